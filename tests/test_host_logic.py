"""Host-side logic of the newer paths, on the CPU: trajectory planning (mixture detection,
Pauli expansion of K'K), parameter-shift recipes, and the measurement sampling rules."""
import numpy as np
import pytest

import mossquantum_b200 as mq
from mossquantum_b200 import trajectories as T
from mossquantum_b200.measurement import _normalize


def test_channel_classification():
    dep = T._compile_channel(mq.Depolarizing(1, 0.1))
    assert dep.mixture and np.isclose(dep.weights.sum(), 1.0)
    for opt in dep.options:
        assert np.allclose(opt.conj().T @ opt, np.eye(2))      # unitary branches
    amp = T._compile_channel(mq.AmplitudeDamping(2, 0.3))
    assert not amp.mixture and len(amp.probes) == 2
    segs = T._plan(mq.QCircuit([mq.HGate(1), mq.Depolarizing(1, 0.1), mq.AmplitudeDamping(2, 0.3), mq.CNOTGate(1, 2)]))
    assert [len(s) for s in segs] == [2, 2]   # a state-dependent channel starts a new segment


def test_pauli_expansion_reconstructs_matrix():
    rng = np.random.default_rng(1)
    for k in (1, 2):
        A = rng.normal(size=(1 << k, 1 << k)) + 1j * rng.normal(size=(1 << k, 1 << k))
        M = A.conj().T @ A
        op = T._pauli_operator(M, list(range(3, 3 + k)))
        got = sum(t.coeff * _kron_term(t, list(range(3, 3 + k))) for t in op.terms)
        assert np.max(np.abs(got - M)) <= 1e-12


def _kron_term(t, positions):
    """Dense matrix of one term's operator product on `positions` (first = least significant)."""
    P = np.array([[1.0 + 0j]])
    for p in reversed(positions):
        m = np.eye(2, dtype=complex)
        for site, o in zip(t.positions, t.op):
            if site == p:
                m = np.asarray(o, dtype=complex)
        P = np.kron(P, m)
    return P


def test_shift_rules():
    r2 = mq.parameter_shift_rule(mq.RxGate(1, 0.3, isparas=True))
    assert r2 == [(0.5, np.pi / 2), (-0.5, -np.pi / 2)]
    r4 = mq.parameter_shift_rule(mq.CRyGate(1, 2, 0.3, isparas=True))
    coeffs = [c for c, _ in r4]
    assert len(r4) == 4 and abs(sum(coeffs)) <= 1e-15
    # the four-term rule differentiates f(t) = a + b cos(t/2) + c sin(t/2) + d cos t + e sin t exactly
    f = lambda t: 0.3 + 0.7 * np.cos(t / 2) - 0.2 * np.sin(t / 2) + 0.5 * np.cos(t) + 0.9 * np.sin(t)
    df = lambda t: -0.35 * np.sin(t / 2) - 0.1 * np.cos(t / 2) - 0.5 * np.sin(t) + 0.9 * np.cos(t)
    x = 0.83
    assert abs(sum(c * f(x + s) for c, s in r4) - df(x)) <= 1e-14
    assert mq.parameter_shift_rule(mq.QuantumGate(1, np.eye(2))) is None
    with pytest.raises(ValueError):
        mq.FiniteDifference(step=0.0)
    with pytest.raises(ValueError):
        mq.SPSAGradient(directions=0)


def test_sampling_rules():
    rng = np.random.default_rng(4)
    draws = [mq.discrete_sample(rng, [0.2, 0.0, 0.8]) for _ in range(4000)]
    assert 1 not in draws and abs(draws.count(2) / 4000 - 0.8) < 0.03
    assert mq.discrete_sample(np.random.default_rng(0), [0.0, 1.0]) == 1
    with pytest.raises(ValueError):
        mq.discrete_sample(rng, [])
    with pytest.raises(ValueError):
        mq.discrete_sample(rng, [0.0, 0.0])
    assert np.allclose(_normalize([0.25, 0.75]), [0.25, 0.75])
    with pytest.raises(ValueError):
        _normalize([0.5, 0.2])
