"""Pins the CPU oracle to the reference's own known answers.

The reference (Julia) cannot run here and ships no golden amplitude vectors; its tests
hold closed forms and a dense-embedding check, restated below:
  test/unit/adjoint_objectives.jl:111-156   Ry/Z value and gradient, damping, shared slots
  test/unit/noise_channels.jl:20-38         depolarizing / phase damping closed forms
  test/regression/kernels.jl:4-70           dense embedding of gates and expectations
  test/cross_backend/runtests.jl:15-19      Bell probabilities
"""
import itertools

import numpy as np
import pytest

from oracle import oracle as O


def embed(n, positions0, m):
    """Full 2^n matrix of a local gate (independent of the oracle's kernels)."""
    dim = 1 << n
    k = len(positions0)
    full = np.zeros((dim, dim), dtype=complex)
    for col in range(dim):
        a = 0
        for j, p in enumerate(positions0):
            a |= ((col >> p) & 1) << j
        base = col
        for p in positions0:
            base &= ~(1 << p)
        for r in range(1 << k):
            row = base
            for j, p in enumerate(positions0):
                row |= ((r >> j) & 1) << p
            full[row, col] = m[r, a]
    return full


def random_unitary(d, rng):
    z = rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def random_state(n, rng):
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


@pytest.mark.parametrize("th", [0.37, -1.2, 2.9])
@pytest.mark.parametrize("dm", [False, True])
def test_ry_z_known_answer(th, dm):
    v, g = O.adjoint([("gate", "RY", (1,), [th], [True], None)], O.zero_state(1, dm), 1, [((1,), ["Z"], 1.0)], dm)
    assert v == pytest.approx(np.cos(th), abs=1e-14)
    assert g[0] == pytest.approx(-np.sin(th), abs=1e-14)


@pytest.mark.parametrize("gamma", [0.23, 1.0])
@pytest.mark.parametrize("dm", [False, True])
def test_amplitude_damping_known_answer(gamma, dm):
    th = 0.37
    specs = [("gate", "RY", (1,), [th], [True], None), ("channel", "AmplitudeDamping", (1,), [gamma], None, None)]
    v, g = O.adjoint(specs, O.zero_state(1, dm), 1, [((1,), ["Z"], 1.0)], dm)
    assert v == pytest.approx(gamma + (1 - gamma) * np.cos(th), abs=1e-13)
    assert g[0] == pytest.approx(-(1 - gamma) * np.sin(th), abs=1e-12)


def test_adjoint_gate_known_answer():
    th = 0.37
    v, g = O.adjoint([("gate", "RY'", (1,), [th], [True], None)], O.zero_state(1), 1, [((1,), ["X"], 1.0)])
    assert v == pytest.approx(-np.sin(th), abs=1e-14)
    assert g[0] == pytest.approx(-np.cos(th), abs=1e-14)


def test_shared_parameter_closed_form():
    t, p = 0.35, -0.47
    specs = [("gate", "RY", (1,), [t], [True], None), ("gate", "RX", (2,), [0.3], [False], None),
             ("gate", "RZ", (1,), [p], [True], None), ("gate", "RY", (1,), [t], [True], None)]
    v, g = O.adjoint(specs, O.zero_state(2), 2, [((1,), ["Z"], 1.0)])
    assert v == pytest.approx(np.cos(t) ** 2 - np.cos(p) * np.sin(t) ** 2, abs=1e-14)
    shared = [g[0] + g[2], g[1]]
    assert shared[0] == pytest.approx(-2 * np.sin(t) * np.cos(t) * (1 + np.cos(p)), abs=1e-13)
    assert shared[1] == pytest.approx(np.sin(p) * np.sin(t) ** 2, abs=1e-13)


def test_bell_probabilities_and_identity_expectation():
    s = O.apply([("gate", "H", (1,), [], [], None), ("gate", "CNOT", (1, 2), [], [], None)], O.zero_state(2), 2)
    np.testing.assert_allclose(O.probabilities(s, 2), [0.5, 0, 0, 0.5], atol=1e-15)
    assert O.expect(O.zero_state(4), 4, [((1, 2, 3, 4), ["Z"] * 4, 2.0)]) == pytest.approx(2.0)


def test_channel_closed_forms():
    rng = np.random.default_rng(172)
    a = rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2))
    rho = a @ a.conj().T
    rho /= np.trace(rho)
    for p in (0.0, 0.5, 1.0, 4 / 3):
        out = O.apply([("channel", "Depolarizing", (1,), [p], None, None)], rho.ravel(order="F"), 1, True)
        np.testing.assert_allclose(out.reshape(2, 2, order="F"), (1 - p) * rho + p * np.eye(2) / 2, atol=1e-14)
    plus = np.full((2, 2), 0.5, dtype=complex)
    out = O.apply([("channel", "PhaseDamping", (1,), [0.36], None, None)], plus.ravel(order="F"), 1, True)
    assert out.reshape(2, 2, order="F")[0, 1] == pytest.approx(0.4)


@pytest.mark.parametrize("n", [5, 7])
def test_gates_match_dense_embedding(n):
    rng = np.random.default_rng(n)
    psi = random_state(n, rng)
    for k in (1, 2, 3, 4, 5):
        for positions in itertools.islice(itertools.permutations(range(1, n + 1), k), 0, 40, 7):
            u = random_unitary(1 << k, rng)
            out = O.apply([("gate", "QuantumGate", positions, [], [], u)], psi, n)
            full = embed(n, [p - 1 for p in positions], u)
            np.testing.assert_allclose(out, full @ psi, atol=1e-11)


def test_density_gate_and_channel_match_dense_embedding():
    n = 3
    rng = np.random.default_rng(5)
    a = rng.normal(size=(8, 8)) + 1j * rng.normal(size=(8, 8))
    rho = a @ a.conj().T
    rho /= np.trace(rho)
    u = random_unitary(4, rng)
    out = O.apply([("gate", "QuantumGate", (3, 1), [], [], u)], rho.ravel(order="F"), n, True)
    full = embed(n, [2, 0], u)
    np.testing.assert_allclose(out.reshape(8, 8, order="F"), full @ rho @ full.conj().T, atol=1e-12)
    ks = O.kraus_matrices("AmplitudeDamping", [0.3], None, 1)
    out = O.apply([("channel", "AmplitudeDamping", (2,), [0.3], None, None)], rho.ravel(order="F"), n, True)
    ref = sum(embed(n, [1], k) @ rho @ embed(n, [1], k).conj().T for k in ks)
    np.testing.assert_allclose(out.reshape(8, 8, order="F"), ref, atol=1e-12)


def test_expectation_matches_dense_embedding():
    n = 6
    rng = np.random.default_rng(11)
    psi = random_state(n, rng)
    for k in (1, 2, 3, 4, 5):
        pos = tuple(rng.choice(np.arange(1, n + 1), size=k, replace=False))
        ops = [rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2)) for _ in range(k)]
        coeff = 0.7 - 0.2j
        keys = O.observable_keys([(pos, ops, coeff)])
        (spos, m), = keys.items()
        full = embed(n, [p - 1 for p in spos], m)
        assert O.expect(psi, n, [(pos, ops, coeff)]) == pytest.approx(np.vdot(psi, full @ psi), abs=1e-12)


def test_probabilities_reject_unnormalised():
    with pytest.raises(ValueError):
        O.probabilities(np.array([1.0, 1.0], dtype=complex), 1)


@pytest.mark.parametrize("k", [4, 5])
def test_high_qubit_gates_match_operator_products(k):
    """test/unit/high_qubit_gates.jl:1-46: a k-body gate from_external(positions, kron(m1..mk))
    applied to a state equals the product QubitsTerm(positions[j] => m_j) applied as an
    operator, for the reference's permuted position orders."""
    import mossquantum_b200 as mq
    rng = np.random.default_rng(40 + k)
    L = 7
    i, j, kk, l, m = 2, 5, 3, 7, 1
    orders = {4: [(i, j, kk, l), (i, j, l, kk), (j, i, kk, l), (j, i, l, kk), (l, kk, j, i), (kk, i, l, j)],
              5: [(i, j, kk, l, m), (i, j, l, m, kk), (j, i, m, kk, l), (j, m, i, l, kk), (l, kk, j, m, i),
                  (m, kk, i, l, j)]}[k]
    for order in orders:
        ms = [random_unitary(2, rng) for _ in range(k)]
        ext = ms[0]
        for x in ms[1:]:
            ext = np.kron(ext, x)          # kron(m1, ..., mk): m1 is the most significant factor
        gate = mq.QuantumGate(tuple(order), O.from_external(ext))
        term = mq.QubitsOperator([mq.QubitsTerm(list(order), ms)])
        psi = random_state(L, rng)
        a = O.apply(mq.QCircuit([gate]).specs(), psi, L)
        b = O.apply_observable(psi, L, term.specs())
        assert np.max(np.abs(a - b)) <= 1e-12, order
