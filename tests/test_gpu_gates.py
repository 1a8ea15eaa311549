"""Gate execution on the GPU vs the CPU oracle (bit layout, ordering, every gate family).

Mirrors test/unit/gate_operations.jl:5-76 (all 1/2/3-position combinations, specialised
gates against the generic QuantumGate) and test/unit/high_qubit_gates.jl (4/5-body gates).
Tolerance: 1e-12 max-abs on amplitudes.
"""
import itertools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-12


def random_unitary(d, rng):
    z = rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def random_state(n, rng):
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def run(mq, circuit, n, psi, plain=False):
    s = mq.StateVector(psi)
    s = mq.apply_(circuit, s, plain=plain)
    return s.to_numpy()


@pytest.mark.parametrize("plain", [False, True])
@pytest.mark.parametrize("n", [5, 9])
def test_random_unitaries_all_position_classes(mq, O, n, plain):
    rng = np.random.default_rng(100 + n)
    psi = random_state(n, rng)
    gates = []
    for k in (1, 2, 3):
        for pos in itertools.permutations(range(1, n + 1), k):
            if rng.random() < (1.0 if k == 1 else 0.25 if k == 2 else 0.05):
                gates.append(mq.QuantumGate(pos, random_unitary(1 << k, rng)))
    for k in (4, 5):
        for _ in range(6):
            pos = tuple(int(x) for x in rng.choice(np.arange(1, n + 1), size=k, replace=False))
            gates.append(mq.QuantumGate(pos, random_unitary(1 << k, rng)))
    c = mq.QCircuit(gates)
    out = run(mq, c, n, psi, plain)
    ref = O.apply(c.specs(), psi, n)
    assert np.max(np.abs(out - ref)) <= TOL


def named_gates(mq, n, rng):
    t = lambda: float(rng.uniform(-np.pi, np.pi))
    g = [mq.XGate(2), mq.YGate(1), mq.ZGate(n), mq.SGate(3), mq.HGate(4), mq.TGate(1), mq.sqrtXGate(2),
         mq.sqrtYGate(n), mq.SWAPGate(n, 1), mq.iSWAPGate(2, 5), mq.CZGate(4, 1), mq.CNOTGate(3, 1),
         mq.CNOTGate(1, n), mq.TOFFOLIGate(n, 1, 3), mq.FREDKINGate(2, n, 1),
         mq.RxGate(1, t()), mq.RyGate(n, t()), mq.RzGate(3, t()), mq.PHASEGate(2, t()),
         mq.CRxGate(4, 2, t()), mq.CRyGate(1, 3, t()), mq.CRzGate(n, 2, t()), mq.CPHASEGate(3, 5, t()),
         mq.CCPHASEGate(5, 1, 2, t()), mq.FSIMGate(2, 4, [t(), t(), t(), t(), t()]),
         mq.CONTROLGate(5, 3, random_unitary(2, rng)), mq.CONTROLCONTROLGate(1, 4, 2, random_unitary(2, rng)),
         mq.RyGate(2, t(), isparas=True).adjoint(), mq.CRxGate(3, 1, t()).adjoint(),
         mq.PHASEGate(4, t()).adjoint(), mq.QuantumGate((3, 1), random_unitary(4, rng)).adjoint()]
    return g


@pytest.mark.parametrize("plain", [False, True])
def test_named_gates(mq, O, plain):
    n = 7
    rng = np.random.default_rng(7)
    psi = random_state(n, rng)
    c = mq.QCircuit(named_gates(mq, n, rng))
    out = run(mq, c, n, psi, plain)
    ref = O.apply(c.specs(), psi, n)
    assert np.max(np.abs(out - ref)) <= TOL


def test_specialised_gates_equal_generic(mq):
    """Each specialised gate equals QuantumGate(positions, mat) (gate_operations.jl:44-76)."""
    n = 6
    rng = np.random.default_rng(3)
    psi = random_state(n, rng)
    for g in named_gates(mq, n, rng):
        a = run(mq, mq.QCircuit([g]), n, psi)
        b = run(mq, mq.QCircuit([mq.QuantumGate(g.positions, g.mat())]), n, psi)
        assert np.max(np.abs(a - b)) <= 1e-13, g


def test_config0_shape_at_n14(mq, O):
    from mossquantum_b200 import workloads as W
    n, depth = 14, 10
    c = W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(0, 14)))
    s = mq.apply_(c, mq.StateVector(n))
    ref = O.apply(c.specs(), O.zero_state(n), n)
    assert np.max(np.abs(s.to_numpy() - ref)) <= TOL
    H = W.tfim(n)
    assert abs(mq.expectation(H, s) - O.expect(ref, n, H.specs())) <= 1e-11


def test_config0_full_size(mq, O):
    """The 20-qubit hardware-efficient workload exactly: 20 qubits, 10 layers, 600 angles, TFIM output."""
    from mossquantum_b200 import workloads as W
    n, depth = 20, 10
    c = W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(0)))
    assert len(c.flat()) == 790 and c.nparameters() == 600
    s = mq.apply_(c, mq.StateVector(n))
    ref = O.apply(c.specs(), O.zero_state(n), n)
    assert np.max(np.abs(s.to_numpy() - ref)) <= TOL
    H = W.tfim(n)
    assert abs(mq.expectation(H, s) - O.expect(ref, n, H.specs())) <= 1e-11


def test_u3_brickwork_small(mq, O):
    from mossquantum_b200 import workloads as W
    for n in (6, 13, 16):
        depth = 6
        c = W.u3_brickwork(n, depth, W.u3_params(n, depth, W.rng_for(1, n)))
        for plain in (False, True):
            s = mq.apply_(c, mq.StateVector(n), plain=plain)
            ref = O.apply(c.specs(), O.zero_state(n), n)
            assert np.max(np.abs(s.to_numpy() - ref)) <= TOL


def test_zero_qubit_gate_and_empty_circuit(mq, O):
    n = 3
    psi = random_state(n, np.random.default_rng(0))
    s = mq.apply_(mq.QCircuit(), mq.StateVector(psi))
    assert np.array_equal(s.to_numpy(), psi)
    ph = np.exp(0.3j)
    s = mq.apply_(mq.QuantumGate((), np.array([[ph]])), mq.StateVector(psi))
    np.testing.assert_allclose(s.to_numpy(), ph * psi, atol=1e-15)


def test_position_validation(mq):
    s = mq.StateVector(3)
    with pytest.raises(ValueError):
        mq.apply_(mq.XGate(4), s)
    with pytest.raises(ValueError):
        mq.QuantumGate((1, 1), np.eye(4))
