"""Runtime-specialised pass kernels vs the oracle (forced on for small states).

The specialised kernels normally serve states of 18+ register bits; here MB_JIT_MIN_BITS
lowers the threshold so the same circuits as the interpreter tests run through them.
Tolerance 1e-12 max-abs.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture
def jit_on():
    old = os.environ.get("MB_JIT_MIN_BITS")
    os.environ["MB_JIT_MIN_BITS"] = "8"
    yield
    if old is None:
        del os.environ["MB_JIT_MIN_BITS"]
    else:
        os.environ["MB_JIT_MIN_BITS"] = old


def used_jit(N):
    rep = N.profile_report()
    return any(k.endswith("_jit") for k in rep)


def test_jit_gates_pure(mq, O, jit_on):
    from mossquantum_b200 import _native as N
    from tests.test_gpu_gates import named_gates, random_state, random_unitary
    rng = np.random.default_rng(41)
    for n in (9, 13):
        psi = random_state(n, rng)
        gates = named_gates(mq, 7, rng)
        gates += [mq.QuantumGate((int(a), int(b)), random_unitary(4, rng))
                  for a, b in rng.choice(np.arange(1, n + 1), size=(6, 2), replace=True) if a != b]
        gates += [mq.QuantumGate(int(q), random_unitary(2, rng)) for q in rng.integers(1, n + 1, size=20)]
        c = mq.QCircuit(gates)
        N.profile(True)
        s = mq.apply_(c, mq.StateVector(psi))
        assert used_jit(N)
        N.profile(False)
        ref = O.apply(c.specs(), psi, n)
        assert np.max(np.abs(s.to_numpy() - ref)) <= 1e-12


def test_jit_workloads(mq, O, jit_on):
    from mossquantum_b200 import workloads as W
    for n, depth in ((12, 6), (15, 4)):
        for c in (W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(9, n))),
                  W.u3_brickwork(n, depth, W.u3_params(n, depth, W.rng_for(10, n)))):
            s = mq.apply_(c, mq.StateVector(n))
            ref = O.apply(c.specs(), O.zero_state(n), n)
            assert np.max(np.abs(s.to_numpy() - ref)) <= 1e-12


def test_jit_density_and_batch(mq, O, jit_on):
    from mossquantum_b200 import workloads as W
    n, depth = 5, 2
    c = W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(11)), noise=(0.01, 0.02))
    s = mq.apply_(c, mq.DensityMatrix(n))
    ref = O.apply(c.specs(), O.zero_state(n, True), n, True)
    assert np.max(np.abs(s.to_numpy().ravel(order="F") - ref)) <= 1e-12
    n, B = 9, 3
    c = W.hea_circuit(n, 2, W.hea_angles(n, 2, W.rng_for(12)))
    thetas = np.random.default_rng(2).uniform(0, 2 * np.pi, size=(B, c.nparameters()))
    s = mq.apply_(c, mq.BatchStateVector(n, B), theta=thetas)
    out = s.to_numpy()
    for b in range(B):
        ref = O.apply(c.copy().reset_parameters(thetas[b]).specs(), O.zero_state(n), n)
        assert np.max(np.abs(out[:, b] - ref)) <= 1e-12


def test_jit_fresh_circuits_same_structure(mq, O, jit_on):
    """Fresh host circuits with new fixed angles lower to passes with the same micro-ops, so
    their schedules reuse the memoised kernel sources; every circuit still gets its own matrix
    values (each result against the oracle)."""
    from mossquantum_b200 import _native as N
    from mossquantum_b200 import workloads as W
    n, depth = 14, 6
    for i in range(3):
        c = W.u3_brickwork(n, depth, W.u3_params(n, depth, W.rng_for(77, i)))
        N.profile(True)
        s = mq.apply_(c, mq.StateVector(n))
        assert used_jit(N)
        N.profile(False)
        ref = O.apply(c.specs(), O.zero_state(n), n)
        assert np.max(np.abs(s.to_numpy() - ref)) <= 1e-12
