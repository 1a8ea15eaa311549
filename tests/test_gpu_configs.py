"""Parity at the benchmarked sizes: the exact workloads bench.py times, against the oracle.

* The 28-qubit scale workload's circuit family (U3 on every qubit + CZ brickwork, 20 layers) at
  26 qubits on the default path (specialised tile passes at 2^11-amplitude tiles), and at 28
  qubits when the host has room for three 4 GiB vectors.
* The gradient workload: 24 qubits, depth 16, 1152 independent angles, forward checkpoints
  every 4 layers, against the oracle's adjoint (1e-10) and central differences (h = 1e-6,
  32 seeded coordinates, 1e-7; the reference's own finite-difference checks use 1e-8..1e-7,
  test/unit/adjoint_objectives.jl:122, test/extensions/batch_density_gradients.jl:48).
* The uneven batch: samples of 18-22 qubits with per-sample angles through a BatchPlan, and
  10-qubit depth-8 noisy density matrices.
* The reference's recorded benchmark circuits (exact angles from
  docs/performance/cpu-scheduling-2026-11-17/baseline-16, committed under tests/golden/).

Tolerances: amplitudes 1e-12 max-abs, expectations 1e-11, gradients 1e-10.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cpu_scan_circuits.json")


def max_abs_diff(a, b, chunk=1 << 24):
    """max |a - b| without full-size temporaries (28-qubit vectors are 4 GiB)."""
    m = 0.0
    for i in range(0, a.size, chunk):
        m = max(m, float(np.max(np.abs(a[i:i + chunk] - b[i:i + chunk]))))
    return m


def host_bytes_available():
    try:
        import psutil
        return psutil.virtual_memory().available
    except ImportError:
        return 0


def run_u3_brickwork(mq, O, n, depth):
    from mossquantum_b200 import _native as N
    from mossquantum_b200 import workloads as W
    c = W.u3_brickwork(n, depth, W.u3_params(n, depth, W.rng_for(1, 0)))
    s = mq.StateVector(n)
    N.profile(True)
    try:
        mq.apply_(c, s)
        rep = N.profile_report()
    finally:
        N.profile(False)
    got = s.to_numpy()
    del s
    ref = O.apply(c.specs(), O.zero_state(n), n)
    return got, ref, rep


def test_scale_workload_26q_default_path(mq, O):
    got, ref, rep = run_u3_brickwork(mq, O, 26, 20)
    # the benchmarked kernel variant: specialised (NVRTC) tile passes
    assert any(k.startswith("k_tile_pass_jit") for k in rep), rep
    assert max_abs_diff(got, ref) <= 1e-12


def test_scale_workload_28q_full(mq, O):
    if host_bytes_available() < (14 << 30):
        pytest.skip("needs about 14 GiB of host memory for the oracle at 28 qubits")
    used, budget = mq.memory_info()
    if budget - used < (6 << 30):
        pytest.skip("needs 6 GiB of the device budget")
    got, ref, rep = run_u3_brickwork(mq, O, 28, 20)
    assert any(k.startswith("k_tile_pass_jit") for k in rep), rep
    assert max_abs_diff(got, ref) <= 1e-12


def test_gradient_workload_24q(mq, O):
    from mossquantum_b200 import workloads as W
    n, depth = 24, 16
    c = W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(3)))
    H = W.tfim(n)
    theta = np.array(c.active_parameters())
    assert theta.size == 1152
    per_layer = 3 * n + (n - 1)
    obj = mq.ExpectationObjective(c, H, mq.StateVector(n))
    v, g = mq.value_and_gradient(mq.AdjointGradient(checkpoint_every=4 * per_layer), obj, theta)
    vr, gr = O.adjoint(c.specs(), O.zero_state(n), n, H.specs())
    assert abs(v - vr) <= 1e-11
    assert np.max(np.abs(g - gr)) <= 1e-10
    idx = np.random.default_rng(24).choice(theta.size, size=32, replace=False)
    h = 1e-6
    for i in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        fd = (obj.evaluate(tp) - obj.evaluate(tm)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7, (i, fd, g[i])


def test_batch_workload_large_pure_samples(mq, O):
    from mossquantum_b200 import workloads as W
    from mossquantum_b200.batch import BatchPlan
    depth = 8
    sizes = {18: 2, 20: 1, 22: 1}
    groups = {n: (W.hea_circuit(n, depth), B) for n, B in sizes.items()}
    plan = BatchPlan(groups, W.xxz)
    rng = np.random.default_rng(22)
    thetas = {n: rng.uniform(0, 2 * np.pi, size=(B, groups[n][0].nparameters())) for n, B in sizes.items()}
    res = plan.run(thetas)
    plan.close()
    for n, B in sizes.items():
        for b in range(B):
            cb = groups[n][0].copy().reset_parameters(thetas[n][b])
            ref = O.expect(O.apply(cb.specs(), O.zero_state(n), n), n, W.xxz(n).specs())
            assert abs(res[n][b] - ref) <= 1e-11, (n, b)


def test_batch_workload_noisy_density_depth8(mq, O):
    from mossquantum_b200 import workloads as W
    from mossquantum_b200.batch import BatchPlan
    n, B, depth = 10, 2, 8
    c = W.hea_circuit(n, depth, noise=(0.01, 0.02))
    plan = BatchPlan({n: (c, B)}, W.xxz, kind="density")
    th = np.random.default_rng(10).uniform(0, 2 * np.pi, size=(B, c.nparameters()))
    res = plan.run({n: th})
    plan.close()
    for b in range(B):
        cb = c.copy().reset_parameters(th[b])
        rho = O.apply(cb.specs(), O.zero_state(n, True), n, True)
        assert abs(res[n][b] - O.expect(rho, n, W.xxz(n).specs(), dm=True)) <= 1e-11
    # and the full density matrix of one sample through the per-call API
    cb = c.copy().reset_parameters(th[0])
    s = mq.apply_(cb, mq.DensityMatrix(n))
    rho = O.apply(cb.specs(), O.zero_state(n, True), n, True)
    assert np.max(np.abs(s.to_numpy().ravel(order="F") - rho)) <= 1e-12


@pytest.mark.parametrize("name", ["n15-d20", "n20-d20", "n25-d10"])
def test_reference_recorded_circuits(mq, O, name):
    from mossquantum_b200 import workloads as W
    with open(GOLDEN) as f:
        case = json.load(f)["cases"][name]
    c = W.cpu_scan_circuit(case["angles_by_layer"])
    n = case["qubits"]
    assert len(c.flat()) == case["depth"] * (2 * n - 1)
    s = mq.apply_(c, mq.StateVector(n))
    got = s.to_numpy()
    del s
    ref = O.apply(c.specs(), O.zero_state(n), n)
    assert max_abs_diff(got, ref) <= 1e-12


@pytest.mark.parametrize("tile_bits", [11, 12])
def test_long_range_gate_beyond_a_tile(mq, O, tile_bits):
    """A dense 3-qubit gate on qubits 4, 12 and 20 of a 20-qubit state needs three windows
    above the lane bits, more than a tile holds: the fused forward runs it as a plain pass,
    and the fused adjoint refuses the schedule so the gradient takes the plain reverse sweep.
    A 2-qubit gate on qubits 4 and 18 fits two windows of one tile."""
    from mossquantum_b200 import _native as N
    from mossquantum_b200 import workloads as W
    n = 20
    rng = np.random.default_rng(14)
    z = rng.normal(size=(8, 8)) + 1j * rng.normal(size=(8, 8))
    u, _ = np.linalg.qr(z)
    z2 = rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4))
    u2, _ = np.linalg.qr(z2)
    gates = [mq.HGate(q) for q in range(1, n + 1)]
    gates += [mq.QuantumGate((4, 12, 20), u), mq.QuantumGate((4, 18), u2)]
    gates += [mq.RyGate(q, float(rng.uniform(0, 2 * np.pi)), isparas=True) for q in range(1, n + 1)]
    gates += [mq.CNOTGate(q, q + 1) for q in range(1, n)]
    gates += [mq.QuantumGate((20, 4, 12), u.conj().T)]
    c = mq.QCircuit(gates)
    from mossquantum_b200 import autotune
    before = autotune.get(n)
    N.check(N.lib().mb_tuning_set(n, tile_bits, 4))
    try:
        s = mq.apply_(c, mq.StateVector(n))
        ref = O.apply(c.specs(), O.zero_state(n), n)
        assert np.max(np.abs(s.to_numpy() - ref)) <= 1e-12
        H = W.tfim(n)
        obj = mq.ExpectationObjective(c, H, mq.StateVector(n))
        v, g = mq.value_and_gradient(mq.AdjointGradient(), obj, np.array(c.active_parameters()))
        vr, gr = O.adjoint(c.specs(), O.zero_state(n), n, H.specs())
        assert abs(v - vr) <= 1e-11
        assert np.max(np.abs(g - gr)) <= 1e-10
    finally:
        autotune.set(n, *before)
