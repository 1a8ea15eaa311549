"""Parameter-shift, finite-difference and SPSA gradients on the batch engine.

Checked against the oracle's adjoint gradient (parameter shifts are exact: 1e-10; central
differences with h = 1e-4 carry O(h^2) truncation: 1e-6), on pure states, a
noisy density-matrix objective and controlled rotations (four-term rule,
sampled_gradients.jl:34-39). SPSA is checked against its definition with the same draws.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_parameter_shift_matches_adjoint(mq, O):
    from mossquantum_b200 import workloads as W
    n, depth = 8, 2
    c = W.hea_circuit(n, depth)
    th = W.hea_angles(n, depth, W.rng_for(8)).reshape(-1)
    obj = mq.ExpectationObjective(c, W.tfim(n), mq.StateVector(n))
    v_ps, g_ps = mq.value_and_gradient(mq.ParameterShift(), obj, th)
    cb = W.hea_circuit(n, depth, th.reshape(depth, n, 3))
    v_ad, g_ad = O.adjoint(cb.specs(), O.zero_state(n), n, W.tfim(n).specs())
    assert abs(v_ps - v_ad) <= 1e-11 and np.max(np.abs(g_ps - g_ad)) <= 1e-10
    v_fd, g_fd = mq.value_and_gradient(mq.FiniteDifference(step=1e-4), obj, th)
    assert np.max(np.abs(g_fd - g_ad)) <= 1e-6
    est = mq.estimate_gradient(mq.ParameterShift(), obj, th)
    assert est.evaluations == 1 + 2 * len(th) and est.shots == 0


def test_parameter_shift_noisy_density_and_controlled(mq, O):
    from mossquantum_b200 import workloads as W
    n = 5
    c = W.hea_circuit(n, 1, noise=(0.02, 0.03))
    th = W.hea_angles(n, 1, W.rng_for(8, 1)).reshape(-1)
    obj = mq.ExpectationObjective(c, W.xxz(n), mq.DensityMatrix(n))
    v, g = mq.value_and_gradient(mq.ParameterShift(), obj, th)
    cb = W.hea_circuit(n, 1, th.reshape(1, n, 3), noise=(0.02, 0.03))
    v_ref, g_ref = O.adjoint(cb.specs(), O.zero_state(n, True), n, W.xxz(n).specs(), dm=True)
    assert abs(v - v_ref) <= 1e-11 and np.max(np.abs(g - g_ref)) <= 1e-10
    cc = mq.QCircuit([mq.HGate(1), mq.HGate(2), mq.CRxGate(1, 2, 0.3, isparas=True), mq.CRyGate(2, 3, 0.5, isparas=True),
                      mq.CRzGate(3, 1, -0.7, isparas=True), mq.RyGate(3, 0.2, isparas=True)])
    objc = mq.ExpectationObjective(cc, W.tfim(3), mq.StateVector(3))
    x = np.array([0.3, 0.5, -0.7, 0.2])
    _, g_ps = mq.value_and_gradient(mq.ParameterShift(), objc, x)
    _, g_ad = O.adjoint(cc.specs(), O.zero_state(3), 3, W.tfim(3).specs())
    assert np.max(np.abs(g_ps - g_ad)) <= 1e-10


def test_batch_objective_and_spsa(mq, O):
    from mossquantum_b200 import workloads as W
    n, B = 6, 3
    c = W.hea_circuit(n, 1)
    th = W.hea_angles(n, 1, W.rng_for(8, 2)).reshape(-1)
    init = mq.BatchStateVector(n, B)
    rng = np.random.default_rng(3)
    psis = rng.normal(size=(1 << n, B)) + 1j * rng.normal(size=(1 << n, B))
    psis /= np.linalg.norm(psis, axis=0)
    init.upload(psis)
    obj = mq.BatchExpectationObjective(c, W.tfim(n), init, reduction="sum")
    _, g_ps = mq.value_and_gradient(mq.ParameterShift(), obj, th)
    cb = W.hea_circuit(n, 1, th.reshape(1, n, 3))
    g_ad = sum(O.adjoint(cb.specs(), psis[:, b], n, W.tfim(n).specs())[1] for b in range(B))
    assert np.max(np.abs(g_ps - g_ad)) <= 1e-10
    m, h = 4, 0.1
    est = mq.estimate_gradient(mq.SPSAGradient(step=h, directions=m), obj, th, rng=np.random.default_rng(5))
    r = np.random.default_rng(5)
    dirs = np.array([[1.0 if r.random() < 0.5 else -1.0 for _ in range(len(th))] for _ in range(m)])
    ref = np.mean([(obj.evaluate(th + h * d) - obj.evaluate(th - h * d)) / (2 * h) * d for d in dirs], axis=0)
    assert np.max(np.abs(est.gradient - ref)) <= 1e-10
