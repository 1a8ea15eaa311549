"""Adjoint gradients on the GPU vs the oracle, closed forms and finite differences.

Mirrors test/unit/adjoint_objectives.jl:111-156, test/extensions/shared_parameter_gradients.jl
and test/integration/noisy_circuit_gradients.jl. Tolerances: 1e-10 vs the oracle, 1e-7 vs
central finite differences (h = 1e-6, accurate to ~1e-9).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def fd(obj, theta, h=1e-6, idx=None):
    idx = range(len(theta)) if idx is None else idx
    g = []
    for i in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        g.append((obj.evaluate(tp) - obj.evaluate(tm)) / (2 * h))
    return np.array(g)


@pytest.mark.parametrize("kind", ["pure", "density"])
def test_ry_known_answer(mq, kind):
    th = 0.37
    init = mq.StateVector(1) if kind == "pure" else mq.DensityMatrix(1)
    obj = mq.ExpectationObjective(mq.QCircuit([mq.RyGate(1, 0.0, isparas=True)]), mq.QubitsTerm([1], ["Z"]), init)
    assert mq.supports_gradient(mq.AdjointGradient(), obj)
    v, g = mq.value_and_gradient(mq.AdjointGradient(), obj, [th])
    assert v == pytest.approx(np.cos(th), abs=1e-14)
    assert g[0] == pytest.approx(-np.sin(th), abs=1e-13)
    for gamma in (0.23, 1.0):
        c = mq.QCircuit([mq.RyGate(1, 0.0, isparas=True), mq.AmplitudeDamping(1, gamma)])
        obj = mq.ExpectationObjective(c, mq.QubitsTerm([1], ["Z"]), init)
        v, g = mq.value_and_gradient(mq.AdjointGradient(), obj, [th])
        assert v == pytest.approx(gamma + (1 - gamma) * np.cos(th), abs=1e-13)
        assert g[0] == pytest.approx(-(1 - gamma) * np.sin(th), abs=1e-12)


def test_adjoint_gate_known_answer(mq):
    th = 0.37
    obj = mq.ExpectationObjective(mq.QCircuit([mq.RyGate(1, 0.0, isparas=True).adjoint()]), mq.QubitsTerm([1], ["X"]),
                                  mq.StateVector(1))
    v, g = mq.value_and_gradient(mq.AdjointGradient(), obj, [th])
    assert v == pytest.approx(-np.sin(th), abs=1e-14) and g[0] == pytest.approx(-np.cos(th), abs=1e-13)


def test_shared_parameter_closed_form(mq):
    template = mq.QCircuit([mq.RyGate(1, 0.0, isparas=True), mq.RxGate(2, 0.3),
                            mq.QCircuit([mq.RzGate(1, 0.0, isparas=True), mq.RyGate(1, 0.0, isparas=True)])])
    pm = mq.ParameterMap(template, [1, 2, 1])
    t, p = 0.35, -0.47
    obj = mq.ExpectationObjective(template, mq.QubitsTerm([1], ["Z"]), mq.StateVector(2), parameter_map=pm)
    v, g = mq.value_and_gradient(mq.AdjointGradient(), obj, [t, p])
    assert v == pytest.approx(np.cos(t) ** 2 - np.cos(p) * np.sin(t) ** 2, abs=1e-13)
    np.testing.assert_allclose(g, [-2 * np.sin(t) * np.cos(t) * (1 + np.cos(p)), np.sin(p) * np.sin(t) ** 2],
                               atol=1e-12)
    assert obj.evaluate([t, p]) == pytest.approx(v, abs=1e-13)


@pytest.mark.parametrize("n,depth", [(6, 3), (10, 4)])
def test_hea_vs_oracle_and_fd(mq, O, n, depth):
    from mossquantum_b200 import workloads as W
    angles = W.hea_angles(n, depth, W.rng_for(3, n))
    c = W.hea_circuit(n, depth, angles)
    H = W.tfim(n)
    obj = mq.ExpectationObjective(c, H, mq.StateVector(n))
    theta = np.array(c.active_parameters())
    v, g = mq.value_and_gradient(mq.AdjointGradient(), obj, theta)
    vr, gr = O.adjoint(c.specs(), O.zero_state(n), n, H.specs())
    assert abs(v - vr) <= 1e-11
    assert np.max(np.abs(g - gr)) <= 1e-10
    idx = np.random.default_rng(0).choice(len(theta), size=min(32, len(theta)), replace=False)
    assert np.max(np.abs(g[idx] - fd(obj, theta, idx=idx))) <= 1e-7


def test_checkpointed_matches_unchecked(mq):
    from mossquantum_b200 import workloads as W
    n, depth = 8, 4
    c = W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(4)))
    obj = mq.ExpectationObjective(c, W.tfim(n), mq.StateVector(n))
    theta = np.array(c.active_parameters())
    v1, g1 = mq.value_and_gradient(mq.AdjointGradient(), obj, theta)
    v2, g2 = mq.value_and_gradient(mq.AdjointGradient(checkpoint_every=7), obj, theta)
    assert abs(v1 - v2) <= 1e-13 and np.max(np.abs(g1 - g2)) <= 1e-12


@pytest.mark.parametrize("kind", ["pure", "density"])
def test_noisy_gradients_vs_oracle(mq, O, kind):
    from mossquantum_b200 import workloads as W
    n, depth = 4, 2
    c = W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(5, n)), noise=(0.01, 0.02))
    H = W.xxz(n)
    init = mq.StateVector(n) if kind == "pure" else mq.DensityMatrix(n)
    obj = mq.ExpectationObjective(c, H, init)
    theta = np.array(c.active_parameters())
    v, g = mq.value_and_gradient(mq.AdjointGradient(), obj, theta)
    vr, gr = O.adjoint(c.specs(), O.zero_state(n, kind == "density"), n, H.specs(), dm=kind == "density")
    assert abs(v - vr) <= 1e-11 and np.max(np.abs(g - gr)) <= 1e-10
    assert np.max(np.abs(g[:8] - fd(obj, theta, idx=range(8)))) <= 1e-7


def test_batch_density_shared_parameters(mq, O):
    from mossquantum_b200 import workloads as W
    n, depth, B = 3, 2, 4
    c = W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(6)), noise=(0.005, 0.0))
    H = W.tfim(n)
    rng = np.random.default_rng(6)
    rhos = []
    for _ in range(B):
        a = rng.normal(size=(8, 8)) + 1j * rng.normal(size=(8, 8))
        r = a @ a.conj().T
        rhos.append(r / np.trace(r))
    init = mq.BatchDensityMatrix(np.stack(rhos, axis=2))
    theta = np.array(c.active_parameters())
    for reduction, weights in (("mean", None), ("sum", None), ("weighted_sum", [0.5, -1.0, 2.0, 0.25])):
        obj = mq.BatchExpectationObjective(c, H, init, reduction=reduction, weights=weights)
        v, g = mq.value_and_gradient(mq.AdjointGradient(), obj, theta)
        w = obj.sample_weights()
        vr, gr = 0.0, 0.0
        for b in range(B):
            vb, gb = O.adjoint(c.specs(), rhos[b].ravel(order="F"), n, H.specs(), dm=True)
            vr += w[b] * vb
            gr = gr + w[b] * gb
        assert abs(v - vr) <= 1e-11 and np.max(np.abs(g - gr)) <= 1e-10
        vals = obj.evaluate_batch(theta)
        assert abs(np.dot(w, vals) - v) <= 1e-12


def test_value_and_pullback(mq):
    obj = mq.ExpectationObjective(mq.QCircuit([mq.RyGate(1, 0.0, isparas=True)]), mq.QubitsTerm([1], ["Z"]),
                                  mq.StateVector(1))
    v, back = mq.value_and_pullback(mq.AdjointGradient(), obj, [0.37])
    assert back(2.0)[0] == pytest.approx(-2 * np.sin(0.37), abs=1e-13)
    assert back(0.0)[0] == 0.0


def _with_env(key, value, fn):
    import os
    old = os.environ.get(key)
    os.environ[key] = value
    try:
        return fn()
    finally:
        if old is None:
            del os.environ[key]
        else:
            os.environ[key] = old


@pytest.mark.parametrize("n,depth,ck", [(10, 3, 0), (13, 4, 17), (16, 2, 0)])
def test_fused_adjoint_vs_plain_and_oracle(mq, O, n, depth, ck):
    """The fused dual-state reverse sweep equals the plain per-gate sweep and the oracle."""
    from mossquantum_b200 import workloads as W
    rng = np.random.default_rng(n)
    c = W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(13, n)))
    t = lambda: float(rng.uniform(-np.pi, np.pi))
    c.push(mq.CRxGate(2, 5, t(), isparas=True))
    c.push(mq.CRyGate(n, 1, t(), isparas=True))
    c.push(mq.CPHASEGate(3, 4, t(), isparas=True))
    c.push(mq.RyGate(6, t(), isparas=True).adjoint())
    c.push(mq.QuantumGate((1, 2, 3), np.linalg.qr(rng.normal(size=(8, 8)) + 1j * rng.normal(size=(8, 8)))[0]))
    c.push(mq.PHASEGate(n, t(), isparas=True))
    H = W.tfim(n) + W.xxz(n) * 0.5
    obj = mq.ExpectationObjective(c, H, mq.StateVector(n))
    theta = np.array(c.active_parameters())
    v, g = mq.value_and_gradient(mq.AdjointGradient(checkpoint_every=ck), obj, theta)
    vp, gp = _with_env("MB_ADJOINT_PLAIN", "1",
                       lambda: mq.value_and_gradient(mq.AdjointGradient(checkpoint_every=ck), obj, theta))
    vr, gr = O.adjoint(c.specs(), O.zero_state(n), n, H.specs())
    assert abs(v - vr) <= 1e-11 and abs(vp - vr) <= 1e-11
    assert np.max(np.abs(g - gr)) <= 1e-10 and np.max(np.abs(gp - gr)) <= 1e-10


def test_fused_adjoint_shared_parameters(mq, O):
    from mossquantum_b200 import workloads as W
    n, depth = 11, 3
    c = W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(14)))
    P = c.nparameters()
    ids = [(i % (P // 3)) + 1 for i in range(P)]
    pm = mq.ParameterMap(c, ids)
    obj = mq.ExpectationObjective(c, W.tfim(n), mq.StateVector(n), parameter_map=pm)
    x = np.random.default_rng(1).uniform(0, 2 * np.pi, size=pm.nparameters())
    v, g = mq.value_and_gradient(mq.AdjointGradient(), obj, x)
    slots = pm.expand(x)
    cb = c.copy().reset_parameters(slots)
    vr, gr = O.adjoint(cb.specs(), O.zero_state(n), n, W.tfim(n).specs())
    assert abs(v - vr) <= 1e-11
    assert np.max(np.abs(g - mq.accumulate_parameter_gradients(pm, gr))) <= 1e-10


def test_density_channel_kinds_forward_and_gradient(mq, O):
    """Every single-qubit channel family after the gates of a 6-qubit density matrix: the ones
    with the real population/coherence pattern run as channel micro-ops (forward, and inverted
    or adjoined in the fused reverse), bit flips keep the dense 4x4. State and gradient against
    the oracle."""
    from mossquantum_b200 import workloads as W
    n, depth = 6, 2
    c0 = W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(6, n)))
    chans = [lambda q: mq.Depolarizing(q, 0.03), lambda q: mq.AmplitudeDamping(q, 0.05),
             lambda q: mq.PhaseDamping(q, 0.04), lambda q: mq.PhaseFlip(q, 0.02),
             lambda q: mq.GeneralizedAmplitudeDamping(q, 0.05, 0.2), lambda q: mq.ResetChannel(q, 0, 0.1),
             lambda q: mq.ThermalRelaxation(q, 50.0, 40.0, 1.0), lambda q: mq.BitFlip(q, 0.02),
             lambda q: mq.BitPhaseFlip(q, 0.01)]
    c = mq.QCircuit()
    for i, g in enumerate(c0.flat()):
        c.push(g)
        for q in g.positions:
            c.push(chans[(i + q) % len(chans)](q))
    s = mq.apply_(c, mq.DensityMatrix(n))
    rho = O.apply(c.specs(), O.zero_state(n, True), n, True)
    assert np.max(np.abs(s.to_numpy().ravel(order="F") - rho)) <= 1e-12
    H = W.tfim(n)
    obj = mq.ExpectationObjective(c, H, mq.DensityMatrix(n))
    theta = np.array(c.active_parameters())
    v, g = mq.value_and_gradient(mq.AdjointGradient(), obj, theta)
    vr, gr = O.adjoint(c.specs(), O.zero_state(n, True), n, H.specs(), dm=True)
    assert abs(v - vr) <= 1e-11 and np.max(np.abs(g - gr)) <= 1e-10
