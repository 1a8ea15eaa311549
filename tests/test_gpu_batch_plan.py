"""Uneven batches replayed from a CUDA graph, and the autotuner, vs the oracle.

Per-sample parameters and mixed register sizes go beyond the reference's batches (one size,
one parameter vector); each sample is checked against the oracle run alone. Tolerance
1e-11 on expectations.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_ragged_plan_two_replays(mq, O):
    from mossquantum_b200 import workloads as W
    from mossquantum_b200.batch import BatchPlan
    sizes = {9: 3, 10: 2, 12: 2, 13: 1}
    depth = 2
    groups = {n: (W.hea_circuit(n, depth), B) for n, B in sizes.items()}
    plan = BatchPlan(groups, W.xxz)
    rng = np.random.default_rng(5)
    for _ in range(2):
        thetas = {n: rng.uniform(0, 2 * np.pi, size=(B, groups[n][0].nparameters())) for n, B in sizes.items()}
        res = plan.run(thetas)
        for n, B in sizes.items():
            for b in range(B):
                c = groups[n][0].copy().reset_parameters(thetas[n][b])
                ref = O.expect(O.apply(c.specs(), O.zero_state(n), n), n, W.xxz(n).specs())
                assert abs(res[n][b] - ref) <= 1e-11
    plan.close()


def test_density_plan(mq, O):
    from mossquantum_b200 import workloads as W
    from mossquantum_b200.batch import BatchPlan
    n, B = 4, 3
    c = W.hea_circuit(n, 1, noise=(0.01, 0.02))
    plan = BatchPlan({n: (c, B)}, W.xxz, kind="density")
    th = np.random.default_rng(6).uniform(0, 2 * np.pi, size=(B, c.nparameters()))
    res = plan.run({n: th})
    for b in range(B):
        cb = c.copy().reset_parameters(th[b])
        rho = O.apply(cb.specs(), O.zero_state(n, True), n, True)
        assert abs(res[n][b] - O.expect(rho, n, W.xxz(n).specs(), dm=True)) <= 1e-11
    plan.close()


def test_autotune_keeps_results(mq, O):
    from mossquantum_b200 import autotune
    from mossquantum_b200 import workloads as W
    n = 14
    c = W.u3_brickwork(n, 4, W.u3_params(n, 4, W.rng_for(20)))
    t, r, ms = autotune.autotune(c, mq.StateVector(n))
    assert (t, r) == autotune.get(n) and ms > 0
    s = mq.apply_(c, mq.StateVector(n))
    ref = O.apply(c.specs(), O.zero_state(n), n)
    assert np.max(np.abs(s.to_numpy() - ref)) <= 1e-12


@pytest.mark.parametrize("form,kernel", [("specialised", "mbk_uneven"), ("interpreted", "k_uneven")])
def test_persistent_uneven_launch(mq, O, monkeypatch, form, kernel):
    """Pure samples of 8..17 qubits with per-sample angles run in one persistent launch (work
    items of (pass, sample, chunk of tiles)); a 6-qubit and an 18-qubit group take the per-size
    path after it. Every sample's expectation and every 8- and 17-qubit amplitude against the
    oracle run alone; the launch list holds exactly one persistent launch per replay, of the
    straight-line form (one device function per pass) or of the micro-op interpreter."""
    if form == "interpreted":
        monkeypatch.setenv("MB_UNEVEN_JIT", "0")
    from mossquantum_b200 import _native as N
    from mossquantum_b200 import workloads as W
    from mossquantum_b200.batch import BatchPlan
    sizes = {6: 2, 8: 3, 11: 2, 14: 2, 17: 2, 18: 1}
    depth = 3
    groups = {n: (W.hea_circuit(n, depth), B) for n, B in sizes.items()}
    plan = BatchPlan(groups, W.xxz, persistent=True)
    assert plan.persistent_info() == (4, 2, 9)
    rng = np.random.default_rng(17)
    thetas = {n: rng.uniform(0, 2 * np.pi, size=(B, groups[n][0].nparameters())) for n, B in sizes.items()}
    res = plan.run(thetas)
    for n, B in sizes.items():
        for b in range(B):
            c = groups[n][0].copy().reset_parameters(thetas[n][b])
            psi = O.apply(c.specs(), O.zero_state(n), n)
            assert abs(res[n][b] - O.expect(psi, n, W.xxz(n).specs())) <= 1e-11, (n, b)
            if n in (8, 17):
                g = [x for x in plan.groups if x["n"] == n][0]
                got = g["state"].to_numpy()[:, b]
                assert np.max(np.abs(got - psi)) <= 1e-12, (n, b)
    # the recorded body run eagerly: one persistent launch for the four middle sizes
    plan._stage(thetas)
    N.profile(True)
    try:
        plan._record_body()
        N.synchronize()
        rep = N.profile_report()
    finally:
        N.profile(False)
    assert rep[kernel][0] == 1, rep
    assert "k_tile_pass" not in rep and ("k_uneven" if form == "specialised" else "mbk_uneven") not in rep, rep
    plan.close()


def test_plan_keeps_the_faster_form(mq, O):
    """The default plan captures the persistent form and per-size specialised launches, keeps
    the faster replay, and either form gives the oracle's expectations."""
    from mossquantum_b200 import workloads as W
    from mossquantum_b200.batch import BatchPlan
    sizes = {10: 3, 12: 2, 15: 2}
    groups = {n: (W.hea_circuit(n, 2), B) for n, B in sizes.items()}
    from mossquantum_b200 import autotune as A
    before = {n: A.get(n) for n in sizes}
    plan = BatchPlan(groups, W.xxz)
    assert plan.choice is not None and plan.choice["chosen"] in ("persistent", "per-size specialised")
    assert {n: A.get(n) for n in sizes} == before   # the choice leaves the process-wide tuning as it was
    rng = np.random.default_rng(23)
    thetas = {n: rng.uniform(0, 2 * np.pi, size=(B, groups[n][0].nparameters())) for n, B in sizes.items()}
    res = plan.run(thetas)
    for n, B in sizes.items():
        for b in range(B):
            c = groups[n][0].copy().reset_parameters(thetas[n][b])
            ref = O.expect(O.apply(c.specs(), O.zero_state(n), n), n, W.xxz(n).specs())
            assert abs(res[n][b] - ref) <= 1e-11
    plan.close()
