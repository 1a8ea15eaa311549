"""Serving loop: results alone and in a mix, against the oracle.

Each request (an ansatz of `repeats` hardware-efficient layers with its own angles, on a pure
state or a noisy density matrix, asking for <H> and possibly its adjoint gradient) must give
the same value and gradient when it runs alone on the server and when it shares batched
launches with a mix of other requests admitted while it runs. Both are checked against the
oracle on the unrolled circuit. Tolerances: 1e-11 on values, 1e-10 on gradients (oracle);
1e-12 / 1e-10 between alone and mix.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _blocks(W):
    cache = {}

    def block(kind, n):
        key = (kind, n)
        if key not in cache:
            cache[key] = W.hea_layer(n, noise=W.SERVING_NOISE if kind == "density" else None)
        return cache[key]
    return block


def _obs(W, name, n):
    return W.tfim(n) if name == "tfim" else W.xxz(n)


def _requests(W):
    rng = W.rng_for(4, 7)
    reqs = W.serving_requests(14, rng, pure_n=(8, 11), dm_n=(3, 4), layers=(2, 4))
    # make sure every combination occurs
    reqs += [("pure", 9, 3, "tfim", True, rng.uniform(0, 2 * np.pi, (3, 27))),
             ("density", 4, 2, "xxz", True, rng.uniform(0, 2 * np.pi, (2, 12))),
             ("density", 3, 3, "tfim", False, rng.uniform(0, 2 * np.pi, (3, 9))),
             ("pure", 10, 2, "xxz", False, rng.uniform(0, 2 * np.pi, (2, 30)))]
    return reqs


def test_serving_alone_vs_mix_vs_oracle(mq, O):
    from mossquantum_b200 import workloads as W
    from mossquantum_b200.serving import Server
    block = _blocks(W)
    reqs = _requests(W)
    with Server(budget_bytes=2 << 30) as srv:
        # the mix: everything submitted at once, plus a second wave while the first runs
        tickets = [srv.submit(block(k, n), n, _obs(W, o, n), th, kind=k, gradient=g) for k, n, L, o, g, th in reqs[:10]]
        tickets += [srv.submit(block(k, n), n, _obs(W, o, n), th, kind=k, gradient=g) for k, n, L, o, g, th in reqs[10:]]
        mix = [srv.wait(t, timeout_s=300) for t in tickets]
        st = srv.stats()
        assert st["completed"] == len(reqs) and st["failed"] == 0
        assert st["iterations"] < sum(r[2] * (2 if r[4] else 1) for r in reqs)  # work was shared
        alone = []
        for k, n, L, o, g, th in reqs:
            t = srv.submit(block(k, n), n, _obs(W, o, n), th, kind=k, gradient=g)
            alone.append(srv.wait(t, timeout_s=300))
    for (k, n, L, o, g, th), a, m in zip(reqs, alone, mix):
        assert abs(a.value - m.value) <= 1e-12, (k, n, a.value, m.value)
        if g:
            assert np.max(np.abs(a.gradient - m.gradient)) <= 1e-10
        dm = k == "density"
        noise = W.SERVING_NOISE if dm else None
        circ = W.unrolled(lambda row: W.hea_layer_bound(n, row, noise=noise), th)
        H = _obs(W, o, n).specs()
        if g:
            v_ref, g_ref = O.adjoint(circ.specs(), O.zero_state(n, dm), n, H, dm=dm)
            assert abs(m.value.real - v_ref) <= 1e-11, (k, n, m.value, v_ref)
            assert np.max(np.abs(m.gradient.reshape(-1) - g_ref)) <= 1e-10, (k, n)
        else:
            ref = O.apply(circ.specs(), O.zero_state(n, dm), n, dm=dm)
            e_ref = O.expect(ref, n, H, dm=dm)
            assert abs(m.value - e_ref) <= 1e-11, (k, n, m.value, e_ref)


def test_serving_admission_budget(mq):
    """A request larger than the budget fails alone; the others still complete."""
    from mossquantum_b200 import workloads as W
    from mossquantum_b200.serving import Server
    small = W.hea_layer(8)
    big = W.hea_layer(15)
    rng = W.rng_for(4, 8)
    # 1 MiB budget: an 8-qubit state is 4 KiB; a 15-qubit gradient request needs its 512 KiB
    # state plus y and delta (another 1 MiB), more than the whole budget
    with Server(budget_bytes=1 << 20) as srv:
        t_ok = [srv.submit(small, 8, W.tfim(8), rng.uniform(0, 6, (3, 24))) for _ in range(4)]
        t_big = srv.submit(big, 15, W.tfim(15), rng.uniform(0, 6, (30, 45)), gradient=True)
        for t in t_ok:
            assert np.isfinite(srv.wait(t, timeout_s=120).value.real)
        with pytest.raises(Exception, match="budget"):
            srv.wait(t_big, timeout_s=120)
        st = srv.stats()
        assert st["peak_bytes"] <= st["budget_bytes"]


def test_serving_rejects_bad_requests(mq):
    from mossquantum_b200 import workloads as W
    from mossquantum_b200.serving import Server
    with Server(budget_bytes=1 << 24) as srv:
        with pytest.raises(ValueError):
            srv.submit(W.hea_layer(8), 8, W.tfim(8), np.zeros((2, 5)))
        with pytest.raises(Exception):
            srv.submit(W.hea_layer(4, noise=W.SERVING_NOISE), 4, W.tfim(4), np.zeros((2, 12)), kind="pure")
