"""Mid-circuit measurement and post-selection on the device.

Restates the reference's known answers (test/unit/measurements.jl:1-54: a measured qubit
measures the same outcome again with probability 1, post-selection of a Bell pair) and checks
every collapse against a numpy restatement of measurement.jl / post_selection.jl applied to
the same state with the same seeded generator (1e-12 max-abs on states, identical records);
the outcome draw is restated here too (sampling.jl:3-18).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rand_state(n, rng):
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def ref_discrete_sample(rng, weights):
    """Inverse-CDF draw (sampling.jl:3-18), restated here so the check does not use the
    product's sampler: the first index whose running sum exceeds u * total, else the last
    index with positive weight."""
    w = np.asarray(weights, dtype=float)
    threshold = rng.random() * float(np.sum(w))
    cumulative, last_positive = 0.0, 0
    for i, x in enumerate(w):
        if x > 0:
            last_positive = i
        cumulative += x
        if threshold < cumulative:
            return i
    return last_positive


def ref_measure(psi, n, pos, auto_reset, rng, mq):
    """measure! on a host vector (measurement.jl:4-18, 151-172)."""
    bit = 1 << (pos - 1)
    idx = np.arange(1 << n)
    p0 = np.sum(np.abs(psi[(idx & bit) == 0]) ** 2)
    l = np.array([p0, 1 - p0])
    l = np.maximum(l, 0) / np.sum(np.maximum(l, 0))
    i = ref_discrete_sample(rng, l)
    p = l[i]
    out = np.zeros_like(psi)
    sel = ((idx & bit) != 0) == bool(i)
    if auto_reset:
        out[idx[sel] & ~bit] = psi[sel] / np.sqrt(p)
    else:
        out[sel] = psi[sel] / np.sqrt(p)
    return out, i, p


def upload(mq, psi):
    n = int(np.log2(len(psi)))
    s = mq.StateVector(n)
    s.upload(psi)
    return s


@pytest.mark.parametrize("auto_reset", [True, False])
def test_measure_in_place_matches_restatement(mq, auto_reset):
    rng = np.random.default_rng(3)
    n = 11
    for pos in (1, 5, 11):
        psi = rand_state(n, rng)
        s = upload(mq, psi)
        seed = int(rng.integers(1 << 30))
        i, p = mq.measure_(s, pos, auto_reset=auto_reset, rng=np.random.default_rng(seed))
        ref, ri, rp = ref_measure(psi, n, pos, auto_reset, np.random.default_rng(seed), mq)
        assert (i, pytest.approx(p, abs=1e-13)) == (ri, rp)
        assert np.max(np.abs(s.to_numpy() - ref)) <= 1e-12
        # the reference's check_measure: measuring again gives the same outcome with p = 1
        _, i2, p2 = mq.measure(s, pos)
        assert i2 == (0 if auto_reset else i) and p2 == pytest.approx(1, abs=1e-10)


def test_batch_and_density_measurement(mq):
    rng = np.random.default_rng(4)
    n, B = 9, 5
    psis = [rand_state(n, rng) for _ in range(B)]
    bs = mq.BatchStateVector(n, B)
    bs.upload(np.stack(psis, axis=1))
    outcomes, probs = mq.measure_(bs, 4, auto_reset=False, rng=np.random.default_rng(10))
    r = np.random.default_rng(10)
    out = bs.to_numpy()
    bit = 1 << 3
    idx = np.arange(1 << n)
    for b in range(B):
        p0 = np.sum(np.abs(psis[b][(idx & bit) == 0]) ** 2)
        dist = np.array([p0, 1 - p0])
        i = ref_discrete_sample(r, dist / dist.sum())
        assert outcomes[b] == i
        ref = np.where(((idx & bit) != 0) == bool(i), psis[b], 0) / np.sqrt(dist[i])
        assert np.max(np.abs(out[:, b] - ref)) <= 1e-12
    # density matrix: rho' = m rho m^dagger with m = |0><i| / sqrt(p) (automatic reset)
    nd = 5
    psi = rand_state(nd, rng)
    rho = np.outer(psi, psi.conj())
    dm = mq.DensityMatrix(nd)
    dm.upload(rho)
    i, p = mq.measure_(dm, 2, auto_reset=True, rng=np.random.default_rng(12))
    P = np.zeros((2, 2))
    P[0, i] = 1 / np.sqrt(p)
    M = np.kron(np.kron(np.eye(1 << (nd - 2)), P), np.eye(2))   # qubit 2 is bit 1
    assert np.max(np.abs(dm.to_numpy() - M @ rho @ M.conj().T)) <= 1e-12
    assert np.trace(dm.to_numpy()).real == pytest.approx(1, abs=1e-12)


def test_measure_removes_qubit(mq):
    rng = np.random.default_rng(5)
    n = 10
    psi = rand_state(n, rng)
    s = upload(mq, psi)
    small, i, p = mq.measure(s, 3, rng=np.random.default_rng(2))
    t = psi.reshape((1 << (n - 3), 2, 4))[:, i, :].reshape(-1) / np.sqrt(p)
    assert small.n == n - 1 and np.max(np.abs(small.to_numpy() - t)) <= 1e-12
    assert np.max(np.abs(s.to_numpy() - psi)) == 0.0   # input unchanged


def test_post_selection_known_answers(mq):
    bell = np.zeros(4, dtype=complex)
    bell[0] = bell[3] = np.sqrt(2) / 2
    for outcome, expected in ((0, [1, 0]), (1, [0, 1])):
        r, p = mq.post_select(upload(mq, bell), 1, outcome)
        assert np.max(np.abs(r.to_numpy() - np.array(expected))) <= 1e-12 and p == pytest.approx(0.5, abs=1e-14)
    rng = np.random.default_rng(6)
    s = upload(mq, rand_state(8, rng))
    mq.post_select_(s, 3, 1)
    _, i, p = mq.measure(s, 3)
    assert i == 1 and p == pytest.approx(1, abs=1e-10)
    zero = upload(mq, np.eye(1, 16, 0)[0].astype(complex))
    with pytest.raises(ValueError):
        mq.post_select_(zero, 2, 1)
    kept, p = mq.post_select(upload(mq, bell), 2, 1, keep=True)
    assert kept.n == 2 and np.max(np.abs(kept.to_numpy() - np.array([0, 0, 0, 1]))) <= 1e-12


def test_simulate_records(mq, O):
    n = 6
    c = mq.QCircuit([mq.HGate(1), mq.CNOTGate(1, 2), mq.RyGate(3, 0.7), mq.QMeasure(1, auto_reset=False),
                     mq.CNOTGate(3, 4), mq.QSelect(4, 1), mq.HGate(5), mq.QMeasure(5)])
    res = mq.simulate(c, mq.StateVector(n), rng=np.random.default_rng(7))
    kinds = [r.kind for r in res.records]
    assert kinds == ["measurement", "postselection", "measurement"]
    # replay on the host with the same generator
    r = np.random.default_rng(7)
    psi = O.apply(mq.QCircuit([mq.HGate(1), mq.CNOTGate(1, 2), mq.RyGate(3, 0.7)]).specs(), O.zero_state(n), n)
    psi, i1, p1 = ref_measure(psi, n, 1, False, r, mq)
    psi = O.apply(mq.QCircuit([mq.CNOTGate(3, 4)]).specs(), psi, n)
    idx = np.arange(1 << n)
    sel = (idx & 8) != 0
    ps = np.sum(np.abs(psi[sel]) ** 2)
    psi = np.where(sel, psi, 0) / np.sqrt(ps)
    psi = O.apply(mq.QCircuit([mq.HGate(5)]).specs(), psi, n)
    psi, i3, p3 = ref_measure(psi, n, 5, True, r, mq)
    assert [x.outcome for x in res.records] == [i1, 1, i3]
    assert np.allclose([x.probability for x in res.records], [p1, ps, p3], atol=1e-13)
    assert np.max(np.abs(res.state.to_numpy() - psi)) <= 1e-12
