"""Batch states on the GPU: shared and per-sample parameters vs single-state runs / oracle.

Mirrors test/regression/kernels.jl:19-43 (batch gate dispatch for batch sizes 1,2,4,5) and
test/unit/batch_expectations.jl. Tolerance 1e-12.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("B", [1, 2, 4, 5])
def test_batch_shared_and_per_sample(mq, O, B):
    from mossquantum_b200 import workloads as W
    n, depth = 7, 2
    c = W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(7)))
    rng = np.random.default_rng(B)
    cols = rng.normal(size=(1 << n, B)) + 1j * rng.normal(size=(1 << n, B))
    cols /= np.linalg.norm(cols, axis=0)
    s = mq.apply_(c, mq.BatchStateVector(cols))
    out = s.to_numpy()
    for b in range(B):
        ref = O.apply(c.specs(), cols[:, b], n)
        assert np.max(np.abs(out[:, b] - ref)) <= 1e-12
    thetas = rng.uniform(0, 2 * np.pi, size=(B, c.nparameters()))
    s = mq.apply_(c, mq.BatchStateVector(cols), theta=thetas)
    out = s.to_numpy()
    H = W.tfim(n)
    ev = mq.expectation(H, s)
    for b in range(B):
        cb = c.copy().reset_parameters(thetas[b])
        ref = O.apply(cb.specs(), cols[:, b], n)
        assert np.max(np.abs(out[:, b] - ref)) <= 1e-12
        assert abs(ev[b] - O.expect(ref, n, H.specs())) <= 1e-11
    probs = mq.probabilities(s, [1, 3])
    assert probs.shape == (4, B)


def test_batch_density_per_sample(mq, O):
    from mossquantum_b200 import workloads as W
    n, depth, B = 3, 2, 3
    c = W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(8)), noise=(0.01, 0.02))
    thetas = np.random.default_rng(1).uniform(0, 2 * np.pi, size=(B, c.nparameters()))
    s = mq.apply_(c, mq.BatchDensityMatrix(n, B), theta=thetas)
    out = s.to_numpy()
    for b in range(B):
        ref = O.apply(c.copy().reset_parameters(thetas[b]).specs(), O.zero_state(n, True), n, True)
        assert np.max(np.abs(out[:, :, b].ravel(order="F") - ref)) <= 1e-12


def test_empty_batch(mq):
    s = mq.BatchStateVector(3, 0)
    s = mq.apply_(mq.HGate(1), s)
    assert mq.expectation(mq.QubitsTerm([1], ["Z"]), s).shape == (0,)


def test_batches_of_varying_size_share_schedules(mq, O):
    """One circuit over batches of 3, 2, 5 and 4 samples with per-sample angles (the serving
    loop's pattern): forward schedules serve every batch up to a power-of-two capacity, so the
    later batches reuse earlier schedules and their per-sample rows; every sample still matches
    the oracle."""
    from mossquantum_b200 import workloads as W
    n, depth = 12, 3
    c = W.hea_circuit(n, depth)
    rng = np.random.default_rng(31)
    for B in (3, 2, 5, 4):
        th = rng.uniform(0, 2 * np.pi, size=(B, c.nparameters()))
        out = mq.apply_(c, mq.BatchStateVector(n, B), theta=th).to_numpy()
        for b in range(B):
            ref = O.apply(c.copy().reset_parameters(th[b]).specs(), O.zero_state(n), n)
            assert np.max(np.abs(out[:, b] - ref)) <= 1e-12, (B, b)
