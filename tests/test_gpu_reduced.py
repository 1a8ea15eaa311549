"""Partial trace and fidelities on the device against numpy restatements of
partial_trace.jl:11-97 and the fidelity definitions (1e-12 max-abs)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rand_state(n, rng):
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def ref_ptrace(rho, n, sites):
    """Reduced density matrix: remaining qubits keep their order as the low bits."""
    t = rho.reshape([2] * (2 * n), order="F")          # axis q-1 = qubit q (row), n + q - 1 (column)
    keep = [q for q in range(1, n + 1) if q not in sites]
    for s in sorted(sites, reverse=True):
        t = np.trace(t, axis1=s - 1, axis2=s - 1 + t.ndim // 2)
    m = len(keep)
    return t.reshape((1 << m, 1 << m), order="F")


def test_partial_trace_density_and_pure(mq):
    rng = np.random.default_rng(1)
    n = 7
    psi = rand_state(n, rng)
    phi = rand_state(n, rng)
    rho = 0.6 * np.outer(psi, psi.conj()) + 0.4 * np.outer(phi, phi.conj())
    dm = mq.DensityMatrix(n)
    dm.upload(rho)
    sv = mq.StateVector(n)
    sv.upload(psi)
    for sites in ([1], [7], [2, 5], [6, 1, 3], [1, 2, 3, 4, 5, 6]):
        r = mq.partial_tr(dm, sites)
        assert r.n == n - len(sites)
        assert np.max(np.abs(r.to_numpy() - ref_ptrace(rho, n, sites))) <= 1e-12
        rp = mq.partial_tr(sv, sites)
        assert np.max(np.abs(rp.to_numpy() - ref_ptrace(np.outer(psi, psi.conj()), n, sites))) <= 1e-12
    assert mq.partial_tr(dm, list(range(1, n + 1))) == pytest.approx(1.0, abs=1e-12)
    with pytest.raises(ValueError):
        mq.partial_tr(dm, [2, 2])
    with pytest.raises(ValueError):
        mq.partial_tr(dm, [8])


def test_partial_trace_batches(mq):
    rng = np.random.default_rng(2)
    n, B = 6, 3
    psis = [rand_state(n, rng) for _ in range(B)]
    bs = mq.BatchStateVector(n, B)
    bs.upload(np.stack(psis, axis=1))
    parts = mq.partial_tr(bs, [2, 4])
    assert len(parts) == B
    for b in range(B):
        ref = ref_ptrace(np.outer(psis[b], psis[b].conj()), n, [2, 4])
        assert np.max(np.abs(parts[b].to_numpy() - ref)) <= 1e-12
    bd = mq.BatchDensityMatrix(n, B)
    rhos = [np.outer(p, p.conj()) for p in psis]
    bd.upload(np.stack(rhos, axis=2))
    r = mq.partial_tr(bd, [1, 6]).to_numpy()
    for b in range(B):
        assert np.max(np.abs(r[:, :, b] - ref_ptrace(rhos[b], n, [1, 6]))) <= 1e-12


def test_fidelities(mq):
    rng = np.random.default_rng(3)
    n = 8
    x, y = rand_state(n, rng), rand_state(n, rng)
    sx, sy = mq.StateVector(n), mq.StateVector(n)
    sx.upload(x)
    sy.upload(y)
    assert mq.fidelity(sx, sy) == pytest.approx(abs(np.vdot(x, y)) ** 2, abs=1e-13)
    assert mq.inner(sx, sy) == pytest.approx(np.vdot(x, y), abs=1e-13)
    rho = np.outer(x, x.conj()) * 0.7 + np.eye(1 << n) * 0.3 / (1 << n)
    d = mq.DensityMatrix(n)
    d.upload(rho)
    ref = np.real(np.vdot(y, rho @ y))
    assert mq.fidelity(d, sy) == pytest.approx(ref, abs=1e-13)
    assert mq.fidelity(sy, d) == pytest.approx(ref, abs=1e-13)
    with pytest.raises(mq.UnsupportedOperation):
        mq.fidelity(d, d)
    B = 4
    xs = [rand_state(n, rng) for _ in range(B)]
    ys = [rand_state(n, rng) for _ in range(B)]
    bx, by = mq.BatchStateVector(n, B), mq.BatchStateVector(n, B)
    bx.upload(np.stack(xs, axis=1))
    by.upload(np.stack(ys, axis=1))
    np.testing.assert_allclose(mq.fidelity(bx, by), [abs(np.vdot(a, b)) ** 2 for a, b in zip(xs, ys)], atol=1e-13)
