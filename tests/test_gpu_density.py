"""Density matrices and Kraus channels on the GPU vs the oracle.

Mirrors test/unit/batch_density_execution.jl:12-45 (U rho U' per sample) and
test/unit/noise_channels.jl:3-40 (channels vs sum K rho K', closed forms).
Tolerance: 1e-12 max-abs on density entries.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-12


def random_density(n, rng, rank=None):
    d = 1 << n
    a = rng.normal(size=(d, rank or d)) + 1j * rng.normal(size=(d, rank or d))
    r = a @ a.conj().T
    return r / np.trace(r)


def test_gates_on_density(mq, O):
    from tests.test_gpu_gates import named_gates
    n = 6
    rng = np.random.default_rng(21)
    rho = random_density(n, rng)
    c = mq.QCircuit(named_gates(mq, n, rng))
    for plain in (False, True):
        s = mq.apply_(c, mq.DensityMatrix(rho), plain=plain)
        ref = O.apply(c.specs(), rho.ravel(order="F"), n, True)
        assert np.max(np.abs(s.to_numpy().ravel(order="F") - ref)) <= TOL


def test_channels(mq, O):
    n = 4
    rng = np.random.default_rng(22)
    rho = random_density(n, rng)
    chans = [mq.AmplitudeDamping(1, 0.3), mq.PhaseDamping(2, gamma=0.4), mq.Depolarizing(3, 0.2),
             mq.Depolarizing((4, 2), 0.3), mq.BitFlip(1, 0.1), mq.PhaseFlip(4, 0.25), mq.BitPhaseFlip(3, 0.3),
             mq.PauliChannel((2, 3), ["XY", "ZI", "II"], [0.2, 0.3, 0.5]),
             mq.GeneralizedAmplitudeDamping(2, 0.3, 0.2), mq.ResetChannel(1, state=1, p=0.4),
             mq.ThermalRelaxation(3, 10.0, 15.0, 2.0)]
    c = mq.QCircuit(chans)
    s = mq.apply_(c, mq.DensityMatrix(rho))
    ref = O.apply(c.specs(), rho.ravel(order="F"), n, True)
    assert np.max(np.abs(s.to_numpy().ravel(order="F") - ref)) <= TOL
    assert abs(np.trace(s.to_numpy()) - 1) < 1e-12


def test_depolarizing_closed_form(mq):
    rng = np.random.default_rng(172)
    rho = random_density(1, rng)
    for p in (0.0, 0.5, 1.0, 4 / 3):
        s = mq.apply_(mq.Depolarizing(1, p), mq.DensityMatrix(rho))
        np.testing.assert_allclose(s.to_numpy(), (1 - p) * rho + p * np.eye(2) / 2, atol=1e-14)


def test_channel_on_pure_state_promotes(mq, O):
    n = 3
    s = mq.apply_(mq.HGate(1), mq.StateVector(n))
    out = mq.apply_(mq.AmplitudeDamping(1, 0.5), s)
    assert isinstance(out, mq.DensityMatrix)
    psi = O.apply([("gate", "H", (1,), [], [], None)], O.zero_state(n), n)
    rho = np.outer(psi, psi.conj()).ravel(order="F")
    ref = O.apply([("channel", "AmplitudeDamping", (1,), [0.5], None, None)], rho, n, True)
    assert np.max(np.abs(out.to_numpy().ravel(order="F") - ref)) <= TOL


def test_noisy_hea(mq, O):
    from mossquantum_b200 import workloads as W
    n, depth = 5, 3
    c = W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(2, 5)), noise=(0.01, 0.02))
    s = mq.apply_(c, mq.DensityMatrix(n))
    ref = O.apply(c.specs(), O.zero_state(n, True), n, True)
    assert np.max(np.abs(s.to_numpy().ravel(order="F") - ref)) <= TOL
    H = W.xxz(n)
    assert abs(mq.expectation(H, s) - O.expect(ref, n, H.specs(), dm=True)) <= 1e-11


@pytest.mark.parametrize("n,jit", [(7, False), (8, False), (9, True)])
def test_noisy_hea_wider_than_a_tile(mq, O, n, jit, monkeypatch):
    """Density matrices of 2n > tile bits: channels on (q, q+n) and both halves of every gate
    fit paired row/column windows; checked against the oracle (1e-12), single and batched."""
    from mossquantum_b200 import workloads as W
    if jit:
        monkeypatch.setenv("MB_JIT_MIN_BITS", "18")
    c = W.hea_circuit(n, 1, W.hea_angles(n, 1, W.rng_for(2, n)), noise=(0.01, 0.02))
    s = mq.apply_(c, mq.DensityMatrix(n))
    ref = O.apply(c.specs(), O.zero_state(n, True), n, True)
    assert np.max(np.abs(s.to_numpy().ravel(order="F") - ref)) <= TOL
    if n == 7:
        B = 2
        ca = W.hea_circuit(n, 1, noise=(0.01, 0.02))
        thetas = np.random.default_rng(n).uniform(0, 2 * np.pi, size=(B, ca.nparameters()))
        sb = mq.apply_(ca, mq.BatchDensityMatrix(n, B), theta=thetas)
        out = sb.to_numpy()
        for b in range(B):
            rb = O.apply(ca.copy().reset_parameters(thetas[b]).specs(), O.zero_state(n, True), n, True)
            assert np.max(np.abs(out[:, :, b].ravel(order="F") - rb)) <= TOL
