"""The fused-pass scheduler on the host (mb_schedule_info needs no GPU).

Every circuit must schedule in bounded time with every fused operation in exactly one pass:
density-matrix channels on qubits farther apart than a tile window (paired row/column
windows), 2-qubit gates between distant qubits (two windows of one tile), gates that need
three windows (a plain pass), the 28-qubit U3 circuit and
the uneven-batch circuits, across tile and register widths.
"""
import ctypes
import time

import numpy as np
import pytest

import mossquantum_b200 as mq
from mossquantum_b200 import _native as N
from mossquantum_b200 import workloads as W


def schedule_info(circ, n, dm=False, t=11, R=3, nsamples=1):
    keep, ops, slot = [], [], 0
    for it in circ.flat():
        o, used = it._ops(slot, keep)
        ops.extend(o)
        slot += used
    arr = (N.MbOp * max(1, len(ops)))(*ops)
    out = [ctypes.c_int() for _ in range(5)]
    rc = N.load().mb_schedule_info(arr, len(ops), n, int(dm), t, R, nsamples, *[ctypes.byref(x) for x in out])
    N.check(rc, "mb_schedule_info")
    npasses, ntile, nreg, nplain, complete = [x.value for x in out]
    assert npasses == ntile + nreg + nplain
    return npasses, ntile, nreg, nplain, complete


@pytest.mark.parametrize("t,R", [(10, 3), (11, 3), (12, 4), (11, 4)])
@pytest.mark.parametrize("n", [6, 9, 10, 12])
def test_noisy_density_circuits_schedule(n, t, R):
    c = W.hea_circuit(n, 2, noise=(0.01, 0.02))
    t0 = time.perf_counter()
    npasses, ntile, nreg, nplain, complete = schedule_info(c, n, dm=True, t=t, R=R, nsamples=8)
    assert complete == 1 and time.perf_counter() - t0 < 20
    assert nplain == 0          # paired windows hold every channel and both halves of every gate


def test_config_circuits_schedule():
    u = W.u3_brickwork(28, 20, W.u3_params(28, 20, W.rng_for(1, 0)))
    assert schedule_info(u, 28) == (15, 15, 0, 0, 1)
    assert schedule_info(u, 28, t=12, R=4)[0] <= 12
    assert schedule_info(W.hea_circuit(10, 8, noise=(0.01, 0.02)), 10, dm=True, nsamples=64)[4] == 1
    for n in (10, 16, 22):
        assert schedule_info(W.hea_circuit(n, 8), n, nsamples=5)[4] == 1


def test_long_range_gates_get_plain_passes():
    rng = np.random.default_rng(3)
    n = 28
    q, _ = np.linalg.qr(rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4)))
    u8, _ = np.linalg.qr(rng.normal(size=(8, 8)) + 1j * rng.normal(size=(8, 8)))
    gates = [mq.HGate(p) for p in range(1, n + 1)]
    # (1, 28) is bits 0 and 27: bit 0 is in every tile, so a window at the top holds it;
    # (6, 26) and (4, 20) fit two windows of one tile; the 3-qubit gates on bits (5, 15, 25)
    # and (3, 11, 19) would need three windows and run as plain passes
    gates += [mq.QuantumGate((6, 26), q), mq.QuantumGate((1, 28), q), mq.QuantumGate((4, 20), q), mq.RyGate(14, 0.3),
              mq.QuantumGate((6, 16, 26), u8), mq.QuantumGate((4, 12, 20), u8)]
    npasses, ntile, nreg, nplain, complete = schedule_info(mq.QCircuit(gates), n)
    assert complete == 1 and nplain == 2


def lowering_errors(circ, n, dm=False, t=11, R=3, seed=1):
    keep, ops, slot = [], [], 0
    for it in circ.flat():
        o, used = it._ops(slot, keep)
        ops.extend(o)
        slot += used
    arr = (N.MbOp * max(1, len(ops)))(*ops)
    ea, eb, ec = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    N.check(N.load().mb_lowering_check(arr, len(ops), n, int(dm), t, R, seed, ctypes.byref(ea), ctypes.byref(eb),
                                       ctypes.byref(ec)), "mb_lowering_check")
    return ea.value, max(eb.value, ec.value)


def random_unitary(d, rng):
    z = rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


# The forward lowering splits fixed single-qubit gates into phase, three-shear rotation and
# phase, merges phases across diagonal gates and runs real / RX-type matrices as real
# micro-ops. On the host, the lowered micro-ops applied in the scheduled order must reproduce
# the compiled instructions on a random vector (random entries of size ~0.5: 1e-12 relative),
# both as fused ops in the scheduled order and as the passes' encoded register-stage micro-ops
# (register indices, selectors, grouped phases).
@pytest.mark.parametrize("t,R", [(8, 3), (10, 3), (11, 3), (12, 4)])
def test_lowering_u3_brickwork(t, R):
    n = 14
    c = W.u3_brickwork(n, 6, W.u3_params(n, 6, W.rng_for(1, 14)))
    ea, eb = lowering_errors(c, n, t=t, R=R)
    assert ea <= 1e-12 and eb <= 1e-12, (ea, eb)


def test_lowering_named_and_random_gates():
    rng = np.random.default_rng(12)
    n = 9
    t = lambda: float(rng.uniform(-np.pi, np.pi))
    gates = [mq.HGate(1), mq.XGate(2), mq.YGate(3), mq.ZGate(4), mq.SGate(5), mq.TGate(6), mq.sqrtXGate(7),
             mq.sqrtYGate(8), mq.RxGate(9, t()), mq.RyGate(1, t()), mq.RzGate(2, t()), mq.PHASEGate(3, t()),
             mq.SWAPGate(4, 8), mq.iSWAPGate(2, 6), mq.CZGate(1, 9), mq.CNOTGate(5, 2), mq.TOFFOLIGate(9, 1, 4),
             mq.FREDKINGate(3, 7, 2), mq.CRxGate(4, 6, t()), mq.CRyGate(8, 1, t()), mq.CRzGate(2, 9, t()),
             mq.CPHASEGate(3, 5, t()), mq.CCPHASEGate(1, 2, 3, t())]
    # parametric families are bound on the device; here they enter as their fixed matrices
    gates = [mq.QuantumGate(g.positions, g.mat()) for g in gates]
    for _ in range(3):
        for q in range(1, n + 1):
            gates.append(mq.QuantumGate(q, random_unitary(2, rng)))
        gates.append(mq.QuantumGate((2, 7), random_unitary(4, rng)))
        gates.append(mq.QuantumGate((9, 3, 5), random_unitary(8, rng)))
        gates.append(mq.QuantumGate(4, np.diag(np.exp(1j * rng.uniform(0, 6, size=2)))))
    c = mq.QCircuit(gates)
    for t_bits, R in ((8, 3), (9, 4)):
        ea, eb = lowering_errors(c, n, t=t_bits, R=R)
        assert ea <= 1e-12 and eb <= 1e-12, (ea, eb)


def test_lowering_density_with_channels():
    n = 5
    c = W.u3_brickwork(n, 4, W.u3_params(n, 4, W.rng_for(1, 5)))
    noisy = mq.QCircuit()
    for g in c.flat():
        noisy.push(g)
        for q in g.positions:
            noisy.push(mq.Depolarizing(q, 0.01))
            noisy.push(mq.AmplitudeDamping(q, 0.02))
    for t_bits, R in ((8, 3), (10, 4)):
        ea, eb = lowering_errors(noisy, n, dm=True, t=t_bits, R=R)
        assert ea <= 1e-12 and eb <= 1e-12, (ea, eb)


def test_lowering_reference_recorded_circuit():
    import json
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cpu_scan_circuits.json")
    with open(path) as f:
        case = json.load(f)["cases"]["n15-d20"]
    c = mq.QCircuit([mq.QuantumGate(g.positions, g.mat()) for g in W.cpu_scan_circuit(case["angles_by_layer"]).flat()])
    ea, eb = lowering_errors(c, 15, t=11, R=3)
    assert ea <= 1e-12 and eb <= 1e-12, (ea, eb)


# Parametric families are bound on the host with the code the device binder runs, so the host
# check also covers the per-sample fusion of single-qubit runs: RX, RY, RZ on one qubit become
# one 2x2 per sample, and on density matrices a gate's two halves with the channels after it
# become one 4x4 superoperator per sample.
@pytest.mark.parametrize("t,R", [(8, 3), (11, 3), (12, 4)])
def test_lowering_parametric_hardware_efficient(t, R):
    n, depth = 12, 3
    c = W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(40)))
    ea, eb = lowering_errors(c, n, t=t, R=R)
    assert ea <= 1e-12 and eb <= 1e-12, (ea, eb)


@pytest.mark.parametrize("t,R", [(8, 3), (10, 4)])
def test_lowering_noisy_density_hardware_efficient(t, R):
    n, depth = 5, 2
    c = W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(41)), noise=(0.01, 0.02))
    ea, eb = lowering_errors(c, n, dm=True, t=t, R=R)
    assert ea <= 1e-12 and eb <= 1e-12, (ea, eb)


def test_lowering_reference_recorded_circuit_families():
    import json
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cpu_scan_circuits.json")
    with open(path) as f:
        case = json.load(f)["cases"]["n15-d20"]
    ea, eb = lowering_errors(W.cpu_scan_circuit(case["angles_by_layer"]), 15, t=11, R=3)
    assert ea <= 1e-12 and eb <= 1e-12, (ea, eb)


# Tiles of bits 0..2 plus two windows let one pass continue a CNOT chain at two places (the
# light cones of consecutive layers): the hardware-efficient ansatz on 20..24 qubits needs
# about one pass per layer instead of three. The two-window passes must still lower exactly.
def test_two_window_tiles_cut_passes():
    assert schedule_info(W.hea_circuit(20, 8), 20, t=11, R=3, nsamples=32)[:2] == (8, 8)
    c24 = W.hea_circuit(24, 16, W.hea_angles(24, 16, W.rng_for(3)))
    assert schedule_info(c24, 24, t=10, R=3)[0] <= 27
    n, depth = 17, 6
    c = W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(42)))
    npasses = schedule_info(c, n, t=9, R=3)[0]
    assert npasses <= 12, npasses
    ea, eb = lowering_errors(c, n, t=9, R=3)
    assert ea <= 1e-12 and eb <= 1e-12, (ea, eb)


# Channels whose supermatrix is real with the population/coherence pattern (depolarizing,
# amplitude and phase damping, phase flip, generalized amplitude damping, reset, thermal
# relaxation) lower to the channel micro-op; bit flips and mixed unitaries keep the dense 4x4.
# Both kinds, fused and unfused, must lower exactly.
def test_lowering_channel_forms():
    n = 5
    c = W.u3_brickwork(n, 2, W.u3_params(n, 2, W.rng_for(1, 7)))
    noisy = mq.QCircuit()
    chans = [lambda q: mq.Depolarizing(q, 0.03), lambda q: mq.AmplitudeDamping(q, 0.05),
             lambda q: mq.PhaseDamping(q, 0.04), lambda q: mq.PhaseFlip(q, 0.02),
             lambda q: mq.GeneralizedAmplitudeDamping(q, 0.05, 0.2), lambda q: mq.ResetChannel(q, 0, 0.1),
             lambda q: mq.ThermalRelaxation(q, 50.0, 40.0, 1.0), lambda q: mq.BitFlip(q, 0.02),
             lambda q: mq.BitPhaseFlip(q, 0.01)]
    for i, g in enumerate(c.flat()):
        noisy.push(g)
        for q in g.positions:
            noisy.push(chans[(i + q) % len(chans)](q))
    for t_bits, R in ((8, 3), (10, 4)):
        ea, eb = lowering_errors(noisy, n, dm=True, t=t_bits, R=R)
        assert ea <= 1e-12 and eb <= 1e-12, (ea, eb)
