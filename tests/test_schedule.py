"""The fused-pass scheduler on the host (mb_schedule_info needs no GPU).

Every circuit must schedule in bounded time with every fused operation in exactly one pass:
density-matrix channels on qubits farther apart than a tile window (paired row/column
windows), 2-qubit gates between distant qubits (a plain pass), the 28-qubit U3 circuit and
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
    assert schedule_info(u, 28) == (20, 20, 0, 0, 1)
    assert schedule_info(W.hea_circuit(10, 8, noise=(0.01, 0.02)), 10, dm=True, nsamples=64)[4] == 1
    for n in (10, 16, 22):
        assert schedule_info(W.hea_circuit(n, 8), n, nsamples=5)[4] == 1


def test_long_range_gates_get_plain_passes():
    rng = np.random.default_rng(3)
    n = 28
    q, _ = np.linalg.qr(rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4)))
    gates = [mq.HGate(p) for p in range(1, n + 1)]
    # (1, 28) is bits 0 and 27: bit 0 is in every tile, so a window at the top holds it;
    # (6, 26) and (4, 20) span more than any window and run as plain passes
    gates += [mq.QuantumGate((6, 26), q), mq.QuantumGate((1, 28), q), mq.QuantumGate((4, 20), q), mq.RyGate(14, 0.3)]
    npasses, ntile, nreg, nplain, complete = schedule_info(mq.QCircuit(gates), n)
    assert complete == 1 and nplain == 2
