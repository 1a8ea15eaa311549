"""The vectorised lowering of circuits made of matrix gates and fixed gates (host, no GPU).

`_plain_lowering` must hand `mb_circuit_create` exactly what the per-instruction lowering
(`_ops`) does: the same records field by field, pointing at the same matrix bytes, and a
signature that tells circuits with different matrices apart. Circuits with any other
instruction take the per-instruction path.
"""
import ctypes

import numpy as np

import mossquantum_b200 as mq
from mossquantum_b200 import workloads as W
from mossquantum_b200.circuit import _plain_lowering


def _unitary(rng, d):
    q, _ = np.linalg.qr(rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d)))
    return q


def _per_instruction(items):
    keep, ops, slot = [], [], 0
    for it in items:
        o, used = it._ops(slot, keep)
        ops.extend(o)
        slot += used
    return ops, keep


def _circuits():
    rng = np.random.default_rng(0)
    yield W.u3_brickwork(12, 3, W.u3_params(12, 3, W.rng_for(1, 0)))
    yield mq.QCircuit()
    c = mq.QCircuit()
    for _ in range(40):
        k = int(rng.integers(1, 4))
        pos = tuple(int(x) for x in rng.choice(np.arange(1, 9), size=k, replace=False))
        r = rng.integers(4)
        if r == 0:
            c.push(mq.QuantumGate(pos, _unitary(rng, 1 << k)))
        elif r == 1:
            c.push(mq.CZGate(pos[0], pos[0] % 8 + 1))
        elif r == 2:
            c.push(mq.HGate(pos[0]))
        else:
            c.push(mq.TOFFOLIGate(1, 2, 3))
    yield c
    yield mq.QCircuit([mq.QCircuit([mq.HGate(1), mq.QuantumGate((2, 5), _unitary(rng, 4))]), mq.SWAPGate(3, 4)])


def test_records_equal_per_instruction_lowering():
    for c in _circuits():
        items = c.flat()
        plain = _plain_lowering(items)
        assert plain is not None
        _, recs, _keep = plain
        ops, _keep2 = _per_instruction(items)
        assert len(ops) == len(recs)
        for a, r in zip(ops, recs):
            assert (a.kind, a.nq, a.family, a.slot, a.flags, a.nkraus, a.value) == (
                r["kind"], r["nq"], r["family"], r["slot"], r["flags"], r["nkraus"], r["value"])
            assert list(a.pos) == list(r["pos"])
            d = 1 << a.nq
            assert ctypes.string_at(a.data, 16 * d * d) == ctypes.string_at(int(r["data"]), 16 * d * d)


def test_other_instructions_take_the_general_path():
    assert _plain_lowering([mq.RxGate(1, 0.3)]) is None
    assert _plain_lowering([mq.HGate(1), mq.AmplitudeDamping(1, 0.1)]) is None


def test_signature_follows_the_matrices():
    a = W.u3_brickwork(6, 2, W.u3_params(6, 2, W.rng_for(1, 0)))
    b = W.u3_brickwork(6, 2, W.u3_params(6, 2, W.rng_for(1, 1)))
    assert _plain_lowering(a.flat())[0] != _plain_lowering(b.flat())[0]
    assert _plain_lowering(a.flat())[0] == _plain_lowering(a.copy().flat())[0]
    # same matrices on other positions
    c = mq.QCircuit([mq.QuantumGate(1, np.eye(2)), mq.CZGate(1, 2)])
    d = mq.QCircuit([mq.QuantumGate(2, np.eye(2)), mq.CZGate(1, 2)])
    assert _plain_lowering(c.flat())[0] != _plain_lowering(d.flat())[0]
