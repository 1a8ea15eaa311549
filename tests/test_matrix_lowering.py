"""The vectorised lowering of circuits made of matrix gates and fixed gates (host, no GPU).

`_matrix_lowering` must hand `mb_circuit_create` exactly what the per-instruction lowering
(`_ops`) does: the same records field by field, pointing at the same matrix bytes, and a
signature that tells circuits with different matrices apart. Circuits with any other
instruction take the per-instruction path.
"""
import ctypes

import numpy as np

import mossquantum_b200 as mq
from mossquantum_b200 import workloads as W
from mossquantum_b200.circuit import _matrix_lowering


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
        plain = _matrix_lowering(items)
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
    assert _matrix_lowering([mq.RxGate(1, 0.3)]) is None
    assert _matrix_lowering([mq.HGate(1), mq.AmplitudeDamping(1, 0.1)]) is None


def test_signature_follows_the_matrices():
    a = W.u3_brickwork(6, 2, W.u3_params(6, 2, W.rng_for(1, 0)))
    b = W.u3_brickwork(6, 2, W.u3_params(6, 2, W.rng_for(1, 1)))
    assert _matrix_lowering(a.flat())[0] != _matrix_lowering(b.flat())[0]
    assert _matrix_lowering(a.flat())[0] == _matrix_lowering(a.copy().flat())[0]
    # same matrices on other positions
    c = mq.QCircuit([mq.QuantumGate(1, np.eye(2)), mq.CZGate(1, 2)])
    d = mq.QCircuit([mq.QuantumGate(2, np.eye(2)), mq.CZGate(1, 2)])
    assert _matrix_lowering(c.flat())[0] != _matrix_lowering(d.flat())[0]


def test_apply_routes_matrix_circuits_through_the_vectorised_lowering(monkeypatch):
    """apply_ on a circuit of matrix and fixed gates lowers it once (the compile cache hit on
    the second call creates nothing), keeps the fused/plain flag the caller asked for, and
    leaves out-of-range positions and other instructions to the general checks."""
    import importlib

    import pytest

    from mossquantum_b200 import _native as N
    from mossquantum_b200.states import StateVector
    backend = importlib.import_module("mossquantum_b200.backend")
    calls = []

    class FakeLib:
        def mb_circuit_create(self, arr, nops, n, out):
            calls.append(("create", nops))
            out._obj.value = 1
            return 0

        def mb_apply(self, circuit, state, theta, ntheta, flags):
            calls.append(("apply", ntheta, flags))
            return 0

        def mb_circuit_free(self, h):
            return 0

    monkeypatch.setattr(N, "lib", lambda: FakeLib())
    state = object.__new__(StateVector)   # a host stand-in: no device memory is touched
    state.n, state.batch, state.handle = 6, 0, ctypes.c_void_p(1)
    c = mq.QCircuit([mq.HGate(1), mq.CZGate(1, 2), mq.QuantumGate((3, 4), np.eye(4))])
    rx = mq.RxGate(1, 0.3)
    try:
        backend.apply_(c, state)
        backend.apply_(c, state, plain=True)
        assert calls == [("create", 3), ("apply", 0, N.MB_APPLY_FUSED), ("apply", 0, N.MB_APPLY_PLAIN)]
        with pytest.raises(ValueError):
            backend.apply_(mq.QCircuit([mq.HGate(7)]), state)
        backend.apply_(rx, state)   # general path
        assert calls[-1][0] == "apply"
    finally:
        # the fake handles must never reach the real library's free
        for circ in (c, getattr(rx, "_as_circuit", None)):
            for h in (getattr(circ, "_compiled", None) or {}).values():
                h._finalizer.detach()
