"""Circuits and parameter binding.

Mirrors ``QCircuit`` (src/quantum_circuits/circuits/circuit.jl:98-130), ``ParameterMap``
(src/api/parameter_map.jl:24-116) and ``bind_parameters`` (src/api/parameter_binding.jl:19-63).
A circuit lowers to the C ABI's ``mb_op`` array once per register size; active
parameters become slots whose values travel as one ``theta`` vector at apply time, so
rebinding never recompiles the circuit.
"""
from __future__ import annotations

import itertools
import weakref

import numpy as np

from . import _native as N
from .channels import QuantumMap
from .gates import Gate, Instruction


class QCircuit(Instruction):
    """Ordered list of instructions, possibly nested."""

    def __init__(self, items=()):
        self.items = []
        for it in items:
            self.push(it)
        self._compiled = {}

    def push(self, item):
        from .measurement import QMeasure, QSelect
        if not isinstance(item, (Gate, QuantumMap, QCircuit, QMeasure, QSelect)):
            raise TypeError(f"unsupported instruction {type(item).__name__}")
        self.items.append(item)
        self._invalidate()
        return self

    append = push

    def extend(self, items):
        for it in items:
            self.push(it)
        return self

    def _invalidate(self):
        for handle in getattr(self, "_compiled", {}).values():
            handle.close()
        self._compiled = {}

    def __iter__(self):
        return iter(self.items)

    def __len__(self):
        return len(self.items)

    def __getitem__(self, i):
        return self.items[i]

    def flat(self):
        """Instructions in execution order with nested circuits expanded."""
        out = []
        for it in self.items:
            if isinstance(it, QCircuit):
                out.extend(it.flat())
            else:
                out.append(it)
        return out

    def __mul__(self, other):
        """a * b executes b then a (operator composition, docs/conventions.md)."""
        if isinstance(other, QCircuit):
            return QCircuit(list(other.items) + list(self.items))
        return NotImplemented

    def adjoint(self):
        return QCircuit([it.adjoint() for it in reversed(self.flat())])

    def has_measurement(self):
        from .measurement import QMeasure, QSelect
        return any(isinstance(it, (QMeasure, QSelect)) for it in self.flat())

    def has_channel(self):
        return any(isinstance(it, QuantumMap) for it in self.flat())

    def max_position(self):
        m = 0
        for it in self.flat():
            if it.positions:
                m = max(m, max(it.positions))
        return m

    # parameters -------------------------------------------------------------------------
    def active_parameters(self):
        out = []
        for it in self.flat():
            out.extend(it.active_parameters())
        return out

    def nparameters(self):
        return sum(it.nparameters() for it in self.flat())

    def parameters(self):
        out = []
        for it in self.flat():
            p = it.parameters() if isinstance(it, Gate) else None
            if p:
                out.extend(p)
        return out

    def reset_parameters(self, values):
        values = list(values)
        if len(values) != self.nparameters():
            raise ValueError(f"expected {self.nparameters()} values, got {len(values)}")
        if not all(np.isfinite(values)):
            raise ValueError("parameter values must be finite")
        pos = 0
        for it in self.flat():
            k = it.nparameters()
            if k:
                it.reset_parameters(values[pos:pos + k])
                pos += k
        return self

    def copy_instruction(self):
        return QCircuit([it.copy_instruction() for it in self.items])

    def copy(self):
        return self.copy_instruction()

    def specs(self):
        return [it.spec() for it in self.flat()]

    # lowering ---------------------------------------------------------------------------
    def compiled(self, n: int, lowered=None) -> "CompiledCircuit":
        """The C-ABI circuit for an n-qubit register (cached; parameter values excluded).
        lowered: this circuit's ``_matrix_lowering`` when the caller has it already."""
        if lowered is None:
            lowered = _matrix_lowering(self.flat())
        key = (n, lowered[0] if lowered is not None else self._signature())
        h = self._compiled.get(key)
        if h is None:
            if len(self._compiled) > 8:
                self._invalidate()
            h = CompiledCircuit(self, n, lowered)
            self._compiled[key] = h
        return h

    def _signature(self):
        sig = []
        for it in self.flat():
            p = it.parameters() if isinstance(it, Gate) else None
            act = it.is_parameters() if isinstance(it, Gate) else None
            frozen = tuple(v for v, a in zip(p, act) if not a) if p else ()
            extra = None
            base = getattr(it, "parent", it)
            if isinstance(it, Gate) and getattr(base, "family", "MATRIX") == "MATRIX":
                extra = it._sig_bytes()
            if isinstance(it, QuantumMap):
                extra = b"".join(k.tobytes() for k in it.kraus)
            if hasattr(it, "signature_data"):
                extra = it.signature_data()
            sig.append((type(it).__name__, getattr(it, "parent", None).__class__.__name__, it.positions,
                        tuple(act or ()), frozen, extra))
        return hash(tuple(sig))

    def theta(self):
        """Current active parameter values in slot order."""
        return np.array(self.active_parameters(), dtype=np.float64)

    def __repr__(self):
        return f"QCircuit({len(self.items)} instructions)"


_OP_DTYPE = np.dtype(N.MbOp)   # mb_op as a numpy record (same layout as the ctypes struct)


def _matrix_lowering(items):
    """Vectorised lowering of a circuit made only of matrix gates (``QuantumGate``) and fixed
    gates: (signature, mb_op records, buffers they point into), or None for any other circuit.

    Every such instruction lowers to one matrix op without parameters, exactly as its own
    ``_ops`` would: the matrices of the matrix gates are packed column-major into one buffer
    per size (fixed gates point at their class's shared copy), and the records are filled as
    columns. The signature hashes the instruction types, positions and matrix bytes; its
    leading tag keeps it apart from the general signature."""
    from .gates import QuantumGate, _FixedGate
    fixed_ops = _FixedGate._ops
    names, positions = [], []
    groups, fixed, bynq = {}, {}, {}
    for i, it in enumerate(items):
        t = type(it)
        if t is QuantumGate:
            groups.setdefault(len(it.pos), []).append(i)
        elif isinstance(it, _FixedGate) and t._ops is fixed_ops:
            fixed.setdefault(t, []).append(i)
        else:
            return None
        names.append(t.__name__)
        positions.append(it.pos)
        bynq.setdefault(len(it.pos), []).append(i)
    m = len(items)
    recs = np.zeros(m, dtype=_OP_DTYPE)
    keep, blobs, classes = [], [], []
    for k in sorted(groups):
        idx = groups[k]
        d = 1 << k
        raw = b"".join([items[i].data.tobytes() for i in idx])   # row-major matrices
        blobs.append(raw)
        mats = np.frombuffer(raw, dtype=np.complex128).reshape(len(idx), d, d)
        buf = np.ascontiguousarray(mats.transpose(0, 2, 1)).view(np.float64)
        keep.append(buf)
        recs["data"][idx] = np.uint64(buf.ctypes.data) + np.arange(len(idx), dtype=np.uint64) * np.uint64(16 * d * d)
    for t in sorted(fixed, key=lambda t: t.__name__):
        b = t._packed_matrix()
        keep.append(b)
        recs["data"][fixed[t]] = b.ctypes.data
        classes.append((t.__name__, b.tobytes()))
    for k, idx in bynq.items():
        flat = np.fromiter(itertools.chain.from_iterable(positions[i] for i in idx), dtype=np.int32,
                           count=len(idx) * k)
        recs["pos"][idx, :k] = flat.reshape(len(idx), k) - 1
        recs["nq"][idx] = k
    recs["kind"] = N.MB_OP_GATE
    recs["family"] = N.FAMILIES["MATRIX"]
    recs["slot"] = -1
    sig = hash(("matrix-and-fixed-gates", tuple(names), tuple(positions), tuple(classes), tuple(blobs)))
    return sig, recs, keep


class CompiledCircuit:
    """Owner of an ``mb_circuit`` handle."""

    def __init__(self, circuit: QCircuit, n: int, lowered=None):
        """lowered: the circuit's ``_matrix_lowering`` result, when it has one."""
        self.n = n
        if lowered is not None:
            _, recs, keep = lowered
            self.nslots = 0
            self.nparams = 0
            self.slot_map = []
            self.gradient_ok = True
            h = N.ctypes.c_void_p()
            arr = recs.ctypes.data_as(N.ctypes.POINTER(N.MbOp))
            N.check(N.lib().mb_circuit_create(arr, len(recs), n, N.ctypes.byref(h)), "mb_circuit_create")
            self.handle = h
            self._finalizer = weakref.finalize(self, _free_circuit, h.value)
            return
        keep = []
        ops = []
        slot = 0
        gradient_ok = True
        from .gates import gate_is_differentiable
        for it in circuit.flat():
            o, used = it._ops(slot, keep)
            if isinstance(it, Gate) and it.nparameters() and not gate_is_differentiable(it):
                gradient_ok = False
            if used == 0 and it.nparameters():
                # A matrix-family gate with active parameters: its values are frozen into the
                # matrix, so it occupies no device slot; record the host slots it covers.
                pass
            ops.extend(o)
            slot += used
        self.nslots = slot
        self.nparams = circuit.nparameters()
        self.slot_map = self._slot_map(circuit)
        self.gradient_ok = gradient_ok and self.nslots == self.nparams
        arr = (N.MbOp * max(1, len(ops)))(*ops)
        h = N.ctypes.c_void_p()
        N.check(N.lib().mb_circuit_create(arr, len(ops), n, N.ctypes.byref(h)), "mb_circuit_create")
        self.handle = h
        self._finalizer = weakref.finalize(self, _free_circuit, h.value)

    @staticmethod
    def _slot_map(circuit):
        """active_parameters index -> device slot (-1 for matrix-frozen parameters)."""
        out = []
        slot = 0
        for it in circuit.flat():
            k = it.nparameters()
            base = it.parent if hasattr(it, "parent") else it
            fam = getattr(base, "family", "MATRIX")
            for _ in range(k):
                if fam != "MATRIX":
                    out.append(slot)
                    slot += 1
                else:
                    out.append(-1)
        return out

    def theta_from(self, values):
        values = np.asarray(values, dtype=np.float64)
        if values.shape[-1] != self.nparams:
            raise ValueError(f"expected {self.nparams} parameter values, got {values.shape[-1]}")
        idx = [i for i, s in enumerate(self.slot_map) if s >= 0]
        return np.ascontiguousarray(values[..., idx])

    def passes(self):
        v = N.ctypes.c_int()
        N.check(N.lib().mb_circuit_passes(self.handle, N.ctypes.byref(v)))
        return v.value

    def close(self):
        self._finalizer()


def _free_circuit(h):
    if h and N._initialised:
        N.lib().mb_circuit_free(N.ctypes.c_void_p(h))


class ParameterMap:
    """ParameterMap(indices): slot -> independent parameter id (1-based, no gaps)."""

    def __init__(self, template_or_indices, indices=None):
        if indices is None and isinstance(template_or_indices, QCircuit):
            indices = list(range(1, template_or_indices.nparameters() + 1))
        elif indices is None:
            indices = template_or_indices
        elif isinstance(template_or_indices, QCircuit) and len(indices) != template_or_indices.nparameters():
            raise ValueError("parameter map length does not match the template's active slots")
        idx = []
        for i in indices:
            if isinstance(i, (bool, np.bool_)) or int(i) != i or int(i) <= 0:
                raise ValueError("parameter ids must be positive integers")
            idx.append(int(i))
        k = max(idx) if idx else 0
        if set(idx) != set(range(1, k + 1)):
            raise ValueError("parameter ids must cover 1:k without gaps")
        self._indices = tuple(idx)

    def parameter_indices(self):
        return list(self._indices)

    def __len__(self):
        return len(self._indices)

    def nparameters(self):
        return max(self._indices) if self._indices else 0

    def expand(self, values):
        values = np.asarray(values, dtype=np.float64)
        if values.shape[-1] != self.nparameters():
            raise ValueError(f"expected {self.nparameters()} values, got {values.shape[-1]}")
        return values[..., [i - 1 for i in self._indices]]

    def __eq__(self, other):
        return isinstance(other, ParameterMap) and other._indices == self._indices

    def __hash__(self):
        return hash(self._indices)


def accumulate_parameter_gradients(parameter_map: ParameterMap, flat_gradient):
    """shared[j] = sum of slot gradients carrying id j (parameter_map.jl:102-116)."""
    g = np.asarray(flat_gradient, dtype=np.float64)
    if g.shape[-1] != len(parameter_map):
        raise ValueError("one gradient entry per slot required")
    out = np.zeros(g.shape[:-1] + (parameter_map.nparameters(),))
    for i, j in enumerate(parameter_map.parameter_indices()):
        out[..., j - 1] += g[..., i]
    return out


def bind_parameters(template: QCircuit, values, parameter_map: ParameterMap | None = None) -> QCircuit:
    """Independent circuit with active slots bound in order (parameter_binding.jl:19-63)."""
    values = np.asarray(values, dtype=np.float64)
    if parameter_map is not None:
        if len(parameter_map) != template.nparameters():
            raise ValueError("parameter map does not match the template")
        values = parameter_map.expand(values)
    if values.shape != (template.nparameters(),):
        raise ValueError(f"expected {template.nparameters()} values")
    if not np.all(np.isfinite(values)):
        raise ValueError("parameter values must be finite")
    out = template.copy()
    out.reset_parameters(values)
    return out
