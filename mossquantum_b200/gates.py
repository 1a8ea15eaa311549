"""Gate descriptions, mirroring MOSSQuantum's ``QuantumCircuits`` gate types.

Positions are the reference's 1-based qubit positions; the first position of a gate is
the least significant bit of its local matrix (docs/conventions.md:15). ``mat()`` returns
the matrix in the gate's own position order, ``ordered_positions()``/``ordered_mat()``
the sorted form (src/quantum_circuits/gates/abstract_gates.jl:76-166).

Reference files: gates/Gates.jl (matrices), gates/one_qubit.jl, two_qubit.jl,
three_qubit.jl, parametric_gates.jl, quantum_gate.jl.
"""
from __future__ import annotations

import numpy as np

from . import _native as N

_X = np.array([[0, 1], [1, 0]], dtype=complex)
_Y = np.array([[0, -1j], [1j, 0]], dtype=complex)
_Z = np.array([[1, 0], [0, -1]], dtype=complex)
_I2 = np.eye(2, dtype=complex)
_UP = np.array([[1, 0], [0, 0]], dtype=complex)
_DOWN = np.array([[0, 0], [0, 1]], dtype=complex)


def rkron(a, b):
    """``rkron(a, b) = kron(b, a)``: a acts on the lower local bit."""
    return np.kron(b, a)


def Rx(t):
    h = t / 2
    return np.array([[np.cos(h), -1j * np.sin(h)], [-1j * np.sin(h), np.cos(h)]], dtype=complex)


def Ry(t):
    h = t / 2
    return np.array([[np.cos(h), -np.sin(h)], [np.sin(h), np.cos(h)]], dtype=complex)


def Rz(t):
    h = t / 2
    return np.array([[np.exp(-1j * h), 0], [0, np.exp(1j * h)]], dtype=complex)


def PHASE(p):
    return np.array([[1, 0], [0, np.exp(1j * p)]], dtype=complex)


def CONTROL(u):
    return rkron(_UP, _I2) + rkron(_DOWN, np.asarray(u, dtype=complex))


def CONTROLCONTROL(u):
    u = np.asarray(u, dtype=complex)
    return (rkron(rkron(_UP, _UP), _I2) + rkron(rkron(_UP, _DOWN), _I2)
            + rkron(rkron(_DOWN, _UP), _I2) + rkron(rkron(_DOWN, _DOWN), u))


def U3(theta, phi, lam):
    """Standard U3 matrix, for building ``QuantumGate(q, U3(...))`` (no reference type)."""
    c, s = np.cos(theta / 2), np.sin(theta / 2)
    return np.array([[c, -np.exp(1j * lam) * s], [np.exp(1j * phi) * s, np.exp(1j * (phi + lam)) * c]], dtype=complex)


SWAP = np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=complex)
iSWAP = np.array([[1, 0, 0, 0], [0, 0, 1j, 0], [0, 1j, 0, 0], [0, 0, 0, 1]], dtype=complex)


def _from_external(m):
    m = np.asarray(m, dtype=complex)
    n = int(round(np.log2(m.shape[0])))
    rev = [int(format(i, f"0{n}b")[::-1], 2) if n else 0 for i in range(m.shape[0])]
    return m[np.ix_(rev, rev)]


def FSIM(theta, phi, dp=0.0, dm=0.0, dmoff=0.0):
    e = np.exp
    m = np.array([[1, 0, 0, 0],
                  [0, e(1j * (dp + dm)) * np.cos(theta), -1j * e(1j * (dp - dmoff)) * np.sin(theta), 0],
                  [0, -1j * e(1j * (dp + dmoff)) * np.sin(theta), e(1j * (dp - dm)) * np.cos(theta), 0],
                  [0, 0, 0, e(1j * (2 * dp - phi))]], dtype=complex)
    return _from_external(m)


def _ordered(positions, m):
    positions = list(positions)
    k = len(positions)
    seq = sorted(range(k), key=lambda j: positions[j])
    perm = []
    for ap in range(1 << k):
        a = 0
        for j in range(k):
            if (ap >> j) & 1:
                a |= 1 << seq[j]
        perm.append(a)
    m = np.asarray(m, dtype=complex)
    return tuple(positions[s] for s in seq), m[np.ix_(perm, perm)]


class Instruction:
    """AbstractInstruction."""

    def nparameters(self) -> int:
        return 0

    def active_parameters(self):
        return []

    def copy_instruction(self):
        return self


class Gate(Instruction):
    """Gate{N}: a unitary on ``positions`` (1-based)."""

    name = "Gate"
    family = "MATRIX"

    def __init__(self, positions):
        if isinstance(positions, int):
            positions = (positions,)
        self.pos = tuple(int(p) for p in positions)
        if any(p <= 0 for p in self.pos) or len(set(self.pos)) != len(self.pos):
            raise ValueError(f"gate positions must be positive and distinct: {self.pos}")

    @property
    def positions(self):
        return self.pos

    @property
    def nqubits(self):
        return len(self.pos)

    def mat(self) -> np.ndarray:
        raise NotImplementedError

    def ordered_positions(self):
        return tuple(sorted(self.pos))

    def ordered_mat(self):
        return _ordered(self.pos, self.mat())[1]

    # parameters -------------------------------------------------------------------------
    def parameters(self):
        return None

    def is_parameters(self):
        return None

    def adjoint(self):
        return AdjointQuantumGate(self)

    @property
    def H(self):
        return self.adjoint()

    def shift(self, j: int):
        g = self.copy_instruction()
        g.pos = tuple(p + j for p in self.pos)
        return g

    # lowering --------------------------------------------------------------------------
    def spec(self):
        return ("gate", self.name, self.pos, list(self.parameters() or []),
                list(self.is_parameters() or []), self._spec_data())

    def _spec_data(self):
        return None

    def _ops(self, next_slot: int, keep: list):
        """mb_op records for this gate; returns (ops, slots used)."""
        op = N.MbOp()
        op.kind = N.MB_OP_GATE
        op.nq = len(self.pos)
        for j, p in enumerate(self.pos):
            op.pos[j] = p - 1
        op.family = N.FAMILIES["MATRIX"]
        op.slot = -1
        m = np.asfortranarray(self.mat().astype(np.complex128))
        buf = m.ravel(order="F").view(np.float64).copy()
        keep.append(buf)
        op.data = buf.ctypes.data
        return [op], 0

    def _sig_bytes(self):
        """Bytes of the matrix, for the compiled-circuit cache key."""
        return self.mat().tobytes()

    def __repr__(self):
        return f"{type(self).__name__}{self.pos}"


class _FixedGate(Gate):
    matrix = None
    _packed = None  # per class: the matrix as column-major interleaved doubles (read-only)

    def __init__(self, *positions):
        super().__init__(positions[0] if len(positions) == 1 and not isinstance(positions[0], int) else positions)

    def mat(self):
        return np.array(self.matrix, dtype=complex)

    @classmethod
    def _packed_matrix(cls):
        if cls.__dict__.get("_packed") is None:
            buf = np.ascontiguousarray(np.array(cls.matrix, dtype=complex).T).view(np.float64)
            buf.flags.writeable = False
            cls._packed = buf
        return cls._packed

    def _sig_bytes(self):
        return self._packed_matrix().tobytes()

    def _ops(self, next_slot: int, keep: list):
        op = N.MbOp()
        op.kind = N.MB_OP_GATE
        op.nq = len(self.pos)
        for j, p in enumerate(self.pos):
            op.pos[j] = p - 1
        op.family = N.FAMILIES["MATRIX"]
        op.slot = -1
        buf = self._packed_matrix()  # shared by every gate of the class; the library copies it
        keep.append(buf)
        op.data = buf.ctypes.data
        return [op], 0

    def copy_instruction(self):
        return type(self)(*self.pos)


def _fixed(name, matrix, arity, selfadjoint=False, sort_positions=False):
    class G(_FixedGate):
        pass

    G.name = name
    G.matrix = matrix
    G.__name__ = G.__qualname__ = name + "Gate"

    def init(self, *positions):
        if len(positions) == 1 and not isinstance(positions[0], int):
            positions = tuple(positions[0])
        if len(positions) != arity:
            raise ValueError(f"{name}Gate needs {arity} positions")
        if sort_positions:
            positions = tuple(sorted(positions))
        Gate.__init__(self, positions)

    G.__init__ = init
    if selfadjoint:
        G.adjoint = lambda self: self
    return G


XGate = _fixed("X", _X, 1, True)
YGate = _fixed("Y", _Y, 1)
ZGate = _fixed("Z", _Z, 1)
SGate = _fixed("S", np.array([[1, 0], [0, 1j]]), 1)
HGate = _fixed("H", (_X + _Z) / np.sqrt(2), 1)
TGate = _fixed("T", np.array([[1, 0], [0, np.exp(1j * np.pi / 4)]]), 1)
sqrtXGate = _fixed("sqrtX", np.array([[1 + 1j, 1 - 1j], [1 - 1j, 1 + 1j]]) / 2, 1)
sqrtYGate = _fixed("sqrtY", np.array([[1j, -1j], [1j, 1j]]) / np.sqrt(2j), 1)
SWAPGate = _fixed("SWAP", SWAP, 2, True, sort_positions=True)
iSWAPGate = _fixed("iSWAP", iSWAP, 2, sort_positions=True)
CZGate = _fixed("CZ", CONTROL(_Z), 2, True, sort_positions=True)
CNOTGate = _fixed("CNOT", CONTROL(_X), 2, True)
TOFFOLIGate = _fixed("TOFFOLI", CONTROLCONTROL(_X), 3, True)
FREDKINGate = _fixed("FREDKIN", rkron(_UP, np.eye(4)) + rkron(_DOWN, SWAP), 3, True)


class QuantumGate(Gate):
    """QuantumGate(positions, matrix): arbitrary matrix in own position order."""

    name = "QuantumGate"

    def __init__(self, positions, m):
        super().__init__(positions)
        m = np.array(m, dtype=complex)
        d = 1 << len(self.pos)
        if m.shape != (d, d):
            raise ValueError("matrix size does not match the number of positions")
        self.data = m

    def mat(self):
        return self.data.copy()

    def _spec_data(self):
        return self.data.copy()

    def _sig_bytes(self):
        return self.data.tobytes()

    def _ops(self, next_slot: int, keep: list):
        op = N.MbOp()
        op.kind = N.MB_OP_GATE
        op.nq = len(self.pos)
        for j, p in enumerate(self.pos):
            op.pos[j] = p - 1
        op.family = N.FAMILIES["MATRIX"]
        op.slot = -1
        # column-major complex128 as interleaved doubles (a fresh buffer the op points into)
        buf = np.ascontiguousarray(self.data.T).view(np.float64)
        keep.append(buf)
        op.data = buf.ctypes.data
        return [op], 0

    def copy_instruction(self):
        return QuantumGate(self.pos, self.data)


def gate(positions, m):
    return QuantumGate(positions, m)


class CONTROLGate(QuantumGate):
    name = "CONTROL"

    def __init__(self, control, target, u):
        self.target = np.array(u, dtype=complex)
        super().__init__((control, target), CONTROL(self.target))

    def _spec_data(self):
        return self.target.copy()

    def copy_instruction(self):
        return CONTROLGate(self.pos[0], self.pos[1], self.target)


class CONTROLCONTROLGate(QuantumGate):
    name = "CONTROLCONTROL"

    def __init__(self, a, b, c, u):
        self.target = np.array(u, dtype=complex)
        super().__init__((a, b, c), CONTROLCONTROL(self.target))

    def _spec_data(self):
        return self.target.copy()

    def copy_instruction(self):
        return CONTROLCONTROLGate(*self.pos, self.target)


class ParametricGate(Gate):
    """ParametricGate{N} with one parameter (FSIM has five)."""

    nparams = 1
    family = "MATRIX"

    def __init__(self, positions, paras, isparas=False):
        super().__init__(positions)
        paras = [float(p) for p in (paras if isinstance(paras, (list, tuple, np.ndarray)) else [paras])]
        if len(paras) != self.nparams:
            raise ValueError(f"{type(self).__name__} expects {self.nparams} parameter(s)")
        self.paras = paras
        if isinstance(isparas, bool):
            isparas = [isparas] * self.nparams
        self.isparas = [bool(x) for x in isparas]

    def parameters(self):
        return self.paras

    def is_parameters(self):
        return self.isparas

    def active_parameters(self):
        return [p for p, a in zip(self.paras, self.isparas) if a]

    def nparameters(self):
        return sum(self.isparas)

    def reset_parameters(self, values):
        values = list(values)
        if len(values) != self.nparameters():
            raise ValueError("wrong number of parameter values")
        it = iter(values)
        self.paras = [float(next(it)) if a else p for p, a in zip(self.paras, self.isparas)]
        return self

    def activate_parameters(self):
        self.isparas = [True] * self.nparams
        return self

    def deactivate_parameters(self):
        self.isparas = [False] * self.nparams
        return self

    def copy_instruction(self):
        g = type(self).__new__(type(self))
        Gate.__init__(g, self.pos)
        g.paras = list(self.paras)
        g.isparas = list(self.isparas)
        return g

    def _ops(self, next_slot, keep):
        if self.family == "MATRIX":
            if any(self.isparas):
                # Bound at compile time; the device adjoint has no derivative rule for it.
                pass
            return super()._ops(next_slot, keep)
        op = N.MbOp()
        op.kind = N.MB_OP_GATE
        op.nq = len(self.pos)
        for j, p in enumerate(self.pos):
            op.pos[j] = p - 1
        op.family = N.FAMILIES[self.family]
        op.value = self.paras[0]
        op.slot = next_slot if self.isparas[0] else -1
        return [op], (1 if self.isparas[0] else 0)


def _param_gate(name, family, arity, matfun, adjoint_negates=False):
    class G(ParametricGate):
        pass

    G.name = name
    G.family = family
    G.__name__ = G.__qualname__ = name + "Gate"

    def init(self, *args, isparas=False, theta=None):
        if theta is not None:
            positions, value = args, theta
        else:
            positions, value = args[:-1], args[-1]
        if len(positions) == 1 and not isinstance(positions[0], int):
            positions = tuple(positions[0])
        if len(positions) != arity:
            raise ValueError(f"{name}Gate needs {arity} positions")
        ParametricGate.__init__(self, positions, value, isparas)

    G.__init__ = init
    G.mat = lambda self: matfun(self.paras[0])
    if adjoint_negates:
        def adj(self):
            g = self.copy_instruction()
            g.paras = [-p for p in self.paras]
            return g
        G.adjoint = adj
    return G


RxGate = _param_gate("RX", "RX", 1, Rx)
RyGate = _param_gate("RY", "RY", 1, Ry)
RzGate = _param_gate("RZ", "RZ", 1, Rz)
PHASEGate = _param_gate("PHASE", "PHASE", 1, PHASE, adjoint_negates=True)
CRxGate = _param_gate("CRX", "CRX", 2, lambda t: CONTROL(Rx(t)))
CRyGate = _param_gate("CRY", "CRY", 2, lambda t: CONTROL(Ry(t)))
CRzGate = _param_gate("CRZ", "CRZ", 2, lambda t: CONTROL(Rz(t)))
CPHASEGate = _param_gate("CPHASE", "CPHASE", 2, lambda t: CONTROL(PHASE(t)), adjoint_negates=True)
CCPHASEGate = _param_gate("CCPHASE", "CCPHASE", 3, lambda t: CONTROLCONTROL(PHASE(t)), adjoint_negates=True)


class FSIMGate(ParametricGate):
    name = "FSIM"
    nparams = 5

    def __init__(self, c, t, params, isparas=False):
        super().__init__((c, t), list(params), isparas)

    def mat(self):
        return FSIM(*self.paras)


class AdjointQuantumGate(Gate):
    """AdjointQuantumGate(parent): U' of the parent (gates/quantum_gate.jl:32-45)."""

    name = "Adjoint"

    def __init__(self, parent: Gate):
        self.parent = parent
        super().__init__(parent.pos)

    def mat(self):
        return self.parent.mat().conj().T

    def parameters(self):
        return self.parent.parameters()

    def is_parameters(self):
        return self.parent.is_parameters()

    def active_parameters(self):
        return self.parent.active_parameters()

    def nparameters(self):
        return self.parent.nparameters()

    def reset_parameters(self, values):
        self.parent.reset_parameters(values)
        return self

    def adjoint(self):
        return self.parent

    def copy_instruction(self):
        return AdjointQuantumGate(self.parent.copy_instruction())

    def spec(self):
        kind, name, pos, params, active, data = self.parent.spec()
        return (kind, name + "'", pos, params, active, data)

    def _ops(self, next_slot, keep):
        ops, used = self.parent._ops(next_slot, keep)
        op = ops[0]
        if op.family == N.FAMILIES["MATRIX"]:
            m = np.asfortranarray(self.mat().astype(np.complex128))
            buf = m.ravel(order="F").view(np.float64).copy()
            keep.append(buf)
            op.data = buf.ctypes.data
        else:
            op.flags |= N.MB_OPF_ADJOINT
        return ops, used

    def __repr__(self):
        return f"{self.parent!r}'"


# Families with a device derivative rule (differentiation.jl): the adjoint gradient supports them.
DIFFERENTIABLE_FAMILIES = {"RX", "RY", "RZ", "PHASE", "CRX", "CRY", "CRZ", "CPHASE", "CCPHASE"}


def gate_is_differentiable(g: Gate) -> bool:
    if g.nparameters() == 0:
        return True
    base = g.parent if isinstance(g, AdjointQuantumGate) else g
    return getattr(base, "family", "MATRIX") in DIFFERENTIABLE_FAMILIES
