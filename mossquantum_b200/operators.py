"""Observables: ``QubitsTerm`` and ``QubitsOperator``.

Mirrors src/quantum_circuits/operators/qubits_term.jl:12-114 and qubits_operator.jl:1-130.
A term is coeff * (tensor product of 2x2 matrices on sorted positions); an operator is a
sum of terms. Positions are 1-based; the first (smallest) position is the least
significant local bit.
"""
from __future__ import annotations

import weakref

import numpy as np

from . import _native as N

OP_MAPPING = {
    "X": np.array([[0, 1], [1, 0]], dtype=complex), "Y": np.array([[0, -1j], [1j, 0]], dtype=complex),
    "Z": np.array([[1, 0], [0, -1]], dtype=complex), "+": np.array([[0, 1], [0, 0]], dtype=complex),
    "-": np.array([[0, 0], [1, 0]], dtype=complex), "I": np.eye(2, dtype=complex),
    "u": np.array([[1, 0], [0, 0]], dtype=complex), "d": np.array([[0, 0], [0, 1]], dtype=complex),
    "0": np.array([[1, 0], [0, 0]], dtype=complex), "1": np.array([[0, 0], [0, 1]], dtype=complex),
}


def _as_matrix(op):
    if isinstance(op, str):
        if op not in OP_MAPPING:
            raise KeyError(f"unknown operator name {op!r}")
        return OP_MAPPING[op].copy()
    m = np.array(op, dtype=complex)
    if m.shape != (2, 2):
        raise ValueError("local operators must be 2x2 matrices")
    return m


class QubitsTerm:
    """QubitsTerm(positions, ops, coeff) or QubitsTerm({pos: op}, coeff=...)."""

    def __init__(self, positions=(), ops=(), coeff=1.0, **kw):
        if isinstance(positions, dict):
            coeff = kw.get("coeff", ops if not isinstance(ops, tuple) else coeff)
            items = list(positions.items())
            positions = [p for p, _ in items]
            ops = [o for _, o in items]
        positions = [int(p) for p in positions]
        ops = list(ops)
        if len(positions) != len(ops):
            raise ValueError("each operator position needs one local matrix")
        if any(p <= 0 for p in positions):
            raise ValueError("operator positions must be positive")
        if len(set(positions)) != len(positions):
            raise ValueError("operator positions must be distinct")
        order = sorted(range(len(positions)), key=lambda j: positions[j])
        self.positions = [positions[j] for j in order]
        self.op = [_as_matrix(ops[j]) for j in order]
        self.coeff = complex(coeff)
        self.names = [ops[j] if isinstance(ops[j], str) else None for j in order]

    @classmethod
    def of(cls, *pairs, coeff=1.0):
        """QubitsTerm(1 => "Z", 2 => "Z"; coeff=-1) spelled QubitsTerm.of((1, "Z"), (2, "Z"), coeff=-1)."""
        return cls([p for p, _ in pairs], [o for _, o in pairs], coeff)

    def __mul__(self, x):
        if isinstance(x, (int, float, complex, np.number)):
            return QubitsTerm(self.positions, self.op, self.coeff * x)
        return NotImplemented

    __rmul__ = __mul__

    def __neg__(self):
        return self * -1

    def __add__(self, other):
        return QubitsOperator([self]) + other

    def adjoint(self):
        return QubitsTerm(self.positions, [m.conj().T for m in self.op], np.conj(self.coeff))

    def nqubits(self):
        return max(self.positions) if self.positions else 0

    def spec(self):
        return (tuple(self.positions), [m.copy() for m in self.op], self.coeff)


class QubitsOperator:
    """Sum of QubitsTerm."""

    def __init__(self, terms=()):
        if isinstance(terms, QubitsTerm):
            terms = [terms]
        self.terms = [QubitsTerm(t.positions, t.op, t.coeff) for t in terms]
        self._handle = None

    def add(self, term: QubitsTerm):
        self.terms.append(QubitsTerm(term.positions, term.op, term.coeff))
        self._handle = None
        return self

    def __add__(self, other):
        out = QubitsOperator(self.terms)
        if isinstance(other, QubitsTerm):
            out.add(other)
        elif isinstance(other, QubitsOperator):
            for t in other.terms:
                out.add(t)
        elif isinstance(other, (int, float, complex)):
            out.add(QubitsTerm([], [], other))
        else:
            return NotImplemented
        return out

    def __mul__(self, x):
        if isinstance(x, (int, float, complex, np.number)):
            return QubitsOperator([t * x for t in self.terms])
        return NotImplemented

    __rmul__ = __mul__

    def __iter__(self):
        return iter(self.terms)

    def __len__(self):
        return len(self.terms)

    def nqubits(self):
        return max((t.nqubits() for t in self.terms), default=0)

    def specs(self):
        return [t.spec() for t in self.terms]

    def matrix(self, n):
        """Dense 2^n x 2^n matrix (test helper; independent of the device path)."""
        dim = 1 << n
        out = np.zeros((dim, dim), dtype=complex)
        for t in self.terms:
            m = np.ones((1, 1), dtype=complex)
            full = [np.eye(2, dtype=complex)] * n
            for p, o in zip(t.positions, t.op):
                full[p - 1] = o
            for q in range(n):
                m = np.kron(full[q], m)
            out += t.coeff * m
        return out

    def is_hermitian(self):
        keys = {}
        for t in self.terms:
            key = tuple(t.positions)
            m = np.ones((1, 1), dtype=complex)
            for o in t.op:
                m = np.kron(o, m)
            keys[key] = keys.get(key, 0) + t.coeff * m
        return all(np.allclose(m, np.conj(m).T, atol=1e-12) for m in keys.values())

    def handle(self):
        """The C-ABI observable (compiled once)."""
        if self._handle is None:
            self._handle = CompiledObservable(self)
        return self._handle


def as_operator(obs) -> QubitsOperator:
    if isinstance(obs, QubitsOperator):
        return obs
    if isinstance(obs, QubitsTerm):
        return QubitsOperator([obs])
    raise TypeError(f"unsupported observable {type(obs).__name__}")


class CompiledObservable:
    def __init__(self, op: QubitsOperator):
        keep = []
        terms = (N.MbTerm * max(1, len(op.terms)))()
        for i, t in enumerate(op.terms):
            terms[i].nsites = len(t.positions)
            for j, p in enumerate(t.positions):
                terms[i].sites[j] = p - 1
            terms[i].coeff[0] = t.coeff.real
            terms[i].coeff[1] = t.coeff.imag
            if t.positions:
                buf = np.concatenate([np.asfortranarray(m).ravel(order="F").view(np.float64) for m in t.op]).copy()
                keep.append(buf)
                terms[i].ops = buf.ctypes.data
        h = N.ctypes.c_void_p()
        N.check(N.lib().mb_observable_create(terms, len(op.terms), N.ctypes.byref(h)), "mb_observable_create")
        self.handle = h
        self.max_site = op.nqubits()
        self._finalizer = weakref.finalize(self, _free_observable, h.value)


def _free_observable(h):
    if h and N._initialised:
        N.lib().mb_observable_free(N.ctypes.c_void_p(h))
