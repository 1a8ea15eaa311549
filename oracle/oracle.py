"""CPU oracle for the B200 backend: ctypes wrapper over ``liboracle.so``.

TEST INFRASTRUCTURE ONLY. Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` may import this module; the product package never does.

The oracle takes *instruction specs*, plain tuples that describe a circuit without any
product code attached, and computes every matrix here with its own restatement of the
reference formulas, so that a mistake in the product's matrices cannot hide itself:

    ("gate", name, positions, params, active, data)
    ("channel", name, positions, params, None, data)

``positions`` are the reference's 1-based qubit positions in the order the gate was
constructed with; ``data`` is the user matrix of a ``QuantumGate`` / ``CONTROL`` gate or
the Kraus list of a ``QuantumMap``.

Reference formulas restated here (paths inside MOSSQuantum):
  gate matrices ........... src/quantum_circuits/gates/Gates.jl:9-93
  gate position order ..... src/quantum_circuits/gates/abstract_gates.jl:88-112,162-166
  derivative generators ... src/quantum_circuits/gates/differentiation.jl:1-132
  channels ................ src/quantum_circuits/channels/one_qubit.jl:1-104,
                            src/quantum_circuits/channels/quantum_map.jl:16-67
  observables ............. src/quantum_circuits/operators/qubits_term.jl:12-114,
                            src/backends/cpu/operators/utils.jl:1-20
"""
from __future__ import annotations

import ctypes
import itertools
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build() -> str:
    """Compile ``liboracle.so`` with the committed Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def _cpu_tag() -> str:
    """Identifies this host's CPU (model and flags), so a -march=native build is only ever run
    on the kind of CPU it was built for."""
    import hashlib
    try:
        with open("/proc/cpuinfo") as f:
            lines = f.read().splitlines()
    except OSError:
        lines = []
    model = next((ln for ln in lines if ln.startswith("model name")), "")
    flags = next((ln for ln in lines if ln.startswith("flags")), "")
    return hashlib.sha1((model + flags).encode()).hexdigest()[:12]


def use_fast() -> str:
    """Switch this module to the host-native build (-O3 -march=native, FMA contraction), used
    only to time the CPU baseline; parity checks use the portable build."""
    global _lib, _LIB_PATH
    sub = os.path.join("_build", "native-" + _cpu_tag())
    subprocess.run(["make", "-s", "-C", _HERE, "fast", f"FAST_DIR={sub}"], check=True)
    _LIB_PATH = os.path.join(_HERE, sub, "liboracle_fast.so")
    _lib = None
    return _LIB_PATH


class OrOp(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("nq", ctypes.c_int32), ("pos", ctypes.c_int32 * 5),
                ("nparams", ctypes.c_int32), ("mat", ctypes.c_void_p), ("gens", ctypes.c_void_p)]


class OrKey(ctypes.Structure):
    _fields_ = [("k", ctypes.c_int32), ("pos", ctypes.c_int32 * 5), ("mat", ctypes.c_void_p)]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
        L.or_set_threads.argtypes = [ctypes.c_int]
        L.or_apply_circuit.argtypes = [ctypes.POINTER(OrOp), ctypes.c_int, dp, ctypes.c_int, ctypes.c_int]
        L.or_apply_matrix.argtypes = [dp, ctypes.c_int64, ctypes.c_int, ip, dp]
        L.or_expect.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(OrKey), ctypes.c_int, dp]
        L.or_cross_expect.argtypes = [dp, dp, ctypes.c_int, ctypes.POINTER(OrKey), ctypes.c_int, dp]
        L.or_apply_observable.argtypes = [dp, dp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(OrKey), ctypes.c_int]
        L.or_probabilities.argtypes = [dp, ctypes.c_int, ctypes.c_int, ip, ctypes.c_int, dp]
        L.or_adjoint.argtypes = [ctypes.POINTER(OrOp), ctypes.c_int, dp, ctypes.c_int, ctypes.c_int,
                                 ctypes.POINTER(OrKey), ctypes.c_int, dp, dp]
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().or_set_threads(int(n))


# ---------------------------------------------------------------------------------------
# Gate matrices (Gates.jl). Each matrix is in the gate's own position order: the first
# position is the least significant local bit.
# ---------------------------------------------------------------------------------------
_X = np.array([[0, 1], [1, 0]], dtype=complex)
_Y = np.array([[0, -1j], [1j, 0]], dtype=complex)
_Z = np.array([[1, 0], [0, -1]], dtype=complex)
_I2 = np.eye(2, dtype=complex)
_UP = np.array([[1, 0], [0, 0]], dtype=complex)
_DOWN = np.array([[0, 0], [0, 1]], dtype=complex)


def rkron(a, b):
    """rkron(a, b) = kron(b, a) (quantum_circuits/utils/tensor_ops.jl:1)."""
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
    return (rkron(rkron(_UP, _UP), _I2) + rkron(rkron(_UP, _DOWN), _I2) + rkron(rkron(_DOWN, _UP), _I2)
            + rkron(rkron(_DOWN, _DOWN), u))


_SWAP = np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=complex)
_ISWAP = np.array([[1, 0, 0, 0], [0, 0, 1j, 0], [0, 1j, 0, 0], [0, 0, 0, 1]], dtype=complex)


def from_external(m):
    """n_qubits_mat_from_external (tensor_ops.jl:6-14): reverse the bit order."""
    m = np.asarray(m, dtype=complex)
    d = m.shape[0]
    n = int(round(np.log2(d)))
    rev = [int(format(i, f"0{n}b")[::-1], 2) if n > 0 else 0 for i in range(d)]
    return m[np.ix_(rev, rev)]


def GFSIM(theta, phi, dp, dm, dmoff):
    e = np.exp
    m = np.array([[1, 0, 0, 0],
                  [0, e(1j * (dp + dm)) * np.cos(theta), -1j * e(1j * (dp - dmoff)) * np.sin(theta), 0],
                  [0, -1j * e(1j * (dp + dmoff)) * np.sin(theta), e(1j * (dp - dm)) * np.cos(theta), 0],
                  [0, 0, 0, e(1j * (2 * dp - phi))]], dtype=complex)
    return from_external(m)


_FIXED = {
    "X": _X, "Y": _Y, "Z": _Z, "S": np.array([[1, 0], [0, 1j]], dtype=complex),
    "H": (_X + _Z) / np.sqrt(2), "T": np.array([[1, 0], [0, np.exp(1j * np.pi / 4)]], dtype=complex),
    "sqrtX": np.array([[1 + 1j, 1 - 1j], [1 - 1j, 1 + 1j]], dtype=complex) / 2,
    "sqrtY": np.array([[1j, -1j], [1j, 1j]], dtype=complex) / np.sqrt(2j),
    "SWAP": _SWAP, "iSWAP": _ISWAP, "CZ": CONTROL(_Z), "CNOT": CONTROL(_X),
    "TOFFOLI": CONTROLCONTROL(_X), "FREDKIN": rkron(_UP, np.eye(4)) + rkron(_DOWN, _SWAP),
}


def gate_matrix(name, params, data=None):
    """mat(gate) in the gate's own position order."""
    if name in _FIXED:
        return _FIXED[name].copy()
    if name == "RX":
        return Rx(params[0])
    if name == "RY":
        return Ry(params[0])
    if name == "RZ":
        return Rz(params[0])
    if name == "PHASE":
        return PHASE(params[0])
    if name == "CRX":
        return CONTROL(Rx(params[0]))
    if name == "CRY":
        return CONTROL(Ry(params[0]))
    if name == "CRZ":
        return CONTROL(Rz(params[0]))
    if name == "CPHASE":
        return CONTROL(PHASE(params[0]))
    if name == "CCPHASE":
        return CONTROLCONTROL(PHASE(params[0]))
    if name == "FSIM":
        return GFSIM(*params)
    if name == "CONTROL":
        return CONTROL(data)
    if name == "CONTROLCONTROL":
        return CONTROLCONTROL(data)
    if name == "QuantumGate":
        return np.asarray(data, dtype=complex).copy()
    raise KeyError(f"oracle has no matrix for gate {name}")


def _phase_mat_diff(p):
    return np.array([[0, 0], [0, 1j * np.exp(1j * p)]], dtype=complex)


def generators(name, params, active):
    """differentiate(gate) (differentiation.jl): (dU/dθ)' U per active parameter."""
    if not any(active):
        return []
    u = gate_matrix(name, params)
    t = params[0]
    if name in ("RX", "RY", "RZ"):
        rot = {"RX": Rx, "RY": Ry, "RZ": Rz}[name]
        return [(0.5 * rot(t + np.pi)).conj().T @ u]
    if name == "PHASE":
        return [_phase_mat_diff(t).conj().T @ u]
    if name in ("CRX", "CRY", "CRZ"):
        rot = {"CRX": Rx, "CRY": Ry, "CRZ": Rz}[name]
        return [rkron(_DOWN, 0.5 * rot(t + np.pi)).conj().T @ u]
    if name == "CPHASE":
        return [rkron(_DOWN, _phase_mat_diff(t)).conj().T @ u]
    if name == "CCPHASE":
        return [rkron(rkron(_DOWN, _DOWN), _phase_mat_diff(t)).conj().T @ u]
    raise KeyError(f"oracle has no derivative rule for {name}")


def ordered(positions, m):
    """_get_norm_order (abstract_gates.jl:162-166): sort positions, permute local bits so
    that local bit j belongs to the j-th smallest position."""
    positions = list(positions)
    k = len(positions)
    seq = sorted(range(k), key=lambda j: positions[j])
    d = 1 << k
    perm = np.zeros(d, dtype=np.int64)
    for a_new in range(d):
        a_old = 0
        for j in range(k):
            if (a_new >> j) & 1:
                a_old |= 1 << seq[j]
        perm[a_new] = a_old
    m = np.asarray(m, dtype=complex)
    return [positions[s] for s in seq], m[np.ix_(perm, perm)]


# ---------------------------------------------------------------------------------------
# Channels (channels/one_qubit.jl, quantum_map.jl)
# ---------------------------------------------------------------------------------------
def _pauli_word_matrix(word):
    lookup = {"I": _I2, "X": _X, "Y": _Y, "Z": _Z}
    m = np.ones((1, 1), dtype=complex)
    for c in word:
        m = np.kron(lookup[c], m)
    return m


def kraus_matrices(name, params, data, nq):
    if name == "AmplitudeDamping":
        g = params[0]
        return [np.array([[1, 0], [0, np.sqrt(1 - g)]], dtype=complex),
                np.array([[0, np.sqrt(g)], [0, 0]], dtype=complex)]
    if name == "PhaseDamping":
        g = params[0]
        return [np.array([[1, 0], [0, np.sqrt(1 - g)]], dtype=complex),
                np.array([[0, 0], [0, np.sqrt(g)]], dtype=complex)]
    if name in ("Depolarizing", "BitFlip", "PhaseFlip", "BitPhaseFlip", "PauliChannel"):
        if name == "Depolarizing":
            p = params[0]
            count = 4 ** nq
            # Iterators.product varies the first factor fastest.
            words = ["".join(reversed(w)) for w in itertools.product("IXYZ", repeat=nq)]
            probs = [p / count] * count
            probs[0] = max(0.0, 1 - (count - 1) * p / count)
        elif name == "PauliChannel":
            words, probs = data
        else:
            p = params[0]
            words = ["I", {"BitFlip": "X", "PhaseFlip": "Z", "BitPhaseFlip": "Y"}[name]]
            probs = [1 - p, p]
        w = np.array(probs, dtype=float)
        w = w / w.sum()
        return [np.sqrt(pi) * _pauli_word_matrix(word) for pi, word in zip(w, words)]
    if name == "QuantumMap":
        return [np.asarray(k, dtype=complex) for k in data]
    raise KeyError(f"oracle has no Kraus rule for channel {name}")


def supermatrix(kraus):
    """_compute_supermat (quantum_map.jl:59-67): S[(a,c),(b,d)] = sum K[a,b] conj(K[c,d]),
    row index a + D*c, column index b + D*d."""
    d = kraus[0].shape[0]
    s = np.zeros((d * d, d * d), dtype=complex)
    for k in kraus:
        s += np.einsum("ab,cd->cadb", k, k.conj()).reshape(d * d, d * d)
    return s


# ---------------------------------------------------------------------------------------
# Observables (qubits_term.jl, operators/utils.jl)
# ---------------------------------------------------------------------------------------
_OPNAMES = {"X": _X, "Y": _Y, "Z": _Z, "+": np.array([[0, 1], [0, 0]], dtype=complex),
            "-": np.array([[0, 0], [1, 0]], dtype=complex), "I": _I2, "u": _UP, "d": _DOWN,
            "0": _UP, "1": _DOWN}


def observable_keys(terms):
    """terms: iterable of (positions (1-based), ops (names or 2x2), coeff). Returns
    {sorted positions tuple: dense local matrix} like QubitsOperator.data + _get_mat."""
    keys = {}
    for pos, ops, coeff in terms:
        pos = list(pos)
        seq = sorted(range(len(pos)), key=lambda j: pos[j])
        spos = tuple(pos[j] for j in seq)
        mats = [np.asarray(_OPNAMES[ops[j]] if isinstance(ops[j], str) else ops[j], dtype=complex)
                for j in seq]
        if not mats:
            m = np.array([[coeff]], dtype=complex)
        else:
            m = np.ones((1, 1), dtype=complex)
            for x in mats:           # _kron_ops(reverse(ops)): first site is the low bit
                m = np.kron(x, m)
            m = m * coeff
        if spos in keys:
            keys[spos] = keys[spos] + m
        else:
            keys[spos] = m
    return keys


# ---------------------------------------------------------------------------------------
# Spec -> C structures
# ---------------------------------------------------------------------------------------
class _Bound:
    """Keeps the numpy buffers alive while the C arrays point into them."""

    def __init__(self):
        self.keep = []

    def ptr(self, a):
        a = np.ascontiguousarray(a)
        self.keep.append(a)
        return a.ctypes.data


def _colmajor(m):
    return np.asfortranarray(np.asarray(m, dtype=np.complex128)).ravel(order="F")


def _ops_from_specs(specs, n, keep):
    ops = (OrOp * max(1, len(specs)))()
    nparams = 0
    for i, spec in enumerate(specs):
        kind, name, positions, params, active, data = spec
        positions = list(positions)
        op = ops[i]
        if any(p < 1 or p > n for p in positions) or len(set(positions)) != len(positions):
            raise ValueError(f"invalid positions {positions} for {n} qubits")
        if kind == "gate":
            if name == "CNOT":
                op.kind, op.nq = 2, 2
                op.pos[0], op.pos[1] = positions[0] - 1, positions[1] - 1
            elif name == "CZ":
                op.kind, op.nq = 3, 2
                op.pos[0], op.pos[1] = positions[0] - 1, positions[1] - 1
            else:
                op.kind = 0
                dagger = name.endswith("'")
                base = name[:-1] if dagger else name
                m = gate_matrix(base, params, data)
                if dagger:
                    m = m.conj().T
                spos, om = ordered(positions, m)
                op.nq = len(spos)
                for j, p in enumerate(spos):
                    op.pos[j] = p - 1
                op.mat = keep.ptr(_colmajor(om))
                act = list(active) if active else []
                gens = generators(base, params, act) if any(act) else []
                if dagger:
                    # differentiate(AdjointQuantumGate) (differentiation.jl:1-9): u D' u'.
                    u = gate_matrix(base, params, data)
                    gens = [u @ g.conj().T @ u.conj().T for g in gens]
                if gens:
                    g = np.concatenate([_colmajor(ordered(positions, x)[1]) for x in gens])
                    op.gens = keep.ptr(g)
                    op.nparams = len(gens)
                    nparams += len(gens)
        elif kind == "channel":
            ks = kraus_matrices(name, params, data, len(positions))
            seq = sorted(range(len(positions)), key=lambda j: positions[j])
            oks = [ordered(positions, k)[1] for k in ks]
            op.kind, op.nq = 1, len(positions)
            for j, s in enumerate(seq):
                op.pos[j] = positions[s] - 1
            op.mat = keep.ptr(_colmajor(supermatrix(oks)))
        else:
            raise ValueError(f"unknown instruction kind {kind}")
    return ops, nparams


def _keys_struct(terms, keep):
    keys = observable_keys(terms)
    arr = (OrKey * max(1, len(keys)))()
    for i, (pos, m) in enumerate(keys.items()):
        arr[i].k = len(pos)
        for j, p in enumerate(pos):
            arr[i].pos[j] = p - 1
        arr[i].mat = keep.ptr(_colmajor(m))
    return arr, len(keys)


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


# ---------------------------------------------------------------------------------------
# Public oracle entry points
# ---------------------------------------------------------------------------------------
def zero_state(n, dm=False):
    dim = 1 << n
    v = np.zeros(dim * dim if dm else dim, dtype=np.complex128)
    v[0] = 1
    return v


def apply(specs, state, n, dm=False):
    """Apply a circuit spec to a copy of ``state``; returns the new state."""
    keep = _Bound()
    ops, _ = _ops_from_specs(specs, n, keep)
    out = np.array(state, dtype=np.complex128, copy=True)
    rc = lib().or_apply_circuit(ops, len(specs), _dptr(out), n, int(dm))
    if rc != 0:
        raise ValueError("channel applied to a pure state; promote to a density matrix first")
    return out


def apply_matrix(state, positions0, mat):
    out = np.array(state, dtype=np.complex128, copy=True)
    pos = (ctypes.c_int * len(positions0))(*positions0)
    m = _colmajor(mat)
    lib().or_apply_matrix(_dptr(out), out.size, len(positions0), pos, _dptr(m))
    return out


def expect(state, n, terms, dm=False):
    keep = _Bound()
    keys, nk = _keys_struct(terms, keep)
    out = np.zeros(2)
    st = np.ascontiguousarray(state, dtype=np.complex128)
    lib().or_expect(_dptr(st), n, int(dm), keys, nk, _dptr(out))
    return complex(out[0], out[1])


def cross_expect(cstate, state, n, terms):
    keep = _Bound()
    keys, nk = _keys_struct(terms, keep)
    out = np.zeros(2)
    c = np.ascontiguousarray(cstate, dtype=np.complex128)
    s = np.ascontiguousarray(state, dtype=np.complex128)
    lib().or_cross_expect(_dptr(c), _dptr(s), n, keys, nk, _dptr(out))
    return complex(out[0], out[1])


def apply_observable(state, n, terms, dm=False):
    keep = _Bound()
    keys, nk = _keys_struct(terms, keep)
    st = np.ascontiguousarray(state, dtype=np.complex128)
    out = np.zeros_like(st)
    lib().or_apply_observable(_dptr(st), _dptr(out), n, int(dm), keys, nk)
    return out


def probabilities(state, n, qubits=None, dm=False):
    qubits = list(range(1, n + 1)) if qubits is None else list(qubits)
    q0 = (ctypes.c_int * max(1, len(qubits)))(*[q - 1 for q in qubits])
    out = np.zeros(1 << len(qubits))
    st = np.ascontiguousarray(state, dtype=np.complex128)
    rc = lib().or_probabilities(_dptr(st), n, int(dm), q0, len(qubits), _dptr(out))
    if rc != 0:
        raise ValueError(f"invalid probabilities (code {rc})")
    return out


def adjoint(specs, state0, n, terms, dm=False):
    """(value, gradient per active slot in forward order) of Re<H> after the circuit."""
    keep = _Bound()
    ops, nparams = _ops_from_specs(specs, n, keep)
    keys, nk = _keys_struct(terms, keep)
    value = np.zeros(1)
    grads = np.zeros(max(1, nparams))
    st = np.ascontiguousarray(state0, dtype=np.complex128)
    w = lib().or_adjoint(ops, len(specs), _dptr(st), n, int(dm), keys, nk, _dptr(value), _dptr(grads))
    assert w == nparams
    return float(value[0]), grads[:nparams]


def sample(rng, probs, shots):
    """Inverse-CDF sampling (probabilities.jl:107-121) with a numpy Generator."""
    probs = np.asarray(probs, dtype=float)
    cum = np.cumsum(probs)
    total = cum[-1]
    last_positive = int(np.nonzero(probs > 0)[0][-1])
    nbits = int(round(np.log2(len(probs))))
    out = np.zeros((shots, nbits), dtype=np.int64)
    for s in range(shots):
        sel = int(np.searchsorted(cum, rng.random() * total, side="right"))
        basis = last_positive if sel >= len(probs) else sel
        for b in range(nbits):
            out[s, b] = (basis >> b) & 1
    return out
