"""Kraus channels, mirroring ``QuantumMap`` and the physical noise constructors.

Reference files: src/quantum_circuits/channels/quantum_map.jl:9-93 (QuantumMap, supermatrix,
validation) and channels/one_qubit.jl:1-104 (AmplitudeDamping ... ThermalRelaxation).
"""
from __future__ import annotations

import itertools

import numpy as np

from . import _native as N
from .gates import Instruction, _I2, _X, _Y, _Z


def _channel_tolerance(atol=None):
    return 1e-8 if atol is None else atol


def _noise_probability(value, name, upper=1.0):
    value = float(value)
    if not (np.isfinite(value) and 0 <= value <= upper):
        raise ValueError(f"{name} must be finite and between 0 and {upper}")
    return value


class QuantumMap(Instruction):
    """QuantumMap(positions, kraus; check_tp=False)."""

    name = "QuantumMap"

    def __init__(self, positions, kraus, check_tp=False, atol=None):
        if isinstance(positions, int):
            positions = (positions,)
        positions = tuple(int(p) for p in positions)
        if not positions or any(p <= 0 for p in positions) or len(set(positions)) != len(positions):
            raise ValueError("channel positions must be positive and distinct")
        if not kraus:
            raise ValueError("a channel needs at least one Kraus matrix")
        d = 1 << len(positions)
        ks = []
        for k in kraus:
            k = np.array(k, dtype=complex)
            if k.shape != (d, d):
                raise ValueError("Kraus dimensions must match the register")
            if not np.all(np.isfinite(k)):
                raise ValueError("Kraus matrices must be finite")
            ks.append(k)
        if check_tp:
            s = sum(k.conj().T @ k for k in ks)
            if not np.allclose(s, np.eye(d), atol=_channel_tolerance(atol), rtol=0):
                raise ValueError("noise must be trace preserving")
        self.pos = positions
        self.kraus = ks
        self.spec_name = "QuantumMap"
        self.spec_params = []

    @property
    def positions(self):
        return self.pos

    @property
    def nqubits(self):
        return len(self.pos)

    def kraus_matrices(self):
        return [k.copy() for k in self.kraus]

    def is_tp(self, atol=1e-8):
        d = 1 << len(self.pos)
        return np.allclose(sum(k.conj().T @ k for k in self.kraus), np.eye(d), atol=atol)

    def spec(self):
        if self.spec_name == "QuantumMap":
            return ("channel", "QuantumMap", self.pos, [], None, self.kraus_matrices())
        return ("channel", self.spec_name, self.pos, list(self.spec_params), None, self._spec_data)

    _spec_data = None

    def _ops(self, next_slot, keep):
        op = N.MbOp()
        op.kind = N.MB_OP_CHANNEL
        op.nq = len(self.pos)
        for j, p in enumerate(self.pos):
            op.pos[j] = p - 1
        op.family = 0
        op.slot = -1
        op.nkraus = len(self.kraus)
        buf = np.concatenate([np.asfortranarray(k).ravel(order="F").view(np.float64) for k in self.kraus]).copy()
        keep.append(buf)
        op.data = buf.ctypes.data
        return [op], 0

    def __repr__(self):
        return f"{self.spec_name}{self.pos}"


def _named(channel, name, params, data=None):
    channel.spec_name = name
    channel.spec_params = list(params)
    channel._spec_data = data
    return channel


def AmplitudeDamping(pos, gamma=None, **kw):
    g = _noise_probability(kw.get("γ", gamma), "γ")
    return _named(QuantumMap(pos, [[[1, 0], [0, np.sqrt(1 - g)]], [[0, np.sqrt(g)], [0, 0]]], check_tp=True),
                  "AmplitudeDamping", [g])


def PhaseDamping(pos, gamma=None, **kw):
    g = _noise_probability(kw.get("γ", gamma), "γ")
    return _named(QuantumMap(pos, [[[1, 0], [0, np.sqrt(1 - g)]], [[0, 0], [0, np.sqrt(g)]]], check_tp=True),
                  "PhaseDamping", [g])


def _word(word):
    lookup = {"I": _I2, "X": _X, "Y": _Y, "Z": _Z}
    m = np.ones((1, 1), dtype=complex)
    for c in word:
        m = np.kron(lookup[c], m)
    return m


def MixedUnitary(pos, unitaries, probabilities):
    if len(unitaries) != len(probabilities) or not unitaries:
        raise ValueError("unitaries and probabilities must match")
    w = np.array([_noise_probability(p, "probability") for p in probabilities])
    if not np.isclose(w.sum(), 1, atol=1e-14, rtol=0):
        raise ValueError("probabilities must sum to one")
    w = w / w.sum()
    ks = []
    for p, u in zip(w, unitaries):
        u = np.array(u, dtype=complex)
        if not np.allclose(u.conj().T @ u, np.eye(u.shape[0]), atol=1e-8):
            raise ValueError("matrix is not unitary")
        ks.append(np.sqrt(p) * u)
    return QuantumMap(pos, ks, check_tp=True)


def PauliChannel(pos, words, probabilities):
    register = (pos,) if isinstance(pos, int) else tuple(pos)
    if not 1 <= len(register) <= 2:
        raise ValueError("PauliChannel supports one or two qubits")
    for w in words:
        if len(w) != len(register) or any(c not in "IXYZ" for c in w):
            raise ValueError("Pauli words must match the register and contain I/X/Y/Z")
    ch = MixedUnitary(register, [_word(w) for w in words], probabilities)
    return _named(ch, "PauliChannel", [], (list(words), [float(p) for p in probabilities]))


def BitFlip(pos, p):
    p = _noise_probability(p, "p")
    return _named(PauliChannel(pos, ["I", "X"], [1 - p, p]), "BitFlip", [p])


def PhaseFlip(pos, p):
    p = _noise_probability(p, "p")
    return _named(PauliChannel(pos, ["I", "Z"], [1 - p, p]), "PhaseFlip", [p])


def BitPhaseFlip(pos, p):
    p = _noise_probability(p, "p")
    return _named(PauliChannel(pos, ["I", "Y"], [1 - p, p]), "BitPhaseFlip", [p])


def Depolarizing(pos, p):
    """(1-p) rho + p tr(rho) I/d on one or two qubits (one_qubit.jl:44-57)."""
    register = (pos,) if isinstance(pos, int) else tuple(pos)
    n = len(register)
    if not 1 <= n <= 2:
        raise ValueError("Depolarizing supports one or two qubits")
    count = 4 ** n
    p = _noise_probability(p, "p", upper=count / (count - 1))
    words = ["".join(reversed(w)) for w in itertools.product("IXYZ", repeat=n)]
    probs = [p / count] * count
    probs[0] = max(0.0, 1 - (count - 1) * p / count)
    ch = MixedUnitary(register, [_word(w) for w in words], probs)
    return _named(ch, "Depolarizing", [p])


def GeneralizedAmplitudeDamping(pos, gamma, excited_population=0.0):
    g = _noise_probability(gamma, "γ")
    e = _noise_probability(excited_population, "excited_population")
    ks = [np.sqrt(1 - e) * np.array([[1, 0], [0, np.sqrt(1 - g)]]), np.sqrt(1 - e) * np.array([[0, np.sqrt(g)], [0, 0]]),
          np.sqrt(e) * np.array([[np.sqrt(1 - g), 0], [0, 1]]), np.sqrt(e) * np.array([[0, 0], [np.sqrt(g), 0]])]
    return QuantumMap(pos, ks, check_tp=True)


def ResetChannel(pos, state=0, p=1.0):
    if state not in (0, 1):
        raise ValueError("reset state must be 0 or 1")
    p = _noise_probability(p, "p")
    a = np.zeros((2, 2))
    b = np.zeros((2, 2))
    a[state, 0] = np.sqrt(p)
    b[state, 1] = np.sqrt(p)
    return QuantumMap(pos, [np.sqrt(1 - p) * np.eye(2), a, b], check_tp=True)


def ThermalRelaxation(pos, T1, T2, duration, excited_population=0.0):
    if not (T1 > 0 and T2 > 0 and T2 / 2 <= T1):
        raise ValueError("require positive T1/T2 and T2 <= 2T1")
    if not (np.isfinite(duration) and duration >= 0):
        raise ValueError("duration must be finite and nonnegative")
    g = -np.expm1(-duration / T1)
    inverse_phi = max(0.0, 1 / T2 - (1 / T1) / 2)
    phase = PhaseDamping(pos, gamma=-np.expm1(-2 * duration * inverse_phi))
    amp = GeneralizedAmplitudeDamping(pos, g, excited_population)
    return QuantumMap(pos, [b @ a for a in amp.kraus for b in phase.kraus], check_tp=True)
