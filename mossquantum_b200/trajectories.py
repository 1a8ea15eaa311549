"""Kraus trajectories: noisy shots as batches of pure states on the device.

Mirrors KrausTrajectory execution (src/execution/noisy_execution.jl:1-334). Every channel of
the circuit becomes a selection instruction (``MB_FAM_SELECT``) that applies one of its Kraus
operators, chosen per trajectory by an integer parameter; a batch of T trajectories is one
batch state whose samples carry their own choices as per-sample parameter rows, so the gates
and channels between two draws run as fused passes over all trajectories at once.

Draws follow the reference's rules per trajectory, each with its own generator seeded from the
caller's (the reference seeds one Xoshiro per shot): a channel whose operators satisfy
K'K = p I (a mixture: depolarizing, Pauli and flip channels) draws branch j with probability
p_j and applies K_j / sqrt(p_j), independent of the state; any other channel (amplitude or
phase damping) draws with weights ||K_j psi||^2, which the device computes as batched
expectations of K_j'K_j, and applies K_j, the state being renormalised at the end (the
weights of later draws are normalised by their sum, so the renormalisation can wait).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _native as N
from .backend import _draw_samples, apply_, expectation, probabilities
from .channels import QuantumMap
from .circuit import QCircuit
from .gates import Gate
from .operators import QubitsOperator, QubitsTerm
from .states import BatchStateVector, StateVector

_PAULI = {"I": np.eye(2), "X": np.array([[0, 1], [1, 0]]), "Y": np.array([[0, -1j], [1j, 0]]),
          "Z": np.diag([1.0, -1.0])}


class KrausTrajectory:
    """Independent pure-state Kraus trajectories (noisy_execution.jl:5)."""

    def __repr__(self):
        return "KrausTrajectory()"


class DensityMatrixEvolution:
    """Exact Kraus sum on density matrices (the default execution method)."""

    def __repr__(self):
        return "DensityMatrixEvolution()"


class KrausSelect(Gate):
    """One of a channel's operators, chosen by an integer parameter (a trajectory branch)."""

    name = "KrausSelect"
    family = "SELECT"

    def __init__(self, positions, options, index=0, isparas=True):
        super().__init__(positions)
        d = 1 << len(self.pos)
        self.options = [np.array(k, dtype=complex) for k in options]
        if not self.options or any(k.shape != (d, d) for k in self.options):
            raise ValueError("selection operators must match the positions")
        self.index = float(index)
        self.isparas = bool(isparas)

    def mat(self):
        return self.options[int(self.index)].copy()

    def parameters(self):
        return [self.index]

    def is_parameters(self):
        return [self.isparas]

    def active_parameters(self):
        return [self.index] if self.isparas else []

    def nparameters(self):
        return 1 if self.isparas else 0

    def reset_parameters(self, values):
        (self.index,) = [float(v) for v in values]
        return self

    def copy_instruction(self):
        return KrausSelect(self.pos, self.options, self.index, self.isparas)

    def signature_data(self):
        return b"".join(k.tobytes() for k in self.options)

    def _ops(self, next_slot, keep):
        op = N.MbOp()
        op.kind = N.MB_OP_GATE
        op.nq = len(self.pos)
        for j, p in enumerate(self.pos):
            op.pos[j] = p - 1
        op.family = N.FAMILIES["SELECT"]
        buf = np.concatenate([np.asfortranarray(k).ravel(order="F").view(np.float64) for k in self.options])
        keep.append(buf)
        op.data = buf.ctypes.data
        op.nkraus = len(self.options)
        op.value = self.index
        op.slot = next_slot if self.isparas else -1
        return [op], (1 if self.isparas else 0)


@dataclass
class _Channel:
    positions: tuple
    kraus: list
    mixture: bool
    weights: np.ndarray | None      # mixture: branch probabilities (p_j > 0 only)
    options: list                   # operators the selection applies
    probes: list | None             # general channel: observables K_j'K_j


def _pauli_operator(M, positions):
    """QubitsOperator equal to the Hermitian matrix M on positions (Pauli expansion)."""
    k = len(positions)
    terms = []
    for idx in range(4 ** k):
        word = [("I", "X", "Y", "Z")[(idx >> (2 * j)) & 3] for j in range(k)]
        P = np.array([[1.0]])
        for w in reversed(word):   # first position = least significant factor
            P = np.kron(P, _PAULI[w])
        c = np.trace(P.conj().T @ M) / (1 << k)
        if abs(c) > 1e-15:
            sites = [p for p, w in zip(positions, word) if w != "I"]
            ops = [w for w in word if w != "I"]
            terms.append(QubitsTerm(sites, ops, complex(c)))
    return QubitsOperator(terms)


def _compile_channel(ch: QuantumMap) -> _Channel:
    ks = [np.array(k, dtype=complex) for k in ch.kraus]
    d = ks[0].shape[0]
    weights = np.array([np.real(np.sum(np.abs(k) ** 2)) / d for k in ks])
    tol = 1e-12
    mixture = all(np.allclose(k.conj().T @ k, p * np.eye(d), atol=tol * max(p, 1e-300), rtol=0) for k, p in zip(ks, weights))
    if mixture:
        keep = [j for j, p in enumerate(weights) if p > 0]
        return _Channel(tuple(ch.positions), ks, True, weights[keep], [ks[j] / np.sqrt(weights[j]) for j in keep], None)
    probes = [_pauli_operator(k.conj().T @ k, list(ch.positions)) for k in ks]
    return _Channel(tuple(ch.positions), ks, False, None, ks, probes)


def _plan(circuit):
    """Segments of the trajectory circuit: each starts at a state-dependent channel (or at the
    beginning) and holds the gates and selections up to the next one."""
    segments = [[]]
    for it in (circuit.flat() if isinstance(circuit, QCircuit) else [circuit]):
        if isinstance(it, QuantumMap):
            ch = _compile_channel(it)
            if not ch.mixture:
                segments.append([])
            segments[-1].append(ch)
        elif isinstance(it, Gate):
            u = it.mat()
            if not (np.all(np.isfinite(u)) and np.allclose(u.conj().T @ u, np.eye(len(u)), atol=1e-12)):
                raise ValueError("trajectory gates must be finite and unitary")
            segments[-1].append(it)
        else:
            raise N.UnsupportedOperation(f"KrausTrajectory cannot run {type(it).__name__}")
    return segments


def _segment_circuit(items):
    c = QCircuit()
    for it in items:
        if isinstance(it, _Channel):
            c.push(KrausSelect(it.positions, it.options, 0, isparas=True))
        else:
            c.push(it)
    return c


def run_trajectories(circuit, initial: StateVector, ntraj: int, rng=None, seeds=None):
    """Final normalised states of `ntraj` trajectories (a BatchStateVector) and their branch
    choices; trajectory t draws from np.random.default_rng(seeds[t]) (seeds drawn from rng)."""
    if not isinstance(initial, StateVector):
        raise TypeError("trajectories start from a StateVector")
    rng = np.random.default_rng() if rng is None else rng
    if seeds is None:
        seeds = rng.integers(0, 2**63 - 1, size=ntraj, dtype=np.int64)
    gens = [np.random.default_rng(int(s)) for s in seeds]
    n = initial.n
    state = BatchStateVector(n, ntraj)
    N.check(N.lib().mb_state_broadcast(initial.handle, state.handle), "broadcast")
    choices = [[] for _ in range(ntraj)]
    for seg in _plan(circuit):
        if not seg:
            continue
        rows = []
        head = seg[0]
        general_w = None
        if isinstance(head, _Channel) and not head.mixture:
            # state-dependent weights ||K_j psi_t||^2 from batched expectations
            general_w = np.stack([np.real(expectation(pr, state)) for pr in head.probes], axis=1)
        for t in range(ntraj):
            row = []
            for it in seg:
                if not isinstance(it, _Channel):
                    continue
                if it.mixture:
                    j = _discrete(gens[t], it.weights)
                else:
                    j = _discrete(gens[t], np.maximum(general_w[t], 0.0))
                row.append(j)
                choices[t].append(j)
            rows.append(row)
        c = _segment_circuit(seg)
        theta = np.asarray(rows, dtype=np.float64).reshape(ntraj, -1)
        state = apply_(c, state, theta=theta if theta.shape[1] else None)
    # renormalise (general branches applied K_j without 1/sqrt(w_j))
    norms = np.real(expectation(QubitsTerm([], [], 1.0), state))
    scale = np.ascontiguousarray(1.0 / np.sqrt(norms))
    N.check(N.lib().mb_scale_samples(state.handle, N.dptr(scale)), "normalize")
    return state, choices, gens


def _discrete(gen, weights):
    from .measurement import discrete_sample
    return discrete_sample(gen, weights)


@dataclass
class CountsResult:
    """Streaming counts (noisy_execution.jl:17-22): shots attempted, shots accepted, the
    readout qubits and the histogram (leftmost character = first qubit)."""
    shots: int
    accepted: int
    qubits: list
    counts: dict


def execute(circuit, initial: StateVector, shots: int, qubits=None, rng=None, method=None, chunk=4096):
    """Noisy shots: with KrausTrajectory each shot is one trajectory followed by one readout
    draw of its final state (from the shot's own generator); trajectories run in batches of
    `chunk`. With DensityMatrixEvolution (default) the exact density matrix is evolved once
    and the shots are drawn from its probabilities."""
    rng = np.random.default_rng() if rng is None else rng
    qubits = list(range(1, initial.n + 1)) if qubits is None else [int(q) for q in qubits]
    hist = {}
    if method is None or isinstance(method, DensityMatrixEvolution):
        from .states import density_of
        rho = apply_(circuit, density_of(initial.copy()) if not initial.is_density else initial.copy())
        draws = _draw_samples(rng, probabilities(rho, qubits), shots, len(qubits))
        for row in draws:
            key = "".join(str(int(x)) for x in row)
            hist[key] = hist.get(key, 0) + 1
        return CountsResult(shots, shots, qubits, hist)
    if not isinstance(method, KrausTrajectory):
        raise ValueError("unsupported noise method")
    done = 0
    while done < shots:
        T = min(chunk, shots - done)
        state, _, gens = run_trajectories(circuit, initial, T, rng)
        probs = probabilities(state, qubits)
        for t in range(T):
            row = _draw_samples(gens[t], probs[:, t], 1, len(qubits))[0]
            key = "".join(str(int(x)) for x in row)
            hist[key] = hist.get(key, 0) + 1
        done += T
    return CountsResult(shots, shots, qubits, hist)
