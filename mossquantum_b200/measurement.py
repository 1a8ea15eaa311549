"""Mid-circuit measurement and post-selection on device states.

Mirrors src/execution/measurement.jl:4-201 (``QMeasure``, ``measure!``, ``measure``, batch
variants), src/execution/post_selection.jl:3-112 (``QSelect``, ``post_select!``,
``post_select``) and the measurement records of ``simulate`` (src/execution/simulation.jl).
The device computes the outcome weights of the qubit (``mb_qubit_weights``) and performs the
collapse (``mb_collapse``, ``mb_remove_qubit``); outcomes are drawn on the host with the
caller's random stream by inverse-CDF sampling (``discrete_sample``, src/execution/sampling.jl:3-18),
so a seeded generator gives the same records for the same state.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _native as N
from .gates import Instruction
from .states import BatchStateVector, StateVector, _DeviceState

_TOL = float(np.sqrt(np.finfo(float).eps))


class QMeasure(Instruction):
    """QMeasure(position; auto_reset=True, keep=True, key=None) (circuits/circuit.jl:7-20)."""

    def __init__(self, position, auto_reset=True, keep=True, key=None):
        self.position = int(position)
        self.auto_reset = bool(auto_reset)
        self.keep = bool(keep)
        self.key = key

    @property
    def positions(self):
        return (self.position,)

    def parameters(self):
        return None


class QSelect(Instruction):
    """QSelect(position, state=0): post-selection of one outcome (circuits/circuit.jl:28-36)."""

    def __init__(self, position, state=0):
        if state not in (0, 1):
            raise ValueError("selected state must be 0 or 1.")
        self.position = int(position)
        self.state = int(state)

    @property
    def positions(self):
        return (self.position,)

    def parameters(self):
        return None


@dataclass
class MeasurementRecord:
    """One recorded measurement or post-selection, before any automatic reset (simulation.jl:2-14)."""
    position: int
    outcome: int
    probability: float
    kind: str                    # "measurement" or "postselection"
    key: object = None


def discrete_sample(rng, weights) -> int:
    """0-based index drawn from finite nonnegative weights (sampling.jl:3-18)."""
    w = np.asarray(weights, dtype=float)
    if w.size == 0:
        raise ValueError("cannot sample an empty distribution")
    if not np.all(np.isfinite(w)) or np.any(w < 0):
        raise ValueError("sampling weights must be finite and nonnegative")
    total = float(np.sum(w))
    if not (np.isfinite(total) and total > 0):
        raise ValueError("sampling weights must have positive finite sum")
    threshold = rng.random() * total
    cumulative, last_positive = 0.0, 0
    for i, x in enumerate(w):
        if x > 0:
            last_positive = i
        cumulative += x
        if threshold < cumulative:
            return i
    return last_positive


def _normalize(p):
    """_normalize_probabilities! (probabilities.jl:23-32)."""
    p = np.asarray(p, dtype=float).copy()
    if not np.all(np.isfinite(p)):
        raise ValueError("probabilities must be finite")
    if np.min(p) < -_TOL:
        raise ValueError("probabilities must be nonnegative")
    p = np.maximum(p, 0.0)
    total = p.sum()
    if not abs(total - 1) <= max(_TOL, _TOL * max(abs(total), 1.0)):
        raise ValueError(f"state probabilities must sum to one; normalize the state first (sum = {total!r})")
    return p / total


def _check_position(state, position):
    if not 1 <= position <= state.n:
        raise ValueError(f"qubit position must be between 1 and {state.n}")


def _weights(state, position):
    w = np.zeros(2 * max(state.batch, 1))
    if state.batch:
        N.check(N.lib().mb_qubit_weights(state.handle, position - 1, N.dptr(w)), "measurement weights")
    return w.reshape(-1, 2)


def _distributions(state, position):
    """Per-sample [p0, p1]: single states use [p0, 1 - p0] (_local_measure), batches both weights."""
    _check_position(state, position)
    w = _weights(state, position)
    if state.is_batch:
        return np.stack([_normalize(row) for row in w]) if state.batch else np.zeros((0, 2))
    return _normalize([w[0, 0], 1.0 - w[0, 0]])[None, :]


def _collapse(state, position, outcomes, probs, auto_reset):
    oc = np.ascontiguousarray(outcomes, dtype=np.int32)
    pr = np.ascontiguousarray(probs, dtype=np.float64)
    if len(oc):
        N.check(N.lib().mb_collapse(state.handle, position - 1, oc.ctypes.data_as(N.ctypes.POINTER(N.ctypes.c_int)),
                                    N.dptr(pr), 1 if auto_reset else 0), "collapse")


def measure_(state, position, auto_reset=True, rng=None):
    """measure!(state, pos; auto_reset): collapse in place; returns (outcome, probability), or
    arrays per sample for batches (draws in column order)."""
    if not isinstance(state, _DeviceState):
        raise TypeError("measure_ needs a B200 state")
    rng = np.random.default_rng() if rng is None else rng
    dist = _distributions(state, position)
    outcomes = np.array([discrete_sample(rng, d) for d in dist], dtype=np.int64)
    probs = dist[np.arange(len(dist)), outcomes] if len(dist) else np.zeros(0)
    _collapse(state, position, outcomes, probs, auto_reset)
    if state.is_batch:
        return outcomes, probs
    return int(outcomes[0]), float(probs[0])


def _remove(state, position, outcomes, scales):
    out = (BatchStateVector(state.n - 1, state.batch) if state.is_batch else StateVector(state.n - 1))
    oc = np.ascontiguousarray(outcomes, dtype=np.int32)
    sc = np.ascontiguousarray(scales, dtype=np.float64)
    if state.batch:
        N.check(N.lib().mb_remove_qubit(state.handle, position - 1, oc.ctypes.data_as(N.ctypes.POINTER(N.ctypes.c_int)),
                                        N.dptr(sc), out.handle), "measure")
    return out


def measure(state, position, rng=None):
    """measure(state, pos): (collapsed state without the qubit, outcome, probability); the
    input is unchanged. Pure states and batches of pure states (measurement.jl:44-56, 94-113)."""
    if not isinstance(state, (StateVector, BatchStateVector)):
        raise TypeError("measure removes a qubit of a pure state or a batch of pure states")
    rng = np.random.default_rng() if rng is None else rng
    dist = _distributions(state, position)
    outcomes = np.array([discrete_sample(rng, d) for d in dist], dtype=np.int64)
    probs = dist[np.arange(len(dist)), outcomes] if len(dist) else np.zeros(0)
    out = _remove(state, position, outcomes, 1.0 / np.sqrt(probs))
    if state.is_batch:
        return out, outcomes, probs
    return out, int(outcomes[0]), float(probs[0])


def _selection_probabilities(state, position, outcome):
    _check_position(state, position)
    w = _weights(state, position)[:, outcome]
    if state.is_batch:
        if np.any(~np.isfinite(w)) or np.any(w <= 0):
            raise ValueError("every batch column must have positive finite post-selection probability")
    elif not w[0] > 0:
        raise ValueError("cannot post-select an outcome with zero probability")
    return w


def post_select_(state, position, outcome=0):
    """post_select!(state, pos, outcome): keep the qubit, renormalise; returns the probability
    (one per sample for batches; every sample is checked before the state changes)."""
    p = _selection_probabilities(state, position, outcome)
    _collapse(state, position, np.full(len(p), outcome), p, False)
    return p if state.is_batch else float(p[0])


def post_select(state, position, outcome=0, keep=False):
    """post_select(state, pos, outcome; keep=False): (new state, probability) without changing
    the input; the selected qubit is removed unless keep=True."""
    p = _selection_probabilities(state, position, outcome)
    if keep:
        out = state.copy()
        _collapse(out, position, np.full(len(p), outcome), p, False)
    else:
        if not isinstance(state, (StateVector, BatchStateVector)):
            raise TypeError("removing the selected qubit needs a pure state")
        out = _remove(state, position, np.full(len(p), outcome), 1.0 / np.sqrt(p))
    return (out, p) if state.is_batch else (out, float(p[0]))


def run_instruction(instruction, state, rng, records):
    """Executes one measurement instruction inside simulate (simulation.jl:145-160)."""
    if isinstance(instruction, QMeasure):
        if not instruction.keep:
            raise ValueError("in-place measurement must keep the measured qubit")
        outcome, prob = measure_(state, instruction.position, instruction.auto_reset, rng)
        if state.is_batch:
            for b in range(state.batch):
                records[b].append(MeasurementRecord(instruction.position, int(outcome[b]), float(prob[b]),
                                                    "measurement", instruction.key))
        else:
            records.append(MeasurementRecord(instruction.position, outcome, prob, "measurement", instruction.key))
        return state
    if isinstance(instruction, QSelect):
        prob = post_select_(state, instruction.position, instruction.state)
        if state.is_batch:
            for b in range(state.batch):
                records[b].append(MeasurementRecord(instruction.position, instruction.state, float(prob[b]),
                                                    "postselection"))
        else:
            records.append(MeasurementRecord(instruction.position, instruction.state, prob, "postselection"))
        return state
    raise TypeError(f"not a measurement instruction: {type(instruction).__name__}")
