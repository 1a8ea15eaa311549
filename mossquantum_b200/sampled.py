"""Parameter-shift, finite-difference and SPSA gradients on the batch engine.

Mirrors src/differentiation/sampled_gradients.jl:1-435 (``ParameterShift``,
``FiniteDifference``, ``SPSAGradient``, ``parameter_shift_rule``, ``estimate_gradient``) for
exact expectation objectives. The reference evaluates every shifted parameter vector as a
separate objective call; here all of them (and the unshifted one) become the samples of one
batch state with per-sample parameters, so one gradient is one batched apply and one batched
expectation (split into chunks that fit the memory limit).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _native as N
from .backend import apply_, expectation
from .gates import AdjointQuantumGate, Gate
from .states import BatchDensityMatrix, BatchStateVector

_TWO_TERM = {"RX", "RY", "RZ", "PHASE", "CPHASE", "CCPHASE"}
_FOUR_TERM = {"CRX", "CRY", "CRZ"}


class ParameterShift:
    """Exact gate-occurrence parameter shifts (sampled_gradients.jl:2)."""

    def __repr__(self):
        return "ParameterShift()"


class FiniteDifference:
    """Central differences with step h (sampled_gradients.jl:4-10)."""

    def __init__(self, step: float = 0.01):
        step = float(step)
        if not (np.isfinite(step) and step > 0):
            raise ValueError("step must be positive and finite")
        self.step = step

    def __repr__(self):
        return f"FiniteDifference(step={self.step})"


class SPSAGradient:
    """Average of `directions` Rademacher simultaneous perturbations (sampled_gradients.jl:12-20)."""

    def __init__(self, step: float = 0.1, directions: int = 8):
        self.step = FiniteDifference(step).step
        if isinstance(directions, bool) or int(directions) != directions or directions < 1:
            raise ValueError("directions must be a positive Int")
        self.directions = int(directions)

    def __repr__(self):
        return f"SPSAGradient(step={self.step}, directions={self.directions})"


SAMPLED_METHODS = (ParameterShift, FiniteDifference, SPSAGradient)


def parameter_shift_rule(gate: Gate, index: int = 1):
    """(coefficient, shift) pairs for the derivative of one active slot, or None."""
    base = gate.parent if isinstance(gate, AdjointQuantumGate) else gate
    fam = getattr(base, "family", "MATRIX")
    if not 1 <= index <= max(1, gate.nparameters()):
        raise IndexError("active parameter index out of range")
    if fam in _TWO_TERM:
        return [(0.5, np.pi / 2), (-0.5, -np.pi / 2)]
    if fam in _FOUR_TERM:
        # controlled rotations have gaps 1/2 and 1: four evaluations
        a = (np.sqrt(2) + 1) / (4 * np.sqrt(2))
        b = (1 - np.sqrt(2)) / (4 * np.sqrt(2))
        return [(a, np.pi / 2), (-a, -np.pi / 2), (b, 3 * np.pi / 2), (-b, -3 * np.pi / 2)]
    return None


def _recipes(template):
    """One shift recipe per active slot of the template, in slot order (None if any is missing)."""
    out = []
    for g in template.flat():
        k = g.nparameters() if isinstance(g, Gate) else 0
        for i in range(k):
            r = parameter_shift_rule(g, i + 1)
            if r is None:
                return None
            out.append(r)
    return out


def supports_sampled(method, objective) -> bool:
    from .objectives import ExpectationObjective
    if not isinstance(objective, ExpectationObjective):
        return False
    if isinstance(method, ParameterShift):
        return _recipes(objective.template) is not None
    return isinstance(method, (FiniteDifference, SPSAGradient))


@dataclass
class GradientEstimate:
    """estimate_gradient's result (sampled_gradients.jl:126-135); exact objectives have zero
    sampling covariance and use no shots."""
    value: float
    gradient: np.ndarray
    covariance: np.ndarray
    shots: int
    evaluations: int


def _evaluate_rows(objective, slot_rows, max_bytes=2 << 30):
    """Objective values for each row of per-slot parameters, as batched device evaluations."""
    from .objectives import BatchExpectationObjective
    init = objective.initial_state
    rows = np.asarray(slot_rows, dtype=np.float64)
    K = rows.shape[0]
    B = init.batch if init.is_batch else 1
    dm = init.is_density or objective.template.has_channel()
    per_sample = 16 * ((1 << (2 * init.n)) if dm else (1 << init.n))
    chunk = max(1, min(K, int(max_bytes // max(1, per_sample * B))))
    weights = objective.sample_weights() if isinstance(objective, BatchExpectationObjective) else np.ones(1)
    out = np.zeros(K)
    for k0 in range(0, K, chunk):
        k1 = min(K, k0 + chunk)
        nk = k1 - k0
        if init.is_batch:
            batch = type(init)(init.n, B * nk)
            N.check(N.lib().mb_state_tile(init.handle, nk, batch.handle), "tile")
            theta = np.repeat(rows[k0:k1], B, axis=0)
        else:
            batch = (BatchDensityMatrix if init.is_density else BatchStateVector)(init.n, nk)
            N.check(N.lib().mb_state_broadcast(init.handle, batch.handle), "broadcast")
            theta = rows[k0:k1]
        res = apply_(objective.template, batch, theta=theta)
        vals = np.real(expectation(objective.observable, res)).reshape(nk, B)
        out[k0:k1] = vals @ weights
    return out


def estimate_gradient(method, objective, values, rng=None) -> GradientEstimate:
    """Gradient of an exact expectation objective by parameter shifts, central differences
    or SPSA, evaluated on the device as batches."""
    from .objectives import UnsupportedGradient
    if not supports_sampled(method, objective):
        raise UnsupportedGradient(f"{method!r} does not support this objective")
    x = np.asarray(values, dtype=np.float64)
    if x.shape != (objective.nparameters(),) or not np.all(np.isfinite(x)):
        raise ValueError(f"expected {objective.nparameters()} finite parameter values")
    pm = objective.parameter_map
    flat = pm.expand(x)
    ids = pm.parameter_indices()
    if isinstance(method, ParameterShift):
        recipes = _recipes(objective.template)
        rows = [flat]
        terms = []
        for slot, recipe in enumerate(recipes):
            for weight, shift in recipe:
                r = flat.copy()
                r[slot] += shift
                rows.append(r)
                terms.append((ids[slot] - 1, weight))
        vals = _evaluate_rows(objective, rows)
        grad = np.zeros(len(x))
        for (target, weight), v in zip(terms, vals[1:]):
            grad[target] += weight * v
        return GradientEstimate(float(vals[0]), grad, np.zeros((len(x), len(x))), 0, len(rows))
    if isinstance(method, FiniteDifference):
        h = method.step
        rows = [flat]
        for i in range(len(x)):
            plus, minus = x.copy(), x.copy()
            plus[i] += h
            minus[i] -= h
            if plus[i] == minus[i]:
                raise ValueError("difference step is below parameter resolution")
            rows += [pm.expand(plus), pm.expand(minus)]
        vals = _evaluate_rows(objective, rows)
        grad = (vals[1::2] - vals[2::2]) / (2 * h)
        return GradientEstimate(float(vals[0]), grad, np.zeros((len(x), len(x))), 0, len(rows))
    # SPSA: directions drawn from rng in order, as in the reference
    rng = np.random.default_rng() if rng is None else rng
    m, h = method.directions, method.step
    dirs = np.array([[1.0 if rng.random() < 0.5 else -1.0 for _ in range(len(x))] for _ in range(m)]).reshape(m, len(x))
    rows = [flat]
    for d in dirs:
        rows += [pm.expand(x + h * d), pm.expand(x - h * d)]
    vals = _evaluate_rows(objective, rows)
    samples = ((vals[1::2] - vals[2::2]) / (2 * h))[:, None] * dirs
    grad = samples.mean(axis=0) if len(x) else np.zeros(0)
    centered = samples - grad
    cov = centered.T @ centered / (m * (m - 1)) if m > 1 else np.zeros((len(x), len(x)))
    return GradientEstimate(float(vals[0]), grad, cov, 0, len(rows))
