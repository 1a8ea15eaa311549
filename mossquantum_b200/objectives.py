"""Objectives and the device adjoint gradient method.

Mirrors src/api/objectives.jl:15-244 (ExpectationObjective, BatchExpectationObjective,
evaluate, evaluate_batch), src/api/gradient_methods.jl:14-138 (value_and_gradient,
value_and_pullback, supports_gradient, differentiable_value) and the AdjointGradient
implementation of src/differentiation/objectives.jl:79-296, which here runs as one
``mb_adjoint`` call on the GPU.
"""
from __future__ import annotations

import numpy as np

from . import _native as N
from .backend import apply_, expectation
from .circuit import ParameterMap, QCircuit, accumulate_parameter_gradients
from .operators import as_operator
from .states import _DeviceState


class UnsupportedGradient(Exception):
    """Mirror of MOSSQuantum.UnsupportedGradient (gradient_methods.jl:20-25)."""


class AdjointGradient:
    """Adjoint reverse sweep on the device (the B200 counterpart of CPU AdjointGradient)."""

    def __init__(self, checkpoint_every: int = 0):
        self.checkpoint_every = int(checkpoint_every)

    def __repr__(self):
        return f"AdjointGradient(checkpoint_every={self.checkpoint_every})"


B200AdjointGradient = AdjointGradient


class ExpectationObjective:
    """Re <H> after ``template`` bound to the input values, on a copy of ``initial_state``."""

    def __init__(self, template: QCircuit, observable, initial_state: _DeviceState, parameter_map=None):
        if not isinstance(template, QCircuit):
            template = QCircuit([template])
        self.template = template
        self.observable = as_operator(observable)
        self.initial_state = initial_state.copy()
        self.parameter_map = parameter_map if parameter_map is not None else ParameterMap(template)
        if len(self.parameter_map) != template.nparameters():
            raise ValueError("parameter map does not match the template")

    def nparameters(self):
        return self.parameter_map.nparameters()

    def _slots(self, values):
        values = np.asarray(values, dtype=np.float64)
        if values.shape != (self.nparameters(),):
            raise ValueError(f"expected {self.nparameters()} parameter values")
        if not np.all(np.isfinite(values)):
            raise ValueError("parameter values must be finite")
        return self.parameter_map.expand(values)

    def _sample_values(self, values):
        state = apply_(self.template, self.initial_state.copy(), theta=self._slots(values))
        return np.real(np.atleast_1d(expectation(self.observable, state)))

    def evaluate(self, values) -> float:
        return float(self._sample_values(values)[0])


class BatchExpectationObjective(ExpectationObjective):
    """Batch objective reduced by ``:mean`` (default), ``:sum`` or ``:weighted_sum``."""

    def __init__(self, template, observable, initial_state, reduction="mean", weights=None, parameter_map=None):
        if not initial_state.is_batch:
            raise ValueError("BatchExpectationObjective needs a batch state")
        if initial_state.batch < 1:
            raise ValueError("scalar batch objectives require at least one sample")
        super().__init__(template, observable, initial_state, parameter_map)
        reduction = reduction.lstrip(":")
        if reduction not in ("mean", "sum", "weighted_sum"):
            raise ValueError("reduction must be mean, sum or weighted_sum")
        if reduction == "weighted_sum":
            if weights is None or len(weights) != initial_state.batch or not np.all(np.isfinite(weights)):
                raise ValueError("weighted_sum needs one finite weight per sample")
        elif weights is not None:
            raise ValueError("weights are only accepted with weighted_sum")
        self.reduction = reduction
        self.weights = None if weights is None else np.asarray(weights, dtype=np.float64)

    def sample_weights(self):
        B = self.initial_state.batch
        if self.reduction == "mean":
            return np.full(B, 1.0 / B)
        if self.reduction == "sum":
            return np.ones(B)
        return self.weights.copy()

    def evaluate_batch(self, values):
        return self._sample_values(values)

    def evaluate(self, values) -> float:
        return float(np.dot(self.sample_weights(), self.evaluate_batch(values)))


def evaluate(objective, values):
    return objective.evaluate(values)


def evaluate_batch(objective, values):
    return objective.evaluate_batch(values)


def supports_gradient(method, objective) -> bool:
    from .sampled import SAMPLED_METHODS, supports_sampled
    if isinstance(method, SAMPLED_METHODS):
        return supports_sampled(method, objective)
    if not isinstance(method, AdjointGradient) or not isinstance(objective, ExpectationObjective):
        return False
    try:
        compiled = objective.template.compiled(objective.initial_state.n)
    except Exception:
        return False
    return compiled.gradient_ok and objective.observable.is_hermitian()


def value_and_gradient(method, objective, values, rng=None):
    """(value, gradient) with one gradient entry per independent parameter. Adjoint gradients
    run as one device reverse sweep; ParameterShift / FiniteDifference / SPSAGradient evaluate
    their shifted parameter vectors as one batch on the device."""
    from .sampled import SAMPLED_METHODS, estimate_gradient
    if isinstance(method, SAMPLED_METHODS):
        est = estimate_gradient(method, objective, values, rng=rng)
        return est.value, est.gradient
    if not supports_gradient(method, objective):
        raise UnsupportedGradient(f"{method!r} does not support this objective")
    slots = objective._slots(values)
    state = objective.initial_state
    compiled = objective.template.compiled(state.n)
    theta = np.ascontiguousarray(compiled.theta_from(slots))
    grad = np.zeros(max(1, compiled.nslots))
    value = np.zeros(1)
    weights = None
    wp = None
    if isinstance(objective, BatchExpectationObjective):
        weights = np.ascontiguousarray(objective.sample_weights())
        wp = N.dptr(weights)
    rc = N.lib().mb_adjoint(compiled.handle, objective.observable.handle().handle, state.handle, N.dptr(theta),
                            theta.size, wp, method.checkpoint_every, N.dptr(value), N.dptr(grad))
    N.check(rc, "value_and_gradient")
    slot_grad = np.zeros(compiled.nparams)
    for i, s in enumerate(compiled.slot_map):
        if s >= 0:
            slot_grad[i] = grad[s]
    return float(value[0]), accumulate_parameter_gradients(objective.parameter_map, slot_grad)


def value_and_pullback(method, objective, values):
    """(value, back) with back(seed) = seed * gradient; the sweep runs once, on first use."""
    if not supports_gradient(method, objective):
        raise UnsupportedGradient(f"{method!r} does not support this objective")
    saved = np.array(values, dtype=np.float64, copy=True)
    value, grad = value_and_gradient(method, objective, saved)

    def back(seed):
        seed = float(seed)
        if seed == 0:
            return np.zeros_like(grad)
        return seed * grad

    return value, back


def differentiable_value(method, objective, values):
    return objective.evaluate(values)
