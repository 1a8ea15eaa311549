"""The B200 backend: MOSSQuantum's selectable-backend operations on device states.

Mirrors the backend protocol of src/api/backend_protocols.jl:10-379 (``backend``,
``supports``, ``apply!``, ``expectation``, ``apply``, ``probabilities``) plus
``sample``/``counts`` (src/execution/probabilities.jl:107-181) and ``simulate``
(src/execution/simulation.jl:174-231). ``apply_`` is the Python spelling of ``apply!``:
it mutates the state in place and returns the resulting state, which is a new density
matrix when a channel meets a pure state (retain the return value, as in the reference).
"""
from __future__ import annotations

import numpy as np

from . import _native as N
from .channels import QuantumMap
from .circuit import QCircuit, _matrix_lowering
from .gates import Gate
from .operators import QubitsOperator, QubitsTerm, as_operator
from .states import (BatchDensityMatrix, BatchStateVector, DensityMatrix, StateVector, _DeviceState, density_of)

UnsupportedOperation = N.UnsupportedOperation


class B200Backend:
    """AbstractBackend for states stored on one B200."""

    name = "B200Backend"

    def __repr__(self):
        return "B200Backend()"


_BACKEND = B200Backend()


def backend(state):
    if isinstance(state, _DeviceState):
        return _BACKEND
    raise TypeError(f"{type(state).__name__} is not a B200 state")


def supports(b, operation, state, action="apply") -> bool:
    """Capability query (backend_protocols.jl:91-201)."""
    if not isinstance(b, B200Backend) or not isinstance(state, _DeviceState):
        return False
    if action == "apply":
        if isinstance(operation, Gate):
            return len(operation.positions) <= 5
        if isinstance(operation, QuantumMap):
            return 1 <= len(operation.positions) <= 2
        if isinstance(operation, QCircuit):
            return all(supports(b, it, state, action) for it in operation.flat())
        return False
    if action == "expectation":
        if isinstance(operation, (QubitsTerm, QubitsOperator)):
            return all(len(t.positions) <= 5 for t in as_operator(operation).terms)
        return False
    if action == "probabilities":
        return True
    return False


def _validate_positions(operation, n):
    for it in (operation.flat() if isinstance(operation, QCircuit) else [operation]):
        if any(p < 1 or p > n for p in it.positions):
            raise ValueError(f"position out of range for {n} qubits in {it!r}")


def _matrix_ops_fit(recs, n):
    """Every record of a matrix lowering acts on at most five qubits, all inside n."""
    if len(recs) == 0:
        return True
    nq = recs["nq"]
    if int(nq.max()) > 5:
        return False
    pos = recs["pos"]
    used = np.arange(5)[None, :] < nq[:, None]
    return bool(np.all(np.where(used, pos, 0) < n))


def _as_circuit(operation):
    if isinstance(operation, QCircuit):
        return operation
    cached = getattr(operation, "_as_circuit", None)
    if cached is None or cached.items[0] is not operation:
        cached = QCircuit([operation])
        try:
            operation._as_circuit = cached
        except AttributeError:
            pass
    return cached


def apply_(operation, state, theta=None, plain=False, tensor=False):
    """apply!(operation, state): execute a gate, channel or circuit on the device.

    theta: optional active-parameter values overriding the circuit's own (shape (P,), or
    (B, P) per-sample values on a batch state). plain=True runs one plain kernel launch per
    gate (the per-call baseline) instead of the fused schedule; tensor=True (with plain) runs
    dense 4-5 qubit gates and 2-qubit channels on the FP64 tensor cores.
    """
    if not isinstance(state, _DeviceState):
        raise TypeError("apply_ needs a B200 state")
    circuit = _as_circuit(operation) if isinstance(operation, (Gate, QCircuit)) else None
    lowered = _matrix_lowering(circuit.flat()) if circuit is not None else None
    if lowered is not None and _matrix_ops_fit(lowered[1], state.n):
        # matrix and fixed gates of at most five qubits inside the register: supported, no
        # channels, no parameters; the lowering doubles as the compile-cache signature
        compiled = circuit.compiled(state.n, lowered=lowered)
        values = np.zeros(0) if theta is None else theta
    else:
        if not supports(_BACKEND, operation, state, "apply"):
            raise UnsupportedOperation(f"B200Backend cannot apply {type(operation).__name__}")
        _validate_positions(operation, state.n)
        circuit = _as_circuit(operation)
        if circuit.has_channel() and not state.is_density:
            state = density_of(state)
        compiled = circuit.compiled(state.n)
        values = circuit.active_parameters() if theta is None else theta
    values = np.asarray(values, dtype=np.float64)
    flags = N.MB_APPLY_PLAIN if plain else N.MB_APPLY_FUSED
    if plain and tensor:
        flags |= N.MB_APPLY_TENSOR
    if values.ndim == 2:
        if not state.is_batch or values.shape[0] != state.batch:
            raise ValueError("per-sample parameters need one row per batch sample")
        flags |= N.MB_APPLY_PER_SAMPLE
    th = np.ascontiguousarray(compiled.theta_from(values), dtype=np.float64)
    N.check(N.lib().mb_apply(compiled.handle, state.handle, N.dptr(th), th.size, flags), "apply!")
    return state


def apply(operation, state, **kw):
    """circuit * state: applies to a copy (backend_protocols.jl:356-362)."""
    return apply_(operation, state.copy(), **kw)


def expectation(observable, state):
    """<H> (complex) for single states, a vector of samples for batches."""
    if not supports(_BACKEND, observable, state, "expectation"):
        raise UnsupportedOperation(f"B200Backend cannot take the expectation of {type(observable).__name__}")
    op = as_operator(observable)
    if op.nqubits() > state.n:
        raise ValueError("observable acts outside the register")
    out = np.zeros(2 * max(state.batch, 1))
    if state.batch == 0:
        return np.zeros(0, dtype=complex)
    N.check(N.lib().mb_expect(op.handle().handle, state.handle, N.dptr(out)), "expectation")
    vals = out[0::2] + 1j * out[1::2]
    return vals if state.is_batch else complex(vals[0])


def apply_observable(observable, state):
    """MOSSQuantum.apply(b, observable, state): the non-mutating H*psi / H*rho."""
    op = as_operator(observable)
    out = type(state).__new__(type(state))
    _DeviceState.__init__(out, state.n, state.batch)
    N.check(N.lib().mb_observable_apply(op.handle().handle, state.handle, out.handle), "apply(observable)")
    return out


def probabilities(state, qubits=None):
    """Marginal computational-basis probabilities; the first qubit is the low bit."""
    qubits = list(range(1, state.n + 1)) if qubits is None else [int(q) for q in qubits]
    if len(set(qubits)) != len(qubits):
        raise ValueError("readout qubits must be distinct")
    if any(q < 1 or q > state.n for q in qubits):
        raise ValueError("readout qubit out of range")
    M = 1 << len(qubits)
    out = np.zeros(M * max(state.batch, 1))
    q0 = (N.ctypes.c_int * max(1, len(qubits)))(*[q - 1 for q in qubits])
    if state.batch:
        N.check(N.lib().mb_probabilities(state.handle, q0, len(qubits), N.dptr(out)), "probabilities")
    if state.is_batch:
        return out[: M * state.batch].reshape((M, state.batch), order="F")
    return out


def _draw_samples(rng, distribution, shots, nbits):
    """Inverse-CDF sampling on the host RNG (probabilities.jl:107-121)."""
    distribution = np.asarray(distribution, dtype=float)
    if not np.all(np.isfinite(distribution)) or np.any(distribution < 0):
        raise ValueError("invalid sampling distribution")
    cum = np.cumsum(distribution)
    total = cum[-1]
    if not (np.isfinite(total) and total > 0):
        raise ValueError("sampling probabilities must have positive finite sum")
    last_positive = int(np.nonzero(distribution > 0)[0][-1])
    out = np.zeros((shots, nbits), dtype=np.int64)
    draws = rng.random(shots) * total
    sel = np.searchsorted(cum, draws, side="right")
    basis = np.where(sel >= len(distribution), last_positive, sel)
    for b in range(nbits):
        out[:, b] = (basis >> b) & 1
    return out


def sample(rng, state, shots, qubits=None):
    """Terminal readout samples (shots x nqubits[, batch]) without collapsing the state."""
    if shots < 0:
        raise ValueError("shots must be nonnegative")
    qubits = list(range(1, state.n + 1)) if qubits is None else list(qubits)
    probs = probabilities(state, qubits)
    if state.is_batch:
        out = np.zeros((shots, len(qubits), state.batch), dtype=np.int64)
        for b in range(state.batch):
            out[:, :, b] = _draw_samples(rng, probs[:, b], shots, len(qubits))
        return out
    return _draw_samples(rng, probs, shots, len(qubits))


def _histogram(draws):
    h = {}
    for row in draws:
        key = "".join(str(int(x)) for x in row)
        h[key] = h.get(key, 0) + 1
    return h


def counts(rng, state, shots, qubits=None):
    """Histogram of samples; the leftmost character is the first requested qubit."""
    draws = sample(rng, state, shots, qubits)
    if draws.ndim == 2:
        return _histogram(draws)
    return [_histogram(draws[:, :, b]) for b in range(draws.shape[2])]


class SimulationResult:
    """Final state and the measurement records in execution order (one list per sample for
    batches), as SimulationResult / BatchSimulationResult (simulation.jl:21-40)."""

    def __init__(self, state, records):
        self.state = state
        self.records = records
        self.measurements = records


def simulate(circuit, state, rng=None):
    """simulate(circuit, state; rng): executes a copy of the state (simulation.jl:174-231).
    Runs of gates and channels execute as fused device passes; QMeasure / QSelect run on the
    device with outcomes drawn from rng in instruction order, then sample order."""
    from .measurement import QMeasure, QSelect, run_instruction
    rng = np.random.default_rng() if rng is None else rng
    out = state.copy()
    records = [[] for _ in range(out.batch)] if out.is_batch else []
    run = []

    def flush(st):
        if run:
            st = apply_(QCircuit(list(run)), st)
            run.clear()
        return st

    for it in _as_circuit(circuit).flat():
        if isinstance(it, (QMeasure, QSelect)):
            out = flush(out)
            out = run_instruction(it, out, rng, records)
        else:
            run.append(it)
    out = flush(out)
    return SimulationResult(out, records)
