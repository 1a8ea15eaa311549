"""Partial trace and fidelities of device states.

Mirrors partial_tr (src/observables/partial_trace.jl:11-97) and fidelity for pure/pure,
density/pure and batch pairs (src/states/state_vector.jl:93, density_matrix.jl:129-130,
batch_state_vector.jl:194-197, batch_density_matrix.jl:187-194). The reductions run on the
device (``mb_partial_trace``, ``mb_inner``, ``mb_sandwich``); only scalars come back to the host.
The fidelity of two mixed states needs matrix square roots (eigendecompositions), which this
backend does not provide: it raises UnsupportedOperation instead of computing on the host.
"""
from __future__ import annotations

import numpy as np

from . import _native as N
from .states import BatchDensityMatrix, BatchStateVector, DensityMatrix, _DeviceState


def _check_sites(sites, n):
    sites = [int(s) for s in sites]
    if len(set(sites)) != len(sites):
        raise ValueError("duplicate sites not allowed.")
    if any(s < 1 or s > n for s in sites):
        raise ValueError("site out of range.")
    return sites


def inner(x, y):
    """dot(x, y) per sample (conjugating x) for pure states of equal shape."""
    out = np.zeros(2 * max(x.batch, 1))
    if x.batch:
        N.check(N.lib().mb_inner(x.handle, y.handle, N.dptr(out)), "dot")
    vals = out[0::2] + 1j * out[1::2]
    return vals[: x.batch] if x.is_batch else complex(vals[0])


def trace(state):
    """tr(rho) (density) or <psi|psi> (pure), per sample for batches."""
    if state.is_density:
        from .backend import expectation
        from .operators import QubitsTerm
        return expectation(QubitsTerm([], [], 1.0), state)
    return inner(state, state)


def partial_tr(state, sites):
    """partial_tr(state, sites): the reduced density matrix of the remaining qubits (same order).
    Empty sites: the state itself for density matrices, DensityMatrix(psi) for pure states;
    all sites: the trace (or squared norm); batch pure input: a list of DensityMatrix."""
    if not isinstance(state, _DeviceState):
        raise TypeError("partial_tr needs a B200 state")
    sites = _check_sites(sites, state.n)
    if not sites:
        if state.is_density:
            return state if not state.is_batch else state.copy()
        from .states import density_of
        return density_of(state.copy())
    if len(sites) == state.n:
        t = trace(state)
        return np.real(t) if not state.is_density else t
    m = state.n - len(sites)
    out = BatchDensityMatrix(m, state.batch) if state.is_batch else DensityMatrix(m)
    arr = (N.ctypes.c_int * len(sites))(*[s - 1 for s in sites])
    if state.batch:
        N.check(N.lib().mb_partial_trace(state.handle, arr, len(sites), out.handle), "partial_tr")
    if isinstance(state, BatchStateVector):
        parts = []
        for b in range(state.batch):
            d = DensityMatrix(m)
            N.check(N.lib().mb_state_extract(out.handle, b, d.handle), "partial_tr")
            parts.append(d)
        return parts
    return out


def fidelity(x, y):
    """fidelity(x, y): |<x|y>|^2 for pure states, <y|rho|y> for a density matrix and a pure
    state (either order), per sample for batch pairs."""
    if x.is_density and y.is_density:
        raise N.UnsupportedOperation("fidelity of two density matrices needs matrix square roots "
                                     "(not provided by the B200 backend)")
    if x.n != y.n or x.batch != y.batch or x.is_batch != y.is_batch:
        raise ValueError("states must have the same number of qubits and samples.")
    if not x.is_density and not y.is_density:
        v = inner(x, y)
        return np.abs(v) ** 2
    rho, psi = (x, y) if x.is_density else (y, x)
    out = np.zeros(2 * max(rho.batch, 1))
    if rho.batch:
        N.check(N.lib().mb_sandwich(rho.handle, psi.handle, N.dptr(out)), "fidelity")
    vals = out[0::2]
    return vals[: rho.batch] if rho.is_batch else float(vals[0])
