"""Device-resident dense states: StateVector, DensityMatrix, BatchStateVector, BatchDensityMatrix.

Mirrors src/states/*.jl. The amplitudes live in HBM behind an ``mb_state`` handle; like the
reference's DemoArray storage family (test/fixtures/MOSSQuantumDemoArrayBackend), a state
never materialises on the host implicitly: ``storage()`` raises, and the only host copy is
the explicit ``to_numpy()``.
"""
from __future__ import annotations

import weakref

import numpy as np

from . import _native as N


class HostConversionError(RuntimeError):
    """Raised on implicit host materialisation of device storage."""


class _DeviceState:
    kind = N.MB_PURE
    is_density = False
    is_batch = False

    def __init__(self, n: int, batch: int = 1, data=None, _handle=None):
        self.n = int(n)
        self.batch = int(batch) if self.is_batch else 1
        if _handle is not None:
            self.handle = _handle
        else:
            h = N.ctypes.c_void_p()
            N.check(N.lib().mb_state_create(self.kind, self.n, self.batch, N.ctypes.byref(h)), "mb_state_create")
            self.handle = h
        self._finalizer = weakref.finalize(self, _free_state, self.handle.value)
        if data is not None:
            self.upload(data)

    # shape -------------------------------------------------------------------------------
    @property
    def nqubits(self):
        return self.n

    def batch_size(self):
        return self.batch

    @property
    def elems(self):
        dim = 1 << self.n
        return dim * dim if self.is_density else dim

    @property
    def nbytes(self):
        return 16 * self.elems * self.batch

    # host transfers (explicit) --------------------------------------------------------------
    def _flat(self, data):
        a = np.asarray(data, dtype=np.complex128)
        if a.size != self.elems * self.batch:
            raise ValueError(f"expected {self.elems * self.batch} amplitudes, got {a.size}")
        return np.ascontiguousarray(a.reshape(-1, order="F") if a.ndim > 1 else a)

    def upload(self, data):
        flat = self._flat(data)
        v = flat.view(np.float64)
        N.check(N.lib().mb_state_upload(self.handle, N.dptr(v), v.size), "upload")
        return self

    def to_numpy(self) -> np.ndarray:
        """Explicit device -> host copy (hostcopy); shaped like the reference storage."""
        out = np.empty(self.elems * self.batch, dtype=np.complex128)
        v = out.view(np.float64)
        N.check(N.lib().mb_state_download(self.handle, N.dptr(v), v.size), "download")
        dim = 1 << self.n
        if self.is_density and self.is_batch:
            return out.reshape((dim, dim, self.batch), order="F")
        if self.is_density:
            return out.reshape((dim, dim), order="F")
        if self.is_batch:
            return out.reshape((dim, self.batch), order="F")
        return out

    hostcopy = to_numpy

    def storage(self):
        raise HostConversionError("device storage cannot be materialised implicitly; use to_numpy()")

    def __array__(self, *a, **k):
        raise HostConversionError("device storage cannot be materialised implicitly; use to_numpy()")

    def device_ptr(self) -> int:
        p = N.ctypes.c_void_p()
        N.check(N.lib().mb_state_device_ptr(self.handle, N.ctypes.byref(p)))
        return p.value or 0

    def set_zero(self):
        N.check(N.lib().mb_state_set_zero(self.handle))
        return self

    def copy(self):
        out = type(self).__new__(type(self))
        _DeviceState.__init__(out, self.n, self.batch)
        N.check(N.lib().mb_state_copy(out.handle, self.handle), "copy")
        return out

    def __repr__(self):
        b = f", batch={self.batch}" if self.is_batch else ""
        return f"{type(self).__name__}(n={self.n}{b})"


def _free_state(h):
    if h and N._initialised:
        N.lib().mb_state_free(N.ctypes.c_void_p(h))


def _n_from_len(length):
    n = int(round(np.log2(length))) if length > 0 else -1
    if n < 0 or (1 << n) != length:
        raise ValueError("state length must be a power of two")
    return n


class StateVector(_DeviceState):
    """StateVector(n) = |0...0>, or StateVector(amplitudes[, n])."""

    kind = N.MB_PURE

    def __init__(self, data, n=None):
        if isinstance(data, (int, np.integer)):
            super().__init__(int(data))
        else:
            a = np.asarray(data, dtype=np.complex128).ravel()
            super().__init__(_n_from_len(a.size) if n is None else n, data=a)


class DensityMatrix(_DeviceState):
    """DensityMatrix(n) = |0><0|, DensityMatrix(StateVector) = psi psi', or from a matrix."""

    kind = N.MB_DENSITY
    is_density = True

    def __init__(self, data, n=None):
        if isinstance(data, (int, np.integer)):
            super().__init__(int(data))
        elif isinstance(data, StateVector):
            super().__init__(data.n)
            N.check(N.lib().mb_state_to_density(data.handle, self.handle), "DensityMatrix(state)")
        else:
            a = np.asarray(data, dtype=np.complex128)
            if a.ndim == 1:
                dim = int(round(np.sqrt(a.size)))
                a = a.reshape((dim, dim), order="F")
            super().__init__(_n_from_len(a.shape[0]) if n is None else n, data=a)


class BatchStateVector(_DeviceState):
    """BatchStateVector(n, B) of |0...0> columns, or from a (2^n, B) array."""

    kind = N.MB_BATCH_PURE
    is_batch = True

    def __init__(self, data, batch=None):
        if isinstance(data, (int, np.integer)):
            super().__init__(int(data), int(batch))
        elif isinstance(data, StateVector):
            raise TypeError("use BatchStateVector.from_states")
        else:
            a = np.asarray(data, dtype=np.complex128)
            if a.ndim != 2:
                raise ValueError("batch storage must be (2^n, B)")
            super().__init__(_n_from_len(a.shape[0]), a.shape[1], data=a)

    @classmethod
    def from_states(cls, states):
        cols = np.stack([s.to_numpy() if isinstance(s, StateVector) else np.asarray(s) for s in states], axis=1)
        return cls(cols)


class BatchDensityMatrix(_DeviceState):
    """BatchDensityMatrix(n, B) of |0><0| slices, or from a (2^n, 2^n, B) array."""

    kind = N.MB_BATCH_DENSITY
    is_density = True
    is_batch = True

    def __init__(self, data, batch=None):
        if isinstance(data, (int, np.integer)):
            super().__init__(int(data), int(batch))
        elif isinstance(data, BatchStateVector):
            super().__init__(data.n, data.batch)
            N.check(N.lib().mb_state_to_density(data.handle, self.handle), "BatchDensityMatrix(batch)")
        else:
            a = np.asarray(data, dtype=np.complex128)
            if a.ndim != 3 or a.shape[0] != a.shape[1]:
                raise ValueError("batch density storage must be (2^n, 2^n, B)")
            super().__init__(_n_from_len(a.shape[0]), a.shape[2], data=a)


def density_of(state):
    """DensityMatrix(state) for pure single or batch states."""
    if isinstance(state, StateVector):
        return DensityMatrix(state)
    if isinstance(state, BatchStateVector):
        return BatchDensityMatrix(state)
    return state
