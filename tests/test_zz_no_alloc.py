"""The allocation-free expectation entry point, called through the C ABI.

mb_expect_local_noalloc exists for callers that cannot allocate device memory (a fixed HBM
pool, a latency-critical loop where cudaMalloc would synchronise the GPU, a plug-in that may
only use memory handed to it): it takes the caller's device state and keeps its reduction
scratch in a static array inside the library. This test compares it with mb_expect (which
uses the library's own workspace) on two calls in a row, at the expectation tolerance used
throughout the suite (1e-11). It sorts last so that a stop-at-first-failure run has already
run every other test.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-11


def _entry():
    from mossquantum_b200 import _native as N
    L = N.lib()
    f = L.mb_expect_local_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
    f.restype = ctypes.c_int
    return N, f


def _term_matrix(ops, coeff):
    m = np.ones((1, 1), dtype=complex)
    for o in ops:                    # first site = least significant local bit
        m = np.kron(o, m)
    return coeff * m


def test_noalloc_matches_expect_twice(mq):
    N, f = _entry()
    rng = np.random.default_rng(2026)
    # (qubits, samples, zero-based sites): k = 1, 2 and 3; several samples at k = 3; and 20
    # qubits with k = 3, where 2^17 blocks exceed the 160 reduction blocks per sample so each
    # block strides over the state
    cases = [(14, 1, [3, 9, 1]), (11, 4, [7, 2]), (12, 3, [5]), (10, 5, [1, 4, 8]), (20, 2, [2, 17, 9])]
    for n, B, sites in cases:
        cols = rng.normal(size=(1 << n, B)) + 1j * rng.normal(size=(1 << n, B))
        cols /= np.linalg.norm(cols, axis=0)
        state = mq.BatchStateVector(cols)
        ops1 = [rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2)) for _ in sites]
        ops2 = [rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2)) for _ in sites]
        c1, c2 = 0.7 - 0.1j, -0.4 + 0.3j
        H = mq.QubitsOperator([mq.QubitsTerm(sites, ops1, c1), mq.QubitsTerm(sites, ops2, c2)])
        expected = mq.expectation(H, state)
        # the same operator as one dense matrix in the given site order
        M = _term_matrix(ops1, c1) + _term_matrix(ops2, c2)
        mcol = np.asfortranarray(M).ravel(order="F").view(np.float64).copy()
        pos = (ctypes.c_int * len(sites))(*[s - 1 for s in sites])
        out = np.zeros(2 * B)
        rc = f(state.device_ptr(), n, B, len(sites), pos, mcol.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
               out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), None)
        assert rc == 0, N.last_error()
        got = out[0::2] + 1j * out[1::2]
        assert np.max(np.abs(got - expected)) <= TOL


def test_noalloc_rejects_oversize(mq):
    N, f = _entry()
    state = mq.BatchStateVector(4, 33)
    pos = (ctypes.c_int * 1)(0)
    m = np.eye(2, dtype=complex).ravel(order="F").view(np.float64).copy()
    out = np.zeros(66)
    rc = f(state.device_ptr(), 4, 33, 1, pos, m.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
           out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), None)
    assert rc == N.MB_EINVAL and "at most 32" in N.last_error()


_FRESH = r"""
import ctypes, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
from mossquantum_b200 import _native as N
L = N.load()                       # the library only: no mb_init in this process
f = L.mb_expect_local_noalloc
f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
              ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
f.restype = ctypes.c_int
rng = np.random.default_rng(8)
n, B, sites = 8, 3, [6, 1, 3]       # zero-based; the first site is the least significant local bit
psi = rng.normal(size=(B, 1 << n)) + 1j * rng.normal(size=(B, 1 << n))
psi /= np.linalg.norm(psi, axis=1, keepdims=True)
M = rng.normal(size=(8, 8)) + 1j * rng.normal(size=(8, 8))
# host reference <psi|M|psi> with M embedded on the sites
idx = np.arange(1 << n)
a = sum(((idx >> s) & 1) << j for j, s in enumerate(sites))
rest = idx & ~sum(1 << s for s in sites)
full = M[a[:, None], a[None, :]] * (rest[:, None] == rest[None, :])
want = np.einsum("bi,ij,bj->b", psi.conj(), full, psi)
dev = torch.from_numpy(psi.reshape(-1).view(np.float64).copy()).to("cuda:0")
torch.cuda.synchronize()
pos = (ctypes.c_int * 3)(*sites)
m = M.ravel(order="F").view(np.float64).copy()
for _ in range(2):
    out = np.zeros(2 * B)
    rc = f(dev.data_ptr(), n, B, 3, pos, m.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
           out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), None)
    assert rc == 0, N.last_error()
    got = out[0::2] + 1j * out[1::2]
    err = float(np.max(np.abs(got - want)))
    assert err <= 1e-11, err
print("fresh ok", err)
"""


def test_noalloc_in_a_fresh_process_without_init():
    """The entry point needs no mb_init: a process that only loads the library and owns its
    device memory (here through torch) gets <psi|M|psi> matching a host computation."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _FRESH, root], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "fresh ok" in r.stdout
