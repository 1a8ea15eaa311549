"""Autotuner for the fused passes: tile bits t (shared-memory tile of 2^t amplitudes), register
bits R (2^R amplitudes per thread, the width of one fused register stage) and the fusion width
(1: every run of operations on one qubit is multiplied into one matrix at bind time; 0: every
gate is its own micro-op).

``autotune`` times every candidate on the caller's circuit and state (``mb_autotune``) and
records the fastest for that register size; ``save``/``load`` persist the table as JSON so a
serving process starts tuned (MB_TUNING_FILE or ~/.cache/mossquantum_b200/tuning.json).
"""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np

from . import _native as N


def default_path():
    return os.environ.get("MB_TUNING_FILE",
                          os.path.join(os.path.expanduser("~"), ".cache", "mossquantum_b200", "tuning.json"))


def autotune(circuit, state, theta=None):
    """Returns (tile_bits, register_bits, ms per apply) chosen for the state's register size."""
    compiled = circuit.compiled(state.n)
    values = circuit.active_parameters() if theta is None else theta
    th = np.ascontiguousarray(compiled.theta_from(np.asarray(values, dtype=np.float64)))
    flags = N.MB_APPLY_PER_SAMPLE if th.ndim == 2 else 0
    t, r, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
    N.check(N.lib().mb_autotune(compiled.handle, state.handle, N.dptr(th), th.size, flags, ctypes.byref(t),
                                ctypes.byref(r), ctypes.byref(ms)), "mb_autotune")
    return t.value, r.value, ms.value


def get(nbits):
    t, r = ctypes.c_int(), ctypes.c_int()
    N.check(N.lib().mb_tuning_get(int(nbits), ctypes.byref(t), ctypes.byref(r)))
    return t.value, r.value


def get_fusion(nbits):
    f = ctypes.c_int()
    N.check(N.lib().mb_tuning_get_fusion(int(nbits), ctypes.byref(f)))
    return f.value


def set_fusion(nbits, fusion):
    N.check(N.lib().mb_tuning_set_fusion(int(nbits), int(fusion)), "mb_tuning_set_fusion")


def set(nbits, tile_bits, reg_bits):  # noqa: A001 - mirrors mb_tuning_set
    N.check(N.lib().mb_tuning_set(int(nbits), int(tile_bits), int(reg_bits)), "mb_tuning_set")


def save(table_bits, path=None):
    path = path or default_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        json.dump({str(n): list(get(n)) + [get_fusion(n)] for n in table_bits}, f, indent=1)
    return path


def load(path=None):
    path = path or default_path()
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        table = json.load(f)
    for n, v in table.items():
        set(int(n), v[0], v[1])
        if len(v) > 2:
            set_fusion(int(n), v[2])
    return {int(n): tuple(v) for n, v in table.items()}
