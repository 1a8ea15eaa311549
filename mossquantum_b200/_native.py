"""ctypes binding of ``libmossb200.so`` (the C ABI declared in include/mossb200.h).

The shared library is built in-tree (``mossquantum_b200/libmossb200.so``). There is no
CPU fallback: if the library or a CUDA device is missing, every numerical call raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmossb200.so")

# status codes (include/mossb200.h)
MB_OK = 0
MB_EINVAL = -1
MB_EUNSUPPORTED = -2
MB_ENOMEM_BUDGET = -3
MB_ETIMEOUT = -4
MB_EDEVICE = -5
MB_ENOTINIT = -6
MB_ENORM = -7
MB_ENOTREADY = -8

MB_PURE, MB_DENSITY, MB_BATCH_PURE, MB_BATCH_DENSITY = 0, 1, 2, 3
MB_OP_GATE, MB_OP_CHANNEL = 0, 1
FAMILIES = {"MATRIX": 0, "RX": 1, "RY": 2, "RZ": 3, "PHASE": 4, "CRX": 5, "CRY": 6, "CRZ": 7,
            "CPHASE": 8, "CCPHASE": 9, "SELECT": 10}
MB_OPF_ADJOINT = 1
MB_APPLY_FUSED, MB_APPLY_PLAIN, MB_APPLY_PER_SAMPLE, MB_APPLY_DEVICE_THETA, MB_APPLY_TENSOR = 0, 1, 2, 4, 8
MB_UNEVEN_ZERO = 1


class BackendError(RuntimeError):
    """A device-side failure reported by libmossb200."""


class UnsupportedOperation(Exception):
    """Mirror of MOSSQuantum.UnsupportedOperation (src/api/backend_protocols.jl:15-36)."""


class BudgetExceeded(MemoryError):
    """The HBM byte budget would be exceeded."""


class MbOp(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("nq", ctypes.c_int32), ("pos", ctypes.c_int32 * 5),
                ("family", ctypes.c_int32), ("slot", ctypes.c_int32), ("flags", ctypes.c_int32),
                ("nkraus", ctypes.c_int32), ("reserved", ctypes.c_int32), ("value", ctypes.c_double),
                ("data", ctypes.c_void_p)]


class MbTerm(ctypes.Structure):
    _fields_ = [("nsites", ctypes.c_int32), ("sites", ctypes.c_int32 * 5), ("coeff", ctypes.c_double * 2),
                ("ops", ctypes.c_void_p)]


class MbServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_size_t), ("max_active", ctypes.c_int), ("reserved", ctypes.c_int * 7)]


class MbRequest(ctypes.Structure):
    _fields_ = [("block", ctypes.c_void_p), ("observable", ctypes.c_void_p), ("kind", ctypes.c_int),
                ("repeats", ctypes.c_int), ("theta", ctypes.c_void_p), ("ntheta", ctypes.c_size_t),
                ("gradient", ctypes.c_int), ("reserved", ctypes.c_int * 5)]


class MbResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("iterations", ctypes.c_int), ("value", ctypes.c_double * 2),
                ("latency_ms", ctypes.c_double), ("queue_ms", ctypes.c_double), ("error", ctypes.c_char * 128)]


class MbServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64),
                ("iterations", ctypes.c_uint64), ("active", ctypes.c_int), ("pending", ctypes.c_int),
                ("bytes_in_use", ctypes.c_size_t), ("peak_bytes", ctypes.c_size_t), ("budget_bytes", ctypes.c_size_t),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("evals_per_s", ctypes.c_double),
                ("jit_compile_ms", ctypes.c_double), ("jit_compiles", ctypes.c_uint64)]


class MbKernelStat(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 48), ("launches", ctypes.c_uint64), ("total_ms", ctypes.c_double),
                ("bytes", ctypes.c_double), ("flops", ctypes.c_double)]


_lib = None
_lock = threading.Lock()
_initialised = False


def load():
    """Load the shared library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise BackendError(f"libmossb200.so is missing ({LIB_PATH}); run __graft_entry__.build() first")
    L = ctypes.CDLL(LIB_PATH)
    vp, dp, ip, sz = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), ctypes.c_size_t
    sig = {
        "mb_init": ([ctypes.c_int, sz], ctypes.c_int),
        "mb_shutdown": ([], ctypes.c_int),
        "mb_last_error": ([], ctypes.c_char_p),
        "mb_memory_info": ([ctypes.POINTER(sz), ctypes.POINTER(sz)], ctypes.c_int),
        "mb_synchronize": ([], ctypes.c_int),
        "mb_version": ([], ctypes.c_int),
        "mb_launch_count": ([ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
        "mb_get_stream": ([ctypes.POINTER(vp)], ctypes.c_int),
        "mb_profile": ([ctypes.c_int], ctypes.c_int),
        "mb_profile_report": ([ctypes.POINTER(MbKernelStat), ctypes.c_int, ip], ctypes.c_int),
        "mb_state_create": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)], ctypes.c_int),
        "mb_state_free": ([vp], ctypes.c_int),
        "mb_state_set_zero": ([vp], ctypes.c_int),
        "mb_state_upload": ([vp, dp, sz], ctypes.c_int),
        "mb_state_download": ([vp, dp, sz], ctypes.c_int),
        "mb_state_copy": ([vp, vp], ctypes.c_int),
        "mb_state_info": ([vp, ip, ip, ip], ctypes.c_int),
        "mb_state_to_density": ([vp, vp], ctypes.c_int),
        "mb_state_device_ptr": ([vp, ctypes.POINTER(vp)], ctypes.c_int),
        "mb_circuit_create": ([ctypes.POINTER(MbOp), sz, ctypes.c_int, ctypes.POINTER(vp)], ctypes.c_int),
        "mb_circuit_free": ([vp], ctypes.c_int),
        "mb_circuit_nslots": ([vp, ip], ctypes.c_int),
        "mb_circuit_passes": ([vp, ip], ctypes.c_int),
        "mb_schedule_info": ([ctypes.POINTER(MbOp), sz, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                              ctypes.c_int, ip, ip, ip, ip, ip], ctypes.c_int),
        "mb_lowering_check": ([ctypes.POINTER(MbOp), sz, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                               ctypes.c_uint64, dp, dp, dp], ctypes.c_int),
        "mb_apply": ([vp, vp, dp, sz, ctypes.c_int], ctypes.c_int),
        "mb_observable_create": ([ctypes.POINTER(MbTerm), sz, ctypes.POINTER(vp)], ctypes.c_int),
        "mb_observable_free": ([vp], ctypes.c_int),
        "mb_expect": ([vp, vp, dp], ctypes.c_int),
        "mb_observable_apply": ([vp, vp, vp], ctypes.c_int),
        "mb_probabilities": ([vp, ip, ctypes.c_int, dp], ctypes.c_int),
        "mb_adjoint": ([vp, vp, vp, dp, sz, dp, ctypes.c_int, dp, dp], ctypes.c_int),
        "mb_theta_upload": ([vp, dp, sz, ctypes.c_int], ctypes.c_int),
        "mb_buffer_alloc": ([sz, ctypes.POINTER(vp)], ctypes.c_int),
        "mb_buffer_free": ([vp], ctypes.c_int),
        "mb_buffer_download": ([vp, vp, sz], ctypes.c_int),
        "mb_expect_to_device": ([vp, vp, vp], ctypes.c_int),
        "mb_graph_begin": ([], ctypes.c_int),
        "mb_graph_end": ([ctypes.POINTER(vp)], ctypes.c_int),
        "mb_graph_launch": ([vp], ctypes.c_int),
        "mb_graph_free": ([vp], ctypes.c_int),
        "mb_uneven_create": ([ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(vp)], ctypes.c_int),
        "mb_uneven_apply": ([vp, ctypes.c_int], ctypes.c_int),
        "mb_uneven_info": ([vp, ip, ip, ip], ctypes.c_int),
        "mb_uneven_free": ([vp], ctypes.c_int),
        "mb_tuning_set": ([ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "mb_tuning_get": ([ctypes.c_int, ip, ip], ctypes.c_int),
        "mb_tuning_set_fusion": ([ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "mb_tuning_get_fusion": ([ctypes.c_int, ip], ctypes.c_int),
        "mb_tuning_set_specialised": ([ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "mb_autotune": ([vp, vp, dp, sz, ctypes.c_int, ip, ip, dp], ctypes.c_int),
        "mb_measure_fp64_peak": ([dp], ctypes.c_int),
        "mb_qubit_weights": ([vp, ctypes.c_int, dp], ctypes.c_int),
        "mb_partial_trace": ([vp, ip, ctypes.c_int, vp], ctypes.c_int),
        "mb_inner": ([vp, vp, dp], ctypes.c_int),
        "mb_sandwich": ([vp, vp, dp], ctypes.c_int),
        "mb_state_extract": ([vp, ctypes.c_int, vp], ctypes.c_int),
        "mb_state_broadcast": ([vp, vp], ctypes.c_int),
        "mb_state_tile": ([vp, ctypes.c_int, vp], ctypes.c_int),
        "mb_collapse": ([vp, ctypes.c_int, ip, dp, ctypes.c_int], ctypes.c_int),
        "mb_remove_qubit": ([vp, ctypes.c_int, ip, dp, vp], ctypes.c_int),
        "mb_scale_samples": ([vp, dp], ctypes.c_int),
        "mb_server_start": ([ctypes.POINTER(MbServerConfig), ctypes.POINTER(vp)], ctypes.c_int),
        "mb_submit": ([vp, ctypes.POINTER(MbRequest), ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
        "mb_poll": ([vp, ctypes.c_uint64, ctypes.POINTER(MbResult), dp, sz], ctypes.c_int),
        "mb_wait": ([vp, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(MbResult), dp, sz], ctypes.c_int),
        "mb_server_stats_get": ([vp, ctypes.POINTER(MbServerStats)], ctypes.c_int),
        "mb_server_stats_reset": ([vp], ctypes.c_int),
        "mb_server_stop": ([vp], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def last_error() -> str:
    return load().mb_last_error().decode(errors="replace")


def check(rc: int, what: str = "") -> None:
    if rc == MB_OK:
        return
    msg = last_error()
    text = f"{what}: {msg}" if what else msg
    if rc == MB_EINVAL:
        raise ValueError(text)
    if rc == MB_EUNSUPPORTED:
        raise UnsupportedOperation(text)
    if rc == MB_ENOMEM_BUDGET:
        raise BudgetExceeded(text)
    if rc == MB_ENORM:
        raise ValueError(text)
    raise BackendError(f"{text} (code {rc})")


def lib():
    """The library, initialised on device 0 on first use (override with init())."""
    if not _initialised:
        init()
    return _lib


def init(device: int = 0, budget_bytes: int = 0) -> None:
    """mb_init: bind the backend to one GPU with an HBM byte budget (0 = 90% of free)."""
    global _initialised
    with _lock:
        L = load()
        check(L.mb_init(int(device), int(budget_bytes)), "mb_init")
        _initialised = True


def memory_info():
    used, budget = ctypes.c_size_t(), ctypes.c_size_t()
    check(lib().mb_memory_info(ctypes.byref(used), ctypes.byref(budget)))
    return used.value, budget.value


def launch_count() -> int:
    v = ctypes.c_uint64()
    check(load().mb_launch_count(ctypes.byref(v)))
    return v.value


def stream_handle() -> int:
    """cudaStream_t of the library (for CUDA-event timing on the launching stream)."""
    p = ctypes.c_void_p()
    check(lib().mb_get_stream(ctypes.byref(p)))
    return p.value or 0


def profile(enable: bool) -> None:
    check(lib().mb_profile(1 if enable else 0))


def profile_report():
    """{kernel name: (launches, total_ms, algorithmic bytes, algorithmic FP64 flops)} since profile(True)."""
    cap = 64
    arr = (MbKernelStat * cap)()
    cnt = ctypes.c_int()
    check(lib().mb_profile_report(arr, cap, ctypes.byref(cnt)))
    return {arr[i].name.decode(): (arr[i].launches, arr[i].total_ms, arr[i].bytes, arr[i].flops)
            for i in range(min(cnt.value, cap))}


def measure_fp64_peak() -> float:
    """FP64 TFLOP/s of a DFMA-only kernel on every SM (the FP64-pipe roofline denominator)."""
    v = ctypes.c_double()
    check(lib().mb_measure_fp64_peak(ctypes.byref(v)), "mb_measure_fp64_peak")
    return v.value


def synchronize() -> None:
    check(lib().mb_synchronize())


def dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
