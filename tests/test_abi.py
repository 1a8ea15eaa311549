"""The C-ABI library loads and exports every function include/mossb200.h declares."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "mossb200.h")).read()
    return sorted(set(re.findall(r"^MB_API\s+[\w\s\*]+?\b(mb_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_api():
    names = declared_functions()
    assert {"mb_init", "mb_apply", "mb_expect", "mb_probabilities", "mb_adjoint"} <= set(names)


def test_library_exports_every_declared_symbol():
    from mossquantum_b200 import _native
    lib = ctypes.CDLL(_native.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_calls_before_init_fail_cleanly():
    from mossquantum_b200 import _native as N
    L = N.load()
    if N._initialised:
        pytest.skip("library already initialised in this process")
    h = ctypes.c_void_p()
    assert L.mb_state_create(0, 3, 1, ctypes.byref(h)) == N.MB_ENOTINIT
    assert b"mb_init" in L.mb_last_error()


def test_init_without_gpu_reports_device_error():
    from mossquantum_b200 import _native as N
    if os.path.exists("/dev/nvidia0") or os.environ.get("CUDA_VISIBLE_DEVICES"):
        pytest.skip("a GPU may be present")
    rc = N.load().mb_init(0, 0)
    assert rc == N.MB_EDEVICE
    with pytest.raises(N.BackendError):
        N.check(rc)


def test_no_undefined_internal_symbols():
    """A library function declared in one file and (by mistake) defined with internal linkage in
    another links into the shared library as an undefined symbol and fails only when loaded:
    none of the library's own symbols may be undefined."""
    import shutil
    import subprocess
    if not shutil.which("nm"):
        pytest.skip("nm not available")
    path = os.path.join(ROOT, "mossquantum_b200", "libmossb200.so")
    out = subprocess.run(["nm", "-D", "-C", "--undefined-only", path], capture_output=True, text=True).stdout
    bad = [ln for ln in out.splitlines() if "mb::" in ln or " mb_" in ln]
    assert not bad, bad
