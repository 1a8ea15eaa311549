"""Generated specialised-kernel sources compile for sm_100a (NVRTC on the host, no GPU).

The harness (tests/jit_sources_harness.cu) links the library's source generator and builds
Pauli expectation passes for nearest-neighbour Hamiltonians (XXZ, TFIM) with the tile's
register bits low and high in the register, and a persistent uneven launch over a 14-qubit
group (with pass-0 generation of |0..0>) and an 8-qubit group whose tiles need fewer threads
than the launch has, a TMA-staged tile pass and a dual-state reverse pass with a gradient
accumulator. Every source must compile; the Pauli passes must fit their register budget
without spills, since a spilling kernel is not used.
"""
import json
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "mossquantum_b200", "csrc")
JIT_OBJ = os.path.join(CSRC, "_build", "jit.o")


@pytest.fixture(scope="module")
def harness_lines(tmp_path_factory):
    if not shutil.which("nvcc") or not os.path.exists(JIT_OBJ):
        pytest.skip("nvcc or the built generator object is missing")
    exe = str(tmp_path_factory.mktemp("jit") / "harness")
    cmd = ["nvcc", "-std=c++17", "-O1", "-I", CSRC, "-I", os.path.join(ROOT, "include"), "-o", exe,
           os.path.join(ROOT, "tests", "jit_sources_harness.cu"), JIT_OBJ, "-ldl", "-lcudart"]
    subprocess.run(cmd, check=True, capture_output=True, timeout=600)
    out = subprocess.run([exe], check=True, capture_output=True, text=True, timeout=600)
    lines = [json.loads(x) for x in out.stdout.splitlines() if x.startswith("{")]
    if any(x.get("error") == "no NVRTC" for x in lines):
        pytest.skip("NVRTC is not available on this host")
    return {x["name"]: x for x in lines}


def test_pauli_pass_sources_compile_without_spills(harness_lines):
    for name in ("pauli_xxz_n20_bits5_9", "pauli_xxz_n20_bits9_13", "pauli_tfim_n22_bits5_9",
                 "pauli_xxz_n22_bits5_9"):
        r = harness_lines[name]
        assert r["bytes"] > 0, name
        assert r["rc"] == 0, name
        assert r["spill"] == 0 and 0 < r["regs"] <= 80, r   # 3 CTAs of 256 threads per SM


def test_persistent_uneven_source_compiles(harness_lines):
    r = harness_lines["uneven_n14_n8"]
    assert r["rc"] == 0 and r["bytes"] > 0, r
    launch = harness_lines["uneven_launch"]
    # 2^10-amplitude tiles with 3 register bits: 128 threads; the tile and the largest matrix
    # copy in dynamic shared memory
    assert launch["threads"] == 128
    assert launch["shm"] >= 16 << 10


def test_tile_and_reverse_pass_sources_compile(harness_lines):
    for name in ("tile_n14", "adjoint_n14"):
        r = harness_lines[name]
        assert r["rc"] == 0 and r["bytes"] > 0 and r["spill"] == 0, r
