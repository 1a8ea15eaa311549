"""Extracts the reference's recorded benchmark circuits into a small committed fixture.

MOSSQuantum's CPU-scheduling benchmark records the exact rotation angles of its 15-, 20- and
25-qubit circuits (docs/performance/cpu-scheduling-2026-11-17/baseline-16/n*-d*.toml, field
`angles_by_layer[layer][qubit]`) together with the SHA-256 of the Julia output amplitudes.
The circuit rule is cpu_scan_circuit in benchmark-source/cpu_thread_scan.jl:4-18: on 1-based
layer l and qubit q the gate is (RX, RY, RZ)[mod1(l + q, 3)] with angle
angles_by_layer[l][q], and each layer ends with CNOT(q, q + 1) for q = 1..n-1.

Run in a checkout that has the reference next to it:
    python tests/golden/make_cpu_scan_fixtures.py /root/reference
It writes tests/golden/cpu_scan_circuits.json (angles, depth, qubits and the recorded hash).
"""
import json
import os
import sys
import tomllib

CASES = ("n15-d20", "n20-d20", "n25-d10")
SUBDIR = os.path.join("docs", "performance", "cpu-scheduling-2026-11-17", "baseline-16")


def main(ref_root):
    out = {"source": SUBDIR, "rule": "benchmark-source/cpu_thread_scan.jl:4-18", "cases": {}}
    for name in CASES:
        with open(os.path.join(ref_root, SUBDIR, name + ".toml"), "rb") as f:
            d = tomllib.load(f)
        angles = d["angles_by_layer"]
        assert len(angles) == d["depth"] and all(len(row) == d["qubits"] for row in angles)
        out["cases"][name] = {"qubits": d["qubits"], "depth": d["depth"], "angles_by_layer": angles,
                              "julia_output_sha256": d["sha256"], "julia_output_bytes": d["bytes"]}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cpu_scan_circuits.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
