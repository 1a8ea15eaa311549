#!/usr/bin/env python
"""Headline benchmark: plain-method circuit at scale on one B200 per rank.

Workload (one "step"): a 28-qubit ComplexF64 StateVector (4 GiB, resident in HBM) is reset
to |0...0> and runs a 20-layer random circuit; each layer is a U3 on every qubit
(theta = arccos(1-2u), phi, lambda uniform) followed by CZ on brickwork pairs. The inputs
are seeded synthetic data. The state is 32x larger than L2, so no L2 flush is needed.

metric: effective gate-kernel HBM GB/s = (bytes the plain per-gate method moves: 32*2^n per
U3 pass, 8*2^n per CZ pass) / step time; layers/s is reported beside it.
--impl reference times the reference's CPU method (the C++ restatement in oracle/) on a
bounded sample of the same workload on the host cores.
Multi-GPU (--gpus N under torchrun): independent replicas, one state per GPU, no
collective on the data path (weak scaling); time = max over ranks of device time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--variant", default="fused", choices=["fused", "plain"])
    ap.add_argument("--qubits", type=int, default=28)
    ap.add_argument("--layers", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--workload", default="scale", choices=["scale", "batch"],
                    help="scale: 28-qubit U3+CZ circuit (headline); batch: uneven batch of 512 pure + 64 density states")
    ap.add_argument("--plain-samples", type=int, default=48)
    return ap.parse_args()


def plain_bytes(n, depth):
    """Bytes of the plain per-gate method: 32*2^n per U3 pass, 8*2^n per CZ pass."""
    ncz = sum(len(range(1 if l % 2 == 0 else 2, n, 2)) for l in range(depth))
    return 32.0 * (1 << n) * n * depth + 8.0 * (1 << n) * ncz


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def build_workload(mq, W, n, depth, seed_stream):
    params = W.u3_params(n, depth, W.rng_for(1, *seed_stream))
    return W.u3_brickwork(n, depth, params)


def cpu_baseline_run(n, layers_sample, threads, W, mq_circuit=None):
    """Times the oracle (restated reference CPU method) on a bounded sample: `layers_sample`
    layers of the same circuit family at the same qubit count, on `threads` host threads."""
    from oracle import oracle as O
    O.set_threads(threads)
    circ = W.u3_brickwork(n, layers_sample, W.u3_params(n, layers_sample, W.rng_for(1, 99)))
    specs = circ.specs()
    state = O.zero_state(n)
    t0 = time.perf_counter()
    O.apply(specs, state, n)
    dt = time.perf_counter() - t0
    return plain_bytes(n, layers_sample) / dt / 1e9, dt


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from mossquantum_b200 import workloads as W
    threads = os.cpu_count() or 1
    n = args.qubits
    sample_layers = 1
    vals = []
    for i in range(args.warmup + args.steps):
        v, dt = cpu_baseline_run(n, sample_layers, threads, W)
        if i >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    sample = f"{sample_layers} of {args.layers} layers at n={n} per step ({n} U3 + CZ brickwork)"
    line = {"metric": "gate-kernel HBM GB/s (effective, plain per-gate bytes)", "value": value, "unit": "GB/s",
            "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128 (f64)",
            "data": "synthetic (seeded)",
            "config": {"workload": f"u3_cz_brickwork n={n} layers={args.layers}", "qubits": n, "layers": args.layers},
            "cpu_baseline": {"value": value, "unit": "GB/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def batch_workload(args):
    """Config 2: 512 pure states with n uniform in 10..22 running the hardware-efficient
    ansatz (depth 8) with per-sample angles, plus 64 ten-qubit density matrices with
    depolarizing (p=0.01) and amplitude damping (gamma=0.02) after every gate; output <XXZ>
    per sample. One step = one evaluation of the whole batch through a BatchPlan (one CUDA
    graph launch). The plain per-call path (each sample alone, one plain kernel per gate) is
    timed on a bounded sample of the same workload."""
    import torch
    import mossquantum_b200 as mq
    from mossquantum_b200 import _native as N
    from mossquantum_b200 import workloads as W
    from mossquantum_b200.batch import BatchPlan, run_plain
    mq.init(0)
    rng = W.rng_for(2)
    sizes = rng.integers(10, 23, size=512)
    counts = {int(n): int((sizes == n).sum()) for n in np.unique(sizes)}
    depth = 8
    groups = {n: (W.hea_circuit(n, depth), B) for n, B in counts.items()}
    dm_groups = {10: (W.hea_circuit(10, depth, noise=(0.01, 0.02)), 64)}
    t0 = time.perf_counter()
    plan = BatchPlan(groups, W.xxz)
    plan_dm = BatchPlan(dm_groups, W.xxz, kind="density")
    prep_s = time.perf_counter() - t0
    def thetas(gr, seed):
        r = np.random.default_rng(seed)
        return {n: r.uniform(0, 2 * np.pi, size=(B, c.nparameters())) for n, (c, B) in gr.items()}
    th, thd = thetas(groups, 1), thetas(dm_groups, 2)
    for _ in range(args.warmup):
        plan.run(th)
        plan_dm.run(thd)
    stream = torch.cuda.ExternalStream(N.stream_handle())
    l0 = N.launch_count()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        t1 = time.perf_counter()
        start.record(stream)
        for _ in range(args.steps):
            plan.run(th)
            plan_dm.run(thd)
        end.record(stream)
        end.synchronize()
        wall = (time.perf_counter() - t1) / args.steps
    ms_step = start.elapsed_time(end) / args.steps
    evals = 512 + 64
    # plain per-call path on a bounded sample (uniform over the same sizes), extrapolated per sample
    sub = {}
    for n in sorted(counts):
        sub[n] = (groups[n][0], min(counts[n], max(1, args.plain_samples * counts[n] // 512)))
    nsub = sum(b for _, b in sub.values())
    run_plain(sub, W.xxz, {n: th[n][:b] for n, (c, b) in sub.items()})
    N.synchronize()
    t2 = time.perf_counter()
    run_plain(sub, W.xxz, {n: th[n][:b] for n, (c, b) in sub.items()})
    N.synchronize()
    plain_per_eval = (time.perf_counter() - t2) / nsub
    # weight plain time by the full size distribution
    per_size = {}
    for n, (c, b) in sub.items():
        t3 = time.perf_counter()
        run_plain({n: (c, 1)}, W.xxz, {n: th[n][:1]})
        N.synchronize()
        per_size[n] = time.perf_counter() - t3
    t4 = time.perf_counter()
    run_plain({10: (dm_groups[10][0], 2)}, W.xxz, {10: thd[10][:2]}, kind="density")
    N.synchronize()
    dm_plain = (time.perf_counter() - t4) / 2
    plain_total = sum(per_size[n] * counts[n] for n in counts) + 64 * dm_plain
    line = {"metric": "circuit-evals/s (uneven batch, per-sample parameters)", "value": evals / (ms_step / 1e3),
            "unit": "evals/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128 (f64)",
            "data": "synthetic (seeded)",
            "config": {"workload": "512 pure (n=10..22, HEA depth 8) + 64 density (n=10, noisy) <XXZ>",
                       "sizes": counts, "plan_build_s": prep_s},
            "plain_per_call": {"value": evals / plain_total, "unit": "evals/s", "seconds_per_batch": plain_total,
                               "sample": f"{nsub} pure samples + 2 density samples timed, weighted by the size mix"},
            "speedup_vs_plain": plain_total / (ms_step / 1e3),
            "e2e": {"value": evals / wall, "unit": "evals/s", "h2d_bytes_per_step": int(8 * sum(
                c.nparameters() * B for c, B in list(groups.values()) + list(dm_groups.values()))),
                "d2h_bytes_per_step": 16 * evals},
            "gpu_launches": N.launch_count() - l0, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload == "batch":
        return batch_workload(args)
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    import mossquantum_b200 as mq
    from mossquantum_b200 import _native as N
    from mossquantum_b200 import workloads as W
    mq.init(local)
    n, depth = args.qubits, args.layers
    circuit = build_workload(mq, W, n, depth, (rank,))
    state = mq.StateVector(n)
    plain = args.variant == "plain"
    stream = torch.cuda.ExternalStream(N.stream_handle(), device=local)

    def step():
        state.set_zero()
        mq.apply_(circuit, state, plain=plain)

    for _ in range(args.warmup):
        step()
    N.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = N.launch_count()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        start.record(stream)
        for _ in range(args.steps):
            step()
        end.record(stream)
        end.synchronize()
    launches = N.launch_count() - l0
    ms = start.elapsed_time(end)
    if world > 1:
        t = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    ms_step = ms / args.steps
    bytes_step = plain_bytes(n, depth)
    value = world * bytes_step / (ms_step / 1e3) / 1e9

    # Per-kernel roofline of the dominant kernel (one profiled step, events on the library stream).
    N.profile(True)
    step()
    rep = N.profile_report()
    N.profile(False)
    dom = max(rep.items(), key=lambda kv: kv[1][1]) if rep else None
    peak, peak_kind = load_peaks()
    roofline = None
    if dom:
        name, (lc, tms, byts) = dom
        achieved = byts / (tms / 1e3) / 1e9
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tpath):
            with open(tpath) as f:
                tj = json.load(f)
            ent = tj.get(f"{name}@n{n}")
            traffic = ent.get("bytes_per_launch") if ent else None
        share = tms / sum(v[1] for v in rep.values())
        roofline = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                    "launches_per_step": lc, "algorithmic_bytes_per_launch": byts / lc, "share_of_step": share,
                    "avg_launch_ms": tms / lc}

    # End to end through the public API: host circuit in, probabilities of 10 qubits out.
    e2e = None
    if not args.no_e2e:
        circuits = [build_workload(mq, W, n, depth, (rank, 1000 + i)) for i in range(args.e2e_steps + 1)]
        h2d = sum(16 * (1 << len(g.positions)) ** 2 for g in circuits[0].flat())
        readout = list(range(1, 11))

        def e2e_step(c):
            state.set_zero()
            mq.apply_(c, state, plain=plain)
            return mq.probabilities(state, readout)

        e2e_step(circuits[0])
        t0 = time.perf_counter()
        for c in circuits[1:]:
            e2e_step(c)
        dt = (time.perf_counter() - t0) / args.e2e_steps
        e2e = {"value": world * bytes_step / dt / 1e9, "unit": "GB/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": 8 * (1 << len(readout)), "ms_per_step": dt * 1e3,
               "note": "circuit lowering + matrix upload + set_zero + apply + 10-qubit probabilities"}

    cpu = None
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        threads = os.cpu_count() or 1
        v, dt = cpu_baseline_run(n, 1, threads, W)
        cpu = {"value": v, "unit": "GB/s", "cores": threads, "kind": "port",
               "sample": f"1 of {depth} layers at n={n} ({dt:.1f} s, oracle C++ restatement)"}

    if rank == 0:
        line = {"metric": "gate-kernel HBM GB/s (effective, plain per-gate bytes)", "value": value, "unit": "GB/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128 (f64)",
                "data": "synthetic (seeded)",
                "config": {"workload": f"u3_cz_brickwork n={n} layers={depth}", "qubits": n, "layers": depth,
                           "state_bytes": 16 << n, "variant": args.variant, "parallelism": f"replicas x{world}",
                           "l2": "state (4 GiB) is larger than L2; no flush needed"},
                "layers_per_s": world * depth / (ms_step / 1e3), "roofline": roofline, "cpu_baseline": cpu,
                "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
