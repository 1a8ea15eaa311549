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
    ap.add_argument("--variant", default="fused", choices=["fused", "plain", "block", "tensor"],
                    help="fused: tiled passes (K1/K2); plain: one K0 sweep per gate; block: gates fused on the "
                         "host into dense <=5-qubit blocks, one K0 sweep each; tensor: the same blocks on the "
                         "FP64 tensor cores (K5)")
    ap.add_argument("--qubits", type=int, default=28)
    ap.add_argument("--layers", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batch (config 2) and serving (config 4) measurements of the default run")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--case", default="all", help="kernel workload: one of " + ", ".join(KERNEL_CASES) + " or all")
    ap.add_argument("--workload", default="scale", choices=["scale", "batch", "grad", "serve", "kernel"],
                    help="scale: 28-qubit U3+CZ circuit (headline); batch: uneven batch of 512 pure + 64 density "
                         "states; grad: adjoint gradients (24 qubits, 1152 angles; 64 noisy density matrices); "
                         "serve: Poisson request stream through the continuous-batching server; kernel: one small "
                         "case per kernel family, each launch timed with CUDA events (the ncu capture command)")
    ap.add_argument("--plain-samples", type=int, default=48)
    ap.add_argument("--rates", default="sat", help="serve: arrival rates (requests/s) to sweep; sat = saturating")
    ap.add_argument("--requests", type=int, default=200, help="serve: requests per rate")
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


def dominant_roofline(N, step, size_key):
    """Roofline of the kernel with the largest share of one profiled step (CUDA events on the
    library stream around every launch). Both views are reported: HBM (algorithmic bytes per
    launch / duration vs the measured copy peak) and FP64 (algorithmic flops per launch /
    duration vs the FP64 rate of a DFMA-only kernel measured here); `bound` is the view with
    the larger fraction."""
    N.profile(True)
    step()
    rep = N.profile_report()
    N.profile(False)
    if not rep:
        return None
    name, (lc, tms, byts, flops) = max(rep.items(), key=lambda kv: kv[1][1])
    peak, peak_kind = load_peaks()
    fp64_peak = N.measure_fp64_peak()
    sec = tms / 1e3
    hbm = {"achieved": byts / sec / 1e9, "peak": peak, "unit": "GB/s", "frac": byts / sec / 1e9 / peak,
           "peak_kind": peak_kind}
    fp = {"achieved": flops / sec / 1e12, "peak": fp64_peak, "unit": "TFLOP/s",
          "frac": flops / sec / 1e12 / fp64_peak if fp64_peak else None,
          "peak_kind": "measured here (DFMA-only kernel, mb_measure_fp64_peak)"}
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            ent = json.load(f).get(f"{name}@{size_key}")
        traffic = ent.get("bytes_per_launch") if ent else None
    main = fp if (fp["frac"] or 0) > hbm["frac"] else hbm
    return {"bound": "fp64" if main is fp else "hbm", "kernel": name, "achieved": main["achieved"],
            "peak": main["peak"], "unit": main["unit"], "frac": main["frac"], "peak_kind": main["peak_kind"],
            "traffic": traffic, "hbm": hbm, "fp64": fp, "launches_per_step": lc,
            "algorithmic_bytes_per_launch": byts / lc, "algorithmic_flops_per_launch": flops / lc,
            "share_of_step": tms / sum(v[1] for v in rep.values()), "avg_launch_ms": tms / lc}


def build_workload(mq, W, n, depth, seed_stream):
    params = W.u3_params(n, depth, W.rng_for(1, *seed_stream))
    return W.u3_brickwork(n, depth, params)


def timing_oracle():
    """The oracle built for this host (-O3 -march=native, FMA contraction; the checker build is
    portable and contraction-free), loaded only for the timed CPU baseline."""
    from oracle import oracle as O
    O.use_fast()
    return O


def cpu_baseline_run(n, layers_sample, threads, W, repeats=3):
    """Times the oracle (restated reference CPU method) on a bounded sample: `layers_sample`
    layers of the same circuit family at the same qubit count, on `threads` host threads.
    One untimed run, then the median of `repeats` runs. Returns (GB/s, seconds per run)."""
    O = timing_oracle()
    O.set_threads(threads)
    circ = W.u3_brickwork(n, layers_sample, W.u3_params(n, layers_sample, W.rng_for(1, 99)))
    specs = circ.specs()
    state = O.zero_state(n)
    O.apply(specs, state, n)
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        O.apply(specs, state, n)
        times.append(time.perf_counter() - t0)
    dt = statistics.median(times)
    return plain_bytes(n, layers_sample) / dt / 1e9, dt


# The reference's own median for its recorded 20-qubit depth-20 circuit (780 gates) with 16
# Julia threads (docs/performance/cpu-scheduling-2026-11-17/summary.csv:94).
REFERENCE_N20_D20_16T_S = 0.23005131


def cpu_anchor(threads):
    """The oracle on the reference's recorded 20-qubit, depth-20 benchmark circuit (exact
    angles, tests/golden/cpu_scan_circuits.json): median of 5 runs after one untimed run,
    reported beside the reference's own Julia time for the same circuit."""
    from mossquantum_b200 import workloads as W
    O = timing_oracle()
    O.set_threads(threads)
    with open(os.path.join(ROOT, "tests", "golden", "cpu_scan_circuits.json")) as f:
        case = json.load(f)["cases"]["n20-d20"]
    specs = W.cpu_scan_circuit(case["angles_by_layer"]).specs()
    state = O.zero_state(20)
    O.apply(specs, state, 20)
    times = []
    for _ in range(5):
        t0 = time.perf_counter()
        O.apply(specs, state, 20)
        times.append(time.perf_counter() - t0)
    return {"circuit": "reference n20-d20 (cpu_thread_scan.jl:4-18, recorded angles)", "threads": threads,
            "oracle_median_s": statistics.median(times), "reference_julia_16_threads_median_s": REFERENCE_N20_D20_16T_S,
            "note": "different hardware; context for the CPU baseline, not a pass/fail"}


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
        v, dt = cpu_baseline_run(n, sample_layers, threads, W, repeats=1)
        if i >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    sample = (f"{sample_layers} of {args.layers} layers at n={n} per step ({n} U3 + CZ brickwork), "
              f"host-native oracle build")
    line = {"metric": "gate-kernel HBM GB/s (effective, plain per-gate bytes)", "value": value, "unit": "GB/s",
            "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128 (f64)",
            "data": "synthetic (seeded)",
            "config": {"workload": f"u3_cz_brickwork n={n} layers={args.layers}", "qubits": n, "layers": args.layers},
            "cpu_baseline": {"value": value, "unit": "GB/s", "cores": threads, "kind": "port", "sample": sample,
                             "anchor": cpu_anchor(threads)},
            "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def batch_measure(steps=3, warmup=2, per_size=3, dm_samples=4):
    """Uneven batch: 512 pure states with n uniform in 10..22 running the hardware-efficient
    ansatz (depth 8) with per-sample angles, plus 64 ten-qubit density matrices with
    depolarizing (p=0.01) and amplitude damping (gamma=0.02) after every gate; output <XXZ>
    per sample. One step = one evaluation of the whole batch through BatchPlans (CUDA graph
    replays). The plain per-call path (each sample alone, one plain kernel per gate) is timed
    on a stratified sample: `per_size` samples of every qubit count and `dm_samples` density
    matrices, each size's mean time weighted by its count in the batch."""
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
    plan = BatchPlan(groups, W.xxz, autotune=True)
    plan_dm = BatchPlan(dm_groups, W.xxz, kind="density", autotune=True)
    prep_s = time.perf_counter() - t0
    log(f"batch: plans ready after {prep_s:.1f} s")

    def thetas(gr, seed):
        r = np.random.default_rng(seed)
        return {n: r.uniform(0, 2 * np.pi, size=(B, c.nparameters())) for n, (c, B) in gr.items()}
    th, thd = thetas(groups, 1), thetas(dm_groups, 2)
    for _ in range(warmup):
        plan.run(th)
        plan_dm.run(thd)
    stream = torch.cuda.ExternalStream(N.stream_handle())
    l0 = N.launch_count()
    start, mid, end = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    with ClockSampler(0) as clk:
        t1 = time.perf_counter()
        pure_ms = dm_ms = 0.0
        for _ in range(steps):
            start.record(stream)
            plan.run(th)
            mid.record(stream)
            plan_dm.run(thd)
            end.record(stream)
            end.synchronize()
            pure_ms += start.elapsed_time(mid)
            dm_ms += mid.elapsed_time(end)
        wall = (time.perf_counter() - t1) / steps
    ms_step = (pure_ms + dm_ms) / steps
    launches = N.launch_count() - l0
    evals = 512 + 64
    # The sizes below 18 qubits replayed alone: in the batch they run in one persistent launch
    # (a CTA per sample); beside it the same sizes with one launch per size and pass.
    small = {n: groups[n] for n in groups if n < 18}
    th_small = {n: th[n] for n in small}
    small_ms = {}
    for persistent in (True, False):
        plan_small = BatchPlan(small, W.xxz, persistent=persistent)
        plan_small.run(th_small)
        start.record(stream)
        for _ in range(steps):
            plan_small.run(th_small)
        end.record(stream)
        end.synchronize()
        small_ms[persistent] = start.elapsed_time(end) / steps
        plan_small.close()
    persistent_info = plan.persistent_info()
    choice = plan.choice
    # plain per-call path: stratified sample
    plain_s = {}
    for n in sorted(counts):
        b = min(per_size, counts[n])
        run_plain({n: (groups[n][0], 1)}, W.xxz, {n: th[n][:1]})      # warm this size
        N.synchronize()
        t2 = time.perf_counter()
        run_plain({n: (groups[n][0], b)}, W.xxz, {n: th[n][:b]})
        N.synchronize()
        plain_s[n] = (time.perf_counter() - t2) / b
    run_plain({10: (dm_groups[10][0], 1)}, W.xxz, {10: thd[10][:1]}, kind="density")
    N.synchronize()
    t4 = time.perf_counter()
    run_plain({10: (dm_groups[10][0], dm_samples)}, W.xxz, {10: thd[10][:dm_samples]}, kind="density")
    N.synchronize()
    dm_plain = (time.perf_counter() - t4) / dm_samples
    plain_total = sum(plain_s[n] * counts[n] for n in counts) + 64 * dm_plain
    log(f"batch: {ms_step:.1f} ms per step, plain per-call {plain_total * 1e3:.0f} ms per batch")
    return {"evals_per_s": evals / (ms_step / 1e3), "ms_per_step": ms_step, "pure_ms_per_step": pure_ms / steps,
            "density_ms_per_step": dm_ms / steps, "small_sizes_ms_per_step": small_ms[True],
            "small_sizes_per_size_launches_ms_per_step": small_ms[False],
            "persistent_launch": {"groups": persistent_info[0], "samples": persistent_info[2],
                                  "groups_on_per_size_path": persistent_info[1], "plan_choice": choice},
            "evals_per_step": evals, "steps": steps, "warmup": warmup,
            "sizes": counts, "plan_build_s": prep_s,
            "autotuned": {str(k): list(v) for k, v in {**plan.tuned, **plan_dm.tuned}.items()},
            "plain_per_call": {"evals_per_s": evals / plain_total, "seconds_per_batch": plain_total,
                               "sample": f"{per_size} samples per qubit count (10..22) and {dm_samples} density "
                                         f"matrices, each timed alone; weighted by the batch's size mix"},
            "speedup_vs_plain": plain_total / (ms_step / 1e3),
            "e2e": {"evals_per_s": evals / wall, "h2d_bytes_per_step": int(8 * sum(
                c.nparameters() * B for c, B in list(groups.values()) + list(dm_groups.values()))),
                "d2h_bytes_per_step": 16 * evals},
            "gpu_launches": launches, "clocks": clk.summary()}


def batch_workload(args):
    r = batch_measure(args.steps, args.warmup)
    line = {"metric": "circuit-evals/s (uneven batch, per-sample parameters)", "value": r["evals_per_s"],
            "unit": "evals/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128 (f64)",
            "data": "synthetic (seeded)",
            "config": {"workload": "512 pure (n=10..22, HEA depth 8) + 64 density (n=10, noisy) <XXZ>",
                       "sizes": r["sizes"], "plan_build_s": r["plan_build_s"], "autotuned": r["autotuned"]},
            "pure_ms_per_step": r["pure_ms_per_step"], "density_ms_per_step": r["density_ms_per_step"],
            "small_sizes_ms_per_step": r["small_sizes_ms_per_step"],
            "small_sizes_per_size_launches_ms_per_step": r["small_sizes_per_size_launches_ms_per_step"],
            "persistent_launch": r["persistent_launch"],
            "plain_per_call": r["plain_per_call"], "speedup_vs_plain": r["speedup_vs_plain"],
            "e2e": {"value": r["e2e"]["evals_per_s"], "unit": "evals/s",
                    "h2d_bytes_per_step": r["e2e"]["h2d_bytes_per_step"],
                    "d2h_bytes_per_step": r["e2e"]["d2h_bytes_per_step"]},
            "gpu_launches": r["gpu_launches"], "clocks": r["clocks"]}
    print(json.dumps(line), flush=True)
    return 0


def _random_unitary(d, rng):
    z = rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def _case_setup(name, mq, W):
    """(description, step) of one kernel case: a small workload (1 GiB states, or two 256 MiB
    states for the adjoint) dominated by one kernel family."""
    rng = np.random.default_rng(7)
    if name in ("dense1_low", "dense1_high"):
        n = 26
        q = 2 if name == "dense1_low" else 26
        c = mq.QCircuit([mq.QuantumGate(q, _random_unitary(2, rng)) for _ in range(4)])
        s = mq.StateVector(n)
        return f"K0 plain sweep: 4 dense 1-qubit gates on qubit {q}, n={n}", lambda: mq.apply_(c, s, plain=True)
    if name == "tile":
        n = 26
        c = W.u3_brickwork(n, 20, W.u3_params(n, 20, W.rng_for(1, 0)))
        s = mq.StateVector(n)
        return f"K1 tile passes: U3 + CZ brickwork, n={n}, 20 layers", lambda: (s.set_zero(), mq.apply_(c, s))
    if name == "density":
        n = 13
        c = W.hea_circuit(n, 1, W.hea_angles(n, 1, W.rng_for(9)), active=False, noise=(0.01, 0.02))
        s = mq.DensityMatrix(n)
        return f"K3 density passes: noisy HEA layer on a {n}-qubit density matrix (26 bits)", \
            lambda: (s.set_zero(), mq.apply_(c, s))
    if name == "pauli":
        n = 26
        s = mq.StateVector(n)
        mq.apply_(W.u3_brickwork(n, 1, W.u3_params(n, 1, W.rng_for(1, 3))), s)
        H = W.tfim(n)
        return f"K4 Pauli pass: TFIM expectation (51 strings), n={n}", lambda: mq.expectation(H, s)
    if name == "adjoint":
        n, depth = 24, 2
        c = W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(3)))
        obj = mq.ExpectationObjective(c, W.tfim(n), mq.StateVector(n))
        th = c.active_parameters()
        return f"K6 adjoint dual-state passes: HEA n={n} depth {depth}", \
            lambda: mq.value_and_gradient(mq.AdjointGradient(), obj, th)
    if name == "grad24":
        # the gradient workload's pure part: 24 qubits, depth 16, 1152 angles, checkpoints
        # every 4 layers (every kernel of one value_and_gradient in the report)
        n, depth = 24, 16
        c = W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(3)))
        obj = mq.ExpectationObjective(c, W.tfim(n), mq.StateVector(n))
        th = c.active_parameters()
        method = mq.AdjointGradient(checkpoint_every=4 * (3 * n + n - 1))
        return f"K6 adjoint gradient: HEA n={n} depth {depth}, 1152 angles", \
            lambda: mq.value_and_gradient(method, obj, th)
    if name == "marginal":
        n = 26
        s = mq.StateVector(n)
        mq.apply_(W.u3_brickwork(n, 1, W.u3_params(n, 1, W.rng_for(1, 4))), s)
        return f"K7 marginal: probabilities of 10 qubits, n={n}", lambda: mq.probabilities(s, list(range(1, 11)))
    if name in ("dmma", "dense5"):
        n = 26
        gates = []
        for layer in range(4):
            for a in range(1 + (layer % 2) * 2, n - 3, 5):
                gates.append(mq.QuantumGate(tuple(range(a, a + 5)), _random_unitary(32, rng)))
        c = mq.QCircuit(gates)
        s = mq.StateVector(n)
        tensor = name == "dmma"
        return (f"K5 {'FP64 tensor cores' if tensor else 'on K0 (CUDA cores)'}: {len(gates)} random dense 5-qubit "
                f"gates in brickwork, n={n}"), lambda: mq.apply_(c, s, plain=True, tensor=tensor)
    if name in ("batch_pure", "batch_pure_small"):
        # the uneven batch's pure part (512 states of 10..22 qubits, HEA depth 8, per-sample
        # angles), applied eagerly group by group; _small keeps the sizes below 18 qubits
        rng2 = W.rng_for(2)
        sizes = rng2.integers(10, 23, size=512)
        counts = {int(n): int((sizes == n).sum()) for n in np.unique(sizes)}
        if name == "batch_pure_small":
            counts = {n: B for n, B in counts.items() if n < 18}
        groups = []
        for n, B in sorted(counts.items()):
            c = W.hea_circuit(n, 8)
            th = np.random.default_rng(n).uniform(0, 2 * np.pi, size=(B, c.nparameters()))
            groups.append((c, mq.BatchStateVector(n, B), th))

        def step():
            for c, st, th in groups:
                st.set_zero()
                mq.apply_(c, st, theta=th)
        return f"uneven batch, pure part: {sum(counts.values())} states, sizes {min(counts)}..{max(counts)}", step
    if name == "uneven":
        # the uneven batch's sizes below 18 qubits in the persistent launch (mbk_uneven, or
        # k_uneven without NVRTC), run eagerly (binding and fused products of all sizes, then
        # the one pass launch)
        from mossquantum_b200.batch import BatchPlan
        rng2 = W.rng_for(2)
        sizes = rng2.integers(10, 23, size=512)
        counts = {int(n): int((sizes == n).sum()) for n in np.unique(sizes) if n < 18}
        groups = {n: (W.hea_circuit(n, 8), B) for n, B in counts.items()}
        plan = BatchPlan(groups, W.xxz, persistent=True)
        th = {n: np.random.default_rng(n).uniform(0, 2 * np.pi, size=(B, c.nparameters()))
              for n, (c, B) in groups.items()}
        plan._stage(th)
        return f"persistent uneven launch: {sum(counts.values())} states, sizes 10..17", plan._record_body
    raise ValueError(f"unknown kernel case {name}")


KERNEL_CASES = ("dense1_low", "dense1_high", "tile", "density", "pauli", "adjoint", "grad24", "marginal", "dmma",
                "dense5", "batch_pure", "batch_pure_small", "uneven")


def kernel_workload(args):
    """One JSON line per kernel case: the case's dominant kernel with its launches, average
    launch time (CUDA events on the library stream) and algorithmic bytes and flops per
    launch, against the measured HBM peak and the FP64 rate of a DFMA-only probe."""
    import mossquantum_b200 as mq
    from mossquantum_b200 import _native as N
    from mossquantum_b200 import workloads as W
    mq.init(0)
    peak, peak_kind = load_peaks()
    fp64 = N.measure_fp64_peak()
    names = KERNEL_CASES if args.case == "all" else [c.strip() for c in args.case.split(",")]
    for name in names:
        desc, step = _case_setup(name, mq, W)
        for _ in range(max(1, args.warmup)):
            step()
        N.synchronize()
        N.profile(True)
        for _ in range(max(1, args.steps)):
            step()
        N.synchronize()
        rep = N.profile_report()
        N.profile(False)
        kern, (lc, tms, byts, flops) = max(rep.items(), key=lambda kv: kv[1][1])
        sec = tms / 1e3 / lc
        line = {"case": name, "what": desc, "kernel": kern, "launches": lc, "avg_launch_ms": tms / lc,
                "share": tms / sum(v[1] for v in rep.values()),
                "algorithmic_bytes_per_launch": byts / lc, "gbs": byts / lc / sec / 1e9,
                "hbm_frac": byts / lc / sec / 1e9 / peak, "hbm_peak": peak, "hbm_peak_kind": peak_kind,
                "algorithmic_flops_per_launch": flops / lc, "tflops": flops / lc / sec / 1e12,
                "fp64_frac": (flops / lc / sec / 1e12 / fp64) if fp64 else None, "fp64_peak_tflops": fp64,
                "others": {k: [v[0], v[1]] for k, v in rep.items() if k != kern}}
        print(json.dumps(line), flush=True)
    return 0


def log(msg):
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def grad_workload(args):
    """Gradients: adjoint gradient of the TFIM loss of a 24-qubit depth-16 hardware-efficient
    ansatz (1152 independent angles) with forward checkpoints every 4 layers, and the
    shared-parameter gradient of 64 ten-qubit density matrices with depolarizing noise
    (p = 0.005) after every gate. One step = one value_and_gradient of each; the plain
    per-call path (one plain kernel per gate and per reverse step) is timed beside it."""
    import torch
    import mossquantum_b200 as mq
    from mossquantum_b200 import _native as N
    from mossquantum_b200 import workloads as W
    mq.init(0)
    n, depth = 24, 16
    angles = W.hea_angles(n, depth, W.rng_for(3))
    c = W.hea_circuit(n, depth, angles)
    H = W.tfim(n)
    per_layer = 3 * n + (n - 1)
    obj = mq.ExpectationObjective(c, H, mq.StateVector(n))
    theta = c.active_parameters()
    cdm = W.hea_circuit(10, 4, W.hea_angles(10, 4, W.rng_for(3, 1)), noise=(0.005, 0.0))
    objb = mq.BatchExpectationObjective(cdm, W.tfim(10), mq.BatchDensityMatrix(10, 64))
    thb = cdm.active_parameters()
    method = mq.AdjointGradient(checkpoint_every=4 * per_layer)
    stream = torch.cuda.ExternalStream(N.stream_handle())

    def step():
        mq.value_and_gradient(method, obj, theta)
        mq.value_and_gradient(mq.AdjointGradient(), objb, thb)

    for _ in range(args.warmup):
        step()
    l0 = N.launch_count()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        t0 = time.perf_counter()
        start.record(stream)
        for _ in range(args.steps):
            step()
        end.record(stream)
        end.synchronize()
        wall = (time.perf_counter() - t0) / args.steps
    ms = start.elapsed_time(end) / args.steps
    launches = N.launch_count() - l0

    def part_ms(fn, reps=3):
        """Median over reps of one call, CUDA events on the library stream."""
        out = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            out.append(a.elapsed_time(b))
        return float(np.median(out))
    t_pure = part_ms(lambda: mq.value_and_gradient(method, obj, theta))
    t_dm = part_ms(lambda: mq.value_and_gradient(mq.AdjointGradient(), objb, thb))
    os.environ["MB_ADJOINT_PLAIN"] = "1"
    try:
        mq.value_and_gradient(method, obj, theta)
        t_plain = part_ms(lambda: mq.value_and_gradient(method, obj, theta), reps=2)
        mq.value_and_gradient(mq.AdjointGradient(), objb, thb)
        t_plain_dm = part_ms(lambda: mq.value_and_gradient(mq.AdjointGradient(), objb, thb), reps=1)
    finally:
        del os.environ["MB_ADJOINT_PLAIN"]
    roofline = dominant_roofline(N, lambda: mq.value_and_gradient(method, obj, theta), f"n{n}")
    line = {"metric": "adjoint gradient evaluations/s", "value": 1e3 / ms, "unit": "gradients/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "complex128 (f64)", "data": "synthetic (seeded)",
            "config": {"workload": "adjoint: 24q HEA depth 16 (1152 angles, checkpoints every 4 layers) + "
                                   "64 x 10q density matrices (depolarizing p=0.005, shared angles)",
                       "l2": "24-qubit states (256 MiB each) exceed L2"},
            "pure_24q_ms": t_pure, "density_batch_ms": t_dm,
            "parts_timing": "median of 3 calls (plain: 2 and 1), CUDA events on the library stream",
            "plain_per_call": {"pure_24q_ms": t_plain, "density_batch_ms": t_plain_dm,
                               "speedup_pure": t_plain / t_pure, "speedup_density": t_plain_dm / t_dm,
                               "speedup": (t_plain + t_plain_dm) / (t_pure + t_dm)},
            "roofline": roofline,
            "e2e": {"value": 1.0 / wall, "unit": "gradients/s", "h2d_bytes_per_step": 8 * (len(theta) + len(thb)),
                    "d2h_bytes_per_step": 8 * (len(theta) + len(thb) + 2)},
            "gpu_launches": launches, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def serve_measure(requests, rate, plain=True, seed_stream=0, log_prefix="serve"):
    """Serving at one arrival rate (None = saturating: every request arrives at t = 0).

    The request mix: 70% pure (8..26 qubits), 30% density matrices (6..12 qubits, depolarizing
    p = 0.01 and amplitude damping gamma = 0.02 after every gate), 4..32 hardware-efficient
    layers with random angles, TFIM or XXZ, half of them adjoint gradients. The server admits
    them against its HBM budget (160 GB or 90% of what the library holds). The plain
    per-request path then replays the same arrivals: each request alone through the per-call
    API (one plain kernel per gate, plain adjoint) in arrival order, its latency measured from
    its arrival to its completion."""
    import mossquantum_b200 as mq
    from mossquantum_b200 import _native as N
    from mossquantum_b200 import workloads as W
    from mossquantum_b200.serving import Server
    mq.init(0)
    budget = min(160 * 10**9, int(mq.memory_info()[1] * 0.9))
    blocks, obs = {}, {}

    def block(kind, n):
        if (kind, n) not in blocks:
            blocks[(kind, n)] = W.hea_layer(n, noise=W.SERVING_NOISE if kind == "density" else None)
        return blocks[(kind, n)]

    def observable(name, n):
        if (name, n) not in obs:
            obs[(name, n)] = W.tfim(n) if name == "tfim" else W.xxz(n)
        return obs[(name, n)]
    srv = Server(budget_bytes=budget)
    t0 = time.perf_counter()
    classes = [("pure", n) for n in range(8, 27)] + [("density", n) for n in range(6, 13)]
    # warm-up: every class alone, then three together (schedules and specialised kernels of both
    # batch shapes), outside the measurement
    for wave in ((("tfim", True),), (("tfim", True), ("xxz", False), ("tfim", False))):
        warm = [srv.submit(block(k, n), n, observable(o, n), np.zeros((2, 3 * n)), kind=k, gradient=g)
                for k, n in classes for o, g in wave]
        for t in warm:
            srv.wait(t)
    warm_s = time.perf_counter() - t0
    log(f"{log_prefix}: warm-up {warm_s:.1f} s")
    rng = W.rng_for(5, seed_stream)
    reqs = W.serving_requests(requests, rng)
    arrivals = np.zeros(len(reqs)) if rate is None else np.cumsum(rng.exponential(1.0 / rate, size=len(reqs)))
    srv.reset_stats()
    l0 = N.launch_count()
    tickets = []
    with ClockSampler(0) as clk:
        t_start = time.perf_counter()
        for (k, n, L, o, g, th), a in zip(reqs, arrivals):
            d = t_start + a - time.perf_counter()
            if d > 0:
                time.sleep(d)
            tickets.append(srv.submit(block(k, n), n, observable(o, n), th, kind=k, gradient=g))
        results = [srv.wait(t) for t in tickets]
        span = time.perf_counter() - t_start
    st = srv.stats()
    launches = N.launch_count() - l0
    srv.close()
    out = {"rate_req_per_s": "saturating" if rate is None else rate, "requests": len(reqs),
           "server": {"p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "evals_per_s": st["evals_per_s"],
                      "wall_evals_per_s": len(reqs) / span, "iterations": st["iterations"],
                      "peak_hbm_bytes": st["peak_bytes"], "warmup_s": warm_s,
                      "jit_compile_ms_in_run": st["jit_compile_ms"], "jit_compiles_in_run": st["jit_compiles"]},
           "gpu_launches": launches, "clocks": clk.summary(),
           "h2d_bytes": int(sum(8 * r[5].size for r in reqs)),
           "d2h_bytes": int(sum(16 + (8 * r[5].size if r[4] else 0) for r in reqs))}
    log(f"{log_prefix}: server p50 {st['p50_ms']:.0f} ms p99 {st['p99_ms']:.0f} ms "
        f"{st['evals_per_s']:.2f} evals/s over {span:.1f} s")
    if not plain:
        return out
    os.environ["MB_ADJOINT_PLAIN"] = "1"
    lat, max_err = [], 0.0
    try:
        t_start = time.perf_counter()
        for ((k, n, L, o, g, th), a), res in zip(zip(reqs, arrivals), results):
            d = t_start + a - time.perf_counter()
            if d > 0:
                time.sleep(d)
            noise = W.SERVING_NOISE if k == "density" else None
            init = mq.DensityMatrix(n) if k == "density" else mq.StateVector(n)
            if g:
                tmpl = W.unrolled(lambda row: W.hea_layer(n, noise=noise), th)
                objp = mq.ExpectationObjective(tmpl, observable(o, n), init)
                v, grad = mq.value_and_gradient(mq.AdjointGradient(), objp, th.reshape(-1))
                max_err = max(max_err, float(np.max(np.abs(grad - res.gradient.reshape(-1)))))
            else:
                circ = W.unrolled(lambda row: W.hea_layer_bound(n, row, noise=noise), th)
                s_ = mq.apply_(circ, init, plain=True)
                v = mq.expectation(observable(o, n), s_).real
            max_err = max(max_err, abs(v - res.value.real))
            lat.append((time.perf_counter() - (t_start + a)) * 1e3)
        pspan = time.perf_counter() - t_start
    finally:
        del os.environ["MB_ADJOINT_PLAIN"]
    out["plain_per_request"] = {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                                "evals_per_s": len(reqs) / pspan,
                                "method": "the same requests replayed at the same arrival times, each alone "
                                          "through the per-call API (one plain kernel per gate, plain adjoint)"}
    out["speedup_evals_per_s"] = out["server"]["evals_per_s"] / out["plain_per_request"]["evals_per_s"]
    out["max_abs_diff_vs_plain"] = max_err
    log(f"{log_prefix}: plain p50 {out['plain_per_request']['p50_ms']:.0f} ms "
        f"{out['plain_per_request']['evals_per_s']:.2f} evals/s")
    return out


def serve_workload(args):
    """Serving: the request mix of serve_measure at each rate of --rates ("sat" = saturating),
    --requests requests per rate, beside the plain per-request path replaying the same
    arrivals."""
    levels = []
    for i, r in enumerate(args.rates.split(",")):
        rate = None if r.strip() in ("sat", "inf") else float(r)
        levels.append(serve_measure(args.requests, rate, seed_stream=i, log_prefix=f"serve[{r}]"))
    best = max(levels, key=lambda lv: lv["server"]["evals_per_s"])
    line = {"metric": "serving circuit-evals/s (continuous batching) with p50/p99 latency",
            "value": best["server"]["evals_per_s"], "unit": "evals/s", "n_gpus": 1, "steps": len(levels),
            "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "complex128 (f64)", "data": "synthetic (seeded)",
            "config": {"workload": "Poisson stream: 70% pure 8..26q, 30% density 6..12q (noisy), 4..32 layers, "
                                   "TFIM/XXZ, 50% adjoint gradients", "requests_per_rate": args.requests},
            "levels": levels,
            "e2e": {"value": best["server"]["wall_evals_per_s"], "unit": "evals/s",
                    "h2d_bytes_per_step": best["h2d_bytes"], "d2h_bytes_per_step": best["d2h_bytes"],
                    "note": "requests submitted from host memory, results read back on the host"},
            "gpu_launches": sum(lv["gpu_launches"] for lv in levels), "clocks": best["clocks"]}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload == "batch":
        return batch_workload(args)
    if args.workload == "grad":
        return grad_workload(args)
    if args.workload == "serve":
        return serve_workload(args)
    if args.workload == "kernel":
        return kernel_workload(args)
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
    if args.variant in ("block", "tensor"):
        circuit = mq.fuse_gates(circuit, max_qubits=5)   # host fusion at bind time, outside the timed region
    state = mq.StateVector(n)
    plain = args.variant != "fused"
    tensor = args.variant == "tensor"
    stream = torch.cuda.ExternalStream(N.stream_handle(), device=local)

    def step():
        state.set_zero()
        mq.apply_(circuit, state, plain=plain, tensor=tensor)

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
    from mossquantum_b200 import replicas
    ms = replicas.max_over_ranks(start.elapsed_time(end), device=f"cuda:{local}")   # slowest replica
    if world > 1:
        dist.barrier()
    ms_step = ms / args.steps
    bytes_step = plain_bytes(n, depth)
    value = replicas.aggregate_rate(bytes_step, world, ms_step / 1e3) / 1e9

    roofline = dominant_roofline(N, step, f"n{n}")

    # End to end through the public API: host circuit in, probabilities of 10 qubits out.
    e2e = None
    if not args.no_e2e:
        circuits = [build_workload(mq, W, n, depth, (rank, 1000 + i)) for i in range(args.e2e_steps + 1)]
        h2d = sum(16 * (1 << len(g.positions)) ** 2 for g in circuits[0].flat())
        readout = list(range(1, 11))

        def e2e_step(c):
            state.set_zero()
            if args.variant in ("block", "tensor"):
                c = mq.fuse_gates(c, max_qubits=5)
            mq.apply_(c, state, plain=plain, tensor=tensor)
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
        v, dt = cpu_baseline_run(n, 1, threads, W, repeats=3)
        cpu = {"value": v, "unit": "GB/s", "cores": threads, "kind": "port",
               "sample": f"1 of {depth} layers at n={n}, median of 3 warm runs ({dt:.2f} s each; C++ restatement "
                         f"of the reference CPU method, host-native build)",
               "anchor": cpu_anchor(threads)}

    # The rest of the headline metric on the same run: circuit-evals/s of the uneven batch against
    # the plain per-call path, and serving p50/p99 and evals/s at a saturating request stream
    # against the plain per-request path replaying the same arrivals (single replica only).
    extras = None
    if not args.no_extras and world == 1:
        extras = {}
        b = batch_measure(steps=3, warmup=2)
        extras["batch"] = {"workload": "512 pure (n=10..22, HEA depth 8, per-sample angles) + 64 density (n=10, "
                                       "noisy) <XXZ>, one CUDA-graph replay per plan",
                           "evals_per_s": b["evals_per_s"], "ms_per_step": b["ms_per_step"],
                           "pure_ms_per_step": b["pure_ms_per_step"], "density_ms_per_step": b["density_ms_per_step"],
                           "plain_per_call_evals_per_s": b["plain_per_call"]["evals_per_s"],
                           "plain_sample": b["plain_per_call"]["sample"], "speedup_vs_plain": b["speedup_vs_plain"],
                           "e2e_evals_per_s": b["e2e"]["evals_per_s"], "plan_build_s": b["plan_build_s"],
                           "gpu_launches": b["gpu_launches"], "clocks": b["clocks"]}
        srv = serve_measure(200, None, seed_stream=0)
        extras["serving"] = {"workload": "200 requests arriving at once (saturating): 70% pure 8..26q, 30% density "
                                         "6..12q (noisy), 4..32 layers, TFIM/XXZ, 50% adjoint gradients",
                             "server": srv["server"], "plain_per_request": srv.get("plain_per_request"),
                             "speedup_evals_per_s": srv.get("speedup_evals_per_s"),
                             "max_abs_diff_vs_plain": srv.get("max_abs_diff_vs_plain"),
                             "gpu_launches": srv["gpu_launches"], "clocks": srv["clocks"]}

    if rank == 0:
        line = {"metric": "gate-kernel HBM GB/s (effective, plain per-gate bytes)", "value": value, "unit": "GB/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128 (f64)",
                "data": "synthetic (seeded)",
                "config": {"workload": f"u3_cz_brickwork n={n} layers={depth}", "qubits": n, "layers": depth,
                           "state_bytes": 16 << n, "variant": args.variant, "parallelism": f"replicas x{world}",
                           "l2": "state (4 GiB) is larger than L2; no flush needed"},
                "layers_per_s": world * depth / (ms_step / 1e3),
                "value_note": "value counts the bytes the plain per-gate method would move (one sweep per gate); "
                              "the fused passes move 32*2^n bytes per pass, see hbm_measured",
                "hbm_measured": ({"gbs": roofline["hbm"]["achieved"], "frac": roofline["hbm"]["frac"],
                                  "peak": roofline["hbm"]["peak"], "kernel": roofline["kernel"]} if roofline else None),
                "roofline": roofline, "cpu_baseline": cpu,
                "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary(), "extras": extras}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
