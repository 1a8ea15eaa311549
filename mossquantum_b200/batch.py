"""Uneven-size batches with per-sample parameters, replayed from a captured CUDA graph.

MOSSQuantum's batches share one register size and one parameter vector
(src/states/batch_state_vector.jl, docs/architecture.md). A ``BatchPlan`` accepts samples
of different qubit counts, each with its own parameters. Pure samples of 8..17 qubits run in
ONE persistent kernel launch (``mb_uneven_apply``): its CTAs take work items (pass, sample,
chunk of tiles) from a work counter, pass by pass, and run them with straight-line code
compiled for the plan's passes, so no launch is spent per size or per pass. Larger samples and
density matrices are grouped by size into device batches that run the fused pass kernels over
all of their samples at once. The whole sequence (reset, parameter binding, passes,
expectations) is recorded once into a CUDA graph; ``run`` uploads the parameters and replays
the graph.
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from . import _native as N
from .backend import apply_
from .circuit import QCircuit
from .operators import as_operator
from .states import BatchDensityMatrix, BatchStateVector


class BatchPlan:
    """groups: {n: (template circuit for n qubits, samples B_n)}; observable_for(n) gives the
    observable evaluated on every sample of size n. kind: "pure" or "density"."""

    def __init__(self, groups, observable_for, kind="pure", autotune=False, autotune_max_bits=24,
                 persistent="auto"):
        """persistent: True runs the pure groups of 8..17 qubits in one persistent launch, False
        runs every group with its own pass launches; "auto" captures both and keeps the faster
        replay (the per-size form then uses the specialised kernels for those sizes too, whose
        compile cost the plan pays once)."""
        self.kind = kind
        self.tuned = {}
        self.groups = []
        total = 0
        for n in sorted(groups):
            circuit, B = groups[n]
            if not isinstance(circuit, QCircuit):
                raise TypeError("each group needs a QCircuit")
            state = BatchDensityMatrix(n, B) if kind == "density" else BatchStateVector(n, B)
            obs = as_operator(observable_for(n))
            compiled = circuit.compiled(n)
            self.groups.append(dict(n=n, B=B, circuit=circuit, compiled=compiled, state=state, obs=obs,
                                    offset=total))
            total += B
        self.total = total
        buf = ctypes.c_void_p()
        N.check(N.lib().mb_buffer_alloc(16 * max(1, total), ctypes.byref(buf)), "mb_buffer_alloc")
        self.results = buf
        self.graph = None
        if autotune:
            # Tile width, register width and fusion width per register size, timed on each
            # group's own batch with random angles (sizes on specialised kernels try a short
            # list, one compilation per candidate); sizes above autotune_max_bits keep defaults.
            from .autotune import autotune as tune, get_fusion
            rng = np.random.default_rng(0)
            for g in self.groups:
                bits = 2 * g["n"] if kind == "density" else g["n"]
                if 8 <= bits <= autotune_max_bits:
                    th = rng.uniform(0, 2 * np.pi, size=(g["B"], g["circuit"].nparameters()))
                    t, r, ms = tune(g["circuit"], g["state"], th)
                    self.tuned[bits] = (t, r, get_fusion(bits), ms)
        # Eager warm-up with zero parameters: builds schedules, kernels and reduction plans.
        self._stage({g["n"]: np.zeros((g["B"], g["circuit"].nparameters())) for g in self.groups})
        self.uneven = None
        self.choice = None
        small = [g["n"] for g in self.groups if 8 <= g["n"] <= 17] if kind == "pure" else []
        if persistent and small:
            cs = (ctypes.c_void_p * len(self.groups))(*[g["compiled"].handle.value for g in self.groups])
            ss = (ctypes.c_void_p * len(self.groups))(*[g["state"].handle.value for g in self.groups])
            u = ctypes.c_void_p()
            N.check(N.lib().mb_uneven_create(cs, ss, len(self.groups), ctypes.byref(u)), "mb_uneven_create")
            self.uneven = u
        self._record_body()
        N.synchronize()
        self._capture()
        if persistent == "auto" and self.uneven is not None:
            self._choose(small)

    def _replay_ms(self, reps=3):
        N.check(N.lib().mb_graph_launch(self.graph), "mb_graph_launch")
        N.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            N.check(N.lib().mb_graph_launch(self.graph), "mb_graph_launch")
        N.synchronize()
        return (time.perf_counter() - t0) * 1e3 / reps

    def _choose(self, small):
        """Times the persistent form against per-size launches of specialised kernels for the
        same groups (both as captured graphs) and keeps the faster."""
        from . import autotune as A
        L = N.lib()
        t_persistent = self._replay_ms()
        graph_p, uneven_p = self.graph, self.uneven
        saved = {n: (A.get(n), A.get_fusion(n)) for n in small}
        self.graph, self.uneven = None, None
        t_specialised = None
        try:
            for n in small:
                N.check(L.mb_tuning_set_specialised(n, 1), "mb_tuning_set_specialised")
                A.set(n, 10, 3)
            self._record_body()
            N.synchronize()
            self._capture()
            t_specialised = self._replay_ms()
        except Exception:  # noqa: BLE001 - any failure keeps the persistent form
            t_specialised = None
        # The captured graph keeps the kernels it was recorded with, so the process-wide
        # settings of these register sizes go back to what they were either way.
        for n in small:
            L.mb_tuning_set_specialised(n, -1)
            (t, r), f = saved[n]
            A.set(n, t, r)
            A.set_fusion(n, f)
        if t_specialised is not None and t_specialised < t_persistent:
            L.mb_graph_free(graph_p)
            L.mb_uneven_free(uneven_p)
            chosen = "per-size specialised"
        else:
            if self.graph is not None:
                L.mb_graph_free(self.graph)
            self.graph, self.uneven = graph_p, uneven_p
            chosen = "persistent"
        self.choice = {"persistent_ms": t_persistent, "per_size_specialised_ms": t_specialised, "chosen": chosen}

    def _stage(self, thetas):
        for g in self.groups:
            th = np.asarray(thetas[g["n"]], dtype=np.float64)
            if th.shape != (g["B"], g["circuit"].nparameters()):
                raise ValueError(f"parameters for n={g['n']} must have shape {(g['B'], g['circuit'].nparameters())}")
            slots = np.ascontiguousarray(g["compiled"].theta_from(th))
            N.check(N.lib().mb_theta_upload(g["compiled"].handle, N.dptr(slots), slots.size, g["B"]),
                    "mb_theta_upload")

    def _record_body(self):
        L = N.lib()
        if self.uneven is not None:
            N.check(L.mb_uneven_apply(self.uneven, N.MB_UNEVEN_ZERO), "uneven apply (recorded)")
        for g in self.groups:
            st = g["state"]
            if self.uneven is None:
                N.check(L.mb_state_set_zero(st.handle))
                N.check(L.mb_apply(g["compiled"].handle, st.handle, None, 0,
                                   N.MB_APPLY_DEVICE_THETA | N.MB_APPLY_PER_SAMPLE), "apply (recorded)")
            out = ctypes.c_void_p(self.results.value + 16 * g["offset"])
            N.check(L.mb_expect_to_device(g["obs"].handle().handle, st.handle, out), "expectation (recorded)")

    def _capture(self):
        L = N.lib()
        N.check(L.mb_graph_begin(), "mb_graph_begin")
        try:
            self._record_body()
        except Exception:
            h = ctypes.c_void_p()
            L.mb_graph_end(ctypes.byref(h))
            if h.value:
                L.mb_graph_free(h)
            raise
        h = ctypes.c_void_p()
        N.check(L.mb_graph_end(ctypes.byref(h)), "mb_graph_end")
        self.graph = h

    def run(self, thetas):
        """thetas: {n: (B_n, P_n) per-sample parameters}. Returns {n: real <H> per sample}."""
        self._stage(thetas)
        N.check(N.lib().mb_graph_launch(self.graph), "mb_graph_launch")
        host = np.zeros(2 * max(1, self.total))
        N.check(N.lib().mb_buffer_download(self.results, host.ctypes.data_as(ctypes.c_void_p), 16 * self.total))
        vals = host[0::2] + 1j * host[1::2]
        return {g["n"]: vals[g["offset"]:g["offset"] + g["B"]] for g in self.groups}

    def persistent_info(self):
        """(groups in the persistent launch, groups on the per-size path, samples in the launch)."""
        if self.uneven is None:
            return 0, len(self.groups), 0
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        N.check(N.lib().mb_uneven_info(self.uneven, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def close(self):
        if self.graph is not None:
            N.lib().mb_graph_free(self.graph)
            self.graph = None
        if getattr(self, "uneven", None) is not None:
            N.lib().mb_uneven_free(self.uneven)
            self.uneven = None
        if self.results:
            N.lib().mb_buffer_free(self.results)
            self.results = ctypes.c_void_p()


def run_plain(groups, observable_for, thetas, kind="pure"):
    """The plain per-call path: every sample separately, one plain kernel launch per gate."""
    from .backend import expectation
    from .states import DensityMatrix, StateVector
    out = {}
    for n in sorted(groups):
        circuit, B = groups[n]
        obs = observable_for(n)
        vals = []
        for b in range(B):
            s = DensityMatrix(n) if kind == "density" else StateVector(n)
            apply_(circuit, s, theta=thetas[n][b], plain=True)
            vals.append(expectation(obs, s))
        out[n] = np.array(vals)
    return out
