"""Continuous-batching server for ansatz evaluations and adjoint gradients.

The reference evaluates one objective per call (``evaluate`` / ``value_and_gradient``,
src/api/objectives.jl:15-244, src/differentiation/objectives.jl:183-296). ``Server`` keeps a
stream of independent requests resident on the GPU instead: a request is ``repeats``
repetitions of a parametrised block circuit (one ansatz layer) with its own parameters per
repetition, on ``|0...0>`` of a pure state or a density matrix, and asks for ``<H>`` and,
optionally, its adjoint gradient. The library's scheduler thread admits requests against the
server's HBM byte budget (16*2^n per pure state, 16*4^n per density matrix, plus gradient
buffers), advances every admitted request by one layer per iteration (requests of the same
block share one batched launch per pass, each with its own parameters), and lets requests
join and leave between iterations (``mb_server_*`` in include/mossb200.h).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .circuit import QCircuit
from .operators import as_operator


@dataclass
class Result:
    value: complex
    gradient: np.ndarray | None   # (repeats, nparameters of the block) for gradient requests
    latency_ms: float
    queue_ms: float
    iterations: int


class Server:
    """Server(budget_bytes=0, max_active=0): start the library's scheduler thread.

    budget_bytes: admission budget (0 = what the library budget leaves); max_active: most
    admitted requests at once (0 = 4096)."""

    def __init__(self, budget_bytes: int = 0, max_active: int = 0):
        cfg = N.MbServerConfig()
        cfg.hbm_budget_bytes = int(budget_bytes)
        cfg.max_active = int(max_active)
        h = ctypes.c_void_p()
        N.check(N.lib().mb_server_start(ctypes.byref(cfg), ctypes.byref(h)), "mb_server_start")
        self._h = h
        self._meta = {}      # ticket -> (repeats, nslots, keep-alive references)
        self._closed = False

    def submit(self, block: QCircuit, n: int, observable, theta, kind: str = "pure", gradient: bool = False) -> int:
        """Queue ``repeats`` layers of ``block`` (compiled for n qubits) with parameters
        ``theta`` of shape (repeats, block.nparameters()); returns a ticket."""
        if self._closed:
            raise ValueError("the server is closed")
        if kind not in ("pure", "density"):
            raise ValueError("kind must be 'pure' or 'density'")
        compiled = block.compiled(n)
        th = np.asarray(theta, dtype=np.float64)
        if th.ndim != 2 or th.shape[1] != block.nparameters():
            raise ValueError(f"theta must have shape (repeats, {block.nparameters()})")
        slots = np.ascontiguousarray(compiled.theta_from(th))
        obs = as_operator(observable).handle()
        req = N.MbRequest()
        req.block = compiled.handle
        req.observable = obs.handle
        req.kind = N.MB_PURE if kind == "pure" else N.MB_DENSITY
        req.repeats = th.shape[0]
        req.theta = slots.ctypes.data if slots.size else None
        req.ntheta = slots.size
        req.gradient = 1 if gradient else 0
        t = ctypes.c_uint64()
        N.check(N.lib().mb_submit(self._h, ctypes.byref(req), ctypes.byref(t)), "mb_submit")
        self._meta[t.value] = (th.shape[0], compiled.nslots, gradient, (compiled, obs, block))
        return t.value

    def _result(self, ticket, rc, res, grad):
        if rc == N.MB_ENOTREADY:
            return None
        N.check(rc, "server result")
        repeats, nslots, gradient, _ = self._meta.pop(ticket)
        if res.status != N.MB_OK:
            raise N.BackendError(f"request {ticket} failed ({res.status}): {res.error.decode(errors='replace')}")
        g = grad.reshape(repeats, nslots) if gradient else None
        return Result(complex(res.value[0], res.value[1]), g, res.latency_ms, res.queue_ms, res.iterations)

    def _grad_buffer(self, ticket):
        repeats, nslots, gradient, _ = self._meta[ticket]
        return np.zeros(max(1, repeats * nslots) if gradient else 1)

    def poll(self, ticket: int) -> Result | None:
        """The result if the request has finished, else None."""
        res = N.MbResult()
        grad = self._grad_buffer(ticket)
        rc = N.lib().mb_poll(self._h, ticket, ctypes.byref(res), N.dptr(grad), grad.size)
        return self._result(ticket, rc, res, grad)

    def wait(self, ticket: int, timeout_s: float | None = None) -> Result:
        res = N.MbResult()
        grad = self._grad_buffer(ticket)
        ms = -1 if timeout_s is None else int(timeout_s * 1e3)
        rc = N.lib().mb_wait(self._h, ticket, ms, ctypes.byref(res), N.dptr(grad), grad.size)
        if rc == N.MB_ETIMEOUT:
            raise TimeoutError(f"request {ticket} still running after {timeout_s} s")
        return self._result(ticket, rc, res, grad)

    def stats(self) -> dict:
        s = N.MbServerStats()
        N.check(N.lib().mb_server_stats_get(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in N.MbServerStats._fields_}

    def reset_stats(self) -> None:
        N.check(N.lib().mb_server_stats_reset(self._h))

    def close(self) -> None:
        if not self._closed:
            self._closed = True
            N.lib().mb_server_stop(self._h)
            self._meta.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
