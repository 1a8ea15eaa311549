"""Seeded synthetic workloads: the circuits and observables the benchmarks and tests use.

The reference publishes no dataset for this path; every input is synthetic and seeded
(base seed 20261203). Shapes follow the reference's hardware-efficient benchmark circuits
(docs/performance/cpu-scheduling-2026-11-17/benchmark-source/cpu_thread_scan.jl:4-18) and
its spin-chain builders (src/utilities/models/spin_hamiltonians.jl:7-63).
"""
from __future__ import annotations

import numpy as np

from .channels import AmplitudeDamping, Depolarizing
from .circuit import QCircuit
from .gates import CNOTGate, CZGate, QuantumGate, RxGate, RyGate, RzGate, U3
from .operators import QubitsOperator, QubitsTerm

BASE_SEED = 20261203


def rng_for(*stream):
    return np.random.default_rng([BASE_SEED, *stream])


def hea_angles(n, depth, rng):
    return rng.uniform(0.0, 2 * np.pi, size=(depth, n, 3))


def hea_circuit(n, depth, angles=None, active=True, noise=None):
    """Layer: RX, RY, RZ on every qubit (in that order per qubit), then CNOT(i, i+1).

    noise=(p, gamma): after every gate, Depolarizing(p) then AmplitudeDamping(gamma) on
    each qubit the gate touches.
    """
    if angles is None:
        angles = np.zeros((depth, n, 3))
    c = QCircuit()

    def add(g):
        c.push(g)
        if noise is not None:
            p, gamma = noise
            for q in g.positions:
                if p:
                    c.push(Depolarizing(q, p))
                if gamma:
                    c.push(AmplitudeDamping(q, gamma))

    for layer in range(depth):
        for q in range(1, n + 1):
            add(RxGate(q, angles[layer, q - 1, 0], isparas=active))
            add(RyGate(q, angles[layer, q - 1, 1], isparas=active))
            add(RzGate(q, angles[layer, q - 1, 2], isparas=active))
        for q in range(1, n):
            add(CNOTGate(q, q + 1))
    return c


def cpu_scan_circuit(angles_by_layer):
    """The reference's CPU-scheduling benchmark circuit (cpu_thread_scan.jl:4-18): on 1-based
    layer l and qubit q a fixed (RX, RY, RZ)[mod1(l + q, 3)] with angle angles_by_layer[l][q],
    then CNOT(q, q + 1) for q = 1..n-1."""
    angles = np.asarray(angles_by_layer, dtype=np.float64)
    depth, n = angles.shape
    rot = (RxGate, RyGate, RzGate)
    c = QCircuit()
    for layer in range(1, depth + 1):
        for q in range(1, n + 1):
            c.push(rot[(layer + q - 1) % 3](q, float(angles[layer - 1, q - 1])))
        for q in range(1, n):
            c.push(CNOTGate(q, q + 1))
    return c


def u3_params(n, depth, rng):
    u = rng.uniform(0.0, 1.0, size=(depth, n))
    theta = np.arccos(1 - 2 * u)
    phi = rng.uniform(0.0, 2 * np.pi, size=(depth, n))
    lam = rng.uniform(0.0, 2 * np.pi, size=(depth, n))
    return np.stack([theta, phi, lam], axis=-1)


def u3_brickwork(n, depth, params):
    """Layer l (0-based): U3 on every qubit, then CZ on (1,2),(3,4),... for even l and
    (2,3),(4,5),... for odd l."""
    c = QCircuit()
    for layer in range(depth):
        for q in range(1, n + 1):
            c.push(QuantumGate(q, U3(*params[layer, q - 1])))
        start = 1 if layer % 2 == 0 else 2
        for q in range(start, n, 2):
            c.push(CZGate(q, q + 1))
    return c


def tfim(n, h=1.0, J=1.0):
    """H = -J sum Z_i Z_{i+1} - h sum X_i (open chain)."""
    terms = [QubitsTerm([i, i + 1], ["Z", "Z"], -J) for i in range(1, n)]
    terms += [QubitsTerm([i], ["X"], -h) for i in range(1, n + 1)]
    return QubitsOperator(terms)


def xxz(n, J=1.0, Jzz=0.5):
    """H = sum (J X_i X_{i+1} + J Y_i Y_{i+1} + Jzz Z_i Z_{i+1})."""
    terms = []
    for i in range(1, n):
        terms += [QubitsTerm([i, i + 1], ["X", "X"], J), QubitsTerm([i, i + 1], ["Y", "Y"], J),
                  QubitsTerm([i, i + 1], ["Z", "Z"], Jzz)]
    return QubitsOperator(terms)


def unrolled(block_for, theta):
    """The full circuit of a layered request: block_for(angles of one layer) per row of theta."""
    c = QCircuit()
    for row in np.asarray(theta):
        c.push(block_for(row))
    return c


def hea_layer(n, noise=None):
    """One hardware-efficient layer with active parameters (3n angles, zeros)."""
    return hea_circuit(n, 1, noise=noise)


def hea_layer_bound(n, row, noise=None):
    """One hardware-efficient layer with its 3n angles bound (row ordered as hea_layer's
    active parameters: RX, RY, RZ per qubit)."""
    return hea_circuit(n, 1, np.asarray(row, dtype=np.float64).reshape(1, n, 3), noise=noise)


SERVING_NOISE = (0.01, 0.02)


def serving_requests(count, rng, pure_n=(8, 26), dm_n=(6, 12), layers=(4, 32), pure_frac=0.7, grad_frac=0.5):
    """Request mix of the serving benchmark: (kind, n, repeats, observable name, gradient,
    theta of shape (repeats, 3n)) per request, drawn from rng."""
    out = []
    for _ in range(count):
        pure = rng.random() < pure_frac
        n = int(rng.integers(pure_n[0], pure_n[1] + 1)) if pure else int(rng.integers(dm_n[0], dm_n[1] + 1))
        L = int(rng.integers(layers[0], layers[1] + 1))
        obs = "tfim" if rng.random() < 0.5 else "xxz"
        grad = bool(rng.random() < grad_frac)
        theta = rng.uniform(0.0, 2 * np.pi, size=(L, 3 * n))
        out.append(("pure" if pure else "density", n, L, obs, grad, theta))
    return out
