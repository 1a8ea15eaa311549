"""Host-side gate fusion: ``fuse_gates`` (src/utilities/algorithms/gate_fusion.jl:10-62).

Adjacent gates are multiplied into one dense gate while their combined support has at most
``max_qubits`` qubits; parameterized gates, channels and circuit boundaries end a block, and
nested circuits are fused recursively, as in the reference. ``bound=True`` extends fusion to
parameterized gates whose parameters are all frozen (their matrices are fixed once bound):
the bound form of a circuit then runs as few dense 4- and 5-qubit blocks, which the library
applies on the FP64 tensor cores (``apply_(..., plain=True, tensor=True)``).
"""
from __future__ import annotations

import numpy as np

from .circuit import QCircuit
from .gates import Gate, QuantumGate


def _eligible(op, max_qubits, bound):
    if not isinstance(op, Gate) or op.nqubits > max_qubits:
        return False
    params = op.parameters()
    if params is None:
        return True
    if not bound:
        return False
    act = op.is_parameters() or []
    return not any(act)


def _fusion_matrix(g: Gate, support):
    """ordered_mat(g) embedded in the sorted support (first qubit = least significant bit)."""
    pos = g.ordered_positions()
    data = g.ordered_mat()
    if tuple(pos) == tuple(support):
        return data
    bits = [support.index(p) for p in pos]
    mask = sum(1 << b for b in bits)
    dim = 1 << len(support)
    cols = np.arange(dim)
    lrows = np.arange(1 << len(bits))
    lcols = np.zeros(dim, dtype=np.int64)
    scatter = np.zeros(len(lrows), dtype=np.int64)
    for j, b in enumerate(bits):
        lcols |= ((cols >> b) & 1) << j
        scatter |= ((lrows >> j) & 1) << b
    rows = (cols & ~mask)[None, :] | scatter[:, None]
    out = np.zeros((dim, dim), dtype=complex)
    out[rows, np.broadcast_to(cols, rows.shape)] = data[lrows[:, None], lcols[None, :]]
    return out


def fuse_gates(circuit: QCircuit, max_qubits: int = 5, bound: bool = False) -> QCircuit:
    """fuse_gates(circuit; max_qubits=5): a new circuit with adjacent eligible gates fused."""
    if not 1 <= max_qubits <= 5:
        raise ValueError("max_qubits must be between 1 and 5.")
    result = QCircuit()
    pending = None
    for op in circuit:
        if not _eligible(op, max_qubits, bound):
            if pending is not None:
                result.push(pending)
                pending = None
            result.push(fuse_gates(op, max_qubits, bound) if isinstance(op, QCircuit) else op)
        elif pending is None:
            pending = op
        else:
            support = sorted(set(pending.positions) | set(op.positions))
            if len(support) <= max_qubits:
                combined = _fusion_matrix(op, support) @ _fusion_matrix(pending, support)
                pending = QuantumGate(tuple(support), combined)
            else:
                result.push(pending)
                pending = op
    if pending is not None:
        result.push(pending)
    return result
