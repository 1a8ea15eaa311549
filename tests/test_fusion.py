"""fuse_gates on the host, checked with the oracle (CPU).

Restates the reference's fusion regression cases (test/regression/operators.jl:139-172):
block counts, boundaries at parameterized gates, channels and nested circuits, and equality
of the fused and unfused circuits on pure and density states (tolerance 1e-12).
"""
import numpy as np
import pytest

import mossquantum_b200 as mq
from mossquantum_b200.fusion import fuse_gates


def run(O, circ, state, n, dm=False):
    return O.apply(circ.specs(), state, n, dm=dm)


def normalized(v):
    v = np.asarray(v, dtype=complex)
    return v / np.linalg.norm(v)


def test_reference_cases(O):
    circuit = mq.QCircuit([mq.HGate(3), mq.CNOTGate(3, 1), mq.TGate(2), mq.SWAPGate(2, 3), mq.YGate(1)])
    state = normalized([1, 2j, 3, 4j, 5, 6j, 7, 8j])
    fused = fuse_gates(circuit)
    assert len(fused) == 1 and len(circuit) == 5
    ref = run(O, circuit, state, 3)
    assert np.max(np.abs(run(O, fused, state, 3) - ref)) <= 1e-12
    rho = np.outer(state, state.conj()).reshape(-1, order="F")
    assert np.max(np.abs(run(O, fused, rho, 3, True) - run(O, circuit, rho, 3, True))) <= 1e-12
    for mqb in (2, 1):
        assert np.max(np.abs(run(O, fuse_gates(circuit, max_qubits=mqb), state, 3) - ref)) <= 1e-12
    assert len(fuse_gates(mq.QCircuit())) == 0
    with pytest.raises(ValueError):
        fuse_gates(circuit, max_qubits=6)

    pgate = mq.RyGate(1, 0.2, isparas=True)
    noise = mq.Depolarizing(1, 0.1)
    noisy = mq.QCircuit([mq.HGate(1), mq.XGate(1), pgate, mq.ZGate(1), mq.XGate(1), noise, mq.XGate(2), mq.ZGate(2)])
    fn = fuse_gates(noisy)
    assert len(fn) == 5 and fn[1] is pgate and fn[3] is noise
    assert fn.active_parameters() == [0.2]
    z = O.zero_state(2, True)
    assert np.max(np.abs(run(O, fn, z, 2, True) - run(O, noisy, z, 2, True))) <= 1e-12

    nested = mq.QCircuit([mq.QCircuit([mq.XGate(1), mq.ZGate(1)]), mq.XGate(2), mq.ZGate(2)])
    assert len(fuse_gates(nested)[0]) == 1
    z = O.zero_state(2)
    assert np.max(np.abs(run(O, fuse_gates(nested), z, 2) - run(O, nested, z, 2))) <= 1e-12

    wide = mq.QCircuit([mq.HGate(1), mq.XGate(5), mq.CNOTGate(5, 2), mq.YGate(4), mq.ZGate(3)])
    s5 = normalized(np.arange(1, 33))
    assert np.max(np.abs(run(O, fuse_gates(wide), s5, 5) - run(O, wide, s5, 5))) <= 1e-12


@pytest.mark.parametrize("max_qubits", [4, 5])
def test_bound_fusion_of_ansatz(O, max_qubits):
    from mossquantum_b200 import workloads as W
    n, depth = 9, 3
    c = W.hea_circuit(n, depth, W.hea_angles(n, depth, W.rng_for(9)), active=False)
    f = fuse_gates(c, max_qubits=max_qubits, bound=True)
    assert len(f) < len(c) // 3
    assert all(len(g.positions) <= max_qubits for g in f)
    assert len(f) < len(fuse_gates(c, max_qubits=max_qubits)) < len(c)  # unbound: only the CNOT ladders fuse
    z = O.zero_state(n)
    assert np.max(np.abs(run(O, f, z, n) - run(O, c, z, n))) <= 1e-12
    u = W.u3_brickwork(n, 2, W.u3_params(n, 2, W.rng_for(9, 1)))
    fu = fuse_gates(u, max_qubits=max_qubits)
    assert np.max(np.abs(run(O, fu, z, n) - run(O, u, z, n))) <= 1e-12
