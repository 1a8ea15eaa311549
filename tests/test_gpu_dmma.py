"""K5: dense 4- and 5-qubit operators on the FP64 tensor cores, against the oracle.

Random unitaries on low, high and mixed position sets, on single and batch pure states and on
density matrices (U on the row bits, conj(U) on the column bits), a 2-qubit channel (a dense
4-bit supermatrix), and host-fused ansatz blocks. Every case is compared with the oracle
(1e-12 max-abs) and the tensor-core path is checked to have launched K5.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def random_unitary(d, rng):
    q, r = np.linalg.qr(rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d)))
    return q * (np.diag(r) / np.abs(np.diag(r)))


def random_state(n, rng):
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def used(N, prefix):
    return any(k.startswith(prefix) for k in N.profile_report())


POSITION_SETS = [(1, 2, 3, 4, 5), (3, 1, 5, 2, 4), (8, 11, 2, 6, 12), (12, 13, 14, 10, 11), (1, 2, 3, 4), (2, 9, 13, 5)]


@pytest.mark.parametrize("positions", POSITION_SETS)
@pytest.mark.parametrize("n", [11, 14])
def test_dense_block_pure(mq, O, positions, n):
    from mossquantum_b200 import _native as N
    if max(positions) > n:
        pytest.skip("positions outside the register")
    rng = np.random.default_rng(hash((positions, n)) % 2**32)
    U = random_unitary(1 << len(positions), rng)
    c = mq.QCircuit([mq.QuantumGate(positions, U), mq.HGate(1), mq.QuantumGate(positions[::-1], U.conj())])
    psi = random_state(n, rng)
    ref = O.apply(c.specs(), psi, n)
    for kw in ({"plain": True, "tensor": True}, {}):
        s = mq.StateVector(n)
        s.upload(psi)
        N.profile(True)
        mq.apply_(c, s, **kw)
        assert used(N, f"k_dmma_block{len(positions)}")
        N.profile(False)
        assert np.max(np.abs(s.to_numpy() - ref)) <= 1e-12, kw
    s = mq.StateVector(n)
    s.upload(psi)
    mq.apply_(c, s, plain=True)   # K0 gives the same answer
    assert np.max(np.abs(s.to_numpy() - ref)) <= 1e-12


def test_dense_block_batch_and_density(mq, O):
    from mossquantum_b200 import _native as N
    rng = np.random.default_rng(5)
    n, B = 12, 3
    U = random_unitary(32, rng)
    c = mq.QCircuit([mq.QuantumGate((2, 7, 4, 12, 1), U)])
    psis = [random_state(n, rng) for _ in range(B)]
    bs = mq.BatchStateVector(n, B)
    bs.upload(np.stack(psis, axis=1))      # storage is (2^n, B), one sample per column
    mq.apply_(c, bs, plain=True, tensor=True)
    out = bs.to_numpy()
    for b in range(B):
        assert np.max(np.abs(out[:, b] - O.apply(c.specs(), psis[b], n))) <= 1e-12
    # density matrix: U on rows, conj(U) on columns (6 qubits = 12 bits, two K5 launches)
    nd = 6
    U4 = random_unitary(16, rng)
    cd = mq.QCircuit([mq.QuantumGate((1, 3, 4, 6), U4), mq.QuantumGate((2, 3, 5, 6, 1), random_unitary(32, rng))])
    psi = random_state(nd, rng)
    rho = np.outer(psi, psi.conj())
    dm = mq.DensityMatrix(nd)
    dm.upload(rho)
    N.profile(True)
    mq.apply_(cd, dm, plain=True, tensor=True)
    assert used(N, "k_dmma_block4") and used(N, "k_dmma_block5")
    N.profile(False)
    ref = O.apply(cd.specs(), rho.reshape(-1, order="F"), nd, dm=True)
    assert np.max(np.abs(dm.to_numpy().reshape(-1, order="F") - ref)) <= 1e-12


def test_two_qubit_channel_supermatrix(mq, O):
    """A 2-qubit channel is a dense 16x16 supermatrix on 4 bits of the vectorised density matrix."""
    from mossquantum_b200 import _native as N
    rng = np.random.default_rng(8)
    n = 6
    ks = [random_unitary(4, rng) * np.sqrt(w) for w in (0.5, 0.3, 0.2)]
    ch = mq.QuantumMap((2, 5), ks, check_tp=True)
    c = mq.QCircuit([mq.HGate(2), mq.CNOTGate(2, 5), ch])
    dm = mq.DensityMatrix(n)
    N.profile(True)
    mq.apply_(c, dm, plain=True, tensor=True)
    assert used(N, "k_dmma_block4")
    N.profile(False)
    ref = O.apply(c.specs(), O.zero_state(n, True), n, dm=True)
    assert np.max(np.abs(dm.to_numpy().reshape(-1, order="F") - ref)) <= 1e-12


def test_fused_ansatz_blocks_on_tensor_cores(mq, O):
    from mossquantum_b200 import workloads as W
    from mossquantum_b200.fusion import fuse_gates
    n = 13
    u = W.u3_brickwork(n, 3, W.u3_params(n, 3, W.rng_for(6)))
    f = fuse_gates(u, max_qubits=5)
    ref = O.apply(u.specs(), O.zero_state(n), n)
    for kw in ({"plain": True, "tensor": True}, {"plain": True}, {}):
        s = mq.apply_(f, mq.StateVector(n), **kw)
        assert np.max(np.abs(s.to_numpy() - ref)) <= 1e-12, kw


@pytest.mark.parametrize("k", [4, 5])
def test_high_qubit_gates_match_operator_products(mq, O, k):
    """test/unit/high_qubit_gates.jl:1-46 on the device: the k-body gate
    from_external(positions, kron(m1..mk)) through K5 equals the operator product
    QubitsTerm(positions[j] => m_j) applied by the observable kernels (1e-12)."""
    rng = np.random.default_rng(60 + k)
    n = 12
    for order in [(2, 9, 4, 12, 7)[:k], (12, 7, 2, 9, 4)[:k], (9, 2, 12, 4, 7)[:k]]:
        ms = [random_unitary(2, rng) for _ in range(k)]
        ext = ms[0]
        for x in ms[1:]:
            ext = np.kron(ext, x)
        gate = mq.QCircuit([mq.QuantumGate(tuple(order), O.from_external(ext))])
        term = mq.QubitsOperator([mq.QubitsTerm(list(order), ms)])
        psi = random_state(n, rng)
        ref = O.apply_observable(psi, n, term.specs())
        for kw in ({"plain": True, "tensor": True}, {}, {"plain": True}):
            s = mq.StateVector(n)
            s.upload(psi)
            mq.apply_(gate, s, **kw)
            assert np.max(np.abs(s.to_numpy() - ref)) <= 1e-12, (order, kw)
        s = mq.StateVector(n)
        s.upload(psi)
        assert np.max(np.abs(mq.apply_observable(term, s).to_numpy() - ref)) <= 1e-12
