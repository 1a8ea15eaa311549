"""Expectations, observable action and readout on the GPU vs the oracle.

Mirrors test/regression/kernels.jl:45-94 (4/5-site and non-Hermitian expectations, H*rho)
and src/execution/probabilities.jl semantics (marginals, normalisation, sampling).
Tolerances: 1e-11 on expectations, 1e-12 on probabilities and amplitudes.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def random_state(n, rng):
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def random_operator(mq, n, rng, hermitian=False):
    names = ["X", "Y", "Z", "+", "-", "I", "u", "d"] if not hermitian else ["X", "Y", "Z", "I"]
    terms = []
    for k in (0, 1, 2, 3, 4, 5):
        for _ in range(3):
            pos = [int(x) for x in rng.choice(np.arange(1, n + 1), size=k, replace=False)]
            ops = [names[rng.integers(len(names))] for _ in range(k)]
            c = complex(rng.normal(), 0 if hermitian else rng.normal())
            terms.append(mq.QubitsTerm(pos, ops, c))
    return mq.QubitsOperator(terms)


@pytest.mark.parametrize("n", [6, 11])
def test_expectation_pure(mq, O, n):
    rng = np.random.default_rng(n)
    psi = random_state(n, rng)
    s = mq.StateVector(psi)
    for herm in (True, False):
        H = random_operator(mq, n, rng, herm)
        assert abs(mq.expectation(H, s) - O.expect(psi, n, H.specs())) <= 1e-11


def test_expectation_density(mq, O):
    n = 5
    rng = np.random.default_rng(1)
    a = rng.normal(size=(32, 32)) + 1j * rng.normal(size=(32, 32))
    rho = a @ a.conj().T
    rho /= np.trace(rho)
    s = mq.DensityMatrix(rho)
    for herm in (True, False):
        H = random_operator(mq, n, rng, herm)
        assert abs(mq.expectation(H, s) - np.trace(H.matrix(n) @ rho)) <= 1e-11


def test_known_expectations(mq):
    s = mq.StateVector(4)
    assert mq.expectation(mq.QubitsTerm([1, 2, 3, 4], ["Z"] * 4, 2.0), s) == pytest.approx(2.0)
    assert mq.expectation(mq.QubitsTerm([], [], 2.5), s) == pytest.approx(2.5)
    d = mq.DensityMatrix(4)
    assert mq.expectation(mq.QubitsTerm([1, 2, 3, 4], ["Z"] * 4, 2.0), d) == pytest.approx(2.0)


def test_observable_action(mq, O):
    n = 7
    rng = np.random.default_rng(2)
    psi = random_state(n, rng)
    H = random_operator(mq, n, rng, False)
    out = mq.apply_observable(H, mq.StateVector(psi)).to_numpy()
    np.testing.assert_allclose(out, O.apply_observable(psi, n, H.specs()), atol=1e-12)


@pytest.mark.parametrize("n", [10, 13])
def test_pauli_passes_expectation_and_action(mq, O, n):
    """From 10 qubits on, expectations and H psi run as Pauli-string passes over shared-memory
    tiles (Hermitian flip groups summed over pairs j, j^x; others over every amplitude);
    strings with flips on up to five bits above the lanes, and Z strings inside, outside and
    across a tile's bits."""
    rng = np.random.default_rng(100 + n)
    psi = random_state(n, rng)
    s = mq.StateVector(psi)
    for herm in (True, False):
        H = random_operator(mq, n, rng, herm)
        assert abs(mq.expectation(H, s) - O.expect(psi, n, H.specs())) <= 1e-11
        out = mq.apply_observable(H, mq.StateVector(psi)).to_numpy()
        np.testing.assert_allclose(out, O.apply_observable(psi, n, H.specs()), atol=1e-12)
    # one Hermitian term with a complex coefficient pair: X1 Y7 Z13-type strings and their sum
    # with a non-Hermitian partner in the same flip group
    terms = [mq.QubitsTerm([1, 7, n], ["X", "Y", "Z"], 0.7), mq.QubitsTerm([1, 7], ["X", "X"], 0.3),
             mq.QubitsTerm([1, 7, 4], ["Y", "X", "Z"], 0.2j)]
    H = mq.QubitsOperator(terms)
    assert abs(mq.expectation(H, s) - O.expect(psi, n, H.specs())) <= 1e-11


def test_probabilities(mq, O):
    n = 9
    rng = np.random.default_rng(3)
    psi = random_state(n, rng)
    s = mq.StateVector(psi)
    for qubits in ([1, 2, 3], [9, 2], [5], list(range(1, 10)), [3, 1, 7, 9, 2, 4, 5, 6, 8]):
        np.testing.assert_allclose(mq.probabilities(s, qubits), O.probabilities(psi, n, qubits), atol=1e-12)
    bell = mq.apply_(mq.QCircuit([mq.HGate(1), mq.CNOTGate(1, 2)]), mq.StateVector(2))
    np.testing.assert_allclose(mq.probabilities(bell), [0.5, 0, 0, 0.5], atol=1e-15)
    d = mq.DensityMatrix(mq.StateVector(psi))
    np.testing.assert_allclose(mq.probabilities(d, [2, 5]), O.probabilities(psi, n, [2, 5]), atol=1e-12)


def test_probabilities_validation(mq):
    s = mq.StateVector(np.array([1.0, 1.0, 0, 0]))
    with pytest.raises(ValueError):
        mq.probabilities(s)
    with pytest.raises(ValueError):
        mq.probabilities(mq.StateVector(3), [1, 1])
    with pytest.raises(ValueError):
        mq.probabilities(mq.StateVector(3), [4])


def test_sampling_matches_oracle_rng(mq, O):
    n = 6
    psi = random_state(n, np.random.default_rng(4))
    s = mq.StateVector(psi)
    a = mq.sample(np.random.default_rng(99), s, 500, qubits=[2, 4, 6])
    b = O.sample(np.random.default_rng(99), O.probabilities(psi, n, [2, 4, 6]), 500)
    assert np.array_equal(a, b)
    c = mq.counts(np.random.default_rng(99), s, 500, qubits=[2, 4, 6])
    assert sum(c.values()) == 500


def test_pauli_pass_matches_dense_keys(mq, O):
    """The fused Pauli-string kernel and the per-key dense kernel agree with the oracle."""
    import os
    from mossquantum_b200 import workloads as W
    rng = np.random.default_rng(77)
    for n in (10, 13, 17):
        psi = random_state(n, rng)
        s = mq.StateVector(psi)
        for H in (W.tfim(n), W.xxz(n), random_operator(mq, n, rng, False)):
            ref = O.expect(psi, n, H.specs())
            fused = mq.expectation(H, s)
            os.environ["MB_EXPECT_KEYS"] = "1"
            try:
                keys = mq.expectation(H, s)
            finally:
                del os.environ["MB_EXPECT_KEYS"]
            assert abs(fused - ref) <= 1e-11 and abs(keys - ref) <= 1e-11
    # batch of states through the fused kernel
    B, n = 3, 11
    cols = rng.normal(size=(1 << n, B)) + 1j * rng.normal(size=(1 << n, B))
    cols /= np.linalg.norm(cols, axis=0)
    ev = mq.expectation(W.xxz(n), mq.BatchStateVector(cols))
    for b in range(B):
        assert abs(ev[b] - O.expect(cols[:, b], n, W.xxz(n).specs())) <= 1e-11


def few_terms(mq, n, rng):
    """A handful of 1..3-site terms (Y, ladder and projector operators, complex coefficients:
    non-Hermitian flip groups) on sites spread over the register, few enough for the
    specialised Pauli passes."""
    names = ["X", "Y", "Z", "+", "-", "u", "d"]
    terms = []
    for k in (1, 2, 2, 3):
        pos = [int(x) for x in rng.choice(np.arange(1, n + 1), size=k, replace=False)]
        ops = [names[rng.integers(len(names))] for _ in range(k)]
        terms.append(mq.QubitsTerm(pos, ops, complex(rng.normal(), rng.normal())))
    return mq.QubitsOperator(terms)


@pytest.mark.parametrize("jit_from", [10, 99])
def test_specialised_pauli_passes(mq, O, monkeypatch, jit_from):
    """Expectations through the specialised Pauli passes (strings' masks compiled in, per-thread
    class factors; jit_from=10) and through the interpreter kernel (jit_from=99) agree with the
    oracle for TFIM, XXZ and random operators (Y strings, complex coefficients, non-Hermitian
    groups, strings straddling the tile bits), on single states and batches."""
    from mossquantum_b200 import _native as N
    from mossquantum_b200 import workloads as W
    monkeypatch.setenv("MB_PAULI_JIT_MIN_BITS", str(jit_from))
    rng = np.random.default_rng(5 + jit_from)
    N.profile(True)
    try:
        for n in (10, 13, 16):
            psi = random_state(n, rng)
            s = mq.StateVector(psi)
            for H in (W.tfim(n), W.xxz(n), random_operator(mq, n, rng, False), random_operator(mq, n, rng, True),
                      few_terms(mq, n, rng)):
                ref = O.expect(psi, n, H.specs())
                assert abs(mq.expectation(H, s) - ref) <= 1e-11, (n, jit_from)
        B, n = 4, 14
        cols = rng.normal(size=(1 << n, B)) + 1j * rng.normal(size=(1 << n, B))
        cols /= np.linalg.norm(cols, axis=0)
        H = few_terms(mq, n, rng)
        ev = mq.expectation(H, mq.BatchStateVector(cols))
        for b in range(B):
            assert abs(ev[b] - O.expect(cols[:, b], n, H.specs())) <= 1e-11
        N.synchronize()
        rep = N.profile_report()
    finally:
        N.profile(False)
    assert ("mbk_pauli" in rep) == (jit_from == 10), rep
