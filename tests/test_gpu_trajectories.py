"""Kraus trajectories on the device (noisy_execution.jl:1-334).

1. Exact replay: trajectories re-run on the host with the oracle, the same per-trajectory
   generators and the reference's branch rules give the same final states (1e-12).
2. Ensemble: the average of psi psi' over many trajectories estimates the density matrix of
   exact Kraus evolution; <H> agrees within 5 standard errors of the trajectory mean.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def noisy_circuit(mq, W, n, layers):
    c = W.hea_circuit(n, layers, W.hea_angles(n, layers, W.rng_for(11)), active=False, noise=(0.05, 0.1))
    return c


def discrete_sample(rng, weights):
    """Inverse-CDF draw (sampling.jl:3-18), restated for the replay."""
    w = np.asarray(weights, dtype=float)
    threshold = rng.random() * float(np.sum(w))
    cumulative, last_positive = 0.0, 0
    for i, x in enumerate(w):
        if x > 0:
            last_positive = i
        cumulative += x
        if threshold < cumulative:
            return i
    return last_positive


def replay(mq, O, circ, n, seed):
    """One trajectory on the host, from the oracle's own Kraus matrices: a channel whose
    operators all satisfy K_j'K_j = p_j I (a mixture) draws p_j and applies K_j/sqrt(p_j);
    any other channel draws with weights ||K_j psi||^2 and applies K_j
    (noisy_execution.jl:1-334); the state is normalised at the end."""
    gen = np.random.default_rng(int(seed))
    psi = O.zero_state(n)
    for spec in circ.specs():
        if spec[0] != "channel":
            psi = O.apply([spec], psi, n)
            continue
        _, name, positions, params, _, data = spec
        assert len(positions) == 1
        ks = O.kraus_matrices(name, params, data, 1)
        pos0 = [positions[0] - 1]
        p = [np.trace(k.conj().T @ k).real / 2 for k in ks]
        if all(np.allclose(k.conj().T @ k, pk * np.eye(2), atol=1e-14) for k, pk in zip(ks, p)):
            keep = [j for j, pk in enumerate(p) if pk > 0]
            j = keep[discrete_sample(gen, [p[i] for i in keep])]
            psi = O.apply_matrix(psi, pos0, ks[j] / np.sqrt(p[j]))
        else:
            cands = [O.apply_matrix(psi, pos0, k) for k in ks]
            j = discrete_sample(gen, [np.vdot(c, c).real for c in cands])
            psi = cands[j]
    return psi / np.linalg.norm(psi)


def test_trajectories_replay_exactly(mq, O):
    from mossquantum_b200 import workloads as W
    from mossquantum_b200.trajectories import run_trajectories
    n = 6
    circ = noisy_circuit(mq, W, n, 2)
    seeds = [11, 22, 33, 44]
    state, choices, _ = run_trajectories(circ, mq.StateVector(n), len(seeds), seeds=seeds)
    out = state.to_numpy()
    for t, s in enumerate(seeds):
        ref = replay(mq, O, circ, n, s)
        assert np.max(np.abs(out[:, t] - ref)) <= 1e-12, t


def test_trajectory_ensemble_matches_density_evolution(mq, O):
    from mossquantum_b200 import workloads as W
    from mossquantum_b200.trajectories import run_trajectories
    n, T = 5, 2048
    circ = noisy_circuit(mq, W, n, 2)
    H = W.tfim(n)
    state, _, _ = run_trajectories(circ, mq.StateVector(n), T, rng=np.random.default_rng(5))
    vals = np.real(mq.expectation(H, state))
    rho = O.apply(circ.specs(), O.zero_state(n, True), n, dm=True)
    exact = O.expect(rho, n, H.specs(), dm=True).real
    se = vals.std(ddof=1) / np.sqrt(T)
    assert abs(vals.mean() - exact) <= 5 * se + 1e-12, (vals.mean(), exact, se)


def test_execute_counts(mq):
    from mossquantum_b200 import workloads as W
    n = 4
    circ = noisy_circuit(mq, W, n, 1)
    r1 = mq.execute(circ, mq.StateVector(n), shots=500, rng=np.random.default_rng(1), method=mq.KrausTrajectory())
    r2 = mq.execute(circ, mq.StateVector(n), shots=500, rng=np.random.default_rng(1), method=mq.KrausTrajectory())
    assert r1.counts == r2.counts and sum(r1.counts.values()) == 500
    rd = mq.execute(circ, mq.StateVector(n), shots=500, rng=np.random.default_rng(1))
    assert sum(rd.counts.values()) == 500
