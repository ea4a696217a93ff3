"""Depolarising-noise trajectories (apply_noise / apply_depolarizing_noise,
src/runtime/quantum_state.rs:839-885): after every gate, for every qubit,
r < p inserts X / Y / Z. Draws come from Philox4x32-10 keyed (seed,
trajectory, event, slot) on both sides, so the engine and the oracle follow
the same trajectory and must agree to 1e-12."""
import numpy as np
import pytest

import qoa_b200 as qb
from qoa_b200 import circuits as C
from oracle import pyoracle as po


def run_pair(n, ops, mode, p, seed, traj, flags):
    arr = C.ops_to_array(ops)
    o = po.OracleState(n, flags)
    o.set_noise(mode, p, seed, traj)
    o.apply(arr)
    cfg = {0: qb.NoiseConfig.Ideal(), 1: qb.NoiseConfig.Fixed(p), 2: qb.NoiseConfig.Random()}[mode]
    with qb.QuantumState(n, cfg, compat_mask_quirk=bool(flags & 1),
                         noise_gate_qubits_only=bool(flags & qb.QOA_FLAG_NOISE_GATE_QUBITS), seed=seed) as e:
        e.set_trajectory(traj)
        e.execute(arr)
        return e.get_state_vector(), o.state()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [6, 13])
@pytest.mark.parametrize("p", [0.02, 0.2])
def test_fixed_noise_trajectory_matches_oracle(n, p):
    ops = C.random_layered(n, 4, 50 + n, initial_h=True)
    got, ref = run_pair(n, ops, 1, p, seed=1234, traj=3, flags=1)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12


@pytest.mark.gpu
def test_random_noise_level_matches_oracle():
    ops = C.random_layered(12, 3, 9, initial_h=True)
    got, ref = run_pair(12, ops, 2, 0.0, seed=77, traj=0, flags=1)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12


@pytest.mark.gpu
def test_noise_on_gate_qubits_only_matches_oracle():
    ops = C.random_layered(13, 4, 3, initial_h=True)
    got, ref = run_pair(13, ops, 1, 0.1, seed=5, traj=1, flags=1 | qb.QOA_FLAG_NOISE_GATE_QUBITS)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12


@pytest.mark.gpu
def test_trajectories_are_independent_and_reproducible():
    n, ops = 12, C.random_layered(12, 4, 8, initial_h=True)
    a, _ = run_pair(n, ops, 1, 0.1, 9, 0, 1)
    b, _ = run_pair(n, ops, 1, 0.1, 9, 0, 1)
    c, _ = run_pair(n, ops, 1, 0.1, 9, 1, 1)
    assert np.array_equal(a, b)
    assert np.linalg.norm(a - c) > 1e-3
