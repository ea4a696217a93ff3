"""Engine vs oracle on seeded circuits: relative L2 <= 1e-12 (FP64)."""
import math

import numpy as np
import pytest

import qoa_b200 as qb
from qoa_b200 import circuits as C
from oracle import pyoracle as po
from tests.test_plan import mixed_circuit

TOL = 1e-12


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def oracle_run(n, ops, flags, init=None):
    po.set_fast(True)
    st = po.OracleState(n, flags)
    if init is not None:
        st.set_state(init)
    st.apply(C.ops_to_array(ops))
    return st.state()


def engine_run(n, ops, quirk, per_gate=False, init=None):
    with qb.QuantumState(n, compat_mask_quirk=quirk, per_gate=per_gate) as st:
        if init is not None:
            st.set_state_vector(init)
        st.execute(C.ops_to_array(ops))
        return st.get_state_vector()


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return v / np.linalg.norm(v)


@pytest.mark.gpu
@pytest.mark.parametrize("quirk", [True, False])
@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 11, 12, 13, 14, 16])
def test_layered_small(n, quirk):
    ops = C.random_layered(n, 6, 100 + n, initial_h=True)
    flags = qb.QOA_FLAG_COMPAT_MASK_QUIRK if quirk else 0
    ref = oracle_run(n, ops, flags)
    got = engine_run(n, ops, quirk)
    assert rel_l2(got, ref) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("per_gate", [False, True])
@pytest.mark.parametrize("n", [12, 13, 15])
def test_mixed_gate_kinds(n, per_gate):
    ops = mixed_circuit(n, 150, 7 * n)
    ref = oracle_run(n, ops, 0)
    got = engine_run(n, ops, False, per_gate=per_gate)
    assert rel_l2(got, ref) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("n", [12, 14])
def test_every_gate_on_every_qubit(n):
    """Each 1-qubit kind on each position, and each 2-qubit kind on every
    ordered pair, from a random start state: covers lane, register, warp and
    outer placements of targets, controls and phase masks in the tile pass."""
    init = random_state(n, n)
    ops = []
    for q in range(n):
        for g in (C.H, C.X, C.Y, C.Z, C.T, C.S, C.P, C.RX, C.RY, C.RZ):
            ops.append(C.Op(g, [q], 0.3 + 0.1 * q))
    for c in range(n):
        for t in range(n):
            if c != t:
                g = (C.CNOT, C.CZ, C.CPHASE, C.CY)[(c + t) % 4]
                ops.append(C.Op(g, [c, t], 0.7 + 0.01 * c))
    for quirk in (False, True):
        flags = qb.QOA_FLAG_COMPAT_MASK_QUIRK if quirk else 0
        ref = oracle_run(n, ops, flags, init)
        got = engine_run(n, ops, quirk, init=init)
        assert rel_l2(got, ref) < TOL


@pytest.mark.gpu
def test_layered_workload_n20_depth40():
    """The 20-qubit, depth-40, 1200-gate layered circuit against the oracle."""
    ops = C.layered_workload()
    ref = oracle_run(20, ops, qb.QOA_FLAG_COMPAT_MASK_QUIRK)
    got = engine_run(20, ops, True)
    assert rel_l2(got, ref) < TOL


@pytest.mark.gpu
def test_layered_h_workload_at_n24():
    """The 30-qubit workload's structure (H layer + 20 layers) at n=24."""
    ops = C.random_layered(24, 20, 1, initial_h=True)
    ref = oracle_run(24, ops, qb.QOA_FLAG_COMPAT_MASK_QUIRK)
    got = engine_run(24, ops, True)
    assert rel_l2(got, ref) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("n", [5, 12, 16])
def test_qft_matches_inverse_dft(n):
    """QFT (physical CPHASE) on a random state equals sqrt(N) * IDFT."""
    init = random_state(n, 3)
    got = engine_run(n, C.qft(n), False, init=init)
    ref = np.fft.ifft(init) * math.sqrt(1 << n)
    assert rel_l2(got, ref) < TOL


@pytest.mark.gpu
def test_per_gate_and_pass_paths_agree():
    ops = C.random_layered(18, 8, 5, initial_h=True)
    a = engine_run(18, ops, True, per_gate=True)
    b = engine_run(18, ops, True, per_gate=False)
    assert rel_l2(a, b) < TOL


@pytest.mark.gpu
def test_round_trip_circuit_then_inverse():
    """Size-independent property: U followed by U^dagger restores |0..0>."""
    n = 22
    fwd = C.random_layered(n, 5, 9, initial_h=True)
    inv = []
    for op in reversed(fwd):
        g, a = op.opcode, op.angle
        if g in (C.H, C.X, C.CNOT, C.CZ):
            inv.append(C.Op(g, op.qubits))
        elif g in (C.RX, C.RY, C.RZ, C.P, C.CPHASE):
            inv.append(C.Op(g, op.qubits, -a))
        elif g == C.T:
            inv.append(C.Op(C.P, op.qubits, -math.pi / 4))
        elif g == C.S:
            inv.append(C.Op(C.P, op.qubits, -math.pi / 2))
    got = engine_run(n, fwd + inv, False)
    assert abs(got[0] - 1.0) < 1e-11
    assert np.linalg.norm(got[1:]) < 1e-11


@pytest.mark.gpu
def test_out_of_range_is_skipped_like_the_reference():
    ops = [C.Op(C.H, [0]), C.Op(C.H, [99]), C.Op(C.CNOT, [0, 0]), C.Op(C.CNOT, [0, 1])]
    with qb.QuantumState(13) as st:
        rc = st.execute(C.ops_to_array(ops))
        assert rc == qb.QOA_E_RANGE
        v = st.get_state_vector()
    ref = oracle_run(13, ops, 0)
    assert rel_l2(v, ref) < TOL


@pytest.mark.gpu
def test_zero_and_nan_states_reset_like_normalize():
    with qb.QuantumState(12) as st:
        st.set_state_vector(np.zeros(1 << 12, dtype=np.complex128))
        v = st.get_state_vector()
        assert v[0] == 1 and np.count_nonzero(v) == 1
        bad = np.full(1 << 12, np.nan, dtype=np.complex128)
        st.set_state_vector(bad)
        st.apply_h(0)
        v = st.get_state_vector()
        assert abs(v[0] - 1 / math.sqrt(2)) < 1e-15 and abs(v[1] - 1 / math.sqrt(2)) < 1e-15
        assert st.get_status()["zero_norm_resets"] >= 2


@pytest.mark.gpu
def test_qinit_recreates_state():
    ops = [C.Op(C.H, [0]), C.Op(C.QINIT, [13]), C.Op(C.H, [12])]
    with qb.QuantumState(3) as st:
        st.execute(C.ops_to_array(ops))
        assert st.n == 13
        v = st.get_state_vector()
    assert abs(v[0] - 1 / math.sqrt(2)) < 1e-15 and abs(v[1 << 12] - 1 / math.sqrt(2)) < 1e-15


def swap_heavy(n, count, seed):
    """SWAPs interleaved with 1-qubit gates, controlled X and phases on the
    swapped qubits (tile passes take SWAPs as relabellings of tile bits)."""
    rng = np.random.default_rng(seed)
    ops = [C.Op(C.H, [q]) for q in range(n)]
    for _ in range(count):
        a, b = (int(x) for x in rng.choice(n, 2, replace=False))
        k = int(rng.integers(6))
        if k < 2:
            ops.append(C.Op(C.SWAP, [a, b]))
        elif k == 2:
            ops.append(C.Op(C.RX, [a], float(rng.uniform(0, 2 * math.pi))))
        elif k == 3:
            ops.append(C.Op(C.CNOT, [a, b]))
        elif k == 4:
            ops.append(C.Op(C.CPHASE, [a, b], float(rng.uniform(0, 2 * math.pi))))
        else:
            ops.append(C.Op(C.T, [a]))
    return ops


@pytest.mark.gpu
@pytest.mark.parametrize("n", [11, 13, 16])
def test_swaps_inside_passes(n):
    ops = swap_heavy(n, 40 * n, n)
    ref = oracle_run(n, ops, 0)
    assert rel_l2(engine_run(n, ops, False), ref) < TOL
    with qb.QuantumState(n, precision="f32") as st:
        st.execute(C.ops_to_array(ops))
        got = st.get_state_vector().astype(np.complex128)
    assert rel_l2(got, ref) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("n", [4, 7, 12, 17])
def test_swap_blocks_as_permutations(n):
    """Runs of >= 3 disjoint SWAPs run as one in-place permutation pass."""
    rng = np.random.default_rng(n)
    ops = [C.Op(C.H, [q]) for q in range(n)] + [C.Op(C.T, [q]) for q in range(0, n, 2)]
    for rep in range(3):
        perm = [int(x) for x in rng.permutation(n)]
        for k in range(0, n - 1, 2):
            ops.append(C.Op(C.SWAP, [perm[k], perm[k + 1]]))
        ops += [C.Op(C.RY, [int(rng.integers(n))], 0.3 + rep), C.Op(C.CNOT, [0, n - 1])]
    ref = oracle_run(n, ops, 0)
    assert rel_l2(engine_run(n, ops, False), ref) < TOL
    with qb.QuantumState(n, precision="f32") as st:
        st.execute(C.ops_to_array(ops))
        got = st.get_state_vector().astype(np.complex128)
    assert rel_l2(got, ref) < 1e-5
