"""Edge cases on the GPU: the smallest states in both precisions, empty op
lists, a state too large for the device (clean QOA_E_OOM), the tile-size
boundary (10/11/12 qubits), and op lists long enough to split passes."""
import numpy as np
import pytest

import qoa_b200 as qb
from qoa_b200 import circuits as C
from oracle import pyoracle as po


def oracle_state(n, ops):
    po.set_fast(True)
    o = po.OracleState(n, 0)
    o.apply(C.ops_to_array(ops))
    s = o.state()
    o.close()
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_one_qubit_states(precision):
    with qb.QuantumState(1, precision=precision) as st:
        st.apply_x(0)
        assert np.allclose(st.get_state_vector(), [0, 1])
        st.apply_h(0)
        assert np.allclose(st.get_state_vector(), [2 ** -0.5, -(2 ** -0.5)], atol=1e-7)
        st.apply_reset_all()
        assert np.allclose(st.get_state_vector(), [1, 0])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_empty_op_list_is_a_no_op(precision):
    with qb.QuantumState(12, precision=precision) as st:
        st.set_random_state(3)
        before = st.get_state_vector()
        st.execute(C.ops_to_array([]))
        after = st.get_state_vector()
        assert np.max(np.abs(after - before)) < (1e-15 if precision == "f64" else 1e-7)


@pytest.mark.gpu
def test_state_too_large_fails_cleanly():
    with pytest.raises(qb.QoaError) as e:
        qb.QuantumState(37)
    assert e.value.code in (qb.QOA_E_OOM, qb.QOA_E_CUDA, qb.QOA_E_ARG)
    with qb.QuantumState(3) as st:   # the device is still usable
        st.apply_h(0)
        assert abs(np.linalg.norm(st.get_state_vector()) - 1) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("n", [10, 11, 12])
def test_tile_size_boundary(n):
    ops = C.random_layered(n, 8, 50 + n, initial_h=True)
    ref = oracle_state(n, ops)
    with qb.QuantumState(n) as st:
        st.execute(C.ops_to_array(ops))
        assert np.linalg.norm(st.get_state_vector() - ref) / np.linalg.norm(ref) < 1e-12
    with qb.QuantumState(n, precision="f32") as st:
        st.execute(C.ops_to_array(ops))
        got = st.get_state_vector().astype(np.complex128)
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-5


@pytest.mark.gpu
def test_long_op_list_splits_passes():
    # thousands of gates on few tile qubits: the pass builder runs out of op
    # slots and splits (or falls back to per-gate kernels) without changing results
    n = 13
    rng = np.random.default_rng(1)
    ops = []
    for _ in range(3000):
        q = int(rng.integers(3))
        ops.append(C.Op([C.H, C.T, C.RX, C.S][int(rng.integers(4))], [q], float(rng.uniform(0, 6.3))))
        if rng.random() < 0.2:
            ops.append(C.Op(C.CPHASE, [q, int(rng.integers(3, n))], float(rng.uniform(0, 6.3))))
    ref = oracle_state(n, ops)
    with qb.QuantumState(n) as st:
        st.execute(C.ops_to_array(ops))
        assert np.linalg.norm(st.get_state_vector() - ref) / np.linalg.norm(ref) < 1e-11
