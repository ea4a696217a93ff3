"""FP32-fused precision form: complex64 state in both of its forms, the fused
tile passes (default) and dense blocks of up to 5 qubits on the tensor cores
(3xTF32, FP32 accumulation, QOA_FLAG_F32_TENSOR). Checked against the FP64
oracle (relative L2 and infidelity) and, for the QFT, against sqrt(N) * IDFT."""
import math

import numpy as np
import pytest

import qoa_b200 as qb
from qoa_b200 import circuits as C
from oracle import pyoracle as po
from tests.test_plan import mixed_circuit

F32_REL_L2 = 1e-5      # FP32 arithmetic over a few fused passes
F32_INFIDELITY = 1e-6  # 1 - |<psi_ref|psi>|^2


def fidelity_err(a, b):
    a = a.astype(np.complex128) / np.linalg.norm(a)
    b = b.astype(np.complex128) / np.linalg.norm(b)
    return 1.0 - abs(np.vdot(b, a)) ** 2


def rel_l2(a, b):
    return float(np.linalg.norm(a.astype(np.complex128) - b) / np.linalg.norm(b))


def f32_run(n, ops, init=None, tensor=False):
    with qb.QuantumState(n, precision="f32", f32_tensor=tensor) as st:
        if init is not None:
            st.set_state_vector(init.astype(np.complex64))
        st.execute(C.ops_to_array(ops))
        return st.get_state_vector()


def oracle_run(n, ops, init=None):
    po.set_fast(True)
    o = po.OracleState(n, 0)
    if init is not None:
        o.set_state(init)
    o.apply(C.ops_to_array(ops))
    return o.state()


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return v / np.linalg.norm(v)


@pytest.mark.gpu
@pytest.mark.parametrize("tensor", [False, True])
@pytest.mark.parametrize("n", [11, 12, 14, 17])
def test_f32_layered_matches_oracle(n, tensor):
    ops = C.random_layered(n, 6, 300 + n, initial_h=True)
    got, ref = f32_run(n, ops, tensor=tensor), oracle_run(n, ops)
    assert got.dtype == np.complex64
    assert rel_l2(got, ref) < F32_REL_L2
    assert fidelity_err(got, ref) < F32_INFIDELITY


@pytest.mark.gpu
@pytest.mark.parametrize("tensor", [False, True])
@pytest.mark.parametrize("n", [12, 15])
def test_f32_mixed_gate_kinds(n, tensor):
    ops = mixed_circuit(n, 150, 11 * n)
    got, ref = f32_run(n, ops, tensor=tensor), oracle_run(n, ops)
    assert rel_l2(got, ref) < F32_REL_L2


@pytest.mark.gpu
@pytest.mark.parametrize("tensor", [False, True])
@pytest.mark.parametrize("n", [11, 14, 18])
def test_f32_qft_matches_inverse_dft(n, tensor):
    init = random_state(n, 4)
    got = f32_run(n, C.qft(n), init=init, tensor=tensor)
    ref = np.fft.ifft(init) * math.sqrt(1 << n)
    assert rel_l2(got, ref) < F32_REL_L2
    assert fidelity_err(got, ref) < F32_INFIDELITY


@pytest.mark.gpu
def test_f32_rejects_non_unitary_ops_and_small_n():
    with pytest.raises(qb.QoaError):
        qb.QuantumState(8, precision="f32", f32_tensor=True)
    for tensor in (False, True):
        with qb.QuantumState(12, precision="f32", f32_tensor=tensor) as st:
            with pytest.raises(qb.QoaError):
                st.execute(C.ops_to_array([C.Op(C.MEASURE, [0])]))


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 4, 9])
def test_f32_small_states_run_per_gate(n):
    ops = mixed_circuit(n, 60, 5 * n) if n >= 3 else C.random_layered(n, 5, 2)
    got, ref = f32_run(n, ops), oracle_run(n, ops)
    assert rel_l2(got, ref) < F32_REL_L2


@pytest.mark.gpu
def test_random_state_and_compare():
    n = 14
    with qb.QuantumState(n) as a, qb.QuantumState(n, precision="f32") as b, qb.QuantumState(n) as c:
        a.set_random_state(7)
        b.set_random_state(7)
        c.set_random_state(8)
        va = a.get_state_vector()
        assert abs(np.linalg.norm(va) - 1) < 1e-12
        # near-Gaussian amplitudes: E|a|^2 = 1/N per amplitude
        assert 0.9 < np.mean(np.abs(va) ** 2) * (1 << n) < 1.1
        r, f = b.compare(a)
        assert r < 1e-6 and abs(f) < 1e-12
        r2, f2 = a.compare(c)
        assert r2 > 1.0 and f2 > 0.9
        r3, f3 = a.compare(a)
        assert r3 == 0.0 and abs(f3) < 1e-14


@pytest.mark.gpu
def test_f32_expect_z_and_sampling():
    n = 13
    ops = C.random_layered(n, 4, 77, initial_h=True)
    ref = oracle_run(n, ops)
    p = np.abs(ref) ** 2
    idx = np.arange(1 << n)
    masks = [1, 0b101, (1 << n) - 1, 1 << 12]
    want = [float(np.sum(np.where(np.array([bin(i & m).count("1") & 1 for i in idx]) == 1, -p, p))) for m in masks]
    with qb.QuantumState(n, precision="f32") as st:
        st.execute(C.ops_to_array(ops))
        got = st.expect_z(masks)
        shots = st.sample(20000, None, mode=1, rng_seed=3)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-5)
    hist = np.bincount((shots & 7).astype(np.int64), minlength=8) / len(shots)
    exp8 = np.array([p[(idx & 7) == k].sum() for k in range(8)])
    assert np.max(np.abs(hist - exp8)) < 0.02
