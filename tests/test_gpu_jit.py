"""Generated (NVRTC-compiled) complex128 pass kernels against the
interpreter kernel and the oracle: the same PassParams must give the same
amplitudes bit for bit, and both must be within 1e-12 (relative L2) of the
oracle."""
import numpy as np
import pytest

import qoa_b200 as qb
from qoa_b200 import circuits as C
from oracle import pyoracle as po
from tests.test_plan import mixed_circuit
from tests.test_gpu_parity import swap_heavy

TOL = 1e-12


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def oracle_run(n, ops, flags):
    po.set_fast(True)
    st = po.OracleState(n, flags)
    st.apply(C.ops_to_array(ops))
    s = st.state()
    st.close()
    return s


def run(n, ops, jit, quirk=False, init_seed=None, precision="f64"):
    with qb.QuantumState(n, compat_mask_quirk=quirk, precision=precision) as st:
        st.set_jit(jit, min_qubits=11)
        if init_seed is not None:
            st.set_random_state(init_seed)
        st.execute(C.ops_to_array(ops))
        return st.get_state_vector(), st.jit_stats()


CASES = [
    ("layered_h_16x8_quirk", 16, True, lambda: C.random_layered(16, 8, 21, initial_h=True)),
    ("layered_18x10", 18, False, lambda: C.random_layered(18, 10, 22)),
    ("qft_17", 17, False, lambda: C.qft(17)),
    ("mixed_14", 14, False, lambda: mixed_circuit(14, 300, 23)),
    ("mixed_17", 17, True, lambda: mixed_circuit(17, 200, 24)),
    ("swaps_15", 15, False, lambda: swap_heavy(15, 600, 25)),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,n,quirk,make", CASES, ids=[c[0] for c in CASES])
def test_generated_passes_match_interpreter_and_oracle(name, n, quirk, make):
    ops = make()
    got_jit, st_jit = run(n, ops, qb.QOA_JIT_SYNC, quirk)
    got_int, st_int = run(n, ops, qb.QOA_JIT_OFF, quirk)
    assert st_jit["launches"] > 0, "the generated kernels did not run"
    assert st_jit["failures"] == 0
    assert st_int["launches"] == 0
    assert np.array_equal(got_jit.view(np.float64), got_int.view(np.float64)), "generated != interpreter"
    ref = oracle_run(n, ops, 1 if quirk else 0)
    assert rel_l2(got_jit, ref) < TOL


@pytest.mark.gpu
def test_generated_passes_from_a_random_state():
    n = 16
    ops = mixed_circuit(n, 150, 31)
    a, s = run(n, ops, qb.QOA_JIT_SYNC, init_seed=5)
    b, _ = run(n, ops, qb.QOA_JIT_OFF, init_seed=5)
    assert s["launches"] > 0
    assert np.array_equal(a.view(np.float64), b.view(np.float64))


@pytest.mark.gpu
def test_async_mode_switches_to_generated_kernels():
    n = 15
    ops = C.ops_to_array(C.random_layered(n, 6, 41, initial_h=True))
    with qb.QuantumState(n) as st:
        st.set_jit(qb.QOA_JIT_ASYNC, min_qubits=11)
        st.execute(ops)          # first sighting: interpreted, nothing compiled
        first = st.get_state_vector()
        assert st.jit_stats()["launches"] == 0
        st.apply_reset_all()
        st.execute(ops)          # second sighting: compiles in the background
        qb.jit_wait()
        st.apply_reset_all()
        st.execute(ops)          # generated kernels now
        third = st.get_state_vector()
        assert st.jit_stats()["launches"] > 0
    assert np.array_equal(first.view(np.float64), third.view(np.float64))


@pytest.mark.gpu
def test_same_structure_reuses_the_compiled_kernel():
    n = 14
    before = qb.jit_stats()
    outs = []
    for angle in (0.3, 1.1):   # same pass structure, other angle values
        ops = [C.Op(C.H, [q]) for q in range(n)] + [C.Op(C.RZ, [q], angle * (q + 1)) for q in range(n)] + \
              [C.Op(C.CPHASE, [q, (q + 5) % n], angle) for q in range(n)] + [C.Op(C.RY, [q], angle) for q in range(n)]
        got, _ = run(n, ops, qb.QOA_JIT_SYNC)
        assert rel_l2(got, oracle_run(n, ops, 0)) < TOL
        outs.append(got)
    after = qb.jit_stats()
    assert after["hits"] > before["hits"], "the second angle set compiled again"
    assert not np.allclose(outs[0], outs[1])


@pytest.mark.gpu
def test_measurement_between_passes_uses_generated_kernels():
    n = 16
    ops = C.random_layered(n, 4, 51, initial_h=True) + [C.Op(C.MEASURE, [3])] + C.random_layered(n, 4, 52)
    with qb.QuantumState(n, seed=9) as st:
        st.set_jit(qb.QOA_JIT_SYNC, min_qubits=11)
        st.execute(C.ops_to_array(ops))
        a = st.get_state_vector()
        assert st.jit_stats()["launches"] > 0
    with qb.QuantumState(n, seed=9) as st:
        st.set_jit(qb.QOA_JIT_OFF)
        st.execute(C.ops_to_array(ops))
        b = st.get_state_vector()
    assert np.array_equal(a.view(np.float64), b.view(np.float64))


@pytest.mark.gpu
@pytest.mark.parametrize("name,n,quirk,make", CASES, ids=[c[0] for c in CASES])
def test_generated_complex64_passes_match_interpreter(name, n, quirk, make):
    """The packed FP32 form: generated kernels against the packed interpreter
    (bit for bit) and against the FP64 oracle (relative L2 < 1e-5)."""
    ops = make()
    got_jit, st_jit = run(n, ops, qb.QOA_JIT_SYNC, quirk, precision="f32")
    got_int, st_int = run(n, ops, qb.QOA_JIT_OFF, quirk, precision="f32")
    assert st_jit["launches"] > 0 and st_jit["failures"] == 0
    assert st_int["launches"] == 0
    assert np.array_equal(got_jit.view(np.float32), got_int.view(np.float32)), "generated != interpreter"
    ref = oracle_run(n, ops, 1 if quirk else 0)
    assert rel_l2(got_jit.astype(np.complex128), ref) < 1e-5


@pytest.mark.gpu
def test_repeated_op_lists_reuse_their_plans():
    """An op list executed again reuses its kept plan (schedule, built passes,
    kernel texts); results stay bit-identical across repeats and another
    list in between does not disturb them."""
    n = 22
    a_ops = C.ops_to_array(C.random_layered(n, 3, 61, initial_h=True))
    b_ops = C.ops_to_array(C.qft(n))
    outs = []
    with qb.QuantumState(n, compat_mask_quirk=True) as st:
        for k in range(4):
            st.apply_reset_all()
            st.execute(a_ops)
            outs.append(st.get_state_vector())
            if k == 1:
                st.apply_reset_all()
                st.execute(b_ops)
            if k == 2:
                qb.jit_wait()
    for o in outs[1:]:
        assert np.array_equal(o.view(np.float64), outs[0].view(np.float64))
    ref = oracle_run(n, C.random_layered(n, 3, 61, initial_h=True), 1)
    assert rel_l2(outs[0], ref) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("grid", ["1", "3", "7"])
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_streamed_passes_with_many_tiles_per_cta(monkeypatch, grid, precision):
    # the streamed form of a generated pass (QOA_JIT_STREAM) is persistent:
    # each CTA walks tiles b, b + grid, ... with two shared-memory buffers
    # whose copies complete on alternating mbarrier phases; a capped grid
    # makes every CTA take many tiles (both buffers, both phases), still
    # bit-identical to the interpreter
    monkeypatch.setenv("QOA_JIT_STREAM_GRID", grid)
    monkeypatch.setenv("QOA_JIT_STREAM", "3")
    n = 17
    ops = C.random_layered(n, 6, 61, initial_h=True)
    got_jit, st_jit = run(n, ops, qb.QOA_JIT_SYNC, True, precision=precision)
    got_int, _ = run(n, ops, qb.QOA_JIT_OFF, True, precision=precision)
    assert st_jit["launches"] > 0 and st_jit["failures"] == 0
    assert np.array_equal(got_jit.view(np.float32 if precision == "f32" else np.float64),
                          got_int.view(np.float32 if precision == "f32" else np.float64))
    tol = 1e-5 if precision == "f32" else TOL
    assert rel_l2(got_jit.astype(np.complex128), oracle_run(n, ops, 1)) < tol
