"""The reference's known-answer tests through the engine's C ABI on the GPU:
vectorization.rs-level cases through the qoa_vec_* shims, instruction-level
cases through qoa_apply on a handle (both CZ-mask modes)."""
import numpy as np
import pytest

import qoa_b200 as qb
from tests.kat_util import case_ops, check_case, cvec, load_cases

VEC = load_cases("vec")
INSTR = load_cases("instr")


@pytest.mark.gpu
@pytest.mark.parametrize("case", VEC, ids=[c["name"] for c in VEC])
def test_vec_kat_gpu(case):
    a = cvec(case["init"]).copy()
    qb.vec_call(case["fn"], a, *case["args"])
    check_case(case, a)


@pytest.mark.gpu
@pytest.mark.parametrize("per_gate", [False, True])
@pytest.mark.parametrize("quirk", [False, True])
@pytest.mark.parametrize("case", INSTR, ids=[c["name"] for c in INSTR])
def test_instr_kat_gpu(case, quirk, per_gate):
    with qb.QuantumState(case["n"], compat_mask_quirk=quirk, per_gate=per_gate) as st:
        if case.get("init"):
            st.set_state_vector(cvec(case["init"]))
        st.execute(case_ops(case))
        check_case(case, st.get_state_vector())
