"""Pins the CPU oracle to the reference's own known-answer tests (src/test.rs)."""
import numpy as np
import pytest

from oracle import pyoracle as po
from tests.kat_util import case_ops, check_case, cvec, load_cases

VEC = load_cases("vec")
INSTR = load_cases("instr")


@pytest.mark.parametrize("case", VEC, ids=[c["name"] for c in VEC])
def test_vec_kat(case):
    a = cvec(case["init"]).copy()
    po.vec_call(case["fn"], a, *case["args"])
    check_case(case, a)


@pytest.mark.parametrize("quirk", [0, 1])
@pytest.mark.parametrize("case", INSTR, ids=[c["name"] for c in INSTR])
def test_instr_kat(case, quirk):
    st = po.OracleState(case["n"], quirk)
    if case.get("init"):
        st.set_state(cvec(case["init"]))
    st.apply(case_ops(case), meas_u=np.full(8, 0.5))
    check_case(case, st.state())


def test_every_case_cites_the_reference():
    for c in VEC + INSTR:
        assert c["src"] and c["src"].startswith("src/test.rs:"), c["name"]
