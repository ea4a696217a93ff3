"""Parity on the plans the 30-qubit headline runs: the pass scheduler's slot
search (taken by every state of 26 or more qubits) makes deeper passes with
more exchanges than the in-order greedy used below 26 qubits.

- Forced slot search (QOA_FLAG_SLOT_SEARCH) at 16-22 qubits, through both the
  generated pass kernels and the interpreter: generated == interpreter bit for
  bit, both within 1e-12 relative L2 of the oracle.
- The layered workload itself (H on every qubit, then random layers; the
  reference's CZ / CPHASE masks) at 26 and 28 qubits, unforced, against the
  oracle (fast mode, per-gate normalize deferred to the end).
- The full headline circuit at 30 qubits (16 GiB) against the oracle is a
  `slow` test (minutes of CPU), run when QOA_SLOW_TESTS=1.

The reference path these replace: src/vectorization.rs:915-1260 with the
per-gate normalize of src/runtime/quantum_state.rs:888-907.
"""
import os

import numpy as np
import pytest

import qoa_b200 as qb
from qoa_b200 import circuits as C
from oracle import pyoracle as po

TOL = 1e-12
QUIRK = qb.QOA_FLAG_COMPAT_MASK_QUIRK


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def oracle_state(n, ops, flags, defer=False):
    po.set_fast(True)
    st = po.OracleState(n, flags)
    if defer:
        st.defer_norm()
    st.apply(ops)
    if defer:
        st.normalize()
    s = st.state()
    st.close()
    return s


def engine_state(n, ops, jit, slot_search, quirk=True):
    with qb.QuantumState(n, compat_mask_quirk=quirk, slot_search=slot_search) as st:
        st.set_jit(jit, min_qubits=11)
        st.execute(ops)
        got = st.get_state_vector()
        assert st.get_status()["copy_timeouts"] == 0
        return got, st.jit_stats()


FORCED = [(16, 12, 31), (18, 12, 32), (20, 14, 33), (22, 16, 34)]


@pytest.mark.parametrize("n,depth,seed", FORCED)
def test_forced_search_makes_other_plans(n, depth, seed):
    # host only: the forced plans are the searched ones, not the greedy
    ops = C.ops_to_array(C.random_layered(n, depth, seed, initial_h=True))
    greedy = qb.plan(n, ops, QUIRK)
    searched = qb.plan(n, ops, QUIRK | qb.QOA_PLAN_SLOT_SEARCH)
    assert searched["npasses"] < greedy["npasses"]


@pytest.mark.gpu
@pytest.mark.parametrize("n,depth,seed", FORCED)
def test_forced_search_generated_and_interpreted_match_oracle(n, depth, seed):
    ops = C.ops_to_array(C.random_layered(n, depth, seed, initial_h=True))
    got_jit, st_jit = engine_state(n, ops, qb.QOA_JIT_SYNC, True)
    got_int, st_int = engine_state(n, ops, qb.QOA_JIT_OFF, True)
    assert st_jit["launches"] > 0 and st_jit["failures"] == 0 and st_int["launches"] == 0
    assert np.array_equal(got_jit.view(np.float64), got_int.view(np.float64)), "generated != interpreter"
    ref = oracle_state(n, ops, QUIRK)
    assert rel_l2(got_jit, ref) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("n,depth", [(26, 20), (28, 6)])
def test_layered_workload_unforced_matches_oracle(n, depth):
    ops = C.ops_to_array(C.layered_h_workload(n, depth, 1))
    got, stats = engine_state(n, ops, qb.QOA_JIT_SYNC, False)
    assert stats["launches"] > 0
    ref = oracle_state(n, ops, QUIRK, defer=True)
    err = rel_l2(got, ref)
    del got, ref
    assert err < TOL


@pytest.mark.gpu
@pytest.mark.slow
@pytest.mark.skipif(os.environ.get("QOA_SLOW_TESTS") != "1", reason="minutes of CPU: set QOA_SLOW_TESTS=1")
def test_headline_30_qubits_matches_oracle():
    n = 30
    ops = C.ops_to_array(C.layered_h_workload(n, 20, 1))
    got, stats = engine_state(n, ops, qb.QOA_JIT_SYNC, False)
    assert stats["launches"] > 0
    ref = oracle_state(n, ops, QUIRK, defer=True)
    err = rel_l2(got, ref)
    print(f"n=30 headline circuit: rel L2 vs oracle {err:.3e}")
    del got, ref
    assert err < TOL
