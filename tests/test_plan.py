"""Host pass scheduler (no GPU): every gate lands in exactly one step, and
replaying the chosen order reproduces the oracle's state, so every reordering
the scheduler made was between commuting gates."""
import math

import numpy as np
import pytest

import qoa_b200 as qb
from qoa_b200 import circuits as C
from oracle import pyoracle as po
from tests.plan_emulator import replay

QOA_PLAN_SLOT_SEARCH = 0x100


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def oracle_state(n, ops, flags):
    po.set_fast(True)
    st = po.OracleState(n, flags)
    st.apply(C.ops_to_array(ops))
    return st.state()


def mixed_circuit(n, count, seed):
    """Every gate kind the engine takes, controls anywhere in the index."""
    rng = C.SplitMix64(seed)
    ops = []
    kinds = [C.H, C.X, C.Y, C.Z, C.T, C.S, C.P, C.RX, C.RY, C.RZ, C.CNOT, C.CZ, C.CPHASE, C.SWAP, C.CSWAP,
             C.TOFFOLI, C.CY, C.U1, C.U2, C.EBELL, C.ECLUSTER]
    for _ in range(count):
        g = kinds[rng.below(len(kinds))]
        qs = []
        while len(qs) < 3:
            q = rng.below(n)
            if q not in qs:
                qs.append(q)
        a = rng.uniform() * 2 * math.pi
        if g in (C.H, C.X, C.Y, C.Z, C.T, C.S, C.P, C.RX, C.RY, C.RZ):
            ops.append(C.Op(g, qs[:1], a))
        elif g in (C.CNOT, C.CZ, C.CPHASE, C.SWAP, C.CY, C.EBELL):
            ops.append(C.Op(g, qs[:2], a))
        elif g in (C.CSWAP, C.TOFFOLI, C.ECLUSTER):
            ops.append(C.Op(g, qs, a))
        elif g == C.U1:
            th, ph, la = rng.uniform() * 3, rng.uniform() * 6, rng.uniform() * 6
            u = np.array([[math.cos(th), -np.exp(1j * la) * math.sin(th)],
                          [np.exp(1j * ph) * math.sin(th), np.exp(1j * (ph + la)) * math.cos(th)]])
            ops.append(C.Op(g, qs[:1], 0.0, u.reshape(-1)))
        else:
            z = np.array([rng.uniform() - 0.5 + 1j * (rng.uniform() - 0.5) for _ in range(16)]).reshape(4, 4)
            q, _ = np.linalg.qr(z)
            ops.append(C.Op(g, qs[:2], 0.0, q.reshape(-1)))
    return ops


CASES = [
    ("layered_h_12x4", 12, lambda: C.random_layered(12, 4, 11, initial_h=True)),
    ("layered_14x6", 14, lambda: C.random_layered(14, 6, 12)),
    ("layered_16x3", 16, lambda: C.random_layered(16, 3, 13, initial_h=True)),
    ("qft_13", 13, lambda: C.qft(13)),
    ("mixed_13", 13, lambda: mixed_circuit(13, 160, 14)),
    ("mixed_15", 15, lambda: mixed_circuit(15, 120, 15)),
]


@pytest.mark.parametrize("search", [0, 1])
@pytest.mark.parametrize("quirk", [0, 1])
@pytest.mark.parametrize("name,n,make", CASES, ids=[c[0] for c in CASES])
def test_plan_replay_matches_oracle(name, n, make, quirk, search):
    """search=1: the slot search (used from 26 qubits on) forced at this size."""
    ops = make()
    flags = (qb.QOA_FLAG_COMPAT_MASK_QUIRK if quirk else 0) | (QOA_PLAN_SLOT_SEARCH if search else 0)
    plan = qb.plan(n, C.ops_to_array(ops), flags)
    assert plan["npasses"] >= 1
    # each expanded gate is in exactly one step, at a distinct slot
    keys = set(zip(plan["pass_of"].tolist(), plan["order"].tolist()))
    assert len(keys) == len(plan["pass_of"])
    got = replay(n, plan)
    ref = oracle_state(n, ops, flags)
    assert rel_l2(got, ref) < 1e-12, rel_l2(got, ref)


def test_layered_30_pass_count():
    """The 930-gate 30-qubit workload packs into far fewer sweeps than gates;
    the slot search (on at this size) packs it into 13."""
    ops = C.layered_h_workload()
    plan = qb.plan(30, C.ops_to_array(ops), qb.QOA_FLAG_COMPAT_MASK_QUIRK)
    assert len(plan["pass_of"]) == 930
    assert plan["npasses"] <= 14


def test_per_gate_flag_gives_one_step_per_gate():
    ops = C.random_layered(14, 2, 3)
    plan = qb.plan(14, C.ops_to_array(ops), qb.QOA_FLAG_PER_GATE)
    assert plan["npasses"] == len(plan["pass_of"]) == C.gate_count(ops)


def test_out_of_range_ops_are_dropped_from_the_plan():
    ops = [C.Op(C.H, [0]), C.Op(C.H, [40]), C.Op(C.CNOT, [1, 1]), C.Op(C.CZ, [0, 12]), C.Op(C.X, [3])]
    plan = qb.plan(12, C.ops_to_array(ops), 0)
    assert len(plan["pass_of"]) == 2
