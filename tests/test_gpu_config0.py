"""The reference-executor workload end to end: a 20-qubit random layered
circuit of depth 40 from |0..0> (the reference's CZ / CPHASE masks), then
1024 shots in measure_all order (src/runtime/quantum_state.rs:909-918: the
state is cloned and qubits 0..n-1 are measured in turn, one uniform each).

- amplitudes within 1e-12 relative L2 of the oracle;
- every shot bit-exact with the oracle's measure_all for the same supplied
  uniforms;
- all 1024 shots against the exact probabilities (chi-square over the 8
  outcomes of qubits 0..2).
"""
import numpy as np
import pytest

import qoa_b200 as qb
from qoa_b200 import circuits as C
from oracle import pyoracle as po

N, DEPTH, SEED, SHOTS = 20, 40, 0, 1024


@pytest.mark.gpu
def test_layered_20_qubits_depth_40_then_1024_shots():
    from scipy.stats import chisquare

    ops = C.ops_to_array(C.random_layered(N, DEPTH, SEED))
    assert len(ops) == DEPTH * (N + N // 2)
    u = np.random.default_rng(2020).random(SHOTS * N)
    with qb.QuantumState(N, compat_mask_quirk=True) as st:
        st.execute(ops)
        got = st.get_state_vector()
        shots = st.sample(SHOTS, u, mode=0)
        # sampling leaves the state as it was (measure_all works on a clone)
        assert np.array_equal(st.get_state_vector().view(np.float64), got.view(np.float64))

    po.set_fast(True)
    o = po.OracleState(N, qb.QOA_FLAG_COMPAT_MASK_QUIRK)
    o.apply(ops)
    ref = o.state()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12
    for s in range(SHOTS):
        assert int(shots[s]) == o.measure_all(u[s * N:(s + 1) * N]), f"shot {s}"
    o.close()

    p = np.abs(ref) ** 2
    exp = np.array([p[np.arange(1 << N) & 7 == k].sum() for k in range(8)]) * SHOTS
    obs = np.bincount((shots & 7).astype(np.int64), minlength=8)
    keep = exp > 5
    stat, pval = chisquare(obs[keep], exp[keep] * obs[keep].sum() / exp[keep].sum())
    assert pval > 1e-4, (stat, pval, obs, exp)
