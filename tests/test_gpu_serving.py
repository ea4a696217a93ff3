"""Serving form: noisy requests through the continuous-batching server.

Checked here: each trajectory's shots equal the oracle's noisy trajectory
sampled by the same inverse-CDF descent with the same counter-based uniforms;
a request's outcomes alone equal its outcomes in a mix of concurrent requests
(bit for bit, both precisions); admission respects the HBM budget; a request
larger than the budget is rejected with QOA_E_OOM."""
import numpy as np
import pytest

import qoa_b200 as qb
from qoa_b200 import circuits as C
from oracle import pyoracle as po


def inverse_cdf_descent(p, n, u):
    """The device's shot rule (k_sample mode 1): walk qubits 0..n-1, taking
    bit q = 0 while the remaining mass is below the marginal of that prefix."""
    idx = np.arange(1 << n)
    out = []
    for x in u:
        t = x * p.sum()
        pre = 0
        for q in range(n):
            sel = (idx & ((2 << q) - 1)) == pre
            left = p[sel].sum()
            if t < left:
                continue
            t -= left
            pre |= 1 << q
        out.append(pre)
    return np.array(out, dtype=np.uint64)


def requests(seed=0, count=8, nmin=5, nmax=15):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(rng.integers(nmin, nmax + 1))
        ops = C.ops_to_array(C.random_layered(n, int(rng.integers(2, 6)), 100 + k))
        out.append(dict(n=n, ops=ops, noise_p=0.02, trajectories=4, shots=8, seed=1000 + k))
    return out


def run(server, reqs):
    ids = [server.submit(r["n"], r["ops"], r["noise_p"], r["trajectories"], r["shots"], r["seed"]) for r in reqs]
    done = {}
    while len(done) < len(ids):
        for res in server.poll(timeout_ms=60000):
            assert res["status"] == 0, res
            done[res["id"]] = res
    return [server.take_shots(i, int(done[i]["shots"])) for i in ids], [done[i] for i in ids]


@pytest.mark.gpu
def test_trajectory_shots_match_oracle():
    n, p, seed, T, S = 7, 0.05, 4242, 3, 32
    ops = C.ops_to_array(C.random_layered(n, 4, 9))
    with qb.Server("f64", hbm_budget_gb=1, workers=2) as srv:
        (shots,), _ = run(srv, [dict(n=n, ops=ops, noise_p=p, trajectories=T, shots=S, seed=seed)])
    po.set_fast(True)
    for t in range(T):
        o = po.OracleState(n, 0)
        o.set_noise(1, p, seed, t)
        o.apply(ops)
        prob = np.abs(o.state()) ** 2
        u = [qb.philox_uniform(seed, t ^ qb.SHOT_STREAM, k, 0) for k in range(S)]
        ref = inverse_cdf_descent(prob / prob.sum(), n, u)
        assert np.array_equal(shots[t * S:(t + 1) * S], ref), t
        o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_alone_equals_in_mix(precision):
    reqs = requests(seed=1, count=8)
    with qb.Server(precision, hbm_budget_gb=4, workers=8) as srv:
        mixed, res = run(srv, reqs)
        st = srv.stats()
    assert st["done"] == len(reqs)
    if precision == "f32":
        assert any(r["precision"] == qb.QOA_PREC_F32 for r in res)
    with qb.Server(precision, hbm_budget_gb=4, workers=1) as srv:
        for k in (0, 3, 6):
            (alone,), _ = run(srv, [reqs[k]])
            assert np.array_equal(alone, mixed[k]), k


@pytest.mark.gpu
def test_admission_respects_budget():
    n = 16
    budget_gb = 3 * ((1 << n) * 24 + (1 << 20)) / (1 << 30)  # room for three states
    reqs = [dict(n=n, ops=C.ops_to_array(C.random_layered(n, 2, k)), noise_p=0.0, trajectories=3, shots=4,
                 seed=k) for k in range(5)]
    with qb.Server("f64", hbm_budget_gb=budget_gb, workers=8) as srv:
        _, res = run(srv, reqs)
        st = srv.stats()
    assert st["peak_bytes_reserved"] <= int(budget_gb * (1 << 30))
    assert st["states_resident"] <= 3
    for r in res:
        assert r["t_submit"] <= r["t_admit"] <= r["t_start"] <= r["t_done"]


@pytest.mark.gpu
def test_request_over_budget_is_rejected():
    with qb.Server("f64", hbm_budget_gb=0.001, workers=1) as srv:
        rid = srv.submit(20, C.ops_to_array(C.random_layered(20, 1, 0)), 0.0, 1, 1, 0)
        res = srv.poll(timeout_ms=60000)
        assert res and res[0]["id"] == rid and res[0]["status"] == qb.QOA_E_OOM
        with pytest.raises(qb.QoaError):
            srv.take_shots(rid, 1)


def state_path_shots(n, ops, p, seed, t, u, precision):
    """One trajectory the way the server runs it on a pooled state handle."""
    with qb.QuantumState(n, precision=precision) as st:
        st.seed_rng(seed)
        st.set_noise_config(qb.NoiseConfig.Fixed(p) if p > 0 else None)
        st.set_trajectory(t)
        st.apply_reset_all()
        st.execute(ops)
        return st.sample(len(u), u=u, mode=1)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("n", [6, 12, 14, 16])
def test_batch_trajectories_match_state_path(precision, n):
    # trajectories as batch circuits (shared-memory route for small n, arena
    # tile passes above) give the shots of the per-state path: the same noise
    # draws, the same inverse-CDF rule
    p, seed, S = 0.03, 777 + n, 24
    ops = C.ops_to_array(C.random_layered(n, 5, 300 + n))
    b = qb.Batch(precision)
    ids, us = [], []
    for t in range(4):
        u = np.array([qb.philox_uniform(seed, t ^ qb.SHOT_STREAM, k, 0) for k in range(S)])
        us.append(u)
        ids.append(b.add_trajectory(n, ops, seed, p, t, u))
    b.run()
    for t in range(4):
        got = b.shots(ids[t])
        ref = state_path_shots(n, ops, p, seed, t, us[t], precision)
        assert np.array_equal(got, ref), (t, got, ref)
    # reuse after reset: a noiseless circuit sampled with many uniforms
    b.reset()
    u = np.array([qb.philox_uniform(seed, 5 ^ qb.SHOT_STREAM, k, 0) for k in range(3 * S)])
    cid = b.add_trajectory(n, ops, seed, 0.0, 0, u)
    b.run()
    assert np.array_equal(b.shots(cid), state_path_shots(n, ops, 0.0, seed, 0, u, precision))


@pytest.mark.gpu
def test_server_runs_trajectory_chunks_and_per_state_fallback():
    reqs = requests(seed=3, count=4, nmin=8, nmax=16)
    meas = dict(n=6, ops=C.ops_to_array([C.Op(C.H, [0]), C.Op(C.CNOT, [0, 1]), C.Op(C.MEASURE, [0]),
                                         C.Op(C.H, [2])]),
                noise_p=0.01, trajectories=3, shots=5, seed=99)
    with qb.Server("f64", hbm_budget_gb=4, workers=4) as srv:
        shots, res = run(srv, reqs + [meas])
        st = srv.stats()
    # the unitary requests ran as batch chunks, the measuring one per state
    assert st["trajectories_batched"] == sum(r["trajectories"] for r in reqs)
    for r, got in zip(reqs, shots):
        for t in (0, r["trajectories"] - 1):
            u = np.array([qb.philox_uniform(r["seed"], t ^ qb.SHOT_STREAM, k, 0) for k in range(r["shots"])])
            ref = state_path_shots(r["n"], r["ops"], r["noise_p"], r["seed"], t, u, "f64")
            assert np.array_equal(got[t * r["shots"]:(t + 1) * r["shots"]], ref)
    assert res[-1]["status"] == 0 and len(shots[-1]) == 15
