"""Batching form: many variational circuits of uneven size in one batch.

Every circuit's <Z_mask> results are checked against the oracle's final state
(FP64: 1e-12 absolute; FP32: 1e-5), the graph replay against the eager first
run, and a circuit's result alone against the same circuit inside a mix."""
import numpy as np
import pytest

import qoa_b200 as qb
from qoa_b200 import circuits as C
from oracle import pyoracle as po

F64_TOL = 1e-12
F32_TOL = 1e-5


def oracle_expz(n, ops, masks):
    po.set_fast(True)
    o = po.OracleState(n, 0)
    o.apply(C.ops_to_array(ops))
    a = o.state()
    p = (a.real ** 2 + a.imag ** 2)
    p = p / p.sum()
    idx = np.arange(1 << n, dtype=np.uint64)
    out = []
    for m in masks:
        par = np.zeros(1 << n, dtype=np.uint8)
        x = idx & np.uint64(m)
        while x.any():
            par ^= (x & np.uint64(1)).astype(np.uint8)
            x >>= np.uint64(1)
        out.append(float(np.sum(np.where(par == 1, -p, p))))
    return np.array(out)


def run_batch(circs, precision, **tuning):
    with qb.Batch(precision) as b:
        if tuning:
            b.set_tuning(**tuning)
        for c in circs:
            b.add(c["n"], c["ops"], c["masks"])
        b.run()  # eager
        first = b.results()
        b.run()  # captured into a graph, then launched
        second = b.results()
        b.run()  # graph replay
        third = b.results()
        info = b.info()
    assert np.array_equal(second, third)
    return first, second, info


def expected(circs):
    return np.concatenate([oracle_expz(c["n"], c["ops"], c["masks"]) for c in circs])


@pytest.fixture(scope="module")
def circs():
    # sizes on both sides of the shared-memory limit, and of the tile size
    return C.variational_batch(count=24, nmin=6, nmax=16, lmin=1, lmax=4, nmasks=8, seed=11)


@pytest.fixture(scope="module")
def ref(circs):
    return expected(circs)


@pytest.mark.gpu
def test_batch_f64_matches_oracle(circs, ref):
    first, second, info = run_batch(circs, "f64")
    assert info["small"] > 0 and info["large"] > 0 and info["graph_ready"] == 1
    np.testing.assert_allclose(first, ref, rtol=0, atol=F64_TOL)
    assert np.array_equal(first, second)


@pytest.mark.gpu
@pytest.mark.parametrize("tensor", [0, 1])
def test_batch_f32_matches_oracle(circs, ref, tensor):
    first, second, info = run_batch(circs, "f32", f32_tensor=tensor)
    assert info["small"] > 0 and info["large"] > 0
    np.testing.assert_allclose(first, ref, rtol=0, atol=F32_TOL)
    assert np.array_equal(first, second)


@pytest.mark.gpu
@pytest.mark.parametrize("tuning", [dict(small_max_n=0), dict(streams=1, small_threads=128),
                                    dict(small_ctas_per_sm=1, small_threads=512, pass_gate_budget=8)])
def test_batch_tunings_agree(circs, ref, tuning):
    first, _, _ = run_batch(circs, "f64", **tuning)
    np.testing.assert_allclose(first, ref, rtol=0, atol=F64_TOL)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_batch_alone_equals_in_mix(circs, precision):
    mixed, _, _ = run_batch(circs, precision)
    off = 0
    for c in circs[::5]:
        k = circs.index(c)
        start = sum(len(x["masks"]) for x in circs[:k])
        alone, _, _ = run_batch([c], precision)
        assert np.array_equal(alone, mixed[start:start + len(c["masks"])])
        off += 1
    assert off > 0


@pytest.mark.gpu
def test_batch_layered_gates_and_empty():
    rng_circs = []
    for n, seed in ((5, 1), (9, 2), (13, 3)):
        rng_circs.append({"n": n, "ops": C.random_layered(n, 3, seed), "masks": [1, (1 << n) - 1, 0b101]})
    rng_circs.append({"n": 7, "ops": [], "masks": [0b11, 0]})
    rng_circs.append({"n": 12, "ops": [], "masks": [0b11]})
    # a SWAP is a per-gate step in complex128: that circuit takes the view route
    rng_circs.append({"n": 13, "ops": C.random_layered(13, 2, 4) + [C.Op(C.SWAP, [0, 12])] + C.random_layered(13, 1, 5),
                      "masks": [1, 1 << 12, 0b1000000000011]})
    rng_circs.append({"n": 14, "ops": [], "masks": [1]})
    ref = expected(rng_circs)
    for prec, tol in (("f64", F64_TOL), ("f32", F32_TOL)):
        first, second, info = run_batch(rng_circs, prec)
        np.testing.assert_allclose(first, ref, rtol=0, atol=tol)
        assert np.array_equal(first, second)


@pytest.mark.gpu
def test_batch_rejects_measurement():
    with qb.Batch("f64") as b:
        with pytest.raises(qb.QoaError):
            b.add(4, [C.Op(C.MEASURE, [0])], [1])


@pytest.mark.gpu
def test_autotune_picks_a_valid_tuning(tmp_path, circs, ref):
    from qoa_b200 import autotune
    cache = str(tmp_path / "tune.json")
    best = autotune.tune(circs, "f64", sample=12, cache=cache, budget_s=20)
    assert set(best) >= {"small_max_n", "small_threads", "small_ctas_per_sm", "pass_gate_budget"}
    assert autotune.tune(circs, "f64", sample=12, cache=cache) == best     # served from the cache
    first, _, _ = run_batch(circs, "f64", **best)
    np.testing.assert_allclose(first, ref, rtol=0, atol=F64_TOL)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_batch_generated_arena_kernels(circs, ref, precision):
    """Arena passes as generated kernels (one per pass structure, compiled
    before the first run) give the interpreter's results bit for bit, and the
    oracle's within tolerance; the graph launches the generated kernels."""
    big = [c for c in circs if c["n"] >= 11] + C.variational_batch(count=6, nmin=13, nmax=15, lmin=2, lmax=3,
                                                                    nmasks=4, seed=12)
    with qb.Batch(precision) as b:
        b.set_tuning(jit=qb.QOA_JIT_SYNC, small_max_n=10, f32_tensor=0)
        for c in big:
            b.add(c["n"], c["ops"], c["masks"])
        b.run()
        gen = b.results()
        b.run()
        b.run()
        info = b.jit_info()
        again = b.results()
    with qb.Batch(precision) as b:
        b.set_tuning(jit=qb.QOA_JIT_OFF, small_max_n=10, f32_tensor=0)
        for c in big:
            b.add(c["n"], c["ops"], c["masks"])
        b.run()
        interp = b.results()
    assert info["structures"] > 0 and info["ready"] == info["structures"]
    assert info["graph_uses_generated"]
    assert np.array_equal(gen, interp)
    assert np.array_equal(gen, again)
    exp = expected(big)
    tol = F64_TOL if precision == "f64" else F32_TOL
    assert np.max(np.abs(gen - exp)) < tol


@pytest.mark.gpu
def test_batch_graph_recaptured_when_kernels_arrive(circs):
    # each structure repeated ten times: shared enough for the default mode
    big = [c for c in circs if c["n"] >= 11] * 10
    with qb.Batch("f64") as b:
        b.set_tuning(jit=qb.QOA_JIT_ASYNC, small_max_n=10)
        for c in big:
            b.add(c["n"], c["ops"], c["masks"])
        b.run()
        first = b.results()
        b.run()
        qb.jit_wait()
        b.launch()          # replays, capturing again with the generated kernels
        replay = b.results()
        assert b.jit_info()["graph_uses_generated"]
    assert np.array_equal(first, replay)
