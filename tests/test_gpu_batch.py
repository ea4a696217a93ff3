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
