"""Measurement: outcomes bit-exact against the oracle for the same supplied
uniforms, and shot histograms against exact probabilities (chi-square)."""
import math

import numpy as np
import pytest

import qoa_b200 as qb
from qoa_b200 import circuits as C
from oracle import pyoracle as po


def prepared(n, seed, quirk=True):
    ops = C.ops_to_array(C.random_layered(n, 4, seed, initial_h=False))
    flags = qb.QOA_FLAG_COMPAT_MASK_QUIRK if quirk else 0
    o = po.OracleState(n, flags)
    o.apply(ops)
    e = qb.QuantumState(n, compat_mask_quirk=quirk)
    e.execute(ops)
    return o, e


@pytest.mark.gpu
@pytest.mark.parametrize("n", [3, 10, 13])
def test_measure_sequence_bit_exact(n):
    o, e = prepared(n, 21 + n)
    rng = np.random.default_rng(n)
    for k in range(2 * n):
        q = int(rng.integers(n))
        u = float(rng.random())
        assert e.measure(q, u) == o.measure(q, u)
        # a few gates between measurements
        ops = C.ops_to_array([C.Op(C.H, [q]), C.Op(C.RY, [(q + 1) % n], 0.4 * k)])
        o.apply(ops)
        e.execute(ops)
    got, ref = e.get_state_vector(), o.state()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12
    e.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 4, 11, 14])
def test_sample_mode0_matches_measure_all(n):
    o, e = prepared(n, 40 + n)
    shots = 256
    u = np.random.default_rng(7).random(shots * n)
    got = e.sample(shots, u, mode=0)
    ref = [o.measure_all(u[s * n:(s + 1) * n]) for s in range(shots)]
    assert [int(x) for x in got] == ref
    e.close()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
def test_shot_histogram_chi_square(mode):
    from scipy.stats import chisquare
    n = 12
    o, e = prepared(n, 77)
    p = np.abs(o.state()) ** 2
    shots = 200_000
    bits = e.sample(shots, None, mode=mode, rng_seed=mode + 1)
    # bin by the low 5 qubits: 32 bins with ample expected counts
    b = (bits & 31).astype(np.int64)
    obs = np.bincount(b, minlength=32)
    exp = np.array([p[np.arange(1 << n) & 31 == k].sum() for k in range(32)]) * shots
    keep = exp > 5
    stat, pval = chisquare(obs[keep], exp[keep] * obs[keep].sum() / exp[keep].sum())
    assert pval > 1e-4, (stat, pval)
    e.close()


@pytest.mark.gpu
def test_probabilities_and_expectations():
    n = 13
    o, e = prepared(n, 5)
    p_ref = np.abs(o.state()) ** 2
    assert np.max(np.abs(e.get_probabilities() - p_ref)) < 1e-14
    masks = [1, 3, 0b1010101, (1 << n) - 1, 0, 1 << 12, 0b110011001100, 7]
    idx = np.arange(1 << n)
    for m, got in zip(masks, e.expect_z(masks)):
        par = np.array([bin(int(i) & m).count("1") & 1 for i in idx])
        ref = float(np.sum(np.where(par, -p_ref, p_ref)))
        assert abs(got - ref) < 1e-12
    e.close()


@pytest.mark.gpu
def test_measure_out_of_range_raises():
    with qb.QuantumState(4) as e:
        with pytest.raises(qb.QoaError):
            e.measure(4, 0.5)


@pytest.mark.gpu
def test_measure_op_inside_apply_uses_seeded_stream():
    n = 12
    ops = C.ops_to_array([C.Op(C.H, [q]) for q in range(n)] + [C.Op(C.MEASURE, [q]) for q in range(0, n, 3)])
    outs = []
    for _ in range(2):
        with qb.QuantumState(n, seed=99) as e:
            e.execute(ops)
            outs.append(e.get_state_vector())
    assert np.array_equal(outs[0], outs[1])
    # the oracle with the same Philox stream (seed 99, stream 0) agrees
    o = po.OracleState(n, 0)
    o.set_noise(0, 0.0, 99, 0)
    o.apply(ops)
    assert np.linalg.norm(outs[0] - o.state()) < 1e-12
