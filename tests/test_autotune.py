"""Batch autotuner, host side: candidate grid and workload signature."""
from qoa_b200 import autotune
from qoa_b200 import circuits as C


def test_candidates_cover_tile_and_fusion_choices():
    for prec, cap in (("f64", 12), ("f32", 13)):
        cands = autotune.candidates(prec)
        assert {c["small_max_n"] for c in cands} == {cap - 2, cap - 1, cap}
        assert {c["pass_gate_budget"] for c in cands} >= {0, 48, 96, 160}
        assert all(c["small_threads"] * c["small_ctas_per_sm"] <= 2048 for c in cands)
    assert any(c.get("f32_tensor") for c in autotune.candidates("f32"))
    assert not any(c.get("f32_tensor") for c in autotune.candidates("f64"))


def test_signature_tracks_size_mix():
    a = C.variational_batch(count=20, seed=1)
    b = C.variational_batch(count=20, seed=2)
    assert autotune.signature(a) == autotune.signature(list(a))
    assert autotune.signature(a) != autotune.signature(b)
