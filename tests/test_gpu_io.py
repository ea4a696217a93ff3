"""Checkpoint I/O and IonQ JSON circuits on the GPU.

Binary checkpoints restore the logical state bit for bit (both precisions);
JSON checkpoints round-trip within 1e-15 and read the reference's serde
layout; IonQ circuits run to the oracle's state within 1e-12 relative L2."""
import json
import os

import numpy as np
import pytest

import qoa_b200 as qb
from qoa_b200 import circuits as C
from qoa_b200 import ionq
from oracle import pyoracle as po


@pytest.mark.gpu
@pytest.mark.parametrize("precision,n", [("f64", 12), ("f32", 13), ("f64", 3)])
def test_binary_checkpoint_round_trip_exact(tmp_path, precision, n):
    with qb.QuantumState(n, precision=precision) as st:
        st.set_random_state(7)
        if n >= 11 or precision == "f64":
            st.execute(C.ops_to_array(C.random_layered(n, 3, 1)))
        path = str(tmp_path / "s.qoas")
        st.save(path)
        want = st.get_state_vector()
    with qb.QuantumState.load(path) as back:
        assert back.n == n and back.precision == precision
        got = back.get_state_vector()
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_binary_checkpoint_continues_a_noisy_trajectory(tmp_path):
    # the checkpoint carries the generator state: a loaded handle draws the
    # same noise and measurement outcomes as the original would have
    n = 10
    first = C.ops_to_array(C.random_layered(n, 3, 5, initial_h=True))
    rest = C.ops_to_array(C.random_layered(n, 4, 6))
    path = str(tmp_path / "noisy.qoas")

    def finish(st):
        st.execute(rest)
        outs = [st.measure(q) for q in range(n)]
        return outs, st.get_state_vector(), st.get_status()

    with qb.QuantumState(n, qb.NoiseConfig.Fixed(0.02), seed=99) as st:
        st.execute(first)
        st.save(path)
        want = finish(st)
    with qb.QuantumState.load(path) as back:
        assert back.get_noise_config().kind == "fixed"
        got = finish(back)
    assert got[0] == want[0]
    assert np.array_equal(got[1], want[1])
    assert got[2] == want[2]


@pytest.mark.gpu
def test_binary_checkpoint_detects_corruption(tmp_path):
    path = str(tmp_path / "s.qoas")
    with qb.QuantumState(6) as st:
        st.apply_h(0)
        st.save(path)
    raw = bytearray(open(path, "rb").read())
    raw[40] ^= 0x01
    open(path, "wb").write(bytes(raw))
    with pytest.raises(qb.QoaError):
        qb.QuantumState.load(path)
    open(path, "wb").write(bytes(raw[:50]))
    with pytest.raises(qb.QoaError):
        qb.QuantumState.load(path)


@pytest.mark.gpu
def test_json_checkpoint_round_trip(tmp_path):
    n = 9
    path = str(tmp_path / "s.json")
    with qb.QuantumState(n, noise_config=qb.NoiseConfig.Fixed(0.125)) as st:
        st.set_noise_config(None)
        st.execute(C.ops_to_array(C.random_layered(n, 4, 3)))
        st.set_noise_config(qb.NoiseConfig.Fixed(0.125))
        want = st.get_state_vector()
        st.save_json(path, [1.5, -2.0, 0.0])
    d = json.load(open(path))
    assert d[0]["n"] == n and len(d[0]["amps"]) == 1 << n and d[0]["noise_config"] == {"Fixed": 0.125}
    assert len(d[0]["regs"]) == 10 and d[1] == [1.5, -2.0, 0.0]
    back, regs = qb.QuantumState.load_json(path)
    with back:
        got = back.get_state_vector()
        assert back.noise_config.kind == "fixed" and back.noise_config.p == 0.125
    assert list(regs) == [1.5, -2.0, 0.0]
    assert np.max(np.abs(got - want)) < 1e-15


@pytest.mark.gpu
@pytest.mark.parametrize("cfg,text", [(None, None), ("ideal", "Ideal")])
def test_json_checkpoint_keeps_none_ideal_status_and_state_registers(tmp_path, cfg, text):
    # what a save / load / save cycle through the reference's serde layout
    # keeps: null against "Ideal", the status flags and the state's own
    # registers as they were loaded
    path, path2 = str(tmp_path / "a.json"), str(tmp_path / "b.json")
    with qb.QuantumState(3, None if cfg is None else qb.NoiseConfig.Ideal()) as st:
        st.apply_h(0)
        st.save_json(path)
    d = json.load(open(path))
    assert d[0]["noise_config"] == text
    d[0]["status"] = {"nan": False, "div_by_zero": True, "overflow": True}
    d[0]["regs"] = [[0.5, -1.0], [2.0, 0.0], [0.0, 3.0]]
    json.dump(d, open(path, "w"))
    back, _ = qb.QuantumState.load_json(path)
    with back:
        back.save_json(path2)
    e = json.load(open(path2))
    assert e[0]["noise_config"] == text
    assert e[0]["status"] == {"nan": False, "div_by_zero": True, "overflow": True}
    assert e[0]["regs"] == [[0.5, -1.0], [2.0, 0.0], [0.0, 3.0]]


@pytest.mark.gpu
def test_json_checkpoint_reads_serde_pretty_layout(tmp_path):
    # the layout serde_json::to_string_pretty writes for (QuantumState, regs)
    text = """[
  {
    "n": 1,
    "amps": [
      [
        0.7071067811865476,
        0.0
      ],
      [
        0.0,
        -0.7071067811865476
      ]
    ],
    "regs": [
      [
        0.0,
        0.0
      ]
    ],
    "status": {
      "nan": false,
      "div_by_zero": false,
      "overflow": false
    },
    "noise_config": "Random"
  },
  [
    3.0,
    1e-17
  ]
]"""
    path = str(tmp_path / "ref.json")
    open(path, "w").write(text)
    st, regs = qb.QuantumState.load_json(path)
    with st:
        v = st.get_state_vector()
        assert st.noise_config.kind == "random"
    assert np.allclose(v, [2 ** -0.5, -1j * 2 ** -0.5], atol=1e-15, rtol=0)
    assert list(regs) == [3.0, 1e-17]


@pytest.mark.gpu
def test_ionq_job_matches_oracle():
    from tests.test_ionq import JOB
    n, ops, _ = ionq.load_array(JOB)
    with qb.QuantumState(n) as st:
        st.execute(ops)
        got = st.get_state_vector()
    po.set_fast(True)
    o = po.OracleState(n, 0)
    o.apply(ops)
    ref = o.state()
    o.close()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12


@pytest.mark.gpu
def test_ionq_job_through_server():
    from tests.test_ionq import JOB
    n, ops, job = ionq.load_array(JOB)
    with qb.Server("f64", hbm_budget_gb=1, workers=2) as srv:
        rid = srv.submit(n, ops, 0.0, 1, job["shots"], 11)
        res = srv.poll(timeout_ms=60000)
        shots = srv.take_shots(rid, job["shots"])
    assert res[0]["status"] == 0 and len(shots) == job["shots"] and shots.max() < (1 << n)
