"""Bytecode front-end on the GPU: the reference's example programs (assembled
from their .qoa sources by this repository's assembler) run through qoa_exe_run on a complex128 state, compared with the oracle
applying the same instruction stream with the same measurement uniforms
(the handle's seeded stream): final amplitudes within 1e-12 relative L2,
and every measurement outcome identical (the collapse would differ otherwise).
"""
import json
import os

import numpy as np
import pytest

import qoa_b200 as qb
from qoa_b200 import qexe
from oracle import pyoracle as po

HERE = os.path.dirname(os.path.abspath(__file__))
PROGRAMS = json.load(open(os.path.join(HERE, "golden", "qexe_programs.json")))
MEAS_STREAM = 0x6D656173


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["teleport", "shor", "aes-decryption-16", "fusion-sim", "hello_world"])
def test_reference_program_matches_oracle(name):
    f = bytes.fromhex(PROGRAMS[name]["hex"])
    n = max(qexe.parse(f)["inferred_qubits"], 1)
    seed = 1234
    ops, tres, tout = qexe.trace(f)
    with qb.QuantumState(n, seed=seed) as st:
        res, out = qexe.run(st, f)
        got = st.get_state_vector()
    assert res["gates"] == tres["gates"] and res["measurements"] == tres["measurements"]
    assert out == tout
    po.set_fast(True)
    o = po.OracleState(n, 0)
    u = [qb.philox_uniform(seed, MEAS_STREAM, k, 0) for k in range(int(tres["measurements"]))]
    o.apply(ops, meas_u=u)
    ref = o.state()
    o.close()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12


@pytest.mark.gpu
def test_charout_prints_measured_bits():
    # X 0, CHAROUT 0 (prints chr(1)), CHAROUT 1 (prints chr(0)), HALT
    f = qexe.write_exe(bytes([0x07, 0, 0x18, 0, 0x18, 1, 0xFF]))
    with qb.QuantumState(2, seed=5) as st:
        res, out = qexe.run(st, f)
    assert out == b"\x01\x00" and res["chars_out"] == 2
