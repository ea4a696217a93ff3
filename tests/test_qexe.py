"""Bytecode front-end (host side): .qexe header parsing and qubit inference,
the run_exe interpreter traced without a GPU, and the assembler.

The reference's own compiled example programs (tests/golden/
reference_qexe.json, made by make_qexe_golden.py) must parse, run to HALT and
infer the qubit counts `qoa run` would; small programs of our own pin the
instruction semantics (jumps, registers, printing, the loop quirk)."""
import json
import os
import struct

import numpy as np
import pytest

import qoa_b200 as qb
from qoa_b200 import circuits as C
from qoa_b200 import qexe

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "reference_qexe.json")))


def prog(src: str, kind="qexe") -> bytes:
    payload, _ = qexe.assemble(src)
    return qexe.write_exe(payload, kind)


def ops_summary(ops):
    return [(int(o["opcode"]), tuple(int(x) for x in o["q"][:o["nq"]]), float(o["angle"])) for o in ops]


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_reference_binaries_parse_and_run_to_halt(name):
    f = bytes.fromhex(GOLDEN[name]["hex"])
    info = qexe.parse(f)
    assert info["kind"] in qexe.MAGIC and info["payload_offset"] == 9
    assert info["payload_len"] == len(f) - 9
    ops, res, out = qexe.trace(f)
    assert res["halted"] == 1 and res["unknown_opcodes"] == 0 and res["loop_errors"] == 0
    assert res["gates"] + res["measurements"] == len(ops)
    # every qubit the program touches lies below the inferred count
    qmax = max((int(o["q"][k]) for o in ops for k in range(o["nq"])), default=-1)
    assert qmax < max(info["inferred_qubits"], 1)


def test_reference_hello_prints():
    ops, res, out = qexe.trace(bytes.fromhex(GOLDEN["hello.qx"]["hex"]))
    assert out == b"Hello, World!\n" and len(ops) == 0 and res["halted"] == 1


def test_reference_qubit_inference():
    got = {k: qexe.parse(bytes.fromhex(v["hex"]))["inferred_qubits"] for k, v in GOLDEN.items()}
    assert got["teleport.qx"] == 25 and got["hello.qx"] == 1 and got["fusion.qx"] == 4


def test_assembler_pinned_against_reference_compiler():
    # recorded when the fixture was made: our assembler reproduced these
    # reference binaries byte for byte from their sources
    matched = [k for k, v in GOLDEN.items() if v.get("assembler_matches_reference")]
    assert {"hello.qx", "teleport.qx", "shor.qx", "aes.qx"} <= set(matched)


def test_quantum_ops_and_run_exe_noops():
    src = """
    QINIT 3
    H 0
    CNOT 0 1
    RZ 1 0.5
    CPHASE 0 2 1.25
    RESET 1
    PHASE 2 0.7
    SETPHASE 2 0.1
    EBELL 0 1
    ROT 2 y 0.3
    T 2
    S 1
    X 2
    Z 0
    SWAP 0 2
    MEASURE 1
    PRINTLN "hi"
    HALT
    X 0
    """
    ops, res, out = qexe.trace(prog(src))
    want = [(C.H, (0,), 0.0), (C.CNOT, (0, 1), 0.0), (C.RZ, (1,), 0.5), (C.CPHASE, (0, 2), 1.25),
            (C.RY, (2,), 0.3), (C.T, (2,), 0.0), (C.S, (1,), 0.0), (C.X, (2,), 0.0), (C.Z, (0,), 0.0),
            (C.SWAP, (0, 2), 0.0), (C.MEASURE, (1,), 0.0)]
    assert ops_summary(ops) == want
    assert out == b"hi\n" and res["halted"] == 1


def test_register_jumps_and_printf():
    # r0 = 0, r1 = 1, r2 = 3; body: H 0, r0 += r1; IFLT r0 r2 jumps back to the body
    body = bytes([0x05, 0]) + bytes([0x54, 0, 0, 1])
    back = -len(body)
    payload = (bytes([0x21, 0]) + struct.pack("<d", 0.0) + bytes([0x21, 1]) + struct.pack("<d", 1.0) +
               bytes([0x21, 2]) + struct.pack("<d", 3.0) + body +
               bytes([0x93, 0, 2]) + struct.pack("<q", back))
    fmt = b"r0=%0 r2=%1 half=%2"
    payload += bytes([0x21, 3]) + struct.pack("<d", 0.5)
    payload += bytes([0x98]) + struct.pack("<Q", len(fmt)) + fmt + bytes([3, 0, 2, 3]) + bytes([0xFF])
    ops, res, out = qexe.trace(qexe.write_exe(payload))
    assert ops_summary(ops) == [(C.H, (0,), 0.0)] * 3
    assert res["registers"][0] == 3.0
    assert out == b"r0=3 r2=3 half=0.5"


def test_loop_quirk_and_loops_flag():
    p = prog("LOOPSTART 3\nX 0\nLOOPEND\nHALT")
    ops, res, _ = qexe.trace(p)
    assert len(ops) == 1 and res["loop_errors"] == 1          # upstream: LOOPSTART pushes nothing
    ops, res, _ = qexe.trace(p, flags=qexe.EXE_LOOPS)
    assert len(ops) == 3 and res["loop_errors"] == 0


def test_bit_ops_charload_and_regdiv():
    payload = (bytes([0x21, 0]) + struct.pack("<d", 12.0) + bytes([0x21, 1]) + struct.pack("<d", 10.0) +
               bytes([0xA5, 2, 0, 1, 0xA6, 3, 0, 1, 0xA7, 4, 0, 1]) +
               bytes([0x21, 5]) + struct.pack("<d", 2.0) + bytes([0xA9, 6, 0, 5, 0xAA, 7, 0, 5]) +
               bytes([0x31, 8, ord("A"), 0]) + bytes([0x57, 9, 0, 5, 0x57, 10, 0, 11]) + bytes([0xFF]))
    _, res, _ = qexe.trace(qexe.write_exe(payload))
    r = res["registers"]
    assert r[2:5] == [8.0, 14.0, 6.0] and r[6:8] == [48.0, 3.0]
    assert r[8] == 65.0 and r[9] == 6.0 and r[10] == 0.0    # divide by zero leaves the register


def test_bad_files_raise():
    with pytest.raises(qb.QoaError):
        qexe.parse(b"QEXE\x01")
    with pytest.raises(qb.QoaError):
        qexe.parse(b"NOPE\x01\x00\x00\x00\x00")
    with pytest.raises(qb.QoaError):   # payload shorter than its header says
        qexe.parse(b"QEXE\x01\x05\x00\x00\x00\x05")
    with pytest.raises(qb.QoaError):   # RZ without its angle
        qexe.trace(qexe.write_exe(bytes([0x0F, 0, 1, 2])))


def test_assembler_rejects_unknown_strict_and_skips_lenient():
    with pytest.raises(ValueError):
        qexe.assemble("FOO 1 2")
    payload, skipped = qexe.assemble("FOO 1 2\nH 0", strict=False)
    assert payload == bytes([0x05, 0]) and skipped == ["FOO 1 2"]


def test_step_limit():
    payload = bytes([0x90]) + struct.pack("<q", 0)   # jmp +0 forever
    with pytest.raises(qb.QoaError):
        qexe.trace(qexe.write_exe(payload), max_steps=1000)
