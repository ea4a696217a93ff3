"""Bytecode front-end (host side): .qexe header parsing and qubit inference,
the run_exe interpreter traced without a GPU, and the assembler.

The fixtures (tests/golden/qexe_programs.json, made by make_qexe_fixtures.py)
are the reference's example sources (qoa_files/*.qoa) assembled by this
repository's own assembler; they must parse, run to HALT and infer the qubit
counts `qoa run` would. The assembler itself is pinned instruction by
instruction against bytes written out by hand from the encode rules of
src/instructions.rs (Instruction::encode, 631-1489); small programs of our
own pin the instruction semantics (jumps, registers, printing, the loop quirk).
"""
import json
import os
import struct

import numpy as np
import pytest

import qoa_b200 as qb
from qoa_b200 import circuits as C
from qoa_b200 import qexe

HERE = os.path.dirname(os.path.abspath(__file__))
PROGRAMS = json.load(open(os.path.join(HERE, "golden", "qexe_programs.json")))


def prog(src: str, kind="qexe") -> bytes:
    payload, _ = qexe.assemble(src)
    return qexe.write_exe(payload, kind)


def ops_summary(ops):
    return [(int(o["opcode"]), tuple(int(x) for x in o["q"][:o["nq"]]), float(o["angle"])) for o in ops]


@pytest.mark.parametrize("name", sorted(PROGRAMS))
def test_example_programs_parse_and_run_to_halt(name):
    f = bytes.fromhex(PROGRAMS[name]["hex"])
    info = qexe.parse(f)
    assert info["kind"] in qexe.MAGIC and info["payload_offset"] == 9
    assert info["payload_len"] == len(f) - 9
    ops, res, out = qexe.trace(f)
    assert res["halted"] == 1 and res["unknown_opcodes"] == 0 and res["loop_errors"] == 0
    assert res["gates"] + res["measurements"] == len(ops)
    # every qubit the program touches lies below the inferred count
    qmax = max((int(o["q"][k]) for o in ops for k in range(o["nq"])), default=-1)
    assert qmax < max(info["inferred_qubits"], 1)


def test_fixtures_are_what_the_assembler_writes_now():
    # a fixture that no longer matches the assembler's output means the
    # assembler changed; regenerate with make_qexe_fixtures.py after review
    for name, rec in PROGRAMS.items():
        f = bytes.fromhex(rec["hex"])
        assert f[:4] == b"QEXE" and f[4] == 1 and struct.unpack("<I", f[5:9])[0] == len(f) - 9, name


def test_hello_world_prints():
    ops, res, out = qexe.trace(bytes.fromhex(PROGRAMS["hello_world"]["hex"]))
    assert out == b"Hello, World!\n" and len(ops) == 0 and res["halted"] == 1


def test_qubit_inference():
    got = {k: qexe.parse(bytes.fromhex(v["hex"]))["inferred_qubits"] for k, v in PROGRAMS.items()}
    assert got == {"teleport": 25, "hello_world": 1, "fusion-sim": 4, "shor": 13, "aes-decryption-16": 25}


# (source line, expected bytes written out from the encode rule, rule's line in src/instructions.rs)
F05 = "000000000000e03f"   # 0.5 as f64, little endian
F10 = "000000000000f03f"   # 1.0
F025 = "000000000000d03f"  # 0.25
F20 = "0000000000000040"   # 2.0
ENCODINGS = [
    ("QINIT 3", "0403", 634), ("QI 3", "0403", 634), ("MEASURE 2", "3202", 639), ("M 2", "3202", 639),
    ("H 1", "0501", 644), ("HAD 1", "0501", 644), ("CNOT 0 1", "170001", 647), ("CN 2 0", "170200", 647),
    ("Z 2", "0602", 650), ("X 2", "0702", 651), ("T 4", "0d04", 652), ("S 4", "0e04", 653),
    ("P 1 0.5", "0801" + F05, 654), ("PHASESHIFT 1 0.5", "0801" + F05, 654),
    ("RESET 1", "0a01", 664), ("RST 1", "0a01", 664), ("SWAP 0 1", "0b0001", 669),
    ("CSWAP 0 1 2", "0c000102", 670), ("ENTANGLE 0 1", "110001", 673), ("EBELL 0 1", "120001", 674),
    ("EMULTI 0 1 2", "1303000102", 677), ("ECLUSTER 0 1 2", "1403000102", 682),
    ("ESWAP 0 1 2 3", "1500010203", 687), ("RESETALL", "1c", 723), ("SETPHASE 1 0.25", "1d01" + F025, 733),
    ("CHARLOAD 2 'A'", "310241", 753), ("CHAROUT 2", "1802", 756),
    ("RX 0 1.0", "2200" + F10, 761), ("RY 0 1.0", "2300" + F10, 766), ("RZ 0 1.0", "0f00" + F10, 771),
    ("PHASE 2 0.5", "2402" + F05, 776), ("CZ 1 0", "1e0100", 781), ("REGSET 3 2.0", "2103" + F20, 790),
    ("LOOPSTART 2", "0102", 799), ("LOOPEND", "10", 802), ("ROT 0 x 0.5", "330078" + F05, 805),
    ("CPHASE 0 1 0.5", "350001" + F05, 822), ("APPLYCPHASE 0 1 0.5", "350001" + F05, 822),
    ("JMP -3", "90fdffffffffffffff", 988), ("REGADD 0 1 2", "54000102", 1029), ("REGCOPY 4 5", "580405", 1041),
    ("HALT", "ff", 1345), ("JMPABS 16", "911000000000000000", 1353),
    ("IFLT 0 1 -4", "930001fcffffffffffffff", 1363),
    ('PRINTF "x" 1 2', "98" + "0100000000000000" + "78" + "020102", 1387),
    ('PRINT "a"', "99" + "0100000000000000" + "61", 1395),
    ('PRINTLN "hi"', "9a" + "0200000000000000" + "6869", 1401),
    ("SEEDRNG 7", "ad0700000000000000", 1476),
]


@pytest.mark.parametrize("line,expect,rule", ENCODINGS, ids=[e[0] for e in ENCODINGS])
def test_assembler_matches_encode_rules(line, expect, rule):
    payload, skipped = qexe.assemble(line)
    assert not skipped
    assert payload == bytes.fromhex(expect), f"src/instructions.rs:{rule}"


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
