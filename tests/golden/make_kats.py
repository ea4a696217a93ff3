"""Writes tests/golden/reference_kats.json: the known-answer tests of the
reference's own test suite (planetryan/qoa src/test.rs), transcribed case by
case. Each record names the test function and its line in src/test.rs; the
expected amplitudes are the hand-computed values those tests assert with
|d re|, |d im| < 1e-9 (assert_complex_approx_eq, src/test.rs:34-58).

Two levels:
  "vec"   — a src/vectorization.rs function applied to a raw slice (src/test.rs:62-472)
  "instr" — QuantumState::execute_arithmetic on a QuantumState (src/test.rs:2199-2667)

Run as `python tests/golden/make_kats.py [path-to-qoa-checkout]`: with the
path, the line numbers are refreshed from its src/test.rs; without it the
previous numbers are kept.
"""
import json
import math
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "reference_kats.json")

R2 = 1.0 / math.sqrt(2.0)
PI = math.pi


def c(re, im=0.0):
    return [float(re), float(im)]


def polar(theta):
    return c(math.cos(theta), math.sin(theta))


def basis(n, idx, val=(1.0, 0.0)):
    v = [c(0.0) for _ in range(1 << n)]
    v[idx] = c(*val)
    return v


def vec(name, fn, args, init, expect):
    return {"name": name, "level": "vec", "fn": fn, "args": args, "init": init, "expect": expect, "tol": 1e-9}


def instr(name, n, ops, init=None, expect=None, expect_at=None, expect_ne=None):
    return {"name": name, "level": "instr", "n": n, "ops": ops, "init": init, "expect": expect,
            "expect_at": expect_at, "expect_ne": expect_ne, "tol": 1e-9}


def op(opcode, qubits, angle=0.0):
    return {"opcode": opcode, "qubits": qubits, "angle": angle}


H, Z, X, P, RST, SWAP, CSWAP, T, S, RZ = 0x05, 0x06, 0x07, 0x08, 0x0A, 0x0B, 0x0C, 0x0D, 0x0E, 0x0F
QINIT, APPLYGATE, EBELL, EMULTI, ECLUSTER, ESWAP, ESWAPM = 0x04, 0x02, 0x12, 0x13, 0x14, 0x15, 0x16
CNOT, ECFB, EDIST, MEASB, RSTALL, SETP, RX, RY, PHASE, MEAS, ROT, CPHASE = (
    0x17, 0x19, 0x1A, 0x1B, 0x1C, 0x1D, 0x22, 0x23, 0x24, 0x32, 0x33, 0x35)

CASES = [
    # ---- src/test.rs:62-472, vectorization.rs functions --------------------
    vec("test_hadamard_on_0_qubit", "hadamard", [R2, 0.0, 0], basis(1, 0), [c(R2), c(R2)]),
    vec("test_hadamard_on_1_qubit", "hadamard", [R2, 0.0, 1], basis(2, 1), [c(0), c(R2), c(0), c(R2)]),
    vec("test_hadamard_on_superposition", "hadamard", [R2, 0.0, 0], [c(R2), c(R2)], [c(1), c(0)]),
    vec("test_x_on_0_qubit", "x", [0], basis(1, 0), [c(0), c(1)]),
    vec("test_x_on_1_qubit", "x", [1], basis(2, 1), basis(2, 3)),
    vec("test_y_on_0_qubit", "y", [0], basis(1, 0), [c(0), c(0, 1)]),
    vec("test_y_on_1_qubit", "y", [0], [c(0, 1), c(0)], [c(0), c(-1)]),
    vec("test_z_on_0_qubit#0", "z", [0], basis(1, 0), basis(1, 0)),
    vec("test_z_on_0_qubit#1", "z", [0], basis(1, 1), [c(0), c(-1)]),
    vec("test_t_on_0_qubit#0", "t", [0], basis(1, 0), basis(1, 0)),
    vec("test_t_on_0_qubit#1", "t", [0], basis(1, 1), [c(0), c(R2, R2)]),
    vec("test_s_on_0_qubit#0", "s", [0], basis(1, 0), basis(1, 0)),
    vec("test_s_on_0_qubit#1", "s", [0], basis(1, 1), [c(0), c(0, 1)]),
    vec("test_phaseshift_on_0_qubit#0", "phaseshift", [0, PI / 3.0], basis(1, 0), basis(1, 0)),
    vec("test_phaseshift_on_0_qubit#1", "phaseshift", [0, PI / 3.0], basis(1, 1),
        [c(0), c(math.cos(PI / 3.0), math.sin(PI / 3.0))]),
    vec("test_reset_on_0_qubit#0", "reset", [0], basis(1, 0), basis(1, 0)),
    vec("test_reset_on_0_qubit#1", "reset", [0], basis(1, 1), basis(1, 0)),
    vec("test_reset_on_0_qubit#2", "reset", [0], [c(R2), c(R2)], basis(1, 0)),
    vec("test_swap_2_qubits", "swap", [0, 1], basis(2, 1), basis(2, 2)),
    vec("test_swap_3_qubits", "swap", [0, 1], basis(3, 1), basis(3, 2)),
    vec("test_controlled_swap_3_qubits", "controlled_swap", [2, 1, 0], basis(3, 5), basis(3, 6)),
    vec("test_rx_on_0_qubit", "rx", [0, PI / 2.0], basis(1, 0),
        [c(math.cos(PI / 4.0)), c(0, -math.sin(PI / 4.0))]),
    vec("test_ry_on_0_qubit", "ry", [0, PI / 2.0], basis(1, 0), [c(math.cos(PI / 4.0)), c(math.sin(PI / 4.0))]),
    vec("test_rz_on_0_qubit#0", "rz", [0, PI / 2.0], basis(1, 0), [polar(-PI / 4.0), c(0)]),
    vec("test_rz_on_0_qubit#1", "rz", [0, PI / 2.0], basis(1, 1), [c(0), polar(PI / 4.0)]),
    vec("test_cnot_2_qubits#0", "cnot", [1, 0], basis(2, 0), basis(2, 0)),
    vec("test_cnot_2_qubits#1", "cnot", [1, 0], basis(2, 2), basis(2, 3)),
    vec("test_cz_2_qubits#0", "cz", [1, 0], basis(2, 0), basis(2, 0)),
    vec("test_cz_2_qubits#1", "cz", [1, 0], basis(2, 3), basis(2, 3, (-1.0, 0.0))),
    vec("test_controlled_phase_rotation_2_qubits#0", "controlled_phase_rotation", [1, 0, PI / 4.0],
        basis(2, 0), basis(2, 0)),
    vec("test_controlled_phase_rotation_2_qubits#1", "controlled_phase_rotation", [1, 0, PI / 4.0],
        basis(2, 3), basis(2, 3, (math.cos(PI / 4.0), math.sin(PI / 4.0)))),
    vec("test_reset_all", "reset_all", [], [c(0.5, 0.5), c(0, 1), c(1, 0), c(0.2, 0.8)], basis(2, 0)),
    # ---- src/test.rs:2199-2667, QuantumState::execute_arithmetic -------------
    instr("test_qinit", 1, [op(QINIT, [0])], init=basis(1, 1), expect=basis(1, 0)),
    instr("test_qinitq_short_for_qinit", 1, [op(QINIT, [0])], init=basis(1, 1), expect=basis(1, 0)),
    instr("test_initqubit_short_for_qinit", 1, [op(QINIT, [0])], init=basis(1, 1), expect=basis(1, 0)),
    instr("test_qmeas", 1, [op(MEAS, [0])], expect=basis(1, 0)),
    instr("test_meas_short_for_qmeas", 1, [op(MEAS, [0])], expect=basis(1, 0)),
    instr("test_measure_short_for_qmeas", 1, [op(MEAS, [0])], expect=basis(1, 0)),
    instr("test_h_short_for_applyhadamard", 1, [op(H, [0])], expect=[c(R2), c(R2)]),
    instr("test_had_short_for_applyhadamard", 1, [op(H, [0])], expect=[c(R2), c(R2)]),
    instr("test_cnot_short_for_controllednot", 2, [op(CNOT, [1, 0])], init=basis(2, 2), expect=basis(2, 3)),
    instr("test_z_short_for_applyphaseflip", 1, [op(Z, [0])], init=basis(1, 1), expect_at={"1": c(-1)}),
    instr("test_x_short_for_applybitflip", 1, [op(X, [0])], expect_at={"1": c(1)}),
    instr("test_t_short_for_applytgate", 1, [op(T, [0])], init=basis(1, 1), expect_at={"1": polar(PI / 4.0)}),
    instr("test_s_short_for_applysgate", 1, [op(S, [0])], init=basis(1, 1), expect_at={"1": polar(PI / 2.0)}),
    instr("test_p_short_for_phaseshift", 1, [op(P, [0], PI / 2.0)], init=basis(1, 1),
          expect_at={"1": polar(PI / 2.0)}),
    instr("test_rst_short_for_reset", 1, [op(RST, [0])], init=basis(1, 1), expect_at={"0": c(1)}),
    instr("test_cswap_short_for_controlledswap", 3, [op(CSWAP, [2, 1, 0])], init=basis(3, 5), expect=basis(3, 6)),
    instr("test_ebell_short_for_entanglebell", 2, [op(EBELL, [0, 1])], expect_at={"0": c(R2), "3": c(R2)}),
    instr("test_emulti_short_for_entanglemulti", 3, [op(EMULTI, [0, 1, 2])], expect_ne={"0": c(1)}),
    instr("test_ecluster_short_for_entanglecluster", 3, [op(ECLUSTER, [0, 1, 2])], expect_ne={"0": c(1)}),
    instr("test_eswap_short_for_entangleswap", 4, [op(ESWAP, [0, 1, 2, 3])], init=basis(4, 3),
          expect_ne={"3": c(1)}),
    instr("test_eswapm_short_for_entangleswapmeasure", 4, [op(ESWAPM, [0, 1, 2, 3])]),
    instr("test_ecfb_short_for_entanglewithclassicalfeedback", 2, [op(ECFB, [0, 1])]),
    instr("test_edist_short_for_entangledistributed", 1, [op(EDIST, [0])]),
    instr("test_measb_short_for_measureinbasis", 1, [op(MEASB, [0, ord("X")])]),
    instr("test_rstall_short_for_resetall", 2, [op(RSTALL, [])], init=basis(2, 3), expect_at={"0": c(1)}),
    instr("test_setp_short_for_setphase", 1, [op(SETP, [0], PI / 2.0)], init=basis(1, 1),
          expect_at={"1": polar(PI / 2.0)}),
    instr("test_agate_short_for_applygate", 1, [op(APPLYGATE, [0, ord("H")])]),
    instr("test_phase_ionq", 1, [op(PHASE, [0], PI / 4.0)], init=basis(1, 1),
          expect_at={"0": c(0), "1": polar(PI / 4.0)}),
    instr("test_applyrotation_x", 1, [op(ROT, [0, ord("X")], PI / 2.0)], expect_at={"0": c(R2), "1": c(0, -R2)}),
    instr("test_rot_short_for_applyrotation", 1, [op(ROT, [0, ord("X")], PI / 2.0)],
          expect_at={"0": c(R2), "1": c(0, -R2)}),
    instr("test_applyrotation_y", 1, [op(ROT, [0, ord("Y")], PI / 2.0)], expect_at={"0": c(R2), "1": c(R2)}),
    instr("test_applyrotation_z", 1, [op(ROT, [0, ord("Z")], PI / 2.0)],
          expect_at={"0": polar(-PI / 4.0), "1": c(0)}),
    instr("test_applycphase", 2, [op(CPHASE, [0, 1], PI / 4.0)], init=basis(2, 3),
          expect_at={"0": c(0), "1": c(0), "2": c(0), "3": polar(PI / 4.0)}),
    instr("test_cphase_short_for_controlledphaserotation", 2, [op(CPHASE, [0, 1], PI / 4.0)], init=basis(2, 3),
          expect_at={"3": polar(PI / 4.0)}),
]


def main(ref=None):
    lines = {}
    old = {}
    if os.path.exists(OUT):
        for rec in json.load(open(OUT))["cases"]:
            old[rec["name"]] = rec.get("src")
    path = os.path.join(ref, "src", "test.rs") if ref else None
    if path and os.path.exists(path):
        for i, line in enumerate(open(path), start=1):
            m = re.match(r"\s*fn (test_\w+)\(", line)
            if m and m.group(1) not in lines:
                lines[m.group(1)] = i
    for rec in CASES:
        base = rec["name"].split("#")[0]
        rec["src"] = f"src/test.rs:{lines[base]}" if base in lines else old.get(rec["name"])
    json.dump({"source": "planetryan/qoa src/test.rs", "tolerance_rule": "abs(re), abs(im) < 1e-9",
               "cases": CASES}, open(OUT, "w"), indent=1)
    print(f"wrote {len(CASES)} cases to {OUT}")


if __name__ == "__main__":
    import sys
    main(sys.argv[1] if len(sys.argv) > 1 else None)
