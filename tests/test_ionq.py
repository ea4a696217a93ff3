"""IonQ-style JSON circuits (host side): parsing into engine ops and the
op-list -> job direction."""
import json
import math

import numpy as np
import pytest

from qoa_b200 import circuits as C
from qoa_b200 import ionq

JOB = {"name": "t", "shots": 64, "target": "simulator",
       "input": {"qubits": 4, "circuit": [
           {"gate": "h", "target": 0}, {"gate": "rz", "target": 2, "angle": 3.0},
           {"gate": "cnot", "control": 0, "target": 1}, {"gate": "cz", "control": 2, "target": 3},
           {"gate": "x", "targets": [1, 3]}, {"gate": "ry", "target": 1, "rotation": 0.25},
           {"gate": "si", "target": 2}, {"gate": "ti", "target": 0}, {"gate": "v", "target": 3},
           {"gate": "x", "controls": [0, 1], "target": 2}, {"gate": "swap", "targets": [0, 3]}]}}


def test_parse_job():
    n, ops, job = ionq.load(json.dumps(JOB))
    assert n == 4 and job["shots"] == 64
    got = [(o.opcode, tuple(o.qubits)) for o in ops]
    assert got == [(C.H, (0,)), (C.RZ, (2,)), (C.CNOT, (0, 1)), (C.CZ, (2, 3)), (C.X, (1,)), (C.X, (3,)),
                   (C.RY, (1,)), (C.P, (2,)), (C.P, (0,)), (C.U1, (3,)), (C.TOFFOLI, (0, 1, 2)), (C.SWAP, (0, 3))]
    assert ops[1].angle == 3.0 and ops[6].angle == 0.25
    assert ops[7].angle == -math.pi / 2 and ops[8].angle == -math.pi / 4
    v = np.array(ops[9].matrix).reshape(2, 2)
    assert np.allclose(v @ v, [[0, 1], [1, 0]])          # V^2 = X


def test_qubit_count_covers_targets():
    n, _, _ = ionq.load({"input": {"qubits": 2, "circuit": [{"gate": "h", "target": 5}]}})
    assert n == 6


@pytest.mark.parametrize("bad", [{"gate": "rx", "target": 0}, {"gate": "foo", "target": 0},
                                 {"gate": "h"}, {"gate": "rz", "controls": [1], "target": 0, "angle": 1.0},
                                 {"gate": "swap", "targets": [0]}])
def test_bad_gates_raise(bad):
    with pytest.raises(ValueError):
        ionq.load({"input": {"qubits": 2, "circuit": [bad]}})


def test_to_job_round_trip():
    ops = [C.Op(C.H, [0]), C.Op(C.RX, [1], 0.5), C.Op(C.CNOT, [0, 1]), C.Op(C.CZ, [1, 2]), C.Op(C.SWAP, [0, 2]),
           C.Op(C.P, [1], -math.pi / 2), C.Op(C.T, [2])]
    job = ionq.to_job(ops, 3, shots=10)
    n, back, _ = ionq.load(job)
    assert n == 3 and [(o.opcode, o.qubits, o.angle) for o in back] == [(o.opcode, o.qubits, o.angle) for o in ops]
    with pytest.raises(ValueError):
        ionq.to_job([C.Op(C.CPHASE, [0, 1], 0.3)], 2)
