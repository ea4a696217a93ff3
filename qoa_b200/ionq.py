"""IonQ-style JSON circuits as an engine op list, and back.

The format is the job description the reference keeps under ionq/ (and that
its `compile-json` command is meant to produce, main.rs:1589-1595 and
4310-4323, where the conversion is left unimplemented):

    {"name": ..., "shots": S, "target": "simulator",
     "input": {"qubits": N, "circuit": [{"gate": "h", "target": 0},
                                         {"gate": "rz", "target": 2, "angle": 3.0},
                                         {"gate": "cnot", "control": 0, "target": 1}, ...]}}

Gates (IonQ's QIS names): h x y z s si t ti v vi rx ry rz cnot cx cz swap,
with "angle" (or "rotation") in radians; "targets" / "controls" lists are
accepted as well as the single "target" / "control". x with one or two
controls is CNOT / Toffoli, y and z with one control are CY / CZ. CZ here is
the physical controlled-Z (both qubits set).
"""
import json
import math
from typing import List, Tuple, Union

from .circuits import (CNOT, CY, CZ, H, P, RX, RY, RZ, S, SWAP, T, TOFFOLI, U1, X, Y, Z, Op,
                       ops_to_array)

_ONE = {"h": H, "x": X, "y": Y, "z": Z, "s": S, "t": T}
_ROT = {"rx": RX, "ry": RY, "rz": RZ}
_V = [complex(0.5, 0.5), complex(0.5, -0.5), complex(0.5, -0.5), complex(0.5, 0.5)]   # sqrt(X)


def _list(g: dict, one: str, many: str) -> List[int]:
    if many in g:
        return [int(q) for q in g[many]]
    if one in g:
        return [int(g[one])]
    return []


def circuit_ops(circuit: List[dict]) -> List[Op]:
    """Engine ops of an IonQ circuit list (raises ValueError on what it lacks)."""
    ops: List[Op] = []
    for k, g in enumerate(circuit):
        name = str(g.get("gate", "")).lower()
        tg = _list(g, "target", "targets")
        ct = _list(g, "control", "controls")
        ang = g.get("angle", g.get("rotation"))
        if not tg:
            raise ValueError(f"gate {k}: no target")
        if name in ("cnot", "cx"):
            if len(ct) != 1 or len(tg) != 1:
                raise ValueError(f"gate {k}: cnot takes one control and one target")
            ops.append(Op(CNOT, [ct[0], tg[0]]))
        elif name == "cz":
            if len(ct) != 1 or len(tg) != 1:
                raise ValueError(f"gate {k}: cz takes one control and one target")
            ops.append(Op(CZ, [ct[0], tg[0]]))
        elif name == "swap":
            if len(tg) != 2 or ct:
                raise ValueError(f"gate {k}: swap takes two targets")
            ops.append(Op(SWAP, tg))
        elif ct:
            if name == "x" and len(ct) == 1:
                ops.append(Op(CNOT, [ct[0], tg[0]]))
            elif name == "x" and len(ct) == 2:
                ops.append(Op(TOFFOLI, [ct[0], ct[1], tg[0]]))
            elif name == "y" and len(ct) == 1:
                ops.append(Op(CY, [ct[0], tg[0]]))
            elif name == "z" and len(ct) == 1:
                ops.append(Op(CZ, [ct[0], tg[0]]))
            else:
                raise ValueError(f"gate {k}: controlled {name} is not supported")
        elif name in _ONE:
            ops += [Op(_ONE[name], [q]) for q in tg]
        elif name in ("si", "ti"):
            ops += [Op(P, [q], -math.pi / (2 if name == "si" else 4)) for q in tg]
        elif name in ("v", "vi"):
            m = _V if name == "v" else [c.conjugate() for c in _V]
            ops += [Op(U1, [q], 0.0, m) for q in tg]
        elif name in _ROT:
            if ang is None:
                raise ValueError(f"gate {k}: {name} needs an angle")
            ops += [Op(_ROT[name], [q], float(ang)) for q in tg]
        else:
            raise ValueError(f"gate {k}: unknown gate {name!r}")
    return ops


def load(job: Union[str, dict]) -> Tuple[int, list, dict]:
    """(qubits, ops, job) from a job dict, JSON text or file path."""
    if isinstance(job, str):
        job = json.loads(job) if job.lstrip().startswith("{") else json.load(open(job))
    inp = job["input"]
    ops = circuit_ops(inp["circuit"])
    n = int(inp.get("qubits", 0))
    used = max((q for o in ops for q in o.qubits), default=-1) + 1
    return max(n, used, 1), ops, job


def load_array(job):
    n, ops, job = load(job)
    return n, ops_to_array(ops), job


def to_job(ops: List[Op], n: int, name: str = "compiled-qoa-circuit", shots: int = 1024) -> dict:
    """IonQ job dict of an engine op list (the compile-json direction) for the
    gates the format has: H X Y Z S T PHASESHIFT(+-pi/2, +-pi/4) RX RY RZ CNOT
    CZ SWAP; anything else raises."""
    inv1 = {H: "h", X: "x", Y: "y", Z: "z", S: "s", T: "t"}
    inv_rot = {RX: "rx", RY: "ry", RZ: "rz"}
    out = []
    for o in ops:
        if o.opcode in inv1:
            out.append({"gate": inv1[o.opcode], "target": o.qubits[0]})
        elif o.opcode in inv_rot:
            out.append({"gate": inv_rot[o.opcode], "target": o.qubits[0], "angle": o.angle})
        elif o.opcode == P and abs(o.angle + math.pi / 2) < 1e-15:
            out.append({"gate": "si", "target": o.qubits[0]})
        elif o.opcode == P and abs(o.angle + math.pi / 4) < 1e-15:
            out.append({"gate": "ti", "target": o.qubits[0]})
        elif o.opcode == CNOT:
            out.append({"gate": "cnot", "control": o.qubits[0], "target": o.qubits[1]})
        elif o.opcode == CZ:
            out.append({"gate": "cz", "control": o.qubits[0], "target": o.qubits[1]})
        elif o.opcode == SWAP:
            out.append({"gate": "swap", "targets": list(o.qubits)})
        else:
            raise ValueError(f"opcode 0x{o.opcode:02X} has no IonQ JSON form")
    return {"name": name, "shots": int(shots), "target": "simulator", "input": {"qubits": int(n), "circuit": out}}
