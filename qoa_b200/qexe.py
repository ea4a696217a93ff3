"""Bytecode front-end: .qoa assembly -> .qexe bytes, and .qexe programs run on
the engine (qoa_exe_* in the C ABI).

`assemble` restates `qoa compile` (compile_qoa_to_bin, main.rs:1677-1700, with
Instruction::parse_instruction / encode, instructions.rs:1849 / 631) for the
quantum instructions and the common classical ones; a line whose mnemonic is
outside that set raises (strict) or is skipped (as upstream skips lines it
cannot parse). `write_exe` adds the file header (write_exe, main.rs:1702-1709).
"""
import ctypes
import struct
from typing import Iterable, List, Optional, Tuple

import numpy as np

from . import OP_DTYPE, QoaError, _check, lib, register_signatures

MAGIC = {"qexe": b"QEXE", "oexe": b"OEXE", "qox": b"QOX ", "xexe": b"XEXE", "qex": b"QEX ", "qx": b"QX\0\0"}
EXE_LOOPS = 0x1

_ALIAS = {
    "QI": "QINIT", "INITQUBIT": "QINIT", "QINITQ": "QINIT", "IQ": "QINIT",
    "QM": "QMEAS", "MEASURE": "QMEAS", "MEAS": "QMEAS", "M": "QMEAS",
    "HAD": "H", "APPLYHADAMARD": "H",
    "CN": "CNOT", "CONTROLLEDNOT": "CNOT",
    "APPLYPHASEFLIP": "Z", "APPLYBITFLIP": "X", "APPLYTGATE": "T", "APPLYSGATE": "S",
    "PHASESHIFT": "P",
    "RST": "RESET", "RSTQ": "RESET", "QRESET": "RESET", "QR": "RESET",
    "CONTROLLEDSWAP": "CSWAP", "CS": "CSWAP",
    "ENTANGLEBELL": "EBELL", "EB": "EBELL", "ENTANGLEMULTI": "EMULTI", "EM": "EMULTI",
    "ENTANGLECLUSTER": "ECLUSTER", "ECR": "ECLUSTER", "ENTANGLESWAP": "ESWAP", "ESP": "ESWAP",
    "RSTALL": "RESETALL", "RSA": "RESETALL",
    "SETP": "SETPHASE", "SPH": "SETPHASE",
    "CLOAD": "CHARLOAD", "CLD": "CHARLOAD", "COUT": "CHAROUT", "CO": "CHAROUT",
    "RSET": "REGSET", "RGST": "REGSET",
    "LSTART": "LOOPSTART", "LS": "LOOPSTART", "LEND": "LOOPEND", "LE": "LOOPEND",
    "ROT": "APPLYROTATION", "AR": "APPLYROTATION",
    "CPHASE": "CPR", "APPLYCPHASE": "CPR", "CONTROLLEDPHASEROTATION": "CPR",
    "PSE": "PHASE",
    "SPOS": "SETPOS", "STP": "SETPOS", "SWL": "SETWL", "SW": "SETWL", "WLS": "WLSHIFT", "WLSH": "WLSHIFT",
    "MOV": "MOVE", "MV": "MOVE", "MOBS": "MARKOBSERVED", "MO": "MARKOBSERVED", "REL": "RELEASE", "RL": "RELEASE",
    "HLT": "HALT", "PLN": "PRINTLN", "VLOG": "VERBOSELOG", "VL": "VERBOSELOG",
    "RADD": "REGADD", "RGA": "REGADD", "RSUB": "REGSUB", "RGS": "REGSUB", "RMUL": "REGMUL", "RM": "REGMUL",
    "RDIV": "REGDIV", "RD": "REGDIV", "RCOPY": "REGCOPY", "RC": "REGCOPY",
    "JABS": "JMPABS", "JMPA": "JMPABS", "IGT": "IFGT", "ILT": "IFLT", "IEQ": "IFEQ", "INE": "IFNE",
    "PF": "PRINTF", "DREGS": "DUMPREGS", "DR": "DUMPREGS", "SRNG": "SEEDRNG", "RN": "RAND",
    "CMT": "COMMENT", "CM": "COMMENT",
}


def _tokens(part: str) -> List[str]:
    """Whitespace tokens; a double-quoted string (quotes kept) is one token."""
    out, cur, in_str = [], "", False
    for c in part:
        if c == '"':
            if in_str:
                out.append(cur + c)
                cur, in_str = "", False
            else:
                if cur:
                    out.append(cur)
                cur, in_str = c, True
        elif c.isspace() and not in_str:
            if cur:
                out.append(cur)
                cur = ""
        else:
            cur += c
    if cur:
        out.append(cur)
    return out


def _u8(s: str) -> int:
    v = int(s, 10)
    if not 0 <= v <= 255 or not s.lstrip("+").isdigit():
        raise ValueError(f"invalid u8: {s}")
    return v


def _f64(s: str) -> bytes:
    return struct.pack("<d", float(s))


def _lit(s: str) -> bytes:
    if len(s) >= 2 and s[0] == '"' and s[-1] == '"':
        return s[1:-1].encode()
    raise ValueError(f"invalid string literal: {s}")


def encode_line(line: str) -> Optional[bytes]:
    """Bytes of one source line (None for a comment, blank or label line)."""
    t = line.strip()
    if not t or t.startswith(";") or t.startswith("//"):
        return None
    if t.endswith(":"):
        return b""
    part = t.split(";")[0].strip()
    if not part:
        return None
    tok = _tokens(part)
    op = tok[0].upper()
    op = _ALIAS.get(op, op)
    a = tok[1:]

    def n(k):
        if len(a) != k:
            raise ValueError(f"{op}: expected {k} operands, got {len(a)}")

    one_q = {"QINIT": 0x04, "QMEAS": 0x32, "H": 0x05, "Z": 0x06, "X": 0x07, "T": 0x0D, "S": 0x0E, "RESET": 0x0A,
             "CHAROUT": 0x18, "MARKOBSERVED": 0x79, "RELEASE": 0x7A, "LOOPSTART": 0x01, "RAND": 0x50}
    q_angle = {"P": 0x08, "RX": 0x22, "RY": 0x23, "RZ": 0x0F, "PHASE": 0x24, "SETPHASE": 0x1D, "REGSET": 0x21,
               "SETWL": 0x75, "WLSHIFT": 0x76}
    two_q = {"CNOT": 0x17, "CZ": 0x1E, "SWAP": 0x0B, "ENTANGLE": 0x11, "EBELL": 0x12, "REGCOPY": 0x58}
    three = {"REGADD": 0x54, "REGSUB": 0x55, "REGMUL": 0x56, "REGDIV": 0x57, "CSWAP": 0x0C}
    if op in one_q:
        n(1)
        return bytes([one_q[op], _u8(a[0])])
    if op in q_angle:
        n(2)
        return bytes([q_angle[op], _u8(a[0])]) + _f64(a[1])
    if op in two_q:
        n(2)
        return bytes([two_q[op], _u8(a[0]), _u8(a[1])])
    if op in three:
        n(3)
        return bytes([three[op], _u8(a[0]), _u8(a[1]), _u8(a[2])])
    if op == "CPR":
        n(3)
        return bytes([0x35, _u8(a[0]), _u8(a[1])]) + _f64(a[2])
    if op in ("EMULTI", "ECLUSTER"):
        qs = [_u8(x) for x in a]
        return bytes([0x13 if op == "EMULTI" else 0x14, len(qs)] + qs)
    if op == "ESWAP":
        n(4)
        return bytes([0x15] + [_u8(x) for x in a])
    if op == "APPLYROTATION":
        n(3)
        if a[1] not in ("x", "y", "z"):
            raise ValueError(f"invalid axis: {a[1]}")
        return bytes([0x33, _u8(a[0]), ord(a[1])]) + _f64(a[2])
    if op in ("SETPOS", "MOVE"):
        n(3)
        return bytes([0x74 if op == "SETPOS" else 0x77, _u8(a[0])]) + _f64(a[1]) + _f64(a[2])
    if op == "CHARLOAD":
        n(2)
        if len(a[1]) == 3 and a[1][0] == "'" and a[1][2] == "'":
            return bytes([0x31, _u8(a[0]), ord(a[1][1]) & 0xFF])
        raise ValueError(f"invalid char literal: {a[1]}")
    if op in ("PRINT", "PRINTLN"):
        n(1)
        s = _lit(a[0])
        return bytes([0x99 if op == "PRINT" else 0x9A]) + struct.pack("<Q", len(s)) + s
    if op == "VERBOSELOG":
        n(2)
        return bytes([0x87, _u8(a[0])]) + _lit(a[1]) + b"\0"
    if op == "COMMENT":
        return bytes([0x88]) + " ".join(a).encode() + b"\0"
    if op in ("LOOPEND", "RESETALL", "HALT", "DUMPREGS"):
        n(0)
        return bytes([{"LOOPEND": 0x10, "RESETALL": 0x1C, "HALT": 0xFF, "DUMPREGS": 0x9D}[op]])
    if op in ("JMP", "JMPABS"):
        n(1)
        return bytes([0x90 if op == "JMP" else 0x91]) + struct.pack("<q" if op == "JMP" else "<Q", int(a[0]))
    if op in ("IFGT", "IFLT", "IFEQ", "IFNE"):
        n(3)
        code = {"IFGT": 0x92, "IFLT": 0x93, "IFEQ": 0x94, "IFNE": 0x95}[op]
        return bytes([code, _u8(a[0]), _u8(a[1])]) + struct.pack("<q", int(a[2]))
    if op == "PRINTF":
        s = _lit(a[0])
        regs = [_u8(x) for x in a[1:]]
        return bytes([0x98]) + struct.pack("<Q", len(s)) + s + bytes([len(regs)] + regs)
    if op == "SEEDRNG":
        n(1)
        return bytes([0xAD]) + struct.pack("<Q", int(a[0]))
    raise KeyError(op)


def assemble(source: str, strict: bool = True) -> Tuple[bytes, List[str]]:
    """Payload bytes of a .qoa source and the lines that were skipped."""
    out, skipped = bytearray(), []
    for line in source.splitlines():
        try:
            b = encode_line(line)
        except (KeyError, ValueError) as e:
            if strict:
                raise ValueError(f"cannot assemble {line.strip()!r}: {e}") from None
            skipped.append(line)
            continue
        if b:
            out += b
    return bytes(out), skipped


def write_exe(payload: bytes, kind: str = "qexe", version: int = 1) -> bytes:
    return MAGIC[kind] + bytes([version]) + struct.pack("<I", len(payload)) + payload


class ExeInfo(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_char * 8), ("version", ctypes.c_uint32), ("inferred_qubits", ctypes.c_uint32),
                ("payload_offset", ctypes.c_uint64), ("payload_len", ctypes.c_uint64)]


class ExeResult(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in ("instructions", "gates", "measurements", "chars_out", "range_errors",
                                               "loop_errors", "unknown_opcodes", "unsupported")] + \
               [("halted", ctypes.c_uint32), ("exit_code", ctypes.c_int32), ("registers", ctypes.c_double * 24)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "registers"}
        d["registers"] = list(self.registers)
        return d


_vp, _sz, _u32, _u64 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint64
register_signatures({
    "qoa_exe_parse": (ctypes.c_int, [ctypes.c_char_p, _sz, ctypes.POINTER(ExeInfo)]),
    "qoa_exe_run": (ctypes.c_int, [_vp, ctypes.c_char_p, _sz, _u32, _u64, ctypes.POINTER(ExeResult),
                                   ctypes.c_char_p, _sz, ctypes.POINTER(_sz)]),
    "qoa_exe_trace": (ctypes.c_int, [ctypes.c_char_p, _sz, _u32, _u64, _vp, _sz, ctypes.POINTER(_sz),
                                     ctypes.POINTER(ExeResult), ctypes.c_char_p, _sz, ctypes.POINTER(_sz)]),
})


def parse(file: bytes) -> dict:
    info = ExeInfo()
    rc = lib.qoa_exe_parse(file, len(file), ctypes.byref(info))
    if rc:
        raise QoaError(rc, (lib.qoa_last_error(None) or b"").decode())
    return {"kind": info.kind.decode(), "version": info.version, "inferred_qubits": info.inferred_qubits,
            "payload_offset": info.payload_offset, "payload_len": info.payload_len}


def _text(buf, n) -> bytes:
    return bytes(buf.raw[:min(n.value, len(buf.raw) - 1)])


def trace(file: bytes, flags: int = 0, max_steps: int = 10_000_000) -> Tuple[np.ndarray, dict, bytes]:
    """Host-only interpretation: (op list, counters, printed bytes)."""
    res, nops, tlen = ExeResult(), ctypes.c_size_t(), ctypes.c_size_t()
    lib.qoa_exe_trace(file, len(file), flags, max_steps, None, 0, ctypes.byref(nops), ctypes.byref(res), None, 0,
                      ctypes.byref(tlen))
    ops = np.zeros(nops.value, dtype=OP_DTYPE)
    buf = ctypes.create_string_buffer(tlen.value + 1)
    rc = lib.qoa_exe_trace(file, len(file), flags, max_steps, ops.ctypes.data if len(ops) else None, len(ops),
                           ctypes.byref(nops), ctypes.byref(res), buf, len(buf), ctypes.byref(tlen))
    if rc:
        raise QoaError(rc, (lib.qoa_last_error(None) or b"").decode())
    return ops, res.as_dict(), _text(buf, tlen)


def run(state, file: bytes, flags: int = 0, max_steps: int = 10_000_000, out_cap: int = 1 << 20) -> Tuple[dict, bytes]:
    """Runs a program on a QuantumState (complex128): (counters, printed bytes)."""
    res, tlen = ExeResult(), ctypes.c_size_t()
    buf = ctypes.create_string_buffer(out_cap)
    rc = lib.qoa_exe_run(state.handle, file, len(file), flags, max_steps, ctypes.byref(res), buf, out_cap,
                         ctypes.byref(tlen))
    _check(rc, state.handle)
    return res.as_dict(), _text(buf, tlen)
