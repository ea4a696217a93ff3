"""Op records and seeded synthetic circuits.

An op is one ``qoa_op`` record of include/qoa_cuda.h: the reference opcode
byte (src/instructions.rs:631-830), up to four qubit operands, an angle, and
pointers for long qubit lists and unitary matrices. ``OP_DTYPE`` is the same
48-byte layout as a numpy structured dtype so whole circuits cross the C ABI
as one buffer.

The generators make the workloads the engine is measured on, from a
splitmix64 stream so every run, test and the CPU oracle see the same gates:
random layered circuits (1-qubit gate on every qubit from {H, T, S, RX, RY,
RZ, PHASESHIFT}, then CNOT / CZ / CPHASE on floor(n/2) disjoint random
pairs), the quantum Fourier transform, and hardware-efficient variational
circuits.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

# reference opcode numbers (src/instructions.rs encode())
H, Z, X, P, RESET, SWAP, CSWAP, T, S, RZ = 0x05, 0x06, 0x07, 0x08, 0x0A, 0x0B, 0x0C, 0x0D, 0x0E, 0x0F
APPLYGATE, QINIT = 0x02, 0x04
ENTANGLE, EBELL, EMULTI, ECLUSTER, ESWAP, ESWAPM = 0x11, 0x12, 0x13, 0x14, 0x15, 0x16
CNOT, ECFB, EDIST, MEASB, RESETALL, SETPHASE, CZ = 0x17, 0x19, 0x1A, 0x1B, 0x1C, 0x1D, 0x1E
RX, RY, PHASE, MEASURE, ROT, CPHASE = 0x22, 0x23, 0x24, 0x32, 0x33, 0x35
# engine extensions (unused reference opcode range 0xF0-0xFE)
Y, U1, U2, TOFFOLI, CY = 0xF0, 0xF1, 0xF2, 0xF3, 0xF4

ONE_QUBIT_GATES = (H, T, S, RX, RY, RZ, P)
TWO_QUBIT_GATES = (CNOT, CZ, CPHASE)
ANGLED = (RX, RY, RZ, P, CPHASE, SETPHASE, PHASE, ROT)

OP_DTYPE = np.dtype([("opcode", "<u4"), ("nq", "<u4"), ("q", "<u4", (4,)), ("angle", "<f8"),
                     ("qlist", "<u8"), ("matrix", "<u8")], align=True)
assert OP_DTYPE.itemsize == 48


@dataclass
class Op:
    opcode: int
    qubits: Sequence[int] = ()
    angle: float = 0.0
    matrix: Optional[np.ndarray] = None

    def __post_init__(self):
        self.qubits = [int(q) for q in self.qubits]


class OpArray(np.ndarray):
    """Structured op array that keeps the buffers its qlist/matrix pointers name."""

    def __array_finalize__(self, obj):
        self._keep = getattr(obj, "_keep", [])


def ops_to_array(ops: Sequence[Op]) -> OpArray:
    arr = np.zeros(len(ops), dtype=OP_DTYPE).view(OpArray)
    keep = []
    for i, op in enumerate(ops):
        arr["opcode"][i] = op.opcode
        qs = list(op.qubits)
        arr["nq"][i] = len(qs)
        if len(qs) <= 4:
            arr["q"][i, : len(qs)] = qs
        else:
            ql = np.ascontiguousarray(np.asarray(qs, dtype=np.uint32))
            keep.append(ql)
            arr["qlist"][i] = ql.ctypes.data
            arr["q"][i, :] = qs[:4]
        arr["angle"][i] = op.angle
        if op.matrix is not None:
            m = np.ascontiguousarray(np.asarray(op.matrix, dtype=np.complex128).reshape(-1))
            keep.append(m)
            arr["matrix"][i] = m.ctypes.data
    arr._keep = keep
    return arr


class SplitMix64:
    """splitmix64 (Steele, Lea, Flood 2014): the seed stream of every generator."""

    MASK = (1 << 64) - 1

    def __init__(self, seed: int):
        self.x = seed & self.MASK

    def next(self) -> int:
        self.x = (self.x + 0x9E3779B97F4A7C15) & self.MASK
        z = self.x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & self.MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & self.MASK
        return z ^ (z >> 31)

    def uniform(self) -> float:
        return (self.next() >> 11) * (1.0 / 9007199254740992.0)

    def below(self, k: int) -> int:
        return min(int(self.uniform() * k), k - 1)


def random_layered(n: int, depth: int, seed: int, initial_h: bool = False) -> List[Op]:
    """Random layered circuit: per layer a 1-qubit gate on every qubit drawn
    from {H, T, S, RX, RY, RZ, PHASESHIFT} (angles U[0, 2pi)), then CNOT / CZ /
    CPHASE on floor(n/2) disjoint pairs from a Fisher-Yates permutation (first
    of a pair = control). `initial_h` prepends H on every qubit."""
    rng = SplitMix64(seed)
    ops: List[Op] = []
    if initial_h:
        ops += [Op(H, [q]) for q in range(n)]
    for _ in range(depth):
        for q in range(n):
            g = ONE_QUBIT_GATES[rng.below(len(ONE_QUBIT_GATES))]
            a = rng.uniform() * 2.0 * math.pi if g in (RX, RY, RZ, P) else 0.0
            ops.append(Op(g, [q], a))
        perm = list(range(n))
        for i in range(n - 1, 0, -1):
            j = rng.below(i + 1)
            perm[i], perm[j] = perm[j], perm[i]
        for k in range(n // 2):
            c, t = perm[2 * k], perm[2 * k + 1]
            g = TWO_QUBIT_GATES[rng.below(len(TWO_QUBIT_GATES))]
            a = rng.uniform() * 2.0 * math.pi if g == CPHASE else 0.0
            ops.append(Op(g, [c, t], a))
    return ops


def layered_workload(n: int = 20, depth: int = 40, seed: int = 0) -> List[Op]:
    """20-qubit depth-40 layered circuit from |0..0> (1200 gates at n=20)."""
    return random_layered(n, depth, seed, initial_h=False)


def layered_h_workload(n: int = 30, depth: int = 20, seed: int = 1) -> List[Op]:
    """30-qubit circuit: H on all qubits, then 20 layers (930 gates at n=30)."""
    return random_layered(n, depth, seed, initial_h=True)


def inverse(ops: Sequence[Op]) -> List[Op]:
    """The adjoint circuit: the gates in reverse order, each inverted (H, X,
    Z, CNOT, CZ, SWAP are their own inverses; T and S become PHASESHIFT by
    -pi/4 and -pi/2; rotations and phases take the negated angle). The
    CZ / CPHASE condition mask is whatever the state's mode makes of the same
    operands, so the inverse holds in both mask modes."""
    out: List[Op] = []
    for op in reversed(list(ops)):
        c = op.opcode
        if c in (H, X, Z, CNOT, CZ, SWAP):
            out.append(Op(c, op.qubits))
        elif c == T:
            out.append(Op(P, op.qubits, -math.pi / 4))
        elif c == S:
            out.append(Op(P, op.qubits, -math.pi / 2))
        elif c in (RX, RY, RZ, P, CPHASE):
            out.append(Op(c, op.qubits, -op.angle))
        else:
            raise ValueError(f"no inverse for opcode {c:#x}")
    return out


def qft(n: int, with_swaps: bool = True) -> List[Op]:
    """Quantum Fourier transform: for q = n-1 .. 0: H(q), then CPHASE(c, q,
    pi/2^k) for the lower qubits c = q-1 .. 0 (k = 1, 2, ...); then the swap
    network (q, n-1-q). n H + n(n-1)/2 CPHASE + floor(n/2) SWAP gates."""
    ops: List[Op] = []
    for q in range(n - 1, -1, -1):
        ops.append(Op(H, [q]))
        for k, c in enumerate(range(q - 1, -1, -1), start=1):
            ops.append(Op(CPHASE, [c, q], math.pi / (2 ** k)))
    if with_swaps:
        for q in range(n // 2):
            ops.append(Op(SWAP, [q, n - 1 - q]))
    return ops


def variational(n: int, layers: int, rng: SplitMix64) -> List[Op]:
    """Hardware-efficient ansatz: per layer RY and RZ on every qubit (angles
    U[-pi, pi)), then a CZ ladder on (i, i+1)."""
    ops: List[Op] = []
    for _ in range(layers):
        for q in range(n):
            ops.append(Op(RY, [q], (rng.uniform() * 2.0 - 1.0) * math.pi))
            ops.append(Op(RZ, [q], (rng.uniform() * 2.0 - 1.0) * math.pi))
        for q in range(n - 1):
            ops.append(Op(CZ, [q, q + 1]))
    return ops


def variational_batch(count: int = 4096, nmin: int = 8, nmax: int = 22, lmin: int = 2, lmax: int = 12,
                      nmasks: int = 8, seed: int = 3):
    """`count` variational circuits with n ~ U{nmin..nmax}, L ~ U{lmin..lmax}
    and `nmasks` Z-string masks each (every qubit in a mask with p = 0.5)."""
    rng = SplitMix64(seed)
    out = []
    for _ in range(count):
        n = nmin + rng.below(nmax - nmin + 1)
        L = lmin + rng.below(lmax - lmin + 1)
        ops = variational(n, L, rng)
        masks = []
        for _ in range(nmasks):
            m = 0
            for q in range(n):
                if rng.uniform() < 0.5:
                    m |= 1 << q
            masks.append(m)
        out.append({"n": n, "layers": L, "ops": ops, "masks": masks})
    return out


def gate_count(ops: Sequence[Op]) -> int:
    """Gates after ENTANGLE* expansion (EBELL = 2, EMULTI = len, ECLUSTER = 2 len - 1)."""
    c = 0
    for op in ops:
        if op.opcode == EBELL:
            c += 2
        elif op.opcode == EMULTI:
            c += len(op.qubits)
        elif op.opcode == ECLUSTER:
            c += max(2 * len(op.qubits) - 1, 0)
        elif op.opcode in (ESWAP,):
            c += 3
        elif op.opcode in (QINIT, EDIST):
            pass
        else:
            c += 1
    return c


def algorithmic_bytes(ops: Sequence[Op], n: int, quirk: bool = False) -> float:
    """Per-gate algorithmic HBM bytes (S = 2^n * 16): H/RX/RY/RZ 2S; P/T/S/Z
    and singly-controlled X S; CZ/CPHASE 2S/2^popcount(mask)."""
    S = 16.0 * (1 << n)
    tot = 0.0
    for op in ops:
        g = op.opcode
        if g in (H, RX, RY, RZ, Y, U1):
            tot += 2 * S
        elif g in (X,):
            tot += 2 * S
        elif g in (T, S, P, Z, PHASE, SETPHASE, CNOT):
            tot += S
        elif g in (CZ, CPHASE):
            c, t = op.qubits[:2]
            m = (c | t) if quirk else ((1 << c) | (1 << t))
            tot += 2 * S / (1 << bin(m).count("1"))
        elif g == SWAP:
            tot += S
        else:
            tot += 2 * S
    return tot
