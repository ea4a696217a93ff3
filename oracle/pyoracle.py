"""ctypes wrapper of liboracle.so (oracle/qoa_oracle.c) — test infrastructure.

The oracle restates the reference's CPU executor (src/runtime/quantum_state.rs
and the x86-64 loops of src/vectorization.rs); it is the checker for the CUDA
engine, never part of it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _load():
    if not os.path.exists(LIB_PATH):
        build()
    lib = ctypes.CDLL(LIB_PATH)
    vp, sz, dbl, u32, u64, i32 = (ctypes.c_void_p, ctypes.c_size_t, ctypes.c_double, ctypes.c_uint32,
                                  ctypes.c_uint64, ctypes.c_int)
    sig = {
        "orc_set_fast": (None, [i32]),
        "orc_get_max_threads": (i32, []),
        "orc_new": (vp, [sz, u32]),
        "orc_free": (None, [vp]),
        "orc_touch": (None, [vp]),
        "orc_set_defer_norm": (None, [vp, i32]),
        "orc_num_qubits": (sz, [vp]),
        "orc_amps": (vp, [vp]),
        "orc_set_noise": (None, [vp, i32, dbl, u64, u64]),
        "orc_zero_resets": (u32, [vp]),
        "orc_normalize": (None, [vp]),
        "orc_measure": (i32, [vp, sz, dbl, ctypes.POINTER(u32)]),
        "orc_measure_all": (u64, [vp, vp]),
        "orc_apply": (i32, [vp, vp, sz, vp, sz]),
        "orc_set_state": (i32, [vp, vp, sz]),
        "orc_get_state": (i32, [vp, vp, sz]),
        "orc_uniform": (dbl, [u64, u64, u64, u32]),
        "orc_vec_hadamard": (None, [vp, sz, dbl, dbl, sz]),
        "orc_vec_x": (None, [vp, sz, sz]),
        "orc_vec_y": (None, [vp, sz, sz]),
        "orc_vec_z": (None, [vp, sz, sz]),
        "orc_vec_t": (None, [vp, sz, sz]),
        "orc_vec_s": (None, [vp, sz, sz]),
        "orc_vec_phaseshift": (None, [vp, sz, sz, dbl]),
        "orc_vec_reset": (None, [vp, sz, sz]),
        "orc_vec_rx": (None, [vp, sz, sz, dbl]),
        "orc_vec_ry": (None, [vp, sz, sz, dbl]),
        "orc_vec_rz": (None, [vp, sz, sz, dbl]),
        "orc_vec_cnot": (None, [vp, sz, sz, sz]),
        "orc_vec_cz": (None, [vp, sz, sz, sz]),
        "orc_vec_cphase": (None, [vp, sz, sz, sz, dbl]),
        "orc_vec_swap": (None, [vp, sz, sz, sz]),
        "orc_vec_cswap": (None, [vp, sz, sz, sz, sz]),
        "orc_vec_reset_all": (None, [vp, sz]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()

# vectorization.rs function name -> oracle symbol (same argument order)
VEC = {
    "hadamard": "orc_vec_hadamard", "x": "orc_vec_x", "y": "orc_vec_y", "z": "orc_vec_z", "t": "orc_vec_t",
    "s": "orc_vec_s", "phaseshift": "orc_vec_phaseshift", "reset": "orc_vec_reset", "rx": "orc_vec_rx",
    "ry": "orc_vec_ry", "rz": "orc_vec_rz", "cnot": "orc_vec_cnot", "cz": "orc_vec_cz",
    "controlled_phase_rotation": "orc_vec_cphase", "swap": "orc_vec_swap", "controlled_swap": "orc_vec_cswap",
    "reset_all": "orc_vec_reset_all",
}


def vec_call(name: str, amps: np.ndarray, *args):
    """Applies the restated vectorization.rs function `name` to amps in place."""
    assert amps.dtype == np.complex128 and amps.flags.c_contiguous
    getattr(lib, VEC[name])(amps.ctypes.data, amps.size, *args)


def set_fast(fast: bool):
    lib.orc_set_fast(1 if fast else 0)


class OracleState:
    """Restated QuantumState (faithful per-gate normalize, supplied uniforms)."""

    def __init__(self, n: int, flags: int = 0):
        self.h = lib.orc_new(n, flags)

    def defer_norm(self, on: bool = True):
        """Skips the per-gate normalize (noiseless unitary circuits at large n;
        call normalize() once at the end)."""
        lib.orc_set_defer_norm(self.h, 1 if on else 0)

    def normalize(self):
        lib.orc_normalize(self.h)

    def touch(self):
        """Maps every page of the state (untimed set-up before a timing)."""
        lib.orc_touch(self.h)

    def close(self):
        if self.h:
            lib.orc_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    @property
    def n(self) -> int:
        return int(lib.orc_num_qubits(self.h))

    def apply(self, ops: np.ndarray, meas_u=None) -> int:
        ops = np.ascontiguousarray(ops)
        if meas_u is None:
            return int(lib.orc_apply(self.h, ops.ctypes.data, len(ops), None, 0))
        mu = np.ascontiguousarray(np.asarray(meas_u, dtype=np.float64))
        return int(lib.orc_apply(self.h, ops.ctypes.data, len(ops), mu.ctypes.data, mu.size))

    def state(self) -> np.ndarray:
        out = np.empty(1 << self.n, dtype=np.complex128)
        lib.orc_get_state(self.h, out.ctypes.data, out.size)
        return out

    def view(self) -> np.ndarray:
        """Zero-copy view of the amplitudes (valid while the state lives)."""
        ptr = lib.orc_amps(self.h)
        buf = (ctypes.c_double * (2 << self.n)).from_address(ptr)
        return np.frombuffer(buf, dtype=np.complex128)

    def set_state(self, amps: np.ndarray) -> int:
        a = np.ascontiguousarray(np.asarray(amps, dtype=np.complex128))
        return int(lib.orc_set_state(self.h, a.ctypes.data, a.size))

    def measure(self, q: int, u: float) -> int:
        out = ctypes.c_uint32()
        rc = lib.orc_measure(self.h, q, u, ctypes.byref(out))
        if rc:
            raise ValueError(f"qubit index {q} out of bounds")
        return int(out.value)

    def measure_all(self, u) -> int:
        u = np.ascontiguousarray(np.asarray(u, dtype=np.float64))
        return int(lib.orc_measure_all(self.h, u.ctypes.data))

    def set_noise(self, mode: int, p: float, seed: int, stream: int = 0):
        lib.orc_set_noise(self.h, mode, p, seed, stream)

    def zero_resets(self) -> int:
        return int(lib.orc_zero_resets(self.h))


def uniform(seed: int, stream: int, event: int, slot: int) -> float:
    return float(lib.orc_uniform(seed, stream, event, slot))
