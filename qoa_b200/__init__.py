"""qoa_b200 — B200 (sm_100a) state-vector engine for the QOA gate-application path.

Python mirror of the reference's ``QuantumState`` (src/runtime/quantum_state.rs)
over the C ABI of ``include/qoa_cuda.h`` (``libqoa_cuda.so``, built in-tree by
``make -C qoa_b200``). Method names, argument meaning and error behaviour follow
the reference: gate methods given an out-of-range qubit print an error and do
nothing (quantum_state.rs:189-195); ``measure`` raises on a bad qubit
(quantum_state.rs:400-402). There is no CPU fallback. The CUDA library is
loaded on the first call into it, not at import, so the seeded circuit
generators (``qoa_b200.circuits``) can be used by code that never touches
the GPU engine; that first call raises ``ImportError`` when the library is
missing.
"""
from __future__ import annotations

import ctypes
import os
import sys
import threading
from typing import Iterable, Optional, Sequence

import numpy as np

from . import circuits  # noqa: F401  (seeded circuit generators)
from .circuits import OP_DTYPE, Op, ops_to_array

_HERE = os.path.dirname(os.path.abspath(__file__))
# QOA_B200_LIB points at an alternative build of the same library (A/B timing).
LIB_PATH = os.environ.get("QOA_B200_LIB") or os.path.join(_HERE, "libqoa_cuda.so")

QOA_OK, QOA_E_RANGE, QOA_E_ARG, QOA_E_OPCODE, QOA_E_CUDA, QOA_E_OOM, QOA_E_STATE, QOA_E_NOGPU = range(8)
QOA_PREC_F64 = 0
QOA_PREC_F32 = 1
QOA_FLAG_COMPAT_MASK_QUIRK = 0x1
QOA_FLAG_F32_TENSOR = 0x10
QOA_JIT_OFF, QOA_JIT_ASYNC, QOA_JIT_SYNC = 0, 1, 2
QOA_FLAG_PER_GATE = 0x2
QOA_FLAG_PROFILE = 0x4
QOA_FLAG_NOISE_GATE_QUBITS = 0x8
QOA_FLAG_SLOT_SEARCH = 0x20
QOA_PLAN_SLOT_SEARCH = 0x100  # qoa_plan only


class QoaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class QoaStatus(ctypes.Structure):
    _fields_ = [("nan_seen", ctypes.c_uint32), ("inf_seen", ctypes.c_uint32),
                ("zero_norm_resets", ctypes.c_uint32), ("copy_timeouts", ctypes.c_uint32)]


class JitStats(ctypes.Structure):
    _fields_ = [("kernels", ctypes.c_uint64), ("hits", ctypes.c_uint64), ("misses", ctypes.c_uint64),
                ("failures", ctypes.c_uint64), ("launches", ctypes.c_uint64), ("compile_ms", ctypes.c_double)]


class BatchTuning(ctypes.Structure):
    _fields_ = [("small_max_n", ctypes.c_uint32), ("small_threads", ctypes.c_uint32),
                ("small_ctas_per_sm", ctypes.c_uint32), ("streams", ctypes.c_uint32),
                ("pass_gate_budget", ctypes.c_uint32), ("f32_tensor", ctypes.c_uint32), ("jit", ctypes.c_uint32)]

    def as_dict(self) -> dict:
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class ServerConfig(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("flags", ctypes.c_uint32), ("hbm_budget_bytes", ctypes.c_uint64),
                ("workers", ctypes.c_uint32)]


class RequestC(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint32), ("ops", ctypes.c_void_p), ("nops", ctypes.c_size_t),
                ("noise_p", ctypes.c_double), ("trajectories", ctypes.c_uint32),
                ("shots_per_trajectory", ctypes.c_uint32), ("seed", ctypes.c_uint64)]


class RequestResult(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint64), ("status", ctypes.c_int), ("n", ctypes.c_uint32),
                ("precision", ctypes.c_int), ("t_submit", ctypes.c_double), ("t_admit", ctypes.c_double),
                ("t_start", ctypes.c_double), ("t_done", ctypes.c_double), ("shots", ctypes.c_uint64)]


class ServerStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in ("submitted", "done", "queued", "admitted", "trajectories_running",
                                               "states_resident", "bytes_reserved", "peak_bytes_reserved",
                                               "trajectories_batched")]


_EXTRA_SIGS: dict = {}


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"qoa_b200: {LIB_PATH} is missing; build it with `make -C qoa_b200` "
                          "(or __graft_entry__.build()). The engine has no CPU fallback.")
    lib = ctypes.CDLL(LIB_PATH)
    vp, u32, u64, sz, dbl, i32 = (ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t,
                                  ctypes.c_double, ctypes.c_int)
    P = ctypes.POINTER
    sig = {
        "qoa_create": (i32, [u32, i32, u32, P(vp)]),
        "qoa_destroy": (i32, [vp]),
        "qoa_num_qubits": (i32, [vp, P(u32)]),
        "qoa_reset_all": (i32, [vp]),
        "qoa_apply": (i32, [vp, vp, sz]),
        "qoa_measure": (i32, [vp, u32, dbl, P(u32)]),
        "qoa_sample": (i32, [vp, vp, sz, i32, vp]),
        "qoa_probabilities": (i32, [vp, vp]),
        "qoa_expect_z": (i32, [vp, vp, sz, vp]),
        "qoa_get_state": (i32, [vp, vp, sz]),
        "qoa_set_state": (i32, [vp, vp, sz]),
        "qoa_seed": (i32, [vp, u64]),
        "qoa_set_random_state": (i32, [vp, u64]),
        "qoa_compare": (i32, [vp, vp, P(dbl), P(dbl)]),
        "qoa_set_noise": (i32, [vp, i32, dbl]),
        "qoa_set_trajectory": (i32, [vp, u64]),
        "qoa_status": (i32, [vp, P(QoaStatus)]),
        "qoa_sync": (i32, [vp]),
        "qoa_stream": (i32, [vp, P(vp)]),
        "qoa_launch_count": (i32, [vp, P(u64)]),
        "qoa_launch_times": (i32, [vp, vp, vp, vp, sz, P(sz)]),
        "qoa_last_error": (ctypes.c_char_p, [vp]),
        "qoa_strerror": (ctypes.c_char_p, [i32]),
        "qoa_batch_create": (i32, [i32, u32, P(vp)]),
        "qoa_batch_add": (i32, [vp, u32, vp, sz, vp, sz, P(u32)]),
        "qoa_batch_set_tuning": (i32, [vp, P(BatchTuning)]),
        "qoa_batch_get_tuning": (i32, [vp, P(BatchTuning)]),
        "qoa_batch_run": (i32, [vp]),
        "qoa_batch_results": (i32, [vp, vp, sz]),
        "qoa_batch_launch": (i32, [vp]),
        "qoa_batch_stream": (i32, [vp, P(vp)]),
        "qoa_batch_info": (i32, [vp, P(u32), P(u32), P(u32), P(u32)]),
        "qoa_batch_traffic": (i32, [vp, P(dbl), P(u32)]),
        "qoa_batch_jit_info": (i32, [vp, P(u32), P(u32), P(u32)]),
        "qoa_batch_add_trajectory": (i32, [vp, u32, vp, sz, u64, dbl, u64, vp, u32, P(u32)]),
        "qoa_batch_shots": (i32, [vp, u32, vp, sz]),
        "qoa_batch_reset": (i32, [vp]),
        "qoa_batch_set_host_threads": (i32, [vp, u32]),
        "qoa_noise_hits": (u64, [u64, u32, u64, u32, dbl]),
        "qoa_ops_unitary": (i32, [u32, u32, vp, sz, P(i32)]),
        "qoa_batch_last_error": (ctypes.c_char_p, [vp]),
        "qoa_batch_destroy": (i32, [vp]),
        "qoa_server_create": (i32, [P(ServerConfig), P(vp)]),
        "qoa_server_submit": (i32, [vp, P(RequestC), P(u64)]),
        "qoa_server_poll": (i32, [vp, P(RequestResult), sz, P(sz), i32]),
        "qoa_server_take_shots": (i32, [vp, u64, vp, sz]),
        "qoa_server_get_stats": (i32, [vp, P(ServerStats)]),
        "qoa_server_now": (dbl, [vp]),
        "qoa_server_destroy": (i32, [vp]),
        "qoa_philox_uniform": (dbl, [u64, u32, u64, u32]),
        "qoa_state_save": (i32, [vp, ctypes.c_char_p]),
        "qoa_state_load": (i32, [ctypes.c_char_p, u32, P(vp)]),
        "qoa_state_save_json": (i32, [vp, vp, sz, ctypes.c_char_p]),
        "qoa_state_load_json": (i32, [ctypes.c_char_p, u32, P(vp), vp, sz, P(sz)]),
        "qoa_get_noise": (i32, [vp, P(ctypes.c_int), P(dbl)]),
        "qoa_get_precision": (i32, [vp, P(ctypes.c_int)]),
        "qoa_plan": (i32, [u32, u32, vp, sz, sz, vp, vp, vp, vp, vp, P(sz), P(sz)]),
        "qoa_set_jit": (i32, [vp, i32, u32]),
        "qoa_jit_wait": (i32, []),
        "qoa_jit_stats_get": (i32, [vp, P(JitStats)]),
        "qoa_jit_translate": (i32, [u32, i32, u32, vp, sz, i32, vp, sz, P(sz), P(sz)]),
        "qoa_vec_apply_hadamard": (i32, [vp, sz, dbl, dbl, sz]),
        "qoa_vec_apply_x": (i32, [vp, sz, sz]),
        "qoa_vec_apply_y": (i32, [vp, sz, sz]),
        "qoa_vec_apply_z": (i32, [vp, sz, sz]),
        "qoa_vec_apply_t": (i32, [vp, sz, sz]),
        "qoa_vec_apply_s": (i32, [vp, sz, sz]),
        "qoa_vec_apply_phaseshift": (i32, [vp, sz, sz, dbl]),
        "qoa_vec_apply_reset": (i32, [vp, sz, sz]),
        "qoa_vec_apply_swap": (i32, [vp, sz, sz, sz]),
        "qoa_vec_apply_controlled_swap": (i32, [vp, sz, sz, sz, sz]),
        "qoa_vec_apply_rx": (i32, [vp, sz, sz, dbl]),
        "qoa_vec_apply_ry": (i32, [vp, sz, sz, dbl]),
        "qoa_vec_apply_rz": (i32, [vp, sz, sz, dbl]),
        "qoa_vec_apply_cnot": (i32, [vp, sz, sz, sz]),
        "qoa_vec_apply_cz": (i32, [vp, sz, sz, sz]),
        "qoa_vec_apply_controlled_phase_rotation": (i32, [vp, sz, sz, sz, dbl]),
        "qoa_vec_apply_reset_all": (i32, [vp, sz]),
    }
    sig.update(_EXTRA_SIGS)
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


class _Library:
    """libqoa_cuda.so, opened (and its signatures declared) on first use."""

    def __init__(self):
        self._cdll = None
        self._lock = threading.Lock()

    def _get(self) -> ctypes.CDLL:
        if self._cdll is None:
            with self._lock:
                if self._cdll is None:
                    self._cdll = _load()
        return self._cdll

    @property
    def loaded(self) -> bool:
        return self._cdll is not None

    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        return getattr(self._get(), name)


lib = _Library()


def register_signatures(sigs: dict):
    """Declares result and argument types of further entry points (used by
    the submodules); applied at load, or at once if the library is open."""
    _EXTRA_SIGS.update(sigs)
    if lib.loaded:
        for name, (res, args) in sigs.items():
            f = getattr(lib._cdll, name)
            f.restype = res
            f.argtypes = args


def _check(rc: int, h=None, allow_range: bool = False) -> int:
    if rc == QOA_OK:
        return rc
    msg = (lib.qoa_last_error(h) or b"").decode(errors="replace")
    if rc == QOA_E_RANGE and allow_range:
        # QuantumState prints the error and leaves the state untouched
        print(f"error: {msg}", file=sys.stderr)
        return rc
    raise QoaError(rc, msg or lib.qoa_strerror(rc).decode())


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class NoiseConfig:
    """NoiseConfig (quantum_state.rs:15-24): Random, Fixed(p) or Ideal."""

    def __init__(self, kind: str, p: float = 0.0):
        if kind not in ("random", "fixed", "ideal"):
            raise ValueError(kind)
        self.kind, self.p = kind, float(p)

    @classmethod
    def Random(cls):
        return cls("random")

    @classmethod
    def Fixed(cls, p: float):
        return cls("fixed", p)

    @classmethod
    def Ideal(cls):
        return cls("ideal")

    @property
    def mode(self) -> int:
        return {"ideal": 0, "fixed": 1, "random": 2}[self.kind]


class QuantumState:
    """Dense complex128 state vector resident in HBM (QuantumState::new,
    quantum_state.rs:56-90)."""

    def __init__(self, n_qubits: int, noise_config: Optional[NoiseConfig] = None, *,
                 compat_mask_quirk: bool = False, per_gate: bool = False, profile: bool = False,
                 noise_gate_qubits_only: bool = False, seed: int = 0, precision: str = "f64",
                 f32_tensor: bool = False, slot_search: bool = False):
        flags = ((QOA_FLAG_F32_TENSOR if f32_tensor else 0)
                 | (QOA_FLAG_SLOT_SEARCH if slot_search else 0)
                 | (QOA_FLAG_COMPAT_MASK_QUIRK if compat_mask_quirk else 0)
                 | (QOA_FLAG_PER_GATE if per_gate else 0)
                 | (QOA_FLAG_PROFILE if profile else 0)
                 | (QOA_FLAG_NOISE_GATE_QUBITS if noise_gate_qubits_only else 0))
        if precision not in ("f64", "f32"):
            raise ValueError("precision must be 'f64' or 'f32'")
        self.precision = precision
        self._dtype = np.complex64 if precision == "f32" else np.complex128
        h = ctypes.c_void_p()
        _check(lib.qoa_create(max(int(n_qubits), 1), QOA_PREC_F32 if precision == "f32" else QOA_PREC_F64, flags,
                              ctypes.byref(h)))
        self._h = h
        self.flags = flags
        self.noise_config = noise_config
        self.seed_rng(seed)
        if noise_config is not None:
            self.set_noise_config(noise_config)

    @classmethod
    def _adopt(cls, h, precision: str, flags: int) -> "QuantumState":
        self = cls.__new__(cls)
        self.precision = precision
        self._dtype = np.complex64 if precision == "f32" else np.complex128
        self._h = h
        self.flags = flags
        self.noise_config = None
        return self

    # ---- checkpoints (--save-state / --load-state, main.rs:3800-3830, 4290-4300) ----
    def save(self, path: str):
        """Exact binary checkpoint (stored amplitudes + norm2)."""
        _check(lib.qoa_state_save(self._h, os.fsencode(path)), self._h)

    @classmethod
    def load(cls, path: str, flags: int = 0) -> "QuantumState":
        h = ctypes.c_void_p()
        _check(lib.qoa_state_load(os.fsencode(path), flags, ctypes.byref(h)))
        p = ctypes.c_int()
        _check(lib.qoa_get_precision(h, ctypes.byref(p)), h)
        st = cls._adopt(h, "f32" if p.value == QOA_PREC_F32 else "f64", flags)
        m, q = ctypes.c_int(), ctypes.c_double()
        _check(lib.qoa_get_noise(h, ctypes.byref(m), ctypes.byref(q)), h)
        st.noise_config = [None, NoiseConfig.Fixed(q.value), NoiseConfig.Random()][m.value]
        return st

    def save_json(self, path: str, registers: Sequence[float] = ()):
        """The reference's serde JSON checkpoint of (QuantumState, registers)."""
        r = np.ascontiguousarray(np.asarray(list(registers), dtype=np.float64))
        _check(lib.qoa_state_save_json(self._h, _ptr(r) if len(r) else None, len(r), os.fsencode(path)), self._h)

    @classmethod
    def load_json(cls, path: str, flags: int = 0):
        """(state, registers) from a reference JSON checkpoint."""
        h = ctypes.c_void_p()
        n = ctypes.c_size_t()
        _check(lib.qoa_state_load_json(os.fsencode(path), flags, ctypes.byref(h), None, 0, ctypes.byref(n)))
        lib.qoa_destroy(h)
        regs = np.zeros(n.value, dtype=np.float64)
        h = ctypes.c_void_p()
        _check(lib.qoa_state_load_json(os.fsencode(path), flags, ctypes.byref(h), _ptr(regs) if len(regs) else None,
                                       len(regs), ctypes.byref(n)))
        st = cls._adopt(h, "f64", flags)
        m, p = ctypes.c_int(), ctypes.c_double()
        _check(lib.qoa_get_noise(h, ctypes.byref(m), ctypes.byref(p)), h)
        st.noise_config = [None, NoiseConfig.Fixed(p.value), NoiseConfig.Random()][m.value]
        return st, regs

    # ---- lifetime -------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            lib.qoa_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    @property
    def n(self) -> int:
        v = ctypes.c_uint32()
        _check(lib.qoa_num_qubits(self._h, ctypes.byref(v)), self._h)
        return int(v.value)

    def get_num_qubits(self) -> int:
        return self.n

    # ---- bulk execution ---------------------------------------------------
    def execute(self, ops) -> int:
        """Applies an op list (qoa_op records, reference opcode numbers)."""
        arr = ops if isinstance(ops, np.ndarray) else ops_to_array(ops)
        if arr.dtype != OP_DTYPE:
            raise TypeError("ops must use circuits.OP_DTYPE")
        arr = np.ascontiguousarray(arr)
        return _check(lib.qoa_apply(self._h, _ptr(arr), len(arr)), self._h, allow_range=True)

    def _one(self, opcode: int, *qs: int, angle: float = 0.0, matrix=None) -> int:
        return self.execute([Op(opcode, list(qs), angle, matrix)])

    # ---- gate methods (quantum_state.rs:171-397, 960-1212) -----------------
    def apply_h(self, q): return self._one(0x05, q)
    def apply_x(self, q): return self._one(0x07, q)
    def apply_y(self, q): return self._one(0xF0, q)
    def apply_phase_flip(self, q): return self._one(0x06, q)
    def apply_t_gate(self, q): return self._one(0x0D, q)
    def apply_s_gate(self, q): return self._one(0x0E, q)
    def apply_phase_shift(self, q, angle): return self._one(0x08, q, angle=angle)
    def apply_rx(self, q, angle): return self._one(0x22, q, angle=angle)
    def apply_ry(self, q, angle): return self._one(0x23, q, angle=angle)
    def apply_rz(self, q, angle): return self._one(0x0F, q, angle=angle)
    def apply_cnot(self, c, t): return self._one(0x17, c, t)
    def apply_cz(self, c, t): return self._one(0x1E, c, t)
    def apply_controlled_phase(self, c, t, angle): return self._one(0x35, c, t, angle=angle)
    def apply_swap(self, a, b): return self._one(0x0B, a, b)
    def apply_controlled_swap(self, c, a, b): return self._one(0x0C, c, a, b)
    def apply_toffoli(self, c1, c2, t): return self._one(0xF3, c1, c2, t)
    def apply_controlled_y(self, c, t): return self._one(0xF4, c, t)
    def reset_qubit(self, q): return self._one(0x0A, q)
    def apply_reset_all(self): return _check(lib.qoa_reset_all(self._h), self._h)

    def apply_custom_unitary(self, q, u: Sequence[complex]):
        m = np.ascontiguousarray(np.asarray(u, dtype=np.complex128).reshape(4))
        return self._one(0xF1, q, matrix=m)

    def apply_two_qubit_unitary(self, q1, q2, u: Sequence[complex]):
        m = np.ascontiguousarray(np.asarray(u, dtype=np.complex128).reshape(16))
        return self._one(0xF2, q1, q2, matrix=m)

    # ---- measurement --------------------------------------------------------
    def measure(self, q: int, u: Optional[float] = None) -> int:
        """measure (quantum_state.rs:399-458): outcome = (u < P0) ? 0 : 1. Without
        `u` the handle's seeded Philox stream supplies the draw."""
        out = ctypes.c_uint32()
        _check(lib.qoa_measure(self._h, int(q), -1.0 if u is None else float(u), ctypes.byref(out)), self._h)
        return int(out.value)

    def sample(self, shots: int, u: Optional[np.ndarray] = None, mode: int = 0, rng_seed: int = 0) -> np.ndarray:
        """Shots without disturbing the state. mode 0 reproduces measure_all's
        qubit-by-qubit draw order (n uniforms per shot); mode 1 is inverse CDF."""
        n = self.n
        need = shots * n if mode == 0 else shots
        if u is None:
            u = np.random.default_rng(rng_seed).random(need)
        u = np.ascontiguousarray(np.asarray(u, dtype=np.float64).reshape(-1))
        if u.size != need:
            raise ValueError(f"need {need} uniforms")
        out = np.empty(shots, dtype=np.uint64)
        _check(lib.qoa_sample(self._h, _ptr(u), shots, mode, _ptr(out)), self._h)
        return out

    def measure_all(self, u: Optional[np.ndarray] = None) -> list:
        """measure_all (quantum_state.rs:909-918): one shot, outcome per qubit."""
        bits = int(self.sample(1, u, mode=0)[0])
        return [(bits >> q) & 1 for q in range(self.n)]

    # ---- state access -------------------------------------------------------
    def get_probabilities(self) -> np.ndarray:
        out = np.empty(1 << self.n, dtype=np.float64)
        _check(lib.qoa_probabilities(self._h, _ptr(out)), self._h)
        return out

    def get_state_vector(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        n = self.n
        if out is None:
            out = np.empty(1 << n, dtype=self._dtype)
        _check(lib.qoa_get_state(self._h, _ptr(out), out.nbytes), self._h)
        return out

    def set_state_vector(self, amps: np.ndarray):
        a = np.ascontiguousarray(np.asarray(amps, dtype=self._dtype))
        _check(lib.qoa_set_state(self._h, _ptr(a), a.nbytes), self._h)

    def set_random_state(self, seed: int):
        """Seeded Gaussian state (re, im i.i.d. N(0,1)), normalised, made on the device."""
        _check(lib.qoa_set_random_state(self._h, int(seed)), self._h)

    def compare(self, other: "QuantumState"):
        """(relative L2, 1 - fidelity) of the two normalised states."""
        r, f = ctypes.c_double(), ctypes.c_double()
        _check(lib.qoa_compare(self._h, other._h, ctypes.byref(r), ctypes.byref(f)), self._h)
        return r.value, f.value

    def expect_z(self, masks: Iterable[int]) -> np.ndarray:
        m = np.ascontiguousarray(np.asarray(list(masks), dtype=np.uint64))
        out = np.empty(len(m), dtype=np.float64)
        _check(lib.qoa_expect_z(self._h, _ptr(m), len(m), _ptr(out)), self._h)
        return out

    # ---- configuration --------------------------------------------------------
    def seed_rng(self, seed: int):
        _check(lib.qoa_seed(self._h, int(seed) & 0xFFFFFFFFFFFFFFFF), self._h)

    def set_trajectory(self, t: int):
        _check(lib.qoa_set_trajectory(self._h, int(t)), self._h)

    def set_noise_config(self, cfg: Optional[NoiseConfig]):
        self.noise_config = cfg
        mode, p = (3, 0.0) if cfg is None else (cfg.mode, cfg.p)  # 3: no config (the Option's None)
        _check(lib.qoa_set_noise(self._h, mode, p), self._h)

    def get_noise_config(self):
        return self.noise_config

    def get_status(self) -> dict:
        st = QoaStatus()
        _check(lib.qoa_status(self._h, ctypes.byref(st)), self._h)
        return {"nan": bool(st.nan_seen), "overflow": bool(st.inf_seen), "zero_norm_resets": st.zero_norm_resets,
                "copy_timeouts": st.copy_timeouts}

    # ---- engine plumbing --------------------------------------------------------
    def sync(self):
        _check(lib.qoa_sync(self._h), self._h)

    def stream_ptr(self) -> int:
        p = ctypes.c_void_p()
        _check(lib.qoa_stream(self._h, ctypes.byref(p)), self._h)
        return int(p.value or 0)

    def set_jit(self, mode: int = QOA_JIT_ASYNC, min_qubits: int = 20):
        """Generated pass kernels for this handle: QOA_JIT_OFF / _ASYNC / _SYNC,
        for states of at least min_qubits qubits."""
        _check(lib.qoa_set_jit(self._h, int(mode), int(min_qubits)), self._h)

    def jit_stats(self) -> dict:
        st = JitStats()
        _check(lib.qoa_jit_stats_get(self._h, ctypes.byref(st)), self._h)
        return {f: getattr(st, f) for f, _ in JitStats._fields_}

    def launch_count(self) -> int:
        v = ctypes.c_uint64()
        _check(lib.qoa_launch_count(self._h, ctypes.byref(v)), self._h)
        return int(v.value)

    def launch_times(self, cap: int = 1 << 16):
        ms = np.empty(cap, dtype=np.float64)
        by = np.empty(cap, dtype=np.float64)
        kd = np.empty(cap, dtype=np.int32)
        n = ctypes.c_size_t()
        _check(lib.qoa_launch_times(self._h, _ptr(ms), _ptr(by), _ptr(kd), cap, ctypes.byref(n)), self._h)
        k = n.value
        return ms[:k].copy(), by[:k].copy(), kd[:k].copy()


def plan(n: int, ops, flags: int = 0):
    """Runs the host pass scheduler without a GPU. Returns per expanded gate
    (pass index, order in pass, kind code, qubits[4], matrix[16] complex) and the
    pass count."""
    arr = np.ascontiguousarray(ops if isinstance(ops, np.ndarray) else ops_to_array(ops))
    ng, npasses = ctypes.c_size_t(), ctypes.c_size_t()
    lib.qoa_plan(n, flags, _ptr(arr), len(arr), 0, None, None, None, None, None, ctypes.byref(ng), ctypes.byref(npasses))
    cap = ng.value
    pass_of = np.empty(max(cap, 1), dtype=np.int32)
    order = np.empty(max(cap, 1), dtype=np.int32)
    kind = np.empty(max(cap, 1), dtype=np.int32)
    qubits = np.empty((max(cap, 1), 4), dtype=np.uint32)
    mat = np.empty((max(cap, 1), 16), dtype=np.complex128)
    _check(lib.qoa_plan(n, flags, _ptr(arr), len(arr), cap, _ptr(pass_of), _ptr(order), _ptr(kind), _ptr(qubits),
                        _ptr(mat), ctypes.byref(ng), ctypes.byref(npasses)))
    k = ng.value
    return {"pass_of": pass_of[:k], "order": order[:k], "kind": kind[:k], "qubits": qubits[:k],
            "matrix": mat[:k], "npasses": npasses.value}


def jit_wait():
    """Blocks until every requested pass-kernel compile has finished."""
    _check(lib.qoa_jit_wait())


def jit_stats() -> dict:
    st = JitStats()
    _check(lib.qoa_jit_stats_get(None, ctypes.byref(st)))
    return {f: getattr(st, f) for f, _ in JitStats._fields_}


def jit_translate(n: int, ops, flags: int = 0, compile: bool = False, precision: str = "f64", arena: bool = False):
    """Host only: the generated CUDA source of every tile pass of `ops` on an
    n-qubit state (precision "f64" or "f32"), and the pass count;
    compile=True also compiles it with NVRTC (raises QoaError with the log
    if it does not compile)."""
    arr = np.ascontiguousarray(ops if isinstance(ops, np.ndarray) else ops_to_array(ops))
    prec = QOA_PREC_F32 if precision == "f32" else QOA_PREC_F64
    ln, npasses = ctypes.c_size_t(), ctypes.c_size_t()
    _check(lib.qoa_jit_translate(n, prec, flags, _ptr(arr), len(arr), 2 if arena else 0, None, 0, ctypes.byref(ln),
                                 ctypes.byref(npasses)))
    buf = ctypes.create_string_buffer(ln.value + 1)
    mode = (1 if compile else 0) | (2 if arena else 0)
    _check(lib.qoa_jit_translate(n, prec, flags, _ptr(arr), len(arr), mode, buf, ln.value + 1,
                                 ctypes.byref(ln), ctypes.byref(npasses)))
    return buf.value.decode(), npasses.value


def vec_call(name: str, amps: np.ndarray, *args) -> int:
    """Calls a vectorization.rs shim (qoa_vec_apply_<name>) on a host
    complex128 array in place."""
    if amps.dtype != np.complex128 or not amps.flags.c_contiguous:
        raise TypeError("amps must be a C-contiguous complex128 array")
    f = getattr(lib, "qoa_vec_apply_" + name)
    return _check(f(_ptr(amps), amps.size, *args))


class Batch:
    """Many circuits run together (qoa_batch_*): each circuit starts in
    |0..0>, applies its unitary op list and yields <Z_mask> of its final
    normalised state for each mask given. Small circuits run whole-state in
    shared memory in one persistent launch; larger ones run as tile passes
    over one packed arena, one launch per pass round across all of them. The
    first run() launches eagerly, the second captures the batch into a CUDA
    graph, later runs replay it."""

    def __init__(self, precision: str = "f64", compat_mask_quirk: bool = False):
        if precision not in ("f64", "f32"):
            raise ValueError("precision must be 'f64' or 'f32'")
        self.precision = precision
        h = ctypes.c_void_p()
        flags = QOA_FLAG_COMPAT_MASK_QUIRK if compat_mask_quirk else 0
        rc = lib.qoa_batch_create(QOA_PREC_F32 if precision == "f32" else QOA_PREC_F64, flags, ctypes.byref(h))
        if rc != QOA_OK:
            raise QoaError(rc, (lib.qoa_last_error(None) or b"").decode())
        self._h = h
        self._nresults = 0
        self._keep = []

    def _check(self, rc: int):
        if rc != QOA_OK:
            raise QoaError(rc, (lib.qoa_batch_last_error(self._h) or b"").decode())

    def add(self, n: int, ops, zmasks: Sequence[int]) -> int:
        arr = ops if isinstance(ops, np.ndarray) else ops_to_array(ops)
        arr = np.ascontiguousarray(arr)
        m = np.ascontiguousarray(np.asarray(list(zmasks), dtype=np.uint64))
        cid = ctypes.c_uint32()
        self._check(lib.qoa_batch_add(self._h, n, _ptr(arr) if len(arr) else None, len(arr),
                                      _ptr(m) if len(m) else None, len(m), ctypes.byref(cid)))
        self._nresults += len(m)
        return cid.value

    def add_trajectory(self, n: int, ops, seed: int, noise_p: float, trajectory: int, u) -> int:
        """Trajectory `trajectory` of the noisy circuit (the draws a state
        seeded `seed` with noise level noise_p makes on that trajectory),
        sampled after the run with one inverse-CDF uniform per shot from u.
        Out-of-range ops are skipped as in qoa_apply."""
        arr = np.ascontiguousarray(ops if isinstance(ops, np.ndarray) else ops_to_array(ops))
        uu = np.ascontiguousarray(np.asarray(u, dtype=np.float64).reshape(-1))
        cid = ctypes.c_uint32()
        rc = lib.qoa_batch_add_trajectory(self._h, n, _ptr(arr) if len(arr) else None, len(arr), seed, float(noise_p),
                                          trajectory, _ptr(uu) if len(uu) else None, len(uu), ctypes.byref(cid))
        if rc != QOA_E_RANGE:
            self._check(rc)
        self._keep.append(uu)
        self._shots = getattr(self, "_shots", {})
        self._shots[cid.value] = len(uu)
        return cid.value

    def shots(self, cid: int) -> np.ndarray:
        out = np.zeros(self._shots[cid], dtype=np.uint64)
        self._check(lib.qoa_batch_shots(self._h, cid, _ptr(out) if len(out) else None, len(out)))
        return out

    def reset(self):
        """Empties the batch for reuse (circuits and device buffers go)."""
        self._check(lib.qoa_batch_reset(self._h))
        self._nresults = 0
        self._keep = []
        self._shots = {}

    def tuning(self) -> dict:
        t = BatchTuning()
        self._check(lib.qoa_batch_get_tuning(self._h, ctypes.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw):
        t = BatchTuning()
        self._check(lib.qoa_batch_get_tuning(self._h, ctypes.byref(t)))
        for k, v in kw.items():
            if not hasattr(t, k):
                raise KeyError(k)
            setattr(t, k, int(v))
        self._check(lib.qoa_batch_set_tuning(self._h, ctypes.byref(t)))

    def run(self):
        self._check(lib.qoa_batch_run(self._h))

    def launch(self):
        """Replays the captured graph without waiting (after a first run())."""
        self._check(lib.qoa_batch_launch(self._h))

    def stream_ptr(self) -> int:
        p = ctypes.c_void_p()
        self._check(lib.qoa_batch_stream(self._h, ctypes.byref(p)))
        return p.value or 0

    def results(self) -> np.ndarray:
        out = np.zeros(self._nresults, dtype=np.float64)
        self._check(lib.qoa_batch_results(self._h, _ptr(out) if len(out) else None, len(out)))
        return out

    def info(self) -> dict:
        v = [ctypes.c_uint32() for _ in range(4)]
        self._check(lib.qoa_batch_info(self._h, *[ctypes.byref(x) for x in v]))
        return dict(zip(("circuits", "small", "large", "graph_ready"), (x.value for x in v)))

    def traffic(self) -> dict:
        by, rounds = ctypes.c_double(), ctypes.c_uint32()
        self._check(lib.qoa_batch_traffic(self._h, ctypes.byref(by), ctypes.byref(rounds)))
        return {"arena_pass_bytes": by.value, "rounds": rounds.value}

    def jit_info(self) -> dict:
        """Generated arena kernels: pass structures, loaded kernels, and
        whether the captured graph launches them."""
        a, r, g = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        self._check(lib.qoa_batch_jit_info(self._h, ctypes.byref(a), ctypes.byref(r), ctypes.byref(g)))
        return {"structures": a.value, "ready": r.value, "graph_uses_generated": bool(g.value)}

    def close(self):
        if getattr(self, "_h", None):
            lib.qoa_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


SHOT_STREAM = 0x73686F74


def philox_uniform(seed: int, stream: int, event: int, slot: int) -> float:
    """The engine's counter-based uniform (Philox4x32-10; stream is 32-bit)."""
    return lib.qoa_philox_uniform(seed, stream & 0xFFFFFFFF, event, slot)


class Server:
    """Serving form (qoa_server_*): a request loop with continuous batching.
    Each request is a circuit with depolarising noise p per gate, run as
    `trajectories` Pauli trajectories of `shots` inverse-CDF shots each;
    trajectory t of a request seeded s uses counter-based streams t (noise)
    and t ^ SHOT_STREAM (shot uniforms), so its outcomes do not depend on the
    other requests or on scheduling. Admission is by HBM footprint."""

    def __init__(self, precision: str = "f64", hbm_budget_gb: float = 150.0, workers: int = 16,
                 compat_mask_quirk: bool = False):
        cfg = ServerConfig(QOA_PREC_F32 if precision == "f32" else QOA_PREC_F64,
                           QOA_FLAG_COMPAT_MASK_QUIRK if compat_mask_quirk else 0,
                           int(hbm_budget_gb * (1 << 30)), int(workers))
        h = ctypes.c_void_p()
        rc = lib.qoa_server_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != QOA_OK:
            raise QoaError(rc, (lib.qoa_last_error(None) or b"").decode())
        self._h = h

    def submit(self, n: int, ops, noise_p: float = 0.0, trajectories: int = 1, shots: int = 1,
               seed: int = 0) -> int:
        arr = np.ascontiguousarray(ops if isinstance(ops, np.ndarray) else ops_to_array(ops))
        req = RequestC(n, _ptr(arr) if len(arr) else None, len(arr), float(noise_p), int(trajectories), int(shots),
                       int(seed))
        rid = ctypes.c_uint64()
        rc = lib.qoa_server_submit(self._h, ctypes.byref(req), ctypes.byref(rid))
        if rc != QOA_OK:
            raise QoaError(rc, (lib.qoa_last_error(None) or b"").decode())
        return rid.value

    def poll(self, timeout_ms: int = -1, cap: int = 256) -> list:
        buf = (RequestResult * cap)()
        got = ctypes.c_size_t()
        _check(lib.qoa_server_poll(self._h, buf, cap, ctypes.byref(got), int(timeout_ms)))
        return [{k: getattr(buf[i], k) for k, _ in RequestResult._fields_} for i in range(got.value)]

    def take_shots(self, rid: int, count: int) -> np.ndarray:
        out = np.zeros(count, dtype=np.uint64)
        rc = lib.qoa_server_take_shots(self._h, rid, _ptr(out) if count else None, count)
        if rc != QOA_OK:
            raise QoaError(rc, (lib.qoa_last_error(None) or b"").decode())
        return out

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib.qoa_server_get_stats(self._h, ctypes.byref(st)))
        return {k: int(getattr(st, k)) for k, _ in ServerStats._fields_}

    def now(self) -> float:
        return lib.qoa_server_now(self._h)

    def close(self):
        if getattr(self, "_h", None):
            lib.qoa_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
