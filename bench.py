#!/usr/bin/env python3
"""Benchmark of the FP64 gate-application path.

Workload (one step): the 30-qubit random layered circuit — H on every qubit,
then 20 layers of (a 1-qubit gate on each of the 30 qubits from {H, T, S, RX,
RY, RZ, PHASESHIFT}, then CNOT/CZ/CPHASE on 15 disjoint random pairs) = 930
gates on a 16 GiB complex128 state from |0..0>, reference CZ/CPHASE mask
semantics. Seeded synthetic circuit (no dataset involved).

  value  gates/s with the state resident in HBM (device time, CUDA events on
         the engine's stream, max over ranks)
  e2e    gates/s through the public C ABI call sequence with host buffers:
         reset, qoa_apply of the host op list, qoa_get_state into pinned host
         memory (16 GiB device->host each step), wall clock; two states
         alternate so each step's copy overlaps the next step's gates
  roofline  the tile-pass kernel: 2 x 16 GiB algorithmic bytes per launch over
         its CUDA-event duration, against MEASURED_PEAKS.json hbm_gbs

--impl reference times the reference's CPU algorithm (the oracle restatement,
gate loops single-threaded as on x86-64, normalize on all cores) on the same
circuit, a bounded number of gates per step.

Multi-GPU: independent replicas, one per rank (the path has no exchange step);
value = all ranks' gates / max rank time.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = {"workload": "random layered circuit, H layer + 20 layers", "n_qubits": 30, "depth": 20, "gates": 930,
            "state_bytes": 16 << 30, "dtype": "complex128", "cz_mask": "reference (index-as-mask)",
            "l2_policy": "inputs larger than L2 (16 GiB state)", "seed": 1}


def set_workload(n: int, depth: int):
    """Smaller instances of the same circuit family (profiling captures)."""
    WORKLOAD.update(n_qubits=n, depth=depth, gates=n + depth * (n + n // 2), state_bytes=16 << n,
                    workload=f"random layered circuit, H layer + {depth} layers",
                    l2_policy="inputs larger than L2" if (16 << n) > (126 << 20) else "state fits in L2")


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def aggregate(elapsed_ms: float, units: float, device=None):
    """Max elapsed and summed units over ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return elapsed_ms, units
    t = torch.tensor([elapsed_ms], dtype=torch.float64, device=device)
    u = torch.tensor([units], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item())


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def pass_traffic_bytes(n: int, kernel: str):
    """DRAM bytes per tile-pass launch at n qubits: the ncu-measured bytes per
    amplitude of a smaller capture of the same kernel (profiles/
    ncu_counters.json, written from the capture's dram__bytes_read.sum +
    dram__bytes_write.sum), scaled by the amplitudes (traffic grows with
    them). None when no capture of that kernel is recorded."""
    p = os.path.join(ROOT, "profiles", "ncu_counters.json")
    try:
        rec = json.load(open(p))[kernel]
        return float(rec["dram_bytes"]) / float(1 << int(rec["n_qubits"])) * (1 << n), rec["source"]
    except (OSError, KeyError, ValueError):
        return None, None


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


GATE_CLASS = {0x05: "H", 0x0D: "T", 0x0E: "S", 0x22: "RX", 0x23: "RY", 0x0F: "RZ", 0x08: "P", 0x17: "CNOT",
              0x1E: "CZ", 0x35: "CPHASE"}
CPU_FORMULA = ("gates/s = G / sum_c N_c * t_c: t_c = measured seconds of one class-c gate of the circuit on the "
               "faithful oracle (single-thread gate loop + all-core normalize), N_c = class-c gates in the circuit, "
               "G = sum_c N_c; every page of the state is written once, untimed, before the first timing")


def gate_classes(ops_arr):
    """(class -> count in the circuit, class -> index of its first gate)."""
    counts, first = {}, {}
    for i, op in enumerate(ops_arr):
        c = GATE_CLASS.get(int(op["opcode"]), "other")
        counts[c] = counts.get(c, 0) + 1
        first.setdefault(c, i)
    return counts, first


def extrapolate(times: dict, counts: dict) -> float:
    """Gates/s of the whole circuit from per-class mean gate times (a class
    not timed yet takes the mean of all timed gates)."""
    timed = [t for v in times.values() for t in v]
    mean_all = sum(timed) / len(timed)
    tot = sum(counts[c] * (sum(times[c]) / len(times[c]) if times.get(c) else mean_all) for c in counts)
    return sum(counts.values()) / tot


class CpuGateTimer:
    """The oracle in the reference's time profile on an n-qubit state, timing
    one gate at a time by class (the state is touched once, untimed)."""

    def __init__(self, n, ops_arr):
        from oracle import pyoracle as po
        self.po = po
        po.set_fast(False)
        self.st = po.OracleState(n, 1)
        self.st.touch()
        self.ops = ops_arr
        self.counts, self.first = gate_classes(ops_arr)
        self.order = [c for c in GATE_CLASS.values() if c in self.counts]
        self.times = {c: [] for c in self.order}
        self.k = 0

    def next(self) -> float:
        """Times the first gate of the next class (round robin) once."""
        c = self.order[self.k % len(self.order)]
        self.k += 1
        i = self.first[c]
        t0 = time.perf_counter()
        self.st.apply(self.ops[i:i + 1])
        dt = time.perf_counter() - t0
        self.times[c].append(dt)
        return dt

    def value(self) -> float:
        return extrapolate(self.times, {c: self.counts[c] for c in self.order})

    def record(self) -> dict:
        return {"per_class_s": {c: sum(v) / len(v) for c, v in self.times.items() if v},
                "class_counts": {c: self.counts[c] for c in self.order}, "formula": CPU_FORMULA}

    def threads(self) -> int:
        return int(self.po.lib.orc_get_max_threads())

    def close(self):
        self.st.close()


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from qoa_b200 import circuits as C  # the generators only: no GPU library is opened
    n = WORKLOAD["n_qubits"]
    ops = C.ops_to_array(C.layered_h_workload(n, WORKLOAD["depth"], WORKLOAD["seed"]))
    timer = CpuGateTimer(n, ops)
    for _ in range(args.warmup):
        timer.next()
    timer.times = {c: [] for c in timer.order}
    dt = 0.0
    for _ in range(args.steps):
        dt += timer.next()
    value = timer.value()
    threads = timer.threads()
    line = {"impl": "reference", "metric": "gates/s", "value": value, "unit": "gates/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(WORKLOAD),
            "cpu_baseline": dict({"value": value, "unit": "gates/s", "cores": threads, "kind": "port",
                                  "sample": f"one gate per step, gate classes in turn (first gate of each class "
                                            f"of the {len(ops)}-gate circuit at n={n}), faithful oracle; "
                                            "extrapolated to the circuit's class mix"}, **timer.record()),
            "e2e": {"value": value, "unit": "gates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    timer.close()
    return 0


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    ws, rank, local = dist_env()
    if ws > 1:
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    import qoa_b200 as qb
    from qoa_b200 import circuits as C

    n = WORKLOAD["n_qubits"]
    ops_list = C.layered_h_workload(n, WORKLOAD["depth"], WORKLOAD["seed"])
    ops = C.ops_to_array(ops_list)
    G = len(ops)

    st = qb.QuantumState(n, compat_mask_quirk=True)
    stream = torch.cuda.ExternalStream(st.stream_ptr(), device=dev)

    def step():
        st.apply_reset_all()
        st.execute(ops)

    st.set_jit(JIT_MODES[args.jit])
    for _ in range(max(args.warmup, 0)):
        step()
    # the warm-up's second sighting of each pass requested its generated
    # kernel; wait for the compiles, then one more untimed step on them
    qb.jit_wait()
    step()
    st.sync()
    if ws > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = st.launch_count()
    j0 = st.jit_stats()["launches"]
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    st.sync()
    torch.cuda.synchronize()
    launches = st.launch_count() - l0
    jit = st.jit_stats()
    jit_timed = jit["launches"] - j0
    elapsed = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    tmax, units = aggregate(elapsed, float(G * args.steps), dev if ws > 1 else None)
    value = units / (tmax / 1e3)
    ms_per_step = tmax / args.steps

    # ---- roofline: per-launch times of the tile-pass kernel ----
    prof = qb.QuantumState(n, compat_mask_quirk=True, profile=True)
    prof.set_jit(JIT_MODES[args.jit])
    prof.apply_reset_all()
    prof.execute(ops)
    prof.sync()
    prof.launch_times()  # drop the warm-up records
    prof.apply_reset_all()
    prof.execute(ops)
    ms, by, kind = prof.launch_times()
    prof_jit = prof.jit_stats()["launches"]
    prof.close()
    streamed = os.environ.get("QOA_JIT_STREAM", "0") in ("1", "3")
    traffic, traffic_src = pass_traffic_bytes(n, ("qoa_jit_pass (streamed, complex128)" if streamed else
                                                  "qoa_jit_pass (complex128)") if prof_jit > 0 else "k_pass (complex128)")
    pass_ms = ms[kind == 0]
    pass_bytes = by[kind == 0]
    peak, peak_src = measured_peaks()
    avg_ms = float(pass_ms.mean()) if pass_ms.size else float("nan")
    achieved = float(pass_bytes.mean() / (avg_ms / 1e3) / 1e9) if pass_ms.size else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None,
                "traffic": traffic, "traffic_source": traffic_src,
                "kernel": "qoa_jit_pass_* (generated tile pass)" if prof_jit > 0 else "k_pass (interpreter)",
                "launches_per_step": int(pass_ms.size), "avg_launch_ms": avg_ms,
                "algorithmic_bytes_per_launch": float(pass_bytes.mean()) if pass_ms.size else None,
                "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peak_src})",
                "pass_share_of_step": float(pass_ms.sum() / ms.sum()) if ms.size else None}

    # ---- e2e: host op list in, full state out to pinned host memory ----
    e2e = None
    if not args.no_e2e:
        # Public-API steps with host buffers: reset, qoa_apply of the host op
        # list, qoa_get_state into pinned host memory. Two states alternate
        # so that step i's 16 GiB device->host copy (its own host thread)
        # overlaps step i+1's gates; every copy finishes inside the timed
        # region (wall clock).
        host = torch.empty((1 << n) * 2, dtype=torch.float64, pin_memory=True)
        hv = host.numpy().view(np.complex128)
        st2 = qb.QuantumState(n, compat_mask_quirk=True)
        st2.set_jit(JIT_MODES[args.jit])
        states = [st, st2]

        def copy_out(s):
            s.get_state_vector(out=hv)

        for s_ in states:  # warm-up
            s_.apply_reset_all()
            s_.execute(ops)
            copy_out(s_)
        if ws > 1:
            dist.barrier()
        k = max(1, min(args.steps, args.e2e_steps))
        t0 = time.perf_counter()
        th = None
        for i in range(k):
            s_ = states[i % 2]
            s_.apply_reset_all()
            s_.execute(ops)
            if th is not None:
                th.join()
            th = threading.Thread(target=copy_out, args=(s_,))
            th.start()
        th.join()
        wall = time.perf_counter() - t0
        et, eu = aggregate(wall * 1e3, float(G * k), dev if ws > 1 else None)
        e2e = {"value": eu / (et / 1e3), "unit": "gates/s", "h2d_bytes_per_step": int(ops.nbytes),
               "d2h_bytes_per_step": int(hv.nbytes), "steps": k, "wall_s": wall,
               "timing": "wall clock, max over ranks; two states alternate so copies overlap the next step"}
        st2.close()
        del host

    # ---- parity at full size (untimed): the same circuit on the per-gate
    # kernels (no passes, no scheduler), and the circuit followed by its
    # inverse, which must give back |0..0>; the oracle itself is checked
    # against these plans in the tests (26 and 28 qubits, and 30 in the slow test)
    parity = None
    if not args.no_parity:
        with qb.QuantumState(n, compat_mask_quirk=True, per_gate=True) as pg:
            pg.execute(ops)
            st.apply_reset_all()
            st.execute(ops)
            r_pg, f_pg = st.compare(pg)
        inv = C.ops_to_array(C.inverse(ops_list))
        st.execute(inv)
        with qb.QuantumState(n, compat_mask_quirk=True) as zero:
            r_inv, f_inv = st.compare(zero)
        parity = {"vs_per_gate_kernels_rel_l2": r_pg, "vs_per_gate_kernels_infidelity": f_pg,
                  "inverse_roundtrip_rel_l2": r_inv, "inverse_roundtrip_infidelity": f_inv,
                  "tolerance": 1e-12,
                  "note": "full-size checks: the pass plan against the per-gate kernels, and circuit + inverse "
                          "= identity; the oracle is compared on the same plans at 26 and 28 qubits (tests) and on this 30-qubit circuit by the slow test (QOA_SLOW_TESTS=1)"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        timer = CpuGateTimer(n, ops)
        spent = 0.0
        while spent < args.cpu_seconds and timer.k < args.cpu_gates:
            spent += timer.next()
        cpu = dict({"value": timer.value(), "unit": "gates/s", "cores": timer.threads(), "kind": "port",
                    "sample": f"{timer.k} gates, one per gate class in turn (the first gate of each class of the "
                              f"same {G}-gate circuit at n={n}), faithful oracle; extrapolated to the circuit's "
                              "class mix"}, **timer.record())
        timer.close()

    frm = None
    if rank == 0 and ws == 1 and not args.no_forms:
        st.close()
        frm = forms(args, ops)

    if rank == 0:
        line = {"metric": "gates/s", "value": value, "unit": "gates/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": dict(WORKLOAD),
                "fusion": {"per_gate_algorithmic_bytes": C.algorithmic_bytes(ops_list, n, quirk=True),
                           "pass_algorithmic_bytes": roofline["algorithmic_bytes_per_launch"] *
                           roofline["launches_per_step"] if roofline["algorithmic_bytes_per_launch"] else None,
                           "note": "bytes the reference's per-gate sweeps would move for one circuit, against "
                                   "the bytes the fused tile passes move"},
                "gpu_launches": int(launches), "clocks": clk, "roofline": roofline, "cpu_baseline": cpu,
                "parity": parity, "forms": frm,
                "e2e": e2e, "impl": "qoa_b200",
                "jit": {"mode": args.jit, "generated_pass_launches_timed": int(jit_timed),
                        "kernels_compiled": int(jit["kernels"]), "compile_ms_total": jit["compile_ms"],
                        "note": "pass kernels compiled once per pass structure during warm-up (NVRTC, "
                                "16 host threads), cached for the process"}}
        print(json.dumps(line), flush=True)
    st.close()
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_qft(args):
    """Precision form: QFT (H + CPHASE(pi/2^k) ladder + swap network) on a seeded
    Gaussian state. FP32-fused (complex64, <=5-qubit blocks on the tensor cores)
    at n = args.qft_qubits for throughput; FP64 plain and FP32-fused both at
    n - 1 for gates/s side by side and for relative L2 / 1 - F between them."""
    import torch
    import qoa_b200 as qb
    from qoa_b200 import circuits as C

    n = args.qft_qubits
    dev = torch.device("cuda", 0)

    def timed(st, ops, steps, warmup, kind):
        stream = torch.cuda.ExternalStream(st.stream_ptr(), device=dev)
        for _ in range(warmup):
            st.execute(ops)
        qb.jit_wait()  # generated pass kernels requested during the warm-up
        st.execute(ops)
        st.sync()
        st.launch_times()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            st.execute(ops)
        e1.record(stream)
        st.sync()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        lm, lb, lk = st.launch_times()
        sel = lk == kind
        passes = int(sel.sum() // steps)
        bw = float(lb[sel].sum() / (lm[sel].sum() / 1e3) / 1e9) if sel.any() else None
        return ms, passes, bw, float(lm[sel].mean()) if sel.any() else None

    out = {"metric": "QFT gates/s, FP32-fused vs FP64 plain", "unit": "gates/s", "impl": "qoa_b200",
           "data": "synthetic (seeded Gaussian input state)", "higher_is_better": True, "n_gpus": 1,
           "steps": args.steps, "warmup": args.warmup}
    ops_n = C.ops_to_array(C.qft(n))
    with qb.QuantumState(n, precision="f32", profile=True) as st:
        st.set_random_state(2)
        ms, passes, bw, avg = timed(st, ops_n, args.steps, args.warmup, 3)
        generated = st.jit_stats()["launches"] > 0
    peak, src = measured_peaks()
    out.update(value=len(ops_n) / (ms / 1e3), dtype="complex64 (FP32 tile passes, FP64-built coefficients)",
               config={"workload": f"QFT n={n}", "gates": len(ops_n), "state_bytes": 8 << n},
               ms_per_step=ms, fp32_passes=passes,
               roofline={"bound": "hbm", "achieved": bw, "peak": peak, "unit": "GB/s",
                         "frac": bw / peak if bw else None,
                         "kernel": "qoa_jit_pass32_* (generated complex64 tile pass)" if generated
                         else "k_pass_p32x2 (interpreter)", "avg_launch_ms": avg,
                         "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({src})"})
    m = n - 1
    ops_m = C.ops_to_array(C.qft(m))
    with qb.QuantumState(m, profile=True) as s64:
        s64.set_random_state(2)
        ms64, p64, bw64, _ = timed(s64, ops_m, args.steps, args.warmup, 0)
    with qb.QuantumState(m, precision="f32", profile=True) as s32:
        s32.set_random_state(2)
        ms32, p32, bw32, _ = timed(s32, ops_m, args.steps, args.warmup, 3)
    with qb.QuantumState(m, precision="f32", profile=True, f32_tensor=True) as s32t:
        s32t.set_random_state(2)
        ms32t, p32t, bw32t, _ = timed(s32t, ops_m, args.steps, args.warmup, 2)
    # accuracy: one QFT from the same input on both precisions
    acc = {}
    for tensor in (False, True):
        with qb.QuantumState(m) as a, qb.QuantumState(m, precision="f32", f32_tensor=tensor) as b:
            a.set_random_state(2)
            b.set_random_state(2)
            a.execute(ops_m)
            b.execute(ops_m)
            acc[tensor] = b.compare(a)
    out.update(at_n_minus_1={"n": m, "fp64_gates_s": len(ops_m) / (ms64 / 1e3),
                             "fp32_gates_s": len(ops_m) / (ms32 / 1e3), "fp32_over_fp64": ms64 / ms32,
                             "fp32_tensor_gates_s": len(ops_m) / (ms32t / 1e3),
                             "fp32_tensor_over_fp64": ms64 / ms32t,
                             "fp64_ms": ms64, "fp32_ms": ms32, "fp32_tensor_ms": ms32t,
                             "fp64_pass_launches": p64, "fp32_pass_launches": p32, "fp32_tensor_passes": p32t,
                             "fp64_pass_gbs": bw64, "fp32_pass_gbs": bw32, "fp32_tensor_pass_gbs": bw32t,
                             "fp32_rel_l2_vs_fp64": acc[False][0], "fp32_infidelity_vs_fp64": acc[False][1],
                             "fp32_tensor_rel_l2_vs_fp64": acc[True][0],
                             "fp32_tensor_infidelity_vs_fp64": acc[True][1]})
    print(json.dumps(out), flush=True)
    return 0


def run_batch(args):
    print(json.dumps(batch_form(args)), flush=True)
    return 0


def batch_form(args) -> dict:
    """Batching form: 4096 hardware-efficient variational circuits (n ~ U{8..22},
    L ~ U{2..12} layers of RY+RZ on every qubit then a CZ ladder, 8 random
    Z-strings each), all in one batch: shared-memory persistent kernel for the
    small ones, arena tile-pass rounds for the rest, replayed as one CUDA graph.
    value = circuits/s of graph replays (device time); e2e = circuits/s of a
    fresh batch per step through the public API (host op lists in, planning,
    upload, eager launch, results out)."""
    import numpy as np
    import torch
    import qoa_b200 as qb
    from qoa_b200 import circuits as C
    from qoa_b200 import autotune

    dev = torch.device("cuda", 0)
    t0 = time.perf_counter()
    circs = C.variational_batch(count=args.batch_count, seed=3)
    for c in circs:
        c["ops"] = C.ops_to_array(c["ops"])
    gen_s = time.perf_counter() - t0
    count = len(circs)
    gates = int(sum(len(c["ops"]) for c in circs))
    out = {"metric": "circuits/s", "unit": "circuits/s", "impl": "qoa_b200", "higher_is_better": True,
           "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "scaling": "weak", "vs_baseline": None,
           "data": "synthetic (seeded variational circuits)",
           "config": {"workload": f"{count} variational circuits, n~U[8,22], L~U[2,12], RY+RZ layers + CZ ladder, "
                                  "8 Z-strings each", "circuits": count, "gates": gates, "seed": 3,
                      "l2_policy": "arena larger than L2"}}
    results = {}
    for prec in args.precisions.split(","):
        t1 = time.perf_counter()
        tuning = autotune.tune(circs, prec, sample=args.tune_sample, budget_s=args.tune_seconds) \
            if args.tune_sample > 0 else None
        tune_s = time.perf_counter() - t1
        b = qb.Batch(prec)
        if tuning:
            b.set_tuning(**tuning)
        t2 = time.perf_counter()
        for c in circs:
            b.add(c["n"], c["ops"], c["masks"])
        b.run()
        first_s = time.perf_counter() - t2
        b.run()
        # generated arena kernels requested at planning: once loaded, the
        # next run captures the graph again with them
        qb.jit_wait()
        b.run()
        info = b.info()
        jit_info = b.jit_info()
        traffic = b.traffic()
        stream = torch.cuda.ExternalStream(b.stream_ptr(), device=dev)
        for _ in range(args.warmup):
            b.launch()
        torch.cuda.synchronize()
        clocks = ClockSampler(0)
        clocks.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            b.launch()
        e1.record(stream)
        torch.cuda.synchronize()
        clk = clocks.stop()
        ms = e0.elapsed_time(e1) / args.steps
        res = b.results()
        b.close()
        results[prec] = res
        peak, peak_src = measured_peaks()
        arena_gbs = traffic["arena_pass_bytes"] / (ms / 1e3) / 1e9
        results[prec + "_line"] = {
            "value": count / (ms / 1e3), "ms_per_step": ms, "tuning": tuning or "defaults",
            "roofline": {"bound": "hbm", "achieved": arena_gbs, "peak": peak, "unit": "GB/s",
                         "frac": arena_gbs / peak, "traffic_basis": "arena tile-pass bytes (2 x state per pass) "
                         "over the whole batch step (small circuits and expectation values included in the time)",
                         "arena_pass_bytes": traffic["arena_pass_bytes"], "rounds": traffic["rounds"],
                         "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peak_src})"},
            "autotune_s": tune_s, "first_run_s": first_s, "routes": info, "clocks": clk, "jit": jit_info,
            "gates_per_s": gates / (ms / 1e3)}
    prim = args.precisions.split(",")[0]
    out.update(roofline=results[prim + "_line"]["roofline"])
    out.update(value=results[prim + "_line"]["value"], ms_per_step=results[prim + "_line"]["ms_per_step"],
               dtype="f64" if prim == "f64" else "complex64 (3xTF32)", clocks=results[prim + "_line"]["clocks"])
    for prec in args.precisions.split(","):
        out[prec] = results[prec + "_line"]
    if "f64" in results and "f32" in results:
        out["f32_vs_f64_max_abs_diff"] = float(np.max(np.abs(results["f32"] - results["f64"])))
    # e2e: a fresh batch per step through the public API
    k = max(1, args.e2e_steps)
    t3 = time.perf_counter()
    for _ in range(k):
        with qb.Batch(prim) as b:
            if results[prim + "_line"]["tuning"] != "defaults":
                b.set_tuning(**results[prim + "_line"]["tuning"])
            for c in circs:
                b.add(c["n"], c["ops"], c["masks"])
            b.run()
            r = b.results()
    e2e_s = (time.perf_counter() - t3) / k
    out["e2e"] = {"value": count / e2e_s, "unit": "circuits/s",
                  "h2d_bytes_per_step": int(sum(c["ops"].nbytes + 8 * len(c["masks"]) for c in circs)),
                  "d2h_bytes_per_step": int(r.nbytes), "steps": k,
                  "note": "wall clock: host planning + upload + eager launches + results; the generated "
                          "arena kernels of these circuits' pass structures are already in the process cache"}
    if not args.no_cpu:
        from oracle import pyoracle as po
        po.set_fast(False)
        rng = np.random.default_rng(5)
        order = rng.permutation(count)
        t_cpu, done = 0.0, 0
        for i in order:
            c = circs[i]
            st = po.OracleState(c["n"], 0)
            tt = time.perf_counter()
            st.apply(c["ops"])
            t_cpu += time.perf_counter() - tt
            st.close()
            done += 1
            if t_cpu > args.cpu_seconds:
                break
        out["cpu_baseline"] = {"value": done / t_cpu, "unit": "circuits/s", "kind": "port",
                               "cores": int(po.lib.orc_get_max_threads()),
                               "sample": f"{done} circuits drawn at random from the same batch, faithful oracle "
                                         "(per-gate loops + normalize after every gate)"}
    out["generate_s"] = gen_s
    return out


def serve_requests(count: int, seed: int = 4, nmax: int = 28, dmax: int = 200, rate: float = 2000.0):
    """Serving workload: random layered circuits (gate mix of the layered
    workload), n log-uniform in [10, nmax], depth uniform in [10, dmax],
    depolarising p = 1e-3 per gate, 64 trajectories x 16 shots, seeded per
    request; Poisson arrival gaps with mean 1/rate s."""
    import numpy as np
    from qoa_b200 import circuits as C
    rng = np.random.default_rng(seed)
    out = []
    t = 0.0
    for k in range(count):
        n = int(np.floor(np.exp(rng.uniform(np.log(10), np.log(nmax + 1)))))
        n = min(max(n, 10), nmax)
        depth = int(rng.integers(10, dmax + 1))
        t += float(rng.exponential(1.0 / rate))
        out.append(dict(n=n, depth=depth, ops=C.ops_to_array(C.random_layered(n, depth, 7000 + k)), noise_p=1e-3,
                        trajectories=64, shots=16, seed=90000 + k, arrival=t))
    return out


def run_serve(args):
    print(json.dumps(serve_form(args)), flush=True)
    return 0


def serve_stream(reqs, prec: str, workers: int) -> dict:
    """One bounded request stream through the continuous-batching server:
    completed circuits/s = requests / (last completion - first submission),
    p50 / p99 of submit-to-done latency, overall and per qubit-count bucket."""
    import numpy as np
    import qoa_b200 as qb
    with qb.Server(prec, hbm_budget_gb=150, workers=workers) as srv:
        t0 = srv.now()
        for r in reqs:
            while srv.now() - t0 < r["arrival"]:
                time.sleep(max(0.0, min(0.001, r["arrival"] - (srv.now() - t0))))
            srv.submit(r["n"], r["ops"], r["noise_p"], r["trajectories"], r["shots"], r["seed"])
        res = []
        while len(res) < len(reqs):
            res += srv.poll(timeout_ms=1000)
        st = srv.stats()
        for x in res:
            if x["status"] == 0:
                srv.take_shots(x["id"], int(x["shots"]))
    lat = np.array([x["t_done"] - x["t_submit"] for x in res])
    buckets = {}
    for lo_n, hi_n in ((10, 14), (15, 19), (20, 24), (25, 28)):
        sel = np.array([lo_n <= x["n"] <= hi_n for x in res])
        if sel.any():
            buckets[f"n{lo_n}-{hi_n}"] = {"requests": int(sel.sum()),
                                          "p50_latency_s": float(np.percentile(lat[sel], 50)),
                                          "p99_latency_s": float(np.percentile(lat[sel], 99))}
    first = min(x["t_submit"] for x in res)
    last = max(x["t_done"] for x in res)
    return {"value": len(res) / (last - first), "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)), "makespan_s": last - first,
            "failed": sum(1 for x in res if x["status"] != 0), "by_qubits": buckets,
            "peak_hbm_reserved_gb": st["peak_bytes_reserved"] / (1 << 30), "workers": workers,
            "trajectories_batched": int(st["trajectories_batched"]),
            "trajectories": int(sum(r["trajectories"] for r in reqs))}


def serve_cpu_baseline(reqs, seconds: float) -> dict:
    """The oracle in the reference's time profile (single-thread gate loops,
    all-core normalize, depolarising draws after every gate) on a sample of
    the requests: the first gates of one trajectory per sampled request are
    timed and extrapolated to the request's gates x 64 trajectories."""
    import numpy as np
    from oracle import pyoracle as po
    po.set_fast(False)
    rng = np.random.default_rng(11)
    t_req, done, spent = [], 0, 0.0
    for i in rng.permutation(len(reqs)):
        r = reqs[i]
        st = po.OracleState(r["n"], 0)
        st.touch()
        st.set_noise(1, r["noise_p"], r["seed"], 0)
        k, tt = 0, 0.0
        while k < len(r["ops"]) and tt < seconds / 4:
            t0 = time.perf_counter()
            st.apply(r["ops"][k:k + 1])
            tt += time.perf_counter() - t0
            k += 1
        st.close()
        t_req.append(tt / k * len(r["ops"]) * r["trajectories"])
        spent += tt
        done += 1
        if spent > seconds:
            break
    return {"value": len(t_req) / sum(t_req), "unit": "circuits/s", "kind": "port",
            "cores": int(po.lib.orc_get_max_threads()),
            "sample": f"{done} requests drawn at random from the stream; per request the first gates of one "
                      "noisy trajectory on the faithful oracle, extrapolated to its gates x 64 trajectories"}


def serve_form(args) -> dict:
    """Serving form: bounded Poisson request streams through the continuous-
    batching server. Per precision, first a stream offered at the top rate of
    args.serve_rates (the server saturated: its completed circuits/s is the
    capacity C and the line's value); then, for the first precision, streams
    offered at 0.5 C and 0.9 C, each sized to ~15 s of arrivals, to show the
    latency of a sustainable load. `sustainable_rate` is the highest offered
    rate whose stream completed at >= 80 % of it (a bounded stream's
    ramp-up and drain keep even an unsaturated one below 100 %)."""
    import numpy as np
    top = max(float(x) for x in str(getattr(args, "serve_rates", "2000")).split(","))
    base = serve_requests(args.serve_requests, nmax=args.serve_max_qubits, dmax=args.serve_max_depth, rate=top)
    out = {"metric": "circuits/s (served, 64 trajectories x 16 shots each), p50/p99 latency", "unit": "circuits/s",
           "impl": "qoa_b200", "higher_is_better": True, "n_gpus": 1, "steps": 1, "warmup": 0, "scaling": "weak",
           "vs_baseline": None, "data": "synthetic (seeded random layered circuits, Poisson arrivals)",
           "config": {"workload": f"{len(base)} requests, n log-uniform [10,{args.serve_max_qubits}], depth "
                                  f"U[10,{args.serve_max_depth}], p=1e-3, 64 traj x 16 shots, HBM budget 150 GB, "
                                  f"offered {top:g} req/s, then 0.5 and 0.9 of the measured capacity",
                      "requests": len(base),
                      "n_hist": np.bincount([r["n"] for r in base], minlength=41)[10:args.serve_max_qubits + 1].tolist(),
                      "gates": int(sum(len(r["ops"]) for r in base))}}
    precs = args.precisions.split(",")
    for i, prec in enumerate(precs):
        rec = serve_stream(base, prec, args.serve_workers)
        rec["offered_rate"] = top
        sweep = [rec]
        if i == 0:
            cap = rec["value"]
            for f in (0.5, 0.9):
                lam = f * cap
                cnt = max(8, min(len(base), int(lam * 15.0)))
                reqs = serve_requests(cnt, nmax=args.serve_max_qubits, dmax=args.serve_max_depth, rate=lam)
                r2 = serve_stream(reqs, prec, args.serve_workers)
                r2["offered_rate"] = lam
                r2["requests"] = cnt
                sweep.append(r2)
        # a bounded stream's completed rate includes its ramp-up and drain,
        # so a rate the server keeps up with completes at ~0.85-0.95 of it
        ok = [r["offered_rate"] for r in sweep if r["value"] >= 0.8 * r["offered_rate"]]
        out[prec] = dict(rec, sweep=[{k: r.get(k) for k in ("offered_rate", "requests", "value", "p50_latency_s",
                                                             "p99_latency_s", "by_qubits", "failed")} for r in sweep],
                         sustainable_rate=max(ok) if ok else None)
    prim = precs[0]
    out.update(value=out[prim]["value"], p50_latency_s=out[prim]["p50_latency_s"],
               p99_latency_s=out[prim]["p99_latency_s"], dtype=prim)
    if not getattr(args, "no_cpu", True):
        out["cpu_baseline"] = serve_cpu_baseline(base, getattr(args, "cpu_seconds", 10.0))
    return out


def per_gate_class_gbs(n: int, ops_arr, layer_ops: int):
    """Config 1 per gate class: the first `layer_ops` gates (the H layer and
    the first random layer) each as its own per-gate kernel (QOA_FLAG_PER_GATE)
    with CUDA-event times; GB/s per class = per-gate algorithmic bytes (2S for
    H / RX / RY / RZ, S for phase gates and CNOT, S/2 for CZ / CPHASE) over the
    class's summed kernel time."""
    import qoa_b200 as qb
    sub = ops_arr[:layer_ops]
    with qb.QuantumState(n, compat_mask_quirk=True, per_gate=True, profile=True) as st:
        st.execute(sub)
        st.sync()
        st.launch_times()
        st.apply_reset_all()
        st.execute(sub)
        st.sync()
        ms, by, kind = st.launch_times()
    gate_ms, gate_by = ms[kind == 1], by[kind == 1]
    out = {}
    if len(gate_ms) != len(sub):
        return {"error": f"{len(gate_ms)} per-gate launches for {len(sub)} gates"}
    peak, _ = measured_peaks()
    for i, op in enumerate(sub):
        c = GATE_CLASS.get(int(op["opcode"]), "other")
        d = out.setdefault(c, {"gates": 0, "ms": 0.0, "bytes": 0.0})
        d["gates"] += 1
        d["ms"] += float(gate_ms[i])
        d["bytes"] += float(gate_by[i])
    for c, d in out.items():
        d["gbs"] = d["bytes"] / (d["ms"] / 1e3) / 1e9
        d["frac_of_peak"] = d["gbs"] / peak
        d["ms_per_gate"] = d["ms"] / d["gates"]
    return out


def qft_form(n: int, steps: int, warmup: int, tensor: bool = True) -> dict:
    """QFT (H + CPHASE(pi/2^k) ladder + swap network) from a seeded Gaussian
    state at n qubits: FP64 plain and FP32-fused gates/s side by side, and
    the FP32 result's relative L2 / 1 - F against the FP64 one."""
    import torch
    import qoa_b200 as qb
    from qoa_b200 import circuits as C
    dev = torch.device("cuda", 0)
    ops = C.ops_to_array(C.qft(n))

    def timed(st, kind):
        stream = torch.cuda.ExternalStream(st.stream_ptr(), device=dev)
        for _ in range(warmup):
            st.execute(ops)
        qb.jit_wait()
        st.execute(ops)
        st.sync()
        st.launch_times()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            st.execute(ops)
        e1.record(stream)
        st.sync()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        lm, lb, lk = st.launch_times()
        sel = lk == kind
        bw = float(lb[sel].sum() / (lm[sel].sum() / 1e3) / 1e9) if sel.any() else None
        return ms, int(sel.sum() // steps), bw

    out = {"workload": f"QFT n={n} from a seeded Gaussian state", "gates": len(ops)}
    with qb.QuantumState(n, profile=True) as s64:
        s64.set_random_state(2)
        ms64, p64, bw64 = timed(s64, 0)
    with qb.QuantumState(n, precision="f32", profile=True) as s32:
        s32.set_random_state(2)
        ms32, p32, bw32 = timed(s32, 3)
    out.update(fp64_gates_s=len(ops) / (ms64 / 1e3), fp32_gates_s=len(ops) / (ms32 / 1e3),
               fp32_over_fp64=ms64 / ms32, fp64_ms=ms64, fp32_ms=ms32, fp64_passes=p64, fp32_passes=p32,
               fp64_pass_gbs=bw64, fp32_pass_gbs=bw32)
    if tensor:
        with qb.QuantumState(n, precision="f32", profile=True, f32_tensor=True) as s32t:
            s32t.set_random_state(2)
            ms32t, p32t, _ = timed(s32t, 2)
        out.update(fp32_tensor_gates_s=len(ops) / (ms32t / 1e3), fp32_tensor_over_fp64=ms64 / ms32t)
    for tens in ((False, True) if tensor else (False,)):
        with qb.QuantumState(n) as a, qb.QuantumState(n, precision="f32", f32_tensor=tens) as b:
            a.set_random_state(2)
            b.set_random_state(2)
            a.execute(ops)
            b.execute(ops)
            r, f = b.compare(a)
        key = "fp32_tensor" if tens else "fp32"
        out[key + "_rel_l2_vs_fp64"] = r
        out[key + "_infidelity_vs_fp64"] = f
    return out


def qft33_fp32(steps: int, warmup: int) -> dict:
    """FP32-fused QFT throughput at 33 qubits (64 GiB complex64)."""
    import torch
    import qoa_b200 as qb
    from qoa_b200 import circuits as C
    ops = C.ops_to_array(C.qft(33))
    with qb.QuantumState(33, precision="f32") as st:
        st.set_random_state(2)
        stream = torch.cuda.ExternalStream(st.stream_ptr(), device=torch.device("cuda", 0))
        for _ in range(warmup):
            st.execute(ops)
        qb.jit_wait()
        st.execute(ops)
        st.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            st.execute(ops)
        e1.record(stream)
        st.sync()
        ms = e0.elapsed_time(e1) / steps
    return {"n": 33, "gates": len(ops), "ms": ms, "gates_s": len(ops) / (ms / 1e3)}


def forms(args, ops_arr) -> dict:
    """The further forms on the default run, each bounded to finish in well
    under a minute: config 1 per gate class, the precision form (QFT), the
    batching form and the serving form (see each function)."""
    out = {}
    t0 = time.perf_counter()
    out["config1_per_gate_class"] = per_gate_class_gbs(WORKLOAD["n_qubits"], ops_arr,
                                                       WORKLOAD["n_qubits"] + WORKLOAD["n_qubits"] * 3 // 2)
    out["precision_qft"] = qft_form(args.forms_qft_qubits, steps=3, warmup=2, tensor=True)
    out["precision_qft"]["fp32_n33"] = qft33_fp32(steps=3, warmup=2)
    bargs = argparse.Namespace(batch_count=4096, precisions="f64,f32", tune_sample=0, tune_seconds=0.0,
                               steps=5, warmup=2, e2e_steps=1, no_cpu=False, cpu_seconds=10.0)
    b = batch_form(bargs)
    out["batch"] = {k: b[k] for k in ("config", "value", "ms_per_step", "roofline", "e2e", "cpu_baseline",
                                      "f32_vs_f64_max_abs_diff") if k in b}
    for prec in ("f64", "f32"):
        if prec in b:
            out["batch"][prec] = {k: b[prec][k] for k in ("value", "ms_per_step", "roofline", "jit", "routes")}
    sargs = argparse.Namespace(serve_requests=args.forms_serve_requests, serve_max_qubits=args.forms_serve_max_qubits,
                               serve_max_depth=200, serve_workers=16, precisions="f64,f32",
                               serve_rates=args.forms_serve_rates, cpu_seconds=10.0, no_cpu=False)
    out["serve"] = serve_form(sargs)
    out["forms_wall_s"] = time.perf_counter() - t0
    return out


JIT_MODES = {"off": 0, "async": 1, "sync": 2}


def run_case(args):
    """Profiling case: two executions of one circuit on one state, nothing
    else (no timing line). --case qft: QFT on a seeded Gaussian state;
    --case layered: the layered circuit (H layer + --depth layers)."""
    import qoa_b200 as qb
    from qoa_b200 import circuits as C
    n = args.qubits
    ops = C.ops_to_array(C.qft(n) if args.case == "qft" else C.layered_h_workload(n, args.depth, 1))
    with qb.QuantumState(n, precision=args.case_precision, compat_mask_quirk=(args.case != "qft"),
                         f32_tensor=args.case_tensor) as st:
        st.set_jit(JIT_MODES[args.jit] if args.jit != "async" else qb.QOA_JIT_SYNC)
        st.set_random_state(2)
        for _ in range(2):
            st.execute(ops)
        st.sync()
        launches = st.launch_count()
    print(json.dumps({"case": args.case, "n": n, "precision": args.case_precision, "ops": len(ops),
                      "launches": launches}), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=4)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-parity", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the precision / batch / serving forms")
    ap.add_argument("--forms-qft-qubits", type=int, default=32)
    ap.add_argument("--forms-serve-requests", type=int, default=120)
    ap.add_argument("--forms-serve-max-qubits", type=int, default=20)
    ap.add_argument("--forms-serve-rates", default="2000",
                    help="top offered request rate (req/s) of the serving streams")
    ap.add_argument("--cpu-gates", type=int, default=10)
    ap.add_argument("--cpu-seconds", type=float, default=60.0)
    ap.add_argument("--ref-gates-per-step", type=int, default=1)
    ap.add_argument("--qubits", type=int, default=30, help="smaller instances for profiling captures")
    ap.add_argument("--depth", type=int, default=20)
    ap.add_argument("--workload", default="layered", choices=["layered", "qft", "batch", "serve", "case"])
    ap.add_argument("--case", default="qft", choices=["qft", "layered"])
    ap.add_argument("--case-precision", default="f64", choices=["f64", "f32"])
    ap.add_argument("--case-tensor", action="store_true", help="complex64 case on the tensor-core block form")
    ap.add_argument("--serve-requests", type=int, default=48)
    ap.add_argument("--serve-workers", type=int, default=16)
    ap.add_argument("--serve-max-qubits", type=int, default=28)
    ap.add_argument("--serve-max-depth", type=int, default=200)
    ap.add_argument("--serve-rates", default="2000", help="offered request rates (req/s), one stream each")
    ap.add_argument("--qft-qubits", type=int, default=33)
    ap.add_argument("--batch-count", type=int, default=4096)
    ap.add_argument("--precisions", default="f64,f32")
    ap.add_argument("--tune-sample", type=int, default=256)
    ap.add_argument("--tune-seconds", type=float, default=60.0)
    ap.add_argument("--jit", default="async", choices=list(JIT_MODES),
                    help="complex128 pass kernels: generated (async / sync compile) or interpreted (off)")
    args = ap.parse_args()
    if args.workload == "qft":
        return run_qft(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "case":
        return run_case(args)
    if (args.qubits, args.depth) != (30, 20):
        set_workload(args.qubits, args.depth)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
