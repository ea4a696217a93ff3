"""Autotuner of the batching form.

Chooses the batch tuning (qoa_batch_tuning) for a workload by timing graph
replays of a sample of its circuits over a grid of candidates:

  small_max_n        where circuits switch from the whole-state-in-shared-
                     memory kernel to arena tile passes (the tile choice)
  small_threads      threads per CTA of the shared-memory kernel
  small_ctas_per_sm  its persistent grid (SMs x this)
  pass_gate_budget   max gates fused into one tile pass (the fusion width;
                     0 = as many as fit)
  f32_tensor         complex64 only: dense tensor-core blocks instead of
                     tile passes

The choice is cached in a JSON file keyed by precision, device name and a
signature of the workload's size mix, so a later process reuses it.
"""
import json
import os
import time
from typing import Dict, List, Optional

import numpy as np

DEFAULT_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "_build", "autotune.json")


def signature(circuits: List[dict]) -> str:
    ns = np.array([c["n"] for c in circuits])
    g = np.array([len(c["ops"]) for c in circuits])
    hist = np.bincount(ns, minlength=41)[:41]
    return "n:" + ",".join(str(int(x)) for x in hist) + f"|ops:{int(g.sum())}"


def candidates(precision: str) -> List[Dict[str, int]]:
    cap = 13 if precision == "f32" else 12
    out = []
    for smax in sorted({cap - 2, cap - 1, cap}):
        for thr in (128, 256, 512):
            for ctas in (1, 2, 4):
                if thr * ctas > 2048:
                    continue
                out.append(dict(small_max_n=smax, small_threads=thr, small_ctas_per_sm=ctas, pass_gate_budget=0))
    for budget in (48, 96, 160):
        out.append(dict(small_max_n=cap, small_threads=256, small_ctas_per_sm=2, pass_gate_budget=budget))
    if precision == "f32":  # the tensor-core block form as well
        out.append(dict(small_max_n=cap, small_threads=256, small_ctas_per_sm=2, pass_gate_budget=0, f32_tensor=1))
    return out


def _time_batch(circuits, precision, tuning, reps=3) -> float:
    import torch
    from . import Batch
    with Batch(precision) as b:
        # the candidates are timed on the interpreted passes: generated
        # kernels would make every candidate pay for its compiles
        b.set_tuning(**dict(tuning, jit=0))
        for c in circuits:
            b.add(c["n"], c["ops"], c["masks"])
        b.run()
        b.run()
        dev = torch.device("cuda", torch.cuda.current_device())
        s = torch.cuda.ExternalStream(b.stream_ptr(), device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(reps):
            b.launch()
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps


def tune(circuits: List[dict], precision: str = "f64", sample: int = 512, seed: int = 0,
         cache: Optional[str] = DEFAULT_CACHE, budget_s: float = 60.0) -> Dict[str, int]:
    """Best tuning for `circuits` (a list of {"n", "ops", "masks"}), measured
    on a seeded sample of at most `sample` circuits within `budget_s`."""
    import torch
    key = f"{precision}|{torch.cuda.get_device_name()}|{signature(circuits)}"
    db = {}
    if cache and os.path.exists(cache):
        try:
            db = json.load(open(cache))
        except (OSError, ValueError):
            db = {}
    if key in db:
        return dict(db[key]["tuning"])
    rng = np.random.default_rng(seed)
    idx = rng.choice(len(circuits), size=min(sample, len(circuits)), replace=False)
    sub = [circuits[i] for i in sorted(idx)]
    best, best_ms, tried = None, float("inf"), []
    t_end = time.time() + budget_s
    for cand in candidates(precision):
        if time.time() > t_end:
            break
        ms = _time_batch(sub, precision, cand)
        tried.append((cand, ms))
        if ms < best_ms:
            best, best_ms = cand, ms
    if cache:
        os.makedirs(os.path.dirname(cache), exist_ok=True)
        db[key] = {"tuning": best, "sample_ms": best_ms, "tried": len(tried)}
        with open(cache, "w") as f:
            json.dump(db, f, indent=1)
    return dict(best)
