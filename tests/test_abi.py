"""The C-ABI library loads without a GPU and exports every entry point that
include/qoa_cuda.h declares (no compute calls here)."""
import ctypes
import os
import re

import qoa_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "qoa_cuda.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(qoa_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_boundary():
    names = declared()
    for must in ("qoa_create", "qoa_apply", "qoa_measure", "qoa_sample", "qoa_get_state", "qoa_set_state",
                 "qoa_vec_apply_hadamard", "qoa_vec_apply_controlled_phase_rotation"):
        assert must in names
    assert sum(n.startswith("qoa_vec_apply_") for n in names) == 17


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(qoa_b200.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_strerror_is_callable_without_gpu():
    assert qoa_b200.lib.qoa_strerror(0) == b"ok"
    assert b"range" in qoa_b200.lib.qoa_strerror(1)


def test_philox_uniform_matches_oracle():
    from oracle import pyoracle as po
    for seed, stream, event, slot in ((0, 0, 0, 0), (5, 7, 3, 1), (2**63 + 11, 0x73686F74 ^ 9, 2**40 + 3, 17)):
        assert qoa_b200.philox_uniform(seed, stream, event, slot) == po.uniform(seed, stream, event, slot)


def test_generators_and_reference_arm_open_no_gpu_library():
    # the reference arm of bench.py times the oracle only: importing the
    # package for its circuit generators must not map libqoa_cuda.so
    import json
    import subprocess
    import sys
    code = ("import sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--qubits', '14', '--depth', '2', "
            "'--steps', '10', '--warmup', '3']; sys.path.insert(0, '.'); import bench; bench.main(); "
            "print(json.dumps({'maps': [l.split()[-1] for l in open('/proc/self/maps') if l.rstrip().endswith('.so')]}))")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = [json.loads(x) for x in out.stdout.splitlines() if x.startswith("{")]
    line, maps = lines[0], lines[1]["maps"]
    assert not any("libqoa_cuda" in m for m in maps)
    assert any("liboracle" in m for m in maps)
    assert line["impl"] == "reference" and line["value"] > 0
    cb = line["cpu_baseline"]
    assert set(cb["per_class_s"]) == set(cb["class_counts"]) and sum(cb["class_counts"].values()) == 14 + 2 * 21
