"""Shared helpers for the reference known-answer tests (tests/golden)."""
import json
import os

import numpy as np

from qoa_b200.circuits import Op, ops_to_array

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_kats.json")


def load_cases(level=None):
    cases = json.load(open(GOLDEN))["cases"]
    return [c for c in cases if level is None or c["level"] == level]


def cvec(pairs):
    return np.array([complex(a, b) for a, b in pairs], dtype=np.complex128)


def case_ops(case):
    return ops_to_array([Op(o["opcode"], o["qubits"], o["angle"]) for o in case["ops"]])


def check_case(case, got):
    """Asserts the reference's |d re|, |d im| < tol on the recorded amplitudes."""
    tol = case["tol"]
    if case.get("expect") is not None:
        exp = cvec(case["expect"])
        assert got.shape == exp.shape, (case["name"], got.shape, exp.shape)
        assert np.all(np.abs(got.real - exp.real) < tol) and np.all(np.abs(got.imag - exp.imag) < tol), (
            case["name"], got, exp)
    for k, v in (case.get("expect_at") or {}).items():
        e = complex(*v)
        g = got[int(k)]
        assert abs(g.real - e.real) < tol and abs(g.imag - e.imag) < tol, (case["name"], k, g, e)
    for k, v in (case.get("expect_ne") or {}).items():
        assert got[int(k)] != complex(*v), (case["name"], k)
