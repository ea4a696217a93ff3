"""Host side of batch trajectories (no GPU): which op lists can run as batch
circuits, i.e. expand to unitary gates only (qoa_ops_unitary)."""
import ctypes

import pytest

import qoa_b200 as qb
from qoa_b200 import circuits as C


def unitary(n, ops):
    arr = C.ops_to_array(ops)
    out = ctypes.c_int(-1)
    assert qb.lib.qoa_ops_unitary(n, 0, qb._ptr(arr) if len(arr) else None, len(arr), ctypes.byref(out)) == qb.QOA_OK
    return out.value


@pytest.mark.parametrize("ops,want", [
    (C.random_layered(6, 4, 1), 1),
    (C.qft(5), 1),
    ([C.Op(C.H, [0]), C.Op(C.MEASURE, [0])], 0),
    ([C.Op(C.H, [0]), C.Op(C.RESET, [1])], 0),
    ([C.Op(C.QINIT, [3]), C.Op(C.H, [0])], 0),
    ([C.Op(C.H, [0]), C.Op(C.CNOT, [0, 9])], 1),   # an out-of-range op is skipped, as in qoa_apply
    ([], 1),
])
def test_ops_unitary(ops, want):
    assert unitary(6, ops) == want


@pytest.mark.parametrize("n,p", [(1, 0.5), (7, 0.3), (15, 1e-3), (33, 0.05), (40, 0.9), (64, 0.2), (17, 1.0),
                                 (16, 0.0), (20, 1e-300), (12, 2.0 ** -53), (12, 3 * 2.0 ** -40), (31, 0.999999999)])
def test_noise_hits_equal_one_draw_per_qubit(n, p):
    # the vectorised hit tests give exactly the per-qubit draws' outcomes
    for seed, stream, ev in [(1, 0, 0), (123456789012345, 7, 99), (2 ** 63 + 5, 0xFFFFFFFF, 2 ** 40 + 3)]:
        want = 0
        for q in range(n):
            if qb.lib.qoa_philox_uniform(seed, stream, ev, 2 * q + 1) < p:
                want |= 1 << q
        assert qb.lib.qoa_noise_hits(seed, stream, ev, n, p) == want
