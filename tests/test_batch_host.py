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
