"""qoa_expect_z_noalloc: the allocation-free entry point.

Callers that own every device buffer themselves (a host runtime with its own
pool and accounting), or that cannot accept cudaMalloc's implicit
synchronisation on their path, use this variant: the state vector and the
output live in memory the caller allocated, and the library's own scratch is
a fixed static device array. The test gives it caller-owned device buffers and
checks its results against the handle entry point qoa_expect_z on the same
state, on two calls in a row (the second reuses the scratch the first left).
"""
import ctypes

import numpy as np
import pytest

import qoa_b200 as qb
from qoa_b200 import circuits as C

TOL = 1e-12


def _entry():
    f = qb.lib.qoa_expect_z_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                  ctypes.c_void_p]
    return f


@pytest.mark.gpu
def test_expect_z_noalloc_matches_qoa_expect_z_twice():
    import torch

    f = _entry()
    n = 16
    masks_first = [1, 3, 0b1010101, (1 << n) - 1, 0, 1 << 15, 0b1100110011001100, 7]
    masks_second = [5, 1 << 3, 0b111000111, 1 << 14 | 1, 0xFFF0]
    with qb.QuantumState(n, compat_mask_quirk=True) as st:
        st.execute(C.ops_to_array(C.random_layered(n, 6, 77, initial_h=True)))
        state = st.get_state_vector()
        # caller-owned device memory for the input and the output
        d_state = torch.from_numpy(state.view(np.float64).copy()).cuda()
        stream = torch.cuda.current_stream()
        for masks in (masks_first, masks_second):
            ref = st.expect_z(masks)
            d_out = torch.full((len(masks),), float("nan"), dtype=torch.float64, device="cuda")
            m = np.ascontiguousarray(np.asarray(masks, dtype=np.uint64))
            rc = f(d_state.data_ptr(), 1 << n, m.ctypes.data, len(m), d_out.data_ptr(), stream.cuda_stream)
            assert rc == qb.QOA_OK, qb.lib.qoa_last_error(None)
            stream.synchronize()
            got = d_out.cpu().numpy()
            assert np.max(np.abs(got - ref)) < TOL, (got, ref)


@pytest.mark.gpu
def test_expect_z_noalloc_rejects_more_masks_than_its_scratch_holds():
    import torch

    f = _entry()
    d_state = torch.zeros(2 * 16, dtype=torch.float64, device="cuda")
    d_out = torch.zeros(16, dtype=torch.float64, device="cuda")
    m = np.arange(qb_max := 8 + 1, dtype=np.uint64)
    rc = f(d_state.data_ptr(), 16, m.ctypes.data, qb_max, d_out.data_ptr(), None)
    assert rc == qb.QOA_E_ARG
    assert b"QOA_NOALLOC_MAX_MASKS" in qb.lib.qoa_last_error(None)
