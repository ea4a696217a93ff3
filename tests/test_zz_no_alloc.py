"""qoa_expect_z_noalloc: the allocation-free entry point.

Callers that own every device buffer themselves (a host runtime with its own
pool and accounting), or that cannot accept cudaMalloc's implicit
synchronisation on their path, use this variant: the state vector and the
output live in memory the caller allocated, and the library's own scratch is
a fixed static device array. The tests give it caller-owned device buffers
and check its results against numpy's sum over the same amplitudes and
against the handle entry point qoa_expect_z, on two calls in a row (the
second reuses the scratch the first left), check that a call leaves the
device's free memory unchanged, and run it in a second CUDA context the
caller made itself, where the scratch array has a different address.
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


def _numpy_expect_z(state: np.ndarray, masks) -> np.ndarray:
    p = np.abs(state) ** 2
    idx = np.arange(state.size, dtype=np.uint64)
    out = []
    for m in masks:
        par = np.zeros(state.size, dtype=np.uint64)
        x = idx & np.uint64(m)
        while x.any():
            par ^= x & np.uint64(1)
            x >>= np.uint64(1)
        out.append(float(np.sum(np.where(par == 1, -p, p))))
    return np.array(out)


@pytest.mark.gpu
def test_expect_z_noalloc_matches_numpy_and_qoa_expect_z_twice():
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
            want = _numpy_expect_z(state, masks)
            d_out = torch.full((len(masks),), float("nan"), dtype=torch.float64, device="cuda")
            m = np.ascontiguousarray(np.asarray(masks, dtype=np.uint64))
            rc = f(d_state.data_ptr(), 1 << n, m.ctypes.data, len(m), d_out.data_ptr(), stream.cuda_stream)
            assert rc == qb.QOA_OK, qb.lib.qoa_last_error(None)
            stream.synchronize()
            got = d_out.cpu().numpy()
            assert np.max(np.abs(got - want)) < TOL, (got, want)
            assert np.max(np.abs(got - ref)) < TOL, (got, ref)
        # a further call takes no device memory (the free figure is unchanged)
        d_out = torch.zeros(3, dtype=torch.float64, device="cuda")
        m = np.array([1, 2, 4], dtype=np.uint64)
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        assert f(d_state.data_ptr(), 1 << n, m.ctypes.data, 3, d_out.data_ptr(), stream.cuda_stream) == qb.QOA_OK
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0
        assert np.max(np.abs(d_out.cpu().numpy() - _numpy_expect_z(state, [1, 2, 4]))) < TOL


@pytest.mark.gpu
def test_expect_z_noalloc_in_a_context_the_caller_made():
    import torch
    from cuda.bindings import driver as drv

    f = _entry()
    n = 14
    with qb.QuantumState(n) as st:
        st.execute(C.ops_to_array(C.random_layered(n, 4, 91, initial_h=True)))
        state = np.ascontiguousarray(st.get_state_vector())
    masks = [1, 6, 0x2AAA, (1 << n) - 1]
    want = _numpy_expect_z(state, masks)
    torch.cuda.synchronize()

    def ok(res):
        err = res[0] if isinstance(res, tuple) else res
        assert err == drv.CUresult.CUDA_SUCCESS, err
        return res[1] if isinstance(res, tuple) and len(res) > 1 else None

    dev = ok(drv.cuDeviceGet(torch.cuda.current_device()))
    ctx = ok(drv.cuCtxCreate(0, dev))  # pushed and current on this thread
    try:
        d_amps = ok(drv.cuMemAlloc(state.nbytes))
        d_out = ok(drv.cuMemAlloc(8 * len(masks)))
        ok(drv.cuMemcpyHtoD(d_amps, state.ctypes.data, state.nbytes))
        m = np.ascontiguousarray(np.asarray(masks, dtype=np.uint64))
        for _ in range(2):
            rc = f(int(d_amps), 1 << n, m.ctypes.data, len(m), int(d_out), None)
            assert rc == qb.QOA_OK, qb.lib.qoa_last_error(None)
            ok(drv.cuCtxSynchronize())
            got = np.zeros(len(masks), dtype=np.float64)
            ok(drv.cuMemcpyDtoH(got.ctypes.data, d_out, got.nbytes))
            assert np.max(np.abs(got - want)) < TOL, (got, want)
        ok(drv.cuMemFree(d_amps))
        ok(drv.cuMemFree(d_out))
    finally:
        ok(drv.cuCtxDestroy(ctx))
    # back in the primary context, the entry point still uses that context's array
    d_state = torch.from_numpy(state.view(np.float64).copy()).cuda()
    d_res = torch.zeros(len(masks), dtype=torch.float64, device="cuda")
    assert f(d_state.data_ptr(), 1 << n, m.ctypes.data, len(m), d_res.data_ptr(), None) == qb.QOA_OK
    torch.cuda.synchronize()
    assert np.max(np.abs(d_res.cpu().numpy() - want)) < TOL


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
