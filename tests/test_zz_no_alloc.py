"""ppb_find_peaks_noalloc: the peak finder for callers that cannot allocate
device memory when they call it (their GPU memory belongs to another
runtime's pool, or they run a fixed-footprint loop where cudaMalloc/cudaFree
are not allowed).  The caller owns every device buffer; the entry point's
only scratch is an array built into the library.

Checked here through the C ABI against ppb_find_peaks on the same inputs, on
two calls in a row (the built-in scratch keeps the previous call's contents,
which must not leak into the next result).  This file is collected last so a
failure here never stops the rest of the GPU suite."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import peakpatch_b200 as pp


def _rt():
    from cuda.bindings import runtime as rt
    return rt


def _h2d(ctx, arr):
    rt = _rt()
    ptr = ctx.alloc_device(max(arr.nbytes, 8))
    (err,) = rt.cudaMemcpy(ptr, arr.ctypes.data, arr.nbytes, rt.cudaMemcpyKind.cudaMemcpyHostToDevice)
    assert err == rt.cudaError_t.cudaSuccess
    return ptr


def _d2h(ptr, dtype, count):
    rt = _rt()
    out = np.empty(count, dtype=dtype)
    if count:
        (err,) = rt.cudaMemcpy(out.ctypes.data, ptr, out.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
        assert err == rt.cudaError_t.cudaSuccess
    return out


def _field(n, seed):
    """A smooth-ish test field: white noise averaged over 3^3 blocks."""
    from numpy.lib.stride_tricks import sliding_window_view
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n + 2, n + 2, n + 2)).astype(np.float32)
    return sliding_window_view(x, (3, 3, 3)).mean(axis=(-1, -2, -3)).astype(np.float32)[:n, :n, :n].copy()


def _noalloc(ctx, d_delta, d_mask, shape, nbuff, fcrit, max_peaks, cap):
    n3, n2, n1 = shape
    outs = [ctx.alloc_device(cap * 8) for _ in range(4)] + [ctx.alloc_device(cap * 4)]
    npk = ctypes.c_int64(-1)
    rc = ctx.L.ppb_find_peaks_noalloc(ctx.h, ctypes.c_void_p(d_delta), ctypes.c_void_p(d_mask), n1, n2, n3, nbuff,
                                      ctypes.c_float(fcrit), max_peaks, *[ctypes.c_void_p(o) for o in outs],
                                      ctypes.byref(npk))
    ctx._check(rc)
    m = npk.value
    res = {k: _d2h(o, np.int64, m) for k, o in zip(("i", "j", "k", "ipp"), outs[:4])}
    res["delta"] = _d2h(outs[4], np.float32, m)
    for o in outs:
        ctx.free_device(o)
    return res


# max_peaks 0 keeps the first peak, as the reference (it tests the count
# after each push); on the 80^3 grid (72^3 inner cells, 365 blocks of the
# ordered compaction, 6707 peaks of which 4736 lie in blocks 0-255) 5500 ends
# the scan inside the second 256-block chunk of the block-offset scan
@pytest.mark.parametrize("max_peaks", [2_000_000, 37, 5500, 0])
def test_noalloc_matches_find_peaks_on_two_consecutive_calls(max_peaks):
    with pp.Context(0) as ctx:
        for call, (n, nbuff, seed) in enumerate([(64, 4, 1), (57, 3, 2), (80, 4, 3)]):
            f = _field(n, seed)
            mask0 = np.zeros(f.shape, np.int8)
            mask0[::7, ::5, ::3] = 1            # a partly masked grid, as across filters
            fcrit = np.float32(0.1)
            # reference: the allocating entry point on host copies
            m_ref = mask0.copy()
            ref = ctx.find_peaks(f, m_ref, 0.0, 0.0, 0.0, 1.0, nbuff, fcrit, max_peaks=max_peaks)
            assert len(ref["i"]) == 1 if max_peaks == 0 else len(ref["i"]) > 30
            # the no-allocation entry point on caller-owned device buffers
            d_f = _h2d(ctx, f)
            d_m = _h2d(ctx, mask0)
            cap = max(1, min(max_peaks, f.size))
            got = _noalloc(ctx, d_f, d_m, f.shape, nbuff, float(fcrit), max_peaks, cap)
            m_got = _d2h(d_m, np.int8, f.size).reshape(f.shape)
            ctx.free_device(d_f)
            ctx.free_device(d_m)
            for k in ("i", "j", "k", "ipp"):
                assert np.array_equal(got[k], ref[k]), (call, k)
            assert got["delta"].tobytes() == ref["delta"].tobytes(), call
            assert np.array_equal(m_got, m_ref), call


def test_noalloc_rejects_host_buffers():
    with pp.Context(0) as ctx:
        f = np.zeros((16, 16, 16), np.float32)
        m = np.zeros(f.shape, np.int8)
        bufs = [np.zeros(8, np.int64) for _ in range(4)] + [np.zeros(8, np.float32)]
        npk = ctypes.c_int64()
        rc = ctx.L.ppb_find_peaks_noalloc(ctx.h, f.ctypes.data_as(ctypes.c_void_p), m.ctypes.data_as(ctypes.c_void_p),
                                          16, 16, 16, 2, ctypes.c_float(1.0), 8,
                                          *[b.ctypes.data_as(ctypes.c_void_p) for b in bufs], ctypes.byref(npk))
        assert rc == -1
