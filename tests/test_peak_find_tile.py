"""ppb_peak_find_tile (peak_find_tile_gpu, src/PeakPatch.jl:341-366) against
the oracle's filter loop: smooth_field (Filters.jl:318-345) and find_peaks
(PeakFind.jl:15-79) per filter, in the given order, the mask carried across
filters.

The GPU transforms in single precision (cuFFT; at 384^3 with the k^2-weighted
twin the x pass of the inverse transform runs fused with the peak search),
the oracle in double precision rounded to Float32, so a cell whose value
ties its largest neighbour or fcrit to within single-precision transform
rounding may be a peak on one side only.  Every disagreement must be such a
cell (or a cell that an earlier disagreement left masked on one side only);
every agreeing peak has the same filter, position and Rf, and FcRf / d2Rf
within transform rounding."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import peakpatch_b200 as pp

# single-precision transform rounding, relative to the field's largest value
ROUND = 3e-6


def oracle_filter_loop(ora, delta, filters, fcrits, mask, alatt, nbuff, wsmooth, ioutshear):
    n = delta.shape[0]
    box = n * alatt
    dk = ora.rfft3(delta)
    out = []
    for Rf, fc in zip(filters, fcrits):
        ds = ora.smooth_field(dk, n, box, Rf, wsmooth)
        ls = ora.smooth_field(dk, n, box, Rf, 3) if ioutshear >= 1 else None
        p = ora.find_peaks(ds, mask, 0.0, 0.0, 0.0, alatt, nbuff, np.float32(fc))
        out.append((ds, ls, p))
    return out


def _margin(ds, i, j, k, fcrit):
    v = float(ds[k - 1, j - 1, i - 1])
    nb = ds[k - 2:k + 1, j - 2:j + 1, i - 2:i + 1].astype(np.float64).copy()
    nb[1, 1, 1] = -np.inf
    return min(abs(v - nb.max()), abs(v - float(np.float32(fcrit))))


def compare(ora_out, gp, filters, fcrits, ioutshear):
    """Returns (number of peaks, disagreements, worst margin of a first
    disagreement relative to the field maximum)."""
    flipped = set()
    nd, worst, total = 0, 0.0, 0
    for f, (ds, ls, op) in enumerate(ora_out):
        sel = gp["filter"] == f + 1
        g = {(int(a), int(b), int(c)): q for q, (a, b, c) in
             enumerate(zip(gp["i"][sel], gp["j"][sel], gp["k"][sel]))}
        o = {(int(a), int(b), int(c)): q for q, (a, b, c) in enumerate(zip(op["i"], op["j"], op["k"]))}
        total += len(o)
        scale = float(np.abs(ds).max())
        for cell in set(g) ^ set(o):
            nd += 1
            if cell in flipped:
                continue
            m = _margin(ds, *cell, fcrits[f]) / scale
            worst = max(worst, m)
            flipped.add(cell)
        common = sorted(set(g) & set(o), key=lambda c: o[c])
        if common:
            gi = np.where(sel)[0][[g[c] for c in common]]
            oi = np.array([o[c] for c in common])
            assert np.all(gp["Rsmooth"][gi] == filters[f])
            for key in ("x", "y", "z", "ipp"):
                assert np.array_equal(gp[key][gi], op[key][oi]), key
            d = np.abs(gp["delta"][gi].astype(np.float64) - op["delta"][oi].astype(np.float64))
            assert d.max() <= ROUND * scale, (f, d.max() / scale)
            if ioutshear:
                lin = op["ipp"][oi] - 1
                lo = ls.reshape(-1)[lin].astype(np.float64)
                dl = np.abs(gp["d2Rf"][gi] - lo)
                assert dl.max() <= ROUND * float(np.abs(ls).max()), (f, dl.max())
        # the GPU's order within a filter is the scan order
        ipp_g = gp["ipp"][sel]
        assert np.all(np.diff(ipp_g) > 0)
    return total, nd, worst


@pytest.mark.parametrize("wsmooth,ioutshear,fused", [(1, 1, -1), (0, 0, -1), (1, 1, 1)])
def test_peak_find_tile_vs_oracle_64(ctx, ora, eh_pk, wsmooth, ioutshear, fused):
    n, alatt, nbuff = 64, 2.0, 4
    delta = ora.generate_grf(n, *eh_pk, n * alatt, 21)
    filters = [12.0, 6.0, 3.0, 1.5]
    fcrits = [1.686, 1.5, 1.686, 1.2]
    mask_o = np.zeros((n, n, n), np.int8)
    mask_o[::9, ::7, ::5] = 1   # a caller's mask, as carried across tiles' filter loops
    mask_g = mask_o.copy()
    oo = oracle_filter_loop(ora, delta, filters, fcrits, mask_o, alatt, nbuff, wsmooth, ioutshear)
    ctx.set_option(pp.OPT_FUSED_X, fused)
    try:
        gp, Rf, FcRf, d2Rf, m = ctx.peak_find_tile(delta, filters, fcrits, mask_g, 0.0, 0.0, 0.0, alatt, nbuff,
                                                   wsmooth, ioutshear)
    finally:
        ctx.set_option(pp.OPT_FUSED_X, -1)
    assert np.array_equal(Rf, gp["Rsmooth"]) and np.array_equal(FcRf, gp["delta"])
    gp = dict(gp, d2Rf=d2Rf)
    total, nd, worst = compare(oo, gp, filters, fcrits, ioutshear)
    assert total > 200
    assert worst <= ROUND and nd <= max(2, total // 1000), (nd, worst)
    if ioutshear == 0:
        assert np.all(d2Rf == 0)
    assert m is mask_g and (nd > 0 or np.array_equal(mask_g, mask_o))


def test_peak_find_tile_capacity_and_coordinates(ctx, ora, eh_pk):
    """Coordinates x = xbx + alatt (i - (n+1)/2) (PeakFind.jl:26-40), the
    1-based filter number, and a capacity too small returns PPB_ERR_CAPACITY
    with the count needed and the mask untouched."""
    import ctypes
    n, alatt = 48, 1.5
    delta = ora.generate_grf(n, *eh_pk, n * alatt, 4)
    mask = np.zeros((n, n, n), np.int8)
    gp, *_ = ctx.peak_find_tile(delta, [5.0, 2.0], [1.0, 1.0], mask, 10.0, -20.0, 30.0, alatt, 2, 1, 0)
    assert len(gp["i"]) > 5 and set(gp["filter"].tolist()) <= {1, 2}
    assert np.allclose(gp["x"], 10.0 + alatt * (gp["i"] - 0.5 * (n + 1)))
    assert np.allclose(gp["z"], 30.0 + alatt * (gp["k"] - 0.5 * (n + 1)))
    m2 = np.zeros((n, n, n), np.int8)
    npk = ctypes.c_int64()
    Rf = np.array([5.0, 2.0])
    fc = np.array([1.0, 1.0])
    rc = ctx.L.ppb_peak_find_tile(ctx.h, delta.ctypes.data_as(ctypes.c_void_p), n, Rf.ctypes.data_as(ctypes.c_void_p),
                                  fc.ctypes.data_as(ctypes.c_void_p), 2, m2.ctypes.data_as(ctypes.c_void_p), 0.0, 0.0,
                                  0.0, alatt, 2, 1, 0, 1, *([None] * 11), ctypes.byref(npk))
    assert rc == -7 and npk.value == len(gp["i"]) and not m2.any()


def test_fused_filter_bank_vs_oracle_384(ctx, ora, eh_pk):
    """The benchmark tile's delta (384^3, box 768 Mpc/h, seed 7) through the
    fused filter bank (window, cuFFT z/y passes, x pass fused with the peak
    search, the k^2-weighted twin at the peaks) against the oracle's
    smooth_field + find_peaks, six filters of the 1.5-30 Mpc/h bank."""
    n, alatt, nbuff = 384, 2.0, 32
    delta = ora.generate_grf(n, *eh_pk, n * alatt, 7)
    filters = [30.0, 16.9, 9.5, 5.35, 3.0, 1.5]
    fcrits = [1.686] * len(filters)
    mask_o = np.zeros((n, n, n), np.int8)
    mask_g = np.zeros((n, n, n), np.int8)
    oo = oracle_filter_loop(ora, delta, filters, fcrits, mask_o, alatt, nbuff, 1, 1)
    gp, _, _, d2Rf, _ = ctx.peak_find_tile(delta, filters, fcrits, mask_g, 0.0, 0.0, 0.0, alatt, nbuff, 1, 1)
    gp = dict(gp, d2Rf=d2Rf)
    total, nd, worst = compare(oo, gp, filters, fcrits, 1)
    print(f"fused filter bank 384^3: {total} oracle peaks, {len(gp['i'])} GPU peaks, {nd} disagreements, "
          f"worst first-disagreement margin {worst:.2e} of the field maximum")
    assert total > 100000
    assert worst <= ROUND and nd <= total // 10000, (nd, worst)
