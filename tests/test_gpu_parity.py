"""GPU parity tests: libppb.so (called through its C ABI) against the CPU
oracle on the same inputs.

Bars (from the path's specification):
  * white noise: bit-exact;
  * peak list: bit-exact (i, j, k, ipp, delta, order) on an identical field;
  * halos: RTHL / mass within 1e-4 relative, at most 0.1 % of halos
    mismatched (a halo on one side only, or outside the tolerance).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, filter_bank
from test_oracle_pins import FORTRAN_GOLDEN, check_fortran_golden, fortran_golden_fields

pytestmark = pytest.mark.gpu

import peakpatch_b200 as pp

RTOL = 1e-4        # halo mass / radius tolerance
MISMATCH = 1e-3    # allowed fraction of mismatched halos


# ------------------------------------------------------------------ noise
@pytest.mark.parametrize("n,seed", [(64, 42), (33, 7), (128, 2**63 + 5), (1, 3), (2, 0)])
def test_noise_bit_exact(ctx, ora, n, seed):
    g = ctx.fill_noise_threefry(n, seed)
    o = ora.noise(n, seed)
    assert g.dtype == np.float32 and g.shape == (n, n, n)
    assert np.array_equal(g.view(np.uint32), o.view(np.uint32))


# ------------------------------------------------------------------ peaks
def _compare_peaks(gp, op):
    for k in ("i", "j", "k", "ipp"):
        assert np.array_equal(gp[k], op[k]), k
    assert np.array_equal(gp["delta"].view(np.uint32), op["delta"].view(np.uint32))
    for k in ("x", "y", "z"):
        assert np.array_equal(gp[k], op[k])


def test_find_peaks_reference_kats(ctx):
    # test/test_peakfind.jl cases through the GPU entry point
    n = 11
    d = np.zeros((n, n, n), np.float32)
    d[5, 5, 5] = 2.0
    m = np.zeros(d.shape, np.int8)
    p = ctx.find_peaks(d, m, 0.0, 0.0, 0.0, 1.0, 1, 1.0, 3.0)
    assert (p["i"].tolist(), p["j"].tolist(), p["k"].tolist()) == ([6], [6], [6]) and m[5, 5, 5] == 1
    assert len(ctx.find_peaks(np.full((n, n, n), 0.5, np.float32), np.zeros(d.shape, np.int8), 0, 0, 0, 1.0, 1,
                              1.0)["i"]) == 0
    mk = np.zeros(d.shape, np.int8)
    mk[5, 5, 5] = 1
    assert len(ctx.find_peaks(d, mk, 0, 0, 0, 1.0, 1, 1.0)["i"]) == 0
    d5 = np.zeros((15,) * 3, np.float32)
    for (i, j, k) in [(4, 4, 4), (4, 4, 12), (12, 12, 4), (12, 12, 12)]:
        d5[k - 1, j - 1, i - 1] = 2.0
    m5 = np.zeros(d5.shape, np.int8)
    p = ctx.find_peaks(d5, m5, 0, 0, 0, 1.0, 1, 1.0, max_peaks=2)
    assert list(zip(p["i"], p["j"], p["k"])) == [(4, 4, 4), (12, 12, 4)]
    assert m5.sum() == 2   # peaks beyond max_peaks stay unmasked, as in the reference
    d21 = np.zeros((21,) * 3, np.float32)
    d21[10, 10, 10] = 2.0
    p = ctx.find_peaks(d21, np.zeros(d21.shape, np.int8), 10.0, 20.0, 30.0, 2.0, 1, 1.0)
    assert (p["x"][0], p["y"][0], p["z"][0]) == (10.0, 20.0, 30.0)


@pytest.mark.parametrize("n,nbuff,seed", [(64, 4, 1), (48, 8, 2), (40, 1, 3)])
def test_find_peaks_bit_exact_on_identical_field(ctx, ora, eh_pk, n, nbuff, seed):
    f = ora.generate_grf(n, *eh_pk, 2.0 * n, seed)
    dk = ora.rfft3(f)
    mask_g = np.zeros(f.shape, np.int8)
    mask_o = np.zeros(f.shape, np.int8)
    # several filters in sequence share the mask, as in run_tile
    for R in (6.0, 3.0, 1.5):
        s = ora.smooth_field(dk, n, 2.0 * n, R, 1)
        gp = ctx.find_peaks(s, mask_g, 0.0, 0.0, 0.0, 2.0, nbuff, np.float32(1.686), R)
        op = ora.find_peaks(s, mask_o, 0.0, 0.0, 0.0, 2.0, nbuff, np.float32(1.686))
        assert len(op["i"]) > 0
        _compare_peaks(gp, op)
        assert np.array_equal(mask_g, mask_o)


def test_find_peaks_ties_and_plateaus(ctx, ora):
    # equal neighbours do not reject a peak (only a strictly larger one does)
    d = np.zeros((12, 12, 12), np.float32)
    d[4:6, 4:6, 4:6] = 3.0
    d[8, 8, 8] = 2.0
    d[8, 8, 9] = 2.0
    mg, mo = np.zeros(d.shape, np.int8), np.zeros(d.shape, np.int8)
    _compare_peaks(ctx.find_peaks(d, mg, 0, 0, 0, 1.0, 1, 1.0), ora.find_peaks(d, mo, 0, 0, 0, 1.0, 1, 1.0))
    assert np.array_equal(mg, mo) and mg.sum() == 10


# ------------------------------------------------------------------ shells
def test_fortran_golden_on_gpu(ctx, fortran_table):
    f = fortran_golden_fields()
    t = pp.read_homeltab(os.path.join(GOLDEN, "HomelTab_fortran.dat"))
    ctx.set_collapse_table(t)
    ipp = 71 + 70 * 142 + 70 * 142 * 142
    for plain in (True, False):
        r = ctx.analyse_peaks(f, [ipp], [4.0], [4], [1.0], [FORTRAN_GOLDEN["fcrit"]], 1.0, 8, plain=plain)[0]
        check_fortran_golden(r, rtol=1e-6)


@pytest.fixture(scope="module")
def shell_case(ora, eh_pk, julia_table):
    """Fields of a 64^3 tile (box 128 Mpc/h) with 2LPT and lapd, the peaks of
    a 6-filter top-hat bank, and the oracle's analyse_peak results."""
    n, box, nbuff = 64, 128.0, 16
    alatt = box / n
    d = ora.generate_grf(n, *eh_pk, box, 11)
    dk = ora.rfft3(d)
    psi = ora.lpt1(dk, n, box)
    psi2 = ora.lpt2(dk, n, box)
    lapd = ora.laplacian(dk, n, box)
    fields = dict(delta=d, etax=psi[0], etay=psi[1], etaz=psi[2], eta2x=psi2[0], eta2y=psi2[1], eta2z=psi2[2],
                  lapd=lapd)
    fcrit = ora.fsc_of_z(0.315, 0.049, 0.685, 0.674, 0.0)
    mask = np.zeros(d.shape, np.int8)
    ipp, Rf = [], []
    for R in (24.0, 12.0, 6.0, 4.0, 2.5, 1.5):
        s = ora.smooth_field(dk, n, box, R, 1)
        p = ora.find_peaks(s, mask, 0, 0, 0, alatt, nbuff, np.float32(fcrit))
        ipp += p["ipp"].tolist()
        Rf += [R] * len(p["ipp"])
    ipp, Rf = np.array(ipp), np.array(Rf)
    ir2 = np.minimum(np.floor((1.75 * Rf / alatt) ** 2), np.floor((40 / alatt - 1) ** 2)).astype(np.int64)
    nhunt = min(nbuff - 1, int(np.floor(24.0 * 1.75 / alatt)))
    res = ora.analyse_peaks(fields, ipp, Rf, ir2, 1.0, fcrit, alatt, ora.precompute_shells(nhunt), julia_table)
    return dict(fields=fields, ipp=ipp, Rf=Rf, ir2=ir2, fcrit=fcrit, alatt=alatt, nhunt=nhunt, res=res, n=n)


def compare_results(g, o, rtol=RTOL):
    """Per-peak comparison; returns (mismatch fraction, worst relative errors
    per field over the agreeing halos)."""
    coll_g, coll_o = g[:, 0] > 0, o[:, 0] > 0
    both = coll_g & coll_o
    rel = lambda a, b: np.abs(a - b) / np.maximum(np.abs(b), 1e-30)
    bad = coll_g != coll_o
    rR = rel(g[both, 0], o[both, 0])
    bad_both = rR > rtol
    bad[np.where(both)[0][bad_both]] = True
    nh = max(1, int(coll_o.sum()))
    errs = {}
    keep = both.copy()
    keep[bad] = False
    for name, sl in pp.RESULT_FIELDS.items():
        a, b = g[keep][:, sl], o[keep][:, sl]
        fin = np.isfinite(b)
        assert np.array_equal(np.isfinite(a), fin), name
        if np.any(fin):
            scale = np.maximum(np.abs(b[fin]), 1e-6 * np.abs(b[fin]).max() + 1e-300)
            errs[name] = float(np.max(np.abs(a[fin] - b[fin]) / scale))
    return bad.sum() / nh, errs


@pytest.mark.parametrize("plain", [True, False])
def test_analyse_peaks_vs_oracle(ctx, shell_case, julia_table, plain):
    c = shell_case
    ctx.set_collapse_table(pp.CollapseTable(julia_table.data, julia_table.x1, julia_table.x2, julia_table.y1,
                                            julia_table.y2, julia_table.z1, julia_table.z2))
    g = ctx.analyse_peaks(c["fields"], c["ipp"], c["Rf"], c["ir2"], 1.0, c["fcrit"], c["alatt"], c["nhunt"],
                          plain=plain)
    assert len(c["ipp"]) > 500
    assert (c["res"][:, 0] > 0).sum() > 100
    frac, errs = compare_results(g, c["res"])
    assert frac <= MISMATCH, (frac, errs)
    # radius and mass (RTHL^3) within 1e-4 on every agreeing halo
    assert errs["RTHL"] < RTOL
    st = ctx.shell_stats()
    assert st["visits"] > 0


@pytest.mark.parametrize("nhunt", [2, 3, 5])
def test_analyse_peaks_short_shell_lists(ctx, ora, shell_case, julia_table, nhunt):
    # short shell lists (cells 1.5-5 Mpc/h wide against the filter radii, as in
    # the reference's multi-resolution sweep) get smaller gather chunks
    c = shell_case
    ctx.set_collapse_table(pp.CollapseTable(julia_table.data, julia_table.x1, julia_table.x2, julia_table.y1,
                                            julia_table.y2, julia_table.z1, julia_table.z2))
    o = ora.analyse_peaks(c["fields"], c["ipp"], c["Rf"], c["ir2"], 1.0, c["fcrit"], c["alatt"],
                          ora.precompute_shells(nhunt), julia_table)
    assert (o[:, 0] > 0).sum() > 20
    for plain in (False, True):
        g = ctx.analyse_peaks(c["fields"], c["ipp"], c["Rf"], c["ir2"], 1.0, c["fcrit"], c["alatt"], nhunt,
                              plain=plain)
        frac, errs = compare_results(g, o)
        assert frac <= MISMATCH, (nhunt, plain, frac, errs)
        assert errs["RTHL"] < RTOL


def test_adaptive_truncation_reads_fewer_cells(ctx, shell_case, julia_table):
    c = shell_case
    ctx.set_collapse_table(pp.CollapseTable(julia_table.data, julia_table.x1, julia_table.x2, julia_table.y1,
                                            julia_table.y2, julia_table.z1, julia_table.z2))
    ctx.analyse_peaks(c["fields"], c["ipp"], c["Rf"], c["ir2"], 1.0, c["fcrit"], c["alatt"], c["nhunt"], plain=True)
    full = ctx.shell_stats()["visits"]
    ctx.analyse_peaks(c["fields"], c["ipp"], c["Rf"], c["ir2"], 1.0, c["fcrit"], c["alatt"], c["nhunt"], plain=False)
    part = ctx.shell_stats()["visits"]
    assert part < full


def test_peaks_near_the_border(ctx, ora, eh_pk, julia_table):
    """Shell cells outside the grid are skipped (no periodic wrap), and d2F
    stops at the first out-of-grid cell, exactly as the reference."""
    n, box = 40, 80.0
    d = ora.generate_grf(n, *eh_pk, box, 5)
    dk = ora.rfft3(d)
    psi = ora.lpt1(dk, n, box)
    lapd = ora.laplacian(dk, n, box)
    fields = dict(delta=d, etax=psi[0], etay=psi[1], etaz=psi[2], lapd=lapd)
    s = ora.smooth_field(dk, n, box, 3.0, 1)
    p = ora.find_peaks(s, np.zeros(d.shape, np.int8), 0, 0, 0, 2.0, 1, np.float32(1.0))
    ipp = p["ipp"]
    assert len(ipp) > 20
    T = julia_table
    ctx.set_collapse_table(pp.CollapseTable(T.data, T.x1, T.x2, T.y1, T.y2, T.z1, T.z2))
    o = ora.analyse_peaks(fields, ipp, 3.0, 6, 1.0, 1.686, 2.0, ora.precompute_shells(10), T)
    for plain in (True, False):
        g = ctx.analyse_peaks(fields, ipp, 3.0, 6, 1.0, 1.686, 2.0, 10, plain=plain)
        frac, errs = compare_results(g, o)
        assert frac <= 0.02 and errs.get("RTHL", 0) < RTOL, (frac, errs)


# ------------------------------------------------------------------ run_tile
def tile_config(n=64, box=128.0, nbuff=16, ioutshear=1, ilpt=2, ievol=0, z_out=0.0, z_max=0.0):
    return pp.PipelineConfig(Omx=0.315 - 0.049, OmB=0.049, Omvac=0.685, h=0.674, n=n, boxsize=box, nbuff=nbuff,
                             z_out=z_out, z_max=z_max, ievol=ievol, ilpt=ilpt, ioutshear=ioutshear, wsmooth=1,
                             rmax2rs=0.0)


def ora_config(ora, cfg):
    return ora.Config(**{k: getattr(cfg, k) for k in ora.Config.__dataclass_fields__})


def small_tile_ok(frac, nhalo):
    """The 0.1 % halo bar on a tile of a few hundred halos: 0.1 % of them is
    less than one halo, so one mismatched halo is allowed there (the
    benchmark-size tiles of test_tile_parity.py apply 0.1 % as it stands)."""
    return frac * nhalo <= max(1.0, MISMATCH * nhalo) + 1e-9


def match_records(rg, ro, nf):
    """Match halos by position and filter radius; returns (mismatch fraction,
    per-field max relative error over matched pairs)."""
    key = lambda r: [tuple(np.round(x, 3)) for x in r[:, [0, 1, 2]]] if nf == 11 else \
        [tuple(np.round(x, 3)) for x in r[:, [0, 1, 2, 27]]]
    kg, ko = key(rg), key(ro)
    ig = {k: i for i, k in enumerate(kg)}
    pairs = [(ig[k], i) for i, k in enumerate(ko) if k in ig]
    unmatched = len(ko) - len(pairs) + len(kg) - len(pairs)
    gi = np.array([p[0] for p in pairs], int)
    oi = np.array([p[1] for p in pairs], int)
    A, B = rg[gi].astype(np.float64), ro[oi].astype(np.float64)
    relR = np.abs(A[:, 6] - B[:, 6]) / B[:, 6]
    bad = relR > RTOL
    errs = {}
    names = pp.EXT_FIELDS if nf == 33 else pp.BASIC_FIELDS
    for c, name in enumerate(names):
        a, b = A[~bad, c], B[~bad, c]
        fin = np.isfinite(b)
        if fin.any():
            sc = np.maximum(np.abs(b[fin]), 1e-3 * np.abs(b[fin]).max() + 1e-30)
            errs[name] = float(np.max(np.abs(a[fin] - b[fin]) / sc))
    return (unmatched + bad.sum()) / max(1, len(ko)), errs


@pytest.fixture(scope="module")
def tile64(ora, eh_pk, julia_table):
    cfg = tile_config()
    filters = filter_bank()
    st = ora.run_tile_stages(ora_config(ora, cfg), 42, *eh_pk, filters, julia_table)
    return cfg, filters, st


@pytest.mark.parametrize("mode", ["auto", "fused", "plain"])
def test_run_tile_vs_oracle(ctx, tile64, eh_pk, julia_table, mode):
    # fused: the filter bank's x pass fused with the peak search forced on at
    # 64^3 (by default it runs for 192, 320, 384 and 448^3 with ioutshear)
    cfg, filters, st = tile64
    T = julia_table
    ctx.set_pk_table(*eh_pk)
    ctx.set_collapse_table(pp.CollapseTable(T.data, T.x1, T.x2, T.y1, T.y2, T.z1, T.z2))
    ctx.set_option(pp.OPT_FUSED_X, 1 if mode == "fused" else -1)
    try:
        rec, rthlmax, npk = ctx.run_tile_arrays(cfg, 42, [f[2] for f in filters], plain=mode == "plain")
    finally:
        ctx.set_option(pp.OPT_FUSED_X, -1)
    ro = st["records"]
    assert rec.shape[1] == 33 and len(ro) > 200
    assert abs(npk - len(st["peaks"]["ipp"])) <= max(1, MISMATCH * npk)
    frac, errs = match_records(rec, ro, 33)
    assert small_tile_ok(frac, len(ro)), (frac, len(ro), errs)
    assert errs["RTHL"] < RTOL
    assert rthlmax == pytest.approx(float(ro[:, 6].max()), rel=RTOL)


def test_run_tile_records_match_oracle_on_identical_fields(ctx, tile64, julia_table):
    """Shell analysis + record packing of run_tile against the oracle on the
    GPU's own peak list: bit-level peak parity is then not needed and the
    halo bar (1e-4, 0.1 %) applies directly."""
    cfg, filters, st = tile64
    c = st
    T = julia_table
    ctx.set_collapse_table(pp.CollapseTable(T.data, T.x1, T.x2, T.y1, T.y2, T.z1, T.z2))
    g = ctx.analyse_peaks(c["fields"], c["peaks"]["ipp"], c["Rf"], c["ir2min"], c["ZZon"], c["fcrit"], c["alatt"],
                          c["nhunt"], plain=False)
    frac, errs = compare_results(g, c["results"])
    assert frac <= MISMATCH, (frac, errs)
    assert errs["RTHL"] < RTOL and errs["Fbarx"] < RTOL


def test_run_tile_lightcone(ctx, ora, eh_pk, julia_table):
    """ievol = 1: per-peak redshift from the comoving distance to the
    observer, per-peak fcrit and growth factor (Pipeline.jl:217-231, 252-271)."""
    cfg = tile_config(ievol=1, z_out=0.0, z_max=0.3)
    cfg.cenx, cfg.ceny, cfg.cenz = -300.0, -300.0, -300.0
    filters = filter_bank()
    st = ora.run_tile_stages(ora_config(ora, cfg), 17, *eh_pk, filters, julia_table)
    T = julia_table
    ctx.set_pk_table(*eh_pk)
    ctx.set_collapse_table(pp.CollapseTable(T.data, T.x1, T.x2, T.y1, T.y2, T.z1, T.z2))
    rec, _, _ = ctx.run_tile_arrays(cfg, 17, [f[2] for f in filters])
    assert len(st["records"]) > 50
    frac, errs = match_records(rec, st["records"], 33)
    assert small_tile_ok(frac, len(st["records"])), (frac, len(st["records"]), errs)
    # radii/masses carry the 1e-4 bar; velocities are means of psi over the
    # collapsed sphere and follow the single-precision FFT differences
    # between cuFFT and the oracle's transforms (a few 1e-5 relative)
    assert errs["RTHL"] < RTOL and errs["vx"] < 1e-3


def test_run_tile_11_field_and_1lpt(ctx, ora, eh_pk, julia_table):
    cfg = tile_config(ioutshear=0, ilpt=1)
    filters = filter_bank(8)
    st = ora.run_tile_stages(ora_config(ora, cfg), 5, *eh_pk, filters, julia_table)
    T = julia_table
    ctx.set_pk_table(*eh_pk)
    ctx.set_collapse_table(pp.CollapseTable(T.data, T.x1, T.x2, T.y1, T.y2, T.z1, T.z2))
    rec, _, _ = ctx.run_tile_arrays(cfg, 5, [f[2] for f in filters])
    assert rec.shape[1] == 11
    frac, errs = match_records(rec, st["records"], 11)
    assert small_tile_ok(frac, len(st["records"])), (frac, len(st["records"]), errs)
    assert np.all(rec[:, 7:10] == 0)


def test_run_tile_rejects_negative_rmax2rs(ctx, eh_pk, julia_table):
    cfg = tile_config()
    cfg.rmax2rs = -1.0
    T = julia_table
    ctx.set_pk_table(*eh_pk)
    ctx.set_collapse_table(pp.CollapseTable(T.data, T.x1, T.x2, T.y1, T.y2, T.z1, T.z2))
    with pytest.raises(pp.PPBError) as e:
        ctx.run_tile_arrays(cfg, 1, [3.0])
    assert e.value.code == -1


def test_run_tile_file_api(ctx, tmp_path, eh_pk):
    """run_tile(cfg; seed) reading the three input files and writing .pksc."""
    from peakpatch_b200 import powerspec
    pk = str(tmp_path / "pk.dat")
    powerspec.write_pk(pk, *eh_pk)
    fb = str(tmp_path / "filters.dat")
    pp.write_filterbank(fb, [f[2] for f in filter_bank(6)])
    cfg = tile_config()
    cfg.pkfile, cfg.filterfile, cfg.tabfile = pk, fb, os.path.join(GOLDEN, "HomelTab_julia.dat")
    cfg.fileout = str(tmp_path / "out.pksc")
    rec = ctx.run_tile(cfg, seed=3)
    r2, rthl, zo = pp.read_pksc(cfg.fileout)
    assert rec.tobytes() == r2.tobytes() and zo == 0.0   # bit for bit, NaN fields included
    assert rthl == pytest.approx(rec[:, 6].max()) if len(rec) else rthl == 0.0


@pytest.mark.parametrize("n,nbuff,ioutshear,seed", [(128, 5, 1, 3), (192, 12, 1, 8), (256, 32, 0, 11)])
def test_fused_filter_bank_matches_full_transforms(ctx, eh_pk, julia_table, n, nbuff, ioutshear, seed):
    """The filter bank with cuFFT's z/y passes and the fused x pass + peak
    search (grid sizes 64 J; PPB_OPT_FUSED_X 1) against the same optimised
    run with full 3-D C2R transforms and the separate peak search
    (PPB_OPT_FUSED_X 0): the same peaks up to single-precision FFT rounding,
    the same halos within the oracle bars."""
    cfg = tile_config(n=n, box=2.0 * n, nbuff=nbuff, ioutshear=ioutshear)
    filters = filter_bank()
    T = julia_table
    ctx.set_pk_table(*eh_pk)
    ctx.set_collapse_table(pp.CollapseTable(T.data, T.x1, T.x2, T.y1, T.y2, T.z1, T.z2))
    rf = [f[2] for f in filters]
    ctx.set_option(pp.OPT_FUSED_X, 1)
    try:
        fused, rmax_f, npk_f = ctx.run_tile_arrays(cfg, seed, rf, plain=False)
        ctx.set_option(pp.OPT_FUSED_X, 0)
        full, rmax_p, npk_p = ctx.run_tile_arrays(cfg, seed, rf, plain=False)
    finally:
        ctx.set_option(pp.OPT_FUSED_X, -1)
    nf = 33 if ioutshear else 11
    assert fused.shape[1] == nf and len(full) > 100
    assert abs(npk_f - npk_p) <= max(1, MISMATCH * npk_p), (npk_f, npk_p)
    frac, errs = match_records(fused, full, nf)
    assert small_tile_ok(frac, len(full)), (frac, len(full), errs)
    assert errs["RTHL"] < RTOL, errs
    assert rmax_f == pytest.approx(rmax_p, rel=RTOL)
