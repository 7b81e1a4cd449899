"""ppb_analyse_peaks_multirf (analyse_peaks_gpu_cuda_multirf,
src/PeakPatch.jl:231-253): batches of peaks, one filter scale each, with the
rmax2rs cell cap and a mask read before and written after each batch.

The oracle side restates the batch order on the host: for each batch, the
pre-mask test of RadialShell.jl:310-316 against the mask as it stood before
the batch, the oracle's analyse_peak (RadialShell.jl:282-891, with the npart
cap of :288-295) for the peaks it does not skip, then the mask writes of
:793-802 for the batch's halos."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import peakpatch_b200 as pp
from test_gpu_parity import MISMATCH, RTOL, compare_results


@pytest.fixture(scope="module")
def mr_case(ora, eh_pk):
    n, box, nbuff = 64, 128.0, 12
    alatt = box / n
    d = ora.generate_grf(n, *eh_pk, box, 23)
    dk = ora.rfft3(d)
    psi = ora.lpt1(dk, n, box)
    psi2 = ora.lpt2(dk, n, box)
    lapd = ora.laplacian(dk, n, box)
    fields = dict(delta=d, etax=psi[0], etay=psi[1], etaz=psi[2], eta2x=psi2[0], eta2y=psi2[1], eta2z=psi2[2],
                  lapd=lapd)
    fcrit = ora.fsc_of_z(0.315, 0.049, 0.685, 0.674, 0.0)
    mask = np.zeros(d.shape, np.int8)
    batches = []
    for R in (16.0, 8.0, 4.0, 2.6, 1.5):
        s = ora.smooth_field(dk, n, box, R, 1)
        p = ora.find_peaks(s, mask, 0, 0, 0, alatt, nbuff, np.float32(fcrit))
        ir2 = int(min(np.floor((1.75 * R / alatt) ** 2), np.floor((40 / alatt - 1) ** 2)))
        batches.append((p["i"].astype(np.int32), p["j"].astype(np.int32), p["k"].astype(np.int32), R, ir2))
    nhunt = min(nbuff - 1, int(np.floor(16.0 * 1.75 / alatt)))
    return dict(fields=fields, batches=batches, fcrit=fcrit, alatt=alatt, nbuff=nbuff, nhunt=nhunt, n=n)


def _table(ctx, T):
    ctx.set_collapse_table(pp.CollapseTable(T.data, T.x1, T.x2, T.y1, T.y2, T.z1, T.z2))


def oracle_multirf(ora, c, T, rmax2rs, mask):
    """The batch order on the host around the oracle's analyse_peak."""
    n, alatt, nbuff = c["n"], c["alatt"], c["nbuff"]
    shells = ora.precompute_shells(c["nhunt"])
    r = np.sqrt(shells[:, 3].astype(np.float64))
    f3p = 4.0 / 3.0 * np.pi
    out = []
    for (pi, pj, pk, Rf, ir2) in c["batches"]:
        ipp = (pi.astype(np.int64) - 1) + n * (pj.astype(np.int64) - 1) + n * n * (pk.astype(np.int64) - 1) + 1
        skip = np.zeros(len(ipp), bool)
        if rmax2rs > 0 and mask is not None:
            skip = mask.reshape(-1)[ipp - 1] > np.floor(Rf / alatt * rmax2rs)
        res = np.zeros((len(ipp), 31))
        res[:, 0] = -1.0
        res[:, 26] = -1.0
        keep = ~skip
        if keep.any():
            res[keep] = ora.analyse_peaks(c["fields"], ipp[keep], Rf, ir2, 1.0, c["fcrit"], alatt, shells, T,
                                          nbuff=nbuff, rmax2rs=rmax2rs)
        if mask is not None:
            npart = len(shells)
            if rmax2rs > 0:
                x = rmax2rs * Rf / alatt
                npart = min(int(np.floor(f3p * (x * x * x))), len(shells))
            flat = mask.reshape(-1)
            for q in np.where(res[:, 0] > 0)[0]:
                sel = np.where(r[:npart] <= res[q, 0])[0]
                iv = np.stack([pi[q] + shells[sel, 0], pj[q] + shells[sel, 1], pk[q] + shells[sel, 2]], 1)
                inside = np.all((iv >= nbuff + 1) & (iv <= n - nbuff), axis=1)
                iv = iv[inside] - 1
                flat[iv[:, 0] + n * iv[:, 1] + n * n * iv[:, 2]] = 1
        out.append(res)
    return out


def test_multirf_matches_flat_entry_point(ctx, mr_case, julia_table):
    """Without rmax2rs and mask the batches give the results of
    ppb_analyse_peaks on the same peaks, bit for bit."""
    c = mr_case
    _table(ctx, julia_table)
    res, _ = ctx.analyse_peaks_multirf(c["fields"], c["batches"], c["nhunt"], c["alatt"], fcrit=c["fcrit"])
    n = c["n"]
    for (pi, pj, pk, Rf, ir2), r in zip(c["batches"], res):
        ipp = (pi - 1) + n * (pj - 1) + n * n * (pk - 1) + 1
        flat = ctx.analyse_peaks(c["fields"], ipp, Rf, ir2, 1.0, c["fcrit"], c["alatt"], c["nhunt"])
        assert r.tobytes() == flat.tobytes()


@pytest.mark.parametrize("rmax2rs", [0.0, 1.0, 1.5])
def test_multirf_mask_and_rmax2rs_vs_oracle(ctx, ora, mr_case, julia_table, rmax2rs):
    c = mr_case
    _table(ctx, julia_table)
    rng = np.random.default_rng(5)
    mask0 = np.zeros((c["n"],) * 3, np.int8)
    # a caller's mask with values above one, so that the pre-mask test skips
    # peaks whose floor(Rf/alatt rmax2rs) is 1 as well
    for (pi, pj, pk, Rf, ir2) in c["batches"]:
        pick = rng.random(len(pi)) < 0.2
        mask0[pk[pick] - 1, pj[pick] - 1, pi[pick] - 1] = rng.integers(1, 3, pick.sum())
    mg, mo = mask0.copy(), mask0.copy()
    res_g, _ = ctx.analyse_peaks_multirf(c["fields"], c["batches"], c["nhunt"], c["alatt"], fcrit=c["fcrit"],
                                         mask=mg, nbuff=c["nbuff"], rmax2rs=rmax2rs)
    res_o = oracle_multirf(ora, c, julia_table, rmax2rs, mo)
    g, o = np.concatenate(res_g), np.concatenate(res_o)
    assert (o[:, 0] > 0).sum() > 100
    frac, errs = compare_results(g, o)
    assert frac <= MISMATCH, (frac, errs)
    assert errs["RTHL"] < RTOL
    if frac == 0:
        assert np.array_equal(mg, mo)
    if rmax2rs > 0:
        assert ((g[:, 0] == -1.0) & (o[:, 0] == -1.0)).sum() > 0


def test_multirf_lightcone_batches(ctx, ora, mr_case, julia_table):
    """7-tuple batches: per-peak ZZon and fcrit (the ievol = 1 caller)."""
    c = mr_case
    _table(ctx, julia_table)
    rng = np.random.default_rng(9)
    b7 = []
    for (pi, pj, pk, Rf, ir2) in c["batches"]:
        Z = 1.0 + rng.uniform(0.0, 0.5, len(pi))
        fc = np.array([ora.fsc_of_z(0.315, 0.049, 0.685, 0.674, z - 1.0) for z in Z])
        b7.append((pi, pj, pk, Rf, ir2, Z, fc))
    res_g, _ = ctx.analyse_peaks_multirf(c["fields"], b7, c["nhunt"], c["alatt"])
    n = c["n"]
    shells = ora.precompute_shells(c["nhunt"])
    for (pi, pj, pk, Rf, ir2, Z, fc), g in zip(b7, res_g):
        ipp = (pi.astype(np.int64) - 1) + n * (pj - 1) + n * n * (pk - 1) + 1
        o = ora.analyse_peaks(c["fields"], ipp, Rf, ir2, Z, fc, c["alatt"], shells, julia_table)
        frac, errs = compare_results(g, o)
        assert frac * max(1, (o[:, 0] > 0).sum()) <= max(1.0, MISMATCH * (o[:, 0] > 0).sum()), (frac, errs)
