"""The batched shell analysis as a stand-alone entry point: per-peak shell-list
limits (ppb_analyse_peaks_lim), a Float64 collapse table and the field
generator (ppb_generate_fields), each against the oracle or against the
existing path."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import peakpatch_b200 as pp
from test_gpu_parity import RTOL, compare_results, tile_config


@pytest.fixture(scope="module")
def setup(ora, julia_table, eh_pk):
    T = julia_table
    n, box = 64, 128.0
    cfg = ora.Config(Omx=0.315 - 0.049, OmB=0.049, Omvac=0.685, h=0.674, n=n, boxsize=box, nbuff=16, z_out=0.0,
                     z_max=0.0, ievol=0, ilpt=2, ioutshear=1, wsmooth=1, rmax2rs=0.0)
    k, P = eh_pk
    d = ora.generate_grf(n, k, P, box, 11)
    dk = ora.rfft3(d)
    psi = ora.lpt1(dk, n, box)
    psi2 = ora.lpt2(dk, n, box)
    fields = dict(delta=d, etax=psi[0], etay=psi[1], etaz=psi[2], eta2x=psi2[0], eta2y=psi2[1], eta2z=psi2[2],
                  lapd=ora.laplacian(dk, n, box))
    # peak cells: the smoothed field's peaks plus uniform cells, 13..51 per axis
    ds = ora.smooth_field(dk, n, box, 6.0, 1)
    pk = ora.find_peaks(ds, np.zeros((n, n, n), np.int8), 0.0, 0.0, 0.0, 2.0, 13, np.float32(0.2))
    rng = np.random.default_rng(4)
    ijk = rng.integers(13, 51, size=(300, 3))
    ipp = np.concatenate([pk["ipp"], 1 + ijk[:, 0] + n * ijk[:, 1] + n * n * ijk[:, 2]]).astype(np.int64)
    R = rng.choice([4, 6, 9, 12], size=len(ipp))
    return dict(T=T, fields=fields, ipp=ipp, R=R, n=n, cfg=cfg)


def _args(S, sel):
    alatt = 2.0
    R = S["R"][sel]
    Rf = R * alatt
    ir2 = np.minimum(np.floor((1.75 * Rf / alatt) ** 2), np.floor((40.0 / alatt - 1) ** 2)).astype(np.int64)
    return S["ipp"][sel], Rf, ir2, np.ones(len(R)), np.full(len(R), 1.686), alatt


@pytest.mark.parametrize("plain", [False, True])
def test_per_peak_shell_limits_vs_oracle(ctx, ora, setup, plain):
    S = setup
    T = S["T"]
    ctx.set_collapse_table(pp.CollapseTable(T.data, T.x1, T.x2, T.y1, T.y2, T.z1, T.z2))
    allsel = np.arange(len(S["ipp"]))
    ipp, Rf, ir2, Z, fc, alatt = _args(S, allsel)
    g = ctx.analyse_peaks(S["fields"], ipp, Rf, ir2, Z, fc, alatt, 12, plain=plain, r2lim=S["R"] ** 2)
    o = np.zeros_like(g)
    for R in np.unique(S["R"]):   # the oracle analyses each limit with its own shell list
        sel = np.where(S["R"] == R)[0]
        a = _args(S, sel)
        o[sel] = ora.analyse_peaks(S["fields"], *a, ora.precompute_shells(int(R)), T)
    assert (o[:, 0] > 0).sum() > 20
    frac, errs = compare_results(g, o)
    assert frac <= 1e-3 and errs.get("RTHL", 0) < RTOL, (frac, errs)
    # the limit matters: the whole 12-cell list gives other results for small R
    g12 = ctx.analyse_peaks(S["fields"], ipp, Rf, ir2, Z, fc, alatt, 12, plain=plain)
    assert not np.array_equal(np.nan_to_num(g12), np.nan_to_num(g))


def test_f64_table_gives_the_f32_table_results(ctx, setup):
    S = setup
    T = S["T"]
    ipp, Rf, ir2, Z, fc, alatt = _args(S, np.arange(len(S["ipp"])))
    ctx.set_collapse_table(pp.CollapseTable(T.data, T.x1, T.x2, T.y1, T.y2, T.z1, T.z2))
    a = ctx.analyse_peaks(S["fields"], ipp, Rf, ir2, Z, fc, alatt, 12, r2lim=S["R"] ** 2)
    ctx.set_collapse_table_f64(T.data.astype(np.float64), (T.x1, T.x2, T.y1, T.y2, T.z1, T.z2))
    b = ctx.analyse_peaks(S["fields"], ipp, Rf, ir2, Z, fc, alatt, 12, r2lim=S["R"] ** 2)
    ctx.set_collapse_table(pp.CollapseTable(T.data, T.x1, T.x2, T.y1, T.y2, T.z1, T.z2))
    assert a.tobytes() == b.tobytes()


def test_generate_fields_vs_oracle(ctx, ora, eh_pk):
    cfg = tile_config(n=64, box=128.0)
    ctx.set_pk_table(*eh_pk)
    g = ctx.generate_fields(cfg, 11)
    k, P = eh_pk
    d = ora.generate_grf(64, k, P, 128.0, 11)
    dk = ora.rfft3(d)
    psi = ora.lpt1(dk, 64, 128.0)
    psi2 = ora.lpt2(dk, 64, 128.0)
    ref = dict(delta=d, etax=psi[0], etay=psi[1], etaz=psi[2], eta2x=psi2[0], eta2y=psi2[1], eta2z=psi2[2],
               lapd=ora.laplacian(dk, 64, 128.0))
    for key, r in ref.items():
        err = np.abs(g[key].astype(np.float64) - r) / np.sqrt(np.mean(r.astype(np.float64) ** 2))
        assert err.max() < 2e-5, (key, err.max())
