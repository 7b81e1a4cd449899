"""Pins of the oracle's multi-resolution restatement (src/MultiResolution.jl)
on CPU.

The reference's own acceptance tests for the split are field-level: per tile,
the split delta and psi_x must track the global-FFT fields on the tile core
(test/test_multiresolution.jl:67-120, thresholds copied from there).  The
residual and coarse noise are also checked against the oracle's global
Threefry noise (src/InitialConditions/RandomField.jl:70-83)."""
import numpy as np
import pytest


def _pk():
    # the P(k) of the reference's test (test/test_multiresolution.jl:52-63)
    k = 10.0 ** np.linspace(-4, 1, 200)
    return k, 1e4 * k ** -1.5


def test_split_tracks_global_fields(ora):
    # "Field-level accuracy (ntile=2, N=120)": nsub 52, nmesh 68, M 10
    for tile, cd, rd, cp, rp in ora.compare_fields_split(*_pk(), 120, 400.0, 42, 2, 5):
        assert cd > 0.999 and rd < 0.05, (tile, cd, rd)
        assert cp > 0.93 and rp < 0.40, (tile, cp, rp)


@pytest.mark.parametrize("cf", [3, 6, 20])
def test_split_coarse_factor_sweep(ora, cf):
    # "Coarse factor sweep (N=120)": mean over tiles
    r = ora.compare_fields_split(*_pk(), 120, 400.0, 42, 2, cf)
    assert np.mean([x[1] for x in r]) > 0.99
    assert np.mean([x[2] for x in r]) < 0.15


def test_residual_is_noise_minus_block_mean(ora):
    # fine noise (the global field's Float32 values) minus the coarse cell
    # times Float32(1/sqrt(block^3)), in Float32, bit for bit
    N, M, nsub, nmesh, seed = 24, 4, 8, 12, 17
    coarse = ora.mr_coarse_noise(N, M, seed)
    g = ora.noise(N, seed)
    b = N // M
    inv = np.float32(1.0 / np.sqrt(float(b) ** 3))
    for tile, nshell in (((1, 1, 1), 0), ((3, 2, 1), 2)):
        r = ora.mr_residual(coarse, M, *tile, nsub, nmesh, N, seed, nshell)
        o = [(t - 1) * nsub - (nmesh - nsub) // 2 - nshell for t in tile]
        ne = nmesh + 2 * nshell
        idx = [np.arange(o[d], o[d] + ne) % N for d in range(3)]
        fine = g[np.ix_(idx[2], idx[1], idx[0])]
        bm = coarse[np.ix_(idx[2] // b, idx[1] // b, idx[0] // b)] * inv
        assert r.tobytes() == (fine - bm).astype(np.float32).tobytes()


def test_coarse_noise_is_scaled_block_sum(ora):
    # block sums of the Float64 deviates vs the Float32-rounded field: equal
    # to the rounding of the stored noise
    N, M, seed = 24, 3, 8
    c = ora.mr_coarse_noise(N, M, seed).astype(np.float64)
    g = ora.noise(N, seed).astype(np.float64)
    b = N // M
    s = g.reshape(M, b, M, b, M, b).sum(axis=(1, 3, 5)) / np.sqrt(b ** 3)
    assert np.abs(c - s).max() < 1e-5


def test_tricubic_reproduces_constant_and_coarse_nodes(ora):
    M, N = 6, 36
    c = np.full((M, M, M), -1.25, np.float32)
    t = ora.mr_tricubic(c, M, 1, 1, 1, 12, 16, N)
    assert np.abs(t + 1.25).max() < 1e-5
    # with block 1 every fine cell sits on a coarse node: interpolation is the
    # identity (Catmull-Rom weights (0, 1, 0, 0) at t = 0)
    rng = np.random.default_rng(1)
    c = rng.standard_normal((8, 8, 8)).astype(np.float32)
    t = ora.mr_tricubic(c, 8, 1, 1, 1, 8, 8, 8)
    assert t.tobytes() == c.tobytes()


def _ref_config(ora, ilpt):
    # _make_config(n=68, boxsize=226.67, z=0, ilpt, nbuff=8) of
    # test/test_multiresolution.jl:10-46
    return ora.Config(Omx=0.261, OmB=0.049, Omvac=0.69, h=0.68, n=68, boxsize=226.67, nbuff=8, z_out=0.0, z_max=0.0,
                      ievol=0, ilpt=ilpt, ioutshear=0, wsmooth=1, rmax2rs=0.0)


@pytest.fixture(scope="module")
def ref_table(ora):
    # make_table for CosmologyParams(0.31, 0.049, 0.69, 0.68) with the default
    # table parameters, stored as Float32 like write_homeltab
    tp = ora.TableParams()
    d = ora.make_table(0.31, 0.049, 0.69, 0.68, tp).astype(np.float32)
    return ora.Table(d, tp.Nx, tp.Ny, tp.Nz, tp.X1, tp.X2, tp.Y1, tp.Y2, tp.Z1, tp.Z2)


REF_FILTERS = [(1, 1.686, 8.0), (2, 1.686, 5.0), (3, 1.686, 3.0)]


@pytest.mark.parametrize("ilpt", [1, 2])
def test_split_halo_count_tracks_global(ora, ref_table, ilpt):
    # "Halo count comparison (ntile=2, 1LPT / 2LPT)"
    # (test/test_multiresolution.jl:123-170): split vs global FFT within 5 %
    cfg = _ref_config(ora, ilpt)
    k, p = _pk()
    g, _ = ora.run_multitile(cfg, 42, k, p, REF_FILTERS, ref_table, ntile=2)
    s, _ = ora.run_multitile_split(cfg, 42, k, p, REF_FILTERS, ref_table, ntile=2, coarse_factor=5)
    assert len(g) > 50
    assert abs(len(s) - len(g)) / len(g) < 0.05 or abs(len(s) - len(g)) <= 3, (len(s), len(g))


def test_split_coarse_grid_choice(ora):
    # coarse_grid wins, then ntile coarse_factor, then the divisor whose block
    # is closest to nmesh/3 (src/MultiResolution.jl:592-612)
    assert ora.split_coarse_grid(120, 68, 2, 5, 0) == 10
    assert ora.split_coarse_grid(120, 68, 2, 5, 24) == 24
    assert ora.split_coarse_grid(120, 68, 2) == 5        # block 24 ~ 68 // 3 = 22 (block 20 ties later)
    assert 120 % ora.split_coarse_grid(120, 60, 3) == 0
