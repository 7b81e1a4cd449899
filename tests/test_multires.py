"""The multi-resolution tile fields of run_multitile_split on the GPU against
the oracle (src/MultiResolution.jl).

Noise, residual and tricubic interpolation are integer/ordered float work
and must match bit for bit.  The FFT stages (isolated convolution, tile 2LPT
and Laplacian, coarse phase) run cuFFT in FP32 against the oracle's FP64
FFTs of the same Float32 inputs, so they are compared with a tolerance
relative to the field's largest value: 2e-5 (a few FP32 ulps of FFT
round-off; an indexing or kernel error is of order 1)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import peakpatch_b200 as pp

FFT_TOL = 2e-5


@pytest.fixture(scope="module")
def mctx(eh_pk):
    with pp.Context(0) as c:
        c.set_pk_table(*eh_pk)
        yield c


def _close(g, o, tol=FFT_TOL):
    g = np.asarray(g, np.float64)
    o = np.asarray(o, np.float64)
    scale = np.abs(o).max()
    assert scale > 0
    err = np.abs(g - o).max() / scale
    assert err <= tol, err
    return err


@pytest.mark.parametrize("N,M,seed", [(64, 8, 42), (60, 4, 7), (45, 5, 3), (32, 32, 11)])
def test_downsample_noise_bit_exact(mctx, ora, N, M, seed):
    # block 8 (Threefry pairs inside rows), 15 and 9 (odd: pairs straddle rows), 1
    g = mctx.downsample_noise(N, M, seed)
    o = ora.mr_coarse_noise(N, M, seed)
    assert g.tobytes() == o.tobytes()
    if N // M > 1:
        assert abs(float(g.std()) - 1.0) < 0.3


@pytest.mark.parametrize("tile,nshell", [((1, 1, 1), 0), ((2, 1, 2), 0), ((1, 2, 1), 3), ((2, 2, 2), 5)])
def test_extended_residual_bit_exact(mctx, ora, tile, nshell):
    N, M, nsub, nmesh, seed = 56, 8, 24, 32, 42
    coarse = ora.mr_coarse_noise(N, M, seed)
    g = mctx.generate_extended_residual(*tile, nsub, nmesh, N, seed, coarse, M, nshell)
    o = ora.mr_residual(coarse, M, *tile, nsub, nmesh, N, seed, nshell)
    assert g.shape == (nmesh + 2 * nshell,) * 3
    assert g.tobytes() == o.tobytes()


def test_residual_has_zero_block_means(mctx, ora):
    # Hoffman-Ribak: a tile covering whole coarse cells has residual block
    # sums of zero up to Float32 rounding
    N, M, seed = 32, 4, 5
    coarse = mctx.downsample_noise(N, M, seed)
    r = mctx.generate_extended_residual(1, 1, 1, 32, 32, N, seed, coarse, M, 0).astype(np.float64)
    b = N // M
    sums = r.reshape(M, b, M, b, M, b).sum(axis=(1, 3, 5))
    assert np.abs(sums).max() < 1e-3


@pytest.mark.parametrize("N,M,tile,nsub,nmesh", [(56, 8, (1, 1, 1), 24, 32), (56, 8, (2, 2, 1), 24, 32),
                                                 (45, 5, (1, 2, 3), 15, 21), (64, 16, (3, 1, 2), 20, 28)])
def test_interpolate_to_tile_bit_exact(mctx, ora, N, M, tile, nsub, nmesh):
    rng = np.random.default_rng(N + M)
    coarse = rng.standard_normal((M, M, M)).astype(np.float32)
    g = mctx.interpolate_to_tile_gpu(coarse, *tile, nsub, nmesh, N, M)
    o = ora.mr_tricubic(coarse, M, *tile, nsub, nmesh, N)
    assert g.tobytes() == o.tobytes()


def test_interpolate_constant_field(mctx):
    # Catmull-Rom weights sum to one: a constant coarse field interpolates to
    # itself up to rounding
    coarse = np.full((6, 6, 6), 2.5, np.float32)
    g = mctx.interpolate_to_tile_gpu(coarse, 1, 1, 1, 12, 16, 36, 6)
    assert np.abs(g - 2.5).max() < 1e-5


KERNELS = [(0, 0, 0), (1, 1, 0), (1, 2, 0), (1, 3, 0), (2, 2, 0), (3, 1, 2), (3, 3, 3), (4, 0, 0)]


@pytest.mark.parametrize("nmesh,nshell", [(24, 0), (20, 2), (25, 0)])
def test_isolated_convolve_vs_oracle(mctx, ora, eh_pk, nmesh, nshell):
    N, M, nsub, seed = 60, 5, nmesh - 4, 9
    alatt = 2.0
    coarse = ora.mr_coarse_noise(N, M, seed)
    resid = ora.mr_residual(coarse, M, 1, 2, 1, nsub, nmesh, N, seed, nshell)
    outs = mctx.isolated_convolve_gpu_multi(resid, None, nmesh * alatt, nmesh, KERNELS, nshell)
    for (kind, d1, d2), g in zip(KERNELS, outs):
        o = ora.isolated_convolve(resid, *eh_pk, nmesh * alatt, nmesh, kind, d1, d2, nshell)
        _close(g, o)


def test_isolated_convolve_region_wider_than_input(mctx, ora, eh_pk):
    # the kept region may reach into the zero padding (n + nshell up to
    # 2 n_input): the pruned inverse then transforms every plane
    rng = np.random.default_rng(5)
    noise = rng.standard_normal((12, 12, 12)).astype(np.float32)
    for n, nshell in ((20, 2), (12, 0), (5, 9)):
        g = mctx.isolated_convolve_gpu_multi(noise, None, 40.0, n, [(0, 0, 0), (1, 3, 0)], nshell)
        for (kind, d1, d2), x in zip([(0, 0, 0), (1, 3, 0)], g):
            _close(x, ora.isolated_convolve(noise, *eh_pk, 40.0, n, kind, d1, d2, nshell))


def test_isolated_convolve_multi_equals_single(mctx, ora):
    # kernels grouped into passes of up to four give the same bits as one
    # kernel per call
    rng = np.random.default_rng(3)
    noise = rng.standard_normal((16, 16, 16)).astype(np.float32)
    multi = mctx.isolated_convolve_gpu_multi(noise, None, 32.0, 16, KERNELS)
    for (kind, d1, d2), g in zip(KERNELS, multi):
        s = mctx.isolated_convolve_gpu(noise, None, 32.0, 16, kind, d1, d2)
        assert s.tobytes() == g.tobytes()


def test_isolated_convolve_is_linear(mctx):
    rng = np.random.default_rng(4)
    a = rng.standard_normal((16, 16, 16)).astype(np.float32)
    b = rng.standard_normal((16, 16, 16)).astype(np.float32)
    ks = [(0, 0, 0), (1, 2, 0)]
    fa = mctx.isolated_convolve_gpu_multi(a, None, 40.0, 16, ks)
    fb = mctx.isolated_convolve_gpu_multi(b, None, 40.0, 16, ks)
    fab = mctx.isolated_convolve_gpu_multi(a + b, None, 40.0, 16, ks)
    for x, y, z in zip(fa, fb, fab):
        _close(z, x.astype(np.float64) + y, 1e-5)


@pytest.mark.parametrize("n", [32, 27])
def test_tile_2lpt_and_laplacian_vs_oracle(mctx, ora, n):
    rng = np.random.default_rng(n)
    delta = rng.standard_normal((n, n, n)).astype(np.float32)
    box = 2.0 * n
    psi2 = mctx.compute_2lpt_gpu(delta, n, box)
    lap = mctx.compute_laplacian_gpu(delta, n, box)
    opsi2, olap = ora.tile_2lpt_laplacian(delta, n, box, 2, True)
    for d in range(3):
        _close(psi2[d], opsi2[d])
    _close(lap, olap)


@pytest.mark.parametrize("M,ilpt,ioutshear", [(16, 2, 1), (15, 1, 0)])
def test_coarse_fields_vs_oracle(mctx, ora, eh_pk, M, ilpt, ioutshear):
    N, seed = 4 * M, 12
    coarse = mctx.downsample_noise(N, M, seed)
    box = N * 2.0
    g = mctx.coarse_fields(coarse, None, box, ilpt, ioutshear)
    d, psi, psi2, lap = ora.coarse_fields(coarse, *eh_pk, box, ilpt, ioutshear)
    _close(g["delta"], d)
    for a in range(3):
        _close(g["psi"][a], psi[a])
    if ilpt >= 2:
        for a in range(3):
            _close(g["psi2"][a], psi2[a])
    else:
        assert g["psi2"] is None
    if ioutshear >= 1:
        _close(g["lapd"], lap)


def test_multires_argument_errors(mctx):
    coarse = np.zeros((4, 4, 4), np.float32)
    with pytest.raises(pp.PPBError):
        mctx.downsample_noise(30, 4, 1)            # N % M != 0
    with pytest.raises(pp.PPBError):
        mctx.generate_extended_residual(0, 1, 1, 8, 8, 32, 1, coarse, 4)   # tiles are 1-based
    noise = np.zeros((8, 8, 8), np.float32)
    with pytest.raises(pp.PPBError):
        mctx.isolated_convolve_gpu(noise, None, 16.0, 8, kernel_fn_id=5)
    with pytest.raises(pp.PPBError):
        mctx.isolated_convolve_gpu(noise, None, 16.0, 8, kernel_fn_id=1, dim1=4)
    with pytest.raises(pp.PPBError):
        mctx.isolated_convolve_gpu(noise, None, 16.0, 12, nshell=5)        # region outside the padded box
    # the context stays usable after rejected calls
    assert mctx.downsample_noise(8, 4, 1).shape == (4, 4, 4)


def test_compare_fields_split_reference_acceptance(mctx, ora):
    # the reference's "Field-level accuracy (ntile=2, N=120)" test
    # (test/test_multiresolution.jl:67-90) through the GPU stages, and the
    # same per-tile figures as the oracle
    from peakpatch_b200 import multires
    k = 10.0 ** np.linspace(-4, 1, 200)
    pk = (k, 1e4 * k ** -1.5)
    g = multires.compare_fields_split(mctx, pk, 120, 400.0, 42, 2, 5)
    o = ora.compare_fields_split(*pk, 120, 400.0, 42, 2, 5)
    assert len(g) == len(o) == 8
    for r, (tile, cd, rd, cp, rp) in zip(g, o):
        assert r["tile"] == tile
        assert r["corr_delta"] > 0.999 and r["rms_delta"] < 0.05
        assert r["corr_psi1"] > 0.93 and r["rms_psi1"] < 0.40
        assert abs(r["corr_delta"] - cd) < 1e-5 and abs(r["rms_delta"] - rd) < 1e-4
        assert abs(r["corr_psi1"] - cp) < 1e-4 and abs(r["rms_psi1"] - rp) < 1e-4
