"""Pins the CPU oracle against the reference's own known-answer tests and
golden values (PeakPatch.jl test/*.jl, read as text), before the oracle is
used to check the GPU path.  CPU only."""
import os
import struct

import numpy as np
import pytest

from conftest import GOLDEN


# ---------------------------------------------------------------- RadialShell
def test_hRinteg_boundary_values(ora):
    # test/test_radialshell.jl:3-26
    assert ora.hRinteg(0.0, 0.0) == pytest.approx(1.4 * 0.0 - 31.0 / 35.0, abs=1e-12)
    assert ora.hRinteg(0.0, 1.5) == pytest.approx(1.4 * 1.5 - 31.0 / 35.0, abs=1e-12)
    assert ora.hRinteg(2.0, 0.0) == 0.0
    assert ora.hRinteg(3.0, 1.0) == 0.0
    assert ora.hRinteg(1.0, 0.0) == pytest.approx(-3.2 / 7.0, abs=1e-12)
    assert ora.hRinteg(0.5, 2.0) == pytest.approx(ora.hRinteg(-0.5, 2.0))
    assert ora.hRinteg(0.5, 1.0) != ora.hRinteg(0.5, 2.0)


def test_atab4(ora):
    # test/test_radialshell.jl:36-52
    akk = ora.atab4()
    assert len(akk) == 1101
    ca = 3.0 / (2.0 * np.pi)
    assert akk[0] == pytest.approx(ca * 2.0 / 3.0, abs=1e-14)
    assert akk[400] == 0.0 and akk[499] == 0.0 and akk[1099] == 0.0
    cb = 1.0 / (4.0 * np.pi)
    assert ca * (2.0 / 3.0 - 1.0 + 0.5) == pytest.approx(cb, abs=1e-14)


def test_precompute_shells(ora):
    # test/test_radialshell.jl:54-71
    c1 = ora.precompute_shells(1)
    assert len(c1) == 7 and c1[0, 3] == 0 and (c1[:, 3] <= 1).all()
    c2 = ora.precompute_shells(2)
    assert len(c2) == 33
    assert (np.diff(c2[:, 3]) >= 0).all()
    # shell geometry used by the configurations: radius 26 -> 73,525 cells in
    # 566 distinct r^2 values; radius 40 -> 267,761 cells
    c26 = ora.precompute_shells(26)
    assert len(c26) == 73525 and len(np.unique(c26[:, 3])) == 566
    assert len(ora.precompute_shells(40)) == 267761


def test_get_evals(ora):
    # test/test_radialshell.jl:73-84
    assert np.allclose(ora.eigvals_sym(np.eye(3)), [1, 1, 1], atol=1e-12)
    assert np.allclose(ora.eigvals_sym(np.diag([1.0, 2.0, 3.0])), [1, 2, 3], atol=1e-12)
    rng = np.random.default_rng(1)
    for _ in range(200):
        a = rng.normal(size=(3, 3))
        a = a + a.T
        assert np.allclose(ora.eigvals_sym(a), np.linalg.eigvalsh(a), rtol=1e-12, atol=1e-12)


def _synthetic_pg(n, fill=0.0):
    z = lambda: np.zeros((n, n, n), np.float32)
    d = np.full((n, n, n), fill, np.float32)
    return dict(delta=d, etax=z(), etay=z(), etaz=z())


def test_analyse_peak_synthetic_collapse(ora):
    # test/test_radialshell.jl:95-130: 20^3, delta 5 in the 3^3 block, 10 at
    # the centre, table of ones, shells(8): collapses
    n = 20
    f = _synthetic_pg(n)
    f["delta"][8:11, 8:11, 8:11] = 5.0
    T = ora.Table(np.ones((3, 3, 5), np.float32), 5, 3, 3, np.log10(1.5), np.log10(8.0), 0.0, 0.5,
                  -1 + 1e-4, 1 - 1e-4)
    ipp = 10 + 9 * n + 9 * n * n
    r = ora.analyse_peaks(f, [ipp], [4.0], [4], [0.0], [1.686], 1.0, ora.precompute_shells(8), T)[0]
    assert r[0] > 0.0 and r[1] > 0.0


def test_analyse_peak_no_collapse(ora):
    # test/test_radialshell.jl:132-156
    n = 20
    f = _synthetic_pg(n, fill=0.5)
    T = ora.Table(np.full((3, 3, 5), 100.0, np.float32), 5, 3, 3, np.log10(1.5), np.log10(8.0), 0.0, 0.5,
                  -1 + 1e-4, 1 - 1e-4)
    ipp = 10 + 9 * n + 9 * n * n
    r = ora.analyse_peaks(f, [ipp], [4.0], [4], [0.0], [1.686], 1.0, ora.precompute_shells(8), T)[0]
    assert r[0] == -1.0


def fortran_golden_fields(n=142):
    """test/test_radialshell_fortran.jl:191-217: delta(71,71,71) = 10, the six
    face neighbours 5, with the listed 1LPT displacements."""
    z = lambda: np.zeros((n, n, n), np.float32)
    d, ex, ey, ez = z(), z(), z(), z()

    def S(a, i, j, k, v):
        a[k - 1, j - 1, i - 1] = v

    S(d, 71, 71, 71, 10.0)
    for (i, j, k) in [(70, 71, 71), (72, 71, 71), (71, 70, 71), (71, 72, 71), (71, 71, 70), (71, 71, 72)]:
        S(d, i, j, k, 5.0)
    for a, vals in ((ex, [0.1, 0.05, 0.15, 0.1, 0.1, 0.1, 0.1]), (ey, [0.2, 0.2, 0.2, 0.1, 0.3, 0.2, 0.2]),
                    (ez, [0.3, 0.3, 0.3, 0.3, 0.3, 0.15, 0.45])):
        for (i, j, k), v in zip([(71, 71, 71), (70, 71, 71), (72, 71, 71), (71, 70, 71), (71, 72, 71),
                                 (71, 71, 70), (71, 71, 72)], vals):
            S(a, i, j, k, v)
    return dict(delta=d, etax=ex, etay=ey, etaz=ez)


FORTRAN_GOLDEN = dict(  # test/test_radialshell_fortran.jl:169-186
    fcrit=1.7161525487899780, RTHL=1.7320507764816284, Srb=1.9020472764968872, Fbarx=2.3230779170989990,
    Sbar=(2.5925926864147186e-02, 5.1851853728294373e-02, 7.7777773141860962e-02),
    strain_diag=(3.8717970252037048e-01, 7.7435940504074097e-01, 1.1615388393402100e+00),
    e_v=1.6666662693023682e-01, p_v=-5.1315236504478889e-08, zvir_half=-1.0)


def check_fortran_golden(r, rtol=0.01):
    G = FORTRAN_GOLDEN
    assert r[0] > 0
    assert abs(r[0] - G["RTHL"]) / G["RTHL"] < rtol
    assert abs(r[1] - G["Srb"]) / G["Srb"] < rtol
    assert abs(r[23] - G["Fbarx"]) / G["Fbarx"] < rtol
    for L in range(3):
        assert abs(r[2 + L] - G["Sbar"][L]) < 0.01 * max(rtol / 0.01, 1)
        assert abs(r[5 + L]) < 0.01
        assert abs(r[17 + L]) < 0.01 and abs(r[20 + L]) < 0.01
    strain = r[8:17].reshape(3, 3, order="F")
    for L in range(3):
        for K in range(3):
            v = G["strain_diag"][L] if L == K else 0.0
            if v:
                assert abs(strain[L, K] - v) / v < rtol
            else:
                assert abs(strain[L, K]) < 0.01
    assert abs(r[24] - G["e_v"]) / G["e_v"] < rtol
    assert abs(r[25] - G["p_v"]) < 0.01
    assert abs(r[26] - G["zvir_half"]) < 0.01


def test_fortran_get_homel_golden(ora, fortran_table):
    f = fortran_golden_fields()
    ipp = 71 + 70 * 142 + 70 * 142 * 142
    r = ora.analyse_peaks(f, [ipp], [4.0], [4], [1.0], [FORTRAN_GOLDEN["fcrit"]], 1.0, ora.precompute_shells(8),
                          fortran_table)[0]
    check_fortran_golden(r, rtol=0.01)
    # the restatement is far tighter than the reference's 1 % tolerance
    check_fortran_golden(r, rtol=1e-6)


# ---------------------------------------------------------------- PeakFind
def _pf(ora, delta, mask=None, nbuff=1, alatt=1.0, box=(0.0, 0.0, 0.0), fcrit=1.0, max_peaks=2000000):
    mask = np.zeros(delta.shape, np.int8) if mask is None else mask
    return ora.find_peaks(delta, mask, *box, alatt, nbuff, fcrit, max_peaks), mask


def _set(a, i, j, k, v):
    a[k - 1, j - 1, i - 1] = v


def test_peakfind_kats(ora):
    # test/test_peakfind.jl:4-118
    n = 11
    d = np.zeros((n, n, n), np.float32)
    _set(d, 6, 6, 6, 2.0)
    p, m = _pf(ora, d)
    assert len(p["i"]) == 1 and (p["i"][0], p["j"][0], p["k"][0]) == (6, 6, 6) and p["delta"][0] == 2.0
    assert m[5, 5, 5] == 1
    p, _ = _pf(ora, np.full((n, n, n), 0.5, np.float32))
    assert len(p["i"]) == 0
    g = np.fromfunction(lambda k, j, i: (i + 1) + (j + 1) + (k + 1), (n, n, n)).astype(np.float32)
    assert len(_pf(ora, g)[0]["i"]) == 0
    mk = np.zeros((n, n, n), np.int8)
    mk[5, 5, 5] = 1
    assert len(_pf(ora, d, mask=mk)[0]["i"]) == 0
    b = np.zeros((n, n, n), np.float32)
    _set(b, 1, 6, 6, 2.0)
    assert len(_pf(ora, b)[0]["i"]) == 0
    n2 = 15
    d2 = np.zeros((n2,) * 3, np.float32)
    _set(d2, 4, 4, 4, 2.0)
    _set(d2, 12, 12, 12, 3.0)
    p, _ = _pf(ora, d2)
    assert list(zip(p["i"], p["j"], p["k"])) == [(4, 4, 4), (12, 12, 12)]
    d3 = np.zeros((n,) * 3, np.float32)
    _set(d3, 3, 5, 7, 2.0)
    p, _ = _pf(ora, d3)
    assert p["ipp"][0] == 3 + 4 * 11 + 6 * 121
    d4 = np.zeros((21,) * 3, np.float32)
    _set(d4, 11, 11, 11, 2.0)
    p, _ = _pf(ora, d4, alatt=2.0, box=(10.0, 20.0, 30.0))
    assert (p["x"][0], p["y"][0], p["z"][0]) == (10.0, 20.0, 30.0)
    d5 = np.zeros((n2,) * 3, np.float32)
    for ijk in [(4, 4, 4), (4, 4, 12), (12, 12, 4), (12, 12, 12)]:
        _set(d5, *ijk, 2.0)
    assert len(_pf(ora, d5, max_peaks=2)[0]["i"]) == 2


# ---------------------------------------------------------------- Filters
def test_windows(ora):
    # test/test_filters.jl:3-55
    for kR in [0.0, 0.1, 0.5, 1.0, 2.0, 5.0]:
        assert ora.window(kR, 1.0, 0) == pytest.approx(np.exp(-kR ** 2 / 8), rel=1e-10)
    for kR in [0.01, 0.1, 0.5, 1.0, 2.0, 5.0]:
        assert ora.window(kR, 1.0, 1) == pytest.approx(3 * (np.sin(kR) - kR * np.cos(kR)) / kR ** 3, rel=1e-10)
    assert ora.window(0.0, 0.0, 1) == 1.0
    assert ora.window(4.0, 1.0, 1) > 0 and ora.window(5.0, 1.0, 1) < 0
    assert ora.window(0.01, 1.0, 1) > 0.999


def test_filterbank_io(ora, tmp_path):
    p = tmp_path / "f.dat"
    p.write_text("3\n1  1.686  2.0\n2  1.686  4.0\n3  1.686  8.0\n")
    assert ora.read_filterbank(str(p)) == [(1, 1.686, 2.0), (2, 1.686, 4.0), (3, 1.686, 8.0)]


# ---------------------------------------------------------------- CollapseTable
def test_trilinear_kats(ora):
    # test/test_ellipsoidalcollapse.jl:127-151: table = x + y + z
    g = np.arange(11) * 0.1
    t = (g[None, None, :] + g[None, :, None] + g[:, None, None]).astype(np.float32)
    T = ora.Table(t, 11, 11, 11, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    assert ora.table_interp(T, 0.0, 0.0, 0.0) == pytest.approx(0.0, abs=1e-5)
    assert ora.table_interp(T, 0.5, 0.0, 0.0) == pytest.approx(0.5, abs=1e-5)
    assert ora.table_interp(T, 0.0, 0.5, 0.0) == pytest.approx(0.5, abs=1e-5)
    assert ora.table_interp(T, 0.25, 0.25, 0.25) == pytest.approx(0.75, abs=1e-4)
    assert ora.table_interp(T, -0.1, 0.0, 0.0) == -1.0
    assert ora.table_interp(T, 1.1, 0.0, 0.0) == -1.0
    assert ora.table_interp(T, float("nan"), 0.0, 0.0) == -1.0


def test_homeltab_fixtures(ora, fortran_table, julia_table):
    # test/data/HomelTab_{fortran,julia}.dat: 50 x 20 x 20 over
    # [log10 1.5, log10 8] x [0, 0.5] x [-0.9999, 0.9999]
    for T in (fortran_table, julia_table):
        assert (T.nx, T.ny, T.nz) == (50, 20, 20)
        assert T.x1 == pytest.approx(np.log10(1.5), rel=1e-6) and T.x2 == pytest.approx(np.log10(8.0), rel=1e-6)
        assert (T.y1, T.y2) == (0.0, 0.5)
        assert T.z1 == pytest.approx(-0.9999, rel=1e-6)
        assert T.data.min() == -1.0
    a, b = fortran_table.data, julia_table.data
    ok = (a > 0) & (b > 0)
    # the two generators agree closely on the collapsed entries
    assert np.median(np.abs(a[ok] - b[ok]) / a[ok]) < 0.01


# ---------------------------------------------------------------- Catalog
def test_pksc_layout(ora, tmp_path):
    # test/test_catalog.jl:71-119: 12-byte header + N * 33 * 4 bytes
    rec = np.arange(2 * 33, dtype=np.float32).reshape(2, 33)
    p = str(tmp_path / "c.pksc")
    ora.write_pksc(p, rec, 3.5, 0.25)
    raw = open(p, "rb").read()
    assert len(raw) == 12 + 2 * 33 * 4
    assert struct.unpack("<i2f", raw[:12]) == (2, 3.5, 0.25)
    assert np.array_equal(np.frombuffer(raw[12:], "<f4").reshape(2, 33), rec)


# ---------------------------------------------------------------- RandomField
def test_threefry_known_answer():
    """Random123's published known-answer value for Threefry-2x64-20 with
    zero key and zero counter."""
    import ctypes, subprocess, tempfile
    src = r'''
#include "ppb_math.h"
#include <cstdio>
int main(){ uint64_t a,b; ppbm::threefry2x64_20(0,0,0,0,&a,&b); printf("%016llx %016llx\n",(unsigned long long)a,(unsigned long long)b); }
'''
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    with tempfile.TemporaryDirectory() as d:
        cpp = os.path.join(d, "k.cpp")
        open(cpp, "w").write(src)
        exe = os.path.join(d, "k")
        subprocess.run(["/usr/bin/g++", "-O2", "-ffp-contract=off", "-I",
                        os.path.join(root, "peakpatch.jl_b200", "csrc"), cpp, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    assert out == ["c2b6e3a8c2c69865", "6f81ed42f350084d"]


def test_noise_determinism_region_decomposition(ora):
    # test/test_randomfield.jl:103-190
    a = ora.noise(32, 42)
    assert np.array_equal(a, ora.noise(32, 42))
    assert not np.array_equal(a, ora.noise(32, 99))
    full = ora.noise(64, 42)
    for (r1, r2, r3) in [((0, 32), (0, 32), (0, 32)), ((32, 64), (0, 64), (0, 64)), ((9, 50), (19, 60), (4, 45)),
                         ((0, 1), (0, 1), (0, 1))]:
        reg = ora.noise_region(64, 42, r1, r2, r3)
        assert np.array_equal(reg, full[r3[0]:r3[1], r2[0]:r2[1], r1[0]:r1[1]])
    assert np.all(np.isfinite(full))


def test_noise_gaussian_statistics(ora):
    # test/test_randomfield.jl:134-158
    x = ora.noise(128, 42).astype(np.float64)
    assert abs(x.mean()) < 0.01 and abs(x.std() - 1.0) < 0.01
    y = ora.noise(128, 77).astype(np.float64)
    s = (y - y.mean()) / y.std()
    assert abs((s ** 3).mean()) < 0.05 and abs((s ** 4).mean() - 3.0) < 0.1


def test_noise_matches_libm_box_muller(ora):
    """The project's own log/sin/cos (ppb_math.h) agree with the platform libm
    to within an ulp, so the Float32 noise equals a libm-based Box-Muller on
    (essentially) every cell: at most 1 in 10^7 may round differently."""
    n = 128
    a = ora.noise(n, 42)
    b = ora.noise_libm(n, 42)
    assert np.count_nonzero(a != b) <= max(1, a.size // 10_000_000)


# ---------------------------------------------------------------- GRF / LPT
def test_grf_variance_flat_spectrum(ora):
    # test/test_randomfield.jl:59-82: P = A -> variance A n^3 dk^3
    n, box, A = 32, 100.0, 0.5
    k = np.logspace(-4, 2, 50)
    f = ora.generate_grf(n, k, np.full_like(k, A), box, 42).astype(np.float64)
    dk = 2 * np.pi / box
    assert f.var() == pytest.approx(A * n ** 3 * dk ** 3, rel=0.05)
    assert abs(f.mean()) < 1e-3 * f.std()


def test_lpt_divergence_identities(ora, eh_pk):
    # test/test_lpt.jl: div psi1 = -delta (spectrally, away from Nyquist)
    n, box = 32, 64.0
    d = ora.generate_grf(n, *eh_pk, box, 3)
    dk_ = ora.rfft3(d)
    psi = ora.lpt1(dk_, n, box)
    kk = 2 * np.pi / box
    kx = np.fft.rfftfreq(n, 1 / n) * kk
    ky = np.fft.fftfreq(n, 1 / n) * kk
    div = 1j * (kx[None, None, :] * ora.rfft3(psi[0]) + ky[None, :, None] * ora.rfft3(psi[1]) +
                ky[:, None, None] * ora.rfft3(psi[2]))
    ny = n // 2
    sel = np.ones(div.shape, bool)
    sel[:, :, -1] = False
    sel[:, ny, :] = False
    sel[ny, :, :] = False
    sel[0, 0, 0] = False
    err = np.abs(div[sel] + dk_[sel]) / (np.abs(dk_[sel]).max())
    assert err.max() < 1e-5


# ---------------------------------------------------------------- Cosmology
def test_growth_and_distance(ora):
    # test/test_cosmology.jl: D(a=1) = 1 (within the table's interpolation),
    # chi(z=1) in (1500, 1600) for Planck-like parameters
    Om, OB, OL, h = 0.2645 + 0.0493, 0.0493, 1.0 - 0.2645 - 0.0493, 0.6735
    assert ora.dlinear(Om, OB, OL, h, [1.0])[0] == pytest.approx(1.0, abs=1e-5)
    assert 1500 < ora.chi(Om, OL, h, 1.0) < 1600
    assert ora.fsc_of_z(0.315, 0.049, 0.685, 0.674, 0.0) == pytest.approx(1.686, rel=1e-5)
    d = ora.dlinear(0.315, 0.049, 0.685, 0.674, [0.25, 0.5, 1.0, 1.5])
    assert np.all(np.diff(d) > 0)
    z = ora.chi_to_z(0.315, 0.685, 0.674, 5.6, [ora.chi(0.315, 0.685, 0.674, zz) for zz in (0.5, 1.0, 3.0)])
    assert np.allclose(z, [0.5, 1.0, 3.0], rtol=1e-4)


# ------------------------------------------------------------------ merge_catalog
def _halos(xyz, r, nf=11):
    rec = np.zeros((len(r), nf), np.float32)
    rec[:, :3] = np.asarray(xyz, np.float32)
    rec[:, 6] = np.asarray(r, np.float32)
    rec[:, 3] = np.arange(len(r))   # tag
    return rec


def test_sphere_overlap_kats(ora):
    # test/test_merger.jl:7-47
    assert ora.sphere_overlap(10.0, 2.0, 3.0) == (0.0, 0.0)
    assert ora.sphere_overlap(5.0, 2.0, 3.0) == (0.0, 0.0)
    assert ora.sphere_overlap(0.5, 3.0, 1.0) == (0.0, 0.0)
    assert ora.sphere_overlap(0.0, 2.0, 2.0) == (0.0, 0.0)
    r = 2.0
    v1, v2 = ora.sphere_overlap(r, r, r)
    h = r / 2.0
    assert v1 == pytest.approx(v2) and v1 == pytest.approx((np.pi / 3.0) * h ** 2 * (3.0 * r - h))
    assert 0 < v1 + v2 < 4 * np.pi / 3 * r ** 3
    v1, v2 = ora.sphere_overlap(3.0, 3.0, 1.0)
    assert 0 < v1 < v2


def test_merge_exclusion_kats(ora):
    # test/test_merger.jl:71-112: A (large) kills B (inside), C far away survives
    out, keep = ora.merge_catalog(_halos([[0, 0, 0], [0.3, 0.3, 0.3], [10, 10, 10]], [2.0, 0.5, 1.0]))
    assert keep.tolist() == [True, False, True]
    # equal radii: the earlier halo of the stable order wins
    out, keep = ora.merge_catalog(_halos([[0, 0, 0], [0.5, 0, 0]], [2.0, 2.0]))
    assert keep.tolist() == [True, False]


def test_merge_volume_reduction_kats(ora):
    # test/test_merger.jl:114-151: overlapping equal pair shrinks symmetrically
    out, keep = ora.merge_catalog(_halos([[0, 0, 0], [3, 0, 0]], [2.0, 2.0]))
    assert keep.all() and out[0, 6] < 2.0 and out[0, 6] == out[1, 6]
    h = 2.0 - 1.5   # cap height at d = 3, r = 2
    cap = np.pi / 3 * h * h * (3 * 2.0 - h)
    assert out[0, 6] == pytest.approx(((4 * np.pi / 3 * 8.0 - cap) / (4 * np.pi / 3)) ** (1 / 3), rel=1e-6)
    out, keep = ora.merge_catalog(_halos([[0, 0, 0], [100, 0, 0]], [2.0, 3.0]))
    assert keep.all() and out[0, 6] == pytest.approx(2.0) and out[1, 6] == pytest.approx(3.0)


# ---------------------------------------------------------------------------
# collapse-table generation (RK4 path of make_table)
# ---------------------------------------------------------------------------
def test_elliptic_rd_and_shape_integrals(ora):
    # test/test_ellipsoidalcollapse.jl:8-38: RD(x,x,x) = x^-3/2; b sums to 1;
    # (1,1,1) is spherical
    for x in (1.0, 2.0, 0.5, 10.0):
        assert ora.elliptic_rd(x, x, x) == pytest.approx(x ** -1.5, rel=1e-10)
    assert ora.elliptic_rd(1.0, 2.0, 3.0) > 0
    assert np.allclose(ora.shape_b2(1.0, 1.0, 1.0), 1.0 / 3.0, rtol=1e-10)
    for a in [(0.5, 0.8, 1.2), (0.3, 0.7, 1.5), (0.9, 0.95, 1.0), (1.2, 0.8, 0.5)]:
        assert ora.shape_b2(*a).sum() == pytest.approx(1.0, rel=1e-10)


def test_single_ellipsoids(ora):
    # test/test_ellipsoidalcollapse.jl:71-98 and :183-186 (RK4): overdensities
    # collapse, more overdense earlier, Frho = 0.5 never (-1)
    tp = ora.TableParams(Nx=2, Ny=2, Nz=2, X1=np.log10(3.0), X2=np.log10(5.0), Y1=0.0, Y2=0.3, Z1=0.0, Z2=0.5)
    t = ora.make_table(0.315, 0.049, 0.685, 0.674, tp)
    assert (t > 0).all()                       # (3, 0.3, 0) and (5, 0, 0) collapse
    assert (t[:, :, 1] > t[:, :, 0]).all()     # higher F, earlier (larger 1 + z)
    sph = ora.make_table(0.315, 0.049, 0.685, 0.674, ora.TableParams(Nx=2, Ny=2, Nz=2, X1=np.log10(1.5),
                                                                     X2=np.log10(1.686), Y2=1e-9, Z1=0.0, Z2=0.1))
    assert sph[0, 0, 1] > 0 and sph[0, 0, 1] > sph[0, 0, 0]   # Frho = 1.686 collapses (zvir > 0)
    low = ora.make_table(0.315, 0.049, 0.685, 0.674, ora.TableParams(Nx=2, Ny=2, Nz=2, X1=np.log10(0.4),
                                                                     X2=np.log10(0.5), Y2=0.1, Z1=0.0, Z2=0.1))
    assert (low == -1.0).all()


def test_make_table_reproduces_the_reference_table(ora, julia_table):
    # tests/golden/HomelTab_julia.dat is the reference's make_table output
    # (RK4 path, default CollapseTableParams) for the Websky cosmology of
    # validation/websky_multitile (Om 0.3138, OB 0.0493, OL 0.6862, h 0.6735):
    # the restatement reproduces every one of its 20,000 Float32 nodes
    t = ora.make_table(0.3138, 0.0493, 0.6862, 0.6735)
    assert t.shape == julia_table.data.shape
    assert np.array_equal(t.astype(np.float32), julia_table.data)


def test_rmax2rs_result_does_not_depend_on_peak_order(ora, eh_pk, julia_table):
    """With rmax2rs > 0 the reference analyses peaks under Threads.@threads
    while each collapsed halo writes the mask (RadialShell.jl:793-802) and
    each peak may read it first (:310-316).  That read can only skip a peak
    with floor(Rf/alatt rmax2rs) = 0, whose cell cap npart (:288-295) is then
    at most floor(4/3 pi) = 4 cells: no shell beyond the centre closes, so
    such a peak returns no_collapse at m0 = 1 (:650-653) whether skipped or
    not.  The oracle shows it: peaks in list order on one thread, and in
    reverse order, and on all threads, give the same results bit for bit,
    and every peak the mask could skip has no halo."""
    n, box, nbuff = 48, 96.0, 12
    cfg = ora.Config(Omx=0.315 - 0.049, OmB=0.049, Omvac=0.685, h=0.674, n=n, boxsize=box, nbuff=nbuff,
                     ilpt=2, ioutshear=1, wsmooth=1, rmax2rs=1.0)
    from conftest import filter_bank
    st = ora.run_tile_stages(cfg, 5, *eh_pk, filter_bank(), julia_table, peak_sample=np.arange(0))
    ipp, Rf, ir2, Z = st["peaks"]["ipp"], st["Rf"], st["ir2min"], st["ZZon"]
    alatt = st["alatt"]
    skippable = np.floor(Rf / alatt * 1.0) == 0
    assert skippable.sum() > 10 and (~skippable).sum() > 100
    runs = []
    for order, serial in ((np.arange(len(ipp)), True), (np.arange(len(ipp))[::-1], True),
                          (np.arange(len(ipp)), False)):
        mask = np.zeros((n, n, n), np.int8)
        r = ora.analyse_peaks(st["fields"], ipp[order], Rf[order], ir2[order], Z[order], st["fcrit"], alatt,
                              st["shells"], julia_table, nbuff=nbuff, rmax2rs=1.0, mask=mask, serial_mask=serial)
        out = np.empty_like(r)
        out[order] = r
        runs.append((out, mask))
    for out, mask in runs[1:]:
        assert np.array_equal(out.view(np.uint64), runs[0][0].view(np.uint64))
        assert np.array_equal(mask, runs[0][1])
    assert np.all(runs[0][0][skippable, 0] == -1.0)
    assert (runs[0][0][:, 0] > 0).sum() > 50


def test_truncated_gather_leg_gives_the_full_results(ora, eh_pk, julia_table):
    """The oracle's truncated gather (each peak stops reading cells once the
    shells its later phases read are in: the first shell beyond ir2min, the
    Rf window and an outward fcrit crossing, plus two cells of radius) gives
    the full-sphere results bit for bit.  The same rule truncates the GPU
    gather; the CPU leg times the reference's algorithm with it."""
    from conftest import filter_bank
    for rmax2rs in (0.0, 1.0):
        cfg = ora.Config(Omx=0.315 - 0.049, OmB=0.049, Omvac=0.685, h=0.674, n=64, boxsize=128.0, nbuff=16,
                         ilpt=2, ioutshear=1, wsmooth=1, rmax2rs=rmax2rs)
        st = ora.run_tile_stages(cfg, 3, *eh_pk, filter_bank(), julia_table, peak_sample=np.arange(0))
        args = (st["fields"], st["peaks"]["ipp"], st["Rf"], st["ir2min"], st["ZZon"], st["fcrit"], st["alatt"],
                st["shells"], julia_table)
        full = ora.analyse_peaks(*args, nbuff=16, rmax2rs=rmax2rs)
        trunc = ora.analyse_peaks(*args, nbuff=16, rmax2rs=rmax2rs, truncate=True)
        assert (full[:, 0] > 0).sum() > 100
        assert np.array_equal(full.view(np.uint64), trunc.view(np.uint64)), rmax2rs
