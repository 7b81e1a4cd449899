"""CPU oracle for PeakPatch.jl's per-tile halo-finding path (run_tile).

TEST INFRASTRUCTURE ONLY: the parity tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use this module as the checker.  The product
(``peakpatch.jl_b200``) never imports it.

The arithmetic lives in ``oracle.cpp`` (a double-precision C++ restatement of
the reference's Julia code, built by ``oracle/Makefile`` into
``oracle/_build/libppb_oracle.so``); this module drives it and supplies the
FFTs.  The reference uses FFTW in single precision; here every transform is
done in double precision (scipy.fft / pocketfft, threaded) and rounded to
single precision where the reference holds a Float32 array, so the oracle's
fields are the correctly rounded values of the same transforms.

Reference files restated (PeakPatch.jl):
  src/Pipeline.jl:66-325            run_tile
  src/InitialConditions/*.jl        noise, P(k), 1LPT/2LPT
  src/HaloFinder/*.jl               filters, peak finding, radial shells
  src/EllipsoidalCollapse/CollapseTable.jl:85-145   HomelTab I/O, lookup
  src/Cosmology/Cosmology.jl        growth tables, chi(z)
  src/IO/Catalog.jl:53-160          .pksc
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
import struct
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libppb_oracle.so")
_lib = None

R_N = 31  # doubles per analyse_peak result (layout documented in oracle.cpp)


def build() -> str:
    """Compile the oracle library with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


P = ctypes.c_void_p
I64 = ctypes.c_int64
D = ctypes.c_double


def _declare(L):
    L.ora_num_threads.restype = ctypes.c_int
    L.ora_set_threads.argtypes = [ctypes.c_int]
    L.ora_noise.argtypes = [P, I64, ctypes.c_uint64]
    L.ora_noise_libm.argtypes = [P, I64, ctypes.c_uint64]
    L.ora_noise_region.argtypes = [P, I64, ctypes.c_uint64, I64, I64, I64, I64, I64, I64]
    L.ora_pk.argtypes = [P, P, ctypes.c_int, D]
    L.ora_pk.restype = D
    L.ora_convolve.argtypes = [P, I64, D, P, P, ctypes.c_int]
    for f in ("ora_lpt1", "ora_phi", "ora_lpt2", "ora_lapd_k"):
        getattr(L, f).argtypes = [P, P, I64, D]
    L.ora_src2.argtypes = [P, P, I64]
    L.ora_window.argtypes = [D, D, ctypes.c_int]
    L.ora_window.restype = D
    L.ora_smooth_k.argtypes = [P, P, I64, D, D, ctypes.c_int]
    L.ora_find_peaks.argtypes = [P, P, I64, I64, I64, D, D, D, D, I64, ctypes.c_float, I64,
                                 P, P, P, P, P, P, P, P]
    L.ora_find_peaks.restype = I64
    L.ora_hRinteg.argtypes = [D, D]
    L.ora_hRinteg.restype = D
    L.ora_make_table.argtypes = [D, D, D, D, P, P, P]
    L.ora_mr_coarse_noise.argtypes = [I64, I64, ctypes.c_uint64, P]
    L.ora_mr_residual.argtypes = [P, I64, I64, I64, I64, I64, I64, I64, ctypes.c_uint64, I64, P]
    L.ora_mr_tricubic.argtypes = [P, I64, I64, I64, I64, I64, I64, I64, P]
    L.ora_mr_transfer.argtypes = [P, I64, D, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.ora_mr_apply_kernel.argtypes = [P, I64, D, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.ora_elliptic_rd.argtypes = [D, D, D]
    L.ora_elliptic_rd.restype = D
    L.ora_shape_b2.argtypes = [D, D, D, P]
    L.ora_atab4.argtypes = [P]
    L.ora_shells.argtypes = [ctypes.c_int, P]
    L.ora_shells.restype = I64
    L.ora_eig3.argtypes = [P, P]
    L.ora_table_interp.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, D, D, D, D, D, D, D, D, D]
    L.ora_table_interp.restype = D
    L.ora_dlinear.argtypes = [D, D, D, D, P, ctypes.c_int, P]
    L.ora_fsc_of_z.argtypes = [D, D, D, D, D]
    L.ora_fsc_of_z.restype = D
    L.ora_chi.argtypes = [D, D, D, D]
    L.ora_chi.restype = D
    L.ora_chi2z.argtypes = [D, D, D, D, P, ctypes.c_int, P]
    L.ora_analyse_peaks.argtypes = [P] * 9 + [I64, I64, I64, P, I64, P, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, D, D, D, D, D, D, I64, P, P, P, P, P, D,
                                              I64, D, ctypes.c_int, ctypes.c_int, P]
    L.ora_dump_counts.argtypes = [P]
    L.ora_pack_records.argtypes = [D, D, D, D, I64, P, P, P, P, P, P, P, D, ctypes.c_int, D, D, D, D,
                                   D, ctypes.c_int, ctypes.c_int, P, P]
    L.ora_pack_records.restype = I64
    L.ora_sphere_overlap.argtypes = [D, D, D, P, P]
    L.ora_merge_catalog.argtypes = [P, I64, ctypes.c_int, P, P]
    L.ora_merge_catalog.restype = I64


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def set_threads(n: int) -> None:
    lib().ora_set_threads(int(n))


def num_threads() -> int:
    return int(lib().ora_num_threads())


# --------------------------------------------------------------------------
# File formats (reference readers restated)
# --------------------------------------------------------------------------
def read_pk(path: str):
    """2-column ASCII (k, P); '#' comments.  PowerSpectrum.jl:11-30."""
    d = np.loadtxt(path, comments="#")
    return np.ascontiguousarray(d[:, 0], dtype=np.float64), np.ascontiguousarray(d[:, 1], dtype=np.float64)


def read_filterbank(path: str):
    """Line 1: count; then 'id fcrit Rf'.  Filters.jl:46-58."""
    with open(path) as f:
        lines = f.read().splitlines()
    nic = int(lines[0].strip())
    out = []
    for i in range(nic):
        p = lines[i + 1].split()
        out.append((int(p[0]), float(p[1]), float(p[2])))
    return out


@dataclass
class Table:
    data: np.ndarray  # float32, shape (nz, ny, nx) C-order == column-major (nx, ny, nz)
    nx: int
    ny: int
    nz: int
    x1: float
    x2: float
    y1: float
    y2: float
    z1: float
    z2: float


def read_homeltab(path: str) -> Table:
    """3 x Int32 + 6 x Float32 header, then Float32 column-major data.
    CollapseTable.jl:102-122."""
    with open(path, "rb") as f:
        raw = f.read()
    nx, ny, nz = struct.unpack("<3i", raw[:12])
    x1, x2, y1, y2, z1, z2 = (float(v) for v in struct.unpack("<6f", raw[12:36]))
    data = np.frombuffer(raw[36:36 + 4 * nx * ny * nz], dtype="<f4").reshape(nz, ny, nx).copy()
    return Table(data, nx, ny, nz, x1, x2, y1, y2, z1, z2)


def write_pksc(path: str, rec: np.ndarray, RTHLmax: float, z_out: float) -> None:
    """Int32 N, Float32 RTHLmax, Float32 z_out, then N x (11|33) Float32.
    Catalog.jl:53-94."""
    rec = np.ascontiguousarray(rec, dtype="<f4")
    with open(path, "wb") as f:
        f.write(struct.pack("<i", rec.shape[0]))
        f.write(struct.pack("<f", RTHLmax))
        f.write(struct.pack("<f", z_out))
        f.write(rec.tobytes())


# --------------------------------------------------------------------------
# FFTs (double precision, rounded to single where the reference stores F32)
# --------------------------------------------------------------------------
def _fft_workers() -> int:
    return max(1, num_threads())


def rfft3(x: np.ndarray) -> np.ndarray:
    import scipy.fft as sf
    return sf.rfftn(x.astype(np.float64), workers=_fft_workers()).astype(np.complex64)


def irfft3(c: np.ndarray, n: int) -> np.ndarray:
    import scipy.fft as sf
    return sf.irfftn(c.astype(np.complex128), s=(n, n, n), workers=_fft_workers()).astype(np.float32)


# --------------------------------------------------------------------------
# Step functions (arrays are C-order [k][j][i] == Julia column-major [i,j,k])
# --------------------------------------------------------------------------
def noise(n: int, seed: int) -> np.ndarray:
    out = np.empty((n, n, n), dtype=np.float32)
    lib().ora_noise(_p(out), n, ctypes.c_uint64(seed))
    return out


def noise_libm(n: int, seed: int) -> np.ndarray:
    """Noise with the platform libm in the Box-Muller step (cross-check)."""
    out = np.empty((n, n, n), dtype=np.float32)
    lib().ora_noise_libm(_p(out), n, ctypes.c_uint64(seed))
    return out


def noise_region(n, seed, irange, jrange, krange) -> np.ndarray:
    """Sub-region with 0-based half-open ranges (RandomField.jl:95-109)."""
    (i0, i1), (j0, j1), (k0, k1) = irange, jrange, krange
    out = np.empty((k1 - k0, j1 - j0, i1 - i0), dtype=np.float32)
    lib().ora_noise_region(_p(out), n, ctypes.c_uint64(seed), i0, i1 - i0, j0, j1 - j0, k0, k1 - k0)
    return out


def convolve(noise_arr: np.ndarray, pk_k, pk_p, boxsize: float) -> np.ndarray:
    n = noise_arr.shape[0]
    nk = rfft3(noise_arr)
    lib().ora_convolve(_p(nk), n, boxsize, _p(pk_k), _p(pk_p), len(pk_k))
    return irfft3(nk, n)


def generate_grf(n, pk_k, pk_p, boxsize, seed) -> np.ndarray:
    """RandomField.jl:123-128."""
    return convolve(noise(n, seed), pk_k, pk_p, boxsize)


def lpt1(delta_k, n, boxsize):
    out = np.empty((3,) + delta_k.shape, dtype=np.complex64)
    lib().ora_lpt1(_p(delta_k), _p(out), n, boxsize)
    return [irfft3(out[c], n) for c in range(3)]


def lpt2(delta_k, n, boxsize):
    phik = np.empty((6,) + delta_k.shape, dtype=np.complex64)
    lib().ora_phi(_p(delta_k), _p(phik), n, boxsize)
    phi = np.stack([irfft3(phik[c], n) for c in range(6)])
    src2 = np.empty((n, n, n), dtype=np.float32)
    lib().ora_src2(_p(phi), _p(src2), n ** 3)
    s2k = rfft3(src2)
    out = np.empty((3,) + delta_k.shape, dtype=np.complex64)
    lib().ora_lpt2(_p(s2k), _p(out), n, boxsize)
    return [irfft3(out[c], n) for c in range(3)]


def laplacian(delta_k, n, boxsize):
    """Pipeline.jl:35-51: irfft(k^2 delta_k) / n^3 (Float32 division)."""
    lk = np.empty_like(delta_k)
    lib().ora_lapd_k(_p(delta_k), _p(lk), n, boxsize)
    return (irfft3(lk, n) / np.float32(float(n) ** 3)).astype(np.float32)


def smooth_field(delta_k, n, boxsize, Rf, wsmooth):
    out = np.empty_like(delta_k)
    lib().ora_smooth_k(_p(delta_k), _p(out), n, boxsize, Rf, wsmooth)
    return irfft3(out, n)


def window(kR: float, k: float, wsmooth: int) -> float:
    return float(lib().ora_window(kR, k, wsmooth))


def find_peaks(delta, mask, xbx, ybx, zbx, alatt, nbuff, fcrit, max_peaks=2000000):
    """PeakFind.jl:15-79.  delta: C-order (n3,n2,n1) float32; mask int8
    (mutated).  Returns dict of arrays; i, j, k, ipp are 1-based."""
    n3, n2, n1 = delta.shape
    cap = int(min(max_peaks, delta.size))
    cap = max(cap, 1)
    bufs = {k: np.empty(cap, dtype=np.int64) for k in ("i", "j", "k", "ipp")}
    bufs.update({k: np.empty(cap, dtype=np.float64) for k in ("x", "y", "z")})
    bufs["delta"] = np.empty(cap, dtype=np.float32)
    npk = lib().ora_find_peaks(_p(delta), _p(mask), n1, n2, n3, xbx, ybx, zbx, alatt, nbuff,
                               ctypes.c_float(fcrit), max_peaks, _p(bufs["i"]), _p(bufs["j"]),
                               _p(bufs["k"]), _p(bufs["ipp"]), _p(bufs["x"]), _p(bufs["y"]),
                               _p(bufs["z"]), _p(bufs["delta"]))
    return {k: v[:npk].copy() for k, v in bufs.items()}


def hRinteg(u0, u12):
    return float(lib().ora_hRinteg(u0, u12))


def atab4():
    a = np.empty(1101, dtype=np.float64)
    lib().ora_atab4(_p(a))
    return a


def precompute_shells(rmax: int) -> np.ndarray:
    n = lib().ora_shells(rmax, None)
    out = np.empty((n, 4), dtype=np.int32)
    lib().ora_shells(rmax, _p(out))
    return out


def eigvals_sym(m) -> np.ndarray:
    a = np.ascontiguousarray(m, dtype=np.float64)
    lam = np.empty(3, dtype=np.float64)
    lib().ora_eig3(_p(a), _p(lam))
    return lam


def table_interp(T: Table, x, y, z) -> float:
    return float(lib().ora_table_interp(_p(T.data), T.nx, T.ny, T.nz, T.x1, T.x2, T.y1, T.y2, T.z1,
                                        T.z2, x, y, z))


def dlinear(Om, OB, OL, h, a) -> np.ndarray:
    a = np.ascontiguousarray(np.atleast_1d(a), dtype=np.float64)
    out = np.empty_like(a)
    lib().ora_dlinear(Om, OB, OL, h, _p(a), len(a), _p(out))
    return out


@dataclasses.dataclass
class TableParams:
    """CollapseTableParams (src/EllipsoidalCollapse/CollapseTable.jl:9-23) and
    the EllipsoidParams defaults of the RK4 path (EllipsoidalCollapse.jl:25-38)."""
    Nx: int = 50
    Ny: int = 20
    Nz: int = 20
    X1: float = float(np.log10(1.5))
    X2: float = float(np.log10(8.0))
    Y1: float = 0.0
    Y2: float = 0.5
    Z1: float = -1.0 + 1e-4
    Z2: float = 1.0 - 1e-4
    iforce_strat: int = 4
    ivir_strat: int = 2
    fcoll_1: float = 0.01
    fcoll_2: float = 0.171
    fcoll_3: float = 0.171
    tfac: float = 0.01
    nstepmax: int = 10000
    zinit_fac: float = 20.0


def make_table(Om, OB, OL, h, tp: TableParams = None) -> np.ndarray:
    """make_table(EllipsoidParams(cosmo; solver=:rk4), tp)
    (src/EllipsoidalCollapse/CollapseTable.jl:33-52): the (Nz, Ny, Nx) array
    (C order, i.e. Julia's [i, j, k]) of 1 + z_vir in double precision; the
    reference stores it rounded to Float32."""
    tp = tp or TableParams()
    ip = np.array([tp.Nx, tp.Ny, tp.Nz, tp.iforce_strat, tp.ivir_strat, tp.nstepmax], np.int32)
    dp = np.array([tp.X1, tp.X2, tp.Y1, tp.Y2, tp.Z1, tp.Z2, tp.fcoll_1, tp.fcoll_2, tp.fcoll_3, tp.tfac,
                   tp.zinit_fac], np.float64)
    out = np.empty((tp.Nz, tp.Ny, tp.Nx), np.float64)
    lib().ora_make_table(Om, OB, OL, h, _p(ip), _p(dp), _p(out))
    return out


def elliptic_rd(x, y, z) -> float:
    return float(lib().ora_elliptic_rd(x, y, z))


def shape_b2(a1, a2, a3) -> np.ndarray:
    b = np.zeros(3)
    lib().ora_shape_b2(a1, a2, a3, _p(b))
    return b


def fsc_of_z(Om, OB, OL, h, z) -> float:
    return float(lib().ora_fsc_of_z(Om, OB, OL, h, z))


def chi(Om, OL, h, z) -> float:
    return float(lib().ora_chi(Om, OL, h, z))


def chi_to_z(Om, OL, h, zmax, chis) -> np.ndarray:
    c = np.ascontiguousarray(np.atleast_1d(chis), dtype=np.float64)
    out = np.empty_like(c)
    lib().ora_chi2z(Om, OL, h, zmax, _p(c), len(c), _p(out))
    return out


def analyse_peaks(fields, ipp, Rf, ir2min, ZZon, fcrit, alatt, shells, T: Table, nbuff=0,
                  rmax2rs=0.0, mask=None, serial_mask=False, truncate=False) -> np.ndarray:
    """RadialShell.jl:282-891 for a batch of peaks.  fields: dict with delta,
    etax, etay, etaz and optional eta2x/eta2y/eta2z/lapd (C-order float32).
    truncate: stop each peak's gather once the shells the later phases read
    are in (the same results; a CPU timing leg, not the reference's loop).
    Returns (npk, 31) float64 results."""
    d = fields["delta"]
    n3, n2, n1 = d.shape
    npk = len(ipp)
    arr = lambda a, t: np.ascontiguousarray(np.broadcast_to(np.asarray(a, dtype=t), (npk,)))
    ipp_a, Rf_a, ir_a, Z_a, fc_a = arr(ipp, np.int64), arr(Rf, np.float64), arr(ir2min, np.int64), \
        arr(ZZon, np.float64), arr(fcrit, np.float64)
    out = np.empty((npk, R_N), dtype=np.float64)
    g = lambda k: fields.get(k)
    sh = np.ascontiguousarray(shells, dtype=np.int32)
    lib().ora_analyse_peaks(_p(d), _p(g("etax")), _p(g("etay")), _p(g("etaz")), _p(g("eta2x")),
                            _p(g("eta2y")), _p(g("eta2z")), _p(g("lapd")), _p(mask), n1, n2, n3,
                            _p(sh), sh.shape[0], _p(T.data), T.nx, T.ny, T.nz, T.x1, T.x2, T.y1, T.y2,
                            T.z1, T.z2, npk, _p(ipp_a), _p(Rf_a), _p(ir_a), _p(Z_a), _p(fc_a), alatt,
                            nbuff, rmax2rs, int(bool(serial_mask)), int(bool(truncate)), _p(out))
    return out


def dump_counts():
    a = np.zeros(5, dtype=np.int64)
    lib().ora_dump_counts(_p(a))
    return dict(zip(("premask", "no_fcrit", "m0_one", "no_collapse", "rthl_neg"), a.tolist()))


# --------------------------------------------------------------------------
# run_tile (Pipeline.jl:66-325)
# --------------------------------------------------------------------------
@dataclass
class Config:
    """PipelineConfig fields used on the path (src/IO/Parameters.jl:17-46)."""
    Omx: float = 0.266
    OmB: float = 0.049
    Omvac: float = 0.685
    h: float = 0.674
    n: int = 142
    boxsize: float = 200.0
    nbuff: int = 4
    z_out: float = 0.0
    z_max: float = 0.0
    ievol: int = 0
    cenx: float = 0.0
    ceny: float = 0.0
    cenz: float = 0.0
    ilpt: int = 2
    ioutshear: int = 0
    wsmooth: int = 0
    rmax2rs: float = 1.0


def run_tile_stages(cfg: Config, seed: int, pk_k, pk_p, filters, T: Table, peak_sample=None,
                    timings: dict | None = None):
    """Runs run_tile and returns all intermediate products (fields, peaks,
    per-peak results, records).  `peak_sample` (optional index array) limits
    the shell analysis to a subset of peaks (CPU-baseline sampling)."""
    import time
    tm = timings if timings is not None else {}
    t0 = time.perf_counter()
    Om = cfg.Omx + cfg.OmB
    filters = sorted(filters, key=lambda f: -f[2])
    n, box = cfg.n, cfg.boxsize
    alatt = box / n
    fcrit_val = fsc_of_z(Om, cfg.OmB, cfg.Omvac, cfg.h, cfg.z_out)
    Rfmax = filters[0][2]
    nhunt = min(cfg.nbuff - 1, int(np.floor(Rfmax * 1.75 / alatt)))
    shells = precompute_shells(nhunt)
    delta = generate_grf(n, pk_k, pk_p, box, seed)
    fcrit = np.float32(fcrit_val)
    delta_k = rfft3(delta)
    psi = lpt1(delta_k, n, box)
    psi2 = lpt2(delta_k, n, box) if cfg.ilpt >= 2 else [None, None, None]
    t1 = time.perf_counter()
    tm["fields_s"] = t1 - t0
    mask = np.zeros((n, n, n), dtype=np.int8)
    peaks = {k: [] for k in ("i", "j", "k", "ipp", "x", "y", "z", "delta")}
    pRf, pFc, pd2 = [], [], []
    for (_, _, Rf) in filters:
        ds = smooth_field(delta_k, n, box, Rf, cfg.wsmooth)
        ls = smooth_field(delta_k, n, box, Rf, 3) if cfg.ioutshear >= 1 else None
        pk = find_peaks(ds, mask, 0.0, 0.0, 0.0, alatt, cfg.nbuff, fcrit)
        for k in peaks:
            peaks[k].append(pk[k])
        npk = len(pk["ipp"])
        pRf.append(np.full(npk, Rf))
        lin = pk["ipp"] - 1
        pFc.append(ds.reshape(-1)[lin])
        pd2.append(ls.reshape(-1)[lin] if ls is not None else np.zeros(npk, np.float32))
    peaks = {k: np.concatenate(v) for k, v in peaks.items()}
    pRf, pFc, pd2 = np.concatenate(pRf), np.concatenate(pFc).astype(np.float32), \
        np.concatenate(pd2).astype(np.float32)
    t2 = time.perf_counter()
    tm["peaks_s"] = t2 - t1
    mask[:] = 0
    lapd = laplacian(delta_k, n, box) if cfg.ioutshear >= 1 else None
    fields = dict(delta=delta, etax=psi[0], etay=psi[1], etaz=psi[2], eta2x=psi2[0], eta2y=psi2[1],
                  eta2z=psi2[2], lapd=lapd)
    npk = len(peaks["ipp"])
    ir2min = np.minimum(np.floor((1.75 * pRf / alatt) ** 2), np.floor((40.0 / alatt - 1) ** 2)).astype(np.int64)
    # per-peak ZZon
    if cfg.ievol == 1:
        dx = peaks["x"] - cfg.cenx
        dy = peaks["y"] - cfg.ceny
        dz = peaks["z"] - cfg.cenz
        zpk = chi_to_z(Om, cfg.Omvac, cfg.h, cfg.z_max + 1.0, np.sqrt(dx * dx + dy * dy + dz * dz))
        ZZon = 1.0 + zpk
        fc_pp = np.array([fsc_of_z(Om, cfg.OmB, cfg.Omvac, cfg.h, z - 1.0) for z in ZZon])
    else:
        ZZon = np.full(npk, 1.0 + cfg.z_out)
        fc_pp = np.full(npk, fcrit_val)
    # analyse_peak computes fcrit from ZZon via fsc_of_z (growth tables given)
    sel = np.arange(npk) if peak_sample is None else np.asarray(peak_sample)
    res = np.zeros((npk, R_N))
    res[:, 0] = -1.0
    res[sel] = analyse_peaks(fields, peaks["ipp"][sel], pRf[sel], ir2min[sel], ZZon[sel], fc_pp[sel],
                             alatt, shells, T, nbuff=cfg.nbuff, rmax2rs=cfg.rmax2rs, mask=mask)
    t3 = time.perf_counter()
    tm["shells_s"] = t3 - t2
    tm["n_analysed"] = int(len(sel))
    st = dict(fields=fields, delta_k=delta_k, peaks=peaks, Rf=pRf, FcollvRf=pFc, d2FRf=pd2,
              ir2min=ir2min, ZZon=ZZon, fcrit=fcrit_val, results=res, shells=shells, nhunt=nhunt, alatt=alatt)
    st["records"] = pack_records(cfg, st, res)
    tm["total_s"] = time.perf_counter() - t0
    return st


def pack_records(cfg: Config, st: dict, res: np.ndarray) -> np.ndarray:
    """Record packing of run_tile (Pipeline.jl:243-308) for the peaks of a
    run_tile_stages result and per-peak analyse_peak results `res`: RTHL > 0
    (and z <= z_max on the lightcone), 11 or 33 Float32 fields, peak order."""
    peaks = st["peaks"]
    npk = len(peaks["ipp"])
    Om = cfg.Omx + cfg.OmB
    nf = 33 if cfg.ioutshear >= 1 else 11
    rec = np.empty((max(npk, 1), nf), dtype=np.float32)
    zz = np.empty(max(npk, 1))
    res = np.ascontiguousarray(res, dtype=np.float64)
    nh = lib().ora_pack_records(Om, cfg.OmB, cfg.Omvac, cfg.h, npk, _p(peaks["x"]), _p(peaks["y"]),
                                _p(peaks["z"]), _p(np.ascontiguousarray(st["Rf"])), _p(st["FcollvRf"]),
                                _p(st["d2FRf"]), _p(res), st["alatt"], cfg.ievol, cfg.z_out, cfg.z_max, cfg.cenx,
                                cfg.ceny, cfg.cenz, cfg.ioutshear, cfg.ilpt, _p(rec), _p(zz))
    return rec[:nh].copy()


def sphere_overlap(d: float, r1: float, r2: float):
    """sphere_overlap (src/Merger/Exclusion.jl:82-100) -> (v1, v2)."""
    v1, v2 = np.zeros(1), np.zeros(1)
    lib().ora_sphere_overlap(float(d), float(r1), float(r2), _p(v1), _p(v2))
    return float(v1[0]), float(v2[0])


def merge_catalog(rec: np.ndarray):
    """merge_catalog (src/Merger/Merger.jl:21-78): returns (survivors with the
    reduced RTHL, keep mask over the input)."""
    rec = np.ascontiguousarray(rec, np.float32)
    n, nf = rec.shape
    out = np.empty_like(rec)
    keep = np.zeros(n, np.int32)
    m = lib().ora_merge_catalog(_p(rec), n, nf, _p(out), _p(keep))
    return out[:m].copy(), keep.astype(bool)


def tile_center(it: int, jt: int, kt: int, ntile: int, dcore: float):
    """tile_center (src/MultiTile.jl:79-86)."""
    cen = (ntile + 1) / 2
    return ((it - cen) * dcore, (jt - cen) * dcore, (kt - cen) * dcore)


def run_multitile(cfg: Config, seed: int, pk_k, pk_p, filters, T: Table, ntile: int, tiles=None):
    """run_multitile (src/MultiTile.jl:108-418): fields on the full periodic
    grid N = nsub ntile + 2 nbuff, the filter bank smoothed globally and the
    peaks found per tile core, the shell analysis per tile on the extracted
    n^3 fields; records in tile order.  `tiles` optionally lists (it, jt, kt)
    (1-based) to process, else every tile in the reference's loop order."""
    Om = cfg.Omx + cfg.OmB
    filters = sorted(filters, key=lambda f: -f[2])
    nm, nbuff = cfg.n, cfg.nbuff
    nsub = nm - 2 * nbuff
    N = nsub * ntile + 2 * nbuff
    alatt = cfg.boxsize / nm
    box = N * alatt
    dcore = nsub * alatt
    fcrit_val = fsc_of_z(Om, cfg.OmB, cfg.Omvac, cfg.h, cfg.z_out)
    nhunt = min(nbuff - 1, int(np.floor(filters[0][2] * 1.75 / alatt)))
    shells = precompute_shells(nhunt)
    delta = generate_grf(N, pk_k, pk_p, box, seed)
    delta_k = rfft3(delta)
    psi = lpt1(delta_k, N, box)
    psi2 = lpt2(delta_k, N, box) if cfg.ilpt >= 2 else [None, None, None]
    lapd = laplacian(delta_k, N, box) if cfg.ioutshear >= 1 else None
    if tiles is None:
        tiles = [(it, jt, kt) for kt in range(1, ntile + 1) for jt in range(1, ntile + 1)
                 for it in range(1, ntile + 1)]
    obs = (cfg.cenx, cfg.ceny, cfg.cenz)
    if cfg.ievol == 1:   # drop tiles beyond chi(z_max) (MultiTile.jl:205-216)
        chi_max = chi(Om, cfg.Omvac, cfg.h, cfg.z_max)
        half = dcore / 2.0
        keep = []
        for t in tiles:
            c = tile_center(*t, ntile, dcore)
            d = [max(abs(c[q] - obs[q]) - half, 0.0) for q in range(3)]
            if np.sqrt(d[0] ** 2 + d[1] ** 2 + d[2] ** 2) <= chi_max:
                keep.append(t)
        tiles = keep
    sl = lambda a, t: a[(t[2] - 1) * nsub:(t[2] - 1) * nsub + nm, (t[1] - 1) * nsub:(t[1] - 1) * nsub + nm,
                        (t[0] - 1) * nsub:(t[0] - 1) * nsub + nm]
    fcrit_t = []
    for t in tiles:
        fc = np.float32(fcrit_val)
        if cfg.ievol == 1:   # fcrit of the tile centre's redshift (MultiTile.jl:238-243)
            c = tile_center(*t, ntile, dcore)
            zt = chi_to_z(Om, cfg.Omvac, cfg.h, cfg.z_max + 1.0,
                          np.array([np.sqrt(sum((c[q] - obs[q]) ** 2 for q in range(3)))]))[0]
            fc = np.float32(fsc_of_z(Om, cfg.OmB, cfg.Omvac, cfg.h, zt))
        fcrit_t.append(fc)
    masks = [np.zeros((nm, nm, nm), np.int8) for _ in tiles]
    tp = [dict(peaks=[], Rf=[], Fc=[], d2=[]) for _ in tiles]
    for (_, _, Rf) in filters:
        ds = smooth_field(delta_k, N, box, Rf, cfg.wsmooth)
        ls = smooth_field(delta_k, N, box, Rf, 3) if cfg.ioutshear >= 1 else None
        for ti, t in enumerate(tiles):
            dst = np.ascontiguousarray(sl(ds, t))
            c = tile_center(*t, ntile, dcore)
            pk = find_peaks(dst, masks[ti], c[0], c[1], c[2], alatt, nbuff, fcrit_t[ti])
            lin = pk["ipp"] - 1
            tp[ti]["peaks"].append(pk)
            tp[ti]["Rf"].append(np.full(len(lin), Rf))
            tp[ti]["Fc"].append(dst.reshape(-1)[lin])
            tp[ti]["d2"].append(np.ascontiguousarray(sl(ls, t)).reshape(-1)[lin] if ls is not None
                                else np.zeros(len(lin), np.float32))
    recs, npk_tot = [], 0
    L = lib()
    for ti, t in enumerate(tiles):
        peaks = {k: np.concatenate([p[k] for p in tp[ti]["peaks"]]) for k in tp[ti]["peaks"][0]}
        pRf = np.concatenate(tp[ti]["Rf"])
        pFc = np.concatenate(tp[ti]["Fc"]).astype(np.float32)
        pd2 = np.concatenate(tp[ti]["d2"]).astype(np.float32)
        npk = len(peaks["ipp"])
        npk_tot += npk
        if npk == 0:
            continue
        fields = dict(delta=np.ascontiguousarray(sl(delta, t)),
                      etax=np.ascontiguousarray(sl(psi[0], t)), etay=np.ascontiguousarray(sl(psi[1], t)),
                      etaz=np.ascontiguousarray(sl(psi[2], t)),
                      eta2x=None if psi2[0] is None else np.ascontiguousarray(sl(psi2[0], t)),
                      eta2y=None if psi2[1] is None else np.ascontiguousarray(sl(psi2[1], t)),
                      eta2z=None if psi2[2] is None else np.ascontiguousarray(sl(psi2[2], t)),
                      lapd=None if lapd is None else np.ascontiguousarray(sl(lapd, t)))
        ir2min = np.minimum(np.floor((1.75 * pRf / alatt) ** 2), np.floor((40.0 / alatt - 1) ** 2)).astype(np.int64)
        if cfg.ievol == 1:
            dx, dy, dz = peaks["x"] - obs[0], peaks["y"] - obs[1], peaks["z"] - obs[2]
            ZZon = 1.0 + chi_to_z(Om, cfg.Omvac, cfg.h, cfg.z_max + 1.0, np.sqrt(dx * dx + dy * dy + dz * dz))
            fc_pp = np.array([fsc_of_z(Om, cfg.OmB, cfg.Omvac, cfg.h, z - 1.0) for z in ZZon])
        else:
            ZZon = np.full(npk, 1.0 + cfg.z_out)
            fc_pp = np.full(npk, fcrit_val)
        res = analyse_peaks(fields, peaks["ipp"], pRf, ir2min, ZZon, fc_pp, alatt, shells, T, nbuff=nbuff,
                            rmax2rs=cfg.rmax2rs)
        nf = 33 if cfg.ioutshear >= 1 else 11
        rec = np.empty((npk, nf), dtype=np.float32)
        zz = np.empty(npk)
        nh = L.ora_pack_records(Om, cfg.OmB, cfg.Omvac, cfg.h, npk, _p(peaks["x"]), _p(peaks["y"]),
                                _p(peaks["z"]), _p(np.ascontiguousarray(pRf)), _p(pFc), _p(pd2), _p(res),
                                alatt, cfg.ievol, cfg.z_out, cfg.z_max, cfg.cenx, cfg.ceny, cfg.cenz,
                                cfg.ioutshear, cfg.ilpt, _p(rec), _p(zz))
        recs.append(rec[:nh])
    nf = 33 if cfg.ioutshear >= 1 else 11
    out = np.concatenate(recs) if recs else np.empty((0, nf), np.float32)
    return out, npk_tot


def run_tile(cfg: Config, seed: int, pk_k, pk_p, filters, T: Table) -> np.ndarray:
    return run_tile_stages(cfg, seed, pk_k, pk_p, filters, T)["records"]


# --------------------------------------------------------------------------
# Multi-resolution (MUSIC-style) per-tile building blocks
# (src/MultiResolution.jl).  Arrays C-order [k][j][i] (Julia [i, j, k]); tile
# numbers (it, jt, kt) 1-based as the reference.
# Kernel kinds: 0 delta, 1 1LPT (i k_d1 / k^2), 2 2LPT (-i k_d1 / k^2),
# 3 phi_ij (-k_d1 k_d2 / k^2), 4 Laplacian (k^2).
# --------------------------------------------------------------------------
def mr_coarse_noise(N: int, M: int, seed: int) -> np.ndarray:
    """_downsample_noise (:68-89): block means of the global Threefry noise,
    summed in double, scaled to unit variance."""
    out = np.empty((M, M, M), np.float32)
    lib().ora_mr_coarse_noise(N, M, seed, _p(out))
    return out


def mr_residual(coarse, M, it, jt, kt, nsub, nmesh, N, seed, nshell=0) -> np.ndarray:
    """_generate_extended_residual (:197-236): fine noise minus its coarse
    cell's block mean on the tile's (nmesh + 2 nshell)^3 region."""
    c = np.ascontiguousarray(coarse, np.float32)
    ne = nmesh + 2 * nshell
    out = np.empty((ne, ne, ne), np.float32)
    lib().ora_mr_residual(_p(c), M, it, jt, kt, nsub, nmesh, N, seed, nshell, _p(out))
    return out


def mr_tricubic(coarse, M, it, jt, kt, nsub, nmesh, N) -> np.ndarray:
    """_interpolate_to_tile (:95-122): Catmull-Rom tricubic interpolation of
    the periodic coarse grid at the tile's fine cells."""
    c = np.ascontiguousarray(coarse, np.float32)
    out = np.empty((nmesh, nmesh, nmesh), np.float32)
    lib().ora_mr_tricubic(_p(c), M, it, jt, kt, nsub, nmesh, N, _p(out))
    return out


def isolated_convolve(noise, pk_k, pk_p, boxsize_local, n, kind=0, d1=0, d2=0, nshell=0) -> np.ndarray:
    """_isolated_convolve (:246-283): zero-pad to twice the input size, rfft,
    multiply by sqrt(P(k) dk^3 n2^3) and the kernel, irfft, keep the n^3 tile
    region (offset nshell)."""
    noise = np.ascontiguousarray(noise, np.float32)
    ni = noise.shape[0]
    n2 = 2 * ni
    padded = np.zeros((n2, n2, n2), np.float32)
    padded[:ni, :ni, :ni] = noise
    pk = np.ascontiguousarray(rfft3(padded))
    kk = np.ascontiguousarray(pk_k, np.float64)
    pp = np.ascontiguousarray(pk_p, np.float64)
    dx = float(boxsize_local) / n
    lib().ora_mr_transfer(_p(pk), n2, n2 * dx, _p(kk), _p(pp), len(kk), kind, d1, d2)
    res = irfft3(pk, n2)
    return np.ascontiguousarray(res[nshell:nshell + n, nshell:nshell + n, nshell:nshell + n])


def mr_apply_kernel(arr_k, n, boxsize, kind, d1=0, d2=0) -> np.ndarray:
    a = np.ascontiguousarray(arr_k, np.complex64).copy()
    lib().ora_mr_apply_kernel(_p(a), n, float(boxsize), kind, d1, d2)
    return a


def tile_2lpt_laplacian(delta_tile, n, boxsize, ilpt=2, want_lap=True):
    """The tile-local 2LPT and Laplacian of run_multitile_split
    (src/MultiResolution.jl:804-847): src2 = delta^2/2 - sum_d phi_dd^2/2 -
    sum_{i<j} phi_ij^2, psi2_d = irfft(-i k_d/k^2 src2_k), lapd =
    irfft(k^2 delta_k), with the kernel applied by _apply_kernel_inplace!.
    Returns (psi2 (3, n, n, n) or None, lapd or None)."""
    d = np.ascontiguousarray(delta_tile, np.float32)
    dk = rfft3(d)
    psi2 = None
    if ilpt >= 2:
        h = np.float32(0.5)
        src2 = np.zeros_like(d)
        src2 = src2 + (d * d) * h
        for a in (1, 2, 3):
            r = irfft3(mr_apply_kernel(dk, n, boxsize, 3, a, a), n)
            src2 = src2 - (r * r) * h
        for a, b in ((1, 2), (1, 3), (2, 3)):
            r = irfft3(mr_apply_kernel(dk, n, boxsize, 3, a, b), n)
            src2 = src2 - r * r
        s2k = rfft3(src2)
        psi2 = np.stack([irfft3(mr_apply_kernel(s2k, n, boxsize, 2, a), n) for a in (1, 2, 3)])
    lap = irfft3(mr_apply_kernel(dk, n, boxsize, 4), n) if want_lap else None
    return psi2, lap


def periodic_convolve(arr_k, pk_k, pk_p, n, boxsize, kind=0, d1=0, d2=0) -> np.ndarray:
    """_periodic_convolve! (:286-309) on a copy of the rfft arr_k of a
    periodic n^3 box of side boxsize."""
    a = np.ascontiguousarray(arr_k, np.complex64).copy()
    kk = np.ascontiguousarray(pk_k, np.float64)
    pp = np.ascontiguousarray(pk_p, np.float64)
    lib().ora_mr_transfer(_p(a), n, float(boxsize), _p(kk), _p(pp), len(kk), kind, d1, d2)
    return a


def coarse_fields(coarse_noise, pk_k, pk_p, boxsize_full, ilpt=2, ioutshear=1):
    """Phase 1a of run_multitile_split (:617-667) on the M^3 coarse noise:
    delta_coarse, psi_coarse (3, M, M, M), psi2_coarse (ilpt >= 2, the
    reference's P(k)-weighted 2LPT multiplier) and lapd_coarse (ioutshear >=
    1), each an irfft of a _periodic_convolve! of the coarse rfft."""
    c = np.ascontiguousarray(coarse_noise, np.float32)
    M = c.shape[0]
    ck = rfft3(c)
    pc = lambda a, kind, d1=0, d2=0: irfft3(periodic_convolve(a, pk_k, pk_p, M, boxsize_full, kind, d1, d2), M)
    delta = pc(ck, 0)
    psi = np.stack([pc(ck, 1, a) for a in (1, 2, 3)])
    psi2 = None
    if ilpt >= 2:
        h = np.float32(0.5)
        src2 = np.zeros_like(c)
        src2 = src2 + (delta * delta) * h
        for a in (1, 2, 3):
            r = pc(ck, 3, a, a)
            src2 = src2 - (r * r) * h
        for a, b in ((1, 2), (1, 3), (2, 3)):
            r = pc(ck, 3, a, b)
            src2 = src2 - r * r
        s2k = rfft3(src2)
        psi2 = np.stack([pc(s2k, 2, a) for a in (1, 2, 3)])
    lap = pc(ck, 4) if ioutshear >= 1 else None
    return delta, psi, psi2, lap


def _correlation(a, b):
    da = a - a.sum() / a.size
    db = b - b.sum() / b.size
    return float((da * db).sum() / np.sqrt((da ** 2).sum() * (db ** 2).sum()))


def _rms_frac(a, b):
    ra = np.sqrt((a ** 2).sum() / a.size)
    return float(np.sqrt(((a - b) ** 2).sum() / a.size) / ra) if ra > 0 else 0.0


def compare_fields_split(pk_k, pk_p, N, boxsize, seed, ntile, coarse_factor, nbuff=8, coarse_grid=0):
    """compare_fields_split (src/MultiResolution.jl:1266-1353): per tile, the
    split delta and psi_x (isolated convolution of the residual plus the
    tricubic coarse field) against the global-FFT fields on the tile core.
    Returns [(tile, corr_delta, rms_delta, corr_psi1, rms_psi1)]."""
    nsub = (N - 2 * nbuff) // ntile
    nmesh = nsub + 2 * nbuff
    assert nsub * ntile + 2 * nbuff == N
    M = coarse_grid if coarse_grid > 0 else ntile * coarse_factor
    assert N % M == 0
    alatt = boxsize / N
    dg = generate_grf(N, pk_k, pk_p, boxsize, seed)
    psig = lpt1(rfft3(dg), N, boxsize)[0]
    cn = mr_coarse_noise(N, M, seed)
    ck = rfft3(cn)
    dc = irfft3(periodic_convolve(ck, pk_k, pk_p, M, boxsize, 0), M)
    pc = irfft3(periodic_convolve(ck, pk_k, pk_p, M, boxsize, 1, 1), M)
    box_tile = nmesh * alatt
    out = []
    for kt in range(1, ntile + 1):
        for jt in range(1, ntile + 1):
            for it in range(1, ntile + 1):
                sl = lambda t: slice((t - 1) * nsub, t * nsub)
                core = slice(nbuff, nbuff + nsub)
                ref_d = dg[sl(kt), sl(jt), sl(it)].astype(np.float64)
                ref_p = psig[sl(kt), sl(jt), sl(it)].astype(np.float64)
                res = mr_residual(cn, M, it, jt, kt, nsub, nmesh, N, seed, 0)
                d = isolated_convolve(res, pk_k, pk_p, box_tile, nmesh, 0) + mr_tricubic(dc, M, it, jt, kt, nsub,
                                                                                          nmesh, N)
                p = isolated_convolve(res, pk_k, pk_p, box_tile, nmesh, 1, 1) + mr_tricubic(pc, M, it, jt, kt, nsub,
                                                                                             nmesh, N)
                d = d[core, core, core].astype(np.float64)
                p = p[core, core, core].astype(np.float64)
                out.append(((it, jt, kt), _correlation(ref_d, d), _rms_frac(ref_d, d), _correlation(ref_p, p),
                            _rms_frac(ref_p, p)))
    return out


def split_coarse_grid(N, nmesh, ntile, coarse_factor=0, coarse_grid=0) -> int:
    """The coarse grid M of run_multitile_split (src/MultiResolution.jl:592-612)."""
    if coarse_grid > 0:
        return coarse_grid
    if coarse_factor > 0:
        return ntile * coarse_factor
    target, best, best_dist = nmesh // 3, 0, N
    for m in range(2, N // 2 + 1):
        if N % m == 0 and abs(N // m - target) < best_dist:
            best, best_dist = m, abs(N // m - target)
    return best


def run_multitile_split(cfg: Config, seed: int, pk_k, pk_p, filters, T: Table, ntile: int, coarse_factor=0,
                        coarse_grid=0, tiles=None):
    """run_multitile_split (src/MultiResolution.jl:523-1236): coarse delta and
    psi on M^3, per tile the split fields (isolated convolution of the
    residual + tricubic coarse field, tile 2LPT and Laplacian), the filter
    bank and peaks on the tile's grid with the tile centre's position (and
    fcrit of its redshift on the lightcone), shells and records; records in
    tile order.  Returns (records, total peaks)."""
    Om = cfg.Omx + cfg.OmB
    filters = sorted(filters, key=lambda f: -f[2])
    nm, nbuff = cfg.n, cfg.nbuff
    nsub = nm - 2 * nbuff
    N = nsub * ntile + 2 * nbuff
    alatt = cfg.boxsize / nm
    box_full, box_local, dcore = N * alatt, nm * alatt, nsub * alatt
    M = split_coarse_grid(N, nm, ntile, coarse_factor, coarse_grid)
    assert M > 0 and N % M == 0
    fcrit_val = fsc_of_z(Om, cfg.OmB, cfg.Omvac, cfg.h, cfg.z_out)
    nhunt = min(nbuff - 1, int(np.floor(filters[0][2] * 1.75 / alatt)))
    shells = precompute_shells(nhunt)
    cn = mr_coarse_noise(N, M, seed)
    ck = rfft3(cn)
    dc = irfft3(periodic_convolve(ck, pk_k, pk_p, M, box_full, 0), M)
    pc = [irfft3(periodic_convolve(ck, pk_k, pk_p, M, box_full, 1, a), M) for a in (1, 2, 3)]
    if tiles is None:
        tiles = [(it, jt, kt) for kt in range(1, ntile + 1) for jt in range(1, ntile + 1)
                 for it in range(1, ntile + 1)]
    obs = (cfg.cenx, cfg.ceny, cfg.cenz)
    if cfg.ievol == 1:   # drop tiles beyond chi(z_max) (:680-692)
        chi_max = chi(Om, cfg.Omvac, cfg.h, cfg.z_max)
        keep = []
        for t in tiles:
            c = tile_center(*t, ntile, dcore)
            d = [max(abs(c[q] - obs[q]) - dcore / 2.0, 0.0) for q in range(3)]
            if np.sqrt(d[0] ** 2 + d[1] ** 2 + d[2] ** 2) <= chi_max:
                keep.append(t)
        tiles = keep
    nf = 33 if cfg.ioutshear >= 1 else 11
    recs, npk_tot = [], 0
    L = lib()
    for t in tiles:
        it, jt, kt = t
        c = tile_center(*t, ntile, dcore)
        fc_t = np.float32(fcrit_val)
        if cfg.ievol == 1:   # fcrit at the tile centre's redshift (:864-871)
            zt = chi_to_z(Om, cfg.Omvac, cfg.h, cfg.z_max + 1.0,
                          np.array([np.sqrt(sum((c[q] - obs[q]) ** 2 for q in range(3)))]))[0]
            fc_t = np.float32(fsc_of_z(Om, cfg.OmB, cfg.Omvac, cfg.h, zt))
        res = mr_residual(cn, M, it, jt, kt, nsub, nm, N, seed, 0)
        d = isolated_convolve(res, pk_k, pk_p, box_local, nm, 0) + mr_tricubic(dc, M, it, jt, kt, nsub, nm, N)
        psi = [isolated_convolve(res, pk_k, pk_p, box_local, nm, 1, a) + mr_tricubic(pc[a - 1], M, it, jt, kt, nsub,
                                                                                      nm, N) for a in (1, 2, 3)]
        psi2, lap = tile_2lpt_laplacian(d, nm, box_local, cfg.ilpt, cfg.ioutshear >= 1)
        dk = rfft3(d)
        mask = np.zeros((nm, nm, nm), np.int8)
        plist, pRf, pFc, pd2 = [], [], [], []
        for (_, _, Rf) in filters:
            ds = smooth_field(dk, nm, box_local, Rf, cfg.wsmooth)
            ls = smooth_field(dk, nm, box_local, Rf, 3) if cfg.ioutshear >= 1 else None
            pk = find_peaks(ds, mask, c[0], c[1], c[2], alatt, nbuff, fc_t)
            lin = pk["ipp"] - 1
            plist.append(pk)
            pRf.append(np.full(len(lin), Rf))
            pFc.append(ds.reshape(-1)[lin])
            pd2.append(ls.reshape(-1)[lin] if ls is not None else np.zeros(len(lin), np.float32))
        peaks = {k: np.concatenate([p[k] for p in plist]) for k in plist[0]}
        pRf = np.concatenate(pRf)
        pFc = np.concatenate(pFc).astype(np.float32)
        pd2 = np.concatenate(pd2).astype(np.float32)
        npk = len(peaks["ipp"])
        npk_tot += npk
        if npk == 0:
            continue
        fields = dict(delta=d, etax=psi[0], etay=psi[1], etaz=psi[2],
                      eta2x=None if psi2 is None else psi2[0], eta2y=None if psi2 is None else psi2[1],
                      eta2z=None if psi2 is None else psi2[2], lapd=lap)
        ir2min = np.minimum(np.floor((1.75 * pRf / alatt) ** 2), np.floor((40.0 / alatt - 1) ** 2)).astype(np.int64)
        if cfg.ievol == 1:
            dx, dy, dz = peaks["x"] - obs[0], peaks["y"] - obs[1], peaks["z"] - obs[2]
            ZZon = 1.0 + chi_to_z(Om, cfg.Omvac, cfg.h, cfg.z_max + 1.0, np.sqrt(dx * dx + dy * dy + dz * dz))
            fc_pp = np.array([fsc_of_z(Om, cfg.OmB, cfg.Omvac, cfg.h, z - 1.0) for z in ZZon])
        else:
            ZZon = np.full(npk, 1.0 + cfg.z_out)
            fc_pp = np.full(npk, fcrit_val)
        r = analyse_peaks(fields, peaks["ipp"], pRf, ir2min, ZZon, fc_pp, alatt, shells, T, nbuff=nbuff,
                          rmax2rs=cfg.rmax2rs)
        rec = np.empty((npk, nf), dtype=np.float32)
        zz = np.empty(npk)
        nh = L.ora_pack_records(Om, cfg.OmB, cfg.Omvac, cfg.h, npk, _p(peaks["x"]), _p(peaks["y"]),
                                _p(peaks["z"]), _p(np.ascontiguousarray(pRf)), _p(pFc), _p(pd2), _p(r),
                                alatt, cfg.ievol, cfg.z_out, cfg.z_max, cfg.cenx, cfg.ceny, cfg.cenz,
                                cfg.ioutshear, cfg.ilpt, _p(rec), _p(zz))
        recs.append(rec[:nh])
    out = np.concatenate(recs) if recs else np.empty((0, nf), np.float32)
    return out, npk_tot
