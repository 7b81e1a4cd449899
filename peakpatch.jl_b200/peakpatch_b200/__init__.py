"""peakpatch_b200 — Python host mirror of PeakPatch.jl's per-tile halo-finding
API over the C-ABI library libppb.so (sm_100a CUDA).

Names, argument meanings and error behaviour follow the reference
(PeakPatch.jl):

  PipelineConfig            src/IO/Parameters.jl:17-125 (kwdef + TOML)
  run_tile(cfg; seed)       src/Pipeline.jl:66-325
  fill_noise_threefry!      src/InitialConditions/RandomField.jl:70-83
  find_peaks                src/HaloFinder/PeakFind.jl:15-79
  analyse_peak (batched)    src/HaloFinder/RadialShell.jl:282-891
  read_homeltab             src/EllipsoidalCollapse/CollapseTable.jl:102-122
  read_filterbank           src/HaloFinder/Filters.jl:46-58
  load_pk (table part)      src/InitialConditions/PowerSpectrum.jl:11-30
  write_pksc / read_pksc    src/IO/Catalog.jl:53-160

Arrays are numpy arrays in C order with shape (n3, n2, n1), which is the
memory layout of Julia's column-major Array{Float32,3} of size (n1, n2, n3);
peak indices i, j, k, ipp are 1-based as in the reference.  All compute runs
in libppb.so on a CUDA device; there is no CPU fallback: without the library
or a GPU the calls raise.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
import struct
from dataclasses import dataclass, field, fields, replace
from typing import Optional, Sequence

import numpy as np

__all__ = [
    "PipelineConfig", "Context", "run_tile", "fill_noise_threefry", "find_peaks", "analyse_peaks",
    "read_homeltab", "read_filterbank", "read_pk_table", "write_pksc", "read_pksc", "PPBError",
    "library_path", "load_library", "EXT_FIELDS", "BASIC_FIELDS", "RESULT_FIELDS",
]

_PKG = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(os.path.dirname(_PKG), "libppb.so")

BASIC_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "RTHL", "vx2", "vy2", "vz2", "overdensity")
EXT_FIELDS = BASIC_FIELDS + (
    "e_v", "p_v", "strain_11", "strain_22", "strain_33", "strain_23", "strain_13", "strain_12",
    "d2F", "zform", "grad_x", "grad_y", "grad_z", "gradf_x", "gradf_y", "gradf_z", "Rf",
    "FcollvRf", "d2FRf", "gradrf_x", "gradrf_y", "gradrf_z")
# per-peak analyse_peak output layout (31 doubles), see include/ppb.h
RESULT_FIELDS = {"RTHL": 0, "Srb": 1, "Sbar": slice(2, 5), "Sbar2": slice(5, 8), "strain": slice(8, 17),
                 "gradpk": slice(17, 20), "gradpkrf": slice(20, 23), "Fbarx": 23, "e_v": 24, "p_v": 25,
                 "zvir_half": 26, "gradpkf": slice(27, 30), "d2F": 30}

PPB_OK = 0
_ERRNAMES = {-1: "INVALID", -2: "CUDA", -3: "NOMEM", -4: "ADMISSION", -5: "TIMEOUT", -6: "UNSUPPORTED",
             -7: "CAPACITY", -8: "NOT_FOUND"}


class PPBError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libppb error {code} ({_ERRNAMES.get(code, '?')}): {msg}")
        self.code = code


# --------------------------------------------------------------------------
# library loading
# --------------------------------------------------------------------------
class _TileParams(ctypes.Structure):
    _fields_ = [("Omx", ctypes.c_double), ("OmB", ctypes.c_double), ("Omvac", ctypes.c_double),
                ("h", ctypes.c_double), ("n", ctypes.c_int32), ("boxsize", ctypes.c_double),
                ("nbuff", ctypes.c_int32), ("z_out", ctypes.c_double), ("z_max", ctypes.c_double),
                ("ievol", ctypes.c_int32), ("cenx", ctypes.c_double), ("ceny", ctypes.c_double),
                ("cenz", ctypes.c_double), ("ilpt", ctypes.c_int32), ("ioutshear", ctypes.c_int32),
                ("wsmooth", ctypes.c_int32), ("rmax2rs", ctypes.c_double), ("seed", ctypes.c_uint64),
                ("plain", ctypes.c_int32), ("reserved0", ctypes.c_int32), ("pk_scale", ctypes.c_double),
                ("reserved", ctypes.c_int32 * 4)]


class _Stats(ctypes.Structure):
    _fields_ = [("tiles_done", ctypes.c_int64), ("peaks_done", ctypes.c_int64), ("halos_done", ctypes.c_int64),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("tiles_per_s", ctypes.c_double),
                ("hbm_in_use", ctypes.c_uint64), ("hbm_budget", ctypes.c_uint64), ("in_flight", ctypes.c_int32),
                ("queued", ctypes.c_int32), ("slots", ctypes.c_int32), ("failed", ctypes.c_int32)]


class _TuneEntry(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("nshell", ctypes.c_int32), ("comp", ctypes.c_int32),
                ("adaptive", ctypes.c_int32), ("limited", ctypes.c_int32), ("brick_shift", ctypes.c_int32),
                ("collapse_threads", ctypes.c_int32), ("long_walk", ctypes.c_int32), ("npk", ctypes.c_int64),
                ("gather_ms", ctypes.c_float * 5), ("collapse_ms", ctypes.c_float * 4),
                ("collapse_order", ctypes.c_int32), ("collapse_ordered_ms", ctypes.c_float * 4),
                ("gather_tex", ctypes.c_int32), ("gather_plain_ms", ctypes.c_float)]


# context options (include/ppb.h)
OPT_GRAPHS, OPT_AUTOTUNE, OPT_TUNE_MIN_PEAKS, OPT_BRICK_SHIFT, OPT_COLLAPSE_THREADS = 1, 2, 3, 4, 5
OPT_FUSED_X = 6
OPT_GATHER_RING = 7
OPT_COLLAPSE_ORDER = 8
OPT_GATHER_TEX = 10
OPT_GRAPH_LAUNCHES, OPT_GRAPH_INSTANTIATIONS, OPT_GRAPH_UPDATES = 16, 17, 18


class _TableParams(ctypes.Structure):
    _fields_ = [("Om", ctypes.c_double), ("OB", ctypes.c_double), ("OL", ctypes.c_double), ("h", ctypes.c_double),
                ("Nx", ctypes.c_int32), ("Ny", ctypes.c_int32), ("Nz", ctypes.c_int32),
                ("iforce_strat", ctypes.c_int32), ("ivir_strat", ctypes.c_int32), ("nstepmax", ctypes.c_int32),
                ("X1", ctypes.c_double), ("X2", ctypes.c_double), ("Y1", ctypes.c_double), ("Y2", ctypes.c_double),
                ("Z1", ctypes.c_double), ("Z2", ctypes.c_double), ("fcoll_1", ctypes.c_double),
                ("fcoll_2", ctypes.c_double), ("fcoll_3", ctypes.c_double), ("tfac", ctypes.c_double),
                ("zinit_fac", ctypes.c_double), ("reserved", ctypes.c_int32 * 4)]


@dataclasses.dataclass
class CollapseTableParams:
    """CollapseTableParams (src/EllipsoidalCollapse/CollapseTable.jl:9-23)
    with the EllipsoidParams settings of the RK4 path
    (src/EllipsoidalCollapse/EllipsoidalCollapse.jl:25-38), defaults as there."""
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


class _HaloBuf(ctypes.Structure):
    _fields_ = [("records", ctypes.c_void_p), ("capacity", ctypes.c_int64), ("count", ctypes.c_int64),
                ("nfields", ctypes.c_int32), ("RTHLmax", ctypes.c_float), ("npeaks", ctypes.c_int64)]


_lib = None

# every function include/ppb.h declares (checked by the CPU test suite)
EXPORTED = (
    "ppb_ctx_create", "ppb_ctx_destroy", "ppb_last_error", "ppb_abi_version", "ppb_set_collapse_table",
    "ppb_set_pk_table", "ppb_run_tile", "ppb_run_tile_timed", "ppb_write_pksc", "ppb_noise_threefry",
    "ppb_find_peaks", "ppb_analyse_peaks", "ppb_event_record", "ppb_event_elapsed", "ppb_synchronize",
    "ppb_launch_count", "ppb_last_shell_stats", "ppb_last_stage_ms", "ppb_alloc_host", "ppb_free_host",
    "ppb_alloc_device", "ppb_free_device", "ppb_shell_counters", "ppb_find_peaks_noalloc",
    "ppb_last_shell_times", "ppb_serve_config", "ppb_submit", "ppb_wait", "ppb_stats_get", "ppb_stats_reset",
    "ppb_run_multitile", "ppb_merge_catalog", "ppb_set_collapse_table_f64", "ppb_generate_fields",
    "ppb_analyse_peaks_lim", "ppb_set_option", "ppb_get_option", "ppb_tune_entries", "ppb_make_collapse_table",
    "ppb_last_table_stats", "ppb_downsample_noise", "ppb_extended_residual", "ppb_isolated_convolve",
    "ppb_interpolate_to_tile", "ppb_compute_2lpt", "ppb_compute_laplacian", "ppb_coarse_fields",
    "ppb_run_multitile_split", "ppb_split_coarse_grid", "ppb_peak_find_tile", "ppb_analyse_peaks_multirf", "ppb_write_catalog_hdf5",
)


def library_path() -> str:
    return os.environ.get("PPB_LIBRARY", _LIB_PATH)


def load_library():
    """Load libppb.so (raises when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise PPBError(-1, f"{path} not found: build it with `python peakpatch.jl_b200/build.py`")
    L = ctypes.CDLL(path)
    P, I32, I64, D = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    L.ppb_ctx_create.argtypes = [I32, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]
    L.ppb_ctx_destroy.argtypes = [P]
    L.ppb_last_error.argtypes = [P, ctypes.c_char_p, ctypes.c_size_t]
    L.ppb_set_collapse_table.argtypes = [P, P, I32, I32, I32, D, D, D, D, D, D]
    L.ppb_set_pk_table.argtypes = [P, P, P, I32]
    L.ppb_run_tile.argtypes = [P, ctypes.POINTER(_TileParams), P, I32, ctypes.POINTER(_HaloBuf)]
    L.ppb_run_tile_timed.argtypes = [P, ctypes.POINTER(_TileParams), P, I32, ctypes.POINTER(_HaloBuf),
                                     ctypes.POINTER(ctypes.c_float)]
    L.ppb_write_pksc.argtypes = [ctypes.c_char_p, P, I64, I32, ctypes.c_float, ctypes.c_float]
    L.ppb_noise_threefry.argtypes = [P, P, I32, ctypes.c_uint64]
    L.ppb_find_peaks.argtypes = [P, P, P, I32, I32, I32, I32, ctypes.c_float, I64, P, P, P, P, P,
                                 ctypes.POINTER(ctypes.c_int64)]
    L.ppb_find_peaks_noalloc.argtypes = L.ppb_find_peaks.argtypes
    L.ppb_analyse_peaks.argtypes = [P] * 9 + [I32, I32, I64, P, P, P, P, P, D, I32, P]
    L.ppb_event_record.argtypes = [P, I32]
    L.ppb_event_elapsed.argtypes = [P, I32, I32, ctypes.POINTER(ctypes.c_float)]
    L.ppb_synchronize.argtypes = [P]
    L.ppb_launch_count.argtypes = [P, ctypes.POINTER(ctypes.c_int64)]
    L.ppb_last_shell_stats.argtypes = [P, ctypes.POINTER(ctypes.c_int64), P, ctypes.POINTER(ctypes.c_float)]
    L.ppb_last_stage_ms.argtypes = [P, P]
    L.ppb_shell_counters.argtypes = [P, P]
    L.ppb_last_shell_times.argtypes = [P, P, P, P]
    L.ppb_serve_config.argtypes = [P, I32]
    L.ppb_submit.argtypes = [P, ctypes.POINTER(_TileParams), P, I32, ctypes.POINTER(ctypes.c_uint64)]
    L.ppb_wait.argtypes = [P, ctypes.c_uint64, I32, ctypes.POINTER(_HaloBuf)]
    L.ppb_stats_get.argtypes = [P, ctypes.POINTER(_Stats)]
    L.ppb_stats_reset.argtypes = [P]
    L.ppb_run_multitile.argtypes = [P, ctypes.POINTER(_TileParams), P, I32, I32, P, I32, ctypes.POINTER(_HaloBuf)]
    L.ppb_merge_catalog.argtypes = [P, P, I64, I32, P, ctypes.POINTER(ctypes.c_int64)]
    L.ppb_set_collapse_table_f64.argtypes = [P, P, I32, I32, I32, D, D, D, D, D, D]
    L.ppb_generate_fields.argtypes = [P, ctypes.POINTER(_TileParams), P, P, P, P]
    L.ppb_analyse_peaks_lim.argtypes = [P] * 9 + [I32, I32, I64, P, P, P, P, P, P, D, I32, P]
    L.ppb_make_collapse_table.argtypes = [P, ctypes.POINTER(_TableParams), P, I32]
    L.ppb_last_table_stats.argtypes = [P, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int64)]
    L.ppb_set_option.argtypes = [P, I32, I64]
    L.ppb_get_option.argtypes = [P, I32, ctypes.POINTER(ctypes.c_int64)]
    L.ppb_tune_entries.argtypes = [P, ctypes.POINTER(_TuneEntry), I32, ctypes.POINTER(ctypes.c_int32)]
    U64 = ctypes.c_uint64
    L.ppb_downsample_noise.argtypes = [P, I64, I32, U64, P]
    L.ppb_extended_residual.argtypes = [P, P, I32, I32, I32, I32, I32, I32, I64, U64, I32, P]
    L.ppb_isolated_convolve.argtypes = [P, P, I32, D, I32, P, I32, I32, P]
    L.ppb_interpolate_to_tile.argtypes = [P, P, I32, I32, I32, I32, I32, I64, I32, P]
    L.ppb_compute_2lpt.argtypes = [P, P, I32, D, P]
    L.ppb_compute_laplacian.argtypes = [P, P, I32, D, P]
    L.ppb_coarse_fields.argtypes = [P, P, I32, D, I32, I32, P, P, P, P]
    L.ppb_run_multitile_split.argtypes = [P, ctypes.POINTER(_TileParams), P, I32, I32, I32, I32, P, I32,
                                          ctypes.POINTER(_HaloBuf)]
    L.ppb_split_coarse_grid.argtypes = [I32, I32, I32, I32, I32]
    L.ppb_write_catalog_hdf5.argtypes = [ctypes.c_char_p, P, I64, I32, D, D, D, D]
    L.ppb_analyse_peaks_multirf.argtypes = [P] * 9 + [I32, I32, I32, P, P, P, P, P, P, P, P, D, D, D, P, I32, D, I32,
                                                       P]
    L.ppb_peak_find_tile.argtypes = [P, P, I32, P, P, I32, P, D, D, D, D, I32, I32, I32, I64] + [P] * 11 + \
        [ctypes.POINTER(ctypes.c_int64)]
    for f in ("ppb_alloc_host", "ppb_alloc_device"):
        getattr(L, f).argtypes = [P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p)]
    for f in ("ppb_free_host", "ppb_free_device"):
        getattr(L, f).argtypes = [P, P]
    _lib = L
    return L


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


# --------------------------------------------------------------------------
# PipelineConfig (src/IO/Parameters.jl:17-125)
# --------------------------------------------------------------------------
@dataclass
class PipelineConfig:
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
    NonGauss: int = 0
    fNL: float = 0.0
    pkfile: str = "pk.dat"
    filterfile: str = "filters.dat"
    tabfile: str = "HomelTab.dat"
    fileout: str = "catalog.pksc"

    @classmethod
    def from_toml(cls, config: dict) -> "PipelineConfig":
        """PipelineConfig(config::Dict) of Parameters.jl:88-125."""
        cosmo, grid, run, files = (config.get(k, {}) for k in ("cosmology", "grid", "run", "files"))
        Om_total = float(cosmo.get("Om", 0.315))
        OmB = float(cosmo.get("OB", 0.049))
        z_out = float(run.get("z_out", 0.0))
        return cls(Omx=Om_total - OmB, OmB=OmB, Omvac=float(cosmo.get("OL", 0.685)), h=float(cosmo.get("h", 0.674)),
                   n=int(grid.get("n", 142)), boxsize=float(grid.get("boxsize", grid.get("dL_box", 200.0))),
                   nbuff=int(grid.get("nbuff", 4)), z_out=z_out, z_max=float(run.get("z_max", z_out)),
                   ievol=int(run.get("ievol", 0)), cenx=float(grid.get("cenx", 0.0)),
                   ceny=float(grid.get("ceny", 0.0)), cenz=float(grid.get("cenz", 0.0)),
                   ilpt=int(run.get("ilpt", 2)), ioutshear=int(run.get("ioutshear", 0)),
                   wsmooth=int(run.get("wsmooth", 0)), rmax2rs=float(run.get("rmax2rs", 1.0)),
                   NonGauss=int(run.get("NonGauss", 0)), fNL=float(run.get("fNL", 0.0)),
                   pkfile=files.get("pk", "pk.dat"), filterfile=files.get("filterbank", "filters.dat"),
                   tabfile=files.get("homeltab", "HomelTab.dat"), fileout=files.get("output", "catalog.pksc"))

    @classmethod
    def from_toml_file(cls, path: str) -> "PipelineConfig":
        import tomllib
        with open(path, "rb") as f:
            return cls.from_toml(tomllib.load(f))


# --------------------------------------------------------------------------
# file formats
# --------------------------------------------------------------------------
@dataclass
class CollapseTable:
    data: np.ndarray          # float32 (Nz, Ny, Nx) C order == column-major (Nx, Ny, Nz)
    X1: float
    X2: float
    Y1: float
    Y2: float
    Z1: float
    Z2: float

    @property
    def shape_xyz(self):
        nz, ny, nx = self.data.shape
        return nx, ny, nz


def read_homeltab(path: str) -> CollapseTable:
    """36-byte header (3 Int32, 6 Float32) + Float32 column-major table."""
    with open(path, "rb") as f:
        raw = f.read()
    nx, ny, nz = struct.unpack("<3i", raw[:12])
    x1, x2, y1, y2, z1, z2 = (float(v) for v in struct.unpack("<6f", raw[12:36]))
    need = 36 + 4 * nx * ny * nz
    if len(raw) < need:
        raise ValueError(f"{path}: truncated collapse table ({len(raw)} < {need} bytes)")
    data = np.frombuffer(raw[36:need], dtype="<f4").reshape(nz, ny, nx).copy()
    return CollapseTable(data, x1, x2, y1, y2, z1, z2)


def write_homeltab(path: str, t: CollapseTable) -> None:
    nx, ny, nz = t.shape_xyz
    with open(path, "wb") as f:
        f.write(struct.pack("<3i", nx, ny, nz))
        f.write(struct.pack("<6f", t.X1, t.X2, t.Y1, t.Y2, t.Z1, t.Z2))
        f.write(np.ascontiguousarray(t.data, dtype="<f4").tobytes())


def read_filterbank(path: str):
    """Returns [(id, fcrit, Rf), ...] in file order."""
    with open(path) as f:
        lines = f.read().splitlines()
    nic = int(lines[0].strip())
    out = []
    for i in range(nic):
        p = lines[i + 1].split()
        out.append((int(p[0]), float(p[1]), float(p[2])))
    return out


def write_filterbank(path: str, Rfs: Sequence[float], fcrit: float = 1.686) -> None:
    with open(path, "w") as f:
        f.write(f"{len(Rfs)}\n")
        for i, R in enumerate(Rfs):
            f.write(f"{i + 1}  {fcrit}  {R!r}\n")


def read_pk_table(path: str):
    d = np.loadtxt(path, comments="#")
    return np.ascontiguousarray(d[:, 0], np.float64), np.ascontiguousarray(d[:, 1], np.float64)


def write_pksc(path: str, records: np.ndarray, RTHLmax: float, z_out: float) -> None:
    rec = np.ascontiguousarray(records, dtype="<f4")
    with open(path, "wb") as f:
        f.write(struct.pack("<i", rec.shape[0]))
        f.write(struct.pack("<f", RTHLmax))
        f.write(struct.pack("<f", z_out))
        f.write(rec.tobytes())


def read_pksc(path: str):
    """Returns (records (N, 11|33) float32, RTHLmax, z_out); the field count
    is inferred from the file size as Catalog.jl:100-120 does."""
    with open(path, "rb") as f:
        raw = f.read()
    nh = struct.unpack("<i", raw[:4])[0]
    rthl, zo = struct.unpack("<2f", raw[4:12])
    nf = (len(raw) - 12) // (nh * 4) if nh > 0 else 11
    rec = np.frombuffer(raw[12:12 + 4 * nh * nf], dtype="<f4").reshape(nh, nf).copy()
    return rec, rthl, zo


# --------------------------------------------------------------------------
# context
# --------------------------------------------------------------------------
class Context:
    """One libppb context on one CUDA device (tables stay resident)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self.L = load_library()
        h = ctypes.c_void_p()
        rc = self.L.ppb_ctx_create(device, hbm_budget, ctypes.byref(h))
        if rc != PPB_OK:
            raise PPBError(rc, "ppb_ctx_create failed (is a CUDA device visible?)")
        self.h = h
        self._table_key = None
        self._pk_key = None

    def close(self):
        if getattr(self, "h", None):
            self.L.ppb_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int):
        if rc != PPB_OK:
            buf = ctypes.create_string_buffer(1024)
            self.L.ppb_last_error(self.h, buf, 1024)
            raise PPBError(rc, buf.value.decode(errors="replace"))

    # tables
    def set_collapse_table(self, t: CollapseTable):
        key = (id(t.data), t.data.shape)
        if key == self._table_key:
            return
        d = np.ascontiguousarray(t.data, dtype=np.float32)
        nz, ny, nx = d.shape
        self._check(self.L.ppb_set_collapse_table(self.h, _p(d), nx, ny, nz, t.X1, t.X2, t.Y1, t.Y2, t.Z1, t.Z2))
        self._table_key = key

    def set_pk_table(self, k: np.ndarray, pk: np.ndarray):
        k = np.ascontiguousarray(k, np.float64)
        pk = np.ascontiguousarray(pk, np.float64)
        self._check(self.L.ppb_set_pk_table(self.h, _p(k), _p(pk), len(k)))

    def launch_count(self) -> int:
        c = ctypes.c_int64()
        self._check(self.L.ppb_launch_count(self.h, ctypes.byref(c)))
        return c.value

    def shell_stats(self):
        v = ctypes.c_int64()
        d = np.zeros(5, np.int64)
        ms = ctypes.c_float()
        self._check(self.L.ppb_last_shell_stats(self.h, ctypes.byref(v), _p(d), ctypes.byref(ms)))
        raw = np.zeros(16, np.int64)
        self._check(self.L.ppb_shell_counters(self.h, _p(raw)))
        kms = np.zeros(4, np.float32)
        rows = ctypes.c_int64()
        nb = ctypes.c_int32()
        self._check(self.L.ppb_last_shell_times(self.h, _p(kms), ctypes.byref(rows), ctypes.byref(nb)))
        return {"visits": v.value, "dumps": dict(zip(("premask", "no_fcrit", "m0_one", "no_collapse", "rthl_neg"),
                                                      d.tolist())), "ms": ms.value, "guard": int(raw[6]),
                "akk_overrun": int(raw[7]), "bad_peaks": int(raw[8]), "walk_steps": int(raw[9]),
                "kernel_ms": dict(zip(("gather", "collapse", "zvir_half", "d2f"), kms.tolist())),
                "pool_rows": rows.value, "batches": nb.value}

    # ---- collapse-table generation ----
    def make_table(self, Om: float, OB: float, OL: float, h: float, tp: "CollapseTableParams" = None,
                   install: int = 0) -> np.ndarray:
        """make_table(EllipsoidParams(cosmo; solver=:rk4), tp) on the GPU
        (src/EllipsoidalCollapse/CollapseTable.jl:33-52): the (Nz, Ny, Nx)
        array (Julia's [i, j, k]) of 1 + z_vir in double precision (the
        reference rounds it to Float32).  Om is the total matter density.
        install = 1 makes it the context's collapse table with Float32 nodes,
        2 with Float64 nodes."""
        tp = tp or CollapseTableParams()
        p = _TableParams(Om=Om, OB=OB, OL=OL, h=h, Nx=tp.Nx, Ny=tp.Ny, Nz=tp.Nz, iforce_strat=tp.iforce_strat,
                         ivir_strat=tp.ivir_strat, nstepmax=tp.nstepmax, X1=tp.X1, X2=tp.X2, Y1=tp.Y1, Y2=tp.Y2,
                         Z1=tp.Z1, Z2=tp.Z2, fcoll_1=tp.fcoll_1, fcoll_2=tp.fcoll_2, fcoll_3=tp.fcoll_3,
                         tfac=tp.tfac, zinit_fac=tp.zinit_fac)
        out = np.empty((tp.Nz, tp.Ny, tp.Nx), np.float64)
        self._check(self.L.ppb_make_collapse_table(self.h, ctypes.byref(p), _p(out), int(install)))
        if install:
            self._table_key = None
        return out

    def table_stats(self):
        ms = ctypes.c_float()
        st = ctypes.c_int64()
        self._check(self.L.ppb_last_table_stats(self.h, ctypes.byref(ms), ctypes.byref(st)))
        return {"ms": ms.value, "rk4_steps": st.value}

    # ---- launch options and the autotuner ----
    def set_option(self, option: int, value: int):
        self._check(self.L.ppb_set_option(self.h, option, int(value)))

    def get_option(self, option: int) -> int:
        v = ctypes.c_int64()
        self._check(self.L.ppb_get_option(self.h, option, ctypes.byref(v)))
        return v.value

    def graph_stats(self):
        return {"launches": self.get_option(OPT_GRAPH_LAUNCHES),
                "instantiations": self.get_option(OPT_GRAPH_INSTANTIATIONS),
                "updates": self.get_option(OPT_GRAPH_UPDATES)}

    def tune_entries(self):
        """The autotuned shell-stage configurations: one dict per kind of batch
        with the chosen gather-order brick (cells on a side, 0 = list order),
        the collapse width and every candidate's time."""
        n = ctypes.c_int32()
        self._check(self.L.ppb_tune_entries(self.h, None, 0, ctypes.byref(n)))
        buf = (_TuneEntry * max(1, n.value))()
        self._check(self.L.ppb_tune_entries(self.h, buf, n.value, ctypes.byref(n)))
        out = []
        for e in buf[:n.value]:
            out.append({"n": e.n, "nshell": e.nshell, "comp": bool(e.comp), "adaptive": bool(e.adaptive),
                        "limited": bool(e.limited), "long_walk": bool(e.long_walk),
                        "brick": (1 << e.brick_shift) if e.brick_shift >= 0 else 0,
                        "collapse_threads": e.collapse_threads, "npk": e.npk,
                        "gather_ms": dict(zip(("brick4", "brick8", "brick16", "brick32", "list"),
                                              [round(x, 4) for x in e.gather_ms])),
                        "collapse_ms": dict(zip(("w1", "w2", "w4", "queue"), [round(x, 4) for x in e.collapse_ms])),
                        "collapse_order": bool(e.collapse_order),
                        "collapse_ordered_ms": dict(zip(("w1", "w2", "w4", "queue"),
                                                        [round(x, 4) for x in e.collapse_ordered_ms])),
                        "gather_tex": bool(e.gather_tex), "gather_plain_ms": round(e.gather_plain_ms, 4)})
        return out

    def stage_ms(self):
        a = np.zeros(4, np.float32)
        self._check(self.L.ppb_last_stage_ms(self.h, _p(a)))
        return dict(zip(("fields", "peaks", "shells", "records"), a.tolist()))

    def event_record(self, slot: int):
        self._check(self.L.ppb_event_record(self.h, slot))

    def event_elapsed(self, a: int, b: int) -> float:
        ms = ctypes.c_float()
        self._check(self.L.ppb_event_elapsed(self.h, a, b, ctypes.byref(ms)))
        return ms.value

    def synchronize(self):
        self._check(self.L.ppb_synchronize(self.h))

    # ---- memory helpers ----
    def alloc_host(self, nbytes: int) -> int:
        p = ctypes.c_void_p()
        self._check(self.L.ppb_alloc_host(self.h, nbytes, ctypes.byref(p)))
        return p.value

    def free_host(self, ptr: int):
        self._check(self.L.ppb_free_host(self.h, ctypes.c_void_p(ptr)))

    def alloc_device(self, nbytes: int) -> int:
        p = ctypes.c_void_p()
        self._check(self.L.ppb_alloc_device(self.h, nbytes, ctypes.byref(p)))
        return p.value

    def free_device(self, ptr: int):
        self._check(self.L.ppb_free_device(self.h, ctypes.c_void_p(ptr)))

    @staticmethod
    def _params(cfg: PipelineConfig, seed: int, plain: bool, pk_scale: float = 1.0) -> _TileParams:
        if cfg.NonGauss not in (0,):
            raise PPBError(-6, "NonGauss modes are outside this path")
        return _TileParams(Omx=cfg.Omx, OmB=cfg.OmB, Omvac=cfg.Omvac, h=cfg.h, n=cfg.n, boxsize=cfg.boxsize,
                           nbuff=cfg.nbuff, z_out=cfg.z_out, z_max=cfg.z_max, ievol=cfg.ievol, cenx=cfg.cenx,
                           ceny=cfg.ceny, cenz=cfg.cenz, ilpt=cfg.ilpt, ioutshear=cfg.ioutshear,
                           wsmooth=cfg.wsmooth, rmax2rs=cfg.rmax2rs, seed=int(seed) & (2**64 - 1),
                           plain=1 if plain else 0, pk_scale=float(pk_scale))

    def run_tile_into(self, cfg: PipelineConfig, seed: int, Rf: Sequence[float], ptr: int, capacity: int,
                      plain: bool = False):
        """run_tile writing records to a caller pointer (pinned host or
        device memory).  Returns (count, RTHLmax, npeaks, device_ms)."""
        p = self._params(cfg, seed, plain)
        rf = np.ascontiguousarray(np.asarray(Rf, dtype=np.float64))
        hb = _HaloBuf(records=ptr, capacity=capacity)
        ms = ctypes.c_float()
        self._check(self.L.ppb_run_tile_timed(self.h, ctypes.byref(p), _p(rf), len(rf), ctypes.byref(hb),
                                              ctypes.byref(ms)))
        return int(hb.count), float(hb.RTHLmax), int(hb.npeaks), ms.value

    # ---- path entry points ----
    def run_tile_arrays(self, cfg: PipelineConfig, seed: int, Rf: Sequence[float], plain: bool = False,
                        capacity: int = 0, timed: bool = False, pk_scale: float = 1.0):
        """run_tile with the tables already set.  Returns (records, RTHLmax,
        npeaks[, device_ms])."""
        p = self._params(cfg, seed, plain, pk_scale)
        rf = np.ascontiguousarray(np.asarray(Rf, dtype=np.float64))
        nf = 33 if cfg.ioutshear >= 1 else 11
        cap = capacity or max(1024, getattr(self, "_last_count", 0) * 2)
        for _ in range(2):
            rec = np.empty((cap, nf), dtype=np.float32)
            hb = _HaloBuf(records=rec.ctypes.data, capacity=cap)
            ms = ctypes.c_float()
            rc = self.L.ppb_run_tile_timed(self.h, ctypes.byref(p), _p(rf), len(rf), ctypes.byref(hb),
                                           ctypes.byref(ms))
            if rc == -7:   # capacity: the tile ran; enlarge and rerun
                cap = int(hb.count) + 16
                continue
            self._check(rc)
            self._last_count = int(hb.count)
            out = (rec[:hb.count].copy(), float(hb.RTHLmax), int(hb.npeaks))
            return out + (ms.value,) if timed else out
        raise PPBError(-7, "record capacity")

    def run_multitile_arrays(self, cfg: PipelineConfig, seed: int, Rf: Sequence[float], ntile: int,
                             tiles=None, plain: bool = False, pk_scale: float = 1.0):
        """run_multitile(cfg; ntile, seed) with the tables set.  tiles: optional
        list of (it, jt, kt), 1-based.  Returns (records, RTHLmax, npeaks)."""
        p = self._params(cfg, seed, plain, pk_scale)
        rf = np.ascontiguousarray(np.asarray(Rf, dtype=np.float64))
        tl = None if tiles is None else np.ascontiguousarray(np.asarray(tiles, dtype=np.int32).reshape(-1, 3))
        nt = 0 if tl is None else len(tl)
        nf = 33 if cfg.ioutshear >= 1 else 11
        # about one halo per 60 core cells (384^3 tiles); grown and rerun when short
        ncore = (cfg.n - 2 * cfg.nbuff) ** 3 * (ntile ** 3 if tl is None else nt)
        cap = max(1024, getattr(self, "_last_count", 0) * 2, ncore // 40)
        for _ in range(2):
            rec = np.empty((cap, nf), dtype=np.float32)
            hb = _HaloBuf(records=rec.ctypes.data, capacity=cap)
            rc = self.L.ppb_run_multitile(self.h, ctypes.byref(p), _p(rf), len(rf), int(ntile),
                                          None if tl is None else _p(tl), nt, ctypes.byref(hb))
            if rc == -7:
                cap = int(hb.count) + 16
                continue
            self._check(rc)
            self._last_count = int(hb.count)
            return rec[:hb.count].copy(), float(hb.RTHLmax), int(hb.npeaks)
        raise PPBError(-7, "record capacity")

    def run_multitile_split_arrays(self, cfg: PipelineConfig, seed: int, Rf: Sequence[float], ntile: int,
                                   coarse_factor: int = 0, coarse_grid: int = 0, tiles=None):
        """run_multitile_split(cfg; ntile, seed, coarse_factor, coarse_grid)
        with the tables set (src/MultiResolution.jl:523-1236).  tiles:
        optional list of (it, jt, kt), 1-based.  Returns (records, RTHLmax,
        npeaks), records in tile order."""
        p = self._params(cfg, seed, False)
        rf = np.ascontiguousarray(np.asarray(Rf, dtype=np.float64))
        tl = None if tiles is None else np.ascontiguousarray(np.asarray(tiles, dtype=np.int32).reshape(-1, 3))
        nt = 0 if tl is None else len(tl)
        nf = 33 if cfg.ioutshear >= 1 else 11
        ncore = (cfg.n - 2 * cfg.nbuff) ** 3 * (ntile ** 3 if tl is None else nt)
        cap = max(1024, getattr(self, "_last_count", 0) * 2, ncore // 30)
        for _ in range(2):
            rec = np.empty((cap, nf), dtype=np.float32)
            hb = _HaloBuf(records=rec.ctypes.data, capacity=cap)
            rc = self.L.ppb_run_multitile_split(self.h, ctypes.byref(p), _p(rf), len(rf), int(ntile),
                                                int(coarse_factor), int(coarse_grid), None if tl is None else _p(tl),
                                                nt, ctypes.byref(hb))
            if rc == -7:
                cap = int(hb.count) + 16
                continue
            self._check(rc)
            self._last_count = int(hb.count)
            return rec[:hb.count].copy(), float(hb.RTHLmax), int(hb.npeaks)
        raise PPBError(-7, "record capacity")

    def merge_catalog(self, records: np.ndarray) -> np.ndarray:
        """merge_catalog(halos): exclusion and volume reduction; returns the
        surviving records (input order) with the reduced RTHL."""
        rec = np.ascontiguousarray(records, dtype=np.float32)
        n, nf = rec.shape if rec.ndim == 2 else (0, 33)
        out = np.empty((max(n, 1), nf), dtype=np.float32)
        m = ctypes.c_int64()
        self._check(self.L.ppb_merge_catalog(self.h, _p(rec) if n else None, n, nf, _p(out), ctypes.byref(m)))
        return out[:m.value].copy()

    # ---- serving ----
    def serve_config(self, slots: int):
        """Number of execution slots of the serving loop (before the first submit)."""
        self._check(self.L.ppb_serve_config(self.h, int(slots)))

    def submit(self, cfg: PipelineConfig, seed: int, Rf: Sequence[float], pk_scale: float = 1.0,
               plain: bool = False) -> int:
        """Queue a tile request; returns its ticket."""
        p = self._params(cfg, seed, plain, pk_scale)
        rf = np.ascontiguousarray(np.asarray(Rf, dtype=np.float64))
        t = ctypes.c_uint64()
        self._check(self.L.ppb_submit(self.h, ctypes.byref(p), _p(rf), len(rf), ctypes.byref(t)))
        return int(t.value)

    def wait(self, ticket: int, timeout_ms: int = -1):
        """Result of a submitted request: (records, RTHLmax, npeaks), or None
        when timeout_ms ran out first."""
        hb = _HaloBuf(records=None, capacity=0)
        rc = self.L.ppb_wait(self.h, ctypes.c_uint64(ticket), int(timeout_ms), ctypes.byref(hb))
        if rc == -5:
            return None
        if rc == -7 or (rc == 0 and hb.count == 0):
            nf = int(hb.nfields) or 33
            rec = np.empty((max(int(hb.count), 1), nf), dtype=np.float32)
            if rc == -7:
                hb2 = _HaloBuf(records=rec.ctypes.data, capacity=rec.shape[0])
                self._check(self.L.ppb_wait(self.h, ctypes.c_uint64(ticket), -1, ctypes.byref(hb2)))
                hb = hb2
            return rec[:hb.count].copy(), float(hb.RTHLmax), int(hb.npeaks)
        self._check(rc)
        raise PPBError(-1, "unexpected ppb_wait result")

    def serve_stats(self) -> dict:
        st = _Stats()
        self._check(self.L.ppb_stats_get(self.h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in _Stats._fields_}

    def serve_stats_reset(self):
        self._check(self.L.ppb_stats_reset(self.h))

    def run_tile(self, cfg: PipelineConfig, seed: int = 42, plain: bool = False, write: bool = True):
        """Pipeline.run_tile(cfg; seed): reads cfg.pkfile / filterfile /
        tabfile, runs the tile, writes cfg.fileout (.pksc) and returns the
        (N, 11|33) float32 records."""
        k, pk = read_pk_table(cfg.pkfile)
        self.set_pk_table(k, pk)
        self.set_collapse_table(read_homeltab(cfg.tabfile))
        Rf = [f[2] for f in read_filterbank(cfg.filterfile)]
        rec, rthlmax, _ = self.run_tile_arrays(cfg, seed, Rf, plain=plain)
        if write:
            write_pksc(cfg.fileout, rec, rthlmax, cfg.z_out)
        return rec

    def fill_noise_threefry(self, n: int, seed: int) -> np.ndarray:
        out = np.empty((n, n, n), dtype=np.float32)
        self._check(self.L.ppb_noise_threefry(self.h, _p(out), n, int(seed) & (2**64 - 1)))
        return out

    def find_peaks(self, delta: np.ndarray, mask: np.ndarray, xbx: float, ybx: float, zbx: float, alatt: float,
                   nbuff: int, fcrit: float, Rsmooth: float = 0.0, max_peaks: int = 2000000):
        """find_peaks(delta, mask, xbx, ybx, zbx, alatt, nbuff, fcrit, Rsmooth):
        mask (int8) is updated in place.  Returns a dict of arrays (i, j, k,
        ipp 1-based; x, y, z physical; delta; Rsmooth)."""
        if delta.dtype != np.float32 or not delta.flags.c_contiguous:
            raise ValueError("delta must be a C-contiguous float32 array")
        if mask.dtype != np.int8 or not mask.flags.c_contiguous or mask.shape != delta.shape:
            raise ValueError("mask must be a C-contiguous int8 array of delta's shape")
        n3, n2, n1 = delta.shape
        cap = int(min(max_peaks, max(1, (n1 - 2 * nbuff) * (n2 - 2 * nbuff) * (n3 - 2 * nbuff))))
        cap = max(cap, 1)
        bi, bj, bk, bp = (np.empty(cap, np.int64) for _ in range(4))
        bd = np.empty(cap, np.float32)
        npk = ctypes.c_int64()
        self._check(self.L.ppb_find_peaks(self.h, _p(delta), _p(mask), n1, n2, n3, nbuff, ctypes.c_float(fcrit),
                                          max_peaks, _p(bi), _p(bj), _p(bk), _p(bp), _p(bd), ctypes.byref(npk)))
        m = npk.value
        i, j, k = bi[:m].copy(), bj[:m].copy(), bk[:m].copy()
        cen = lambda nn: 0.5 * (nn + 1)
        return {"i": i, "j": j, "k": k, "ipp": bp[:m].copy(), "x": xbx + alatt * (i - cen(n1)),
                "y": ybx + alatt * (j - cen(n2)), "z": zbx + alatt * (k - cen(n3)), "delta": bd[:m].copy(),
                "Rsmooth": np.full(m, float(Rsmooth))}

    def peak_find_tile(self, delta_tile: np.ndarray, filters, fcrits, tile_masks_in: np.ndarray, xbx: float,
                       ybx: float, zbx: float, alatt: float, nbuff: int, wsmooth: int, ioutshear: int):
        """peak_find_tile_gpu (src/PeakPatch.jl:341-366): the filter loop of
        smooth_field + find_peaks on a tile's own periodic grid.  filters:
        radii (Mpc/h) or (id, fcrit, Rf) tuples, processed in the given
        order; fcrits: one per filter.  tile_masks_in (int8, the field's
        shape) is updated in place.  Returns (peaks, Rf, FcRf, d2Rf, mask),
        peaks a dict of arrays (i, j, k, ipp, x, y, z, delta, Rsmooth,
        filter) in (filter, scan) order."""
        d = np.ascontiguousarray(delta_tile, dtype=np.float32)
        n = d.shape[0]
        if d.shape != (n, n, n):
            raise ValueError("peak_find_tile needs a cubic field")
        m = tile_masks_in
        if m.dtype != np.int8 or not m.flags.c_contiguous or m.shape != d.shape:
            raise ValueError("tile_masks_in must be a C-contiguous int8 array of the field's shape")
        Rf = np.ascontiguousarray([f[2] if isinstance(f, (tuple, list)) else f for f in filters], dtype=np.float64)
        fc = np.ascontiguousarray(np.broadcast_to(np.asarray(fcrits, dtype=np.float64), Rf.shape))
        cap = max(1, n ** 3 // 40)
        while True:
            o32 = [np.empty(cap, np.int32) for _ in range(4)]
            o64 = np.empty(cap, np.int64)
            od = [np.empty(cap, np.float64) for _ in range(4)]
            of = [np.empty(cap, np.float32) for _ in range(2)]
            npk = ctypes.c_int64()
            rc = self.L.ppb_peak_find_tile(self.h, _p(d), n, _p(Rf), _p(fc), len(Rf), _p(m), xbx, ybx, zbx, alatt,
                                           nbuff, wsmooth, ioutshear, cap, _p(o32[0]), _p(o32[1]), _p(o32[2]),
                                           _p(o64), _p(od[0]), _p(od[1]), _p(od[2]), _p(of[0]), _p(od[3]),
                                           _p(of[1]), _p(o32[3]), ctypes.byref(npk))
            if rc == -7:
                cap = npk.value
                continue
            self._check(rc)
            break
        c = npk.value
        peaks = {"i": o32[0][:c].astype(np.int64), "j": o32[1][:c].astype(np.int64),
                 "k": o32[2][:c].astype(np.int64), "ipp": o64[:c].copy(), "x": od[0][:c].copy(),
                 "y": od[1][:c].copy(), "z": od[2][:c].copy(), "delta": of[0][:c].copy(),
                 "Rsmooth": od[3][:c].copy(), "filter": o32[3][:c].copy()}
        return peaks, peaks["Rsmooth"].copy(), peaks["delta"].copy(), of[1][:c].copy(), m

    def analyse_peaks_multirf(self, fields: dict, batches, nhunt: int, alatt: float, ZZon: float = 1.0,
                              fcrit: float = 1.686, mask: np.ndarray = None, nbuff: int = 0, rmax2rs: float = 0.0,
                              plain: bool = False):
        """analyse_peaks_gpu_cuda_multirf (src/PeakPatch.jl:231-253): batches
        of (pi, pj, pk, Rf, ir2min[, ZZon_pp, fcrit_pp]) tuples, 1-based
        indices, one filter scale per batch.  mask (int8, the fields' shape)
        is read and updated in place.  Returns (list of (npk_b, 31) result
        arrays, mask)."""
        d = fields["delta"]
        n = d.shape[0]
        if d.shape != (n, n, n):
            raise ValueError("analyse_peaks_multirf needs a cubic grid")
        if mask is not None and (mask.dtype != np.int8 or not mask.flags.c_contiguous or mask.shape != d.shape):
            raise ValueError("mask must be a C-contiguous int8 array of the fields' shape")
        g = lambda key: None if fields.get(key) is None else np.ascontiguousarray(fields[key], np.float32)
        f = {k: g(k) for k in ("delta", "etax", "etay", "etaz", "eta2x", "eta2y", "eta2z", "lapd")}
        pp_ = len(batches) > 0 and len(batches[0]) >= 7
        cat = lambda i, t: np.ascontiguousarray(np.concatenate([np.asarray(b[i], t) for b in batches])
                                                if batches else np.zeros(0, t))
        boff = np.zeros(len(batches) + 1, np.int64)
        boff[1:] = np.cumsum([len(b[0]) for b in batches])
        pi, pj, pk = cat(0, np.int32), cat(1, np.int32), cat(2, np.int32)
        Rf = np.ascontiguousarray([float(b[3]) for b in batches], np.float64)
        ir2 = np.ascontiguousarray([int(b[4]) for b in batches], np.int64)
        Zpp = cat(5, np.float64) if pp_ else None
        fpp = cat(6, np.float64) if pp_ else None
        out = np.empty((max(int(boff[-1]), 1), 31), np.float64)
        self._check(self.L.ppb_analyse_peaks_multirf(
            self.h, _p(f["delta"]), _p(f["etax"]), _p(f["etay"]), _p(f["etaz"]), _p(f["eta2x"]), _p(f["eta2y"]),
            _p(f["eta2z"]), _p(f["lapd"]), n, nhunt, len(batches), _p(boff), _p(pi), _p(pj), _p(pk), _p(Rf),
            _p(ir2), _p(Zpp), _p(fpp), ZZon, fcrit, alatt, _p(mask), nbuff, rmax2rs, 1 if plain else 0, _p(out)))
        return [out[boff[b]:boff[b + 1]].copy() for b in range(len(batches))], mask

    def analyse_peaks(self, fields: dict, ipp, Rf, ir2min, ZZon, fcrit, alatt: float, nhunt: int,
                      plain: bool = False, r2lim=None) -> np.ndarray:
        """analyse_peak over a batch (rmax2rs = 0).  fields: delta, etax, etay,
        etaz and optional eta2x/eta2y/eta2z/lapd (C-order float32, cubic;
        numpy arrays or device pointers as ints).  r2lim: optional per-peak
        shell-list limit r^2 <= r2lim (cells^2).  Returns (npk, 31) float64
        (layout RESULT_FIELDS)."""
        d = fields["delta"]
        n = d.shape[0]
        if d.shape != (n, n, n):
            raise ValueError("analyse_peaks needs a cubic grid")
        npk = len(ipp)
        arr = lambda a, t: np.ascontiguousarray(np.broadcast_to(np.asarray(a, dtype=t), (npk,)))
        g = lambda key: None if fields.get(key) is None else np.ascontiguousarray(fields[key], np.float32)
        f = {k: g(k) for k in ("delta", "etax", "etay", "etaz", "eta2x", "eta2y", "eta2z", "lapd")}
        out = np.empty((npk, 31), dtype=np.float64)
        a_ipp, a_Rf, a_ir2, a_Z, a_fc = arr(ipp, np.int64), arr(Rf, np.float64), arr(ir2min, np.int64), \
            arr(ZZon, np.float64), arr(fcrit, np.float64)
        lim = None if r2lim is None else arr(r2lim, np.int32)
        self._check(self.L.ppb_analyse_peaks_lim(self.h, _p(f["delta"]), _p(f["etax"]), _p(f["etay"]),
                                                 _p(f["etaz"]), _p(f["eta2x"]), _p(f["eta2y"]), _p(f["eta2z"]),
                                                 _p(f["lapd"]), n, nhunt, npk, _p(a_ipp), _p(a_Rf), _p(a_ir2),
                                                 _p(a_Z), _p(a_fc), _p(lim), alatt, 1 if plain else 0, _p(out)))
        return out

    def set_collapse_table_f64(self, data: np.ndarray, ranges):
        """Collapse table with Float64 nodes; data C-order (nz, ny, nx), ranges
        (X1, X2, Y1, Y2, Z1, Z2)."""
        d = np.ascontiguousarray(data, dtype=np.float64)
        nz, ny, nx = d.shape
        self._check(self.L.ppb_set_collapse_table_f64(self.h, _p(d), nx, ny, nz, *[float(v) for v in ranges]))
        self._table_key = None

    def generate_fields(self, cfg: PipelineConfig, seed: int, pk_scale: float = 1.0) -> dict:
        """run_tile's fields (generate_grf, 1LPT, 2LPT, Laplacian) for cfg and
        seed as C-order float32 host arrays: delta, etax/etay/etaz,
        eta2x/eta2y/eta2z (ilpt = 2), lapd (ioutshear >= 1)."""
        p = self._params(cfg, seed, False, pk_scale)
        n = cfg.n
        d = np.empty((n, n, n), np.float32)
        psi = np.empty((3, n, n, n), np.float32)
        psi2 = np.empty((3, n, n, n), np.float32) if cfg.ilpt >= 2 else None
        lap = np.empty((n, n, n), np.float32) if cfg.ioutshear >= 1 else None
        self._check(self.L.ppb_generate_fields(self.h, ctypes.byref(p), _p(d), _p(psi), _p(psi2), _p(lap)))
        out = dict(delta=d, etax=psi[0], etay=psi[1], etaz=psi[2], lapd=lap)
        if psi2 is not None:
            out.update(eta2x=psi2[0], eta2y=psi2[1], eta2z=psi2[2])
        return out

    # ---- multi-resolution tile fields (src/MultiResolution.jl) -------------
    # Arrays are C-order float32 (k, j, i) = Julia's column-major [i, j, k];
    # tiles (it, jt, kt) are 1-based.  P(k) is the resident table: pass
    # pk=(k, P) to install one first, or None to use the installed one.
    def _pk(self, pk):
        if pk is not None:
            self.set_pk_table(np.asarray(pk[0], np.float64), np.asarray(pk[1], np.float64))

    @staticmethod
    def _f32(a, name):
        a = np.ascontiguousarray(a, np.float32)
        if a.ndim != 3 or not a.shape[0] == a.shape[1] == a.shape[2]:
            raise ValueError(f"{name} must be a cubic 3-D array")
        return a

    def downsample_noise(self, N: int, M: int, seed: int) -> np.ndarray:
        """_downsample_noise(N, M, seed) (src/MultiResolution.jl:68-89)."""
        out = np.empty((M, M, M), np.float32)
        self._check(self.L.ppb_downsample_noise(self.h, N, M, int(seed) & (2**64 - 1), _p(out)))
        return out

    def generate_extended_residual(self, it: int, jt: int, kt: int, nsub: int, nmesh: int, N: int, seed: int,
                                   coarse_noise: np.ndarray, M: int, nshell: int = 0) -> np.ndarray:
        """_generate_extended_residual (src/MultiResolution.jl:197-236)."""
        c = self._f32(coarse_noise, "coarse_noise")
        if c.shape[0] != M:
            raise ValueError("coarse_noise must be M^3")
        ne = nmesh + 2 * nshell
        out = np.empty((ne, ne, ne), np.float32)
        self._check(self.L.ppb_extended_residual(self.h, _p(c), M, it, jt, kt, nsub, nmesh, N,
                                                 int(seed) & (2**64 - 1), nshell, _p(out)))
        return out

    def isolated_convolve_gpu_multi(self, noise: np.ndarray, pk, boxsize_local: float, n: int,
                                    kernels=((0, 0, 0), (1, 1, 0), (1, 2, 0), (1, 3, 0)), nshell: int = 0):
        """isolated_convolve_gpu_multi (src/PeakPatch.jl:280-298): one
        zero-padded rfft of the noise, then per (kernel_fn_id, dim1, dim2)
        the transfer multiply and irfft; returns one n^3 array per kernel."""
        self._pk(pk)
        x = self._f32(noise, "noise")
        ks = np.ascontiguousarray(np.asarray(kernels, np.int32).reshape(-1, 3))
        out = np.empty((len(ks), n, n, n), np.float32)
        self._check(self.L.ppb_isolated_convolve(self.h, _p(x), x.shape[0], float(boxsize_local), n, _p(ks), len(ks),
                                                 nshell, _p(out)))
        return [out[i] for i in range(len(ks))]

    def isolated_convolve_gpu(self, noise: np.ndarray, pk, boxsize_local: float, n: int, kernel_fn_id: int = 0,
                              dim1: int = 0, dim2: int = 0, nshell: int = 0) -> np.ndarray:
        """isolated_convolve_gpu (src/PeakPatch.jl:255-278)."""
        return self.isolated_convolve_gpu_multi(noise, pk, boxsize_local, n, ((kernel_fn_id, dim1, dim2),),
                                                nshell)[0]

    def interpolate_to_tile_gpu(self, coarse: np.ndarray, it: int, jt: int, kt: int, nsub: int, nmesh: int, N: int,
                                M: int) -> np.ndarray:
        """interpolate_to_tile_gpu (src/PeakPatch.jl:329-339)."""
        c = self._f32(coarse, "coarse")
        if c.shape[0] != M:
            raise ValueError("coarse must be M^3")
        out = np.empty((nmesh, nmesh, nmesh), np.float32)
        self._check(self.L.ppb_interpolate_to_tile(self.h, _p(c), it, jt, kt, nsub, nmesh, N, M, _p(out)))
        return out

    def compute_2lpt_gpu(self, delta_tile: np.ndarray, nmesh: int, boxsize_local: float):
        """compute_2lpt_gpu (src/PeakPatch.jl:300-316): [psi2_x, psi2_y, psi2_z]."""
        d = self._f32(delta_tile, "delta_tile")
        out = np.empty((3, nmesh, nmesh, nmesh), np.float32)
        self._check(self.L.ppb_compute_2lpt(self.h, _p(d), nmesh, float(boxsize_local), _p(out)))
        return [out[0], out[1], out[2]]

    def compute_laplacian_gpu(self, delta_tile: np.ndarray, nmesh: int, boxsize_local: float) -> np.ndarray:
        """compute_laplacian_gpu (src/PeakPatch.jl:318-327)."""
        d = self._f32(delta_tile, "delta_tile")
        out = np.empty((nmesh, nmesh, nmesh), np.float32)
        self._check(self.L.ppb_compute_laplacian(self.h, _p(d), nmesh, float(boxsize_local), _p(out)))
        return out

    def coarse_fields(self, coarse_noise: np.ndarray, pk, boxsize_full: float, ilpt: int = 2,
                      ioutshear: int = 1) -> dict:
        """The coarse phase of run_multitile_split (src/MultiResolution.jl:
        617-667): delta, psi (3, M, M, M), psi2 (ilpt >= 2), lapd
        (ioutshear >= 1)."""
        self._pk(pk)
        c = self._f32(coarse_noise, "coarse_noise")
        M = c.shape[0]
        d = np.empty((M, M, M), np.float32)
        psi = np.empty((3, M, M, M), np.float32)
        psi2 = np.empty((3, M, M, M), np.float32) if ilpt >= 2 else None
        lap = np.empty((M, M, M), np.float32) if ioutshear >= 1 else None
        self._check(self.L.ppb_coarse_fields(self.h, _p(c), M, float(boxsize_full), ilpt, ioutshear, _p(d), _p(psi),
                                             _p(psi2), _p(lap)))
        return dict(delta=d, psi=psi, psi2=psi2, lapd=lap)


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def run_tile(cfg: PipelineConfig, seed: int = 42, verbose: bool = False, plain: bool = False):
    """Drop-in for Pipeline.run_tile(cfg; seed): returns the halo records and
    writes cfg.fileout."""
    rec = default_context().run_tile(cfg, seed=seed, plain=plain)
    if verbose:
        print(f"run_tile: {rec.shape[0]} halos -> {cfg.fileout}")
    return rec


def fill_noise_threefry(n: int, seed: int) -> np.ndarray:
    return default_context().fill_noise_threefry(n, seed)


def find_peaks(delta, mask, xbx, ybx, zbx, alatt, nbuff, fcrit, Rsmooth=0.0, max_peaks=2000000):
    return default_context().find_peaks(delta, mask, xbx, ybx, zbx, alatt, nbuff, fcrit, Rsmooth, max_peaks)


def analyse_peaks(fields, ipp, Rf, ir2min, ZZon, fcrit, alatt, nhunt, plain=False):
    return default_context().analyse_peaks(fields, ipp, Rf, ir2min, ZZon, fcrit, alatt, nhunt, plain)
