"""Host-side checks of the C-ABI library and the Python mirror of the
reference API.  CPU only: nothing here launches GPU work."""
import ctypes
import os
import re
import struct

import numpy as np
import pytest

from conftest import ROOT, GOLDEN

import peakpatch_b200 as pp


def _declared_functions():
    src = open(os.path.join(ROOT, "include", "ppb.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ppb_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = pp.load_library()
    declared = _declared_functions()
    assert len(declared) >= 15
    missing = [f for f in declared if not hasattr(L, f)]
    assert not missing, missing
    assert set(pp.EXPORTED) == set(declared)


def test_abi_version():
    assert pp.load_library().ppb_abi_version() == 5


def test_tile_params_layout_matches_the_header():
    # ppb_tile_params: 168 bytes, pk_scale at offset 144 (after plain and reserved0)
    assert ctypes.sizeof(pp._TileParams) == 168
    assert pp._TileParams.pk_scale.offset == 144
    assert ctypes.sizeof(pp._Stats) == 8 * 6 + 8 * 2 + 4 * 4


def test_tune_entry_layout_and_option_entry_points():
    # ppb_tune_entry: 8 int32, an int64, 5 + 4 floats, an int32, 4 floats, an int32, a float
    assert ctypes.sizeof(pp._TuneEntry) == 8 * 4 + 8 + 9 * 4 + 4 + 4 * 4 + 8
    assert pp._TuneEntry.gather_ms.offset == 40
    assert pp._TuneEntry.collapse_order.offset == 76 and pp._TuneEntry.collapse_ordered_ms.offset == 80
    L = pp.load_library()
    v = ctypes.c_int64()
    n = ctypes.c_int32()
    assert L.ppb_set_option(None, pp.OPT_GRAPHS, 1) == -1
    assert L.ppb_get_option(None, pp.OPT_GRAPHS, ctypes.byref(v)) == -1
    assert L.ppb_tune_entries(None, None, 0, ctypes.byref(n)) == -1


def test_table_params_layout_matches_the_header():
    # ppb_table_params: 4 doubles, 6 int32, 11 doubles, 4 int32 = 160 bytes
    assert ctypes.sizeof(pp._TableParams) == 160
    assert pp._TableParams.X1.offset == 56 and pp._TableParams.zinit_fac.offset == 136
    L = pp.load_library()
    assert L.ppb_make_collapse_table(None, None, None, 0) == -1


def test_serving_entry_points_reject_bad_arguments():
    L = pp.load_library()
    assert L.ppb_submit(None, None, None, 0, None) == -1
    assert L.ppb_wait(None, 1, 0, None) == -1
    assert L.ppb_stats_get(None, None) == -1
    assert L.ppb_serve_config(None, 4) == -1


def test_write_pksc_through_the_abi(tmp_path):
    L = pp.load_library()
    rec = np.arange(3 * 33, dtype=np.float32).reshape(3, 33)
    p = str(tmp_path / "a.pksc").encode()
    assert L.ppb_write_pksc(p, rec.ctypes.data_as(ctypes.c_void_p), 3, 33, ctypes.c_float(7.5),
                            ctypes.c_float(0.5)) == 0
    r, rthl, zo = pp.read_pksc(p.decode())
    assert np.array_equal(r, rec) and rthl == 7.5 and zo == 0.5
    # 11-field layout and the empty catalogue
    p2 = str(tmp_path / "b.pksc")
    pp.write_pksc(p2, np.zeros((0, 11), np.float32), 0.0, 0.0)
    raw = open(p2, "rb").read()
    assert len(raw) == 12 and struct.unpack("<i", raw[:4])[0] == 0
    assert L.ppb_write_pksc(p, rec.ctypes.data_as(ctypes.c_void_p), 3, 12, 0.0, 0.0) != 0


def test_invalid_arguments_fail_loudly_without_a_context():
    L = pp.load_library()
    assert L.ppb_ctx_destroy(None) == -1
    assert L.ppb_run_tile(None, None, None, 0, None) == -1
    assert L.ppb_set_pk_table(None, None, None, 0) == -1


def test_pipeline_config_from_toml():
    cfg = pp.PipelineConfig.from_toml({
        "cosmology": {"Om": 0.315, "OB": 0.049, "OL": 0.685, "h": 0.674},
        "grid": {"n": 128, "boxsize": 256.0, "nbuff": 32},
        "run": {"z_out": 0.5, "ilpt": 2, "ioutshear": 1, "wsmooth": 1, "rmax2rs": 0.0},
        "files": {"pk": "a.dat", "filterbank": "b.dat", "homeltab": "c.dat", "output": "o.pksc"}})
    assert cfg.Omx == pytest.approx(0.315 - 0.049) and cfg.n == 128 and cfg.nbuff == 32
    assert cfg.z_max == 0.5 and cfg.ioutshear == 1 and cfg.pkfile == "a.dat" and cfg.fileout == "o.pksc"
    d = pp.PipelineConfig()
    assert (d.n, d.boxsize, d.nbuff, d.rmax2rs, d.wsmooth) == (142, 200.0, 4, 1.0, 0)


def test_file_io_mirror(tmp_path):
    t = pp.read_homeltab(os.path.join(GOLDEN, "HomelTab_julia.dat"))
    assert t.shape_xyz == (50, 20, 20)
    p = str(tmp_path / "t.dat")
    pp.write_homeltab(p, t)
    assert open(p, "rb").read() == open(os.path.join(GOLDEN, "HomelTab_julia.dat"), "rb").read()
    fb = str(tmp_path / "f.dat")
    pp.write_filterbank(fb, [3.0, 1.5])
    assert pp.read_filterbank(fb) == [(1, 1.686, 3.0), (2, 1.686, 1.5)]
    k, P = pp.read_pk_table(os.path.join(GOLDEN, "test_pk.dat"))
    assert len(k) == 500 and k[0] == 1e-5 and k[-1] == 100.0


def test_eh_power_spectrum_normalisation():
    from peakpatch_b200 import powerspec as ps
    k, P = ps.eh_table(sigma8=0.808)
    Pstd = P * (2 * np.pi) ** 3
    assert ps.sigma_R(k, Pstd, 8.0) == pytest.approx(0.808, rel=2e-3)
    assert len(k) == 500 and k[0] == pytest.approx(1e-5) and k[-1] == pytest.approx(100.0)
    # shape: P rises at low k and falls at high k
    assert P[0] < P.max() and P[-1] < P.max()
    assert np.allclose(ps.rescale_sigma8(P, 0.75), P * (0.75 / 0.808) ** 2)


def test_product_never_uses_the_oracle():
    """The product package neither imports nor links the oracle: every
    compute entry point goes through libppb.so."""
    pkg = os.path.join(ROOT, "peakpatch.jl_b200")
    bad = re.compile(r"import\s+oracle|from\s+oracle|libppb_oracle|oracle\.cpp|oracle/")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cpp", ".h", ".cuh", ".jl")):
                txt = open(os.path.join(dirpath, f), errors="replace").read()
                assert not bad.search(txt), f
