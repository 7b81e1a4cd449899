"""HDF5 catalogue output (write_catalog_hdf5, ext/HDF5Ext.jl:47-104) without
libhdf5: the library's writer against the package's reader of the same
subset of the format, and the derived columns against their definitions.
CPU only (the writer is host code)."""
import struct

import numpy as np
import pytest

import peakpatch_b200 as pp
from peakpatch_b200.hdf5 import read_catalog_hdf5, write_catalog_hdf5

OM, OL, H = 0.315, 0.685, 0.674


def _records(n, nf, seed=0):
    rng = np.random.default_rng(seed)
    r = rng.normal(size=(n, nf)).astype(np.float32)
    r[:, :3] = rng.uniform(-900, 900, size=(n, 3))   # positions, Mpc/h
    r[:, 6] = rng.uniform(1.0, 20.0, size=n)          # RTHL, Mpc/h
    return r


@pytest.mark.parametrize("nf", [11, 33])
def test_hdf5_round_trip_and_columns(ora, tmp_path, nf):
    rec = _records(257, nf)
    path = str(tmp_path / "cat.h5")
    write_catalog_hdf5(path, rec, OM, OL, H, z_max=10.0)
    d = read_catalog_hdf5(path)
    base = ["x", "y", "z", "ra", "dec", "redshift", "chi", "M200m", "RTHL", "vx", "vy", "vz"]
    ext = ["vx2", "vy2", "vz2", "overdensity", "e_v", "p_v", "Rf", "zform"]
    assert sorted(d) == sorted(base + (ext if nf == 33 else []))
    for name in d:
        assert d[name].dtype == np.float32 and d[name].shape == (len(rec),), name
    col = {"x": 0, "y": 1, "z": 2, "vx": 3, "vy": 4, "vz": 5, "RTHL": 6, "vx2": 7, "vy2": 8, "vz2": 9,
           "overdensity": 10, "e_v": 11, "p_v": 12, "Rf": 27, "zform": 20}
    for name, c in col.items():
        if name in d:
            assert np.array_equal(d[name], rec[:, c]), name
    x, y, z = (rec[:, i].astype(np.float64) for i in range(3))
    r = np.sqrt(x * x + y * y + z * z)
    assert np.array_equal(d["chi"], r.astype(np.float32))
    # M200m = 4/3 pi rho_m RTHL^3, rho_m = 2.775e11 Om h^2 (ext/HDF5Ext.jl:58, 64)
    R = rec[:, 6].astype(np.float64)
    m = (4.0 / 3.0 * np.pi * (2.775e11 * OM * H * H) * R ** 3).astype(np.float32)
    assert np.allclose(d["M200m"], m, rtol=1e-6)
    assert np.allclose(d["dec"], np.arcsin(np.clip(z / r, -1, 1)).astype(np.float32), rtol=0, atol=1e-6)
    assert np.allclose(d["ra"], np.arctan2(y, x).astype(np.float32), rtol=0, atol=1e-6)
    # redshift from the reference's chi -> z table (build_chi_to_z, 2000 points to z_max)
    zo = ora.chi_to_z(OM, OL, H, 10.0, d["chi"].astype(np.float64)).astype(np.float32)
    assert np.allclose(d["redshift"], zo, rtol=1e-6, atol=1e-7)
    # the superblock's end-of-file address is the file's length
    raw = open(path, "rb").read()
    assert struct.unpack_from("<Q", raw, 40)[0] == len(raw)


def test_hdf5_empty_catalogue(tmp_path):
    path = str(tmp_path / "empty.h5")
    write_catalog_hdf5(path, np.zeros((0, 33), np.float32), OM, OL, H)
    assert read_catalog_hdf5(path) == {}


def test_hdf5_from_run_records_and_reader_rejects_other_files(tmp_path):
    p = str(tmp_path / "a.pksc")
    pp.write_pksc(p, _records(5, 33), 1.0, 0.0)
    with pytest.raises(ValueError):
        read_catalog_hdf5(p)
    rec, _, _ = pp.read_pksc(p)
    h = str(tmp_path / "a.h5")
    write_catalog_hdf5(h, rec, OM, OL, H)
    assert np.array_equal(read_catalog_hdf5(h)["Rf"], rec[:, 27])
