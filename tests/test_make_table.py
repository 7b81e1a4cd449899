"""Collapse-table generation on the GPU (make_table, RK4 path) against the
oracle, bit for bit, and against the reference's own table file."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import peakpatch_b200 as pp
from conftest import filter_bank
from test_gpu_parity import match_records, tile_config

WEBSKY = (0.3138, 0.0493, 0.6862, 0.6735)   # the cosmology HomelTab_julia.dat was made for


@pytest.fixture(scope="module")
def gctx():
    with pp.Context(0) as c:
        yield c


def test_default_table_is_the_reference_table(gctx, ora, julia_table):
    g = gctx.make_table(*WEBSKY)
    o = ora.make_table(*WEBSKY)
    assert g.tobytes() == o.tobytes()                         # FP64 nodes identical to the oracle
    assert np.array_equal(g.astype(np.float32), julia_table.data)   # and to the reference's file
    st = gctx.table_stats()
    assert st["ms"] > 0 and st["rk4_steps"] > 20000


@pytest.mark.parametrize("iforce,ivir", [(0, 2), (1, 2), (3, 2), (4, 1), (5, 1), (6, 2)])
def test_force_and_virialisation_strategies(gctx, ora, iforce, ivir):
    tp = pp.CollapseTableParams(Nx=9, Ny=5, Nz=4, iforce_strat=iforce, ivir_strat=ivir)
    otp = ora.TableParams(Nx=9, Ny=5, Nz=4, iforce_strat=iforce, ivir_strat=ivir)
    g = gctx.make_table(0.315, 0.049, 0.685, 0.674, tp)
    o = ora.make_table(0.315, 0.049, 0.685, 0.674, otp)
    assert (o > 0).any() or iforce == 6   # strategy 6 collapses nothing on this grid
    assert g.tobytes() == o.tobytes(), (iforce, ivir, np.abs(g - o).max())


def test_installed_table_runs_the_tile_like_the_file(gctx, julia_table, eh_pk):
    RF = [f[2] for f in filter_bank()]
    cfg = tile_config()
    gctx.set_pk_table(*eh_pk)
    T = julia_table
    gctx.set_collapse_table(pp.CollapseTable(T.data, T.x1, T.x2, T.y1, T.y2, T.z1, T.z2))
    a, _, _ = gctx.run_tile_arrays(cfg, 17, RF)
    gctx.make_table(*WEBSKY, install=1)                 # Float32 nodes, as the file
    b, _, _ = gctx.run_tile_arrays(cfg, 17, RF)
    # the same nodes; the file stores the axis ranges as Float32, the
    # in-process table keeps them in double (as make_table's own result), so
    # a lookup may differ in the last bits
    frac, errs = match_records(b, a, 33)
    assert len(a) > 20 and frac <= 0.01 and errs["RTHL"] < 1e-5, (frac, errs)
    gctx.make_table(0.315, 0.049, 0.685, 0.674, install=2)   # another cosmology, Float64 nodes
    c, _, _ = gctx.run_tile_arrays(cfg, 17, RF)
    assert len(c) > 20 and c.tobytes() != a.tobytes()


def test_bad_parameters_are_rejected(gctx):
    with pytest.raises(pp.PPBError):
        gctx.make_table(0.3, 0.05, 0.7, 0.7, pp.CollapseTableParams(Nx=1))
    with pytest.raises(pp.PPBError):
        gctx.make_table(0.3, 0.05, 0.7, 0.7, pp.CollapseTableParams(iforce_strat=2))
