"""CUDA-graph launches and the shell-stage autotuner.  Neither may change a
result: the records of run_tile and run_multitile are compared byte for byte
with graphs on and off and under every gather-order brick and collapse width
the autotuner chooses from."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import peakpatch_b200 as pp
from conftest import filter_bank
from test_gpu_parity import tile_config

RF = [f[2] for f in filter_bank()]


@pytest.fixture(scope="module")
def tctx(julia_table, eh_pk):
    T = julia_table
    with pp.Context(0) as c:
        c.set_pk_table(*eh_pk)
        c.set_collapse_table(pp.CollapseTable(T.data, T.x1, T.x2, T.y1, T.y2, T.z1, T.z2))
        yield c


def _defaults(c):
    c.set_option(pp.OPT_GRAPHS, 1)
    c.set_option(pp.OPT_AUTOTUNE, 0)
    c.set_option(pp.OPT_BRICK_SHIFT, -2)
    c.set_option(pp.OPT_COLLAPSE_THREADS, 0)
    c.set_option(pp.OPT_TUNE_MIN_PEAKS, 16384)
    c.set_option(pp.OPT_COLLAPSE_ORDER, -1)
    c.set_option(pp.OPT_GATHER_TEX, -1)


def test_graphs_on_and_off_give_the_same_records(tctx):
    _defaults(tctx)
    cfg = tile_config()
    tctx.set_option(pp.OPT_GRAPHS, 0)
    a, _, _ = tctx.run_tile_arrays(cfg, 31, RF)
    g0 = tctx.graph_stats()
    tctx.set_option(pp.OPT_GRAPHS, 1)
    b, _, _ = tctx.run_tile_arrays(cfg, 31, RF)
    g1 = tctx.graph_stats()
    assert g1["launches"] >= g0["launches"] + 3   # fields, filter bank, shell stage
    c, _, _ = tctx.run_tile_arrays(cfg, 32, RF)   # another seed: the graphs are updated in place
    d, _, _ = tctx.run_tile_arrays(cfg, 31, RF)
    g3 = tctx.graph_stats()
    assert g3["updates"] >= g1["updates"] + 4
    assert a.tobytes() == b.tobytes() == d.tobytes()
    assert c.tobytes() != a.tobytes()


def test_multitile_chain_graphs_on_and_off(tctx):
    _defaults(tctx)
    cfg = tile_config()
    tctx.set_option(pp.OPT_GRAPHS, 0)
    a, _, _ = tctx.run_multitile_arrays(cfg, 5, RF, ntile=2, tiles=[(1, 1, 1), (2, 2, 1)])
    tctx.set_option(pp.OPT_GRAPHS, 1)
    b, _, _ = tctx.run_multitile_arrays(cfg, 5, RF, ntile=2, tiles=[(1, 1, 1), (2, 2, 1)])
    assert len(a) > 20 and a.tobytes() == b.tobytes()


@pytest.mark.parametrize("brick", [-1, 2, 3, 4, 5])
def test_every_order_brick_and_collapse_width_gives_the_same_records(tctx, brick):
    _defaults(tctx)
    cfg = tile_config()
    ref, _, _ = tctx.run_tile_arrays(cfg, 41, RF)
    tctx.set_option(pp.OPT_BRICK_SHIFT, brick)
    for w in (1, 2, 4, 8):
        tctx.set_option(pp.OPT_COLLAPSE_THREADS, w)
        g, _, _ = tctx.run_tile_arrays(cfg, 41, RF)
        assert g.tobytes() == ref.tobytes(), (brick, w)
    _defaults(tctx)


def test_autotuner_times_every_candidate_and_keeps_the_records(tctx):
    _defaults(tctx)
    cfg = tile_config()
    ref, _, _ = tctx.run_tile_arrays(cfg, 43, RF)
    tctx.set_option(pp.OPT_TUNE_MIN_PEAKS, 1)
    tctx.set_option(pp.OPT_AUTOTUNE, 2)   # clear the table, tune on next use
    a, _, npk = tctx.run_tile_arrays(cfg, 43, RF)
    ents = tctx.tune_entries()
    assert len(ents) == 1
    e = ents[0]
    assert e["n"] == cfg.n and e["comp"] and e["adaptive"] and not e["limited"] and e["npk"] == npk
    assert all(v > 0 for v in e["gather_ms"].values()) and all(v > 0 for v in e["collapse_ms"].values())
    assert all(v > 0 for v in e["collapse_ordered_ms"].values())
    assert e["brick"] in (0, 4, 8, 16, 32) and e["collapse_threads"] in (0, 1, 2, 4, 8)
    b, _, _ = tctx.run_tile_arrays(cfg, 43, RF)   # runs with the tuned choice, no new entry
    assert len(tctx.tune_entries()) == 1
    assert ref.tobytes() == a.tobytes() == b.tobytes()
    _defaults(tctx)


@pytest.mark.parametrize("plain", [False, True])
def test_tma_staged_gather_gives_the_same_records(tctx, plain):
    """Records gathered through the per-lane TMA rings (tile::gather4 copies
    into shared memory) equal those of plain loads byte for byte: the same
    cells in the same order reach the same sums.  Also for a multi-tile run
    (the tile's own record array) and with the compensated sums off."""
    _defaults(tctx)
    cfg = tile_config()
    try:
        tctx.set_option(pp.OPT_GATHER_RING, 0)
        a, _, _ = tctx.run_tile_arrays(cfg, 51, RF, plain=plain)
        m0, _, _ = tctx.run_multitile_arrays(cfg, 5, RF, ntile=2, tiles=[(1, 1, 1), (2, 2, 1)])
        tctx.set_option(pp.OPT_GATHER_RING, 1)
        b, _, _ = tctx.run_tile_arrays(cfg, 51, RF, plain=plain)
        m1, _, _ = tctx.run_multitile_arrays(cfg, 5, RF, ntile=2, tiles=[(1, 1, 1), (2, 2, 1)])
        assert tctx.get_option(pp.OPT_GATHER_RING) == 1
    finally:
        tctx.set_option(pp.OPT_GATHER_RING, 0)
    assert len(a) > 100 and a.tobytes() == b.tobytes()
    assert m0.tobytes() == m1.tobytes()


def test_collapse_order_gives_the_same_records(tctx):
    """The collapse kernels taking the peaks by descending crossing shell
    (PPB_OPT_COLLAPSE_ORDER) give the records of list order, byte for byte,
    under every collapse width."""
    _defaults(tctx)
    cfg = tile_config()
    try:
        tctx.set_option(pp.OPT_COLLAPSE_ORDER, 0)
        ref, _, _ = tctx.run_tile_arrays(cfg, 61, RF)
        tctx.set_option(pp.OPT_COLLAPSE_ORDER, 1)
        for w in (0, 1, 2, 4, 8):
            tctx.set_option(pp.OPT_COLLAPSE_THREADS, w)
            g, _, _ = tctx.run_tile_arrays(cfg, 61, RF)
            assert g.tobytes() == ref.tobytes(), w
    finally:
        tctx.set_option(pp.OPT_COLLAPSE_ORDER, -1)
        tctx.set_option(pp.OPT_COLLAPSE_THREADS, 0)
    assert len(ref) > 100


def test_texture_and_plain_record_loads_give_the_same_records(tctx):
    """The gather's records fetched through the texture pipe (the default) or
    with 256-bit loads: byte-identical records, tile and multi-tile."""
    _defaults(tctx)
    cfg = tile_config()
    try:
        tctx.set_option(pp.OPT_GATHER_TEX, 0)
        a, _, _ = tctx.run_tile_arrays(cfg, 71, RF)
        m0, _, _ = tctx.run_multitile_arrays(cfg, 5, RF, ntile=2, tiles=[(1, 1, 1), (2, 2, 1)])
        tctx.set_option(pp.OPT_GATHER_TEX, 1)
        b, _, _ = tctx.run_tile_arrays(cfg, 71, RF)
        m1, _, _ = tctx.run_multitile_arrays(cfg, 5, RF, ntile=2, tiles=[(1, 1, 1), (2, 2, 1)])
        assert tctx.get_option(pp.OPT_GATHER_TEX) == 1
    finally:
        tctx.set_option(pp.OPT_GATHER_TEX, -1)
    assert len(a) > 100 and a.tobytes() == b.tobytes() and m0.tobytes() == m1.tobytes()
