"""Serving loop (ppb_serve_config / ppb_submit / ppb_wait / ppb_stats_get).

The serving loop runs tile requests of different grid sizes, seeds and
cosmologies on several execution slots at once.  Its contract: every result
equals the result of the same request run alone through ppb_run_tile, no
matter what ran beside it; requests that can never fit the HBM budget fail
with PPB_ERR_ADMISSION; a bounded wait returns PPB_ERR_TIMEOUT and leaves the
request in place."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import peakpatch_b200 as pp
from conftest import GOLDEN, filter_bank

RF = [f[2] for f in filter_bank()]


def _cfg(n, ievol=0, box_per_cell=2.0):
    box = box_per_cell * n
    z_max = 1.0 if ievol else 0.0
    cen = -box / 2 if ievol else 0.0
    return pp.PipelineConfig(Omx=0.315 - 0.049, OmB=0.049, Omvac=0.685, h=0.674, n=n, boxsize=box, nbuff=16,
                             z_out=0.0, z_max=z_max, ievol=ievol, ilpt=2, ioutshear=1, wsmooth=1, rmax2rs=0.0,
                             cenx=cen, ceny=cen, cenz=cen)


def _tables(ctx):
    from peakpatch_b200 import powerspec
    k, P = powerspec.eh_table()
    ctx.set_pk_table(k, P)
    ctx.set_collapse_table(pp.read_homeltab(os.path.join(GOLDEN, "HomelTab_julia.dat")))


# (n, seed, sigma8, ievol): mixed sizes, seeds and cosmologies
MIX = [(64, 11, 0.808, 0), (96, 12, 0.78, 1), (128, 13, 0.84, 0), (64, 14, 0.75, 1), (96, 15, 0.82, 0),
       (128, 16, 0.808, 1), (64, 17, 0.80, 0), (96, 18, 0.85, 0)]


def test_each_result_is_the_same_alone_and_in_the_mix():
    with pp.Context(0) as ctx:
        _tables(ctx)
        alone = []
        for n, seed, s8, ievol in MIX:
            rec, rmax, npk = ctx.run_tile_arrays(_cfg(n, ievol), seed, RF, pk_scale=(s8 / 0.808) ** 2)
            assert len(rec) > 0
            alone.append((rec, rmax, npk))
        ctx.serve_config(3)
        tickets = [ctx.submit(_cfg(n, ievol), seed, RF, pk_scale=(s8 / 0.808) ** 2) for n, seed, s8, ievol in MIX]
        for t, (rec0, rmax0, npk0), m in zip(tickets, alone, MIX):
            rec, rmax, npk = ctx.wait(t)
            assert npk == npk0, m
            assert rec.shape == rec0.shape, m
            assert rec.tobytes() == rec0.tobytes(), m
            assert rmax == rmax0, m
        st = ctx.serve_stats()
        assert st["tiles_done"] == len(MIX) and st["failed"] == 0
        assert st["p99_ms"] >= st["p50_ms"] > 0 and st["tiles_per_s"] > 0
        assert st["slots"] == 3 and st["queued"] == 0 and st["in_flight"] == 0


def test_tight_budget_evicts_resident_sizes_and_keeps_every_result():
    # about 900 MB: a 128^3 request's estimate is ~0.8 GB (0.33 GB of grid-size
    # buffers, the rest shell-stage buffers of its slot), so three slots
    # cycling through the mix must give resident sizes back to admit the next
    with pp.Context(0, hbm_budget=900 << 20) as ctx:
        _tables(ctx)
        alone = [ctx.run_tile_arrays(_cfg(n, ievol), seed, RF, pk_scale=(s8 / 0.808) ** 2)
                 for n, seed, s8, ievol in MIX]
        ctx.serve_config(3)
        tickets = [ctx.submit(_cfg(n, ievol), seed, RF, pk_scale=(s8 / 0.808) ** 2) for n, seed, s8, ievol in MIX]
        for t, (rec0, rmax0, npk0), m in zip(tickets, alone, MIX):
            rec, rmax, npk = ctx.wait(t)
            assert npk == npk0 and rec.tobytes() == rec0.tobytes() and rmax == rmax0, m
        st = ctx.serve_stats()
        assert st["failed"] == 0 and st["tiles_done"] == len(MIX)
        # admission works on estimates; what the slots then hold may exceed them a little
        assert st["hbm_in_use"] <= 1.25 * (900 << 20)


def test_sigma8_rescale_changes_the_catalogue():
    with pp.Context(0) as ctx:
        _tables(ctx)
        a, _, _ = ctx.run_tile_arrays(_cfg(64), 5, RF)
        b, _, _ = ctx.run_tile_arrays(_cfg(64), 5, RF, pk_scale=1.0)
        c, _, _ = ctx.run_tile_arrays(_cfg(64), 5, RF, pk_scale=(0.85 / 0.808) ** 2)
        assert a.tobytes() == b.tobytes()        # pk_scale 1 is the unscaled table
        assert len(c) > len(a)                   # more power, more collapsed halos


def test_admission_refuses_a_request_larger_than_the_budget():
    with pp.Context(0, hbm_budget=256 << 20) as ctx:
        _tables(ctx)
        t = ctx.submit(_cfg(128), 1, RF)
        with pytest.raises(pp.PPBError) as e:
            ctx.wait(t)
        assert e.value.code == -4
        assert ctx.serve_stats()["failed"] == 1


def test_bounded_wait_times_out_and_leaves_the_request():
    with pp.Context(0) as ctx:
        _tables(ctx)
        ctx.serve_config(1)
        t1 = ctx.submit(_cfg(128), 1, RF)
        t2 = ctx.submit(_cfg(128), 2, RF)
        assert ctx.wait(t2, timeout_ms=0) is None      # queued behind t1 on the only slot
        r1 = ctx.wait(t1)
        r2 = ctx.wait(t2)
        assert len(r1[0]) > 0 and len(r2[0]) > 0
        with pytest.raises(pp.PPBError) as e:
            ctx.wait(t2)
        assert e.value.code == -8                       # each ticket is collected once
