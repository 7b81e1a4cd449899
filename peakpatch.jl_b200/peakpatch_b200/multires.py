"""Host side of the multi-resolution (MUSIC-style) split of
src/MultiResolution.jl on the library's GPU stages.

The split replaces one global FFT of the N^3 grid by a coarse periodic M^3
grid for the long modes (interpolated to each tile with Catmull-Rom
weights) plus, per tile, an isolated zero-padded convolution of the
Hoffman–Ribak residual (fine noise minus its coarse block mean).  Every
array stage runs in libppb (Context.downsample_noise, coarse_fields,
generate_extended_residual, isolated_convolve_gpu_multi,
interpolate_to_tile_gpu, compute_2lpt_gpu, compute_laplacian_gpu); this
module only sequences them.
"""
from __future__ import annotations

from typing import List

import numpy as np

from . import Context, PipelineConfig


def split_geometry(N: int, ntile: int, nbuff: int, coarse_factor: int = 0, coarse_grid: int = 0):
    """(nsub, nmesh, M) of compare_fields_split (src/MultiResolution.jl:
    1269-1276): N = nsub ntile + 2 nbuff, nmesh = nsub + 2 nbuff, M =
    coarse_grid or ntile coarse_factor; N % M == 0."""
    nsub = (N - 2 * nbuff) // ntile
    nmesh = nsub + 2 * nbuff
    if nsub < 1 or nsub * ntile + 2 * nbuff != N:
        raise ValueError(f"N={N} not consistent with ntile={ntile}, nbuff={nbuff}")
    M = coarse_grid if coarse_grid > 0 else ntile * coarse_factor
    if M < 1 or N % M != 0:
        raise ValueError(f"N={N} must be divisible by M={M}")
    return nsub, nmesh, M


def _correlation(a, b):
    da = a - a.sum() / a.size
    db = b - b.sum() / b.size
    return float((da * db).sum() / np.sqrt((da ** 2).sum() * (db ** 2).sum()))


def _rms_frac(a, b):
    ra = np.sqrt((a ** 2).sum() / a.size)
    return float(np.sqrt(((a - b) ** 2).sum() / a.size) / ra) if ra > 0 else 0.0


def compare_fields_split(ctx: Context, pk, N: int, boxsize: float, seed: int, ntile: int, coarse_factor: int,
                         nbuff: int = 8, coarse_grid: int = 0) -> List[dict]:
    """compare_fields_split (src/MultiResolution.jl:1266-1353): per tile
    (it fastest), the split delta and psi_x against the global-FFT fields
    (generate_grf and displacements_1lpt on N^3) on the tile core.  pk =
    (k, P) installs a P(k) table first; None uses the resident one.
    Returns dicts with tile, corr_delta, rms_delta, corr_psi1, rms_psi1,
    std_global_delta."""
    nsub, nmesh, M = split_geometry(N, ntile, nbuff, coarse_factor, coarse_grid)
    alatt = boxsize / N
    ctx._pk(pk)
    cfg = PipelineConfig(n=N, boxsize=float(boxsize), nbuff=nbuff, ilpt=1, ioutshear=0)
    glob = ctx.generate_fields(cfg, seed)
    coarse_noise = ctx.downsample_noise(N, M, seed)
    cf = ctx.coarse_fields(coarse_noise, None, boxsize, ilpt=1, ioutshear=0)
    box_tile = nmesh * alatt
    out = []
    core = slice(nbuff, nbuff + nsub)
    for kt in range(1, ntile + 1):
        for jt in range(1, ntile + 1):
            for it in range(1, ntile + 1):
                sl = lambda t: slice((t - 1) * nsub, t * nsub)
                ref_d = glob["delta"][sl(kt), sl(jt), sl(it)].astype(np.float64)
                ref_p = glob["etax"][sl(kt), sl(jt), sl(it)].astype(np.float64)
                res = ctx.generate_extended_residual(it, jt, kt, nsub, nmesh, N, seed, coarse_noise, M, 0)
                d_self, p_self = ctx.isolated_convolve_gpu_multi(res, None, box_tile, nmesh, ((0, 0, 0), (1, 1, 0)))
                d = d_self + ctx.interpolate_to_tile_gpu(cf["delta"], it, jt, kt, nsub, nmesh, N, M)
                p = p_self + ctx.interpolate_to_tile_gpu(cf["psi"][0], it, jt, kt, nsub, nmesh, N, M)
                d = d[core, core, core].astype(np.float64)
                p = p[core, core, core].astype(np.float64)
                out.append(dict(tile=(it, jt, kt), corr_delta=_correlation(ref_d, d), rms_delta=_rms_frac(ref_d, d),
                                corr_psi1=_correlation(ref_p, p), rms_psi1=_rms_frac(ref_p, p),
                                std_global_delta=float(np.sqrt((ref_d ** 2).mean()))))
    return out


def coarse_grid_size(n: int, nbuff: int, ntile: int, coarse_factor: int = 0, coarse_grid: int = 0) -> int:
    """The coarse grid M run_multitile_split uses for tile size n (src/
    MultiResolution.jl:592-612)."""
    from . import load_library
    m = load_library().ppb_split_coarse_grid(n, nbuff, ntile, coarse_factor, coarse_grid)
    if m < 0:
        raise ValueError("invalid tile geometry")
    return m


def run_multitile_split(cfg: PipelineConfig, ntile: int, seed: int = 42, verbose: bool = False,
                        coarse_factor: int = 0, coarse_grid: int = 0, use_gpu: bool = True, devices=None,
                        profile: bool = False, ctx: Context = None, Rf=None, pk=None, table=None):
    """Drop-in for run_multitile_split(cfg; ntile, seed, verbose,
    coarse_factor, coarse_grid, use_gpu, devices, profile)
    (src/MultiResolution.jl:523-1236); returns the records array (11 or 33
    Float32 fields per halo).

    Every stage runs on the GPU whatever `use_gpu` says (this library has no
    CPU path).  devices=[d0, d1, ...] splits the tiles round-robin over one
    worker per device (tile i to worker (i mod n_workers)) and concatenates
    the workers' records in worker order, as the reference does
    (:1183-1213); otherwise one context (ctx, or a new one on device 0)
    processes the tiles in order.  pk = (k, P), table (a CollapseTable) and
    Rf (filter radii) are installed when given; otherwise a new context reads
    them from cfg's pkfile, tabfile and filterfile, and a given ctx keeps the
    tables it holds."""
    import threading
    import time
    from . import read_filterbank, read_homeltab, read_pk_table

    def setup(c: Context, fresh: bool):
        if pk is not None:
            c.set_pk_table(np.asarray(pk[0], np.float64), np.asarray(pk[1], np.float64))
        elif fresh:
            c.set_pk_table(*read_pk_table(cfg.pkfile))
        if table is not None:
            c.set_collapse_table(table)
        elif fresh:
            c.set_collapse_table(read_homeltab(cfg.tabfile))
        return list(Rf) if Rf is not None else [f[2] for f in read_filterbank(cfg.filterfile)]

    t0 = time.perf_counter()
    tile_ids = [(it, jt, kt) for kt in range(1, ntile + 1) for jt in range(1, ntile + 1) for it in range(1, ntile + 1)]
    if devices:
        nw = len(devices)
        parts = [None] * nw
        errs = []

        def work(w):
            try:
                mine = [t for i, t in enumerate(tile_ids) if i % nw == w]
                if not mine:
                    parts[w] = np.zeros((0, 33 if cfg.ioutshear >= 1 else 11), np.float32)
                    return
                with Context(int(devices[w])) as c:
                    rf = setup(c, True)
                    parts[w] = c.run_multitile_split_arrays(cfg, seed, rf, ntile, coarse_factor, coarse_grid,
                                                            tiles=mine)[0]
            except Exception as e:   # surfaced after join
                errs.append(e)

        th = [threading.Thread(target=work, args=(w,)) for w in range(nw)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        if errs:
            raise errs[0]
        rec = np.concatenate(parts, axis=0)
    else:
        c = ctx if ctx is not None else Context(0)
        rf = setup(c, ctx is None)
        rec = c.run_multitile_split_arrays(cfg, seed, rf, ntile, coarse_factor, coarse_grid)[0]
    if verbose or profile:
        print(f"run_multitile_split: {len(rec)} halos, ntile={ntile}, nmesh={cfg.n}, "
              f"{time.perf_counter() - t0:.2f} s")
    return rec
