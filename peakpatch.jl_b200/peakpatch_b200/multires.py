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
