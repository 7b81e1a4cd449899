"""run_multitile across ranks, one process per GPU.

The tiles of a multi-tile run are independent once the global fields exist
(src/MultiTile.jl:284-402): every rank computes the fields and the filter
bank on the full grid, analyses its share of the tiles (round-robin over the
tile list), and rank 0 gathers the records, restores the single-process
tile order and applies merge_catalog (src/Merger/Merger.jl:21-78).  The only
collective is that gather of records; it runs over torch.distributed (gloo or
NCCL) as a pickled object gather, so it needs no device buffers.

A single run_tile does not shard (one periodic tile would need distributed-FFT
transposes): ranks run replicas of it instead.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

Tile = Tuple[int, int, int]


def tile_list(ntile: int, tiles: Optional[Sequence[Tile]] = None) -> List[Tile]:
    """The tiles of a run in processing order: the given list, else every
    tile of the ntile^3 grid in the reference's (kt, jt, it) loop order."""
    if tiles is not None:
        return [tuple(int(v) for v in t) for t in tiles]
    return [(it, jt, kt) for kt in range(1, ntile + 1) for jt in range(1, ntile + 1) for it in range(1, ntile + 1)]


def shard_tiles(tiles: Sequence[Tile], rank: int, world: int) -> List[Tile]:
    """Round-robin share of `rank` (tiles rank, rank + world, ...)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    return list(tiles[rank::world])


def tile_of_records(records: np.ndarray, ntile: int, dcore: float) -> np.ndarray:
    """(it, jt, kt) of each record from its Lagrangian position (fields 0-2).
    Tile (it, jt, kt) has its core centred at ((it - (ntile+1)/2) dcore, ...)
    (src/MultiTile.jl:79-86) and peaks lie half a cell or more inside a core,
    so the position decides the tile without ambiguity."""
    if len(records) == 0:
        return np.zeros((0, 3), np.int64)
    x = records[:, :3].astype(np.float64)
    return np.floor(x / dcore + ntile / 2.0).astype(np.int64) + 1


def split_by_tile(records: np.ndarray, tiles: Sequence[Tile], ntile: int, dcore: float) -> List[np.ndarray]:
    """The records of each listed tile, in the list's order (records of one
    tile keep their order)."""
    t = tile_of_records(records, ntile, dcore)
    out = []
    for tt in tiles:
        sel = (t[:, 0] == tt[0]) & (t[:, 1] == tt[1]) & (t[:, 2] == tt[2])
        out.append(records[sel])
    return out


def gather_tile_records(parts: dict, all_tiles: Sequence[Tile], nfields: int, group=None) -> Optional[np.ndarray]:
    """Gather {tile: records} from every rank to rank 0 and concatenate them
    in the order of `all_tiles`; other ranks get None."""
    import torch.distributed as dist
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    got = [None] * world if rank == 0 else None
    dist.gather_object(parts, got, dst=0, group=group)
    if rank != 0:
        return None
    merged = {}
    for d in got:
        merged.update(d)
    chunks = [merged[t] for t in all_tiles if t in merged and len(merged[t])]
    if not chunks:
        return np.zeros((0, nfields), np.float32)
    return np.concatenate(chunks, axis=0)


def run_multitile_sharded(run: Callable[[List[Tile]], np.ndarray], ntile: int, dcore: float, nfields: int,
                          tiles: Optional[Sequence[Tile]] = None, merge: Optional[Callable] = None,
                          group=None) -> Optional[np.ndarray]:
    """run_multitile over the ranks of `group`.

    run(tiles) analyses the given tiles on this rank's GPU and returns their
    records in that order (e.g. ``lambda t: ctx.run_multitile_arrays(cfg, seed,
    Rf, ntile, tiles=t)[0]``); merge(records) is applied on rank 0 (e.g.
    ``ctx.merge_catalog``).  Returns the catalogue on rank 0, None elsewhere.
    The catalogue equals the single-process one: the same records in the same
    tile order."""
    import torch.distributed as dist
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    all_tiles = tile_list(ntile, tiles)
    mine = shard_tiles(all_tiles, rank, world)
    rec = run(mine) if mine else np.zeros((0, nfields), np.float32)
    parts = dict(zip(mine, split_by_tile(rec, mine, ntile, dcore)))
    out = gather_tile_records(parts, all_tiles, nfields, group=group)
    if out is not None and merge is not None:
        out = merge(out)
    return out
