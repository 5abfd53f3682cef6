"""Partition of a tile list over GPUs, one process per GPU.

Tiles are independent (no exchange step), so N GPUs decode N disjoint
shards of one global tile list and nothing crosses between them on the data
path.  Shards are balanced by coded bytes, the quantity the decode time
follows, the way the reference's CPU tile batch splits its jobs over workers
by contiguous chunks (crates/signinum-j2k/src/batch.rs:110-147) but weighted
by size, since tiles of a batch are uneven.

The balancing starts from a round-robin assignment (tile g to rank g mod N),
which lets each rank produce its own candidates without any other rank's
data, and then moves single tiles from the heaviest shard to the lightest
while that lowers the heaviest; every rank runs the same deterministic steps
on the same all-gathered sizes, so all agree on the shards without a
coordinator.
"""
from __future__ import annotations

from typing import Callable, Dict, List, Sequence, Tuple


def round_robin(n_total: int, world: int, rank: int) -> List[int]:
    return list(range(rank, n_total, world))


def balance_by_coded_bytes(sizes: Sequence[int], world: int,
                           owners: Sequence[int] | None = None) -> List[List[int]]:
    """Shards (ascending tile indices per rank) of tiles with `sizes` coded
    bytes over `world` ranks.  Starting from `owners` (default round robin),
    a tile moves from the heaviest shard to the lightest while its size is
    below their gap; each move lowers the sum of squared loads, so the loop
    ends, with every shard within the largest tile's size of every other."""
    n = len(sizes)
    if owners is None:
        owners = [g % world for g in range(n)]
    shards: List[set] = [set() for _ in range(world)]
    loads = [0] * world
    for g, r in enumerate(owners):
        shards[r].add(g)
        loads[r] += sizes[g]
    while world > 1:
        h = max(range(world), key=lambda r: (loads[r], -r))
        lo = min(range(world), key=lambda r: (loads[r], r))
        gap = loads[h] - loads[lo]
        best = None
        for g in shards[h]:
            if sizes[g] < gap and (best is None or (sizes[g], g) > (sizes[best], best)):
                best = g
        if best is None or sizes[best] == 0:
            break
        shards[h].remove(best)
        shards[lo].add(best)
        loads[h] -= sizes[best]
        loads[lo] += sizes[best]
    return [sorted(s) for s in shards]


def shard_tiles(dist, n_total: int, encode: Callable[[List[int]], list]) -> Tuple[List[int], list, Dict]:
    """This rank's shard of a global list of n_total tiles.

    encode(indices) returns the tiles (objects with .codestream, .width,
    .height) of the given global indices; tile g is a pure function of g,
    so any rank can produce any tile.  Each rank encodes its round-robin
    candidates, the ranks all-gather their coded sizes (a few kilobytes,
    before any timing), every rank computes the same balanced shards and
    encodes the few tiles moved to it.  Returns (indices, tiles, summary)
    with the global loads in the summary.  dist None means one rank."""
    world = dist.get_world_size() if dist else 1
    rank = dist.get_rank() if dist else 0
    mine = round_robin(n_total, world, rank)
    tiles = dict(zip(mine, encode(mine)))
    local = [(g, len(tiles[g].codestream), tiles[g].width * tiles[g].height) for g in mine]
    if dist:
        gathered: list = [None] * world
        dist.all_gather_object(gathered, local)
    else:
        gathered = [local]
    sizes = [0] * n_total
    pixels = [0] * n_total
    for part in gathered:
        for g, s, p in part:
            sizes[g] = s
            pixels[g] = p
    shards = balance_by_coded_bytes(sizes, world)
    want = shards[rank]
    missing = [g for g in want if g not in tiles]
    if missing:
        tiles.update(zip(missing, encode(missing)))
    loads = [sum(sizes[g] for g in s) for s in shards]
    summary = {"tiles_total": n_total, "tiles_per_rank": [len(s) for s in shards],
               "coded_bytes_per_rank": loads, "pixels_total": sum(pixels),
               "moved_tiles": sum(1 for r, s in enumerate(shards) for g in s if g % world != r)}
    return want, [tiles[g] for g in want], summary
