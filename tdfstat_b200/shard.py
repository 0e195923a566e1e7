"""Sharding of a search over several GPUs (one process per GPU).

Sky points are independent (jobcore.c:105-156: each job_core() call reads
only the segment inputs and writes its own records), so a run splits its
point list into contiguous shards, one per rank, with no data exchange.
Concatenating the ranks' records in rank order reproduces the
single-process record order (pm -> mm -> nn -> ss, jobcore.c:88-111).
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np


def shard_range(n: int, rank: int, world: int) -> Tuple[int, int]:
    """[a, b) of the n points that rank `rank` of `world` processes."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("rank %d of world %d" % (rank, world))
    return rank * n // world, (rank + 1) * n // world


def shard_points(pm: Sequence[int], mm: Sequence[float], nn: Sequence[float], rank: int, world: int):
    a, b = shard_range(len(pm), rank, world)
    return (np.asarray(pm, np.int32)[a:b], np.asarray(mm, np.float32)[a:b], np.asarray(nn, np.float32)[a:b])


def balanced_ranges(costs: Sequence[float], world: int) -> List[Tuple[int, int]]:
    """Contiguous ranges with about equal total cost (e.g. spindowns per
    sky point in an all-sky run, where the count varies with the point)."""
    c = np.cumsum(np.asarray(costs, dtype=np.float64))
    total = c[-1] if len(c) else 0.0
    out, a = [], 0
    for r in range(world):
        target = total * (r + 1) / world
        if r == world - 1:
            b = len(costs)
        else:
            # cut after the point whose prefix cost is closest to the target
            j = int(np.searchsorted(c, target, side="left"))
            cands = [k for k in (j, j + 1) if a <= k <= len(costs)]
            b = min(cands, key=lambda k: abs((c[k - 1] if k else 0.0) - target)) if cands else a
        b = max(b, a)
        out.append((a, b))
        a = b
    return out


def segment_cost(templates: int, nfftf: int, nifo: int, N: int) -> float:
    """Estimated device time of one segment's search: per template two FFTs
    of nfftf (5 nfftf log2 nfftf flops each) and the demodulation of nifo*N
    samples (about 40 flops each)."""
    return float(templates) * (10.0 * nfftf * np.log2(nfftf) + 40.0 * nifo * N)


def assign_segments(costs: Sequence[float], world: int) -> List[List[int]]:
    """Whole segments to ranks (the reference runs one segment per process,
    so a segment's records never need merging): longest first, each to the
    rank with the least cost so far (ties: the lower rank); every rank's
    list in segment order.  The most loaded rank carries at most
    4/3 of the optimum (Graham's bound for this rule)."""
    if world < 1:
        raise ValueError("world %d" % world)
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for k in sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(k)
        load[r] += float(costs[k])
    return [sorted(x) for x in out]


def merge_records(parts):
    """Concatenates per-rank (hdr, lens, pairs_flat) in rank order; returns
    the same triple for the whole run."""
    hdrs = [p[0] for p in parts]
    lens = [p[1] for p in parts]
    flats = [p[2] for p in parts]
    return (np.concatenate(hdrs) if hdrs else np.zeros((0, 6), np.float32),
            np.concatenate(lens) if lens else np.zeros(0, np.int64),
            np.concatenate(flats) if flats else np.zeros(0, np.float32))
