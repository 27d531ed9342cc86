"""Data-parallel layout of the search over ranks (one process per GPU).

Particles are independent and the references are small and read-only, so every
rank holds all references and searches a contiguous block of particles; the only
exchange is the all-gather of the 16-byte per-particle results
(pftcc_best: iref, irot, ishift, corr).  For a queue of uneven chunks (several
geometries) chunks are assigned whole, longest-processing-time first, with the
cost of a chunk taken as nptcls * nrefs * nshifts * nrots * nshells.
"""
from __future__ import annotations

import heapq

import numpy as np
import torch
import torch.distributed as dist


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """contiguous balanced block [lo, hi) of n items for rank of world"""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def chunk_cost(nptcls: int, nrefs: int, nshifts: int, nrots: int, nshells: int) -> float:
    return float(nptcls) * nrefs * nshifts * nrots * nshells


def assign_chunks(costs, world: int) -> list[list[int]]:
    """longest-processing-time-first assignment of whole chunks to ranks"""
    heap = [(0.0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda i: -costs[i]):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    for lst in out:
        lst.sort()
    return out


def gather_results(best_local: torch.Tensor, n_total: int, world: int, group=None) -> torch.Tensor:
    """all-gather of each rank's (n_local, 4) int32 result records into the (n_total, 4)
    array in particle order (rank r holds shard_range(n_total, r, world))"""
    if world == 1:
        return best_local
    sizes = [shard_range(n_total, r, world) for r in range(world)]
    width = max(hi - lo for lo, hi in sizes)
    buf = torch.zeros((width, 4), dtype=torch.int32, device=best_local.device)
    buf[: best_local.shape[0]] = best_local
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return torch.cat([parts[r][: hi - lo] for r, (lo, hi) in enumerate(sizes)])


def as_records(iref, irot, ishift, corr) -> np.ndarray:
    """pack per-particle results into the 16-byte int32 records gathered across ranks"""
    rec = np.zeros((len(iref), 4), np.int32)
    rec[:, 0], rec[:, 1], rec[:, 2] = iref, irot, ishift
    rec[:, 3] = np.asarray(corr, np.float32).view(np.int32)
    return rec
