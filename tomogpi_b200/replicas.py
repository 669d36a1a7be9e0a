"""Multi-GPU form: whole reconstructions as replicas, one process per GPU.

Every workload of this path fits one B200 with room to spare, so N GPUs run N independent
job streams with no data-path collective (weak scaling). The operators themselves would
shard without a collective as well -- projection by detector rows, backprojection by
z-slabs (RegularSamplingProjector_compute_CUDA_mem_CPU.cu:243-278,
VIBackProjector_compute_CUDA_mem_CPU.cu:214-245) -- but nothing here needs that.

Host logic only: rank set-up from the torchrun environment, a deterministic assignment of
jobs to ranks (longest processing time first), device time as the maximum over ranks, and
rank 0 collecting the served results. The collectives are torch.distributed calls, so the
same code runs over NCCL on GPUs and over gloo on CPU (the tests).
"""
from __future__ import annotations

import heapq
import os
from typing import Callable, List, Sequence, Tuple


def dist_env() -> Tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment (1, 0, 0 without it)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def assign_jobs(works: Sequence[float], world: int) -> List[List[int]]:
    """Job indices per rank: longest job first onto the least-loaded rank (ties to the lower
    rank), so that every rank computes the same assignment without communicating."""
    if world < 1:
        raise ValueError("world size must be positive")
    heap = [(0.0, r) for r in range(world)]
    out: List[List[int]] = [[] for _ in range(world)]
    for j in sorted(range(len(works)), key=lambda j: (-float(works[j]), j)):
        load, r = heapq.heappop(heap)
        out[r].append(j)
        heapq.heappush(heap, (load + float(works[j]), r))
    for lst in out:
        lst.sort()
    return out


def max_over_ranks(value: float, device=None) -> float:
    """The largest value over all ranks (device times are reported this way); the value
    itself without an initialised process group."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def serve_replicated(requests: Sequence, work: Callable[[object], float], serve: Callable[[list], list]):
    """Serves `requests` over all ranks: each rank runs `serve` (e.g. a ``serve.Server``'s
    ``run``) on the requests assigned to it by their `work`; rank 0 returns every rank's
    results (in request order of the ranks' lists), the other ranks None."""
    import torch.distributed as dist

    multi = dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1
    world = dist.get_world_size() if multi else 1
    rank = dist.get_rank() if multi else 0
    mine = [requests[j] for j in assign_jobs([work(r) for r in requests], world)[rank]]
    results = serve(mine)
    if not multi:
        return list(results)
    gathered = [None] * world
    dist.all_gather_object(gathered, list(results))
    if rank != 0:
        return None
    return [r for part in gathered for r in part]
