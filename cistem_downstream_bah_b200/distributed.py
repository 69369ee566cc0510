"""One process per GPU for the match_template search: the rank plumbing and the
one exchange step the search has.

The reference distributes a search by splitting the Euler-sphere search
positions of one image into jobs (src/gui/MatchTemplatePanel.cpp:674-784);
each worker job searches its range and sends one flat result array to the
master, which merges them (AggregatedTemplateResult::AddResult,
src/programs/match_template/match_template.cpp:2015-2103) and computes the
statistics.  Here a rank is a job: `rank_search_range` gives its positions,
and `gather_merge` is the exchange -- every rank's result array is gathered on
one rank in rank order and merged there as the master merges.  The search
itself has no data-path collective.  Backend "nccl" on GPUs (tensors staged
through the device), "gloo" on CPU.
"""
from __future__ import annotations

import os
from datetime import timedelta

import numpy as np

from . import hostprep as H


def init_from_env(backend: str | None = None, timeout_s: float = 600.0):
    """(world, rank, local_rank) from torchrun's environment; joins the process
    group when world > 1 (nccl with the local GPU selected, unless `backend`
    says otherwise)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        backend = backend or "nccl"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return world, rank, local


def _device():
    import torch
    import torch.distributed as dist
    return torch.device("cuda") if dist.get_backend() == "nccl" else torch.device("cpu")


def barrier(world: int) -> None:
    if world > 1:
        import torch
        import torch.distributed as dist
        dist.barrier()
        if _device().type == "cuda":
            torch.cuda.synchronize()


def max_over_ranks(world: int, v: float) -> float:
    if world <= 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(world: int, v: float) -> float:
    if world <= 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def rank_search_range(n_positions: int, rank: int, world: int) -> tuple[int, int]:
    """[first, last] search positions of this rank: job `rank` of `world` jobs
    as the reference's panel splits them."""
    return H.job_search_ranges(n_positions, world)[rank]


def gather_merge(result_array: np.ndarray, dst: int = 0, use_gpu: bool = True):
    """Gathers every rank's worker result array (pack_worker_result) on rank
    `dst`, in rank order, and merges them as the master does.  Returns the
    merge (hostprep.merge_results) on `dst` and None elsewhere.  All ranks
    take the same collective steps; arrays of different lengths raise
    ValueError on every rank before the gather."""
    import torch
    import torch.distributed as dist
    world, rank = dist.get_world_size(), dist.get_rank()
    dev = _device()
    a = np.ascontiguousarray(result_array, dtype=np.float32)
    n = torch.tensor([a.size], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n)
    if any(int(s.item()) != a.size for s in sizes):
        raise ValueError("result arrays of different lengths: " + str([int(s.item()) for s in sizes]))
    t = torch.from_numpy(a).to(dev)
    parts = [torch.empty_like(t) for _ in range(world)] if rank == dst else None
    dist.gather(t, parts, dst=dst)
    if rank != dst:
        return None
    return H.merge_results([p.cpu().numpy() for p in parts], use_gpu=use_gpu)
