"""Walkers over ranks: one process per GPU, independent walkers, no data-path collective.

Saddle searches and relaxations of different walkers never exchange data, so the walker
set is split across ranks and each rank runs its share on its own GPU.  The only exchange
is after the searches: every rank contributes fixed-size per-walker records (status,
saddle energy, barrier, walker id, force calls) and rank 0 receives all of them -- the
step the reference's KMC master does by receiving each worker's events
(kmc/KineticMonteCarlo.cpp:352-464) -- with the device time of the searches taken as the
maximum over ranks.

Works with any torch.distributed backend: NCCL between GPUs, gloo on the host (tests).
"""
from __future__ import annotations

import numpy as np

RECORD_FIELDS = ("walker", "status", "energy", "barrier", "force_calls")


def shard_indices(n_walkers: int, rank: int, world: int) -> np.ndarray:
    """Walkers of this rank: a contiguous block, sizes differing by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n_walkers, world)
    start = rank * base + min(rank, extra)
    return np.arange(start, start + base + (1 if rank < extra else 0), dtype=np.int64)


def records(walker_ids, results, e_min) -> np.ndarray:
    """(n, 5) float64 records of this rank's walkers: id, status, E_saddle, barrier, calls."""
    ids = np.asarray(walker_ids, dtype=np.float64)
    out = np.zeros((len(ids), len(RECORD_FIELDS)), dtype=np.float64)
    out[:, 0] = ids
    out[:, 1] = results["status"]
    out[:, 2] = results["energy"]
    out[:, 3] = results["energy"] - np.asarray(e_min, dtype=np.float64)
    out[:, 4] = results["force_calls"]
    return out


def _device(device):
    """The device of a collective's tensors: the caller's, else the current CUDA device under
    NCCL (which takes CUDA tensors only) and the host otherwise."""
    import torch
    import torch.distributed as dist
    if device is not None:
        return device
    if dist.is_available() and dist.is_initialized() and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def gather_records(local: np.ndarray, n_walkers: int, device=None):
    """Every rank's records on rank 0, ordered by walker id (None on other ranks).  One
    fixed-size all-gather: each rank pads its block to the largest shard."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size()
    device = _device(device)
    width = len(RECORD_FIELDS)
    cap = -(-n_walkers // world)
    buf = torch.full((cap, width), -1.0, dtype=torch.float64, device=device)
    buf[: len(local)] = torch.as_tensor(local, dtype=torch.float64, device=device)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    if dist.get_rank() != 0:
        return None
    allr = torch.cat(parts).cpu().numpy()
    allr = allr[allr[:, 0] >= 0]
    return allr[np.argsort(allr[:, 0], kind="stable")]


def max_over_ranks(seconds: float, device=None) -> float:
    """The job's time: the slowest rank's."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([seconds], dtype=torch.float64, device=_device(device))
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, device=None):
    """The sum of a count over ranks (the value itself on one rank)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device(device))
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
