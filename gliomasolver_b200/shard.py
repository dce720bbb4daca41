"""The path across ranks: one process per GPU, no data-path collective.

A single solve does not shard (a 256^3 FP32 pool is 270 MB), so N GPUs run N
independent replicas of the step.  What does shard is a TMCMC stage: its
samples are independent forward solves (the reference hands them to its task
engine one by one, tools/pi4u_lite/Inference/engine_tmcmc.c:597-624), so each
rank runs a ``tmcmc.Batch`` over its own share.  The only collectives are the
host-side bookkeeping below: the max over ranks of a device-timed duration and
the gather of per-sample results to rank 0.
"""
from __future__ import annotations

import heapq

import torch
import torch.distributed as dist


def stage_shards(nsteps, world: int):
    """Samples of a stage per rank, balanced by time steps: longest
    processing time first, each sample to the rank with the fewest steps so
    far (ties to the lower rank).  Deterministic; every rank computes the
    same assignment.  Returns ``world`` lists of sample indices, each sorted."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(nsteps)), key=lambda i: (-int(nsteps[i]), i))
    heap = [(0, r) for r in range(world)]
    shards = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + int(nsteps[i]), r))
    return [sorted(s) for s in shards]


def _device():
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(value: float) -> float:
    """The largest of every rank's ``value`` (a duration): all ranks call it
    in the same order.  Without an initialised process group it is ``value``."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_results(local: dict):
    """Per-sample results ``{sample index: value}`` of every rank merged on
    rank 0 (None on the other ranks).  A sample reported by two ranks is an
    error."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return dict(local)
    parts = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(dict(local), parts, dst=0)
    if dist.get_rank() != 0:
        return None
    merged = {}
    for part in parts:
        for k, v in part.items():
            if k in merged:
                raise RuntimeError(f"sample {k} reported by two ranks")
            merged[k] = v
    return merged
