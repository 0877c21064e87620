"""Multi-GPU runs as independent replicas (one process per GPU).

A batch of independent simulations has no cross-simulation coupling, so
several GPUs split the simulations between them; no collective touches the
particle data.  This module holds the host-side logic: the assignment of
simulations to ranks (balancing particles x steps), per-rank seeds, and the
max-over-ranks reduction of device timings.  It works with any
``torch.distributed`` backend (NCCL between GPUs, gloo on the CPU).
"""
import heapq

import torch

__all__ = ['assign', 'replica_seed', 'max_over_ranks', 'gather_counts']


def assign(costs, world):
  """Split simulations with per-simulation ``costs`` (e.g. particles x
  steps) between ``world`` ranks: longest-processing-time first, each to the
  currently least loaded rank.  Returns, per rank, the sorted list of
  simulation indices; deterministic, so every rank computes the same
  answer without communicating."""
  if world < 1:
    raise ValueError('world must be >= 1')
  order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
  heap = [(0.0, r) for r in range(world)]
  heapq.heapify(heap)
  parts = [[] for _ in range(world)]
  for i in order:
    load, r = heapq.heappop(heap)
    parts[r].append(i)
    heapq.heappush(heap, (load + float(costs[i]), r))
  return [sorted(p) for p in parts]


def replica_seed(base, rank):
  """Seed of rank ``rank``'s replica: distinct per rank, reproducible."""
  return int(base) * 1000003 + int(rank)


def max_over_ranks(value, group=None, device=None):
  """Max of a float over all ranks (identity without a process group)."""
  import torch.distributed as dist
  if not dist.is_available() or not dist.is_initialized():
    return float(value)
  t = torch.tensor([float(value)], dtype=torch.float64, device=device)
  dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
  return float(t.item())


def gather_counts(count, group=None, device=None):
  """Sum of an integer over all ranks (e.g. particle-updates done)."""
  import torch.distributed as dist
  if not dist.is_available() or not dist.is_initialized():
    return int(count)
  t = torch.tensor([int(count)], dtype=torch.int64, device=device)
  dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
  return int(t.item())
