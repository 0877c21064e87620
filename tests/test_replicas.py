"""Multi-rank replica logic on the CPU: two gloo ranks split the C3
simulation mix, agree on the split without communicating, reduce timings
to the max and work counts to the sum (the N > 1 path of bench.py)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from flowpm_b200 import replicas

C3 = [32**3 * s for s in (10, 12, 15, 20, 11, 18, 13, 16)] + \
     [64**3 * s for s in (14, 10, 20, 17, 12, 19, 11, 15)] + \
     [128**3 * s for s in (16, 10, 20, 13)]


def test_assign_partitions_and_balances():
  for world in (1, 2, 3, 4, 8):
    parts = replicas.assign(C3, world)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(C3)))
    loads = [sum(C3[i] for i in p) for p in parts]
    # LPT guarantee: max load <= 4/3 of the optimum (>= mean, >= max item)
    bound = max(sum(C3) / world, max(C3))
    assert max(loads) <= 4.0 / 3.0 * bound + 1
  assert replicas.assign([], 2) == [[], []]
  with pytest.raises(ValueError):
    replicas.assign(C3, 0)


def test_seeds_distinct():
  seeds = {replicas.replica_seed(7, r) for r in range(64)}
  assert len(seeds) == 64


def _free_port():
  with socket.socket() as s:
    s.bind(('127.0.0.1', 0))
    return s.getsockname()[1]


def _worker(rank, world, port, out):
  os.environ['MASTER_ADDR'] = '127.0.0.1'
  os.environ['MASTER_PORT'] = str(port)
  dist.init_process_group('gloo', rank=rank, world_size=world)
  try:
    parts = replicas.assign(C3, world)
    mine = parts[rank]
    work = sum(C3[i] for i in mine)
    total = replicas.gather_counts(work)
    t = replicas.max_over_ranks(1.0 + rank)
    # every rank computed the same split
    obj = [None] * world
    dist.all_gather_object(obj, parts)
    out.put((rank, total, t, all(o == parts for o in obj)))
  finally:
    dist.destroy_process_group()


def test_two_gloo_ranks():
  ctx = mp.get_context('spawn')
  q = ctx.Queue()
  port = _free_port()
  procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
  for p in procs:
    p.start()
  res = [q.get(timeout=120) for _ in procs]
  for p in procs:
    p.join(timeout=60)
    assert p.exitcode == 0
  for rank, total, t, same in res:
    assert total == sum(C3)
    assert t == 2.0
    assert same
