"""Multi-rank host logic of bench.py, run as two gloo ranks on the CPU.

The GPU path shards ensemble members / field batches across ranks as
independent replicas; the only cross-rank step is the max-over-ranks timing
reduction, tested here without a GPU.
"""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
  with socket.socket() as s:
    s.bind(('127.0.0.1', 0))
    return s.getsockname()[1]


def _worker(rank, world, port, out):
  import bench
  os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
  dist.init_process_group('gloo', rank=rank, world_size=world)
  try:
    ms_local = 10.0 + 5.0 * rank
    ms_max = bench.max_over_ranks(ms_local)
    tflops = bench.aggregate_tflops(1e12, world, ms_max)
    seeds = [None] * world
    dist.all_gather_object(seeds, bench.replica_seed(rank))
    out[rank] = (ms_max, tflops, tuple(seeds))
  finally:
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_max_time():
  port = _free_port()
  manager = mp.get_context('spawn').Manager()
  out = manager.dict()
  mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True,
                     start_method='spawn')
  assert out[0][0] == out[1][0] == 15.0
  assert out[0][1] == pytest.approx(2 * 1e12 / 15e-3 / 1e12)
  assert len(set(out[0][2])) == 2  # distinct replica seeds


def test_single_process_passthrough():
  import bench
  assert not dist.is_initialized()
  assert bench.max_over_ranks(3.5) == 3.5
