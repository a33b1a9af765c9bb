"""The multi-GPU path is replicas only (the path does not shard): every rank
runs its own rollout, ranks meet only at barriers and in the max-over-ranks
timing reduction.  That host logic runs here on CPU as two gloo ranks."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = [120.0, 150.0][rank]  # rank 1 is the slow replica
        ms = bench.max_over_ranks(local_ms, dist, torch.device("cpu"))
        dist.barrier()
        out[rank] = (ms, bench.job_rate(world, 20, ms))
    finally:
        dist.destroy_process_group()


def test_replica_timing_is_max_over_two_gloo_ranks():
    world = 2
    out = mp.Manager().dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
    assert out[0][0] == out[1][0] == 150.0
    assert out[0][1] == pytest.approx(world * 20 / 0.150)


def test_single_rank_reduction_is_identity():
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.job_rate(1, 10, 500.0) == pytest.approx(20.0)


def test_algorithmic_bytes_model():
    # per-launch algorithmic bytes of the dealiased RHS kernels at 512^3 (compact extents)
    b = bench.kernel_alg_bytes(512)
    A, Bx, Cx = 341 * 341 * 171, 512 * 341 * 171, 512 * 512 * 171
    assert b["z-pass"] == 9 * Cx * 8
    assert b["y-inverse"] == (6 * Bx + 6 * Cx) * 8
    assert b["x-inverse"] == (3 * A + 6 * Bx) * 8
    assert bench.spectral_bytes(512) * 127 == 68448944128
