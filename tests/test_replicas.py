"""Multi-rank host logic of bench.py on CPU: world_size 2 over gloo.

Each rank steps its own replica (here the CPU oracle on a small scene, a
different jitter per rank), the ranks meet only at the barriers and the one
max-reduction of the time, and the whole-job value counts every replica.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    import time

    import numpy as np
    import torch.distributed as dist

    from oracle import Oracle
    from sources_b200 import replicas, scenes

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = scenes.jitter(scenes.small("granular_column"), 0.0002, seed=100 + rank)
        o = Oracle(s)
        replicas.barrier(dist)
        t0 = time.perf_counter()
        assert o.time_integration(3) == 0
        ms = (time.perf_counter() - t0) * 1000.0 + rank   # ranks differ on purpose
        replicas.barrier(dist)
        ms_max = replicas.max_over_ranks(ms, dist)
        value = replicas.weak_scaling_value(world, s.n_particles, 3, ms_max)
        x = o.download(1).x
        out[rank] = (ms, ms_max, value, float(np.abs(x).sum()), s.n_particles)
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_on_gloo():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    r0, r1 = out[0], out[1]
    assert r0[1] == r1[1] == max(r0[0], r1[0])          # same max on every rank
    assert r0[2] == r1[2]
    assert abs(r0[2] - world * r0[4] * 3 / (r0[1] / 1000.0)) < 1e-6 * r0[2]
    assert r0[3] != r1[3]                                # independent replicas


def test_single_rank_needs_no_process_group():
    from sources_b200 import replicas
    assert replicas.max_over_ranks(3.5, None) == 3.5
    assert replicas.weak_scaling_value(1, 1000, 10, 10.0) == 1000 * 10 / 0.01
