"""The replica path (bench.py --gpus N under torchrun) on CPU: two gloo ranks.
Each rank stands for one GPU running its own instance; the harness must line
the ranks up, take the slowest rank's time and count the work of all ranks,
and independent replicas must get independent inputs."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      LOCAL_RANK=str(rank), WORLD_SIZE=str(world))
    from bfps_b200 import ic, replicas
    w, r, local, pg = replicas.setup("gloo", timeout_s=60)
    assert (w, r, local) == (world, rank, rank)
    replicas.barrier(pg)
    # a rank's "device time" for K steps; the slowest rank sets the job time
    ms = 10.0 + 5.0 * rank
    ms_max = replicas.allmax(pg, ms)
    rate = replicas.whole_job_rate(w, 20, ms_max / 1e3)
    # replicas draw their inputs from their own seeds (bench.py make_inputs)
    field = ic.vorticity_ic(8, seed=r)
    out[rank] = (ms_max, rate, float(np.abs(field).sum()))
    replicas.barrier(pg)
    replicas.teardown(pg)


def test_two_gloo_replicas():
    world = 2
    mgr = mp.get_context("spawn").Manager()  # no fork of this multi-threaded process
    out = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    (m0, r0, f0), (m1, r1, f1) = out[0], out[1]
    assert m0 == m1 == 15.0                      # max over ranks, on every rank
    assert r0 == r1 == pytest.approx(2 * 20 / 0.015)  # work of all ranks / slowest time
    assert f0 != f1                              # independent inputs


def test_single_process_needs_no_group():
    from bfps_b200 import replicas
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    w, r, local, pg = replicas.setup()
    assert (w, r, local, pg) == (1, 0, 0, None)
    assert replicas.allmax(pg, 3.5) == 3.5
    replicas.barrier(pg)
