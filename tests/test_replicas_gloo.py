"""The N > 1 path on CPU: two gloo ranks run independent replicas (the oracle step on a small
shell, each with its own seed) and reduce their times with the max, as bench.py does over NCCL."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import time
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    from aturan_b200 import params as P, replicas, state as S
    from oracle import Oracle
    p = P.default_params(9, 13, 17)
    st = S.synthetic_state(p, seed=replicas.replica_seed(100, rank))
    t0 = time.perf_counter()
    Oracle().step(p, st, P.PRESS_GS_LEX)
    local = time.perf_counter() - t0
    mx = replicas.max_over_ranks(local, dist)
    out[rank] = (local, mx, float(np.abs(st["t"]).sum()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas_reduce_max_time():
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    (l0, m0, s0), (l1, m1, s1) = out[0], out[1]
    assert m0 == m1 == max(l0, l1)
    assert s0 != s1                      # independent replicas: different seeded states

    # each replica equals a single-process run with its seed
    from aturan_b200 import params as P, replicas, state as S
    from oracle import Oracle
    p = P.default_params(9, 13, 17)
    st = S.synthetic_state(p, seed=replicas.replica_seed(100, 1))
    Oracle().step(p, st, P.PRESS_GS_LEX)
    assert float(np.abs(st["t"]).sum()) == s1


def test_throughput_is_whole_job():
    from aturan_b200 import replicas
    assert replicas.throughput(100, 10, 4, 2.0) == 2000.0
