"""The N > 1 path of bench.py: independent replicas, max-over-ranks timing, the job
throughput sum, run as two gloo ranks on the CPU (127.0.0.1)."""
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


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from lsbflow_b200 import replicas
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, w, _ = replicas.rank_info()
        elapsed = 1.0 + r  # rank 1 is the slow one
        m = replicas.max_over_ranks(elapsed, w)
        dist.barrier()
        out[r] = (m, replicas.job_throughput(1000, 10, w, m), replicas.replica_seed(1000, r))
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas():
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    assert out[0][0] == out[1][0] == 2.0            # max over ranks
    assert out[0][1] == 1000 * 10 * 2 / 2.0          # both runs count
    assert out[0][2] != out[1][2]                    # independent seeds
