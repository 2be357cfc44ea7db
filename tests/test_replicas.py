"""The multi-GPU form of the benchmark is replicas of independent ensembles (no data-path
collective): every rank steps its own peaks and the job's rate is the particles of all ranks
over the slowest rank's time.  This runs the aggregation on two gloo ranks on the CPU, and
checks that ranks draw different peaks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    t_local = [0.5, 0.8][rank]                 # rank 1 is the slow one
    t, value = bench.replica_throughput(t_local, 1000, 10, dist)
    specs, _ = bench.workload_specs("batched", 8, 1234, rank)
    out[rank] = (t, value, [s.seed for s in specs])
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_take_the_slowest_rank_and_distinct_peaks():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    for r in (0, 1):
        t, value, _ = res[r]
        assert t == pytest.approx(0.8)
        assert value == pytest.approx(2 * 1000 * 10 / 0.8)
    assert set(res[0][2]).isdisjoint(res[1][2])
