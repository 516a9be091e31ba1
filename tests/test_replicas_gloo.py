"""The N-GPU path of bench.py is replicas only: each rank advances its own
seeded run and the whole-job rate is all ranks' steps over the slowest rank's
device time.  This covers that aggregation and the per-rank workloads with two
gloo ranks on the CPU (no GPU, no NCCL)."""
import datetime
import os
import socket

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    import bench
    value, ms_max = bench.aggregate(10, 100.0 + 50.0 * rank, ws, device="cpu")
    _, phi, _ = bench.workload(rank)
    q.put((rank, value, ms_max, float(np.sum(phi[0, ::64, ::64]))))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_aggregation_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every rank reports the same whole-job value: 2 x 10 steps over the slower rank's 150 ms
    for _, value, ms_max, _ in res:
        assert ms_max == 150.0
        assert abs(value - 2 * 10 / 0.150) < 1e-9
    # the ranks advance different seeded runs
    assert res[0][3] != res[1][3]
