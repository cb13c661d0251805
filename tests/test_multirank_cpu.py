"""The multi-GPU path of bench.py on CPU: two gloo ranks, each with its own shard of columns
(different seeds), no collective on the data path, the device time reduced as the max over ranks
and the whole-job throughput computed from it."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path[:0] = [REPO, os.path.join(REPO, "oracle"), os.path.join(REPO, "hpc-and-climate-model_b200")]
    import datetime
    import torch.distributed as dist
    import bench
    import oracle
    import soundings
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        s = soundings.make_soundings(64, 30, seed=bench.shard_seed(rank), rh_pbl=bench.RH_PBL)
        oracle.init_default()
        out = oracle.compute(s, diag=False, nthreads=1)
        local_ms = 10.0 + 5.0 * rank          # stands in for this rank's device time
        ms = bench.max_over_ranks(dist, local_ms, "cpu")
        q.put((rank, float(np.sum(out["precip"])), float(s["ps0"][0, 0]), ms,
               bench.job_throughput(world, 64, ms * 1e-3)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, prec0, ps0, ms0, v0), (r1, prec1, ps1, ms1, v1) = res
    assert (r0, r1) == (0, 1)
    assert ps0 != ps1                       # different shards
    assert ms0 == ms1 == 15.0               # max over ranks, the same on every rank
    assert v0 == v1 == 2 * 64 / 15e-3       # whole-job columns/s
