"""The multi-rank plumbing (opencaeporo_b200/shards.py) on CPU: two gloo
ranks, each flashing its own seeded shard through the plain-C oracle; the
timing reduction is the maximum over ranks and the shards are distinct."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    os.environ.update({"WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from oracle import oracle as O
    from opencaeporo_b200 import shards, synth
    from opencaeporo_b200.workload import SEED, bench_fluid
    assert shards.init("gloo", timeout_s=60) == world
    fl = bench_fluid()
    w = synth.uniform_states(fl, 256, shards.shard_seed(SEED, rank))
    r = O.flash_fim("port", fl, w["P"], w["T"], w["Ni"], nthreads=1)
    shards.barrier()
    mx = shards.max_over_ranks([r["seconds"], float(rank), -float(rank)])
    shards.finalize()
    q.put((rank, float(w["P"][0]), int((r["NPhc"] == 2).sum()), mx, r["seconds"]))


def test_two_ranks_max_over_ranks_and_distinct_shards():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, p0, n0, mx0, t0), (r1, p1, n1, mx1, t1) = res
    assert mx0 == mx1                      # every rank sees the same reduction
    assert mx0[0] == max(t0, t1)           # job time = slowest rank
    assert mx0[1] == 1.0 and mx0[2] == 0.0
    assert p0 != p1                        # independent shards
    assert 0 < n0 < 256 and 0 < n1 < 256
