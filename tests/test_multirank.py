"""The multi-GPU form is replicas only: every rank runs its own seeded copy of the plain workload, the
batched replica set is split across the ranks by beads, and the reported rate is all ranks'
particle-steps over the slowest rank's time.  These tests run that host logic (the rank seeds, the
replica split, the max/sum reductions and the aggregate) on two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import conftest  # noqa: F401  (registers the package in spawned ranks too)
import bench
from protocell_genesis_b200 import config as cfgm


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    import datetime
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        w, r, _ = bench.dist_init()
        ms = 10.0 + 5.0 * r                      # the slower rank sets the time
        beads = 1000 * (r + 1)                   # batched replica sets differ between ranks
        ms_max = bench.max_over_ranks(ms, dist, "cpu")
        total = bench.sum_over_ranks(beads, dist, "cpu")
        plain_seed, batch_seed = bench.rank_seeds(r)
        cfg = cfgm.resolve(bench.workload_opts(cfgm, seed=plain_seed, scale=0.02))
        items = bench.batched_configs(cfgm, seed=batch_seed, replicas=16)
        share = bench.replica_share([int(c.n) for c, _, _ in items], w, r)
        mine = int(sum(int(items[i][0].n) for i in share))
        all_beads = bench.sum_over_ranks(mine, dist, "cpu")
        q.put((r, w, ms_max, total, bench.aggregate_rate(w, 500, 100, ms_max), plain_seed, batch_seed,
               int(cfg.seed), tuple(cfg.box), tuple(share), mine, all_beads, sum(int(c.n) for c, _, _ in items)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_time_and_units():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, (rr, w, ms_max, total, rate, ps, bs, seed, box, share, mine, all_beads, set_beads) in enumerate(out):
        assert rr == r and w == ws
        assert ms_max == 15.0                         # max over ranks
        assert total == 3000                          # sum over ranks
        assert rate == pytest.approx(2 * 500 * 100 / 0.015)
        assert all_beads == set_beads                 # the ranks' shares make up the one replica set
    assert out[0][5] != out[1][5]                     # plain replicas are seeded apart
    assert out[0][6] == out[1][6]                     # one batched replica set, split
    assert out[0][7] != out[1][7] and out[0][8] == out[1][8]   # same geometry, different seed
    assert not set(out[0][9]) & set(out[1][9]) and len(out[0][9]) + len(out[1][9]) == 16
    assert abs(out[0][10] - out[1][10]) < 0.1 * out[0][12]     # balanced by beads
