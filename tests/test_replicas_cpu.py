"""Runs on several ranks, on CPU with the gloo backend (world size 2).

bench.py --gpus N runs one process per GPU as independent replicas: each rank
builds the same plan from the same SPR structure, times its own factor+solve,
and the job time is the maximum over ranks.  Many independent systems shard
round robin.  This test runs that bookkeeping on two gloo ranks: identical
plans on both ranks, the max-over-ranks reduction, the sharding (every
system exactly once) and the whole-job rate.
"""
import os
import socket
import tempfile

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, outdir):
    import datetime
    import json
    import torch.distributed as dist
    import sam_lib_b200 as spr
    from sam_lib_b200.replicas import max_over_ranks, shard, whole_job_rate
    from sam_lib_b200.system import load_structure
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        st = load_structure(6)
        out = np.zeros(13)
        rc = spr.load(8).spr_b200_plan_check(spr._ptr(st['mspar']), spr._ptr(st['mtrees']),
                                             spr._ptr(st['msifa']), spr._ptr(out))
        plans = [None] * world
        dist.all_gather_object(plans, out.tolist())
        t = max_over_ranks(1.0 + 0.5 * rank, dist)
        owned = shard(10, rank, world)
        owners = [None] * world
        dist.all_gather_object(owners, owned)
        rate = whole_job_rate(3.0, world, t)
        with open(os.path.join(outdir, 'rank%d.json' % rank), 'w') as f:
            json.dump(dict(rc=rc, plans=plans, t=t, owners=owners, rate=rate), f)
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_replica_bookkeeping():
    import json
    import torch.multiprocessing as mp
    world = 2
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(world, _free_port(), d), nprocs=world, join=True,
                           start_method='spawn')
        res = [json.load(open(os.path.join(d, 'rank%d.json' % r))) for r in range(world)]
    for r in res:
        assert r['rc'] == 0
        assert r['plans'][0] == r['plans'][1]            # the same plan on every rank
        assert r['plans'][0][0] == 0.0                    # build_plan status
        assert r['t'] == 1.5                              # the slowest rank's time
        assert r['rate'] == pytest.approx(2 * 3.0 / 1.5)
        flat = sorted(i for o in r['owners'] for i in o)
        assert flat == list(range(10))                    # every system exactly once
        assert set(r['owners'][0]).isdisjoint(r['owners'][1])


def test_shard_and_rate_edges():
    from sam_lib_b200.replicas import shard, whole_job_rate, max_over_ranks
    assert shard(3, 0, 4) == [0] and shard(3, 3, 4) == []
    with pytest.raises(ValueError):
        shard(3, 4, 4)
    with pytest.raises(ValueError):
        whole_job_rate(1.0, 1, 0.0)
    assert max_over_ranks(2.5) == 2.5
