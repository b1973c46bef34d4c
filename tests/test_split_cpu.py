"""One system split across ranks (CPU parts).

* The subtree partition of the benchmark structures: every supernode owned
  once, subtrees contiguous in postorder with their parents inside them
  except the root's (a top node), top nodes' parents in the top; with one
  rank nothing is split.  The top's share of RINFO(3) bounds the speed-up
  (the separators near the root carry most of the work).
* The exchange protocol of SplitSolver on two and three gloo ranks on CPU,
  with a stand-in for the engine that writes rank-tagged values: every
  subtree-root block and update vector reaches rank 0 before its top phase,
  every rank's D/LNZ ranges land in rank 0's SM, the top equations' solution
  reaches every rank before its back sweep, every rank's solution ranges
  land in rank 0's B, and the combined outcome counts each supernode's
  negative pivots once and finds the first failing supernode in postorder.
"""
import os
import socket
import tempfile

import numpy as np
import pytest

from sam_lib_b200.split import tree, partition, check_partition, combine


@pytest.mark.parametrize('n', [12, 24, 48])
def test_partition_of_the_benchmark_structures(n):
    from sam_lib_b200.system import load_structure
    st = load_structure(n)
    t = tree(st['mspar'], st['mtrees'], st['msifa'])
    assert abs(t['flops'].sum() - st['rinfo'][2]) <= 1e-9 * st['rinfo'][2]      # RINFO(3)
    for world in (1, 2, 3, 4, 8):
        p = partition(t, world)
        assert check_partition(t, p) == 0
        assert sorted(set(p['owner'].tolist())) == list(range(min(world, len(set(p['owner'].tolist())))))
        if world == 1:
            assert p['top'] == [] and np.all(p['owner'] == 0)
        else:
            loads = p['load'][1:]
            assert loads.min() > 0.0
            assert abs(p['load'].sum() - t['flops'].sum()) <= 1e-9 * t['flops'].sum()


def test_combine_first_failure_in_postorder():
    t = dict(ns=6, fst=np.array([0, 3, 6, 9, 12, 15]))
    def rec(mask, neg, fail, tol2=0.5, lierr=0):
        return dict(mask=np.array(mask, bool), neg=np.array(neg), fail=np.array(fail), trace=10.0,
                    res=dict(lierr=lierr, numneg=int(np.sum(neg)), supeqt=0, tol2=tol2, tol3=1.0))
    a = rec([1, 1, 0, 0, 0, 0], [1, 0, 0, 0, 0, 0], [-1, -1, -1, -1, -1, -1], tol2=0.5)
    b = rec([0, 0, 1, 1, 0, 0], [0, 0, 2, 0, 0, 0], [-1, -1, -1, 1, -1, -1], tol2=-1e-14, lierr=-30)
    top = rec([0, 0, 0, 0, 1, 1], [0, 0, 0, 0, 3, 0], [-1] * 6, tol2=0.25)
    out = combine(t, top, [a, b], 2.0)
    assert out['lierr'] == -30 and out['supeqt'] == 9 + 1 + 1 and out['numneg'] == 3
    b2 = rec([0, 0, 1, 1, 0, 0], [0, 0, 2, 0, 0, 0], [-1] * 6, tol2=0.4)
    out = combine(t, top, [a, b2], 2.0)
    assert out['lierr'] == 0 and out['numneg'] == 6 and out['tol3'] == 5.0
    assert out['tol2'] == pytest.approx(0.25)


class _Stand:
    """SplitRank's interface with rank-tagged values instead of the engine."""

    def __init__(self, t, part, rank, world, neq):
        import torch
        self.t, self.part, self.rank, self.world, self.neq = t, part, rank, world, neq
        ns = t['ns']
        self.is_top = np.zeros(ns, dtype=bool)
        self.is_top[part['top']] = True
        self.own = (part['owner'] == rank) & ~self.is_top
        self.links = [(r, k) for (r, k, f0) in part['roots'] if t['parent'][r] >= 0]
        self.own_ranges = []
        for (r, k, f0) in part['roots']:
            if k == rank:
                self.own_ranges.append((int(t['fst'][f0]), int(t['fst'][r] + t['S'][r]), int(t['lnz_off'][f0]),
                                        int(t['lnz_off'][r] + t['lnz_len'][r])))
        keep = [r for (r, k) in self.links if k == rank or rank == 0]
        self.blocks = {r: torch.zeros(5) for r in keep}
        self.vecs = {r: torch.zeros(3) for r in keep}
        self.seen = []

    def _rec(self, mask):
        ns = self.t['ns']
        neg = np.where(mask, 1, 0).astype(np.int32)
        return dict(res=dict(lierr=0, numneg=int(neg.sum()), supeqt=0, tol2=0.5, tol3=1.0), trace=3.0,
                    neg=neg, fail=-np.ones(ns, dtype=np.int32))

    def factor_subtrees(self, d_sm, tol1=1e-12):
        for e0, e1, l0, l1 in self.own_ranges:
            d_sm[e0:e1] = self.rank + 1
            d_sm[self.neq + l0: self.neq + l1] = self.rank + 1
        for (r, k) in self.links:
            if k == self.rank:
                self.blocks[r].fill_(r + 0.5)
        return self._rec(self.own)

    def factor_top(self, d_sm, tol1=1e-12):
        for (r, k) in self.links:
            assert float(self.blocks[r][0]) == r + 0.5, ('block', r)
        return self._rec(self.is_top)

    def forward_subtrees(self, d_sm, d_b, nrhs):
        for (r, k) in self.links:
            if k == self.rank:
                self.vecs[r].fill_(r + 0.25)

    def forward_top(self, d_sm, d_b, nrhs):
        for (r, k) in self.links:
            assert float(self.vecs[r][0]) == r + 0.25, ('vector', r)

    def back_top(self, d_sm, d_b, nrhs):
        top_eq = np.concatenate([np.arange(self.t['fst'][j], self.t['fst'][j] + self.t['S'][j]) for j in self.part['top']])
        d_b[:, top_eq] = 7.0

    def back_subtrees(self, d_sm, d_b, nrhs):
        top_eq = np.concatenate([np.arange(self.t['fst'][j], self.t['fst'][j] + self.t['S'][j]) for j in self.part['top']])
        assert bool((d_b[:, top_eq] == 7.0).all())
        for e0, e1, _, _ in self.own_ranges:
            d_b[:, e0:e1] = self.rank + 10

    def close(self):
        pass


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, outdir):
    import datetime
    import json
    import torch
    import torch.distributed as dist
    from sam_lib_b200.system import load_structure
    from sam_lib_b200.split import SplitSolver
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        st = load_structure(12)
        ms, mt, mf = st['mspar'], st['mtrees'], st['msifa']
        t = tree(ms, mt, mf)
        part = partition(t, world)
        neq = int(ms[7])
        stand = _Stand(t, part, rank, world, neq)
        sv = SplitSolver(ms, mt, mf, dist, rank_impl=stand)
        d_sm = torch.zeros(neq + int(ms[15]), dtype=torch.float64)
        out = sv.factor(d_sm)
        d_b = torch.zeros((2, neq), dtype=torch.float64)
        sv.solve(d_sm, d_b, 2)
        res = dict(out=out)
        if rank == 0:
            owner_sm = np.zeros(neq, dtype=np.int64)
            owner_b = np.zeros(neq)
            for (r, k, f0) in part['roots']:
                e0, e1 = int(t['fst'][f0]), int(t['fst'][r] + t['S'][r])
                owner_sm[e0:e1] = k + 1
                owner_b[e0:e1] = k + 10
            for j in part['top']:
                owner_b[t['fst'][j]: t['fst'][j] + t['S'][j]] = 7.0
            res['sm_ok'] = bool(np.array_equal(d_sm[:neq].numpy()[owner_sm > 0], owner_sm[owner_sm > 0]))
            res['b_ok'] = bool(np.array_equal(d_b[0].numpy(), owner_b) and np.array_equal(d_b[1].numpy(), owner_b))
            res['numneg_expected'] = int(t['ns'])
        with open(os.path.join(outdir, 'rank%d.json' % rank), 'w') as f:
            json.dump(res, f)
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.parametrize('world', [2, 3])
def test_split_protocol_on_gloo_ranks(world):
    import json
    import torch.multiprocessing as mp
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(world, _free_port(), d), nprocs=world, join=True,
                           start_method='spawn')
        res = [json.load(open(os.path.join(d, 'rank%d.json' % r))) for r in range(world)]
    r0 = res[0]
    assert r0['sm_ok'] and r0['b_ok']
    for r in res:
        assert r['out'] == r0['out']                      # every rank gets the same outcome
    assert r0['out']['lierr'] == 0 and r0['out']['numneg'] == r0['numneg_expected']
