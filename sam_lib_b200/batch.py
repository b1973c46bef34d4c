"""Many independent SPR systems factored as one forest.

SPR supports a forest of elimination trees: SIBL(NSUPER+1) holds the number of
roots, and the roots occupy the last positions of SIBL (src/SPR/sprtrs.f:1592-
1597).  Independent systems therefore merge into a single SPR structure by
concatenation: equations, supernodes, row lists and LNZ blocks are shifted by
the running offsets, and each system's postorder stays a postorder of the
forest.  The GPU engine then factors every front of a tree level, of every
system, in one batched launch per kernel, and per-system inertia is read from
the per-supernode negative-pivot counts.
"""
import numpy as np


def _parts(mspar, mtrees, msifa):
    ns = int(mspar[10])
    xs = mtrees[mspar[44] - 1: mspar[44] - 1 + ns + 1]
    xsibl = mtrees[mspar[44] - 1 + ns + 1: mspar[44] - 1 + 2 * (ns + 1)]
    sibl = mtrees[mspar[44] - 1 + 2 * (ns + 1): mspar[44] - 1 + 3 * (ns + 1)]
    xl = mtrees[mspar[45] - 1: mspar[45] - 1 + ns + 1]
    lindx = msifa[mspar[46] - 1: mspar[46] - 1 + int(mspar[14])]
    xlnz = msifa[mspar[47] - 1: mspar[47] - 1 + ns + 1]
    return ns, xs, xsibl, sibl, xl, lindx, xlnz


class Forest:
    """Merged SPR structure of several systems (INTEGER*8 arrays)."""

    def __init__(self, structures):
        eq_off = sn_off = lnz_off = lx_off = 0
        xs_all, xl_all, lindx_all, xlnz_all, child_lists, roots = [], [], [], [], [], []
        self.eq_off, self.sn_off, self.lnz_off, self.neq_i, self.nzerol_i = [], [], [], [], []
        maxsup = mfront = 0
        for (mspar, mtrees, msifa) in structures:
            ns, xs, xsibl, sibl, xl, lindx, xlnz = _parts(mspar, mtrees, msifa)
            neq, nzerol = int(mspar[7]), int(mspar[15])
            self.eq_off.append(eq_off)
            self.sn_off.append(sn_off)
            self.lnz_off.append(lnz_off)
            self.neq_i.append(neq)
            self.nzerol_i.append(nzerol)
            xs_all.append(xs[:-1] + eq_off)
            xl_all.append(xl[:-1] + lx_off)
            lindx_all.append(lindx + eq_off)
            xlnz_all.append(xlnz[:-1] + lnz_off)
            has_parent = np.zeros(ns, dtype=bool)
            for js in range(ns):
                ch = sibl[xsibl[js] - 1: xsibl[js + 1] - 1]
                has_parent[ch - 1] = True
                child_lists.append(ch + sn_off)
            roots.extend((np.nonzero(~has_parent)[0] + 1 + sn_off).tolist())
            maxsup = max(maxsup, int(mspar[12]))
            mfront = max(mfront, int(mspar[13]))
            eq_off += neq
            sn_off += ns
            lnz_off += nzerol
            lx_off += int(mspar[14])
        self.nsys = len(structures)
        self.neq, self.nsuper, self.nzerol, self.nofsub = eq_off, sn_off, lnz_off, lx_off
        ns = self.nsuper
        xsuper = np.concatenate(xs_all + [[self.neq + 1]]).astype(np.int64)
        xsibl = np.empty(ns + 1, dtype=np.int64)
        pos = 1
        for js, ch in enumerate(child_lists):
            xsibl[js] = pos
            pos += len(ch)
        xsibl[ns] = pos
        sibl = np.concatenate(child_lists + [np.array(roots, dtype=np.int64),
                                             np.array([len(roots)], dtype=np.int64)]).astype(np.int64)
        assert len(sibl) == ns + 1
        xlindx = np.concatenate(xl_all + [[self.nofsub + 1]]).astype(np.int64)
        lindx = np.concatenate(lindx_all).astype(np.int64)
        xlnz = np.concatenate(xlnz_all + [[self.nzerol + 1]]).astype(np.int64)
        supsup = np.zeros(ns, dtype=np.int64)
        self.mtrees = np.concatenate([xsuper, xsibl, sibl, xlindx, supsup, [1, 0]]).astype(np.int64)
        self.msifa = np.concatenate([lindx, xlnz, np.ones(ns, dtype=np.int64), [0]]).astype(np.int64)
        m = np.zeros(60, dtype=np.int64)
        m[0] = 4
        m[2] = len(self.msifa)
        m[3] = len(self.mtrees)
        m[7] = self.neq
        m[10] = ns
        m[12] = maxsup
        m[13] = mfront
        m[14] = self.nofsub
        m[15] = self.nzerol
        m[16] = max(int(s[0][16]) for s in structures)
        m[44] = 1
        m[45] = 1 + 3 * (ns + 1)
        m[46] = 1
        m[47] = 1 + self.nofsub
        self.mspar = m

    def merge_sm(self, sms, out=None):
        """[D | LNZ] of the forest from each system's SM."""
        sm = np.empty(self.neq + self.nzerol) if out is None else out
        for i, s in enumerate(sms):
            neq = self.neq_i[i]
            sm[self.eq_off[i]: self.eq_off[i] + neq] = s[:neq]
            sm[self.neq + self.lnz_off[i]: self.neq + self.lnz_off[i] + self.nzerol_i[i]] = s[neq:]
        return sm

    def split_sm(self, sm):
        return [np.concatenate([sm[self.eq_off[i]: self.eq_off[i] + self.neq_i[i]],
                                sm[self.neq + self.lnz_off[i]:
                                   self.neq + self.lnz_off[i] + self.nzerol_i[i]]])
                for i in range(self.nsys)]

    def per_system(self, per_supernode):
        """Sums a per-supernode count (e.g. negative pivots) over each system."""
        bounds = self.sn_off + [self.nsuper]
        return np.array([int(np.sum(per_supernode[bounds[i]:bounds[i + 1]])) for i in range(self.nsys)])


class BatchSolver:
    """Factor + solve of many independent systems in one batched pass on the GPU.

    systems: list of dicts with 'hs' (a HexSystem-like object with mspar,
    mtrees, msifa, neq), 'sm' (assembled SM) and 'b' (NEQ x NRHS, column-major).
    """

    def __init__(self, systems):
        import torch
        from . import DeviceSolver
        self.systems = systems
        self.forest = Forest([(s['hs'].mspar, s['hs'].mtrees, s['hs'].msifa) for s in systems])
        self.ds = DeviceSolver(self.forest.mspar, self.forest.mtrees, self.forest.msifa)
        f = self.forest
        self.sm0 = torch.from_numpy(f.merge_sm([s['sm'] for s in systems])).cuda()
        self.nrhs = systems[0]['b'].shape[1]
        B = np.zeros((self.nrhs, f.neq))
        for i, s in enumerate(systems):
            B[:, f.eq_off[i]: f.eq_off[i] + f.neq_i[i]] = s['b'].T
        self.b0 = torch.from_numpy(B).cuda()
        self.sm = torch.empty_like(self.sm0)
        self.b = torch.empty_like(self.b0)

    def run(self, solve=True):
        """One batched factor (+ solve); returns (factor result, per-system NUMNEG)."""
        self.sm.copy_(self.sm0)
        self.b.copy_(self.b0)
        r = self.ds.factor(self.sm)
        if solve:
            self.ds.solve(self.sm, self.b, self.nrhs)
        return r

    def numneg(self):
        neg, _ = self.ds.sn_stats(self.forest.nsuper)
        return self.forest.per_system(neg)

    def solutions(self):
        X = self.b.cpu().numpy()
        f = self.forest
        return [X[:, f.eq_off[i]: f.eq_off[i] + f.neq_i[i]].T for i in range(f.nsys)]
