"""Batched forests on the CPU: the merged SPR structure of several systems.

sam_lib_b200.batch.Forest concatenates independent systems into one SPR
forest (SIBL(NSUPER+1) = number of roots, src/SPR/sprtrs.f:1592-1597).  The
reference and the oracle factor and solve that forest exactly as they do each
system alone, so the per-system parts of the forest's SM and solution are bit
for bit the systems' own; the GPU plan of the forest passes its self-check.
"""
import numpy as np

import sam_lib_b200 as spr
from conftest import ref_system, shifted_sm
from test_oracle import run_sprsol, rhs
from sam_lib_b200.batch import Forest


class _RS:
    """The fields of a RefSystem that run_sprsol reads."""

    def __init__(self, mspar, mtrees, msifa):
        self.mspar, self.mtrees, self.msifa = mspar, mtrees, msifa
        self.neq = int(mspar[7])


def _systems():
    rs3, sm3 = ref_system(3)
    rs4, sm4 = ref_system(4, 'loguniform')
    rs3b, _ = ref_system(3)
    return [(rs3, sm3), (rs4, sm4), (rs3b, shifted_sm(rs3b, sm3, 0.1))]


def test_forest_factor_and_solve_equal_the_systems_alone():
    systems = _systems()
    f = Forest([(rs.mspar, rs.mtrees, rs.msifa) for rs, _ in systems])
    frs = _RS(f.mspar, f.mtrees, f.msifa)
    bs = [rhs(rs.neq, 2, 80 + i) for i, (rs, _) in enumerate(systems)]
    sm = f.merge_sm([s for _, s in systems])
    B = np.zeros((f.neq, 2))
    for i, b in enumerate(bs):
        B[f.eq_off[i]: f.eq_off[i] + f.neq_i[i]] = b
    ref = run_sprsol('ref', frs, sm, B)
    orc = run_sprsol('orc', frs, sm, B)
    assert ref['ierr'] == orc['ierr'] == 0
    assert np.array_equal(ref['sm'], orc['sm']) and np.array_equal(ref['b'], orc['b'])
    numneg = 0
    for i, ((rs, s), b) in enumerate(zip(systems, bs)):
        alone = run_sprsol('orc', rs, s, b, iop=1)
        numneg += alone['mspar'][25]
        assert np.array_equal(f.split_sm(orc['sm'])[i], alone['sm'])
        alone = run_sprsol('orc', rs, s, b)
        assert np.array_equal(orc['b'][f.eq_off[i]: f.eq_off[i] + f.neq_i[i]], alone['b'])
    assert orc['mspar'][25] == numneg > 0


def test_forest_plan_self_check():
    systems = _systems()
    f = Forest([(rs.mspar, rs.mtrees, rs.msifa) for rs, _ in systems])
    out = np.zeros(13)
    rc = spr.load(8).spr_b200_plan_check(spr._ptr(f.mspar), spr._ptr(f.mtrees), spr._ptr(f.msifa), spr._ptr(out))
    assert rc == 0 and out[0] == 0
    assert out[1] == f.nsuper
    assert out[4] == 0 and out[5] == 0 and out[11] == 0 and out[12] == 0
    assert abs(out[6] - sum(rs.rinfo[2] for rs, _ in systems)) <= 1e-12 * out[6]
