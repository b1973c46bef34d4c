"""One system split across GPUs: the data path on one GPU (GPU).

``split.emulate`` runs the ranks of a split run one after another on the
current GPU, each with its own engine and SM copy, moving the subtree-root
update blocks, the D/LNZ ranges, the update vectors and the solution ranges
between them with device copies - the same phases and the same exchange
lists as ``SplitSolver`` over NCCL, without any kernel waiting for another
rank's.  Against the one-engine factorisation of the same system: the same
kernels per supernode in the same order, so the factor must agree to
rounding level (max |dSM| <= 1e-13 max |SM|), NUMNEG exactly, TOL(2:3) to
1e-13, and the solution to 1e-12 (E = 1, shifted and not).
"""
import numpy as np
import pytest

import sam_lib_b200 as spr
from conftest import ref_system, shifted_sm
from test_oracle import rhs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('n,sigma,world', [(12, 0.0, 2), (12, 8e-3, 3), (16, 0.0, 2), (16, 3e-3, 4)])
def test_emulated_split_equals_one_engine(n, sigma, world):
    import torch
    from sam_lib_b200.split import emulate
    rs, sm = ref_system(n)
    if sigma:
        sm = shifted_sm(rs, sm, sigma)
    b = rhs(rs.neq, 3, 21 + n)
    ds = spr.DeviceSolver(rs.mspar, rs.mtrees, rs.msifa)
    d_sm = torch.from_numpy(sm).cuda()
    r1 = ds.factor(d_sm)
    d_b = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    ds.solve(d_sm, d_b, 3)
    sm1, x1 = d_sm.cpu().numpy(), d_b.cpu().numpy().T
    ds.close()
    out, sm2, x2 = emulate(rs.mspar, rs.mtrees, rs.msifa, sm, b, world)
    assert out['lierr'] == r1['lierr'] == 0
    assert out['numneg'] == r1['numneg']
    if sigma:
        assert r1['numneg'] > 0
    dsm = np.max(np.abs(sm2 - sm1)) / np.max(np.abs(sm1))
    assert dsm <= 1e-13, dsm
    assert abs(out['tol2'] - r1['tol2']) <= 1e-13 * abs(r1['tol2'])
    assert abs(out['tol3'] - r1['tol3']) <= 1e-13 * abs(r1['tol3'])
    dx = np.linalg.norm(x2 - x1) / np.linalg.norm(x1)
    assert dx <= 1e-12, dx
    print('split %d ranks, %d^3: max|dSM| %.1e, solution %.1e, bitwise SM %s' % (world, n, dsm, dx,
                                                                             np.array_equal(sm1, sm2)))
