"""The two eliminations of the diagonal-block kernel agree bit for bit (GPU).

k_diag has two forms of its 64 x 64 LDL' elimination: the block in registers
over 256 threads (SPR_B200_DIAG=0) and the default, row pairs in shared
memory.  Both apply a_ij -= (a_ik / d_k) a_jk in the same order per entry, so
their factors must be identical: SM, NUMNEG, IERR, TOL and the solution, for
SPRFC1's pivot test, SPRFC3's replacement (a free box) and a pivot failure
inside a dense front, through the Fortran entry points (each run in a fresh
library context, the variable read when a context is created).
"""
import os

import numpy as np
import pytest

import sam_lib_b200 as spr
from conftest import ref_system, shifted_sm

pytestmark = pytest.mark.gpu


def _run(fn, alg):
    old = os.environ.get('SPR_B200_DIAG')
    os.environ['SPR_B200_DIAG'] = alg
    try:
        spr.release_all()
        return fn()
    finally:
        spr.release_all()
        if old is None:
            del os.environ['SPR_B200_DIAG']
        else:
            os.environ['SPR_B200_DIAG'] = old


def _sprsol(rs, sm, tol1=1e-12):
    def go():
        g_sm = sm.copy()
        b = np.asfortranarray(np.random.default_rng(3).uniform(-1, 1, size=(rs.neq, 2)))
        msp = rs.mspar.copy()
        tol = np.array([tol1, 0.0, 0.0])
        ierr = spr.sprsol(3, msp, rs.mtrees, rs.msifa, g_sm, b, rs.neq, 2, tol)
        return ierr, g_sm, b, tol, msp
    return go


@pytest.mark.parametrize('n,sigma', [(12, 0.0), (12, 2.0e-3), (16, 0.0)])
def test_diag_eliminations_bitwise_equal(n, sigma):
    rs, sm = ref_system(n)
    if sigma:
        sm = shifted_sm(rs, sm, sigma)
    a = _run(_sprsol(rs, sm), '0')
    b = _run(_sprsol(rs, sm), '1')
    assert a[0] == b[0]
    for x, y in zip(a[1:], b[1:]):
        assert np.array_equal(x, y)


def test_diag_eliminations_agree_on_replaced_and_failed_pivots():
    rs, sm = ref_system(8, clamp=False)

    def fc3():
        g_sm = sm.copy()
        msp = rs.mspar.copy()
        tol = np.array([1e-8, 0.0, 0.0, 1e-2])
        dcor = np.full(2 * rs.neq, 7.0)
        ierr = spr.sprfc3(msp, rs.mtrees, rs.msifa, g_sm, tol, dcor)
        return ierr, g_sm, tol, dcor, msp
    a, b = _run(fc3, '0'), _run(fc3, '1')
    assert a[0] == b[0]
    for x, y in zip(a[1:], b[1:]):
        assert np.array_equal(x, y)
    # a pivot driven to zero in the middle of the largest (dense-path) front
    from sam_lib_b200.system import diag_positions
    rs2, sm2 = ref_system(8)
    sp = rs2.mspar
    ns = int(sp[10])
    xs = rs2.mtrees[sp[44] - 1: sp[44] + ns]
    F = np.diff(rs2.mtrees[sp[45] - 1: sp[45] + ns])
    js = int(np.argmax(F))
    assert F[js] > 176
    j = int(xs[js] - 1 + (xs[js + 1] - xs[js]) // 2)
    d = _run(_sprsol(rs2, sm2), '1')[1][j]
    z = sm2.copy()
    z[diag_positions(rs2.mspar, rs2.mtrees, rs2.msifa)[j]] -= d
    a = _run(_sprsol(rs2, z, tol1=1e-8), '0')
    b = _run(_sprsol(rs2, z, tol1=1e-8), '1')
    assert a[0] == b[0] == -3
    assert a[4][26] == b[4][26] == j + 1
    assert np.array_equal(a[4], b[4]) and np.array_equal(a[3], b[3])
