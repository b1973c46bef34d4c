"""The streamed factorisation of the Fortran entry points (GPU).

When SM lies in page-locked host memory, SPRFC1 (and SPRSOL with IOP <= 3)
uploads LNZ level group by level group on a copy stream while the lower
levels factor, and downloads each level's finished columns while the higher
levels factor; the zero-diagonal test reads a host-gathered diagonal first.
The results must be those of the plain path (pageable SM, one upload, one
download) bit for bit: SM, B, TOL, MSPAR and IERR, also on the error paths
(a zero diagonal, a failed pivot) and for a partial factorisation.
"""
import numpy as np
import pytest

import sam_lib_b200 as spr
from conftest import ref_system, shifted_sm
from test_oracle import rhs

pytestmark = pytest.mark.gpu


def _pinned(a):
    import torch
    t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
    v = t.numpy()
    v[...] = a
    return t, v


def _run(rs, sm, b, iop, pinned, mspar=None, ldb=None, tol1=1e-12):
    ldb = rs.neq if ldb is None else ldb
    msp = (rs.mspar if mspar is None else mspar).copy()
    tol = np.array([tol1, 0.0, 0.0])
    B = np.asfortranarray(b.copy())
    if pinned:
        keep, smv = _pinned(sm)
        tb, bt = _pinned(np.ascontiguousarray(B.T))
        Bv = bt.T
    else:
        smv, Bv = sm.copy(), B
    ierr = spr.sprsol(iop, msp, rs.mtrees, rs.msifa, smv, Bv, ldb, B.shape[1], tol)
    return dict(ierr=ierr, sm=np.array(smv), b=np.array(Bv), tol=tol, mspar=msp)


def _same(a, b):
    assert a['ierr'] == b['ierr'], (a['ierr'], b['ierr'])
    assert np.array_equal(a['mspar'], b['mspar'])
    assert np.array_equal(a['tol'], b['tol'])
    assert np.array_equal(a['sm'], b['sm'])
    assert np.array_equal(a['b'], b['b'])


@pytest.mark.parametrize('n,sigma,iop', [(12, 0.0, 3), (12, 8e-3, 3), (10, 0.0, 1), (16, 0.0, 3)])
def test_streamed_equals_plain(n, sigma, iop):
    rs, sm = ref_system(n)
    if sigma:
        sm = shifted_sm(rs, sm, sigma)
    b = rhs(rs.neq, 2, n)
    _same(_run(rs, sm, b, iop, True), _run(rs, sm, b, iop, False))
    spr.release_all()


def test_streamed_error_paths_equal_plain():
    rs, sm = ref_system(8)
    b = rhs(rs.neq, 1, 3)
    z = sm.copy()
    from sam_lib_b200.system import diag_positions
    pos = diag_positions(rs.mspar, rs.mtrees, rs.msifa)
    z[pos[rs.neq - 5]] = 0.0                           # a zero diagonal in the root supernode
    p, q = _run(rs, z, b, 3, True), _run(rs, z, b, 3, False)
    assert p['ierr'] == -3 and p['mspar'][26] == rs.neq - 4
    _same(p, q)
    # a pivot that fails the TOL(1) test in a top-level front
    p, q = _run(rs, sm, b, 1, True, tol1=0.6), _run(rs, sm, b, 1, False, tol1=0.6)
    assert p['ierr'] == -3
    _same(p, q)
    spr.release_all()


def test_streamed_partial_factorisation_equals_plain():
    rs, sm = ref_system(8, retain=True)
    msp = rs.mspar.copy()
    msp[56] = 1
    b = rhs(rs.neq, 2, 5)
    _same(_run(rs, sm, b, 1, True, mspar=msp), _run(rs, sm, b, 1, False, mspar=msp))
    spr.release_all()
