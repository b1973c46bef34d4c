"""GPU parity of SPR's partial factorisation (MSPAR(57) = 1, superelements).

A hex box whose face x=n is external (MSC = 2) makes the reference pipeline
number the face's equations last and mark their supernode retained
(SUPSUP > 0).  SPRFC1 then assembles that front without eliminating it, so
its LNZ columns hold the Schur complement (the condensed stiffness), and the
solves skip it: a forward sweep over all NEQ rows leaves the condensed load
in the retained rows, and LDB < NEQ solves for the internal equations with
the retained ones held at zero (sprfc1.f:463-608, sprfs1.f:201/371,
sprbs1.f:189/347).  The oracle is pinned bitwise to the reference on the
same cases (test_oracle.py).

Tolerances as the other parity tests: factor 1e-10 of max|SM|, solutions
1e-9 relative; IERR and MSPAR exact; D of the retained equations exactly 0.
"""
import numpy as np
import pytest

import sam_lib_b200 as spr
from conftest import ref_system, dense_from_sm
from test_oracle import run_sprsol, run_sprfc3, rhs, retained_info, _sprsol_ldb
from test_gpu_parity import close_factor, relerr

pytestmark = pytest.mark.gpu


def gpu_solve(rs, sm, b, iop, mspar, ldb):
    sm = sm.copy()
    B = np.asfortranarray(b.copy())
    msp = mspar.copy()
    tol = np.array([1e-12, 0.0, 0.0])
    ierr = spr.sprsol(iop, msp, rs.mtrees, rs.msifa, sm, B, ldb, B.shape[1], tol)
    return dict(sm=sm, b=B, tol=tol, ierr=ierr, mspar=msp)


@pytest.mark.parametrize('n', [6, 8])
def test_partial_factorisation_matches_oracle(n):
    """6^3: the retained root (F = 147) is a one-CTA small front; 8^3: it is a
    dense front (F = 243) assembled by the blocked path and written back
    without any panel or update launch."""
    rs, sm = ref_system(n, retain=True)
    msp = rs.mspar.copy()
    msp[56] = 1
    first, nret = retained_info(rs)
    b = rhs(rs.neq, 3, 50 + n)
    o = run_sprsol('orc', rs, sm, b, iop=1, mspar=msp)
    g = gpu_solve(rs, sm, b, 1, msp, rs.neq)
    assert g['ierr'] == o['ierr'] == 0
    assert np.array_equal(g['mspar'], o['mspar'])
    assert close_factor(g['sm'], o['sm'])
    assert not np.any(g['sm'][first:rs.neq])
    assert abs(g['tol'][1] - o['tol'][1]) <= 1e-10 * abs(o['tol'][1])
    assert abs(g['tol'][2] - o['tol'][2]) <= 1e-10 * abs(o['tol'][2])
    # the retained LNZ is the condensed stiffness
    K = dense_from_sm(rs, sm)
    S = K[first:, first:] - K[first:, :first] @ np.linalg.solve(K[:first, :first], K[:first, first:])
    Kg = dense_from_sm(rs, g['sm'])
    assert np.max(np.abs(Kg[first:, first:] - S)) <= 1e-10 * np.max(np.abs(S))
    # forward sweep over all rows: condensed load in the retained rows
    of = run_sprsol('orc', rs, o['sm'], b, iop=5, mspar=o['mspar'])
    gf = gpu_solve(rs, g['sm'], b, 5, g['mspar'], rs.neq)
    assert gf['ierr'] == of['ierr'] == 0
    assert relerr(gf['b'], of['b']) <= 1e-9
    # factor + both sweeps with LDB = internal equations, one call (IOP = 3)
    bi = np.asfortranarray(b[:first].copy())
    o3 = _sprsol_ldb('orc', rs, sm, bi, msp, first)
    g3 = gpu_solve(rs, sm, bi, 3, msp, first)
    assert g3['ierr'] == o3['ierr'] == 0
    assert relerr(g3['b'], o3['b']) <= 1e-9
    xi = np.linalg.solve(K[:first, :first], b[:first])
    assert relerr(g3['b'], xi) <= 1e-9
    # the same through SPRFS1 and SPRBS1 separately on the factored SM
    B = np.asfortranarray(b[:first].copy())
    fac, msp2 = g['sm'].copy(), g['mspar'].copy()
    assert spr.sprfs1(msp2, rs.mtrees, rs.msifa, fac, B, first, 3) == 0
    assert spr.sprbs1(msp2, rs.mtrees, rs.msifa, fac, B, first, 3) == 0
    assert relerr(B, o3['b']) <= 1e-9


def test_partial_sprfc3_leaves_retained_dcor_zero():
    rs, sm = ref_system(8, retain=True)
    msp = rs.mspar.copy()
    msp[56] = 1
    first, _ = retained_info(rs)
    o = run_sprfc3('orc', rs, sm, 1e-12, 1.0, mspar=msp)
    smg = sm.copy()
    mg = msp.copy()
    tol = np.array([1e-12, 0.0, 0.0, 1.0])
    dcor = np.full(2 * rs.neq, 7.0)
    ierr = spr.sprfc3(mg, rs.mtrees, rs.msifa, smg, tol, dcor)
    assert ierr == o['ierr'] == 0
    assert np.array_equal(mg, o['mspar'])
    assert not np.any(dcor.reshape(-1, 2)[first:])
    assert np.array_equal(dcor.reshape(-1, 2), o['dcor'])
    assert close_factor(smg, o['sm'])
