"""GPU parity of SPR's Cholesky family: SPRFC2 (C C' factorisation, MSPAR(1)
= 6), SPRFS2 (C y = b) and SPRBS2 (C' x = y, MSPAR(1) = 8) through
sprfc2_/sprfs2_/sprbs2_ of libspr_b200.so, against the oracle (pinned
bitwise to the translated reference in test_oracle.py).

The GPU factors in L D L' form with SPRF27's pivot rule (a non-positive
pivot stops) and hands the host C = L D^1/2; its sweeps apply the L D L'
solves with a D^1/2 scaling.  Tolerances as the other parity tests: factor
1e-10 of max|SM|, solutions 1e-9 relative (1e-6 with E over four decades);
IERR and MSPAR exact; TOL(2:3) 1e-10.
"""
import numpy as np
import pytest

import sam_lib_b200 as spr
from conftest import ref_system, shifted_sm, dense_from_sm
from test_oracle import run_chol, rhs, retained_info
from test_gpu_parity import close_factor, relerr

pytestmark = pytest.mark.gpu


def gpu_chol(rs, sm, b, tol1=1e-12, mspar=None, ldb=None, steps='fsb'):
    sm = sm.copy()
    ldb = rs.neq if ldb is None else ldb
    B = np.asfortranarray(b.copy())
    msp = rs.mspar.copy() if mspar is None else mspar.copy()
    tol = np.array([tol1, 0.0, 0.0])
    ierrs = []
    for st in steps:
        if st == 'f':
            ierrs.append(spr.sprfc2(msp, rs.mtrees, rs.msifa, sm, tol))
        elif st == 's':
            ierrs.append(spr.sprfs2(msp, rs.mtrees, rs.msifa, sm, B, ldb, B.shape[1]))
        else:
            ierrs.append(spr.sprbs2(msp, rs.mtrees, rs.msifa, sm, B, ldb, B.shape[1]))
        if ierrs[-1] < 0:
            break
    return dict(sm=sm, b=B, tol=tol, ierr=ierrs, mspar=msp)


@pytest.mark.parametrize('n,emod', [(6, 'loguniform'), (8, 'uniform'), (12, 'uniform')])
def test_sprfc2_factor_and_sweeps_match_oracle(n, emod):
    rs, sm = ref_system(n, emod)
    b = rhs(rs.neq, 3, 70 + n)
    rt = 1e-9 if emod == 'uniform' else 1e-6
    of = run_chol('orc', rs, sm, b, steps='f')
    gf = gpu_chol(rs, sm, b, steps='f')
    assert gf['ierr'] == of['ierr'] == [0]
    assert np.array_equal(gf['mspar'], of['mspar']) and gf['mspar'][0] == 6
    assert close_factor(gf['sm'], of['sm'])
    assert abs(gf['tol'][1] - of['tol'][1]) <= 1e-10 * abs(of['tol'][1])
    assert abs(gf['tol'][2] - of['tol'][2]) <= 1e-10 * abs(of['tol'][2])
    os_ = run_chol('orc', rs, sm, b, steps='fs')
    gs = gpu_chol(rs, sm, b, steps='fs')
    assert gs['ierr'] == os_['ierr'] == [0, 0] and gs['mspar'][0] == 8
    assert relerr(gs['b'], os_['b']) <= rt
    o = run_chol('orc', rs, sm, b)
    g = gpu_chol(rs, sm, b)
    assert g['ierr'] == o['ierr'] == [0, 0, 0]
    assert relerr(g['b'], o['b']) <= rt
    K = dense_from_sm(rs, sm) if n <= 8 else None
    if K is not None:
        assert np.linalg.norm(K @ g['b'] - b) <= 1e-10 * np.linalg.norm(b)


def test_sprfc2_errors_match_oracle():
    """An indefinite shift stops at the first non-positive pivot (MSPAR(27),
    TOL(2) = that pivot, TOL(3) = its original diagonal), an exact zero
    diagonal gives -35's mapping, and a preceding error is reported."""
    from scipy.linalg import eigh
    from sam_lib_b200.system import diag_positions
    rs, sm = ref_system(6)
    b = rhs(rs.neq, 1, 71)
    K = dense_from_sm(rs, sm)
    M = np.diag(K.diagonal() - dense_from_sm(rs, shifted_sm(rs, sm, 1.0)).diagonal())
    w = eigh(K, M, eigvals_only=True)
    ssm = shifted_sm(rs, sm, 0.5 * (w[7] + w[8]))
    o = run_chol('orc', rs, ssm, b, steps='f')
    g = gpu_chol(rs, ssm, b, steps='f')
    assert g['ierr'] == o['ierr'] == [-3]
    assert np.array_equal(g['mspar'], o['mspar'])
    assert g['tol'][2] == o['tol'][2]
    assert abs(g['tol'][1] - o['tol'][1]) <= 1e-9 * abs(o['tol'][2])
    z = sm.copy()
    z[diag_positions(rs.mspar, rs.mtrees, rs.msifa)[rs.neq - 30]] = 0.0
    o = run_chol('orc', rs, z, b, steps='f')
    g = gpu_chol(rs, z, b, steps='f')
    assert g['ierr'] == o['ierr'] == [-3]
    assert np.array_equal(g['mspar'], o['mspar'])
    bad = rs.mspar.copy()
    bad[0] = -2
    for st, state in (('f', -6), ('s', -8), ('b', -8)):
        g = gpu_chol(rs, sm, b, mspar=bad, steps=st)
        assert g['ierr'] == [-1] and g['mspar'][0] == state


def test_sprfc2_partial_factorisation_and_host_factor():
    """MSPAR(57) = 1 with the dense retained root of the 8^3 box: internal
    solution with LDB < NEQ; then the sweeps on a C C' factor the host made
    (the oracle's), which the GPU converts on upload."""
    rs, sm = ref_system(8, retain=True)
    msp = rs.mspar.copy()
    msp[56] = 1
    first, _ = retained_info(rs)
    b = rhs(rs.neq, 2, 72)
    o = run_chol('orc', rs, sm, b[:first], mspar=msp, ldb=first)
    g = gpu_chol(rs, sm, b[:first], mspar=msp, ldb=first)
    assert g['ierr'] == o['ierr'] == [0, 0, 0]
    assert np.array_equal(g['mspar'], o['mspar'])
    assert close_factor(g['sm'], o['sm'])
    assert relerr(g['b'], o['b']) <= 1e-9
    K = dense_from_sm(rs, sm)
    assert relerr(g['b'], np.linalg.solve(K[:first, :first], b[:first])) <= 1e-9
    # the oracle's C C' factor of the plain 6^3 box, solved on the GPU
    rs6, sm6 = ref_system(6)
    b6 = rhs(rs6.neq, 2, 73)
    of = run_chol('orc', rs6, sm6, b6, steps='f')
    ox = run_chol('orc', rs6, sm6, b6)
    g = gpu_chol(rs6, of['sm'], b6, mspar=of['mspar'], steps='sb')
    assert g['ierr'] == [0, 0]
    assert relerr(g['b'], ox['b']) <= 1e-9
