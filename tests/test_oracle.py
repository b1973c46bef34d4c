"""Oracle pinning (CPU): the C restatement against the translated reference.

The oracle (oracle/spr_oracle.c) must reproduce the reference SPR numeric
phase bit for bit: same factor in SM, same solution, same TOL/MSPAR/IERR.
The reference itself is the machine translation of the Fortran sources
(oracle/f77c.py -> oracle/_ref/libsprref.so).
"""
import ctypes as C

import numpy as np
import pytest

from conftest import ref_system, shifted_sm, dense_from_sm


_L = None


def _lib():
    global _L
    if _L is None:
        import os
        here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        _L = C.CDLL(os.path.join(here, 'oracle', '_ref', 'liboracle.so'))
    return _L


def run_sprsol(which, rs, sm, b, iop=3, tol1=1e-12, mspar=None):
    from oracle.refpipe import lib as reflib, _p, _i
    sm = sm.copy()
    b = np.asfortranarray(b.copy())
    nrhs = 1 if b.ndim == 1 else b.shape[1]
    msp = rs.mspar.copy() if mspar is None else mspar.copy()
    tol = np.array([tol1, 0.0, 0.0])
    iw = np.zeros(int(rs.mspar[13]) + int(rs.mspar[12]) + 8, dtype=np.int64)
    rw = np.zeros(int(rs.mspar[16]) + int(rs.mspar[13]) + 8)
    ierr = C.c_int64(0)
    f = reflib().sprsol_ if which == 'ref' else _lib().orc_sprsol_
    f(_i(iop), _p(msp), _p(rs.mtrees), _p(rs.msifa), _p(sm), _p(b), _i(rs.neq), _i(nrhs),
      _p(tol), _p(iw), _p(rw), _i(-1), C.byref(ierr))
    return dict(sm=sm, b=b, tol=tol, ierr=ierr.value, mspar=msp)


def rhs(neq, nrhs, seed):
    return np.random.default_rng(seed).uniform(-1.0, 1.0, size=(neq, nrhs))


@pytest.mark.parametrize('n,emod', [(3, 'uniform'), (6, 'uniform'), (6, 'loguniform'), (9, 'loguniform')])
def test_oracle_bitwise_equals_reference(n, emod):
    rs, sm = ref_system(n, emod)
    b = rhs(rs.neq, 3, n)
    r = run_sprsol('ref', rs, sm, b)
    o = run_sprsol('orc', rs, sm, b)
    assert r['ierr'] == o['ierr'] == 0
    assert np.array_equal(r['sm'], o['sm'])
    assert np.array_equal(r['b'], o['b'])
    assert np.array_equal(r['tol'], o['tol'])
    assert np.array_equal(r['mspar'], o['mspar'])


def test_reference_solution_is_accurate():
    rs, sm = ref_system(6)
    K = dense_from_sm(rs, sm)
    b = rhs(rs.neq, 2, 0)
    r = run_sprsol('ref', rs, sm, b)
    res = np.linalg.norm(K @ r['b'] - b) / np.linalg.norm(b)
    assert res < 1e-12


def test_inertia_matches_eigenvalues_and_reference():
    rs, sm = ref_system(3)
    from scipy.linalg import eigh
    K = dense_from_sm(rs, sm)
    M = np.diag(K.diagonal() - dense_from_sm(rs, shifted_sm(rs, sm, 1.0)).diagonal())
    w = eigh(K, M, eigvals_only=True)
    sigma = 0.5 * (w[3] + w[4])           # between the 4th and 5th eigenvalue
    ssm = shifted_sm(rs, sm, sigma)
    b = rhs(rs.neq, 1, 1)
    r = run_sprsol('ref', rs, ssm, b, iop=1)
    o = run_sprsol('orc', rs, ssm, b, iop=1)
    assert r['ierr'] == 3 and o['ierr'] == 3          # not positive definite warning
    assert r['mspar'][25] == o['mspar'][25] == 4      # NUMNEG = eigenvalues below sigma
    assert np.array_equal(r['sm'], o['sm'])
    # SPRSOL IOP=3: the solves reset IERR to 0 (sprfs1.f:143-144), NUMNEG stays
    r = run_sprsol('ref', rs, ssm, b, iop=3)
    o = run_sprsol('orc', rs, ssm, b, iop=3)
    assert r['ierr'] == o['ierr'] == 0
    assert r['mspar'][25] == o['mspar'][25] == 4
    assert np.array_equal(r['b'], o['b'])


def test_error_codes_match_reference():
    rs, sm = ref_system(3)
    b = rhs(rs.neq, 1, 2)
    # preceding error not cleared (sprfc1.f:140-148)
    bad = rs.mspar.copy()
    bad[0] = -3
    r = run_sprsol('ref', rs, sm, b, mspar=bad)
    o = run_sprsol('orc', rs, sm, b, mspar=bad)
    assert r['ierr'] == o['ierr'] == -1 and r['mspar'][0] == o['mspar'][0] == -5
    # exact zero diagonal (sprfc1.f:474-488): IERR=-3, MSPAR(27)=first equation
    z = sm.copy()
    neq = rs.neq
    sp = rs.mspar
    xlnz1 = int(rs.msifa[sp[47] - 1 + 5])       # first LNZ entry of supernode 6
    z[neq + xlnz1 - 1] = 0.0
    r = run_sprsol('ref', rs, z, b, iop=1)
    o = run_sprsol('orc', rs, z, b, iop=1)
    assert r['ierr'] == o['ierr'] == -3
    assert r['mspar'][26] == o['mspar'][26] and r['mspar'][25] == o['mspar'][25] == 1
    assert np.array_equal(r['tol'], o['tol'])
    # pivot below threshold (sprfc1.f:1274-1279): huge TOL(1)
    r = run_sprsol('ref', rs, sm, b, iop=1, tol1=0.9)
    o = run_sprsol('orc', rs, sm, b, iop=1, tol1=0.9)
    assert r['ierr'] == o['ierr'] == -3
    assert r['mspar'][26] == o['mspar'][26]
    assert r['mspar'][25] == o['mspar'][25]
    assert np.array_equal(r['tol'], o['tol'])


# ---------------------------------------------------------------------------
# SPRFC3 (src/SPR/sprfc3.f): singular pivots replaced and recorded in DCOR
# ---------------------------------------------------------------------------

def run_sprfc3(which, rs, sm, tol1, tol4, mspar=None):
    from oracle.refpipe import lib as reflib, _p, _i
    sm = sm.copy()
    msp = rs.mspar.copy() if mspar is None else mspar.copy()
    tol = np.array([tol1, 0.0, 0.0, tol4])
    dcor = np.full(2 * rs.neq, 7.0)        # every entry is written (sprfc3.f:564-565)
    iw = np.zeros(int(rs.mspar[13]) + 8, dtype=np.int64)
    rw = np.zeros(int(rs.mspar[16]) + 8)
    ierr = C.c_int64(0)
    if which == 'ref':
        R = reflib()
        R.sprfc3_(_p(msp), _p(rs.mtrees), _p(rs.msifa), _p(sm), _p(tol), _p(iw), _p(rw),
                  _p(dcor), _i(-1), C.byref(ierr), C.cast(R.lmvy18_, C.c_void_p),
                  C.cast(R.lmmy18_, C.c_void_p))
    else:
        _lib().orc_sprfc3_(_p(msp), _p(rs.mtrees), _p(rs.msifa), _p(sm), _p(tol), _p(iw),
                           _p(rw), _p(dcor), _i(-1), C.byref(ierr))
    return dict(sm=sm, tol=tol, dcor=dcor.reshape(-1, 2), ierr=ierr.value, mspar=msp)


def _same(r, o):
    assert r['ierr'] == o['ierr']
    assert np.array_equal(r['sm'], o['sm'])
    assert np.array_equal(r['tol'], o['tol'])
    assert np.array_equal(r['dcor'], o['dcor'])
    assert np.array_equal(r['mspar'], o['mspar'])


def test_sprfc3_rigid_body_modes_match_reference():
    """Free box: the six rigid-body modes give six pivots at rounding level,
    each replaced by sign(TOL(1) max(1, |TOL(4) a_jj|), d)."""
    rs, sm = ref_system(4, clamp=False)
    r = run_sprfc3('ref', rs, sm, 1e-8, 1e-2)
    o = run_sprfc3('orc', rs, sm, 1e-8, 1e-2)
    _same(r, o)
    assert o['ierr'] == -3 and o['mspar'][0] == 5
    assert o['mspar'][26] == -6                   # MSPAR(27) = -(number replaced)
    rep = np.nonzero(o['dcor'][:, 1])[0]
    assert len(rep) == 6
    from sam_lib_b200.system import diag_positions
    adiag = sm[diag_positions(rs.mspar, rs.mtrees, rs.msifa)]
    np.testing.assert_array_equal(np.abs(o['dcor'][rep, 1]),
                                  1e-8 * np.maximum(1.0, np.abs(1e-2 * adiag[rep])))


def test_sprfc3_zero_diagonal_indefinite_and_threshold_match_reference():
    from sam_lib_b200.system import diag_positions
    rs, sm = ref_system(5)
    pos = diag_positions(rs.mspar, rs.mtrees, rs.msifa)
    # an exact zero diagonal becomes 1 (DCOR(2,j) = 1, sprfc3.f:566-571)
    z = sm.copy()
    j = rs.neq // 2
    z[pos[j]] = 0.0
    r = run_sprfc3('ref', rs, z, 1e-12, 1.0)
    o = run_sprfc3('orc', rs, z, 1e-12, 1.0)
    _same(r, o)
    assert o['dcor'][j, 1] == 1.0
    # an indefinite shift: DCOR(1,j) holds the negative pivots, IERR = 3
    from scipy.linalg import eigh
    rs3, sm3 = ref_system(3)
    K = dense_from_sm(rs3, sm3)
    M = np.diag(K.diagonal() - dense_from_sm(rs3, shifted_sm(rs3, sm3, 1.0)).diagonal())
    w = eigh(K, M, eigvals_only=True)
    ssm = shifted_sm(rs3, sm3, 0.5 * (w[5] + w[6]))
    r = run_sprfc3('ref', rs3, ssm, 1e-12, 1.0)
    o = run_sprfc3('orc', rs3, ssm, 1e-12, 1.0)
    _same(r, o)
    assert o['ierr'] == 3 and o['mspar'][25] == 6
    assert np.count_nonzero(o['dcor'][:, 0] < 0.0) == 6
    # a large TOL(1): regular pivots replaced, the factor still completes
    r = run_sprfc3('ref', rs, sm, 0.45, 0.5)
    o = run_sprfc3('orc', rs, sm, 0.45, 0.5)
    _same(r, o)
    assert o['ierr'] == -3 and o['mspar'][26] < 0 and o['mspar'][0] == 5
    # preceding error not cleared (sprfc3.f:139-143)
    bad = rs.mspar.copy()
    bad[0] = -2
    r = run_sprfc3('ref', rs, sm, 1e-12, 1.0, mspar=bad)
    o = run_sprfc3('orc', rs, sm, 1e-12, 1.0, mspar=bad)
    assert r['ierr'] == o['ierr'] == -1 and r['mspar'][0] == o['mspar'][0] == -5


# ---------------------------------------------------------------------------
# Partial factorisation (MSPAR(57) = 1): retained supernodes of external DOFs
# ---------------------------------------------------------------------------

def retained_info(rs):
    """(first retained equation, 0-based; number of retained equations)."""
    sp = rs.mspar
    ns = int(sp[10])
    xs = rs.mtrees[sp[44] - 1: sp[44] + ns]
    supsup = rs.mtrees[sp[45] + ns: sp[45] + 2 * ns]
    ret = np.nonzero(supsup > 0)[0]
    first = int(xs[ret[0]] - 1)
    return first, rs.neq - first


@pytest.mark.parametrize('n', [3, 6])
def test_partial_factorisation_matches_reference(n):
    """SPRSOL with MSPAR(57) = 1 on a box whose face x=n is external (MSC=2):
    the factor (retained supernodes assembled, not eliminated), the condensed
    load (forward with LDB = NEQ), and the internal solution for zero
    retained displacements (LDB < NEQ) are the reference's bit for bit."""
    rs, sm = ref_system(n, retain=True)
    msp = rs.mspar.copy()
    msp[56] = 1
    first, nret = retained_info(rs)
    assert nret == 3 * (n + 1) ** 2
    b = rhs(rs.neq, 2, 40 + n)
    r = run_sprsol('ref', rs, sm, b, iop=1, mspar=msp)
    o = run_sprsol('orc', rs, sm, b, iop=1, mspar=msp)
    assert r['ierr'] == o['ierr'] == 0
    assert np.array_equal(r['sm'], o['sm'])
    assert np.array_equal(r['tol'], o['tol'])
    assert np.array_equal(r['mspar'], o['mspar'])
    assert not np.any(o['sm'][first:rs.neq])          # D of the retained equations stays 0
    # forward reduction over all NEQ rows: the retained rows get the condensed load
    fac = o['sm']
    r = run_sprsol('ref', rs, fac, b, iop=5, mspar=r['mspar'])
    o = run_sprsol('orc', rs, fac, b, iop=5, mspar=o['mspar'])
    assert r['ierr'] == o['ierr'] == 0
    assert np.array_equal(r['b'], o['b'])
    # factor + forward + back with LDB = number of internal equations
    bi = np.asfortranarray(b[:first].copy())
    r = _sprsol_ldb('ref', rs, sm, bi, msp, first)
    o = _sprsol_ldb('orc', rs, sm, bi, msp, first)
    assert r['ierr'] == o['ierr'] == 0
    assert np.array_equal(r['b'], o['b'])
    # which is the internal solution with the retained DOFs held at zero
    K = dense_from_sm(rs, sm)
    xi = np.linalg.solve(K[:first, :first], b[:first])
    assert np.max(np.abs(o['b'] - xi)) <= 1e-10 * np.max(np.abs(xi))
    # and the retained supernodes of LNZ hold the Schur complement
    S = K[first:, first:] - K[first:, :first] @ np.linalg.solve(K[:first, :first], K[:first, first:])
    Kf = dense_from_sm(rs, fac)
    assert np.max(np.abs(Kf[first:, first:] - S)) <= 1e-10 * np.max(np.abs(S))
    # SPRFC3 with MSPAR(57) = 1: DCOR of the retained equations stays 0 (sprfc3.f:551-554)
    r = run_sprfc3('ref', rs, sm, 1e-12, 1.0, mspar=msp)
    o = run_sprfc3('orc', rs, sm, 1e-12, 1.0, mspar=msp)
    _same(r, o)
    assert not np.any(o['dcor'][first:])


def _sprsol_ldb(which, rs, sm, b, mspar, ldb):
    from oracle.refpipe import lib as reflib, _p, _i
    sm = sm.copy()
    b = np.asfortranarray(b.copy())
    msp = mspar.copy()
    tol = np.array([1e-12, 0.0, 0.0])
    iw = np.zeros(int(rs.mspar[13]) + int(rs.mspar[12]) + 8, dtype=np.int64)
    rw = np.zeros(int(rs.mspar[16]) + int(rs.mspar[13]) + 8)
    ierr = C.c_int64(0)
    f = reflib().sprsol_ if which == 'ref' else _lib().orc_sprsol_
    f(_i(3), _p(msp), _p(rs.mtrees), _p(rs.msifa), _p(sm), _p(b), _i(ldb), _i(b.shape[1]),
      _p(tol), _p(iw), _p(rw), _i(-1), C.byref(ierr))
    return dict(sm=sm, b=b, tol=tol, ierr=ierr.value, mspar=msp)


# ---------------------------------------------------------------------------
# Cholesky C C' (src/SPR/sprfc2.f, sprfs2.f, sprbs2.f, cmvy18.f, cmmy18.f)
# ---------------------------------------------------------------------------

def run_chol(which, rs, sm, b, tol1=1e-12, mspar=None, ldb=None, steps='fsb'):
    """SPRFC2 (f), SPRFS2 (s: forward) and SPRBS2 (b: back), in that order,
    as `steps` lists them."""
    from oracle.refpipe import lib as reflib, _p, _i
    sm = sm.copy()
    ldb = rs.neq if ldb is None else ldb
    b = np.asfortranarray(b.copy())
    nrhs = b.shape[1]
    msp = rs.mspar.copy() if mspar is None else mspar.copy()
    tol = np.array([tol1, 0.0, 0.0])
    iw = np.zeros(int(rs.mspar[13]) + int(rs.mspar[12]) + 8, dtype=np.int64)
    rw = np.zeros(int(rs.mspar[16]) + int(rs.mspar[13]) + 8)
    ierr = C.c_int64(0)
    ierrs = []
    R = reflib()
    for st in steps:
        ierr.value = 0
        if st == 'f':
            if which == 'ref':
                R.sprfc2_(_p(msp), _p(rs.mtrees), _p(rs.msifa), _p(sm), _p(tol), _p(iw), _p(rw), _i(-1),
                          C.byref(ierr), C.cast(R.cmvy18_, C.c_void_p), C.cast(R.cmmy18_, C.c_void_p))
            else:
                _lib().orc_sprfc2_(_p(msp), _p(rs.mtrees), _p(rs.msifa), _p(sm), _p(tol), _p(iw), _p(rw),
                                   _i(-1), C.byref(ierr))
        elif st == 's':
            f = R.sprfs2_ if which == 'ref' else _lib().orc_sprfs2_
            f(_p(msp), _p(rs.mtrees), _p(rs.msifa), _p(sm), _p(b), _i(ldb), _i(nrhs), _p(iw), _p(rw), _i(-1),
              C.byref(ierr))
        else:
            f = R.sprbs2_ if which == 'ref' else _lib().orc_sprbs2_
            f(_p(msp), _p(rs.mtrees), _p(rs.msifa), _p(sm), _p(b), _i(ldb), _i(nrhs), _p(rw), _i(-1),
              C.byref(ierr))
        ierrs.append(ierr.value)
        if ierr.value < 0:
            break
    return dict(sm=sm, b=b, tol=tol, ierr=ierrs, mspar=msp)


def _same_chol(r, o):
    assert r['ierr'] == o['ierr']
    for k in ('sm', 'b', 'tol', 'mspar'):
        assert np.array_equal(r[k], o[k]), k


@pytest.mark.parametrize('n,emod', [(3, 'uniform'), (6, 'loguniform'), (8, 'uniform')])
def test_cholesky_bitwise_equals_reference(n, emod):
    rs, sm = ref_system(n, emod)
    b = rhs(rs.neq, 2, 60 + n)
    r = run_chol('ref', rs, sm, b)
    o = run_chol('orc', rs, sm, b)
    _same_chol(r, o)
    assert o['ierr'] == [0, 0, 0] and o['mspar'][0] == 8
    K = dense_from_sm(rs, sm)
    assert np.linalg.norm(K @ o['b'] - b) <= 1e-12 * np.linalg.norm(b)


def test_cholesky_error_paths_match_reference():
    rs, sm = ref_system(3)
    b = rhs(rs.neq, 1, 61)
    # an indefinite shift: the first non-positive pivot stops it (sprfc2.f:1001-1008)
    from scipy.linalg import eigh
    K = dense_from_sm(rs, sm)
    M = np.diag(K.diagonal() - dense_from_sm(rs, shifted_sm(rs, sm, 1.0)).diagonal())
    w = eigh(K, M, eigvals_only=True)
    ssm = shifted_sm(rs, sm, 0.5 * (w[3] + w[4]))
    r = run_chol('ref', rs, ssm, b, steps='f')
    o = run_chol('orc', rs, ssm, b, steps='f')
    _same_chol(r, o)
    assert o['ierr'] == [-3] and o['mspar'][26] > 0 and o['tol'][1] <= 0.0
    # an exact zero diagonal (-35: MSPAR(26) counts them, MSPAR(27) the first)
    from sam_lib_b200.system import diag_positions
    z = sm.copy()
    z[diag_positions(rs.mspar, rs.mtrees, rs.msifa)[7]] = 0.0
    r = run_chol('ref', rs, z, b, steps='f')
    o = run_chol('orc', rs, z, b, steps='f')
    _same_chol(r, o)
    assert o['ierr'] == [-3] and o['mspar'][26] == 8 and o['mspar'][25] == 1
    # preceding error not cleared
    bad = rs.mspar.copy()
    bad[0] = -2
    for st in 'fsb':
        r = run_chol('ref', rs, sm, b, mspar=bad, steps=st)
        o = run_chol('orc', rs, sm, b, mspar=bad, steps=st)
        _same_chol(r, o)
        assert o['ierr'] == [-1] and o['mspar'][0] == (-6 if st == 'f' else -8)


def test_cholesky_partial_factorisation_matches_reference():
    rs, sm = ref_system(6, retain=True)
    msp = rs.mspar.copy()
    msp[56] = 1
    first, _ = retained_info(rs)
    b = rhs(rs.neq, 2, 62)
    r = run_chol('ref', rs, sm, b[:first], mspar=msp, ldb=first)
    o = run_chol('orc', rs, sm, b[:first], mspar=msp, ldb=first)
    _same_chol(r, o)
    K = dense_from_sm(rs, sm)
    xi = np.linalg.solve(K[:first, :first], b[:first])
    assert np.max(np.abs(o['b'] - xi)) <= 1e-10 * np.max(np.abs(xi))
    r = run_chol('ref', rs, sm, b, mspar=msp, steps='fs')
    o = run_chol('orc', rs, sm, b, mspar=msp, steps='fs')
    _same_chol(r, o)


def run_sprfc4(which, rs, sm, tol1, tol4, mspar=None):
    from oracle.refpipe import lib as reflib, _p, _i
    sm = sm.copy()
    msp = rs.mspar.copy() if mspar is None else mspar.copy()
    tol = np.array([tol1, 0.0, 0.0, tol4])
    dcor = np.full(2 * rs.neq, 7.0)
    iw = np.zeros(int(rs.mspar[13]) + 8, dtype=np.int64)
    rw = np.zeros(int(rs.mspar[16]) + 8)
    ierr = C.c_int64(0)
    if which == 'ref':
        R = reflib()
        R.sprfc4_(_p(msp), _p(rs.mtrees), _p(rs.msifa), _p(sm), _p(tol), _p(iw), _p(rw),
                  _p(dcor), _i(-1), C.byref(ierr), C.cast(R.cmvy18_, C.c_void_p),
                  C.cast(R.cmmy18_, C.c_void_p))
    else:
        _lib().orc_sprfc4_(_p(msp), _p(rs.mtrees), _p(rs.msifa), _p(sm), _p(tol), _p(iw),
                           _p(rw), _p(dcor), _i(-1), C.byref(ierr))
    return dict(sm=sm, tol=tol, dcor=dcor.reshape(-1, 2), ierr=ierr.value, mspar=msp)


def test_sprfc4_matches_reference():
    """SPRFC4 (sprfc4.f), the Cholesky form of SPRFC3: rigid-body pivots of a
    free box replaced by +TOL(1) max(1, |TOL(4) a_jj|) (IERR -3, MSPAR(27) = -6,
    a complete factor); an indefinite shift stopped at its first pivot below
    -TOL(1)|a_jj| (MSPAR(27) = that equation); an SPD box; a zero diagonal."""
    rs, sm = ref_system(4, clamp=False)
    r = run_sprfc4('ref', rs, sm, 1e-8, 1e-2)
    o = run_sprfc4('orc', rs, sm, 1e-8, 1e-2)
    _same(r, o)
    assert o['ierr'] == -3 and o['mspar'][26] == -6 and o['mspar'][0] == 6
    assert np.count_nonzero(o['dcor'][:, 1]) == 6 and np.all(o['dcor'][:, 1] >= 0.0)
    rs3, sm3 = ref_system(3)
    from scipy.linalg import eigh
    K = dense_from_sm(rs3, sm3)
    M = np.diag(K.diagonal() - dense_from_sm(rs3, shifted_sm(rs3, sm3, 1.0)).diagonal())
    w = eigh(K, M, eigvals_only=True)
    ssm = shifted_sm(rs3, sm3, 0.5 * (w[3] + w[4]))
    r = run_sprfc4('ref', rs3, ssm, 1e-12, 1.0)
    o = run_sprfc4('orc', rs3, ssm, 1e-12, 1.0)
    _same(r, o)
    assert o['ierr'] == -3 and o['mspar'][26] > 0 and o['tol'][1] < 0.0
    r = run_sprfc4('ref', rs3, sm3, 1e-12, 1.0)
    o = run_sprfc4('orc', rs3, sm3, 1e-12, 1.0)
    _same(r, o)
    assert o['ierr'] == 0 and not np.any(o['dcor'])
    from sam_lib_b200.system import diag_positions
    z = sm3.copy()
    z[diag_positions(rs3.mspar, rs3.mtrees, rs3.msifa)[20]] = 0.0
    r = run_sprfc4('ref', rs3, z, 1e-12, 1.0)
    o = run_sprfc4('orc', rs3, z, 1e-12, 1.0)
    _same(r, o)
    assert o['dcor'][20, 1] == 1.0
