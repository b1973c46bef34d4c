"""GPU parity: the C-ABI entry points against the oracle on the same inputs.

Every case calls the product through the Fortran ABI (sprsol_/sprfc1_/
sprfs1_/sprbs1_ of libspr_b200.so) with the structures produced by the
reference host pipeline, and compares with the oracle restatement (which is
itself pinned bitwise to the reference in test_oracle.py).

Tolerances (FP64, different summation order than the reference):
  factor  : max |SM_gpu - SM_oracle| <= 1e-10 * max |SM_oracle|
  solution: ||x_gpu - x_oracle|| / ||x_oracle|| <= 1e-9 (E = 1) or 1e-6
            (log-uniform E over four decades, condition number ~1e9)
  inertia : NUMNEG (MSPAR(26)) bit-exact; IERR, MSPAR(1), MSPAR(27) exact
"""
import ctypes as C

import numpy as np
import pytest

import sam_lib_b200 as spr
from conftest import ref_system, shifted_sm, dense_from_sm
from test_oracle import run_sprsol, rhs

pytestmark = pytest.mark.gpu


def gpu_sprsol(rs, sm, b, iop=3, tol1=1e-12, mspar=None, ldb=None):
    sm = sm.copy()
    nrhs = 1 if b.ndim == 1 else b.shape[1]
    ldb = rs.neq if ldb is None else ldb
    B = np.zeros((ldb, nrhs), order='F')
    B[:rs.neq, :] = b.reshape(rs.neq, nrhs)
    msp = rs.mspar.copy() if mspar is None else mspar.copy()
    tol = np.array([tol1, 0.0, 0.0])
    ierr = spr.sprsol(iop, msp, rs.mtrees, rs.msifa, sm, B, ldb, nrhs, tol)
    return dict(sm=sm, b=B[:rs.neq], tol=tol, ierr=ierr, mspar=msp)


def close_factor(a, b, rtol=1e-10):
    return np.max(np.abs(a - b)) <= rtol * np.max(np.abs(b))


def relerr(x, y):
    return np.linalg.norm(x - y) / np.linalg.norm(y)


@pytest.mark.parametrize('n,emod,nrhs', [(3, 'uniform', 1), (6, 'uniform', 3), (6, 'loguniform', 2),
                                         (12, 'uniform', 1), (12, 'loguniform', 4)])
def test_sprsol_factor_and_solve_match_oracle(n, emod, nrhs):
    rs, sm = ref_system(n, emod)
    b = rhs(rs.neq, nrhs, 10 + n)
    o = run_sprsol('orc', rs, sm, b)
    g = gpu_sprsol(rs, sm, b)
    assert g['ierr'] == o['ierr'] == 0
    assert np.array_equal(g['mspar'], o['mspar'])
    assert close_factor(g['sm'], o['sm'])
    assert relerr(g['b'], o['b']) <= (1e-9 if emod == 'uniform' else 1e-6)
    assert abs(g['tol'][1] - o['tol'][1]) <= 1e-10 * abs(o['tol'][1])
    assert abs(g['tol'][2] - o['tol'][2]) <= 1e-10 * abs(o['tol'][2])


def test_config1_residual_and_reference_difference():
    """12^3 box, one RHS U[-1,1] seed 0: ||Ku-f||/||f|| and max rel. diff vs the reference."""
    rs, sm = ref_system(12)
    f = np.random.default_rng(0).uniform(-1.0, 1.0, size=(rs.neq, 1))
    r = run_sprsol('ref', rs, sm, f)
    g = gpu_sprsol(rs, sm, f)
    K = dense_from_sm(rs, sm)
    res = np.linalg.norm(K @ g['b'] - f) / np.linalg.norm(f)
    assert res < 1e-12
    assert np.max(np.abs(g['b'] - r['b'])) / np.max(np.abs(r['b'])) < 1e-10


def test_factor_then_separate_solves_reuse_device_factor():
    rs, sm = ref_system(6, 'loguniform')
    b = rhs(rs.neq, 2, 3)
    o = run_sprsol('orc', rs, sm, b)
    g1 = gpu_sprsol(rs, sm, b, iop=1)
    assert g1['ierr'] == 0
    # IOP=4 on the factored SM; then forward and back through SPRFS1/SPRBS1
    g2 = gpu_sprsol(rs, g1['sm'], b, iop=4)
    assert relerr(g2['b'], o['b']) < 1e-6
    fsm = g1['sm'].copy()
    B = np.asfortranarray(b.copy())
    msp = rs.mspar.copy()
    assert spr.sprfs1(msp, rs.mtrees, rs.msifa, fsm, B, rs.neq, 2) == 0
    y = run_sprsol('orc', rs, o['sm'], b, iop=5)['b']
    assert relerr(B, y) < 1e-6
    assert spr.sprbs1(msp, rs.mtrees, rs.msifa, fsm, B, rs.neq, 2) == 0
    assert relerr(B, o['b']) < 1e-6
    assert msp[0] == 7


def test_ldb_larger_than_neq():
    rs, sm = ref_system(6)
    b = rhs(rs.neq, 3, 4)
    o = run_sprsol('orc', rs, sm, b)
    g = gpu_sprsol(rs, sm, b, ldb=rs.neq + 5)
    assert relerr(g['b'], o['b']) < 1e-9


def test_indefinite_shift_inertia_exact():
    from scipy.linalg import eigh
    for n, k in ((3, 4), (6, 11)):
        rs, sm = ref_system(n)
        K = dense_from_sm(rs, sm)
        M = np.diag(K.diagonal() - dense_from_sm(rs, shifted_sm(rs, sm, 1.0)).diagonal())
        w = eigh(K, M, eigvals_only=True)
        sigma = 0.5 * (w[k - 1] + w[k])
        ssm = shifted_sm(rs, sm, sigma)
        b = rhs(rs.neq, 1, 5)
        o = run_sprsol('orc', rs, ssm, b, iop=1)
        g = gpu_sprsol(rs, ssm, b, iop=1)
        assert o['ierr'] == g['ierr'] == 3
        assert o['mspar'][25] == g['mspar'][25] == k
        assert close_factor(g['sm'], o['sm'], 1e-8)


def test_error_codes_match_oracle():
    rs, sm = ref_system(6)
    b = rhs(rs.neq, 1, 6)
    bad = rs.mspar.copy()
    bad[0] = -3
    o = run_sprsol('orc', rs, sm, b, mspar=bad)
    g = gpu_sprsol(rs, sm, b, mspar=bad)
    assert g['ierr'] == o['ierr'] == -1 and g['mspar'][0] == o['mspar'][0] == -5
    # exact zero diagonal
    z = sm.copy()
    sp = rs.mspar
    p = int(rs.msifa[sp[47] - 1 + 7])
    z[rs.neq + p - 1] = 0.0
    o = run_sprsol('orc', rs, z, b, iop=1)
    g = gpu_sprsol(rs, z, b, iop=1)
    assert g['ierr'] == o['ierr'] == -3
    assert g['mspar'][26] == o['mspar'][26] and g['mspar'][25] == o['mspar'][25]
    assert np.array_equal(g['sm'][:rs.neq], o['sm'][:rs.neq])
    # pivot failure
    for tol1 in (0.9, 0.5):
        o = run_sprsol('orc', rs, sm, b, iop=3, tol1=tol1)
        g = gpu_sprsol(rs, sm, b, iop=3, tol1=tol1)
        assert g['ierr'] == o['ierr'] == -3
        assert g['mspar'][26] == o['mspar'][26]
        assert g['mspar'][25] == o['mspar'][25]
        assert np.allclose(g['tol'], o['tol'], rtol=1e-10, atol=0)


def test_partial_factorisation_without_retained_dofs_is_a_full_factor():
    """MSPAR(57) = 1 on a structure without external DOFs (no SUPSUP > 0):
    nothing is retained, so factor and solution are the full ones."""
    rs, sm = ref_system(3)
    msp = rs.mspar.copy()
    msp[56] = 1
    b = rhs(rs.neq, 1, 7)
    o = run_sprsol('orc', rs, sm, b, mspar=msp)
    g = gpu_sprsol(rs, sm, b, mspar=msp)
    assert g['ierr'] == o['ierr'] == 0
    assert np.array_equal(g['mspar'], o['mspar'])
    assert close_factor(g['sm'], o['sm'])
    assert relerr(g['b'], o['b']) <= 1e-9


def test_pivot_failure_inside_a_dense_front():
    """A pivot driven to zero inside the largest (dense-path) front: IERR -3,
    the failing equation (MSPAR(27)), NUMNEG of the columns before it and
    TOL(2:3) as the oracle reports them (SPRF17's test, sprfc1.f:1272-1294)."""
    from sam_lib_b200.system import diag_positions
    rs, sm = ref_system(8)
    sp = rs.mspar
    ns = int(sp[10])
    xs = rs.mtrees[sp[44] - 1: sp[44] + ns]
    xl = rs.mtrees[sp[45] - 1: sp[45] + ns]
    F = np.diff(xl)
    js = int(np.argmax(F))
    assert F[js] > 176                       # a dense-path front
    j = int(xs[js] - 1 + (xs[js + 1] - xs[js]) // 2)
    pos = diag_positions(rs.mspar, rs.mtrees, rs.msifa)
    o1 = run_sprsol('orc', rs, sm, rhs(rs.neq, 1, 8), iop=1)
    z = sm.copy()
    z[pos[j]] -= o1['sm'][pos[j]]            # the pivot of column j becomes (nearly) zero
    b = rhs(rs.neq, 1, 8)
    o = run_sprsol('orc', rs, z, b, iop=1, tol1=1e-8)
    g = gpu_sprsol(rs, z, b, iop=1, tol1=1e-8)
    assert o['ierr'] == g['ierr'] == -3
    assert g['mspar'][26] == o['mspar'][26] == j + 1
    assert g['mspar'][25] == o['mspar'][25]
    # TOL(3) is the column's original diagonal; TOL(2) the failing pivot, a
    # rounding-level remainder whose value depends on the summation order
    assert abs(g['tol'][2] - o['tol'][2]) <= 1e-12 * abs(o['tol'][2])
    assert abs(g['tol'][1]) <= 1e-8 * abs(o['tol'][2])


def test_integer4_abi_matches_oracle():
    """libspr_b200_i4.so (INTEGER*4 build) through sprsol_ gives the INTEGER*8 results."""
    rs, sm = ref_system(6, 'loguniform')
    b = rhs(rs.neq, 2, 9)
    o = run_sprsol('orc', rs, sm, b)
    sm4 = sm.copy()
    B = np.asfortranarray(b.copy())
    msp4 = rs.mspar.astype(np.int32)
    tol = np.array([1e-12, 0.0, 0.0])
    ierr = spr.sprsol(3, msp4, rs.mtrees.astype(np.int32), rs.msifa.astype(np.int32), sm4, B, rs.neq, 2, tol,
                      int_kind=4)
    assert ierr == o['ierr'] == 0
    assert np.array_equal(msp4.astype(np.int64), o['mspar'])
    assert close_factor(sm4, o['sm'])
    assert relerr(B, o['b']) <= 1e-6
