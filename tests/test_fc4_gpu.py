"""GPU parity of SPRFC4 (src/SPR/sprfc4.f): the Cholesky factorisation C C'
with SPRF47's pivot replacement, through sprfc4_ of libspr_b200.so, against
the oracle (pinned bitwise to the reference in test_oracle.py), and the
C C' sweeps SPRFS2/SPRBS2 on the factor it leaves.

Tolerances:
  deterministic replacements (pivots with a clear margin to TOL(1)|a_jj|):
    IERR, MSPAR, replaced equations exact; factor, DCOR, TOL(2:3) within
    1e-10 relative; solutions within 1e-9
  rigid-body modes of a free box (pivots at rounding level): the replaced
    equations and DCOR(2,j) exact, C C' = K + diag(DCOR(2,j) - DCOR(1,j)) to
    1e-10 of max|K|
  a negative pivot: the stopping equation MSPAR(27), TOL(3) = its a_jj and
    DCOR(1:2, j) = TOL(2) = its pivot (to 1e-9 of |a_jj|)
"""
import numpy as np
import pytest

import sam_lib_b200 as spr
from conftest import ref_system, shifted_sm, dense_from_sm
from test_oracle import run_sprfc4, run_chol, rhs
from test_gpu_parity import relerr

pytestmark = pytest.mark.gpu


def gpu_sprfc4(rs, sm, tol1, tol4, mspar=None):
    sm = sm.copy()
    msp = rs.mspar.copy() if mspar is None else mspar.copy()
    tol = np.array([tol1, 0.0, 0.0, tol4])
    dcor = np.full(2 * rs.neq, 7.0)
    ierr = spr.sprfc4(msp, rs.mtrees, rs.msifa, sm, tol, dcor)
    return dict(sm=sm, tol=tol, dcor=dcor.reshape(-1, 2), ierr=ierr, mspar=msp)


def _cct_defect(rs, K, g):
    rep = np.nonzero(g['dcor'][:, 1])[0]
    Cf = dense_from_sm(rs, g['sm'])
    Cm = np.tril(Cf)
    delta = np.zeros(rs.neq)
    delta[rep] = g['dcor'][rep, 1] - g['dcor'][rep, 0]
    return np.max(np.abs(Cm @ Cm.T - (K + np.diag(delta)))) / np.max(np.abs(K))


@pytest.mark.parametrize('n', [4, 8])
def test_sprfc4_rigid_body_modes(n):
    """Free box: six rounding-level pivots replaced, in the small-front kernel
    (4^3) and the dense diagonal-block kernel (8^3)."""
    rs, sm = ref_system(n, clamp=False)
    o = run_sprfc4('orc', rs, sm, 1e-8, 1e-2)
    g = gpu_sprfc4(rs, sm, 1e-8, 1e-2)
    assert g['ierr'] == o['ierr'] == -3
    assert g['mspar'][0] == o['mspar'][0] == 6
    assert g['mspar'][26] == o['mspar'][26] == -6
    assert g['mspar'][25] == o['mspar'][25] == 0
    rep_o = np.nonzero(o['dcor'][:, 1])[0]
    rep_g = np.nonzero(g['dcor'][:, 1])[0]
    assert np.array_equal(rep_g, rep_o)
    np.testing.assert_array_equal(g['dcor'][rep_g, 1], o['dcor'][rep_o, 1])
    keep = np.ones(rs.neq, dtype=bool)
    keep[rep_g] = False
    assert not np.any(g['dcor'][keep])
    assert _cct_defect(rs, dense_from_sm(rs, sm), g) <= 1e-10


def test_sprfc4_threshold_replacements_and_sweeps_match_oracle():
    """TOL(1) = 0.6 on the clamped 8^3 box: the 8 regular pivots below 0.6 a_jj
    are replaced by 0.6 max(1, |TOL(4) a_jj|); then SPRFS2 + SPRBS2 on that factor."""
    rs, sm = ref_system(8)
    tol1, tol4 = 0.6, 0.5
    o = run_sprfc4('orc', rs, sm, tol1, tol4)
    g = gpu_sprfc4(rs, sm, tol1, tol4)
    rep = np.nonzero(o['dcor'][:, 1])[0]
    assert len(rep) >= 5          # pivots at 0.552..0.598 a_jj; the others at >= 0.605 a_jj
    assert g['ierr'] == o['ierr'] == -3
    assert np.array_equal(g['mspar'], o['mspar'])
    assert np.array_equal(np.nonzero(g['dcor'][:, 1])[0], rep)
    assert np.max(np.abs(g['sm'] - o['sm'])) <= 1e-10 * np.max(np.abs(o['sm']))
    assert np.max(np.abs(g['dcor'] - o['dcor'])) <= 1e-10 * np.max(np.abs(o['dcor']))
    for k in (1, 2):
        assert abs(g['tol'][k] - o['tol'][k]) <= 1e-10 * abs(o['tol'][k])
    b = rhs(rs.neq, 2, 41)
    ro = run_chol('orc', rs, o['sm'], b, mspar=o['mspar'], steps='sb')
    B = np.asfortranarray(b.copy())
    msp = g['mspar'].copy()
    msp[0] = 6
    assert spr.sprfs2(msp, rs.mtrees, rs.msifa, g['sm'], B, rs.neq, 2) == 0
    assert spr.sprbs2(msp, rs.mtrees, rs.msifa, g['sm'], B, rs.neq, 2) == 0
    assert relerr(B, ro['b']) <= 1e-9


def test_sprfc4_negative_pivot_stops():
    rs, sm = ref_system(3)
    ssm = shifted_sm(rs, sm, 0.12)
    o = run_sprfc4('orc', rs, ssm, 1e-12, 1.0)
    g = gpu_sprfc4(rs, ssm, 1e-12, 1.0)
    assert g['ierr'] == o['ierr'] == -3
    j = int(o['mspar'][26])
    assert j > 0 and g['mspar'][26] == j
    assert g['mspar'][0] == o['mspar'][0] and g['mspar'][25] == o['mspar'][25] == 0
    assert g['tol'][2] == o['tol'][2]                     # a_jj of the stopping equation
    assert abs(g['tol'][1] - o['tol'][1]) <= 1e-9 * abs(o['tol'][2])
    assert abs(g['dcor'][j - 1, 0] - o['dcor'][j - 1, 0]) <= 1e-9 * abs(o['tol'][2])
    assert g['dcor'][j - 1, 0] == g['dcor'][j - 1, 1] < 0


def test_sprfc4_zero_diagonal_and_spd_box():
    rs, sm = ref_system(3)
    o = run_sprfc4('orc', rs, sm, 1e-12, 1.0)
    g = gpu_sprfc4(rs, sm, 1e-12, 1.0)
    assert g['ierr'] == o['ierr'] == 0 and np.array_equal(g['mspar'], o['mspar'])
    assert np.max(np.abs(g['sm'] - o['sm'])) <= 1e-10 * np.max(np.abs(o['sm']))
    from sam_lib_b200.system import diag_positions
    z = sm.copy()
    pos = diag_positions(rs.mspar, rs.mtrees, rs.msifa)
    z[pos[7]] = 0.0
    o = run_sprfc4('orc', rs, z, 1e-12, 1.0)
    g = gpu_sprfc4(rs, z, 1e-12, 1.0)
    assert g['ierr'] == o['ierr'] and np.array_equal(g['mspar'], o['mspar'])
    assert g['dcor'][7, 1] == o['dcor'][7, 1] == 1.0
    assert np.max(np.abs(g['sm'] - o['sm'])) <= 1e-10 * np.max(np.abs(o['sm']))
    assert np.max(np.abs(g['dcor'] - o['dcor'])) <= 1e-10 * max(1.0, np.max(np.abs(o['dcor'])))
