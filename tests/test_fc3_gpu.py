"""GPU parity of SPRFC3 (src/SPR/sprfc3.f): the factorisation that replaces
singular pivots instead of stopping, through sprfc3_ of libspr_b200.so and
the device entry point spr_b200_factor3_dev, against the oracle (pinned
bitwise to the reference in test_oracle.py).

Tolerances:
  deterministic replacements (pivots with a clear margin to TOL(1)):
    IERR, MSPAR, replaced equations exact; factor, DCOR and TOL(2:3)
    within 1e-10 relative
  rigid-body modes (pivots at rounding level, their sign is noise): the
    replaced equations and |DCOR(2,j)| exact; the factor satisfies
    L D L' = K + diag(DCOR(2,j) - DCOR(1,j)) to 1e-10 of max|K|
"""
import numpy as np
import pytest

import sam_lib_b200 as spr
from conftest import ref_system, shifted_sm, dense_from_sm
from test_oracle import run_sprfc3, run_sprsol, rhs
from test_gpu_parity import close_factor, relerr, gpu_sprsol

pytestmark = pytest.mark.gpu


def gpu_sprfc3(rs, sm, tol1, tol4, mspar=None):
    sm = sm.copy()
    msp = rs.mspar.copy() if mspar is None else mspar.copy()
    tol = np.array([tol1, 0.0, 0.0, tol4])
    dcor = np.full(2 * rs.neq, 7.0)
    ierr = spr.sprfc3(msp, rs.mtrees, rs.msifa, sm, tol, dcor)
    return dict(sm=sm, tol=tol, dcor=dcor.reshape(-1, 2), ierr=ierr, mspar=msp)


def _front_order_of_columns(rs):
    sp = rs.mspar
    ns = int(sp[10])
    xs = rs.mtrees[sp[44] - 1: sp[44] + ns]
    xl = rs.mtrees[sp[45] - 1: sp[45] + ns]
    return np.repeat(np.diff(xl), np.diff(xs))


def _ldlt_defect(rs, K, g):
    """max |L D L' - (K + diag(delta))| / max |K| for the GPU factor g."""
    rep = np.nonzero(g['dcor'][:, 1])[0]
    Lf = dense_from_sm(rs, g['sm'])
    L = np.tril(Lf, -1) + np.eye(rs.neq)
    D = g['sm'][:rs.neq]
    delta = np.zeros(rs.neq)
    delta[rep] = g['dcor'][rep, 1] - g['dcor'][rep, 0]
    return np.max(np.abs((L * D) @ L.T - (K + np.diag(delta)))) / np.max(np.abs(K))


@pytest.mark.parametrize('n', [3, 8])
def test_sprfc3_rigid_body_modes(n):
    """Free box: six rounding-level pivots replaced by +-TOL(1) max(1, |TOL(4) a_jj|),
    in the one-CTA small-front kernel (3^3, root F = 66) and in the dense
    diagonal-block kernel (8^3, root F = 354)."""
    rs, sm = ref_system(n, clamp=False)
    o = run_sprfc3('orc', rs, sm, 1e-8, 1e-2)
    g = gpu_sprfc3(rs, sm, 1e-8, 1e-2)
    assert g['ierr'] == o['ierr'] == -3
    assert g['mspar'][0] == o['mspar'][0] == 5
    assert g['mspar'][26] == o['mspar'][26] == -6
    rep_o = np.nonzero(o['dcor'][:, 1])[0]
    rep_g = np.nonzero(g['dcor'][:, 1])[0]
    assert np.array_equal(rep_g, rep_o)
    assert np.all(_front_order_of_columns(rs)[rep_g] == (66 if n == 3 else 354))
    np.testing.assert_array_equal(np.abs(g['dcor'][rep_g, 1]), np.abs(o['dcor'][rep_o, 1]))
    # every other DCOR entry: DCOR(1) zero (no negative pivot), DCOR(2) zero
    keep = np.ones(rs.neq, dtype=bool)
    keep[rep_g] = False
    assert not np.any(g['dcor'][keep])
    # the inertia apart from the replaced pivots, whose signs are rounding noise
    assert g['mspar'][25] - np.sum(g['dcor'][rep_g, 1] < 0) == 0
    assert o['mspar'][25] - np.sum(o['dcor'][rep_o, 1] < 0) == 0
    assert _ldlt_defect(rs, dense_from_sm(rs, sm), g) <= 1e-10


def test_sprfc3_threshold_replacements_match_oracle():
    """TOL(1) = 0.65 on the 8^3 box: 62 regular pivots (53 in dense fronts)
    fall below the threshold with a margin of 4.7e-4 and are replaced; every
    later column sees the modified pivots.  The factor then solves through
    SPRFS1/SPRBS1 like the oracle's."""
    rs, sm = ref_system(8)
    tol1, tol4 = 0.65, 0.5
    o = run_sprfc3('orc', rs, sm, tol1, tol4)
    g = gpu_sprfc3(rs, sm, tol1, tol4)
    assert g['ierr'] == o['ierr'] == -3
    assert np.array_equal(g['mspar'], o['mspar'])
    assert o['mspar'][26] == -62
    rep_o = np.nonzero(o['dcor'][:, 1])[0]
    assert np.array_equal(np.nonzero(g['dcor'][:, 1])[0], rep_o)
    assert np.sum(_front_order_of_columns(rs)[rep_o] > 176) == 53
    assert close_factor(g['sm'], o['sm'])
    assert close_factor(g['dcor'], o['dcor'])
    assert abs(g['tol'][1] - o['tol'][1]) <= 1e-10 * abs(o['tol'][1])
    assert abs(g['tol'][2] - o['tol'][2]) <= 1e-10 * abs(o['tol'][2])
    # solves on the completed factor (MSPAR(1) = 5 after IERR = -3)
    b = rhs(rs.neq, 2, 21)
    os_ = run_sprsol('orc', rs, o['sm'], b, iop=4, mspar=o['mspar'])
    gs = gpu_sprsol(rs, g['sm'], b, iop=4, mspar=g['mspar'])
    assert gs['ierr'] == os_['ierr'] == 0
    assert relerr(gs['b'], os_['b']) <= 1e-9


def test_sprfc3_zero_diagonal_and_negative_pivots():
    """A zero diagonal becomes 1 (DCOR(2,j) = 1) and an indefinite shift puts
    its negative pivots in DCOR(1,j); IERR = 3 with the oracle's inertia."""
    from sam_lib_b200.system import diag_positions
    from scipy.linalg import eigh
    rs, sm = ref_system(6)
    K = dense_from_sm(rs, sm)
    M = np.diag(K.diagonal() - dense_from_sm(rs, shifted_sm(rs, sm, 1.0)).diagonal())
    w = eigh(K, M, eigvals_only=True)
    ssm = shifted_sm(rs, sm, 0.5 * (w[7] + w[8]))     # a gap of 11 %: pivots >= 0.06 |a_jj|
    o = run_sprfc3('orc', rs, ssm, 1e-12, 1.0)
    g = gpu_sprfc3(rs, ssm, 1e-12, 1.0)
    assert g['ierr'] == o['ierr'] == 3
    assert np.array_equal(g['mspar'], o['mspar'])
    assert g['mspar'][25] == 8
    neg = np.nonzero(o['dcor'][:, 0])[0]
    assert len(neg) == 8
    assert np.array_equal(np.nonzero(g['dcor'][:, 0])[0], neg)
    assert close_factor(g['dcor'], o['dcor'])
    assert close_factor(g['sm'], o['sm'])
    pos = diag_positions(rs.mspar, rs.mtrees, rs.msifa)
    z = sm.copy()
    j = rs.neq - 40
    z[pos[j]] = 0.0
    o = run_sprfc3('orc', rs, z, 1e-12, 1.0)
    g = gpu_sprfc3(rs, z, 1e-12, 1.0)
    assert g['ierr'] == o['ierr']
    assert np.array_equal(g['mspar'], o['mspar'])
    assert g['dcor'][j, 1] == o['dcor'][j, 1] == 1.0
    assert close_factor(g['dcor'], o['dcor'])
    assert close_factor(g['sm'], o['sm'])
    # preceding error not cleared (sprfc3.f:139-143)
    bad = rs.mspar.copy()
    bad[0] = -2
    g = gpu_sprfc3(rs, sm, 1e-12, 1.0, mspar=bad)
    assert g['ierr'] == -1 and g['mspar'][0] == -5


def test_factor3_device_entry_matches_fortran_entry():
    """spr_b200_factor3_dev on torch buffers equals sprfc3_ on host arrays."""
    import torch
    rs, sm = ref_system(8)
    h = gpu_sprfc3(rs, sm, 0.65, 0.5)
    ds = spr.DeviceSolver(rs.mspar, rs.mtrees, rs.msifa)
    d_sm = torch.from_numpy(sm.copy()).cuda()
    d_dcor = torch.zeros(2 * rs.neq, dtype=torch.float64, device='cuda')
    r = ds.factor3(d_sm, d_dcor, 0.65, 0.5)
    torch.cuda.synchronize()
    assert r['lierr'] == -31 and r['supeqt'] == -h['mspar'][26] == 62
    assert r['numneg'] == h['mspar'][25]
    assert np.array_equal(d_sm.cpu().numpy(), h['sm'])
    assert np.array_equal(d_dcor.cpu().numpy().reshape(-1, 2), h['dcor'])
    assert r['tol2'] == h['tol'][1] and r['tol3'] == h['tol'][2]
