"""Failure detection on the GPU, in forms that fault, trap or hang nothing.

* NaN in an element matrix: the NaN reaches a pivot through the Schur
  updates; the pivot test treats a non-finite pivot as failed, so SPRSOL
  returns IERR = -3 (MSPAR(1) = -5 is not set: -3 is the reference's
  pivot-failure code, sprfc1.f:251-265) instead of a factor full of NaN.
* Watchdog of the tensor-core update: with a short wait limit and the test
  switch that makes one CTA skip its first operand load, that CTA's bounded
  mbarrier waits run out; the kernel frees its tensor memory and returns,
  the factorisation reports -4, and the next factorisation on the same
  engine is correct.
* Residency of the device factor: a host edit of one factor entry between
  SPRFC1 and SPRFS1/SPRBS1 is seen (full content hash), so the solves use
  the edited factor, as the reference's would.
* MVMULT/MMMULT: the reference's own LMVY18/LMMY18 pass the probe and the
  factor equals the one with null callbacks.
"""
import ctypes as C

import numpy as np
import pytest

import sam_lib_b200 as spr
from conftest import ref_system
from test_oracle import run_sprsol, rhs
from test_gpu_parity import gpu_sprsol, close_factor, relerr

pytestmark = pytest.mark.gpu


def test_nan_in_element_matrix_is_an_error():
    from oracle.refpipe import RefSystem
    from sam_lib_b200.fe import HexBox, hex8_stiffness
    rs = RefSystem(HexBox(4))
    ke = hex8_stiffness()
    bad = ke.copy()
    bad[5, 7] = bad[7, 5] = np.nan
    sm = rs.assemble(lambda e: bad if e == 17 else ke)
    assert np.isnan(sm).any()
    g = gpu_sprsol(rs, sm, rhs(rs.neq, 1, 2))
    assert g['ierr'] == -3, g['ierr']
    assert 1 <= g['mspar'][26] <= rs.neq            # MSPAR(27): the equation that failed


def test_watchdog_timeout_is_reported_and_engine_stays_usable():
    import torch
    rs, sm = ref_system(12)
    ds = spr.DeviceSolver(rs.mspar, rs.mtrees, rs.msifa)
    st = torch.cuda.Stream()
    ds.set_stream(st.cuda_stream)
    d0 = torch.from_numpy(sm).cuda()
    ds.set_mode(1)                                   # tensor-core updates
    ds.set_watchdog(0.05, drop=True)
    d = d0.clone()
    with pytest.raises(RuntimeError, match='-4'):
        ds.factor(d)
    ds.set_watchdog(2.0, drop=False)
    d = d0.clone()
    r = ds.factor(d)
    assert r['lierr'] == 0 and r['numneg'] == 0
    ds.set_mode(0)
    d64 = d0.clone()
    r64 = ds.factor(d64)
    assert r64['lierr'] == 0
    dmax = float((d - d64).abs().max() / d64.abs().max())
    assert 0.0 < dmax <= 1e-5, dmax                   # the mixed factor ran, and correctly
    ds.close()


def test_solve_watchdog_timeout_is_reported_and_engine_stays_usable():
    """One task of each solve triangle launch never reports its block: the
    tasks waiting for it give up after the short limit, the solve returns -4,
    and the next solve on the same engine is correct."""
    import torch
    rs, sm = ref_system(12)
    ds = spr.DeviceSolver(rs.mspar, rs.mtrees, rs.msifa)
    d = torch.from_numpy(sm).cuda()
    ds.factor(d)
    b = rhs(rs.neq, 2, 6)
    d_b0 = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    ds.set_watchdog(0.05, drop=True)
    d_b = d_b0.clone()
    with pytest.raises(RuntimeError, match='-4'):
        ds.solve(d, d_b, 2)
    ds.set_watchdog(2.0, drop=False)
    d_b = d_b0.clone()
    ds.solve(d, d_b, 2)
    o = run_sprsol('orc', rs, sm, b)
    assert relerr(d_b.cpu().numpy().T, o['b']) <= 1e-9
    ds.close()


def test_edit_of_the_factor_between_calls_is_seen():
    rs, sm = ref_system(6, 'loguniform')
    b = rhs(rs.neq, 2, 9)
    g = gpu_sprsol(rs, sm, b, iop=1)
    assert g['ierr'] == 0
    fsm = g['sm'].copy()
    k = rs.neq + 11                                   # one entry of L
    fsm[k] *= 1.5
    msp = g['mspar'].copy()
    B = np.asfortranarray(b.copy())
    assert spr.sprfs1(msp, rs.mtrees, rs.msifa, fsm, B, rs.neq, 2) == 0
    assert spr.sprbs1(msp, rs.mtrees, rs.msifa, fsm, B, rs.neq, 2) == 0
    o = run_sprsol('orc', rs, fsm, b, iop=4)          # the reference's solves on the edited factor
    assert relerr(B, o['b']) <= 1e-9
    u = run_sprsol('orc', rs, g['sm'], b, iop=4)      # ... which differ from the unedited ones
    assert relerr(o['b'], u['b']) > 1e-6


def test_reference_callbacks_give_the_same_factor():
    from oracle.refpipe import lib as reflib
    rs, sm = ref_system(6)
    msp = rs.mspar.copy()
    s1 = sm.copy()
    tol = np.array([1e-12, 0.0, 0.0])
    assert spr.sprfc1(msp, rs.mtrees, rs.msifa, s1, tol) == 0
    lib = spr.load(8)
    msp2 = rs.mspar.copy()
    s2 = sm.copy()
    tol2 = np.array([1e-12, 0.0, 0.0])
    ierr = C.c_int64(0)
    mv = C.cast(reflib().lmvy18_, C.c_void_p)
    mm = C.cast(reflib().lmmy18_, C.c_void_p)
    lib.sprfc1_(spr._ptr(msp2), spr._ptr(rs.mtrees), spr._ptr(rs.msifa), spr._ptr(s2), spr._ptr(tol2),
                spr._ptr(np.zeros(1, dtype=np.int64)), spr._ptr(np.zeros(1)), C.byref(C.c_int64(-1)),
                C.byref(ierr), mv, mm)
    assert ierr.value == 0
    assert np.array_equal(s1, s2) and np.array_equal(msp, msp2)
