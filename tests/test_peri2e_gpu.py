"""The PERI2E solve path (MSPAR(58) >= 1) against the reference (GPU).

SPRABC (sprabc.f:5-66) writes the internal->external permutation PERI2E and
its inverse first in MSIFA and sets MSPAR(58) = 2; SPRSMB and SPRPMP then
place LINDX and XLNZ 2*NEQ further on (sprsmb.f:181, sprpmp.f:47-48).  The
structure here is built the same way from the reference pipeline's arrays,
with a seeded permutation, and B is given in the external numbering.  The
reference (the translated SPR, which runs SPRFS4/SPRFB3/SPRFB4 and SPRBS5,
sprfs1.f:396-900, sprbs1.f:371-495) is compared with the GPU library on:
  * a full solve (MSPAR(57) = 0) with every equation permuted;
  * a partial factorisation (MSPAR(57) = 1, face x=n retained) with LDB =
    the number of internal equations, internal equations permuted among
    themselves: the internal solution for zero retained displacements;
  * the same with one internal equation numbered beyond LDB: the library
    refuses it (IERR = -4), since its sweeps would not drop that row's
    updates as SPRFB3/SPRFB4 do inside every supernode.
"""
import ctypes as C

import numpy as np
import pytest

import sam_lib_b200 as spr
from conftest import ref_system
from test_oracle import rhs, retained_info
from test_gpu_parity import relerr

pytestmark = pytest.mark.gpu


def with_peri2e(rs, peri2e):
    """(MSPAR, MSIFA) of the structure with PERI2E (1-based, internal -> external)."""
    neq = rs.neq
    pere2i = np.empty(neq, dtype=np.int64)
    pere2i[peri2e - 1] = np.arange(1, neq + 1)
    ms = rs.mspar.copy()
    nmsifa = int(ms[2])
    msifa = np.concatenate([peri2e.astype(np.int64), pere2i, rs.msifa[:nmsifa]]).astype(np.int64)
    ms[57] = 2
    ms[46] += 2 * neq
    ms[47] += 2 * neq
    ms[2] += 2 * neq
    return ms, msifa


def ref_sprsol(rs, ms, msifa, sm, b, ldb, iop=3):
    from oracle.refpipe import lib as reflib, _p, _i
    sm = sm.copy()
    b = np.asfortranarray(b.copy())
    msp = ms.copy()
    tol = np.array([1e-12, 0.0, 0.0])
    iw = np.zeros(int(ms[13]) + int(ms[12]) + 8, dtype=np.int64)
    rw = np.zeros(int(ms[16]) + int(ms[13]) + 8)
    ierr = C.c_int64(0)
    reflib().sprsol_(_i(iop), _p(msp), _p(rs.mtrees), _p(msifa), _p(sm), _p(b), _i(ldb), _i(b.shape[1]),
                     _p(tol), _p(iw), _p(rw), _i(-1), C.byref(ierr))
    return ierr.value, msp, sm, b


def gpu_sprsol(rs, ms, msifa, sm, b, ldb, iop=3):
    sm = sm.copy()
    b = np.asfortranarray(b.copy())
    msp = ms.copy()
    tol = np.array([1e-12, 0.0, 0.0])
    ierr = spr.sprsol(iop, msp, rs.mtrees, msifa, sm, b, ldb, b.shape[1], tol)
    return ierr, msp, sm, b


@pytest.mark.parametrize('n,emod', [(6, 'uniform'), (8, 'loguniform')])
def test_peri2e_full_solve_matches_reference(n, emod):
    rs, sm = ref_system(n, emod)
    peri2e = np.random.default_rng(n).permutation(rs.neq) + 1
    ms, msifa = with_peri2e(rs, peri2e)
    b = rhs(rs.neq, 3, 70 + n)                       # external numbering
    ri, rm, rsm, rb = ref_sprsol(rs, ms, msifa, sm, b, rs.neq)
    gi, gm, gsm, gb = gpu_sprsol(rs, ms, msifa, sm, b, rs.neq)
    assert ri == gi == 0 and np.array_equal(rm, gm)
    assert relerr(gb, rb) <= (1e-9 if emod == 'uniform' else 1e-6)
    # the permutation really applies: the solution differs from the unpermuted solve
    ri2, _, _, rb2 = ref_sprsol(rs, rs.mspar, rs.msifa, sm, b, rs.neq)
    assert relerr(rb2, rb) > 1e-3
    # SPRFS1 then SPRBS1 separately on the GPU factor
    B = np.asfortranarray(b.copy())
    msp = gm.copy()
    assert spr.sprfs1(msp, rs.mtrees, msifa, gsm, B, rs.neq, 3) == 0
    assert spr.sprbs1(msp, rs.mtrees, msifa, gsm, B, rs.neq, 3) == 0
    assert relerr(B, rb) <= (1e-9 if emod == 'uniform' else 1e-6)


@pytest.mark.parametrize('n', [6, 8])
def test_peri2e_partial_factorisation_internal_solution(n):
    rs, sm = ref_system(n, retain=True)
    first, nret = retained_info(rs)
    peri2e = np.arange(1, rs.neq + 1)
    peri2e[:first] = np.random.default_rng(n + 1).permutation(first) + 1
    ms, msifa = with_peri2e(rs, peri2e)
    ms[56] = 1
    b = rhs(first, 2, 80 + n)                        # internal equations, external numbering
    ri, rm, rsm, rb = ref_sprsol(rs, ms, msifa, sm, b, first)
    gi, gm, gsm, gb = gpu_sprsol(rs, ms, msifa, sm, b, first)
    assert ri == gi == 0 and np.array_equal(rm, gm)
    assert np.max(np.abs(gsm - rsm)) <= 1e-10 * np.max(np.abs(rsm))
    assert relerr(gb, rb) <= 1e-9


def test_peri2e_internal_row_beyond_ldb_is_refused():
    rs, sm = ref_system(6, retain=True)
    first, nret = retained_info(rs)
    peri2e = np.arange(1, rs.neq + 1)
    peri2e[[5, first + 3]] = peri2e[[first + 3, 5]]  # an internal equation numbered beyond LDB
    ms, msifa = with_peri2e(rs, peri2e)
    ms[56] = 1
    b = rhs(first, 1, 90)
    gi, gm, _, _ = gpu_sprsol(rs, ms, msifa, sm, b, first)
    assert gi == -4 and gm[0] == -7, (gi, gm[0])
