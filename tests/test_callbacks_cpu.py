"""MVMULT/MMMULT callbacks of SPRFC1/SPRFC3/SPRFC2 (host side, no GPU needed).

The reference calls the routines it is given (sprfc1.f:1138-1175); the GPU
path applies the updates of LMVY18/LMMY18 (CMVY18/CMMY18 for SPRFC2) itself.
The library therefore runs a non-null routine once on a small probe and
refuses the call (IERR = -4, MSPAR(1) < 0, a message on LPU >= 0) unless the
routine computes those updates.  The reference's own kernels (from the
translated reference build) and null pointers pass the probe; routines with
the right signature but another update are refused before any GPU work.
"""
import ctypes as C

import numpy as np
import pytest

import sam_lib_b200 as spr
from conftest import ref_system

I = C.c_int64
P = C.POINTER
LMV = C.CFUNCTYPE(None, P(I), P(I), P(C.c_double), P(C.c_double), P(I), P(C.c_double))
LMM = C.CFUNCTYPE(None, P(I), P(I), P(I), P(I), P(C.c_double), P(C.c_double), P(C.c_double), P(I))
CMV = C.CFUNCTYPE(None, P(I), P(I), P(C.c_double), P(I), P(C.c_double))
CMM = C.CFUNCTYPE(None, P(I), P(I), P(I), P(I), P(C.c_double), P(C.c_double), P(I))
MSG = 'MVMULT/MMMULT DO NOT COMPUTE'


def _mv_no_d(m, n, y, d, apnt, a):
    """LMVY18's signature with the C C' update (D ignored): not the LDL' kernel."""
    M, N = m[0], n[0]
    for j in range(N):
        off = apnt[j + 1] - (M + 1)
        s = -a[off]
        for i in range(M):
            y[i] += s * a[off + i]


def _noop(*args):
    return None


def _call(fn, mv, mm, capfd, lpu=6):
    rs, sm = ref_system(3)
    msp = rs.mspar.copy()
    tol = np.array([1e-12, 0.0, 0.0, 1.0])
    ierr = I(0)
    lib = spr.load(8)
    args = [spr._ptr(msp), spr._ptr(rs.mtrees), spr._ptr(rs.msifa), spr._ptr(sm.copy()), spr._ptr(tol),
            spr._ptr(np.zeros(1, dtype=np.int64)), spr._ptr(np.zeros(1))]
    if fn == 'sprfc3_':
        args.append(spr._ptr(np.zeros(2 * rs.neq)))
    args += [C.byref(I(lpu)), C.byref(ierr), mv, mm]
    getattr(lib, fn)(*args)
    err = capfd.readouterr().err
    return ierr.value, int(msp[0]), err


def _ref_fn(name):
    from oracle.refpipe import lib as reflib
    return C.cast(getattr(reflib(), name), C.c_void_p)


@pytest.mark.parametrize('fn', ['sprfc1_', 'sprfc3_'])
def test_foreign_ldlt_callbacks_are_refused(fn, capfd):
    bad_mv, bad_mm, ok_mm = LMV(_mv_no_d), LMM(_noop), _ref_fn('lmmy18_')
    for mv, mm in ((bad_mv, ok_mm), (_ref_fn('lmvy18_'), bad_mm)):
        ierr, state, err = _call(fn, C.cast(mv, C.c_void_p), C.cast(mm, C.c_void_p), capfd)
        assert ierr == -4 and state == -5, (ierr, state)
        assert MSG in err


@pytest.mark.parametrize('fn', ['sprfc1_', 'sprfc3_'])
def test_reference_ldlt_kernels_and_null_pass_the_probe(fn, capfd):
    for mv, mm in ((_ref_fn('lmvy18_'), _ref_fn('lmmy18_')), (None, None)):
        ierr, state, err = _call(fn, mv, mm, capfd)
        assert MSG not in err
        # with a GPU the factorisation runs (a clamped box: IERR 0); without
        # one the context set-up fails after the probe
        assert ierr in (0, -4)


def test_sprfc2_probe_uses_the_cholesky_kernels(capfd):
    ierr, state, err = _call('sprfc2_', _ref_fn('cmvy18_'), _ref_fn('cmmy18_'), capfd)
    assert MSG not in err and ierr in (0, -4)
    ierr, state, err = _call('sprfc2_', C.cast(CMV(_noop), C.c_void_p), _ref_fn('cmmy18_'), capfd)
    assert ierr == -4 and state == -6 and MSG in err
