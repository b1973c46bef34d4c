"""B200 implementation of the numeric phase of SAM's SPR sparse solver.

The product is the C-ABI library ``libspr_b200.so`` (built in-tree by
``sam_lib_b200.build``): it exports the reference's Fortran entry points
``sprsol_``, ``sprfc1_``, ``sprfc2_``, ``sprfc3_``, ``sprfc4_``, ``sprfs1_``, ``sprfs2_``,
``sprbs1_`` and ``sprbs2_`` (INTEGER*8 ABI;
``libspr_b200_i4.so`` has the INTEGER*4 ABI) plus a device-level API.  This
module is the Python mirror of that interface: the same routine names,
argument meaning and IERR conventions as src/SPR/sprsol.f, sprfc1.f,
sprfc2.f, sprfc3.f, sprfs1.f, sprfs2.f, sprbs1.f and sprbs2.f, with numpy
arrays standing in for the Fortran arrays.

There is no CPU fallback: if the library is missing, importing the
interface raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_I8 = os.path.join(HERE, 'libspr_b200.so')
LIB_I4 = os.path.join(HERE, 'libspr_b200_i4.so')

_libs = {}


def load(int_kind=8):
    """Loads the in-tree GPU library (raises if it has not been built)."""
    path = LIB_I8 if int_kind == 8 else LIB_I4
    lib = _libs.get(path)
    if lib is None:
        if not os.path.exists(path):
            raise RuntimeError('spr_b200: %s is missing; run `python -m sam_lib_b200.build`' % path)
        lib = C.CDLL(path)
        vp = C.c_void_p
        lib.spr_b200_open.argtypes = [vp, vp, vp, C.POINTER(vp)]
        lib.spr_b200_open.restype = C.c_int
        lib.spr_b200_close.argtypes = [vp]
        lib.spr_b200_close.restype = None
        lib.spr_b200_set_stream.argtypes = [vp, vp]
        lib.spr_b200_factor_dev.argtypes = [vp, vp, C.c_double, vp]
        lib.spr_b200_factor_dev.restype = C.c_int
        lib.spr_b200_factor3_dev.argtypes = [vp, vp, vp, vp, vp]
        lib.spr_b200_factor3_dev.restype = C.c_int
        lib.spr_b200_solve_dev.argtypes = [vp, vp, vp, C.c_int64, C.c_int64, C.c_int]
        lib.spr_b200_solve_dev.restype = C.c_int
        lib.spr_b200_info.argtypes = [vp, vp]
        lib.spr_b200_info.restype = C.c_int
        lib.spr_b200_sn_stats.argtypes = [vp, vp, vp]
        lib.spr_b200_sn_stats.restype = C.c_int
        lib.spr_b200_build_residual.argtypes = [vp, vp]
        lib.spr_b200_build_residual.restype = C.c_int
        lib.spr_b200_refine.argtypes = [vp, vp, vp, vp, C.c_int64, C.c_int64, C.c_double, C.c_int, vp]
        lib.spr_b200_refine.restype = C.c_int
        lib.spr_b200_set_mode.argtypes = [vp, C.c_int]
        lib.spr_b200_set_mode.restype = C.c_int
        lib.spr_b200_set_inertia_guard.argtypes = [vp, C.c_double]
        lib.spr_b200_set_inertia_guard.restype = C.c_int
        lib.spr_b200_set_watchdog.argtypes = [vp, C.c_double, C.c_int]
        lib.spr_b200_set_watchdog.restype = C.c_int
        lib.spr_b200_set_skip.argtypes = [vp, vp]
        lib.spr_b200_set_skip.restype = C.c_int
        lib.spr_b200_set_exchange.argtypes = [vp, C.c_int64, vp, vp, C.c_int64, vp, vp, C.c_int64, vp, vp,
                                              C.c_int64, vp, vp]
        lib.spr_b200_set_exchange.restype = C.c_int
        lib.spr_b200_autotune.argtypes = [vp, vp, vp]
        lib.spr_b200_autotune.restype = C.c_int
        lib.spr_b200_autotune_tiles.argtypes = [vp, vp, vp]
        lib.spr_b200_autotune_tiles.restype = C.c_int
        lib.spr_b200_set_small_tile.argtypes = [vp, C.c_int]
        lib.spr_b200_set_small_tile.restype = C.c_int
        lib.spr_b200_tc_stats.argtypes = [vp, vp]
        lib.spr_b200_tc_stats.restype = C.c_int
        lib.spr_b200_phase_ms.argtypes = [vp, vp]
        lib.spr_b200_phase_ms.restype = C.c_int
        lib.spr_b200_set_profile.argtypes = [vp, C.c_int]
        lib.spr_b200_set_profile.restype = C.c_int
        lib.spr_b200_release_all.argtypes = []
        lib.spr_b200_release_all.restype = None
        _libs[path] = lib
    return lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _ref(v, dtype):
    return C.byref(dtype(int(v)))


def _ints(int_kind):
    return (np.int64, C.c_int64) if int_kind == 8 else (np.int32, C.c_int32)


def _check_int(a, np_t, name):
    if a.dtype != np_t or not a.flags['C_CONTIGUOUS']:
        raise TypeError('%s must be a contiguous %s array' % (name, np.dtype(np_t).name))


def sprsol(iop, mspar, mtrees, msifa, sm, b, ldb, nrhs, tol, iwork=None, rwork=None, lpu=-1,
           int_kind=8):
    """SPRSOL (src/SPR/sprsol.f:5): returns IERR; SM, B, TOL, MSPAR updated in place."""
    np_t, c_t = _ints(int_kind)
    for a, n in ((mspar, 'MSPAR'), (mtrees, 'MTREES'), (msifa, 'MSIFA')):
        _check_int(a, np_t, n)
    if sm.dtype != np.float64 or b.dtype != np.float64 or tol.dtype != np.float64:
        raise TypeError('SM, B and TOL must be float64')
    if not b.flags['F_CONTIGUOUS']:
        raise TypeError('B must be Fortran-ordered (LDB, NRHS)')
    iwork = np.zeros(1, dtype=np_t) if iwork is None else iwork
    rwork = np.zeros(1) if rwork is None else rwork
    ierr = c_t(0)
    load(int_kind).sprsol_(_ref(iop, c_t), _ptr(mspar), _ptr(mtrees), _ptr(msifa), _ptr(sm),
                           _ptr(b), _ref(ldb, c_t), _ref(nrhs, c_t), _ptr(tol), _ptr(iwork),
                           _ptr(rwork), _ref(lpu, c_t), C.byref(ierr))
    return ierr.value


def sprfc1(mspar, mtrees, msifa, sm, tol, iwork=None, rwork=None, lpu=-1, int_kind=8):
    """SPRFC1 (src/SPR/sprfc1.f:5): LDL' factorisation of SM; returns IERR."""
    np_t, c_t = _ints(int_kind)
    iwork = np.zeros(1, dtype=np_t) if iwork is None else iwork
    rwork = np.zeros(1) if rwork is None else rwork
    ierr = c_t(0)
    load(int_kind).sprfc1_(_ptr(mspar), _ptr(mtrees), _ptr(msifa), _ptr(sm), _ptr(tol),
                           _ptr(iwork), _ptr(rwork), _ref(lpu, c_t), C.byref(ierr), None, None)
    return ierr.value


def sprfc3(mspar, mtrees, msifa, sm, tol, dcor, iwork=None, rwork=None, lpu=-1, int_kind=8):
    """SPRFC3 (src/SPR/sprfc3.f:5): LDL' factorisation that replaces singular pivots.

    TOL has 4 entries (TOL(1) zero threshold, TOL(4) replacement scale on
    entry; TOL(2), TOL(3) on exit); DCOR is a float64 array of 2*NEQ entries
    (DCOR(2,NEQ) column-major).  Returns IERR: -3 with MSPAR(27) = -(number of
    replaced pivots) still leaves a complete factor in SM.
    """
    np_t, c_t = _ints(int_kind)
    if tol.dtype != np.float64 or tol.size < 4:
        raise TypeError('TOL must be a float64 array of 4 entries')
    if dcor.dtype != np.float64 or dcor.size < 2 * int(mspar[7]):
        raise TypeError('DCOR must be a float64 array of 2*NEQ entries')
    iwork = np.zeros(1, dtype=np_t) if iwork is None else iwork
    rwork = np.zeros(1) if rwork is None else rwork
    ierr = c_t(0)
    load(int_kind).sprfc3_(_ptr(mspar), _ptr(mtrees), _ptr(msifa), _ptr(sm), _ptr(tol),
                           _ptr(iwork), _ptr(rwork), _ptr(dcor), _ref(lpu, c_t), C.byref(ierr),
                           None, None)
    return ierr.value


def sprfc4(mspar, mtrees, msifa, sm, tol, dcor, iwork=None, rwork=None, lpu=-1, int_kind=8):
    """SPRFC4 (src/SPR/sprfc4.f:5): Cholesky factorisation C C' that replaces
    small pivots (TOL(1), TOL(4); 4 TOL entries) and records them in DCOR
    (2*NEQ); returns IERR (-3 with MSPAR(27) = -(number replaced) still leaves
    a complete factor)."""
    np_t, c_t = _ints(int_kind)
    if tol.dtype != np.float64 or tol.size < 4:
        raise TypeError('TOL must be a float64 array of 4 entries')
    if dcor.dtype != np.float64 or dcor.size < 2 * int(mspar[7]):
        raise TypeError('DCOR must be a float64 array of 2*NEQ entries')
    iwork = np.zeros(1, dtype=np_t) if iwork is None else iwork
    rwork = np.zeros(1) if rwork is None else rwork
    ierr = c_t(0)
    load(int_kind).sprfc4_(_ptr(mspar), _ptr(mtrees), _ptr(msifa), _ptr(sm), _ptr(tol),
                           _ptr(iwork), _ptr(rwork), _ptr(dcor), _ref(lpu, c_t), C.byref(ierr),
                           None, None)
    return ierr.value


def sprfc2(mspar, mtrees, msifa, sm, tol, iwork=None, rwork=None, lpu=-1, int_kind=8):
    """SPRFC2 (src/SPR/sprfc2.f:5): Cholesky factorisation C C' of SM; returns IERR."""
    np_t, c_t = _ints(int_kind)
    iwork = np.zeros(1, dtype=np_t) if iwork is None else iwork
    rwork = np.zeros(1) if rwork is None else rwork
    ierr = c_t(0)
    load(int_kind).sprfc2_(_ptr(mspar), _ptr(mtrees), _ptr(msifa), _ptr(sm), _ptr(tol),
                           _ptr(iwork), _ptr(rwork), _ref(lpu, c_t), C.byref(ierr), None, None)
    return ierr.value


def sprfs2(mspar, mtrees, msifa, sm, b, ldb, nrhs, iwork=None, rwork=None, lpu=-1, int_kind=8):
    """SPRFS2 (src/SPR/sprfs2.f:5): forward sweep C y = b on a C C' factor; returns IERR."""
    np_t, c_t = _ints(int_kind)
    iwork = np.zeros(1, dtype=np_t) if iwork is None else iwork
    rwork = np.zeros(1) if rwork is None else rwork
    ierr = c_t(0)
    load(int_kind).sprfs2_(_ptr(mspar), _ptr(mtrees), _ptr(msifa), _ptr(sm), _ptr(b),
                           _ref(ldb, c_t), _ref(nrhs, c_t), _ptr(iwork), _ptr(rwork),
                           _ref(lpu, c_t), C.byref(ierr))
    return ierr.value


def sprbs2(mspar, mtrees, msifa, sm, b, ldb, nrhs, rwork=None, lpu=-1, int_kind=8):
    """SPRBS2 (src/SPR/sprbs2.f:5): back sweep C' x = y; returns IERR."""
    _, c_t = _ints(int_kind)
    rwork = np.zeros(1) if rwork is None else rwork
    ierr = c_t(0)
    load(int_kind).sprbs2_(_ptr(mspar), _ptr(mtrees), _ptr(msifa), _ptr(sm), _ptr(b),
                           _ref(ldb, c_t), _ref(nrhs, c_t), _ptr(rwork), _ref(lpu, c_t),
                           C.byref(ierr))
    return ierr.value


def sprfs1(mspar, mtrees, msifa, sm, b, ldb, nrhs, iwork=None, rwork=None, lpu=-1, int_kind=8):
    """SPRFS1 (src/SPR/sprfs1.f:5): forward reduction + diagonal scaling; returns IERR."""
    np_t, c_t = _ints(int_kind)
    iwork = np.zeros(1, dtype=np_t) if iwork is None else iwork
    rwork = np.zeros(1) if rwork is None else rwork
    ierr = c_t(0)
    load(int_kind).sprfs1_(_ptr(mspar), _ptr(mtrees), _ptr(msifa), _ptr(sm), _ptr(b),
                           _ref(ldb, c_t), _ref(nrhs, c_t), _ptr(iwork), _ptr(rwork),
                           _ref(lpu, c_t), C.byref(ierr))
    return ierr.value


def sprbs1(mspar, mtrees, msifa, sm, b, ldb, nrhs, rwork=None, lpu=-1, int_kind=8):
    """SPRBS1 (src/SPR/sprbs1.f:5): back substitution; returns IERR."""
    _, c_t = _ints(int_kind)
    rwork = np.zeros(1) if rwork is None else rwork
    ierr = c_t(0)
    load(int_kind).sprbs1_(_ptr(mspar), _ptr(mtrees), _ptr(msifa), _ptr(sm), _ptr(b),
                           _ref(ldb, c_t), _ref(nrhs, c_t), _ptr(rwork), _ref(lpu, c_t),
                           C.byref(ierr))
    return ierr.value


def release_all():
    """Frees the device contexts cached by the Fortran entry points."""
    load(8).spr_b200_release_all()


class DeviceSolver:
    """Device-resident factor/solve on one SPR structure (INTEGER*8 arrays).

    ``factor(d_sm)`` and ``solve(d_sm, d_b)`` take device pointers (ints) or
    torch CUDA tensors: SM = [D(NEQ) | LNZ(NZEROL)] and B (NEQ x NRHS,
    column-major, i.e. a torch tensor of shape (NRHS, NEQ)).
    """

    def __init__(self, mspar, mtrees, msifa):
        self.lib = load(8)
        self.h = C.c_void_p()
        rc = self.lib.spr_b200_open(_ptr(mspar), _ptr(mtrees), _ptr(msifa), C.byref(self.h))
        if rc != 0:
            raise RuntimeError('spr_b200_open failed with %d' % rc)
        self.neq = int(mspar[7])
        self.nzerol = int(mspar[15])

    @staticmethod
    def _dev(x):
        return x if isinstance(x, int) else x.data_ptr()

    def set_stream(self, stream_ptr):
        self.lib.spr_b200_set_stream(self.h, C.c_void_p(stream_ptr))

    def factor(self, d_sm, tol1=1.0e-12):
        """Returns dict(tol2, tol3, numneg, supeqt, lierr) like SPRF11."""
        out = np.zeros(5)
        rc = self.lib.spr_b200_factor_dev(self.h, C.c_void_p(self._dev(d_sm)), tol1, _ptr(out))
        if rc != 0:
            raise RuntimeError('spr_b200_factor_dev failed with %d' % rc)
        return dict(tol2=out[0], tol3=out[1], numneg=int(out[2]), supeqt=int(out[3]),
                    lierr=int(out[4]))

    def factor3(self, d_sm, d_dcor, tol1=1.0e-12, tol4=1.0):
        """SPRFC3 semantics (SPRF31, sprfc3.f:372): singular pivots are replaced
        and recorded in the device DCOR(2,NEQ) (2*NEQ doubles); returns the dict
        of factor(), with lierr = -31 and supeqt = the number replaced if any."""
        out = np.zeros(5)
        tol = np.array([tol1, tol4])
        rc = self.lib.spr_b200_factor3_dev(self.h, C.c_void_p(self._dev(d_sm)), _ptr(tol),
                                           C.c_void_p(self._dev(d_dcor)), _ptr(out))
        if rc != 0:
            raise RuntimeError('spr_b200_factor3_dev failed with %d' % rc)
        return dict(tol2=out[0], tol3=out[1], numneg=int(out[2]), supeqt=int(out[3]),
                    lierr=int(out[4]))

    def solve(self, d_sm, d_b, nrhs, ldb=None, which=3):
        ldb = self.neq if ldb is None else ldb
        rc = self.lib.spr_b200_solve_dev(self.h, C.c_void_p(self._dev(d_sm)),
                                         C.c_void_p(self._dev(d_b)), ldb, nrhs, which)
        if rc != 0:
            raise RuntimeError('spr_b200_solve_dev failed with %d' % rc)

    def info(self):
        out = np.zeros(15)
        self.lib.spr_b200_info(self.h, _ptr(out))
        keys = ('factor_flops', 'solve_flops', 'arena_bytes', 'levels', 'factor_ms', 'solve_ms',
                'launches', 'gemm_launches', 'gemm_ms', 'gemm_flops', 'solve_launches', 'nzerol',
                'near_pivots', 'fp64_redo', 'trace')
        return dict(zip(keys, out.tolist()))

    def sn_stats(self, nsuper):
        neg = np.zeros(nsuper, dtype=np.int32)
        fail = np.zeros(nsuper, dtype=np.int32)
        self.lib.spr_b200_sn_stats(self.h, _ptr(neg), _ptr(fail))
        return neg, fail

    def build_residual(self, d_sm_assembled):
        rc = self.lib.spr_b200_build_residual(self.h, C.c_void_p(self._dev(d_sm_assembled)))
        if rc != 0:
            raise RuntimeError('spr_b200_build_residual failed with %d' % rc)

    def refine(self, d_sm, d_b, d_x, nrhs, tol=1e-12, maxit=30, ld=None):
        """Iterative refinement; returns (corrections, backward error, solve ms)."""
        ld = self.neq if ld is None else ld
        out = np.zeros(3)
        rc = self.lib.spr_b200_refine(self.h, C.c_void_p(self._dev(d_sm)), C.c_void_p(self._dev(d_b)),
                                      C.c_void_p(self._dev(d_x)), ld, nrhs, tol, maxit, _ptr(out))
        if rc != 0:
            raise RuntimeError('spr_b200_refine failed with %d' % rc)
        return int(out[0]), float(out[1]), float(out[2])

    def set_mode(self, mixed):
        """0/False = FP64, 1/True = 3xTF32 on tcgen05, 2 = 3xTF32 through mma.sync."""
        rc = self.lib.spr_b200_set_mode(self.h, int(mixed))
        if rc != 0:
            raise ValueError('unknown factorisation mode %r' % (mixed,))

    def set_inertia_guard(self, tau):
        """Mixed modes: redo the factorisation in FP64 when a pivot has
        |d| < tau |a_jj| or fails the pivot test (default 1e-3, 0 = off)."""
        if self.lib.spr_b200_set_inertia_guard(self.h, float(tau)) != 0:
            raise ValueError('bad inertia-guard tolerance %r' % (tau,))

    def set_watchdog(self, wait_s=2.0, drop=False):
        """Wait limit of the tensor-core kernel's barriers; drop=True is the
        test switch that makes one CTA's waits run out."""
        if self.lib.spr_b200_set_watchdog(self.h, float(wait_s) * 1e9, 1 if drop else 0) != 0:
            raise ValueError('bad watchdog limit %r' % (wait_s,))

    def set_skip(self, mask):
        """Split runs: supernodes with mask[js] (NSUPER bools) are left alone; None clears."""
        if mask is None:
            rc = self.lib.spr_b200_set_skip(self.h, None)
        else:
            m = np.ascontiguousarray(mask, dtype=np.uint8)
            rc = self.lib.spr_b200_set_skip(self.h, _ptr(m))
        if rc != 0:
            raise RuntimeError('spr_b200_set_skip failed with %d' % rc)

    def set_exchange(self, factor_out=(), factor_in=(), vec_out=(), vec_in=()):
        """Split runs: lists of (node, device buffer) for the update blocks of
        the following factorisations and the update vectors of the following
        forward sweeps (see include/spr_b200.h)."""
        def arr(lst):
            nodes = np.array([int(n) for n, _ in lst], dtype=np.int32)
            bufs = (C.c_void_p * max(1, len(lst)))(*[C.c_void_p(self._dev(b)) for _, b in lst])
            return len(lst), nodes, bufs
        parts = [arr(l) for l in (factor_out, factor_in, vec_out, vec_in)]
        args = []
        for n, nodes, bufs in parts:
            args += [n, _ptr(nodes), C.cast(bufs, C.c_void_p)]
        rc = self.lib.spr_b200_set_exchange(self.h, *args)
        if rc != 0:
            raise RuntimeError('spr_b200_set_exchange failed with %d' % rc)

    def autotune(self, d_sm_assembled):
        """Mixed-mode autotuner on a copy of the assembled SM; returns the choice and times."""
        out = np.zeros(5)
        rc = self.lib.spr_b200_autotune(self.h, C.c_void_p(self._dev(d_sm_assembled)), _ptr(out))
        if rc != 0:
            raise RuntimeError('spr_b200_autotune failed with %d' % rc)
        return dict(tc_min_flops=out[0], far_sm_quarters=int(out[1]), factor_ms=out[2], default_ms=out[3],
                    candidates=int(out[4]))

    def autotune_tiles(self, d_sm_assembled):
        """Times the small Schur updates with 64x64 and 32x32 tiles on a copy
        of the assembled SM and keeps the faster; returns the choice."""
        out = np.zeros(3)
        rc = self.lib.spr_b200_autotune_tiles(self.h, C.c_void_p(self._dev(d_sm_assembled)), _ptr(out))
        if rc != 0:
            raise RuntimeError('spr_b200_autotune_tiles failed with %d' % rc)
        return {'small_tile': int(out[0]), 'factor_ms_64': out[1], 'factor_ms_32': out[2]}

    def set_small_tile(self, tile):
        self.lib.spr_b200_set_small_tile(self.h, int(tile))

    def tc_stats(self):
        """Mixed mode: (tensor-core update flops, their time in the last profiled factor, ms)."""
        out = np.zeros(2)
        self.lib.spr_b200_tc_stats(self.h, _ptr(out))
        return float(out[0]), float(out[1])

    def phase_ms(self):
        """Profile mode: last factorisation's time by phase (ms)."""
        out = np.zeros(20)
        self.lib.spr_b200_phase_ms(self.h, _ptr(out))
        keys = ('prepass', 'small_fronts', 'extend_add', 'diag', 'trsm', 'updates', 'outer_update',
                'writeback', 'end', 'fwd_small', 'fwd_gather', 'fwd_blocks', 'fwd_rect', 'fwd_finish',
                'bwd_small', 'bwd_gather', 'bwd_rect', 'bwd_blocks', 'unused', 'bwd_finish')
        return dict(zip(keys, out.tolist()))

    def set_profile(self, on=True):
        self.lib.spr_b200_set_profile(self.h, 1 if on else 0)

    def close(self):
        if self.h:
            self.lib.spr_b200_close(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
