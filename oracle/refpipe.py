"""Drive the machine-translated reference SPR library (oracle/_ref/libsprref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
CPU-baseline leg of bench.py, never by the product.

Runs the reference host sequence exactly as a Fortran FE program would:

    SPRPRP -> SPRSAS -> SPRRNM -> SPRTRS -> SPRSMB -> SPRPMP
           -> SPRADM (once per element) -> SPRSOL

(call sequence from ``src/SPR/sprprp.f:5``, ``sprsas.f:5``, ``sprrnm.f:5``,
``sprtrs.f:5``, ``sprsmb.f:5``, ``sprpmp.f:5``, ``spradm.f:5``,
``sprsol.f:5``).  All INTEGER arrays are int64 (the default SPR_I8 build);
every routine receives its arguments by reference through ctypes.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, '_ref', 'libsprref.so')
NSPAR = 60

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError('oracle reference library missing: %s (run make -C oracle)' % LIB_PATH)
        _lib = C.CDLL(LIB_PATH)
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _i(v):
    return C.byref(C.c_int64(int(v)))


class RefSystem:
    """One SPR system prepared by the reference host pipeline."""

    def __init__(self, box, lpu=-1):
        self.box = box
        L = lib()
        ierr = C.c_int64(0)
        self.mpar = box.mpar.copy()
        self.mspar = np.zeros(NSPAR, dtype=np.int64)
        self.meqn = np.zeros(box.ndof, dtype=np.int64)
        msc = box.msc.copy()
        mwork = np.zeros(2 * box.ndof + box.nanod + 8, dtype=np.int64)
        L.sprprp_(_p(box.madof), _p(box.minex), _p(box.mpmnpc), _p(box.mmnpc),
                  _p(box.mpmceq), _p(box.mmceq), _p(msc), _i(NSPAR), _i(lpu),
                  _p(self.mpar), _p(self.mspar), _p(self.meqn), _p(mwork), C.byref(ierr))
        self._check('SPRPRP', ierr)
        self.msc = msc
        nmsica = int(self.mspar[34])
        self.msica = np.zeros(nmsica, dtype=np.int64)
        L.sprsas_(_p(self.mpar), _p(box.mpmnpc), _p(box.mmnpc), _p(box.madof), _p(msc),
                  _p(box.mpmceq), _p(box.mmceq), _p(self.meqn), _p(self.mspar), _p(self.msica),
                  _p(mwork), _i(NSPAR), _i(lpu), C.byref(ierr))
        self._check('SPRSAS', ierr, allow_positive=True)
        iw = np.zeros(int(self.mspar[36]) + 8, dtype=np.int64)
        L.sprrnm_(_p(self.mspar), _p(self.msica), _p(iw), _i(lpu), C.byref(ierr))
        self._check('SPRRNM', ierr)
        ntrees = int(self.mspar[35])
        self.mtrees = np.zeros(ntrees, dtype=np.int64)
        niwork = int(self.mspar[37]) + 8
        iw = np.zeros(niwork, dtype=np.int64)
        self.rinfo = np.zeros(4, dtype=np.float64)
        L.sprtrs_(_p(self.mspar), _p(self.msica), _p(self.mtrees), _p(self.meqn), _i(NSPAR),
                  _i(nmsica), _i(ntrees), _i(box.ndof), _i(niwork), _p(iw), _p(self.rinfo),
                  _i(lpu), C.byref(ierr))
        self._check('SPRTRS', ierr)
        self.msifa = np.zeros(int(self.mspar[2]) + 8, dtype=np.int64)
        iw = np.zeros(3 * int(self.mspar[5]) + 2 * int(self.mspar[7]) + 8, dtype=np.int64)
        L.sprsmb_(_p(self.mspar), _p(self.msica), _p(self.mtrees), _p(self.msifa),
                  _p(self.meqn), _p(iw), _i(lpu), C.byref(ierr))
        self._check('SPRSMB', ierr)
        neq = int(self.mspar[7])
        self.mdofnc = np.zeros(2 * neq + 8, dtype=np.int64)
        L.sprpmp_(_p(self.msica), _p(self.mtrees), _p(self.meqn), _p(self.mpar),
                  _p(self.mspar), _p(self.mdofnc))
        self.neq = neq
        self.nzerol = int(self.mspar[15])

    @staticmethod
    def _check(name, ierr, allow_positive=False):
        v = ierr.value
        if v < 0 or (v > 0 and not allow_positive):
            raise RuntimeError('%s returned IERR=%d' % (name, v))

    # ---------------------------------------------------------------
    def assemble(self, ke_list, nsv=0):
        """SPRADM once per element; ke_list(iel) -> 24x24 matrix (0-based iel).

        Returns SM = [D(NEQ) | LNZ(NZEROL)] with the assembled matrix in LNZ;
        with nsv = 1 (or -1) returns (SM, SV), SV(NEQ) the right-hand side of
        the prescribed values of the box's constraint equations (TTCC).
        """
        L = lib()
        box = self.box
        sm = np.zeros(self.neq + self.nzerol, dtype=np.float64)
        sv = np.zeros(max(self.neq, 1), dtype=np.float64)
        ttcc = np.ascontiguousarray(getattr(box, 'ttcc', np.zeros(1)), dtype=np.float64)
        iw = np.zeros(int(self.mspar[38]) + 64, dtype=np.int64)
        ierr = C.c_int64(0)
        nedof = 8 * box.nndof
        for iel in range(box.nel):
            em = np.asfortranarray(ke_list(iel), dtype=np.float64)
            L.spradm_(_p(em), _p(ttcc), _p(self.mpar), _p(self.mspar), _p(box.madof),
                      _p(self.meqn), _p(box.mpmnpc), _p(box.mmnpc), _p(box.mpmceq),
                      _p(box.mmceq), _p(self.msica), _p(self.mtrees), _p(self.msifa),
                      _p(self.mdofnc), _p(sm), _p(sv), _p(iw), _i(iel + 1), _i(nedof),
                      _i(-1), _i(nsv), C.byref(ierr))
            if ierr.value < 0:
                raise RuntimeError('SPRADM(%d) returned IERR=%d' % (iel + 1, ierr.value))
        return (sm, sv) if nsv else sm

    def rhs_to_internal(self, f_dof):
        """Map a per-DOF vector (length NDOF) to SPR equation order via MEQN."""
        b = np.zeros(self.neq)
        m = self.meqn
        sel = m > 0
        b[m[sel] - 1] = f_dof[sel]
        return b

    def sprsol(self, iop, sm, b, tol1=1.0e-12, lpu=-1):
        """Call the reference SPRSOL; returns (IERR, TOL(3), NUMNEG)."""
        L = lib()
        b = np.asfortranarray(b)
        nrhs = 1 if b.ndim == 1 else b.shape[1]
        tol = np.array([tol1, 0.0, 0.0])
        mfront = int(self.mspar[13])
        iwork = np.zeros(max(mfront + 1, int(self.mspar[12])) + 8, dtype=np.int64)
        rwork = np.zeros(max(int(self.mspar[16]), mfront) + 8, dtype=np.float64)
        ierr = C.c_int64(0)
        L.sprsol_(_i(iop), _p(self.mspar), _p(self.mtrees), _p(self.msifa), _p(sm), _p(b),
                  _i(self.neq), _i(nrhs), _p(tol), _p(iwork), _p(rwork), _i(lpu), C.byref(ierr))
        return ierr.value, tol, int(self.mspar[25])
