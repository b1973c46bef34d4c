"""SPRLAN (src/SPR/sprlan.f:5, the reference's shift-invert Lanczos) on a
clamped hex box with lumped mass, through the translated reference library.

Run as a script it prints a JSON line with the results; the GPU test runs it
in a child process with libspr_b200.so preloaded (LD_PRELOAD), so that the
reference's SPRLAN reaches the GPU through its calls to SPRFC1, SPRFS1 and
SPRBS1 (sprlan.f:703, sprsmm.f), exactly as a Fortran host linked against
the GPU library would.

Options (MIP, as SPRLAX sets them, sprlax.f:24-30, with KSB = 2): A the
original sparse matrix (KSA = 1), B = the lumped mass as a diagonal (KSB =
2), random start vector (KSR = 1), full reorthogonalisation (KORT = 2), KEX =
2, A - SHIFT B indefinite (KPD = 2), so MOP(4) is the Sturm count MSPAR(26).
"""
import ctypes as C
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for _p in (ROOT, HERE):
    if _p not in sys.path:
        sys.path.insert(0, _p)


def run(n, shift, neval=6, maxlan=40):
    from conftest import ref_system
    from oracle.refpipe import lib as reflib, _p, _i
    rs, sm = ref_system(n)
    a = sm.copy()
    neq = rs.neq
    mass = np.zeros(neq)
    sel = rs.meqn > 0
    mass[rs.meqn[sel] - 1] = rs.box.lumped_mass()[sel]
    ms = rs.mspar.copy()
    msb = rs.mspar.copy()
    tol = np.zeros(3)
    mip = np.array([1, 2, -1, 2, 2, 2, 0], dtype=np.int64)
    mop = np.zeros(10, dtype=np.int64)
    msing = np.zeros(neq + 16, dtype=np.int64)
    evl = np.zeros(maxlan)
    everr = np.zeros(maxlan)
    v = np.zeros((maxlan, neq))          # V(N, MAXLAN), column-major
    r = np.zeros(2 * neq + 16)
    nrwa = int(ms[16]) + int(ms[13]) + maxlan * (maxlan + 8) + 1024
    rwa = np.zeros(nrwa)
    lwa = np.zeros(2 * neq + int(ms[13]) + 4 * maxlan + 1024, dtype=np.int64)
    sh = C.c_double(shift)
    ierr = C.c_int64(0)
    R = reflib()
    R.sprlan_(_p(a), _p(mass), _p(tol), _p(ms), _p(rs.mtrees), _p(rs.msifa), _p(msb), _p(rs.mtrees),
              _p(rs.msifa), _p(mip), _p(mop), _p(msing), _p(evl), _p(everr), _p(v), _p(r), _p(rwa), _p(lwa),
              C.byref(sh), _i(neq), _i(neval), _i(0), _i(maxlan), _i(-1), _i(-1), C.byref(ierr),
              C.cast(R.lmvy18_, C.c_void_p), C.cast(R.lmmy18_, C.c_void_p),
              C.cast(R.cmvy18_, C.c_void_p), C.cast(R.cmmy18_, C.c_void_p))
    return dict(ierr=int(ierr.value), evl=evl.tolist(), mop=mop.tolist(), numneg=int(ms[25]),
                state=int(ms[0]))


if __name__ == '__main__':
    n, shift = int(sys.argv[1]), float(sys.argv[2])
    print(json.dumps(run(n, shift)))
