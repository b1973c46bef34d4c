"""Oracle runs of the benchmark-scale parity tests (CPU, in worker processes).

Each case is an n^3 hex box (the reference's structure, SM assembled by the
SPRADM main add), optionally shifted to K - sigma M (lumped mass, SPRSHA
KSB=2), with seeded right-hand sides.  The oracle restatement
(oracle/spr_oracle.c, pinned bitwise to the reference) runs SPRSOL IOP=3;
the factor, solution, TOL, MSPAR and IERR go to .npy files, so that the
parent process only loads what it compares.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

# lowest eigenvalue of (K, M) for the clamped n^3 box: lambda1(20) = 1.1190e-3
# from shift-invert Lanczos, scaled by (20/n)^2 (at 24^3 the scaled value is
# 7.771e-4 against 7.763e-4 computed)
LAMBDA1_20 = 1.1190368512857803e-3


def lambda1_est(n):
    return LAMBDA1_20 * (20.0 / n) ** 2


def _paths():
    for p in (ROOT, HERE):
        if p not in sys.path:
            sys.path.insert(0, p)


def case_system(n, emod, sigma_factor):
    """(HexSystem, SM) of one case."""
    _paths()
    from sam_lib_b200.fe import element_moduli
    from sam_lib_b200.system import HexSystem, diag_positions, shift_diagonal
    hs = HexSystem(n, moduli=element_moduli(n ** 3, emod, seed=2))
    sm = hs.assemble()
    if sigma_factor:
        pos = diag_positions(hs.mspar, hs.mtrees, hs.msifa)
        mass = hs.to_internal(hs.box.lumped_mass())
        sm = shift_diagonal(sm, pos, mass, sigma_factor * lambda1_est(n))
    return hs, sm


def case_rhs(neq, nrhs, seed):
    return np.asfortranarray(np.random.default_rng(seed).uniform(-1.0, 1.0, size=(neq, nrhs)))


def run_case(args):
    """Worker: oracle SPRSOL IOP=3 of one case; returns the output prefix."""
    n, emod, sigma_factor, nrhs, seed, out = args
    _paths()
    import oracle.refpipe as rp
    from sam_lib_b200.system import diag_positions
    hs, sm = case_system(n, emod, sigma_factor)
    adiag = sm[diag_positions(hs.mspar, hs.mtrees, hs.msifa)].copy()
    b = case_rhs(hs.neq, nrhs, seed)
    lib = C.CDLL(os.path.join(ROOT, 'oracle', '_ref', 'liboracle.so'))
    msp = hs.mspar.copy()
    tol = np.array([1e-12, 0.0, 0.0])
    iw = np.zeros(int(hs.mspar[13]) + int(hs.mspar[12]) + 8, dtype=np.int64)
    rw = np.zeros(int(hs.mspar[16]) + int(hs.mspar[13]) + 8)
    ierr = C.c_int64(0)
    lib.orc_sprsol_(rp._i(3), rp._p(msp), rp._p(hs.mtrees), rp._p(hs.msifa), rp._p(sm), rp._p(b),
                    rp._i(hs.neq), rp._i(nrhs), rp._p(tol), rp._p(iw), rp._p(rw), rp._i(-1), C.byref(ierr))
    d = sm[:hs.neq]
    np.save(out + '.sm.npy', sm)
    np.save(out + '.b.npy', b)
    np.savez(out + '.meta.npz', tol=tol, mspar=msp, ierr=ierr.value,
             min_ratio=float(np.min(np.abs(d) / np.abs(adiag))))
    return out


def batch_numneg(args):
    """Worker: oracle NUMNEG of systems [i0, i1) of the 512-system workload."""
    i0, i1 = args
    _paths()
    import oracle.refpipe as rp
    from sam_lib_b200.workloads import config4_system_sm
    lib = C.CDLL(os.path.join(ROOT, 'oracle', '_ref', 'liboracle.so'))
    out = []
    for i in range(i0, i1):
        _, _, sm, hs = config4_system_sm(i)
        b = np.zeros((hs.neq, 1), order='F')
        msp = hs.mspar.copy()
        tol = np.array([1e-12, 0.0, 0.0])
        iw = np.zeros(int(hs.mspar[13]) + int(hs.mspar[12]) + 8, dtype=np.int64)
        rw = np.zeros(int(hs.mspar[16]) + int(hs.mspar[13]) + 8)
        ierr = C.c_int64(0)
        lib.orc_sprsol_(rp._i(1), rp._p(msp), rp._p(hs.mtrees), rp._p(hs.msifa), rp._p(sm), rp._p(b),
                        rp._i(hs.neq), rp._i(1), rp._p(tol), rp._p(iw), rp._p(rw), rp._i(-1), C.byref(ierr))
        out.append((int(ierr.value), int(msp[25])))
    return out
