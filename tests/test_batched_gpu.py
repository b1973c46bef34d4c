"""Config 4 on the GPU: many uneven shifted (indefinite) systems in one batched
factorisation; per-system inertia bit-exact against the reference, solutions
against the oracle."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def oracle_solve(hs, sm, b):
    from test_oracle import _lib
    import oracle.refpipe as rp
    sm = sm.copy()
    b = np.asfortranarray(b.copy())
    msp = hs.mspar.copy()
    tol = np.array([1e-12, 0.0, 0.0])
    iw = np.zeros(int(hs.mspar[13]) + 8, dtype=np.int64)
    rw = np.zeros(int(hs.mspar[16]) + int(hs.mspar[13]) + 8)
    ierr = C.c_int64(0)
    _lib().orc_sprsol_(rp._i(3), rp._p(msp), rp._p(hs.mtrees), rp._p(hs.msifa), rp._p(sm), rp._p(b),
                       rp._i(hs.neq), rp._i(b.shape[1]), rp._p(tol), rp._p(iw), rp._p(rw), rp._i(-1),
                       C.byref(ierr))
    return ierr.value, int(msp[25]), b


def test_batched_shifted_systems_inertia_and_solutions():
    from sam_lib_b200.workloads import config4
    from sam_lib_b200.batch import BatchSolver
    systems = config4()[:40]
    bs = BatchSolver(systems)
    r = bs.run()
    assert r['lierr'] == 0
    neg = bs.numneg()
    xs = bs.solutions()
    assert neg.sum() == r['numneg']
    assert (neg > 0).any() and (neg == 0).any()       # both definite and indefinite systems
    for i, s in enumerate(systems):
        ierr, nn, x = oracle_solve(s['hs'], s['sm'], s['b'])
        assert ierr == 0
        assert neg[i] == nn, (i, s['n'], neg[i], nn)
        assert np.linalg.norm(xs[i] - x) <= 1e-8 * np.linalg.norm(x), i
