"""K - sigma M (SPRSHA with a diagonal B, KSB = 2, src/SPR/sprsha.f:86-93) and
the diagonal pointers of SPRDG1 (sprdg1.f:5): the restatements the tests and
the batched workload use (conftest.shifted_sm, system.diag_positions /
shift_diagonal) against the translated reference, bit for bit (CPU)."""
import ctypes as C

import numpy as np
import pytest

from conftest import ref_system, shifted_sm


def ref_sprsha(rs, sm, mass, sigma):
    from oracle.refpipe import lib as reflib, _p, _i
    a = sm.copy()
    msp = rs.mspar.copy()
    mdloc = np.zeros(rs.neq, dtype=np.int64)
    b = np.ascontiguousarray(mass, dtype=np.float64)
    ierr = C.c_int64(0)
    reflib().sprsha_(_p(msp), _p(rs.mtrees), _p(rs.msifa), _p(msp), _p(rs.mtrees), _p(rs.msifa), _p(mdloc),
                     _p(a), _p(b), C.byref(C.c_double(sigma)), _i(rs.neq), _i(2), _i(-1), C.byref(ierr))
    return ierr.value, msp, mdloc, a


@pytest.mark.parametrize('n,sigma', [(3, 0.12), (6, 0.031), (9, 7.5e-3)])
def test_sprsha_diagonal_shift_matches_reference(n, sigma):
    from sam_lib_b200.system import diag_positions, shift_diagonal
    rs, sm = ref_system(n)
    mass = np.zeros(rs.neq)
    sel = rs.meqn > 0
    mass[rs.meqn[sel] - 1] = rs.box.lumped_mass()[sel]
    ierr, msp, mdloc, a = ref_sprsha(rs, sm, mass, sigma)
    assert ierr == 0 and msp[0] == 66                      # sprsha.f:95
    pos = diag_positions(rs.mspar, rs.mtrees, rs.msifa)
    assert np.array_equal(pos, mdloc - 1)                  # SPRDG1's pointers, 0-based
    assert np.array_equal(shifted_sm(rs, sm, sigma), a)
    assert np.array_equal(shift_diagonal(sm, pos, mass, sigma), a)
