"""The library's host SPRADM with constraint equations, and general hex8
element matrices, against the translated reference's SPRADM (CPU).

The box ties the x-DOFs of its face x=n to two master DOFs (multi-point
constraints with a constant term, one with a zero coefficient) and
prescribes the z-DOFs of one edge (src/SPR/sprseq.f:120-145 layout).  SPRADM
then adds, besides the free-DOF entries, the master-weighted entries of the
slaves into SM and the prescribed values' products into SV
(src/SPR/spradm.f:868-1002).  The library's assembly must give the same SM
and SV bit for bit, for NSV = 0, 1 and -1.
"""
import ctypes as C
import functools

import numpy as np
import pytest

import sam_lib_b200 as spr
from sam_lib_b200.fe import HexBox, element_moduli, hex8_stiffness, hex8_stiffness_xyz

I8 = C.c_int64


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


@functools.lru_cache(maxsize=None)
def tied(n):
    from oracle.refpipe import RefSystem
    box = HexBox(n, ties=True)
    return box, RefSystem(box)


def host_assemble(box, rs, em, scale, nsv):
    """spr_b200_assemble_ceq -> (rc, SM, SV)."""
    sm = np.zeros(rs.neq + rs.nzerol)
    sv = np.zeros(rs.neq)
    rc = spr.load(8).spr_b200_assemble_ceq(
        _p(rs.mspar), _p(rs.mtrees), _p(rs.msifa), _p(rs.meqn), _p(box.madof), _p(box.mpmnpc),
        _p(box.mmnpc), _p(box.mpmceq), _p(box.mmceq), _p(box.ttcc), I8(box.nceq), I8(box.nel), I8(24),
        _p(em), _p(scale), I8(nsv), _p(sm), _p(sv))
    return rc, sm, sv


def element_matrices(box, kind):
    """(reference callback, library em, library scale) for the element set."""
    if kind == 'scaled':
        ke = np.asfortranarray(hex8_stiffness())
        E = element_moduli(box.nel, 'loguniform', seed=2)
        # SPRADM receives the matrix the host formed: E_e * K_ref, rounded
        return (lambda e: ke * E[e]), ke, E
    xe = box.element_coords(box.distorted_coords(seed=5))
    K = hex8_stiffness_xyz(xe, element_moduli(box.nel, 'loguniform', seed=3))
    em = np.ascontiguousarray(K.transpose(0, 2, 1))       # column-major per element
    return (lambda e: K[e]), em, None


@pytest.mark.parametrize('n', [3, 5])
@pytest.mark.parametrize('nsv', [0, 1, -1])
@pytest.mark.parametrize('kind', ['scaled', 'distorted'])
def test_constrained_assembly_bitwise_equals_spradm(n, nsv, kind):
    box, rs = tied(n)
    assert box.nceq > 0 and rs.mpar[15] == len(box.mmceq)     # MPAR(16) = NMMCEQ from SPRSEQ
    cb, em, scale = element_matrices(box, kind)
    ref = rs.assemble(cb, nsv=nsv)
    rc, sm, sv = host_assemble(box, rs, em, scale, nsv)
    assert rc == 0
    if nsv == 0:
        assert np.array_equal(sm, ref)
        return
    sm_ref, sv_ref = ref
    assert np.array_equal(sv, sv_ref[:rs.neq])
    assert np.count_nonzero(sv) > 0
    assert np.array_equal(sm, sm_ref)
    if nsv == -1:
        assert not sm.any()


def test_constrained_system_solves_like_the_reference():
    """The assembled tied system factored and solved by the reference: the
    slaves' masters carry the coupling, the solution satisfies K u = SV."""
    box, rs = tied(4)
    cb, em, scale = element_matrices(box, 'scaled')
    rc, sm, sv = host_assemble(box, rs, em, scale, 1)
    assert rc == 0
    sm_f = sm.copy()
    ierr, _, numneg = rs.sprsol(3, sm_f, sv.copy())
    assert ierr == 0 and numneg == 0


def test_unsupported_nsv_and_pattern_errors():
    box, rs = tied(3)
    cb, em, scale = element_matrices(box, 'scaled')
    assert host_assemble(box, rs, em, scale, 2)[0] == -2
    bad = rs.meqn.copy()
    # an element DOF numbered into a column whose pattern lacks the pairing
    free = np.nonzero(bad > 0)[0]
    bad[free[0]], bad[free[-1]] = bad[free[-1]], bad[free[0]]
    sm = np.zeros(rs.neq + rs.nzerol)
    rc = spr.load(8).spr_b200_assemble_ceq(
        _p(rs.mspar), _p(rs.mtrees), _p(rs.msifa), _p(bad), _p(box.madof), _p(box.mpmnpc), _p(box.mmnpc),
        _p(box.mpmceq), _p(box.mmceq), _p(box.ttcc), I8(box.nceq), I8(box.nel), I8(24), _p(em), _p(scale),
        I8(0), _p(sm), None)
    assert rc == -3


def test_general_hex8_matrix_reduces_to_the_unit_cube():
    box = HexBox(2)
    K = hex8_stiffness_xyz(box.element_coords(box.node_coords()), np.full(box.nel, 2.5))
    assert np.allclose(K, 2.5 * hex8_stiffness()[None], rtol=0, atol=1e-15)
    # a stretched element (h = 2 along every axis) scales by h
    K2 = hex8_stiffness_xyz(2.0 * box.element_coords(box.node_coords())[:1], np.ones(1))
    assert np.allclose(K2[0], hex8_stiffness(h=2.0), rtol=0, atol=1e-15)
