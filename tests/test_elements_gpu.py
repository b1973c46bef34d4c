"""Device element stiffness and SPRADM with constraint equations (GPU).

* spr_b200_elem_hex8 (isoparametric hex8, 2x2x2 Gauss, from node
  coordinates) against the numpy restatement fe.hex8_stiffness_xyz on a
  distorted box with log-uniform moduli: max |difference| <= 1e-13 of
  max |K| (the two sum the same terms in different orders);
* device assembly of the device matrices equals the host SPRADM
  restatement of the same matrices bit for bit, and the factor + solve of
  that system through sprsol_ matches the translated reference's SPRSOL on
  the same SM;
* the constrained box: device SM and SV (spr_b200_elem_assemble_ceq) equal
  the host assembly, which the CPU tests pin to the reference's SPRADM,
  bit for bit; the GPU solve of K u = SV matches the reference's solve.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

I8 = C.c_int64


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _ops_and_matrices(n, seed=5):
    import torch
    from oracle.refpipe import RefSystem
    from sam_lib_b200.adjoint import ElementOps
    from sam_lib_b200.fe import HexBox, element_moduli
    box = HexBox(n)
    rs = RefSystem(box)
    xyz = box.distorted_coords(seed)
    E = element_moduli(box.nel, 'loguniform', seed=3)
    ops = ElementOps(rs)
    d_em = ops.hex8(torch.from_numpy(xyz).cuda(), torch.from_numpy(E).cuda(), 0.3)
    return box, rs, ops, xyz, E, d_em


@pytest.mark.parametrize('n', [4, 10])
def test_hex8_kernel_matches_numpy(n):
    from sam_lib_b200.fe import hex8_stiffness_xyz
    box, rs, ops, xyz, E, d_em = _ops_and_matrices(n)
    K = d_em.cpu().numpy().transpose(0, 2, 1)               # column-major per element
    Kn = hex8_stiffness_xyz(box.element_coords(xyz), E)
    scale = np.abs(Kn).max(axis=(1, 2))
    err = (np.abs(K - Kn).max(axis=(1, 2)) / scale).max()
    assert err <= 1e-13, err
    assert np.array_equal(K, K.transpose(0, 2, 1))          # exactly symmetric


def test_hex8_unit_cube_equals_reference_element():
    import torch
    from oracle.refpipe import RefSystem
    from sam_lib_b200.adjoint import ElementOps
    from sam_lib_b200.fe import HexBox, hex8_stiffness
    box = HexBox(3)
    ops = ElementOps(RefSystem(box))
    d_em = ops.hex8(torch.from_numpy(box.node_coords()).cuda(), torch.ones(box.nel, dtype=torch.float64,
                                                                             device='cuda'))
    K = d_em.cpu().numpy().transpose(0, 2, 1)
    assert np.abs(K - hex8_stiffness()[None]).max() <= 1e-15


@pytest.mark.parametrize('n', [8])
def test_device_hex8_system_factor_and_solve_match_reference(n):
    import torch
    import sam_lib_b200 as spr
    box, rs, ops, xyz, E, d_em = _ops_and_matrices(n)
    d_sm = torch.full((rs.neq + rs.nzerol,), np.nan, dtype=torch.float64, device='cuda')
    ops.assemble(d_sm, d_em)
    sm = d_sm.cpu().numpy()
    em = d_em.cpu().numpy().reshape(-1)
    host = np.zeros_like(sm)
    rc = spr.load(8).spr_b200_assemble(_p(rs.mspar), _p(rs.mtrees), _p(rs.msifa), _p(rs.meqn), _p(box.madof),
                                       _p(box.mpmnpc), _p(box.mmnpc), I8(box.nel), I8(24), _p(em), None,
                                       _p(host))
    assert rc == 0 and np.array_equal(sm, host)
    b = np.asfortranarray(np.random.default_rng(7).uniform(-1, 1, size=(rs.neq, 2)))
    ref_sm, ref_b = sm.copy(), b.copy(order='F')
    ierr, tol_r, nneg = rs.sprsol(3, ref_sm, ref_b)
    assert ierr == 0
    g_sm, g_b = sm.copy(), b.copy(order='F')
    tol = np.array([1e-12, 0.0, 0.0])
    ms = rs.mspar.copy()
    assert spr.sprsol(3, ms, rs.mtrees, rs.msifa, g_sm, g_b, rs.neq, 2, tol) == 0
    assert ms[25] == nneg
    assert np.abs(g_sm - ref_sm).max() <= 1e-10 * np.abs(ref_sm).max()
    assert np.linalg.norm(g_b - ref_b) <= 1e-10 * np.linalg.norm(ref_b)
    spr.release_all()


@pytest.mark.parametrize('n', [4, 7])
def test_constrained_device_assembly_and_solve(n):
    import torch
    import sam_lib_b200 as spr
    from test_assembly_ceq_cpu import element_matrices, host_assemble, tied
    box, rs = tied(n)
    cb, em, scale = element_matrices(box, 'distorted')
    rc, sm_h, sv_h = host_assemble(box, rs, em, scale, 1)
    assert rc == 0
    from sam_lib_b200.adjoint import ElementOps
    ops = ElementOps(rs)
    d_em = torch.from_numpy(em.reshape(-1)).cuda()
    d_tt = torch.from_numpy(box.ttcc).cuda()
    d_sm = torch.full((rs.neq + rs.nzerol,), np.nan, dtype=torch.float64, device='cuda')
    d_sv = torch.full((rs.neq,), np.nan, dtype=torch.float64, device='cuda')
    ops.assemble(d_sm, d_em, d_sv=d_sv, d_ttcc=d_tt)
    assert np.array_equal(d_sm.cpu().numpy(), sm_h)
    assert np.array_equal(d_sv.cpu().numpy(), sv_h)
    # NSV = -1 (SV only) and NSV = 0 (SM only)
    d_sv2 = torch.full_like(d_sv, np.nan)
    ops.assemble(None, d_em, d_sv=d_sv2, d_ttcc=d_tt)
    assert np.array_equal(d_sv2.cpu().numpy(), sv_h)
    d_sm2 = torch.full_like(d_sm, np.nan)
    ops.assemble(d_sm2, d_em, d_ttcc=d_tt)
    assert np.array_equal(d_sm2.cpu().numpy(), sm_h)
    # K u = SV on the GPU against the reference's SPRSOL
    ref_sm, ref_b = sm_h.copy(), sv_h.copy()
    ierr, _, nneg = rs.sprsol(3, ref_sm, ref_b)
    assert ierr == 0
    g_sm, g_b = sm_h.copy(), np.asfortranarray(sv_h.reshape(-1, 1).copy())
    ms = rs.mspar.copy()
    assert spr.sprsol(3, ms, rs.mtrees, rs.msifa, g_sm, g_b, rs.neq, 1,
                      np.array([1e-12, 0.0, 0.0])) == 0
    assert ms[25] == nneg
    assert np.linalg.norm(g_b[:, 0] - ref_b) <= 1e-10 * np.linalg.norm(ref_b)
    spr.release_all()
