"""Adjoint sensitivities (SIMP compliance) on the GPU.

* device assembly (spr_b200_elem_assemble) equals the host SPRADM main add
  bit for bit;
* dL/dtheta from the hand-written backward (one solve on the stored factor +
  spr_b200_elem_grad) equals the gradient built from the reference CPU solve
  (the translated SPR Fortran) to 1e-9, normwise;
* 32^3 box (104,544 equations), theta ~ U[0.2, 1] seed 4, L = f^T u:
  within 1e-6 (normwise relative) of central finite differences on 64
  random elements, Richardson-extrapolated over steps h and h/2
  (h = 1% of theta_e; truncation O(h^4) and rounding both ~1e-8 here).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_device_assembly_bitwise_equals_host():
    import torch
    from sam_lib_b200.adjoint import ElementOps
    from sam_lib_b200.system import HexSystem
    theta = np.random.default_rng(4).uniform(0.2, 1.0, size=12 ** 3)
    scale = theta ** 3
    hs = HexSystem(12, moduli=scale)
    host = hs.assemble()
    ops = ElementOps(hs)
    d_sm = torch.full((hs.neq + hs.nzerol,), np.nan, dtype=torch.float64, device='cuda')
    d_ke = torch.from_numpy(np.asfortranarray(hs.ke).ravel(order='F').copy()).cuda()
    ops.assemble(d_sm, d_ke, torch.from_numpy(scale).cuda())
    assert np.array_equal(d_sm.cpu().numpy(), host)
    # per-element matrices (scale is None): same result
    d_em = torch.from_numpy(np.concatenate([s * hs.ke.ravel(order='F') for s in scale])).cuda()
    d_sm2 = torch.zeros_like(d_sm)
    ops.assemble(d_sm2, d_em)
    assert np.array_equal(d_sm2.cpu().numpy(), host)


def test_adjoint_gradient_matches_reference_cpu_solve():
    import torch
    from conftest import ref_system  # noqa: F401  (sys.path)
    from oracle.refpipe import RefSystem
    from test_oracle import run_sprsol
    from sam_lib_b200.adjoint import SimpModel, simp_solve, tip_load
    from sam_lib_b200.fe import HexBox, hex8_stiffness
    from sam_lib_b200.system import HexSystem
    n = 12
    theta = np.random.default_rng(4).uniform(0.2, 1.0, size=n ** 3)
    hs = HexSystem(n)
    f = tip_load(hs)
    # reference: SPRADM assembly of sum theta^3 K0 and SPRSOL on the CPU
    rs = RefSystem(HexBox(n))
    ke = hex8_stiffness()
    sm = rs.assemble(lambda e: ke * theta[e] ** 3)
    u_ref = run_sprsol('ref', rs, sm, f.reshape(-1, 1).copy())['b'][:, 0]
    eq = hs.element_equations()
    ue = np.where(eq >= 0, u_ref[np.maximum(eq, 0)], 0.0)
    g_ref = -3.0 * theta ** 2 * np.einsum('ei,ij,ej->e', ue, ke, ue)
    # GPU: autograd through the C ABI
    model = SimpModel(hs)
    th = torch.tensor(theta, device='cuda', requires_grad=True)
    ft = torch.tensor(f, device='cuda')
    u = simp_solve(th, ft, model)
    L = torch.dot(ft, u)
    L.backward()
    g = th.grad.cpu().numpy()
    assert np.linalg.norm(u.detach().cpu().numpy() - u_ref) <= 1e-10 * np.linalg.norm(u_ref)
    assert np.linalg.norm(g - g_ref) <= 1e-9 * np.linalg.norm(g_ref)
    assert np.all(g < 0)                        # stiffening any element lowers the compliance


def test_adjoint_gradient_matches_finite_differences_32():
    import torch
    from sam_lib_b200.adjoint import SimpModel, simp_solve, simp_workload
    hs, theta, f = simp_workload(32, seed=4)
    model = SimpModel(hs)
    th = torch.tensor(theta, device='cuda', requires_grad=True)
    ft = torch.tensor(f, device='cuda')
    u = simp_solve(th, ft, model)
    L = torch.dot(ft, u)
    L.backward()
    g = th.grad.cpu().numpy()
    picks = np.random.default_rng(5).choice(theta.size, size=64, replace=False)

    def loss(t):
        with torch.no_grad():
            return float(torch.dot(ft, simp_solve(t, ft, model)))

    base = torch.tensor(theta, device='cuda')
    fd = np.empty(64)
    for i, e in enumerate(picks):
        h = 0.01 * theta[e]
        d = []
        for step in (h, h / 2):
            tp, tm = base.clone(), base.clone()
            tp[e] += step
            tm[e] -= step
            d.append((loss(tp) - loss(tm)) / (2 * step))
        fd[i] = (4 * d[1] - d[0]) / 3
    err = np.linalg.norm(g[picks] - fd) / np.linalg.norm(fd)
    assert err <= 1e-6, err
