"""Mixed precision: 3xTF32 Schur updates with FP64 iterative refinement.

The factor of the large fronts uses split-TF32 products (three tensor-core
products per update): mode 1 on tcgen05 (TMA-fed, FP32 accumulation in
tensor memory over the whole update), mode 2 through mma.sync (FP32
accumulation per 64-wide slice, FP64 across slices); diagonal blocks,
pivots, TRSM and storage stay FP64.  Refinement
runs against the FP64 matrix (CSR compacted from the assembled SM on the
device) until the normwise backward error

    max|b - K x| / (||K||inf max|x| + max|b|)  <=  1e-12

Checks: inertia (NUMNEG) equal to the FP64 factor's; for SPD systems the
mixed factor within 1e-5 of the FP64 factor (relative to max|SM|; an
indefinite LDL' without pivoting amplifies the perturbation through its
element growth, so there only the refined result is checked); the
backward error the device reports is recomputed on the host from scipy's
product; the refined solution agrees with the FP64 solution.
"""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


def _system(n, emod, sigma_factor):
    from sam_lib_b200.fe import element_moduli
    from sam_lib_b200.system import HexSystem, diag_positions, shift_diagonal, sm_to_csr
    from sam_lib_b200.workloads import lambda1
    hs = HexSystem(n, moduli=element_moduli(n ** 3, emod, seed=2))
    sm = hs.assemble()
    if sigma_factor:
        pos = diag_positions(hs.mspar, hs.mtrees, hs.msifa)
        mass = hs.to_internal(hs.box.lumped_mass())
        sm = shift_diagonal(sm, pos, mass, sigma_factor * lambda1(n))
    K = sm_to_csr(hs.mspar, hs.mtrees, hs.msifa, sm)
    return hs, sm, K


def _host_berr(K, x, b):
    r = b - K @ x
    knorm = abs(K).sum(axis=1).max()
    return max(np.max(np.abs(r[:, q])) / (knorm * np.max(np.abs(x[:, q])) + np.max(np.abs(b[:, q])))
               for q in range(b.shape[1]))


@pytest.mark.parametrize('mode', [1, 2])
@pytest.mark.parametrize('n,emod,sigma_factor', [(16, 'uniform', 0.0), (16, 'loguniform', 0.0),
                                                 (20, 'uniform', 2.5)])
def test_mixed_factor_refined_to_fp64_backward_error(n, emod, sigma_factor, mode):
    import torch
    import sam_lib_b200 as spr
    hs, sm, K = _system(n, emod, sigma_factor)
    nrhs = 4
    b = np.random.default_rng(7).uniform(-1.0, 1.0, size=(hs.neq, nrhs))
    ds = spr.DeviceSolver(hs.mspar, hs.mtrees, hs.msifa)
    d_sm0 = torch.from_numpy(sm).cuda()
    ds.build_residual(d_sm0)
    d_b = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()      # (NRHS, NEQ) = column-major B

    # FP64 reference factor + solve
    d_f64 = d_sm0.clone()
    r64 = ds.factor(d_f64)
    x64 = d_b.clone()
    ds.solve(d_f64, x64, nrhs)
    # FP64 residual through the device operator: backward error at rounding level
    d_x = torch.empty_like(d_b)
    it0, berr64, _ = ds.refine(d_f64, d_b, d_x, nrhs, tol=1e-12, maxit=0)
    assert it0 == 0 and berr64 <= 1e-13

    # mixed factor + refinement
    ds.set_mode(mode)
    d_mx = d_sm0.clone()
    rmx = ds.factor(d_mx)
    ds.set_mode(False)
    assert rmx['lierr'] == 0 and r64['lierr'] == 0
    assert rmx['numneg'] == r64['numneg']
    if sigma_factor:
        assert rmx['numneg'] > 0
    f64, fmx = d_f64.cpu().numpy(), d_mx.cpu().numpy()
    dmax = np.max(np.abs(fmx - f64)) / np.max(np.abs(f64))
    assert dmax > 0.0                                # the mixed path really ran
    if not sigma_factor:
        assert dmax <= 1e-5, dmax
    d_x.zero_()
    it, berr, _ = ds.refine(d_mx, d_b, d_x, nrhs, tol=1e-12, maxit=20)
    assert berr <= 1e-12 and 1 <= it <= 10, (it, berr)
    x = d_x.cpu().numpy().T
    hb = _host_berr(K, x, b)
    assert hb <= 2e-12, hb
    assert abs(hb - berr) <= 0.5 * max(hb, berr)
    xr = x64.cpu().numpy().T
    assert np.linalg.norm(x - xr) <= (1e-9 if emod == 'uniform' else 1e-5) * np.linalg.norm(xr)
    ds.close()


def test_autotune_keeps_refinement_to_fp64_backward_error():
    """The autotuner picks the tensor-core/FP64 split of the mixed factor on a
    copy of the assembled SM; the chosen setting still refines to 1e-12 with
    the FP64 factor's inertia."""
    import torch
    import sam_lib_b200 as spr
    hs, sm, K = _system(20, 'uniform', 2.5)
    nrhs = 2
    b = np.random.default_rng(3).uniform(-1.0, 1.0, size=(hs.neq, nrhs))
    ds = spr.DeviceSolver(hs.mspar, hs.mtrees, hs.msifa)
    st = torch.cuda.Stream()
    ds.set_stream(st.cuda_stream)
    d_sm0 = torch.from_numpy(sm).cuda()
    ds.build_residual(d_sm0)
    ref = ds.factor(d_sm0.clone())
    tuned = ds.autotune(d_sm0)
    assert tuned['candidates'] == 13 and tuned['factor_ms'] > 0 and tuned['far_sm_quarters'] in (2, 3, 4)
    assert np.array_equal(d_sm0.cpu().numpy(), sm)                  # the caller's SM is untouched
    ds.set_mode(1)
    d_mx = d_sm0.clone()
    r = ds.factor(d_mx)
    assert r['numneg'] == ref['numneg'] and r['lierr'] == 0
    d_b = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    d_x = torch.empty_like(d_b)
    it, berr, _ = ds.refine(d_mx, d_b, d_x, nrhs, tol=1e-12, maxit=20)
    assert berr <= 1e-12, (it, berr)
    assert _host_berr(K, d_x.cpu().numpy().T, b) <= 2e-12
    ds.close()
