"""Adjoint sensitivities of element-parametrised systems through the C ABI.

For K(theta) u = f with K = sum_e s(theta_e) K_e, a loss L(u) has

    K^T lambda = dL/du,      dL/dtheta_e = -lambda_e^T (dK_e/dtheta_e) u_e,
    dL/df = lambda,

where lambda_e, u_e are the element's DOF values.  K is symmetric, so the
adjoint solve reuses the factor of the forward solve (forward + back sweep
of SPRFS1/SPRBS1 semantics, src/SPR/sprfs1.f:5, sprbs1.f:5).  The element
gradient and the assembly (the SPRADM main add, src/SPR/spradm.f:818-859)
are device kernels behind spr_b200_elem_grad / spr_b200_elem_assemble.

``simp_solve(theta, f, model)`` is the torch.autograd entry point for SIMP
stiffness s(theta) = E0 * theta^p: forward = assemble + factor + solve,
backward = one more solve on the stored factor + the element gradient.
Vectors are in SPR equation order (``HexSystem.to_internal``); right-hand
sides are (NRHS, NEQ) tensors, i.e. column-major B.
"""
import ctypes as C

import numpy as np
import torch

from . import DeviceSolver, load, _ptr


def _vp(t):
    return C.c_void_p(0 if t is None else t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class ElementOps:
    """Device element operations of one system: SPRADM assembly (with the
    box's constraint equations, if it has any), hex8 element stiffness and
    the adjoint element gradient.  ``hs`` holds the structure (mspar,
    mtrees, msifa, meqn, neq) and the SAM topology (``hs.box``)."""

    def __init__(self, hs):
        lib = load(8)
        vp = C.c_void_p
        i8 = C.c_int64
        lib.spr_b200_elem_open.argtypes = [vp] * 7 + [i8, i8, C.POINTER(vp)]
        lib.spr_b200_elem_open.restype = C.c_int
        lib.spr_b200_elem_open_ceq.argtypes = [vp] * 9 + [i8, i8, i8, C.POINTER(vp)]
        lib.spr_b200_elem_open_ceq.restype = C.c_int
        lib.spr_b200_elem_close.argtypes = [vp]
        lib.spr_b200_elem_close.restype = None
        lib.spr_b200_elem_assemble.argtypes = [vp, vp, vp, vp, vp]
        lib.spr_b200_elem_assemble.restype = C.c_int
        lib.spr_b200_elem_assemble_ceq.argtypes = [vp] * 7
        lib.spr_b200_elem_assemble_ceq.restype = C.c_int
        lib.spr_b200_elem_hex8.argtypes = [vp, vp, vp, C.c_double, vp, vp]
        lib.spr_b200_elem_hex8.restype = C.c_int
        lib.spr_b200_elem_grad.argtypes = [vp, vp, vp, i8, i8, vp, vp, vp, vp]
        lib.spr_b200_elem_grad.restype = C.c_int
        self.lib = lib
        self.h = C.c_void_p()
        b = hs.box
        self.nceq = int(getattr(b, 'nceq', 0))
        if self.nceq > 0:
            rc = lib.spr_b200_elem_open_ceq(_ptr(hs.mspar), _ptr(hs.mtrees), _ptr(hs.msifa), _ptr(hs.meqn),
                                            _ptr(b.madof), _ptr(b.mpmnpc), _ptr(b.mmnpc), _ptr(b.mpmceq),
                                            _ptr(b.mmceq), self.nceq, b.nel, 24, C.byref(self.h))
        else:
            rc = lib.spr_b200_elem_open(_ptr(hs.mspar), _ptr(hs.mtrees), _ptr(hs.msifa), _ptr(hs.meqn),
                                        _ptr(b.madof), _ptr(b.mpmnpc), _ptr(b.mmnpc), b.nel, 24, C.byref(self.h))
        if rc != 0:
            raise RuntimeError('spr_b200_elem_open failed with %d' % rc)
        self.nel = b.nel
        self.neq = hs.neq

    def assemble(self, d_sm, d_em, d_scale=None, d_sv=None, d_ttcc=None):
        """SM (and SV) = SPRADM over every element; d_ttcc: the constraint
        coefficients on the device (boxes with constraint equations)."""
        if self.nceq > 0 or d_sv is not None:
            rc = self.lib.spr_b200_elem_assemble_ceq(self.h, _vp(d_sm), _vp(d_sv), _vp(d_em), _vp(d_scale),
                                                     _vp(d_ttcc), _stream())
        else:
            rc = self.lib.spr_b200_elem_assemble(self.h, _vp(d_sm), _vp(d_em), _vp(d_scale), _stream())
        if rc != 0:
            raise RuntimeError('spr_b200_elem_assemble failed with %d' % rc)

    def hex8(self, d_xyz, d_E, nu=0.3, out=None):
        """(NEL, 24, 24) element stiffness matrices from node coordinates
        (NANOD, 3) and moduli (NEL,), all on the device; out[e] holds K_e
        column-major (out[e].T is K_e)."""
        out = torch.empty((self.nel, 24, 24), dtype=torch.float64, device=d_xyz.device) if out is None else out
        rc = self.lib.spr_b200_elem_hex8(self.h, _vp(d_xyz), _vp(d_E), float(nu), _vp(out), _stream())
        if rc != 0:
            raise RuntimeError('spr_b200_elem_hex8 failed with %d' % rc)
        return out

    def grad(self, d_u, d_lam, nrhs, d_em, d_dscale=None, out=None):
        out = torch.empty(self.nel, dtype=torch.float64, device=d_u.device) if out is None else out
        rc = self.lib.spr_b200_elem_grad(self.h, _vp(d_u), _vp(d_lam), self.neq, nrhs, _vp(d_em),
                                         _vp(d_dscale), _vp(out), _stream())
        if rc != 0:
            raise RuntimeError('spr_b200_elem_grad failed with %d' % rc)
        return out

    def close(self):
        if self.h:
            self.lib.spr_b200_elem_close(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SimpModel:
    """Device state of a SIMP-parametrised hex system: structure, element
    matrix, SM buffer (holds the factor of the last forward) and solver."""

    def __init__(self, hs, penal=3.0, e0=1.0, device='cuda'):
        self.hs = hs
        self.penal = float(penal)
        self.e0 = float(e0)
        self.solver = DeviceSolver(hs.mspar, hs.mtrees, hs.msifa)
        self.elements = ElementOps(hs)
        self.d_ke = torch.from_numpy(np.asfortranarray(hs.ke).ravel(order='F').copy()).to(device)
        self.d_sm = torch.empty(hs.neq + hs.nzerol, dtype=torch.float64, device=device)
        self.version = 0
        self.last = None

    def factor(self, theta):
        scale = self.e0 * theta.detach() ** self.penal
        self.elements.assemble(self.d_sm, self.d_ke, scale.contiguous())
        r = self.solver.factor(self.d_sm)
        if r['lierr'] != 0:
            raise RuntimeError('factorisation failed: LIERR %d at equation %d' % (r['lierr'], r['supeqt']))
        self.version += 1
        self.last = r
        return r

    def solve(self, b):
        """Solves with the stored factor; b (NEQ,) or (NRHS, NEQ) is not modified."""
        x = b.detach().clone().contiguous()
        self.solver.solve(self.d_sm, x, 1 if x.dim() == 1 else x.shape[0])
        return x


class SimpSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, f, model):
        model.factor(theta)
        u = model.solve(f)
        ctx.model = model
        ctx.version = model.version
        ctx.save_for_backward(theta, u)
        return u

    @staticmethod
    def backward(ctx, gu):
        model = ctx.model
        theta, u = ctx.saved_tensors
        if model.version != ctx.version:
            raise RuntimeError('the factor of this forward was replaced by a later forward; '
                               'run backward before the next forward on the same model')
        lam = model.solve(gu)
        nrhs = 1 if u.dim() == 1 else u.shape[0]
        dscale = (model.e0 * model.penal) * theta.detach() ** (model.penal - 1.0)
        g = model.elements.grad(u, lam, nrhs, model.d_ke, dscale.contiguous())
        return g, lam, None


def simp_solve(theta, f, model):
    """u = K(theta)^-1 f with K = sum_e E0 theta_e^p K_e; differentiable in theta and f."""
    return SimpSolve.apply(theta, f, model)


def tip_load(hs, total=1.0):
    """Downward (-z) load of the given resultant on the face x = n, spread as a
    uniform traction (each face cell sends a quarter to each of its nodes);
    returned in equation order."""
    b = hs.box
    n1 = b.n + 1
    f = np.zeros(b.ndof)
    share = total / (b.n * b.n) / 4.0
    for k in range(b.n):
        for j in range(b.n):
            for dj, dk in ((0, 0), (1, 0), (0, 1), (1, 1)):
                node = b.n + n1 * ((j + dj) + n1 * (k + dk))
                f[3 * node + 2] -= share
    return hs.to_internal(f)


def simp_workload(n=32, seed=4):
    """theta_e ~ U[0.2, 1] (numpy default_rng(seed)), and the tip load."""
    from .system import HexSystem
    hs = HexSystem(n)
    theta = np.random.default_rng(seed).uniform(0.2, 1.0, size=hs.box.nel)
    return hs, theta, tip_load(hs)
