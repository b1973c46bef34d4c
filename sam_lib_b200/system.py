"""An SPR system on the host: structure + assembled SM, as a Fortran host holds it.

The symbolic structure (MSPAR, MTREES, MSIFA, MEQN) is the reference's own:
SPR's minimum-degree ordering, supernode partition and symbolic factorisation
run on the host in the reference library (src/SPR/sprrnm.f, sprtrs.f,
sprsmb.f).  For the seeded benchmark meshes their outputs are stored as
compressed package data (sam_lib_b200/structures/hex<n>.npz, produced by
tests/golden/make_structures.py from the reference pipeline).  Assembly into SM is done here by the
library's own bit-exact SPRADM main add (spr_b200_assemble).
"""
import ctypes as C
import os

import numpy as np

from . import load
from .fe import HexBox, hex8_stiffness

STRUCT_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'structures')


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def load_structure(n):
    """MSPAR (60), MTREES, MSIFA, MEQN, RINFO of the n^3 box (int64)."""
    z = np.load(os.path.join(STRUCT_DIR, 'hex%d.npz' % n))
    und = lambda d: np.cumsum(d.astype(np.int64))   # noqa: E731
    return dict(mspar=z['mspar'].astype(np.int64).copy(), mtrees=und(z['mtrees_d']),
                msifa=und(z['msifa_d']), meqn=und(z['meqn_d']), rinfo=z['rinfo'].copy())


class HexSystem:
    """n^3 hex8 box: SAM control arrays, SPR structure and assembled SM."""

    def __init__(self, n, moduli=None, nu=0.3):
        self.box = HexBox(n)
        st = load_structure(n)
        self.mspar, self.mtrees, self.msifa = st['mspar'], st['mtrees'], st['msifa']
        self.meqn, self.rinfo = st['meqn'], st['rinfo']
        self.neq = int(self.mspar[7])
        self.nzerol = int(self.mspar[15])
        self.ke = np.asfortranarray(hex8_stiffness(1.0, nu))
        self.moduli = np.ones(self.box.nel) if moduli is None else np.asarray(moduli, dtype=np.float64)

    def assemble(self, out=None):
        """SM = [D(NEQ) | LNZ(NZEROL)] with K = sum_e E_e K_ref (SPRADM order)."""
        sm = np.zeros(self.neq + self.nzerol) if out is None else out
        if out is not None:
            sm[:] = 0.0
        rc = load(8).spr_b200_assemble(
            _p(self.mspar), _p(self.mtrees), _p(self.msifa), _p(self.meqn), _p(self.box.madof),
            _p(self.box.mpmnpc), _p(self.box.mmnpc), C.c_int64(self.box.nel), C.c_int64(24),
            _p(self.ke), _p(self.moduli), _p(sm))
        if rc != 0:
            raise RuntimeError('spr_b200_assemble failed: %d' % rc)
        return sm

    def to_internal(self, f_dof):
        """Per-DOF vector (NDOF) -> SPR equation order via MEQN."""
        b = np.zeros(self.neq)
        sel = self.meqn > 0
        b[self.meqn[sel] - 1] = f_dof[sel]
        return b

    def element_equations(self):
        """(NEL, 24) equation numbers (0-based, -1 for fixed DOFs)."""
        dofs = (self.box.conn - 1)[:, :, None] * 3 + np.arange(3)[None, None, :]
        return self.meqn[dofs.reshape(self.box.nel, 24)] - 1

    def matvec(self, x):
        """K x from the element matrices (for residuals): x (NEQ,) or (NEQ, k)."""
        eq = self.element_equations()
        x2 = x.reshape(self.neq, -1)
        out = np.zeros_like(x2)
        m = eq >= 0
        xe = np.where(m[:, :, None], x2[np.maximum(eq, 0)], 0.0)
        ye = np.einsum('ij,ejk->eik', self.ke, xe) * self.moduli[:, None, None]
        np.add.at(out, eq[m], ye[m])
        return out.reshape(x.shape)


def diag_positions(mspar, mtrees, msifa):
    """0-based index into SM of each equation's diagonal (inside LNZ), cf. SPRDG1."""
    neq, ns = int(mspar[7]), int(mspar[10])
    xs = mtrees[mspar[44] - 1: mspar[44] + ns]
    xl = mtrees[mspar[45] - 1: mspar[45] + ns]
    xlnz = msifa[mspar[47] - 1: mspar[47] + ns]
    pos = np.empty(neq, dtype=np.int64)
    for js in range(ns):
        F = xl[js + 1] - xl[js]
        j = np.arange(xs[js + 1] - xs[js])
        pos[xs[js] - 1 + j] = neq + (xlnz[js] - 1) + j * F - (j * (j - 1)) // 2
    return pos


def shift_diagonal(sm, pos, mass, sigma):
    """A - sigma*B for a diagonal B (SPRSHA KSB=2, src/SPR/sprsha.f:86-93)."""
    out = sm.copy()
    out[pos] -= sigma * mass
    return out


def sm_to_csr(mspar, mtrees, msifa, sm):
    """Full symmetric scipy CSR of the matrix held (lower part) in LNZ, zeros dropped."""
    import scipy.sparse as sp
    neq, ns = int(mspar[7]), int(mspar[10])
    xs = mtrees[mspar[44] - 1: mspar[44] + ns]
    xl = mtrees[mspar[45] - 1: mspar[45] + ns]
    lindx = msifa[mspar[46] - 1:]
    xlnz = msifa[mspar[47] - 1: mspar[47] + ns]
    rows, cols, vals = [], [], []
    lnz = sm[neq:]
    for js in range(ns):
        F = int(xl[js + 1] - xl[js])
        r = lindx[xl[js] - 1: xl[js + 1] - 1] - 1
        p = int(xlnz[js] - 1)
        for j in range(int(xs[js + 1] - xs[js])):
            v = lnz[p: p + F - j]
            nz = v != 0.0
            rows.append(r[j:][nz])
            cols.append(np.full(int(nz.sum()), xs[js] - 1 + j))
            vals.append(v[nz])
            p += F - j
    rows, cols, vals = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
    L = sp.coo_matrix((vals, (rows, cols)), shape=(neq, neq)).tocsr()
    return (L + sp.tril(L, -1).T).tocsr()
