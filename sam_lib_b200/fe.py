"""Synthetic finite-element host data: hex8 boxes in SAM's control-array form.

SPR is called by a finite-element host program that owns the SAM control
arrays (MPAR, MADOF, MINEX, MPMNPC, MMNPC, MPMCEQ, MMCEQ, MSC) and computes
the element matrices.  The reference ships no element routines, so this
module plays the host's part for the seeded workloads:

* an ``n x n x n`` box of unit-cube 8-node trilinear hex elements, 3 DOF per
  node, the face x=0 clamped through status code MSC=0
  (the status-code meaning follows ``src/SPR/sprseq.f:60-80``: 1 and 2 are
  free, 0 is fixed);
* the 24x24 isotropic linear-elastic hex8 stiffness with 2x2x2 Gauss
  integration, scaled per element by its Young's modulus;
* a lumped (diagonal) mass with density 1 (nodal mass = sum of volume/8).

Arrays are 1-based Fortran-style contents stored in 0-based numpy arrays,
exactly as a Fortran host would pass them.
"""
import numpy as np

HEX8_CORNERS = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                         [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=np.int64)


class HexBox:
    """SAM control arrays of an n^3 hex8 box, face x=0 clamped.

    retain_face=True marks the DOFs of the face x=n as external (MSC = 2): the
    reference pipeline then numbers them last and makes their supernodes the
    retained (superelement) ones, SUPSUP > 0 (src/SPR/sprtrs.f:1142-1204)."""

    def __init__(self, n, ndof_per_node=3, clamp_face=True, retain_face=False):
        self.n = int(n)
        n1 = self.n + 1
        self.nanod = n1 ** 3
        self.nel = self.n ** 3
        self.nndof = ndof_per_node
        self.ndof = self.nanod * ndof_per_node
        # node (i,j,k) -> 1 + i + n1*(j + n1*k); i runs along x
        i, j, k = np.meshgrid(np.arange(self.n), np.arange(self.n), np.arange(self.n),
                              indexing='ij')
        i = i.transpose(2, 1, 0).ravel()
        j = j.transpose(2, 1, 0).ravel()
        k = k.transpose(2, 1, 0).ravel()
        conn = np.empty((self.nel, 8), dtype=np.int64)
        for c, (di, dj, dk) in enumerate(HEX8_CORNERS):
            conn[:, c] = 1 + (i + di) + n1 * ((j + dj) + n1 * (k + dk))
        self.conn = conn                                    # 1-based node numbers
        self.mpmnpc = np.arange(1, 8 * self.nel + 2, 8, dtype=np.int64)
        self.mmnpc = conn.ravel().copy()
        self.madof = np.arange(1, self.ndof + 2, ndof_per_node, dtype=np.int64)
        self.minex = np.arange(1, self.nanod + 1, dtype=np.int64)
        self.mpmceq = np.ones(1, dtype=np.int64)
        self.mmceq = np.zeros(1, dtype=np.int64)
        msc = np.ones(self.ndof, dtype=np.int64)
        if clamp_face:
            node_i = (np.arange(self.nanod) % n1)
            fixed_nodes = np.nonzero(node_i == 0)[0]
            for d in range(ndof_per_node):
                msc[fixed_nodes * ndof_per_node + d] = 0
        if retain_face:
            node_i = (np.arange(self.nanod) % n1)
            ext_nodes = np.nonzero(node_i == self.n)[0]
            for d in range(ndof_per_node):
                msc[ext_nodes * ndof_per_node + d] = 2
        self.msc = msc
        self.mpar = np.zeros(50, dtype=np.int64)
        self.mpar[0] = self.nanod       # MPAR(1) NANOD
        self.mpar[1] = self.nel         # MPAR(2) NEL
        self.mpar[2] = self.ndof        # MPAR(3) NDOF
        self.mpar[6] = 0                # MPAR(7) NCEQ

    @property
    def neq(self):
        return int(np.count_nonzero(self.msc))

    def node_coords(self):
        n1 = self.n + 1
        idx = np.arange(self.nanod)
        return np.stack([idx % n1, (idx // n1) % n1, idx // (n1 * n1)], axis=1).astype(np.float64)

    def lumped_mass(self, density=1.0):
        """Nodal lumped mass per DOF (length NDOF): sum over elements of vol/8."""
        m = np.zeros(self.nanod)
        np.add.at(m, self.conn.ravel() - 1, density / 8.0)
        return np.repeat(m, self.nndof)


def hex8_stiffness(E=1.0, nu=0.3, h=1.0):
    """24x24 stiffness of a cube of side h, 2x2x2 Gauss, node-major DOFs."""
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[0, 0] = D[1, 1] = D[2, 2] = lam + 2 * mu
    D[3, 3] = D[4, 4] = D[5, 5] = mu
    sgn = 2 * HEX8_CORNERS - 1                   # corner signs in [-1,1]^3
    g = 1.0 / np.sqrt(3.0)
    K = np.zeros((24, 24))
    for xi in (-g, g):
        for eta in (-g, g):
            for zeta in (-g, g):
                # derivatives of N_a = (1+xi xi_a)(1+eta eta_a)(1+zeta zeta_a)/8
                dN = np.empty((8, 3))
                dN[:, 0] = sgn[:, 0] * (1 + eta * sgn[:, 1]) * (1 + zeta * sgn[:, 2]) / 8
                dN[:, 1] = sgn[:, 1] * (1 + xi * sgn[:, 0]) * (1 + zeta * sgn[:, 2]) / 8
                dN[:, 2] = sgn[:, 2] * (1 + xi * sgn[:, 0]) * (1 + eta * sgn[:, 1]) / 8
                dNdx = dN * (2.0 / h)            # J = (h/2) I
                detJ = (h / 2.0) ** 3
                B = np.zeros((6, 24))
                for a in range(8):
                    bx, by, bz = dNdx[a]
                    c = 3 * a
                    B[0, c] = bx
                    B[1, c + 1] = by
                    B[2, c + 2] = bz
                    B[3, c] = by
                    B[3, c + 1] = bx
                    B[4, c + 1] = bz
                    B[4, c + 2] = by
                    B[5, c] = bz
                    B[5, c + 2] = bx
                K += B.T @ D @ B * detJ
    return 0.5 * (K + K.T)


def element_moduli(nel, kind='uniform', seed=None, lo=1.0, hi=1.0e4):
    """Per-element Young's modulus for the seeded workloads."""
    if kind == 'uniform':
        return np.ones(nel)
    rng = np.random.default_rng(seed)
    if kind == 'loguniform':
        return np.exp(rng.uniform(np.log(lo), np.log(hi), size=nel))
    raise ValueError(kind)
