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
* a lumped (diagonal) mass with density 1 (nodal mass = sum of volume/8);
* the same stiffness for general (distorted) hexahedra from nodal
  coordinates (isoparametric map, 2x2x2 Gauss), the host restatement of the
  device element kernel;
* optionally, SAM constraint equations (MPMCEQ/MMCEQ/TTCC): the x-DOFs of the
  face x=n tied to two master nodes (multi-point constraints) and the
  z-DOFs of one edge prescribed (the layout of ``src/SPR/sprseq.f:120-145``:
  MMCEQ(MPMCEQ(i)) is the slave or prescribed DOF with MSC = 0, the entries
  after it its masters; TTCC(MPMCEQ(i)) the constant term, then the master
  coefficients).

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

    def __init__(self, n, ndof_per_node=3, clamp_face=True, retain_face=False, ties=False,
                 prescribed=-0.01):
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
        self.ttcc = np.zeros(1)
        if ties:
            self._tie_face(msc, prescribed)
        self.msc = msc
        self.mpar = np.zeros(50, dtype=np.int64)
        self.mpar[0] = self.nanod       # MPAR(1) NANOD
        self.mpar[1] = self.nel         # MPAR(2) NEL
        self.mpar[2] = self.ndof        # MPAR(3) NDOF
        self.mpar[6] = len(self.mpmceq) - 1 if ties else 0   # MPAR(7) NCEQ

    @property
    def nceq(self):
        return int(self.mpar[6])

    def _tie_face(self, msc, prescribed):
        """Constraint equations on the face x=n (not clamped, not retained):
        u_x(s) = c0 + 0.3 u_x(m1) + 0.7 u_x(m2) for every face node s but the
        masters m1 = (n,0,0) and m2 = (n,n,n), with c0 = prescribed/5 (the
        first one u_x(s) = u_x(m1) + 0 u_x(m2), a zero coefficient); u_z =
        prescribed (a constraint equation without masters) on the edge
        x=n, y=n below m2."""
        n1 = self.n + 1
        nd = self.nndof
        face = [self.n + n1 * (j + n1 * k) for k in range(n1) for j in range(n1)]
        m1, m2 = self.n, self.n + n1 * (self.n + n1 * self.n)
        ptr, mm, tt = [1], [], []
        for node in face:
            if node in (m1, m2):
                continue
            slave = node * nd + 1                      # 1-based x-DOF
            mm += [slave, m1 * nd + 1, m2 * nd + 1]
            tt += [0.0, 1.0, 0.0] if len(ptr) == 1 else [prescribed / 5, 0.3, 0.7]
            ptr.append(ptr[-1] + 3)
            msc[slave - 1] = 0
        for k in range(self.n):
            node = self.n + n1 * (self.n + n1 * k)
            dof = node * nd + 3                        # 1-based z-DOF
            mm.append(dof)
            tt.append(prescribed)
            ptr.append(ptr[-1] + 1)
            msc[dof - 1] = 0
        self.mpmceq = np.array(ptr, dtype=np.int64)
        self.mmceq = np.array(mm, dtype=np.int64)
        self.ttcc = np.array(tt, dtype=np.float64)

    @property
    def neq(self):
        return int(np.count_nonzero(self.msc))

    def node_coords(self):
        n1 = self.n + 1
        idx = np.arange(self.nanod)
        return np.stack([idx % n1, (idx // n1) % n1, idx // (n1 * n1)], axis=1).astype(np.float64)

    def distorted_coords(self, seed, amp=0.15):
        """Node coordinates of the box with every node moved by U[-amp, amp]
        per direction (numpy default_rng(seed), one (NANOD, 3) draw); for
        amp < 0.25 every element keeps a positive Jacobian."""
        rng = np.random.default_rng(seed)
        return self.node_coords() + rng.uniform(-amp, amp, size=(self.nanod, 3))

    def element_coords(self, xyz):
        """(NEL, 8, 3) corner coordinates of every element in MMNPC order."""
        return xyz[self.conn - 1]

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


def hex8_stiffness_xyz(xe, E, nu=0.3):
    """24x24 stiffness of general hexahedra, node-major DOFs, 2x2x2 Gauss:
    xe (nel, 8, 3) corner coordinates in HEX8_CORNERS order, E (nel,).
    K_e = sum_g det J_g B_g^T D B_g with B from dN/dx = J^-1 dN/dxi and
    J_ij = sum_a dN_a/dxi_i x_a,j.  Returns (nel, 24, 24)."""
    xe = np.asarray(xe, dtype=np.float64)
    E = np.asarray(E, dtype=np.float64)
    nel = xe.shape[0]
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    D = np.zeros((nel, 6, 6))
    D[:, :3, :3] = lam[:, None, None]
    for i in range(3):
        D[:, i, i] = lam + 2 * mu
        D[:, 3 + i, 3 + i] = mu
    sgn = 2 * HEX8_CORNERS - 1
    g = 1.0 / np.sqrt(3.0)
    K = np.zeros((nel, 24, 24))
    for zeta in (-g, g):
        for eta in (-g, g):
            for xi in (-g, g):
                dN = np.empty((8, 3))
                dN[:, 0] = sgn[:, 0] * (1 + eta * sgn[:, 1]) * (1 + zeta * sgn[:, 2]) / 8
                dN[:, 1] = sgn[:, 1] * (1 + xi * sgn[:, 0]) * (1 + zeta * sgn[:, 2]) / 8
                dN[:, 2] = sgn[:, 2] * (1 + xi * sgn[:, 0]) * (1 + eta * sgn[:, 1]) / 8
                J = np.einsum('ai,eaj->eij', dN, xe)
                detJ = np.linalg.det(J)
                dNdx = np.linalg.solve(J, np.broadcast_to(dN.T, (nel, 3, 8)))   # (nel, 3, 8)
                B = np.zeros((nel, 6, 24))
                for a in range(8):
                    bx, by, bz = dNdx[:, 0, a], dNdx[:, 1, a], dNdx[:, 2, a]
                    c = 3 * a
                    B[:, 0, c] = bx
                    B[:, 1, c + 1] = by
                    B[:, 2, c + 2] = bz
                    B[:, 3, c] = by
                    B[:, 3, c + 1] = bx
                    B[:, 4, c + 1] = bz
                    B[:, 4, c + 2] = by
                    B[:, 5, c] = bz
                    B[:, 5, c + 2] = bx
                K += np.einsum('eki,ekl,elj->eij', B, D, B) * detJ[:, None, None]
    return K


def element_moduli(nel, kind='uniform', seed=None, lo=1.0, hi=1.0e4):
    """Per-element Young's modulus for the seeded workloads."""
    if kind == 'uniform':
        return np.ones(nel)
    rng = np.random.default_rng(seed)
    if kind == 'loguniform':
        return np.exp(rng.uniform(np.log(lo), np.log(hi), size=nel))
    raise ValueError(kind)
