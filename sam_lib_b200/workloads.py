"""Seeded synthetic workloads of the benchmark configurations.

All meshes are n^3 boxes of unit-cube hex8 elements, 3 DOF per node, nu=0.3,
face x=0 clamped; structures are the reference's (see system.py).

Config 4 (batched uneven shifted LDL'), draw order from
numpy.random.default_rng(3): the 512 box sizes n ~ U{3..12}; then the 512
shift factors U[0.5, 2]; then, system by system, 16 right-hand sides
U[-1, 1] of that system's NEQ (column-major).  Each system is K - sigma*M
with lumped mass (density 1), sigma = factor * lambda1(n), lambda1(n) the
lowest eigenvalue of (K, M) from shift-invert Lanczos (scipy eigsh, sigma=0,
v0 = ones).
"""
import functools

import numpy as np

from .system import HexSystem, diag_positions, shift_diagonal, sm_to_csr


@functools.lru_cache(maxsize=None)
def hex_system(n):
    hs = HexSystem(n)
    sm = hs.assemble()
    sm.setflags(write=False)
    pos = diag_positions(hs.mspar, hs.mtrees, hs.msifa)
    mass = hs.to_internal(hs.box.lumped_mass())
    return hs, sm, pos, mass


@functools.lru_cache(maxsize=None)
def lambda1(n):
    """Lowest eigenvalue of K x = lambda M x for the n^3 box (shift-invert Lanczos)."""
    import scipy.sparse as sp
    from scipy.sparse.linalg import eigsh
    hs, sm, pos, mass = hex_system(n)
    K = sm_to_csr(hs.mspar, hs.mtrees, hs.msifa, sm)
    M = sp.diags(mass)
    w = eigsh(K, k=1, M=M, sigma=0.0, which='LM', v0=np.ones(hs.neq), return_eigenvectors=False)
    return float(w[0])


def config4_draws(count=512, seed=3):
    """(rng, box sizes n, shift factors) of the first two draws of config4."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(3, 13, size=count)
    fac = rng.uniform(0.5, 2.0, size=count)
    return rng, ns, fac


def config4_system_sm(i, count=512, seed=3):
    """(n, sigma, shifted SM) of system i of config4, without the right-hand sides."""
    _, ns, fac = config4_draws(count, seed)
    n = int(ns[i])
    hs, sm, pos, mass = hex_system(n)
    sigma = float(fac[i] * lambda1(n))
    return n, sigma, shift_diagonal(sm, pos, mass, sigma), hs


def config4(count=512, seed=3, nrhs=16):
    rng, ns, fac = config4_draws(count, seed)
    systems = []
    for i in range(count):
        n = int(ns[i])
        hs, sm, pos, mass = hex_system(n)
        sigma = float(fac[i] * lambda1(n))
        b = np.asfortranarray(rng.uniform(-1.0, 1.0, size=(nrhs, hs.neq)).T)
        systems.append(dict(n=n, sigma=sigma, sm=shift_diagonal(sm, pos, mass, sigma), b=b, hs=hs))
    return systems
