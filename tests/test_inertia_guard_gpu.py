"""Exact inertia under mixed precision (GPU).

A shift sigma within 1e-6 (relative) of an eigenvalue of (K, M) puts a pivot
of K - sigma M close to zero, where the TF32 rounding of the tensor-core
Schur updates (relative error ~1e-6) could flip its sign.  The mixed mode's
inertia guard counts pivots with |d| < 1e-3 |a_jj| and redoes such a
factorisation in FP64 (from a copy of the assembled SM), so NUMNEG equals
the reference's (the oracle, pinned bitwise to it) and the number of
eigenvalues below sigma, on both sides of the eigenvalue.  Away from the
eigenvalues the guard stays quiet and the mixed factor is kept.
"""
import functools

import numpy as np
import pytest

import sam_lib_b200 as spr
from conftest import ref_system, shifted_sm
from test_oracle import run_sprsol, rhs

pytestmark = pytest.mark.gpu


@functools.lru_cache(maxsize=None)
def _eigs(n, k):
    """The k lowest eigenvalues of K x = lambda M x (lumped mass), shift-invert."""
    import scipy.sparse as sp
    from scipy.sparse.linalg import eigsh
    from sam_lib_b200.system import sm_to_csr
    rs, sm = ref_system(n)
    K = sm_to_csr(rs.mspar, rs.mtrees, rs.msifa, sm)
    M = sm_to_csr(rs.mspar, rs.mtrees, rs.msifa, sm) - sm_to_csr(rs.mspar, rs.mtrees, rs.msifa,
                                                                   shifted_sm(rs, sm, 1.0))
    w = eigsh(K.tocsc(), k=k, M=M.tocsc(), sigma=0.0, which='LM', v0=np.ones(rs.neq), tol=1e-14,
              return_eigenvectors=False)
    return np.sort(w)


def _factor(ds, d_sm0, mode):
    d = d_sm0.clone()
    ds.set_mode(mode)
    r = ds.factor(d)
    inf = ds.info()
    ds.set_mode(0)
    return r, inf


@pytest.mark.parametrize('n', [12])
def test_mixed_inertia_near_an_eigenvalue_equals_the_oracle(n):
    import torch
    w = _eigs(n, 10)
    # a simple eigenvalue (the lowest two are a degenerate bending pair)
    gaps = np.minimum(np.diff(w)[:-1], np.diff(w)[1:]) / w[1:-1]
    k = 1 + int(np.argmax(gaps > 1e-3))
    lam = w[k]
    rs, sm = ref_system(n)
    ds = spr.DeviceSolver(rs.mspar, rs.mtrees, rs.msifa)
    for side, expect in ((+1, k + 1), (-1, k)):
        sigma = lam * (1.0 + side * 1e-6)
        ssm = shifted_sm(rs, sm, sigma)
        o = run_sprsol('orc', rs, ssm, rhs(rs.neq, 1, 4), iop=1)
        assert o['ierr'] == 3 and o['mspar'][25] == expect, (o['ierr'], o['mspar'][25], expect)
        d0 = torch.from_numpy(ssm).cuda()
        r64, _ = _factor(ds, d0, 0)
        assert r64['numneg'] == expect
        rmx, inf = _factor(ds, d0, 1)
        assert inf['near_pivots'] >= 1 and inf['fp64_redo'] == 1, inf
        assert rmx['numneg'] == expect and rmx['lierr'] == 0
    # away from the eigenvalues: no near-zero pivot, the mixed factor is kept
    sigma = 0.5 * (w[k] + w[k + 1])
    d0 = torch.from_numpy(shifted_sm(rs, sm, sigma)).cuda()
    r64, _ = _factor(ds, d0, 0)
    rmx, inf = _factor(ds, d0, 1)
    assert inf['fp64_redo'] == 0 and inf['near_pivots'] == 0, inf
    assert rmx['numneg'] == r64['numneg'] == k + 1
    ds.close()
