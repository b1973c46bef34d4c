"""The translated reference SPRLAN (oracle build) on its own, CPU: the
eigenvalues of (K, M) closest to the shift agree with scipy's shift-invert
Lanczos, and MOP(4) is the number of eigenvalues below the shift (the Sturm
count of the shifted LDL' factorisation, MSPAR(26)).  This pins the
translation that test_lanczos_gpu.py then runs with the GPU library
interposed."""
import numpy as np

from conftest import ref_system, shifted_sm
from lanczos_case import run


def test_translated_sprlan_finds_the_eigenvalues_near_the_shift():
    import scipy.sparse as sp
    from scipy.sparse.linalg import eigsh
    from sam_lib_b200.system import sm_to_csr
    n, shift = 5, 0.05
    res = run(n, shift)
    assert res['ierr'] >= 0, res
    rs, sm = ref_system(n)
    K = sm_to_csr(rs.mspar, rs.mtrees, rs.msifa, sm)
    M = K - sm_to_csr(rs.mspar, rs.mtrees, rs.msifa, shifted_sm(rs, sm, 1.0))
    w = np.sort(eigsh(K.tocsc(), k=20, M=M.tocsc(), sigma=shift, which='LM', return_eigenvectors=False))
    got = np.array(res['evl'][:6])
    assert res['mop'][0] >= 6, res['mop']                        # accepted eigenvalues
    for x in got:
        assert np.min(np.abs(w - x)) <= 1e-8 * abs(x), (x, w)
    below = int(np.sum(np.linalg.eigvalsh(np.linalg.solve(np.diag(np.sqrt(M.diagonal())),
                                                          np.linalg.solve(np.diag(np.sqrt(M.diagonal())),
                                                                          K.toarray()).T)) < shift))
    assert res['mop'][3] == below == res['numneg'], (res['mop'], below)
