"""The allocation-free entry point against the regular one (GPU).

spr_b200_dense_ldlt_noalloc is for callers that must not allocate device
memory (their own allocator owns it, or an allocation would stall a
time-critical loop): it factors a dense front in place using only a fixed
file-scope scratch array.  Here it must reproduce what the regular device
entry point (spr_b200_factor_dev on the same front as a one-supernode SPR
structure) computes, on two calls in a row.  This file is collected last on
purpose, so a run that stops at the first failure has run everything else.
"""
import ctypes as C

import numpy as np
import pytest

import sam_lib_b200 as spr
from dense_structure import dense_chain, pack_dense

pytestmark = pytest.mark.gpu

RTOL = 1e-10          # same factor tolerance as the parity tests


def _lib():
    lib = spr.load(8)
    lib.spr_b200_dense_ldlt_noalloc.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_double,
                                                C.c_void_p, C.c_void_p, C.c_void_p]
    lib.spr_b200_dense_ldlt_noalloc.restype = C.c_int
    return lib


def _matrix(n, shift, seed):
    rng = np.random.default_rng(seed)
    Q = rng.standard_normal((n, n))
    A = Q @ Q.T / n + np.eye(n)
    return A - shift * np.eye(n)


def _regular(A):
    """Factor with the regular device entry point; returns (L lower with d, d, numneg)."""
    import torch
    n = A.shape[0]
    ms, mt, mf = dense_chain([n])
    sm = torch.from_numpy(pack_dense(A, ms, mt, mf)).cuda()
    ds = spr.DeviceSolver(ms, mt, mf)
    r = ds.factor(sm, 1e-12)
    smh = sm.cpu().numpy()
    ds.close()
    lnz = smh[n:]
    L = np.zeros((n, n))
    p = 0
    for j in range(n):
        L[j:, j] = lnz[p:p + n - j]
        p += n - j
    return L, smh[:n], r['numneg']


def _noalloc(lib, A, lda):
    import torch
    n = A.shape[0]
    buf = torch.zeros((n, lda), dtype=torch.float64, device='cuda')   # row j = column j (column-major)
    buf[:, :n] = torch.from_numpy(A.T.copy())
    d = torch.zeros(n, dtype=torch.float64, device='cuda')
    out = np.zeros(5)
    rc = lib.spr_b200_dense_ldlt_noalloc(buf.data_ptr(), n, lda, 1e-12, d.data_ptr(),
                                         torch.cuda.current_stream().cuda_stream,
                                         out.ctypes.data_as(C.c_void_p))
    torch.cuda.synchronize()
    L = np.tril(buf[:, :n].cpu().numpy().T)
    return rc, L, d.cpu().numpy(), out


@pytest.mark.parametrize('n,shift', [(1000, 0.0), (777, 2.5)])
def test_noalloc_matches_regular_entry_point_twice(n, shift):
    lib = _lib()
    A = _matrix(n, shift, seed=n)
    Lr, dr, negr = _regular(A)
    scale = np.max(np.abs(Lr))
    for call in range(2):
        rc, L, d, out = _noalloc(lib, A, lda=n + (4 - n % 4) % 4 + 4)
        assert rc == 0, (call, rc)
        assert np.max(np.abs(np.tril(L) - np.tril(Lr))) <= RTOL * scale, call
        assert np.max(np.abs(d - dr)) <= RTOL * np.max(np.abs(dr)), call
        assert int(out[0]) == negr, call
        assert out[1] == 0
    if shift > 0:
        assert negr > 0


def _numpy_ldlt(A):
    """Unpivoted L D L' of A (the SPRF17 recurrence, column by column); returns L, d."""
    W = np.array(A, dtype=np.float64)
    n = W.shape[0]
    d = np.zeros(n)
    for j in range(n):
        d[j] = W[j, j]
        if j + 1 < n:
            col = W[j + 1:, j] / d[j]
            W[j + 1:, j + 1:] -= np.outer(col, W[j + 1:, j])
            W[j + 1:, j] = col
    return np.tril(W, -1) + np.eye(n), d


_FRESH = r"""
import ctypes as C, json, sys
import numpy as np
import torch
sys.path.insert(0, %(root)r)
import sam_lib_b200 as spr
lib = spr.load(8)
f = lib.spr_b200_dense_ldlt_noalloc
f.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
f.restype = C.c_int
A = np.load(%(path)r)
n = A.shape[0]
lda = n + (4 - n %% 4) %% 4
res = []
for call in range(2):
    buf = torch.zeros((n, lda), dtype=torch.float64, device='cuda')
    buf[:, :n] = torch.from_numpy(A.T.copy())
    d = torch.zeros(n, dtype=torch.float64, device='cuda')
    out = np.zeros(5)
    rc = f(buf.data_ptr(), n, lda, 1e-12, d.data_ptr(), None, out.ctypes.data_as(C.c_void_p))
    torch.cuda.synchronize()
    np.save(%(path)r + '.L%%d.npy' %% call, np.tril(buf[:, :n].cpu().numpy().T))
    np.save(%(path)r + '.d%%d.npy' %% call, d.cpu().numpy())
    res.append([rc] + out.tolist())
print(json.dumps(res))
"""


def test_noalloc_first_call_in_a_fresh_process(tmp_path):
    """The allocation-free call must work as the very first call of this
    library in a process (no other entry point has set anything up), and
    agree with a numpy L D L'."""
    import json
    import os
    import subprocess
    import sys
    n = 700                                   # several 64-wide panels, a partial last one
    A = _matrix(n, 1.5, seed=11)
    path = str(tmp_path / 'a.npy')
    np.save(path, A)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, '-c', _FRESH % {'root': root, 'path': path}],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    Ln, dn = _numpy_ldlt(A)
    for call in range(2):
        rc, numneg, fail = res[call][0], res[call][1], res[call][2]
        assert rc == 0 and fail == 0, res[call]
        L = np.load(path + '.L%d.npy' % call)
        d = np.load(path + '.d%d.npy' % call)
        assert int(numneg) == int(np.sum(dn < 0)) > 0
        # numpy's column-by-column recurrence and the blocked GPU factor round
        # differently; the unpivoted indefinite LDL' grows (max |d| ~ 340 for
        # a_jj ~ 1), so they agree to about 1e-9 of the largest entry
        assert np.max(np.abs(d - dn)) <= 1e-8 * np.max(np.abs(dn)), call
        assert np.max(np.abs(np.tril(L, -1) - np.tril(Ln, -1))) <= 1e-8 * np.max(np.abs(Ln)), call


def test_noalloc_pivot_failure_column():
    """A matrix built as L diag(d) L' with d_k = 0 fails the pivot test at
    column k+1 (1-based), reported with the original a_jj, as SPRF17 does."""
    import torch
    lib = _lib()
    n, k = 300, 137
    rng = np.random.default_rng(5)
    L = np.tril(rng.uniform(-0.5, 0.5, (n, n)), -1) + np.eye(n)
    dd = rng.uniform(1.0, 2.0, n)
    dd[k] = 0.0
    A = (L * dd) @ L.T
    lda = n + (4 - n % 4) % 4
    for call in range(2):
        buf = torch.zeros((n, lda), dtype=torch.float64, device='cuda')
        buf[:, :n] = torch.from_numpy(A.T.copy())
        d = torch.zeros(n, dtype=torch.float64, device='cuda')
        out = np.zeros(5)
        rc = lib.spr_b200_dense_ldlt_noalloc(buf.data_ptr(), n, lda, 1e-12, d.data_ptr(), None,
                                             out.ctypes.data_as(C.c_void_p))
        torch.cuda.synchronize()
        assert rc == 0, call
        assert int(out[1]) == k + 1, (call, out)
        assert out[3] == A[k, k], (call, out)
        assert abs(out[2]) <= 1e-12 * abs(A[k, k]), (call, out)


def test_noalloc_rejects_sizes_and_layouts_without_running():
    lib = _lib()
    out = np.zeros(5)
    # larger than the fixed scratch allows: rejected before any GPU work
    assert lib.spr_b200_dense_ldlt_noalloc(None, 9000, 9000, 1e-12, None, None,
                                           out.ctypes.data_as(C.c_void_p)) == -3
    import torch
    a = torch.zeros(16 * 18, dtype=torch.float64, device='cuda')
    d = torch.zeros(16, dtype=torch.float64, device='cuda')
    # leading dimension not a multiple of 4
    assert lib.spr_b200_dense_ldlt_noalloc(a.data_ptr(), 16, 18, 1e-12, d.data_ptr(), None,
                                           out.ctypes.data_as(C.c_void_p)) == -2
