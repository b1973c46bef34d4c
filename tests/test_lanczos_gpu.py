"""SPRLAN end to end with the GPU library interposed (GPU).

The translated reference's SPRLAN (shift-invert Lanczos, src/SPR/sprlan.f)
runs twice in child processes on the same problem: once on its own (all
CPU), once with libspr_b200.so preloaded (LD_PRELOAD), as a Fortran host
linked against the GPU library would run it: its SPRFC1 factorisation of
K - SHIFT M (sprlan.f:703) and the SPRFS1/SPRBS1 solves of every Lanczos step
(SPRSMM) then run on the device, while SPRSHA, the Lanczos recurrence and the
tridiagonal eigensolver stay in the reference.  The Sturm count MOP(4) =
MSPAR(26) must be equal, and the GPU library must have served the calls (it
holds a device context afterwards).  Every eigenvalue either run reports must
be an eigenvalue of K x = lambda M x to 1e-9 relative (scipy's shift-invert
eigsh on the same matrices), and the two runs must find the same distinct
eigenvalues nearest the shift.  Copies of a multiple eigenvalue are not
compared one by one: the box's y-z symmetry gives double eigenvalues, and
single-vector Lanczos finds a second copy only through rounding, which the
two factorisations do differently.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(ROOT, 'sam_lib_b200', 'libspr_b200.so')

_SCRIPT = r"""
import ctypes, json, sys
sys.path.insert(0, %(here)r)
from lanczos_case import run
res = run(%(n)d, %(shift)r)
if %(pre)r:
    res['contexts'] = ctypes.CDLL(%(lib)r).spr_b200_contexts()
print(json.dumps(res))
"""


def _child(n, shift, preload):
    env = dict(os.environ)
    if preload:
        env['LD_PRELOAD'] = LIB
    code = _SCRIPT % {'here': HERE, 'n': n, 'shift': shift, 'pre': preload, 'lib': LIB}
    r = subprocess.run([sys.executable, '-c', code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.mark.parametrize('n,shift', [(8, 0.02), (12, 0.008)])
def test_sprlan_with_the_gpu_library_interposed(n, shift):
    cpu = _child(n, shift, False)
    gpu = _child(n, shift, True)
    assert cpu['ierr'] == gpu['ierr'] == 0
    assert gpu['contexts'] >= 1                         # the calls reached the device
    assert gpu['mop'][3] == cpu['mop'][3] == cpu['numneg'] > 0     # Sturm count
    k = min(cpu['mop'][0], gpu['mop'][0])
    assert k >= 6
    a, b = np.array(cpu['evl'][:k]), np.array(gpu['evl'][:k])
    exact = _exact_spectrum(n, shift)
    for run in (a, b):
        near = np.min(np.abs(run[:, None] - exact[None, :]) / np.abs(run[:, None]), axis=1)
        assert near.max() <= 1e-9, (run, exact)
        for lam in run:                    # no more copies than the exact multiplicity
            assert np.sum(np.isclose(run, lam, rtol=1e-9, atol=0)) <= \
                np.sum(np.isclose(exact, lam, rtol=1e-7, atol=0)), (run, exact)
    da, db = _distinct(a, shift), _distinct(b, shift)
    m = min(len(da), len(db)) - 1          # the farthest one found may differ
    assert m >= 3
    assert np.allclose(da[:m], db[:m], rtol=1e-9, atol=0), (da, db)


def _distinct(v, shift):
    """Distinct values of v (1e-9 relative), ordered by distance from the shift."""
    out = []
    for x in sorted(v, key=lambda x: abs(x - shift)):
        if not any(abs(x - y) <= 1e-9 * abs(y) for y in out):
            out.append(x)
    return np.array(out)


def _exact_spectrum(n, shift, k=16):
    """The k eigenvalues of K x = lambda M x nearest the shift (scipy, CPU)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla
    sys.path.insert(0, HERE)
    from conftest import ref_system
    from sam_lib_b200.system import sm_to_csr
    rs, sm = ref_system(n)
    K = sm_to_csr(rs.mspar, rs.mtrees, rs.msifa, sm)
    mass = np.zeros(rs.neq)
    sel = rs.meqn > 0
    mass[rs.meqn[sel] - 1] = rs.box.lumped_mass()[sel]
    w = sla.eigsh(K.tocsc(), k=k, M=sp.diags(mass).tocsc(), sigma=shift, which='LM',
                  return_eigenvectors=False, tol=1e-14)
    return np.sort(w)
