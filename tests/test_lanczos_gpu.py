"""SPRLAN end to end with the GPU library interposed (GPU).

The translated reference's SPRLAN (shift-invert Lanczos, src/SPR/sprlan.f)
runs twice in child processes on the same problem: once on its own (all
CPU), once with libspr_b200.so preloaded (LD_PRELOAD), as a Fortran host
linked against the GPU library would run it: its SPRFC1 factorisation of
K - SHIFT M (sprlan.f:703) and the SPRFS1/SPRBS1 solves of every Lanczos step
(SPRSMM) then run on the device, while SPRSHA, the Lanczos recurrence and the
tridiagonal eigensolver stay in the reference.  The eigenvalues must agree to
1e-9 relative, and the Sturm count MOP(4) = MSPAR(26) exactly; the GPU
library must have served the calls (it holds a device context afterwards).
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
    assert np.max(np.abs(a - b) / np.abs(a)) <= 1e-9, (a, b)
