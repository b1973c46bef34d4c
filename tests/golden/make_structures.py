"""Generates the reference SPR structures of the benchmark meshes.

Runs the reference host pipeline (SPRPRP -> SPRSAS -> SPRRNM -> SPRTRS ->
SPRSMB -> SPRPMP, from the oracle build oracle/_ref/libsprref.so, i.e. the
reference's own minimum-degree ordering, supernode partition and symbolic
factorisation) on n^3 hex8 boxes with the face x=0 clamped, and stores its
outputs -- MSPAR, MTREES, MSIFA, MEQN, RINFO -- as compressed package data
(the benchmark and the tests read them as a Fortran host's structure arrays):

    sam_lib_b200/structures/hex<n>.npz

The GPU product consumes these exactly as it would consume the arrays a
Fortran host passes after calling those reference routines.

    python tests/golden/make_structures.py 3 4 ... 12 32 48
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.refpipe import RefSystem          # noqa: E402
from sam_lib_b200.fe import HexBox             # noqa: E402


def delta(a):
    return np.diff(a.astype(np.int64), prepend=0).astype(np.int32)


def make(n):
    rs = RefSystem(HexBox(n))
    sp = rs.mspar
    out = os.path.join(ROOT, 'sam_lib_b200', 'structures', 'hex%d.npz' % n)
    np.savez_compressed(out, n=n, mspar=sp, rinfo=rs.rinfo,
                        mtrees_d=delta(rs.mtrees[:sp[3]]), msifa_d=delta(rs.msifa[:sp[2]]),
                        meqn_d=delta(rs.meqn))
    print('%s  NEQ=%d NSUPER=%d NZEROL=%d  %.1f kB' % (out, sp[7], sp[10], sp[15], os.path.getsize(out) / 1e3))


if __name__ == '__main__':
    for a in sys.argv[1:] or ['3', '4', '5', '6', '7', '8', '9', '10', '11', '12', '32', '48']:
        make(int(a))
