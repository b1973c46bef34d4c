"""Shared fixtures: SPR systems prepared by the reference host pipeline.

The reference pipeline (SPRPRP -> ... -> SPRADM) runs from the oracle build
(oracle/_ref/libsprref.so, the machine-translated reference); the GPU product
is then compared against the oracle restatement and the reference on the same
inputs.
"""
import functools
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200)')


def _have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _have_gpu():
        return
    skip = pytest.mark.skip(reason='no CUDA device')
    for it in items:
        if 'gpu' in it.keywords:
            it.add_marker(skip)


@functools.lru_cache(maxsize=None)
def ref_system(n, emod='uniform', seed=2, clamp=True, retain=False):
    """(RefSystem, assembled SM) for an n^3 hex box, cached per process.

    clamp=False leaves the box free: K is singular with the six rigid-body
    modes in its null space.  retain=True makes the face x=n external (MSC=2):
    its equations are numbered last and form the retained supernodes of a
    partial factorisation (MSPAR(57) = 1)."""
    from oracle.refpipe import RefSystem
    from sam_lib_b200.fe import HexBox, hex8_stiffness, element_moduli
    box = HexBox(n, clamp_face=clamp, retain_face=retain)
    rs = RefSystem(box)
    ke = hex8_stiffness()
    E = element_moduli(box.nel, emod, seed=seed)
    sm = rs.assemble(lambda e: ke * E[e])
    sm.setflags(write=False)
    return rs, sm


def shifted_sm(rs, sm, sigma):
    """SM of K - sigma*M with the lumped mass on the diagonal (SPRSHA KSB=2, sprsha.f:86-93)."""
    out = sm.copy()
    mass = rs.box.lumped_mass()
    meqn = rs.meqn
    neq = rs.neq
    m_int = np.zeros(neq)
    sel = meqn > 0
    m_int[meqn[sel] - 1] = mass[sel]
    mt, ms, sp = rs.mtrees, rs.msifa, rs.mspar
    nsuper = int(sp[10])
    xsuper = mt[sp[44] - 1: sp[44] + nsuper]
    xlindx = mt[sp[45] - 1: sp[45] + nsuper]
    xlnz = ms[sp[47] - 1: sp[47] + nsuper]
    for js in range(nsuper):
        f = xlindx[js + 1] - xlindx[js]
        p = xlnz[js] - 1
        for j in range(xsuper[js], xsuper[js + 1]):
            out[neq + p] -= sigma * m_int[j - 1]
            p += f
            f -= 1
    return out


def dense_from_sm(rs, sm):
    """Dense symmetric matrix from the assembled LNZ pattern (small systems only)."""
    mt, ms, sp = rs.mtrees, rs.msifa, rs.mspar
    nsuper = int(sp[10])
    neq = rs.neq
    xsuper = mt[sp[44] - 1: sp[44] + nsuper]
    xlindx = mt[sp[45] - 1: sp[45] + nsuper]
    lindx = ms[sp[46] - 1:]
    xlnz = ms[sp[47] - 1: sp[47] + nsuper]
    K = np.zeros((neq, neq))
    lnz = sm[neq:]
    for js in range(nsuper):
        rows = lindx[xlindx[js] - 1: xlindx[js + 1] - 1]
        p = xlnz[js] - 1
        for jc, col in enumerate(range(xsuper[js], xsuper[js + 1])):
            r = rows[jc:]
            K[r - 1, col - 1] = lnz[p:p + len(r)]
            p += len(r)
    return np.tril(K) + np.tril(K, -1).T
