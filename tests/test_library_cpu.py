"""CPU checks of the product library: it loads, exports the declared ABI,
and its host-side plan is self-consistent (no GPU is touched)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import sam_lib_b200 as spr
from conftest import ref_system

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, 'include', 'spr_b200.h')).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(spr\w+_|spr_b200_\w+)\s*\(', text)))


@pytest.mark.parametrize('kind', [8, 4])
def test_library_exports_declared_abi(kind):
    lib = spr.load(kind)
    syms = declared_symbols()
    assert {'sprsol_', 'sprfc1_', 'sprfs1_', 'sprbs1_'} <= set(syms)
    for s in syms:
        assert hasattr(lib, s), s


@pytest.mark.parametrize('n', [3, 6, 12])
def test_plan_self_check(n):
    rs, _ = ref_system(n)
    out = np.zeros(13)
    rc = spr.load(8).spr_b200_plan_check(rs.mspar.ctypes.data_as(C.c_void_p),
                                         rs.mtrees.ctypes.data_as(C.c_void_p),
                                         rs.msifa.ctypes.data_as(C.c_void_p),
                                         out.ctypes.data_as(C.c_void_p))
    assert rc == 0 and out[0] == 0
    assert out[1] == rs.mspar[10]                 # NSUPER
    assert out[4] == 0, 'buffers outside the arena'
    assert out[5] == 0, 'live buffers overlap'
    assert abs(out[6] - rs.rinfo[2]) <= 1e-12 * rs.rinfo[2]   # RINFO(3)
    assert out[11] == 0 and out[12] == 0, 'Schur-update K ranges do not tile every column exactly once'


def test_plan_check_i4_abi():
    rs, _ = ref_system(6)
    out = np.zeros(13)
    m4 = [a.astype(np.int32) for a in (rs.mspar, rs.mtrees, rs.msifa)]
    rc = spr.load(4).spr_b200_plan_check(*[a.ctypes.data_as(C.c_void_p) for a in m4],
                                         out.ctypes.data_as(C.c_void_p))
    assert rc == 0 and out[4] == 0 and out[5] == 0
    assert abs(out[6] - rs.rinfo[2]) <= 1e-12 * rs.rinfo[2]


@pytest.mark.parametrize('n', [24, 48])
def test_plan_self_check_benchmark_structures(n):
    """The benchmark meshes' plans (reference structures from tests/golden):
    buffers inside the arena, no overlap of live buffers, and every column's
    Schur updates tile its earlier panels exactly once, in the FP64 launch
    lists and in the mixed mode's (side-stream and tensor-core) lists."""
    from sam_lib_b200.system import load_structure
    st = load_structure(n)
    out = np.zeros(13)
    rc = spr.load(8).spr_b200_plan_check(spr._ptr(st['mspar']), spr._ptr(st['mtrees']), spr._ptr(st['msifa']),
                                         spr._ptr(out))
    assert rc == 0 and out[0] == 0
    assert out[4] == 0 and out[5] == 0
    assert out[11] == 0 and out[12] == 0
    assert abs(out[6] - st['rinfo'][2]) <= 1e-12 * st['rinfo'][2]


@pytest.mark.parametrize('n', [6, 8])
def test_plan_self_check_partial_factorisation(n):
    """MSPAR(57) = 1 on a box with an external face: the retained root front
    (small at 6^3, dense at 8^3) gets no elimination or update launches, the
    arena stays consistent, and RINFO(3) excludes it as the reference does
    (src/SPR/sprtrs.f:1956)."""
    rs, _ = ref_system(n, retain=True)
    msp = rs.mspar.copy()
    msp[56] = 1
    out = np.zeros(13)
    rc = spr.load(8).spr_b200_plan_check(spr._ptr(msp), spr._ptr(rs.mtrees), spr._ptr(rs.msifa), spr._ptr(out))
    assert rc == 0 and out[0] == 0
    assert out[4] == 0 and out[5] == 0
    assert out[11] == 0 and out[12] == 0
    assert abs(out[6] - rs.rinfo[2]) <= 1e-12 * rs.rinfo[2]
