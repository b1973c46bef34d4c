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
    assert out[4] == 0, 'buffers outside the arena or index-map entries out of range'
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


def test_length_checks_match_reference_without_a_gpu():
    """MSPAR claiming a shorter MTREES or MSIFA than the structure needs, or
    LDB < NEQ, gives IERR = -2 and MSPAR(1) = -2 from every entry point, as
    from the reference (src/SPR/sprfc1.f:205-236, sprfs1.f:203-226,
    sprbs1.f:191-215, sprfc2.f, sprfs2.f, sprbs2.f, sprfc3.f:209-234); the
    checks come before any device work."""
    from oracle.refpipe import lib as reflib, _p, _i
    rs, sm = ref_system(3)
    R = reflib()
    b = np.asfortranarray(np.ones((rs.neq, 1)))
    iw = np.zeros(int(rs.mspar[13]) + int(rs.mspar[12]) + 8, dtype=np.int64)
    rw = np.zeros(int(rs.mspar[16]) + int(rs.mspar[13]) + 8)
    dcor = np.zeros(2 * rs.neq)
    # MSPAR(4) = NTREES one short; MSPAR(3) = NMSIFA one short of what the
    # factorisation uses (SPLIT + NBLOCK) or of what the solves use (LINDX + NOFSUB - 1)
    mlused_solve = int(rs.mspar[46] + rs.mspar[14] - 1)
    cases = [(3, lambda name: rs.mspar[3] - 1),
             (2, lambda name: rs.mspar[2] - 1 if name.startswith('sprfc') else mlused_solve - 1)]
    for slot, short in cases:
        for name in ('sprfc1', 'sprfc2', 'sprfc3', 'sprfs1', 'sprbs1', 'sprfs2', 'sprbs2'):
            msp = rs.mspar.copy()
            msp[slot] = short(name)
            mr, mg = msp.copy(), msp.copy()
            er, eg = C.c_int64(0), None
            tol = np.array([1e-12, 0.0, 0.0, 1.0])
            if name in ('sprfc1', 'sprfc2'):
                mv = R.cmvy18_ if name == 'sprfc2' else R.lmvy18_
                mm = R.cmmy18_ if name == 'sprfc2' else R.lmmy18_
                getattr(R, name + '_')(_p(mr), _p(rs.mtrees), _p(rs.msifa), _p(sm.copy()), _p(tol), _p(iw),
                                       _p(rw), _i(-1), C.byref(er), C.cast(mv, C.c_void_p),
                                       C.cast(mm, C.c_void_p))
                eg = getattr(spr, name)(mg, rs.mtrees, rs.msifa, sm.copy(), tol.copy())
            elif name == 'sprfc3':
                R.sprfc3_(_p(mr), _p(rs.mtrees), _p(rs.msifa), _p(sm.copy()), _p(tol), _p(iw), _p(rw),
                          _p(dcor), _i(-1), C.byref(er), C.cast(R.lmvy18_, C.c_void_p),
                          C.cast(R.lmmy18_, C.c_void_p))
                eg = spr.sprfc3(mg, rs.mtrees, rs.msifa, sm.copy(), tol.copy(), dcor.copy())
            elif name in ('sprfs1', 'sprfs2'):
                getattr(R, name + '_')(_p(mr), _p(rs.mtrees), _p(rs.msifa), _p(sm.copy()), _p(b.copy()),
                                       _i(rs.neq), _i(1), _p(iw), _p(rw), _i(-1), C.byref(er))
                eg = getattr(spr, name)(mg, rs.mtrees, rs.msifa, sm.copy(), b.copy(), rs.neq, 1)
            else:
                getattr(R, name + '_')(_p(mr), _p(rs.mtrees), _p(rs.msifa), _p(sm.copy()), _p(b.copy()),
                                       _i(rs.neq), _i(1), _p(rw), _i(-1), C.byref(er))
                eg = getattr(spr, name)(mg, rs.mtrees, rs.msifa, sm.copy(), b.copy(), rs.neq, 1)
            assert er.value == eg == -2, (name, slot, er.value, eg)
            assert mr[0] == mg[0] == -2, (name, slot)
    # LDB < NEQ without a partial factorisation
    for name in ('sprfs1', 'sprbs1', 'sprfs2', 'sprbs2'):
        mg = rs.mspar.copy()
        bs = np.asfortranarray(np.ones((rs.neq - 1, 1)))
        eg = getattr(spr, name)(mg, rs.mtrees, rs.msifa, sm.copy(), bs, rs.neq - 1, 1)
        assert eg == -2 and mg[0] == -2, name


@pytest.mark.parametrize('which', ['box12', 'gold24', 'gold48', 'retained8'])
def test_factor_stream_schedule_is_race_free(which):
    """Happens-before replay of the factorisation's three-stream schedule (the
    far trailing updates on a side stream, the in-super-panel columns after
    the next panel on a look-ahead stream, both forked and joined by events):
    no panel starts before its columns have all their earlier updates, no
    update reads a panel that is not final, no two unordered launches write a
    common element, in the FP64 and the tensor-core form.  Without either
    stream's joins the same check must fail wherever that stream has launches
    (a self-test of the check)."""
    from sam_lib_b200.system import load_structure
    if which == 'box12':
        rs, _ = ref_system(12)
        ms, mt, mf = rs.mspar, rs.mtrees, rs.msifa
    elif which == 'retained8':
        rs, _ = ref_system(8, retain=True)
        ms, mt, mf = rs.mspar.copy(), rs.mtrees, rs.msifa
        ms[56] = 1
    else:
        st = load_structure(int(which[4:]))
        ms, mt, mf = st['mspar'], st['mtrees'], st['msifa']
    out = np.zeros(6)
    rc = spr.load(8).spr_b200_schedule_check(spr._ptr(ms), spr._ptr(mt), spr._ptr(mf), spr._ptr(out))
    assert rc == 0
    assert out[0] == 0 and out[1] == 0, 'ordering violations in the factor schedule'
    if out[3] > 0:
        assert out[2] > 0, 'the check does not see the missing far joins'
    if out[5] > 0:
        assert out[4] > 0, 'the check does not see the missing look-ahead joins'
    if which.startswith('gold'):
        assert out[3] > 0 and out[5] > 0


@pytest.mark.parametrize('which', ['box6', 'box12', 'gold24', 'gold48', 'retained8'])
def test_solve_plan_is_consistent(which):
    """The solves' plan: every triangle block of every eliminated large front
    is one task of its level's dataflow launch, listed after the block above
    it (the forward sweep's dependency order; the back sweep takes the list
    in reverse), with its own ready flag; rectangle and forward-rows jobs
    match the fronts, and the partial-sum ranges of a level do not overlap.
    Two planted mistakes (blocks swapped, partial ranges made to overlap)
    must be reported (a self-test of the check)."""
    from sam_lib_b200.system import load_structure
    if which.startswith('box'):
        rs, _ = ref_system(int(which[3:]))
        ms, mt, mf = rs.mspar, rs.mtrees, rs.msifa
    elif which == 'retained8':
        rs, _ = ref_system(8, retain=True)
        ms, mt, mf = rs.mspar.copy(), rs.mtrees, rs.msifa
        ms[56] = 1
    else:
        st = load_structure(int(which[4:]))
        ms, mt, mf = st['mspar'], st['mtrees'], st['msifa']
    out = np.zeros(5)
    rc = spr.load(8).spr_b200_solve_plan_check(spr._ptr(ms), spr._ptr(mt), spr._ptr(mf), spr._ptr(out))
    assert rc == 0 and out[0] == 0
    assert out[1] == 0, 'solve plan violations'
    assert out[3] != 0 and out[4] != 0
    if which.startswith('gold'):
        assert out[2] > 0 and out[3] > 0 and out[4] > 0


def test_product_does_not_reach_the_oracle_or_the_tests():
    """The package imports neither the oracle nor the test tree, and none of
    its code (docstrings and comments aside) names their files: the checker
    is never part of the product path."""
    import ast
    pkg = os.path.join(ROOT, 'sam_lib_b200')
    pat = re.compile(r'\boracle\b|refpipe|liboracle|libsprref|\btests?/|conftest')
    hits = []
    for d, _, files in os.walk(pkg):
        if '_build' in d or '__pycache__' in d:
            continue
        for f in files:
            path = os.path.join(d, f)
            rel = os.path.relpath(path, ROOT)
            if f.endswith('.py'):
                tree = ast.parse(open(path, encoding='utf-8').read())
                docs = set()
                for node in ast.walk(tree):
                    if isinstance(node, (ast.Module, ast.FunctionDef, ast.ClassDef, ast.AsyncFunctionDef)):
                        if node.body and isinstance(node.body[0], ast.Expr) and \
                                isinstance(node.body[0].value, ast.Constant):
                            docs.add(id(node.body[0].value))
                for node in ast.walk(tree):
                    if isinstance(node, ast.Import):
                        names = [a.name for a in node.names]
                    elif isinstance(node, ast.ImportFrom):
                        names = [node.module or '']
                    elif isinstance(node, ast.Constant) and isinstance(node.value, str) and id(node) not in docs:
                        names = [node.value]
                    else:
                        continue
                    for nm in names:
                        if pat.search(nm) or nm.split('.')[0] in ('oracle', 'tests', 'conftest'):
                            hits.append('%s:%d: %s' % (rel, node.lineno, nm[:80]))
            elif f.endswith(('.cu', '.cpp', '.h', '.cuh')):
                text = re.sub(r'/\*.*?\*/', '', open(path, encoding='utf-8').read(), flags=re.S)
                for k, line in enumerate(text.splitlines(), 1):
                    if pat.search(line.split('//')[0]):
                        hits.append('%s: %s' % (rel, line.strip()))
    assert not hits, '\n'.join(hits)
