"""Product host pieces against the reference (CPU): the committed reference
structures and the library's SPRADM assembly."""
import numpy as np
import pytest

from conftest import ref_system
from sam_lib_b200.system import HexSystem, load_structure
from sam_lib_b200.fe import element_moduli


@pytest.mark.parametrize('n', [3, 6, 12])
def test_committed_structure_equals_reference_pipeline(n):
    rs, _ = ref_system(n)
    st = load_structure(n)
    sp = rs.mspar
    assert np.array_equal(st['mspar'], sp)
    assert np.array_equal(st['mtrees'], rs.mtrees[:sp[3]])
    assert np.array_equal(st['msifa'], rs.msifa[:sp[2]])
    assert np.array_equal(st['meqn'], rs.meqn)
    assert np.array_equal(st['rinfo'], rs.rinfo)


@pytest.mark.parametrize('n,emod', [(3, 'uniform'), (6, 'loguniform'), (12, 'loguniform')])
def test_assembly_bitwise_equals_spradm(n, emod):
    rs, sm_ref = ref_system(n, emod)
    hs = HexSystem(n, moduli=element_moduli(n ** 3, emod, seed=2))
    sm = hs.assemble()
    assert np.array_equal(sm, sm_ref)


def test_matvec_matches_dense():
    from conftest import dense_from_sm
    rs, sm = ref_system(3, 'loguniform')
    hs = HexSystem(3, moduli=element_moduli(27, 'loguniform', seed=2))
    x = np.random.default_rng(0).standard_normal(hs.neq)
    K = dense_from_sm(rs, sm)
    assert np.allclose(hs.matvec(x), K @ x, rtol=1e-12, atol=1e-12)


def test_forest_merge_matches_individual_systems_bitwise():
    """Independent systems merged into one SPR forest: the oracle factors the
    forest exactly as it factors each system (solutions bitwise equal)."""
    from sam_lib_b200.workloads import config4
    from sam_lib_b200.batch import Forest
    from test_batched_gpu import oracle_solve
    systems = config4()[:6]
    fo = Forest([(s['hs'].mspar, s['hs'].mtrees, s['hs'].msifa) for s in systems])
    sm = fo.merge_sm([s['sm'] for s in systems])
    B = np.zeros((fo.neq, 16), order='F')
    for i, s in enumerate(systems):
        B[fo.eq_off[i]:fo.eq_off[i] + fo.neq_i[i]] = s['b']

    class H:
        mspar, mtrees, msifa, neq = fo.mspar, fo.mtrees, fo.msifa, fo.neq
    ierr, nn, X = oracle_solve(H, sm, B)
    assert ierr == 0
    tot = 0
    for i, s in enumerate(systems):
        e, n1, x = oracle_solve(s['hs'], s['sm'], s['b'])
        tot += n1
        assert np.array_equal(x, X[fo.eq_off[i]:fo.eq_off[i] + fo.neq_i[i]])
    assert nn == tot
