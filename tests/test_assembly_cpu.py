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
