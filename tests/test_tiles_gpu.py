"""The tile autotuner's two shapes of the small FP64 Schur updates (GPU).

Updates with fewer than 256 rows run in 64 x 64 or, as the autotuner may
choose, 32 x 32 lower-triangle tiles.  Every entry sums its K products in the
same order either way, so the factors must agree bit for bit; the autotuner
must return one of the two shapes with both timings.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _factor(ds, d_sm0, tile):
    import torch
    ds.set_small_tile(tile)
    d = d_sm0.clone()
    r = ds.factor(d)
    torch.cuda.synchronize()
    return r, d.cpu().numpy()


@pytest.mark.parametrize('which', ['box12', 'forest'])
def test_small_update_tiles_agree_bitwise(which):
    import torch
    import sam_lib_b200 as spr
    from conftest import ref_system, shifted_sm
    if which == 'box12':
        rs, sm = ref_system(12)
        sm = shifted_sm(rs, sm, 1.0e-3)
        ds = spr.DeviceSolver(rs.mspar, rs.mtrees, rs.msifa)
        d_sm0 = torch.from_numpy(sm.copy()).cuda()
    else:
        from sam_lib_b200.batch import BatchSolver
        from sam_lib_b200.workloads import config4
        bs = BatchSolver(config4()[:40])
        ds, d_sm0 = bs.ds, bs.sm0
    r64, s64 = _factor(ds, d_sm0, 64)
    r32, s32 = _factor(ds, d_sm0, 32)
    assert r64['lierr'] == r32['lierr'] == 0 and r64['numneg'] == r32['numneg']
    assert np.array_equal(s64, s32)
    t = ds.autotune_tiles(d_sm0)
    assert t['small_tile'] in (32, 64) and t['factor_ms_64'] > 0 and t['factor_ms_32'] > 0
    ds.close()
