"""Detector::Calc_kMap on the GPU against the oracle (bit for bit)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ny,nx,gap", [(128, 128, 0.0), (512, 1024, 2e-3), (7, 5, 0.0)])
def test_kmap_bit_exact(ctx, oracle_lib, ny, nx, gap):
    import torch
    from incohautocorrelate_b200 import workloads as W
    pm = W.flat_pixel_map(ny, nx, gap_x=gap, gap_after=nx // 2 if gap else None)
    rng = np.random.default_rng(ny * nx)
    pm = (pm * (1 + 0.01 * rng.standard_normal(pm.shape))).astype(np.float32)  # tilted, uneven
    want, mq_want = oracle_lib.calc_kmap(pm)
    d_pm = torch.from_numpy(pm).cuda()
    d_km = torch.empty_like(d_pm)
    mq = ctx.calc_kmap(d_pm, pm.size // 3, d_km)
    np.testing.assert_array_equal(d_km.cpu().numpy(), want)
    assert mq == [np.float32(v) for v in mq_want]
