"""GPU parity of the spectral operators (filter_fftw.f90, tridv.f90) against
the oracle, through the C ABI operator entry points."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12   # FP64: relative to max |reference|
TOL32 = 2e-5    # FP32 form


def _t(a, dtype):
    import torch
    return torch.tensor(a, dtype=dtype, device="cuda")


@pytest.mark.parametrize("n1,n2", [(16, 24), (64, 96), (96, 64), (192, 128), (768, 32), (576, 24)])
def test_xderiv_yderiv_match_oracle(gpu_lib, product, n1, n2):
    import torch
    rng = np.random.default_rng(n1 * 7 + n2)
    a = rng.standard_normal((3, n2, n1))
    xl, yl = 2 * np.pi, np.pi
    ref_x = np.stack([O.xderiv(p, xl) for p in a])
    ref_y = np.stack([O.yderiv(p, yl) for p in a])
    for dt, tol in ((torch.float64, TOL64), (torch.float32, TOL32)):
        gx = product.xderiv(_t(a, dt), xl).cpu().numpy()
        gy = product.yderiv(_t(a, dt), yl).cpu().numpy()
        assert np.abs(gx - ref_x).max() <= tol * np.abs(ref_x).max()
        assert np.abs(gy - ref_y).max() <= tol * np.abs(ref_y).max()


@pytest.mark.parametrize("nx,ny", [(16, 16), (64, 32), (128, 128), (512, 256)])
def test_expand_compress_deal_match_oracle(gpu_lib, product, nx, ny):
    import torch
    rng = np.random.default_rng(nx + ny)
    a = rng.standard_normal((2, ny, nx))
    b = rng.standard_normal((2, 3 * ny // 2, 3 * nx // 2))
    ref_e = np.stack([O.expand(p) for p in a])
    ref_c = np.stack([O.compress(p) for p in b])
    ref_d = np.stack([O.deal(p) for p in a])
    for dt, tol in ((torch.float64, TOL64), (torch.float32, TOL32)):
        ge = product.expand(_t(a, dt)).cpu().numpy()
        gc = product.compress(_t(b, dt)).cpu().numpy()
        gd = product.deal(_t(a, dt)).cpu().numpy()
        assert np.abs(ge - ref_e).max() <= tol * np.abs(ref_e).max()
        assert np.abs(gc - ref_c).max() <= tol * np.abs(ref_c).max()
        assert np.abs(gd - ref_d).max() <= tol * np.abs(ref_d).max()


def test_tridv_matches_oracle(gpu_lib, product):
    import torch
    rng = np.random.default_rng(4)
    ny, n = 37, 65
    bd = np.zeros((4, n, ny))
    bd[0] = 1.0; bd[2] = 1.0
    bd[1] = -2.0 - np.abs(rng.standard_normal((n, ny)))
    bd[3] = rng.standard_normal((n, ny))
    ref = O.tridv(bd)
    got = product.tridv(torch.tensor(bd, device="cuda")).cpu().numpy()
    np.testing.assert_allclose(got[3], ref[3], rtol=1e-13, atol=1e-13 * np.abs(ref[3]).max())
    np.testing.assert_allclose(got[1], ref[1], rtol=1e-14)


def test_fma_probe_rates(gpu_lib, product):
    """The compute roof of the transform kernels: the device's vector FMA
    rate from the library's own probe kernel, FP32 above FP64, both above
    1 TFLOP/s (a B200 delivers tens)."""
    f32 = product.fma_rate(4)
    f64 = product.fma_rate(8)
    assert f32 > 1e12 and f64 > 1e12
    assert f32 > f64
