"""GPU regrid (les_gpu_regrid, the device form of redim.f90 plus the
restart's deal) against the numpy restatement in oracle/redim.py, on states
produced by a few solver steps: refinement and coarsening in x, y and z, both
precisions; argument checks; the file-level redim (regrid_field) against the
handle-level call; and a regridded state that steps on."""
import numpy as np
import pytest

from oracle import redim as R

pytestmark = pytest.mark.gpu


def _src(product, nx, ny, nz, precision, steps=3):
    cfg = product.channel_config(nx, ny, nz, dt=1e-3, re_tau=180.0, precision=precision)
    g = product.LesGpu(cfg)
    g.make_ic(seed=7, amp=0.3, re_tau=180.0)
    dt = g.cfl_dt(0.5)
    for i in range(steps):
        g.step(it=i + 1, dt=dt)
    g.sync()
    return g


CASES = [
    (16, 16, 8, 32, 32, 12),   # refine x, y, z
    (32, 32, 12, 16, 16, 8),   # coarsen x, y, z
    (16, 32, 8, 64, 16, 8),    # refine x, coarsen y, same z
]


@pytest.mark.parametrize("prec,tol", [(0, 1e-12), (1, 2e-5)])
@pytest.mark.parametrize("case", CASES)
def test_regrid_matches_restatement(gpu_lib, product, case, prec, tol):
    nxi, nyi, nzi, nxo, nyo, nzo = case
    precision = product.PREC_FP64 if prec == 0 else product.PREC_MIXED
    src = _src(product, nxi, nyi, nzi, precision)
    f = src.download()
    ref = R.restart_state(R.redim_fields(f["u"], f["v"], f["w"], f["e"], f["p"], 2.0, nxo, nyo, nzo,
                                         nyquist=False))
    dst = product.LesGpu(product.channel_config(nxo, nyo, nzo, dt=1e-3, re_tau=180.0, precision=precision))
    dst.regrid_from(src)
    got = dst.download()
    for k in "uvwep":
        scale = max(np.abs(ref[k]).max(), 1e-30)
        assert np.abs(ref[k]).max() > 0, k
        np.testing.assert_allclose(got[k], ref[k], rtol=0, atol=tol * scale, err_msg=k)
    assert np.all(got["w"][-1] == 0)
    dst.close()
    src.close()


def test_refine_then_coarsen_returns_the_plane_modes(gpu_lib, product):
    src = _src(product, 16, 16, 8, product.PREC_FP64)
    a = src.download()
    fine = product.LesGpu(product.channel_config(64, 32, 8, re_tau=180.0))
    back = product.LesGpu(product.channel_config(16, 16, 8, re_tau=180.0))
    fine.regrid_from(src)
    back.regrid_from(fine)
    b = back.download()
    for k in "uvwp":
        np.testing.assert_allclose(b[k], a[k], rtol=0, atol=1e-12 * np.abs(a[k]).max(), err_msg=k)
    for h in (fine, back, src):
        h.close()


def test_regrid_rejects_mismatched_handles(gpu_lib, product):
    a = product.LesGpu(product.channel_config(16, 16, 8, re_tau=180.0))
    b = product.LesGpu(product.channel_config(32, 32, 8, re_tau=180.0, precision=product.PREC_MIXED))
    c = product.channel_config(32, 32, 8, re_tau=180.0)
    c.xl = 4.0
    d = product.LesGpu(c)
    for dst, src in ((b, a), (a, a), (d, a)):
        with pytest.raises(product.LesError) as ei:
            dst.regrid_from(src)
        assert ei.value.code == product.LES_EINVAL
    for h in (a, b, d):
        h.close()


def test_regrid_field_file_and_stepping(gpu_lib, product, tmp_path):
    src = _src(product, 16, 16, 8, product.PREC_FP64)
    pin, pout = str(tmp_path / "coarse.field"), str(tmp_path / "fine.field")
    src.write_field(pin, time=3.5)
    product.regrid_field(pin, pout, 32, 32, 16)
    dims, hdr = product.field_header(pout)
    assert dims == (32, 32, 16) and hdr["time"] == 3.5
    direct = product.LesGpu(product.channel_config(32, 32, 16, re_tau=180.0))
    direct.regrid_from(src)
    loaded = product.LesGpu(product.channel_config(32, 32, 16, re_tau=180.0))
    loaded.read_field(pout)
    a, b = direct.download(), loaded.download()
    for k in "uvwep":
        np.testing.assert_allclose(b[k], a[k], rtol=0, atol=1e-13 * max(np.abs(a[k]).max(), 1e-30), err_msg=k)
    # the regridded state steps on
    dt = direct.cfl_dt(0.5)
    for i in range(3):
        direct.step(it=i + 1, dt=dt)
    direct.sync()
    s = direct.download()
    assert all(np.isfinite(s[k]).all() for k in "uvwep")
    for h in (direct, loaded, src):
        h.close()
