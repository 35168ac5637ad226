"""CPU tests of the oracle restatement against analytic known answers and the
independent numpy restatement (oracle/mini.py).  The reference ships no
tests or golden vectors, so these are what pin the oracle."""
import numpy as np
import pytest

from oracle import mini
from oracle import oracle as O


@pytest.mark.parametrize("n", [8, 12, 16, 24, 48, 64, 96, 144, 192, 384, 768])
def test_dft_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    np.testing.assert_allclose(O.dft(x, -1), np.fft.fft(x), rtol=0, atol=1e-12 * np.abs(x).sum())
    np.testing.assert_allclose(O.dft(x, +1), np.fft.ifft(x) * n, rtol=0, atol=1e-12 * np.abs(x).sum())


def trig_plane(nx, ny, xl, yl, kxmax, kymax, seed=0):
    """Band-limited random trigonometric polynomial and its exact x, y derivatives."""
    rng = np.random.default_rng(seed)
    x = np.arange(nx) * xl / nx
    y = np.arange(ny) * yl / ny
    X, Y = np.meshgrid(x, y)
    f = np.zeros((ny, nx)); fx = np.zeros_like(f); fy = np.zeros_like(f)
    for kx in range(0, kxmax + 1):
        for ky in range(-kymax, kymax + 1):
            a, b = rng.standard_normal(2)
            ph = 2 * np.pi * (kx * X / xl + ky * Y / yl)
            f += a * np.cos(ph) + b * np.sin(ph)
            d = -a * np.sin(ph) + b * np.cos(ph)
            fx += d * 2 * np.pi * kx / xl
            fy += d * 2 * np.pi * ky / yl
    return f, fx, fy


@pytest.mark.parametrize("nx,ny", [(16, 16), (24, 32), (96, 96), (64, 128)])
def test_xderiv_yderiv_exact_on_trig_polynomials(nx, ny):
    xl, yl = 2 * np.pi, np.pi
    f, fx, fy = trig_plane(nx, ny, xl, yl, nx // 2 - 1, ny // 2 - 1, seed=nx + ny)
    np.testing.assert_allclose(O.xderiv(f, xl), fx, atol=1e-10 * np.abs(fx).max())
    np.testing.assert_allclose(O.yderiv(f, yl), fy, atol=1e-10 * np.abs(fy).max())
    np.testing.assert_allclose(mini.xderiv(f, xl), fx, atol=1e-10 * np.abs(fx).max())


def test_xderiv_zeroes_dc_and_nyquist():
    nx, ny = 16, 8
    x = np.arange(nx)
    f = np.tile(3.0 + np.cos(np.pi * x), (ny, 1))  # DC + Nyquist only
    assert np.abs(O.xderiv(f, 2 * np.pi)).max() < 1e-13


@pytest.mark.parametrize("nx,ny", [(16, 16), (32, 24), (64, 64)])
def test_expand_compress_roundtrip_and_interpolation(nx, ny):
    xl, yl = 2 * np.pi, np.pi
    f, _, _ = trig_plane(nx, ny, xl, yl, nx // 2 - 1, ny // 2 - 1, seed=3)
    big = O.expand(f)
    # the padded plane is the same trigonometric polynomial sampled on the 3/2 grid
    fb, _, _ = trig_plane(3 * nx // 2, 3 * ny // 2, xl, yl, nx // 2 - 1, ny // 2 - 1, seed=3)
    np.testing.assert_allclose(big, fb, atol=1e-11 * np.abs(fb).max())
    np.testing.assert_allclose(O.compress(big), f, atol=1e-11 * np.abs(f).max())
    np.testing.assert_allclose(mini.expand(f), big, atol=1e-12 * np.abs(big).max())
    np.testing.assert_allclose(mini.compress(big), O.compress(big), atol=1e-12 * np.abs(f).max())


def test_deal_removes_nyquist_only():
    nx, ny = 16, 12
    rng = np.random.default_rng(1)
    f = rng.standard_normal((ny, nx))
    g = O.deal(f)
    z = np.fft.rfft2(g)
    assert np.abs(z[:, nx // 2]).max() < 1e-12
    assert np.abs(z[ny // 2, :]).max() < 1e-12
    zf = np.fft.rfft2(f)
    keep = np.ones_like(zf, dtype=bool); keep[:, nx // 2] = False; keep[ny // 2, :] = False
    np.testing.assert_allclose(z[keep], zf[keep], atol=1e-11)
    np.testing.assert_allclose(O.deal(g), g, atol=1e-13)


def test_tridv_matches_dense_solve():
    rng = np.random.default_rng(2)
    ny, n = 5, 9
    bd = np.zeros((4, n, ny))
    bd[0] = rng.standard_normal((n, ny))
    bd[2] = rng.standard_normal((n, ny))
    bd[1] = 4.0 + np.abs(rng.standard_normal((n, ny)))
    bd[3] = rng.standard_normal((n, ny))
    out = O.tridv(bd)
    for j in range(ny):
        A = np.diag(bd[1][:, j]) + np.diag(bd[0][1:, j], -1) + np.diag(bd[2][:-1, j], 1)
        np.testing.assert_allclose(out[3][:, j], np.linalg.solve(A, bd[3][:, j]), rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(out[1][:, 0][j] if False else out[1][0, j], 1.0 / bd[1][0, j])


def _divergence(f, cfg):
    """Discrete divergence used by the projection: spectral dx, dy on the
    small grid plus the staggered dz of w (w(0)=w(nnz)=0)."""
    u, v, w = f["u"], f["v"], f["w"]
    nz = cfg.nnz
    ww = w.copy(); ww[nz - 1] = 0.0
    wm = np.concatenate([np.zeros_like(ww[:1]), ww[:-1]])
    return mini.xderiv(u, cfg.xl) + mini.yderiv(v, cfg.yl) + (ww - wm) / (cfg.zl / nz)


@pytest.mark.parametrize("nx,ny,nz", [(16, 16, 8), (32, 24, 16)])
def test_initial_condition_is_projected(nx, ny, nz):
    cfg = O.make_config(nx, ny, nz, dt=1e-3)
    o = O.Oracle(cfg)
    o.make_ic(seed=12345, amp=0.1)
    f = o.get_fields()
    div = _divergence(f, cfg)
    scale = np.abs(mini.xderiv(f["u"], cfg.xl)).max() + np.abs(f["v"]).max()
    assert np.abs(div).max() < 1e-11 * max(scale, 1.0)
    assert np.abs(f["w"].mean(axis=(1, 2))).max() < 1e-14
    assert np.all(f["e"] >= cfg.emin)
    # perturbation statistics: amplitude 0.1*utau, zero-mean, Nyquist-free
    z = np.fft.rfft2(f["v"])
    assert np.abs(z[:, :, nx // 2]).max() < 1e-10


CASES = [
    dict(nx=16, ny=16, nz=8, imodel=3, isurface=6, prod=0),
    dict(nx=16, ny=16, nz=8, imodel=4, isurface=1, prod=1),
    dict(nx=24, ny=16, nz=12, imodel=3, isurface=1, prod=1),
    # the other wall models of lowerbc.f90:126-161 / upperbc.f90:124-158
    dict(nx=16, ny=16, nz=8, imodel=3, isurface=2, prod=0),
    dict(nx=16, ny=16, nz=8, imodel=3, isurface=3, prod=0),
    dict(nx=16, ny=16, nz=8, imodel=3, isurface=4, prod=1),
    dict(nx=16, ny=16, nz=8, imodel=4, isurface=5, prod=0),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "{nx}x{ny}x{nz}-m{imodel}-s{isurface}-p{prod}".format(**c))
def test_oracle_matches_level_form(case):
    """The ring-buffer restatement and the level-parallel numpy restatement
    agree after two full RK3 steps."""
    cfg = O.make_config(case["nx"], case["ny"], case["nz"], dt=2e-3, imodel=case["imodel"],
                        isurface=case["isurface"], tke_production=case["prod"])
    o = O.Oracle(cfg)
    o.make_ic(seed=7, amp=0.3)
    f = o.get_fields()
    m = mini.MiniLes(cfg)
    m.u, m.v, m.w, m.e = [f[k].copy() for k in "uvwe"]
    for it in range(2):
        for s in (1, 2, 3):
            o.stage(it, 1, s)
            m.stage(1, s)
    g = o.get_fields()
    t = o.get_tendencies()
    for k in "uvwe":
        ref = np.abs(g[k]).max()
        assert np.abs(g[k] - getattr(m, k)).max() <= 1e-12 * ref, k
    for k in ("ru", "rv", "rw", "re"):
        ref = max(np.abs(t[k]).max(), 1e-30)
        assert np.abs(t[k] - getattr(m, k)).max() <= 1e-10 * ref, k
    assert np.abs(g["p"] - m.p).max() <= 1e-10 * np.abs(g["p"]).max()
    mb, sc = o.stats()
    np.testing.assert_allclose(sc[:4], [m.utau, m.utau_s, m.dudt, m.dvdt], rtol=1e-10, atol=1e-14)
    for r in (17, 18):  # uwsb, vwsb include the wall stresses: O(utau^2)
        np.testing.assert_allclose(mb[r], m.meanbuf[r], rtol=1e-9, atol=1e-15)


def test_fp32_oracle_tracks_fp64():
    """The shipped single-precision form stays within an FP32 envelope of the
    FP64 form over a few steps (error envelope for the mixed form)."""
    cfg = O.make_config(16, 16, 8, dt=2e-3)
    o64 = O.Oracle(cfg, 8)
    o64.make_ic(seed=3)
    f = o64.get_fields()
    o32 = O.Oracle(cfg, 4)
    o32.set_fields(**f)
    o64.step(0, 3, 1)
    o32.step(0, 3, 1)
    a, b = o64.get_fields(), o32.get_fields()
    scale = np.abs(a["u"]).max()  # velocity scale
    for k in "uvw":
        err = np.abs(a[k] - b[k]).max() / scale
        assert err < 1e-5, (k, err)


def test_rk3_mean_constraints():
    """w and rw plane means vanish after every step (comp2.f90:30,39)."""
    cfg = O.make_config(16, 16, 8, dt=2e-3)
    o = O.Oracle(cfg)
    o.make_ic(seed=5)
    o.step(0, 2, 1)
    f, t = o.get_fields(), o.get_tendencies()
    assert np.abs(f["w"].mean(axis=(1, 2))).max() < 1e-15
    assert np.abs(t["rw"].mean(axis=(1, 2))).max() < 1e-14
    assert np.abs(f["w"][-1]).max() < 1e-15 and np.abs(t["rw"][-1]).max() == 0.0


def test_spectra_variance_identity():
    """sum of the 1D x-spectrum equals the plane variance (the identity the
    reference checks in its commented-out lines, spectra2.f90:149-154)."""
    cfg = O.make_config(16, 16, 8, dt=2e-3)
    o = O.Oracle(cfg)
    o.make_ic(seed=9)
    f = o.get_fields()
    zx, z2 = o.spectra(1, 3)  # v at level 3
    plane = f["v"][2]
    assert abs(zx.sum() - (plane ** 2).mean()) < 1e-12 * (plane ** 2).mean()
