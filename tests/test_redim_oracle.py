"""CPU tests of the numpy restatement of redim.f90 (oracle/redim.py): the z
walk against hand-derived tables, exactness on fields the scheme reproduces
(linear profiles in z, band-limited planes in x-y), the Nyquist bookkeeping,
the e clamp, and the equality of the reference form and the GPU form
(nyquist=False) when the grid is refined."""
import numpy as np
import pytest

from oracle import redim as R


def test_z_table_same_levels_is_identity():
    t = R.z_table(6, 6, 2.0)
    # level 1: extrapolated from (1, 2) with c = -1, i.e. level 1 itself
    assert t[0][:2] == (1, 2) and t[0][2] == pytest.approx(-1.0)
    for n in range(1, 6):
        a, b, c, f0, f1, d = t[n]
        assert (a, b) == (n, n + 1) and c == pytest.approx(0.0, abs=1e-14)
        assert f1 == n + 1 and d == pytest.approx(0.0, abs=1e-14)
    # first face: from (0, 1) = (wall, level 1) with d = 0
    assert t[0][3:5] == (0, 1) and t[0][5] == pytest.approx(0.0, abs=1e-14)


def test_z_table_doubling():
    t = R.z_table(4, 8, 2.0)  # dz 0.5 -> 0.25
    # new centre 0.125 from old centres 0.25 (1), 0.75 (2): c = (0.125 - 0.75)/0.5
    assert t[0][:3] == (1, 2, pytest.approx(-1.25))
    # new centre 1.875 lies above the last old centre 1.75: extrapolated from (3, 4)
    assert t[7][:3] == (3, 4, pytest.approx(0.25))
    # new face 0.25 lies between the wall (0) and old face 0.5 (level 1)
    assert t[0][3:6] == (0, 1, pytest.approx(-0.5))


def _grid(nx, ny, nz, zl=2.0, xl=2 * np.pi, yl=np.pi):
    x = np.arange(nx) * xl / nx
    y = np.arange(ny) * yl / ny
    zc = (np.arange(nz) + 0.5) * zl / nz
    zf = (np.arange(nz) + 1.0) * zl / nz
    return x, y, zc, zf


@pytest.mark.parametrize("nzi,nzo", [(8, 12), (12, 8), (8, 8), (6, 16)])
def test_linear_profiles_and_low_modes_are_reproduced(nzi, nzo):
    nxi, nyi, nxo, nyo = 16, 16, 32, 8
    x, y, zc, zf = _grid(nxi, nyi, nzi)
    X, Y = np.meshgrid(x, y, indexing="xy")
    mode = np.cos(2 * X) + 0.5 * np.sin(2 * np.pi * 2 * Y / np.pi + 0.3)  # |kx| = 2, |ky| = 2
    u = (1.0 + 0.3 * zc)[:, None, None] * (1 + 0.1 * mode)[None]
    v = (0.5 - 0.2 * zc)[:, None, None] * np.ones_like(mode)[None]
    w = (0.7 * zf)[:, None, None] * mode[None]
    e = 0.01 * np.ones((nzi, nyi, nxi)) + 0.001 * mode[None]
    p = (2.0 * zc)[:, None, None] * mode[None]
    out = R.redim_fields(u, v, w, e, p, 2.0, nxo, nyo, nzo)
    xo, yo, zco, zfo = _grid(nxo, nyo, nzo)
    Xo, Yo = np.meshgrid(xo, yo, indexing="xy")
    mo = np.cos(2 * Xo) + 0.5 * np.sin(2 * np.pi * 2 * Yo / np.pi + 0.3)
    np.testing.assert_allclose(out["u"], (1.0 + 0.3 * zco)[:, None, None] * (1 + 0.1 * mo)[None], atol=1e-12)
    np.testing.assert_allclose(out["v"], (0.5 - 0.2 * zco)[:, None, None] * np.ones_like(mo)[None], atol=1e-12)
    np.testing.assert_allclose(out["w"], (0.7 * zfo)[:, None, None] * mo[None], atol=1e-12)
    np.testing.assert_allclose(out["p"], (2.0 * zco)[:, None, None] * mo[None], atol=1e-12)
    np.testing.assert_allclose(out["e"], 0.01 + 0.001 * mo[None] * np.ones((nzo, 1, 1)), atol=1e-12)


def test_modes_above_the_coarse_grid_are_removed():
    nx, ny = 32, 32
    x, y, _, _ = _grid(nx, ny, 1)
    X, Y = np.meshgrid(x, y, indexing="xy")
    low = np.cos(3 * X)
    f = low + np.cos(12 * X) + np.sin(2 * np.pi * 10 * Y / np.pi)  # kx 12, ky 10 >= 16/2
    g = R.regrid_plane(f, 16, 16)
    xo, _, _, _ = _grid(16, 16, 1)
    np.testing.assert_allclose(g, np.cos(3 * xo)[None, :] * np.ones((16, 1)), atol=1e-13)


def test_coarse_nyquist_mode_kept_by_redim_and_removed_by_deal():
    # the +8 x-mode of a 32-grid lands on the 16-grid's Nyquist column:
    # redim keeps it, the restart's deal removes it
    x, y, _, _ = _grid(32, 32, 1)
    f = np.cos(8 * x)[None, :] * np.ones((32, 1))
    g = R.regrid_plane(f, 16, 16)
    assert np.abs(g).max() > 0.5
    assert np.abs(R.deal(g)).max() < 1e-13
    assert np.abs(R.regrid_plane(f, 16, 16, nyquist=False)).max() < 1e-13


def test_e_clamp():
    nz, ny, nx = 4, 8, 8
    rng = np.random.default_rng(3)
    e = 1e-3 * rng.standard_normal((nz, ny, nx))  # half negative
    z = np.zeros((nz, ny, nx))
    out = R.redim_fields(z, z, z, e, z, 2.0, 16, 16, nz)
    assert out["e"].min() >= 1e-10
    t = R.z_table(nz, nz, 2.0)
    for n, (_, _, _, f0, f1, d) in enumerate(t):
        e0 = e[0] if f0 == 0 else e[f0 - 1]
        assert out["e"][n].max() <= (e[f1 - 1] + (e[f1 - 1] - e0) * d).max() + 1e-15


@pytest.mark.parametrize("dims", [(16, 16, 8, 32, 32, 12), (16, 32, 6, 32, 64, 6)])
def test_reference_and_device_forms_agree_when_refining(dims):
    nxi, nyi, nzi, nxo, nyo, nzo = dims
    rng = np.random.default_rng(5)
    f = {k: R.deal(rng.standard_normal((nzi, nyi, nxi))) for k in "uvwp"}
    f["e"] = 1e-3 * (1.0 + 0.5 * R.deal(rng.standard_normal((nzi, nyi, nxi))))
    a = R.redim_fields(f["u"], f["v"], f["w"], f["e"], f["p"], 2.0, nxo, nyo, nzo, nyquist=True)
    b = R.redim_fields(f["u"], f["v"], f["w"], f["e"], f["p"], 2.0, nxo, nyo, nzo, nyquist=False)
    for k in "uvwep":
        np.testing.assert_allclose(a[k], b[k], atol=1e-14)
