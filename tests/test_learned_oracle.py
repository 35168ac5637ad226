"""CPU tests of the oracle's learned closure (les_oracle.cpp learned_prepare)
against the independent numpy restatement in oracle/learned.py (gradients
by numpy.fft, the network in numpy with the same bfloat16 rounding, the
dissipation test, the dealiased stress divergence), a stage whose network
is anti-dissipative falling back to the Deardorff stresses exactly, and
known answers of the training-data filter."""
import numpy as np
import pytest

from oracle import learned as LN
from oracle import oracle as O

NX, NY, NZ = 16, 16, 8
RE_TAU = 180.0


def make_case(sign):
    cfg = O.make_config(NX, NY, NZ, re_tau=RE_TAU, imodel=5)
    o = O.Oracle(cfg)
    o.make_ic(seed=3, amp=0.3, re_tau=RE_TAU)
    o.dt_used = o.cfl_dt(0.5)
    o.set_dt(o.dt_used)
    cfg.dt = o.dt_used
    fl = o.get_fields()
    P = O.mlp_init(seed=31)
    N = np.concatenate([np.zeros(11), np.full(9, 3.0), [0.2, 2.0], np.full(6, sign * 0.02), np.zeros(6)])
    return cfg, o, fl, P, N


def np_learned(cfg, fl, P, N):
    u, v, w = fl["u"], fl["v"], fl["w"]
    f, sc = LN.features(u, v, w, cfg.xl, cfg.yl, cfg.zl)
    y = LN.mlp(P, (f - N[:11]) * N[11:22])
    raw = ((y * N[22:28] + N[28:34]) * (sc ** 2)[:, None]).T.reshape(6, NZ, NY, NX)
    g = LN.gradients(u, v, w, cfg.xl, cfg.yl, cfg.zl)
    tau = LN.project_backscatter(g, raw)
    dz = cfg.zl / NZ
    xkmax = dz * dz / cfg.dt / 5.0
    nut = LN.network_viscosity(g, tau, xkmax)
    dsl = (cfg.xl / NX * cfg.yl / NY * dz) ** (1.0 / 3.0)
    dis_r = LN.reference_dissipation(g, dsl)
    return (LN.dissipation(g, raw), LN.dissipation(g, tau), dis_r,
            LN.divergence(tau, cfg.xl, cfg.yl, cfg.zl, u, v, nut))


@pytest.mark.parametrize("guard", [0.0, 4.0, 1e6])
@pytest.mark.parametrize("sign", [1.0, -1.0])
def test_learned_prepare_matches_numpy(sign, guard):
    cfg, o, fl, P, N = make_case(sign)
    o.set_mlp(P, N, RE_TAU)
    o.set_learned_guard(guard)
    o.stage(0, 0, 1)
    used, dis = o.learned_status()
    raw_np, dis_np, dis_r_np, (lru, lrv, lrw) = np_learned(cfg, fl, P, N)
    assert abs(dis - dis_np) <= 1e-9 * abs(dis_np)
    assert abs(o.learned_raw() - raw_np) <= 1e-9 * abs(raw_np)
    assert abs(o.learned_reference() - dis_r_np) <= 1e-9 * abs(dis_r_np) and dis_r_np > 0
    assert dis_np >= max(raw_np, 0.0) - 1e-12 * abs(raw_np)  # the projection only removes backscatter
    assert used == LN.network_used(raw_np, dis_np, dis_r_np, guard)
    if used:
        a, b, c = o.learned_divergence()
        for x, y in ((a, lru), (b, lrv), (c, lrw)):
            assert np.abs(y).max() > 0
            np.testing.assert_allclose(x, y, rtol=0, atol=1e-10 * np.abs(y).max())


def test_anti_dissipative_network_falls_back_to_deardorff():
    for sign in (1.0, -1.0):
        cfg, o, fields, P, N = make_case(sign)
        o.set_mlp(P, N, RE_TAU)
        o.set_learned_guard(0.0)
        o.stage(0, 0, 1)
        used, dis = o.learned_status()
        if used:
            continue
        assert o.learned_raw() < 0 and dis >= 0  # the applied (projected) stress never injects energy
        cfg3 = O.make_config(NX, NY, NZ, re_tau=RE_TAU, imodel=3)
        d = O.Oracle(cfg3)
        d.set_fields(**fields)
        d.set_dt(o.dt_used)
        d.stage(0, 0, 1)
        a, b = o.get_fields(), d.get_fields()
        for k in "uvwe":
            np.testing.assert_array_equal(a[k], b[k])
        return
    pytest.fail("neither sign gave an anti-dissipative network")


def _grid(nx, ny, nz, xl, yl, zl):
    x = np.arange(nx) * xl / nx
    y = np.arange(ny) * yl / ny
    zc = (np.arange(nz) + 0.5) * zl / nz
    return np.meshgrid(zc, y, x, indexing="ij")


def test_filter_transfer_of_single_modes():
    nx, ny, nz, xl, yl, zl = 32, 32, 8, 2 * np.pi, np.pi, 2.0
    Z, Y, X = _grid(nx, ny, nz, xl, yl, zl)
    kx, ky = 3, 2
    u = np.cos(kx * X) * np.ones_like(Z)
    v = np.sin(2 * np.pi * ky * Y / yl) * (1 + Z)
    w = np.zeros_like(u)
    out = LN.filter_fields(u, v, w, xl, yl, 4, 2)
    Zc, Yc, Xc = _grid(nx // 4, ny // 4, nz // 2, xl, yl, zl)
    gx = LN.box_transfer(np.array([kx * 2 * np.pi / xl]), xl / (nx // 4))[0]
    gy = LN.box_transfer(np.array([ky * 2 * np.pi / yl]), yl / (ny // 4))[0]
    np.testing.assert_allclose(out[0], gx * np.cos(kx * Xc), atol=1e-13)
    # z: the pair average of a linear profile is its value at the coarse centre
    np.testing.assert_allclose(out[1], gy * np.sin(2 * np.pi * ky * Yc / yl) * (1 + Zc), atol=1e-13)
    # no w: the w stresses vanish
    for i in (2, 5, 7, 8):
        assert np.abs(out[i]).max() < 1e-14


def test_filter_constants_and_z_box():
    nx, ny, nz, xl, yl, zl = 32, 32, 8, 2 * np.pi, np.pi, 2.0
    rng = np.random.default_rng(1)
    c = rng.standard_normal(3)
    u = np.full((nz, ny, nx), c[0]); v = np.full_like(u, c[1])
    w = np.full_like(u, c[2]); w[-1] = 0
    out = LN.filter_fields(u, v, w, xl, yl, 4, 1)
    np.testing.assert_allclose(out[0], c[0], atol=1e-14)
    for i in (3, 4, 6):
        assert np.abs(out[i]).max() < 1e-13
    # a field that varies only in z sees only the z box (a positive kernel):
    # tau11 is the variance of each pair of fine levels
    uz = rng.standard_normal(nz)
    u = np.broadcast_to(uz[:, None, None], (nz, ny, nx)).copy()
    out = LN.filter_fields(u, v, w, xl, yl, 4, 2)
    np.testing.assert_allclose(out[3][:, 0, 0], 0.25 * (uz[0::2] - uz[1::2]) ** 2, rtol=1e-12)


@pytest.mark.parametrize("fz", [2, 4])
def test_filter_z_box_of_w_is_exact_for_linear_profiles(fz):
    """w at the coarse faces: the trapezoid box of fz fine cells centred on
    the face reproduces a w that is linear in z (away from the top wall,
    where w(nz) = 0 breaks the line)."""
    nx, ny, nz, xl, yl, zl = 16, 16, 16, 2 * np.pi, np.pi, 2.0
    k = np.arange(1, nz + 1, dtype=np.float64)
    w = np.broadcast_to((0.3 + 0.05 * k)[:, None, None], (nz, ny, nx)).copy()
    w[-1] = 0.0
    u = np.zeros_like(w)
    out = LN.filter_fields(u, u, w, xl, yl, 4, fz)
    nzc = nz // fz
    for K in range(1, nzc):
        if fz * K + fz // 2 <= nz - 1:
            np.testing.assert_allclose(out[2][K - 1], 0.3 + 0.05 * fz * K, rtol=1e-13)
