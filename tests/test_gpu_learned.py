"""GPU parity of the RK3 stage with the learned closure (imodel = 5) against
the oracle's learned stage, through the C ABI.

The network runs in bfloat16 on the tensor cores and the oracle emulates
the bf16 rounding of inputs, weights and activations, so the two networks'
stresses agree to about 1%; the learned part of a stage's change is
dtab1 times the stress divergence, and the tolerance below is 5% of that on
top of the FP64 (or mixed-form) tolerance of the Deardorff stage.  A stage
whose network is anti-dissipative must reproduce the Deardorff stage
bit for bit."""
import numpy as np
import pytest

from oracle import oracle as O
from test_gpu_stage import make_pair, relerr

pytestmark = pytest.mark.gpu
RE_TAU = 180.0


def params():
    """A seeded network with the dimensionless closure's normalisation:
    inputs g/|G| in [-1, 1], min(z_w/Delta, 16), z_w/h in [0, 1]; outputs
    c of order 0.02 (tau = (Delta |G|)^2 c)."""
    P = O.mlp_init(seed=31).astype(np.float32).astype(np.float64)
    N = np.concatenate([np.zeros(11), np.full(9, 3.0), [0.2, 2.0], np.full(6, 0.02), np.zeros(6)])
    return P, N


def learned_pair(product, sign, precision=8, nx=32, ny=32, nz=16, guard=0.0):
    """Oracle and GPU handle with the seeded network; guard = the factor of
    the fallback test against the Deardorff dissipation (0: the sign test
    only, so that the seeded network's stresses are exercised)."""
    o, g, f = make_pair(product, nx, ny, nz, precision=precision, imodel=5, re_tau=RE_TAU)
    P, N = params()
    N[22:28] *= sign
    o.set_mlp(P, N, RE_TAU)
    m = product.Mlp(P, N)
    g.set_mlp(m, RE_TAU)
    o.set_learned_guard(guard)
    g.set_learned_guard(guard)
    return o, g, m, f


_SIGNS = {}


def dissipative_sign(product, n=32, nz=16):
    """Output sign that makes the seeded network dissipative on the seeded
    field of this size (the oracle's own test, computed once per size)."""
    if (n, nz) not in _SIGNS:
        o, g, m, f = learned_pair(product, 1.0, nx=n, ny=n, nz=nz)
        o.stage(0, 0, 1)
        used, _ = o.learned_status()
        _SIGNS[(n, nz)] = 1.0 if used else -1.0
    return _SIGNS[(n, nz)]


# 32x32x16, and the bench width 512 (nz = 4 keeps the oracle to seconds):
# the gradient, network and divergence kernels at the shapes the bench runs
@pytest.mark.parametrize("n,nz", [(32, 16), (512, 4)])
@pytest.mark.parametrize("precision", [8, 4])
def test_learned_stage_matches_oracle(gpu_lib, product, precision, n, nz):
    sign = dissipative_sign(product, n, nz)
    o, g, m, f = learned_pair(product, sign, precision=precision, nx=n, ny=n, nz=nz)
    o.stage(0, 1, 1)
    g.stage(0, True, 1)
    used_o, dis_o = o.learned_status()
    used_g, dis_g = g.learned_status()
    assert used_o == 1 and used_g == 1
    assert abs(dis_g - dis_o) <= 0.05 * abs(dis_o)
    lru, lrv, lrw = o.learned_divergence()
    lscale = max(np.abs(lru).max(), np.abs(lrv).max(), np.abs(lrw).max())
    dtab1 = o.cfg.dt * 8.0 / 15.0
    fo, fg = o.get_fields(), g.download()
    to_, tg = o.get_tendencies(), g.download_tendencies()
    vscale = np.abs(fo["u"]).max()
    rscale = max(np.abs(to_[k]).max() for k in ("ru", "rv", "rw"))
    base_f, base_t = (1e-11, 1e-9) if precision == 8 else (2e-5, 2e-4)
    for k in "uvw":
        err = np.abs(fg[k] - fo[k]).max()
        assert err <= 0.05 * dtab1 * lscale + base_f * vscale, (k, err, dtab1 * lscale, vscale)
    for k in ("ru", "rv", "rw"):
        err = np.abs(tg[k] - to_[k]).max()
        assert err <= 0.05 * lscale + base_t * rscale, (k, err, lscale, rscale)
    assert relerr(fg["e"], fo["e"]) <= (1e-10 if precision == 8 else 1e-4)


def test_anti_dissipative_network_reproduces_deardorff(gpu_lib, product):
    sign = -dissipative_sign(product)
    o, g, m, f = learned_pair(product, sign)
    g.stage(0, True, 1)
    used, dis = g.learned_status()
    assert used == 0 and dis >= 0  # rejected on the raw sign; the applied stress is projected
    _, d, _ = make_pair(product, 32, 32, 16, imodel=3, re_tau=RE_TAU)
    d.stage(0, True, 1)
    a, b = g.download(), d.download()
    for k in "uvwep":
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("guard", [1.5, 4.0, 1e6])
def test_dissipation_guard_matches_oracle(gpu_lib, product, guard):
    """The second fallback test: the reference (Smagorinsky) mean
    dissipation and the decision agree with the oracle's; a rejected network
    reproduces the Deardorff stage bit for bit."""
    sign = dissipative_sign(product)
    o, g, m, f = learned_pair(product, sign, guard=guard)
    o.stage(0, 1, 1)
    g.stage(0, True, 1)
    used_o, dis_o = o.learned_status()
    used_g, dis_g = g.learned_status()
    dd_o, dd_g = o.learned_reference(), g.learned_reference()
    assert dd_o > 0 and abs(dd_g - dd_o) <= 0.02 * dd_o
    ratio = max(dis_o / dd_o, dd_o / dis_o)
    if abs(ratio / guard - 1.0) > 0.1:  # decisions near the threshold may differ by rounding
        assert used_g == used_o == (1 if ratio <= guard else 0)
    if used_g == 0:
        _, d, _ = make_pair(product, 32, 32, 16, imodel=3, re_tau=RE_TAU)
        d.stage(0, True, 1)
        a, b = g.download(), d.download()
        for k in "uvwep":
            assert np.array_equal(a[k], b[k]), k


def test_guard_is_on_by_default(gpu_lib, product):
    o, g, f = make_pair(product, 16, 16, 8, imodel=5, re_tau=RE_TAU)
    P, N = params()
    m = product.Mlp(P, N)
    g.set_mlp(m, RE_TAU)
    o.set_mlp(P, N, RE_TAU)
    o.stage(0, 1, 1)
    g.stage(0, True, 1)
    used_o, _ = o.learned_status()
    assert g.learned_status()[0] == used_o  # both apply the default factor 4
    with pytest.raises(product.LesError):
        g.set_learned_guard(float("nan"))


def test_learned_graph_step_matches_stages(gpu_lib, product):
    sign = dissipative_sign(product)
    _, g1, m1, _ = learned_pair(product, sign)
    _, g2, m2, _ = learned_pair(product, sign)
    for it in range(2):
        g1.step(it=it, mnout=False)
        for s in (1, 2, 3):
            g2.stage(it, False, s)
    assert g1.learned_status()[0] == 1
    a, b = g1.download(), g2.download()
    for k in "uvwe":
        assert np.array_equal(a[k], b[k]), k


def test_set_mlp_rejects_other_closures(gpu_lib, product):
    _, g, _ = make_pair(product, 16, 16, 8, imodel=3)
    P, N = params()
    m = product.Mlp(P, N)
    with pytest.raises(product.LesError) as ei:
        g.set_mlp(m, RE_TAU)
    assert ei.value.code == product.LES_EINVAL


@pytest.mark.parametrize("with_model", [False, True])
def test_learn_filter_matches_numpy(gpu_lib, product, with_model):
    from oracle import learned as LN
    o, g, f = make_pair(product, 64, 64, 16, imodel=3)
    c = o.cfg
    e = 1e-3 * (1.0 + 0.5 * LN.Spec(64, 64, c.xl, c.yl).deal(np.random.default_rng(5).uniform(-1, 1, f["u"].shape)))
    g.upload(f["u"], f["v"], f["w"], e, f["p"])
    out = g.learn_filter(4, 2, with_model=with_model).cpu().numpy()
    tm = LN.model_stress(f["u"], f["v"], f["w"], e, c.xl, c.yl, c.zl, c.emin) if with_model else None
    ref = LN.filter_fields(f["u"], f["v"], f["w"], c.xl, c.yl, 4, 2, tau_model=tm)
    assert out.shape == ref.shape == (9, 8, 16, 16)
    us = np.abs(f["u"]).max()
    # the fine run's model stress comes from the f32 feature kernel
    ms = np.abs(tm).max() if with_model else 0.0
    for i in range(9):
        tol = 1e-12 * (us if i < 3 else us * us) + (2e-6 * ms if i >= 3 else 0.0)
        err = np.abs(out[i] - ref[i]).max()
        assert err <= tol, (i, err, tol)
    assert np.abs(ref[3]).max() > 1e-6  # the stresses are not trivially zero


def test_learned_features_match_numpy(gpu_lib, product):
    from oracle import learned as LN
    o, g, f = make_pair(product, 32, 32, 16, imodel=3)
    feat = g.learned_features().cpu().numpy()
    ref, sc = LN.features(f["u"], f["v"], f["w"], o.cfg.xl, o.cfg.yl, o.cfg.zl)
    assert np.all(feat[:, 12:] == 0)
    for j in range(11):
        scale = np.abs(ref[:, j]).max()
        err = np.abs(feat[:, j] - ref[:, j]).max()
        assert err <= 1e-6 * scale + 1e-30, (j, err, scale)  # f32 output
    assert np.abs(feat[:, 11] - sc).max() <= 1e-6 * sc.max()
    assert np.abs(np.sqrt((ref[:, :9] ** 2).sum(1)) - 1.0).max() < 1e-12  # unit-norm gradient inputs


def test_mma_wait_limit_in_the_learned_stage(gpu_lib, product):
    """A tensor-core wait that runs out inside the solver's learned stage is
    reported by les_gpu_sync as LES_ETIMEOUT (the handle's error word is
    sticky); a new handle on the same context with the limit restored
    reproduces the stage of a handle that never timed out."""
    sign = dissipative_sign(product)
    o, g, m, f = learned_pair(product, sign)
    m.set_wait_limit(0.0)
    g.stage(0, True, 1)
    with pytest.raises(product.LesError) as ei:
        g.sync()
    assert ei.value.code == product.LES_ETIMEOUT
    g.close()
    m.set_wait_limit(1.0)
    _, g2, m2, _ = learned_pair(product, sign)
    g2.stage(0, True, 1)
    g2.sync()
    g3 = product.LesGpu(g2.cfg)
    g3.upload(f["u"], f["v"], f["w"], f["e"], f["p"])
    g3.set_mlp(m, RE_TAU)
    g3.set_learned_guard(0.0)
    g3.stage(0, True, 1)
    g3.sync()
    a, b = g2.download(), g3.download()
    for k in "uvwe":
        assert np.array_equal(a[k], b[k]), k
