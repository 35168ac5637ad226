"""CPU tests of the learned closure's FP64 perceptron (oracle/mlp_oracle.h):
the analytic gradient against central finite differences, Adam against a
numpy restatement of Kingma & Ba's update, and the bfloat16 rounding helper
against numpy's float32 bit manipulation."""
import numpy as np

from oracle import oracle as O


def _batch(n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, O.MLP_NIN)), rng.standard_normal((n, O.MLP_NOUT))


def test_mlp_gradient_matches_finite_differences():
    p = O.mlp_init(seed=1)
    x, t = _batch(64, 2)
    loss, g = O.mlp_loss_grad(p, x, t)
    assert abs(loss - O.mlp_loss(p, x, t)) < 1e-12 * loss
    rng = np.random.default_rng(3)
    # a sample of every parameter block, plus every bias of the output layer
    idx = set(rng.integers(0, O.MLP_NPARAM, 60).tolist())
    for (o, sh) in O.mlp_slices():
        idx.add(o)
        idx.add(o + int(np.prod(sh)) - 1)
    for i in sorted(idx):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (O.mlp_loss(pp, x, t) - O.mlp_loss(pm, x, t)) / (2 * h)
        assert abs(g[i] - fd) <= 1e-5 * max(abs(fd), 1e-3), (i, g[i], fd)


def test_mlp_gradient_is_batch_mean():
    p = O.mlp_init(seed=4)
    x, t = _batch(40, 5)
    _, g = O.mlp_loss_grad(p, x, t)
    _, g1 = O.mlp_loss_grad(p, x[:20], t[:20])
    _, g2 = O.mlp_loss_grad(p, x[20:], t[20:])
    np.testing.assert_allclose(g, 0.5 * (g1 + g2), rtol=1e-12, atol=1e-15)


def test_adam_matches_numpy_restatement():
    rng = np.random.default_rng(6)
    n = 100
    p = rng.standard_normal(n); m = np.zeros(n); v = np.zeros(n)
    pr, mr, vr = p.copy(), m.copy(), v.copy()
    for step in range(1, 6):
        g = rng.standard_normal(n)
        O.mlp_adam(p, m, v, g, 1e-3, step)
        mr = 0.9 * mr + 0.1 * g
        vr = 0.999 * vr + 0.001 * g * g
        pr = pr - 1e-3 * (mr / (1 - 0.9 ** step)) / (np.sqrt(vr / (1 - 0.999 ** step)) + 1e-8)
    np.testing.assert_allclose(p, pr, rtol=1e-13, atol=1e-15)


def test_bf16_round_is_nearest_even():
    rng = np.random.default_rng(7)
    a = np.concatenate([rng.standard_normal(2000) * 10.0 ** rng.integers(-20, 20, 2000),
                        [0.0, -0.0, 1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 65504.0]])
    f = a.astype(np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32).view(np.float32)
    np.testing.assert_array_equal(O.bf16_round(a), r.astype(np.float64))
    # ties go to even: 1 + 2^-8 sits halfway between 1 and 1 + 2^-7
    assert O.bf16_round(1.0 + 2.0 ** -8) == 1.0
    assert O.bf16_round(1.0 + 3 * 2.0 ** -8) == 1.0 + 2.0 ** -6


def test_mlp_bf16_emulation_is_close():
    p = O.mlp_init(seed=8)
    x, _ = _batch(256, 9)
    y = O.mlp_forward(p, x)
    yb = O.mlp_forward(p, x, bf16=True)
    err = np.abs(y - yb).max() / np.abs(y).max()
    assert 1e-4 < err < 3e-2
