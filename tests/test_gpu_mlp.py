"""GPU parity of the learned closure's tensor-core perceptron (les_mlp.h)
against the FP64 oracle (oracle/mlp_oracle.h): inference, the loss and its
gradient, the Adam update, and a short training run.

Tolerances: the product stores weights, inputs and hidden activations in
bfloat16 (8-bit significand) and evaluates GELU in bf16x2 arithmetic, so
outputs agree with the FP64 network to about 1% of their scale; a wrong
operand layout or accumulator mapping gives O(1) errors."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _inputs(n, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    x = O.bf16_round(rng.standard_normal((n, O.MLP_NIN)) * scale)
    t = rng.standard_normal((n, O.MLP_NOUT))
    return x, t


@pytest.fixture(scope="module")
def mlp(product, gpu_lib):
    m = product.Mlp(O.mlp_init(seed=11))
    yield m
    m.close()


@pytest.mark.parametrize("n", [1, 127, 128, 1000, 200003])
def test_forward_matches_oracle(product, mlp, n):
    p = O.mlp_init(seed=11)
    mlp.set_params(p)
    x, _ = _inputs(n, seed=n)
    y = mlp.forward(product.to_feat(x)).cpu().numpy()
    ref = O.mlp_forward(p, x, bf16=True)
    assert np.all(y[:, 6:] == 0)
    err = y[:, :6] - ref
    scale = np.sqrt(np.mean(ref ** 2))
    assert np.sqrt(np.mean(err ** 2)) <= 0.02 * scale, (np.sqrt(np.mean(err ** 2)), scale)
    assert np.abs(err).max() <= 0.1 * np.abs(ref).max() + 1e-3


def test_forward_uses_every_weight(product, mlp):
    """Perturbing one weight of each layer changes the outputs the way the
    oracle says (catches a transposed or misplaced tile)."""
    base = O.mlp_init(seed=12)
    x, _ = _inputs(512, seed=5)
    feat = product.to_feat(x)
    for (off, sh) in O.mlp_slices():
        p = base.copy()
        idx = off + (int(np.prod(sh)) // 3)
        p[idx] += 1.0
        mlp.set_params(p)
        d_gpu = mlp.forward(feat).cpu().numpy()[:, :6]
        mlp.set_params(base)
        d_gpu = d_gpu - mlp.forward(feat).cpu().numpy()[:, :6]
        d_ref = O.mlp_forward(p, x, bf16=True) - O.mlp_forward(base, x, bf16=True)
        num = np.sqrt(np.mean((d_gpu - d_ref) ** 2))
        den = np.sqrt(np.mean(d_ref ** 2))
        assert num <= 0.1 * den + 1e-3, (off, sh, num, den)


def test_loss_and_gradient_match_oracle(product, mlp):
    p = O.mlp_init(seed=13)
    mlp.set_params(p)
    n = 5000
    x, t = _inputs(n, seed=14)
    loss, g = mlp.loss_grad(product.to_feat(x), product.to_target(t))
    ref_loss, ref_g = O.mlp_loss_grad(p, x, t)
    assert abs(loss - ref_loss) <= 0.02 * ref_loss
    g = g.cpu().numpy().astype(np.float64)
    for (off, sh) in O.mlp_slices():
        k = int(np.prod(sh))
        a, b = g[off:off + k], ref_g[off:off + k]
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert rel <= 0.05, (off, sh, rel)


def test_gradient_is_deterministic(product, mlp):
    p = O.mlp_init(seed=15)
    mlp.set_params(p)
    x, t = _inputs(70000, seed=16)
    f, tt = product.to_feat(x), product.to_target(t)
    l1, g1 = mlp.loss_grad(f, tt)
    l2, g2 = mlp.loss_grad(f, tt)
    assert l1 == l2
    assert bool((g1 == g2).all())


def test_adam_step_matches_oracle_update(product, mlp):
    p = O.mlp_init(seed=17)
    mlp.set_params(p)
    x, t = _inputs(4096, seed=18)
    f, tt = product.to_feat(x), product.to_target(t)
    _, g = mlp.loss_grad(f, tt)
    g = g.cpu().numpy().astype(np.float64)
    mlp.adam_step(f, tt, lr=1e-3)
    p_gpu, _ = mlp.get_params()
    pr = p.astype(np.float32).astype(np.float64)
    m = np.zeros_like(pr); v = np.zeros_like(pr)
    O.mlp_adam(pr, m, v, g, 1e-3, 1)
    np.testing.assert_allclose(p_gpu, pr, rtol=0, atol=2e-6)


def test_training_reduces_loss(product, mlp):
    """Fit a teacher network: 300 Adam steps at batch 8192 cut the loss by
    more than 10x."""
    teacher = O.mlp_init(seed=19, scale=0.7)
    n = 8192 * 4
    x, _ = _inputs(n, seed=20)
    t = O.mlp_forward(teacher, x)
    f, tt = product.to_feat(x), product.to_target(t)
    mlp.set_params(O.mlp_init(seed=21))
    first = None
    for it in range(300):
        lo = (it % 4) * 8192
        l = mlp.adam_step(f[lo:lo + 8192], tt[lo:lo + 8192], lr=1e-3, want_loss=(it == 0 or it == 299))
        if it == 0:
            first = l
        last = l
    assert last < 0.1 * first, (first, last)


def test_mma_wait_limit_runs_out_and_context_stays_usable(product, gpu_lib):
    """The bounded tensor-core waits: with the limit set to 0 from the host,
    the training kernel gives up at its first unfinished MMA, drains it
    (fixed 1 s bound), frees its tensor memory and the host gets
    LES_ETIMEOUT; with the limit back at 1 s the same call on the same
    context reproduces the earlier result bit for bit."""
    m = product.Mlp(O.mlp_init(seed=23))
    x, t = _inputs(8192, seed=24)
    f, tt = product.to_feat(x), product.to_target(t)
    l_ref, g_ref = m.loss_grad(f, tt)
    m.set_wait_limit(0.0)
    with pytest.raises(product.LesError) as ei:
        m.loss_grad(f, tt)
    assert ei.value.code == product.LES_ETIMEOUT
    m.set_wait_limit(1.0)
    l2, g2 = m.loss_grad(f, tt)
    assert l2 == l_ref and bool((g2 == g_ref).all())
    with pytest.raises(product.LesError):
        m.set_wait_limit(-1.0)
    m.close()
