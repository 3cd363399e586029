"""The closure network's GPU kernels through the C ABI against the FP64
oracle (oracle/mlp_oracle.py).  The kernels compute in bfloat16 with FP32
accumulation, so the bars are those of bfloat16: the forward pass agrees
with the oracle that rounds weights and activations the same way to 1e-3
relative L2 and with the plain FP64 oracle to 2e-2; the gradient of the
trained parameters agrees with the FP64 gradient to 3e-2 relative L2 (and
per layer to 5e-2); Adam training lowers the loss."""
import numpy as np
import pytest

from diablo_b200 import mlp as ML
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def data(seed, n):
    rng = np.random.default_rng(seed)
    m = max(n, 4096)          # normalisation from at least 4096 samples
    x = rng.normal(size=(m, 11)) * rng.uniform(0.5, 3.0, 11) + rng.normal(size=11)
    mean, scale = x.mean(axis=0), x.std(axis=0)
    # a smooth target of the inputs, as a closure's stresses are
    z = (x - mean) / scale
    t = np.stack([np.tanh(z[:, 0] * z[:, 1]), np.sin(z[:, 2]) + 0.3 * z[:, 3], z[:, 4] ** 2 - 1,
                  z[:, 5] * z[:, 6], np.exp(-z[:, 7] ** 2), 0.5 * z[:, 8] - z[:, 9] * z[:, 10]], axis=1) * 1e-3
    osc = t.std(axis=0)
    return x[:n], t[:n], ML.init_params(seed, mean, scale, osc)


@pytest.mark.parametrize("n", [1, 15, 16, 1000, 70001])
def test_forward_matches_oracle(n):
    x, _, p = data(5, n)
    with ML.SgsMlp(p) as m:
        y = m.forward(x)
        p32 = m.params().astype(np.float64)
    assert np.array_equal(p32, p.astype(np.float64))
    assert relerr(y, M.forward(p32, x, emulate_bf16=True)) < 1e-3
    assert relerr(y, M.forward(p32, x)) < 2e-2


def test_gradient_matches_oracle():
    x, t, p = data(6, 4000)
    with ML.SgsMlp(p) as m:
        loss, g = m.gradient(x, t)
        loss2, g2 = m.gradient(x, t)           # the state is not changed by a gradient call
    lo, go = M.loss_grad(p.astype(np.float64), x, t)
    assert abs(loss - lo) <= 2e-2 * lo
    assert relerr(g, go) < 3e-2
    o = 0
    for name, shape in M.SHAPES:
        k = int(np.prod(shape))
        assert relerr(g[o:o + k], go[o:o + k]) < 5e-2, name
        o += k
    assert abs(loss2 - loss) <= 1e-6 * loss and relerr(g2, g) < 1e-5


def test_gradient_with_dissipation_term_matches_oracle():
    """The loss with the subgrid-dissipation term and its gradient against
    the FP64 oracle, at the bars of the plain gradient.  The weight is 5 over
    the variance of the targets' dissipation, as closure.train_and_evaluate
    sets it."""
    from diablo_b200.closure import dissipation

    x, t, p = data(6, 4000)
    w = 5.0 / float(np.var(dissipation(x, t)))
    with ML.SgsMlp(p) as m:
        m.set_dissipation_weight(w)
        loss, g = m.gradient(x, t)
    lo, go = M.loss_grad(p.astype(np.float64), x, t, diss_weight=w)
    lo0, go0 = M.loss_grad(p.astype(np.float64), x, t)
    assert relerr(go, go0) > 0.05                  # the term changes the gradient
    assert abs(loss - lo) <= 2e-2 * lo
    assert relerr(g, go) < 3e-2


def test_training_lowers_loss():
    x, t, p = data(7, 20000)
    rng = np.random.default_rng(8)
    perm = rng.permutation(x.shape[0])
    x, t = x[perm], t[perm]
    with ML.SgsMlp(p) as m:
        before, _ = m.gradient(x, t)
        losses = m.train(x, t, batch=512, steps=600, lr=2e-3)
        after, _ = m.gradient(x, t)
        q = m.params()
    assert np.isfinite(losses).all()
    assert after < 0.2 * before, (before, after)
    assert np.array_equal(q[M.NTRAIN:], p[M.NTRAIN:])      # normalisation is not trained


def test_training_is_reproducible():
    """Two trainings from the same seed and data on fresh networks.  The
    gradient sums use FP32 atomics, whose order varies from run to run, so
    the two loss curves agree statistically rather than bit for bit: the
    means of the last 100 mini-batch losses within 5% and the final
    full-data losses within 5%."""
    x, t, p = data(9, 20000)
    runs = []
    for _ in range(2):
        with ML.SgsMlp(p) as m:
            losses = m.train(x, t, batch=512, steps=600, lr=2e-3)
            after, _ = m.gradient(x, t)
        runs.append((losses, after))
    (l0, a0), (l1, a1) = runs
    assert np.isfinite(l0).all() and np.isfinite(l1).all()
    assert abs(l0[0] - l1[0]) <= 1e-5 * l0[0]        # the first mini-batch sees identical weights
    m0, m1 = l0[-100:].mean(), l1[-100:].mean()
    assert abs(m0 - m1) <= 0.05 * max(m0, m1), (m0, m1)
    assert abs(a0 - a1) <= 0.05 * max(a0, a1), (a0, a1)
