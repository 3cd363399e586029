"""CPU checks of the closure network's FP64 oracle (oracle/mlp_oracle.py):
its analytic gradient against central differences, the bfloat16 rounding it
uses to mirror the tensor-core kernels, and one Adam step."""
import numpy as np

from diablo_b200 import mlp as ML
from oracle import mlp_oracle as M


def sample(seed, n=24):
    rng = np.random.default_rng(seed)
    p = ML.init_params(seed, mean=rng.normal(size=11), scale=rng.uniform(0.5, 2.0, 11),
                       out_scale=rng.uniform(0.5, 2.0, 6)).astype(np.float64)
    p[:M.NTRAIN] += 0.05 * rng.normal(size=M.NTRAIN)     # non-zero biases too
    x = rng.normal(size=(n, 11)) * 1.5 + 0.3
    t = rng.normal(size=(n, 6))
    return p, x, t


def test_layout_sizes():
    assert M.NTRAIN == ML.NTRAIN == 9478 and M.NPARAM == ML.NPARAM == 9506


def test_gradient_matches_central_differences():
    p, x, t = sample(1)
    loss, g = M.loss_grad(p, x, t)
    rng = np.random.default_rng(2)
    idx = np.concatenate([rng.choice(M.NTRAIN, 60, replace=False), [0, 703, 704, 767, M.NTRAIN - 1]])
    h = 1e-6
    for i in idx:
        q1, q2 = p.copy(), p.copy()
        q1[i] += h
        q2[i] -= h
        fd = (M.loss_grad(q1, x, t)[0] - M.loss_grad(q2, x, t)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(g[i]), (i, fd, g[i])


def test_forward_matches_loss_definition():
    p, x, t = sample(3)
    y = M.forward(p, x)
    q = M.unpack(p)
    e = (y - t) / q["oscale"]
    assert np.isclose(M.loss_grad(p, x, t)[0], 0.5 * np.sum(e * e) / x.shape[0], rtol=1e-12)


def test_bf16_rounding():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7, 1.0 + 3 * 2 ** -8, -2.5, 3.14159265])
    r = M.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0                  # tie to even
    assert r[2] == 1.0 + 2 ** -7
    assert r[3] == 1.0 + 2 ** -6                        # tie to even (up)
    assert r[4] == -2.5
    assert abs(r[5] - np.pi) < 2 ** -7 * 4


def test_adam_first_step_moves_by_lr():
    p, x, t = sample(4)
    _, g = M.loss_grad(p, x, t)
    q, m1, m2 = M.adam_step(p, g, np.zeros_like(g), np.zeros_like(g), 1, 1e-3)
    d = (q - p)[:M.NTRAIN]
    nz = np.abs(g) > 1e-4      # |g|/(|g|+eps) within 1e-4 of 1
    assert np.allclose(d[nz], -1e-3 * np.sign(g[nz]), rtol=1e-3)
    assert np.array_equal(q[M.NTRAIN:], p[M.NTRAIN:])


def test_dissipation_term_gradient_and_definition():
    """The subgrid-dissipation term of the loss: its value from the stresses
    and gradient features directly (Pi = -tau_ij S_ij, off-diagonals twice),
    and the analytic gradient of the whole loss against central differences."""
    p, x, t = sample(5)
    w = 0.7
    q = M.unpack(p)
    y = M.forward(p, x)                          # physical stresses
    g = x[:, :9].reshape(-1, 3, 3)
    s = 0.5 * (g + g.transpose(0, 2, 1))

    def pi(tau):
        full = np.zeros((tau.shape[0], 3, 3))
        for k, (a, b) in enumerate([(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]):
            full[:, a, b] = full[:, b, a] = tau[:, k]
        return -np.einsum("nij,nij->n", full, s)

    e = (y - t) / q["oscale"]
    want = 0.5 * np.sum(e * e) / x.shape[0] + 0.5 * w * np.sum((pi(y) - pi(t)) ** 2) / x.shape[0]
    loss, grad = M.loss_grad(p, x, t, diss_weight=w)
    assert np.isclose(loss, want, rtol=1e-12)
    rng = np.random.default_rng(6)
    h = 1e-6
    for i in rng.choice(M.NTRAIN, 40, replace=False):
        q1, q2 = p.copy(), p.copy()
        q1[i] += h
        q2[i] -= h
        fd = (M.loss_grad(q1, x, t, w)[0] - M.loss_grad(q2, x, t, w)[0]) / (2 * h)
        assert abs(fd - grad[i]) <= 1e-7 + 1e-5 * abs(grad[i]), (i, fd, grad[i])
