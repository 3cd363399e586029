"""FP64 restatement of the learned subgrid-stress closure (the MLP of
diablo_b200/csrc/mlp.cu): forward pass, loss, analytic gradient and one Adam
step, in numpy.

TEST INFRASTRUCTURE ONLY: the checker of the GPU kernels in tests/ (the
forward values and the gradients they compute), never imported by the
diablo_b200 package.  The reference has no such model, so this oracle is
checked against finite differences of itself (tests/test_oracle_mlp.py).

Parameter vector layout (float, as the C ABI): W1[64][11] b1[64] W2[64][64]
b2[64] W3[64][64] b3[64] W4[6][64] b4[6] | in_mean[11] in_scale[11]
out_scale[6].  GELU is its tanh form, 0.5 z (1 + tanh(sqrt(2/pi) (z +
0.044715 z^3))).
"""
from __future__ import annotations

import math

import numpy as np

NIN, NH, NOUT = 11, 64, 6
SHAPES = [("W1", (NH, NIN)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NH, NH)), ("b3", (NH,)),
          ("W4", (NOUT, NH)), ("b4", (NOUT,))]
NTRAIN = sum(int(np.prod(s)) for _, s in SHAPES)
NPARAM = NTRAIN + NIN + NIN + NOUT

_C = math.sqrt(2.0 / math.pi)


def unpack(p: np.ndarray) -> dict:
    p = np.asarray(p, dtype=np.float64)
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape)
        o += n
    out["mean"] = p[o:o + NIN]
    out["scale"] = p[o + NIN:o + 2 * NIN]
    out["oscale"] = p[o + 2 * NIN:o + 2 * NIN + NOUT]
    return out


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to bfloat16 (round to nearest even on the float32 bits), as
    __float2bfloat16_rn does; returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(_C * (z + 0.044715 * z ** 3)))


def gelu_d(z):
    t = np.tanh(_C * (z + 0.044715 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * _C * (1.0 + 3 * 0.044715 * z * z)


def forward(p: np.ndarray, x: np.ndarray, emulate_bf16: bool = False, keep: bool = False):
    """Stresses (physical units) for features x [n][11].  With emulate_bf16
    the weights, the normalised inputs and the hidden activations are rounded
    to bfloat16 as the tensor-core kernels see them."""
    q = unpack(p)
    r = bf16 if emulate_bf16 else (lambda a: a)
    h = r((np.asarray(x, dtype=np.float64) - q["mean"]) / q["scale"])
    hs, zs = [h], []
    for l in (1, 2, 3):
        z = h @ r(q[f"W{l}"]).T + q[f"b{l}"]
        zs.append(z)
        h = r(gelu(z))
        hs.append(h)
    y = h @ r(q["W4"]).T + q["b4"]
    if keep:
        return y, hs, zs
    return y * q["oscale"]


_PAIRS = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]


def dissipation_weights(x: np.ndarray, oscale: np.ndarray) -> np.ndarray:
    """pe[n][6]: Pi(tau) = sum_k pe_k y_k for tau_k = out_scale_k y_k,
    Pi = -sum_ij tau_ij S_ij with S_ij the symmetric part of the gradient
    features g_ij = x[3i+j] (off-diagonal pairs counted twice)."""
    g = np.asarray(x, dtype=np.float64)[:, :9].reshape(-1, 3, 3)
    s = 0.5 * (g + g.transpose(0, 2, 1))
    sv = np.stack([s[:, a, b] for a, b in _PAIRS], axis=1)
    c = np.array([1.0, 1.0, 1.0, 2.0, 2.0, 2.0])
    return -c * np.asarray(oscale, dtype=np.float64) * sv


def loss_grad(p: np.ndarray, x: np.ndarray, t: np.ndarray, diss_weight: float = 0.0):
    """Loss sum (y - t/out_scale)^2 / (2n) over samples and outputs (y the
    normalised output), plus diss_weight/(2n) sum (Pi(y) - Pi(t))^2 over
    samples (the subgrid dissipation, dissipation_weights), and its gradient
    with respect to the trained parameters, FP64."""
    q = unpack(p)
    n = x.shape[0]
    y, hs, zs = forward(p, x, keep=True)
    e = y - np.asarray(t, dtype=np.float64) / q["oscale"]
    loss = 0.5 * float(np.sum(e * e)) / n
    d = e / n
    if diss_weight:
        pe = dissipation_weights(x, q["oscale"])
        dpi = np.sum(pe * e, axis=1)
        loss += 0.5 * diss_weight * float(np.sum(dpi * dpi)) / n
        d = d + diss_weight * dpi[:, None] * pe / n
    grads = {"W4": d.T @ hs[3], "b4": d.sum(axis=0)}
    g = d @ q["W4"]
    for l in (3, 2, 1):
        dl = g * gelu_d(zs[l - 1])
        grads[f"W{l}"] = dl.T @ hs[l - 1]
        grads[f"b{l}"] = dl.sum(axis=0)
        g = dl @ q[f"W{l}"]
    return loss, np.concatenate([grads[name].reshape(-1) for name, _ in SHAPES])


def adam_step(p, grad, m1, m2, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update of the trained parameters (step counts from 1)."""
    p = np.array(p, dtype=np.float64)
    m1 = b1 * m1 + (1 - b1) * grad
    m2 = b2 * m2 + (1 - b2) * grad * grad
    p[:NTRAIN] -= lr * (m1 / (1 - b1 ** step)) / (np.sqrt(m2 / (1 - b2 ** step)) + eps)
    return p, m1, m2
