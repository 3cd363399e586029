"""numpy restatement of the closure's training samples (the sampler of
diablo_b200/csrc/les.cu, k_sgs_samples): features and targets of a w x w
top-hat filter in x and z at GYF points J = 2..NY-1.

TEST INFRASTRUCTURE ONLY: the checker of diablo_gpu_sgs_samples in tests/.
The reference has no such sampler.
"""
from __future__ import annotations

import numpy as np


def samples(u1, u2, u3, gyf, dyf, dx, dz, nu, w, stride):
    """u1, u2, u3: physical fields [NY+2][NZ][NX] (U2 at GY points).
    Returns the dimensionless features [n][11] (g_ij/G, y+, Delta), targets
    [n][6] (tau_ij / s) and scales s = Delta^2 G^2 [n] in FP64, n = (NY-2) *
    ceil(NX/stride) * ceil(NZ/stride), J-major then z then x."""
    ny = u1.shape[0] - 2
    u2f = np.zeros_like(u2)
    u2f[:-1] = 0.5 * (u2[:-1] + u2[1:])
    us = [u1, u2f, u3]
    hw = (w - 1) // 2

    def box(a):
        out = np.zeros_like(a)
        for dk in range(-hw, hw + 1):
            for di in range(-hw, hw + 1):
                out += np.roll(np.roll(a, -dk, axis=-2), -di, axis=-1)
        return out / (w * w)

    ub = [box(a) for a in us]
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    tau = [box(us[a] * us[b]) - ub[a] * ub[b] for a, b in pairs]
    js = np.arange(2, ny)
    feats = []
    for c in range(3):
        f = ub[c]
        feats.append((np.roll(f, -1, axis=-1) - np.roll(f, 1, axis=-1))[js] / (2 * dx))
        hy = (gyf[js + 1] - gyf[js - 1])[:, None, None]
        feats.append((f[js + 1] - f[js - 1]) / hy)
        feats.append((np.roll(f, -1, axis=-2) - np.roll(f, 1, axis=-2))[js] / (2 * dz))
    shape = feats[0].shape
    dwall = np.minimum(gyf[js] - gyf[1], gyf[ny] - gyf[js])
    feats.append(np.broadcast_to((dwall / nu)[:, None, None], shape))
    feats.append(np.broadcast_to(np.cbrt(w * dx * dyf[js] * w * dz)[:, None, None], shape))
    sl = (slice(None), slice(None, None, stride), slice(None, None, stride))
    x = np.stack([f[sl].reshape(-1) for f in feats], axis=1)
    t = np.stack([a[js][sl].reshape(-1) for a in tau], axis=1)
    g2 = np.sum(x[:, :9] ** 2, axis=1)
    G = np.sqrt(g2)
    x[:, :9] = np.where(G[:, None] > 0, x[:, :9] / np.where(G > 0, G, 1.0)[:, None], 0.0)
    s = x[:, 10] ** 2 * g2
    t = np.where(s[:, None] > 0, t / np.where(s > 0, s, 1.0)[:, None], 0.0)
    return x, t, s
