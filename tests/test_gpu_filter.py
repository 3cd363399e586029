"""filter_chan (filter.f:1-98) on the GPU against the CPU FP64 oracle, and the
oracle against a direct numpy restatement of the filter on one column."""
import numpy as np
import pytest

from diablo_b200 import grid as G, ics, layout, params as P
from oracle.oracle import Oracle


def case(nx=48, ny=33, nz=36, seed=4):
    p = P.kelvin_helmholtz(nx, ny, nz)
    g = G.channel_grid(G.create_grid(2, ny, 20.0, 1.5))
    u, th = ics.shear_layer(p, g, seed=seed, amp=0.2)
    return p, g, u, th


def test_oracle_filter_matches_direct_formula():
    p, g, u, th = case()
    o = Oracle(p, g, 0.01)
    o.init_from_physical(u, th)
    c0 = o.cth[0].copy()
    o.filter_chan(1)
    c1 = o.cth[0]
    i, k = 5, 7                                    # a column with I >= 1, K >= 1
    kx = i * 2 * np.pi / p.lx
    kz = k * 2 * np.pi / p.lz
    s0 = 0.5 * (1 + np.cos(np.hypot(kx * p.lx / p.nx, kz * p.lz / p.nz)))
    sg = s0 ** 4 * (35 - 84 * s0 + 70 * s0 ** 2 - 20 * s0 ** 3)
    h = c0[:, k, i].copy()
    h[: p.ny + 1] *= sg
    ref = h.copy()
    for j in range(2, p.ny):
        ref[j] = 5 / 8 * h[j] + 0.25 * (h[j + 1] + h[j - 1]) - 1 / 16 * (h[j + 2] + h[j - 2])
    assert np.allclose(c1[:, k, i], ref, rtol=1e-13, atol=1e-15 * np.abs(ref).max())
    # the mean mode and the kx = 0 / kz = 0 columns get only the horizontal factor
    assert np.array_equal(c1[:, 0, 0], c0[:, 0, 0])
    assert np.array_equal(c1[p.ny + 1], c0[p.ny + 1])


@pytest.mark.gpu
def test_filter_chan_matches_oracle():
    from diablo_b200.channel import Channel
    p, g, u, th = case()
    o = Oracle(p, g, 0.01)
    o.init_from_physical(u, th)
    with Channel(p, g, 0.01) as c:
        c.upload([x.copy() for x in o.cu], o.cp.copy(), o.cth.copy())
        c.filter_chan(1)
        o.filter_chan(1)
        got = layout.dealiased(p, c.download()["cth"][0])
        ref = layout.dealiased(p, o.cth[0])
        assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)
