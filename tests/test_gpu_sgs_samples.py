"""The closure's sampler (diablo_gpu_sgs_samples) against its numpy
restatement (oracle/sgs_oracle.py) on the same state: the GPU's physical
fields come from its own transforms, the oracle's from the CPU oracle's
FFT_XZ_TO_PHYSICAL of the downloaded state, so the comparison covers both.
Outputs are float32: per column, agreement to 1e-5 of the column's scale
(the targets, divided by the small scale Delta^2 G^2, to 1e-4)."""
import numpy as np
import pytest

from diablo_b200 import grid as G, ics, params as P
from diablo_b200.channel import Channel
from diablo_b200.layout import new_physical
from oracle.oracle import Oracle
from oracle import sgs_oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("width,stride", [(1, 1), (3, 1), (3, 2), (5, 3)])
def test_samples_match_oracle(width, stride):
    p = P.turbulent_channel(32, 33, 24, re_tau=180.0, variable_dt=False)
    g = G.channel_grid(G.create_grid(1, p.ny, 2.0, 1.75))
    u, th = ics.poiseuille(p, g, u_center=10.0, seed=9, noise=0.5)
    o = Oracle(p, g, 2e-4)
    o.init_from_physical(u, th)
    with Channel(p, g, 2e-4) as c:
        c.upload([x.copy() for x in o.cu], o.cp.copy(), o.cth.copy())
        c.step(2)
        x, t, sc = c.sgs_samples(width, stride)
        s = c.download()
    phys = []
    for k in range(3):
        v = new_physical(p)
        o.fft_xz_to_physical(s["cu"][k].copy(), v, 0, p.ny + 1)
        phys.append(v[:, : p.nz, : p.nx].copy())
    xo, to, so = sgs_oracle.samples(*phys, g.gyf, g.dyf, p.lx / p.nx, p.lz / p.nz, p.nu, width, stride)
    assert x.shape == xo.shape and t.shape == to.shape and sc.shape == so.shape
    for a, b in ((x, xo), (t, to), (sc[:, None], so[:, None])):
        scale = np.abs(b).max(axis=0)
        scale[scale == 0] = 1.0
        tol = 1e-4 if a is t else 1e-5
        assert (np.abs(a - b).max(axis=0) <= tol * scale).all(), np.abs(a - b).max(axis=0) / scale
    if width > 1:
        assert np.abs(t[:, 0]).max() > 0          # the filter leaves a subfilter stress
