"""GPU parity of POISSON_P_CHAN and the SAVE_STATS_CHAN plane statistics
against the CPU FP64 oracle, through the C ABI.

Both are FP64 on the device.  The GPU sums the pressure source in physical
space and transforms it once (the oracle transforms each product group and
sums in Fourier space), and its plane sums run in a different order, so the
agreement is to round-off: 1e-10 relative L2."""
import numpy as np
import pytest

from diablo_b200 import grid as G, ics, layout, params as P, workloads
from diablo_b200.channel import Channel
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
TOL = 1e-10

FIRST_ORDER = ["ume", "vme", "wme", "urms", "vrms", "wrms", "dudy", "dwdy", "thme", "dthdy", "thrms"]
SECOND_ORDER = ["uv", "uw", "wv", "cp", "shear", "thv"]
INDEX = {"ume": 0, "vme": 1, "wme": 2, "urms": 3, "vrms": 4, "wrms": 5, "uv": 6, "uw": 7, "wv": 8,
         "dudy": 9, "dwdy": 10, "cp": 11, "shear": 12, "thme": 13, "dthdy": 14, "thrms": 15, "thv": 16}


def relerr(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def kh_pair(nx, ny, nz, steps, stretched=True, seed=11):
    p = P.kelvin_helmholtz(nx, ny, nz)
    gy = G.create_grid(2, ny, 20.0, 1.5) if stretched else G.uniform_gy(ny, -10.0, 10.0)
    g = G.channel_grid(gy)
    u, th = ics.shear_layer(p, g, seed=seed, amp=0.05)
    o = Oracle(p, g, 0.02)
    o.init_from_physical(u, th)
    o.step(steps)
    return p, g, o


def channel_pair(nx, ny, nz, steps):
    w = workloads.channel(nx, ny, nz)
    w.p.variable_dt = 0
    u, th = w.initial_fields()
    o = Oracle(w.p, w.grid, w.dt)
    o.init_from_physical(u, th)
    o.step(steps)
    return w.p, w.grid, o


def upload(p, g, o, dt):
    c = Channel(p, g, dt)
    c.upload([x.copy() for x in o.cu], o.cp.copy(), o.cth.copy(), [x.copy() for x in o.cf])
    return c


@pytest.mark.parametrize("case", ["kh", "channel"])
def test_poisson_p_chan_matches_oracle(case):
    if case == "kh":
        p, g, o = kh_pair(48, 33, 36, steps=3)
        dt = 0.02
    else:
        p, g, o = channel_pair(48, 33, 40, steps=2)
        dt = 1e-3
    with upload(p, g, o, dt) as c:
        c.poisson_p_chan()
        o.poisson_p_chan()
        s = c.download()
        a = layout.dealiased(p, s["cp"])[1:p.ny + 1]
        b = layout.dealiased(p, o.cp)[1:p.ny + 1]
        assert np.linalg.norm(b) > 0
        assert relerr(a, b) < TOL
        # the velocity and scalars are inputs only
        for f in range(3):
            assert np.array_equal(layout.dealiased(p, s["cu"][f]), layout.dealiased(p, o.cu[f]))


def test_poisson_p_chan_idempotent():
    """A second call on the same state gives the same CP (idempotent)."""
    p, g, o = kh_pair(32, 17, 24, steps=2, stretched=False)
    with upload(p, g, o, 0.02) as c:
        c.poisson_p_chan()
        first = c.download()["cp"].copy()
        c.poisson_p_chan()
        second = c.download()["cp"]
        assert np.array_equal(first, second)


@pytest.mark.parametrize("case", ["kh", "channel"])
def test_stats_match_oracle(case):
    if case == "kh":
        p, g, o = kh_pair(48, 33, 36, steps=3)
        dt = 0.02
    else:
        p, g, o = channel_pair(48, 33, 40, steps=2)
        dt = 1e-3
    with upload(p, g, o, dt) as c:
        got = c.stats()
        ref = o.stats()
        for group in (FIRST_ORDER, SECOND_ORDER):
            floor = 1e-3 * max(np.linalg.norm(ref[INDEX[k]]) for k in group)
            for k in group:
                r, a = ref[INDEX[k]], got[INDEX[k]]
                err = float(np.linalg.norm(a - r) / max(np.linalg.norm(r), floor))
                assert err < TOL, (k, err)
        # APPLY_BC_VEL is the one state change the statistics keep
        s = c.download()
        for f in range(3):
            assert relerr(layout.dealiased(p, s["cu"][f]), layout.dealiased(p, o.cu[f])) < 1e-14


def kh2_pair(nx, ny, nz, steps):
    """A shear layer with a second, passive scalar (Pr 2)."""
    p = P.kelvin_helmholtz(nx, ny, nz)
    p.n_th = 2
    p.pr[1], p.ri[1] = 2.0, 0.0
    p.th_bc_ymin[1] = p.th_bc_ymax[1] = 1
    g = G.channel_grid(G.create_grid(2, ny, 20.0, 1.5))
    u, th1 = ics.shear_layer(p, g, seed=5, amp=0.1)
    th = np.stack([th1[0], 0.5 * th1[0] ** 2 + 0.1 * u[0]])
    o = Oracle(p, g, 0.02)
    o.init_from_physical(u, th)
    o.step(steps)
    return p, g, o


@pytest.mark.parametrize("case", ["kh2", "channel"])
def test_mean_stats_match_oracle(case):
    """Every mean.h5 / tke.h5 profile (vorticity, pseudo-dissipation, the
    per-scalar profiles) against the oracle's restatement of save_stats.f."""
    if case == "kh2":
        p, g, o = kh2_pair(48, 33, 36, steps=3)
        dt = 0.02
    else:
        p, g, o = channel_pair(48, 33, 40, steps=2)
        dt = 1e-3
    with upload(p, g, o, dt) as c:
        got = c.mean_stats()
        ref = o.mean_stats()
        assert sorted(got) == sorted(ref)
        for k, r in ref.items():
            a = got[k]
            scale = max(np.abs(r).max(), 1e-300)
            err = float(np.abs(a - r).max() / scale)
            assert err < 1e-11, (k, err)
        assert np.abs(ref["omega_z"]).max() > 0 and np.abs(ref["epsilon"]).max() > 0
        if p.n_th > 1:
            assert np.abs(ref["pe_diss02"]).max() > 0 and not np.allclose(ref["thrms02"], ref["thrms01"])


def test_les_epsilon_sgs_matches_oracle(tmp_path):
    """tkebudget_chan_les through the statistics writer on an LES instance
    (NU_T and the state from the device) against the oracle."""
    from diablo_b200 import statsfile
    from test_gpu_les import les_channel
    p, g, u, th = les_channel(32, 33, 24)
    o = Oracle(p, g, 1e-3)
    o.init_from_physical(u, th)
    with Channel(p, g, 1e-3) as c:
        c.upload([x.copy() for x in o.cu], o.cp.copy(), o.cth.copy())
        for _ in range(2):
            o.step()
            c.step()
        m = statsfile.StatsWriter(str(tmp_path)).save(c)
        ref = o.epsilon_sgs()
        rows = slice(1, p.ny + 1)
        scale = np.abs(ref[rows]).max()
        assert scale > 0
        assert np.abs(m["epsilon_sgs"][rows] - ref[rows]).max() <= 1e-8 * scale
        assert statsfile.read(str(tmp_path / "tke.h5"))["epsilon_sgs"]["SAMPLES"] == 1
