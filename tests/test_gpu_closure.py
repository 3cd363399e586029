"""What the learned closure gains over the method without it.

A priori: the network, trained by the library's own kernels on box-filtered
snapshots of this solver's DNS (Kelvin-Helmholtz layer, 64x65x64, 3x3
top-hat in x and z, seeded 80/20 split by snapshot), predicts the held-out
snapshots' deviatoric subfilter stresses with a smaller error than the best
eddy viscosity -- Smagorinsky with its coefficient fitted to each y-plane of
the training snapshots, a lower bound for the dynamic model's a-priori error.

A posteriori: trained on the stresses of the spectral cutoff that the LES
resolves (closure.cutoff_snapshots: Kelvin-Helmholtz DNS 96x65x96, LES
32x65x32), the closure run inside the LES for 2010 steps from the truncated
initial state gives mean-velocity and u'v' profiles closer to the truncated
DNS than the LES without a model -- on the Kelvin-Helmholtz layer and in a
turbulent channel at Re_tau 180 (DNS 192x65x192, LES 64x65x64)."""
import numpy as np
import pytest

from diablo_b200 import closure, grid as G, ics, params as P
from diablo_b200.channel import Channel
from diablo_b200.layout import dealiased

pytestmark = pytest.mark.gpu


def test_closure_beats_best_eddy_viscosity_on_held_out_snapshots():
    p = P.kelvin_helmholtz(64, 65, 64)
    g = G.channel_grid(G.uniform_gy(p.ny, -10.0, 10.0))
    u, th = ics.shear_layer(p, g, seed=31, amp=0.2)
    data = closure.dns_snapshots(p, g, 0.01, u, th, count=40, every=3, warmup=10, width=3, stride=2)
    rep = closure.train_and_evaluate(data, seed=32, steps=8000, batch=1024, lr=2e-3)
    # mini-batch losses (normalised stresses: a zero prediction scores about 3)
    assert np.isfinite(rep.losses).all() and rep.losses[-500:].mean() < 0.8 * rep.losses[:50].mean()
    assert rep.mlp_test_error_deviatoric < 0.8 * rep.eddy_viscosity_test_error, rep.summary()


def test_cutoff_targets_share_the_les_feature_points():
    """The host-side truncated field that the cutoff stresses are formed from
    is the field the sampler differentiates: its centred x and z differences
    at the LES points equal the sampler's gradient features (times G)."""
    p = P.kelvin_helmholtz(96, 65, 96)
    g = G.channel_grid(G.uniform_gy(p.ny, -10.0, 10.0))
    u, th = ics.shear_layer(p, g, seed=41, amp=0.2)
    q = p.copy()
    q.nx, q.nz = 32, 32
    with Channel(p, g, 0.01) as c, Channel(q, g, 0.01) as lc:
        c.init_from_physical(u, th)
        c.step(20)
        s = c.download()
        lc.upload([closure.coarsen(p, s["cu"][k], q) for k in range(3)], closure.coarsen(p, s["cp"], q),
                  np.stack([closure.coarsen(p, s["cth"][0], q)]))
        x, _, sc = lc.sgs_samples(1, 1)
    u1 = closure._to_physical(dealiased(p, s["cu"][0])[2:p.ny][:, closure._les_kz(p, 10)][:, :, :11], 32, 32)
    gn = np.sqrt(sc.astype(np.float64)) / x[:, 10].astype(np.float64)
    for axis, h, col in ((2, p.lx / 32, 0), (1, p.lz / 32, 2)):
        host = ((np.roll(u1, -1, axis=axis) - np.roll(u1, 1, axis=axis)) / (2 * h)).reshape(-1)
        dev = x[:, col].astype(np.float64) * gn
        assert np.linalg.norm(dev - host) < 1e-6 * np.linalg.norm(host)


def test_cutoff_trained_closure_beats_no_model_a_posteriori():
    p = P.kelvin_helmholtz(96, 65, 96)
    g = G.channel_grid(G.uniform_gy(p.ny, -10.0, 10.0))
    u, th = ics.shear_layer(p, g, seed=41, amp=0.2)
    data = closure.cutoff_snapshots(p, g, 0.01, u, th, count=400, every=5, warmup=10)
    rep = closure.train_and_evaluate(data, seed=42, steps=20000, batch=4096, lr=2e-3)
    assert rep.mlp_test_error_deviatoric < rep.eddy_viscosity_test_error, rep.summary()
    ap = closure.a_posteriori(p, g, 0.01, u, th, 2010, rep.params)
    cl, nm = ap["closure"]["profile_errors"], ap["no_model"]["profile_errors"]
    assert cl["ume"] < nm["ume"] and cl["uv"] < nm["uv"], ap


def test_channel_les_closure_beats_no_model_a_posteriori():
    """Channel LES at Re_tau 180 (DNS 192x65x192, LES 64x65x64, 2000 LES
    steps, profiles averaged every 100 steps): the closure trained on the
    DNS's spectral-cutoff stresses gives mean-velocity and u'v' profiles
    closer to the truncated DNS than the LES without a model."""
    out = closure.channel_les_study(snapshots=60, every=30)
    ap = out["a_posteriori"]
    cl, nm = ap["closure"]["profile_errors"], ap["no_model"]["profile_errors"]
    assert cl["ume"] < nm["ume"] and cl["uv"] < nm["uv"], ap
