"""What the learned closure gains over the method without it, a priori: the
network, trained by the library's own kernels on box-filtered snapshots of
this solver's DNS (Kelvin-Helmholtz layer, 64x65x64, 3x3 top-hat in x and
z, seeded 80/20 split by snapshot), predicts the held-out snapshots'
deviatoric subfilter stresses with a smaller error than the best eddy
viscosity -- Smagorinsky with its coefficient fitted to each y-plane of the
training snapshots, a lower bound for the dynamic model's a-priori error."""
import numpy as np
import pytest

from diablo_b200 import closure, grid as G, ics, params as P

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
