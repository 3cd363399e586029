"""GPU parity on the three benchmark configurations at their own sizes and
step counts, against the CPU FP64 oracle.

* Kelvin-Helmholtz shear layer 64x65x64, fixed dt = 0.01, 100 steps: the
  oracle runs beside the GPU in the test.
* Wall-bounded channel 192x129x160 (Re_tau 180 scale, passive scalar,
  CFL-adaptive dt), 200 steps; and the 512x257x384 precision workload, 100
  steps: the oracle needs minutes to hours on the CPU for these, so its
  results are committed fixtures (tests/golden/make_config_fixtures.py):
  per-plane norms, the plane means and the modes |kx|, |kz| <= 6 of every
  plane of CU1, CU2, CU3, CTH and CP, and the DELTA_T of every step.

The all-FP64 GPU path must agree with the oracle to 1e-10 relative L2 per
field in each field's own norm, except CP: CP accumulates phi/h, and phi
solves for the divergence of a nearly solenoidal field, so the round-off of
the O(1) velocity (1e-16) reaches CP amplified by the cancellation and by
1/h -- in both codes, which then agree only to that level.  CP is held to
1e-8 in its own norm and 1e-10 against the dynamic-pressure scale |U|^2.
The FP32-split path, at the benchmark size, agrees to 1e-5 in each field's
own norm."""
import importlib.util
import os

import numpy as np
import pytest

from diablo_b200 import layout, params as P, workloads
from diablo_b200.channel import Channel
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL64 = 1e-10
TOL32 = 1e-5
NAMES = ("cu1", "cu2", "cu3", "cth1", "cp")


def _fixture_module():
    spec = importlib.util.spec_from_file_location("make_config_fixtures",
                                                  os.path.join(GOLDEN, "make_config_fixtures.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def relerr(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


CP_OWN = 1e-8


def check64(err, pscale_err=None):
    """FP64 bar: every field but CP to 1e-10 in its own norm; CP to 1e-8 in
    its own norm (and, when given, 1e-10 against the pressure scale)."""
    rest = {k: v for k, v in err.items() if k != "cp"}
    assert max(rest.values()) < TOL64, err
    assert err["cp"] < CP_OWN, err
    if pscale_err is not None:
        assert pscale_err < TOL64, (pscale_err, err)


def pressure_scale_error(p, s, o):
    u = [layout.dealiased(p, o.cu[c]) for c in range(3)]
    uscale = float(np.sqrt(sum(np.linalg.norm(x) ** 2 for x in u)))
    d = np.linalg.norm(layout.dealiased(p, s["cp"]) - layout.dealiased(p, o.cp))
    return float(d / (uscale ** 2 / np.sqrt(u[0].size)))


def own_norm_errors(p, s, o):
    """Relative L2 of every field's dealiased block in its own norm."""
    a = [s["cu"][0], s["cu"][1], s["cu"][2], s["cth"][0], s["cp"]]
    b = [o.cu[0], o.cu[1], o.cu[2], o.cth[0], o.cp]
    return {n: relerr(layout.dealiased(p, x), layout.dealiased(p, y)) for n, x, y in zip(NAMES, a, b)}


def summary_errors(p, s, ref):
    """Errors of a downloaded state against a fixture summary, per field:
    the low modes, the plane norms and the mean profile, each in its own
    norm."""
    m = _fixture_module()
    k = int(ref["k"])
    got = m.summarise(p, m.state_fields(s), k)
    out = {}
    for i, n in enumerate(NAMES):
        out[n] = max(relerr(got["low_modes"][i], ref["low_modes"][i]),
                     relerr(got["plane_norm"][i], ref["plane_norm"][i]),
                     relerr(got["mean"][i], ref["mean"][i]))
    return out


def test_kh_64x65x64_100_steps_matches_oracle():
    """Config 1: KH shear layer, Re 1000, Pr 1, Ri 0.1, dt 0.01, 100 steps."""
    w = workloads.kh(64, 65, 64)
    u, th = w.initial_fields()
    o = Oracle(w.p, w.grid, w.dt)
    o.init_from_physical(u, th)
    with Channel(w.p, w.grid, w.dt) as c:
        c.upload([x.copy() for x in o.cu], o.cp.copy(), o.cth.copy())
        o.step(100)
        c.step(100)
        s = c.download()
    check64(own_norm_errors(w.p, s, o), pressure_scale_error(w.p, s, o))


def _run_against_fixture(w, steps, ref, check_dt):
    with Channel(w.p, w.grid, w.dt) as c:
        u, th = w.initial_fields()
        c.init_from_physical(u, th)
        dts = []
        for _ in range(steps):
            c.step()
            dts.append(c.delta_t)
        s = c.download()
    if check_dt:
        dref = np.asarray(ref["delta_t"])
        assert np.max(np.abs(np.array(dts) - dref) / dref) < 1e-10
    return summary_errors(w.p, s, ref)


def test_channel_192x129x160_200_steps_matches_oracle_fixture():
    """Config 2: Re_tau 180 channel, tanh grid, no-slip walls, constant
    pressure gradient, passive scalar Pr 0.71, CFL-adaptive dt, 200 steps."""
    ref = np.load(os.path.join(GOLDEN, "oracle_channel_192x129x160_200steps.npz"))
    w = workloads.channel(192, 129, 160)
    check64(_run_against_fixture(w, 200, ref, check_dt=True))


PRECISION_FIXTURE = os.path.join(GOLDEN, "oracle_precision_512x257x384_100steps.npz")


@pytest.mark.skipif(not os.path.exists(PRECISION_FIXTURE), reason="precision fixture not generated")
@pytest.mark.parametrize("prec", [P.PREC_FP64, P.PREC_FP32SPLIT])
def test_precision_512x257x384_100_steps_matches_oracle_fixture(prec):
    """Config 3 grid and fields, 100 steps: the FP64 path to 1e-10 and the
    FP32-split path to 1e-5, each field in its own norm."""
    ref = np.load(PRECISION_FIXTURE)
    w = workloads.precision(512, 257, 384, prec=prec)
    err = _run_against_fixture(w, 100, ref, check_dt=False)
    if prec == P.PREC_FP64:
        check64(err)
    else:
        assert max(err.values()) < TOL32, err
