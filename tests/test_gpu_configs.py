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
field in each field's own norm, with two documented exceptions, both
round-off of the O(1) fields seen through a much smaller one:

* CP accumulates phi/h, and phi solves for the divergence of a nearly
  solenoidal field, so the round-off of the O(1) velocity (1e-16) reaches CP
  amplified by the cancellation and by 1/h -- in both codes, which then
  agree only to that level.  CP is held to 1e-10 against the
  dynamic-pressure scale |U|^2 (its L2 norm over the points, |U|^2 / sqrt(N)),
  and to 1e-8 in its own norm unless CP itself is below 1e-3 of that scale
  (the nearly laminar 512x257x384 workload, where CP is 6e-4 of it).
* A velocity component whose norm is below 1e-3 of the velocity norm (U2
  and U3 of the nearly laminar 512x257x384 workload, 3e4 times smaller than
  U1) receives the O(1) fields' round-off through the projection.  It is
  held to 1e-8 in its own norm and 1e-13 against the velocity norm.

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
SMALL_FIELD = 1e-3      # a velocity component below this fraction of |U| is "small"
SMALL_VS_U = 1e-13      # bar of a small component against |U|


def small_components(norms):
    """Velocity components (cu1..cu3) whose norm is below SMALL_FIELD of the
    velocity norm, with their norm as a fraction of it."""
    vel = float(np.sqrt(sum(norms[n] ** 2 for n in ("cu1", "cu2", "cu3"))))
    return {n: norms[n] / vel for n in ("cu1", "cu2", "cu3") if norms[n] < SMALL_FIELD * vel}


def check64(err, pscale_err=None, small=None, cp_small=False):
    """FP64 bar: every field to 1e-10 in its own norm, except CP (1e-10
    against the pressure scale when given, and 1e-8 in its own norm unless
    `cp_small`) and the small velocity components in `small` (name -> norm /
    |U|): 1e-8 in their own norm and 1e-13 against |U|."""
    small = small or {}
    rest = {k: v for k, v in err.items() if k != "cp" and k not in small}
    assert max(rest.values()) < TOL64, err
    if not cp_small:
        assert err["cp"] < CP_OWN, err
    for n, frac in small.items():
        assert err[n] < CP_OWN and err[n] * frac < SMALL_VS_U, (n, frac, err)
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
    the largest of the L2 differences of the low modes, the plane norms and
    the mean profile, each divided by the field's own L2 norm (the root sum
    of squares of its plane norms).  A part of a field can itself be
    round-off -- the plane mean of U2 is 1e-26 at 512x257x384 -- so it is
    not divided by its own norm."""
    m = _fixture_module()
    k = int(ref["k"])
    got = m.summarise(p, m.state_fields(s), k)
    out = {}
    for i, n in enumerate(NAMES):
        scale = float(np.linalg.norm(ref["plane_norm"][i]))
        scale = scale if scale > 0 else 1.0
        out[n] = max(float(np.linalg.norm(got[part][i] - ref[part][i])) / scale
                     for part in ("low_modes", "plane_norm", "mean"))
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
    """Errors against the fixture (summary_errors), and the number of
    dealiased points of a field."""
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
    return summary_errors(w.p, s, ref), layout.dealiased(w.p, s["cp"]).size


def check64_fixture(err, npts, ref):
    """check64 for a fixture comparison: the small velocity components and
    the pressure scale |U|^2 / sqrt(N) from the fixture's own norms."""
    norms = {n: float(np.linalg.norm(ref["plane_norm"][i])) for i, n in enumerate(NAMES)}
    u2 = sum(norms[n] ** 2 for n in ("cu1", "cu2", "cu3"))
    pscale = u2 / np.sqrt(npts)
    check64(err, pscale_err=err["cp"] * norms["cp"] / pscale, small=small_components(norms),
            cp_small=norms["cp"] < SMALL_FIELD * pscale)


def test_channel_192x129x160_200_steps_matches_oracle_fixture():
    """Config 2: Re_tau 180 channel, tanh grid, no-slip walls, constant
    pressure gradient, passive scalar Pr 0.71, CFL-adaptive dt, 200 steps."""
    ref = np.load(os.path.join(GOLDEN, "oracle_channel_192x129x160_200steps.npz"))
    w = workloads.channel(192, 129, 160)
    check64_fixture(*_run_against_fixture(w, 200, ref, check_dt=True), ref)


PRECISION_FIXTURE = os.path.join(GOLDEN, "oracle_precision_512x257x384_100steps.npz")


@pytest.mark.skipif(not os.path.exists(PRECISION_FIXTURE), reason="precision fixture not generated")
@pytest.mark.parametrize("prec", [P.PREC_FP64, P.PREC_FP32SPLIT])
def test_precision_512x257x384_100_steps_matches_oracle_fixture(prec):
    """Config 3 grid and fields, 100 steps: the FP64 path to 1e-10 (with the
    small-field and pressure bars of the module) and the FP32-split path to
    1e-5, each field in its own norm."""
    ref = np.load(PRECISION_FIXTURE)
    w = workloads.precision(512, 257, 384, prec=prec)
    err, npts = _run_against_fixture(w, 100, ref, check_dt=False)
    if prec == P.PREC_FP64:
        check64_fixture(err, npts, ref)
    else:
        assert max(err.values()) < TOL32, err
