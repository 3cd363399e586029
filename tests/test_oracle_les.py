"""CPU tests of the oracle's constant-Smagorinsky LES branch (les.f,
channel.f LES branches): properties of the model that hold whatever the
flow, checked without a GPU."""
import numpy as np
import pytest

from diablo_b200 import grid as G, ics, params as P
from oracle.oracle import Oracle


def channel_case(les, create_new_flow=0, noise=0.5, neumann_top=False, nx=32, ny=33, nz=24, seed=3, model=1):
    p = P.turbulent_channel(nx, ny, nz, re_tau=180.0, variable_dt=False)
    p.les, p.les_model_type, p.create_new_flow = les, model, create_new_flow
    if neumann_top:
        p.u_bc_ymax = p.w_bc_ymax = 1
        p.u_bc_ymax_c1 = 0.1
    P.validate(p)
    g = G.channel_grid(G.create_grid(1, p.ny, 2.0, 1.75))
    u, th = ics.poiseuille(p, g, u_center=10.0, seed=seed, noise=noise)
    o = Oracle(p, g, 2e-4)
    o.init_from_physical(u, th)
    return p, o


def state(o):
    return [x.copy() for x in o.cu] + [o.cp.copy()] + [x.copy() for x in o.cth]


def test_eddy_viscosity_rows_and_sign():
    """NU_T = C_s^2 Delta^2 |S| >= 0; GHOST_LES zeroes rows 1, 2, NY, NY+1
    and row 0 is never written (mpi.f:494-507)."""
    p, o = channel_case(1)
    o.step(2)
    nt = o.nu_t
    assert np.isfinite(nt).all() and nt.min() >= 0.0
    for j in (0, 1, 2, p.ny, p.ny + 1):
        assert not nt[j].any(), j
    assert nt[3: p.ny].min() > 0.0


def test_laminar_profile_has_no_subgrid_stress():
    """A plane-parallel flow has |S| = 0 once the mean shear is removed
    (les.f:113-160), so NU_T vanishes to round-off and LES reproduces the
    DNS step."""
    _, a = channel_case(1, noise=0.0)
    _, b = channel_case(0, noise=0.0)
    a.step(3)
    b.step(3)
    # |S| is round-off of the O(10) shear, and so is every difference
    assert a.nu_t.max() < 1e-14
    scale = np.abs(b.cu[0]).max()
    for x, y in zip(state(a), state(b)):
        assert np.abs(x - y).max() <= 1e-12 * scale


def test_spin_up_wait_leaves_dns_untouched():
    """With CREATE_NEW_FLOW the subgrid model waits until TIME_STEP > 100
    (channel.f:303): until then NU_T stays zero and the LES terms add exact
    zeros, so the state matches the DNS bit for bit."""
    _, a = channel_case(1, create_new_flow=1)
    _, b = channel_case(0, create_new_flow=1)
    a.step(2)
    b.step(2)
    assert not a.nu_t.any()
    for x, y in zip(state(a), state(b)):
        assert np.array_equal(x, y)


def test_model_switches_on_after_step_100():
    _, a = channel_case(1, create_new_flow=1)
    t, dt, _, _ = a.time()
    a.set_time(t, dt, 100)
    a.step()     # TIME_STEP 101
    assert a.nu_t.max() > 0.0


@pytest.mark.parametrize("neumann_top", [False, True])
def test_subgrid_model_dissipates_fluctuations(neumann_top):
    """The eddy viscosity drains fluctuation energy: after a few steps the
    LES run holds less of it than the DNS from the same state."""
    _, a = channel_case(1, neumann_top=neumann_top)
    _, b = channel_case(0, neumann_top=neumann_top)
    a.step(6)
    b.step(6)

    def fluct(o):
        e = 0.0
        for c in o.cu:
            f = c.copy()
            f[:, 0, 0] = 0.0
            e += float(np.sum(np.abs(f) ** 2))
        return e
    assert all(np.isfinite(x).all() for x in state(a))
    assert fluct(a) < fluct(b)


def test_validate_les_model_types():
    p = P.turbulent_channel(32, 33, 24)
    p.les = 1
    p.les_model_type = 3
    with pytest.raises(ValueError):
        P.validate(p)
    p.les_model_type = 2
    P.validate(p)
    p.les_model_type = 1
    p.v_bc_ymin = 2
    with pytest.raises(ValueError):
        P.validate(p)
    p.v_bc_ymin = 0
    P.validate(p)


# --- dynamic Smagorinsky (LES_MODEL_TYPE 2, written for this library) -------

def kh_dynamic(shift=0.0, seed=5):
    p = P.kelvin_helmholtz(32, 33, 24)
    p.les, p.les_model_type, p.create_new_flow = 1, 2, 0
    P.validate(p)
    g = G.channel_grid(G.uniform_gy(p.ny, -10.0, 10.0))
    u, th = ics.shear_layer(p, g, seed=seed, amp=0.2)
    u[0] += shift
    o = Oracle(p, g, 0.01)
    o.init_from_physical(u, th)
    return p, o


@pytest.mark.parametrize("model", [1, 2])
def test_dynamic_model_rows_sign_and_finite(model):
    p, o = channel_case(1, model=model)
    o.step(2)
    nt = o.nu_t
    assert np.isfinite(nt).all() and nt.min() >= 0.0
    for j in (0, 1, 2, p.ny, p.ny + 1):
        assert not nt[j].any(), j
    assert all(np.isfinite(x).all() for x in state(o))


def test_dynamic_model_differs_from_constant():
    _, a = channel_case(1, model=1)
    _, b = channel_case(1, model=2)
    a.rk_chan_1(1)
    b.rk_chan_1(1)
    assert np.abs(a.nu_t - b.nu_t).max() > 1e-3 * np.abs(a.nu_t).max()


def test_dynamic_coefficient_is_galilean_invariant():
    """A uniform streamwise velocity changes neither the Leonard stress L_ij
    (the test filter keeps constants), the strain rates nor the mean-shear
    removal, so NU_T of the first substage is the same."""
    _, a = kh_dynamic(0.0)
    _, b = kh_dynamic(0.7)
    a.rk_chan_1(1)
    b.rk_chan_1(1)
    na, nb = a.nu_t, b.nu_t
    assert na.max() > 0.0
    assert np.abs(na - nb).max() <= 1e-9 * na.max()


def test_dynamic_model_laminar_profile_has_no_eddy_viscosity():
    _, o = channel_case(1, noise=0.0, model=2)
    o.step(2)
    assert o.nu_t.max() < 1e-14
