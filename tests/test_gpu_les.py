"""GPU parity of the LES branch against the oracle, for the constant
Smagorinsky model (LES_MODEL_TYPE 1) and this library's dynamic model (2): the
state after several RK3 steps and the eddy viscosity NU_T, through the
C ABI, to the FP64 bar of the other parity tests (1e-10 relative L2, the
small velocity components and the pressure measured against the velocity
and pressure scales)."""
import ctypes

import numpy as np
import pytest

from diablo_b200 import grid as G, ics, params as P
from diablo_b200.channel import Batch, Channel, DiabloError, DIABLO_ENOTSUP, load_library
from oracle.oracle import Oracle
from test_gpu_parity import TOL64, relerr, state_errors

pytestmark = pytest.mark.gpu


def les_channel(nx=32, ny=33, nz=24, n_th=1, neumann_top=False, variable_dt=False, create_new_flow=0, model=1):
    p = P.turbulent_channel(nx, ny, nz, re_tau=180.0, variable_dt=variable_dt)
    p.les, p.les_model_type, p.create_new_flow = 1, model, create_new_flow
    p.n_th = n_th
    for n in range(1, n_th):
        p.pr[n], p.ri[n] = 1.0 + n, 0.0
        p.th_bc_ymin[n], p.th_bc_ymax[n] = 1, 0      # Neumann bottom: JSTART_TH = 1
        p.th_bc_ymin_c1[n], p.th_bc_ymax_c1[n] = 0.5, 1.0
    if neumann_top:
        p.u_bc_ymax = p.w_bc_ymax = 1
        p.u_bc_ymax_c1, p.w_bc_ymax_c1 = 0.1, -0.05
    g = G.channel_grid(G.create_grid(1, p.ny, 2.0, 1.75))
    u, th = ics.poiseuille(p, g, u_center=10.0, seed=3, noise=0.5)
    if n_th > 1:
        th[1:] = th[:1] * 0.5 + 0.1
    return p, g, u, th


def run(p, g, u, th, dt, steps, start_step=0):
    o = Oracle(p, g, dt)
    o.init_from_physical(u, th)
    c = Channel(p, g, dt)
    c.upload([x.copy() for x in o.cu], o.cp.copy(), o.cth.copy())
    if start_step:
        t, d, _, _ = o.time()
        o.set_time(t, d, start_step)
        c.time_step = start_step
    with c:
        for _ in range(steps):
            o.step()
            c.step()
            if p.variable_dt:
                assert c.delta_t == pytest.approx(o.time()[1], rel=1e-12)
        err = state_errors(p, c, o, scaled=True)
        plain = state_errors(p, c, o)
        nut = relerr(c.download_nu_t(), o.nu_t)
    return err, plain, nut, o


@pytest.mark.parametrize("model", [1, 2])
def test_les_channel_dirichlet(model):
    """Closed channel, no-slip walls, one scalar: 4 steps with the model on."""
    p, g, u, th = les_channel(model=model)
    err, plain, nut, o = run(p, g, u, th, 2e-4, 4)
    assert o.nu_t.max() > 0.0
    assert nut < TOL64, nut
    assert max(err.values()) < TOL64, (err, plain)


@pytest.mark.parametrize("model", [1, 2])
def test_les_neumann_top_two_scalars_variable_dt(model):
    """Stress-free upper wall (APPLY_BC_LES rewrites row NY), a second scalar
    with a Neumann lower wall (JSTART_TH = 1), CFL-adaptive dt, radix-3 x;
    NX = 48 is not a multiple of the dynamic model's 32-point tiles."""
    p, g, u, th = les_channel(nx=48, ny=33, nz=24, n_th=2, neumann_top=True, variable_dt=True, model=model)
    err, plain, nut, _ = run(p, g, u, th, 2e-4, 3)
    assert nut < TOL64, nut
    assert max(err.values()) < TOL64, (err, plain)


def test_les_spin_up_switch():
    """CREATE_NEW_FLOW: step 100 runs without the model, 101 and 102 with it."""
    p, g, u, th = les_channel(create_new_flow=1)
    err, plain, nut, o = run(p, g, u, th, 2e-4, 3, start_step=99)
    assert o.nu_t.max() > 0.0
    assert nut < TOL64, nut
    assert max(err.values()) < TOL64, (err, plain)


def test_les_rejected_configurations():
    p, g, _, _ = les_channel()
    q = p.copy()
    q.les_model_type = 3     # the reference stops here too (les.f:269-272)
    L = load_library()
    h = ctypes.c_void_p()
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (g.gy, g.gyf, g.dy, g.dyf)]
    ptr = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert L.diablo_gpu_create(ctypes.byref(q), *[ptr(a) for a in arrs], ctypes.byref(h)) == DIABLO_ENOTSUP
    q = p.copy()
    q.precision = P.PREC_FP32SPLIT
    with pytest.raises(DiabloError) as e:
        Channel(q, g, 2e-4)
    assert e.value.code == DIABLO_ENOTSUP
    with Channel(p, g, 2e-4) as c:
        with pytest.raises(DiabloError) as e:
            Batch([c])
        assert e.value.code == DIABLO_ENOTSUP


# --- the learned closure (LES_MODEL_TYPE 4) ----------------------------------

def closure_params(seed=21, out=1e-3):
    """A seeded network whose inputs are normalised by the features' typical
    sizes (the gradients enter divided by their norm) and whose
    dimensionless stresses are O(out)."""
    from diablo_b200 import mlp as ML
    mean = np.zeros(11)
    scale = np.concatenate([np.full(9, 0.3), [60.0, 0.1]])
    return ML.init_params(seed, mean, scale, np.full(6, out))


def run_closure(p, g, u, th, dt, steps, params):
    from diablo_b200.mlp import SgsMlp
    o = Oracle(p, g, dt)
    o.init_from_physical(u, th)
    if params is not None:
        o.set_mlp(params)
    c = Channel(p, g, dt)
    c.upload([x.copy() for x in o.cu], o.cp.copy(), o.cth.copy())
    m = SgsMlp(params) if params is not None else None
    with c:
        if m is not None:
            c.set_sgs_mlp(m)
        for _ in range(steps):
            o.step()
            c.step()
        err = state_errors(p, c, o, scaled=True)
        plain = state_errors(p, c, o)
        s = c.download()
    if m is not None:
        m.close()
    return err, plain, s, o


def test_learned_closure_matches_oracle():
    """Closure stresses from the same BF16 network on both sides (the
    oracle rounds weights, inputs and activations to bfloat16 as the tensor
    cores do, and accumulates in FP64 where the GPU uses FP32).  After 3
    steps the velocity agrees to 1e-9; CF and CP, which carry the stresses
    directly (CP through phi/h), to 5e-7 -- the size of the few activations
    that round to different bfloat16 neighbours -- while the closure itself
    changes CF by far more than that."""
    p, g, u, th = les_channel(model=4)
    err, plain, s, o = run_closure(p, g, u, th, 2e-4, 3, closure_params())
    for k in ("cu1", "cu2", "cu3", "cth1"):
        assert err[k] < 1e-9, (err, plain)
    assert max(err.values()) < 5e-7, (err, plain)
    # the closure's own effect, from the run without any model
    q = p.copy()
    q.les = 0
    o0 = Oracle(q, g, 2e-4)
    o0.init_from_physical(u, th)
    o0.step(3)
    effect = max(relerr(o.cf[c][2:p.ny + 1], o0.cf[c][2:p.ny + 1]) for c in range(3))
    assert effect > 200 * max(err[k] for k in ("cf1", "cf2", "cf3")), (effect, err)


def test_learned_closure_falls_back_to_dynamic_model():
    p, g, u, th = les_channel(model=4)
    err, plain, _, _ = run_closure(p, g, u, th, 2e-4, 3, None)
    assert max(err.values()) < TOL64, (err, plain)
