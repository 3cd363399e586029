"""GPU parity on the configurations the headline cases do not reach: no
scalar (three fields), four scalars with mixed boundary conditions (seven
fields: the 16-warp column kernel and the chunked product extraction),
radix-3 and radix-5 transform lengths through whole steps, and wall-normal
sizes that select each partition width of the column solve (3, 5, 9 and 17
rows per lane).  Each compares the FP64 GPU path with the oracle after a few
full RK3 steps to the same 1e-10 relative L2 bar as the other parity tests."""
import numpy as np
import pytest

from diablo_b200 import grid as G, ics, params as P
from diablo_b200.channel import Channel
from oracle.oracle import Oracle
from test_gpu_parity import TOL32, TOL64, state_errors

pytestmark = pytest.mark.gpu


def run_pair(p, g, u, th, dt, steps):
    o = Oracle(p, g, dt)
    o.init_from_physical(u, th)
    c = Channel(p, g, dt)
    c.upload([x.copy() for x in o.cu], o.cp.copy(), o.cth.copy())
    with c:
        for _ in range(steps):
            o.step()
            c.step()
            if p.variable_dt:
                assert c.delta_t == pytest.approx(o.time()[1], rel=1e-12)
        return state_errors(p, c, o, scaled=True), state_errors(p, c, o)


def scalar_layers(p, g, seed):
    """Shear layer whose scalars differ from one another: each a tanh of its
    own thickness plus seeded noise."""
    u, th = ics.shear_layer(p, g, seed=seed, amp=1e-2)
    rng = np.random.default_rng(seed + 1)
    y = np.asarray(g.gyf, dtype=np.float64)
    for n in range(p.n_th):
        prof = np.tanh(y[1: p.ny + 1] / (1.0 + 0.5 * n))
        noise = 1e-2 * rng.standard_normal((p.ny, p.nz, p.nx))
        th[n, 1: p.ny + 1, : p.nz, : p.nx] = prof[:, None, None] + noise
    return u, th


def test_no_scalar_channel_variable_dt():
    """N_TH = 0: three fields through products, z-forward and column solve."""
    p = P.turbulent_channel(32, 17, 24, re_tau=180.0)
    p.n_th = 0
    g = G.channel_grid(G.create_grid(1, p.ny, 2.0, 1.75))
    u, th = ics.poiseuille(p, g, u_center=10.0, seed=5, noise=0.1)
    assert th.shape[0] == 0
    err, plain = run_pair(p, g, u, th, 1e-3, 6)
    assert max(err.values()) < TOL64, (err, plain)


def four_scalar_case(nx, ny, nz, precision=P.PREC_FP64):
    """Four scalars with distinct Ri and Pr and every BC kind: Dirichlet at
    both walls with nonzero values, Neumann with nonzero gradient, and mixed."""
    p = P.kelvin_helmholtz(nx, ny, nz, precision=precision)
    p.n_th = 4
    ri = [0.1, 0.05, 0.0, 0.2]
    pr = [1.0, 0.71, 7.0, 2.0]
    bc = [(1, 1, 0.0, 0.0), (0, 0, -1.0, 1.0), (1, 0, 0.02, 1.0), (0, 1, -1.0, -0.01)]
    for n in range(4):
        p.ri[n], p.pr[n] = ri[n], pr[n]
        p.th_bc_ymin[n], p.th_bc_ymax[n], p.th_bc_ymin_c1[n], p.th_bc_ymax_c1[n] = bc[n]
    g = G.channel_grid(G.create_grid(2, ny, 20.0, 1.5))
    u, th = scalar_layers(p, g, seed=11)
    return p, g, u, th


def test_four_scalars_mixed_bcs_radix5():
    """Seven fields, NX=40 and NZ=30 (radix 5 and 3 in both transforms),
    stretched grid."""
    p, g, u, th = four_scalar_case(40, 33, 30)
    err, plain = run_pair(p, g, u, th, 0.02, 5)
    assert max(err.values()) < TOL64, (err, plain)


def test_four_scalars_fp32_split():
    """The FP32-split path with seven fields against the FP64 oracle."""
    p, g, u, th = four_scalar_case(48, 33, 40, precision=P.PREC_FP32SPLIT)
    p64 = p.copy()
    p64.precision = P.PREC_FP64
    o = Oracle(p64, g, 0.02)
    o.init_from_physical(u, th)
    with Channel(p, g, 0.02) as c:
        c.upload([x.copy() for x in o.cu], o.cp.copy(), o.cth.copy())
        o.step(5)
        c.step(5)
        err = state_errors(p, c, o, with_cf=False)       # own norms
        assert max(err.values()) < TOL32, err


@pytest.mark.parametrize("ny,rc", [(129, 5), (257, 9), (513, 17)])
def test_partition_widths(ny, rc):
    """NY+2 rows split over 32 lanes of RC rows each; two scalars so that the
    17-row case still fits the column kernel's shared memory."""
    assert 32 * rc >= ny + 2 > 32 * {5: 3, 9: 5, 17: 9}[rc]
    p = P.kelvin_helmholtz(16, ny, 12)
    p.n_th = 2
    p.ri[1], p.pr[1] = 0.02, 0.5
    p.th_bc_ymin[1], p.th_bc_ymax[1] = 0, 0
    p.th_bc_ymin_c1[1], p.th_bc_ymax_c1[1] = -1.0, 1.0
    g = G.channel_grid(G.create_grid(2, ny, 20.0, 1.5))
    u, th = scalar_layers(p, g, seed=ny)
    err, plain = run_pair(p, g, u, th, 0.02, 3)
    assert max(err.values()) < TOL64, (err, plain)
