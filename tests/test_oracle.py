"""CPU tests of the oracle: transform conventions, reference fixtures and
known-answer tests of the channel timestep (no GPU)."""
import math
import os

import numpy as np
import pytest

from diablo_b200 import grid as G, ics, layout, params as P
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def relerr(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.mark.parametrize("n", [16, 24, 32, 40, 64, 96, 128, 160, 192, 384, 512])
def test_cdft_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    assert np.abs(O.cdft(x, -1) - np.fft.fft(x)).max() < 1e-12 * n
    assert np.abs(O.cdft(x, +1) - np.fft.ifft(x) * n).max() < 1e-12 * n


def test_cdft_rejects_bad_radix():
    with pytest.raises(ValueError):
        O.cdft(np.zeros(14, complex), -1)


def _numpy_fourier(p, v):
    """FFT_XZ_TO_FOURIER by numpy: r2c in x / NX, c2c in z / NZ, truncation
    and kz packing (mpi.f:1493-1539); returns the dealiased block."""
    nx, nz = p.nx, p.nz
    phys = v[:, :nz, :nx]
    a = np.fft.rfft(phys, axis=2) / nx
    a = np.fft.fft(a, axis=1) / nz
    out = np.zeros((v.shape[0], p.tnkz + 1, p.nkx + 1), complex)
    out[:, : p.nkz + 1] = a[:, : p.nkz + 1, : p.nkx + 1]
    for k in range(1, p.nkz + 1):
        out[:, p.nkz + k] = a[:, nz - 1 + k - p.nkz, : p.nkx + 1]
    return out


@pytest.mark.parametrize("dims", [(32, 9, 24), (48, 7, 40), (64, 5, 96)])
def test_fft_xz_conventions_vs_numpy(dims):
    nx, ny, nz = dims
    p = P.kelvin_helmholtz(nx, ny, nz)
    g = G.channel_grid(G.uniform_gy(ny, -1.0, 1.0))
    o = O.Oracle(p, g, 0.01)
    rng = np.random.default_rng(1)
    v = layout.new_physical(p)
    v[:, :nz, :nx] = rng.standard_normal((ny + 2, nz, nx))
    vv = layout.new_fourier(p)
    buf = v.copy()
    o.fft_xz_to_fourier(buf, vv, 0, ny + 1)
    ref = _numpy_fourier(p, v)
    assert relerr(layout.dealiased(p, vv), ref) < 1e-14
    # modes above NKX are zero, the x-Nyquist column too
    assert np.all(vv[:, : p.tnkz + 1, p.nkx + 1:] == 0)
    # inverse: the dealiased (filtered) field
    back = layout.new_physical(p)
    o.fft_xz_to_physical(vv.copy(), back, 0, ny + 1)
    full = np.zeros((ny + 2, nz, nx // 2 + 1), complex)
    full[:, : p.nkz + 1, : p.nkx + 1] = ref[:, : p.nkz + 1]
    for k in range(1, p.nkz + 1):
        full[:, nz - 1 + k - p.nkz, : p.nkx + 1] = ref[:, p.nkz + k]
    filt = np.fft.irfft(np.fft.ifft(full, axis=1) * nz, n=nx, axis=2) * nx
    assert np.abs(back[:, :nz, :nx] - filt).max() < 1e-12


def test_single_mode_coefficients():
    p = P.kelvin_helmholtz(48, 5, 36)
    g = G.channel_grid(G.uniform_gy(p.ny, -1.0, 1.0))
    o = O.Oracle(p, g, 0.01)
    x = np.arange(p.nx) * p.lx / p.nx
    z = np.arange(p.nz) * p.lz / p.nz
    a, b = 3, -5
    v = layout.new_physical(p)
    v[:, : p.nz, : p.nx] = np.cos(2 * np.pi * a * x[None, :] / p.lx + 2 * np.pi * b * z[:, None] / p.lz)
    vv = layout.new_fourier(p)
    o.fft_xz_to_fourier(v.copy(), vv, 0, p.ny + 1)
    m = p.tnkz + 1 + b  # packed slot of kz = b < 0
    blk = layout.dealiased(p, vv)
    expect = np.zeros_like(blk)
    expect[:, m, a] = 0.5
    assert np.abs(blk - expect).max() < 1e-14


def test_grid_generator_reproduces_reference_grid_h5():
    """KH_test/grid.h5 of the reference = create_grid_h5.m type 2, L=20, CS=1.5."""
    gy_ref = np.loadtxt(os.path.join(GOLDEN, "kh_grid_y.txt"))
    gy = G.create_grid(2, 65, 20.0, 1.5)
    assert np.abs(gy - gy_ref).max() < 1e-13
    cg = G.channel_grid(gy_ref)
    assert abs(cg.gyf[1] + 10.0) < 1e-12 and abs(cg.gyf[65] - 10.0) < 1e-12
    assert cg.gy[0] == 0.0 and cg.dyf[66] == cg.dyf[65]


def test_uniform_grid_walls():
    cg = G.channel_grid(G.uniform_gy(65, -10.0, 10.0))
    assert abs(cg.gyf[1] + 10) < 1e-12 and abs(cg.gyf[65] - 10) < 1e-12
    assert np.allclose(cg.dy[1:66], 20.0 / 64) and np.allclose(cg.dyf[1:66], 20.0 / 64)


def test_input_file_parsers_on_reference_kh_files():
    p = P.DiabloParams()
    p.nx, p.ny, p.nz, p.n_th = 128, 65, 16, 1
    ctl = P.RunControl()
    P.read_input_dat(open(os.path.join(GOLDEN, "KH_test_input.dat")).read(), p, ctl)
    P.read_input_chan_dat(open(os.path.join(GOLDEN, "KH_test_input_chan.dat")).read(), p, ctl)
    assert (p.nu, p.beta, p.lx, p.ly, p.lz) == (0.001, 1.0, 30.0, 20.0, 4.0)
    assert p.variable_dt == 1 and p.cfl == 0.5 and p.update_dt == 1
    assert ctl.n_time_steps == 5000 and ctl.delta_t == 0.1 and ctl.save_stats_int == 20
    assert p.ri[0] == 0.15 and p.pr[0] == 1.0
    assert ctl.ic_type == 3 and ctl.kick == 0.1
    assert (p.grav_x, p.grav_y, p.grav_z) == (0.0, 1.0, 0.0)
    assert p.f_type == 3 and p.px0 == -1.0
    assert (p.u_bc_ymin, p.v_bc_ymin, p.w_bc_ymin, p.u_bc_ymax, p.v_bc_ymax, p.w_bc_ymax) == (1, 0, 1, 1, 0, 1)
    assert p.th_bc_ymin[0] == 1 and p.th_bc_ymax[0] == 1
    assert p.les_model_type == 1
    P.validate(p)


def test_validate_rejects_bad_parameters():
    p = P.kelvin_helmholtz(28, 17, 16)
    with pytest.raises(ValueError):
        P.validate(p)
    p = P.kelvin_helmholtz(32, 3, 16)
    with pytest.raises(ValueError):
        P.validate(p)


def _divergence(o):
    p, g = o.p, o.grid
    kx = np.arange(p.nkx + 1) * 2 * np.pi / p.lx
    kz = np.zeros(p.tnkz + 1)
    kz[: p.nkz + 1] = np.arange(p.nkz + 1) * 2 * np.pi / p.lz
    for k in range(1, p.nkz + 1):
        kz[p.tnkz + 1 - k] = -k * 2 * np.pi / p.lz
    cu = [layout.dealiased(p, c) for c in o.cu]
    worst = 0.0
    for j in range(2, p.ny):
        d = 1j * kx[None, :] * cu[0][j] + (cu[1][j + 1] - cu[1][j]) / g.dyf[j] + 1j * kz[:, None] * cu[2][j]
        worst = max(worst, np.abs(d).max())
    return worst


def test_rem_div_leaves_discrete_divergence_free_field():
    p = P.kelvin_helmholtz(32, 25, 24)
    g = G.channel_grid(G.create_grid(2, 25, 20.0, 1.5))
    o = O.Oracle(p, g, 0.01)
    u, th = ics.shear_layer(p, g, seed=5, amp=0.1)
    o.init_from_physical(u, th)
    scale = max(np.abs(c).max() for c in o.cu)
    assert _divergence(o) < 1e-12 * scale
    o.step(2)
    assert _divergence(o) < 1e-12 * scale


def test_couette_is_steady():
    p = P.kelvin_helmholtz(16, 17, 16)
    p.u_bc_ymin, p.u_bc_ymax = 0, 0
    p.u_bc_ymin_c1, p.u_bc_ymax_c1 = -1.0, 1.0
    p.ri[0] = 0.0
    g = G.channel_grid(G.create_grid(1, 17, 2.0, 1.75))
    o = O.Oracle(p, g, 0.01)
    u = layout.new_physical(p, 3)
    th = layout.new_physical(p, 1)
    u[0, : p.ny + 1, : p.nz, : p.nx] = g.gyf[: p.ny + 1, None, None]
    o.init_from_physical(u, th)
    before = o.cu[0][:, 0, 0].real.copy()
    o.step(5)
    after = o.cu[0][:, 0, 0].real
    assert np.abs(after[1: p.ny + 1] - g.gyf[1: p.ny + 1]).max() < 1e-12
    assert np.abs(after[1: p.ny + 1] - before[1: p.ny + 1]).max() < 1e-12


def test_poiseuille_is_steady_on_uniform_grid():
    p = P.turbulent_channel(16, 17, 16, variable_dt=False)
    p.n_th = 0
    uc = 2.0
    p.px0 = -2.0 * p.nu * uc
    g = G.channel_grid(G.uniform_gy(p.ny, -1.0, 1.0))
    o = O.Oracle(p, g, 0.01)
    u = layout.new_physical(p, 3)
    u[0, : p.ny + 1, : p.nz, : p.nx] = (uc * (1 - g.gyf[: p.ny + 1] ** 2))[:, None, None]
    o.init_from_physical(u, layout.new_physical(p, 1))
    o.step(5)
    prof = o.cu[0][1: p.ny + 1, 0, 0].real
    assert np.abs(prof - uc * (1 - g.gyf[1: p.ny + 1] ** 2)).max() < 1e-11


def test_horizontal_diffusion_matches_rk3_amplification():
    """A y-independent scalar mode cos(2 pi x/Lx) decays by the discrete
    low-storage RK3 factor of channel.f:175-189 / 581-595."""
    p = P.kelvin_helmholtz(16, 9, 16)
    p.ri[0] = 0.0
    p.nu = 0.05
    g = G.channel_grid(G.uniform_gy(p.ny, -1.0, 1.0))
    dt = 0.02
    o = O.Oracle(p, g, dt)
    th = layout.new_physical(p, 1)
    x = np.arange(p.nx) * p.lx / p.nx
    th[0, :, : p.nz, : p.nx] = np.cos(2 * np.pi * x / p.lx)[None, None, :]
    o.init_from_physical(layout.new_physical(p, 3), th)
    c0 = o.cth[0][4, 0, 1].real
    lam = (p.nu / p.pr[0]) * (2 * np.pi / p.lx) ** 2
    hb = [dt * 8 / 15, dt * 2 / 15, dt * 5 / 15]
    be, ze = [1.0, 25 / 8, 9 / 4], [0.0, -17 / 8, -5 / 4]
    th_, fold = c0, 0.0
    nsteps = 4
    for _ in range(nsteps):
        for r in range(3):
            fnew = -lam * th_
            th_ = th_ + ze[r] * hb[r] * fold + be[r] * hb[r] * fnew
            fold = fnew
    o.step(nsteps)
    assert abs(o.cth[0][4, 0, 1].real - th_) < 1e-13
    assert abs(o.cth[0][4, 0, 1].real - c0 * math.exp(-lam * dt * nsteps)) < 1e-6


def test_oracle_matches_committed_regression_vectors():
    ref = np.load(os.path.join(GOLDEN, "oracle_kh_small.npz"))
    p = P.kelvin_helmholtz(24, 17, 16)
    g = G.channel_grid(G.uniform_gy(p.ny, -10.0, 10.0))
    o = O.Oracle(p, g, 0.05)
    o.init_from_physical(ref["u"], ref["th"])
    for c in range(3):
        assert relerr(layout.dealiased(p, o.cu[c]), ref[f"init_cu{c}"]) < 1e-13
    o.step(3)
    for c in range(3):
        assert relerr(layout.dealiased(p, o.cu[c]), ref[f"cu{c}"]) < 1e-12
    assert relerr(layout.dealiased(p, o.cth), ref["cth"]) < 1e-12
    assert relerr(layout.dealiased(p, o.cp), ref["cp"]) < 1e-12
    st = o.stats()
    assert np.allclose(st, ref["stats"], rtol=1e-10, atol=1e-14)


def test_courant_limits():
    p = P.turbulent_channel(16, 17, 16)
    g = G.channel_grid(G.create_grid(1, 17, 2.0, 1.75))
    o = O.Oracle(p, g, 0.01)
    u = layout.new_physical(p, 3)
    u[0, :, : p.nz, : p.nx] = 2.0
    o.raw(O.ORC_U1)[:] = u[0].reshape(-1)
    o.raw(O.ORC_U2)[:] = 0.0
    o.raw(O.ORC_U3)[:] = 0.0
    o.courant()
    _, dt, _, hb = o.time()
    dx = p.lx / p.nx
    lim = 0.5 * min(dx, g.dy[1]) ** 2 / p.nu
    lim = min(lim, lim * p.pr[0])
    assert dt == pytest.approx(min(lim, p.cfl * dx / 2.0), rel=1e-15)
    assert hb[0] == pytest.approx(dt * 8 / 15)
