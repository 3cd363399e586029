"""Seeded synthetic initial fields (physical space, Fortran layout).

The reference's CREATE_FLOW_CHAN (for/set_ics.f:2-200) draws uniform KICK
noise from the compiler's RANDOM_NUMBER with seed RANK+k+999; that stream is
compiler-specific, so runs here use this project's own portable generator
instead: splitmix64 -> 53-bit uniforms -> Box-Muller normals, fully
determined by the seed and the array shape.  Profiles follow IC_TYPE 0 and 3
of set_ics.f (laminar Poiseuille, tanh shear layer) and CREATE_TH_CHAN
(set_ics.f:204-273).
"""
from __future__ import annotations

import numpy as np

from .grid import ChannelGrid
from .layout import new_physical
from .params import DiabloParams

_MASK = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(seed: int, n: int) -> np.ndarray:
    """n consecutive outputs of splitmix64 started at `seed`."""
    with np.errstate(over="ignore"):
        idx = np.arange(1, n + 1, dtype=np.uint64)
        z = (np.uint64(seed) + idx * np.uint64(0x9E3779B97F4A7C15)) & _MASK
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _MASK
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _MASK
        z = z ^ (z >> np.uint64(31))
    return z


def normals(seed: int, n: int) -> np.ndarray:
    """n standard normal deviates (Box-Muller on splitmix64 uniforms)."""
    m = (n + 1) // 2
    bits = splitmix64(seed, 2 * m)
    u = ((bits >> np.uint64(11)).astype(np.float64) + 0.5) * (1.0 / 9007199254740992.0)
    u1, u2 = u[0::2], u[1::2]
    r = np.sqrt(-2.0 * np.log(u1))
    z = np.empty(2 * m)
    z[0::2] = r * np.cos(2.0 * np.pi * u2)
    z[1::2] = r * np.sin(2.0 * np.pi * u2)
    return z[:n]


def shear_layer(p: DiabloParams, grid: ChannelGrid, seed: int = 1234, amp: float = 1e-3,
                delta: float = 1.0) -> tuple[np.ndarray, np.ndarray]:
    """U1 = tanh(y/delta), U2 = U3 = 0 on J=0..NY and TH = tanh(y/delta) on
    J=1..NY (IC_TYPE 3), plus amp*exp(-(y/delta)^2)*N(0,1) on the three
    velocity components on J=0..NY+1.  Returns (u[3], th[N_TH]) physical."""
    u = new_physical(p, 3)
    th = new_physical(p, max(p.n_th, 1))
    nx, nz, ny = p.nx, p.nz, p.ny
    y = grid.gyf / delta
    u[0, : ny + 1, :nz, :nx] = np.tanh(y[: ny + 1])[:, None, None]
    env = np.exp(-(y ** 2))[:, None, None]
    for c in range(3):
        z = normals(seed + 7919 * c, (ny + 2) * nz * nx).reshape(ny + 2, nz, nx)
        u[c, :, :nz, :nx] += amp * env * z
    for n in range(p.n_th):
        th[n, 1: ny + 1, :nz, :nx] = np.tanh(y[1: ny + 1])[:, None, None]
    return u, th[: p.n_th]


def poiseuille(p: DiabloParams, grid: ChannelGrid, u_center: float, seed: int = 1234,
               noise: float = 0.1) -> tuple[np.ndarray, np.ndarray]:
    """U1 = u_center*(1-GYF^2) (IC_TYPE 0 with UBULK0 = 2/3 u_center) on
    J=0..NY plus noise*u_center*N(0,1)*(1-GYF^2) on all components (the
    projection that follows makes it divergence-free); TH linear between the
    wall values (IC_TYPE 1/2 form of CREATE_TH_CHAN)."""
    u = new_physical(p, 3)
    th = new_physical(p, max(p.n_th, 1))
    nx, nz, ny = p.nx, p.nz, p.ny
    y = grid.gyf
    u[0, : ny + 1, :nz, :nx] = (u_center * (1.0 - y[: ny + 1] ** 2))[:, None, None]
    env = np.clip(1.0 - y ** 2, 0.0, None)[:, None, None]
    for c in range(3):
        z = normals(seed + 7919 * c, (ny + 2) * nz * nx).reshape(ny + 2, nz, nx)
        u[c, :, :nz, :nx] += noise * u_center * env * z
    for n in range(p.n_th):
        lo, hi = p.th_bc_ymin_c1[n], p.th_bc_ymax_c1[n]
        prof = (hi - lo) * (y[1: ny + 1] + 1.0) / 2.0 + lo
        th[n, 1: ny + 1, :nz, :nx] = prof[:, None, None]
    return u, th[: p.n_th]


def tripped_poiseuille(p: DiabloParams, grid: ChannelGrid, u_center: float, seed: int = 1234,
                       amp: float = 0.3, kx_max: int = 3, kz_max: int = 6) -> tuple[np.ndarray, np.ndarray]:
    """The Poiseuille field of `poiseuille` without its white noise, plus a
    large-scale perturbation that trips a channel to turbulence: seeded
    normals low-pass filtered to |kx| <= kx_max, |kz| <= kz_max, scaled to
    unit RMS over planes 1..NY and then by amp*u_center*(1-GYF^2), on every
    component (the projection that follows makes it divergence-free).  White
    noise of the same amplitude decays before the flow transitions; this one
    gives a Re_tau 180 channel its turbulent statistics after about 25 time
    units."""
    u, th = poiseuille(p, grid, u_center, seed=seed, noise=0.0)
    nx, nz, ny = p.nx, p.nz, p.ny
    env = np.clip(1.0 - grid.gyf ** 2, 0.0, None)[:, None, None]
    kz = np.abs(np.fft.fftfreq(nz, 1.0 / nz))[:, None]
    keep = (kz <= kz_max) & (np.arange(nx // 2 + 1)[None, :] <= kx_max)
    for c in range(3):
        r = normals(seed + 104729 * (c + 1), (ny + 2) * nz * nx).reshape(ny + 2, nz, nx)
        lp = np.fft.irfft2(np.fft.rfft2(r, axes=(1, 2)) * keep[None], s=(nz, nx), axes=(1, 2))
        lp /= lp[1: ny + 1].std()
        u[c, :, :nz, :nx] += amp * u_center * env * lp
    return u, th
