"""Named synthetic workloads of the channel timestep.

Seeded synthetic fields stand in for any dataset (the reference ships none):

* ``kh``        -- stratified shear layer, 64x65x64, Lx=4pi, Lz=2pi, y uniform
                   on [-10,10], Re=1000, Pr=1, Ri=0.1, dt=0.01 fixed; the BCs
                   of the reference's KH_test/input_chan.dat.
* ``channel``   -- wall-bounded channel at Re_tau=180 scale, 192x129x160,
                   Lx=4pi, Lz=4pi/3, tanh-stretched y (CS=1.75) on [-1,1],
                   no-slip walls, constant pressure gradient, passive scalar
                   Pr=0.71, CFL-adaptive dt.
* ``batched``   -- many independent shear layers of uneven sizes: NX from
                   {64,96,128}, NY from {65,129}, NZ from {32,64,128}, Ri
                   uniform in [0.05,0.3], Re uniform in [500,3000] (nu=1/Re),
                   Pr=1, the ``kh`` domain and BCs, per-instance seeds,
                   FP32-split, dt=0.01 fixed.
* ``precision`` -- the benchmark grid 512x257x384: tanh-stretched y (CS=1.75)
                   on [-1,1]; the shear layer of ``kh`` rescaled to
                   thickness delta=0.1 (U1 = TH = tanh(y/delta), noise
                   1e-3 exp(-(y/delta)^2)), Re = U delta/nu = 1000 (nu=1e-4),
                   RI = Ri/delta = 1, Lx = 0.8 pi and Lz = 0.6 pi (dx = dz),
                   KH boundary conditions, dt = 1e-3 fixed (CFL ~0.2).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import grid as G, ics, params as P


@dataclass
class Workload:
    name: str
    p: P.DiabloParams
    grid: G.ChannelGrid
    dt: float
    ic: str
    ic_kw: dict
    meta: dict

    def initial_fields(self) -> tuple[np.ndarray, np.ndarray]:
        if self.ic == "shear":
            return ics.shear_layer(self.p, self.grid, **self.ic_kw)
        return ics.poiseuille(self.p, self.grid, **self.ic_kw)


def kh(nx: int = 64, ny: int = 65, nz: int = 64, precision: int = P.PREC_FP64, seed: int = 1234) -> Workload:
    p = P.kelvin_helmholtz(nx, ny, nz, precision=precision)
    g = G.channel_grid(G.uniform_gy(ny, -10.0, 10.0))
    return Workload("kh", p, g, 0.01, "shear", dict(seed=seed, amp=1e-3, delta=1.0),
                    dict(nu=p.nu, ri=p.ri[0], pr=p.pr[0], lx=p.lx, lz=p.lz, y="uniform [-10,10]"))


def channel(nx: int = 192, ny: int = 129, nz: int = 160, precision: int = P.PREC_FP64,
            seed: int = 1234) -> Workload:
    p = P.turbulent_channel(nx, ny, nz, re_tau=180.0, precision=precision)
    g = G.channel_grid(G.create_grid(1, ny, 2.0, 1.75))
    return Workload("channel", p, g, 1e-3, "poiseuille", dict(u_center=18.0, seed=seed, noise=0.1),
                    dict(nu=p.nu, re_tau=180.0, pr=p.pr[0], lx=p.lx, lz=p.lz, y="tanh CS=1.75 [-1,1]",
                         variable_dt=True, cfl=p.cfl))


def precision(nx: int = 512, ny: int = 257, nz: int = 384, prec: int = P.PREC_FP32SPLIT,
              seed: int = 1234) -> Workload:
    delta = 0.1
    p = P.kelvin_helmholtz(nx, ny, nz, precision=prec)
    p.nu = 1.0e-4
    p.ri[0] = 1.0
    p.lx, p.ly, p.lz = 0.8 * math.pi, 2.0, 0.6 * math.pi
    g = G.channel_grid(G.create_grid(1, ny, 2.0, 1.75))
    return Workload("precision", p, g, 1.0e-3, "shear", dict(seed=seed, amp=1e-3, delta=delta),
                    dict(nu=p.nu, ri=p.ri[0], pr=p.pr[0], lx=p.lx, lz=p.lz, delta=delta,
                         y="tanh CS=1.75 [-1,1]", dt=1.0e-3))


def batched(n: int = 64, seed: int = 2024, prec: int = P.PREC_FP32SPLIT) -> list[Workload]:
    """n shear-layer instances with sizes, Ri and Re drawn from a seeded
    generator (the instance list is a pure function of n and seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nx = int(rng.choice([64, 96, 128]))
        ny = int(rng.choice([65, 129]))
        nz = int(rng.choice([32, 64, 128]))
        w = kh(nx, ny, nz, precision=prec, seed=seed + 1 + i)
        w.p.ri[0] = float(rng.uniform(0.05, 0.3))
        w.p.nu = 1.0 / float(rng.uniform(500.0, 3000.0))
        w.name = "batched"
        w.meta.update(nu=w.p.nu, ri=w.p.ri[0], grid=(nx, ny, nz))
        out.append(w)
    return out
