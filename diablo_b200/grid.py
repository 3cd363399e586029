"""Wall-normal (y) grid of the channel solver.

* `create_grid` restates the reference's grid generator
  (pre_process/create_grid_h5.m:30-79): G on j=0..N with one of three
  stretching functions, GF halfway between, both rescaled and shifted so that
  GF(1) and GF(N) sit on the walls; it returns the N+1 values the script
  writes to grid.h5:/grids/y.
* `channel_grid` turns those N+1 values into the /GRID_PARAMS/ arrays exactly
  as ReadGridHDF5 (for/hdf5.f:548-710) and CREATE_GRID_CHAN
  (for/channel.f:1646-1652) do: GY(1..NY+1) from the file, GYF at midpoints,
  extrapolated GYF ghosts, DY and DYF.  GY(0) is never assigned on that path
  and stays 0, as in the reference's COMMON block.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def create_grid(grid_type: int, n: int, length: float, cs: float) -> np.ndarray:
    """The N+1 GY values of create_grid_h5.m for GRID_TYPE 1, 2 or 3."""
    g = np.zeros(n + 3)
    gf = np.zeros(n + 3)
    for jj in range(1, n + 2):
        x = (2.0 * (jj - 1)) / n - 1.0
        if grid_type == 1:
            g[jj + 1] = (length / 2.0) * np.tanh(cs * x) / np.tanh(cs)
        elif grid_type == 2:
            g[jj + 1] = (length / 2.0) * (cs * x ** 3 + x) / (cs + 1)
        elif grid_type == 3:
            g[jj + 1] = (length / 2.0) * np.tanh(cs * x) / np.tanh(cs) + length / 2.0
        else:
            raise ValueError("grid type must be 1, 2 or 3")
    for jj in range(1, n + 1):
        gf[jj + 1] = (g[jj + 1] + g[jj + 2]) / 2.0
    gf_lower, gf_upper, g_lower, g_upper = gf[2], gf[n + 1], g[2], g[n + 2]
    for jj in range(1, n + 1):
        gf[jj + 1] = gf[jj + 1] * (g_upper - g_lower) / (gf_upper - gf_lower)
    for jj in range(1, n + 2):
        g[jj + 1] = g[jj + 1] * (g_upper - g_lower) / (gf_upper - gf_lower)
    gf_lower = gf[2]
    shift = g_lower - gf_lower
    for jj in range(1, n + 1):
        gf[jj + 1] = gf[jj + 1] + shift
    for jj in range(1, n + 2):
        g[jj + 1] = g[jj + 1] + shift
    return g[2:n + 3].copy()


def uniform_gy(ny: int, ymin: float, ymax: float) -> np.ndarray:
    """N+1 GY values of a uniform grid whose GYF(1), GYF(NY) are the walls."""
    d = (ymax - ymin) / (ny - 1)
    return ymin - 0.5 * d + d * np.arange(ny + 1, dtype=np.float64)


@dataclass
class ChannelGrid:
    gy: np.ndarray    # GY(0:NY+1)
    gyf: np.ndarray   # GYF(0:NY+1)
    dy: np.ndarray    # DY(0:NY+1)
    dyf: np.ndarray   # DYF(0:NY+1)

    @property
    def ny(self) -> int:
        return self.gy.shape[0] - 2


def channel_grid(gy_file: np.ndarray) -> ChannelGrid:
    """/GRID_PARAMS/ from the NY+1 values stored in grid.h5:/grids/y."""
    gy_file = np.asarray(gy_file, dtype=np.float64)
    ny = gy_file.shape[0] - 1
    gy = np.zeros(ny + 2)
    gyf = np.zeros(ny + 2)
    gy[1:ny + 2] = gy_file
    for j in range(1, ny + 1):
        gyf[j] = 0.5 * (gy[j] + gy[j + 1])
    gyf[0] = 2.0 * gyf[1] - gyf[2]
    gyf[ny + 1] = 2.0 * gyf[ny] - gyf[ny - 1]
    dy = np.zeros(ny + 2)
    dyf = np.zeros(ny + 2)
    for j in range(1, ny + 2):
        dy[j] = gyf[j] - gyf[j - 1]
    for j in range(1, ny + 1):
        dyf[j] = gy[j + 1] - gy[j]
    dyf[ny + 1] = dyf[ny]
    return ChannelGrid(gy=gy, gyf=gyf, dy=dy, dyf=dyf)
