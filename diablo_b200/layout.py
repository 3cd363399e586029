"""Host array layouts shared by the Fortran host and the C ABI.

A Fortran COMMON array ``CU1(0:NXP,0:NZ+1,0:NY+1)`` of COMPLEX*16 is, in
numpy's C order, an array of shape ``(NY+2, NZ+2, NXP+1)`` indexed
``[j, k, i]``; the physical array ``U1(0:NX+1,0:NZ+1,0:NY+1)`` of REAL*8 is
``(NY+2, NZ+2, NX+2)``.  Both occupy the same number of bytes, which is what
the reference's EQUIVALENCE (for/header:245-255) relies on; `as_fourier` and
`as_physical` give the two views of one buffer.
"""
from __future__ import annotations

import numpy as np

from .params import DiabloParams


def fourier_shape(p: DiabloParams) -> tuple[int, int, int]:
    return (p.ny + 2, p.nz + 2, p.nx // 2 + 1)


def physical_shape(p: DiabloParams) -> tuple[int, int, int]:
    return (p.ny + 2, p.nz + 2, p.nx + 2)


def new_fourier(p: DiabloParams, count: int | None = None) -> np.ndarray:
    shape = fourier_shape(p) if count is None else (count,) + fourier_shape(p)
    return np.zeros(shape, dtype=np.complex128)


def new_physical(p: DiabloParams, count: int | None = None) -> np.ndarray:
    shape = physical_shape(p) if count is None else (count,) + physical_shape(p)
    return np.zeros(shape, dtype=np.float64)


def as_fourier(p: DiabloParams, buf: np.ndarray) -> np.ndarray:
    """Complex view of a buffer holding one (or, with a leading axis, several) fields."""
    flat = np.ascontiguousarray(buf).view(np.float64).reshape(-1)
    n = 2 * int(np.prod(fourier_shape(p)))
    lead = flat.size // n
    v = flat.view(np.complex128).reshape((lead,) + fourier_shape(p))
    return v if buf.ndim > 3 else v[0]


def as_physical(p: DiabloParams, buf: np.ndarray) -> np.ndarray:
    flat = np.ascontiguousarray(buf).view(np.float64).reshape(-1)
    n = int(np.prod(physical_shape(p)))
    lead = flat.size // n
    v = flat.reshape((lead,) + physical_shape(p))
    return v if buf.ndim > 3 else v[0]


def dealiased(p: DiabloParams, cu: np.ndarray) -> np.ndarray:
    """The block of a Fourier array that every Fourier-space loop of the
    reference visits: I in [0,NKX], K in [0,TNKZ], all planes."""
    return cu[..., : p.tnkz + 1, : p.nkx + 1]
