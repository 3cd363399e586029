"""ctypes binding of the CPU FP64 oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by the cpu_baseline / reference legs of bench.py, where it is the checker or
the timed CPU baseline -- never by the diablo_b200 package.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from diablo_b200.grid import ChannelGrid
from diablo_b200.layout import as_fourier, as_physical, fourier_shape, physical_shape
from diablo_b200.params import DiabloParams

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")

(ORC_U1, ORC_U2, ORC_U3, ORC_P, ORC_R1, ORC_R2, ORC_R3, ORC_F1, ORC_F2, ORC_F3, ORC_S1,
 ORC_TH, ORC_CTH, ORC_FTH, ORC_CFTH, ORC_RTH, ORC_CRTH,
 ORC_GY, ORC_GYF, ORC_DY, ORC_DYF, ORC_KX, ORC_KZ, ORC_NU_T) = range(24)


USER_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p)


def build() -> str:
    """Compile liboracle.so with the committed Makefile if it is missing or stale."""
    src = [os.path.join(_HERE, f) for f in ("diablo_oracle.c", "diablo_oracle.h", "Makefile")]
    if not os.path.exists(_LIB) or any(os.path.getmtime(f) > os.path.getmtime(_LIB) for f in src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB)
        vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int
        L.orc_create.restype = vp
        L.orc_create.argtypes = [ctypes.POINTER(DiabloParams), dp, dp, ctypes.c_double]
        L.orc_destroy.argtypes = [vp]
        L.orc_array.restype = dp
        L.orc_array.argtypes = [vp, ip]
        L.orc_array_doubles.restype = ctypes.c_size_t
        L.orc_array_doubles.argtypes = [vp, ip]
        L.orc_get_time.argtypes = [vp, dp, dp, ctypes.POINTER(ctypes.c_int), dp]
        L.orc_set_time.argtypes = [vp, ctypes.c_double, ctypes.c_double, ip]
        L.orc_set_threads.argtypes = [ip]
        L.orc_filter_chan.argtypes = [vp, ip]
        for name in ("orc_fft_xz_to_fourier", "orc_fft_xz_to_physical"):
            getattr(L, name).argtypes = [vp, dp, dp, ip, ip]
        L.orc_rk_chan_1.argtypes = [vp, ip]
        for name in ("orc_rem_div_chan", "orc_poisson_p_chan", "orc_courant", "orc_apply_bc_vel",
                     "orc_apply_bc_scalar", "orc_step"):
            getattr(L, name).argtypes = [vp]
        L.orc_stats.argtypes = [vp, dp]
        L.orc_mean_stats.argtypes = [vp, dp, dp, dp]
        L.orc_set_user_rhs.argtypes = [vp, ip, USER_FN, vp]
        L.orc_epsilon_sgs.argtypes = [vp, dp]
        L.orc_epsilon_field.argtypes = [vp, dp]
        L.orc_set_mlp.argtypes = [vp, ctypes.POINTER(ctypes.c_float)]
        L.orc_cdft.restype = ip
        L.orc_cdft.argtypes = [ip, dp, ip]
        _lib = L
    return _lib


def _dptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def cdft(x: np.ndarray, sign: int) -> np.ndarray:
    """Complex DFT of the oracle's transform kernel (unnormalised)."""
    y = np.ascontiguousarray(x, dtype=np.complex128).copy()
    if lib().orc_cdft(y.shape[0], _dptr(y.view(np.float64)), sign) != 0:
        raise ValueError("length must be a product of 2, 3 and 5")
    return y


def set_threads(n: int) -> None:
    lib().orc_set_threads(n)


class Oracle:
    """The reference's channel state and routines, restated on the CPU."""

    def __init__(self, p: DiabloParams, grid: ChannelGrid, delta_t: float):
        self.p = p.copy()
        self.grid = grid
        L = lib()
        gy = np.ascontiguousarray(grid.gy, dtype=np.float64)
        gyf = np.ascontiguousarray(grid.gyf, dtype=np.float64)
        self._h = L.orc_create(ctypes.byref(self.p), _dptr(gy), _dptr(gyf), float(delta_t))
        if not self._h:
            raise ValueError("oracle: NX and NZ must be products of 2, 3 and 5")

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    # --- raw arrays -------------------------------------------------------
    def raw(self, which: int) -> np.ndarray:
        L = lib()
        n = L.orc_array_doubles(self._h, which)
        ptr = L.orc_array(self._h, which)
        return np.ctypeslib.as_array(ptr, shape=(n,))

    def fourier(self, which: int, n: int | None = None) -> np.ndarray:
        v = as_fourier(self.p, self.raw(which).reshape((-1,) + fourier_shape(self.p)))
        return v if n is None else v[n]

    def physical(self, which: int, n: int | None = None) -> np.ndarray:
        v = as_physical(self.p, self.raw(which).reshape((-1,) + physical_shape(self.p)))
        return v if n is None else v[n]

    @property
    def cu(self) -> list[np.ndarray]:
        return [self.fourier(ORC_U1, 0), self.fourier(ORC_U2, 0), self.fourier(ORC_U3, 0)]

    @property
    def cp(self) -> np.ndarray:
        return self.fourier(ORC_P, 0)

    @property
    def cth(self) -> np.ndarray:
        return self.fourier(ORC_CTH)[: self.p.n_th]

    @property
    def cf(self) -> list[np.ndarray]:
        return [self.fourier(ORC_F1, 0), self.fourier(ORC_F2, 0), self.fourier(ORC_F3, 0)]

    @property
    def cfth(self) -> np.ndarray:
        return self.fourier(ORC_CFTH)[: self.p.n_th]

    @property
    def nu_t(self) -> np.ndarray:
        """NU_T(0:NX-1, 0:NZ-1, 0:NY+1) at GY points, as [J][K][I] (LES only)."""
        if not self.p.les:
            raise ValueError("NU_T exists only when LES is set")
        return self.physical(ORC_NU_T, 0)[:, : self.p.nz, : self.p.nx]

    @property
    def phi(self) -> np.ndarray:
        """CR1, where REM_DIV_CHAN leaves phi (channel.f:1196-1199)."""
        return self.fourier(ORC_R1, 0)

    # --- time ---------------------------------------------------------------
    def time(self) -> tuple[float, float, int, np.ndarray]:
        t, dt, ts = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        hb = np.zeros(3)
        lib().orc_get_time(self._h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(ts), _dptr(hb))
        return t.value, dt.value, ts.value, hb

    def set_time(self, time: float, delta_t: float, time_step: int) -> None:
        lib().orc_set_time(self._h, time, delta_t, time_step)

    # --- routines of the reference -----------------------------------------
    def fft_xz_to_fourier(self, v: np.ndarray, vv: np.ndarray, jmin: int, jmax: int) -> None:
        lib().orc_fft_xz_to_fourier(self._h, _dptr(v.view(np.float64)), _dptr(vv.view(np.float64)),
                                    jmin, jmax)

    def fft_xz_to_physical(self, vv: np.ndarray, v: np.ndarray, jmin: int, jmax: int) -> None:
        lib().orc_fft_xz_to_physical(self._h, _dptr(vv.view(np.float64)), _dptr(v.view(np.float64)),
                                     jmin, jmax)

    def rk_chan_1(self, rk_step: int) -> None:
        lib().orc_rk_chan_1(self._h, rk_step)

    def step(self, n: int = 1) -> None:
        for _ in range(n):
            lib().orc_step(self._h)

    def rem_div_chan(self) -> None:
        lib().orc_rem_div_chan(self._h)

    def poisson_p_chan(self) -> None:
        lib().orc_poisson_p_chan(self._h)

    def courant(self) -> None:
        lib().orc_courant(self._h)

    def apply_bc_vel(self) -> None:
        lib().orc_apply_bc_vel(self._h)

    def filter_chan(self, n: int = 1) -> None:
        lib().orc_filter_chan(self._h, n)

    def epsilon_sgs(self) -> np.ndarray:
        """tkebudget_chan_les's epsilon_sgs (plane sums, rows 1..NY)."""
        out = np.zeros(self.p.ny + 2)
        lib().orc_epsilon_sgs(self._h, _dptr(out))
        return out

    def epsilon_field(self) -> np.ndarray:
        """tkebudget_chan's F1 as [J][K][I] (NY+2, NZ, NX), rows 2..NY-1."""
        buf = np.zeros(physical_shape(self.p))
        lib().orc_epsilon_field(self._h, _dptr(buf))
        return buf[:, : self.p.nz, : self.p.nx].copy()

    def set_user_rhs(self, kind: int, fn) -> None:
        """USER_RHS_CHAN_FOURIER (kind 0) / _PHYSICAL (kind 1): fn(oracle)
        runs at that point of RK_CHAN_1 and may change self.cf / self.cfth
        in place; None removes it."""
        if not hasattr(self, "_user"):
            self._user = {}
        if fn is None:
            self._user.pop(kind, None)
            lib().orc_set_user_rhs(self._h, kind, USER_FN(), None)
            return
        cb = USER_FN(lambda _: fn(self))
        self._user[kind] = cb
        lib().orc_set_user_rhs(self._h, kind, cb, None)

    def set_mlp(self, params) -> None:
        """The learned closure's parameters (LES_MODEL_TYPE 4), or None."""
        if params is None:
            lib().orc_set_mlp(self._h, None)
            return
        self._mlp = np.ascontiguousarray(params, dtype=np.float32)
        lib().orc_set_mlp(self._h, self._mlp.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))

    def stats(self) -> np.ndarray:
        out = np.zeros((17, self.p.ny + 2))
        lib().orc_stats(self._h, _dptr(out))
        return out

    def mean_stats(self) -> dict:
        """Every mean.h5 / tke.h5 profile, keyed as Channel.mean_stats."""
        from diablo_b200.channel import MEAN_NAMES, SCAL_NAMES
        p = self.p
        ny2 = p.ny + 2
        chan = np.zeros((len(MEAN_NAMES), ny2))
        scal = np.zeros((max(p.n_th, 1), len(SCAL_NAMES), ny2))
        eps = np.zeros(ny2)
        lib().orc_mean_stats(self._h, _dptr(chan), _dptr(scal), _dptr(eps))
        out = {name: chan[k] for k, name in enumerate(MEAN_NAMES)}
        for n in range(p.n_th):
            for k, name in enumerate(SCAL_NAMES):
                out[f"{name}{n + 1:02d}"] = scal[n, k]
        out["epsilon"] = eps
        return out

    # --- initial condition (CREATE_TH_CHAN then CREATE_FLOW_CHAN) ------------
    def init_from_physical(self, u: np.ndarray, th: np.ndarray) -> None:
        """Physical fields -> Fourier state: scalars transformed
        (set_ics.f:265-268), velocity transformed, APPLY_BC_VEL, REM_DIV
        (set_ics.f:125-183).  CP and CF start at zero."""
        ny = self.p.ny
        for n in range(self.p.n_th):
            s1 = self.raw(ORC_S1)
            s1[:] = th[n].reshape(-1)
            self.fft_xz_to_fourier(s1, s1, 0, ny + 1)
            self.raw(ORC_CTH).reshape(self.p.n_th, -1)[n][:] = s1
        for c, which in enumerate((ORC_U1, ORC_U2, ORC_U3)):
            buf = self.raw(which)
            buf[:] = u[c].reshape(-1)
            self.fft_xz_to_fourier(buf, buf, 0, ny + 1)
        self.raw(ORC_P)[:] = 0.0
        for which in (ORC_F1, ORC_F2, ORC_F3, ORC_CFTH):
            self.raw(which)[:] = 0.0
        self.apply_bc_vel()
        self.rem_div_chan()
