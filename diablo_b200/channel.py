"""ctypes binding of libdiablo_gpu.so and the host-side time loop.

`Channel` is the host mirror of the reference's channel solver: it owns the
/RUNTIME_VARS/ and /RKW3_PARAMS/ scalars (TIME, TIME_STEP, DELTA_T, H_BAR,
BETA_BAR, ZETA_BAR) like the Fortran host does and calls the library's C ABI
for everything that runs on the GPU.  Method names follow the reference
routines they replace.  There is no CPU fallback: a missing or unloadable
library raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .grid import ChannelGrid
from .layout import new_fourier, physical_shape, fourier_shape
from .params import DiabloParams, validate

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdiablo_gpu.so")

DIABLO_OK, DIABLO_EINVAL, DIABLO_ERADIX, DIABLO_ECUDA, DIABLO_ENOTSUP, DIABLO_ENAN, DIABLO_ENOMEM, DIABLO_ETIMEOUT = (
    0, -1, -2, -3, -4, -5, -6, -7)
NSTATS = 17
# profiles of diablo_gpu_mean_stats: chan rows, then per scalar the SCAL rows
MEAN_NAMES = ["ume", "vme", "wme", "urms", "vrms", "wrms", "uv", "uw", "wv", "dudy", "dwdy", "cp", "shear",
              "omega_x", "omega_y", "omega_z"]
SCAL_NAMES = ["thme", "dthdy", "thrms", "thv", "pe_diss"]
# DIABLO_STAT_* rows of diablo_gpu_stats
STAT_INDEX = {"ume": 0, "vme": 1, "wme": 2, "urms": 3, "vrms": 4, "wrms": 5, "uv": 6, "uw": 7, "wv": 8,
              "dudy": 9, "dwdy": 10, "cp": 11, "shear": 12, "thme": 13, "dthdy": 14, "thrms": 15, "thv": 16}

# C entry points declared in include/diablo_gpu.h
EXPORTS = [
    "diablo_gpu_create", "diablo_gpu_destroy", "diablo_gpu_upload_state", "diablo_gpu_download_state",
    "diablo_gpu_rk_chan_1", "diablo_gpu_rk_chan_2", "diablo_gpu_fft_xz_to_fourier",
    "diablo_gpu_fft_xz_to_physical", "diablo_gpu_rem_div_chan", "diablo_gpu_download_phi",
    "diablo_gpu_poisson_p_chan", "diablo_gpu_apply_bc_vel", "diablo_gpu_courant", "diablo_gpu_stats",
    "diablo_gpu_synchronize", "diablo_gpu_kernel_launches", "diablo_gpu_last_error",
    "diablo_gpu_get_stream", "diablo_gpu_set_profiling", "diablo_gpu_kernel_times",
    "diablo_gpu_rem_div_chan_noalloc", "diablo_gpu_autotune", "diablo_gpu_batch_create",
    "diablo_gpu_batch_step", "diablo_gpu_batch_destroy", "diablo_gpu_filter_chan", "diablo_gpu_download_nu_t",
    "diablo_gpu_mean_stats", "diablo_gpu_set_user_rhs",
    "diablo_gpu_sgs_samples", "diablo_gpu_set_sgs_mlp", "diablo_gpu_step_graph",
]
KERNEL_NAMES = ["zinv", "products", "zfwd_nl", "cn_coef", "column", "remdiv", "cfl", "other"]


class UserRhsArgs(ctypes.Structure):
    """diablo_user_rhs_args: what a USER_RHS_CHAN_FOURIER / _PHYSICAL
    callback receives (device pointers, strides, the handle's stream)."""
    _fields_ = [("rk_step", ctypes.c_int), ("time_step", ctypes.c_int), ("time", ctypes.c_double),
                ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("n_th", ctypes.c_int),
                ("nkx", ctypes.c_int), ("tnkz", ctypes.c_int),
                ("s_field", ctypes.c_longlong), ("s_plane", ctypes.c_longlong), ("s_row", ctypes.c_longlong),
                ("p_field", ctypes.c_longlong), ("p_plane", ctypes.c_longlong),
                ("cu", ctypes.c_void_p), ("cf_add", ctypes.c_void_p), ("u", ctypes.c_void_p),
                ("f_add", ctypes.c_void_p), ("stream", ctypes.c_void_p)]


USER_RHS_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.POINTER(UserRhsArgs))
USER_RHS_FOURIER, USER_RHS_PHYSICAL = 0, 1


class DiabloError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what} failed with status {code}: {last_error()}")
        self.code = code


_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m diablo_b200.build`")
    L = ctypes.CDLL(path)
    vp, dp, ip, dd = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_double
    L.diablo_gpu_create.argtypes = [ctypes.POINTER(DiabloParams), dp, dp, dp, dp, ctypes.POINTER(vp)]
    L.diablo_gpu_destroy.argtypes = [vp]
    L.diablo_gpu_upload_state.argtypes = [vp] + [dp] * 9
    L.diablo_gpu_download_state.argtypes = [vp] + [dp] * 9
    L.diablo_gpu_rk_chan_1.argtypes = [vp, ip, ip, dd, dp, dp, dp, dp]
    L.diablo_gpu_rk_chan_2.argtypes = [vp]
    L.diablo_gpu_fft_xz_to_fourier.argtypes = [vp, dp, dp, ip, ip]
    L.diablo_gpu_fft_xz_to_physical.argtypes = [vp, dp, dp, ip, ip]
    for name in ("diablo_gpu_rem_div_chan", "diablo_gpu_poisson_p_chan", "diablo_gpu_apply_bc_vel",
                 "diablo_gpu_synchronize"):
        getattr(L, name).argtypes = [vp]
    L.diablo_gpu_download_phi.argtypes = [vp, dp]
    L.diablo_gpu_courant.argtypes = [vp, dp, dp]
    L.diablo_gpu_stats.argtypes = [vp, dp]
    L.diablo_gpu_mean_stats.argtypes = [vp, dp, dp, dp]
    L.diablo_gpu_set_user_rhs.argtypes = [vp, ip, USER_RHS_FN, vp]
    L.diablo_gpu_kernel_launches.argtypes = [vp]
    L.diablo_gpu_kernel_launches.restype = ctypes.c_longlong
    L.diablo_gpu_last_error.restype = ctypes.c_char_p
    L.diablo_gpu_get_stream.argtypes = [vp, ctypes.POINTER(vp)]
    L.diablo_gpu_set_profiling.argtypes = [vp, ip]
    L.diablo_gpu_kernel_times.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong), dp]
    L.diablo_gpu_rem_div_chan_noalloc.argtypes = [ctypes.POINTER(DiabloParams), dp, dp, vp, vp, vp, vp, vp]
    L.diablo_gpu_autotune.argtypes = [vp, ctypes.POINTER(ip), ctypes.POINTER(ip)]
    L.diablo_gpu_batch_create.argtypes = [ctypes.POINTER(vp), dp, ip, ctypes.POINTER(vp)]
    L.diablo_gpu_batch_step.argtypes = [vp, ip]
    L.diablo_gpu_step_graph.argtypes = [vp, ip, ip, dp, dp, dp]
    L.diablo_gpu_batch_destroy.argtypes = [vp]
    L.diablo_gpu_filter_chan.argtypes = [vp, ip]
    L.diablo_gpu_download_nu_t.argtypes = [vp, dp]
    L.diablo_gpu_set_sgs_mlp.argtypes = [vp, vp]
    L.diablo_gpu_sgs_samples.argtypes = [vp, ip, ip, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                         ctypes.POINTER(ctypes.c_float), ctypes.c_longlong,
                                         ctypes.POINTER(ctypes.c_longlong)]
    _lib = L
    return L


def last_error() -> str:
    if _lib is None:
        return ""
    return (_lib.diablo_gpu_last_error() or b"").decode()


def _dp(a: np.ndarray | None):
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("host arrays must be C-contiguous (Fortran layout viewed in C order)")
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _check(rc: int, what: str) -> None:
    if rc != DIABLO_OK:
        raise DiabloError(rc, what)


class Channel:
    """One channel instance on the current GPU (one library handle)."""

    def __init__(self, p: DiabloParams, grid: ChannelGrid, delta_t: float):
        validate(p)
        self.L = load_library()
        self.p = p.copy()
        self.grid = grid
        self._h = ctypes.c_void_p()
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (grid.gy, grid.gyf, grid.dy, grid.dyf)]
        _check(self.L.diablo_gpu_create(ctypes.byref(self.p), *[_dp(a) for a in arrs], ctypes.byref(self._h)),
               "diablo_gpu_create")
        # /RUNTIME_VARS/ and /RKW3_PARAMS/ (diablo_io.f:116-124)
        self.time = 0.0
        self.time_step = 0
        self.delta_t = float(delta_t)
        self.h_bar = np.array([delta_t * 8.0 / 15.0, delta_t * 2.0 / 15.0, delta_t * 5.0 / 15.0])
        self.beta_bar = np.array([1.0, 25.0 / 8.0, 9.0 / 4.0])
        self.zeta_bar = np.array([0.0, -17.0 / 8.0, -5.0 / 4.0])

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self.L.diablo_gpu_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --- state transfer ----------------------------------------------------
    def upload(self, cu: list[np.ndarray], cp: np.ndarray, cth: np.ndarray | None,
               cf: list[np.ndarray] | None = None, cfth: np.ndarray | None = None) -> None:
        def f64(a):
            return None if a is None else np.ascontiguousarray(a).view(np.float64)
        cfl = cf or [None, None, None]
        _check(self.L.diablo_gpu_upload_state(
            self._h, _dp(f64(cu[0])), _dp(f64(cu[1])), _dp(f64(cu[2])), _dp(f64(cp)),
            _dp(f64(cth)) if self.p.n_th else None,
            _dp(f64(cfl[0])), _dp(f64(cfl[1])), _dp(f64(cfl[2])),
            _dp(f64(cfth)) if (cfth is not None and self.p.n_th) else None), "diablo_gpu_upload_state")

    def download(self) -> dict:
        p = self.p
        out = {
            "cu": [new_fourier(p) for _ in range(3)],
            "cp": new_fourier(p),
            "cth": new_fourier(p, max(p.n_th, 1)),
            "cf": [new_fourier(p) for _ in range(3)],
            "cfth": new_fourier(p, max(p.n_th, 1)),
        }
        v = lambda a: _dp(a.view(np.float64))
        _check(self.L.diablo_gpu_download_state(
            self._h, v(out["cu"][0]), v(out["cu"][1]), v(out["cu"][2]), v(out["cp"]), v(out["cth"]),
            v(out["cf"][0]), v(out["cf"][1]), v(out["cf"][2]), v(out["cfth"])), "diablo_gpu_download_state")
        out["cth"] = out["cth"][: p.n_th]
        out["cfth"] = out["cfth"][: p.n_th]
        return out

    def download_into(self, cu: list[np.ndarray], cp: np.ndarray, cth: list[np.ndarray]) -> None:
        """Download CU1..3, CP and CTH into caller-owned Fortran-layout arrays."""
        v = lambda a: _dp(a.view(np.float64)) if a is not None else None
        if self.p.n_th > 1:
            tmp = np.empty((self.p.n_th,) + fourier_shape(self.p), dtype=np.complex128)
            th_ptr = v(tmp)
        else:
            tmp = None
            th_ptr = v(cth[0]) if self.p.n_th else None
        _check(self.L.diablo_gpu_download_state(self._h, v(cu[0]), v(cu[1]), v(cu[2]), v(cp), th_ptr,
                                                None, None, None, None), "diablo_gpu_download_state")
        if tmp is not None:
            for n in range(self.p.n_th):
                cth[n][...] = tmp[n]

    def download_phi(self) -> np.ndarray:
        phi = new_fourier(self.p)
        _check(self.L.diablo_gpu_download_phi(self._h, _dp(phi.view(np.float64))), "diablo_gpu_download_phi")
        return phi

    def download_nu_t(self) -> np.ndarray:
        """NU_T at GY points as [J][K][I] (NY+2, NZ, NX); LES only."""
        buf = np.zeros(physical_shape(self.p))
        _check(self.L.diablo_gpu_download_nu_t(self._h, _dp(buf)), "diablo_gpu_download_nu_t")
        return buf[:, : self.p.nz, : self.p.nx].copy()

    def set_user_rhs(self, kind: int, fn) -> None:
        """USER_RHS_CHAN_FOURIER (kind USER_RHS_FOURIER) or _PHYSICAL
        (USER_RHS_PHYSICAL): fn(args: UserRhsArgs) runs once per substage and
        writes the terms to add to CF into args.cf_add / args.f_add on
        args.stream; None removes the hook."""
        if not hasattr(self, "_user_rhs"):
            self._user_rhs = {}
        if fn is None:
            self._user_rhs.pop(kind, None)
            _check(self.L.diablo_gpu_set_user_rhs(self._h, kind, USER_RHS_FN(), None), "diablo_gpu_set_user_rhs")
            return
        cb = USER_RHS_FN(lambda _user, args: fn(args.contents))
        self._user_rhs[kind] = cb
        _check(self.L.diablo_gpu_set_user_rhs(self._h, kind, cb, None), "diablo_gpu_set_user_rhs")

    def set_sgs_mlp(self, mlp) -> None:
        """Attach a closure network (diablo_b200.mlp.SgsMlp) for
        LES_MODEL_TYPE 4, or detach it with None."""
        self._mlp = mlp
        _check(self.L.diablo_gpu_set_sgs_mlp(self._h, mlp.handle if mlp is not None else None),
               "diablo_gpu_set_sgs_mlp")

    def sgs_samples(self, width: int = 3, stride: int = 1):
        """Closure training samples of the current state for a width x width
        x-z top-hat filter: dimensionless features [n][11], dimensionless
        targets [n][6] and the stress scales [n] (tau = target * scale)."""
        p = self.p
        n = (p.ny - 2) * (-(-p.nx // stride)) * (-(-p.nz // stride))
        x = np.zeros((n, 11), dtype=np.float32)
        t = np.zeros((n, 6), dtype=np.float32)
        s = np.zeros(n, dtype=np.float32)
        cnt = ctypes.c_longlong()
        fp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        _check(self.L.diablo_gpu_sgs_samples(self._h, width, stride, fp(x), fp(t), fp(s), n, ctypes.byref(cnt)),
               "diablo_gpu_sgs_samples")
        assert cnt.value == n
        return x, t, s

    # --- routines of the reference ------------------------------------------
    def rk_chan_1(self, rk_step: int) -> None:
        """One RK substage (RK_CHAN_1); DELTA_T/H_BAR change if COURANT ran."""
        dt = ctypes.c_double(self.delta_t)
        hb = np.ascontiguousarray(self.h_bar, dtype=np.float64)
        _check(self.L.diablo_gpu_rk_chan_1(self._h, rk_step, self.time_step, self.time, ctypes.byref(dt),
                                           _dp(hb), _dp(self.beta_bar), _dp(self.zeta_bar)),
               "diablo_gpu_rk_chan_1")
        self.delta_t = dt.value
        self.h_bar = hb

    def rk_chan_2(self) -> None:
        _check(self.L.diablo_gpu_rk_chan_2(self._h), "diablo_gpu_rk_chan_2")

    def step(self, n: int = 1) -> None:
        """n time steps of the loop in diablo.f:66-111 (no statistics or I/O)."""
        for _ in range(n):
            self.time_step += 1
            for rk in (1, 2, 3):
                self.rk_chan_1(rk)
            self.time += self.delta_t

    def step_graph(self, n: int = 1) -> bool:
        """n time steps as replays of one CUDA graph of a whole RK3 step
        (diablo_gpu_step_graph): the same results as step(n), with one
        launch per step instead of one per kernel.  Falls back to step(n) and
        returns False when the step is not static (variable dt, time-dependent
        forcing, a user right-hand side, profiling, or an LES whose subgrid
        model starts within these steps)."""
        if n <= 0:
            return True
        hb = np.ascontiguousarray(self.h_bar, dtype=np.float64)
        bb = np.ascontiguousarray(self.beta_bar, dtype=np.float64)
        zb = np.ascontiguousarray(self.zeta_bar, dtype=np.float64)
        rc = self.L.diablo_gpu_step_graph(self._h, int(n), self.time_step, _dp(hb), _dp(bb), _dp(zb))
        if rc == DIABLO_ENOTSUP:
            self.step(n)
            return False
        _check(rc, "diablo_gpu_step_graph")
        self.time_step += n
        self.time += n * self.delta_t
        return True

    def synchronize(self) -> None:
        _check(self.L.diablo_gpu_synchronize(self._h), "diablo_gpu_synchronize")

    def rem_div_chan(self) -> None:
        _check(self.L.diablo_gpu_rem_div_chan(self._h), "diablo_gpu_rem_div_chan")

    def poisson_p_chan(self) -> None:
        _check(self.L.diablo_gpu_poisson_p_chan(self._h), "diablo_gpu_poisson_p_chan")

    def apply_bc_vel(self) -> None:
        _check(self.L.diablo_gpu_apply_bc_vel(self._h), "diablo_gpu_apply_bc_vel")

    def courant(self) -> None:
        dt = ctypes.c_double(self.delta_t)
        hb = np.zeros(3)
        _check(self.L.diablo_gpu_courant(self._h, ctypes.byref(dt), _dp(hb)), "diablo_gpu_courant")
        self.delta_t = dt.value
        self.h_bar = hb

    def stats(self) -> np.ndarray:
        out = np.zeros((NSTATS, self.p.ny + 2))
        _check(self.L.diablo_gpu_stats(self._h, _dp(out)), "diablo_gpu_stats")
        return out

    def mean_stats(self) -> dict:
        """Every mean.h5 / tke.h5 profile of SAVE_STATS_CHAN (NY+2 values
        each): MEAN_NAMES, SCAL_NAMES with the scalar's two-digit number
        (thme01, ...), and epsilon (rows 2..NY-1)."""
        p = self.p
        ny2 = p.ny + 2
        chan = np.zeros((len(MEAN_NAMES), ny2))
        scal = np.zeros((max(p.n_th, 1), len(SCAL_NAMES), ny2))
        eps = np.zeros(ny2)
        _check(self.L.diablo_gpu_mean_stats(self._h, _dp(chan), _dp(scal), _dp(eps)), "diablo_gpu_mean_stats")
        out = {name: chan[k] for k, name in enumerate(MEAN_NAMES)}
        for n in range(p.n_th):
            for k, name in enumerate(SCAL_NAMES):
                out[f"{name}{n + 1:02d}"] = scal[n, k]
        out["epsilon"] = eps
        return out

    def fft_xz_to_fourier(self, v: np.ndarray, vv: np.ndarray, jmin: int, jmax: int) -> None:
        assert v.shape[-3:] == physical_shape(self.p) and vv.shape[-3:] == fourier_shape(self.p)
        _check(self.L.diablo_gpu_fft_xz_to_fourier(self._h, _dp(v), _dp(vv.view(np.float64)), jmin, jmax),
               "diablo_gpu_fft_xz_to_fourier")

    def fft_xz_to_physical(self, vv: np.ndarray, v: np.ndarray, jmin: int, jmax: int) -> None:
        assert v.shape[-3:] == physical_shape(self.p) and vv.shape[-3:] == fourier_shape(self.p)
        _check(self.L.diablo_gpu_fft_xz_to_physical(self._h, _dp(vv.view(np.float64)), _dp(v), jmin, jmax),
               "diablo_gpu_fft_xz_to_physical")

    def filter_chan(self, n: int = 1) -> None:
        _check(self.L.diablo_gpu_filter_chan(self._h, n), "diablo_gpu_filter_chan")

    def autotune(self) -> tuple[int, int]:
        """Pick the products plane chunk and the z-forward planes per block by
        timing this instance's grid; the state is left as it was."""
        pc, zp = ctypes.c_int(), ctypes.c_int()
        _check(self.L.diablo_gpu_autotune(self._h, ctypes.byref(pc), ctypes.byref(zp)), "diablo_gpu_autotune")
        return pc.value, zp.value

    def kernel_launches(self) -> int:
        return int(self.L.diablo_gpu_kernel_launches(self._h))

    def stream(self) -> int:
        """The handle's cudaStream_t as an integer (for timing events)."""
        s = ctypes.c_void_p()
        _check(self.L.diablo_gpu_get_stream(self._h, ctypes.byref(s)), "diablo_gpu_get_stream")
        return int(s.value or 0)

    def set_profiling(self, on: bool) -> None:
        _check(self.L.diablo_gpu_set_profiling(self._h, int(on)), "diablo_gpu_set_profiling")

    def kernel_times(self) -> dict:
        """{kernel kind: (launches, total ms)} since profiling was switched on."""
        n = (ctypes.c_longlong * len(KERNEL_NAMES))()
        ms = np.zeros(len(KERNEL_NAMES))
        _check(self.L.diablo_gpu_kernel_times(self._h, n, _dp(ms)), "diablo_gpu_kernel_times")
        return {KERNEL_NAMES[k]: (int(n[k]), float(ms[k])) for k in range(len(KERNEL_NAMES)) if n[k]}

    # --- initial condition (CREATE_TH_CHAN then CREATE_FLOW_CHAN) ------------
    def init_from_physical(self, u: np.ndarray, th: np.ndarray) -> None:
        """Transform physical fields with this library, upload with CP = CF = 0,
        then APPLY_BC_VEL and REM_DIV_CHAN (set_ics.f:125-183, 265-268)."""
        p = self.p
        cu = [new_fourier(p) for _ in range(3)]
        for c in range(3):
            self.fft_xz_to_fourier(np.ascontiguousarray(u[c]), cu[c], 0, p.ny + 1)
        cth = new_fourier(p, max(p.n_th, 1))
        for n in range(p.n_th):
            self.fft_xz_to_fourier(np.ascontiguousarray(th[n]), cth[n], 0, p.ny + 1)
        self.upload(cu, new_fourier(p), cth)
        self.apply_bc_vel()
        self.rem_div_chan()


class Batch:
    """Many channel instances advanced together: one CUDA graph holds a full
    RK3 step of every instance (one stream branch each); step(n) launches it n
    times.  Instances need a fixed time step; they stay usable on their own
    (upload / download) between batch steps."""

    def __init__(self, channels: list[Channel], delta_t: list[float] | None = None):
        self.L = load_library()
        self.channels = list(channels)
        n = len(self.channels)
        hs = (ctypes.c_void_p * n)(*[c._h.value for c in self.channels])
        dts = np.ascontiguousarray([c.delta_t for c in self.channels] if delta_t is None else delta_t,
                                   dtype=np.float64)
        self._b = ctypes.c_void_p()
        _check(self.L.diablo_gpu_batch_create(hs, _dp(dts), n, ctypes.byref(self._b)), "diablo_gpu_batch_create")
        self._dts = dts

    def step(self, n: int = 1) -> None:
        _check(self.L.diablo_gpu_batch_step(self._b, int(n)), "diablo_gpu_batch_step")
        for c, dt in zip(self.channels, self._dts):
            c.time += n * float(dt)
            c.time_step += n

    def close(self) -> None:
        if getattr(self, "_b", None) and self._b.value:
            self.L.diablo_gpu_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
