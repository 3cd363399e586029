"""The learned subgrid-stress closure through the C ABI (diablo_mlp_*).

An MLP from 11 features -- the 9 resolved velocity gradients du_i/dx_j
(i-major), the wall distance in viscous units y+ and the filter width -- to
the 6 stresses (tau_11, tau_22, tau_33, tau_12, tau_13, tau_23), with 3
hidden layers of 64 GELU units, BF16 weights and activations on the tensor
cores and FP32 accumulation.  The reference has no such model.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .channel import DIABLO_OK, DiabloError, load_library

NIN, NH, NOUT = 11, 64, 6
NTRAIN = NH * NIN + NH + NH * NH + NH + NH * NH + NH + NOUT * NH + NOUT
NPARAM = NTRAIN + 2 * NIN + NOUT


def _bind(L):
    if getattr(L, "_mlp_bound", False):
        return L
    vp, fp, dp, ll = ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double), ctypes.c_longlong
    L.diablo_mlp_create.argtypes = [ctypes.POINTER(vp)]
    L.diablo_mlp_destroy.argtypes = [vp]
    L.diablo_mlp_set_params.argtypes = [vp, fp]
    L.diablo_mlp_get_params.argtypes = [vp, fp]
    L.diablo_mlp_forward.argtypes = [vp, fp, ll, fp]
    L.diablo_mlp_gradient.argtypes = [vp, fp, fp, ll, dp, fp]
    L.diablo_mlp_train.argtypes = [vp, fp, fp, ll, ctypes.c_int, ctypes.c_int, ctypes.c_float, dp]
    L.diablo_mlp_set_dissipation_weight.argtypes = [vp, ctypes.c_float]
    L._mlp_bound = True
    return L


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _fp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _check(rc: int, what: str) -> None:
    if rc != DIABLO_OK:
        raise DiabloError(rc, what)


def init_params(seed: int, mean=None, scale=None, out_scale=None) -> np.ndarray:
    """Seeded Xavier-uniform weights, zero biases and the given normalisation
    (identity when omitted)."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_out, fan_in in ((NH, NIN), (NH, NH), (NH, NH), (NOUT, NH)):
        lim = np.sqrt(6.0 / (fan_in + fan_out))
        parts.append(rng.uniform(-lim, lim, size=fan_out * fan_in))
        parts.append(np.zeros(fan_out))
    parts.append(np.zeros(NIN) if mean is None else np.asarray(mean, dtype=np.float64))
    parts.append(np.ones(NIN) if scale is None else np.asarray(scale, dtype=np.float64))
    parts.append(np.ones(NOUT) if out_scale is None else np.asarray(out_scale, dtype=np.float64))
    p = np.concatenate(parts).astype(np.float32)
    assert p.size == NPARAM
    return p


def normalisation(x: np.ndarray, t: np.ndarray):
    """Input means and scales and output scales from training data."""
    mean = x.mean(axis=0)
    scale = x.std(axis=0)
    scale[scale == 0] = 1.0
    osc = t.std(axis=0)
    osc[osc == 0] = 1.0
    return mean, scale, osc


class SgsMlp:
    """One closure network on the current GPU."""

    def __init__(self, params: np.ndarray | None = None, seed: int = 0):
        self.L = _bind(load_library())
        self._h = ctypes.c_void_p()
        _check(self.L.diablo_mlp_create(ctypes.byref(self._h)), "diablo_mlp_create")
        self.set_params(init_params(seed) if params is None else params)

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self.L.diablo_mlp_destroy(self._h)
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

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def set_params(self, p: np.ndarray) -> None:
        p = _f32(p)
        assert p.size == NPARAM
        _check(self.L.diablo_mlp_set_params(self._h, _fp(p)), "diablo_mlp_set_params")

    def set_dissipation_weight(self, w: float) -> None:
        """Weight of the subgrid-dissipation term of the training loss:
        w/2 (Pi(y) - Pi(t))^2 per sample, Pi = -tau_ij S_ij."""
        _check(self.L.diablo_mlp_set_dissipation_weight(self._h, float(w)), "diablo_mlp_set_dissipation_weight")

    def params(self) -> np.ndarray:
        p = np.zeros(NPARAM, dtype=np.float32)
        _check(self.L.diablo_mlp_get_params(self._h, _fp(p)), "diablo_mlp_get_params")
        return p

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = _f32(x).reshape(-1, NIN)
        y = np.zeros((x.shape[0], NOUT), dtype=np.float32)
        _check(self.L.diablo_mlp_forward(self._h, _fp(x), x.shape[0], _fp(y)), "diablo_mlp_forward")
        return y

    def gradient(self, x: np.ndarray, t: np.ndarray):
        x = _f32(x).reshape(-1, NIN)
        t = _f32(t).reshape(-1, NOUT)
        g = np.zeros(NTRAIN, dtype=np.float32)
        loss = ctypes.c_double()
        _check(self.L.diablo_mlp_gradient(self._h, _fp(x), _fp(t), x.shape[0], ctypes.byref(loss), _fp(g)),
               "diablo_mlp_gradient")
        return loss.value, g

    def train(self, x: np.ndarray, t: np.ndarray, batch: int, steps: int, lr: float) -> np.ndarray:
        x = _f32(x).reshape(-1, NIN)
        t = _f32(t).reshape(-1, NOUT)
        losses = np.zeros(steps)
        _check(self.L.diablo_mlp_train(self._h, _fp(x), _fp(t), x.shape[0], batch, steps, lr,
                                       losses.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "diablo_mlp_train")
        return losses
