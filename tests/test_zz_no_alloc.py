"""The no-allocation REM_DIV_CHAN entry point against the handle-based one.

diablo_gpu_rem_div_chan_noalloc serves hosts that own their device arrays
and cannot let a library call cudaMalloc; it works in place on device arrays
in the Fortran layout and keeps its scratch in static device memory.  This
test owns the device arrays itself (torch allocates them, the entry point
does not) and checks two consecutive calls, with different fields, against
diablo_gpu_rem_div_chan on a library handle and against the CPU oracle's
REM_DIV_CHAN.  The file name makes pytest collect it last."""
import ctypes

import numpy as np
import pytest

from diablo_b200 import layout, workloads
from diablo_b200.channel import DIABLO_EINVAL, DIABLO_OK, Channel, load_library

pytestmark = pytest.mark.gpu
TOL64 = 1e-10


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _random_velocity(p, rng):
    cu = [layout.new_fourier(p) for _ in range(3)]
    for c in cu:
        blk = c[:, : p.tnkz + 1, : p.nkx + 1]
        blk[...] = rng.standard_normal(blk.shape) + 1j * rng.standard_normal(blk.shape)
    return cu


def _relerr(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_rem_div_noalloc_matches_handle_path_on_two_calls():
    import torch

    L = load_library()
    w = workloads.kh(48, 33, 36)
    p, g = w.p, w.grid
    rng = np.random.default_rng(2024)
    dy = np.ascontiguousarray(g.dy)
    dyf = np.ascontiguousarray(g.dyf)
    for call in range(2):
        cu = _random_velocity(p, rng)
        with Channel(p, g, w.dt) as ch:
            ch.upload([x.copy() for x in cu], layout.new_fourier(p), layout.new_fourier(p, 1))
            ch.rem_div_chan()
            ref = ch.download()
            ref_phi = ch.download_phi()
        dev = [torch.from_numpy(x.view(np.float64).reshape(-1).copy()).cuda() for x in cu]
        phi = torch.full_like(dev[0], float("nan"))
        stream = torch.cuda.current_stream().cuda_stream
        rc = L.diablo_gpu_rem_div_chan_noalloc(ctypes.byref(p), _dp(dy), _dp(dyf), dev[0].data_ptr(),
                                                dev[1].data_ptr(), dev[2].data_ptr(), phi.data_ptr(),
                                                ctypes.c_void_p(stream))
        assert rc == DIABLO_OK, L.diablo_gpu_last_error()
        torch.cuda.synchronize()
        out = [t.cpu().numpy().view(np.complex128).reshape(layout.fourier_shape(p)) for t in dev]
        for k in range(3):
            a = layout.dealiased(p, out[k])[1: p.ny + 1]
            b = layout.dealiased(p, ref["cu"][k])[1: p.ny + 1]
            assert _relerr(a, b) < TOL64, (call, k)
        phi_h = phi.cpu().numpy().view(np.complex128).reshape(layout.fourier_shape(p))
        assert _relerr(layout.dealiased(p, phi_h)[1: p.ny + 1], layout.dealiased(p, ref_phi)[1: p.ny + 1]) < TOL64


def test_rem_div_noalloc_matches_oracle_on_two_calls():
    """Two calls in a row on the same device arrays (the second starts from
    the first one's projected field plus new noise), each against the CPU
    oracle's REM_DIV_CHAN on the same input: CU1..CU3 and phi on J = 1..NY."""
    import torch

    from oracle.oracle import ORC_U1, ORC_U2, ORC_U3, Oracle

    L = load_library()
    w = workloads.kh(40, 17, 30)
    p, g = w.p, w.grid
    rng = np.random.default_rng(77)
    dy = np.ascontiguousarray(g.dy)
    dyf = np.ascontiguousarray(g.dyf)
    cu = _random_velocity(p, rng)
    dev = [torch.from_numpy(x.view(np.float64).reshape(-1).copy()).cuda() for x in cu]
    phi = torch.full_like(dev[0], float("nan"))
    o = Oracle(p, g, w.dt)
    for call in range(2):
        if call:
            noise = _random_velocity(p, rng)
            for k in range(3):
                dev[k] += torch.from_numpy(0.5 * noise[k].view(np.float64).reshape(-1)).cuda()
        start = [t.cpu().numpy().copy() for t in dev]
        for k, which in enumerate((ORC_U1, ORC_U2, ORC_U3)):
            o.raw(which)[:] = start[k]
        o.rem_div_chan()
        stream = torch.cuda.current_stream().cuda_stream
        rc = L.diablo_gpu_rem_div_chan_noalloc(ctypes.byref(p), _dp(dy), _dp(dyf), dev[0].data_ptr(),
                                                dev[1].data_ptr(), dev[2].data_ptr(), phi.data_ptr(),
                                                ctypes.c_void_p(stream))
        assert rc == DIABLO_OK, L.diablo_gpu_last_error()
        torch.cuda.synchronize()
        for k in range(3):
            a = layout.dealiased(p, dev[k].cpu().numpy().view(np.complex128).reshape(layout.fourier_shape(p)))
            b = layout.dealiased(p, o.cu[k])
            assert _relerr(a[1: p.ny + 1], b[1: p.ny + 1]) < TOL64, (call, k)
        phi_h = phi.cpu().numpy().view(np.complex128).reshape(layout.fourier_shape(p))
        assert _relerr(layout.dealiased(p, phi_h)[1: p.ny + 1], layout.dealiased(p, o.phi)[1: p.ny + 1]) < TOL64


def test_rem_div_noalloc_rejects_grids_beyond_its_scratch():
    import torch

    L = load_library()
    w = workloads.kh(512, 257, 384)
    p, g = w.p, w.grid
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = L.diablo_gpu_rem_div_chan_noalloc(ctypes.byref(p), _dp(np.ascontiguousarray(g.dy)),
                                            _dp(np.ascontiguousarray(g.dyf)), t.data_ptr(), t.data_ptr(),
                                            t.data_ptr(), t.data_ptr(), None)
    assert rc == DIABLO_EINVAL
    assert b"too large" in L.diablo_gpu_last_error()
