"""USER_RHS_CHAN_FOURIER / USER_RHS_CHAN_PHYSICAL (for/user_rhs.f) through
the library's hooks against the oracle with the same terms: a linear damping
CF += -alpha CU, the example of user_rhs.f:14-40 and 90-120.  The GPU
callbacks write their terms with torch on the handle's stream."""
import numpy as np
import pytest

from diablo_b200 import layout, params as P
from diablo_b200.channel import USER_RHS_FOURIER, USER_RHS_PHYSICAL, Channel
from oracle.oracle import Oracle
from test_gpu_les import les_channel
from test_gpu_parity import TOL32, TOL64, kh_case, state_errors

pytestmark = pytest.mark.gpu
ALPHA = 0.7


class _Dev:
    """A device buffer of n float64 values as __cuda_array_interface__."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def fourier_damping(args):
    import torch
    n = 2 * args.s_field * (3 + args.n_th)
    with torch.cuda.stream(torch.cuda.ExternalStream(args.stream)):
        cu = torch.as_tensor(_Dev(args.cu, n), device="cuda")
        add = torch.as_tensor(_Dev(args.cf_add, n), device="cuda")
        add.copy_(-ALPHA * cu)


def physical_damping(args):
    import torch
    n = args.p_field * (3 + args.n_th)
    with torch.cuda.stream(torch.cuda.ExternalStream(args.stream)):
        u = torch.as_tensor(_Dev(args.u, n), device="cuda")
        add = torch.as_tensor(_Dev(args.f_add, n), device="cuda")
        add.copy_(-ALPHA * u)


def oracle_damping(o):
    for cf, cu in zip(o.cf, o.cu):
        cf -= ALPHA * cu
    for n in range(o.p.n_th):
        o.cfth[n] -= ALPHA * o.cth[n]


def start(p, g, u, th, dt):
    o = Oracle(p, g, dt)
    o.init_from_physical(u, th)
    c = Channel(p, g, dt)
    c.upload([x.copy() for x in o.cu], o.cp.copy(), o.cth.copy())
    return o, c


@pytest.mark.parametrize("case", ["kh", "les"])
def test_fourier_hook_matches_oracle(case):
    if case == "kh":
        p, g, u, th, dt = kh_case(32, 33, 24, dt=0.01)
    else:
        p, g, u, th = les_channel(32, 33, 24, model=1)
        dt = 1e-3
    o, c = start(p, g, u, th, dt)
    _, ref_c = start(p, g, u, th, dt)              # the same run without the hook
    with c, ref_c:
        o.set_user_rhs(0, oracle_damping)
        c.set_user_rhs(USER_RHS_FOURIER, fourier_damping)
        for _ in range(3):
            o.step()
            c.step()
            ref_c.step()
        err = state_errors(p, c, o, with_cf=False, scaled=True)
        assert max(err.values()) < TOL64, err
        # the hook changed the run by far more than the tolerance
        a = layout.dealiased(p, c.download()["cu"][0])
        b = layout.dealiased(p, ref_c.download()["cu"][0])
        assert np.linalg.norm(a - b) > 1e3 * TOL64 * np.linalg.norm(b)
        c.set_user_rhs(USER_RHS_FOURIER, None)     # removed: the plain step again
        c.step()


def test_physical_hook_equals_fourier_hook():
    """-alpha U in physical space, transformed, is -alpha CU (U is band-limited)."""
    p, g, u, th, dt = kh_case(32, 33, 24, dt=0.01)
    o = Oracle(p, g, dt)
    o.init_from_physical(u, th)
    with Channel(p, g, dt) as a, Channel(p, g, dt) as b:
        for c in (a, b):
            c.upload([x.copy() for x in o.cu], o.cp.copy(), o.cth.copy())
        a.set_user_rhs(USER_RHS_FOURIER, fourier_damping)
        b.set_user_rhs(USER_RHS_PHYSICAL, physical_damping)
        a.step(3)
        b.step(3)
        sa, sb = a.download(), b.download()
        for f in range(3):
            x, y = layout.dealiased(p, sb["cu"][f]), layout.dealiased(p, sa["cu"][f])
            assert np.linalg.norm(x - y) <= 1e-12 * np.linalg.norm(y), f


def test_fourier_hook_fp32_split():
    p, g, u, th, dt = kh_case(32, 33, 24, precision=P.PREC_FP32SPLIT, dt=0.01)
    p64 = p.copy()
    p64.precision = P.PREC_FP64
    o = Oracle(p64, g, dt)
    o.init_from_physical(u, th)
    with Channel(p, g, dt) as c:
        c.upload([x.copy() for x in o.cu], o.cp.copy(), o.cth.copy())
        o.set_user_rhs(0, oracle_damping)
        c.set_user_rhs(USER_RHS_FOURIER, fourier_damping)
        for _ in range(3):
            o.step()
            c.step()
        err = state_errors(p, c, o, with_cf=False, scaled=True)
        assert max(err.values()) < TOL32, err
