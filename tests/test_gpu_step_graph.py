"""One RK3 step as a CUDA graph (diablo_gpu_step_graph, Channel.step_graph):
the replayed graph gives the state of the same number of substage calls,
on the Fourier-space path in FP64 and FP32-split and on the LES branch, over
a first call (one direct step, then capture) and later calls that only
replay; a step that is not static falls back to the substage calls."""
import numpy as np
import pytest

from diablo_b200 import grid as G, ics, params as P, workloads
from diablo_b200.channel import Channel
from test_gpu_les import les_channel

pytestmark = pytest.mark.gpu


def _max_rel(a, b):
    out = 0.0
    for k in ("cu", "cth"):
        for x, y in zip(a[k], b[k]):
            out = max(out, float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300)))
    out = max(out, float(np.linalg.norm(a["cp"] - b["cp"]) / max(np.linalg.norm(b["cp"]), 1e-300)))
    return out


def _pair(p, g, dt, u, th):
    a, b = Channel(p, g, dt), Channel(p, g, dt)
    for c in (a, b):
        c.init_from_physical(u, th)
    return a, b


@pytest.mark.parametrize("prec", [P.PREC_FP64, P.PREC_FP32SPLIT])
def test_step_graph_equals_substage_calls(prec):
    w = workloads.kh(48, 65, 32, precision=prec)
    u, th = w.initial_fields()
    a, b = _pair(w.p, w.grid, w.dt, u, th)
    with a, b:
        a.step(6)
        assert b.step_graph(6)            # one direct step, capture, five replays
        assert _max_rel(b.download(), a.download()) < 1e-14
        l0 = b.kernel_launches()
        a.step(4)
        assert b.step_graph(4)            # replays only
        assert b.kernel_launches() > l0
        assert b.time_step == a.time_step and b.time == pytest.approx(a.time)
        assert _max_rel(b.download(), a.download()) < 1e-14


def test_step_graph_les_constant_model():
    p, g, u, th = les_channel(model=1)
    a, b = _pair(p, g, 2e-4, u, th)
    with a, b:
        a.step(3)
        assert b.step_graph(3)
        a.step(3)
        assert b.step_graph(3)
        assert _max_rel(b.download(), a.download()) < 1e-13


def test_step_graph_falls_back_when_not_static():
    p, g, u, th = les_channel(model=1, variable_dt=True)
    p.les = 0
    a, b = _pair(p, g, 2e-4, u, th)
    with a, b:
        a.step(3)
        assert not b.step_graph(3)        # CFL-adaptive dt: the substage calls instead
        assert b.delta_t == a.delta_t
        assert _max_rel(b.download(), a.download()) == 0.0
