"""Flow files written and read through the library (save/load with the
GPU transforms, POISSON_P_CHAN, COURANT and APPLY_BC_VEL) against the CPU
oracle running the reference's SAVE_FLOW / READ_FLOW steps."""
import numpy as np
import pytest

from diablo_b200 import checkpoint as ck, layout
from diablo_b200.channel import Channel
from oracle.oracle import ORC_P, Oracle
from test_checkpoint import channel, kh, oracle_load, oracle_load_legacy, oracle_save, rel
from test_gpu_parity import TOL64, state_errors

pytestmark = pytest.mark.gpu


def oracle_run(p, g, u, th, dt, steps):
    o = Oracle(p, g, dt)
    o.init_from_physical(u, th)
    o.step(steps)
    return o


def to_gpu(o):
    """A Channel holding the oracle's state, TIME, TIME_STEP and DELTA_T."""
    p = o.p
    c = Channel(p, o.grid, o.time()[1])
    c.upload([x.copy() for x in o.cu], o.cp.copy(), o.cth.copy(), [x.copy() for x in o.cf], o.cfth.copy())
    t, dto, ts, hb = o.time()
    c.time, c.time_step, c.delta_t, c.h_bar = t, ts, dto, hb.copy()
    return c


def test_save_matches_oracle(tmp_path):
    p, g, u, th = kh(48, 33, 36)
    o = oracle_run(p, g, u, th, 0.01, 3)
    with to_gpu(o) as c:
        ck.save(c, str(tmp_path / "gpu.h5"), save_pressure=True)
    oracle_save(o, str(tmp_path / "cpu.h5"), save_pressure=True)
    a, b = ck.datasets(str(tmp_path / "gpu.h5")), ck.datasets(str(tmp_path / "cpu.h5"))
    assert sorted(a) == sorted(b)
    for k in ("U", "V", "W", "TH01", "P"):
        assert a[k].shape == (p.nz, p.ny, p.nx)
        assert rel(a[k], b[k]) < 1e-13, k
    assert float(a["Time"]) == float(b["Time"]) and int(a["Timestep"]) == 3


@pytest.mark.parametrize("save_pressure", [False, True])
def test_load_and_continue_matches_oracle(tmp_path, save_pressure):
    """A variable-DT wall-bounded channel: COURANT, POISSON_P_CHAN (file
    without P) and APPLY_BC_VEL after the read, then three steps."""
    p, g, u, th = channel(48, 33, 40)
    o = oracle_run(p, g, u, th, 1e-3, 3)
    path = str(tmp_path / "out.h5")
    oracle_save(o, path, save_pressure)
    o2 = Oracle(p, g, 1e-3)
    oracle_load(o2, path)
    with Channel(p, g, 1e-3) as c2:
        info = ck.load(c2, path)
        assert info["pressure"] == save_pressure
        _, dto, tso, _ = o2.time()
        assert c2.time_step == tso and c2.delta_t == pytest.approx(dto, rel=1e-12)
        err = state_errors(p, c2, o2, with_cf=False)
        assert max(err.values()) < 1e-12, err
        o2.step(3)
        c2.step(3)
        err = state_errors(p, c2, o2)
        assert max(err.values()) < TOL64, err


def test_legacy_round_trip_and_continue(tmp_path):
    p, g, u, th = kh(48, 33, 36)
    o = oracle_run(p, g, u, th, 0.01, 3)
    flow, sp = str(tmp_path / "diablo.saved"), str(tmp_path / "diablo_th01.saved")
    with to_gpu(o) as c, Channel(p, g, 0.01) as c2:
        ck.save_legacy(c, flow, [sp])
        ref = c.download()
        c2.upload([layout.new_fourier(p)] * 3, ref["cp"], ref["cth"])
        ck.load_legacy(c2, flow, {0: sp})
        got = c2.download()
        blk = np.s_[2 : p.ny, : p.tnkz + 1, : p.nkx + 1]
        for a, b in zip(got["cu"] + [got["cth"][0]], ref["cu"] + [ref["cth"][0]]):
            assert np.array_equal(a[blk], b[blk])               # interior planes bit for bit
        assert (c2.time, c2.time_step) == (c.time, c.time_step)
        o2 = Oracle(p, g, 0.01)
        o2.fourier(ORC_P, 0)[...] = ref["cp"]                   # READ_FLOW keeps CP
        oracle_load_legacy(o2, flow, {0: sp})
        err = state_errors(p, c2, o2, with_cf=False)
        assert max(err.values()) < 1e-13, err
        o2.step(3)
        c2.step(3)
        err = state_errors(p, c2, o2)
        assert max(err.values()) < TOL64, err
