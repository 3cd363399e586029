"""DIABLO_ENAN: a non-finite value in the state is flagged by the kernels that
write CU and reported once by the next call that synchronises.  NaN
arithmetic does not fault the GPU; the state is simply not finite."""
import numpy as np
import pytest

from diablo_b200 import grid as G, ics, layout, params as P
from diablo_b200.channel import DIABLO_ENAN, Channel, DiabloError
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def state(p, g, dt):
    u, th = ics.shear_layer(p, g, seed=3, amp=0.05)
    o = Oracle(p, g, dt)
    o.init_from_physical(u, th)
    return [x.copy() for x in o.cu], o.cp.copy(), o.cth.copy()


@pytest.mark.parametrize("variable_dt", [False, True])
def test_nan_in_state_is_reported_once(variable_dt):
    p = P.kelvin_helmholtz(32, 33, 24)
    p.variable_dt = int(variable_dt)
    g = G.channel_grid(G.create_grid(2, p.ny, 20.0, 1.5))
    cu, cp, cth = state(p, g, 0.01)
    with Channel(p, g, 0.01) as c:
        c.upload(cu, cp, cth)
        c.step(1)
        c.synchronize()                                  # a finite state: no status
        bad = [x.copy() for x in cu]
        bad[0][p.ny // 2, 3, 2] = np.nan                 # one interior coefficient of CU1
        c.upload(bad, cp, cth)
        dt0 = c.delta_t
        with pytest.raises(DiabloError) as e:
            c.step(1)                                    # COURANT at RK step 3 synchronises
            c.synchronize()
        assert e.value.code == DIABLO_ENAN
        if variable_dt:
            assert c.delta_t == dt0                      # DELTA_T kept when COURANT saw the flag
        c.synchronize()                                  # reported once, then cleared
        s = c.download()
        assert not np.isfinite(layout.dealiased(p, s["cu"][0])).all()
