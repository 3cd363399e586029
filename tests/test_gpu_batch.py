"""GPU tests of the batched path and of the launch-shape autotuner.

The batch groups its instances by shape; each kernel of a substage is one
launch over a whole group, reading every instance's arrays and parameters
from device tables, and one CUDA graph holds the step of all groups.  It runs
the same kernel bodies with the same arithmetic as single-instance steps (the
autotuner only regroups planes into blocks), so the results must equal those
of the plain path: compared here to 1e-14 relative L2 per field, i.e. to the
last bits.  A second test pins batched instances directly to the CPU oracle."""
import numpy as np
import pytest

from diablo_b200 import grid as G, ics, layout, params as P
from diablo_b200.channel import Batch, Channel, DiabloError

pytestmark = pytest.mark.gpu
TOL = 1e-14

# two instances share the first shape (one group of two), the others differ
SIZES = [(32, 17, 24), (48, 33, 36), (64, 33, 32), (32, 17, 24)]


def relerr(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def instance(nx, ny, nz, precision, seed, ri):
    p = P.kelvin_helmholtz(nx, ny, nz, precision=precision)
    p.ri[0] = ri
    g = G.channel_grid(G.uniform_gy(ny, -10.0, 10.0))
    u, th = ics.shear_layer(p, g, seed=seed, amp=1e-2)
    return p, g, u, th


def state_of(c):
    s = c.download()
    return [layout.dealiased(c.p, a) for a in (s["cu"][0], s["cu"][1], s["cu"][2], s["cp"], s["cth"][0])]


def same(a, b):
    return max(relerr(x, y) for x, y in zip(a, b))


@pytest.mark.parametrize("precision", [P.PREC_FP64, P.PREC_FP32SPLIT])
def test_batch_equals_instances_stepped_alone(precision):
    """Three instances of uneven sizes (different NX, NY, NZ, Ri): two batched
    steps agree with two plain steps of each instance on its own."""
    batched, alone = [], []
    for i, (nx, ny, nz) in enumerate(SIZES):
        p, g, u, th = instance(nx, ny, nz, precision, seed=10 + i, ri=0.05 + 0.1 * i)
        for lst in (batched, alone):
            c = Channel(p, g, 0.01 * (1 + i))
            c.init_from_physical(u, th)
            lst.append(c)
    with Batch(batched) as b:
        b.step(2)
    for c in alone:
        c.step(2)
    for cb, ca in zip(batched, alone):
        assert cb.time_step == ca.time_step == 2
        assert same(state_of(cb), state_of(ca)) < TOL
    for c in batched + alone:
        c.close()


def test_batched_instances_match_oracle():
    """Three FP64 instances, two of one shape with different Ri, Re and dt and
    one of another, two batched steps against the CPU oracle's steps of each
    instance: 1e-10 relative L2 per field (CU2, CU3, CP against the velocity
    and pressure scales, as in the other shear-layer parity tests)."""
    from oracle.oracle import Oracle
    from test_gpu_parity import state_errors

    cases = [((32, 17, 24), 0.05, 1e-3, 0.01), ((32, 17, 24), 0.2, 2e-3, 0.02), ((48, 33, 36), 0.1, 1e-3, 0.015)]
    chans, oracles = [], []
    for i, ((nx, ny, nz), ri, nu, dt) in enumerate(cases):
        p, g, u, th = instance(nx, ny, nz, P.PREC_FP64, seed=40 + i, ri=ri)
        p.nu = nu
        o = Oracle(p, g, dt)
        o.init_from_physical(u, th)
        c = Channel(p, g, dt)
        c.upload([x.copy() for x in o.cu], o.cp.copy(), o.cth.copy())
        chans.append(c)
        oracles.append(o)
    with Batch(chans) as b:
        b.step(2)
    for c, o in zip(chans, oracles):
        o.step(2)
        err = state_errors(c.p, c, o, with_cf=False, scaled=True)
        assert max(err.values()) < 1e-10, err
        c.close()


def test_batch_can_step_again_after_host_upload():
    """Instances stay usable on their own between batch steps: a state uploaded
    by the host is what the next graph launch advances."""
    p, g, u, th = instance(32, 17, 24, P.PREC_FP64, seed=3, ri=0.1)
    a, ref = Channel(p, g, 0.01), Channel(p, g, 0.01)
    a.init_from_physical(u, th)
    ref.init_from_physical(u, th)
    with Batch([a]) as b:
        b.step(1)
        s = ref.download()
        a.upload(s["cu"], s["cp"], s["cth"], s["cf"], s["cfth"])   # back to the initial state
        b.step(1)
    ref.step(1)
    assert same(state_of(a), state_of(ref)) < TOL
    a.close()
    ref.close()


def test_batch_rejects_variable_time_step():
    p, g, u, th = instance(32, 17, 24, P.PREC_FP64, seed=1, ri=0.1)
    p.variable_dt = 1
    p.update_dt = 1
    with Channel(p, g, 0.01) as c:
        with pytest.raises(DiabloError):
            Batch([c])


@pytest.mark.parametrize("precision", [P.PREC_FP64, P.PREC_FP32SPLIT])
def test_autotune_keeps_state_and_results(precision):
    p, g, u, th = instance(64, 33, 48, precision, seed=5, ri=0.1)
    tuned, plain = Channel(p, g, 0.01), Channel(p, g, 0.01)
    tuned.init_from_physical(u, th)
    plain.init_from_physical(u, th)
    before = state_of(tuned)
    chunk, planes = tuned.autotune()
    assert chunk in (4, 8, 16, 32, 64) and planes in (4, 8, 16)
    assert same(state_of(tuned), before) == 0.0          # the state is restored exactly
    tuned.step(2)
    plain.step(2)
    assert same(state_of(tuned), state_of(plain)) < TOL
    tuned.close()
    plain.close()
