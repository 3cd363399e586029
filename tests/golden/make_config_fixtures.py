"""Oracle fixtures of the wall-bounded channel (192x129x160) and the
precision workload (512x257x384), for the GPU parity tests at full size.

    python tests/golden/make_config_fixtures.py [--which channel|precision|both] [--threads N]

Each run starts from the workload's seeded physical fields, applies the
oracle's own initialisation (transform, APPLY_BC_VEL, REM_DIV_CHAN) and
advances the CPU FP64 oracle by the stated number of RK3 steps.  A full
state at these sizes is tens to hundreds of MB, so the fixture keeps what a
comparison needs in a few MB:

* ``plane_norm``   -- [field][J]: L2 norm of each plane's dealiased block
                      (fields CU1, CU2, CU3, CTH, CP);
* ``low_modes``    -- [field][J][kz][kx]: the modes |kx| <= K, |kz| <= K of
                      every plane (kz in packed order: 0..K, then -K..-1);
* ``mean``         -- [field][J]: the (0,0) mode, real part (the mean profiles);
* ``delta_t``      -- DELTA_T after every step (CFL-adaptive runs);
* ``time``, ``steps``, ``k``.

The oracle runs on the CPU; at 512x257x384 a step takes about a minute on
8 threads, so the precision fixture takes 1 to 2 hours.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

K_LOW = 6
FIXTURES = {
    # name: (workload factory arguments, steps)
    "channel": ((192, 129, 160), 200),
    "precision": ((512, 257, 384), 100),
}


def low_mode_index(p, k: int):
    """Packed kz indices of |kz| <= k and kx indices 0..k."""
    kz = list(range(0, k + 1)) + list(range(p.tnkz + 1 - k, p.tnkz + 1))
    return np.array(kz), np.arange(k + 1)


def summarise(p, fields, k: int) -> dict:
    from diablo_b200.layout import dealiased
    kz, kx = low_mode_index(p, k)
    norms, lows, means = [], [], []
    for f in fields:
        b = dealiased(p, f)
        norms.append(np.sqrt((np.abs(b) ** 2).sum(axis=(1, 2))))
        lows.append(b[:, kz][:, :, kx].copy())
        means.append(b[:, 0, 0].real.copy())
    return {"plane_norm": np.array(norms), "low_modes": np.array(lows), "mean": np.array(means)}


def state_fields(s) -> list:
    """CU1, CU2, CU3, CTH(1), CP from an oracle or a downloaded GPU state."""
    if isinstance(s, dict):
        return [s["cu"][0], s["cu"][1], s["cu"][2], s["cth"][0], s["cp"]]
    return [s.cu[0], s.cu[1], s.cu[2], s.cth[0], s.cp]


def workload(name: str):
    from diablo_b200 import params as P, workloads
    dims, steps = FIXTURES[name]
    if name == "channel":
        return workloads.channel(*dims, precision=P.PREC_FP64), steps
    return workloads.precision(*dims, prec=P.PREC_FP64), steps


def make(name: str, threads: int) -> str:
    from oracle.oracle import Oracle, set_threads

    set_threads(threads)
    w, steps = workload(name)
    u, th = w.initial_fields()
    o = Oracle(w.p, w.grid, w.dt)
    o.init_from_physical(u, th)
    dts = []
    t0 = time.time()
    for s in range(steps):
        o.step()
        t, dt, ts, _ = o.time()
        dts.append(dt)
        if s % 10 == 9:
            print(f"{name}: step {s + 1}/{steps}, {time.time() - t0:.0f} s", flush=True)
    t, dt, ts, _ = o.time()
    out = summarise(w.p, state_fields(o), K_LOW)
    path = os.path.join(HERE, f"oracle_{name}_{'x'.join(map(str, FIXTURES[name][0]))}_{steps}steps.npz")
    np.savez_compressed(path, **out, delta_t=np.array(dts), time=t, steps=steps, k=K_LOW,
                        grid=np.array(FIXTURES[name][0]))
    print(f"{name}: wrote {path} ({os.path.getsize(path) / 1e6:.1f} MB) in {time.time() - t0:.0f} s", flush=True)
    return path


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--which", choices=["channel", "precision", "both"], default="both")
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    a = ap.parse_args()
    for name in (["channel", "precision"] if a.which == "both" else [a.which]):
        make(name, a.threads)


if __name__ == "__main__":
    main()
