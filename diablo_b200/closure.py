"""Training and a-priori evaluation of the learned subgrid-stress closure.

The closure (diablo_b200.mlp) is trained on snapshots of this solver's own
DNS: every `every` steps the state is filtered by a `width` x `width` top-hat
in x and z on the GPU (Channel.sgs_samples), which gives the resolved
velocity gradients (divided by their norm G), y+ and the filter width Delta
as features and the subfilter stresses tau_ij = bar(u_i u_j) - ubar_i
ubar_j divided by Delta^2 G^2 as targets; this dimensionless form lets
snapshots of a decaying flow weigh alike.  Snapshots are
split 80/20 with a seeded permutation; the network is trained by the
library's own kernels (diablo_mlp_train) on the training snapshots, whose
samples are drawn with probabilities proportional to s^2 = (Delta^2 G^2)^2
so that the dimensionless loss weighs samples as the error of the
dimensional stresses does (otherwise the quiescent regions, where tau/s is
noise over a small G^2, would dominate it).

For an LES, the stresses the model must supply are those of the filter the
LES itself applies: the spectral cutoff at its resolved modes, not a
top-hat.  cutoff_snapshots collects those: the DNS state truncated to the
LES modes is put on an LES-grid instance, whose sampler (width 1) gives the
features the LES computes at run time at every LES point, and the targets
tau_ij = T(u_i u_j) - T(T(u_i) T(u_j)) (T the truncation) are formed on the
host by FFT from the DNS velocity.  Trained on these, the closure improves
the LES a posteriori (a_posteriori); trained on top-hat stresses, which are
larger than the cutoff's at the same width, it over-dissipates.

The method without the network is an eddy viscosity: tau^d_ij = -2 C Delta^2
|S| S_ij for the deviatoric stresses.  Its a-priori error is bounded below
by the best coefficient for each y-plane fitted by least squares to the
training snapshots' (dimensional) stresses -- the best any such model, the dynamic one
included, can do at a plane -- and that fit is the baseline the network is
compared with on the held-out snapshots.
"""
from __future__ import annotations

import time as _time
from dataclasses import dataclass, field

import numpy as np

from .channel import Channel
from .layout import dealiased
from .mlp import NIN, NOUT, SgsMlp, init_params, normalisation

_PAIRS = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]


@dataclass
class Snapshots:
    x: np.ndarray            # [n][11] dimensionless features
    t: np.ndarray            # [n][6] dimensionless subfilter stresses
    s: np.ndarray            # [n] stress scales Delta^2 G^2
    snap: np.ndarray         # [n] snapshot index of each sample
    per_snapshot: int
    seconds: float = 0.0


def dns_snapshots(p, grid, dt, u, th, count: int, every: int, warmup: int = 0, width: int = 3,
                  stride: int = 1) -> Snapshots:
    """Run the DNS on the GPU and collect `count` filtered snapshots, one
    every `every` steps after `warmup` steps."""
    t0 = _time.perf_counter()
    xs, ts, ss = [], [], []
    with Channel(p, grid, dt) as c:
        c.init_from_physical(u, th)
        c.step(warmup)
        for _ in range(count):
            c.step(every)
            x, t, s = c.sgs_samples(width, stride)
            xs.append(x)
            ts.append(t)
            ss.append(s)
    m = xs[0].shape[0]
    snap = np.repeat(np.arange(count), m)
    return Snapshots(np.concatenate(xs), np.concatenate(ts), np.concatenate(ss), snap, m,
                     _time.perf_counter() - t0)


def _to_physical(spec: np.ndarray, nx: int, nz: int) -> np.ndarray:
    """Dealiased Fourier block [planes][2 nkz + 1][nkx + 1] (kz = -k at index
    2 nkz + 1 - k, coefficients normalised by NX NZ) to physical values
    [planes][nz][nx] on an nx x nz grid: the plain sum over the modes."""
    nkz, nkx = (spec.shape[1] - 1) // 2, spec.shape[2] - 1
    full = np.zeros((spec.shape[0], nz, nx // 2 + 1), dtype=np.complex128)
    full[:, : nkz + 1, : nkx + 1] = spec[:, : nkz + 1]
    for k in range(1, nkz + 1):
        full[:, nz - k, : nkx + 1] = spec[:, 2 * nkz + 1 - k]
    return np.fft.irfft(np.fft.ifft(full, axis=1, norm="forward"), n=nx, axis=2, norm="forward")


def _to_fourier(f: np.ndarray, nkx: int, nkz: int) -> np.ndarray:
    """Physical [planes][nz][nx] to the dealiased block of modes |kx| <= nkx,
    |kz| <= nkz (the inverse of _to_physical on those modes)."""
    nz = f.shape[1]
    full = np.fft.fft(np.fft.rfft(f, axis=2, norm="forward"), axis=1, norm="forward")
    out = np.zeros((f.shape[0], 2 * nkz + 1, nkx + 1), dtype=np.complex128)
    out[:, : nkz + 1] = full[:, : nkz + 1, : nkx + 1]
    for k in range(1, nkz + 1):
        out[:, 2 * nkz + 1 - k] = full[:, nz - k, : nkx + 1]
    return out


def cutoff_stresses(p, q, s: dict) -> np.ndarray:
    """Subgrid stresses of the spectral cutoff that an LES on q's grid
    resolves (the modes coarsen keeps), at q's physical points of planes
    J = 2..NY-1 in the sampler's order [J][z][x][6]:
    tau_ij = T(u_i u_j) - T(T(u_i) T(u_j)), T the truncation to the LES modes
    and u the DNS velocity of state s (U2 averaged to GYF, as the sampler
    does).  The DNS products are formed on p's grid, where the 2/3 rule
    keeps their aliases off the LES modes; the resolved products on q's
    grid, likewise."""
    ny = p.ny
    nkx, nkz = q.nx // 3, q.nz // 3
    cu = s["cu"]

    def dns(k, lo, hi):
        return _to_physical(dealiased(p, cu[k])[lo:hi], p.nx, p.nz)

    def les(k, lo, hi):
        return _to_physical(dealiased(p, cu[k])[lo:hi][:, _les_kz(p, nkz)][:, :, : nkx + 1], q.nx, q.nz)

    u = [dns(0, 2, ny), 0.5 * (dns(1, 2, ny) + dns(1, 3, ny + 1)), dns(2, 2, ny)]
    uc = [les(0, 2, ny), 0.5 * (les(1, 2, ny) + les(1, 3, ny + 1)), les(2, 2, ny)]
    out = np.empty((ny - 2, q.nz, q.nx, 6), dtype=np.float64)
    for n, (a, b) in enumerate(_PAIRS):
        full = _to_physical(_to_fourier(u[a] * u[b], nkx, nkz), q.nx, q.nz)
        res = _to_physical(_to_fourier(uc[a] * uc[b], nkx, nkz), q.nx, q.nz)
        out[..., n] = full - res
    return out


def _les_kz(p, nkz: int) -> np.ndarray:
    """Indices, in p's dealiased kz order, of the modes |kz| <= nkz in the
    same order for the smaller grid (0..nkz, then -nkz..-1)."""
    tf = 2 * (p.nz // 3)
    return np.array(list(range(nkz + 1)) + [tf + 1 - k for k in range(nkz, 0, -1)])


def cutoff_snapshots(p, grid, dt, u, th, count: int, every: int, warmup: int = 0, factor: int = 3,
                     start: dict | None = None) -> Snapshots:
    """Run the DNS on the GPU and collect `count` snapshots for an LES on the
    grid `factor` times coarser in x and z, one every `every` steps after
    `warmup`: the features at every LES point of planes 2..NY-1 are those
    the LES computes at run time (Channel.sgs_samples with width 1 on an LES
    grid instance holding the DNS state truncated to the LES modes), and the
    targets are the spectral-cutoff stresses (cutoff_stresses) in the same
    dimensionless form.  The DNS starts from `start` (a downloaded state)
    when given, else from the physical fields u, th."""
    from .params import PREC_FP64

    t0 = _time.perf_counter()
    q = p.copy()
    q.nx, q.nz = p.nx // factor, p.nz // factor
    q.precision = PREC_FP64
    xs, ts, ss = [], [], []
    with Channel(p, grid, dt) as c, Channel(q, grid, dt) as lc:
        if start is None:
            c.init_from_physical(u, th)
        else:
            c.upload(start["cu"], start["cp"], start["cth"] if p.n_th else None)
        c.step(warmup)
        for _ in range(count):
            c.step(every)
            s = c.download()
            lc.upload([coarsen(p, s["cu"][k], q) for k in range(3)], coarsen(p, s["cp"], q),
                      np.stack([coarsen(p, s["cth"][n], q) for n in range(p.n_th)]) if p.n_th else None)
            x, _, sc = lc.sgs_samples(1, 1)
            tau = cutoff_stresses(p, q, s).reshape(-1, 6)
            inv = np.where(sc > 0, 1.0 / np.maximum(sc.astype(np.float64), 1e-300), 0.0)
            xs.append(x)
            ts.append((tau * inv[:, None]).astype(np.float32))
            ss.append(sc)
    m = xs[0].shape[0]
    snap = np.repeat(np.arange(count), m)
    return Snapshots(np.concatenate(xs), np.concatenate(ts), np.concatenate(ss), snap, m,
                     _time.perf_counter() - t0)


def split(count: int, seed: int, frac: float = 0.8):
    """Seeded split of snapshot indices into training and held-out sets."""
    perm = np.random.default_rng(seed).permutation(count)
    k = int(round(frac * count))
    return np.sort(perm[:k]), np.sort(perm[k:])


def deviatoric(t: np.ndarray) -> np.ndarray:
    d = np.array(t, dtype=np.float64, copy=True)
    tr = (d[:, 0] + d[:, 1] + d[:, 2]) / 3.0
    d[:, :3] -= tr[:, None]
    return d


def _norm2(a: np.ndarray) -> np.ndarray:
    """Squared tensor norm with the off-diagonal pairs counted twice."""
    return np.sum(a[:, :3] ** 2, axis=1) + 2.0 * np.sum(a[:, 3:] ** 2, axis=1)


def eddy_viscosity_basis(x: np.ndarray) -> np.ndarray:
    """m_ij = -2 Delta^2 |S| S_ij / (Delta^2 G^2) from the dimensionless
    features (S_ij the symmetric part of the gradient g_ij / G, |S| =
    sqrt(2 S_ij S_ij)): the eddy viscosity's stresses in the targets' form."""
    g = np.asarray(x[:, :9], dtype=np.float64).reshape(-1, 3, 3)
    s = 0.5 * (g + g.transpose(0, 2, 1))
    sv = np.stack([s[:, a, b] for a, b in _PAIRS], axis=1)
    smag = np.sqrt(2.0 * _norm2(sv))
    return -2.0 * smag[:, None] * sv


def dissipation(x: np.ndarray, t: np.ndarray) -> np.ndarray:
    """Subgrid dissipation Pi = -tau_ij S_ij of dimensionless stresses t from
    the dimensionless gradient features x (S_ij the symmetric part of g_ij)."""
    g = np.asarray(x[:, :9], dtype=np.float64).reshape(-1, 3, 3)
    s = 0.5 * (g + g.transpose(0, 2, 1))
    sv = np.stack([s[:, a, b] for a, b in _PAIRS], axis=1)
    c = np.array([1.0, 1.0, 1.0, 2.0, 2.0, 2.0])
    return -np.sum(c * sv * np.asarray(t, dtype=np.float64), axis=1)


def plane_coefficients(x: np.ndarray, t: np.ndarray, s: np.ndarray) -> dict:
    """Least-squares C for each plane (keyed by its y+ feature) from samples,
    minimising the error of the dimensional stresses (weights s^2)."""
    m = eddy_viscosity_basis(x)
    d = deviatoric(t)
    w = np.asarray(s, dtype=np.float64) ** 2
    num = w * (np.sum(d[:, :3] * m[:, :3], axis=1) + 2.0 * np.sum(d[:, 3:] * m[:, 3:], axis=1))
    den = w * _norm2(m)
    key = np.round(np.asarray(x[:, 9], dtype=np.float64), 6)
    out = {}
    for k in np.unique(key):
        sel = key == k
        out[k] = float(num[sel].sum() / den[sel].sum()) if den[sel].sum() > 0 else 0.0
    return out


def eddy_viscosity_predict(x: np.ndarray, coef: dict) -> np.ndarray:
    key = np.round(np.asarray(x[:, 9], dtype=np.float64), 6)
    c = np.array([coef.get(k, 0.0) for k in key])
    return c[:, None] * eddy_viscosity_basis(x)


def relative_error(pred: np.ndarray, true: np.ndarray, s: np.ndarray) -> float:
    """Tensor-norm relative L2 error over all samples of the dimensional
    stresses (dimensionless values times the scales s)."""
    s = np.asarray(s, dtype=np.float64)[:, None]
    return float(np.sqrt(_norm2((pred - true) * s).sum() / _norm2(true * s).sum()))


@dataclass
class ClosureReport:
    train_samples: int
    test_samples: int
    train_seconds: float
    losses: np.ndarray
    mlp_test_error: float             # full tau, held-out snapshots
    mlp_test_error_deviatoric: float
    eddy_viscosity_test_error: float  # deviatoric, best per-plane coefficient
    params: np.ndarray = field(repr=False, default=None)

    def summary(self) -> dict:
        # mini-batch losses of heavy-tailed targets are noisy: window means
        return {"train_samples": self.train_samples, "test_samples": self.test_samples,
                "train_seconds": self.train_seconds, "final_loss": float(np.mean(self.losses[-1000:])),
                "first_loss": float(np.mean(self.losses[:10])),
                "loss_windows": "first: mean of the first 10 mini-batches; final: of the last 1000",
                "mlp_test_error": self.mlp_test_error,
                "mlp_test_error_deviatoric": self.mlp_test_error_deviatoric,
                "eddy_viscosity_best_plane_fit_test_error": self.eddy_viscosity_test_error}


def train_and_evaluate(data: Snapshots, seed: int, steps: int, batch: int = 1024, lr: float = 2e-3,
                       frac: float = 0.8, max_stats: int = 2_000_000, diss_weight: float = 0.0) -> ClosureReport:
    """Train on the training snapshots (seeded split and shuffle) and compare
    the network with the best per-plane eddy viscosity on the held-out ones.
    The normalisation, the per-plane coefficients and the held-out errors use
    seeded subsamples of at most max_stats samples (training uses all).
    diss_weight > 0 adds the subgrid-dissipation term to the loss
    (SgsMlp.set_dissipation_weight), measured against the spread of the
    training targets' dissipation: the weight passed on is
    diss_weight / var(Pi(t)), so that diss_weight = 1 weighs a dissipation
    error of one standard deviation like a stress error of one output scale."""
    count = int(data.snap.max()) + 1
    tr, te = split(count, seed, frac)
    mtr = np.isin(data.snap, tr)
    xtr, ttr, strn = data.x[mtr], data.t[mtr], data.s[mtr]
    xte, tte, ste = data.x[~mtr], data.t[~mtr], data.s[~mtr]
    w = strn.astype(np.float64) ** 2
    draw = np.random.default_rng(seed + 1).choice(xtr.shape[0], xtr.shape[0], replace=True, p=w / w.sum())
    xtr, ttr, strn = xtr[draw], ttr[draw], strn[draw]
    rng = np.random.default_rng(seed + 2)
    sub = lambda n: slice(None) if n <= max_stats else np.sort(rng.choice(n, max_stats, replace=False))
    st = sub(xtr.shape[0])
    se = sub(xte.shape[0])
    mean, scale, osc = normalisation(xtr[st].astype(np.float64), ttr[st].astype(np.float64))
    t0 = _time.perf_counter()
    with SgsMlp(init_params(seed, mean, scale, osc)) as m:
        if diss_weight:
            pi_t = dissipation(xtr[st], ttr[st])
            m.set_dissipation_weight(diss_weight / max(float(np.var(pi_t)), 1e-300))
        losses = m.train(xtr, ttr, batch, steps, lr)
        train_seconds = _time.perf_counter() - t0
        pred = m.forward(xte[se]).astype(np.float64)
        params = m.params()
    coef = plane_coefficients(xtr[st], ttr[st], strn[st])
    ev = eddy_viscosity_predict(xte[se], coef)
    tsel = tte[se].astype(np.float64)
    ssel = ste[se]
    dte = deviatoric(tsel)
    return ClosureReport(xtr.shape[0], xte.shape[0], train_seconds, losses,
                         relative_error(pred, tsel, ssel),
                         relative_error(deviatoric(pred), dte, ssel),
                         relative_error(ev, dte, ssel), params)


assert NIN == 11 and NOUT == 6


# --- a-posteriori comparison ---------------------------------------------------

def coarsen(p_fine, a: np.ndarray, p_coarse) -> np.ndarray:
    """Spectral truncation of a Fortran-layout Fourier array to the modes a
    coarser x-z grid keeps (same y grid); the coefficients are normalised by
    NX NZ on both grids, so they carry over unchanged."""
    from .layout import new_fourier
    out = new_fourier(p_coarse)
    nkx, nkz = p_coarse.nx // 3, p_coarse.nz // 3
    tf, tc = 2 * (p_fine.nz // 3), 2 * nkz
    out[:, : nkz + 1, : nkx + 1] = a[:, : nkz + 1, : nkx + 1]
    for k in range(1, nkz + 1):
        out[:, tc + 1 - k, : nkx + 1] = a[:, tf + 1 - k, : nkx + 1]
    return out


def _profiles(stats: np.ndarray) -> dict:
    from .channel import STAT_INDEX
    return {k: stats[STAT_INDEX[k]] for k in ("ume", "urms", "vrms", "wrms", "uv")}


def a_posteriori(p, grid, dt, u, th, steps: int, params: np.ndarray, factor: int = 3, start: dict | None = None,
                 average_every: int = 0) -> dict:
    """DNS on p's grid and LES on the grid coarsened `factor` times in x and
    z, from the DNS's initial state truncated to the LES modes, `steps`
    steps each; mean-velocity and Reynolds-stress profiles of each LES (no
    model, the dynamic model, the closure with `params`) against the
    filtered DNS (the DNS state truncated the same way) as relative L2
    errors over the planes.  The initial state is `start` (a downloaded DNS
    state) when given, else the physical fields u, th.  With average_every
    > 0 the profiles are means over the states every average_every steps
    (a turbulent flow's instantaneous plane averages fluctuate); else those
    of the final states.  p's dt must be fixed, so that the runs meet at the
    same times."""
    from .mlp import SgsMlp
    from .params import PREC_FP64

    q = p.copy()
    q.nx, q.nz = p.nx // factor, p.nz // factor
    q.les, q.create_new_flow = 1, 0
    q.precision = PREC_FP64          # the LES branch runs in FP64
    chunk = average_every if average_every > 0 else steps

    def coarse_channel(s, model):
        r = q.copy()
        if model == 0:
            r.les = 0
        else:
            r.les_model_type = model
        ch = Channel(r, grid, dt)
        ch.upload([coarsen(p, s["cu"][k], q) for k in range(3)], coarsen(p, s["cp"], q),
                  np.stack([coarsen(p, s["cth"][n], q) for n in range(p.n_th)]) if p.n_th else None)
        return ch

    def mean_profiles(samples):
        return {k: np.mean([smp[k] for smp in samples], axis=0) for k in samples[0]}

    targets = []
    with Channel(p, grid, dt) as c:
        if start is None:
            c.init_from_physical(u, th)
        else:
            c.upload(start["cu"], start["cp"], start["cth"] if p.n_th else None)
        s0 = c.download()
        t0 = _time.perf_counter()
        done = 0
        while done < steps:
            n = min(chunk, steps - done)
            c.step(n)
            done += n
            with coarse_channel(c.download(), 0) as ref:
                targets.append(_profiles(ref.stats()))
        c.synchronize()
        dns_seconds = _time.perf_counter() - t0
    target = mean_profiles(targets)
    out = {"dns_grid": [p.nx, p.ny, p.nz], "les_grid": [q.nx, q.ny, q.nz], "steps": steps, "dt": dt,
           "dns_seconds": dns_seconds, "profile_samples": len(targets)}
    for name, model in (("no_model", 0), ("dynamic", 2), ("closure", 4)):
        ch = coarse_channel(s0, model)
        m = None
        if model == 4:
            m = SgsMlp(params)
            ch.set_sgs_mlp(m)
        t0 = _time.perf_counter()
        samples, done = [], 0
        while done < steps:
            n = min(chunk, steps - done)
            ch.step(n)
            done += n
            samples.append(_profiles(ch.stats()))
        ch.synchronize()
        el = _time.perf_counter() - t0
        prof = mean_profiles(samples)
        ch.close()
        if m is not None:
            m.close()
        err = {}
        for k, ref_prof in target.items():
            d = np.linalg.norm(prof[k] - ref_prof)
            err[k] = float(d / max(np.linalg.norm(ref_prof), 1e-300)) if np.isfinite(d) else float("inf")
        out[name] = {"profile_errors": err, "seconds": el}
    return out


def channel_les_study(snapshots: int = 60, every: int = 30, spin: int = 20000, adam_steps: int = 20000,
                      les_steps: int = 2000, seed: int = 42, dt: float = 1.2e-3) -> dict:
    """The learned closure in a channel LES: turbulent channel at Re_tau 180,
    DNS on 192x65x192 (FP32-split, fixed dt), LES on 64x65x64 (the DNS grid
    coarsened 3 times in x and z, same y grid).  The DNS starts from
    ics.tripped_poiseuille and runs `spin` steps to a turbulent state S;
    after 4000 more steps `snapshots` cutoff snapshots are taken one every
    `every` steps (cutoff_snapshots), the closure is trained on them
    (`adam_steps` Adam steps of 4096, seeded 80/20 split by snapshot), and
    from S -- before the training window -- the LES with no model, the
    dynamic model and the closure run `les_steps` steps beside the DNS, with
    the profiles averaged every 100 steps (a_posteriori)."""
    from . import grid as G, ics, params as P

    p = P.turbulent_channel(192, 65, 192, re_tau=180.0, precision=P.PREC_FP32SPLIT, variable_dt=False)
    g = G.channel_grid(G.create_grid(1, 65, 2.0, 1.75))
    u, th = ics.tripped_poiseuille(p, g, 18.0, seed=5)
    t0 = _time.perf_counter()
    with Channel(p, g, dt) as c:
        c.init_from_physical(u, th)
        c.step(spin)
        start = c.download()
    spin_seconds = _time.perf_counter() - t0
    data = cutoff_snapshots(p, g, dt, None, None, count=snapshots, every=every, warmup=4000, start=start)
    rep = train_and_evaluate(data, seed=seed, steps=adam_steps, batch=4096, lr=2e-3)
    out = rep.summary()
    out.update({"snapshots": snapshots, "snapshot_every": every, "snapshot_seconds": data.seconds,
                "spin_up_steps": spin, "spin_up_seconds": spin_seconds, "adam_steps": adam_steps, "batch": 4096,
                "workload": f"channel Re_tau 180: DNS 192x65x192 FP32-split, LES 64x65x64, dt {dt}; tripped "
                            f"Poiseuille, {spin} spin-up steps; {snapshots} spectral-cutoff snapshots one every "
                            f"{every} steps after 4000 more; seeded 80/20 split by snapshot"})
    out["a_posteriori"] = a_posteriori(p, g, dt, None, None, les_steps, rep.params, start=start, average_every=100)
    return out
