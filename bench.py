#!/usr/bin/env python3
"""RK3 steps/s of DIABLO's channel timestep at 512x257x384 on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (diablo_b200.workloads.precision): channel 512x257x384 (NX x NY x
NZ), tanh-stretched y (CS=1.75) on [-1,1], seeded shear-layer fields, one
scalar, fixed dt; the headline number is the FP32-split path (transforms and
products in FP32, solves, state and the projection in FP64).  Besides the
device-timed value the line carries: the all-FP64 path's steps/s and its
difference from the FP32-split state after the same steps, the end-to-end
rate through the C ABI with host buffers, the roofline of the dominant
kernel, a CPU baseline, the SM clocks seen during the timed region, the
batched form, and the constant-Smagorinsky LES step against the FP64 DNS
step.

Multi-GPU: independent replicas, one process per GPU (torchrun); no data-path
collective (the single-instance path does not shard).  The reference arm
times the CPU restatement of the reference (oracle/) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "RK3 steps/s at 512×257×384: FP32-split vs FP64 on 1 B200, err vs FP64 oracle"
FALLBACK_HBM_GBS = 6650.0

# DRAM traffic per launch (dram__bytes_read.sum + dram__bytes_write.sum) per
# y-plane of the grid, from one ncu capture (one pass, nothing replayed) of
# each kernel at 512x257x384, FP32-split; scaled to other grids by their
# number of planes.
TRAFFIC_PER_PLANE = {
    "zinv": (749.9e6 + 513.5e6) / 259.0,
    "products": (562.9e6 + 1052.9e6) / 259.0,
    "zfwd_nl": (1114.5e6 + 359.9e6) / 259.0,
    "column": (2293.7e6 + 1630.3e6) / 259.0,
}


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--grid", default="512,257,384", help="NX,NY,NZ")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-les", action="store_true")
    ap.add_argument("--no-closure", action="store_true")
    ap.add_argument("--closure-snapshots", type=int, default=60)
    ap.add_argument("--closure-steps", type=int, default=20000)
    ap.add_argument("--only", choices=["les", "closure"], default=None,
                    help="run one leg alone and print its JSON (for profiling captures)")
    ap.add_argument("--error-steps", type=int, default=2000,
                    help="last step count at which FP32-split is compared with FP64 (besides 100 and 500)")
    return ap.parse_args()


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# --------------------------------------------------------------------------
# clocks during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            cmd = ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "100"]
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 10:
                continue
            if self.uuid and self.uuid not in parts[1]:
                continue
            rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        smax = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[6 + i].lower() == "active"})
        loaded = [s for s in sm if smax and s > 0.5 * max(smax)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons, "samples": len(rows)}


# --------------------------------------------------------------------------
# algorithmic bytes per launch (per RK substage), the roofline numerators
# --------------------------------------------------------------------------
def algorithmic_bytes(p, prec: str) -> dict:
    nkxp, nkzt, nyp, nz = p.nx // 3 + 1, 2 * (p.nz // 3) + 1, p.ny + 2, p.nz
    nf = 3 + p.n_th
    tb = 8 if prec == "fp32split" else 16          # complex element of the transform path
    A = nkxp * nkzt                                  # dealiased modes per plane
    X = nz * nkxp                                    # x-spectrum entries per plane
    planes_p = p.ny - 1                              # product planes 2..NY
    col = (nf * 16 + (2.0 / 3.0) * nf * 16 + nf * tb + 16    # read CU, CF (rk>1), NL, CP
           + nf * 16 + nf * 16 + 16)                          # write CU, CF, CP
    nq = 2 * nf                                      # product outputs (ikx*Pa + Pflux, Pz per field)
    return {
        "zinv": nf * nyp * (A * 16 + X * tb),
        "products": nf * nyp * X * tb + nq * planes_p * X * tb,
        "zfwd_nl": nq * planes_p * X * tb + nf * planes_p * A * tb,
        "column": col * A * nyp,
    }


# --------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------
def make_channel(w, prec, u=None, th=None):
    from diablo_b200.channel import Channel
    p = w.p.copy()
    p.precision = prec
    c = Channel(p, w.grid, w.dt)
    if u is None:
        u, th = w.initial_fields()
    c.init_from_physical(u, th)
    return c, u, th


def timed_steps(c, steps, torch):
    """Device time of `steps` time steps on the library's stream (ms)."""
    stream = torch.cuda.ExternalStream(c.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    c.synchronize()
    e0.record(stream)
    c.step(steps)
    e1.record(stream)
    c.synchronize()
    return e0.elapsed_time(e1)


def rel_errors(p, a, b):
    from diablo_b200.layout import dealiased
    out = {}
    refs = [dealiased(p, b["cu"][k]) for k in range(3)]
    uscale = float(np.sqrt(sum(np.linalg.norm(r) ** 2 for r in refs)))
    for k in range(3):
        d = np.linalg.norm(dealiased(p, a["cu"][k]) - refs[k])
        out[f"cu{k + 1}"] = float(d / max(np.linalg.norm(refs[k]), 1e-300))
        out[f"cu{k + 1}_vs_velocity_scale"] = float(d / uscale)
    for n in range(p.n_th):
        r = dealiased(p, b["cth"][n])
        out[f"cth{n + 1}"] = float(np.linalg.norm(dealiased(p, a["cth"][n]) - r) / np.linalg.norm(r))
    r = dealiased(p, b["cp"])
    d = np.linalg.norm(dealiased(p, a["cp"]) - r)
    out["cp"] = float(d / max(np.linalg.norm(r), 1e-300))
    out["cp_vs_pressure_scale"] = float(d / (uscale ** 2 / math.sqrt(refs[0].size)))
    return out


def profile_errors(p, a, b):
    """Mean-profile errors (the (0,0) modes of U1 and TH, SAVE_STATS_CHAN's
    ume/thme) relative to the profile's norm."""
    out = {}
    for name, x, y in (("ume", a["cu"][0], b["cu"][0]), ("thme", a["cth"][0], b["cth"][0])):
        px, py = x[:, 0, 0].real, y[:, 0, 0].real
        out[f"mean_profile_{name}"] = float(np.linalg.norm(px - py) / max(np.linalg.norm(py), 1e-300))
    return out


def divergence_norm(p, g, s):
    """Discrete divergence of the downloaded velocity on J = 2..NY-1 (the rows
    REM_DIV_CHAN makes divergence-free), relative L2 against the velocity
    norm: ikx CU1 + (CU2(j+1)-CU2(j))/DYF(j) + ikz CU3."""
    from diablo_b200.layout import dealiased
    nkx, nkz = p.nx // 3, p.nz // 3
    kx = np.arange(nkx + 1) * 2 * np.pi / p.lx
    kz = np.concatenate([np.arange(nkz + 1), -np.arange(nkz, 0, -1)]) * 2 * np.pi / p.lz
    u1, u2, u3 = (dealiased(p, s["cu"][c]) for c in range(3))
    j = np.arange(2, p.ny)
    div = (1j * kx[None, None, :] * u1[j] + (u2[j + 1] - u2[j]) / np.asarray(g.dyf)[j][:, None, None]
           + 1j * kz[None, :, None] * u3[j])
    scale = np.sqrt(sum(np.linalg.norm(x[j]) ** 2 for x in (u1, u2, u3)))
    return float(np.linalg.norm(div) / scale)


def e2e_rate(c, steps, torch):
    """Steps/s through the C ABI with pinned host buffers in the Fortran
    layout: every step uploads CU1..3, CP, CTH, runs the three substages and
    downloads the same arrays."""
    from diablo_b200.layout import fourier_shape
    p = c.p
    shape = fourier_shape(p)
    n = int(np.prod(shape)) * 2

    def pinned():
        t = torch.empty(n, dtype=torch.float64).pin_memory()
        return t, t.numpy().view(np.complex128).reshape(shape)

    bufs = [pinned() for _ in range(4 + max(p.n_th, 1))]
    host = [b[1] for b in bufs]
    c.download_into(host[0:3], host[3], host[4:4 + p.n_th])
    per_field = (p.nx // 3 + 1) * (2 * (p.nz // 3) + 1) * (p.ny + 2) * 16
    nfields = 4 + p.n_th
    c.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        c.upload(host[0:3], host[3], np.stack(host[4:4 + p.n_th]) if p.n_th > 1 else host[4][None])
        c.step(1)
        c.download_into(host[0:3], host[3], host[4:4 + p.n_th])
    el = time.perf_counter() - t0
    return steps / el, nfields * per_field, nfields * per_field


def batched_rates(steps: int, n: int = 64) -> dict:
    """The batched form: n shear layers of uneven sizes (workloads.batched),
    autotuned, advanced together by one CUDA graph per step, against the same
    instances stepped one after another.  Wall clock around synchronised calls
    (the host-side launch cost is part of what batching removes)."""
    from diablo_b200 import workloads
    from diablo_b200.channel import Batch, Channel

    ws = workloads.batched(n)
    chans = []
    for w in ws:
        c = Channel(w.p, w.grid, w.dt)
        u, th = w.initial_fields()
        c.init_from_physical(u, th)
        chans.append(c)
    shapes = [c.autotune() for c in chans]
    for c in chans:                       # one untimed step each
        c.step(1)
        c.synchronize()
    t0 = time.perf_counter()
    for c in chans:
        c.step(steps)
        c.synchronize()
    seq = time.perf_counter() - t0
    with Batch(chans) as b:
        b.step(1)
        t0 = time.perf_counter()
        b.step(steps)
        bat = time.perf_counter() - t0
    cells = sum(w.p.nx * w.p.ny * w.p.nz for w in ws)
    for c in chans:
        c.close()
    return {"instances": n, "steps": steps, "precision": "fp32split",
            "aggregate_instance_steps_per_s": n * steps / bat,
            "sequential_instance_steps_per_s": n * steps / seq,
            "speedup_vs_sequential": seq / bat,
            "grid_points": cells,
            "autotuned_shapes": {f"{a}x{b}": shapes.count((a, b)) for a, b in sorted(set(shapes))},
            "workload": "workloads.batched: NX in {64,96,128}, NY in {65,129}, NZ in {32,64,128}, "
                        "Ri U[0.05,0.3], Re U[500,3000], Pr 1, seeded",
            "timing": "wall clock around synchronised calls"}


def les_rates(w, u, th, steps: int, warmup: int, torch, cpu: bool) -> dict:
    """The constant-Smagorinsky LES branch (LES_MODEL_TYPE 1, CREATE_NEW_FLOW
    off so the model runs from the first step) on the same grid and fields,
    FP64, against the FP64 DNS step; device time on the library's stream.
    With cpu, the oracle's LES step on the bounded y-sample of cpu_sample."""
    from diablo_b200.params import PREC_FP64
    from diablo_b200.channel import Channel

    from diablo_b200.mlp import SgsMlp, init_params

    out = {"workload": "same grid and initial fields, LES=1, CREATE_NEW_FLOW=F, FP64; les: LES_MODEL_TYPE=1 "
                       "(C_s=0.13), les_dynamic: 2, les_closure: 4 with a seeded untrained network whose output "
                       "scale is 1e-3 (the cost does not depend on the weights; at scale 1 its random stresses "
                       "are anti-dissipative somewhere and the run goes non-finite)"}
    for key, les, model in (("dns", 0, 1), ("les", 1, 1), ("les_dynamic", 1, 2), ("les_closure", 1, 4)):
        p = w.p.copy()
        p.precision = PREC_FP64
        p.les, p.les_model_type, p.create_new_flow = les, model, 0
        c = Channel(p, w.grid, w.dt)
        m = None
        if model == 4:
            m = SgsMlp(init_params(7, out_scale=np.full(6, 1e-3)))
            c.set_sgs_mlp(m)
        c.init_from_physical(u, th)
        c.step(warmup)
        n0 = c.kernel_launches()
        ms = timed_steps(c, steps, torch)
        launches = c.kernel_launches() - n0
        out[f"{key}_steps_per_s"] = steps / (ms / 1e3)
        out[f"{key}_ms_per_step"] = ms / steps
        out[f"{key}_gpu_launches_per_step"] = launches / steps
        if key == "les":
            out["nu_t_max"] = float(c.download_nu_t().max())
        c.close()
        if m is not None:
            m.close()
    out["les_cost_vs_dns"] = out["les_ms_per_step"] / out["dns_ms_per_step"]
    out["les_dynamic_cost_vs_dns"] = out["les_dynamic_ms_per_step"] / out["dns_ms_per_step"]
    out["les_closure_cost_vs_dns"] = out["les_closure_ms_per_step"] / out["dns_ms_per_step"]
    # closure inference: MLP flops per resolved point, 2 (11*64 + 2*64*64 + 64*6), over (NY-2) NX NZ points
    # per substage
    fl = 2 * (11 * 64 + 2 * 64 * 64 + 64 * 6) * (w.p.ny - 2) * w.p.nx * w.p.nz * 3
    out["closure_network_gflop_per_step"] = fl / 1e9
    if cpu:
        from diablo_b200 import workloads
        from oracle.oracle import Oracle
        nx, ny, nz = w.p.nx, w.p.ny, w.p.nz
        nys = min(SAMPLE_NY, ny)
        ws = workloads.precision(nx, nys, nz)
        p = ws.p.copy()
        p.les, p.les_model_type, p.create_new_flow = 1, 1, 0
        o = Oracle(p, ws.grid, ws.dt)
        uu, tt = ws.initial_fields()
        o.init_from_physical(uu, tt)
        o.step(1)
        t0 = time.perf_counter()
        o.step(1)
        el = time.perf_counter() - t0
        scale = (ny + 2) / (nys + 2)
        cores = os.cpu_count() or 1
        out["cpu_baseline"] = {"value": 1.0 / (el * scale), "unit": "steps/s", "cores": cores, "kind": "port",
                               "sample": f"1 LES RK3 step of {nx}x{nys}x{nz}, {el:.3f} s scaled x{scale:.2f}; "
                                         f"OpenMP on {cores} threads"}
    return out


def closure_rates(snapshots: int, steps: int) -> dict:
    """The learned closure in a channel LES (closure.channel_les_study):
    Re_tau 180 channel DNS 192x65x192 and LES 64x65x64, `snapshots`
    spectral-cutoff snapshots, `steps` Adam steps of 4096 samples, a-priori
    errors on the held-out snapshots against the best per-plane eddy
    viscosity, then 2000 LES steps with no model, the dynamic model and the
    trained closure against the truncated DNS, profiles averaged every 100
    steps."""
    from diablo_b200 import closure

    out = closure.channel_les_study(snapshots=snapshots, adam_steps=steps)
    flop_per_sample = 3 * 2 * (11 * 64 + 2 * 64 * 64 + 64 * 6)     # forward + backward
    out.update({"train_samples_per_s": steps * 4096 / out["train_seconds"],
                "train_tflops": steps * 4096 * flop_per_sample / out["train_seconds"] / 1e12})
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    from diablo_b200 import build, workloads
    from diablo_b200.params import PREC_FP32SPLIT, PREC_FP64

    build.build()
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    nx, ny, nz = (int(v) for v in args.grid.split(","))
    w = workloads.precision(nx, ny, nz)
    if args.only == "closure":
        out = closure_rates(args.closure_snapshots, args.closure_steps) if rank == 0 else None
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"closure": out}), flush=True)
        return
    if args.only == "les":
        u, th = w.initial_fields()
        out = les_rates(w, u, th, args.steps, args.warmup, torch, cpu=False)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"grid": [nx, ny, nz], "les": out}), flush=True)
        return
    try:
        uuid = str(torch.cuda.get_device_properties(local_rank).uuid)
    except Exception:
        uuid = None

    c32, u, th = make_channel(w, PREC_FP32SPLIT)
    c32.step(args.warmup)
    c32.synchronize()
    if dist:
        dist.barrier()
    n0 = c32.kernel_launches()
    with ClockSampler(uuid) as clk:
        ms = timed_steps(c32, args.steps, torch)
    launches = c32.kernel_launches() - n0
    t = torch.tensor([ms], device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    ms_max = float(t.item())
    value = world * args.steps / (ms_max / 1e3)

    # per-kernel device time of one step (events on the launching stream)
    c32.set_profiling(True)
    c32.step(1)
    ktimes = c32.kernel_times()
    c32.set_profiling(False)

    # all-FP64 path from the same initial fields: rate and state difference
    fp64 = None
    if not args.no_fp64:
        c64, _, _ = make_channel(w, PREC_FP64, u, th)
        c64.step(args.warmup)
        ms64 = timed_steps(c64, args.steps, torch)
        c64.close()
        # error of FP32-split against the all-FP64 path from the same start,
        # after 100, 500 and args.error_steps time steps
        c64, _, _ = make_channel(w, PREC_FP64, u, th)
        c32b, _, _ = make_channel(w, PREC_FP32SPLIT, u, th)
        errs = {}
        done = 0
        for n in sorted({100, 500, args.error_steps}):
            c64.step(n - done)
            c32b.step(n - done)
            done = n
            a32, a64 = c32b.download(), c64.download()
            e = rel_errors(w.p, a32, a64)
            e.update(profile_errors(w.p, a32, a64))
            e["divergence_fp32split"] = divergence_norm(w.p, w.grid, a32)
            e["divergence_fp64"] = divergence_norm(w.p, w.grid, a64)
            errs[f"after_{n}_steps"] = e
        fp64 = {"steps_per_s": args.steps / (ms64 / 1e3), "ms_per_step": ms64 / args.steps, "err": errs}
        c64.close()
        c32b.close()

    e2e = None
    if not args.no_e2e:
        rate, bi, bo = e2e_rate(c32, max(3, min(args.steps, 20)), torch)
        e2e = {"value": world * rate, "unit": "steps/s", "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo}

    batched = None
    if not args.no_batched:
        batched = batched_rates(max(3, min(args.steps, 20)))

    closure_line = None
    if not args.no_closure and rank == 0:
        closure_line = closure_rates(args.closure_snapshots, args.closure_steps)

    les = None
    if not args.no_les:
        les = les_rates(w, u, th, max(3, min(args.steps, 20)), 3, torch,
                        cpu=(rank == 0 and world == 1 and not args.no_cpu_baseline))

    peak, peak_kind = hbm_peak()
    alg = algorithmic_bytes(w.p, "fp32split")
    dom = max(ktimes, key=lambda k: ktimes[k][1])
    dom_launches, dom_ms = ktimes[dom]
    avg_s = dom_ms / dom_launches / 1e3
    achieved = alg.get(dom, 0.0) / avg_s / 1e9 if dom in alg else None
    traffic = TRAFFIC_PER_PLANE[dom] * (w.p.ny + 2) if dom in TRAFFIC_PER_PLANE else None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                "traffic": traffic, "algorithmic_bytes_per_launch": alg.get(dom),
                "avg_launch_ms": avg_s * 1e3}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample(w, nx, ny, nz)

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    kernel_ms = {k: round(v[1] / max(v[0], 1) * 3, 4) for k, v in ktimes.items()}
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 transforms/products + f64 solves/state",
        "data": "synthetic (seeded shear layer, splitmix64/Box-Muller)",
        "config": {"workload": f"channel {nx}x{ny}x{nz}, tanh y CS=1.75, shear layer delta=0.1, FP32-split",
                   "grid": [nx, ny, nz], "n_th": w.p.n_th, "dt": w.dt, "nu": w.p.nu, "ri": w.p.ri[0],
                   "lx": w.p.lx, "lz": w.p.lz, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (each state field 187 MB)"},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
        "clocks": clk.summary(), "fp64": fp64,
        "fp32_split_speedup_vs_fp64": (value / world) / fp64["steps_per_s"] if fp64 else None,
        "fp32split_vs_cpu_baseline": (value / world) / cpu["value"] if cpu else None,
        "fp64_vs_cpu_baseline": fp64["steps_per_s"] / cpu["value"] if (cpu and fp64) else None,
        "kernel_ms_per_step": kernel_ms, "batched": batched, "les": les, "closure": closure_line,
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# CPU: the oracle (a restatement of the reference, OpenMP) on the host cores
# --------------------------------------------------------------------------
SAMPLE_NY = 33


def cpu_sample(w, nx, ny, nz, steps: int = 2):
    """One bounded sample: full NX x NZ planes, a y-subset of SAMPLE_NY
    planes, `steps` RK steps after one untimed step; per-step time scaled by
    (NY+2)/(SAMPLE_NY+2), the work of the path being proportional to the
    number of planes."""
    from diablo_b200 import workloads
    from oracle.oracle import Oracle

    nys = min(SAMPLE_NY, ny)
    ws = workloads.precision(nx, nys, nz)
    o = Oracle(ws.p, ws.grid, ws.dt)
    u, th = ws.initial_fields()
    o.init_from_physical(u, th)
    o.step(1)
    t0 = time.perf_counter()
    o.step(steps)
    el = (time.perf_counter() - t0) / steps
    scale = (ny + 2) / (nys + 2)
    cores = os.cpu_count() or 1
    return {"value": 1.0 / (el * scale), "unit": "steps/s", "cores": cores, "kind": "port",
            "sample": f"{steps} RK3 steps of {nx}x{nys}x{nz} (full x-z planes, {nys + 2} of {ny + 2} y-planes), "
                      f"{el:.3f} s/step scaled x{scale:.2f} to {ny + 2} planes; OpenMP on {cores} threads"}


def run_reference(args, rank):
    """The reference's algorithm on the host cores: the oracle (a line-by-line
    FP64 restatement of RK_CHAN_1 and its routines, OpenMP over y-planes) on
    the full workload -- every y-plane of the grid -- for W untimed and K
    timed RK3 steps.  The Fortran reference itself needs gfortran, MPI, HDF5
    and FFTW, none of which this image has."""
    if rank != 0:
        return
    from diablo_b200 import workloads
    from oracle.oracle import Oracle, build as build_oracle

    build_oracle()
    nx, ny, nz = (int(v) for v in args.grid.split(","))
    w = workloads.precision(nx, ny, nz)
    p = w.p.copy()
    from diablo_b200.params import PREC_FP64
    p.precision = PREC_FP64
    o = Oracle(p, w.grid, w.dt)
    u, th = w.initial_fields()
    o.init_from_physical(u, th)
    o.step(args.warmup)
    t0 = time.perf_counter()
    o.step(args.steps)
    el = (time.perf_counter() - t0) / args.steps
    value = 1.0 / el
    cores = os.cpu_count() or 1
    sample = (f"the whole workload: {args.steps} RK3 steps of {nx}x{ny}x{nz} (all {ny + 2} y-planes) after "
              f"{args.warmup} untimed; OpenMP on {cores} threads")
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded shear layer)", "impl": "reference",
        "config": {"workload": f"channel {nx}x{ny}x{nz}, tanh y CS=1.75, shear layer delta=0.1",
                   "grid": [nx, ny, nz], "parallelism": "cpu"},
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "timed_region_s": el * args.steps,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
