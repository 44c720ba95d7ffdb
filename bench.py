#!/usr/bin/env python
"""Throughput of the ICLS per-timestep hot path on B200, in Mcell-steps/s.

One "step" is one full main-loop iteration (src/main.f90:107-210 of the
reference): level-set advection/reinitialisation/mass correction for every
drop, materials, AB2 predictor, Poisson RHS with GFM jumps, FFT/Thomas
pressure solve, projection, pressure update.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --drift-steps 1000 [--inflate-step S] [--mass-threshold T] [--dt DT] [--gain-one]
                                                  (volume record, no timing)
  python bench.py --rise-steps 2000 [--gain-one] [--workload rising_bubble_128]
                                                  (rising bubble: centroid, rise velocity, drift)

Default workload: the 256^3 box with 48 seeded drops.  The headline value is
the FP32 form with the learned curvature in the loop (FP64 kept for the
Poisson solve, pressures, volume integral and GFM jumps), whose network is
first trained on the GPU (4M seeded samples, 20 epochs); the same line
carries the plain FP64 path on the same workload (value, per-kernel shares,
roofline), the FP32 form with the plain stencil, and the form's errors
against the FP64 run and against the analytic curvature of the seeded
spheres.  Inputs (several GB of level sets and fields) are far larger than
the 126 MB L2, so no flush is needed between steps.  Under torchrun each
rank runs its own replica of the workload (the path is not sharded across
GPUs), the timed region is bracketed by a barrier and synchronisation on
every rank, and the reported time is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (ROOT, os.path.join(ROOT, "icls-release_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

METRIC = "Mcell-steps/s at 256\u00b3: FP32+learned-\u03ba vs plain FP64 on B200, at stated vol/\u03ba error"
UNIT = "Mcell-steps/s"


# ------------------------------------------------------------------ workload
MULTI_DROP = {"multi_drop_256_48": dict(n=256, ndrop=48, seed=2024),
              "multi_drop_256_4": dict(n=256, ndrop=4, seed=2024),
              "multi_drop_128_12": dict(n=128, ndrop=12, seed=2024, rmin=0.06, rmax=0.12)}


def make_workload(name):
    from icls_gpu.config import combined, multi_drop, rising_bubble, static_drop
    if name in MULTI_DROP:
        return multi_drop(**MULTI_DROP[name])
    if name.endswith("_walls") and name[:-len("_walls")] in MULTI_DROP:
        # the same kind of box between walls at y = 0 and y = ly (BC_in_y =
        # 'Walls'), its drops seeded clear of them as of the z walls
        wl = multi_drop(**MULTI_DROP[name[:-len("_walls")]], y_walls=True)
        wl.name = name
        return wl
    if name == "static_drop_64":
        return static_drop(64)
    if name == "static_drop_256":  # one drop: full-size field kernels with a few GB on the device
        return static_drop(256)
    if name == "rising_bubble_128":
        return rising_bubble(128)
    if name == "combined_96_12":  # the same kinds of input at 96^3 (16 x 6), 12 drops of 7-10 cells
        return combined(96, 12, rmin=0.07, rmax=0.1)
    raise SystemExit("unknown workload %s" % name)


def initial_state(wl):
    from icls_gpu.config import init_drops, init_drops_boxed, workload_velocity
    cfg = wl.cfg
    if wl.all_images and cfg.itot >= 128:
        ls = init_drops_boxed(cfg, wl.centres, wl.radii)
    else:
        ls = init_drops(cfg, wl.centres, wl.radii, wl.all_images)
    u, v, w = workload_velocity(wl)
    return ls, u, v, w


# -------------------------------------------------- algorithmic byte model
# Compulsory HBM values of one launcher scope (the unit the per-kernel device
# timer brackets), as (bulk values, FP64 values, unit): bulk values are the
# form's field type (8 B in plain FP64, 4 B in the FP32 form: velocities,
# materials, AB2 history, level sets, and the pressures pnew, pold with the
# face jumps p_x,y,z and their old values), FP64 values stay 8 B in both (the
# Poisson work array p and the jump Laplacian p_jump).  Units: N interior
# cells, B band cells of all drops (one batched scope covers every drop),
# S |phi| <= 2dz shell cells of all drops.
ALG_VALUES = {
    "ab2": (24, 0, "N"),             # u,v,w,miu,rho_uvw,duold x3,pnew,pold,p_xyz,p_xyz_old -> dudt x3,duold x3
    "correc": (12, 1, "N"),          # dudt x3,p_xyz | p -> u,v,w, ucc,vcc,wcc
    "fillps": (3, 2, "N"),           # dudt x3 | pjump -> p
    "solver2d": (3, 2, "N"),         # dudt x3 | p_jump -> p: fillps folded into the first pass (the transposes and sweeps between are not compulsory)
    "pressure_update": (3, 1, "N"),  # pnew | p -> pnew, pold
    "stream_vel": (1, 0, "N"),
    "materials_final": (6, 0, "N"),  # jiemian -> miu, rho, rho_uvw
    "tube": (2, 0, "B"),             # phi -> clipped phi on the band
    "adv_stage": (17.0 / 3.0, 0, "B"),  # one RK3 stage on the band
    "heaviside": (1, 0, "B"),
    "curvature": (2, 0, "S"),
    "recurvature": (2, 0, "S"),
    "jumps": (8, 2, "S"),            # phi, kappa_re, p_xyz (read+write) | p_jump (read+write)
}


# tensor-core FLOPs of one network evaluation: the three BF16 tile products
# (layer 1 takes its 32 inputs as hi + lo pairs, K = 64)
MLP_FLOPS_PER_CELL = 2 * (128 * 64 + 128 * 128 + 64 * 128)

# DRAM bytes (read + write) of one launch of the dominant kernel at 256^3,
# (kernel, FP32 form) -> bytes: ncu's dram__bytes_read.sum + write.sum of the
# launch in a capture of the static_drop_256 workload (the predictor's grid
# and fields do not depend on the drops)
TRAFFIC = {("ab2", False): 2.504199e9 + 0.801062e9, ("ab2", True): 1.245101e9 + 0.389982e9}


def alg_bytes_per_launch(name, cfg, stats, f32=False):
    """Compulsory HBM bytes of one scope of the named launcher."""
    e = ALG_VALUES.get(name)
    if e is None:
        return None
    bulk, f64, unit = e
    n = {"N": cfg.itot * cfg.jtot * cfg.ktot, "B": stats.get("band_total", 0.0),
         "S": stats.get("shell_total", 0.0)}[unit]
    return (bulk * (4.0 if f32 else 8.0) + f64 * 8.0) * n


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [x.strip() for x in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        finally:
            os.unlink(self.path)
        if not rows:
            return None

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, val in zip(names, r[5:9]):
                if val.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ---------------------------------------------------------------- helpers
def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(x, world):
    """The maximum of x over the ranks (the job's time is its slowest rank's),
    on the process group's own device (NCCL: the GPU; gloo: the host)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def shell_and_band(wl, ls):
    """Mean |phi|<=2dz shell size per drop from the initial level sets."""
    dz = wl.cfg.lz / wl.cfg.ktot
    inner = ls[2:-4, 2:-4, 2:-4]
    return float(np.mean([(np.abs(inner[..., l]) <= 2 * dz).sum() for l in range(ls.shape[-1])]))


def cpu_sample(wl, ls, u, v, w, steps, threads):
    """The oracle (C++ restatement of the reference) on the host cores."""
    from oracle.oracle import Oracle, set_threads
    n = set_threads(threads)
    o = Oracle(wl.cfg)
    o.setup(ls, u, v, w)
    o.step(1, 0)  # first step (AB2 start, pressure normalisation branch)
    t0 = time.perf_counter()
    for s in range(2, 2 + steps):
        o.step(s, 0)
    dt = time.perf_counter() - t0
    cells = wl.cfg.itot * wl.cfg.jtot * wl.cfg.ktot
    return cells * steps / dt / 1e6, n, dt


# ---------------------------------------------------------------- arms
def reference_arm(args):
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    wl = make_workload(args.workload)
    ls, u, v, w = initial_state(wl)
    steps = max(1, min(args.steps, 2))
    threads = os.cpu_count() or 1
    value, n, dt = cpu_sample(wl, ls, u, v, w, steps, threads)
    sample = "%d timed step(s) of %s after one untimed step (of %d requested)" % (steps, wl.name, args.steps)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": steps, "warmup": 1, "ms_per_step": 1000.0 * dt / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_block(wl, world, "fp64 (the reference's only form)"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": n, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "C++ restatement of the reference (oracle/, OpenMP); the Fortran/MPI reference cannot be "
                "built here (no Fortran compiler, MPI or LAPACK)",
    }
    print(json.dumps(line))
    return 0


def config_block(wl, world, form):
    c = wl.cfg
    return {"workload": wl.name, "grid": [c.itot, c.jtot, c.ktot], "drops": c.lmax,
            "dt": c.timestep, "scheme": "HOUC5" if c.ls_adv_space == 0 else "WENO5",
            "reinit_step": c.reinit_step, "reinit_iter_max": c.reinit_iter_max,
            "inflate_step": c.inflate_step, "form": form,
            "l2": "inputs larger than L2 (no flush)", "parallelism": "replicas x%d" % world}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def timed_steps(s, args, world, torch, istep, label, sampler=None):
    """W warm-up steps, then K steps between barriers and synchronisations,
    timed with CUDA events on the context's stream; max over ranks.  The K
    steps sit in the NVTX push/pop range `label` (an ncu launch list of one
    form selects them with --nvtx --nvtx-include "<label>/")."""
    stream = torch.cuda.ExternalStream(s.stream_ptr())
    for _ in range(args.warmup):
        istep += 1
        s.step(istep, 0)
    launches0 = s.launch_count()
    if sampler:
        sampler.start()
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push(label)
    e0.record(stream)
    for _ in range(args.steps):
        istep += 1
        s.step(istep, 0)
    e1.record(stream)
    torch.cuda.nvtx.range_pop()
    e1.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop() if sampler else None
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    return ms, istep, s.launch_count() - launches0, clocks


def step_roofline(roof, ms_step):
    """The whole step against the HBM roofline: the algorithmic bytes of
    every scope with a byte model (ALG_VALUES), per step, over the measured
    (unprofiled) step time."""
    peak = load_peaks().get("hbm_gbs", 6650.0)
    b = roof.get("step_alg_bytes") or 0.0
    roof["step_ms"] = ms_step
    roof["step_frac"] = (b / (ms_step / 1000.0) / 1e9 / peak) if ms_step > 0 else None


def dominant_scope(table):
    """The roofline's dominant kernel: the largest scope of one kernel launch
    (solver2d, for one, is five kernels: the x and y transforms both ways
    and the z sweeps); the largest scope if none is single."""
    single = {k: e for k, e in table.items() if e["timed"] > 0 and e["launches"] == e["timed"]}
    return max((single or table).items(), key=lambda kv: kv[1]["ms"])


def kernel_table(s, args, cfg, stats, istep, f32, mlp_cells=None):
    """K more steps with every launcher scope bracketed by CUDA events: the
    per-kernel shares and the roofline of the dominant one.  The network's
    scope (gather + tiles) is rated against the tensor peak by its products'
    FLOPs, mlp_cells evaluated cells per step."""
    s.profile(True)
    s.profile_reset()
    for _ in range(args.steps):
        istep += 1
        s.step(istep, 0)
    table = s.profile_table()
    s.profile(False)
    tot = sum(e["ms"] for e in table.values()) or 1.0
    name, ent = dominant_scope(table)
    per_launch_ms = ent["ms"] / max(ent["timed"], 1)
    alg = alg_bytes_per_launch(name, cfg, stats, f32)
    peaks = load_peaks()
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = (alg / (per_launch_ms / 1000.0) / 1e9) if alg else None
    # the network runs inside a long step: its denominator is the sustained
    # bf16 figure (the power-capped clock), not the burst one
    tpeak = peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops", 1590.0))
    tsrc = ("measured (cuBLAS bf16 sustained)" if "bf16_tflops_sustained" in peaks else
            "measured (cuBLAS bf16 burst)" if "bf16_tflops" in peaks else "fallback")
    if name == "mlp_curvature" and mlp_cells:
        tf = MLP_FLOPS_PER_CELL * mlp_cells / (per_launch_ms / 1000.0) / 1e12
        roofline = {"bound": "tensor", "kernel": name, "achieved": tf, "peak": tpeak, "unit": "TFLOP/s",
                    "frac": tf / tpeak, "traffic": TRAFFIC.get((name, f32)), "flops": MLP_FLOPS_PER_CELL * mlp_cells,
                    "share": ent["ms"] / tot, "launch_ms": per_launch_ms, "peak_source": tsrc}
    else:
        roofline = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": (achieved / peak) if achieved else None, "traffic": TRAFFIC.get((name, f32)),
                    "alg_bytes": alg, "share": ent["ms"] / tot, "launch_ms": per_launch_ms,
                    "peak_source": "measured (burst copy)" if "hbm_gbs" in peaks else "fallback"}
    kernels = {}
    step_bytes = 0.0  # algorithmic bytes of one step: the scopes with a byte model
    for k, e in table.items():
        ab = alg_bytes_per_launch(k, cfg, stats, f32)
        if ab:
            step_bytes += ab * e["timed"] / args.steps
    roofline["step_alg_bytes"] = step_bytes
    for k, e in sorted(table.items(), key=lambda kv: -kv[1]["ms"]):
        if e["timed"] == 0:
            continue
        ms1 = e["ms"] / e["timed"]
        ab = alg_bytes_per_launch(k, cfg, stats, f32)
        kernels[k] = {"share": round(e["ms"] / tot, 4), "scopes": e["timed"], "ms_per_scope": round(ms1, 5),
                      "hbm_frac": round(ab / (ms1 / 1000.0) / 1e9 / peak, 3) if ab else None}
        if k == "mlp_curvature" and mlp_cells:
            tf = MLP_FLOPS_PER_CELL * mlp_cells / (ms1 / 1000.0) / 1e12
            kernels[k].update({"tflops": round(tf, 2), "tensor_frac": round(tf / tpeak, 4), "cells": mlp_cells})
    return roofline, kernels, istep


def drop_shells(wl):
    """Per drop, the shape-C cells with ||x - c| - R| <= 1.5 dx (minimum image
    in x and y) from the seeded geometry: flat Fortran-order indices and
    distances |x - c|.  The drops move by far less than a cell in the steps
    the bench runs, so the initial spheres locate the shells."""
    cfg = wl.cfg
    n1, n2, n3 = cfg.itot + 2, cfg.jtot + 2, cfg.ktot + 2
    h = cfg.lz / cfg.ktot
    out = []
    for c, R in zip(wl.centres, wl.radii):
        ax = []
        for d, (nn, L) in enumerate(((n1, cfg.lx), (n2, cfg.ly), (n3, cfg.lz))):
            lo = int(np.floor((c[d] - R - 2 * h) / h)) + 1
            hi = int(np.ceil((c[d] + R + 2 * h) / h)) + 1
            idx = np.arange(lo, hi + 1)
            x = (idx - 0.5) * h
            if d < 2:
                idx = (idx - 1) % (nn - 2) + 1  # interior image of a periodic index
                dd = x - c[d]
            else:
                keep = (idx >= 0) & (idx < nn)
                idx, dd = idx[keep], (x - c[d])[keep]
            ax.append((idx, dd))
        I, J, K = np.meshgrid(ax[0][0], ax[1][0], ax[2][0], indexing="ij")
        X, Y, Z = np.meshgrid(ax[0][1], ax[1][1], ax[2][1], indexing="ij")
        r = np.sqrt(X * X + Y * Y + Z * Z)
        m = np.abs(r - R) <= 1.5 * h
        flat = (I[m] + n1 * (J[m] + n2 * K[m])).astype(np.int64)
        out.append((flat, r[m]))
    return out


def train_network(torch):
    """The learned curvature's network, trained on the GPU by the project's
    own kernels: 4M seeded sphere/ellipsoid samples, 20 epochs of batch 8192,
    Adam lr 1e-3 with a cosine decay to 1e-5."""
    from icls_gpu.binding import Mlp
    net = Mlp(2024)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    net.make_data(99, 1 << 22, 1 << 16)
    t1 = time.perf_counter()
    losses = net.train(epochs=20, batch=8192, lr=1e-3, lr_final=1e-5, seed=5)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    ev = net.evaluate()
    info = {"samples": 1 << 22, "held_out": int(ev["samples"]), "epochs": 20, "batch": 8192,
            "generate_s": round(t1 - t0, 3), "train_s": round(t2 - t1, 3),
            "loss_first_epoch": losses[0], "loss_last_epoch": losses[-1],
            "held_out_kdx_rms_vs_analytic": {"network": ev["rms_mlp_analytic"], "stencil": ev["rms_plain_analytic"],
                                             "refined_label": ev["rms_label_analytic"]}}
    return net, info


def ours_arm(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from icls_gpu import CURV_MLP, FP32, Solver
    from icls_gpu.binding import curvature_stats
    from icls_gpu.config import IclsConfig
    wl = make_workload(args.workload)
    cfg = wl.cfg
    ls, u, v, w = initial_state(wl)
    cells = cfg.itot * cfg.jtot * cfg.ktot
    h = cfg.lz / cfg.ktot
    shells = drop_shells(wl)
    shell = shell_and_band(wl, ls)

    # ---- the network: trained before any timing --------------------------
    net, net_info = (None, None)
    if not args.no_forms:
        net, net_info = train_network(torch)

    # ---- plain FP64 -------------------------------------------------------
    ref = Solver(cfg)
    ref.setup(ls, u, v, w)
    ms64, istep, launches64, clocks64 = timed_steps(ref, args, world, torch, 0, "fp64", ClockSampler(local))
    stats = {"band_total": float(sum(ref.band_count(l + 1) for l in range(cfg.lmax))),
             "shell_total": shell * cfg.lmax}
    roof64, kern64, istep = kernel_table(ref, args, cfg, stats, istep, False)
    step_roofline(roof64, ms64 / args.steps)
    v64 = cells * args.steps * world / (ms64 / 1000.0) / 1e6
    plain = {"value": v64, "unit": UNIT, "ms_per_step": ms64 / args.steps, "dtype": "f64",
             "gpu_launches": launches64, "clocks": clocks64, "roofline": roof64, "kernels": kern64}
    torch.cuda.synchronize()

    form = None
    if not args.no_forms:
        # ---- FP32 + learned curvature (the headline form) -------------------
        cf = IclsConfig.from_buffer_copy(cfg)
        cf.precision = FP32
        cf.curvature_model = CURV_MLP
        s = Solver(cf)
        net.attach(s)
        s.setup(ls, u, v, w)
        ms, istep_f, launches, clocks = timed_steps(s, args, world, torch, 0, "fp32_learned_kappa",
                                                     ClockSampler(local))
        ev, fb = curvature_stats(s, reset=True)
        roof, kern, istep_f = kernel_table(s, args, cfg, stats, istep_f, True,
                                           ev / max(args.warmup + args.steps, 1))
        step_roofline(roof, ms / args.steps)
        assert istep_f == istep
        errors = form_errors(s, ref, wl, shells, h, istep)
        errors["fallback_fraction"] = fb / max(ev, 1)
        errors["network_cells_per_step"] = ev / max(args.warmup + args.steps, 1)
        form = {"value": cells * args.steps * world / (ms / 1000.0) / 1e6, "ms_per_step": ms / args.steps,
                "gpu_launches": launches, "clocks": clocks, "roofline": roof, "kernels": kern, "errors": errors}
        del s
        torch.cuda.synchronize()
        # ---- FP32 with the plain stencil (splits the gain) -------------------
        cs = IclsConfig.from_buffer_copy(cfg)
        cs.precision = FP32
        s = Solver(cs)
        s.setup(ls, u, v, w)
        ms32, _, _, _ = timed_steps(s, args, world, torch, 0, "fp32_stencil")
        form["fp32_stencil"] = {"value": cells * args.steps * world / (ms32 / 1000.0) / 1e6,
                                "ms_per_step": ms32 / args.steps}
        del s
        torch.cuda.synchronize()
    del ref
    torch.cuda.synchronize()

    # ---- end to end through the per-subroutine C ABI, host buffers -------
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, wl, ls, u, v, w, torch, world, net)

    # ---- volume drift over 1000 steps: both contexts side by side from the
    # initial state, the gain-one mass correction at the workload's cadence
    # with a 1e-7 trigger (icls_config.mass_gain_one / mass_threshold)
    drift = None
    if world == 1 and net is not None and not args.no_drift:
        drift = drift_record(wl, ls, u, v, w, net, 1000, torch, mass_threshold=1e-7, gain_one=True)

    # ---- CPU baseline: the oracle on a bounded sample ---------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        cv, n, dt = cpu_sample(wl, ls, u, v, w, 1, threads)
        cpu = {"value": cv, "unit": UNIT, "cores": n, "kind": "port",
               "sample": "one plain FP64 time step of %s on %d host threads after one untimed step (%.1f s)"
                         % (wl.name, n, dt)}
    if net is not None:
        net.close()

    if rank == 0:
        if form is not None:
            line = {
                "metric": METRIC, "value": form["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": form["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 (f64 Poisson/pressure, volume integral, GFM jumps; bf16 network, f32 accumulate)",
                "data": "synthetic (seeded drops; network trained on seeded spheres/ellipsoids)",
                "config": config_block(wl, world, "fp32+learned-curvature"),
                "roofline": form["roofline"], "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": form["gpu_launches"], "clocks": form["clocks"],
                "speedup_vs_fp64": form["value"] / v64, "errors": form["errors"],
                "plain_fp64": plain, "fp32_stencil": form["fp32_stencil"], "network": net_info,
                "kernels": form["kernels"], "volume_drift_1000": drift}
        else:
            line = {
                "metric": METRIC, "value": v64, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms64 / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded drops)",
                "config": config_block(wl, world, "fp64"), "roofline": roof64, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": launches64, "clocks": clocks64, "kernels": kern64}
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def form_errors(s, ref, wl, shells, h, istep):
    """The form against the plain FP64 context after the same steps from the
    same initial state: phi on the |phi| <= 4dz band (first four drops),
    velocities, per-drop volume; each context's volume drift since the
    initial state; and, drop by drop, the curvature get_curvature gives on
    the drop's shell (the network's, with its fallback, in the form) against
    the FP64 stencil's and against the analytic -2/r of the seeded sphere."""
    def rel(a, b):
        return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
    band = 0.0
    for l in range(1, min(wl.cfg.lmax, 4) + 1):
        pa, pb = s.download("lvset", l), ref.download("lvset", l)
        m = np.abs(pb) <= 4.0 * h
        band = max(band, rel(pa[m], pb[m]))
    va, va0 = s.volumes()
    vb, vb0 = ref.volumes()
    out = {
        "steps": istep, "drops_compared_phi": min(wl.cfg.lmax, 4), "phi_band_rel_l2": band,
        "u_rel_l2": rel(s.download("u"), ref.download("u")), "v_rel_l2": rel(s.download("v"), ref.download("v")),
        "w_rel_l2": rel(s.download("w"), ref.download("w")),
        "volume_max_rel_vs_fp64": float(np.max(np.abs(va - vb) / vb)),
        "volume_drift_max_rel": {"form": float(np.max(np.abs(va - va0) / va0)),
                                 "fp64": float(np.max(np.abs(vb - vb0) / vb0))},
    }
    acc = {"form": [0.0, 0.0], "fp64_stencil": [0.0, 0.0]}
    d2, p2, cells = 0.0, 0.0, 0
    for l, (flat, r) in enumerate(shells, start=1):
        kap = {}
        for name, ctx in (("form", s), ("fp64_stencil", ref)):
            ctx.get_curvature(l)
            kap[name] = ctx.download("curv").ravel(order="F")[flat]
            acc[name][0] += float(np.sum((kap[name] + 2.0 / r) ** 2))
        acc["form"][1] += float(np.sum((2.0 / r) ** 2))
        d2 += float(np.sum((kap["form"] - kap["fp64_stencil"]) ** 2))
        p2 += float(np.sum(kap["fp64_stencil"] ** 2))
        cells += flat.size
    out["curv_shell_rel_l2_vs_fp64"] = float(np.sqrt(d2 / max(p2, 1e-300)))
    out["curv_vs_analytic"] = {
        name: {"kdx_rms": float(np.sqrt(e2 / max(cells, 1))) * h, "rel": float(np.sqrt(e2 / acc["form"][1]))}
        for name, (e2, _) in acc.items()}
    out["curv_vs_analytic"]["shell_cells"] = cells
    return out


def run_e2e(args, wl, ls, u, v, w, torch, world, net=None):
    """Upload the initial state from pinned host memory, init_program, K steps
    through the subroutines main.f90 calls (with its per-step NaN probe),
    download the final fields; all inside the timed region.  With a network
    the context is the FP32 + learned-curvature form."""
    from icls_gpu import CURV_MLP, FP32, Solver
    from icls_gpu.config import IclsConfig
    cfg = IclsConfig.from_buffer_copy(wl.cfg)
    if net is not None:
        cfg.precision = FP32
        cfg.curvature_model = CURV_MLP

    def pinned(a):
        t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
        t.numpy()[:] = np.asfortranarray(a).ravel(order="F")
        return t

    hu, hv, hw = pinned(u), pinned(v), pinned(w)
    hp = pinned(np.zeros_like(u))
    hls = [pinned(ls[..., l]) for l in range(cfg.lmax)]
    out_c = [torch.empty(u.size, dtype=torch.float64, pin_memory=True) for _ in range(4)]
    out_l = [torch.empty(hls[0].numel(), dtype=torch.float64, pin_memory=True) for _ in range(cfg.lmax)]
    h2d = 8 * (4 * u.size + cfg.lmax * hls[0].numel())
    d2h = 8 * (4 * u.size + cfg.lmax * hls[0].numel())
    s = Solver(cfg)
    if net is not None:
        net.attach(s)
    stream = torch.cuda.ExternalStream(s.stream_ptr())
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.upload_ptr("u", hu.data_ptr())
    s.upload_ptr("v", hv.data_ptr())
    s.upload_ptr("w", hw.data_ptr())
    s.upload_ptr("pnew", hp.data_ptr())
    for l in range(cfg.lmax):
        s.upload_ptr("lvset", hls[l].data_ptr(), l + 1)
    s.init_program()
    probes = 0
    for istep in range(1, args.steps + 1):
        s.ls_main(istep)
        s.average_stream_vel()
        s.ab2()
        s.fillps()
        s.gfm4p()
        s.add_pjump()
        s.solver2d()
        s.boundp("p")
        s.correc()
        s.bounduvw("u")
        s.pressure_update(istep, 0)
        s.average_vel_at_center()
        if np.isnan(s.probe("v", 1, 1, 1)):
            raise RuntimeError("NaN at step %d" % istep)
        probes += 1
    for t, name in zip(out_c, ("u", "v", "w", "pnew")):
        s.download_ptr(name, t.data_ptr())
    for l in range(cfg.lmax):
        s.download_ptr("lvset", out_l[l].data_ptr(), l + 1)
    e1.record(stream)
    e1.synchronize()
    wall = time.perf_counter() - t0
    barrier(world)
    ms = max_over_ranks(max(e0.elapsed_time(e1), 1000.0 * wall), world)
    cells = cfg.itot * cfg.jtot * cfg.ktot
    del s
    return {"value": cells * args.steps * world / (ms / 1000.0) / 1e6, "unit": UNIT,
            "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": (d2h + 8 * probes) / args.steps,
            "path": "per-subroutine C ABI (FP64 host arrays; upload, init_program, ls_main..average_vel_at_center, "
                    "download)", "form": "fp32+learned-curvature" if net is not None else "fp64",
            "ms_total": ms}


def combined_full(args):
    """The combined configuration at its full size (384^3, 200 drops of
    radius 0.02-0.04, random solenoidal k^-5/3 velocity, rms 0.2): the plain
    FP64 context, then the FP32 + learned-curvature form, each alone on the
    device (together they would not fit: 200 whole-domain level sets are
    95 GB in FP64).  Each drop's level set is built on the host and uploaded
    one at a time.  After the FP64 run, the quantities the form is compared
    with (velocities, volumes, the first four drops' bands, the first eight
    drops' shell curvature) are kept on the host.  One JSON line."""
    import gc
    import torch
    from icls_gpu import CURV_MLP, FP32, Solver, field_shape
    from icls_gpu.binding import curvature_stats
    from icls_gpu.config import IclsConfig, combined, init_drops_boxed, workload_velocity
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    wl = combined()
    cfg = wl.cfg
    if args.gain_one:  # a stable correction for long runs (at 384^3 the reference's gain is about -7)
        cfg.mass_gain_one = 1
    if args.mass_threshold:
        cfg.mass_threshold = args.mass_threshold
    if args.inflate_step:
        cfg.inflate_step = args.inflate_step
    h = cfg.lz / cfg.ktot
    cells = cfg.itot * cfg.jtot * cfg.ktot
    u, v, w = workload_velocity(wl)
    zeros = np.zeros(field_shape(cfg, "p"), order="F")
    shells = drop_shells(wl)[:8]
    net, net_info = train_network(torch)
    torch.cuda.empty_cache()  # the training's cached blocks back to the device

    def start(c, attach):
        s = Solver(c)
        if attach:
            net.attach(s)
        for name, a in (("u", u), ("v", v), ("w", w), ("pnew", zeros)):
            s.upload(name, a)
        for l, (cen, r) in enumerate(zip(wl.centres, wl.radii), start=1):
            s.upload("lvset", init_drops_boxed(cfg, [cen], [r])[..., 0], l)
        s.init_program()
        return s

    band_idx = []  # the FP64 run's |phi| <= 4dz cells of drops 1-4 (flat indices)

    def state(s):
        out = {k: s.download(k) for k in ("u", "v", "w")}
        out["vol"], out["vol0"] = s.volumes()
        out["bands"] = []
        for l in range(1, 5):
            phi = s.download("lvset", l).ravel(order="F")
            if len(band_idx) < l:
                band_idx.append(np.flatnonzero(np.abs(phi) <= 4 * h))
            out["bands"].append(phi[band_idx[l - 1]].copy())
            del phi
        out["curv"] = []
        for l, (flat, r) in enumerate(shells, start=1):
            s.get_curvature(l)
            out["curv"].append(s.download("curv").ravel(order="F")[flat].copy())
        return out

    res = {}
    for label, c, attach in (("fp64", cfg, False), ("fp32_learned_kappa", None, True)):
        if c is None:
            c = IclsConfig.from_buffer_copy(cfg)
            c.precision = FP32
            c.curvature_model = CURV_MLP
        s = start(c, attach)
        ms, istep, launches, clocks = timed_steps(s, args, world, torch, 0, label, ClockSampler(local))
        r = {"value": cells * args.steps / (ms / 1000.0) / 1e6, "ms_per_step": ms / args.steps,
             "gpu_launches": launches, "clocks": clocks}
        if attach:
            ev, fb = curvature_stats(s, reset=True)
            r["fallback_fraction"] = fb / max(ev, 1)
            r["network_cells_per_step"] = ev / max(args.warmup + args.steps, 1)
        r["state"] = state(s)
        # per-scope times over K more steps (the compared state is taken first)
        stats = {"band_total": float(sum(s.band_count(l + 1) for l in range(cfg.lmax))), "shell_total": 0.0}
        _, r["kernels"], istep = kernel_table(s, args, cfg, stats, istep, attach)
        res[label] = r
        s.close()
        del s
        gc.collect()
        torch.cuda.synchronize()

    def rel(a, b):
        return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
    a, b = res["fp32_learned_kappa"].pop("state"), res["fp64"].pop("state")
    band = max(rel(pa, pb) for pa, pb in zip(a["bands"], b["bands"]))
    e_form = sum(float(np.sum((ka + 2.0 / r) ** 2)) for ka, (_, r) in zip(a["curv"], shells))
    e_fp64 = sum(float(np.sum((kb + 2.0 / r) ** 2)) for kb, (_, r) in zip(b["curv"], shells))
    ncell = sum(f.size for f, _ in shells)
    errors = {
        "steps": args.warmup + args.steps, "phi_band_rel_l2_first4": band,
        "u_rel_l2": rel(a["u"], b["u"]), "v_rel_l2": rel(a["v"], b["v"]), "w_rel_l2": rel(a["w"], b["w"]),
        "volume_max_rel_vs_fp64": float(np.max(np.abs(a["vol"] - b["vol"]) / b["vol"])),
        "volume_drift_max_rel": {"form": float(np.max(np.abs(a["vol"] - a["vol0"]) / a["vol0"])),
                                 "fp64": float(np.max(np.abs(b["vol"] - b["vol0"]) / b["vol0"]))},
        "curv_vs_analytic_first8": {"form_kdx_rms": float(np.sqrt(e_form / max(ncell, 1))) * h,
                                    "fp64_stencil_kdx_rms": float(np.sqrt(e_fp64 / max(ncell, 1))) * h,
                                    "shell_cells": ncell},
    }
    form = res["fp32_learned_kappa"]
    line = {"metric": "Mcell-steps/s at 384\u00b3 with 200 drops: FP32+learned-\u03ba vs plain FP64 on B200",
            "workload": "combined_384_200", "value": form["value"], "unit": UNIT,
            "ms_per_step": form["ms_per_step"], "steps": args.steps, "warmup": args.warmup,
            "dtype": "f32 (f64 Poisson/pressure, volume integral, GFM jumps; bf16 network, f32 accumulate)",
            "data": "synthetic (seeded drops, seeded solenoidal velocity)",
            "config": {"grid": [cfg.itot, cfg.jtot, cfg.ktot], "drops": cfg.lmax, "dt": cfg.timestep,
                       "We": cfg.We, "Re": cfg.Re, "inflate_step": cfg.inflate_step,
                       "mass_threshold": cfg.mass_threshold or 1e-5, "gain_one": bool(cfg.mass_gain_one)},
            "fp32_learned_kappa": form, "plain_fp64": res["fp64"],
            "speedup_vs_fp64": form["value"] / res["fp64"]["value"], "errors": errors, "network": net_info}
    if rank == 0:
        print(json.dumps(line))
    return 0


def drift_record(wl, ls, u, v, w, net, n, torch, inflate_step=0, mass_threshold=0.0, dt=0.0, gain_one=False,
                 record_every=0):
    """The plain FP64 context and the FP32 + learned-curvature form advance
    the same initial state side by side for n steps; every drop's volume is
    read after every step.  Returns the largest |V - V0| / V0 of each
    context over the run and at its end, the form's largest per-drop volume
    difference from FP64, and at the end the phi band and velocity
    differences."""
    from icls_gpu import CURV_MLP, FP32, Solver
    from icls_gpu.binding import curvature_stats
    from icls_gpu.config import IclsConfig
    cfg = IclsConfig.from_buffer_copy(wl.cfg)
    if dt:
        cfg.timestep = dt
    if inflate_step:
        cfg.inflate_step = inflate_step
    if mass_threshold:
        cfg.mass_threshold = mass_threshold
    cfg.mass_gain_one = 1 if gain_one else 0
    h = cfg.lz / cfg.ktot
    ref = Solver(cfg)
    ref.setup(ls, u, v, w)
    cf = IclsConfig.from_buffer_copy(cfg)
    cf.precision = FP32
    cf.curvature_model = CURV_MLP
    s = Solver(cf)
    net.attach(s)
    s.setup(ls, u, v, w)
    every = record_every or max(n // 50, 1)
    worst = {"form": 0.0, "fp64": 0.0}
    worst_step = {"form": 0, "fp64": 0}
    vs_fp64 = 0.0
    record = []
    last = (0.0, 0.0)
    stopped = None
    t0 = time.perf_counter()
    for istep in range(1, n + 1):
        try:
            ref.step(istep, 0)
            s.step(istep, 0)
        except Exception as e:  # a divergence or time-step check of either context
            stopped = {"step": istep, "error": str(e)}
            break
        va, va0 = s.volumes()
        vb, vb0 = ref.volumes()
        da = float(np.max(np.abs(va - va0) / va0))
        db = float(np.max(np.abs(vb - vb0) / vb0))
        for key, d in (("form", da), ("fp64", db)):
            if d > worst[key]:
                worst[key], worst_step[key] = d, istep
        vs_fp64 = max(vs_fp64, float(np.max(np.abs(va - vb) / vb)))
        last = (da, db)
        if istep % every == 0 or istep == n:
            record.append([istep, da, db])
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0

    def rel(a, b):
        return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
    band = 0.0
    for l in range(1, min(cfg.lmax, 4) + 1):
        pa, pb = s.download("lvset", l), ref.download("lvset", l)
        m = np.abs(pb) <= 4.0 * h
        band = max(band, rel(pa[m], pb[m]))
    ev, fb = curvature_stats(s, reset=True)
    sc = ref.scalars()
    out = {
        "steps": n, "dt": sc["dt"], "time": sc["time"], "inflate_step": cfg.inflate_step,
        "reinit_step": cfg.reinit_step, "drops": cfg.lmax, "mass_threshold": cfg.mass_threshold or 1e-5,
        "gain_one": bool(gain_one), "sampled": "every step",
        "drift_max_rel_over_run": worst, "at_step": worst_step,
        "drift_max_rel_at_end": {"form": last[0], "fp64": last[1]},
        "volume_max_rel_form_vs_fp64": vs_fp64,
        "at_end": {"phi_band_rel_l2_first4": band, "u_rel_l2": rel(s.download("u"), ref.download("u")),
                   "v_rel_l2": rel(s.download("v"), ref.download("v")),
                   "w_rel_l2": rel(s.download("w"), ref.download("w"))},
        "network_fallback_fraction": fb / max(ev, 1),
        "record_step_drift_form_fp64": record, "stopped": stopped, "wall_s": round(wall, 1)}
    s.close()
    ref.close()
    return out


def rise_record(args):
    """The rising bubble's record (--rise-steps N): the plain FP64 context
    alone for N steps on its workload (default rising_bubble_128: 128 x 128 x
    256 on [0,1]x[0,1]x[0,2], reinitialisation and the mass-correction check
    every step), the bubble's centroid z and rise velocity (disp_cg,
    disp_speed, write_vtk.f90:438-566) and its volume drift every --record
    steps, and the device time per step.  --gain-one takes the gain-one mass
    correction (the reference's, at inflate_step = 1, multiplies the volume
    error by about 1 - 0.44 n = -55 per correction at this resolution)."""
    import torch
    rank, world, local = dist_env()
    if world != 1:
        raise SystemExit("--rise-steps runs on one GPU")
    torch.cuda.set_device(local)
    from icls_gpu import Solver
    wl = make_workload(args.workload if args.workload != "multi_drop_256_48" else "rising_bubble_128")
    cfg = wl.cfg
    if args.dt:
        cfg.timestep = args.dt
    if args.inflate_step:
        cfg.inflate_step = args.inflate_step
    if args.mass_threshold:
        cfg.mass_threshold = args.mass_threshold
    cfg.mass_gain_one = 1 if args.gain_one else 0
    ls, u, v, w = initial_state(wl)
    s = Solver(cfg)
    s.setup(ls, u, v, w)
    stream = torch.cuda.ExternalStream(s.stream_ptr())
    cg0, _ = s.disp(1)
    every = max(args.record, 1)
    rec, worst, stopped = [], 0.0, None
    ms = 0.0
    for istep in range(1, args.rise_steps + 1):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        try:
            s.step(istep, 0)
        except Exception as e:  # the reference's divergence or NaN checks
            stopped = {"step": istep, "error": str(e)}
            break
        e1.record(stream)
        e1.synchronize()
        ms += e0.elapsed_time(e1)
        vol, v0 = s.volumes()
        d = abs(vol[0] - v0[0]) / v0[0]
        worst = max(worst, d)
        if istep % every == 0 or istep == args.rise_steps:
            cg, vel = s.disp(1)
            sc = s.scalars()
            rec.append([istep, sc["time"], cg[2], vel[2], d])
    cells = cfg.itot * cfg.jtot * cfg.ktot
    n = rec[-1][0] if rec else 0
    line = {"report": "rising_bubble", "workload": wl.name, "steps": args.rise_steps, "dt": cfg.timestep,
            "inflate_step": cfg.inflate_step, "reinit_step": cfg.reinit_step,
            "mass_threshold": cfg.mass_threshold or 1e-5, "gain_one": bool(args.gain_one),
            "centroid_z0": cg0[2], "volume_drift_max_rel": worst,
            "mcell_steps_per_s": cells * n / (ms / 1000.0) / 1e6 if ms > 0 else None,
            "ms_per_step": ms / max(n, 1),
            "record_step_time_cgz_wz_drift": rec, "stopped": stopped}
    s.close()
    print(json.dumps(line))
    return 0


def volume_drift(args):
    """The volume record over a long run (drift_record), as its own JSON
    line: a report, not a throughput line."""
    import torch
    rank, world, local = dist_env()
    if world != 1:
        raise SystemExit("--drift-steps runs on one GPU")
    torch.cuda.set_device(local)
    wl = make_workload(args.workload)
    ls, u, v, w = initial_state(wl)
    net, net_info = train_network(torch)
    line = {"report": "volume_drift", "workload": wl.name}
    line.update(drift_record(wl, ls, u, v, w, net, args.drift_steps, torch, args.inflate_step,
                             args.mass_threshold, args.dt, args.gain_one))
    line["network"] = net_info
    net.close()
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="multi_drop_256_48")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-drift", action="store_true", help="skip the 1000-step volume record")
    ap.add_argument("--rise-steps", type=int, default=0,
                    help="the rising bubble's centroid / rise-velocity / volume record over N steps")
    ap.add_argument("--record", type=int, default=50, help="with --rise-steps: record every N steps")
    ap.add_argument("--no-forms", action="store_true",
                    help="plain FP64 only (no network training, no FP32 forms)")
    ap.add_argument("--dt", type=float, default=0.0, help="with --drift-steps: the time step (default: the workload's)")
    ap.add_argument("--inflate-step", type=int, default=0,
                    help="with --drift-steps: the mass-correction cadence (default: the workload's)")
    ap.add_argument("--mass-threshold", type=float, default=0.0,
                    help="with --drift-steps: the volume error that triggers a correction (default 1e-5)")
    ap.add_argument("--gain-one", action="store_true",
                    help="with --drift-steps: the gain-one mass correction (icls_config.mass_gain_one)")
    ap.add_argument("--drift-steps", type=int, default=0,
                    help="instead of timing: run FP64 and the form side by side this many steps, "
                         "report the drop volumes' drift")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)
    if args.drift_steps > 0:
        return volume_drift(args)
    if args.rise_steps > 0:
        return rise_record(args)
    if args.workload == "combined_384_200":
        return combined_full(args)
    return ours_arm(args)


if __name__ == "__main__":
    sys.exit(main())
