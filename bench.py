#!/usr/bin/env python
"""Throughput of the ICLS per-timestep hot path on B200, in Mcell-steps/s.

One "step" is one full main-loop iteration (src/main.f90:107-210 of the
reference): level-set advection/reinitialisation/mass correction for every
drop, materials, AB2 predictor, Poisson RHS with GFM jumps, FFT/Thomas
pressure solve, projection, pressure update.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Default workload: the 256^3 box with 48 seeded drops (plain FP64).  Inputs
(seven-plus GB of level sets and fields) are far larger than the 126 MB L2,
so no flush is needed between steps.  Under torchrun each rank runs its own
replica of the workload (the path is not sharded across GPUs here), the
timed region is bracketed by a barrier and synchronisation on every rank,
and the reported time is the max over ranks.
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

METRIC = "Mcell-steps/s at 256^3 (plain FP64 time step)"
UNIT = "Mcell-steps/s"


# ------------------------------------------------------------------ workload
def make_workload(name):
    from icls_gpu.config import multi_drop, rising_bubble, static_drop
    if name == "multi_drop_256_48":
        return multi_drop(n=256, ndrop=48, seed=2024)
    if name == "multi_drop_256_4":
        return multi_drop(n=256, ndrop=4, seed=2024)
    if name == "multi_drop_128_12":
        return multi_drop(n=128, ndrop=12, seed=2024, rmin=0.06, rmax=0.12)
    if name == "static_drop_64":
        return static_drop(64)
    if name == "rising_bubble_128":
        return rising_bubble(128)
    raise SystemExit("unknown workload %s" % name)


def initial_state(wl):
    from icls_gpu.config import init_drops, init_drops_boxed, initial_velocity
    cfg = wl.cfg
    if wl.all_images and cfg.itot >= 128:
        ls = init_drops_boxed(cfg, wl.centres, wl.radii)
    else:
        ls = init_drops(cfg, wl.centres, wl.radii, wl.all_images)
    u, v, w = initial_velocity(cfg, wl.shear_v)
    return ls, u, v, w


# -------------------------------------------------- algorithmic byte model
def alg_bytes_per_launch(name, cfg, stats):
    """Compulsory HBM bytes of one launch of the named launcher group: the
    per-cell value counts of an ideal fused implementation (8 B per FP64
    value) times the cells that launch covers.  N = interior cells,
    Nb = band cells of one drop, Ng = its |phi|<=2dz shell."""
    N = cfg.itot * cfg.jtot * cfg.ktot
    Nb = stats.get("band_mean", 0.0)
    Ng = stats.get("shell_mean", 0.0)
    v = {
        "ab2": 24 * N,                  # u,v,w,miu,rho_uvw,duold x3,pnew,pold,p_xyz,p_xyz_old -> dudt x3,duold x3
        "correc": 13 * N,               # dudt x3, p, p_xyz -> u,v,w, ucc,vcc,wcc
        "fillps": 5 * N,                # dudt x3, p_jump -> p
        "solver2d": 10 * N / 5,         # 5 passes read+write, per launch
        "pressure_update": 4 * N / 2,   # p, pnew -> pnew, pold over two launches
        "stream_vel": 1 * N / 2,
        "materials_final": 6 * N / 2,   # jiemian -> miu, rho, rho_uvw
        "tube": 2 * Nb,                 # phi -> clipped phi on the band
        "adv_stage": (17.0 / 3.0) * Nb, # RK3 on the band, per stage
        "heaviside_drop": 1 * Nb,       # phi read per band cell
        "curvature": 2 * Ng,
        "recurvature": 2 * Ng,
        "jumps": 10 * Ng,
        "reinit_stage": (11.0 / 3.0) * N,  # reinit region is the whole grid after clipping
    }.get(name)
    return None if v is None else 8.0 * v


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
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
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
        "config": config_block(wl, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": n, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "C++ restatement of the reference (oracle/, OpenMP); the Fortran/MPI reference cannot be "
                "built here (no Fortran compiler, MPI or LAPACK)",
    }
    print(json.dumps(line))
    return 0


def config_block(wl, world):
    c = wl.cfg
    return {"workload": wl.name, "grid": [c.itot, c.jtot, c.ktot], "drops": c.lmax,
            "dt": c.timestep, "scheme": "HOUC5" if c.ls_adv_space == 0 else "WENO5",
            "reinit_step": c.reinit_step, "reinit_iter_max": c.reinit_iter_max,
            "inflate_step": c.inflate_step, "precision": "fp64",
            "l2": "inputs larger than L2 (no flush)", "parallelism": "replicas x%d" % world}


def ours_arm(args):
    import torch
    rank, world, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(local)
    from icls_gpu import Solver
    wl = make_workload(args.workload)
    cfg = wl.cfg
    ls, u, v, w = initial_state(wl)
    cells = cfg.itot * cfg.jtot * cfg.ktot
    shell = shell_and_band(wl, ls)

    s = Solver(cfg)
    s.setup(ls, u, v, w)
    stream = torch.cuda.ExternalStream(s.stream_ptr())
    istep = 0
    for _ in range(args.warmup):
        istep += 1
        s.step(istep, 0)
    sampler = ClockSampler(local)
    launches0 = s.launch_count()
    sampler.start()
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        istep += 1
        s.step(istep, 0)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    launches = s.launch_count() - launches0
    value = cells * args.steps * world / (ms / 1000.0) / 1e6

    # ---- per-kernel device times over the same number of steps ----------
    s.profile(True)
    s.profile_reset()
    for _ in range(args.steps):
        istep += 1
        s.step(istep, 0)
    table = s.profile_table()
    s.profile(False)
    bands = [s.band_count(l + 1) for l in range(cfg.lmax)]
    stats = {"band_mean": float(np.mean(bands)), "shell_mean": shell}
    tot = sum(e["ms"] for e in table.values()) or 1.0
    top = max(table.items(), key=lambda kv: kv[1]["ms"])
    name, ent = top
    per_launch_ms = ent["ms"] / max(ent["timed"], 1)
    alg = alg_bytes_per_launch(name, cfg, stats)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = (alg / (per_launch_ms / 1000.0) / 1e9) if alg else None
    roofline = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "traffic": None,
                "share": ent["ms"] / tot, "launch_ms": per_launch_ms,
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"}
    kernels = {k: {"share": round(e["ms"] / tot, 4), "launches": e["timed"],
                   "ms_per_launch": e["ms"] / max(e["timed"], 1)} for k, e in table.items()}
    torch.cuda.synchronize()

    # ---- the precision form on the same workload ------------------------
    prec = None
    if not args.no_forms:
        prec = precision_leg(args, wl, ls, u, v, w, torch, world, istep, s)
        prec["speedup_vs_fp64"] = prec["value"] / value
    del s
    torch.cuda.synchronize()

    # ---- end to end through the per-subroutine C ABI, host buffers -------
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, wl, ls, u, v, w, torch, world)

    # ---- CPU baseline: the oracle on a bounded sample ---------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        cv, n, dt = cpu_sample(wl, ls, u, v, w, 1, threads)
        cpu = {"value": cv, "unit": UNIT, "cores": n, "kind": "port",
               "sample": "one time step of %s on %d host threads after one untimed step (%.1f s)" % (wl.name, n, dt)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded drops)",
            "config": config_block(wl, world), "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches, "clocks": clocks, "kernels": kernels, "precision_form": prec,
        }
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def precision_leg(args, wl, ls, u, v, w, torch, world, fp64_solver_steps, ref):
    """The precision form (FP32 bulk, FP64 Poisson / volume / jumps) on the
    same workload: the same warm-up and timed steps, timed like the plain
    path; then its errors against the plain FP64 context `ref`, which has run
    fp64_solver_steps steps from the same initial state."""
    from icls_gpu import FP32, Solver
    from icls_gpu.config import IclsConfig
    cfg = IclsConfig.from_buffer_copy(wl.cfg)
    cfg.precision = FP32
    s = Solver(cfg)
    s.setup(ls, u, v, w)
    stream = torch.cuda.ExternalStream(s.stream_ptr())
    istep = 0
    for _ in range(args.warmup):
        istep += 1
        s.step(istep, 0)
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        istep += 1
        s.step(istep, 0)
    e1.record(stream)
    e1.synchronize()
    barrier(world)
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    cells = cfg.itot * cfg.jtot * cfg.ktot
    out = {"value": cells * args.steps * world / (ms / 1000.0) / 1e6, "unit": UNIT,
           "ms_per_step": ms / args.steps, "dtype": "f32 bulk, f64 Poisson/volume/jumps"}
    # errors after the same number of steps as the FP64 reference context
    while istep < fp64_solver_steps:
        istep += 1
        s.step(istep, 0)
    if istep == fp64_solver_steps:
        def rel(a, b):
            return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
        dz = wl.cfg.lz / wl.cfg.ktot
        band = 0.0
        for l in range(1, min(wl.cfg.lmax, 4) + 1):
            pa, pb = s.download("lvset", l), ref.download("lvset", l)
            m = np.abs(pb) <= 4.0 * dz
            band = max(band, rel(pa[m], pb[m]))
        va, vb = s.volumes()[0], ref.volumes()[0]
        out["errors_vs_fp64"] = {
            "steps": istep, "phi_band_rel_l2": band,
            "u_rel_l2": rel(s.download("u"), ref.download("u")),
            "w_rel_l2": rel(s.download("w"), ref.download("w")),
            "volume_max_rel": float(np.max(np.abs(va - vb) / vb)),
            "curv_rel_l2": rel(s.download("curv"), ref.download("curv")),
            "drops_compared_phi": min(wl.cfg.lmax, 4)}
    del s
    return out


def run_e2e(args, wl, ls, u, v, w, torch, world):
    """Upload the initial state from pinned host memory, init_program, K steps
    through the subroutines main.f90 calls (with its per-step NaN probe),
    download the final fields; all inside the timed region."""
    from icls_gpu import Solver
    cfg = wl.cfg

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
            "path": "per-subroutine C ABI (upload, init_program, ls_main..average_vel_at_center, download)",
            "ms_total": ms}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="multi_drop_256_48")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the precision-form leg")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)
    return ours_arm(args)


if __name__ == "__main__":
    sys.exit(main())
