#!/usr/bin/env python3
"""Benchmark of the direct-sum gravity time step on B200.

Workload (one "step"): predictor -> FP32 direct-sum force pass -> corrector
over one 786,432-body disk galaxy (262,144 stars + 524,288 dark-matter bodies,
masses 1.0 / 6.699356, eps 0.004, dt 0.002), generated from a seed (the
reference's own start_DM0.txt is not shipped).  The metric is pair
interactions per second (n^2 per force pass, j = i counted as the reference
does); the roofline of the force kernel is FP32: 20 flops per interaction
(n^2 per pass) over the nominal FP32 peak, and beside it the flops the kernel
executes (an FMA counts 2; the pair kernel evaluates each unordered pair once
for both bodies, so it executes fewer than 20 per interaction).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl khrr|reference]

N > 1 (under torchrun) runs N independent replicas (the path is pinned to one
GPU per galaxy; there is no data-path collective), timed as the max over ranks.
--impl reference times the reference's own ACCEL_kernel compiled for the host
(oracle/_ref, OpenMP over all host threads) on a bounded target sample.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import pathlib
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "khrr-nbody_b200"))

METRIC = "G interactions/s & %FP32 peak at 786k bodies; batched vs plain; err vs FP64"
UNIT = "G interactions/s"
N_STARS, N_DM = 262144, 524288
DT = 0.002
SEED = 1000
FLOPS_PER_PAIR = 20  # the n-body literature's convention per interaction
SMS, FP32_LANES = 148, 128
PAIR_BLOCK = 1024    # bodies per block of the symmetric pair kernel


def force_flops(n: int, pair: bool) -> float:
    """FP32 flops one force launch executes on one n-body system (uniform
    softening, tile-uniform masses; an FMA counts 2).  One-sided kernel: every
    ordered pair, 3 sub + 3 fma (r^2) + 2 mul (r^-3) + 3 fma = 17.  Pair kernel:
    each unordered pair of different 1024-blocks once, 17 + 3 fma for the
    reaction = 23; the pairs within a block one-sided (17)."""
    if not pair:
        return 17.0 * n * n
    blocks = [PAIR_BLOCK] * (n // PAIR_BLOCK) + ([n % PAIR_BLOCK] if n % PAIR_BLOCK else [])
    own = float(sum(b * b for b in blocks))
    return 23.0 * (float(n) * n - own) / 2.0 + 17.0 * own


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["khrr", "reference"], default="khrr")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 64-galaxy batched-vs-plain leg")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mesh", action="store_true", help="skip the p2mesh (binning, scan, wave) leg")
    ap.add_argument("--mesh-max-iter", type=int, default=0, help="cap on wave iterations (0 = to tolerance)")
    ap.add_argument("--n-stars", type=int, default=N_STARS)
    ap.add_argument("--n-dm", type=int, default=N_DM)
    return ap.parse_args()


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            return {}
    return {}


def workload(ns, nd):
    from khrr.galaxy import make_galaxy
    pos, vel, mass, eps = make_galaxy(ns, nd, SEED).arrays()
    return pos, vel, mass, eps * eps


def config(args, extra=None):
    c = {"workload": f"disk galaxy N={args.n_stars + args.n_dm} ({args.n_stars} stars + {args.n_dm} DM), "
                     f"eps 0.004, dt {DT}, predictor-force-corrector step",
         "n_bodies": args.n_stars + args.n_dm, "dt": DT, "seed": SEED,
         "l2": "256 MB buffer written between timed steps (inside the timed region)",
         "parallelism": f"replicas x{args.gpus}" if args.gpus > 1 else "single GPU"}
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.proc = None
        self.gpu_id = gpu_id

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu_id)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        if not getattr(self, "lines", None):
            return None
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for k, name in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "samples": len(sm),
                "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
# reference arm: the reference's ACCEL_kernel compiled for the host
# ---------------------------------------------------------------------------
def cpu_reference_sample(pos, mass, eps2, seconds, rng):
    """Times the host-compiled reference (or the oracle port when _ref is
    absent) on a seeded target subset; returns (pairs/s, cores, kind, sample)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle
    n = len(mass)
    try:
        ref = pyoracle.Reference()
        run = ref.accel
        cores = ref.max_threads()
        kind = "reference"
        what = "ACCEL_kernel (nbody-kernel.cuh:89-142) FP64, host build of the reference (oracle/_ref)"
    except FileNotFoundError:
        orc = pyoracle.Oracle()
        run = orc.accel_f64
        cores = orc.max_threads()
        kind = "port"
        what = "FP64 direct sum, oracle restatement (oracle/oracle.c)"
    t_cal = max(2 * cores, 16)
    tg = rng.choice(n, t_cal, replace=False)
    t0 = time.perf_counter()
    run(pos, mass, eps2, tg)
    rate = t_cal * n / (time.perf_counter() - t0)
    nt = int(min(n, max(t_cal, rate * seconds / n)))
    tg = rng.choice(n, nt, replace=False)
    t0 = time.perf_counter()
    run(pos, mass, eps2, tg)
    dt = time.perf_counter() - t0
    return nt * n / dt, cores, kind, f"{nt} seeded targets x {n} sources, {what}", dt


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    pos, vel, mass, eps2 = workload(args.n_stars, args.n_dm)
    rng = np.random.default_rng(7)
    rates, total_t, pairs = [], 0.0, 0.0
    for k in range(args.warmup + args.steps):
        rate, cores, kind, sample, dt = cpu_reference_sample(pos, mass, eps2, 6.0, rng)
        if k >= args.warmup:
            rates.append(rate)
            total_t += dt
            pairs += rate * dt
    value = pairs / total_t / 1e9
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": (len(mass) ** 2) / (value * 1e9) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": config(args),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                             "sample": sample + "; ms_per_step extrapolates one full n^2 force pass"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def ensemble_leg(khrr, ctx_device, torch, steps=8):
    """Configs' 64-galaxy uneven ensemble: one batched step launch vs one
    force launch per system (the plain path), in galaxy-steps/s."""
    from khrr.galaxy import ensemble_sizes, make_galaxy
    sizes = ensemble_sizes(64, seed=77)
    parts = [make_galaxy(ns, nd, 2000 + k).arrays() for k, (ns, nd) in enumerate(sizes)]
    pos = np.concatenate([p[0] for p in parts])
    vel = np.concatenate([p[1] for p in parts])
    mass = np.concatenate([p[2] for p in parts])
    eps2 = np.concatenate([p[3] ** 2 for p in parts])
    off = np.cumsum([0] + [len(p[2]) for p in parts])
    out = {"galaxies": 64, "bodies": int(off[-1]), "pairs_per_step": float(sum(len(p[2]) ** 2 for p in parts))}
    ctx = khrr.Context(ctx_device)
    try:
        # the batched path's kernel shape from the autotuner (cached per layout)
        ctx.upload(pos, vel, mass, eps2, offsets=off)
        ctx.autotune(ROOT / "khrr-nbody_b200" / "build" / f"autotune_cache.{ctx_device}.json")
        out["tuning"] = ctx.get_tuning()
        for label, flags in (("batched", 0), ("plain", khrr.PLAIN)):
            ctx.upload(pos, vel, mass, eps2, offsets=off)
            ctx.forces(khrr.ACC | (flags & khrr.PLAIN))
            ctx.step(DT, 2, flags)
            s = torch.cuda.ExternalStream(ctx.stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ctx.synchronize()
            e0.record(s)
            ctx.step(DT, steps, flags)
            e1.record(s)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            out[label + "_galaxy_steps_per_s"] = 64 * steps / (ms * 1e-3)
            out[label + "_ms_per_step"] = ms / steps
        # accuracy of the batched pass vs FP64 on sampled bodies of every galaxy
        ctx.upload(pos, vel, mass, eps2, offsets=off)
        ctx.forces(khrr.ACC)
        acc = ctx.download(pos=False, vel=False, phi=False)["acc"]
        rng = np.random.default_rng(3)
        tg = np.sort(rng.choice(len(mass), 4096, replace=False))
        ref, _ = ctx.accel_fp64_sample(tg)
        out["acc_rel_rms_vs_fp64"] = float(np.sqrt(((acc[tg] - ref) ** 2).sum() / (ref ** 2).sum()))
    finally:
        ctx.close()
    out["batched_over_plain"] = out["batched_galaxy_steps_per_s"] / out["plain_galaxy_steps_per_s"]
    return out


def mesh_leg(khrr, device, torch, hbm_gbs, iter_cap=0):
    """p2mesh on the configs' meshes: the two-galaxy encounter (786,432 bodies,
    128^3 cells over [-4,4]^3, residual 1e-5) and the large system (2,097,152
    bodies, 256^3 cells, residual 1e-6).  Algorithmic bytes: binning + mass
    deposit + scan = 40 B per body (FP64 position and mass read, cell id and
    slot written) + 24 B per cell (count and mass zeroed, count read, both
    start views written); one FP32 stencil iteration = 16 B per cell (phi,
    phi_old, mass read, phi_new written)."""
    import ctypes as C
    from khrr.galaxy import assemble, make_galaxy, two_galaxy_encounter
    cases = {
        "encounter_128": (lambda: two_galaxy_encounter(), 128, 4.0, 1e-5, 40000),
        "large_256": (lambda: assemble([make_galaxy(698368, 1398784, 4000, eps_stars=0.002, eps_dm=0.002)],
                                       [(0.0, (0, 0, 0), (0, 0, 0))]), 256, 4.0, 1e-6, 20000),
    }
    out = {}
    ctx = khrr.Context(device)
    try:
        for label, (gen, nx, L, tol, max_iter) in cases.items():
            pos, vel, mass, eps2 = gen()
            n, ncells = len(mass), nx ** 3
            ctx.upload(pos, vel, mass, eps2)
            s = torch.cuda.ExternalStream(ctx.stream)
            mesh = khrr.Mesh.make((-L,) * 3, (2 * L / nx,) * 3, (nx, nx, nx))
            nul = [None] * 6
            ctx._check(ctx.L.khrr_bin(ctx.h, C.byref(mesh), *nul))
            best = 1e30
            for _ in range(5):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(s)
                ctx._check(ctx.L.khrr_bin(ctx.h, C.byref(mesh), *nul))
                e1.record(s)
                e1.synchronize()
                best = min(best, e0.elapsed_time(e1))
            bin_bytes = 40.0 * n + 24.0 * ncells
            W = khrr.WaveParams.make(nx, 2 * L / nx)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            if iter_cap > 0:
                max_iter = min(max_iter, iter_cap)
            it, res, _ = ctx.wave_solve(W, tol=tol, max_iter=max_iter, check_every=50, cold=True, want_phi=False)
            e1.record(s)
            e1.synchronize()
            wms = e0.elapsed_time(e1)
            per_it = wms / max(it, 1)
            wave_gbs = 16.0 * ncells / (per_it * 1e-3) / 1e9

            def timed(fn, reps=5):
                best = 1e30
                for _ in range(reps):
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(s)
                    fn()
                    b.record(s)
                    b.synchronize()
                    best = min(best, a.elapsed_time(b))
                return best

            # CIC deposit (the configs bin CIC) and the counting-sort order of the bin.
            P = torch.as_tensor(np.ascontiguousarray(pos).reshape(-1), device=device)
            M = torch.as_tensor(np.ascontiguousarray(mass), device=device)
            CM = torch.zeros(ncells, dtype=torch.float64, device=device)
            torch.cuda.synchronize()

            def cic():
                ctx._check(ctx.L.khrr_cic_deposit(ctx.h, P.data_ptr(), M.data_ptr(), n, C.byref(mesh), CM.data_ptr()))
            cic_ms = timed(cic)
            cic_bytes = 32.0 * n + 16.0 * ncells
            sort_ms = timed(lambda: ctx.sort_by_cell(want=False))
            del P, M, CM
            out[label] = {
                "bodies": n, "cells": ncells,
                "bin_scan_deposit_ms": best, "bin_gbs": bin_bytes / (best * 1e-3) / 1e9,
                "bin_frac_of_hbm": bin_bytes / (best * 1e-3) / 1e9 / hbm_gbs,
                "wave_iterations": it, "wave_residual": res, "wave_ms_per_iteration": per_it,
                "wave_gbs": wave_gbs, "wave_frac_of_hbm": wave_gbs / hbm_gbs,
                "wave_working_set_mb": 16.0 * ncells / 1e6,
                "wave_note": "L2-resident working set" if 16.0 * ncells < 126e6 else "HBM-resident",
                "cic_deposit_ms": cic_ms, "cic_gbs": cic_bytes / (cic_ms * 1e-3) / 1e9,
                "cic_bytes_note": "32 B per body (FP64 position, mass) + 16 B per cell (zeroed, summed)",
                "sort_ms": sort_ms, "sort_gbs": 16.0 * n / (sort_ms * 1e-3) / 1e9,
            }
            if label == "large_256":
                # The reference's own FP64 stencil (wave_diss_iteration's
                # expression, khrr_wave_iteration) on the same mesh: 32 B/cell.
                f64 = [torch.zeros(ncells, dtype=torch.float64, device=device) for _ in range(3)]
                m64 = torch.rand(ncells, dtype=torch.float64, device=device) * 1e-4  # timing only: values do not matter
                torch.cuda.synchronize()
                k = [0]

                def f64_iter():
                    o, c, nx_ = f64[k[0] % 3], f64[(k[0] + 1) % 3], f64[(k[0] + 2) % 3]
                    ctx.wave_iteration(nx_.data_ptr(), c.data_ptr(), o.data_ptr(), m64.data_ptr(), W)
                    k[0] += 1
                f64_iter()

                def f64_run():
                    for _ in range(20):
                        f64_iter()
                f64_ms = timed(f64_run, reps=3) / 20
                out[label].update({"wave_f64_ms_per_iteration": f64_ms,
                                   "wave_f64_gbs": 32.0 * ncells / (f64_ms * 1e-3) / 1e9,
                                   "wave_f64_frac_of_hbm": 32.0 * ncells / (f64_ms * 1e-3) / 1e9 / hbm_gbs})
                del f64, m64
            if label == "encounter_128":
                # The reference's Wave mode on this mesh: FP32 stencil, CIC,
                # (int)(dt / dt_wave) iterations per dt = 0.002 step.
                ips = int(0.002 / W.dt)
                ctx.set_mesh_solver(W, assign=khrr.ASSIGN_CIC, fp64=False, iters_per_step=ips, setup_iters=2000)
                try:
                    ctx.forces(khrr.ACC | khrr.MESH)
                    ctx.step(0.002, 3, khrr.MESH)   # builds the graphs of all three ring rotations
                    step_ms = timed(lambda: ctx.step(0.002, 1, khrr.MESH), reps=3)
                finally:
                    ctx.set_mesh_solver(None)
                out[label].update({"wave_mode_step_ms": step_ms, "wave_mode_iters_per_step": ips,
                                   "wave_mode_gbs": 16.0 * ncells * ips / (step_ms * 1e-3) / 1e9})
    finally:
        ctx.close()
    return out


def kick_drift_leg(khrr, ctx, torch, n, hbm_gbs):
    """The predictor and corrector as the reference launches them
    (khrr_integ_time = kernelNbody_integTime, nbody-kernel.cuh:144-193) on n
    bodies in device memory, in achieved GB/s of algorithmic bytes: predictor
    120 B per body (read acc, pos, vel; write pos_t, vel_t), corrector 168 B
    (read acc, pos, vel, vel_t; write pos_t, vel_t, acc0)."""
    g = torch.Generator(device="cuda").manual_seed(3)
    arr = lambda: torch.randn((n, 3), dtype=torch.float64, device="cuda", generator=g)
    acc, pos, vel, pos_t, vel_t, acc0 = arr(), arr(), arr(), arr(), arr(), arr()
    s = torch.cuda.ExternalStream(ctx.stream)
    torch.cuda.synchronize()
    out = {}
    for istep, label, nbytes in ((0, "predictor", 120), (1, "corrector", 168)):
        call = lambda: ctx.integ_time(acc.data_ptr(), pos_t.data_ptr(), vel_t.data_ptr(), pos.data_ptr(),
                                      vel.data_ptr(), DT, istep, 0.0, acc0.data_ptr(), n)
        for _ in range(3):
            call()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 20
        e0.record(s)
        for _ in range(reps):
            call()
        e1.record(s)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / reps
        gbs = nbytes * n / (ms * 1e-3) / 1e9
        out[label] = {"ms": ms, "gbs": gbs, "frac_of_hbm": gbs / hbm_gbs, "bytes_per_body": nbytes}
    out["bodies"] = n
    out["note"] = f"{120 * n / 1e6:.0f}-{168 * n / 1e6:.0f} MB per pass (above the 126 MB L2)"
    return out


def max_over_ranks(dist, values, device="cpu"):
    """Element-wise maximum of per-rank timings over all ranks (the identity
    without a process group).  Every rank calls it at the same point."""
    if not dist:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def replica_rate(world, pairs_per_step, steps, ms_max):
    """Whole-job interactions per second (G/s) of `world` independent
    replicas, each doing `steps` steps of `pairs_per_step` pairs, timed as the
    slowest rank's `ms_max`."""
    return world * pairs_per_step * steps / (ms_max * 1e-3) / 1e9


def run_khrr(args):
    import torch
    import khrr

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist:
            dist.barrier()

    pos, vel, mass, eps2 = workload(args.n_stars, args.n_dm)
    n = len(mass)
    ctx = khrr.Context(local)
    ctx.upload(pos, vel, mass, eps2)
    # kernel shape picked by the autotuner (timed candidates, cached per layout;
    # one cache file per local rank, so replicas never write the same file)
    ctx.autotune(ROOT / "khrr-nbody_b200" / "build" / f"autotune_cache.{local}.json")
    ctx.forces(khrr.ACC)

    # accuracy vs FP64 on 4096 seeded targets (GPU FP64 direct sum)
    acc0 = ctx.download(pos=False, vel=False, phi=False)["acc"]
    rng = np.random.default_rng(11)
    tg = np.sort(rng.choice(n, min(4096, n), replace=False))
    ref, _ = ctx.accel_fp64_sample(tg)
    err = float(np.sqrt(((acc0[tg] - ref) ** 2).sum() / (ref ** 2).sum()))
    err_max = float(np.max(np.linalg.norm(acc0[tg] - ref, axis=1) / np.linalg.norm(ref, axis=1)))

    # conservation at the start (potentials of the current positions)
    ctx.forces(khrr.ACC | khrr.PHI)
    lie0 = ctx.conservation()

    stream = torch.cuda.ExternalStream(ctx.stream)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        ctx.step(DT, 1)
        with torch.cuda.stream(stream):
            flush.zero_()
    ctx.synchronize()
    barrier()
    torch.cuda.synchronize()
    ctx.enable_timing(True)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    gpu_id = local
    try:
        gpu_id = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    with ClockSampler(gpu_id) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            ctx.step(DT, 1)
            with torch.cuda.stream(stream):
                flush.zero_()
        ev1.record(stream)
        ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    force_ms, launches, pairs_timed = ctx.force_timing()
    ctx.enable_timing(False)
    tuning = ctx.get_tuning()
    if launches < 1 or force_ms <= 0.0:
        raise RuntimeError("force-kernel timing events recorded nothing")
    # conservation after warm-up + timed steps (one more step, with potentials,
    # outside the timed region): relative energy and L_z drift over the run
    ctx.step(DT, 1, khrr.PHI)
    lie1 = ctx.conservation()
    drift = {"steps": args.warmup + args.steps + 1,
             "energy_rel": abs(lie1["E"] / lie0["E"] - 1.0),
             "lz_rel": abs(lie1["Lz"] / lie0["Lz"] - 1.0) if lie0["Lz"] != 0 else None}

    # the plain path on the same galaxy: the conventional one-body-per-thread
    # FP32 kernel, one launch per system (CUDA events, outside the timed region)
    ctx.upload(pos, vel, mass, eps2)
    ctx.forces(khrr.ACC | khrr.PLAIN)
    ctx.step(DT, 1, khrr.PLAIN)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    ctx.step(DT, 2, khrr.PLAIN)
    p1.record(stream)
    p1.synchronize()
    plain_ms = p0.elapsed_time(p1) / 2
    plain = {"value": float(n) * n / (plain_ms * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": plain_ms,
             "what": "KHRR_PLAIN: one i body per thread, 256-body shared-memory j tiles, one launch per system"}

    barrier()
    (ms_max,) = max_over_ranks(dist, [ms], device="cuda")
    pairs_step = float(n) * n
    value = replica_rate(world, pairs_step, args.steps, ms_max)

    # end to end through the C ABI: pinned host inputs -> step -> host outputs
    pin = lambda shape: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
    h_pos, h_vel, h_mass, h_eps2, h_acc = pin((n, 3)), pin((n, 3)), pin(n), pin(n), pin((n, 3))
    o_pos, o_vel, o_acc = pin((n, 3)), pin((n, 3)), pin((n, 3))
    h_pos[:], h_vel[:], h_mass[:], h_eps2[:], h_acc[:] = pos, vel, mass, eps2, acc0
    ptr = lambda a: a.ctypes.data
    e2e_ms = []
    for k in range(args.warmup + args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.upload_ptrs(n, ptr(h_pos), ptr(h_vel), ptr(h_mass), ptr(h_eps2))
        ctx.set_accelerations_ptr(ptr(h_acc))
        ctx.step(DT, 1)
        ctx.download_into(o_pos.ctypes.data, o_vel.ctypes.data, o_acc.ctypes.data, None)
        e1.record(stream)
        e1.synchronize()
        if k >= args.warmup:
            e2e_ms.append(e0.elapsed_time(e1))
    (e2e_total,) = max_over_ranks(dist, [sum(e2e_ms)], device="cuda")
    e2e_value = replica_rate(world, pairs_step, args.steps, e2e_total)

    peaks = measured_peaks()
    sm_max = float(peaks.get("sm_max_mhz", 1965.0))
    peak_tflops = SMS * FP32_LANES * 2 * sm_max * 1e6 / 1e12
    avg_launch_s = force_ms / max(launches, 1) * 1e-3
    pair_kernel = tuning["packed"] == 2
    achieved = FLOPS_PER_PAIR * (pairs_timed / max(launches, 1)) / avg_launch_s / 1e12
    executed = force_flops(n, pair_kernel) / avg_launch_s / 1e12
    probe = ctx.fp32_probe()

    kick = None
    if rank == 0:
        kick = kick_drift_leg(khrr, ctx, torch, 4 * n, float(peaks.get("hbm_gbs", 6650.0)))
    ens = None
    if not args.no_ensemble and rank == 0:
        ens = ensemble_leg(khrr, local, torch)
    mesh = None
    if not args.no_mesh and rank == 0:
        mesh = mesh_leg(khrr, local, torch, float(peaks.get("hbm_gbs", 6650.0)), args.mesh_max_iter)
    ctx.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, cores, kind, sample, _ = cpu_reference_sample(pos, mass, eps2, 15.0, np.random.default_rng(5))
        cpu = {"value": rate / 1e9, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "steps_per_s": 1e3 * args.steps / ms_max,
        "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 pair terms (compensated sums), f64 integrator",
        "data": "synthetic (seeded disk-galaxy generator)",
        "config": config(args, {"tuning": tuning}),
        "pct_fp32_peak": 100.0 * achieved / peak_tflops,
        "pct_fp32_peak_executed": 100.0 * executed / peak_tflops,
        "acc_rel_rms_vs_fp64": err, "acc_rel_max_vs_fp64": err_max, "acc_err_targets": int(len(tg)),
        "drift": drift,
        "plain": plain,
        "roofline": {"bound": "fp32", "kernel": "pair_kernel" if pair_kernel else "force_kernel",
                     "achieved": achieved, "peak": peak_tflops,
                     "unit": "TFLOP/s", "frac": achieved / peak_tflops,
                     # DRAM read+write of one force launch from ncu captures: the
                     # pair kernel's 6.09 GB at 786,432 bodies (its FP32 partial
                     # slots, ~n x blocks / 2 of them) scaled by n^2; the one-sided
                     # kernel's 2.80 MB at 131,072 (the shadow, once) by n.
                     "traffic": 6.09e9 * (n / 786432) ** 2 if pair_kernel else 2.80e6 * n / 131072,
                     "flops_per_pair": FLOPS_PER_PAIR, "pairs_per_launch": pairs_timed / max(launches, 1),
                     "executed": {"tflops": executed, "frac": executed / peak_tflops,
                                  "flops_per_launch": force_flops(n, pair_kernel),
                                  "what": "FP32 flops the kernel executes (FMA = 2): pair kernel 23 per "
                                          "unordered pair of different blocks + 17 per pair inside a block; "
                                          "one-sided kernel 17 per ordered pair"},
                     "avg_launch_ms": avg_launch_s * 1e3,
                     "peak_basis": f"nominal FP32: {SMS} SMs x {FP32_LANES} lanes x 2 flops x {sm_max:.0f} MHz "
                                   "(sm_max_mhz of MEASURED_PEAKS.json)",
                     "fp32_fma_probe_tflops": probe},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": int(n * (24 + 24 + 8 + 8 + 24)),
                "d2h_bytes_per_step": int(n * (24 + 24 + 24)),
                "what": "khrr_upload_state + khrr_set_accelerations (pinned host) + khrr_step(1) + "
                        "khrr_download_state(pos, vel, acc)"},
        "gpu_launches": 2 * args.steps,
        "clocks": clk.summary(),
        "kick_drift": kick,
        "ensemble": ens,
        "mesh": mesh,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_khrr(args)


if __name__ == "__main__":
    sys.exit(main())
