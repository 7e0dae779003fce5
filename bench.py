#!/usr/bin/env python
"""Benchmark of the msbg-rs sparse-grid hot path on B200.

Workloads (--workload; every input is seeded synthetic data, no dataset
exists for this path):

flip (default): one FLIP transfer step.  256^3 domain, 16^3 blocks, three
  resolution levels chosen per block by the distance of its centre to the
  sphere |x - c| = 89.6 (< 16 cells: level 0, < 48: level 1, else level 2), 8
  particles per level-0 cell uniformly jittered inside the cell (25,427,968
  particles), velocities N(0, 1), mass 1, in shuffled order.  One step:
    1. Morton sort of the particles by morton3 of their cell (21 bits per axis)
       and the payload gather into sorted order,
    2. P2G: splat of mass and momentum to the MAC faces (r_p = 2) + normalise,
    3. 2^3 downsample of the splatted x-face mass to the coarse level and 10
       sweeps of the 19-tap mean-curvature smoother (dt 0.025) over the level-0
       blocks, halos of coarser neighbours sampled from the coarse level,
    4. G2P: trilinear MAC sample at every particle + FLIP/PIC blend (alpha 0.95).
  metric = particles through the whole step per second.  Inputs (713 MB of
  particle data) are larger than L2: no flush needed.

smoother: the single-level shell (blocks meeting |‖x - c‖ - 0.35 size| <= 6),
  U[-1, 1] values; one step = 10 in-place 8-colour sweeps of the 7-tap stencil
  (dt 0.025).  Default size 2048 (56,056 blocks, 918 MB, larger than L2).
  metric = cell-updates per second; the 19- and 25-tap stencils and 10 sweeps
  of the weighted-Jacobi Poisson relaxation (w = 2/3) are reported beside it.

poisson: the pressure solve on the level-0 blocks of the FLIP layout (776
  blocks, 3.18 M unknowns, zero Dirichlet outside), right-hand side the
  divergence of a random smooth velocity field (32 Gaussian blobs).  One step =
  one solve from x = 0 to 1e-6 relative residual; metric = milliseconds per
  solve (lower is better); plain multigrid V-cycles and MG-preconditioned CG
  are timed beside the learned-preconditioned CG (the network alone, and a
  V-cycle plus the network's correction of its error, the headline), whose
  network is first trained on the device on (residual, multigrid error)
  pairs the solver generates for other right-hand sides.

batched: 64 independent sparse Poisson problems (edges from {32, 64, 128,
  256}, 8^3 or 16^3 blocks, active fraction 5-60 % as random shells,
  right-hand sides U[-1, 1] with the mean removed) solved together to 1e-8
  relative residual: MG-preconditioned CG with per-problem scalars on the
  device, one CUDA graph launch per cycle of 8 iterations, FP64 solution and
  residual replacement, launch shapes autotuned per level; errors against the
  FP64 oracle are reported for the smallest problems.

phasefield: the full phase-field FLIP step on a 512^3 domain of 16^3 blocks:
  a sphere of radius 0.3 * 512 perturbed by 3-octave value noise (amplitude
  10 cells), 4 levels by distance to the surface, 8 particles per cell in a
  band of width 24 (52.8 M particles), a BF16 phase field on the level-0
  blocks.  One step = Morton sort, P2G, 10 sweeps of the 25-tap
  smoother on the BF16 phase field, divergence, pressure solve to 1e-6
  (learned V-cycle/network/V-cycle CG, timed beside MG-PCG and plain MG),
  G2P + blend.  The BF16 storage error is stated against the same sweeps
  with f32 storage.

--impl reference times the reference algorithm on the host CPU (the C++
restatement in oracle/, all host threads) on a bounded sample of the same
workload.  With --gpus N > 1 every rank runs an independent replica (the
path has no exchange step).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "FLIP transfer step throughput (Morton sort + P2G + 19-tap multires smoother + G2P)"
UNIT = "particles/s"
R_P = 2.0
DT = 0.025
SWEEPS = 10
ALPHA = 0.95


def load_package():
    import importlib.util

    if "msbg_rs_b200" in sys.modules:
        return sys.modules["msbg_rs_b200"]
    pkg_dir = os.path.join(ROOT, "msbg-rs_b200")
    spec = importlib.util.spec_from_file_location("msbg_rs_b200", os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["msbg_rs_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sms, maxes, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sms.append(float(f[1]))
                maxes.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sms) if sms else None, "sm_max_mhz": max(maxes) if maxes else None,
                "reasons": sorted(reasons), "samples": len(sms)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def make_workload(msbg, size):
    from msbg_rs_b200 import workloads

    ft = workloads.flip_transfer(size=size, bsx=16, seed=2, ppc=8)
    order = np.random.default_rng(12).permutation(ft.n)  # particles arrive unsorted
    return ft, ft.pos[order], ft.vel[order], ft.mass[order]


def timing_report(msbg, ctx, reset=True):
    n = C.c_size_t()
    msbg._lib.call("msbg_ctx_timing_report", ctx.handle, 0, None, 0, C.byref(n))
    buf = C.create_string_buffer(n.value + 1)
    msbg._lib.call("msbg_ctx_timing_report", ctx.handle, int(reset), buf, n.value + 1, C.byref(n))
    out = {}
    for line in buf.value.decode().splitlines():
        name, cnt, ms = line.split()
        out[name] = (int(cnt), float(ms))
    return out


def run_ours(args, world, rank, local):
    import torch

    msbg = load_package()
    from msbg_rs_b200._lib import call, ptr

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta

        dist_mod.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
        dist = dist_mod

    ft, pos_h, vel_h, mass_h = make_workload(msbg, args.size)
    n = ft.n
    ctx = msbg.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    pos = torch.from_numpy(pos_h).to(dev)
    vel = torch.from_numpy(vel_h).to(dev)
    mass = torch.from_numpy(mass_h).to(dev)
    keys = torch.empty(n, dtype=torch.int64, device=dev)
    perm = torch.empty(n, dtype=torch.int32, device=dev)
    spos = torch.empty_like(pos)
    svel = torch.empty_like(vel)
    smass = torch.empty_like(mass)
    u = torch.empty_like(vel)
    u_new = torch.empty_like(vel)
    torch.cuda.synchronize()

    mac = msbg.MacGrid(ctx, args.size, args.size, args.size, 16)
    coarse = msbg.SparseGrid(ctx, args.size // 2, args.size // 2, args.size // 2, 0.0, 0.0, 8, name="coarse_mass_x")
    levels = ft.levels
    sweeper = msbg.Sweeper(mac.mass(0))
    sampler = msbg.MacSampler(mac, msbg.CLAMP)
    fine_set = None
    state = {}

    def step(p=pos, v=vel, m=mass, events=None, before_blend=None):
        def mark(name):
            if events is not None:
                e = torch.cuda.Event(enable_timing=True)
                e.record(stream)
                events.append((name, e))

        mark("start")
        call("msbg_morton_sort_device", ctx.handle, ptr(p), n, ptr(keys), ptr(perm))
        # the particles into Morton order: the splat's gather and G2P then read
        # them in cell order (measured: gathering through the permutation
        # inside P2G and G2P in the caller's order cost 0.6 ms more a step)
        call("msbg_permute_device", ctx.handle, ptr(perm), n, 3, ptr(p), ptr(spos))
        call("msbg_permute_device", ctx.handle, ptr(perm), n, 3, ptr(v), ptr(svel))
        call("msbg_permute_device", ctx.handle, ptr(perm), n, 1, ptr(m), ptr(smass))
        mark("sort")
        msbg.particles_to_grid_sorted_device(mac, spos, svel, smass, keys, n, R_P)
        mark("p2g")
        act = mac.active_blocks()
        fine = act[levels[act.astype(np.int64)] == 0]
        state["active"], state["fine"] = act, fine
        msbg.downsample_channel_avg(coarse, mac.mass(0))
        sweeper.sweep_multires(coarse, levels, fine, msbg.Stencil.MeanCurvature, msbg.PdeParams(DT, SWEEPS, False))
        mark("smooth")
        if before_blend is not None:
            before_blend()  # u_new of the previous step has been read back
        # MacSampler::sample and g2p_blend in one pass (u_tilde = the sample)
        msbg.g2p_flip_device(sampler, spos, n, svel, ALPHA, u_new)
        mark("g2p")

    # warm-up
    for _ in range(args.warmup):
        step()
    ctx.synchronize()
    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = ctx.kernel_launches()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    phase_ms = {}
    all_events = []
    t0.record(stream)
    for _ in range(args.steps):
        ev = []
        step(events=ev)
        all_events.append(ev)
    t1.record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = ctx.kernel_launches() - launches0
    ms = t0.elapsed_time(t1) / args.steps
    for ev in all_events:
        for (a, ea), (b, eb) in zip(ev[:-1], ev[1:]):
            phase_ms[b] = phase_ms.get(b, 0.0) + ea.elapsed_time(eb) / args.steps
    ms = _max_over_ranks(dist, ms, dev)
    # per-kernel device times: a separate pass with an event pair around every
    # library launch (kept out of the timed region above)
    prof_steps = max(1, min(args.steps, 5))
    call_timing(msbg, ctx, True)
    for _ in range(prof_steps):
        step()
    kernels = timing_report(msbg, ctx, reset=True)
    call_timing(msbg, ctx, False)

    # ---- end to end through the C ABI with host buffers ----------------------
    pin_pos = torch.from_numpy(pos_h).pin_memory()
    pin_vel = torch.from_numpy(vel_h).pin_memory()
    pin_mass = torch.from_numpy(mass_h).pin_memory()
    pin_out = torch.empty((n, 3), dtype=torch.float32).pin_memory()
    # Every step copies its inputs from pinned host memory and reads its new
    # velocities back.  The copies run on two copy streams, overlapped with
    # the device work: the inputs are double-buffered, so the next step's
    # inputs go up while this step runs (into the buffers the previous step
    # has finished with), and this step's result comes down while the next
    # step runs (its blend waits for that read).  The library's own small
    # reads (status words, counts) bypass the copy engines, so they do not
    # wait behind these transfers.
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e2e_steps = max(1, min(args.steps, 10))
    up = torch.cuda.Stream(device=dev)
    down = torch.cuda.Stream(device=dev)
    held = {}
    sets = [(pos, vel, mass), (torch.empty_like(pos), torch.empty_like(vel), torch.empty_like(mass))]

    def upload(k):
        with torch.cuda.stream(up):
            p_, v_, m_ = sets[k % 2]
            p_.copy_(pin_pos, non_blocking=True)
            v_.copy_(pin_vel, non_blocking=True)
            m_.copy_(pin_mass, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(up)
        held[("inputs", k)] = ev

    e0.record(stream)
    up.wait_event(e0)
    upload(0)
    for i in range(e2e_steps):
        stream.wait_event(held[("inputs", i)])
        if i + 1 < e2e_steps:
            if "done" in held:
                up.wait_event(held["done"])  # step i - 1 is done with the buffers of step i + 1
            upload(i + 1)

        def before_blend():
            if "read" in held:
                stream.wait_event(held["read"])

        step(*sets[i % 2], before_blend=before_blend)
        oe = torch.cuda.Event()
        oe.record(stream)
        held["done"] = oe
        down.wait_event(oe)
        with torch.cuda.stream(down):
            pin_out.copy_(u_new, non_blocking=True)
            rd = torch.cuda.Event()
            rd.record(down)
        held["read"] = rd
    e1.record(down)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    h2d = pin_pos.numel() * 4 + pin_vel.numel() * 4 + pin_mass.numel() * 4
    d2h = pin_out.numel() * 4
    if dist:
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())

    # ---- end to end through the host-array entry point ----------------------
    # msbg_flip_step: one call per step copies the step's inputs up from the
    # (page-locked) host arrays, runs the whole step and returns once the new
    # velocities are in the host output array -- what a host caller of the
    # C ABI gets per step.  The pipelined figure above overlaps the copies of
    # neighbouring steps with torch streams around the device-pointer entry
    # points instead.
    fstep = msbg.FlipStep(mac, coarse, levels)
    fargs = (pin_pos.data_ptr(), pin_vel.data_ptr(), pin_mass.data_ptr(), n, R_P, int(msbg.Stencil.MeanCurvature), DT,
             SWEEPS, ALPHA, pin_out.data_ptr())
    fstep.step_ptrs(*fargs)  # sizes the step's device arrays
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(e2e_steps):
        fstep.step_ptrs(*fargs)
    f1.record(stream)
    torch.cuda.synchronize()
    abi_ms = _max_over_ranks(dist, f0.elapsed_time(f1) / e2e_steps, dev)
    fstep.close()

    # ---- roofline of the dominant kernel ------------------------------------
    peak, peak_kind = load_peaks()
    dom = max(kernels.items(), key=lambda kv: kv[1][1]) if kernels else ("none", (1, 1.0))
    n_fine = len(state["fine"])
    n_active = len(state["active"])
    algo = algorithmic_bytes(dom[0], n=n, n_fine=n_fine, n_active=n_active, launches=dom[1][0])
    roof = None
    if algo is not None:
        achieved = algo / (dom[1][1] * 1e-3) / 1e9
        per_launch = algo / dom[1][0]
        traffic = measured_traffic(dom[0], n=n)
        roof = {"kernel": dom[0], "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "traffic": traffic, "algorithmic_bytes_per_launch": per_launch, "launches": dom[1][0],
                "avg_launch_us": round(dom[1][1] / dom[1][0] * 1e3, 2)}
        ipu = INST_PER_UNIT.get(dom[0])
        if ipu is not None:
            sms = torch.cuda.get_device_properties(dev).multi_processor_count
            mhz = (clk or {}).get("sm_mhz") or (clk or {}).get("sm_max_mhz") or 1965.0
            ach = ipu * n * dom[1][0] / (dom[1][1] * 1e-3) / 1e9
            pk = 4.0 * sms * mhz * 1e6 / 1e9
            roof["issue"] = {"inst_per_particle_per_launch": round(ipu, 1), "achieved_ginst_s": round(ach, 1),
                             "peak_ginst_s": round(pk, 1), "frac": round(ach / pk, 4),
                             "source": "warp instructions per particle and launch from ncu at 128^3; peak = 4 per "
                                       "SM per clock at the sampled SM clock"}
    sweep_k = sweep_kernel_time(kernels)
    smoother = None
    if sweep_k:
        cells = n_fine * 4096 * SWEEPS * prof_steps
        smoother = {"cell_updates_per_s": cells / (sweep_k[1] * 1e-3), "gbs_algorithmic": 8 * cells / (sweep_k[1] * 1e-3) / 1e9,
                    "frac_of_hbm": 8 * cells / (sweep_k[1] * 1e-3) / 1e9 / peak}

    value = world * n / (ms * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded; no dataset exists for this path)",
        "config": {"workload": f"FLIP transfer {args.size}^3, 16^3 blocks, 3 levels, 8 particles per level-0 cell",
                   "particles": n, "level_blocks": np.bincount(ft.levels, minlength=3).tolist(),
                   "p2g_active_blocks": n_active, "smoothed_level0_blocks": n_fine, "r_p": R_P,
                   "sweeps": SWEEPS, "stencil": "19-tap mean curvature", "parallelism": f"replicas x{world}",
                   "l2": "inputs (713 MB) larger than L2, no flush"},
        "e2e": {"value": world * n / (abi_ms * 1e-3), "unit": UNIT, "ms_per_step": abi_ms, "steps": e2e_steps,
                "api": "msbg_flip_step (C ABI, host arrays in page-locked memory; returns with the new velocities "
                       "in the host array, in the caller's particle order)",
                "copies": "every step: positions, velocities and masses host->device (velocities and masses beside "
                          "the sort), new velocities device->host",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "pipelined_device_api": {
                    "value": world * n / (e2e_ms * 1e-3), "ms_per_step": e2e_ms,
                    "copies": "the same bytes on two torch copy streams, overlapped with the device work of "
                              "neighbouring steps (double-buffered inputs; identical inputs every step)"}},
        "gpu_launches": launches,
        "phases_ms": {k: round(v, 4) for k, v in phase_ms.items()},
        "kernels_ms_per_step": {k: round(v[1] / prof_steps, 4) for k, v in sorted(kernels.items(), key=lambda kv: -kv[1][1])},
        "submetrics": {"p2g_particles_per_s": n / (phase_ms.get("p2g", float("nan")) * 1e-3),
                       "smoother": smoother},
        "roofline": roof,
        "clocks": clk,
    }
    if world == 1 and not args.no_submetrics:
        # the other two parts of the metric, on their own configurations:
        # smoother GB/s on the 2048^3 shell and the pressure solve's time to
        # 1e-6 (plain MG, MG-PCG, learned PCG) on the 256^3 layout
        del pos, vel, mass, keys, perm, spos, svel, smass, u, u_new, sets
        mac.close()
        coarse.close()
        torch.cuda.empty_cache()
        line["submetrics"].update(submetric_lines(args, rank, local))
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(ft, pos_h, vel_h, mass_h, budget_s=args.cpu_budget)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def submetric_lines(args, rank, local):
    """Smoother and pressure-solve parts of the metric, measured in this
    process after the FLIP step (world size 1)."""
    sub = argparse.Namespace(**vars(args))
    sub.size, sub.steps, sub.warmup, sub.stencil = 2048, 3, 1, "laplacian"
    sm = run_smoother(sub, 1, rank, local, emit=False)
    sub = argparse.Namespace(**vars(args))
    sub.size, sub.steps, sub.warmup = 256, 3, 1
    po = run_poisson(sub, 1, rank, local, emit=False)
    m = po["methods"]
    head = po["learned"]["head"]
    return {
        "smoother_shell2048": {
            "config": sm["config"], "cell_updates_per_s_7tap": sm["value"], "ms_per_10_sweeps_7tap": sm["ms_per_step"],
            "roofline_7tap": sm["roofline"], "other_stencils": sm["submetrics"]["other_stencils"],
            "jacobi": sm["submetrics"]["jacobi"], "clocks": sm["clocks"]},
        "poisson_256": {
            "config": po["config"], "metric": "time to 1e-6 relative residual (ms), FP64 true residual",
            "plain_mg_ms": m["plain_mg"]["ms"], "plain_mg_vcycles": m["plain_mg"]["iterations"],
            "mg_pcg_ms": m["mg_pcg"]["ms"], "mg_pcg_iterations": m["mg_pcg"]["iterations"],
            "learned_pcg_ms": m[head]["ms"], "learned_pcg_iterations": m[head]["iterations"],
            "learned_method": head,
            "plain_mg_over_learned": m["plain_mg"]["ms"] / m[head]["ms"],
            "mg_pcg_over_learned": m["mg_pcg"]["ms"] / m[head]["ms"],
            "methods": {k: {"ms": v["ms"], "iterations": v["iterations"]} for k, v in m.items()},
            "training": {k: po["learned"][k] for k in ("pairs", "adam_steps", "train_s", "loss_first", "loss_last")},
            "training_outside_timed_region": True,
            "roofline_jacobi": po["roofline"], "clocks": po["clocks"]},
    }


def algorithmic_bytes(kernel, n, n_fine, n_active, launches):
    """Algorithmic HBM bytes moved by `launches` launches of `kernel` in one
    FLIP transfer step's accounting: 8 B per f32 cell-update for the in-place
    smoother; 28 B per particle once per P2G for the splat (position, velocity
    and mass read once: P2G_SPLAT_LAUNCHES launches make one P2G); 24 B
    written per face-cell of the active blocks for the combine; 12 B read + 12
    B written per particle for G2P; 24 B per element per onesweep radix pass
    (3 passes per sort)."""
    if kernel == "sweep_wave_kernel":  # every phase of the SWEEPS sweeps in one launch
        return 8.0 * n_fine * 4096 * SWEEPS * launches
    if kernel in SWEEP_KERNELS:
        return 8.0 * n_fine * 4096 * SWEEPS * launches / 80
    if kernel == "p2g_cells_kernel":
        return 28.0 * n * launches / P2G_SPLAT_LAUNCHES
    if kernel == "p2g_r2_kernel":
        return 28.0 * n * launches
    if kernel == "p2g_combine_kernel":
        return 24.0 * n_active * 4096 * launches
    if kernel == "g2p_kernel":
        return 24.0 * n * launches
    if kernel == "os_pass_kernel":
        return 24.0 * n * launches
    if kernel == "permute_kernel":
        return 28.0 * n * launches
    return None


# Launches of the general splat kernel per P2G (one per face direction; the
# r_p = 2 kernel does the three directions in one launch).
P2G_SPLAT_LAUNCHES = 3

# DRAM bytes (read + write) per launch measured by ncu on a smaller case of
# the same kernel, per unit of work: p2g_cells_kernel at 128^3 (5,767,168
# particles, one direction per launch) read 167.28 MB and wrote 3.96 MB
# (profiles/p2g_cells_kernel_flip128.txt); traffic grows with the particle
# count, so it is scaled by particles.
TRAFFIC_PER_UNIT = {"p2g_cells_kernel": (167.28e6 + 3.96e6) / 5767168,
                    # r_p = 2 kernel, all three directions in one launch at 128^3
                    # (profiles/p2g_r2_kernel_flip128.txt): 308.83 MB read, 47.21 MB written
                    "p2g_r2_kernel": (308.83e6 + 47.21e6) / 5767168}

# Warp instructions per unit of work from the same capture (575,950,823 per
# launch at 128^3): the splat is bound by instruction issue, not by DRAM, so
# its second roofline is issue slots (4 warp instructions per SM per clock).
INST_PER_UNIT = {"p2g_cells_kernel": 575950823 / 5767168,
                 "p2g_r2_kernel": 1073931570 / 5767168}


# The smoother's sweep kernels (one of them runs, by element type, halo and
# active-set size).
SWEEP_KERNELS = ("sweep_compact_kernel", "sweep_pipe_kernel", "sweep_phase_kernel", "sweep_wave_kernel")


def sweep_kernel_time(kern):
    """(launches, ms) summed over the sweep kernels in a timing report, or None."""
    hits = [kern[k] for k in SWEEP_KERNELS if k in kern]
    return (sum(h[0] for h in hits), sum(h[1] for h in hits)) if hits else None


def sweep_kernel_name(kern):
    hits = [k for k in SWEEP_KERNELS if k in kern]
    return "+".join(hits) if hits else "sweep_compact_kernel"


def measured_traffic(kernel, n):
    per = TRAFFIC_PER_UNIT.get(kernel)
    return None if per is None else per * n


def cpu_baseline(ft, pos_h, vel_h, mass_h, budget_s=20.0):
    """The reference algorithm on the host (oracle/, all host threads) on a
    sample: the particles of the first k level-0 blocks (in block order)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    res = run_cpu_sample(oracle, ft, budget_s)
    return {"value": res["value"], "unit": UNIT, "cores": res["threads"], "kind": "port", "sample": res["sample"]}


def run_cpu_sample(oracle, ft, budget_s, full=False):
    """Times Morton sort + P2G + downsample + 10 multires sweeps + G2P on the
    host for the particles of a contiguous run of level-0 blocks (full: all
    particles, the whole step)."""
    threads = oracle.num_threads()
    size, bsx = ft.size, ft.bsx
    per_block = 8 * bsx ** 3
    k = len(ft.fine_blocks) if full else 8
    results = None
    while True:
        sel = slice(0, ft.n) if full else slice(0, k * per_block)
        pos, vel, mass = ft.pos[sel], ft.vel[sel], ft.mass[sel]
        t = time.perf_counter()
        keys, perm = oracle.morton_sort(pos)
        pos_s, vel_s, mass_s = pos[perm], vel[perm], mass[perm]
        act, ch = oracle.p2g(pos_s, vel_s, mass_s, size, size, size, bsx, R_P, threads=threads)
        msbg = load_package()
        fine = msbg.HostGrid("mass_x", size, size, size, 0.0, 0.0, bsx)
        coarse = msbg.HostGrid("coarse", size // 2, size // 2, size // 2, 0.0, 0.0, bsx // 2)
        for j, b in enumerate(act):
            fine.ensure_block(int(b))
            fine.blocks[int(b)][:] = ch[0][j]
        cblocks = oracle.downsample_avg(ch[0], bsx)
        for j, b in enumerate(act):
            coarse.ensure_block(int(b))
            coarse.blocks[int(b)][:] = cblocks[j]
        lv = ft.levels
        fine_act = [int(b) for b in act if lv[int(b)] == 0]
        oracle.sweep_multires(fine, coarse, lv, fine_act, 1, DT, SWEEPS, False, threads=threads)
        vg = []
        for a in range(3):
            g = msbg.HostGrid(f"v{a}", size, size, size, 0.0, 0.0, bsx)
            for j, b in enumerate(act):
                g.ensure_block(int(b))
                g.blocks[int(b)][:] = ch[3 + a][j]
            vg.append(g)
        u = oracle.mac_sample(vg[0], vg[1], vg[2], pos_s, 0)
        oracle.g2p_blend(vel_s, u, u, ALPHA)
        el = time.perf_counter() - t
        results = {"value": len(pos) / el, "threads": threads, "seconds": el,
                   "sample": f"{len(pos)} particles ({k} level-0 blocks of {len(ft.fine_blocks)}), full step pipeline, "
                             f"{el:.1f} s"}
        if full or el > budget_s / 4 or k * 2 > len(ft.fine_blocks):
            return results
        k *= 2


def run_reference(args, world, rank, local):
    """Reference arm: the reference algorithm (C++ restatement of the crate's
    CPU path, oracle/) timed on the host cores, same metric and workload."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    msbg = load_package()
    from msbg_rs_b200 import workloads

    ft = workloads.flip_transfer(size=args.size, bsx=16, seed=2, ppc=8)
    # every step is the whole step on every particle (the same configuration
    # as the GPU arm); the warm-up steps are the same work, untimed
    for _ in range(args.warmup):
        run_cpu_sample(oracle, ft, budget_s=0.0, full=True)
    vals = [run_cpu_sample(oracle, ft, budget_s=0.0, full=True) for _ in range(args.steps)]
    step_s = statistics.mean(r["seconds"] for r in vals)
    v = ft.n / step_s
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": f"FLIP transfer {args.size}^3, 16^3 blocks, 3 levels, 8 particles per level-0 cell",
                   "particles": ft.n, "parallelism": "host CPU"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": vals[0]["threads"], "kind": "port",
                         "sample": f"the whole step on all {ft.n} particles, every step"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _dist_init(world, local):
    import torch

    torch.cuda.set_device(local)
    if world <= 1:
        return None
    import torch.distributed as dist_mod
    from datetime import timedelta

    dist_mod.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    return dist_mod


def _max_over_ranks(dist, v, dev):
    import torch

    if not dist:
        return v
    t = torch.tensor([v], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _finish(dist):
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# DRAM bytes per launch of the 7-tap sweep phase on the 2048^3 shell (7,007
# blocks per colour), mean of two ncu-captured launches of the compact kernel
# (profiles/sweep_compact_kernel_shell2048.txt): 160.23 MB read + 74.49 MB written.
SWEEP_TRAFFIC_2048 = 160.23e6 + 74.49e6

SMOOTHER_STENCILS = {0: "7-tap laplacian", 1: "19-tap mean curvature", 2: "25-tap bilaplacian"}


def run_smoother(args, world, rank, local, emit=True):
    """10 in-place sweeps of the 7-tap stencil over the shell per step.
    emit=False: no process group, no CPU baseline; returns the line."""
    import torch

    msbg = load_package()
    from msbg_rs_b200 import workloads

    dist = _dist_init(world, local) if emit else None
    dev = torch.device("cuda", local)
    size = args.size or 2048
    sp = workloads.shell_problem(size, 16, seed=1)
    nb = len(sp.active)
    ctx = msbg.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    grid = msbg.SparseGrid(ctx, size, size, size, 0.0, 1.0, 16)
    grid.write_blocks(sp.active, sp.values)
    sw = msbg.Sweeper(grid)
    params = msbg.PdeParams(DT, SWEEPS, False)
    ctx.synchronize()

    def timed(stencil, steps, warmup):
        """Device time per step (no per-launch events), then the per-kernel
        times of a separate pass of `steps` steps with an event pair around
        every launch."""
        for _ in range(warmup):
            sw.sweep(sp.active, stencil, params)
        ctx.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(steps):
            sw.sweep(sp.active, stencil, params)
        t1.record(stream)
        ctx.synchronize()
        call_timing(msbg, ctx, True)
        for _ in range(steps):
            sw.sweep(sp.active, stencil, params)
        kern = timing_report(msbg, ctx, reset=True)
        call_timing(msbg, ctx, False)
        return t0.elapsed_time(t1) / steps, kern

    stencil = {"laplacian": 0, "meancurv": 1, "bilaplacian": 2}[args.stencil]
    for _ in range(args.warmup):
        sw.sweep(sp.active, stencil, params)
    ctx.synchronize()
    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = ctx.kernel_launches()
    ms, kern = timed(stencil, args.steps, 0)
    clk = clocks.stop()
    launches = (ctx.kernel_launches() - launches0) // 2
    ms = _max_over_ranks(dist, ms, dev)
    cells = nb * 4096 * SWEEPS
    peak, peak_kind = load_peaks()
    sk = sweep_kernel_time(kern) or (0, float("nan"))
    k_ms = sk[1] / args.steps
    achieved = 8.0 * cells / (k_ms * 1e-3) / 1e9
    roof = {"kernel": sweep_kernel_name(kern), "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
            "traffic": SWEEP_TRAFFIC_2048 if size == 2048 and stencil == 0 else None,
            "algorithmic_bytes_per_launch": 8.0 * cells / max(sk[0] / args.steps, 1),
            "launches": sk[0], "avg_launch_us": round(sk[1] / max(sk[0], 1) * 1e3, 2),
            "algorithmic": "8 B per f32 cell-update (read + in-place write)"}
    others = {}
    for st in (0, 1, 2):
        if st == stencil:
            continue
        o_ms, o_k = timed(st, 2, 1)
        ok = sweep_kernel_time(o_k) or (1, float("nan"))
        o_gbs = 8.0 * cells / (ok[1] / 2 * 1e-3) / 1e9
        others[SMOOTHER_STENCILS[st]] = {"ms_per_10_sweeps": o_ms, "cell_updates_per_s": cells / (o_ms * 1e-3),
                                         "kernel_gbs_algorithmic": o_gbs, "frac_of_hbm": o_gbs / peak,
                                         "kernel": sweep_kernel_name(o_k)}
    # weighted-Jacobi relaxation of the Poisson operator on the same blocks
    P = msbg.Poisson(ctx, size, size, size, 16, sp.active)
    tuning = P.autotune()  # the library's launch-choice autotuner, outside the timed region
    x = torch.empty(P.n, device=dev)
    b = torch.empty(P.n, device=dev)
    x.uniform_(-1, 1)
    b.uniform_(-1, 1)
    torch.cuda.synchronize()
    P.jacobi(x, b, 2.0 / 3.0, 2)
    ctx.synchronize()
    call_timing(msbg, ctx, True)
    P.jacobi(x, b, 2.0 / 3.0, SWEEPS)
    jk = timing_report(msbg, ctx, reset=True)
    call_timing(msbg, ctx, False)
    jac = jk.get("pk_block16_jacobi") or jk.get("pk_jacobi", (1, float("nan")))
    jacobi = {"sweeps": SWEEPS, "kernel_ms": jac[1], "cell_updates_per_s": P.n * SWEEPS / (jac[1] * 1e-3),
              "gbs_algorithmic": 12.0 * P.n * SWEEPS / (jac[1] * 1e-3) / 1e9,
              "frac_of_hbm": 12.0 * P.n * SWEEPS / (jac[1] * 1e-3) / 1e9 / peak,
              "algorithmic": "12 B per cell-update (x, b read, x written)",
              "autotuned": "per level (Jacobi shape, residual shape, tile): " + str(tuning.tolist())}
    P.close()
    # end to end through the C ABI: host payload in, 10 sweeps, host payload out
    e2e_steps = max(1, min(args.steps, 3))
    t = time.perf_counter()
    for _ in range(e2e_steps):
        grid.write_blocks(sp.active, sp.values)
        sw.sweep(sp.active, stencil, params)
        out = grid.read_blocks(sp.active)
    e2e_ms = (time.perf_counter() - t) * 1e3 / e2e_steps
    e2e_ms = _max_over_ranks(dist, e2e_ms, dev)
    value = world * cells / (ms * 1e-3)
    line = {
        "metric": "smoother cell-updates per second (10 in-place 8-colour sweeps)", "value": value,
        "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded U[-1,1] values; no dataset exists for this path)",
        "config": {"workload": f"shell {size}^3, 16^3 blocks, radius 0.35*size, thickness 12", "blocks": nb,
                   "stencil": SMOOTHER_STENCILS[stencil], "sweeps": SWEEPS, "dt": DT,
                   "parallelism": f"replicas x{world}", "l2": f"grid payload {nb * 16384 / 1e6:.0f} MB; larger than L2, no flush" if nb * 16384 > 126e6 else "grid fits in L2"},
        "e2e": {"value": world * cells / (e2e_ms * 1e-3), "unit": "cell-updates/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": int(sp.values.nbytes), "d2h_bytes_per_step": int(out.nbytes)},
        "gpu_launches": launches,
        "kernels_ms_per_step": {k: round(v[1] / args.steps, 4) for k, v in kern.items()},
        "submetrics": {"gbs_algorithmic": achieved, "other_stencils": others, "jacobi": jacobi},
        "roofline": roof,
        "clocks": clk,
    }
    if not emit:
        grid.close()
        ctx.close()
        return line
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_smoother(sp, stencil, args.cpu_budget)
    if rank == 0:
        print(json.dumps(line), flush=True)
    _finish(dist)


def call_timing(msbg, ctx, on):
    from msbg_rs_b200._lib import call

    call("msbg_ctx_set_timing", ctx.handle, 1 if on else 0)
    if on:
        timing_report(msbg, ctx, reset=True)


def run_cpu_smoother(oracle, sp, stencil, budget_s):
    """The oracle's colour-ordered sweep (10 sweeps) on the first k shell
    blocks, k doubling until the run takes a quarter of the budget."""
    msbg = load_package()
    threads = oracle.num_threads()
    k = 64
    while True:
        sel = sp.active[:k]
        g = msbg.HostGrid("shell", sp.size, sp.size, sp.size, 0.0, 1.0, 16)
        for j, bid in enumerate(sel):
            g.ensure_block(int(bid))
            g.blocks[int(bid)][:] = sp.values[j]
        t = time.perf_counter()
        oracle.sweep(g, sel.astype(np.int64), stencil, DT, SWEEPS, False, threads=threads)
        el = time.perf_counter() - t
        cells = k * 4096 * SWEEPS
        res = {"value": cells / el, "threads": threads, "seconds": el,
               "sample": f"{k} of {len(sp.active)} shell blocks, 10 sweeps, {el:.1f} s"}
        if el > budget_s / 4 or k * 2 > len(sp.active):
            return res
        k *= 2


def cpu_baseline_smoother(sp, stencil, budget_s):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    r = run_cpu_smoother(oracle, sp, stencil, budget_s)
    return {"value": r["value"], "unit": "cell-updates/s", "cores": r["threads"], "kind": "port", "sample": r["sample"]}


def poisson_problem(size=256):
    from msbg_rs_b200 import workloads

    ft = workloads.flip_transfer(size=size, bsx=16, particles=False)
    active = np.unique(ft.fine_blocks)
    b = workloads.smooth_divergence_rhs(size, 16, active, seed=4)
    return active, b


def run_poisson(args, world, rank, local, emit=True):
    """Time to 1e-6 relative residual, plain V-cycles and MG-PCG.
    emit=False: no process group, no CPU baseline; returns the line."""
    import torch

    msbg = load_package()
    dist = _dist_init(world, local) if emit else None
    dev = torch.device("cuda", local)
    size = args.size or 256
    active, bh = poisson_problem(size)
    ctx = msbg.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    P = msbg.Poisson(ctx, size, size, size, 16, active)
    tuning = P.autotune()  # outside the timed region
    b = torch.from_numpy(bh.reshape(-1)).to(dev)
    x = torch.zeros(P.n, device=dev, dtype=torch.float64)
    torch.cuda.synchronize()
    # the learned preconditioner, trained on pairs the solver generates on
    # this geometry (right-hand sides of other seeds than the timed one)
    net = msbg.UNet(ctx, size, size, size, active, seed=1)
    P.set_preconditioner(net)
    t_train = time.perf_counter()
    hist = P.train_preconditioner(n_rhs=args.train_rhs, mg_iters=args.train_iters, steps_per_rhs=args.train_iters,
                                  pool=64, lr=1e-3, target=1, seed=7)
    ctx.synchronize()
    t_train = time.perf_counter() - t_train
    ev = P.eval_preconditioner(n_rhs=2, mg_iters=10, seed=99)
    # (method, network lead applications for LEARNED_LEAD)
    methods = {"plain_mg": (msbg.MG, 0), "mg_pcg": (msbg.PCG, 0), "learned_pcg": (msbg.LEARNED, 0),
               "hybrid_pcg": (msbg.HYBRID, 0), "learned_mg": (msbg.LEARNED_MG, 0),
               "lead1_pcg": (msbg.LEARNED_LEAD, 1), "lead2_pcg": (msbg.LEARNED_LEAD, 2),
               "lead3_pcg": (msbg.LEARNED_LEAD, 3), "lead1_nopost_pcg": (msbg.LEARNED_LEAD, -1)}
    head = "lead1_pcg"

    def one(spec):
        method, lead = spec
        P.set_network_lead(lead)
        x.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        it, rel, hist = P.solve_device(x, b, method=method, tol=1e-6, max_iter=400)
        e1.record(stream)
        ctx.synchronize()
        return e0.elapsed_time(e1), it, rel

    for _ in range(args.warmup):
        one(methods[head])
    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = ctx.kernel_launches()
    times, its = [], []
    for _ in range(args.steps):
        t, it, rel = one(methods[head])
        times.append(t)
        its.append(it)
    clk = clocks.stop()
    launches = ctx.kernel_launches() - launches0
    call_timing(msbg, ctx, True)
    prof_steps = max(1, min(args.steps, 3))
    for _ in range(prof_steps):
        one(methods[head])
    kern = timing_report(msbg, ctx, reset=True)
    call_timing(msbg, ctx, False)
    ms = _max_over_ranks(dist, statistics.mean(times), dev)
    per_method = {}
    for name, m in methods.items():
        one(m)
        t, it, rel = one(m)
        per_method[name] = {"ms": t, "iterations": it, "rel_residual": rel, **P.solve_stats(),
                            "history": [float("%.3g" % v) for v in P.last_history[:12]]}
    # end to end through the C ABI with host arrays: one untimed call, then
    # the mean of `steps` calls (each copies b and x up and x down)
    P.set_network_lead(methods[head][1])
    P.solve(bh.reshape(-1), method=methods[head][0], tol=1e-6, max_iter=400)
    t = time.perf_counter()
    for _ in range(args.steps):
        _, it_h, rel_h, _ = P.solve(bh.reshape(-1), method=methods[head][0], tol=1e-6, max_iter=400)
    e2e_ms = (time.perf_counter() - t) * 1e3 / args.steps
    learned = {"pairs": args.train_rhs * args.train_iters, "adam_steps": int(len(hist)), "train_s": t_train,
               "loss_first": float(np.mean(hist[:20])) if len(hist) else None,
               "loss_last": float(np.mean(hist[-20:])) if len(hist) else None,
               "rel_error_fresh_pairs": ev,
               "head": head,
               "speedup_vs_plain_mg": per_method["plain_mg"]["ms"] / per_method[head]["ms"],
               "speedup_vs_mg_pcg": per_method["mg_pcg"]["ms"] / per_method[head]["ms"]}
    peak, peak_kind = load_peaks()
    # the level-0 Jacobi kernel (16^3 blocks), timed over 20 back-to-back
    # sweeps (inside a solve it runs in captured V-cycles, and per-launch
    # events there would time the host's launch rate)
    n_cells = P.n
    xj = torch.zeros(P.n, device=dev)
    P.jacobi(xj, b, 2.0 / 3.0, 2)
    ja, jb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ja.record(stream)
    P.jacobi(xj, b, 2.0 / 3.0, 20)
    jb.record(stream)
    ctx.synchronize()
    jac_us = ja.elapsed_time(jb) * 1e3 / 20
    jac_gbs = 12.0 * n_cells / (jac_us * 1e-6) / 1e9
    line = {
        "metric": "time to 1e-6 relative residual (Poisson, 7-point, learned-preconditioned CG)", "value": ms, "unit": "ms",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 dots and coarsest solve)",
        "data": "synthetic (seeded smooth-divergence right-hand side; no dataset exists for this path)",
        "config": {"workload": f"Poisson on the level-0 blocks of the {size}^3 3-level layout, 16^3 blocks",
                   "blocks": int(len(active)), "unknowns": int(n_cells), "tol": 1e-6,
                   "smoother": "weighted Jacobi w=2/3, 2+2 sweeps", "parallelism": f"replicas x{world}",
                   "autotuned": tuning.tolist(),
                   "l2": "working set (~64 MB) fits in L2; solves run back to back"},
        "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": int(bh.nbytes) * 2, "d2h_bytes_per_step": int(bh.nbytes)},
        "gpu_launches": launches,
        "iterations": its[0],
        "methods": per_method,
        "learned": learned,
        "kernels_ms_per_step": {k: round(v[1] / prof_steps, 4) for k, v in sorted(kern.items(), key=lambda kv: -kv[1][1])},
        "roofline": {"kernel": "pk_block16_jacobi", "bound": "hbm", "achieved": round(jac_gbs, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(jac_gbs / peak, 4), "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "traffic": None, "algorithmic": "12 B per level-0 cell-update (x, b read, x' written); the "
                                                     "level-0 vectors (38 MB) stay in L2 between sweeps",
                     "launches": 20, "avg_launch_us": round(jac_us, 2)},
        "clocks": clk,
    }
    P.close()
    if not emit:
        net.close()
        ctx.close()
        return line
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_poisson(active, bh, size)
    if rank == 0:
        print(json.dumps(line), flush=True)
    _finish(dist)


def cpu_baseline_poisson(active, bh, size):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    n = size // 16
    t = time.perf_counter()
    _, hist = oracle.poisson_solve(np.asarray(active, np.int64), n, n, n, 16, bh.reshape(-1).astype(np.float64), mode=1,
                                   tol=1e-6, max_iter=400)
    el = time.perf_counter() - t
    return {"value": el * 1e3, "unit": "ms", "cores": 1, "kind": "port",
            "sample": f"the whole solve ({len(hist)} MG-PCG iterations, FP64, one thread)"}


def run_batched(args, world, rank, local):
    """64 independent sparse Poisson problems to 1e-8 in one batch."""
    import torch

    msbg = load_package()
    from msbg_rs_b200 import workloads

    dist = _dist_init(world, local)
    dev = torch.device("cuda", local)
    probs = workloads.batched_problems(n=args.problems, seed=3)
    ctx = msbg.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    t_build = time.perf_counter()
    B = msbg.Batch(ctx, [(d, bs, a) for d, bs, a, _ in probs], tune=True)
    t_build = time.perf_counter() - t_build
    for p, (_, _, _, b) in enumerate(probs):
        B.set_rhs(p, b)
    cells = int(sum(len(a) * bs ** 3 for _, bs, a, _ in probs))

    def one():
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        its, rel, cyc = B.solve(tol=1e-8, iters_per_cycle=8, max_cycles=60)
        e1.record(stream)
        ctx.synchronize()
        return e0.elapsed_time(e1), its, rel, cyc

    for _ in range(args.warmup):
        one()
    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = ctx.kernel_launches()
    res = [one() for _ in range(args.steps)]
    clk = clocks.stop()
    launches = ctx.kernel_launches() - launches0
    ms = _max_over_ranks(dist, statistics.mean(r[0] for r in res), dev)
    _, its, rel, cyc = res[-1]
    # end to end through the public API: every right-hand side from the host,
    # the solve, every FP64 solution back to the host
    sols = [np.empty(len(a) * bs ** 3, np.float64) for _, bs, a, _ in probs]
    e2e_steps = max(1, min(args.steps, 3))
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(e2e_steps):
        for p, (_, _, _, b) in enumerate(probs):
            B.set_rhs(p, b)
        B.solve(tol=1e-8, iters_per_cycle=8, max_cycles=60)
        for p in range(len(probs)):
            sols[p][:] = B.solution(p)
    e2e_ms = _max_over_ranks(dist, (time.perf_counter() - t) * 1e3 / e2e_steps, dev)
    # error of the FP64 solutions against the FP64 oracle on the smallest problems
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    order = sorted(range(len(probs)), key=lambda p: len(probs[p][2]) * probs[p][1] ** 3)[: args.check]
    errs = {}
    t_cpu = 0.0
    for p in order:
        dims, bs, act, b = probs[p]
        n = dims[0] // bs
        t0 = time.perf_counter()
        xo, _ = oracle.poisson_solve(act.astype(np.int64), n, n, n, bs, b.reshape(-1).astype(np.float64), mode=1,
                                     tol=1e-10, max_iter=400)
        t_cpu += time.perf_counter() - t0
        x = B.solution(p)
        errs[str(p)] = float(np.linalg.norm(x - xo) / np.linalg.norm(xo))
    tun = {str(g): B.tuning(g)[0].tolist() for g in range(B.n_groups)}
    line = {
        "metric": "batched Poisson solve: all problems to 1e-8 relative residual (MG-PCG, FP64 refinement)",
        "value": ms, "unit": "ms", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 solution, dots, refinement)",
        "data": "synthetic (seeded shells and uniform right-hand sides; no dataset exists for this path)",
        "config": {"workload": f"{len(probs)} problems, edges from {{32,64,128,256}}, 8^3 or 16^3 blocks, "
                               "active fraction 5-60 %", "unknowns": cells, "groups": B.n_groups,
                   "iters_per_cycle": 8, "parallelism": f"replicas x{world}", "l2": "solves run back to back"},
        "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": int(4 * cells),
                "d2h_bytes_per_step": int(8 * cells + 16 * 8 * len(probs)),
                "api": "msbg_batch_set_rhs per problem (host f32), msbg_batch_solve, msbg_batch_get_solution per "
                       "problem (host FP64); host wall clock"},
        "gpu_launches": launches,
        "graph_launches_per_solve": 1,
        "cycles_per_solve": cyc,
        "iterations": {"min": int(its.min()), "max": int(its.max()), "mean": float(its.mean())},
        "max_rel_residual": float(rel.max()),
        "error_vs_fp64_oracle": errs,
        "autotuned_shapes": tun,
        "build_s": t_build,
        "clocks": clk,
    }
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = {"value": t_cpu * 1e3, "unit": "ms", "cores": 1, "kind": "port",
                                "sample": f"FP64 oracle MG-PCG solves of the {len(order)} smallest problems"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    B.close()
    _finish(dist)


def run_phasefield(args, world, rank, local):
    """The full phase-field FLIP step on the noisy-sphere band."""
    import torch

    msbg = load_package()
    from msbg_rs_b200 import workloads
    from msbg_rs_b200._lib import call, ptr

    dist = _dist_init(world, local)
    dev = torch.device("cuda", local)
    size = args.size or 512
    t_gen = time.perf_counter()
    pf = workloads.phase_field(size)
    t_gen = time.perf_counter() - t_gen
    n = pf.n
    fine = pf.fine_blocks
    nf = len(fine)
    ctx = msbg.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    pos = torch.from_numpy(pf.pos).to(dev)
    vel = torch.from_numpy(pf.vel).to(dev)
    mass = torch.from_numpy(pf.mass).to(dev)
    keys = torch.empty(n, dtype=torch.int64, device=dev)
    perm = torch.empty(n, dtype=torch.int32, device=dev)
    u, u_new = torch.empty_like(vel), torch.empty_like(vel)
    mac = msbg.MacGrid(ctx, size, size, size, 16)
    sampler = msbg.MacSampler(mac, msbg.CLAMP)
    phase = msbg.SparseGrid(ctx, size, size, size, 0.0, 1.0, 16, dtype="bf16", name="phase")
    phase_bits = workloads.bf16_bits(pf.phase)
    phase.write_blocks(fine, phase_bits)
    sweeper = msbg.Sweeper(phase)
    divg = msbg.SparseGrid(ctx, size, size, size, 0.0, 0.0, 16, name="divergence")
    divg.ensure_blocks(fine)
    P = msbg.Poisson(ctx, size, size, size, 16, fine)
    P.autotune()  # outside the timed region
    net = msbg.UNet(ctx, size, size, size, fine, seed=1)
    P.set_preconditioner(net)
    t_train = time.perf_counter()
    hist = P.train_preconditioner(n_rhs=args.train_rhs, mg_iters=args.train_iters, steps_per_rhs=args.train_iters,
                                  pool=32, lr=1e-3, target=1, seed=7)
    ctx.synchronize()
    t_train = time.perf_counter() - t_train
    b = torch.empty(P.n, device=dev)
    x = torch.zeros(P.n, dtype=torch.float64, device=dev)
    fine_h = np.ascontiguousarray(fine, np.uint64)
    params = msbg.PdeParams(0.01, SWEEPS, True)

    def step(method, events=None):
        def mark(name):
            if events is not None:
                e = torch.cuda.Event(enable_timing=True)
                e.record(stream)
                events.append((name, e))

        mark("start")
        call("msbg_morton_sort_device", ctx.handle, ptr(pos), n, ptr(keys), ptr(perm))
        msbg.particles_to_grid_permuted_device(mac, pos, vel, mass, keys, perm, n, R_P)
        mark("p2g")
        sweeper.sweep(fine_h, msbg.Stencil.BiLaplacian, params)
        mark("phase")
        mac.divergence(divg, fine_h)
        call("msbg_grid_read_blocks_device", divg.handle, ptr(fine_h), nf, ptr(b))
        b.neg_()  # A p = -div u for A = 6 x - sum of neighbours
        x.zero_()
        it, rel, _ = P.solve_device(x, b, method=method, tol=1e-6, max_iter=400)
        mark("pressure")
        sampler.sample_device(pos, n, u)
        msbg.g2p_blend_device(ctx, vel, u, u, n, ALPHA, u_new)
        mark("g2p")
        return it, rel

    # learned PCG: the network in the first preconditioner application, then
    # CG restarted with V-cycles (LEARNED_LEAD); the V-net-V preconditioner
    # throughout (HYBRID) beside it
    methods = {"learned_pcg": (msbg.LEARNED_LEAD, 1), "learned_hybrid_pcg": (msbg.HYBRID, 0),
               "mg_pcg": (msbg.PCG, 0), "plain_mg": (msbg.MG, 0)}
    out = {}
    for name, (m, lead) in methods.items():
        P.set_network_lead(lead)
        for _ in range(args.warmup):
            step(m)
        ctx.synchronize()
        clocks = ClockSampler(local)
        clocks.start()
        launches0 = ctx.kernel_launches()
        evs = []
        for _ in range(args.steps):
            ev = []
            it, rel = step(m, ev)
            evs.append(ev)
        ctx.synchronize()
        clk = clocks.stop()
        ph = {}
        for ev in evs:
            for (a_, ea), (b_, eb) in zip(ev[:-1], ev[1:]):
                ph[b_] = ph.get(b_, 0.0) + ea.elapsed_time(eb) / args.steps
        total = sum(ev[0][1].elapsed_time(ev[-1][1]) for ev in evs) / args.steps
        out[name] = {"ms_per_step": total, "phases_ms": {k: round(v, 3) for k, v in ph.items()}, "pressure_iterations": it,
                     "pressure_rel_residual": rel, "launches": ctx.kernel_launches() - launches0, "clocks": clk,
                     **P.solve_stats()}
    # BF16 storage error: the same 10 sweeps on an f32 copy of the phase field
    ref = msbg.SparseGrid(ctx, size, size, size, 0.0, 1.0, 16, name="phase_f32")
    ref.write_blocks(fine, pf.phase)
    p16 = msbg.SparseGrid(ctx, size, size, size, 0.0, 1.0, 16, dtype="bf16", name="phase_bf16")
    p16.write_blocks(fine, phase_bits)
    msbg.Sweeper(ref).sweep(fine_h, msbg.Stencil.BiLaplacian, params)
    msbg.Sweeper(p16).sweep(fine_h, msbg.Stencil.BiLaplacian, params)
    r32 = ref.read_blocks(fine).astype(np.float64)
    r16 = (p16.read_blocks(fine).astype(np.uint32) << 16).view(np.float32).astype(np.float64)
    bf16_err = {"max_abs": float(np.max(np.abs(r16 - r32))),
                "rel_l2": float(np.linalg.norm(r16 - r32) / max(np.linalg.norm(r32), 1e-30)),
                "reference": "the same 10 sweeps with f32 storage"}
    head = out["learned_pcg"]
    ms = _max_over_ranks(dist, head["ms_per_step"], dev)
    line = {
        "metric": "full phase-field FLIP step (sort, P2G, BF16 25-tap phase field x10, pressure to 1e-6, G2P)",
        "value": ms, "unit": "ms", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (bf16 phase field, FP64 dots)",
        "data": "synthetic (seeded noisy sphere, particles and velocities; no dataset exists for this path)",
        "config": {"workload": f"phase-field FLIP {size}^3, 16^3 blocks, 4 levels, 8 particles per cell in a band of "
                               "width 24 around a noisy sphere", "particles": n, "level_blocks": np.bincount(pf.levels, minlength=4).tolist(),
                   "pressure_unknowns": int(P.n), "parallelism": f"replicas x{world}", "l2": "inputs larger than L2"},
        "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                "note": "particles stay resident between steps"},
        "gpu_launches": head["launches"],
        "solvers": out,
        "bf16_storage_error": bf16_err,
        "learned": {"pairs": args.train_rhs * args.train_iters, "train_s": t_train,
                    "loss_first": float(np.mean(hist[:10])) if len(hist) else None,
                    "loss_last": float(np.mean(hist[-10:])) if len(hist) else None},
        "generation_s": t_gen,
        "clocks": head["clocks"],
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    _finish(dist)


def run_reference_smoother(args, world, rank, local):
    """Reference arm of the smoother workload: the oracle sweep on the host."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    load_package()
    from msbg_rs_b200 import workloads

    sp = workloads.shell_problem(args.size, 16, seed=1)
    stencil = {"laplacian": 0, "meancurv": 1, "bilaplacian": 2}[args.stencil]
    for _ in range(args.warmup):
        run_cpu_smoother(oracle, sp, stencil, budget_s=2.0)
    vals = [run_cpu_smoother(oracle, sp, stencil, budget_s=args.cpu_budget) for _ in range(args.steps)]
    v = statistics.median(r["value"] for r in vals)
    cells = len(sp.active) * 4096 * SWEEPS
    print(json.dumps({
        "impl": "reference", "metric": "smoother cell-updates per second (10 in-place 8-colour sweeps)", "value": v,
        "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": cells / v * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": f"shell {args.size}^3, 16^3 blocks, radius 0.35*size, thickness 12",
                   "blocks": len(sp.active), "stencil": SMOOTHER_STENCILS[stencil], "parallelism": "host CPU"},
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": vals[0]["threads"], "kind": "port",
                         "sample": vals[0]["sample"]},
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_reference_poisson(args, world, rank, local):
    """Reference arm of the Poisson workload: the FP64 oracle MG-PCG solve."""
    if rank != 0:
        return
    load_package()
    active, bh = poisson_problem(args.size)
    steps = max(1, min(args.steps, 3))
    vals = [cpu_baseline_poisson(active, bh, args.size) for _ in range(steps)]
    v = statistics.median(r["value"] for r in vals)
    print(json.dumps({
        "impl": "reference", "metric": "time to 1e-6 relative residual (Poisson, 7-point, MG-preconditioned CG)",
        "value": v, "unit": "ms", "n_gpus": world, "steps": steps, "warmup": 0, "ms_per_step": v,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": f"Poisson on the level-0 blocks of the {args.size}^3 3-level layout, 16^3 blocks",
                   "blocks": int(len(active)), "parallelism": "host CPU"},
        "cpu_baseline": dict(vals[0], value=v),
        "e2e": {"value": v, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_reference_batched(args, world, rank, local):
    """Reference arm of the batched workload: the FP64 oracle solving every
    problem in turn (bounded: the smallest --check problems), one thread."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    load_package()
    from msbg_rs_b200 import workloads

    probs = workloads.batched_problems(n=args.problems, seed=3)
    order = sorted(range(len(probs)), key=lambda p: len(probs[p][2]) * probs[p][1] ** 3)[: args.check]
    t0 = time.perf_counter()
    for p in order:
        dims, bs, act, b = probs[p]
        n = dims[0] // bs
        oracle.poisson_solve(act.astype(np.int64), n, n, n, bs, b.reshape(-1).astype(np.float64), mode=1, tol=1e-8,
                             max_iter=400)
    v = (time.perf_counter() - t0) * 1e3
    print(json.dumps({
        "impl": "reference", "metric": "batched Poisson solve: all problems to 1e-8 relative residual (MG-PCG, FP64 refinement)",
        "value": v, "unit": "ms", "n_gpus": world, "steps": 1, "warmup": 0, "ms_per_step": v, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": f"{len(order)} smallest of {len(probs)} batched problems", "parallelism": "host CPU"},
        "cpu_baseline": {"value": v, "unit": "ms", "cores": 1, "kind": "port",
                         "sample": f"the {len(order)} smallest of {len(probs)} problems, solved one after another"},
        "e2e": {"value": v, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["flip", "smoother", "poisson", "batched", "phasefield"], default="flip")
    ap.add_argument("--stencil", choices=["laplacian", "meancurv", "bilaplacian"], default="laplacian")
    ap.add_argument("--size", type=int, default=None)
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-submetrics", action="store_true",
                    help="flip: skip the smoother (2048^3 shell) and pressure-solve (256^3) parts of the metric")
    ap.add_argument("--train-rhs", type=int, default=100, help="poisson: right-hand sides generating training pairs")
    ap.add_argument("--problems", type=int, default=64, help="batched: number of problems")
    ap.add_argument("--check", type=int, default=8, help="batched: problems checked against the FP64 oracle")
    ap.add_argument("--train-iters", type=int, default=40, help="poisson: V-cycles (pairs) and Adam steps per rhs")
    args = ap.parse_args()
    if args.size is None:
        args.size = {"flip": 256, "smoother": 2048, "poisson": 256, "batched": 0, "phasefield": 512}[args.workload]
    world, rank, local = dist_setup()
    if args.impl == "reference":
        {"flip": run_reference, "smoother": run_reference_smoother, "poisson": run_reference_poisson,
         "batched": run_reference_batched, "phasefield": run_reference}[args.workload](args, world, rank, local)
    else:
        {"flip": run_ours, "smoother": run_smoother, "poisson": run_poisson, "batched": run_batched,
         "phasefield": run_phasefield}[args.workload](args, world, rank, local)


if __name__ == "__main__":
    main()
