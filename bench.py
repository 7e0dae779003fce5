#!/usr/bin/env python
"""Benchmark: one FLIP transfer step of the msbg-rs sparse-grid hot path on B200.

Workload (the FLIP transfer configuration): 256^3 domain, 16^3 blocks, three
resolution levels chosen per block by the distance of its centre to the
sphere |x - c| = 89.6 (< 16 cells: level 0, < 48: level 1, else level 2), 8
particles per level-0 cell uniformly jittered inside the cell (25,427,968
particles), velocities N(0, 1), mass 1, all from a fixed seed, in shuffled
order.  One step:
  1. Morton sort of the particles by morton3 of their cell (21 bits per axis)
     and the payload gather into sorted order,
  2. P2G: splat of mass and momentum to the MAC faces (r_p = 2) + normalise,
  3. 2^3 downsample of the splatted x-face mass to the coarse level and 10
     sweeps of the 19-tap mean-curvature smoother (dt 0.025) over the level-0
     blocks, halos of coarser neighbours sampled from the coarse level,
  4. G2P: trilinear MAC sample at every particle + FLIP/PIC blend (alpha 0.95).
metric = particles through the whole step per second.  Inputs are resident in
HBM when the timed region starts and are far larger than L2 (713 MB of
particle data), so no L2 flush is needed.

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
                                          "--format=csv,noheader,nounits", "-lms", "200"],
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

    def step(events=None):
        def mark(name):
            if events is not None:
                e = torch.cuda.Event(enable_timing=True)
                e.record(stream)
                events.append((name, e))

        mark("start")
        call("msbg_morton_sort_device", ctx.handle, ptr(pos), n, ptr(keys), ptr(perm))
        call("msbg_permute_device", ctx.handle, ptr(perm), n, 3, ptr(pos), ptr(spos))
        call("msbg_permute_device", ctx.handle, ptr(perm), n, 3, ptr(vel), ptr(svel))
        call("msbg_permute_device", ctx.handle, ptr(perm), n, 1, ptr(mass), ptr(smass))
        mark("sort")
        msbg.particles_to_grid_sorted_device(mac, spos, svel, smass, keys, n, R_P)
        mark("p2g")
        act = mac.active_blocks()
        fine = act[levels[act.astype(np.int64)] == 0]
        state["active"], state["fine"] = act, fine
        msbg.downsample_channel_avg(coarse, mac.mass(0))
        sweeper.sweep_multires(coarse, levels, fine, msbg.Stencil.MeanCurvature, msbg.PdeParams(DT, SWEEPS, False))
        mark("smooth")
        sampler.sample_device(spos, n, u)
        msbg.g2p_blend_device(ctx, svel, u, u, n, ALPHA, u_new)
        mark("g2p")

    # warm-up
    for _ in range(args.warmup):
        step()
    ctx.synchronize()
    call("msbg_ctx_set_timing", ctx.handle, 1)
    timing_report(msbg, ctx, reset=True)
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
        step(ev)
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
    kernels = timing_report(msbg, ctx, reset=True)
    call("msbg_ctx_set_timing", ctx.handle, 0)
    if dist:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    # ---- end to end through the C ABI with host buffers ----------------------
    pin_pos = torch.from_numpy(pos_h).pin_memory()
    pin_vel = torch.from_numpy(vel_h).pin_memory()
    pin_mass = torch.from_numpy(mass_h).pin_memory()
    pin_out = torch.empty((n, 3), dtype=torch.float32).pin_memory()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e2e_steps = max(1, min(args.steps, 5))
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(e2e_steps):
            pos.copy_(pin_pos, non_blocking=True)
            vel.copy_(pin_vel, non_blocking=True)
            mass.copy_(pin_mass, non_blocking=True)
            step()
            pin_out.copy_(u_new, non_blocking=True)
        e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    h2d = pin_pos.numel() * 4 + pin_vel.numel() * 4 + pin_mass.numel() * 4
    d2h = pin_out.numel() * 4
    if dist:
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())

    # ---- roofline of the dominant kernel ------------------------------------
    peak, peak_kind = load_peaks()
    dom = max(kernels.items(), key=lambda kv: kv[1][1]) if kernels else ("none", (1, 1.0))
    n_fine = len(state["fine"])
    n_active = len(state["active"])
    algo = algorithmic_bytes(dom[0], n=n, n_fine=n_fine, n_active=n_active, steps=args.steps)
    roof = None
    if algo is not None:
        achieved = algo / (dom[1][1] * 1e-3) / 1e9
        roof = {"kernel": dom[0], "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "traffic": None, "launches": dom[1][0], "avg_launch_us": round(dom[1][1] / dom[1][0] * 1e3, 2)}
    sweep_k = kernels.get("sweep_phase_kernel")
    smoother = None
    if sweep_k:
        cells = n_fine * 4096 * SWEEPS * args.steps
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
        "e2e": {"value": world * n / (e2e_ms * 1e-3), "unit": UNIT, "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "phases_ms": {k: round(v, 4) for k, v in phase_ms.items()},
        "kernels_ms_per_step": {k: round(v[1] / args.steps, 4) for k, v in sorted(kernels.items(), key=lambda kv: -kv[1][1])},
        "submetrics": {"p2g_particles_per_s": n / (phase_ms.get("p2g", float("nan")) * 1e-3),
                       "smoother": smoother},
        "roofline": roof,
        "clocks": clk,
    }
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(ft, pos_h, vel_h, mass_h, budget_s=args.cpu_budget)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def algorithmic_bytes(kernel, n, n_fine, n_active, steps):
    """Algorithmic HBM bytes moved by all launches of `kernel` in the timed
    region (the per-unit figures: 8 B per f32 cell-update for the in-place
    smoother; 28 B read per particle for the P2G splat plus 24 B written per
    face-cell of the active blocks for the combine; 12 B read + 12 B written
    per particle for G2P; 24 B per element per radix pass)."""
    if kernel == "sweep_phase_kernel":
        return 8.0 * n_fine * 4096 * SWEEPS * steps
    if kernel == "p2g_cells_kernel":
        return 28.0 * n * steps
    if kernel == "p2g_combine_kernel":
        return 24.0 * n_active * 4096 * steps
    if kernel == "g2p_kernel":
        return 24.0 * n * steps
    if kernel in ("rs_scatter_kernel",):
        return 24.0 * n * steps * 3  # one sort of 3 passes
    if kernel == "permute_kernel":
        return 2 * 28.0 * n * steps
    return None


def cpu_baseline(ft, pos_h, vel_h, mass_h, budget_s=20.0):
    """The reference algorithm on the host (oracle/, all host threads) on a
    sample: the particles of the first k level-0 blocks (in block order)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    res = run_cpu_sample(oracle, ft, budget_s)
    return {"value": res["value"], "unit": UNIT, "cores": res["threads"], "kind": "port", "sample": res["sample"]}


def run_cpu_sample(oracle, ft, budget_s):
    """Times Morton sort + P2G + downsample + 10 multires sweeps + G2P on the
    host for the particles of a contiguous run of level-0 blocks."""
    threads = oracle.num_threads()
    size, bsx = ft.size, ft.bsx
    per_block = 8 * bsx ** 3
    k = 8
    results = None
    while True:
        sel = slice(0, k * per_block)
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
        if el > budget_s / 4 or k * 2 > len(ft.fine_blocks):
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
    for _ in range(args.warmup):
        run_cpu_sample(oracle, ft, budget_s=4.0)
    vals = [run_cpu_sample(oracle, ft, budget_s=args.cpu_budget) for _ in range(args.steps)]
    v = statistics.median(r["value"] for r in vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ft.n / v * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": f"FLIP transfer {args.size}^3, 16^3 blocks, 3 levels, 8 particles per level-0 cell",
                   "particles": ft.n, "parallelism": "host CPU"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": vals[0]["threads"], "kind": "port",
                         "sample": vals[0]["sample"]},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank, local)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
