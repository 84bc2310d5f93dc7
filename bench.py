#!/usr/bin/env python
"""Benchmark of the B200 particle step on the 1D3V capacitive RF discharge
with null-collision MCC (512 cells, 512 electrons + 512 He+ per cell).

One JSON line on rank 0.  A step is one PIC step of that discharge: push
(gather, kick, drift, walls), CIC deposit, Poisson solve and MCC.

  value  device-resident throughput (particle-steps/s), L2 flushed between
         timed steps, max over ranks, summed over ranks (weak scaling: each
         rank runs its own discharge, no collective on the data path)
  e2e    the same metric through the C ABI with host buffers: every step loads
         the particles from pinned host memory, resumes, steps and reads the
         particles back
  roofline  the fused particle-pass kernel against measured HBM bandwidth
  cpu_baseline  the reference's own CPU step (compiled from its sources) on
         this host's cores, on a bounded sample of the same workload

`--impl reference` times the reference's CPU implementation alone (rank 0).
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
sys.path.insert(0, os.path.join(ROOT, "aurora-pic_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "particle-steps/s (push+deposit+MCC)"
WORKLOAD = "ccp_helium_1d3v: Dirichlet 0.067 m, 512 cells, 450 V 13.56 MHz, dt=1/(400 f), " \
           "2x262144 particles (e-, He+ 4 amu), He 9.64e20 m^-3 300 K, 5-channel MCC"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ppc", type=int, default=512)
    ap.add_argument("--cells", type=int, default=512)
    ap.add_argument("--e2e-steps", type=int, default=30)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(", ") for r in open(self.path).read().strip().splitlines()]
        except Exception:
            rows = []
        rows = [r for r in rows if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, nm in enumerate(names):
                if r[5 + k].strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": sorted(reasons),
                "samples": len(rows)}


def cpu_reference_sample(wl, seconds, threads):
    """The reference's own Simulation::step on this host (oracle/_ref), or the C
    restatement when the reference library is absent: a bounded sample."""
    import pyoracle as po
    tabs = po.TableSet()
    work = tempfile.mkdtemp(prefix="apic_ref_")
    n_per = len(wl.species[0].x)
    if po.reference_available():
        cfg = po.config_from_workload(wl, tabs, seed=12345, threads=threads, own_loading=True)
        sim = po.Ref1D(cfg, work)
        sim.initialize()
        kind, cores = "reference", threads
    else:
        cfg = po.config_from_workload(wl, tabs, seed=12345)
        sim = po.Sim1D(cfg, 0)
        for i, s in enumerate(wl.species):
            sim.load(i, s.x, s.v, s.v, s.vy, s.vz)
        sim.initialize()
        kind, cores = "port", 1
    sim.step(1)  # warm
    steps = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        sim.step(1)
        steps += 1
    dt = time.perf_counter() - t0
    psteps = steps * n_per * len(wl.species)
    return {"value": psteps / dt, "unit": "particle-steps/s", "cores": cores, "kind": kind,
            "sample": f"{steps} full steps of the same discharge ({n_per * len(wl.species)} particles) "
                      f"in {dt:.1f} s"}


def run_reference(args):
    from apic import workloads as W
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wl = W.ccp_helium(particles_per_cell=args.ppc, cells=args.cells, seed=7)
    threads = os.cpu_count() or 1
    import pyoracle as po
    tabs = po.TableSet()
    work = tempfile.mkdtemp(prefix="apic_ref_")
    n = sum(len(s.x) for s in wl.species)
    if po.reference_available():
        cfg = po.config_from_workload(wl, tabs, seed=12345, threads=threads, own_loading=True)
        sim = po.Ref1D(cfg, work)
        sim.initialize()
        kind = "reference"
    else:
        cfg = po.config_from_workload(wl, tabs, seed=12345)
        sim = po.Sim1D(cfg, 0)
        for i, s in enumerate(wl.species):
            sim.load(i, s.x, s.v, s.v, s.vy, s.vz)
        sim.initialize()
        kind, threads = "port", 1
    # each bench step is a bounded sample of CPU steps so the run ends in minutes
    # the reference's thermal-neutral frequency bound scans every table row per
    # candidate (src/Collision.cpp:627-685): about 2-3 s per step here, so one
    # CPU step per bench step and at most 10 of them
    per_step = 1
    sim.step(per_step * max(1, min(args.warmup, 2)))
    t0 = time.perf_counter()
    k = max(1, min(args.steps, 10))
    sim.step(per_step * k)
    dt = time.perf_counter() - t0
    value = n * per_step * k / dt
    line = {"metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": args.gpus, "steps": k,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / (per_step * k), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": WORKLOAD, "particles": n, "parallelism": "cpu threads"},
            "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": threads, "kind": kind,
                             "sample": f"{per_step * k} steps of the full discharge"},
            "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import numpy as np
    import torch
    import apic
    from apic import workloads as W

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    wl = W.ccp_helium(particles_per_cell=args.ppc, cells=args.cells, seed=7 + rank)
    cfg, tabs = W.to_device_config(wl, precision=apic.FP64, seed=1000 + rank)
    sim = apic.Simulation1D(cfg, tabs)
    for i, s in enumerate(wl.species):
        sim.load(i, s.x, s.v, None, s.vy, s.vz)
    sim.initialize()
    sim.step(args.warmup)
    sim.synchronize()

    ext = torch.cuda.ExternalStream(sim.cuda_stream())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > 126 MB L2
    flush_sink = torch.empty((), dtype=torch.float32, device="cuda")
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    n_before = sum(sim.count(s) for s in range(len(wl.species)))
    sim.set_kernel_timing(True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        with torch.cuda.stream(ext):
            for i in range(args.steps):
                # write a buffer larger than L2, then read it back so the dirty
                # lines are written out before the timed step starts
                flush.zero_()
                flush_sink.copy_(flush.sum())
                starts[i].record(ext)
                sim.step(1)
                ends[i].record(ext)
        sim.synchronize()
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends))
    pass_ms, post_ms, passes = sim.kernel_times()
    sim.set_kernel_timing(False)
    n_after = sum(sim.count(s) for s in range(len(wl.species)))
    psteps = args.steps * 0.5 * (n_before + n_after)
    t = torch.tensor([ms, psteps], dtype=torch.float64, device="cuda")
    if dist:
        mx = t.clone()
        dist.all_reduce(mx[0:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(mx[1:2], op=dist.ReduceOp.SUM)
        ms_max, total_psteps = float(mx[0]), float(mx[1])
    else:
        ms_max, total_psteps = ms, psteps
    value = total_psteps / (ms_max * 1e-3)

    # ---- end to end through the C ABI with pinned host buffers ----
    ns = len(wl.species)
    cap = [wl.species[s].capacity for s in range(ns)]
    host = [{k: torch.empty(cap[s], dtype=torch.float64, pin_memory=True).numpy() for k in ("x", "v", "vh", "vy", "vz")}
            for s in range(ns)]
    counts = []
    for s in range(ns):
        p = sim.particles(s)
        n = len(p["x"])
        counts.append(n)
        for k in ("x", "v", "vh", "vy", "vz"):
            host[s][k][:n] = p[k]
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    t_sim, k_sim = sim.time, sim.step_count
    h2d = d2h = 0
    e2e_ms = 0.0
    L = apic.lib()
    got = apic.C.c_size_t()
    for it in range(args.e2e_steps):
        e_start.record(ext)
        for s in range(ns):
            n = counts[s]
            h = host[s]
            apic._check(L.apic_sim1d_load_particles(sim.h, s, n, *[apic.dptr(h[k]) for k in ("x", "v", "vh", "vy", "vz")],
                                                    None), sim.h)
            if it == 0:
                h2d += 5 * 8 * n
        sim.resume(t_sim, k_sim)
        sim.step(1)
        for s in range(ns):
            h = host[s]
            apic._check(L.apic_sim1d_read_particles(sim.h, s, cap[s], *[apic.dptr(h[k]) for k in ("x", "v", "vh", "vy", "vz")],
                                                    apic.C.byref(got)), sim.h)
            counts[s] = got.value
            if it == 0:
                d2h += 5 * 8 * got.value
        e_end.record(ext)
        e_end.synchronize()
        e2e_ms += e_start.elapsed_time(e_end)
        t_sim, k_sim = sim.time, sim.step_count
    e2e_psteps = args.e2e_steps * 0.5 * (n_before + n_after)
    te = torch.tensor([e2e_ms, e2e_psteps], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(te[0:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(te[1:2], op=dist.ReduceOp.SUM)
    e2e_value = float(te[1]) / (float(te[0]) * 1e-3)

    # ---- roofline of the fused particle pass ----
    hbm, peak_kind = peaks()
    bytes_per_pstep = 64  # FP64 1D3V: read + write x, v_half, v_y, v_z
    per_pass_ms = pass_ms / max(passes, 1)
    achieved = bytes_per_pstep * 0.5 * (n_before + n_after) / (per_pass_ms * 1e-3) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "pass1d_fp64_ccp_traffic.json")
    if os.path.exists(prof):
        try:
            traffic = json.load(open(prof)).get("bytes_per_launch_full_size")
        except Exception:
            traffic = None

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                cpu = cpu_reference_sample(wl, args.cpu_seconds, os.cpu_count() or 1)
            except Exception as e:  # reported, never fatal
                cpu = {"value": None, "error": str(e)}
        line = {
            "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "particles": int(0.5 * (n_before + n_after)),
                       "form": "FP64 particles (bit-faithful arithmetic)", "l2": "flushed between timed steps",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_value, "unit": "particle-steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "k_pass1d<3,true>", "bytes_per_particle_step": bytes_per_pstep,
                         "pass_ms": per_pass_ms, "post_ms": post_ms / max(passes, 1)},
            "gpu_launches": 2 * args.steps,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    sim.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
