#!/usr/bin/env python
"""Benchmark of the B200 particle step.

Default workload: the 1D3V capacitive RF discharge with null-collision MCC
(512 cells, 512 electrons + 512 He+ per cell).  `--workload plasma2d` /
`plasma3d` run the 512^2 x 64 ppc 2D3V and 256^3 x 8 ppc 3D3V periodic decks
(FP32 particles by default, `--precision fp64` for the plain form).

One JSON line on rank 0.  A step is one PIC step: push (gather, kick, drift,
walls or wrap), CIC deposit, Poisson solve, and for the discharge MCC.

  value  device-resident throughput (particle-steps/s), max over ranks for
         time, summed over ranks for work (weak scaling: each rank runs its own
         deck, no collective on the data path)
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
WORKLOAD_CCP = "ccp_helium_1d3v: Dirichlet 0.067 m, 512 cells, 450 V 13.56 MHz, dt=1/(400 f), " \
               "2x262144 particles (e-, He+ 4 amu), He 9.64e20 m^-3 300 K, 5-channel MCC"
WORKLOAD_2D = "plasma_2d3v_bz: periodic 512x512 cells (cell = lambda_D at 1e16 m^-3, 2 eV), 64 ppc e- + 64 ppc " \
              "ions (33,554,432 particles), Bz 0.01 T, Te 2 eV, Ti 0.03 eV, m_i/m_e 1836, dt 0.1/omega_pe"
WORKLOAD_3D = "plasma_3d3v_bx: periodic 256^3 cells, 8 ppc e- + 8 ppc ions (268,435,456 particles), " \
              "Bx 0.005 T, Te 1 eV, Ti 0.025 eV, m_i/m_e 1836, dt 0.1/omega_pe"
WORKLOAD_SWARM = "swarm_serving: electron swarms in a 4-process gas (elastic, excitations 11.5 / 13.0 eV, " \
                 "ionization 15.8 eV) at 2.45e25 m^-3, 300 K; E/N log-uniform 10-1000 Td, electrons log-normal " \
                 "(median 100k, sigma 1, clipped 10k-4M), Poisson arrivals at 80% of measured capacity, each run " \
                 "until drift velocity and mean energy converge to 1% or 20k steps"
# algorithmic bytes per particle-step: read + write of the persistent state once
BYTES_PER_PSTEP = {("plasma2d", "fp64"): 80, ("plasma3d", "fp64"): 96,
                   ("plasma2d", "fp32"): 48, ("plasma3d", "fp32"): 56}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=None)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ccp1d", choices=["ccp1d", "plasma2d", "plasma3d", "swarm"])
    ap.add_argument("--requests", type=int, default=96, help="swarm: requests in the Poisson serving phase")
    ap.add_argument("--mixed-requests", type=int, default=64,
                    help="swarm: swarm requests of the mixed phase (two-stream decks arrive at half that rate)")
    ap.add_argument("--batch", type=int, default=8, help="ccp1d: discharges stepped together for the batched line")
    ap.add_argument("--precision", default=None, choices=["fp64", "fp32"])
    ap.add_argument("--ppc", type=int, default=None)
    ap.add_argument("--cells", type=int, default=None, help="cells per axis")
    ap.add_argument("--sort-interval", type=int, default=0, help="plasma: 0 = chosen by the autotuner")
    ap.add_argument("--push-items", type=int, default=0, help="plasma FP32: particles per thread (0 = autotuned)")
    ap.add_argument("--steps-per-launch", type=int, default=0, help="swarm: graph length (0 = autotuned)")
    ap.add_argument("--no-other-configs", action="store_true",
                    help="ccp1d at N=1: skip the nested 2D3V / 3D3V / swarm-serving records")
    ap.add_argument("--no-autotune", action="store_true", help="skip the autotuner (fixed defaults)")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    a = ap.parse_args()
    big = a.workload in ("plasma2d", "plasma3d")
    if a.workload == "swarm":
        a.precision = a.precision or "fp32"
    if a.steps is None:
        a.steps = {"ccp1d": 200, "plasma2d": 100, "plasma3d": 20, "swarm": 48}[a.workload]
    if a.warmup is None:
        a.warmup = 5 if big else 20
    if a.e2e_steps is None:
        a.e2e_steps = 2 if big else 30
    if a.precision is None:
        a.precision = "fp32" if big else "fp64"
    return a


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
            # the sampler is running before the timed region starts, so even a
            # region shorter than the sampling period gets its first sample
            # (waited for at most 3 s)
            t0 = time.time()
            while time.time() - t0 < 3.0 and self.proc.poll() is None:
                self.f.flush()
                if os.path.getsize(self.path) > 0:
                    break
                time.sleep(0.02)
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


# ---------------------------------------------------------------- CPU side

def _ccp_cpu_sim(wl, threads):
    """The reference's Simulation (oracle/_ref) on this host, or the C
    restatement when the reference library is absent."""
    import pyoracle as po
    tabs = po.TableSet()
    work = tempfile.mkdtemp(prefix="apic_ref_")
    if po.reference_available():
        cfg = po.config_from_workload(wl, tabs, seed=12345, threads=threads, own_loading=True)
        sim = po.Ref1D(cfg, work)
        sim.initialize()
        return sim, "reference", threads, tabs
    cfg = po.config_from_workload(wl, tabs, seed=12345)
    sim = po.Sim1D(cfg, 0)
    for i, s in enumerate(wl.species):
        sim.load(i, s.x, s.v, s.v, s.vy, s.vz)
    sim.initialize()
    return sim, "port", 1, tabs


def _plasma_cpu_sim(plan, threads):
    """The reference's Simulation2D / Simulation3D on a scaled mesh with the
    same particles per cell (the full decks take minutes per CPU step)."""
    import pyoracle as po
    from apic import workloads as W
    cells = (128, 128) if plan.dims == 2 else (64, 64, 64)
    small = W.plasma_plan(plan.dims, cells=cells, ppc=plan.species[0][3] // int(_prod(plan.n)))
    sp = [(q, m, w, n, 0.0, vt) for (q, m, w, n, vt, seed) in small.species]
    if po.reference_available():
        sim = po.RefND(small.dims, small.n, small.length, small.dt, True, small.B, sp, seed=12345, threads=threads)
        kind = "reference"
    else:
        raise RuntimeError("the reference library was not built on this host")
    sim.initialize()
    return sim, kind, threads, small


def _prod(t):
    r = 1
    for x in t:
        r *= x
    return r


def _swarm_cpu_sample(seconds, threads):
    """The reference's run_swarm_benchmark on this host: one serial run per
    core (the reference runs fields one after another), each sized to about
    `seconds` of work, on the serving deck's gas and timestep."""
    import concurrent.futures as cf
    import pyoracle as po
    from apic import workloads as W
    if not po.reference_available():
        raise RuntimeError("the reference library was not built on this host")
    spec = W.swarm_c5()
    T = po.TableSet()
    cfg, gas = po.swarm_from_spec(spec, T)
    cfg.particles, cfg.steps, cfg.burn_in_steps = 2000, 100, 50
    t0 = time.perf_counter()
    po.ref_swarm_run(cfg, gas, [100.0], tempfile.mkdtemp())
    rate = cfg.particles * cfg.steps / (time.perf_counter() - t0)
    steps = 200
    cfg.steps, cfg.burn_in_steps = steps, 100
    cfg.particles = int(min(max(rate * seconds / steps, 1000), 200_000))

    def one(k):
        return po.ref_swarm_run(cfg, gas, [100.0 + 10.0 * k], tempfile.mkdtemp())

    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(threads) as ex:  # ctypes calls release the GIL
        list(ex.map(one, range(threads)))
    dt = time.perf_counter() - t0
    return threads * cfg.particles * steps / dt, dt, cfg.particles, steps


def cpu_reference_sample(args, wl, seconds, threads):
    """A bounded sample of the reference's CPU step on this host's cores."""
    if args.workload == "swarm":
        v, dt, n, steps = _swarm_cpu_sample(seconds, threads)
        return {"value": v, "unit": "particle-steps/s", "cores": threads, "kind": "reference",
                "sample": f"{threads} concurrent run_swarm_benchmark runs (one field each, {n} electrons x {steps} "
                          f"steps, 100-{100 + 10 * (threads - 1)} Td) in {dt:.1f} s"}
    if args.workload == "ccp1d":
        sim, kind, cores, _ = _ccp_cpu_sim(wl, threads)
        n = sum(len(s.x) for s in wl.species)
        what = f"full steps of the same discharge ({n} particles)"
    else:
        sim, kind, cores, small = _plasma_cpu_sim(wl, threads)
        n = small.particles
        what = f"steps of the same deck on a {'x'.join(map(str, small.n))} mesh ({n} particles, same ppc)"
    sim.step(1)  # warm
    steps = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        sim.step(1)
        steps += 1
    dt = time.perf_counter() - t0
    return {"value": steps * n / dt, "unit": "particle-steps/s", "cores": cores, "kind": kind,
            "sample": f"{steps} {what} in {dt:.1f} s"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from apic import workloads as W
    threads = os.cpu_count() or 1
    if args.workload == "swarm":
        value, dt, n, steps = _swarm_cpu_sample(min(20.0, 2.0 * max(1, min(args.steps, 10))), threads)
        line = {"metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": args.gpus, "steps": steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": {"workload": WORKLOAD_SWARM, "parallelism": "one serial run per host thread"},
                "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": threads, "kind": "reference",
                                 "sample": f"{threads} concurrent runs of {n} electrons x {steps} steps"},
                "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    if args.workload == "ccp1d":
        wl = W.ccp_helium(particles_per_cell=args.ppc or 512, cells=args.cells or 512, seed=7)
        sim, kind, threads, _ = _ccp_cpu_sim(wl, threads)
        n = sum(len(s.x) for s in wl.species)
        workload, sample = WORKLOAD_CCP, "full discharge"
        # the reference's thermal-neutral frequency bound scans every table row
        # per candidate (src/Collision.cpp:627-685): 2-3 s per step here, so
        # one CPU step per bench step and at most 10 of them
        kmax = 10
    else:
        plan = W.plasma_plan(2 if args.workload == "plasma2d" else 3)
        sim, kind, threads, small = _plasma_cpu_sim(plan, threads)
        n = small.particles
        workload = WORKLOAD_2D if plan.dims == 2 else WORKLOAD_3D
        sample = f"{'x'.join(map(str, small.n))} mesh, same ppc ({n} particles)"
        kmax = 10
    sim.step(max(1, min(args.warmup, 2)))
    k = max(1, min(args.steps, kmax))
    t0 = time.perf_counter()
    sim.step(k)
    dt = time.perf_counter() - t0
    value = n * k / dt
    line = {"metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": args.gpus, "steps": k,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / k, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": workload, "particles": n, "parallelism": "cpu threads"},
            "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": threads, "kind": kind,
                             "sample": f"{k} steps of the {sample}"},
            "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU side

def _profiled_traffic(name):
    """DRAM bytes (read + write) per launch of the dominant kernel, from the
    committed ncu summary of the same workload (None when absent)."""
    import re
    try:
        m = re.search(r"traffic_bytes_per_launch: (\d+)", open(os.path.join(ROOT, "profiles", name)).read())
        return int(m.group(1)) if m else None
    except OSError:
        return None


def _reduce(dist, t_ms, work, device="cuda"):
    """Whole-job figures of the replicas: the slowest rank's device time (the
    job ends when it does) and the work summed over ranks.  `device` is the
    process group's tensor device ("cuda" for NCCL, "cpu" for gloo)."""
    import torch
    t = torch.tensor([t_ms, work], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(t[0:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:2], op=dist.ReduceOp.SUM)
    return float(t[0]), float(t[1])


def bench_ccp1d(args, rank, dist):
    """Returns the workload-specific part of the JSON line."""
    import torch
    import apic
    from apic import workloads as W

    prec = apic.FP32 if args.precision == "fp32" else apic.FP64
    wl = W.ccp_helium(particles_per_cell=args.ppc or 512, cells=args.cells or 512, seed=7 + rank)
    cfg, tabs = W.to_device_config(wl, precision=prec, seed=1000 + rank)
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
    with Clocks(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
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
    mean_n = 0.5 * (n_before + n_after)
    ms_max, total = _reduce(dist, ms, args.steps * mean_n)
    value = total / (ms_max * 1e-3)

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
    e_ms, e_total = _reduce(dist, e2e_ms, args.e2e_steps * mean_n)

    hbm, peak_kind = peaks()
    # read + write of the particle state: FP64 x, v_half, v_y, v_z 8+8+8+8;
    # FP32 cell form cell, offset, v_half, v_y, v_z 4+4+4+4+4
    bytes_per_pstep = 64 if prec == apic.FP64 else 40
    per_pass_ms = pass_ms / max(passes, 1)
    achieved = bytes_per_pstep * mean_n / (per_pass_ms * 1e-3) / 1e9
    traffic = _profiled_traffic("k_pass1d_ccp1d_fp64.md" if prec == apic.FP64 else "k_pass1d_c32_ccp1d_fp32.md")
    sim.close()
    # the other storage form of the same discharge, device-timed the same way
    other = apic.FP32 if prec == apic.FP64 else apic.FP64
    other_ps, other_ms = _single_ccp(args, rank, other, max(50, args.steps // 2))
    forms = {("fp64" if prec == apic.FP64 else "fp32"): {"particle_steps_per_s": value, "ms_per_step": ms_max / args.steps},
             ("fp32" if other == apic.FP32 else "fp64"): {"particle_steps_per_s": other_ps, "ms_per_step": other_ms},
             "fp32_error": FP32_1D_ERROR}
    batched = _batched_ccp(args, rank) if args.batch > 1 else None
    if batched:
        batched["vs_plain_fp64_single_run"] = batched["value"] / forms["fp64"]["particle_steps_per_s"]
    return {
        "batched": batched,
        "forms": forms,
        "value": value, "ms_per_step": ms_max / args.steps, "dtype": "f64",
        "config": {"workload": WORKLOAD_CCP, "particles": int(mean_n),
                   "form": "FP64 particles (bit-faithful arithmetic)" if prec == apic.FP64 else
                   "FP32 cell form: int32 cell + FP32 offset + FP32 velocities, FP32 particle and collision "
                   "arithmetic; fixed-point charge, FP64 solve and ledgers; " + FP32_1D_ERROR,
                   "l2": "flushed between timed steps"},
        "e2e": {"value": e_total / (e_ms * 1e-3), "unit": "particle-steps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": "k_pass1d<3,true,false,false>" if prec == apic.FP64 else "k_pass1d_c32<3,true>",
                     "bytes_per_particle_step": bytes_per_pstep,
                     "pass_ms": per_pass_ms, "post_ms": post_ms / max(passes, 1)},
        "gpu_launches": 2 * args.steps,
        "clocks": clk.summary(),
    }


FP32_1D_ERROR = ("error against the FP64 oracle (tests/test_gpu_1d_fp32_cell.py): collisionless runs over "
                 "50 steps positions < 1e-4 cell, velocities < 1e-4 of the largest speed, fields < 1e-4; "
                 "the discharge over 6 seeds x 40 steps: per-channel collision counts, wall losses and mean "
                 "energies within 3 standard errors and within 1% where the counts exceed 1e4")


def _single_ccp(args, rank, prec, steps):
    """One discharge in the given storage form, device-timed over `steps`
    steps with the L2 flushed between steps; (particle-steps/s, ms/step)."""
    import torch
    import apic
    from apic import workloads as W
    wl = W.ccp_helium(particles_per_cell=args.ppc or 512, cells=args.cells or 512, seed=7 + rank)
    cfg, tabs = W.to_device_config(wl, precision=prec, seed=1000 + rank)
    sim = apic.Simulation1D(cfg, tabs)
    for i, s in enumerate(wl.species):
        sim.load(i, s.x, s.v, None, s.vy, s.vz)
    sim.initialize()
    sim.step(args.warmup)
    sim.synchronize()
    ext = torch.cuda.ExternalStream(sim.cuda_stream())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    flush_sink = torch.empty((), dtype=torch.float32, device="cuda")
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    n0 = sum(sim.count(s) for s in range(len(wl.species)))
    torch.cuda.synchronize()
    with torch.cuda.stream(ext):
        for i in range(steps):
            flush.zero_()
            flush_sink.copy_(flush.sum())
            starts[i].record(ext)
            sim.step(1)
            ends[i].record(ext)
    sim.synchronize()
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends))
    n1 = sum(sim.count(s) for s in range(len(wl.species)))
    sim.close()
    return steps * 0.5 * (n0 + n1) / (ms * 1e-3), ms / steps


def _batched_ccp(args, rank):
    """`args.batch` independent discharges in the FP32 particle form stepped
    together through apic_sim1d_step_group (their kernels overlap on the GPU):
    aggregate particle-steps/s, device time from one event before the launches
    to the last run's end event (host launch time included)."""
    import torch
    import apic
    from apic import workloads as W
    batch = args.batch
    tuned = None
    if not args.no_autotune:
        from apic import autotune

        def make(k):
            wl = W.ccp_helium(particles_per_cell=args.ppc or 512, cells=args.cells or 512, seed=200 + k)
            cfg, tabs = W.to_device_config(wl, precision=apic.FP32, seed=7000 + k)
            sim = apic.Simulation1D(cfg, tabs)
            for i, s in enumerate(wl.species):
                sim.load(i, s.x, s.v, None, s.vy, s.vz)
            sim.initialize()
            return sim, tabs

        tuned = autotune.tune_group(make, sizes=(2, 4, 8, 16))
        batch = tuned["runs"]
    sims = []
    for k in range(batch):
        wl = W.ccp_helium(particles_per_cell=args.ppc or 512, cells=args.cells or 512, seed=100 + 31 * rank + k)
        cfg, tabs = W.to_device_config(wl, precision=apic.FP32, seed=5000 + 31 * rank + k)
        sim = apic.Simulation1D(cfg, tabs)
        for i, s in enumerate(wl.species):
            sim.load(i, s.x, s.v, None, s.vy, s.vz)
        sim.initialize()
        sims.append((sim, tabs))
    group = [s for s, _ in sims]
    apic.step_group(group, max(args.warmup, 4))
    for s in group:
        s.synchronize()
    n0 = sum(s.count(i) for s in group for i in range(2))
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    start.record()
    apic.step_group(group, args.steps)
    ends = []
    for s in group:
        e = torch.cuda.Event(enable_timing=True)
        e.record(torch.cuda.ExternalStream(s.cuda_stream()))
        ends.append(e)
    torch.cuda.synchronize()
    ms = max(start.elapsed_time(e) for e in ends)
    n1 = sum(s.count(i) for s in group for i in range(2))
    for s in group:
        s.close()
    psteps = args.steps * 0.5 * (n0 + n1)
    return {"decks": batch, "autotuned": tuned["table"] if tuned else None,
            "value": psteps / (ms * 1e-3), "unit": "particle-steps/s",
            "ms_per_step": ms / args.steps,
            "form": "FP32 cell form, runs stepped together (apic_sim1d_step_group)",
            "l2": f"{batch} discharges' state larger than L2"}


def bench_plasma(args, rank, dist):
    """The 2D3V / 3D3V periodic decks, particles generated on the device."""
    import numpy as np
    import torch
    import apic
    from apic import workloads as W

    dims = 2 if args.workload == "plasma2d" else 3
    cells = None if args.cells is None else (args.cells,) * dims
    plan = W.plasma_plan(dims, cells=cells, ppc=args.ppc, seed=11 + 2 * rank)
    prec = apic.FP32 if args.precision == "fp32" else apic.FP64
    tuned = None
    sort_interval, push_items = args.sort_interval or 16, args.push_items
    if not args.no_autotune and not args.sort_interval:
        from apic import autotune
        tuned = autotune.tune_plasma(plan, prec, steps=32)
        sort_interval, push_items = tuned["sort_interval"], tuned["push_items"]
    sim = apic.SimulationND(plan.config(precision=prec, sort_interval=sort_interval, push_items=push_items))
    plan.load(sim)
    sim.initialize()
    sim.step(args.warmup)
    sim.synchronize()
    P = plan.particles
    ext = torch.cuda.ExternalStream(sim.cuda_stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches0 = sim.launch_count()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        e0.record(ext)
        sim.step(args.steps)  # one CUDA graph launch per step
        e1.record(ext)
        sim.synchronize()
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    launches = sim.launch_count() - launches0
    # per-kernel breakdown: the same number of steps again, kernel by kernel
    # with events between sort, push and solve (outside the timed region)
    sim.set_kernel_timing(True)
    sim.step(args.steps)
    sim.synchronize()
    push_ms, solve_ms, sort_ms, nsteps = sim.kernel_times()
    sim.set_kernel_timing(False)
    ms_max, total = _reduce(dist, ms, args.steps * P)
    value = total / (ms_max * 1e-3)

    # ---- end to end: pinned host state in, one step, state out ----
    ns = len(plan.species)
    host = []
    for k in range(ns):
        n = plan.species[k][3]
        host.append([torch.empty((3, n), dtype=torch.float64, pin_memory=True).numpy() for _ in range(3)])
    L = apic._bind_nd()
    got = apic.C.c_size_t()
    for k in range(ns):
        pos, v, vh = host[k]
        apic._check_nd(L.apic_simnd_read_particles(sim.h, k, pos.shape[1], apic.dptr(pos), apic.dptr(v),
                                                   apic.dptr(vh), apic.C.byref(got)), sim.h)
    s0 = sim.sample()
    t_sim, k_sim = s0.time, s0.step
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    e2e_ms, h2d, d2h = 0.0, 0, 0
    for it in range(args.e2e_steps):
        e_start.record(ext)
        for k in range(ns):
            pos, v, vh = host[k]  # rows 0..dims-1 of pos are the [dims][n] block load reads
            n = pos.shape[1]
            apic._check_nd(L.apic_simnd_load_particles(sim.h, k, n, apic.dptr(pos),
                                                       apic.dptr(v), apic.dptr(vh)), sim.h)
            if it == 0:
                h2d += (dims + 6) * 8 * n
        sim.resume(t_sim, k_sim)
        sim.step(1)
        for k in range(ns):
            pos, v, vh = host[k]
            apic._check_nd(L.apic_simnd_read_particles(sim.h, k, pos.shape[1], apic.dptr(pos), apic.dptr(v),
                                                       apic.dptr(vh), apic.C.byref(got)), sim.h)
            if it == 0:
                d2h += (dims + 6) * 8 * got.value
        e_end.record(ext)
        e_end.synchronize()
        e2e_ms += e_start.elapsed_time(e_end)
        t_sim, k_sim = t_sim + plan.dt, k_sim + 1
    e_ms, e_total = _reduce(dist, e2e_ms, args.e2e_steps * P)

    hbm, peak_kind = peaks()
    bpp = BYTES_PER_PSTEP[(args.workload, args.precision)]
    per_step_push = push_ms / max(nsteps, 1)
    achieved = bpp * P / (per_step_push * 1e-3) / 1e9
    # DRAM bytes per push launch from the committed ncu capture of a smaller
    # case of the same deck, scaled by the particles per launch (the state is
    # streamed once per launch, so traffic grows in proportion)
    traffic, traffic_note = None, None
    items = push_items or (4 if dims == 2 else 2)
    run_kernel = prec == apic.FP32 and items in (2, 4)  # consecutive particles per thread (k_push32_run)
    if prec == apic.FP32:
        captured = {2: 4194304, 3: 16777216}[dims]
        name = f"k_push32_run_plasma{dims}d_fp32.md" if run_kernel else f"k_push32_plasma{dims}d_fp32.md"
        t = _profiled_traffic(name)
        if t:
            traffic = t * (P / 2) / captured
            traffic_note = f"ncu capture ({name}) of {captured} particles per launch scaled to {P // 2}"
    form = ("FP32 particles: packed int32 cell + FP32 offsets + FP32 velocities; FP64 fixed-point deposit, "
            "FP64 spectral solve; error against the FP64 oracle after 10 steps (tests/test_gpu_nd.py): positions "
            "< 1e-5 cell, velocities < 1e-5 thermal, fields < 1e-4") if prec == apic.FP32 else \
        "FP64 particles (bit-faithful arithmetic)"
    sim.close()
    return {
        "value": value, "ms_per_step": ms_max / args.steps, "dtype": "f32" if prec == apic.FP32 else "f64",
        "config": {"workload": WORKLOAD_2D if dims == 2 else WORKLOAD_3D, "particles": P, "form": form,
                   "sort_interval": sort_interval, "push_items": push_items or ("4" if dims == 2 else "2"),
                   "autotuned": tuned["table"] if tuned else None,
                   "l2": f"inputs larger than L2 ({bpp // 2 * P / 1e9:.1f} GB of particle state)"},
        "e2e": {"value": e_total / (e_ms * 1e-3), "unit": "particle-steps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": traffic, "traffic_note": traffic_note, "peak_kind": peak_kind,
                     "kernel": (("k_push32_run" if run_kernel else "k_push32_step") if prec == apic.FP32 else "k_push")
                     + f"<{dims}, boris, items={items}>",
                     "bytes_per_particle_step": bpp, "push_ms": per_step_push,
                     "solve_ms": solve_ms / max(nsteps, 1), "sort_ms_per_step": sort_ms / max(nsteps, 1)},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }


def _swarm_draw(rng, spec, W, k, seed_base):
    """One serving request: E/N log-uniform in 10-1000 Td, electrons
    log-normal (median 100k, sigma 1) clipped to 10k-4M, 1% tolerance or 20k
    steps, 2000 burn-in steps."""
    import numpy as np
    td = float(np.exp(rng.uniform(np.log(10.0), np.log(1000.0))))
    n = int(np.clip(np.exp(rng.normal(np.log(1e5), 1.0)), 1e4, 4e6))
    return W.swarm_request(spec, td, particles=n, seed=seed_base + k, steps=20000, burn_in_steps=2000, tolerance=0.01)


def _mixed_serving(args, srv, spec, rng, rate, rank):
    """Swarm requests (Poisson, `rate`) mixed with small 1D two-stream decks
    (Poisson at rate / 2; Nx log-uniform over 64..1024, 64 particles per cell
    per beam, 2000 steps).  The swarm batch's graph and the decks' steps
    overlap on the GPU: each iteration launches the swarm batch, steps the
    active decks (apic_sim1d_step_group on their own streams), then completes
    the swarm batch.  Decks come from a pool created up front (no device
    allocation while serving)."""
    import numpy as np
    import apic
    from apic import workloads as W
    nxs = (64, 128, 256, 512, 1024)
    pool = {nx: [] for nx in nxs}
    for nx in nxs:
        for k in range(4):
            wl = W.two_stream(particles_per_beam=64 * nx, nx=nx, seed=1)
            cfg, tabs = W.to_device_config(wl, seed=9000 + k)
            pool[nx].append((apic.Simulation1D(cfg, tabs), tabs))
    free = {nx: list(range(4)) for nx in nxs}
    n_sw = args.mixed_requests
    n_dk = max(1, n_sw // 2)
    sw_arr = np.cumsum(rng.exponential(1.0 / rate, n_sw))
    dk_arr = np.cumsum(rng.exponential(2.0 / rate, n_dk))
    sw_req = [_swarm_draw(rng, spec, W, k, 40_000_000 + 1000 * rank) for k in range(n_sw)]
    dk_nx = [nxs[int(rng.integers(0, len(nxs)))] for _ in range(n_dk)]
    deck_steps, per_iter = 2000, 100
    _, ps0, _ = srv.stats()
    t0 = time.perf_counter()
    sw_sub, dk_wait, active = {}, [], []  # active: [sim, nx, slot, arrival, steps]
    sw_lat, dk_lat = [], []
    i_sw = i_dk = 0
    deck_psteps = 0
    while len(sw_lat) < n_sw or len(dk_lat) < n_dk:
        now = time.perf_counter() - t0
        while i_sw < n_sw and sw_arr[i_sw] <= now:
            sw_sub[srv.submit(sw_req[i_sw])] = sw_arr[i_sw]
            i_sw += 1
        while i_dk < n_dk and dk_arr[i_dk] <= now:
            dk_wait.append((dk_nx[i_dk], dk_arr[i_dk], i_dk))
            i_dk += 1
        for item in list(dk_wait):  # admit decks into free pool slots
            nx, arr, k = item
            if free[nx]:
                slot = free[nx].pop()
                sim = pool[nx][slot][0]
                wl = W.two_stream(particles_per_beam=64 * nx, nx=nx, seed=500 + k)
                for sp_i, sp in enumerate(wl.species):
                    sim.load(sp_i, sp.x, sp.v)
                sim.initialize()
                active.append([sim, nx, slot, arr, 0, 2 * 64 * nx])
                dk_wait.remove(item)
        srv.launch()
        if active:
            apic.step_group([a[0] for a in active], per_iter)
        srv.complete()
        now = time.perf_counter() - t0
        for i in list(sw_sub):
            r = srv.poll(i)
            if r is not None:
                sw_lat.append(now - sw_sub.pop(i))
        for a in list(active):
            a[4] += per_iter
            deck_psteps += per_iter * a[5]
            if a[4] >= deck_steps:
                a[0].sample()  # waits for the deck and reads its diagnostics
                dk_lat.append(time.perf_counter() - t0 - a[3])
                free[a[1]].append(a[2])
                active.remove(a)
        if not sw_sub and not active and not dk_wait:
            nxt = []
            if i_sw < n_sw:
                nxt.append(sw_arr[i_sw])
            if i_dk < n_dk:
                nxt.append(dk_arr[i_dk])
            if nxt:
                time.sleep(max(0.0, min(nxt) - (time.perf_counter() - t0)))
    wall = time.perf_counter() - t0
    _, ps1, _ = srv.stats()
    for nx in nxs:
        for sim, _ in pool[nx]:
            sim.close()
    sw_lat, dk_lat = np.array(sw_lat), np.array(dk_lat)
    return {"swarm_requests": n_sw, "deck_requests": n_dk,
            "swarm_p50_latency_s": float(np.percentile(sw_lat, 50)), "swarm_p99_latency_s": float(np.percentile(sw_lat, 99)),
            "deck_p50_latency_s": float(np.percentile(dk_lat, 50)), "deck_p99_latency_s": float(np.percentile(dk_lat, 99)),
            "particle_steps_per_s": ((ps1 - ps0) + deck_psteps) / wall,
            "decks": "two-stream 1D1V, Nx in 64..1024 (64 particles per cell per beam), 2000 steps, FP64"}


def bench_swarm(args, rank, dist):
    """Batched swarm serving: saturation throughput, then Poisson arrivals at
    80% of the measured capacity with p50 / p99 request latency."""
    import numpy as np
    import torch
    import apic
    from apic import workloads as W

    spec = W.swarm_c5()
    prec = apic.FP32 if args.precision == "fp32" else apic.FP64
    cfg, gas, tabs = W.to_device_swarm(spec, prec)
    free, _ = torch.cuda.mem_get_info()
    budget = int(min(64 << 30, 0.6 * free))
    rng = np.random.default_rng(5 + rank)
    spl, tuned = args.steps_per_launch or 200, None
    if not args.no_autotune and not args.steps_per_launch:
        from apic import autotune
        sample = [_swarm_draw(rng, spec, W, k, 5_000_000) for k in range(12)]
        tuned = autotune.tune_swarm_server(gas, sample, prec, min(budget, 16 << 30))
        spl = tuned["steps_per_launch"]
    srv = apic.SwarmServer(gas, budget, max_runs=256, precision=prec, steps_per_launch=spl)
    ext = torch.cuda.ExternalStream(srv.cuda_stream())

    def drain(ids, submit_at=None, pending=None):
        done = {}
        while len(done) < len(ids):
            srv.advance()
            for i in ids:
                if i not in done:
                    r = srv.poll(i)
                    if r is not None:
                        done[i] = r
        return done

    # warm-up: graph capture and first-touch of the pool
    drain([srv.submit(_swarm_draw(rng, spec, W, k, 10_000_000)) for k in range(max(args.warmup, 3))])

    # -- saturation: a full queue, device time over the whole batch --
    batch = [_swarm_draw(rng, spec, W, k, 20_000_000 + 1000 * rank) for k in range(args.steps)]
    _, ps0, _ = srv.stats()
    ids = [srv.submit(r) for r in batch]
    srv.set_kernel_timing(True)  # the first two advances time the push kernel one launch at a time
    srv.advance()
    srv.advance()
    push_ms, collide_ms, push_launches, push_bytes = srv.kernel_times()
    srv.set_kernel_timing(False)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    with Clocks(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        e0.record(ext)
        g0 = srv.stats()[0]
        k0 = srv.kernel_launches()
        res = drain(ids)
        k1 = srv.kernel_launches()
        e1.record(ext)
        e1.synchronize()
    t_sat = e0.elapsed_time(e1) * 1e-3
    g1, ps1, _ = srv.stats()
    sat_psteps = ps1 - ps0
    # the two timed advances ran before e0: count only the work inside the region
    ms_max, total = _reduce(dist, t_sat * 1e3, float(sat_psteps))
    value = total / (ms_max * 1e-3)
    capacity = len(batch) / t_sat
    assert all(r.status == 0 for r in res.values()), [r.message for r in res.values() if r.status]

    # -- serving: Poisson arrivals at 80% of capacity --
    rate = 0.8 * capacity
    gaps = rng.exponential(1.0 / rate, args.requests)
    arrivals = np.cumsum(gaps)
    reqs = [_swarm_draw(rng, spec, W, k, 30_000_000 + 1000 * rank) for k in range(args.requests)]
    g2, ps2, _ = srv.stats()
    h2d0, d2h0 = srv.copy_bytes()
    t0 = time.perf_counter()
    sub, lat, results = {}, [], []
    nxt = 0
    while len(lat) < args.requests:
        now = time.perf_counter() - t0
        while nxt < args.requests and arrivals[nxt] <= now:
            sub[srv.submit(reqs[nxt])] = arrivals[nxt]
            nxt += 1
        active, queued = srv.advance()
        now = time.perf_counter() - t0
        for i in list(sub):
            r = srv.poll(i)
            if r is not None:
                lat.append(now - sub.pop(i))
                results.append(r)
        if not active and not queued and nxt < args.requests:
            time.sleep(max(0.0, arrivals[nxt] - (time.perf_counter() - t0)))
    t_serve = time.perf_counter() - t0
    g3, ps3, _ = srv.stats()
    h2d1, d2h1 = srv.copy_bytes()
    serve_steps = max(1, (g3 - g2) * spl)  # device steps of the serving phase
    serve_value = (ps3 - ps2) / t_serve
    mixed = _mixed_serving(args, srv, spec, rng, rate, rank) if args.mixed_requests > 0 else None
    srv.close()
    lat = np.array(lat)
    hbm, peak_kind = peaks()
    achieved = push_bytes / (push_ms * 1e-3) / 1e9 if push_ms > 0 else None
    steps_done = np.array([r.steps_done for r in results])
    return {
        "value": value, "ms_per_step": 1e3 * t_sat / max(1, (g1 - g0) * spl), "dtype": "f32" if prec == apic.FP32 else "f64",
        "config": {"workload": WORKLOAD_SWARM, "form": ("FP32 electron velocity + displacement and FP32 collision "
                                                        "loops; FP64 tallies; error against the FP64 form "
                                                        "(tests/test_gpu_swarm.py): over 12 seeds per field the "
                                                        "ensemble means of drift velocity, mean energy and the "
                                                        "ionization rate coefficient within 3 combined standard "
                                                        "errors") if prec == apic.FP32 else
                   "FP64 electrons", "saturation_requests": len(batch), "steps_per_launch": spl,
                   "autotuned": tuned["table"] if tuned else None,
                   "l2": "electron state of the batch larger than L2"},
        "e2e": {"value": serve_value, "unit": "particle-steps/s",
                "h2d_bytes_per_step": (h2d1 - h2d0) / serve_steps, "d2h_bytes_per_step": (d2h1 - d2h0) / serve_steps,
                "note": ("Poisson serving phase through the swarm server API, host wall clock: requests and "
                         "results are host structs; bytes per device step are the server's own copies (run "
                         "set-up, chunk tables, samples read for the convergence test, results)")},
        "swarm": {"p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
                  "capacity_requests_per_s": capacity, "arrival_rate_requests_per_s": rate,
                  "requests": int(args.requests), "converged_fraction": float(np.mean([r.converged for r in results])),
                  "mean_steps": float(steps_done.mean()), "serving_particle_steps_per_s": serve_value,
                  "mixed": mixed},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm if achieved else None, "traffic": None,
                     "traffic_note": "no ncu capture at the saturation size: the pool there spans tens of GB",
                     "peak_kind": peak_kind, "kernel": "k_swarm_push<float>",
                     "bytes_per_particle_step": "24 (burn-in) / 48 (sampling)",
                     "push_ms_per_launch": push_ms / max(push_launches, 1),
                     "collide_ms_per_launch": collide_ms / max(push_launches, 1)},
        "gpu_launches": int(k1 - k0),
        "clocks": clk.summary(),
    }


# The nested records of the default run: the other benchmark shapes with the
# settings the autotuner picked for them on the B200 (sort interval and
# particles per thread of the plasma decks, graph length of the swarm server),
# a few timed steps each and a shorter CPU sample, so the whole default run
# stays within a few minutes.
OTHER_CONFIGS = {
    "plasma2d": {"sort_interval": 8, "push_items": 4, "e2e_steps": 2},
    "plasma3d": {"sort_interval": 3, "push_items": 2, "e2e_steps": 1},
    "swarm": {"steps_per_launch": 100, "requests": 48, "mixed_requests": 16},
}


def bench_other_configs(args, rank, dist, world):
    """The 2D3V (512^2 x 64 ppc), 3D3V (256^3 x 8 ppc) and swarm-serving
    shapes measured the way their own --workload runs measure them, each with
    its roofline, end-to-end figure, clocks and CPU baseline."""
    out = {}
    for wk, over in OTHER_CONFIGS.items():
        a = argparse.Namespace(**vars(args))
        a.workload, a.precision, a.no_autotune = wk, "fp32", True
        a.steps = max(args.steps, 20)
        a.warmup = max(args.warmup, 3)
        for k, v in over.items():
            setattr(a, k, v)
        t0 = time.perf_counter()
        try:
            part = bench_swarm(a, rank, dist) if wk == "swarm" else bench_plasma(a, rank, dist)
        except Exception as e:  # reported in the record, never fatal to the headline
            out[wk] = {"error": f"{type(e).__name__}: {e}"}
            continue
        rec = {k: part[k] for k in ("value", "ms_per_step", "dtype", "config", "e2e", "roofline", "gpu_launches",
                                    "clocks") if k in part}
        rec["unit"] = "particle-steps/s"
        rec["steps"], rec["warmup"] = a.steps, a.warmup
        if "swarm" in part:
            rec["swarm"] = part["swarm"]
        rec["cpu_baseline"] = None
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            try:
                from apic import workloads as W
                wl = None if wk == "swarm" else W.plasma_plan(2 if wk == "plasma2d" else 3)
                rec["cpu_baseline"] = cpu_reference_sample(a, wl, min(args.cpu_seconds, 10.0), os.cpu_count() or 1)
            except Exception as e:
                rec["cpu_baseline"] = {"value": None, "error": str(e)}
        rec["wall_s"] = time.perf_counter() - t0
        out[wk] = rec
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    others = None
    if args.workload == "ccp1d":
        part = bench_ccp1d(args, rank, dist)
        if world == 1 and not args.no_other_configs:
            others = bench_other_configs(args, rank, dist, world)
    elif args.workload == "swarm":
        part = bench_swarm(args, rank, dist)
    else:
        part = bench_plasma(args, rank, dist)

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                from apic import workloads as W
                wl = (W.ccp_helium(particles_per_cell=args.ppc or 512, cells=args.cells or 512, seed=7)
                      if args.workload == "ccp1d" else None if args.workload == "swarm"
                      else W.plasma_plan(2 if args.workload == "plasma2d" else 3))
                cpu = cpu_reference_sample(args, wl, args.cpu_seconds, os.cpu_count() or 1)
            except Exception as e:  # reported, never fatal
                cpu = {"value": None, "error": str(e)}
        cfg = dict(part["config"])
        cfg["parallelism"] = f"replicas x{world}"
        line = {
            "metric": METRIC, "value": part["value"], "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": part["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": part["dtype"],
            "data": "synthetic", "config": cfg, "e2e": part["e2e"], "roofline": part["roofline"],
            "gpu_launches": part["gpu_launches"], "clocks": part["clocks"], "cpu_baseline": cpu,
        }
        if "swarm" in part:
            line["swarm"] = part["swarm"]
        if part.get("forms"):
            line["forms"] = part["forms"]
        if part.get("batched"):
            b = dict(part["batched"])
            b["vs_single_run"] = b["value"] / part["value"]
            line["batched"] = b
        if others:
            line["configs"] = others
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
