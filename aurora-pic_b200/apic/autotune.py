"""Autotuner of the launch and schedule parameters that do not change results.

Each tuner times a short run of the caller's own workload for every candidate
on the current GPU (CUDA events on the library's stream) and returns the
fastest, with the table of timings.  Results can be cached in a JSON file keyed
by the workload shape and the device name, so a service tunes once per shape.

* ``tune_plasma``: 2D3V/3D3V decks - cell-sort interval x particles per thread
  of the FP32 step push (``apic_config_nd.sort_interval``, ``push_items``).
* ``tune_swarm_server``: steps per graph launch of the swarm server (the
  convergence-check cadence trades latency against launch overhead).
* ``tune_group``: how many 1D runs to step together on one GPU.
"""
from __future__ import annotations

import json
import os
import time

import numpy as np


def _device_name():
    import torch
    return torch.cuda.get_device_name()


def _cache_get(path, key):
    if not path or not os.path.exists(path):
        return None
    try:
        return json.load(open(path)).get(key)
    except (OSError, ValueError):
        return None


def _cache_put(path, key, value):
    if not path:
        return
    data = {}
    if os.path.exists(path):
        try:
            data = json.load(open(path))
        except (OSError, ValueError):
            data = {}
    data[key] = value
    with open(path, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)


def tune_plasma(plan, precision, sort_intervals=(2, 3, 4, 6, 8, 16), push_items=(1, 2, 4, 8), steps=None, cache=None):
    """Fastest (sort_interval, push_items) for a workloads.PlasmaPlan deck:
    each candidate runs one full sort period (at least `steps` steps) after a
    warm-up and is timed per step, sort included."""
    import torch
    import apic
    key = f"plasma/{plan.dims}/{'x'.join(map(str, plan.n))}/{plan.particles}/{precision}/{_device_name()}"
    hit = _cache_get(cache, key)
    if hit:
        return hit
    items = push_items if precision == apic.FP32 else (0,)
    table = []
    for si in sort_intervals:
        for it in items:
            sim = apic.SimulationND(plan.config(precision=precision, sort_interval=si, push_items=it))
            plan.load(sim)
            sim.initialize()
            sim.step(2)
            sim.synchronize()
            n = max(si, steps or si)
            ext = torch.cuda.ExternalStream(sim.cuda_stream())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            sim.step(n)
            e1.record(ext)
            e1.synchronize()
            table.append({"sort_interval": si, "push_items": it, "ms_per_step": e0.elapsed_time(e1) / n})
            sim.close()
    best = min(table, key=lambda r: r["ms_per_step"])
    out = {"sort_interval": best["sort_interval"], "push_items": best["push_items"], "table": table}
    _cache_put(cache, key, out)
    return out


def tune_swarm_server(gas, requests, precision, memory_budget_bytes, candidates=(50, 100, 200, 400), cache=None):
    """Fastest steps_per_launch of an apic.SwarmServer on a sample batch of
    `requests` (apic.SwarmRequest): the batch is run to completion for each
    candidate; particle-steps per second decide."""
    import apic
    key = f"swarm/{len(requests)}/{sum(r.particles for r in requests)}/{precision}/{_device_name()}"
    hit = _cache_get(cache, key)
    if hit:
        return hit
    table = []
    for spl in candidates:
        srv = apic.SwarmServer(gas, memory_budget_bytes, max_runs=max(len(requests), 1), precision=precision,
                               steps_per_launch=spl)
        ids = [srv.submit(r) for r in requests]
        t0 = time.perf_counter()
        done = set()
        while len(done) < len(ids):
            srv.advance()
            for i in ids:
                if i not in done and srv.poll(i) is not None:
                    done.add(i)
        dt = time.perf_counter() - t0
        psteps = srv.stats()[1]
        srv.close()
        table.append({"steps_per_launch": spl, "particle_steps_per_s": psteps / dt})
    best = max(table, key=lambda r: r["particle_steps_per_s"])
    out = {"steps_per_launch": best["steps_per_launch"], "table": table}
    _cache_put(cache, key, out)
    return out


def tune_group(make_run, sizes=(1, 2, 4, 8, 16), steps=40, cache=None, key=None):
    """Number of 1D runs to step together: `make_run(k)` builds and
    initialises run k (an apic.Simulation1D); aggregate particle-steps per
    second decide (the GPU fills up, then extra runs only queue).  Each size
    is warmed up for 8 steps (every run's step graphs exist by then) and timed
    twice over `steps` steps; the faster repetition counts."""
    import torch
    import apic
    ck = f"group/{key}/{_device_name()}" if key else None
    hit = _cache_get(cache, ck) if ck else None
    if hit:
        return hit
    table = []
    for k in sizes:
        runs = [make_run(i) for i in range(k)]
        apic.step_group([r[0] for r in runs], 8)
        for r in runs:
            r[0].synchronize()
        rate = 0.0
        for _rep in range(2):
            n = sum(r[0].count(s) for r in runs for s in range(2))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            apic.step_group([r[0] for r in runs], steps)
            for r in runs:
                r[0].synchronize()
            rate = max(rate, n * steps / (time.perf_counter() - t0))
        table.append({"runs": k, "particle_steps_per_s": rate})
        for r in runs:
            r[0].close()
    best = max(table, key=lambda r: r["particle_steps_per_s"])
    out = {"runs": best["runs"], "table": table}
    if ck:
        _cache_put(cache, ck, out)
    return out
