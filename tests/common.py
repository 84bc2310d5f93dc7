"""Shared helpers of the parity tests: build the oracle's configuration from
the same workload the device library runs, and compare results."""
from __future__ import annotations

import numpy as np

import pyoracle as po
from apic import workloads as W


def oracle_config(wl: W.Workload1D, tables: po.TableSet, seed=12345, threads=0, particles=None):
    return po.config_from_workload(wl, tables, seed=seed, threads=threads, particles=particles)


def load_oracle(sim: po.Sim1D, wl: W.Workload1D):
    for i, s in enumerate(wl.species):
        sim.load(i, s.x, s.v, s.v, s.vy, s.vz)


def load_device(sim, wl: W.Workload1D):
    for i, s in enumerate(wl.species):
        sim.load(i, s.x, s.v, None, s.vy, s.vz)


def rel_max(a, b):
    """max |a - b| / max |b| (norm-relative error)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.shape != b.shape:
        raise AssertionError(f"shape mismatch {a.shape} vs {b.shape}")
    scale = np.max(np.abs(b)) if b.size else 0.0
    if scale == 0.0:
        return float(np.max(np.abs(a))) if a.size else 0.0
    return float(np.max(np.abs(a - b)) / scale)
