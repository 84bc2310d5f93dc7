"""Shared helpers of the parity tests: build the oracle's configuration from
the same workload the device library runs, and compare results."""
from __future__ import annotations

import numpy as np

import pyoracle as po
from apic import workloads as W


def oracle_config(wl: W.Workload1D, tables: po.TableSet, seed=12345, threads=0, particles=None):
    models = []
    for m in wl.models:
        chans = [tables.channel(c.process, c.energy, c.sigma, c.threshold, c.secondary, c.ion) for c in m.channels]
        models.append(po.make_model(m.species, chans, m.neutral_density, m.max_frequency, m.neutral_mass,
                                    m.neutral_temperature, 1 if wl.si else 0, m.max_candidates))
    species = []
    for s in wl.species:
        n = len(s.x) if particles is None else particles
        species.append((s.charge, s.mass, s.weight, n, 0.0, 0.0, 0.0, 0.0))
    return po.config1d(dirichlet=int(wl.dirichlet), vdim=wl.vdim, si=int(wl.si), nx=wl.nx, length=wl.length,
                       dt=wl.dt, species=species, models=models, phi_left=wl.phi_left, phi_right=wl.phi_right,
                       drive_left=wl.drive_left, drive_right=wl.drive_right, seed=seed, threads=threads,
                       max_particles=max(s.capacity for s in wl.species))


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
