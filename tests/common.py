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


def swarm_cases():
    """The small swarm decks pinned by golden vectors from the reference's
    run_swarm_benchmark (tests/golden/swarm_*.npz)."""
    fixed = W.swarm_c5(fields_td=(10.0, 300.0), particles=200, steps=300, burn_in_steps=100)
    ch, mn = W.swarm_gas_anisotropic(attachment=True)
    ng, T = 1e24, 300.0
    nu = W.swarm_max_frequency(ch, ng, mn, T, 150.0)
    branching = W.SwarmSpec("aniso_attach", ch, mn, ng, T, nu, 0.08 / nu, 400, 200, 300, [50.0, 400.0],
                            branching=True, uncertainty_blocks=10, initial_mean_energy_ev=2.0, max_energy_ev=150.0,
                            seed=99)
    return {"swarm_fixed": fixed, "swarm_branching": branching}


SWARM_KEYS = ("mean_velocity_x", "mean_velocity_x_se", "drift_velocity", "reduced_mobility", "mean_energy_ev",
              "mean_energy_se_ev", "diffusion_longitudinal", "diffusion_transverse", "max_observed_energy_ev",
              "final_weight", "final_particles", "growth_rate", "growth_rate_se", "ionization_rate",
              "ionization_rate_se", "attachment_rate", "attachment_rate_se", "net_rate", "townsend_growth",
              "townsend_rate", "candidates", "null_collisions")


ENSEMBLE_SEEDS = 12


def swarm_ensemble_cases():
    """Decks whose seed ensembles (ENSEMBLE_SEEDS reference runs each, in
    tests/golden/swarm_ensemble_*.npz) pin the device statistically: the
    anisotropic gas at 1e24 m^-3 relaxes within the burn-in, and ensemble
    averages over independent seeds carry honest standard errors (block errors
    of one branching run understate the step-to-step correlation that
    resampling creates)."""
    out = {}
    for name, att in (("ens_fixed", False), ("ens_branching", True)):
        ch, mn = W.swarm_gas_anisotropic(attachment=att)
        ng, T = 1e24, 300.0
        nu = W.swarm_max_frequency(ch, ng, mn, T, 199.0)
        out[name] = W.SwarmSpec(name, ch, mn, ng, T, nu, 0.08 / nu, 600, 300, 2000, [50.0, 250.0],
                                branching=att, uncertainty_blocks=10, initial_mean_energy_ev=2.0,
                                max_energy_ev=199.0, seed=1000)
    return out


ENSEMBLE_KEYS = ("mean_velocity_x", "mean_energy_ev", "ionization_rate", "attachment_rate")
