"""The 1D FP32 cell form (APIC_FP32: int32 cell + float offset positions, float
velocities, FP32 particle arithmetic and FP32 null-collision loops; 64-bit
fixed-point charge, FP64 field solve and energy ledgers) through the C ABI.

Its error against the FP64 oracle, stated per quantity for collisionless runs:
  positions  1e-4 of a cell (periodic distance)
  velocities 1e-4 of the largest speed
  fields     1e-4 relative (max norm)
and statistically for runs with collisions (the FP32 loop draws its own
uniforms, so trajectories differ once a particle collides): over seeds, the
per-channel collision counts, wall losses and mean kinetic energies of the
discharge agree with the FP64 form within 3 combined standard errors, and
within 1% wherever the FP64 form's mean count is large enough (>= 10^4) for
1% to lie above the statistical noise."""
import numpy as np
import pytest

import apic
import pyoracle as po
from apic import workloads as W
from common import load_device, load_oracle, oracle_config, rel_max

pytestmark = pytest.mark.gpu
TOL_X = 1e-4   # of a cell
TOL_V = 1e-4   # of the largest speed
TOL_F = 1e-4   # fields, relative


def _pair(wl, steps, seed=0x5EED):
    cfg, tabs = W.to_device_config(wl, precision=apic.FP32, seed=seed)
    dev = apic.Simulation1D(cfg, tabs)
    load_device(dev, wl)
    dev.initialize()
    T = po.TableSet()
    ora = po.Sim1D(oracle_config(wl, T), 1, seed)
    load_oracle(ora, wl)
    ora.initialize()
    dev.step(steps)
    ora.step(steps)
    return dev, ora, (T, tabs)


def _compare_state(wl, dev, ora, s):
    a, b = dev.particles(s), ora.particles(s)
    assert len(a["x"]) == len(b["x"]), (s, len(a["x"]), len(b["x"]))
    dx = wl.length / (wl.nx - 1 if wl.dirichlet else wl.nx)
    d = np.abs(a["x"] - b["x"])
    if not wl.dirichlet:
        d = np.minimum(d, wl.length - d)
    assert d.max() < TOL_X * dx, (s, d.max() / dx)
    keys = ("vh", "v", "vy", "vz") if wl.vdim == 3 else ("vh", "v")
    vmax = max(float(np.max(np.abs(b[k]))) for k in keys)
    for k in keys:
        assert np.max(np.abs(a[k] - b[k])) < TOL_V * vmax, (s, k, np.max(np.abs(a[k] - b[k])) / vmax)
    # the stored components really are floats
    for k in ("vh", "vy", "vz") if wl.vdim == 3 else ("vh",):
        assert np.array_equal(a[k], a[k].astype(np.float32).astype(np.float64)), k


@pytest.mark.parametrize("steps", [1, 10, 50])
def test_cell_form_two_stream_against_fp64_oracle(steps):
    wl = W.two_stream(particles_per_beam=2048, nx=64, seed=3)
    dev, ora, _keep = _pair(wl, steps)
    for s in range(2):
        _compare_state(wl, dev, ora, s)
    for a, b in zip(dev.fields(), ora.fields()):
        assert rel_max(a, b) < TOL_F, rel_max(a, b)
    dev.close()


def test_cell_form_rf_walls_against_fp64_oracle():
    wl = W.ccp_helium(particles_per_cell=32, cells=64, seed=11, table_rows=1024, te_ev=4.0)
    wl.models = []
    dev, ora, _keep = _pair(wl, 40)
    lost = 0
    for s in range(2):
        b = dev.boundary_losses(s)
        l, r, el, er = ora.losses(s)
        assert (b.absorbed_left, b.absorbed_right) == (l, r)
        lost += l + r
        if l + r:
            e_dev = b.kinetic_energy_left + b.kinetic_energy_right
            assert abs(e_dev - (el + er)) <= 1e-4 * (el + er)
        _compare_state(wl, dev, ora, s)
    assert lost > 0  # the walls absorbed something
    for a, b in zip(dev.fields(), ora.fields()):
        assert rel_max(a, b) < TOL_F, rel_max(a, b)
    dev.close()


def test_cell_form_load_readback_and_reproducibility():
    """Read-back right after the load gives the loaded state rounded to the
    form (positions to 2^-24 of a cell, velocities to float); two identical
    runs with collisions and ionization products end bit-identical."""
    wl = W.ccp_helium(particles_per_cell=16, cells=64, seed=3, table_rows=512, te_ev=30.0)
    cfg, tabs = W.to_device_config(wl, precision=apic.FP32, seed=9)
    dev = apic.Simulation1D(cfg, tabs)
    load_device(dev, wl)
    dx = wl.length / (wl.nx - 1)
    for s, sp in enumerate(wl.species):
        a = dev.particles(s)
        assert np.max(np.abs(a["x"] - sp.x)) <= 1.2e-7 * dx
        assert np.array_equal(a["vy"], sp.vy.astype(np.float32).astype(np.float64))
    runs = []
    for _ in range(2):
        sim = apic.Simulation1D(cfg, tabs)
        load_device(sim, wl)
        sim.initialize()
        sim.step(30)
        runs.append(sim)
    t = runs[0].collision_totals()
    assert t.channel_collisions[0][2] > 0  # ionization happened
    for s in range(2):
        a, b = runs[0].particles(s), runs[1].particles(s)
        for k in a:
            assert np.array_equal(a[k], b[k]), k
    for a, b in zip(runs[0].fields(), runs[1].fields()):
        assert np.array_equal(a, b)
    for sim in runs + [dev]:
        sim.close()


def test_cell_form_step_group_matches_single_runs():
    decks = [W.ccp_helium(particles_per_cell=16, cells=64, seed=3, table_rows=256, te_ev=12.0),
             W.two_stream(particles_per_beam=2048, nx=64, seed=4)]

    def make(wl, k):
        cfg, tabs = W.to_device_config(wl, precision=apic.FP32, seed=77 + k)
        sim = apic.Simulation1D(cfg, tabs)
        load_device(sim, wl)
        sim.initialize()
        return sim, tabs

    grouped = [make(wl, k) for k, wl in enumerate(decks)]
    single = [make(wl, k) for k, wl in enumerate(decks)]
    apic.step_group([g for g, _ in grouped], 9)
    for s, _ in single:
        s.step(9)
    for (g, _), (s, _), wl in zip(grouped, single, decks):
        for k in range(len(wl.species)):
            a, b = g.particles(k), s.particles(k)
            for key in a:
                assert np.array_equal(a[key], b[key]), key


def _discharge_tallies(precision, seed, steps, te_ev):
    wl = W.ccp_helium(particles_per_cell=512, cells=512, seed=100 + seed, te_ev=te_ev)
    cfg, tabs = W.to_device_config(wl, precision=precision, seed=1000 + seed)
    sim = apic.Simulation1D(cfg, tabs)
    load_device(sim, wl)
    sim.initialize()
    sim.step(steps)
    t = sim.collision_totals()
    smp = sim.sample()
    out = {"candidates": t.candidates}
    for m, nch in ((0, 3), (1, 2)):
        for c in range(nch):
            out[f"m{m}c{c}"] = t.channel_collisions[m][c]
    for s in range(2):
        b = sim.boundary_losses(s)
        out[f"lost{s}"] = b.absorbed_left + b.absorbed_right
        out[f"ke{s}"] = smp.kinetic_by_species[s] / smp.live_by_species[s]
    sim.close()
    return out


def test_cell_form_discharge_statistics_match_fp64():
    """The full discharge (512 cells, 512 electrons + 512 He+ per cell, Te
    10 eV so that every channel fires), 6 seeds x 40 steps in each form."""
    seeds, steps = 6, 40
    f64 = [_discharge_tallies(apic.FP64, k, steps, 10.0) for k in range(seeds)]
    f32 = [_discharge_tallies(apic.FP32, k, steps, 10.0) for k in range(seeds)]
    for key in f64[0]:
        a = np.array([r[key] for r in f64], dtype=np.float64)
        b = np.array([r[key] for r in f32], dtype=np.float64)
        ma, mb = a.mean(), b.mean()
        se = np.sqrt(a.var(ddof=1) / seeds + b.var(ddof=1) / seeds)
        # counts: add the Poisson floor so that identical small counts pass
        floor = np.sqrt(max(ma, 1.0) / seeds) if not key.startswith("ke") else 0.0
        assert abs(mb - ma) <= 3.0 * max(se, floor), (key, ma, mb, se)
        if (key.startswith("ke") or ma >= 1e4):
            assert abs(mb - ma) <= 0.01 * abs(ma), (key, ma, mb)
