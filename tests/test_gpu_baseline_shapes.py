"""Parity at the benchmark shapes (not only on small decks):

* the 1D3V capacitive discharge at its full size (512 cells, 512 electrons +
  512 He+ per cell) for a few steps against the oracle's device form with the
  same Philox streams: collision counts exact, particle state within 1e-11;
* the 1D1V two-stream deck at its full size (Nx 256, 2 x 16384) over 100 steps,
  FP64 within 1e-12;
* the 2D3V and 3D3V periodic decks with their real particles per cell (64 and
  8) and the benchmark's sort interval and particles per thread, on meshes
  scaled to 64^2 and 32^3: FP64 within 1e-12, the FP32 form within its stated
  bounds against the FP64 oracle (positions 1e-5 cell, velocities 1e-5 of the
  largest speed, fields 1e-4)."""
import numpy as np
import pytest

import apic
import pyoracle as po
from apic import workloads as W
from common import load_device, load_oracle, oracle_config, rel_max

pytestmark = pytest.mark.gpu


def test_full_discharge_against_the_oracle():
    wl = W.ccp_helium(particles_per_cell=512, cells=512, seed=7)
    seed = 0x5EED
    cfg, tabs = W.to_device_config(wl, seed=seed)
    dev = apic.Simulation1D(cfg, tabs)
    load_device(dev, wl)
    dev.initialize()
    T = po.TableSet()
    ora = po.Sim1D(oracle_config(wl, T), 1, seed)
    load_oracle(ora, wl)
    ora.initialize()
    steps = 3
    dev.step(steps)
    ora.step(steps)
    tot = dev.collision_totals()
    c, nl, per = ora.collisions()
    assert tot.candidates == c and tot.null_collisions == nl
    for m in range(2):
        assert list(tot.channel_collisions[m])[:len(per[m])] == list(per[m])
    for s in range(2):
        a, b = dev.particles(s), ora.particles(s)
        assert len(a["x"]) == len(b["x"])
        for k in ("x", "v", "vh", "vy", "vz"):
            assert rel_max(a[k], b[k]) < 1e-11, (s, k, rel_max(a[k], b[k]))
        bl = dev.boundary_losses(s)
        assert (bl.absorbed_left, bl.absorbed_right) == tuple(ora.losses(s)[:2])
    for a, b in zip(dev.fields(), ora.fields()):
        assert rel_max(a, b) < 1e-11
    dev.close()


def test_full_two_stream_deck():
    wl = W.two_stream()
    cfg, tabs = W.to_device_config(wl)
    dev = apic.Simulation1D(cfg, tabs)
    load_device(dev, wl)
    dev.initialize()
    T = po.TableSet()
    ora = po.Sim1D(oracle_config(wl, T), 1)
    load_oracle(ora, wl)
    ora.initialize()
    dev.step(100)
    ora.step(100)
    for s in range(2):
        a, b = dev.particles(s), ora.particles(s)
        for k in ("x", "v", "vh"):
            assert rel_max(a[k], b[k]) < 1e-12, (s, k)
    for a, b in zip(dev.fields(), ora.fields()):
        assert rel_max(a, b) < 1e-12


def _scaled(dims):
    if dims == 2:
        return W.plasma_2d(cells=(64, 64), ppc=64, seed=21), 8, 4
    return W.plasma_3d(cells=(32, 32, 32), ppc=8, seed=23), 8, 2


@pytest.mark.parametrize("dims", [2, 3])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_plasma_decks_at_benchmark_particles_per_cell(dims, precision):
    wl, sort_interval, items = _scaled(dims)
    prec = apic.FP64 if precision == "fp64" else apic.FP32
    cfg = W.to_device_config_nd(wl, precision=prec, sort_interval=sort_interval)
    cfg.push_items = items
    dev = apic.SimulationND(cfg)
    ora = po.SimND(wl.dims, wl.n, wl.length, wl.dt, W.EPS0, wl.B, [(q, m, w) for (q, m, w, pos, v) in wl.species])
    for k, (q, m, w, pos, v) in enumerate(wl.species):
        dev.load(k, pos, v)
        ora.load(k, pos, v, v)
    dev.initialize()
    ora.initialize()
    steps = 10  # spans a re-sort of the electrons
    dev.step(steps)
    ora.step(steps)
    for k in range(2):
        a, b = dev.particles(k), ora.particles(k)
        if prec == apic.FP64:
            for name, x, y in zip(("pos", "v", "vh"), a, b):
                assert rel_max(x[:dims] if name == "pos" else x, y[:dims] if name == "pos" else y) < 1e-12, (k, name)
        else:
            cell = wl.length[0] / wl.n[0]
            d = np.abs(a[0][:dims] - b[0][:dims])
            d = np.minimum(d, np.array(wl.length)[:dims, None] - d)
            assert d.max() < 1e-5 * cell, (k, d.max() / cell)
            vs = np.max(np.abs(b[2]))
            assert np.max(np.abs(a[2] - b[2])) < 1e-5 * vs
    tol = 1e-12 if prec == apic.FP64 else 1e-4
    for name, x, y in zip(("rho", "phi", "E"), dev.fields(), ora.fields()):
        y = np.asarray(y).reshape(-1, int(np.prod(wl.n)))[:dims] if name == "E" else y
        assert rel_max(x, y) < tol, (name, rel_max(x, y))
    dev.close()
