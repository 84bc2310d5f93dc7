"""Device sample() against the reference's diagnostic sums evaluated on the
oracle's state (tests/diag_formulas.py, pinned to the reference's own
Simulation::sample by tests/test_diag_formulas.py).  FP64 form: 1e-12
relative, counts exact.  FP32 particle forms: against the FP64 oracle within
the forms' stated bounds (energies 1e-4 relative)."""
import numpy as np
import pytest

import apic
import pyoracle as po
from apic import workloads as W
from common import load_device, load_oracle, oracle_config
from diag_formulas import sample_1d, sample_nd

pytestmark = pytest.mark.gpu
TOL = 1e-12
FP32_TOL = 1e-4


def _check_1d(s, ref, tol, exact_counts=True):
    for k in ("kinetic_energy", "field_energy", "total_energy", "charge_l1"):
        got, want = getattr(s, k), ref[k]
        assert abs(got - want) <= tol * abs(want), (k, got, want)
    for i, ke in enumerate(ref["kinetic_by_species"]):
        assert abs(s.kinetic_by_species[i] - ke) <= tol * abs(ke), (i, s.kinetic_by_species[i], ke)
    if exact_counts:
        assert s.live_particles == ref["live_particles"]
        assert list(s.live_by_species)[:len(ref["live_by_species"])] == ref["live_by_species"]
    if "phi_left" in ref:
        assert abs(s.phi_left - ref["phi_left"]) <= 1e-12 * max(1.0, abs(ref["phi_left"]))
        assert abs(s.phi_right - ref["phi_right"]) <= 1e-12 * max(1.0, abs(ref["phi_right"]))


def _run_1d(wl, steps, precision, seed=0x5EED):
    cfg, tabs = W.to_device_config(wl, seed=seed, precision=precision)
    dev = apic.Simulation1D(cfg, tabs)
    load_device(dev, wl)
    dev.initialize()
    T = po.TableSet()
    ora = po.Sim1D(oracle_config(wl, T), 1, seed)
    load_oracle(ora, wl)
    ora.initialize()
    dev.step(steps)
    ora.step(steps)
    eps = W.EPS0 if wl.si else 1.0
    dx = wl.length / (wl.nx - 1 if wl.dirichlet else wl.nx)
    rho, phi, E = ora.fields()
    ref = sample_1d([(s.mass, s.weight) for s in wl.species], [ora.particles(s) for s in range(len(wl.species))],
                    rho, E, phi, eps, wl.dirichlet, dx)
    return dev, ref


@pytest.mark.parametrize("case", ["two_stream", "rf", "mcc"])
def test_sample_1d_fp64(case):
    if case == "two_stream":
        wl = W.two_stream(particles_per_beam=2048, nx=64, seed=3)
        steps = 25
    else:
        wl = W.ccp_helium(particles_per_cell=32, cells=64, seed=11, table_rows=1024)
        if case == "rf":
            wl.models = []
        steps = 20
    dev, ref = _run_1d(wl, steps, apic.FP64)
    s = dev.sample()
    assert s.step == steps
    _check_1d(s, ref, TOL)
    dev.close()


@pytest.mark.parametrize("case", ["two_stream", "rf"])
def test_sample_1d_fp32_form(case):
    if case == "two_stream":
        wl = W.two_stream(particles_per_beam=2048, nx=64, seed=3)
    else:
        wl = W.ccp_helium(particles_per_cell=32, cells=64, seed=11, table_rows=1024)
        wl.models = []
    dev, ref = _run_1d(wl, 10, apic.FP32)
    s = dev.sample()
    _check_1d(s, ref, FP32_TOL, exact_counts=(case == "two_stream"))
    dev.close()


def _run_nd(wl, steps, precision):
    cfg = W.to_device_config_nd(wl, sort_interval=4, precision=precision)
    dev = apic.SimulationND(cfg)
    eps = W.EPS0 if wl.si else 1.0
    ora = po.SimND(wl.dims, wl.n, wl.length, wl.dt, eps, wl.B, [(q, m, w) for (q, m, w, pos, v) in wl.species])
    for k, (q, m, w, pos, v) in enumerate(wl.species):
        dev.load(k, pos, v)
        ora.load(k, pos, v, v)
    dev.initialize()
    ora.initialize()
    dev.step(steps)
    ora.step(steps)
    vol = float(np.prod([L / n for L, n in zip(wl.length, wl.n)]))
    rho, phi, E = ora.fields()
    E = np.asarray(E).reshape(-1, int(np.prod(wl.n)))[: wl.dims]
    ref = sample_nd([(m, w) for (q, m, w, pos, v) in wl.species], [ora.particles(k) for k in range(len(wl.species))],
                    rho, E, eps, vol)
    return dev, ref


@pytest.mark.parametrize("dims", [2, 3])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_sample_nd(dims, precision):
    wl = W.plasma_2d(cells=(32, 16), ppc=8, seed=3) if dims == 2 else W.plasma_3d(cells=(16, 8, 8), ppc=4, seed=5)
    steps = 12
    dev, ref = _run_nd(wl, steps, apic.FP64 if precision == "fp64" else apic.FP32)
    s = dev.sample()
    tol = TOL if precision == "fp64" else FP32_TOL
    assert s.step == steps
    for k in ("kinetic_energy", "total_energy", "charge_l1"):
        assert abs(getattr(s, k) - ref[k]) <= tol * abs(ref[k]), (k, getattr(s, k), ref[k])
    # the field energy of a 1e-3 perturbation is a difference-sensitive quantity:
    # FP32 particle positions move it at the 1e-3 level
    fe_tol = tol if precision == "fp64" else 1e-2
    assert abs(s.field_energy - ref["field_energy"]) <= fe_tol * abs(ref["field_energy"]), \
        (s.field_energy, ref["field_energy"])
    for i, ke in enumerate(ref["kinetic_by_species"]):
        assert abs(s.kinetic_by_species[i] - ke) <= tol * abs(ke)
    assert s.live_particles == ref["live_particles"]
    dev.close()
