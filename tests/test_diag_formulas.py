"""The restated sample() sums (tests/diag_formulas.py) agree with the
reference's own Simulation::sample on a short run of the reference compiled
from its sources (the same library the golden vectors come from)."""
import tempfile

import numpy as np
import pytest

import pyoracle as po
from apic import workloads as W
from diag_formulas import sample_1d


@pytest.mark.parametrize("case", ["two_stream", "ccp"])
def test_sample_formulas_match_the_reference(case):
    if not po.reference_available():
        pytest.skip("reference library not built on this host")
    if case == "two_stream":
        wl = W.two_stream(particles_per_beam=256, nx=32, seed=3)
    else:
        wl = W.ccp_helium(particles_per_cell=8, cells=32, seed=11, table_rows=256)
    T = po.TableSet()
    cfg = po.config_from_workload(wl, T, seed=777)
    ref = po.Ref1D(cfg, tempfile.mkdtemp())
    ref.initialize()
    ref.step(7)
    ke, fe, live = ref.sample()
    parts = [ref.particles(s) for s in range(len(wl.species))]
    rho, phi, E = ref.fields()
    eps = W.EPS0 if wl.si else 1.0
    dx = wl.length / (wl.nx - 1 if wl.dirichlet else wl.nx)
    got = sample_1d([(s.mass, s.weight) for s in wl.species], parts, rho, E, phi, eps, wl.dirichlet, dx)
    for s in range(len(wl.species)):
        assert abs(got["kinetic_by_species"][s] - ke[s]) <= 1e-13 * abs(ke[s])
        assert got["live_by_species"][s] == live[s]
    assert abs(got["field_energy"] - fe) <= 1e-13 * abs(fe)
