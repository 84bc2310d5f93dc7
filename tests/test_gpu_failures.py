"""Failure detection of the 1D step, injected from the host: inputs that make
the reference throw (src/Collision.cpp:620-623, :680-684, :910-916, :938-943,
src/Simulation.cpp:941-964) set the device error word, which the next
synchronising call returns as the matching status with the reference's
message.  Nothing here traps, faults or spins on the device: the kernels flag
and drop the offending particle or product, and the host's wait on the
stream is bounded."""
import numpy as np
import pytest

import apic
from apic import workloads as W
from common import load_device

pytestmark = pytest.mark.gpu

ERR_CAPACITY, ERR_MAJORANT, ERR_CANDIDATES, ERR_NONFINITE, ERR_TIMEOUT = 3, 4, 5, 6, 7


def _deck(te_ev=1.0):
    return W.ccp_helium(particles_per_cell=32, cells=64, seed=11, table_rows=1024, te_ev=te_ev)


def _run(wl, steps, precision=apic.FP64):
    cfg, tabs = W.to_device_config(wl, seed=99, precision=precision)
    dev = apic.Simulation1D(cfg, tabs)
    load_device(dev, wl)
    dev.initialize()
    dev.step(steps)
    with pytest.raises(apic.ApicError) as e:
        dev.synchronize()
    return dev, e.value


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_max_frequency_below_the_rate_bound(precision):
    wl = _deck(te_ev=20.0)
    wl.models[0].max_frequency *= 0.02  # far below the electrons' total collision rate
    dev, err = _run(wl, 3, apic.FP64 if precision == "fp64" else apic.FP32)
    assert err.status == ERR_MAJORANT, err
    assert "exceeds configured max_frequency" in str(err)
    dev.close()


def test_candidate_limit():
    wl = _deck()
    m = wl.models[1]  # ions in a gas 200x denser: many candidates per particle per step
    m.neutral_density *= 200.0
    m.max_frequency *= 200.0
    m.max_candidates = 1
    dev, err = _run(wl, 2)
    assert err.status == ERR_CANDIDATES, err
    assert "candidate limit" in str(err)
    dev.close()


def test_capacity_too_small_for_ionization_products():
    wl = _deck(te_ev=40.0)
    for s in wl.species:
        s.capacity = len(s.x)  # no room for a single product
    dev, err = _run(wl, 20)
    assert err.status == ERR_CAPACITY, err
    assert "max_particles_per_species" in str(err)
    dev.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_non_finite_velocity_loaded_from_the_host(precision):
    wl = _deck()
    wl.species[0].v[17] = np.nan
    dev, err = _run(wl, 2, apic.FP64 if precision == "fp64" else apic.FP32)
    assert err.status == ERR_NONFINITE, err
    assert "non-finite" in str(err)
    dev.close()


def test_bounded_wait_gives_up_and_a_later_wait_completes():
    """A wait limit far below the time of the enqueued steps ends the
    synchronising call with APIC_ERR_TIMEOUT; the work itself runs on, and a
    synchronise with a normal limit then succeeds with the run intact."""
    wl = W.ccp_helium(particles_per_cell=256, cells=256, seed=5, table_rows=1024)
    cfg, tabs = W.to_device_config(wl, seed=3)
    dev = apic.Simulation1D(cfg, tabs)
    load_device(dev, wl)
    dev.initialize()
    dev.synchronize()
    dev.set_wait_limit(1e-5)
    dev.step(400)
    with pytest.raises(apic.ApicError) as e:
        dev.synchronize()
    assert e.value.status == ERR_TIMEOUT
    dev.set_wait_limit(120.0)
    dev.synchronize()
    assert dev.sample().step == 400
    dev.close()
