"""CCP campaign diagnostics on the device (spatial average, RF phase bins,
spatial collision energy, phase EEDF; src/Simulation.cpp:1163-1370) and the
electric-work ledger (src/Simulation.cpp:1047-1056, :1094-1132) against
the oracle, whose restatement is pinned bit for bit to the reference's own
accumulators and CSV output (tests/test_oracle_golden.py).

FP64 form: sample counts and EEDF observation counts exact; every per-node sum
within 1e-12 of the oracle relative to the largest magnitude of its row (the
device adds with FP64 atomics, so only the order of the additions differs).
FP32 storage form: against oracle mode 2 within the FP32 form's bounds."""
import numpy as np
import pytest

import apic
import pyoracle as po
from apic import workloads as W
from common import load_device, load_oracle, oracle_config, rel_max

pytestmark = pytest.mark.gpu

F = 13.56e6
EEDF = dict(eedf_species=0, eedf_bins=48, eedf_energy_max=60.0,
            eedf_regions=((0.0, 0.02), (0.02, 0.067), (0.03, 0.04)))
# the discharge driven at 10 F: one RF cycle is 40 steps, short enough that
# the device and oracle trajectories stay within 1e-12 of each other
SHORT = dict(interval=2, start_step=1, end_step=40, rf_frequency=10 * F, rf_cycles=1, phase_bins=4, **EEDF)
# the 13.56 MHz discharge over one cycle (400 steps)
RF = dict(interval=4, start_step=1, end_step=400, rf_frequency=F, rf_cycles=1, phase_bins=4, **EEDF)
WINDOW = dict(interval=5, start_step=3, end_step=37)
TOL = 1e-12
# over 400 steps the device and oracle trajectories drift apart (the field
# solves round differently and a plasma amplifies differences); the sums then
# agree to this bound
LONG_TOL = 1e-9


def _deck(frequency=F):
    wl = W.ccp_helium(particles_per_cell=16, cells=64, seed=11, steps=400, table_rows=256, te_ev=12.0)
    wl.drive_right = (450.0, frequency, 0.0)
    return wl


def _device(wl, kw, precision=apic.FP64, seed=0x5EED, ledger=False):
    cfg, tabs = W.to_device_config(wl, precision=precision, seed=seed)
    dev = apic.Simulation1D(cfg, tabs)
    load_device(dev, wl)
    if kw is not None:
        dev.enable_spatial_average(apic.spatial_average1d(**kw))
    if ledger:
        dev.enable_power_transfer()
    dev.initialize()
    return dev, tabs


def _oracle(wl, kw, mode, seed=0x5EED):
    T = po.TableSet()
    ora = po.Sim1D(oracle_config(wl, T), mode, seed)
    load_oracle(ora, wl)
    if kw is not None:
        ora.enable_spatial_average(po.spatial_average1d(**kw))
    ora.initialize()
    return ora, T


def _check_work(dev, ora, nspecies, tol):
    for s in range(nspecies):
        w, wo = dev.electric_work(s), ora.electric_work(s)
        assert abs(w - wo) <= tol * (abs(wo) + ora.kinetic(s)), (s, w, wo)
        assert wo != 0.0


def _compare(dev, ora, kw, nspecies, nch, tol, count_tol=0.0):
    P = kw.get("phase_bins", 0)
    a, b = dev.spatial_counts(), ora.spatial_counts()
    assert a[0] == b[0] and a[1] == b[1], (a, b)
    assert np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3])
    assert a[0] > 0
    for phase in [-1] + list(range(P)):
        for q in range(5):
            for s in range(nspecies):
                x, y = dev.spatial_sums(q, s, phase), ora.spatial_sums(q, s, phase)
                assert rel_max(x, y) < tol, (phase, q, s, rel_max(x, y))
        for q in (apic.SA_POTENTIAL, apic.SA_ELECTRIC, apic.SA_ELECTRIC_SQUARED):
            x, y = dev.spatial_sums(q, 0, phase), ora.spatial_sums(q, 0, phase)
            assert rel_max(x, y) < tol, (phase, q, rel_max(x, y))
        for c in range(nch):
            x, y = dev.spatial_sums(apic.SA_COLLISION_ENERGY, c, phase), ora.spatial_sums(po.SA_COLLISION, c, phase)
            assert rel_max(x, y) < tol, (phase, c, rel_max(x, y))
    if kw.get("eedf_species", -1) >= 0:
        for p in range(P):
            for r in range(len(kw["eedf_regions"])):
                (c1, s1, h1), (c2, s2, h2) = dev.phase_eedf(p, r), ora.phase_eedf(p, r)
                assert np.all(np.abs(c1.astype(np.int64) - c2.astype(np.int64)) <= count_tol * c2), (p, r, c1, c2)
                assert c2[0] > 0
                for k in range(7):
                    assert abs(s1[k] - s2[k]) <= tol * max(abs(s2[k]), abs(s2[0])), (p, r, k, s1[k], s2[k])
                assert rel_max(h1, h2) < tol, (p, r)


def test_rf_phase_bins_and_eedf_match_oracle_fp64():
    """One RF cycle (40 steps) sampled every 2 steps into 4 phase bins with a
    3-region EEDF; the state is read part way through (the read applies the
    pending collision part once, as a sample does) and the run goes on."""
    wl = _deck(10 * F)
    dev, _t1 = _device(wl, SHORT)
    ora, _t2 = _oracle(wl, SHORT, 1)
    dev.step(23)
    ora.step(23)
    assert dev.spatial_counts()[:2] == ora.spatial_counts()[:2]
    dev.step(17)
    ora.step(17)
    nch = sum(len(m.channels) for m in wl.models)
    _compare(dev, ora, SHORT, 2, nch, TOL)
    assert np.any(dev.spatial_sums(apic.SA_COLLISION_ENERGY, 2) != 0.0)  # ionization deposits


def test_bgk_collision_energy_and_ledger_match_oracle_fp64():
    """The legacy BGK model (src/Simulation.cpp:772-834) deposits each
    relaxation's energy change in its one "bgk" channel; with the phase bins,
    EEDF and the electric-work ledger over one 40-step RF cycle everything
    agrees with the oracle as for MCC."""
    wl = W.ccp_helium(particles_per_cell=16, cells=64, seed=11, steps=40, table_rows=64, te_ev=4.0,
                      bgk=(2.0e8, 3.0e5))
    wl.drive_right = (450.0, 10 * F, 0.0)
    dev, _t1 = _device(wl, SHORT, ledger=True)
    ora, _t2 = _oracle(wl, SHORT, 1)
    dev.step(40)
    ora.step(40)
    _compare(dev, ora, SHORT, 2, 1, TOL)
    _check_work(dev, ora, 2, TOL)
    assert np.any(dev.spatial_sums(apic.SA_COLLISION_ENERGY, 0) != 0.0)


def test_long_rf_cycle_fp64_and_unperturbed_trajectory():
    """The 13.56 MHz discharge over a whole cycle (400 steps, 100 samples):
    counts exact, sums within the long-run bound; and the diagnostics leave
    the FP64 trajectory bit for bit as a run without them."""
    wl = _deck()
    dev, _t1 = _device(wl, RF)
    ora, _t2 = _oracle(wl, RF, 1)
    dev.step(400)
    ora.step(400)
    nch = sum(len(m.channels) for m in wl.models)
    _compare(dev, ora, RF, 2, nch, LONG_TOL, count_tol=0.01)
    plain, _t3 = _device(wl, None)
    plain.step(400)
    for s in range(2):
        a, b = dev.particles(s), plain.particles(s)
        for k in a:
            assert np.array_equal(a[k], b[k]), (s, k)
    ta, tb = dev.collision_totals(), plain.collision_totals()
    assert ta.candidates == tb.candidates


def test_window_without_rf_contract_through_step_group():
    wl = _deck()
    dev, _t1 = _device(wl, WINDOW)
    ora, _t2 = _oracle(wl, WINDOW, 1)
    apic.step_group([dev], 40)
    ora.step(40)
    nch = sum(len(m.channels) for m in wl.models)
    _compare(dev, ora, WINDOW, 2, nch, TOL)
    samples, csteps, _, _ = dev.spatial_counts()
    assert samples == len(range(3, 38, 5)) and csteps == 35


def test_fp32_form_matches_oracle_mode2():
    """The FP32 storage form: every sample stores the state as the read-back
    does; against oracle mode 2 the sums agree within the FP32 form's bounds."""
    wl = _deck(10 * F)
    dev, _t1 = _device(wl, SHORT, precision=apic.FP32_STORAGE)
    ora, _t2 = _oracle(wl, SHORT, 2)
    dev.step(40)
    ora.step(40)
    nch = sum(len(m.channels) for m in wl.models)
    _compare(dev, ora, SHORT, 2, nch, 1e-5, count_tol=0.01)


def test_electric_work_ledger_with_walls_and_products_fp64():
    """The work of every synchronisation and wall crossing (products pushed
    in the post kernel included), read part way through and at the end; the
    ledger leaves the FP64 trajectory bit for bit as a run without it."""
    wl = _deck(10 * F)
    dev, _t1 = _device(wl, None, ledger=True)
    ora, _t2 = _oracle(wl, None, 1)
    dev.step(17)
    ora.step(17)
    _check_work(dev, ora, 2, TOL)
    dev.step(23)
    ora.step(23)
    _check_work(dev, ora, 2, TOL)
    assert dev.boundary_losses(0).absorbed_left + dev.boundary_losses(0).absorbed_right > 0
    plain, _t3 = _device(wl, None)
    plain.step(40)
    for s in range(2):
        a, b = dev.particles(s), plain.particles(s)
        for k in a:
            assert np.array_equal(a[k], b[k]), (s, k)


def test_electric_work_ledger_two_stream_graphs_and_fp32():
    """Periodic two-stream deck stepped through step_group (the graph path),
    FP64 against oracle mode 1; the FP32 storage form against oracle mode 2."""
    wl = W.two_stream(particles_per_beam=512, nx=64, seed=3, steps=50)
    dev, _t1 = _device(wl, None, ledger=True)
    ora, _t2 = _oracle(wl, None, 1)
    apic.step_group([dev], 50)
    ora.step(50)
    _check_work(dev, ora, 2, TOL)
    dev32, _t3 = _device(wl, None, precision=apic.FP32_STORAGE, ledger=True)
    ora2, _t4 = _oracle(wl, None, 2)
    dev32.step(50)
    ora2.step(50)
    _check_work(dev32, ora2, 2, 1e-5)


def test_ledger_and_spatial_average_together():
    wl = _deck(10 * F)
    dev, _t1 = _device(wl, SHORT, ledger=True)
    ora, _t2 = _oracle(wl, SHORT, 1)
    dev.step(40)
    ora.step(40)
    _check_work(dev, ora, 2, TOL)
    nch = sum(len(m.channels) for m in wl.models)
    _compare(dev, ora, SHORT, 2, nch, TOL)


def test_enable_after_initialize_is_refused():
    wl = _deck()
    dev, _t = _device(wl, None)
    with pytest.raises(apic.ApicError, match="before initialize"):
        dev.enable_spatial_average(apic.spatial_average1d(**WINDOW))
    with pytest.raises(apic.ApicError, match="before initialize"):
        dev.enable_power_transfer()
    with pytest.raises(apic.ApicError, match="not enabled"):
        dev.electric_work(0)
