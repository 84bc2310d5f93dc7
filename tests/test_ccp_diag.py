"""CCP campaign-diagnostics settings on the CPU: the device library's
validation (apic_spatial_average1d_validate, no device needed) raises the
reference's messages (validate_spatial_average_1d, src/Config.cpp:1377-1524),
checked against the reference itself where it is built."""
import tempfile

import pytest

import apic
import pyoracle as po
from apic import workloads as W

F = 13.56e6
EEDF = dict(eedf_species=0, eedf_bins=32, eedf_energy_max=50.0, eedf_regions=((0.0, 0.02),))
RF = dict(interval=4, start_step=1, end_step=400, rf_frequency=F, rf_cycles=1, phase_bins=4)

CASES = [
    (dict(RF), None),
    (dict(RF, **EEDF), None),
    (dict(interval=5, start_step=3, end_step=37), None),
    (dict(interval=0, start_step=1, end_step=5), "spatial_average_interval must be positive"),
    (dict(interval=1, start_step=0, end_step=5), "spatial_average requires 1 <= start_step <= end_step"),
    (dict(interval=1, start_step=6, end_step=5), "spatial_average requires 1 <= start_step <= end_step"),
    (dict(interval=1, start_step=1, end_step=5, phase_bins=2),
     "spatial_average_rf_cycles requires positive spatial_average_rf_frequency"),
    (dict(RF, rf_frequency=-1.0), "spatial_average_rf_frequency must be non-negative and finite"),
    (dict(RF, rf_cycles=0), "positive spatial_average_rf_frequency requires positive spatial_average_rf_cycles"),
    (dict(RF, rf_frequency=F * 1.1), "spatial-average RF period must contain an integer number of timesteps"),
    (dict(RF, end_step=399), "spatial-average step window does not span the configured whole RF cycles"),
    (dict(RF, start_step=2, end_step=401), "spatial-average RF window must end at the time-zero drive phase"),
    (dict(RF, interval=3, phase_bins=0), "spatial_average_interval must divide RF steps per cycle"),
    (dict(RF, phase_bins=3), "spatial_average_phase_bins must divide the sampled RF cycle"),
    (dict(RF, rf_frequency=2 * F, end_step=200, phase_bins=2), "spatial-average RF frequency does not match the electrode drive"),
    (dict(RF, phase_bins=0, **EEDF), "phase_eedf requires spatial averaging with phase bins"),
    (dict(RF, **dict(EEDF, eedf_bins=0)),
     "phase_eedf requires a species, 1..1000000 bins, a positive energy maximum, and at least one region"),
    (dict(RF, **dict(EEDF, eedf_energy_max=0.0)),
     "phase_eedf requires a species, 1..1000000 bins, a positive energy maximum, and at least one region"),
    (dict(RF, **dict(EEDF, eedf_regions=((0.01, 0.5),))),
     "phase_eedf regions require unique safe names and 0 <= x_min < x_max <= length"),
    (dict(RF, **dict(EEDF, eedf_regions=((0.03, 0.02),))),
     "phase_eedf regions require unique safe names and 0 <= x_min < x_max <= length"),
    (dict(RF, eedf_bins=4), "disabled phase_eedf cannot configure species, bins, energy maximum, or regions"),
]


def _deck():
    return W.ccp_helium(particles_per_cell=8, cells=32, seed=5, steps=10, table_rows=96)


@pytest.mark.parametrize("kw,message", CASES)
def test_validation_messages_match_the_reference(kw, message):
    wl = _deck()
    cfg, _tabs = W.to_device_config(wl)
    try:
        apic.validate_spatial_average(cfg, apic.spatial_average1d(**kw))
        got = None
    except apic.ApicError as e:
        got = str(e.args[1] if len(e.args) > 1 else e)
    assert (got is None) == (message is None), got
    if message is not None:
        assert message in got, got
    if po.reference_available():
        T = po.TableSet()
        ocfg = po.config_from_workload(wl, T, seed=2024)
        ref = po.ref_validate_spatial_average(ocfg, po.spatial_average1d(**kw), tempfile.mkdtemp())
        assert (ref is None) == (message is None), ref
        if message is not None:
            assert ref == message, ref
