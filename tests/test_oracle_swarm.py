"""The CPU oracle's electron swarm (run_field, systematic_resample,
block_mean_and_error) and Henyey-Greenstein scattering against golden
vectors that the reference's own run_swarm_benchmark and
NullCollisionModel::collide produced (tests/golden/make_golden.py)."""
import ctypes as C
import os

import numpy as np
import pytest

import pyoracle as po
from apic import workloads as W
from common import SWARM_KEYS, swarm_cases

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(G, name))


def _hg_model(T):
    ch, mn = W.swarm_gas_anisotropic(attachment=True)
    chans = [T.channel(c.process, c.energy, c.sigma, c.threshold, 0 if c.process == W.IONIZATION else -1,
                       1 if c.process == W.IONIZATION else -1, angular=c.angular, mu_energy=c.mu_energy, mu=c.mu)
             for c in ch]
    nu = W.swarm_max_frequency(ch, 1e24, mn, 300.0, 200.0)
    return po.make_model(0, chans, 1e24, nu, mn, 300.0, 1, 64)


def test_collide3_henyey_greenstein_attachment_bit_exact():
    f = load("collide3_hg.npz")
    T = po.TableSet()
    m = _hg_model(T)
    assert m.max_frequency == float(f["nu"])
    O = po.oracle()
    col = (C.c_byte * 8192)()
    assert O.ora_collider_init(col, C.byref(m), W.M_E) == 0
    dt = float(f["dt"])
    for i in range(len(f["seeds"])):
        mt = (C.c_uint64 * 313)()
        O.ora_mt64_seed(C.byref(mt), C.c_uint64(int(f["seeds"][i])))
        r = po.Rng()
        r.kind = 0
        r.mt = C.cast(C.byref(mt), C.c_void_p)
        st = po.CollideStats()
        v = np.ascontiguousarray(f["v_in"][i].copy())
        assert O.ora_collide3(col, po.dptr(v), dt, C.byref(r), C.byref(st)) == 0
        assert np.array_equal(v, f["v_out"][i]), i
        assert st.candidates == f["candidates"][i]
        assert list(st.channel_collisions) == list(f["channels"][i])
        assert st.nsecondaries == f["nsec"][i] and st.removed == f["removed"][i]
        assert st.draws == f["draws"][i]
        for k in range(min(st.nsecondaries, 4)):
            assert np.array_equal(np.array(st.secondary_velocity[k]), f["sec_v"][i][k])
    ch = f["channels"].sum(axis=0)
    assert ch[0] > 100 and ch[2] > 0 and ch[3] > 0  # elastic, ionization and attachment all exercised


@pytest.mark.parametrize("name", ["swarm_fixed", "swarm_branching"])
def test_swarm_run_field_bit_exact(name):
    f = load(f"{name}.npz")
    spec = swarm_cases()[name]
    T = po.TableSet()
    cfg, gas = po.swarm_from_spec(spec, T)
    for k, td in enumerate(spec.fields_td):
        res, _ = po.swarm_run_field(cfg, gas, td, spec.seed + k, 0)
        for key in SWARM_KEYS:
            assert getattr(res, key) == f[key][k], (name, td, key, getattr(res, key), f[key][k])
        assert list(res.channel_collisions)[: res.nch] == list(f["channel_collisions"][k])
        assert list(res.channel_rate)[: res.nch] == list(f["channel_rate"][k])


def test_block_statistics():
    x = np.arange(1.0, 11.0)
    m, e = po.block_mean_and_error(x, 5)  # block means 1.5, 3.5, ..., 9.5
    assert m == 5.5
    assert abs(e - np.sqrt(np.sum((np.arange(1.5, 10, 2) - 5.5) ** 2) / 20)) < 1e-15
    with pytest.raises(ValueError):
        po.block_mean_and_error(x, 11)


@pytest.mark.parametrize("branching", [False, True])
def test_device_forms_agree_with_reference_form(branching):
    """Modes 1 (device FP64 form: Philox streams, displacement tallies, index
    resampling) and 2 (FP32 storage) against mode 0 (the reference's form):
    different random streams, so drift velocity and mean energy must agree
    within 4 combined standard errors."""
    spec = swarm_cases()["swarm_branching"]  # relaxes within the burn-in
    spec.branching = branching
    if not branching:  # fixed population: no attachment (src/Swarm.cpp:505-511)
        spec.channels = [c for c in spec.channels if c.process != W.ATTACHMENT]
    spec.particles, spec.steps, spec.burn_in_steps = 1000, 800, 300
    spec.max_energy_ev = 199.0  # room for the 400 Td tail within the 200 eV tables
    spec.max_frequency = W.swarm_max_frequency(spec.channels, spec.neutral_density, spec.neutral_mass,
                                               spec.neutral_temperature, 199.0)
    spec.timestep = 0.08 / spec.max_frequency
    T = po.TableSet()
    cfg, gas = po.swarm_from_spec(spec, T)
    for k, td in enumerate(spec.fields_td):
        ref, _ = po.swarm_run_field(cfg, gas, td, spec.seed + k, 0)
        for mode in (1, 2):
            got, _ = po.swarm_run_field(cfg, gas, td, spec.seed + k, mode)
            for key, se in (("mean_velocity_x", "mean_velocity_x_se"), ("mean_energy_ev", "mean_energy_se_ev")):
                a, b = getattr(got, key), getattr(ref, key)
                s = np.hypot(getattr(got, se), getattr(ref, se))
                assert abs(a - b) <= 4 * s + 1e-12 * abs(b), (branching, td, mode, key, a, b, s)


def test_fp32_storage_tracks_fp64_form():
    """Same Philox streams: mode 2 differs from mode 1 only by FP32 rounding
    of the stored state, which moves the ensemble averages by ~1e-6."""
    spec = swarm_cases()["swarm_fixed"]
    T = po.TableSet()
    cfg, gas = po.swarm_from_spec(spec, T)
    a, sa = po.swarm_run_field(cfg, gas, 300.0, 7, 1, samples=True)
    b, sb = po.swarm_run_field(cfg, gas, 300.0, 7, 2, samples=True)
    assert abs(a.mean_energy_ev - b.mean_energy_ev) < 1e-4 * a.mean_energy_ev
    assert abs(a.mean_velocity_x - b.mean_velocity_x) < 1e-3 * abs(a.mean_velocity_x)


def test_spatial_townsend_bit_exact_against_reference():
    """run_spatial_townsend (src/Swarm.cpp:645-938): oracle mode 0 against the
    reference's own run_swarm_benchmark over two fields (seed + f, one
    particle-update scan across the fields): result fields and the flux
    profile bit for bit (tests/golden/swarm_townsend.npz)."""
    import os
    from golden.make_golden import townsend_deck
    f = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "swarm_townsend.npz"))
    spec, sp = townsend_deck()
    T = po.TableSet()
    cfg, gas = po.swarm_from_spec(spec, T)
    scan = 0
    for k, td in enumerate(spec.fields_td):
        r, prof, _, scan = po.swarm_spatial_townsend(cfg, sp, gas, td, spec.seed + k, 0, scan)
        assert np.array_equal(np.array([r.townsend_1_m, r.townsend_se_1_m, r.fit_r_squared]), f[f"f{k}_scalars"])
        assert [r.histories_completed, r.maximum_active_particles, r.particle_updates] == list(f[f"f{k}_counts"])
        assert np.array_equal(prof, f[f"f{k}_profile"])
    assert scan == int(f["f0_counts"][2] + f["f1_counts"][2])


def test_spatial_townsend_device_form_is_consistent():
    """Mode 1 (the device form, per-history Philox streams) estimates the same
    Townsend coefficient within the combined standard errors."""
    from golden.make_golden import townsend_deck
    spec, sp = townsend_deck()
    T = po.TableSet()
    cfg, gas = po.swarm_from_spec(spec, T)
    for k, td in enumerate(spec.fields_td):
        a = po.swarm_spatial_townsend(cfg, sp, gas, td, spec.seed + k, 0)[0]
        b = po.swarm_spatial_townsend(cfg, sp, gas, td, spec.seed + k, 1)[0]
        assert abs(a.townsend_1_m - b.townsend_1_m) < 3.0 * np.hypot(a.townsend_se_1_m, b.townsend_se_1_m)
