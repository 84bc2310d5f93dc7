"""The device electron swarm (apic_swarm_run / the swarm server) against the
CPU oracle's device form (same Philox streams), the reference's own results
(golden vectors from run_swarm_benchmark), and itself alone versus batched."""
import os

import numpy as np
import pytest

import apic
import pyoracle as po
from apic import workloads as W
from common import ENSEMBLE_KEYS, SWARM_KEYS, swarm_cases, swarm_ensemble_cases

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# FP64 form against oracle mode 1: the same electrons, collisions and random
# streams; CUDA's log/sin/cos differ from glibc's by an ulp or two and the
# device sums in another order, so ensemble means agree to ~1e-13 and the
# block standard errors / displacement variances (differences of nearly equal
# numbers) to ~1e-10.
TOL_MEAN = 1e-10
TOL_SPREAD = 1e-7
MEANS = ("mean_velocity_x", "drift_velocity", "reduced_mobility", "mean_energy_ev", "final_weight",
         "ionization_rate", "attachment_rate", "net_rate", "growth_rate", "townsend_growth", "townsend_rate")
SPREADS = ("mean_velocity_x_se", "mean_energy_se_ev", "diffusion_longitudinal", "diffusion_transverse",
           "growth_rate_se", "ionization_rate_se")
COUNTS = ("candidates", "null_collisions", "final_particles")


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300) if b != 0 else abs(a)


def _device(spec, precision):
    cfg, gas, tabs = W.to_device_swarm(spec, precision)
    return apic.swarm_run(cfg, gas, spec.fields_td)


@pytest.mark.parametrize("name", ["swarm_fixed", "swarm_branching"])
def test_fp64_form_matches_oracle(name):
    spec = swarm_cases()[name]
    dev = _device(spec, apic.FP64)
    T = po.TableSet()
    cfg, gas = po.swarm_from_spec(spec, T)
    for k, td in enumerate(spec.fields_td):
        ora, _ = po.swarm_run_field(cfg, gas, td, spec.seed + k, 1)
        d = dev[k]
        assert d.status == 0, d.message
        assert d.steps_done == spec.steps
        for key in COUNTS:
            assert getattr(d, key) == getattr(ora, key), (name, td, key)
        assert list(d.channel_collisions)[: ora.nch] == list(ora.channel_collisions)[: ora.nch]
        assert d.max_observed_energy_ev == pytest.approx(ora.max_observed_energy_ev, rel=1e-12)
        for key in MEANS:
            assert rel(getattr(d, key), getattr(ora, key)) < TOL_MEAN, (name, td, key, getattr(d, key), getattr(ora, key))
        for key in SPREADS:
            assert rel(getattr(d, key), getattr(ora, key)) < TOL_SPREAD, (name, td, key, getattr(d, key), getattr(ora, key))


@pytest.mark.parametrize("name", ["swarm_fixed", "swarm_branching"])
def test_fp32_form_statistically_matches_fp64_form(name):
    """The FP32 form (float electron state, FP32 collision loops on their own
    uniforms) against the FP64 form over 12 seeds per field: ensemble means of
    drift velocity, mean energy and the ionization rate coefficient within 3
    combined standard errors, candidates within 3 standard errors."""
    spec = swarm_cases()[name]
    res = {}
    for prec in (apic.FP64, apic.FP32):
        cfg, gas, tabs = W.to_device_swarm(spec, prec)
        runs = []
        for k in range(12):
            cfg.seed = spec.seed + 1000 * k
            runs.append(apic.swarm_run(cfg, gas, spec.fields_td))
        res[prec] = runs
    for j, td in enumerate(spec.fields_td):
        for key in ("drift_velocity", "mean_energy_ev", "ionization_rate", "candidates"):
            a = np.array([float(getattr(r[j], key)) for r in res[apic.FP64]])
            b = np.array([float(getattr(r[j], key)) for r in res[apic.FP32]])
            assert all(r[j].status == 0 for r in res[apic.FP32])
            if np.all(a == 0) and np.all(b == 0):
                continue
            se = np.hypot(a.std(ddof=1), b.std(ddof=1)) / np.sqrt(len(a))
            assert abs(a.mean() - b.mean()) <= 3 * max(se, 1e-12 * abs(a.mean())), (name, td, key, a.mean(), b.mean(), se)


@pytest.mark.parametrize("name", ["ens_fixed", "ens_branching"])
def test_ensemble_statistically_consistent_with_reference(name):
    """Seed ensembles of device FP32 runs (Philox streams, batched on the
    server) against seed ensembles of the reference's own run_swarm_benchmark
    (mt19937_64): drift velocity, mean energy, ionization and attachment rate
    coefficients within 3 combined standard errors of the ensemble means."""
    f = np.load(os.path.join(G, f"swarm_ensemble_{name}.npz"))
    spec = swarm_ensemble_cases()[name]
    srv = _server(spec, max_runs=64, spl=60)
    ids = {}
    for k in range(16):
        for j, td in enumerate(spec.fields_td):
            ids[srv.submit(W.swarm_request(spec, td, seed=7000 + 31 * k))] = j
    res = _drain(srv, list(ids))
    srv.close()
    for j, td in enumerate(spec.fields_td):
        runs = [r for i, r in res.items() if ids[i] == j]
        assert all(r.status == 0 for r in runs)
        for key in ENSEMBLE_KEYS:
            dev = np.array([getattr(r, key) for r in runs])
            ref = f[key][:, j]
            if np.all(ref == 0) and np.all(dev == 0):
                continue
            s = np.hypot(dev.std(ddof=1) / np.sqrt(len(dev)), ref.std(ddof=1) / np.sqrt(len(ref)))
            assert abs(dev.mean() - ref.mean()) <= 3 * s, (name, td, key, dev.mean(), ref.mean(), s)


def _server(spec, budget=1 << 30, max_runs=16, precision=apic.FP32, spl=32):
    cfg, gas, tabs = W.to_device_swarm(spec, precision)
    srv = apic.SwarmServer(gas, budget, max_runs=max_runs, precision=precision, steps_per_launch=spl)
    srv._tabs = tabs
    return srv


def _drain(srv, ids):
    out = {}
    for _ in range(100000):
        active, queued = srv.advance()
        for i in ids:
            if i not in out:
                r = srv.poll(i)
                if r is not None:
                    out[i] = r
        if len(out) == len(ids):
            return out
        assert active or queued
    raise AssertionError("server did not finish")


def _result_tuple(r):
    keys = [k for k, _ in apic.SwarmResult._fields_ if k not in ("id", "latency_s", "queue_s", "message")]
    vals = []
    for k in keys:
        v = getattr(r, k)
        vals.append(tuple(v) if not isinstance(v, (int, float, bytes)) else v)
    return tuple(vals)


def test_result_identical_alone_and_in_the_mix():
    """Continuous batching: a request's result does not depend on what else
    shares the GPU (admission time, neighbours, chunk positions)."""
    spec = W.swarm_c5(particles=5000, steps=640, burn_in_steps=320)
    probe = W.swarm_request(spec, 200.0, particles=7000, seed=77)
    alone = _server(spec)
    a_id = alone.submit(probe)
    a = _drain(alone, [a_id])[a_id]
    h2d, d2h = alone.copy_bytes()
    alone.close()
    assert a.status == 0, a.message
    # the server's own traffic: at least the run's state record in, and the
    # sampled drift and energy series (steps after burn-in, 8 B each) out
    assert h2d > 0 and d2h >= 2 * (640 - 320) * 8
    mix = _server(spec, max_runs=4)
    ids = [mix.submit(W.swarm_request(spec, td, particles=n, seed=s))
           for td, n, s in ((30.0, 3000, 1), (500.0, 12000, 2), (80.0, 2500, 3))]
    mix.advance()
    mix.advance()
    p_id = mix.submit(probe)  # admitted later, next to runs already in flight
    ids += [p_id, mix.submit(W.swarm_request(spec, 900.0, particles=1500, seed=4))]
    res = _drain(mix, ids)
    mix.close()
    assert all(r.status == 0 for r in res.values())
    assert _result_tuple(res[p_id]) == _result_tuple(a)


def test_convergence_retires_runs_early_and_budget_admission():
    spec = W.swarm_c5(particles=4000, steps=20000, burn_in_steps=200)
    per_run = 4000 * 24 + 3 * (20000 - 200) * 8  # FP32 state + samples
    srv = _server(spec, budget=int(2.5 * per_run) + (1 << 20), max_runs=8, spl=64)
    ids = [srv.submit(W.swarm_request(spec, td, tolerance=0.02)) for td in (300.0, 500.0, 700.0, 900.0)]
    first = srv.advance()
    assert first[0] <= 8 and first[0] + first[1] == 4
    res = _drain(srv, ids)
    for r in res.values():
        assert r.status == 0 and r.converged == 1 and r.steps_done < 20000
        assert r.mean_energy_se_ev <= 0.02 * r.mean_energy_ev
    assert max(r.queue_s for r in res.values()) > 0.0


def test_run_errors_are_reported_per_run():
    spec = W.swarm_c5(particles=2000, steps=400, burn_in_steps=100, max_energy_ev=1000.0)
    srv = _server(spec)
    bad = W.swarm_request(spec, 1000.0)
    bad.max_energy_ev = 2.0  # electrons exceed it within a few steps
    good = W.swarm_request(spec, 100.0)
    ids = [srv.submit(bad), srv.submit(good)]
    res = _drain(srv, ids)
    assert res[ids[0]].status != 0 and b"max_energy_ev" in res[ids[0]].message
    assert res[ids[1]].status == 0
    with pytest.raises(apic.ApicError):
        srv.submit(W.swarm_request(spec, 100.0, particles=20_000_000))


def test_collide_henyey_greenstein_attachment_replay_against_reference():
    """NullCollisionModel::collide with Henyey-Greenstein elastic scattering,
    ionization and attachment on the device, fed the reference's own
    std::mt19937_64 draws: every count exact, velocities within 1e-12."""
    f = np.load(os.path.join(G, "collide3_hg.npz"))
    ch, mn = W.swarm_gas_anisotropic(attachment=True)
    tabs = apic.Tables()
    chans = [tabs.channel(c.process, c.energy, c.sigma, c.threshold, angular=c.angular, mu_energy=c.mu_energy, mu=c.mu)
             for c in ch]
    model = apic.mcc_model(0, chans, 1e24, float(f["nu"]), mn, 300.0, 1, 64)
    O = po.oracle()
    n = len(f["seeds"])
    draws = []
    for i in range(n):
        mt = (po.C.c_uint64 * 313)()
        O.ora_mt64_seed(po.C.byref(mt), po.C.c_uint64(int(f["seeds"][i])))
        draws.append(np.array([O.ora_mt64_next(po.C.byref(mt)) for _ in range(int(f["draws"][i]))], np.uint64))
    offsets = np.concatenate([[0], np.cumsum([len(d) for d in draws])]).astype(np.uint64)
    out_v, stats = apic.collide3(model, W.M_E, f["v_in"], float(f["dt"]), np.concatenate(draws), offsets)
    scale = np.max(np.abs(f["v_out"]))
    assert np.max(np.abs(out_v - f["v_out"])) < 1e-12 * scale
    for i in range(n):
        s = stats[i]
        assert s.candidates == f["candidates"][i]
        assert list(s.channel_collisions)[:4] == list(f["channels"][i])[:4]
        assert s.removed == f["removed"][i]
        assert (s.draws & 0x7FFFFFFF) == f["draws"][i]


def test_launch_complete_overlapping_1d_decks_keeps_results():
    """Launching the swarm batch, stepping 1D decks on their own streams, then
    completing the batch changes neither the swarm result nor the decks'."""
    spec = W.swarm_c5(particles=3000, steps=400, burn_in_steps=200)
    req = W.swarm_request(spec, 150.0, seed=5)
    alone = _server(spec, spl=40)
    a_id = alone.submit(req)
    a = _drain(alone, [a_id])[a_id]
    alone.close()
    wl = W.two_stream(particles_per_beam=4096, nx=128, seed=9)
    decks = []
    for k in range(2):
        cfg, tabs = W.to_device_config(wl, seed=3 + k)
        d = apic.Simulation1D(cfg, tabs)
        for i, sp in enumerate(wl.species):
            d.load(i, sp.x, sp.v)
        d.initialize()
        decks.append((d, tabs))
    ref = apic.Simulation1D(*W.to_device_config(wl, seed=3))
    for i, sp in enumerate(wl.species):
        ref.load(i, sp.x, sp.v)
    ref.initialize()
    mix = _server(spec, spl=40)
    m_id = mix.submit(req)
    done, steps = None, 0
    while done is None:
        mix.launch()
        apic.step_group([d for d, _ in decks], 10)
        steps += 10
        mix.complete()
        done = mix.poll(m_id)
    mix.close()
    assert _result_tuple(done) == _result_tuple(a)
    ref.step(steps)
    for k in range(2):
        x, y = decks[0][0].particles(k), ref.particles(k)
        for key in x:
            assert np.array_equal(x[key], y[key])


def test_spatial_townsend_matches_oracle_device_form():
    """run_spatial_townsend on the device against oracle mode 1 (the same
    per-history Philox streams): per-history net crossings, the flux profile
    and the fitted coefficient, over two fields sharing one work-item scan."""
    from golden.make_golden import townsend_deck
    spec, osp = townsend_deck()
    T = po.TableSet()
    ocfg, ogas = po.swarm_from_spec(spec, T)
    cfg, gas, _tabs = W.to_device_swarm(spec)
    sp = apic.SpatialTownsendConfig(osp.histories, osp.length_m, osp.bins, osp.fit_begin_bin, osp.fit_end_bin,
                                    osp.max_steps, osp.work_item_limit, osp.min_r_squared)
    scan_d = scan_o = 0
    for k, td in enumerate(spec.fields_td):
        d, dprof, dcross, scan_d = apic.swarm_spatial_townsend(cfg, sp, gas, td, spec.seed + k, scan_d, True)
        o, oprof, ocross, scan_o = po.swarm_spatial_townsend(ocfg, osp, ogas, td, spec.seed + k, 1, scan_o)
        assert (d.histories_completed, d.maximum_active_particles, d.particle_updates) == \
            (o.histories_completed, o.maximum_active_particles, o.particle_updates)
        assert np.max(np.abs(dcross - ocross)) <= 1e-12 * np.max(np.abs(ocross))
        assert np.max(np.abs(dprof - oprof)) <= 1e-12 * np.max(np.abs(oprof))
        assert abs(d.townsend_1_m - o.townsend_1_m) <= 1e-10 * abs(o.townsend_1_m)
        assert abs(d.townsend_standard_error_1_m - o.townsend_se_1_m) <= 1e-8 * o.townsend_se_1_m
    assert scan_d == scan_o


def test_spatial_townsend_errors_match_reference_messages():
    from golden.make_golden import townsend_deck
    spec, osp = townsend_deck()
    cfg, gas, _tabs = W.to_device_swarm(spec)
    sp = apic.SpatialTownsendConfig(osp.histories, osp.length_m, osp.bins, osp.fit_begin_bin, osp.fit_end_bin,
                                    osp.max_steps, osp.work_item_limit, osp.min_r_squared)
    bad = apic.SpatialTownsendConfig(sp.histories, sp.length_m, 3, 0, 0, sp.max_steps, 0, 0.0)
    with pytest.raises(apic.ApicError, match="spatial_bins must be at least 4"):
        apic.swarm_spatial_townsend(cfg, bad, gas, 600.0, 1)
    short = apic.SpatialTownsendConfig(sp.histories, sp.length_m, sp.bins, 1, 0, 20, 0, 0.0)
    with pytest.raises(apic.ApicError, match="did not terminate within spatial_max_steps"):
        apic.swarm_spatial_townsend(cfg, short, gas, 600.0, 1)
    tiny = apic.SpatialTownsendConfig(sp.histories, sp.length_m, sp.bins, 1, 0, sp.max_steps, 1000, 0.0)
    with pytest.raises(apic.ApicError, match="exceeded spatial_work_item_limit"):
        apic.swarm_spatial_townsend(cfg, tiny, gas, 600.0, 1)
