"""Parity of the device 1D particle step against the CPU oracle, through the
C ABI.  FP64 form: tolerance 1e-12 relative (max-norm) for fields and particle
state; exact for counts and collision decisions."""
import numpy as np
import pytest

import apic
import pyoracle as po
from apic import workloads as W
from common import load_device, load_oracle, oracle_config, rel_max

pytestmark = pytest.mark.gpu
TOL = 1e-12


def small_two_stream():
    return W.two_stream(particles_per_beam=512, nx=64, seed=3, steps=50)


def small_ccp(ppc=16, cells=64):
    return W.ccp_helium(particles_per_cell=ppc, cells=cells, seed=11, steps=20, table_rows=1024)


@pytest.mark.parametrize("boundary", [apic.PERIODIC, apic.DIRICHLET])
def test_deposit_solve_gather(boundary):
    rng = np.random.default_rng(5)
    nx, L = 97, 3.7
    xs = [rng.uniform(0, L, 5000), rng.uniform(0, L, 3000)]
    xs[0][:3] = [0.0, L, L * (1 - 1e-17)]
    q, w = [-1.0, 1.0], [0.013, 0.02]
    xq = rng.uniform(-0.5, L + 0.5, 777)
    rho, phi, E, eq = apic.deposit_solve_gather_1d(boundary, nx, L, 1.3, 0.4, -2.0, q, w, xs, xq)
    dir_ = int(boundary == apic.DIRICHLET)
    dx = L / (nx - 1 if dir_ else nx)
    O = po.oracle()
    rr = np.zeros(nx)
    for s in range(2):
        x = np.ascontiguousarray(xs[s])
        O.ora_deposit1d(po.dptr(rr), nx, L, dx, dir_, q[s], w[s], len(x), po.dptr(x), None)
    assert rel_max(rho, rr) < TOL
    pr, er = np.zeros(nx), np.zeros(nx)
    r2 = rr.copy()
    O.ora_solve1d(po.dptr(r2), po.dptr(pr), po.dptr(er), nx, L, dx, dir_, 1.3, 0.4, -2.0)
    assert rel_max(phi, pr) < TOL
    assert rel_max(E, er) < TOL
    eo = np.array([O.ora_gather1d(po.dptr(E), nx, L, dx, dir_, x) for x in xq])
    assert rel_max(eq, eo) < TOL


def _oracle_collider(wl, model_index, tables):
    cfg = oracle_config(wl, tables)
    col = (po.C.c_byte * 8192)()
    m = cfg.models[model_index]
    O = po.oracle()
    assert O.ora_collider_init(col, po.C.byref(m), wl.species[m.species].mass) == 0
    return col, m


@pytest.mark.parametrize("model_index", [0, 1])
@pytest.mark.parametrize("source", ["replay", "philox"])
def test_collide3(model_index, source):
    wl = small_ccp()
    tables = po.TableSet()
    col, om = _oracle_collider(wl, model_index, tables)
    sp = wl.species[om.species]
    rng = np.random.default_rng(9)
    n = 4000
    # fast particles so that collisions, ionization and the threshold paths all occur
    scale = 5e6 if model_index == 0 else 6e4
    v3 = rng.standard_normal((n, 3)) * scale
    dt = wl.dt * 40  # several candidates per particle
    O = po.oracle()
    draws_per = 4096
    seeds = rng.integers(1, 2 ** 63, n, dtype=np.uint64)
    ref_v = v3.copy()
    ref_stats = []
    all_draws = []
    for i in range(n):
        r = po.Rng()
        if source == "replay":
            mt = (po.C.c_uint64 * 313)()
            O.ora_mt64_seed(po.C.byref(mt), po.C.c_uint64(int(seeds[i])))
            raw = np.array([O.ora_mt64_next(po.C.byref(mt)) for _ in range(draws_per)], dtype=np.uint64)
            all_draws.append(raw)
            r.kind = po.ORA_SRC_ARRAY if hasattr(po, "ORA_SRC_ARRAY") else 2
            r.array = raw.ctypes.data_as(po.C.POINTER(po.C.c_uint64))
            r.array_len = draws_per
        else:
            r.kind = 1
            r.key[0], r.key[1] = 0x1234567, 0x89ABCDE
            r.ctr[0], r.ctr[1], r.ctr[2] = i, 17, 3
        st = po.CollideStats()
        vv = np.ascontiguousarray(ref_v[i])
        rc = O.ora_collide3(col, po.dptr(vv), dt, po.C.byref(r), po.C.byref(st))
        assert rc == 0, po.oracle().ora_last_error()
        ref_v[i] = vv
        ref_stats.append(st)
    dm = apic.mcc_model(0, [apic.McChannel(*[getattr(om.ch[c], f) for f, _ in po.Channel._fields_])
                            for c in range(om.nch)], om.neutral_density, om.max_frequency, om.neutral_mass,
                        om.neutral_temperature, om.si, om.max_candidates)
    if source == "replay":
        offsets = np.arange(0, (n + 1) * draws_per, draws_per, dtype=np.uint64)
        out_v, stats = apic.collide3(dm, sp.mass, v3, dt, np.concatenate(all_draws), offsets)
    else:
        out_v, stats = apic.collide3(dm, sp.mass, v3, dt, seed=(0x89ABCDE << 32) | 0x1234567, step=17, stream=3)
    cand = 0
    for i in range(n):
        a, b = stats[i], ref_stats[i]
        assert a.candidates == b.candidates and a.null_collisions == b.null_collisions, i
        assert (a.draws & 0x7FFFFFFF) == b.draws and not (a.draws & 0x80000000), i
        assert list(a.channel_collisions)[:om.nch] == list(b.channel_collisions)[:om.nch], i
        assert a.nsecondaries == b.nsecondaries
        for k in range(min(a.nsecondaries, 4)):
            assert rel_max(np.array(a.secondary_velocity[k]), np.array(b.secondary_velocity[k])) < 1e-12
        cand += a.candidates
    assert cand > n  # the test exercised the collision loop
    assert rel_max(out_v, ref_v) < TOL


def _compare_species(dev, ora, s, tol=TOL):
    a = dev.particles(s)
    b = ora.particles(s)
    assert len(a["x"]) == len(b["x"]), (s, len(a["x"]), len(b["x"]))
    for k in ("x", "v", "vh", "vy", "vz"):
        assert rel_max(a[k], b[k]) < tol, (s, k, rel_max(a[k], b[k]))


@pytest.mark.parametrize("steps", [1, 10, 50])
def test_two_stream_parity(steps):
    wl = small_two_stream()
    cfg, tabs = W.to_device_config(wl)
    dev = apic.Simulation1D(cfg, tabs)
    load_device(dev, wl)
    dev.initialize()
    T = po.TableSet()
    ora = po.Sim1D(oracle_config(wl, T), 1)
    load_oracle(ora, wl)
    ora.initialize()
    dev.step(steps)
    ora.step(steps)
    for s in range(2):
        _compare_species(dev, ora, s)
    for a, b in zip(dev.fields(), ora.fields()):
        assert rel_max(a, b) < TOL
    smp = dev.sample()
    assert abs(smp.field_energy - ora.field_energy()) <= 1e-12 * abs(ora.field_energy())
    assert smp.step == steps


def test_dirichlet_rf_without_collisions():
    wl = small_ccp()
    wl.models = []
    cfg, tabs = W.to_device_config(wl)
    dev = apic.Simulation1D(cfg, tabs)
    load_device(dev, wl)
    dev.initialize()
    T = po.TableSet()
    ora = po.Sim1D(oracle_config(wl, T), 1)
    load_oracle(ora, wl)
    ora.initialize()
    dev.step(40)
    ora.step(40)
    for s in range(2):
        _compare_species(dev, ora, s)
        b = dev.boundary_losses(s)
        l, r, el, er = ora.losses(s)
        assert (b.absorbed_left, b.absorbed_right) == (l, r)
    assert sum(ora.losses(0)[:2]) > 0  # walls absorbed something
    for a, b in zip(dev.fields(), ora.fields()):
        assert rel_max(a, b) < TOL


def test_ccp_mcc_parity_philox():
    """Full steps with MCC: the oracle in device layout with the same Philox
    streams must agree exactly on every decision."""
    wl = small_ccp(ppc=32, cells=64)
    seed = 0x5EED
    cfg, tabs = W.to_device_config(wl, seed=seed)
    dev = apic.Simulation1D(cfg, tabs)
    load_device(dev, wl)
    dev.initialize()
    T = po.TableSet()
    ora = po.Sim1D(oracle_config(wl, T), 1, seed)
    load_oracle(ora, wl)
    ora.initialize()
    dev.step(20)
    ora.step(20)
    tot = dev.collision_totals()
    c, nl, per = ora.collisions()
    assert tot.candidates == c and tot.null_collisions == nl
    for m in range(2):
        assert list(tot.channel_collisions[m])[:3] == list(per[m])[:3]
    for s in range(2):
        _compare_species(dev, ora, s, tol=1e-11)


@pytest.mark.parametrize("precision", ["fp64", "fp32_storage"])
def test_ccp_mcc_1v_parity_philox(precision):
    """The 1D1V discharge through the 1V collision interface
    (NullCollisionModel::collide(double&), src/Collision.cpp:831-905): the
    oracle in device layout with the same Philox streams agrees on every
    collision decision; the FP32 storage form against oracle mode 2."""
    wl = W.ccp_helium(particles_per_cell=64, cells=64, seed=5, steps=10, table_rows=256, te_ev=12.0, vdim=1)
    seed = 0x5EED
    prec = apic.FP64 if precision == "fp64" else apic.FP32_STORAGE
    cfg, tabs = W.to_device_config(wl, precision=prec, seed=seed)
    dev = apic.Simulation1D(cfg, tabs)
    load_device(dev, wl)
    dev.initialize()
    T = po.TableSet()
    ora = po.Sim1D(oracle_config(wl, T), 1 if prec == apic.FP64 else 2, seed)
    load_oracle(ora, wl)
    ora.initialize()
    dev.step(40)
    ora.step(40)
    tot = dev.collision_totals()
    c, nl, per = ora.collisions()
    assert tot.candidates == c and tot.null_collisions == nl and c > 100
    for m in range(2):
        assert list(tot.channel_collisions[m])[:2] == list(per[m])[:2]
    assert min(int(per[0][0]), int(per[0][1]), int(per[1][0]) + int(per[1][1])) > 0
    for s in range(2):
        _compare_species(dev, ora, s, tol=1e-11 if prec == apic.FP64 else 1e-6)
    dev.close()


BGK = (2.0e8, 3.0e5)  # frequency (1/s), neutral_temperature_velocity (m/s)


@pytest.mark.parametrize("vdim,precision", [(3, "fp64"), (1, "fp64"), (3, "fp32_storage")])
def test_bgk_parity_philox(vdim, precision):
    """The legacy BGK branch (src/Simulation.cpp:772-834) on the RF discharge
    deck: the oracle in device layout with the same Philox streams agrees on
    every relaxation (counts exact), state within 1e-11 (FP64) or against
    oracle mode 2 within 1e-6 (FP32 storage form); the channel's energy change
    within 1e-9 (the device sums it with FP64 atomics in another order)."""
    wl = W.ccp_helium(particles_per_cell=64, cells=64, seed=6, steps=10, table_rows=64, te_ev=4.0, vdim=vdim,
                      bgk=BGK)
    seed = 0xB6C
    prec = apic.FP64 if precision == "fp64" else apic.FP32_STORAGE
    cfg, tabs = W.to_device_config(wl, precision=prec, seed=seed)
    dev = apic.Simulation1D(cfg, tabs)
    load_device(dev, wl)
    dev.initialize()
    T = po.TableSet()
    ora = po.Sim1D(oracle_config(wl, T), 1 if prec == apic.FP64 else 2, seed)
    load_oracle(ora, wl)
    ora.initialize()
    dev.step(40)
    ora.step(40)
    tot = dev.collision_totals()
    c, nl, per = ora.collisions()
    assert tot.candidates == c == int(per[0][0]) == tot.channel_collisions[0][0] and c > 1000
    assert tot.null_collisions == nl == 0
    e, eo = tot.channel_energy_change[0][0], ora.bgk_energy()
    assert abs(e - eo) <= 1e-9 * abs(eo) and eo != 0.0, (e, eo)
    for s in range(2):
        _compare_species(dev, ora, s, tol=1e-11 if prec == apic.FP64 else 1e-6)
        b = dev.boundary_losses(s)
        assert (b.absorbed_left, b.absorbed_right) == ora.losses(s)[:2]
    dev.close()


def test_bgk_rejections():
    """BGK excludes named MCC models (the reference's message) and the FP32
    cell form does not take it."""
    wl = W.ccp_helium(particles_per_cell=4, cells=16, seed=5, steps=10, table_rows=64, bgk=BGK)
    cfg, tabs = W.to_device_config(wl, precision=apic.FP32, seed=1)
    with pytest.raises(apic.ApicError) as e:
        apic.Simulation1D(cfg, tabs)
    assert "legacy BGK" in str(e.value)


def test_1v_mcc_rejections():
    """The 1V interface takes no ionization or anisotropic channel (the
    reference's logic_error), and the FP32 cell form's collisions are 3V."""
    wl = W.ccp_helium(particles_per_cell=4, cells=16, seed=5, steps=10, table_rows=64, te_ev=12.0, vdim=1)
    wl3 = W.ccp_helium(particles_per_cell=4, cells=16, seed=5, steps=10, table_rows=64, te_ev=12.0)
    wl.models[0].channels.append(wl3.models[0].channels[2])  # ionization
    cfg, tabs = W.to_device_config(wl, seed=1)
    with pytest.raises(apic.ApicError) as e:
        apic.Simulation1D(cfg, tabs)
    assert "require the 3V collision interface" in str(e.value)
    wl.models[0].channels.pop()
    cfg, tabs = W.to_device_config(wl, precision=apic.FP32, seed=1)
    with pytest.raises(apic.ApicError) as e:
        apic.Simulation1D(cfg, tabs)
    assert "velocity_dimensions = 3" in str(e.value)


def test_step_group_matches_individual_steps():
    """Runs stepped together (overlapping streams, two steps per graph launch)
    end in exactly the state of the same runs stepped one by one."""
    decks = [W.ccp_helium(particles_per_cell=16, cells=64, seed=3, table_rows=256, te_ev=12.0),
             W.two_stream(particles_per_beam=2048, nx=64, seed=4),
             W.ccp_helium(particles_per_cell=8, cells=128, seed=5, table_rows=256, te_ev=12.0)]

    def make(wl, k):
        cfg, tabs = W.to_device_config(wl, seed=77 + k)
        sim = apic.Simulation1D(cfg, tabs)
        load_device(sim, wl)
        sim.initialize()
        return sim, tabs

    grouped = [make(wl, k) for k, wl in enumerate(decks)]
    single = [make(wl, k) for k, wl in enumerate(decks)]
    apic.step_group([g for g, _ in grouped], 9)
    apic.step_group([g for g, _ in grouped], 4)
    for s, _ in single:
        s.step(13)
    for (g, _), (s, _), wl in zip(grouped, single, decks):
        assert g.step_count == s.step_count == 13
        for k in range(len(wl.species)):
            a, b = g.particles(k), s.particles(k)
            for key in a:
                assert np.array_equal(a[key], b[key]), key
        for x, y in zip(g.fields(), s.fields()):
            assert np.array_equal(x, y)


def test_cpp20_facade_on_the_device(tmp_path):
    import subprocess
    from test_abi import build_facade_check
    out = subprocess.run([str(build_facade_check(tmp_path))], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "device step=3 live=8" in out.stdout
