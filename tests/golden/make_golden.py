"""Generates the golden vectors under tests/golden/ by running the reference
itself (its library compiled from the reference sources by oracle/Makefile,
driven through oracle/ref_harness.cpp).  Run from the repository root:

    make -C oracle ref && python tests/golden/make_golden.py [fixture ...]

(no names: every fixture; a name such as `mixed` writes only that one).

The fixtures pin the CPU oracle (oracle/apic_oracle.c) in
tests/test_oracle_golden.py; the GPU parity tests then compare the device
library with the oracle.
"""
from __future__ import annotations

import ctypes as C
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "aurora-pic_b200"))

import pyoracle as po  # noqa: E402
from apic import workloads as W  # noqa: E402


def rng_fixture():
    R = po.ref()
    raw = np.zeros(1000, np.uint64)
    R.ref_mt64(42, 1000, po.u64ptr(raw))
    dists = np.zeros((4, 500))
    for k in range(4):
        d = np.zeros(500)
        R.ref_dist(k, 7, 500, po.dptr(d))
        dists[k] = d
    np.savez_compressed(os.path.join(HERE, "rng.npz"), mt64_seed42=raw, dist_seed7=dists)


def grid_fixture():
    R = po.ref()
    rng = np.random.default_rng(21)
    for name, dirichlet in (("periodic", 0), ("dirichlet", 1)):
        nx, L, eps = 67, 2.3, 1.7
        xs = [rng.uniform(0, L, 700), rng.uniform(0, L, 500)]
        xs[0][:2] = [0.0, L]
        q = np.array([-1.0, 1.0])
        w = np.array([0.011, 0.017])
        xq = rng.uniform(-0.3, L + 0.3, 300)
        counts = (C.c_size_t * 2)(len(xs[0]), len(xs[1]))
        ptrs = (C.POINTER(C.c_double) * 2)(po.dptr(xs[0]), po.dptr(xs[1]))
        rho, phi, E, eq = np.zeros(nx), np.zeros(nx), np.zeros(nx), np.zeros(len(xq))
        rc = R.ref_deposit_solve_gather_1d(dirichlet, nx, L, eps, 0.3, -1.1, 2, po.dptr(q), po.dptr(w), counts, ptrs,
                                           po.dptr(rho), po.dptr(phi), po.dptr(E), len(xq), po.dptr(xq), po.dptr(eq))
        assert rc == 0, R.ref_last_error()
        np.savez_compressed(os.path.join(HERE, f"grid1d_{name}.npz"), nx=nx, length=L, eps=eps, phi_left=0.3,
                            phi_right=-1.1, q=q, w=w, x0=xs[0], x1=xs[1], xq=xq, rho=rho, phi=phi, E=E, eq=eq)


def small_ccp(ppc=8, cells=32, rows=96):
    return W.ccp_helium(particles_per_cell=ppc, cells=cells, seed=5, steps=10, table_rows=rows)


def collide_fixture():
    R = po.ref()
    wl = small_ccp()
    out = {}
    for mi, scale in ((0, 5e6), (1, 6e4)):
        T = po.TableSet()
        cfg = po.config_from_workload(wl, T)
        m = cfg.models[mi]
        rng = np.random.default_rng(100 + mi)
        n = 300
        v = rng.standard_normal((n, 3)) * scale
        seeds = rng.integers(1, 2 ** 62, n, dtype=np.uint64)
        stats = (po.CollideStats * n)()
        vv = np.ascontiguousarray(v.copy())
        dt = wl.dt * 40
        work = tempfile.mkdtemp()
        rc = R.ref_collide3(C.byref(m), wl.species[m.species].mass, work.encode(), n, po.dptr(vv.reshape(-1)),
                            po.u64ptr(seeds), dt, stats, None, 0)
        assert rc == 0, R.ref_last_error()
        ch = [m.ch[i] for i in range(m.nch)]
        out[f"m{mi}_v_in"] = v
        out[f"m{mi}_v_out"] = vv
        out[f"m{mi}_seeds"] = seeds
        out[f"m{mi}_dt"] = dt
        out[f"m{mi}_candidates"] = np.array([s.candidates for s in stats], np.uint64)
        out[f"m{mi}_nulls"] = np.array([s.null_collisions for s in stats], np.uint64)
        out[f"m{mi}_channels"] = np.array([list(s.channel_collisions) for s in stats], np.uint64)
        out[f"m{mi}_nsec"] = np.array([s.nsecondaries for s in stats], np.int32)
        out[f"m{mi}_draws"] = np.array([s.draws for s in stats], np.uint64)
        out[f"m{mi}_sec_v"] = np.array([[list(s.secondary_velocity[k]) for k in range(4)] for s in stats])
    np.savez_compressed(os.path.join(HERE, "collide3.npz"), **out)


def sim_fixture(name, wl, steps, with_rng=False, with_energy=False):
    T = po.TableSet()
    cfg = po.config_from_workload(wl, T, seed=2024, own_loading=True)
    work = tempfile.mkdtemp()
    R = po.Ref1D(cfg, work)
    R.initialize()
    out = {"steps": steps}
    for s in range(cfg.nspecies):
        p = R.particles(s)
        for k, v in p.items():
            out[f"init_s{s}_{k}"] = v
    if with_rng:
        out["rng_state"] = R.rng_state()
    R.step(steps)
    for s in range(cfg.nspecies):
        p = R.particles(s)
        for k, v in p.items():
            out[f"final_s{s}_{k}"] = v
        out[f"losses_s{s}"] = np.array(R.losses(s)[:2], np.uint64)
        out[f"electric_work_s{s}"] = R.electric_work(s)
    rho, phi, E = R.fields()
    out.update(rho=rho, phi=phi, E=E, time=R.time())
    c, nl, per = R.collisions()
    out.update(candidates=c, nulls=nl, per_channel=per)
    if with_energy:
        out["channel_energy"] = R.channel_energy()
    np.savez_compressed(os.path.join(HERE, f"sim1d_{name}.npz"), **out)


ND_CASES = {
    # name: dims, cells, B, steps
    "sim2d_boris": (2, (16, 8), (0.0, 0.0, 0.7), 25),
    "sim2d_leapfrog": (2, (8, 8), (0.0, 0.0, 0.0), 25),
    "sim3d_boris": (3, (8, 4, 8), (0.3, 0.0, 0.0), 25),
}
ND_SPECIES = [(-1.0, 1.0, 0.05, 400, 0.3, 0.4), (1.0, 50.0, 0.05, 400, 0.0, 0.05)]


# magnetic_field_profile cases: B tabulated along one axis (uniform B zero)
PROFILE_CASES = {
    # name: dims, cells, axis, steps
    "sim2d_bprofile": (2, (16, 8), 0, 25),
    "sim3d_bprofile": (3, (8, 4, 8), 2, 25),
}


def bprofile_table(axis_length, rows=9):
    """A smooth B(s) table covering [0, axis_length] (rows unevenly spaced)."""
    c = axis_length * (np.linspace(0.0, 1.0, rows) ** 1.3)
    v = np.stack([0.2 * np.sin(3.0 * c / axis_length), 0.1 + 0.0 * c, 0.8 + 0.4 * np.cos(2.0 * c / axis_length)],
                 axis=1)
    return c, v


def bprofile_fixture():
    for name, (dims, n, axis, steps) in PROFILE_CASES.items():
        L = [1.3 * ni for ni in n]
        c, v = bprofile_table(L[axis])
        _nd_run(name, dims, n, L, (0.0, 0.0, 0.0), steps, profile=(axis, c, v))


def nd_fixture(name):
    dims, n, B, steps = ND_CASES[name]
    L = [1.3 * ni for ni in n]
    _nd_run(name, dims, n, L, B, steps)


def _nd_run(name, dims, n, L, B, steps, profile=None, walls=None):
    R = po.RefND(dims, n, L, 0.1, 0, B, ND_SPECIES, seed=9, profile=profile, walls=walls)
    R.initialize()
    out = {"steps": steps}
    for k in range(len(ND_SPECIES)):
        for key, arr in zip(("pos", "v", "vh"), R.particles(k)):
            out[f"init_s{k}_{key}"] = arr
    R.step(steps)
    for k in range(len(ND_SPECIES)):
        for key, arr in zip(("pos", "v", "vh"), R.particles(k)):
            out[f"final_s{k}_{key}"] = arr
        if walls is not None:
            al, lo = R.alive_losses(k)
            out[f"final_s{k}_alive"] = al
            out[f"losses_s{k}"] = lo
    rho, phi, E = R.fields()
    out.update(rho=rho, phi=phi, E=E, time=R.time())
    if walls is not None and dims == 3:
        out.update(walls_particle=np.array(walls))
    elif walls is not None:
        out.update(walls_dirichlet=np.array(walls[0]), walls_potentials=np.array(walls[1]),
                   walls_particle=np.array(walls[2]))
    if profile is not None:
        out.update(prof_axis=profile[0], prof_c=profile[1], prof_v=profile[2])
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


# 2D runs with walls: name -> cells, B, Dirichlet axes, side potentials, particle
# boundaries (left, right, bottom, top: 0 periodic, 1 absorbing, 2 reflecting)
WALL_CASES = {
    "sim2d_walls_mixed": ((17, 8), (0.0, 0.0, 0.7), (1, 0), (0.0, 0.4, 0.0, 0.0), (1, 2, 0, 0)),
    "sim2d_walls_dirichlet": ((17, 9), (0.0, 0.0, 0.0), (1, 1), (1.0, -0.5, 0.25, 0.0), (1, 1, 2, 1)),
}


def walls_fixture():
    """Simulation2D with a wall axis (mixed solve) and with walls on every side
    (the reference's SOR): absorbing and reflecting particle boundaries, 25 steps."""
    for name, (n, B, d, pot, pb) in WALL_CASES.items():
        _nd_run(name, 2, n, (4.0, 2.0), B, 25, walls=(d, pot, pb))


# 3D runs with walls (a grounded Dirichlet mesh): name -> nodes, B, particle
# boundaries (left, right, bottom, top, back, front: 0 periodic, 1 absorbing,
# 2 reflecting)
WALL3_CASES = {
    "sim3d_walls_boris": ((17, 9, 9), (0.3, 0.0, 0.5), (1, 2, 1, 2, 1, 1)),
    "sim3d_walls_leapfrog": ((9, 9, 17), (0.0, 0.0, 0.0), (2, 1, 0, 0, 1, 2)),
}
WALL3_LENGTH = (4.0, 2.0, 3.0)


def walls3d_fixture():
    """Simulation3D on a Dirichlet mesh: clamped trilinear CIC over the
    half-cell wall volumes, the warm-started SOR, absorbing, reflecting and
    periodic particle boundaries with the run's loss ledger, 25 steps."""
    for name, (n, B, pb) in WALL3_CASES.items():
        _nd_run(name, 3, n, WALL3_LENGTH, B, 25, walls=pb)


def collide_hg_fixture():
    """NullCollisionModel::collide with Henyey-Greenstein elastic scattering,
    ionization and attachment (electron projectile, thermal neutrals)."""
    R = po.ref()
    ch, mn = W.swarm_gas_anisotropic(attachment=True)
    T = po.TableSet()
    chans = [T.channel(c.process, c.energy, c.sigma, c.threshold, 0 if c.process == W.IONIZATION else -1,
                       1 if c.process == W.IONIZATION else -1, angular=c.angular, mu_energy=c.mu_energy, mu=c.mu)
             for c in ch]
    nu = W.swarm_max_frequency(ch, 1e24, mn, 300.0, 200.0)
    m = po.make_model(0, chans, 1e24, nu, mn, 300.0, 1, 64)
    rng = np.random.default_rng(300)
    n = 400
    v = rng.standard_normal((n, 3)) * 1.2e6
    seeds = rng.integers(1, 2 ** 62, n, dtype=np.uint64)
    stats = (po.CollideStats * n)()
    vv = np.ascontiguousarray(v.copy())
    dt = 2.0 / nu
    rc = R.ref_collide3(C.byref(m), W.M_E, tempfile.mkdtemp().encode(), n, po.dptr(vv.reshape(-1)),
                        po.u64ptr(seeds), dt, stats, None, 0)
    assert rc == 0, R.ref_last_error()
    np.savez_compressed(os.path.join(HERE, "collide3_hg.npz"), v_in=v, v_out=vv, seeds=seeds, dt=dt, nu=nu,
                        candidates=np.array([s.candidates for s in stats], np.uint64),
                        channels=np.array([list(s.channel_collisions) for s in stats], np.uint64),
                        nsec=np.array([s.nsecondaries for s in stats], np.int32),
                        removed=np.array([s.removed for s in stats], np.int32),
                        draws=np.array([s.draws for s in stats], np.uint64),
                        sec_v=np.array([[list(s.secondary_velocity[k]) for k in range(4)] for s in stats]))


def swarm_fixture():
    """pic::run_swarm_benchmark on the small decks of tests/common.py."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from common import swarm_cases, SWARM_KEYS
    for name, spec in swarm_cases().items():
        T = po.TableSet()
        cfg, gas = po.swarm_from_spec(spec, T)
        res = po.ref_swarm_run(cfg, gas, spec.fields_td, tempfile.mkdtemp())
        out = {k: np.array([getattr(r, k) for r in res]) for k in SWARM_KEYS}
        out["channel_collisions"] = np.array([list(r.channel_collisions)[: r.nch] for r in res], np.uint64)
        out["channel_rate"] = np.array([list(r.channel_rate)[: r.nch] for r in res])
        out["fields_td"] = np.array(spec.fields_td)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


def swarm_ensemble_fixture():
    """run_swarm_benchmark over ENSEMBLE_SEEDS seeds of each ensemble deck."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from common import ENSEMBLE_KEYS, ENSEMBLE_SEEDS, swarm_ensemble_cases
    for name, spec in swarm_ensemble_cases().items():
        T = po.TableSet()
        cfg, gas = po.swarm_from_spec(spec, T)
        rows = []
        for k in range(ENSEMBLE_SEEDS):
            cfg.seed = spec.seed + 100 * k
            rows.append(po.ref_swarm_run(cfg, gas, spec.fields_td, tempfile.mkdtemp()))
        out = {key: np.array([[getattr(r, key) for r in row] for row in rows]) for key in ENSEMBLE_KEYS}
        out["fields_td"] = np.array(spec.fields_td)
        np.savez_compressed(os.path.join(HERE, f"swarm_ensemble_{name}.npz"), **out)


MIXED_CASES = {
    # name: (n, L, periodic axis, lower / upper wall potentials)
    "mixed2d_xperiodic": ((64, 33), (0.02, 0.015), 0, (0.0, 12.5)),
    "mixed2d_yperiodic": ((17, 32), (0.01, 0.03), 1, (-3.0, 7.0)),
}


def mixed_fixture():
    """FieldSolver::solve(Mesh2D&) on meshes with one periodic axis (the
    spectral-tridiagonal solve), from seeded charge densities."""
    eps = 8.8541878128e-12
    for k, (name, (n, L, axis, (lo, hi))) in enumerate(MIXED_CASES.items()):
        rng = np.random.default_rng(90 + k)
        nx, ny = n
        x = np.arange(nx)[None, :] / nx
        y = np.arange(ny)[:, None] / ny
        rho = 1e-6 * (1.0 + 0.3 * np.sin(2 * np.pi * x) * np.cos(np.pi * y) + 0.05 * rng.standard_normal((ny, nx)))
        phi, E = po.ref_solve_mixed_2d(rho, n, L, axis, eps, lo, hi)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), n=np.array(n), L=np.array(L), axis=axis, eps=eps,
                            lower=lo, upper=hi, rho=rho.ravel(), phi=phi, E=E)


DIRICHLET_CASES = {
    # name: (n, L, side potentials left, right, bottom, top)
    "dirichlet2d": ((17, 9), (0.02, 0.01), (0.0, 50.0, -10.0, 5.0)),
    "dirichlet3d": ((9, 5, 9), (0.01, 0.005, 0.01), (0.0, 0.0, 0.0, 0.0)),
}


def dirichlet_fixture():
    """FieldSolver::solve on fully Dirichlet meshes (the reference's SOR)."""
    eps = 8.8541878128e-12
    for k, (name, (n, L, pot)) in enumerate(DIRICHLET_CASES.items()):
        rng = np.random.default_rng(70 + k)
        rho = 1e-6 * (1.0 + 0.3 * rng.standard_normal(int(np.prod(n))))
        phi, E = po.ref_solve_dirichlet_nd(rho, n, L, eps, pot)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), n=np.array(n), L=np.array(L), eps=eps,
                            pot=np.array(pot), rho=rho, phi=phi, E=E)


CCP_DIAG_CASES = {
    # name: steps, spatial-average settings
    "rf": (400, dict(interval=4, start_step=1, end_step=400, rf_frequency=13.56e6, rf_cycles=1, phase_bins=4,
                     eedf_species=0, eedf_bins=32, eedf_energy_max=50.0,
                     eedf_regions=((0.0, 0.02), (0.02, 0.067)))),
    "window": (40, dict(interval=5, start_step=3, end_step=37)),
}


def ccp_diag_deck():
    return W.ccp_helium(particles_per_cell=8, cells=32, seed=5, steps=10, table_rows=96, te_ev=12.0)


def _read_csv(path):
    import csv
    with open(path) as f:
        rows = list(csv.reader(f))
    return rows[0], rows[1:]


def ccp_diag_fixture():
    """Campaign diagnostics of a small RF discharge: the collision-energy and
    phase-EEDF accumulators read through the reference's accessors after
    initialize + step, and the spatial-average CSV files of Simulation::run
    over the same steps (values printed with 17 significant digits)."""
    wl = ccp_diag_deck()
    for name, (steps, kw) in CCP_DIAG_CASES.items():
        T = po.TableSet()
        cfg = po.config_from_workload(wl, T, seed=2024, own_loading=True)
        sa = po.spatial_average1d(**kw)
        R = po.Ref1D(cfg, tempfile.mkdtemp(), spatial_average=sa)
        R.initialize()
        out = {"steps": steps}
        for s in range(cfg.nspecies):
            for k, v in R.particles(s).items():
                out[f"init_s{s}_{k}"] = v
        out["rng_state"] = R.rng_state()
        R.step(steps)
        nch = sum(cfg.models[m].nch for m in range(cfg.nmodels))
        P = int(sa.phase_bins)
        out["collision_energy"] = np.array([R.collision_energy(c) for c in range(nch)])
        if P:
            out["collision_energy_phase"] = np.array([[R.collision_energy(c, p) for c in range(nch)]
                                                      for p in range(P)])
        cs, ps = R.collision_steps()
        out["collision_steps"] = cs
        out["collision_phase_steps"] = ps
        if sa.eedf_species >= 0:
            cnt, sums, hist = [], [], []
            for p in range(P):
                for r in range(sa.eedf_regions):
                    c, sm, h = R.phase_eedf(p, r)
                    cnt.append(c); sums.append(sm); hist.append(h)
            out["eedf_counts"] = np.array(cnt)
            out["eedf_sums"] = np.array(sums)
            out["eedf_hist"] = np.array(hist)
        folder = po.ref_run_spatial_average(cfg, sa, steps, tempfile.mkdtemp())
        files = ["spatial_average", "spatial_kinetic_energy", "spatial_field_average"]
        if P:
            files += ["spatial_phase_moments", "spatial_phase_fields"]
        for f in files:
            header, rows = _read_csv(os.path.join(folder, f + ".csv"))
            numeric = [i for i, h in enumerate(header) if h != "species"]
            out[f"csv_{f}"] = np.array([[float(r[i]) for i in numeric] for r in rows])
            out[f"csv_{f}_header"] = np.array([header[i] for i in numeric])
        np.savez_compressed(os.path.join(HERE, f"ccp_diag_{name}.npz"), **out)


def townsend_deck():
    """A swarm deck whose spatial Townsend pass is short: the 4-process gas at
    1e23 m^-3, two fields, ten electrons per history population (so the
    cascades are resampled), 50 histories over 2 mm and 8 planes."""
    ch, mn = W.swarm_gas_4process(table_rows=512, e_max_ev=400.0)
    ng, T = 1e23, 300.0
    nu = W.swarm_max_frequency(ch, ng, mn, T, 200.0)
    spec = W.SwarmSpec("townsend", ch, mn, ng, T, nu, 0.1 / nu, 100, 50, 10, [450.0, 600.0], branching=True,
                       uncertainty_blocks=5, initial_mean_energy_ev=1.0, max_energy_ev=200.0, seed=77)
    sp = po.spatial_config(histories=50, length_m=2e-3, bins=8, fit_begin_bin=1, max_steps=200000)
    return spec, sp


def townsend_fixture():
    """run_swarm_benchmark with the spatial Townsend controls: per field the
    spatial result fields and the flux profile."""
    spec, sp = townsend_deck()
    T = po.TableSet()
    cfg, gas = po.swarm_from_spec(spec, T)
    rows = po.ref_swarm_run_spatial(cfg, sp, gas, spec.fields_td, tempfile.mkdtemp())
    out = {}
    for f, (_, r, prof) in enumerate(rows):
        out[f"f{f}_scalars"] = np.array([r.townsend_1_m, r.townsend_se_1_m, r.fit_r_squared])
        out[f"f{f}_counts"] = np.array([r.histories_completed, r.maximum_active_particles, r.particle_updates],
                                       np.uint64)
        out[f"f{f}_profile"] = prof
    np.savez_compressed(os.path.join(HERE, "swarm_townsend.npz"), **out)


def mcc1v_fixture():
    """The 1D1V discharge with the 1V collision interface (elastic and
    excitation electrons, elastic and charge-exchange ions), shared engine."""
    hot = W.ccp_helium(particles_per_cell=32, cells=32, seed=5, steps=10, table_rows=96, te_ev=12.0, vdim=1)
    sim_fixture("mcc1v", hot, 400, with_rng=True)


BGK = (2.0e8, 3.0e5)  # frequency (1/s), neutral_temperature_velocity (m/s)


def bgk_fixture():
    """The RF discharge deck with the legacy BGK model instead of MCC, 1D3V and
    1D1V (electrons and ions relax to one neutral Maxwellian), shared engine."""
    for vdim in (3, 1):
        wl = W.ccp_helium(particles_per_cell=32, cells=32, seed=6, steps=10, table_rows=96, te_ev=4.0,
                          vdim=vdim, bgk=BGK)
        sim_fixture(f"bgk{vdim}v", wl, 60, with_rng=True, with_energy=True)


def main(names=None):
    if names:
        for n in names:
            globals()[f"{n}_fixture"]()
        print("golden vectors written to", HERE)
        return
    ccp_diag_fixture()
    townsend_fixture()
    walls_fixture()
    walls3d_fixture()
    mixed_fixture()
    dirichlet_fixture()
    bprofile_fixture()
    swarm_ensemble_fixture()
    swarm_fixture()
    collide_hg_fixture()
    for name in ND_CASES:
        nd_fixture(name)
    rng_fixture()
    grid_fixture()
    collide_fixture()
    ts = W.two_stream(particles_per_beam=256, nx=32, seed=4, steps=30)
    sim_fixture("two_stream", ts, 30)
    rf = small_ccp()
    rf.models = []
    sim_fixture("rf", rf, 30)
    hot = W.ccp_helium(particles_per_cell=8, cells=32, seed=5, steps=10, table_rows=96, te_ev=12.0)
    sim_fixture("mcc", hot, 30, with_rng=True)
    mcc1v_fixture()
    bgk_fixture()
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main(sys.argv[1:])
