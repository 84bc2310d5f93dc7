"""The CPU oracle against golden vectors produced by the reference itself
(tests/golden/make_golden.py).  Bit-exact where the oracle restates the
reference operation by operation (random numbers, particle state, fields)."""
import ctypes as C
import os

import numpy as np
import pytest

import pyoracle as po
from apic import workloads as W

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(G, name))


def test_mt19937_64_and_libstdcxx_distributions():
    f = load("rng.npz")
    L = po.oracle()
    g = (C.c_uint64 * 313)()
    L.ora_mt64_seed(C.byref(g), C.c_uint64(42))
    raw = np.array([L.ora_mt64_next(C.byref(g)) for _ in range(1000)], np.uint64)
    assert np.array_equal(raw, f["mt64_seed42"])
    for kind in range(4):
        mt = (C.c_uint64 * 313)()
        L.ora_mt64_seed(C.byref(mt), C.c_uint64(7))
        r = po.Rng()
        r.kind = 0
        r.mt = C.cast(C.byref(mt), C.c_void_p)
        nst = (C.c_double * 2)()
        out = []
        for _ in range(500):
            if kind == 0:
                out.append(L.ora_uniform01(C.byref(r)))
            elif kind == 1:
                out.append(L.ora_normal_draw(C.byref(nst), C.byref(r), C.c_double(0.0), C.c_double(1.0)))
            elif kind == 2:
                out.append(float(L.ora_bit(C.byref(r))))
            else:
                out.append(L.ora_canonical(C.byref(r)))
        assert np.array_equal(np.array(out), f["dist_seed7"][kind]), kind


@pytest.mark.parametrize("name,dirichlet", [("periodic", 0), ("dirichlet", 1)])
def test_deposit_solve_gather(name, dirichlet):
    f = load(f"grid1d_{name}.npz")
    nx, L, eps = int(f["nx"]), float(f["length"]), float(f["eps"])
    dx = L / (nx - 1 if dirichlet else nx)
    O = po.oracle()
    rho = np.zeros(nx)
    for s, key in enumerate(("x0", "x1")):
        x = np.ascontiguousarray(f[key])
        O.ora_deposit1d(po.dptr(rho), nx, L, dx, dirichlet, float(f["q"][s]), float(f["w"][s]), len(x), po.dptr(x),
                        None)
    assert np.array_equal(rho, f["rho"])
    phi, E = np.zeros(nx), np.zeros(nx)
    O.ora_solve1d(po.dptr(rho), po.dptr(phi), po.dptr(E), nx, L, dx, dirichlet, eps, float(f["phi_left"]),
                  float(f["phi_right"]))
    assert np.array_equal(phi, f["phi"])
    assert np.array_equal(E, f["E"])
    eq = np.array([O.ora_gather1d(po.dptr(E), nx, L, dx, dirichlet, x) for x in f["xq"]])
    assert np.array_equal(eq, f["eq"])


def small_ccp():
    return W.ccp_helium(particles_per_cell=8, cells=32, seed=5, steps=10, table_rows=96)


@pytest.mark.parametrize("mi", [0, 1])
def test_collide3(mi):
    f = load("collide3.npz")
    wl = small_ccp()
    T = po.TableSet()
    cfg = po.config_from_workload(wl, T)
    m = cfg.models[mi]
    O = po.oracle()
    col = (C.c_byte * 8192)()
    assert O.ora_collider_init(col, C.byref(m), wl.species[m.species].mass) == 0
    v_in, seeds = f[f"m{mi}_v_in"], f[f"m{mi}_seeds"]
    dt = float(f[f"m{mi}_dt"])
    for i in range(len(seeds)):
        mt = (C.c_uint64 * 313)()
        O.ora_mt64_seed(C.byref(mt), C.c_uint64(int(seeds[i])))
        r = po.Rng()
        r.kind = 0
        r.mt = C.cast(C.byref(mt), C.c_void_p)
        st = po.CollideStats()
        v = np.ascontiguousarray(v_in[i].copy())
        assert O.ora_collide3(col, po.dptr(v), dt, C.byref(r), C.byref(st)) == 0
        assert np.array_equal(v, f[f"m{mi}_v_out"][i]), i
        assert st.candidates == f[f"m{mi}_candidates"][i]
        assert st.null_collisions == f[f"m{mi}_nulls"][i]
        assert list(st.channel_collisions) == list(f[f"m{mi}_channels"][i])
        assert st.nsecondaries == f[f"m{mi}_nsec"][i]
        assert st.draws == f[f"m{mi}_draws"][i]
        for k in range(min(st.nsecondaries, 4)):
            assert np.array_equal(np.array(st.secondary_velocity[k]), f[f"m{mi}_sec_v"][i][k])
    assert f[f"m{mi}_candidates"].sum() > 100


def _run_sim(name, wl):
    f = load(f"sim1d_{name}.npz")
    T = po.TableSet()
    cfg = po.config_from_workload(wl, T, seed=2024)
    sim = po.Sim1D(cfg, 0)
    for s in range(cfg.nspecies):
        sim.load(s, *[f[f"init_s{s}_{k}"] for k in ("x", "v", "vh", "vy", "vz", "alive")])
    sim.initialize_fields(0.0, 0)
    if "rng_state" in f.files:
        sim.set_mt(f["rng_state"])
    sim.step(int(f["steps"]))
    for s in range(cfg.nspecies):
        p = sim.particles(s)
        for k in ("x", "v", "vh", "vy", "vz", "alive"):
            assert np.array_equal(p[k], f[f"final_s{s}_{k}"]), (name, s, k)
        assert sim.losses(s)[:2] == tuple(int(v) for v in f[f"losses_s{s}"])
        assert sim.electric_work(s) == float(f[f"electric_work_s{s}"]), (name, s)
    rho, phi, E = sim.fields()
    assert np.array_equal(rho, f["rho"]) and np.array_equal(phi, f["phi"]) and np.array_equal(E, f["E"])
    assert sim.time() == float(f["time"])
    return sim, f


def test_two_stream_run_bit_exact():
    _run_sim("two_stream", W.two_stream(particles_per_beam=256, nx=32, seed=4, steps=30))


def test_dirichlet_rf_run_bit_exact():
    wl = small_ccp()
    wl.models = []
    _run_sim("rf", wl)


def test_mcc_run_bit_exact():
    """Shared mt19937_64 stream, ionization products in the first dead slot."""
    hot = W.ccp_helium(particles_per_cell=8, cells=32, seed=5, steps=10, table_rows=96, te_ev=12.0)
    sim, f = _run_sim("mcc", hot)
    c, nl, per = sim.collisions()
    assert c == int(f["candidates"]) and nl == int(f["nulls"])
    ref_per = f["per_channel"]
    assert list(per[0][:3]) + list(per[1][:2]) == [int(v) for v in ref_per]
    assert ref_per[2] > 0  # ionization happened


def test_mcc_1v_run_bit_exact():
    """The 1D1V discharge through NullCollisionModel::collide(double&)
    (src/Collision.cpp:831-905): scalar thermal neutrals, random-sign
    scattering, elastic recoil, excitation and charge exchange; shared
    mt19937_64 stream, 400 steps, bit-exact."""
    hot = W.ccp_helium(particles_per_cell=32, cells=32, seed=5, steps=10, table_rows=96, te_ev=12.0, vdim=1)
    sim, f = _run_sim("mcc1v", hot)
    c, nl, per = sim.collisions()
    assert c == int(f["candidates"]) and nl == int(f["nulls"])
    ref_per = f["per_channel"]
    assert list(per[0][:2]) + list(per[1][:2]) == [int(v) for v in ref_per]
    assert min(int(v) for v in ref_per) > 0  # every channel fired


BGK = (2.0e8, 3.0e5)  # frequency (1/s), neutral_temperature_velocity (m/s)


@pytest.mark.parametrize("vdim", [3, 1])
def test_bgk_run_bit_exact(vdim):
    """The legacy BGK branch of apply_collisions (src/Simulation.cpp:772-834)
    on the RF discharge deck: every species relaxes to one neutral Maxwellian,
    the engine and each species' normal_distribution (with its saved value)
    shared, 60 steps; state, counts and the channel's energy change bit-exact."""
    wl = W.ccp_helium(particles_per_cell=32, cells=32, seed=6, steps=10, table_rows=96, te_ev=4.0,
                      vdim=vdim, bgk=BGK)
    sim, f = _run_sim(f"bgk{vdim}v", wl)
    c, nl, per = sim.collisions()
    assert c == int(f["candidates"]) and nl == int(f["nulls"]) == 0
    assert per[0][0] == int(f["per_channel"][0]) == c > 1000
    assert sim.bgk_energy() == float(f["channel_energy"][0])


def test_bgk_validation_messages():
    """Simulation's collision checks (src/Simulation.cpp:95-100, :388-392)."""
    wl = W.ccp_helium(particles_per_cell=4, cells=8, seed=6, steps=1, table_rows=16, bgk=BGK)
    T = po.TableSet()
    for bgk, msg in (((-1.0, 1.0), "collision frequency must be non-negative and finite"),
                     ((float("nan"), 1.0), "collision frequency must be non-negative and finite"),
                     ((1.0, float("inf")), "neutral_temperature_velocity must be non-negative and finite")):
        wl.bgk = bgk
        with pytest.raises(RuntimeError, match=msg):
            po.Sim1D(po.config_from_workload(wl, T), 0)
    wl.bgk = BGK
    cfg = po.config_from_workload(W.ccp_helium(particles_per_cell=4, cells=8, seed=6, steps=1, table_rows=16), T)
    cfg.bgk, cfg.bgk_frequency, cfg.bgk_neutral_velocity = 1, *BGK
    with pytest.raises(RuntimeError, match="named collision models cannot be combined"):
        po.Sim1D(cfg, 0)


ND_CASES = {
    "sim2d_boris": (2, (16, 8), (0.0, 0.0, 0.7)),
    "sim2d_leapfrog": (2, (8, 8), (0.0, 0.0, 0.0)),
    "sim3d_boris": (3, (8, 4, 8), (0.3, 0.0, 0.0)),
}
ND_SPECIES = [(-1.0, 1.0, 0.05), (1.0, 50.0, 0.05)]


@pytest.mark.parametrize("name", sorted(ND_CASES))
def test_structured_periodic_run_bit_exact(name):
    """Simulation2D / Simulation3D with Boris or leapfrog pushers, CIC deposit,
    FFT spectral Poisson: 25 steps, bit-exact."""
    dims, n, B = ND_CASES[name]
    f = load(f"{name}.npz")
    L = [1.3 * ni for ni in n]
    sim = po.SimND(dims, n, L, 0.1, 1.0, B, ND_SPECIES)
    for k in range(2):
        sim.load(k, f[f"init_s{k}_pos"], f[f"init_s{k}_v"], f[f"init_s{k}_vh"])
    sim.initialize_fields()
    sim.step(int(f["steps"]))
    for k in range(2):
        for key, arr in zip(("pos", "v", "vh"), sim.particles(k)):
            assert np.array_equal(arr, f[f"final_s{k}_{key}"]), (name, k, key)
    rho, phi, E = sim.fields()
    assert np.array_equal(rho, f["rho"]) and np.array_equal(phi, f["phi"]) and np.array_equal(E, f["E"])


@pytest.mark.parametrize("name", ["mixed2d_xperiodic", "mixed2d_yperiodic"])
def test_mixed_spectral_tridiagonal_solve_bit_exact(name):
    """FieldSolver::solve(Mesh2D&) with one periodic axis and wall potentials on
    the other (FFT along the periodic axis, one tridiagonal solve per mode,
    finite-difference E): phi and E bit-exact."""
    f = load(f"{name}.npz")
    phi, E = po.solve_mixed_2d(f["rho"], tuple(int(v) for v in f["n"]), f["L"], int(f["axis"]), float(f["eps"]),
                               float(f["lower"]), float(f["upper"]))
    assert np.array_equal(phi, f["phi"]) and np.array_equal(E, f["E"])


@pytest.mark.parametrize("name,dims,n", [("sim2d_bprofile", 2, (16, 8)), ("sim3d_bprofile", 3, (8, 4, 8))])
def test_tabulated_magnetic_field_run_bit_exact(name, dims, n):
    """Simulation2D / Simulation3D with magnetic_field_profile (B tabulated along
    one axis, evaluated at each particle's position in every Boris kick):
    25 steps, bit-exact."""
    f = load(f"{name}.npz")
    L = [1.3 * ni for ni in n]
    sim = po.SimND(dims, n, L, 0.1, 1.0, (0.0, 0.0, 0.0), ND_SPECIES)
    sim.set_profile(int(f["prof_axis"]), f["prof_c"], f["prof_v"])
    for k in range(2):
        sim.load(k, f[f"init_s{k}_pos"], f[f"init_s{k}_v"], f[f"init_s{k}_vh"])
    sim.initialize_fields()
    sim.step(int(f["steps"]))
    for k in range(2):
        for key, arr in zip(("pos", "v", "vh"), sim.particles(k)):
            assert np.array_equal(arr, f[f"final_s{k}_{key}"]), (name, k, key)
    rho, phi, E = sim.fields()
    assert np.array_equal(rho, f["rho"]) and np.array_equal(phi, f["phi"]) and np.array_equal(E, f["E"])


@pytest.mark.parametrize("name", ["dirichlet2d", "dirichlet3d"])
def test_dirichlet_sor_solve_bit_exact(name):
    """FieldSolver::solve on fully Dirichlet meshes (2D side potentials with the
    corner rule, 3D grounded): the restated SOR is bit-exact with the reference."""
    f = load(f"{name}.npz")
    n = tuple(int(v) for v in f["n"])
    pot = f["pot"] if len(n) == 2 else None
    phi, E = po.solve_dirichlet_nd(f["rho"], n, f["L"], float(f["eps"]), pot)
    assert np.array_equal(phi, f["phi"]) and np.array_equal(E, f["E"])


# ---- CCP campaign diagnostics (src/Simulation.cpp:1163-1560) ----------------

E_CHARGE = 1.602176634e-19


def _ccp_diag_setup(name):
    from golden.make_golden import CCP_DIAG_CASES, ccp_diag_deck
    steps, kw = CCP_DIAG_CASES[name]
    f = load(f"ccp_diag_{name}.npz")
    wl = ccp_diag_deck()
    T = po.TableSet()
    cfg = po.config_from_workload(wl, T, seed=2024)
    sim = po.Sim1D(cfg, 0)
    sa = po.spatial_average1d(**kw)
    sim.enable_spatial_average(sa)
    for s in range(cfg.nspecies):
        sim.load(s, *[f[f"init_s{s}_{k}"] for k in ("x", "v", "vh", "vy", "vz", "alive")])
    sim.initialize_fields(0.0, 0)
    sim.set_mt(f["rng_state"])
    sim.step(steps)
    return sim, sa, cfg, wl, f, T


def _csv_tables(sim, sa, cfg, wl):
    """write_spatial_average's derived columns (src/Simulation.cpp:1372-1560)
    from the oracle's sums, without the node coordinate column."""
    nx, ns = cfg.nx, cfg.nspecies
    samples, _, psamples, _ = sim.spatial_counts()
    dims = float(cfg.vdim)
    dens = [sim.spatial_sums(po.SA_DENSITY, s) for s in range(ns)]
    ke = [sim.spatial_sums(po.SA_KINETIC, s) for s in range(ns)]
    t = {"spatial_average": [], "spatial_kinetic_energy": [], "spatial_field_average": []}
    for s in range(ns):
        for i in range(nx):
            t["spatial_average"].append([s, i, dens[s][i] / float(samples)])
            me = ke[s][i] / dens[s][i] / E_CHARGE if dens[s][i] > 0.0 else 0.0
            t["spatial_kinetic_energy"].append([s, i, me, 2.0 * me / dims])
    phi, E, E2 = (sim.spatial_sums(q) for q in (po.SA_POTENTIAL, po.SA_ELECTRIC, po.SA_ELECTRIC2))
    for i in range(nx):
        t["spatial_field_average"].append([i, phi[i] / float(samples), E[i] / float(samples),
                                           np.sqrt(E2[i] / float(samples))])
    P = int(sa.phase_bins)
    if P:
        t["spatial_phase_moments"], t["spatial_phase_fields"] = [], []
        for p in range(P):
            n = float(psamples[p])
            frac = (float(p) + 0.5) / float(P)
            for s in range(ns):
                m = [sim.spatial_sums(q, s, p) for q in range(5)]
                mass = wl.species[s].mass
                for i in range(nx):
                    d = m[0][i]
                    ux = m[1][i] / d if d > 0.0 else 0.0
                    uy = m[2][i] / d if d > 0.0 else 0.0
                    uz = m[3][i] / d if d > 0.0 else 0.0
                    me = m[4][i] / d / E_CHARGE if d > 0.0 else 0.0
                    drift = 0.5 * mass * (ux * ux + uy * uy + uz * uz) / E_CHARGE
                    temp = 2.0 / dims * max(0.0, me - drift)
                    t["spatial_phase_moments"].append([p, frac, n, s, i, d / n if n > 0 else 0.0, ux, uy, uz, me,
                                                       temp])
            fphi, fE, fE2 = (sim.spatial_sums(q, 0, p) for q in (po.SA_POTENTIAL, po.SA_ELECTRIC, po.SA_ELECTRIC2))
            for i in range(nx):
                t["spatial_phase_fields"].append([p, frac, n, i, fphi[i] / n, fE[i] / n, np.sqrt(fE2[i] / n)])
    return {k: np.array(v) for k, v in t.items()}


@pytest.mark.parametrize("name", ["rf", "window"])
def test_ccp_campaign_diagnostics_bit_exact(name):
    """Oracle mode 0 against the reference's own run: the collision-energy
    and phase-EEDF accumulators bit for bit, and every derived column of the
    spatial-average CSV files (17 significant digits round-trip a double)."""
    sim, sa, cfg, wl, f, _keep = _ccp_diag_setup(name)
    P = int(sa.phase_bins)
    samples, csteps, psamples, pcoll = sim.spatial_counts()
    assert csteps == int(f["collision_steps"])
    assert np.array_equal(pcoll, f["collision_phase_steps"])
    nch = f["collision_energy"].shape[0]
    for c in range(nch):
        assert np.array_equal(sim.spatial_sums(po.SA_COLLISION, c), f["collision_energy"][c]), c
        for p in range(P):
            assert np.array_equal(sim.spatial_sums(po.SA_COLLISION, c, p), f["collision_energy_phase"][p][c])
    assert np.any(f["collision_energy"] != 0.0)
    if sa.eedf_species >= 0:
        k = 0
        for p in range(P):
            for r in range(sa.eedf_regions):
                cnt, sums, hist = sim.phase_eedf(p, r)
                assert np.array_equal(cnt, f["eedf_counts"][k]), (p, r)
                assert np.array_equal(sums, f["eedf_sums"][k]), (p, r)
                assert np.array_equal(hist, f["eedf_hist"][k]), (p, r)
                k += 1
    tables = _csv_tables(sim, sa, cfg, wl)
    for key, mine in tables.items():
        ref = f[f"csv_{key}"]
        header = list(f[f"csv_{key}_header"])
        cols = [i for i, h in enumerate(header) if not h.startswith("x_")]
        assert np.array_equal(ref[:, cols], mine), key


@pytest.mark.parametrize("name", ["sim2d_walls_mixed", "sim2d_walls_dirichlet"])
def test_2d_run_with_walls_bit_exact(name):
    """Simulation2D with walls: clamped CIC deposit over half-cell wall areas,
    clamped gather, absorbing and reflecting particle boundaries with the
    per-side loss ledger, and the mixed spectral-tridiagonal or the SOR
    Dirichlet solve (src/Simulation2D.cpp:38-97, :1309-1364, src/Mesh2D.cpp:77-144,
    src/FieldSolver.cpp:389-397): 25 steps, bit-exact."""
    from golden.make_golden import WALL_CASES
    n, B, d, pot, pb = WALL_CASES[name]
    f = load(f"{name}.npz")
    sim = po.SimND(2, n, (4.0, 2.0), 0.1, 1.0, B, ND_SPECIES)
    sim.set_walls(d, pot, pb)
    for k in range(2):
        sim.load(k, f[f"init_s{k}_pos"], f[f"init_s{k}_v"], f[f"init_s{k}_vh"])
    sim.initialize_fields()
    sim.step(int(f["steps"]))
    for k in range(2):
        al, lo = sim.alive_losses(k)
        assert np.array_equal(al, f[f"final_s{k}_alive"]), (name, k)
        assert np.array_equal(lo, f[f"losses_s{k}"]), (name, k)
        for key, arr in zip(("pos", "v", "vh"), sim.particles(k)):
            assert np.array_equal(arr, f[f"final_s{k}_{key}"]), (name, k, key)
    rho, phi, E = sim.fields()
    assert np.array_equal(rho, f["rho"]) and np.array_equal(phi, f["phi"])
    assert np.array_equal(E[:2].ravel(), f["E"].ravel()[: 2 * len(rho)])


@pytest.mark.parametrize("name", ["sim3d_walls_boris", "sim3d_walls_leapfrog"])
def test_3d_run_with_walls_bit_exact(name):
    """Simulation3D on a Dirichlet mesh: clamped trilinear CIC over the half-cell
    wall volumes, clamped gather, the warm-started SOR with grounded walls,
    absorbing, reflecting and periodic particle boundaries in the order left,
    right, bottom, top, back, front (src/Simulation3D.cpp:25-97, :309-365,
    src/Mesh3D.cpp:52-126, src/FieldSolver.cpp:830-907, :978-1038): 25 steps,
    bit-exact.  The reference keeps one loss ledger for the run; the oracle's
    per-species counts add up to it."""
    from golden.make_golden import WALL3_CASES, WALL3_LENGTH
    n, B, pb = WALL3_CASES[name]
    f = load(f"{name}.npz")
    sim = po.SimND(3, n, WALL3_LENGTH, 0.1, 1.0, B, ND_SPECIES)
    sim.set_walls3d(pb)
    for k in range(2):
        sim.load(k, f[f"init_s{k}_pos"], f[f"init_s{k}_v"], f[f"init_s{k}_vh"])
    sim.initialize_fields()
    sim.step(int(f["steps"]))
    total = np.zeros(6, np.uint64)
    for k in range(2):
        al, lo = sim.alive_losses(k)
        total += lo
        assert np.array_equal(al, f[f"final_s{k}_alive"]), (name, k)
        for key, arr in zip(("pos", "v", "vh"), sim.particles(k)):
            assert np.array_equal(arr, f[f"final_s{k}_{key}"]), (name, k, key)
    assert np.array_equal(total, f["losses_s0"]) and total.sum() > 0
    rho, phi, E = sim.fields()
    assert np.array_equal(rho, f["rho"]) and np.array_equal(phi, f["phi"])
    assert np.array_equal(E.ravel()[: 3 * len(rho)], f["E"].ravel())
