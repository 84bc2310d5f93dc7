"""Parity of the device 2D3V / 3D3V periodic step against the CPU oracle
(itself bit-exact with Simulation2D / Simulation3D), through the C ABI.
FP64 form: particle state and fields within 1e-12 relative (max-norm)."""
import os

import numpy as np
import pytest

import apic
import pyoracle as po
from apic import workloads as W
from common import rel_max

pytestmark = pytest.mark.gpu
TOL = 1e-12


def run_pair(wl, steps, sort_interval=4):
    cfg = W.to_device_config_nd(wl, sort_interval=sort_interval)
    dev = apic.SimulationND(cfg)
    eps = 8.8541878128e-12 if wl.si else 1.0
    ora = po.SimND(wl.dims, wl.n, wl.length, wl.dt, eps, wl.B, [(q, m, w) for (q, m, w, pos, v) in wl.species])
    for k, (q, m, w, pos, v) in enumerate(wl.species):
        dev.load(k, pos, v)
        ora.load(k, pos, v, v)
    dev.initialize()
    ora.initialize()
    dev.step(steps)
    ora.step(steps)
    return dev, ora


@pytest.mark.parametrize("case", ["2d_boris", "2d_leapfrog", "3d_boris"])
@pytest.mark.parametrize("steps", [1, 12])
def test_structured_step_parity(case, steps):
    if case.startswith("2d"):
        wl = W.plasma_2d(cells=(32, 16), ppc=8, seed=3)
        if case == "2d_leapfrog":
            wl.B = (0.0, 0.0, 0.0)
    else:
        wl = W.plasma_3d(cells=(16, 8, 8), ppc=4, seed=5)
    dev, ora = run_pair(wl, steps)
    for k in range(2):
        a, b = dev.particles(k), ora.particles(k)
        for name, x, y in zip(("pos", "v", "vh"), a, b):
            assert rel_max(x[: 3 if wl.dims == 3 else 2] if name == "pos" else x,
                           y[: 3 if wl.dims == 3 else 2] if name == "pos" else y) < TOL, (case, k, name)
    fa, fb = dev.fields(), ora.fields()
    for name, x, y in zip(("rho", "phi", "E"), fa, fb):
        assert rel_max(x, y) < TOL, (case, name, rel_max(x, y))
    s = dev.sample()
    assert s.step == steps and s.live_particles == wl.particles


@pytest.mark.parametrize("dims,n", [(2, (64, 32)), (3, (32, 16, 8)), (3, (8, 8, 8)),
                                    (2, (256, 64)), (2, (32, 256)), (3, (256, 16, 8)), (3, (16, 256, 8)),
                                    (3, (8, 16, 256)), (3, (256, 256, 64))])
def test_periodic_solve_against_oracle(dims, n):
    """Every pass kernel: the shared-memory tile FFTs and, along 256-node axes,
    the register four-step FFTs (x pass and strided y / z passes)."""
    rng = np.random.default_rng(2)
    N = int(np.prod(n))
    L = [0.7 * (a + 1) for a in range(dims)]
    rho = rng.standard_normal(N) + 3.0
    phi, E = apic.field_solve_periodic_nd(dims, n, L, 1.3, rho)
    pr, Er = np.zeros(N), np.zeros(3 * N)
    po._nd_bind().ora_solve_nd(po.dptr(rho), po.dptr(pr), po.dptr(Er), dims, po.sizes3(n), po.dptr(po.arr3(L)), 1.3)
    assert rel_max(phi, pr) < TOL
    assert rel_max(E, Er[: dims * N].reshape(dims, N)) < TOL


@pytest.mark.parametrize("n,L,axis,walls", [((64, 33), (0.02, 0.015), 0, (0.0, 12.5)),
                                             ((17, 32), (0.01, 0.03), 1, (-3.0, 7.0)),
                                             ((256, 3), (1.0, 0.5), 0, (1.0, -1.0)),
                                             ((129, 512), (0.2, 0.1), 1, (0.0, 0.0))])
def test_mixed_periodic_wall_solve_against_oracle(n, L, axis, walls):
    """FieldSolver::solve(Mesh2D&) with one periodic axis (spectral along it,
    tridiagonal across the walls): phi and E within 1e-12 of the oracle, which
    is bit-exact with the reference on the golden meshes."""
    rng = np.random.default_rng(sum(n) + axis)
    nx, ny = n
    rho = 1e-6 * (1.0 + 0.3 * rng.standard_normal((ny, nx)))
    eps = 8.8541878128e-12
    phi, E = apic.field_solve_mixed_2d(n, L, axis, eps, walls[0], walls[1], rho)
    pr, Er = po.solve_mixed_2d(rho, n, L, axis, eps, walls[0], walls[1])
    assert rel_max(phi, pr) < TOL
    assert rel_max(E, Er) < TOL


def test_mixed_solve_rejects_unsupported_meshes():
    with pytest.raises(apic.ApicError):
        apic.field_solve_mixed_2d((24, 9), (1.0, 1.0), 0, 1.0, 0.0, 0.0, np.zeros(24 * 9))  # periodic 24
    with pytest.raises(apic.ApicError):
        apic.field_solve_mixed_2d((16, 2), (1.0, 1.0), 0, 1.0, 0.0, 0.0, np.zeros(32))  # two wall nodes


def test_sort_keeps_identity_and_fields():
    """Sorting every step versus never: identical particles (by load order) and fields."""
    wl = W.plasma_2d(cells=(32, 32), ppc=4, seed=8)
    dev_a, _ = run_pair(wl, 6, sort_interval=1)
    cfg = W.to_device_config_nd(wl, sort_interval=1000)
    dev_b = apic.SimulationND(cfg)
    for k, (q, m, w, pos, v) in enumerate(wl.species):
        dev_b.load(k, pos, v)
    dev_b.initialize()
    dev_b.step(6)
    for k in range(2):
        for x, y in zip(dev_a.particles(k), dev_b.particles(k)):
            assert np.array_equal(x, y)
    for x, y in zip(dev_a.fields(), dev_b.fields()):
        assert np.array_equal(x, y)  # fixed-point deposit: independent of particle order


@pytest.mark.parametrize("case", ["2d_boris", "3d_boris"])
def test_fp32_form_against_fp64_oracle(case):
    """FP32 particles (packed cell + float offsets + float velocities) against the
    FP64 oracle on the same inputs: positions within 1e-5 of a cell, velocities
    within 1e-5 of the thermal scale, fields within 1e-4 (max-norm relative)."""
    wl = W.plasma_2d(cells=(32, 16), ppc=8, seed=3) if case == "2d_boris" else W.plasma_3d(cells=(16, 8, 8), ppc=4, seed=5)
    steps = 10
    cfg = W.to_device_config_nd(wl, precision=apic.FP32, sort_interval=4)
    dev = apic.SimulationND(cfg)
    eps = 8.8541878128e-12
    ora = po.SimND(wl.dims, wl.n, wl.length, wl.dt, eps, wl.B, [(q, m, w) for (q, m, w, pos, v) in wl.species])
    for k, (q, m, w, pos, v) in enumerate(wl.species):
        dev.load(k, pos, v)
        ora.load(k, pos, v, v)
    dev.initialize()
    ora.initialize()
    dev.step(steps)
    ora.step(steps)
    for k in range(2):
        a, b = dev.particles(k), ora.particles(k)
        cell = wl.length[0] / wl.n[0]
        dpos = np.abs(a[0][: wl.dims] - b[0][: wl.dims])
        dpos = np.minimum(dpos, np.array(wl.length)[: wl.dims, None] - dpos)  # periodic distance
        assert dpos.max() < 1e-5 * cell, (k, dpos.max() / cell)
        vs = np.max(np.abs(b[2]))
        assert np.max(np.abs(a[2] - b[2])) < 1e-5 * vs
    fa, fb = dev.fields(), ora.fields()
    for name, x, y in zip(("rho", "phi", "E"), fa, fb):
        assert rel_max(x, y) < 1e-4, (name, rel_max(x, y))


def test_fp32_energy_conservation_2d():
    """A larger FP32 2D run conserves total energy like the FP64 form does."""
    wl = W.plasma_2d(cells=(64, 64), ppc=16, seed=21)
    res = {}
    for prec in (apic.FP64, apic.FP32):
        dev = apic.SimulationND(W.to_device_config_nd(wl, precision=prec))
        for k, (q, m, w, pos, v) in enumerate(wl.species):
            dev.load(k, pos, v)
        dev.initialize()
        e0 = dev.sample().total_energy
        dev.step(50)
        e1 = dev.sample().total_energy
        res[prec] = (e0, e1)
    drift64 = abs(res[apic.FP64][1] - res[apic.FP64][0]) / res[apic.FP64][0]
    drift32 = abs(res[apic.FP32][1] - res[apic.FP32][0]) / res[apic.FP32][0]
    assert abs(res[apic.FP32][0] - res[apic.FP64][0]) < 1e-5 * res[apic.FP64][0]
    assert drift32 < max(2 * drift64, 1e-4), (drift32, drift64)


@pytest.mark.parametrize("dims,cells,ppc,sort_interval,steps", [
    (2, (64, 64), 16, 4, 9), (3, (16, 16, 16), 8, 4, 9), (3, (32, 32, 32), 8, 1000, 30)])
def test_push_items_leave_results_unchanged(dims, cells, ppc, sort_interval, steps):
    """The FP32 push's particles-per-thread knob changes only speed: every
    setting (one particle per thread, the shared-memory box pushes at 2 and 4,
    8 per thread) gives the same particles and fields, also when the particles
    have drifted far from their sorted order (sorted once, 30 steps: many
    gather and deposit outside their CTA's box)."""
    plan = W.plasma_plan(dims, cells=cells, ppc=ppc, seed=4)
    ref = None
    for items in (1, 2, 4, 8):
        sim = apic.SimulationND(plan.config(precision=apic.FP32, sort_interval=sort_interval, push_items=items))
        plan.load(sim)
        sim.initialize()
        sim.step(steps)
        got = [sim.particles(k) for k in range(2)] + [sim.fields()]
        sim.close()
        if ref is None:
            ref = got
        else:
            for a, b in zip(got, ref):
                for x, y in zip(a, b):
                    assert np.array_equal(x, y), items


def test_autotuner_returns_a_candidate():
    """The autotuner returns one of the candidates with its timing table."""
    from apic import autotune
    plan = W.plasma_plan(2, cells=(64, 64), ppc=16, seed=4)
    out = autotune.tune_plasma(plan, apic.FP32, sort_intervals=(4, 8), push_items=(1, 4), steps=8)
    assert out["sort_interval"] in (4, 8) and out["push_items"] in (1, 4)
    assert len(out["table"]) == 4 and all(r["ms_per_step"] > 0 for r in out["table"])


def _with_profile(cfg, axis, coords, values):
    """Switch a device config to a tabulated B (uniform B cleared)."""
    import ctypes as C
    pc = np.ascontiguousarray(coords, dtype=np.float64)
    pv = np.ascontiguousarray(values, dtype=np.float64).ravel()
    cfg._profile_keep = (pc, pv)
    cfg.magnetic_field[:] = [0.0, 0.0, 0.0]
    cfg.profile_axis, cfg.profile_rows = axis, pc.size
    cfg.profile_coordinates = pc.ctypes.data_as(C.POINTER(C.c_double))
    cfg.profile_values = pv.ctypes.data_as(C.POINTER(C.c_double))
    return cfg


def _profile_for(wl, axis, rows=11):
    Lax = wl.length[axis] if axis < wl.dims else 0.0
    c = np.linspace(0.0, Lax if Lax > 0 else 1.0, rows) ** 1.0
    if axis >= wl.dims:
        c = np.linspace(-1.0, 1.0, rows)
    B0 = np.linalg.norm(wl.B) or 0.01
    u = c / (np.max(np.abs(c)) or 1.0)
    v = np.stack([0.3 * B0 * np.sin(2.0 * u), 0.1 * B0 + 0.0 * u, B0 * (1.0 + 0.5 * np.cos(3.0 * u))], axis=1)
    return c, v


@pytest.mark.parametrize("dims,axis", [(2, 0), (2, 1), (2, 2), (3, 2), (3, 0)])
def test_tabulated_magnetic_field_parity(dims, axis):
    """magnetic_field_profile: B piecewise linear along one axis, evaluated at
    each particle in every Boris kick.  FP64 form against the oracle (bit-exact
    with the reference on the golden runs) within 1e-12; FP32 form within the
    FP32 bounds of the uniform-B case."""
    wl = W.plasma_2d(cells=(32, 16), ppc=8, seed=3) if dims == 2 else W.plasma_3d(cells=(16, 8, 8), ppc=4, seed=5)
    c, v = _profile_for(wl, axis)
    eps = 8.8541878128e-12
    for prec in (apic.FP64, apic.FP32):
        cfg = _with_profile(W.to_device_config_nd(wl, precision=prec, sort_interval=4), axis, c, v)
        dev = apic.SimulationND(cfg)
        ora = po.SimND(wl.dims, wl.n, wl.length, wl.dt, eps, (0.0, 0.0, 0.0),
                       [(q, m, w) for (q, m, w, pos, vv) in wl.species])
        ora.set_profile(axis, c, v)
        for k, (q, m, w, pos, vv) in enumerate(wl.species):
            dev.load(k, pos, vv)
            ora.load(k, pos, vv, vv)
        dev.initialize()
        ora.initialize()
        dev.step(10)
        ora.step(10)
        for k in range(2):
            a, b = dev.particles(k), ora.particles(k)
            if prec == apic.FP64:
                for name, x, y in zip(("pos", "v", "vh"), a, b):
                    x, y = (x[: wl.dims], y[: wl.dims]) if name == "pos" else (x, y)
                    assert rel_max(x, y) < TOL, (dims, axis, k, name, rel_max(x, y))
            else:
                cell = wl.length[0] / wl.n[0]
                dpos = np.abs(a[0][: wl.dims] - b[0][: wl.dims])
                dpos = np.minimum(dpos, np.array(wl.length)[: wl.dims, None] - dpos)
                assert dpos.max() < 1e-5 * cell, (dims, axis, k, dpos.max() / cell)
                assert np.max(np.abs(a[2] - b[2])) < 1e-5 * np.max(np.abs(b[2]))
        if prec == apic.FP64:
            for name, x, y in zip(("rho", "phi", "E"), dev.fields(), ora.fields()):
                assert rel_max(x, y) < TOL, (name, rel_max(x, y))
        dev.close()


def test_tabulated_magnetic_field_rejections():
    wl = W.plasma_2d(cells=(16, 16), ppc=2, seed=3)
    c, v = _profile_for(wl, 0)
    cfg = W.to_device_config_nd(wl)
    cfg = _with_profile(cfg, 0, c, v)
    cfg.magnetic_field[:] = [0.0, 0.0, 0.01]
    with pytest.raises(apic.ApicError, match="mutually exclusive"):
        apic.SimulationND(cfg)
    short = _with_profile(W.to_device_config_nd(wl), 0, c[:-2], v[:-2])  # stops before length_x
    with pytest.raises(apic.ApicError, match="cover"):
        apic.SimulationND(short)


def test_particle_state_file_drives_a_device_run(tmp_path):
    """An .aps initial state (written, then parsed by the library) loaded into a
    2D3V device run gives the oracle's run on the same records (1e-12)."""
    wl = W.plasma_2d(cells=(32, 16), ppc=4, seed=9)
    names = ["electrons", "ions"]
    sp = {names[k]: (np.asarray(pos, dtype=np.float64), np.asarray(v, dtype=np.float64))
          for k, (q, m, w, pos, v) in enumerate(wl.species)}
    for k in sp:
        p3 = np.zeros((3, sp[k][0].shape[1]))
        p3[:2] = sp[k][0][:2]
        sp[k] = (p3, sp[k][1])
    path = str(tmp_path / "init.aps")
    apic.ParticleState.write(path, 2, apic.SI, sp)
    st = apic.ParticleState(path)
    assert st.dimension == 2 and sorted(st.species) == names
    cfg = W.to_device_config_nd(wl, sort_interval=4)
    dev = apic.SimulationND(cfg)
    ora = po.SimND(wl.dims, wl.n, wl.length, wl.dt, 8.8541878128e-12, wl.B,
                   [(q, m, w) for (q, m, w, pos, v) in wl.species])
    for k, name in enumerate(names):
        pos, vel = st.species[name]
        dev.load(k, pos, vel)
        ora.load(k, pos, vel, vel)
    dev.initialize()
    ora.initialize()
    dev.step(5)
    ora.step(5)
    for k in range(2):
        a, b = dev.particles(k), ora.particles(k)
        for name, x, y in zip(("pos", "v", "vh"), a, b):
            x, y = (x[:2], y[:2]) if name == "pos" else (x, y)
            assert rel_max(x, y) < TOL, (k, name)


def _exact_dirichlet(rho, n, L, eps, pot):
    """Direct sparse solve of the same discrete Dirichlet system (5/7-point
    Laplacian, wall potentials on the neighbours of the walls)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    dims = len(n)
    h = [L[a] / (n[a] - 1) for a in range(dims)]
    M = [n[a] - 2 for a in range(dims)]
    ops = []
    for a in range(dims):
        d = sp.diags([-np.ones(M[a] - 1), 2 * np.ones(M[a]), -np.ones(M[a] - 1)], [-1, 0, 1]) / h[a] ** 2
        mats = [sp.identity(M[b]) if b != a else d for b in range(dims)]
        k = mats[dims - 1]
        for b in range(dims - 2, -1, -1):
            k = sp.kron(k, mats[b])
        ops.append(k)
    A = sum(ops).tocsc()
    full = np.zeros(tuple(reversed(n)))
    if dims == 2:
        left, right, bottom, top = pot
        full[:, 0], full[:, -1], full[0, :], full[-1, :] = left, right, bottom, top
        full[0, 0], full[0, -1] = 0.5 * (left + bottom), 0.5 * (right + bottom)
        full[-1, 0], full[-1, -1] = 0.5 * (left + top), 0.5 * (right + top)
    r = np.asarray(rho).reshape(tuple(reversed(n)))
    inner = tuple(slice(1, -1) for _ in range(dims))
    b = r[inner] / eps
    if dims == 2:
        b = b.copy()
        b[:, 0] += full[1:-1, 0] / h[0] ** 2
        b[:, -1] += full[1:-1, -1] / h[0] ** 2
        b[0, :] += full[0, 1:-1] / h[1] ** 2
        b[-1, :] += full[-1, 1:-1] / h[1] ** 2
    full[inner] = spl.spsolve(A, b.ravel()).reshape(b.shape)
    return full.ravel()


@pytest.mark.parametrize("n,L,pot", [((17, 9), (0.02, 0.01), (0.0, 50.0, -10.0, 5.0)),
                                     ((65, 33), (0.03, 0.01), (100.0, 0.0, 0.0, 20.0)),
                                     ((9, 5, 9), (0.01, 0.005, 0.01), None),
                                     ((33, 17, 9), (0.02, 0.01, 0.005), None)])
def test_dirichlet_solve_against_exact_and_reference_sor(n, L, pot):
    """Walls on every side: the direct device solve equals the exact solution of
    the discrete system within 1e-12 and the reference's SOR result (the oracle,
    bit-exact with the reference on the golden meshes) within 1e-8, the SOR
    convergence of a 1e-11 update."""
    rng = np.random.default_rng(len(n) * 100 + n[0])
    N = int(np.prod(n))
    rho = 1e-6 * (1.0 + 0.3 * rng.standard_normal(N))
    eps = 8.8541878128e-12
    phi, E = apic.field_solve_dirichlet_nd(n, L, eps, rho, pot)
    exact = _exact_dirichlet(rho, n, L, eps, pot if pot is not None else (0.0,) * 4)
    assert rel_max(phi, exact) < TOL
    pr, Er = po.solve_dirichlet_nd(rho, n, L, eps, pot)
    assert rel_max(phi, pr) < 1e-8
    assert rel_max(E, Er) < 1e-7


def test_dirichlet_solve_rejects_other_extents():
    with pytest.raises(apic.ApicError, match="2\\^k \\+ 1"):
        apic.field_solve_dirichlet_nd((16, 9), (1.0, 1.0), 1.0, np.zeros(16 * 9))


# ---- 2D runs with walls ---------------------------------------------------------

WALL_SPECIES = [(-1.0, 1.0, 0.05, 400), (1.0, 50.0, 0.05, 400)]


def _walls_pair(name):
    from golden.make_golden import WALL_CASES
    n, B, d, pot, pb = WALL_CASES[name]
    f = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", f"{name}.npz"))
    # the device's particle-boundary codes: 0 auto, 1 absorbing, 2 reflecting, 3 periodic
    dev_pb = [3 if k == 0 else k for k in pb]
    cfg = apic.config_nd(dims=2, n=n, length=(4.0, 2.0), dt=0.1, magnetic_field=B,
                         species=[(q, m, w, cap) for q, m, w, cap in WALL_SPECIES], walls=(d, pot, dev_pb))
    dev = apic.SimulationND(cfg)
    ora = po.SimND(2, n, (4.0, 2.0), 0.1, 1.0, B, [(q, m, w) for q, m, w, _ in WALL_SPECIES])
    ora.set_walls(d, pot, pb)
    for k in range(2):
        pos, v, vh = f[f"init_s{k}_pos"], f[f"init_s{k}_v"], f[f"init_s{k}_vh"]
        dev.load(k, pos[:2], v, vh)
        ora.load(k, pos, v, vh)
    dev.resume(0.0, 0)
    ora.initialize_fields()
    return dev, ora, f


@pytest.mark.parametrize("name,tol", [("sim2d_walls_mixed", 1e-12), ("sim2d_walls_dirichlet", 1e-6)])
def test_2d_walls_against_oracle(name, tol):
    """2D runs with walls on the device against the oracle (bit-exact with the
    reference): one wall axis (mixed solve) within 1e-12; walls on every side
    within 1e-6, since the device solves the discrete system directly while the
    reference's SOR stops at a 1e-11 update (about 1e-8 in the potential).
    Absorbed particles and the per-side loss counts exact."""
    dev, ora, f = _walls_pair(name)
    dev.step(25)
    ora.step(25)
    for k in range(2):
        al, lo = ora.alive_losses(k)
        assert np.array_equal(dev.alive(k), al), (name, k)
        assert np.array_equal(dev.boundary_losses(k), lo), (name, k)
        dpos, _, dvh = dev.particles(k)
        opos, _, ovh = ora.particles(k)
        keep = al == 1
        assert rel_max(dpos[:2][:, keep], opos[:2][:, keep]) < tol, (name, k)
        assert rel_max(dvh[:, keep], ovh[:, keep]) < tol, (name, k)
    assert f["losses_s0"].sum() > 0


def _walls3_pair(name):
    from golden.make_golden import WALL3_CASES, WALL3_LENGTH
    n, B, pb = WALL3_CASES[name]
    f = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", f"{name}.npz"))
    dev_pb = [3 if k == 0 else k for k in pb]  # device codes: 0 auto, 1 absorbing, 2 reflecting, 3 periodic
    cfg = apic.config_nd(dims=3, n=n, length=WALL3_LENGTH, dt=0.1, magnetic_field=B,
                         species=[(q, m, w, cap) for q, m, w, cap in WALL_SPECIES], walls=((1, 1, 1), None, dev_pb))
    dev = apic.SimulationND(cfg)
    ora = po.SimND(3, n, WALL3_LENGTH, 0.1, 1.0, B, [(q, m, w) for q, m, w, _ in WALL_SPECIES])
    ora.set_walls3d(pb)
    for k in range(2):
        pos, v, vh = f[f"init_s{k}_pos"], f[f"init_s{k}_v"], f[f"init_s{k}_vh"]
        dev.load(k, pos, v, vh)
        ora.load(k, pos, v, vh)
    dev.resume(0.0, 0)
    ora.initialize_fields()
    return dev, ora, f


@pytest.mark.parametrize("name", ["sim3d_walls_boris", "sim3d_walls_leapfrog"])
def test_3d_walls_against_oracle(name):
    """3D runs on a Dirichlet mesh (grounded walls on every side) against the
    oracle, which is bit-exact with the reference's Simulation3D: positions and
    v_half of the live particles within 1e-6 (the device solves the discrete
    Poisson system directly while the reference's SOR stops at a 1e-11 update),
    alive flags and the per-side loss counts exact (their sum over the species
    is the reference's run ledger), live counts of sample() exact."""
    dev, ora, f = _walls3_pair(name)
    dev.step(25)
    ora.step(25)
    total = np.zeros(6, np.uint64)
    live = 0
    for k in range(2):
        al, lo = ora.alive_losses(k)
        total += lo
        live += int(al.sum())
        assert np.array_equal(dev.alive(k), al), (name, k)
        assert np.array_equal(dev.boundary_losses(k), lo), (name, k)
        dpos, _, dvh = dev.particles(k)
        opos, _, ovh = ora.particles(k)
        keep = al == 1
        assert rel_max(dpos[:, keep], opos[:, keep]) < 1e-6, (name, k)
        assert rel_max(dvh[:, keep], ovh[:, keep]) < 1e-6, (name, k)
    assert np.array_equal(total, f["losses_s0"]) and total.sum() > 0
    assert dev.sample().live_particles == live
    rho_d, phi_d, E_d = dev.fields()
    rho_o, phi_o, E_o = ora.fields()
    assert rel_max(rho_d, rho_o) < 1e-6
    assert rel_max(phi_d, phi_o) < 1e-6
    assert rel_max(E_d, E_o[:3]) < 1e-6
    dev.close()


def test_2d_walls_sample_counts_live_particles():
    """sample().live_particles leaves out absorbed particles (live_count,
    src/Diagnostics.cpp:111-137)."""
    dev, ora, _ = _walls_pair("sim2d_walls_dirichlet")
    dev.step(25)
    ora.step(25)
    live = sum(int(ora.alive_losses(k)[0].sum()) for k in range(2))
    assert live < 800 and dev.sample().live_particles == live
    dev.close()


def test_small_solve_does_not_break_a_large_simulation():
    """The FFT kernels' shared-memory limit belongs to the kernel functions and
    is shared by every simulation in the process: a small stand-alone solve made
    after a 512^2 simulation was created must leave that simulation steppable."""
    plan = W.plasma_plan(2, cells=(512, 512), ppc=1, seed=4)
    sim = apic.SimulationND(plan.config(precision=apic.FP64, sort_interval=16))
    plan.load(sim)
    sim.initialize()
    rng = np.random.default_rng(9)
    apic.field_solve_periodic_nd(2, (64, 64), (1.0, 1.0), 1.0, rng.standard_normal(64 * 64))
    sim.step(2)
    sim.synchronize()
    assert sim.sample().step == 2
    sim.close()
