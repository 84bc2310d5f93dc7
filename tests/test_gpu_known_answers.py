"""The reference's own analytic known-answer tests, run on the device through
the C ABI (tests/test_core.cpp of the reference: the spectral Poisson
benchmarks :980-1066 and the permittivity contract :267-300, the MCC
envelopes :336-432, the constant-acceleration leapfrog :1068-1107, the Boris
cyclotron rotations :1220-1358, the CIC deposit checks :1874-1966 and
:2133-2146 and the zero-cross-section swarm :6187-6233), with the reference's
tolerances where the device runs the same operation.  The periodic device
solve takes power-of-two extents, so the Poisson and CIC benchmarks use
power-of-two meshes near the reference's, with the same Fourier modes and
particle positions."""
import math

import numpy as np
import pytest

import apic
from apic import workloads as W

pytestmark = pytest.mark.gpu


def _nodes(n, L):
    return [np.arange(k) * (l / k) for k, l in zip(n, L)]  # periodic node positions, Mesh2D/3D::node_x


def test_poisson_2d_sine_cosine_benchmark():
    """rho = sin(kx x) cos(ky y): phi = rho / k^2 and E = -grad phi at every node
    within 1e-12 (the reference's M1 2D benchmark, on 16 x 8 nodes)."""
    n, L = (16, 8), (1.0, 1.5)
    kx, ky = 2 * math.pi * 2 / L[0], 2 * math.pi * 3 / L[1]
    k2 = kx * kx + ky * ky
    x, y = _nodes(n, L)
    X, Y = np.meshgrid(x, y)  # [ny][nx]: index j * nx + i
    rho = (np.sin(kx * X) * np.cos(ky * Y)).ravel()
    phi, E = apic.field_solve_periodic_nd(2, n, L, 1.0, rho)
    assert np.max(np.abs(phi - rho / k2)) < 1e-12
    assert np.max(np.abs(E[0] - (-kx * np.cos(kx * X) * np.cos(ky * Y) / k2).ravel())) < 1e-12
    assert np.max(np.abs(E[1] - (ky * np.sin(kx * X) * np.sin(ky * Y) / k2).ravel())) < 1e-12


def test_poisson_3d_sine_cosine_benchmark():
    """rho = sin(kx x) cos(ky y) sin(kz z) on 8 x 8 x 16 nodes: phi and the three
    field components within 1e-12 (the reference's M1 3D benchmark)."""
    n, L = (8, 8, 16), (1.0, 1.25, 1.5)
    kx, ky, kz = 2 * math.pi * 1 / L[0], 2 * math.pi * 2 / L[1], 2 * math.pi * 3 / L[2]
    k2 = kx * kx + ky * ky + kz * kz
    x, y, z = _nodes(n, L)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")  # [nz][ny][nx]
    sx, cx, sy, cy, sz, cz = np.sin(kx * X), np.cos(kx * X), np.sin(ky * Y), np.cos(ky * Y), np.sin(kz * Z), np.cos(kz * Z)
    rho = (sx * cy * sz).ravel()
    phi, E = apic.field_solve_periodic_nd(3, n, L, 1.0, rho)
    assert np.max(np.abs(phi - rho / k2)) < 1e-12
    assert np.max(np.abs(E[0] - (-kx * cx * cy * sz / k2).ravel())) < 1e-12
    assert np.max(np.abs(E[1] - (ky * sx * sy * sz / k2).ravel())) < 1e-12
    assert np.max(np.abs(E[2] - (-kz * sx * cy * cz / k2).ravel())) < 1e-12


def test_poisson_field_scales_inversely_with_permittivity():
    """A doubled permittivity halves the field (1e-13), as the reference's
    FieldSolver(2.0) against FieldSolver()."""
    n, L = (32, 16), (1.0, 1.0)
    x, y = _nodes(n, L)
    X, Y = np.meshgrid(x, y)
    rho = (np.sin(2 * math.pi * X) + 0.3 * np.cos(4 * math.pi * Y)).ravel()
    _p1, E1 = apic.field_solve_periodic_nd(2, n, L, 1.0, rho)
    _p2, E2 = apic.field_solve_periodic_nd(2, n, L, 2.0, rho)
    assert np.max(np.abs(E2 - 0.5 * E1)) < 1e-13


def test_leapfrog_constant_acceleration_through_the_1d_step():
    """A charge-free test particle between electrodes at 0 and -5 V over 2 m
    (uniform E = 2.5, q/m = 1) follows x0 + v0 t + a t^2 / 2 and v0 + a t after
    8 steps of 0.125 (the reference's 1D leapfrog benchmark: initialize, then
    kick, drift, synchronize each step), within 1e-12."""
    dt, a, x0, v0 = 0.125, 2.5, 0.2, -0.4
    cfg = apic.config1d(boundary=apic.DIRICHLET, velocity_dimensions=1, units=apic.NORMALIZED, nx=33, length=2.0,
                        dt=dt, species=[(1.0, 1.0, 0.0, 16)], phi_left=0.0, phi_right=-5.0)
    sim = apic.Simulation1D(cfg)
    sim.load(0, [x0], [v0])
    sim.initialize()
    sim.step(8)
    p = sim.particles(0)
    t = 8 * dt
    assert abs(p["x"][0] - (x0 + v0 * t + 0.5 * a * t * t)) < 1e-12
    assert abs(p["v"][0] - (v0 + a * t)) < 1e-12
    sim.close()


def _boris_angle(b, qm, dt):
    """The Boris rotation per step about B, -2 atan(q B dt / 2 m)."""
    return -2.0 * math.atan(0.5 * qm * b * dt)


def _rotate(v, axis, angle):
    c, s = math.cos(angle), math.sin(angle)
    return v * c + np.cross(axis, v) * s + axis * np.dot(axis, v) * (1.0 - c)


def _gyrate(dims, B, qm, dt, steps, v0):
    """One test particle of weight 1e-30 (no self-field) in uniform B on a
    periodic mesh: its time-centred velocity after `steps` FP64 steps."""
    n = (8,) * dims
    cfg = apic.config_nd(dims=dims, n=n, length=(1.0,) * dims, dt=dt, species=[(qm, 1.0, 1e-30, 16)],
                         magnetic_field=B)
    sim = apic.SimulationND(cfg)
    pos = np.full((3, 1), 0.25)
    sim.load(0, pos, np.array(v0, dtype=np.float64).reshape(3, 1))
    sim.initialize()
    sim.step(steps)
    sim.synchronize()
    v = sim.particles(0)[1][:, 0].copy()
    sim.close()
    return v


def test_boris_cyclotron_rotation_2d():
    """The reference's M5 run: a 2D periodic simulation with uniform Bz = 1.7,
    q/m = 1.25, dt = 0.04; after 37 steps the velocity is the initial one
    rotated by 37 Boris angles, speed conserved (1e-10)."""
    dt, steps, qm, bz = 0.04, 37, 1.25, 1.7
    v0 = np.array([0.8, -0.35, 0.0])
    v = _gyrate(2, (0.0, 0.0, bz), qm, dt, steps, v0)
    ang = steps * _boris_angle(abs(bz), qm, dt)
    assert abs(v[0] - (v0[0] * math.cos(ang) - v0[1] * math.sin(ang))) < 1e-10
    assert abs(v[1] - (v0[0] * math.sin(ang) + v0[1] * math.cos(ang))) < 1e-10
    assert abs(np.hypot(v[0], v[1]) - np.hypot(v0[0], v0[1])) < 1e-10


@pytest.mark.parametrize("dims", [3, 2])
def test_boris_arbitrary_axis_rotation(dims):
    """B = (0.4, -0.8, 1.1), q/m = -0.75, dt = 0.03, 29 steps: the velocity is
    the initial one rotated about B by 29 Boris angles, with speed and the
    parallel component conserved (3D3V and 2D3V, 1e-10)."""
    dt, steps, qm = 0.03, 29, -0.75
    B = np.array([0.4, -0.8, 1.1])
    v0 = np.array([0.6, -0.25, 0.9])
    v = _gyrate(dims, tuple(B), qm, dt, steps, v0)
    bm = np.linalg.norm(B)
    axis = B / bm
    expected = _rotate(v0, axis, steps * _boris_angle(bm, qm, dt))
    assert np.max(np.abs(v - expected)) < 1e-10
    assert abs(np.linalg.norm(v) - np.linalg.norm(v0)) < 1e-10
    assert abs(np.dot(v, axis) - np.dot(v0, axis)) < 1e-10


def test_zero_cross_section_swarm_drift_and_energy():
    """Four electrons at rest in a gas that never collides (1 Td at 1e20 m^-3,
    0.1 V/m), 6 steps of 1e-8 s after 2 burn-in steps: drift 4.5 a dt and mean
    energy m (a dt)^2 21.5 / (2 e) within 1e-13 relative, no longitudinal
    diffusion and no collisions (the reference's zero-cross-section swarm)."""
    me, e = 9.1093837139e-31, 1.602176634e-19
    energy = np.array([0.0, 1.0, 50.0]) * e
    gas = [W.ChannelSpec(W.ELASTIC, energy, np.zeros(3))]
    spec = W.SwarmSpec("zero_sigma", gas, 6.6335209e-26, 1e20, 300.0, 1e6, 1e-8, 6, 2, 4, [1.0],
                       uncertainty_blocks=2, initial_mean_energy_ev=0.0, max_energy_ev=1.0, seed=17)
    cfg, g, _tabs = W.to_device_swarm(spec, apic.FP64)
    r = apic.swarm_run(cfg, g, spec.fields_td)[0]
    assert r.status == 0, r.message
    adt = e * 0.1 / me * 1e-8
    assert abs(r.drift_velocity - 4.5 * adt) <= 1e-13 * 4.5 * adt, (r.drift_velocity, 4.5 * adt)
    mean = 0.5 * me * adt * adt * 21.5 / e
    assert abs(r.mean_energy_ev - mean) <= 1e-13 * mean, (r.mean_energy_ev, mean)
    assert abs(r.diffusion_longitudinal) <= 1e-30
    assert r.channel_collisions[0] == 0


def test_cic_1d_dirichlet_boundary_half_volume():
    """A particle on the left electrode (charge 2, weight 0.5, 5 nodes over
    1 m) puts its whole charge on node 0 over half a control volume: rho[0] = 8
    and the charge is conserved (the reference's 1D Dirichlet CIC check, 1e-12)."""
    rho, _phi, _E, _eq = apic.deposit_solve_gather_1d(apic.DIRICHLET, 5, 1.0, 1.0, 0.0, 0.0, [2.0], [0.5],
                                                      [np.array([0.0])])
    vol = np.full(5, 0.25)
    vol[0] = vol[-1] = 0.125
    assert abs(rho[0] - 8.0) < 1e-12
    assert abs(np.sum(rho * vol) - 1.0) < 1e-12


def _deposit_nd(n, L, charge, weight, pos):
    """rho of the periodic FP64 mesh after loading particles at `pos` ([dims][k])."""
    dims = len(n)
    cfg = apic.config_nd(dims=dims, n=n, length=L, dt=0.1, species=[(charge, 1.0, weight, 16)])
    sim = apic.SimulationND(cfg)
    pos = np.asarray(pos, dtype=np.float64)
    p3 = np.zeros((3, pos.shape[1]))
    p3[:dims] = pos
    sim.load(0, p3, np.zeros((3, pos.shape[1])))
    sim.initialize()
    rho = sim.fields()[0]
    sim.close()
    return rho


@pytest.mark.parametrize("dims", [2, 3])
def test_cic_wrapped_deposit(dims):
    """Two live particles of charge 2 x weight 0.5 on a periodic 4^dims mesh,
    one of them outside the box (wrapped): the weights on the corner, x, y (and
    z) nodes and the total charge of the reference's CIC check (1e-12)."""
    n = (4,) * dims
    if dims == 2:
        rho = _deposit_nd(n, (1.0, 1.0), 2.0, 0.5, [[0.125, 1.125], [0.125, -0.125]])
        idx = lambda i, j: j * 4 + i
        assert abs(rho[idx(0, 0)] - 8.0) < 1e-12 and abs(rho[idx(1, 0)] - 8.0) < 1e-12
        assert abs(rho[idx(0, 1)] - 4.0) < 1e-12
        assert abs(rho.sum() * 0.25 * 0.25 - 2.0) < 1e-12
    else:
        rho = _deposit_nd(n, (1.0, 1.0, 1.0), 2.0, 0.5, [[0.125, 1.125], [0.125, -0.125], [0.125, 0.875]])
        idx = lambda i, j, k: (k * 4 + j) * 4 + i
        assert abs(rho[idx(0, 0, 0)] - 16.0) < 1e-12 and abs(rho[idx(1, 0, 0)] - 16.0) < 1e-12
        assert abs(rho[idx(0, 1, 0)] - 8.0) < 1e-12 and abs(rho[idx(0, 0, 3)] - 8.0) < 1e-12
        assert abs(rho.sum() * 0.25 ** 3 - 2.0) < 1e-12


@pytest.mark.parametrize("dims", [2, 3])
def test_cic_exact_shape_function(dims):
    """One interior particle: the 4 (8) node densities are the bilinear
    (trilinear) shape-function weights of the reference's M1 CIC benchmark and
    the charge is conserved (1e-12; power-of-two meshes)."""
    if dims == 2:
        n, L, pos, q, w = (8, 8), (1.0, 1.5), (0.31, 0.44), -1.5, 2.0
    else:
        n, L, pos, q, w = (8, 8, 4), (1.2, 1.0, 0.8), (0.37, 0.46, 0.51), 1.25, 0.8
    d = [l / k for l, k in zip(L, n)]
    rho = _deposit_nd(n, L, q, w, [[p] for p in pos])
    g = [p / dd for p, dd in zip(pos, d)]
    i0 = [int(math.floor(x)) for x in g]
    f = [x - i for x, i in zip(g, i0)]
    expected = np.zeros(int(np.prod(n)))
    cellvol = float(np.prod(d))
    for corner in range(1 << dims):
        w_c, idx, stride = 1.0, 0, 1
        for a in range(dims):
            b = (corner >> a) & 1
            w_c *= f[a] if b else 1.0 - f[a]
            idx += ((i0[a] + b) % n[a]) * stride
            stride *= n[a]
        expected[idx] += q * w * w_c / cellvol
    assert np.max(np.abs(rho - expected)) < 1e-12
    assert abs(rho.sum() * cellvol - q * w) < 1e-12


def _elastic_model(angular=False):
    """The reference's envelope gas: sigma(E) on the table (0, 0), (1, 0.5),
    (2, 1), neutral density 1, max_frequency 2, infinitely heavy neutrals
    (neutral_mass 0), unit particle mass; Henyey-Greenstein with a constant
    mean cosine 0.8 when `angular`."""
    tabs = apic.Tables()
    kw = dict(angular=apic.HENYEY_GREENSTEIN, mu_energy=[0.0, 2.0], mu=[0.8, 0.8]) if angular else {}
    ch = tabs.channel(W.ELASTIC, [0.0, 1.0, 2.0], [0.0, 0.5, 1.0], **kw)
    return apic.mcc_model(0, [ch], 1.0, 2.0, 0.0, 0.0, 0, 64), tabs


def test_mcc_elastic_envelopes():
    """10000 collide calls at |v| = sqrt(2) over dt = 0.1 (the reference's MCC
    envelope checks, on the device's Philox streams): candidates within
    (1800, 2200), accepted elastic collisions within (620, 800), the speed kept
    to 1e-14 and the scattered directions isotropic."""
    m, _tabs = _elastic_model()
    n = 10000
    v0 = np.zeros((n, 3))
    v0[:, 0] = math.sqrt(2.0)
    v, stats = apic.collide3(m, 1.0, v0, 0.1, seed=8128, step=0, stream=0)
    cand = sum(s.candidates for s in stats)
    hits = np.array([s.channel_collisions[0] for s in stats])
    assert 1800 < cand < 2200, cand
    assert 620 < hits.sum() < 800, hits.sum()
    assert np.max(np.abs(np.linalg.norm(v, axis=1) - math.sqrt(2.0))) < 1e-14
    mean_dir = (v[hits > 0] / math.sqrt(2.0)).sum(axis=0)
    assert np.all(np.abs(mean_dir) < 0.1 * hits.sum()), mean_dir


def test_mcc_henyey_greenstein_mean_cosine():
    """20000 calls with Henyey-Greenstein scattering of mean cosine 0.8: the
    particles scattered exactly once keep the configured mean cosine within
    0.04 and their speed to 1e-14 (the reference's anisotropic envelope)."""
    m, _tabs = _elastic_model(angular=True)
    n = 20000
    v0 = np.zeros((n, 3))
    v0[:, 0] = math.sqrt(2.0)
    v, stats = apic.collide3(m, 1.0, v0, 0.1, seed=161803, step=0, stream=0)
    once = np.array([s.channel_collisions[0] == 1 for s in stats])
    assert np.max(np.abs(np.linalg.norm(v, axis=1) - math.sqrt(2.0))) < 1e-14
    assert once.sum() > 1200
    assert abs(np.mean(v[once, 0] / math.sqrt(2.0)) - 0.8) < 0.04
