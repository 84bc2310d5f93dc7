"""Synthetic inputs for the named workloads of the particle step.

Every workload is seeded and fully determined by its arguments.  The same
arrays feed the device library, the CPU oracle and the reference harness, so
parity tests and benchmarks run on identical inputs.

Cross sections are analytic forms tabulated once on a shared energy grid
(the reference reads tables, src/Collision.cpp:158-219, and interpolates
linearly, :221-237):

* electron elastic momentum transfer  6e-20 / sqrt(1 + E/10 eV) m^2
* electron excitation, threshold 19.8 eV: 1.5e-21 * t * exp(1 - t) m^2,
  t = (E - 19.8 eV) / (60 eV - 19.8 eV)          (peak 1.5e-21 m^2 at 60 eV)
* electron ionization, threshold 24.6 eV: 3.5e-21 * t * exp(1 - t) m^2,
  t = (E - 24.6 eV) / (120 eV - 24.6 eV)         (peak 3.5e-21 m^2 at 120 eV)
* ion isotropic elastic 2e-19 m^2 and resonant charge exchange 5e-19 m^2.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

E_CHARGE = 1.602176634e-19
M_E = 9.1093837139e-31
AMU = 1.66053906660e-27
K_B = 1.380649e-23
EPS0 = 8.8541878128e-12

ELASTIC, EXCITATION, IONIZATION, ATTACHMENT, CHARGE_EXCHANGE = range(5)


def hump(E, threshold, peak_energy, peak):
    t = np.clip((E - threshold) / (peak_energy - threshold), 0.0, None)
    return peak * t * np.exp(1.0 - t)


@dataclass
class ChannelSpec:
    process: int
    energy: np.ndarray  # J
    sigma: np.ndarray   # m^2
    threshold: float = 0.0  # J
    secondary: int = -1
    ion: int = -1
    angular: int = 0        # 0 isotropic, 1 backward, 2 Henyey-Greenstein
    mu_energy: np.ndarray | None = None  # J, Henyey-Greenstein mean-cosine table
    mu: np.ndarray | None = None


@dataclass
class ModelSpec:
    species: int
    channels: list
    neutral_density: float
    max_frequency: float
    neutral_mass: float
    neutral_temperature: float
    max_candidates: int = 64


@dataclass
class SpeciesSpec:
    charge: float
    mass: float
    weight: float
    capacity: int
    x: np.ndarray
    v: np.ndarray
    vy: np.ndarray | None = None
    vz: np.ndarray | None = None
    drift: float = 0.0     # Maxwellian parameters of the loading (for codes that load their own)
    thermal: float = 0.0


@dataclass
class Workload1D:
    name: str
    dirichlet: bool
    vdim: int
    si: bool
    nx: int
    length: float
    dt: float
    species: list
    models: list = field(default_factory=list)
    phi_left: float = 0.0
    phi_right: float = 0.0
    drive_left: tuple = (0.0, 0.0, 0.0)
    drive_right: tuple = (0.0, 0.0, 0.0)
    steps: int = 100
    bgk: tuple = None  # (frequency, neutral_temperature_velocity): the legacy BGK model

    @property
    def particles(self) -> int:
        return sum(len(s.x) for s in self.species)


def two_stream(particles_per_beam=16384, nx=256, seed=1, steps=2000) -> Workload1D:
    """1D1V electrostatic two-stream instability in normalized units
    (omega_p = 1, lambda_D = 1): L = 2 pi / 0.5, beams at +/-1.0 with 0.01
    Maxwellian spread, positions U[0, L) plus a 1e-3 cos(k x) displacement."""
    L = 2 * math.pi / 0.5
    k = 2 * math.pi / L
    n = 2 * particles_per_beam
    w = L / n  # unit mean density
    rx = np.random.default_rng(seed)
    rv = np.random.default_rng(seed + 1)
    sp = []
    for sign in (1.0, -1.0):
        x = rx.uniform(0.0, L, particles_per_beam)
        x = np.mod(x + 1e-3 * np.cos(k * x), L)
        v = sign * 1.0 + 0.01 * rv.standard_normal(particles_per_beam)
        sp.append(SpeciesSpec(-1.0, 1.0, w, particles_per_beam, x, v, drift=sign * 1.0, thermal=0.01))
    return Workload1D("two_stream_1d1v", False, 1, False, nx, L, 0.1, sp, steps=steps)


def landau(particles=1 << 20, nx=64, k=0.5, alpha=0.05, seed=3, steps=400) -> Workload1D:
    """1D1V Landau damping in normalized units: Maxwellian electrons (v_th = 1)
    over an immobile neutralising background, L = 2 pi / k, density
    1 + alpha cos(k x) from a position displacement, dt = 0.1.  Linear theory at
    k lambda_D = 0.5: omega = 1.4156 - 0.1533 i."""
    L = 2 * math.pi / k
    w = L / particles
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.0, L, particles)
    x = np.mod(x + alpha / k * np.sin(k * x), L)
    v = rng.standard_normal(particles)
    sp = [SpeciesSpec(-1.0, 1.0, w, particles, x, v, thermal=1.0)]
    return Workload1D("landau_1d1v", False, 1, False, nx, L, 0.1, sp, steps=steps)


def _rate_bound(mass, channels, e_max_ev, neutral_density, neutral_mass, temperature, grid=20001):
    s_max = math.sqrt(2 * e_max_ev * E_CHARGE / mass)
    v = np.linspace(0.0, s_max, grid)
    spread = 8.0 * math.sqrt(K_B * temperature / neutral_mass) if temperature > 0 else 0.0
    tot = np.zeros_like(v)
    for ch in channels:
        E = 0.5 * mass * v ** 2
        tot += np.where(E >= ch.threshold, np.interp(E, ch.energy, ch.sigma), 0.0)
    return float(np.max(neutral_density * tot * (v + spread)))


def ccp_helium(particles_per_cell=512, cells=512, seed=7, steps=4000, table_rows=4096, te_ev=1.0,
               vdim=3, bgk=None) -> Workload1D:
    """1D3V capacitive RF discharge with null-collision MCC: Dirichlet gap
    0.067 m, `cells` cells, grounded left electrode, right electrode driven at
    450 V / 13.56 MHz, dt = 1 / (400 f); electrons and He+ (4 amu) at
    particles_per_cell per cell each, Maxwellian Te = 1 eV, Ti = 0.026 eV;
    neutral helium 9.64e20 m^-3 at 300 K (thermal neutrals).  max_frequency is
    1.25 x the thermal-neutral rate bound over each table's energy range.
    vdim = 1 gives the 1D1V form of the same discharge: one velocity component
    and the 1V collision interface, which has no ionization channel (the
    electrons keep elastic scattering and excitation).  bgk = (frequency,
    neutral_temperature_velocity) replaces the MCC models by the legacy BGK
    model, which relaxes every species to that neutral Maxwellian."""
    f_rf = 13.56e6
    L = 0.067
    nx = cells + 1
    n = particles_per_cell * cells
    n0 = 2.56e14
    w = n0 * L / n
    m_he = 4 * AMU
    ng = 9.64e20
    T = 300.0
    Ee = np.concatenate([[0.0], np.logspace(-3, 4, table_rows - 1)])
    Ei = np.concatenate([[0.0], np.logspace(-3, math.log10(2000.0), table_rows // 2 - 1)])
    e_ch = [
        ChannelSpec(ELASTIC, Ee * E_CHARGE, 6e-20 / np.sqrt(1 + Ee / 10.0)),
        ChannelSpec(EXCITATION, Ee * E_CHARGE, hump(Ee, 19.8, 60.0, 1.5e-21), 19.8 * E_CHARGE),
        ChannelSpec(IONIZATION, Ee * E_CHARGE, hump(Ee, 24.6, 120.0, 3.5e-21), 24.6 * E_CHARGE, 0, 1),
    ][: 3 if vdim == 3 else 2]
    i_ch = [
        ChannelSpec(ELASTIC, Ei * E_CHARGE, np.full_like(Ei, 2e-19)),
        ChannelSpec(CHARGE_EXCHANGE, Ei * E_CHARGE, np.full_like(Ei, 5e-19)),
    ]
    nu_e = 1.25 * _rate_bound(M_E, e_ch, 1e4, ng, m_he, T)
    nu_i = 1.25 * _rate_bound(m_he, i_ch, 2000.0, ng, m_he, T)
    rng = np.random.default_rng(seed)
    ve = math.sqrt(E_CHARGE * te_ev / M_E)
    vi = math.sqrt(E_CHARGE * 0.026 / m_he)
    cap = int(n * 1.5) + 4096
    sp = []
    for q, m, vt in ((-E_CHARGE, M_E, ve), (E_CHARGE, m_he, vi)):
        x = rng.uniform(0.0, L, n)
        v3 = vt * rng.standard_normal((3, n))
        if vdim == 3:
            sp.append(SpeciesSpec(q, m, w, cap, x, v3[0].copy(), v3[1].copy(), v3[2].copy(), thermal=vt))
        else:
            sp.append(SpeciesSpec(q, m, w, cap, x, v3[0].copy(), thermal=vt))
    models = [
        ModelSpec(0, e_ch, ng, nu_e, m_he, T),
        ModelSpec(1, i_ch, ng, nu_i, m_he, T),
    ]
    name = "ccp_helium_1d3v" if vdim == 3 else "ccp_helium_1d1v"
    if bgk is not None:
        models, name = [], name + "_bgk"
    return Workload1D(name, True, vdim, True, nx, L, 1.0 / (400 * f_rf), sp, models,
                      drive_right=(450.0, f_rf, 0.0), steps=steps, bgk=bgk)


def to_device_config(wl: Workload1D, precision=0, seed=1):
    """Builds the device library's apic_config1d (and the table keeper)."""
    from . import (DIRICHLET, PERIODIC, SI, NORMALIZED, Tables, config1d, mcc_model)
    tabs = Tables()
    models = []
    for m in wl.models:
        chans = [tabs.channel(c.process, c.energy, c.sigma, c.threshold, c.secondary, c.ion) for c in m.channels]
        models.append(mcc_model(m.species, chans, m.neutral_density, m.max_frequency, m.neutral_mass,
                                m.neutral_temperature, 1 if wl.si else 0, m.max_candidates))
    cfg = config1d(boundary=DIRICHLET if wl.dirichlet else PERIODIC, velocity_dimensions=wl.vdim,
                   units=SI if wl.si else NORMALIZED, nx=wl.nx, length=wl.length, dt=wl.dt,
                   species=[(s.charge, s.mass, s.weight, s.capacity) for s in wl.species], models=models,
                   phi_left=wl.phi_left, phi_right=wl.phi_right, drive_left=wl.drive_left,
                   drive_right=wl.drive_right, precision=precision, seed=seed, bgk=wl.bgk)
    return cfg, tabs


# ---------------------------------------------------------------------------
# Structured periodic plasmas (2D3V with Bz, 3D3V with Bx)

@dataclass
class WorkloadND:
    name: str
    dims: int
    n: tuple
    length: tuple
    dt: float
    B: tuple
    species: list  # (charge, mass, weight, pos[3][np], v[3][np])
    si: bool = True
    steps: int = 100

    @property
    def particles(self) -> int:
        return sum(s[3].shape[1] for s in self.species)


def _plasma_nd(dims, cells, ppc, te_ev, ti_ev, mass_ratio, B, modes, n0, seed, steps, name, dt_wpe=0.1):
    """Maxwellian electrons and ions, cell size = Debye length at (n0, Te),
    density perturbed by 1e-3 cos(k . x) on the given modes (position
    displacement, like the two-stream loading)."""
    rng = np.random.default_rng(seed)
    lam = math.sqrt(EPS0 * te_ev * E_CHARGE / (n0 * E_CHARGE ** 2))
    wpe = math.sqrt(n0 * E_CHARGE ** 2 / (EPS0 * M_E))
    L = tuple(c * lam for c in cells)
    ncell = int(np.prod(cells))
    npart = ppc * ncell
    volume = float(np.prod(L))
    w = n0 * volume / npart
    species = []
    for q, m, t_ev in ((-E_CHARGE, M_E, te_ev), (E_CHARGE, M_E * mass_ratio, ti_ev)):
        pos = np.zeros((3, npart))
        for a in range(dims):
            pos[a] = rng.uniform(0.0, L[a], npart)
        for mode in modes:
            a = mode
            k = 2 * math.pi / L[a]
            pos[a] = np.mod(pos[a] + 1e-3 / k * np.sin(k * pos[a]), L[a])
        vt = math.sqrt(t_ev * E_CHARGE / m)
        v = vt * rng.standard_normal((3, npart))
        species.append((q, m, w, pos, v))
    return WorkloadND(name, dims, tuple(cells), L, dt_wpe / wpe, B, species, steps=steps)


def plasma_2d(cells=(512, 512), ppc=64, seed=11, steps=500):
    """2D3V periodic plasma, uniform Bz = 0.01 T: cell = lambda_D at
    n0 = 1e16 m^-3 and Te = 2 eV, Ti = 0.03 eV, m_i/m_e = 1836,
    1e-3 perturbation on the lowest kx and ky modes, dt = 0.1 / omega_pe."""
    return _plasma_nd(2, cells, ppc, 2.0, 0.03, 1836.0, (0.0, 0.0, 0.01), (0, 1), 1e16, seed, steps,
                      "plasma_2d3v_bz")


def plasma_3d(cells=(256, 256, 256), ppc=8, seed=13, steps=200):
    """3D3V periodic Langmuir oscillation, uniform Bx = 0.005 T: Te = 1 eV,
    m_i/m_e = 1836, 1e-3 perturbation on mode (1,0,0), dt = 0.1 / omega_pe."""
    return _plasma_nd(3, cells, ppc, 1.0, 0.025, 1836.0, (0.005, 0.0, 0.0), (0,), 1e16, seed, steps,
                      "plasma_3d3v_bx")


def to_device_config_nd(wl: WorkloadND, precision=0, capacity_factor=1.0, sort_interval=16):
    from . import SI, NORMALIZED, config_nd
    sp = [(q, m, w, int(pos.shape[1] * capacity_factor) + 1) for (q, m, w, pos, v) in wl.species]
    return config_nd(dims=wl.dims, n=wl.n, length=wl.length, dt=wl.dt, species=sp, magnetic_field=wl.B,
                     units=SI if wl.si else NORMALIZED, precision=precision, sort_interval=sort_interval)


@dataclass
class PlasmaPlan:
    """A 2D3V / 3D3V periodic deck whose particles are generated on the device
    (sizes too large to stage through host arrays)."""
    name: str
    dims: int
    n: tuple
    length: tuple
    dt: float
    B: tuple
    perturb_axis: int
    amplitude: float
    species: list  # (charge, mass, weight, count, thermal speed, seed)

    @property
    def particles(self) -> int:
        return sum(s[3] for s in self.species)

    def config(self, precision=0, sort_interval=16, capacity_factor=1.0, push_items=0, ion_sort_factor=16):
        """The ions (thermal speed 40-270x below the electrons') are re-sorted
        ion_sort_factor times less often than the electrons."""
        from . import SI, config_nd
        sp = [(q, m, w, int(n * capacity_factor) + 1) for (q, m, w, n, vt, seed) in self.species]
        return config_nd(dims=self.dims, n=self.n, length=self.length, dt=self.dt, species=sp,
                         magnetic_field=self.B, units=SI, precision=precision, sort_interval=sort_interval,
                         push_items=push_items,
                         species_sort_interval=[sort_interval, sort_interval * ion_sort_factor])

    def load(self, sim):
        for k, (q, m, w, n, vt, seed) in enumerate(self.species):
            amp = self.amplitude if k == 0 else 0.0
            sim.load_maxwellian(k, n, seed, vt, 0.0, self.perturb_axis, amp)


def plasma_plan(dims, cells=None, ppc=None, seed=11):
    """The 512^2 x 64 ppc 2D3V deck (Bz = 0.01 T, Te 2 eV, Ti 0.03 eV,
    perturbation on the lowest kx and ky modes) or the 256^3 x 8 ppc 3D3V deck
    (Bx = 0.005 T, Te 1 eV, Ti 0.025 eV, mode (1,0,0)); m_i/m_e = 1836,
    cell = lambda_D at n0 = 1e16 m^-3, dt = 0.1 / omega_pe, electrons
    perturbed by 1e-3."""
    if dims == 2:
        cells = tuple(cells or (512, 512))
        ppc = ppc or 64
        te, ti, B, axis, name = 2.0, 0.03, (0.0, 0.0, 0.01), -1, "plasma_2d3v_bz"
    else:
        cells = tuple(cells or (256, 256, 256))
        ppc = ppc or 8
        te, ti, B, axis, name = 1.0, 0.025, (0.005, 0.0, 0.0), 0, "plasma_3d3v_bx"
    n0 = 1e16
    lam = math.sqrt(EPS0 * te * E_CHARGE / (n0 * E_CHARGE ** 2))
    wpe = math.sqrt(n0 * E_CHARGE ** 2 / (EPS0 * M_E))
    L = tuple(c * lam for c in cells)
    npart = ppc * int(np.prod(cells))
    w = n0 * float(np.prod(L)) / npart
    mi = M_E * 1836.0
    species = [(-E_CHARGE, M_E, w, npart, math.sqrt(te * E_CHARGE / M_E), seed),
               (E_CHARGE, mi, w, npart, math.sqrt(ti * E_CHARGE / mi), seed + 1)]
    return PlasmaPlan(name, dims, cells, L, 0.1 / wpe, B, axis, 1e-3, species)


# ---------------------------------------------------------------------------
# Homogeneous electron swarms (run_swarm_benchmark)

TOWNSEND = 1.0e-21


def bethe(E, threshold, sigma0):
    """sigma0 ln(u) / u, u = E / threshold (zero below threshold, peak sigma0 / e at u = e)."""
    u = np.maximum(E / threshold, 1.0)
    return sigma0 * np.log(u) / u


@dataclass
class SwarmSpec:
    """One run_swarm_benchmark deck: a gas, the run controls and the reduced
    fields (each field f runs with seed + f, like the reference)."""
    name: str
    channels: list          # ChannelSpec, projectile-frame energies in J
    neutral_mass: float
    neutral_density: float
    neutral_temperature: float
    max_frequency: float
    timestep: float
    steps: int
    burn_in_steps: int
    particles: int
    fields_td: list
    branching: bool = False
    population_limit: int = 0
    uncertainty_blocks: int = 10
    initial_mean_energy_ev: float = 1.0
    max_energy_ev: float = 1000.0
    seed: int = 12345
    max_candidates: int = 64


def swarm_gas_4process(table_rows=2048, e_max_ev=2000.0):
    """Synthetic 4-process electron gas: elastic momentum transfer
    1e-20 (1.5 + 10 x^1.2 / (1 + x^2)) m^2 with x = E / 10 eV; excitations
    at 11.5 eV and 13.0 eV and ionization at 15.8 eV with Bethe-like shapes
    sigma0 ln(u)/u peaking at 3e-21, 5e-21 and 3e-20 m^2.  Argon-like
    neutral mass (39.948 amu)."""
    E = np.concatenate([[0.0], np.logspace(-3, math.log10(e_max_ev), table_rows - 1)])
    x = E / 10.0
    el = 1e-20 * (1.5 + 10.0 * x ** 1.2 / (1.0 + x ** 2))
    ch = [
        ChannelSpec(ELASTIC, E * E_CHARGE, el),
        ChannelSpec(EXCITATION, E * E_CHARGE, bethe(E, 11.5, 3e-21 * math.e), 11.5 * E_CHARGE),
        ChannelSpec(EXCITATION, E * E_CHARGE, bethe(E, 13.0, 5e-21 * math.e), 13.0 * E_CHARGE),
        ChannelSpec(IONIZATION, E * E_CHARGE, bethe(E, 15.8, 3e-20 * math.e), 15.8 * E_CHARGE, 0, 1),
    ]
    return ch, 39.948 * AMU


def swarm_gas_anisotropic(table_rows=512, e_max_ev=200.0, attachment=False):
    """A small synthetic gas that exercises Henyey-Greenstein elastic
    scattering (mean cosine rising from 0 to 0.6 over 0-100 eV), one
    excitation at 4 eV, ionization at 9 eV and optionally a dissociative
    attachment band near 2 eV."""
    E = np.concatenate([[0.0], np.logspace(-3, math.log10(e_max_ev), table_rows - 1)])
    mu_e = np.array([0.0, 1.0, 10.0, 100.0, E[-1]])
    mu = np.array([0.0, 0.05, 0.3, 0.6, 0.6])
    ch = [
        ChannelSpec(ELASTIC, E * E_CHARGE, 8e-20 / np.sqrt(1.0 + E / 5.0), angular=2, mu_energy=mu_e * E_CHARGE, mu=mu),
        ChannelSpec(EXCITATION, E * E_CHARGE, bethe(E, 4.0, 4e-21 * math.e), 4.0 * E_CHARGE),
        ChannelSpec(IONIZATION, E * E_CHARGE, bethe(E, 9.0, 2e-20 * math.e), 9.0 * E_CHARGE, 0, 1),
    ]
    if attachment:
        ch.append(ChannelSpec(ATTACHMENT, E * E_CHARGE, 6e-21 * np.exp(-((E - 2.0) / 0.8) ** 2)))
    return ch, 28.0 * AMU


def swarm_max_frequency(channels, neutral_density, neutral_mass, temperature, e_max_ev, margin=1.05):
    """A max_frequency that bounds the total rate of every electron up to
    e_max_ev (thermal neutrals add 8 sigma of relative speed)."""
    return margin * _rate_bound(M_E, channels, e_max_ev, neutral_density, neutral_mass, temperature)


def swarm_c5(fields_td=(10.0, 100.0, 1000.0), particles=100_000, steps=2000, burn_in_steps=1000, seed=12345,
             max_energy_ev=1000.0, branching=False) -> SwarmSpec:
    """The batched-serving swarm deck: the 4-process gas at 2.45e25 m^-3 and
    300 K, dt = 0.1 / max_frequency (the reference's bound,
    src/Swarm.cpp:300-303, at equality)."""
    ch, mn = swarm_gas_4process(e_max_ev=2.0 * max_energy_ev)
    ng, T = 2.45e25, 300.0
    nu = swarm_max_frequency(ch, ng, mn, T, max_energy_ev)
    return SwarmSpec("swarm_4process", ch, mn, ng, T, nu, 0.1 / nu, steps, burn_in_steps, particles,
                     list(fields_td), branching=branching, initial_mean_energy_ev=1.0,
                     max_energy_ev=max_energy_ev, seed=seed)


def to_device_swarm(spec: SwarmSpec, precision=0):
    """(apic.SwarmConfig, apic.MccModel, Tables) of a swarm deck."""
    from . import SWARM_BRANCHING, SWARM_FIXED, SwarmConfig, Tables, mcc_model
    tabs = Tables()
    chans = [tabs.channel(c.process, c.energy, c.sigma, c.threshold, c.secondary, c.ion, angular=c.angular,
                          mu_energy=c.mu_energy, mu=c.mu) for c in spec.channels]
    gas = mcc_model(0, chans, spec.neutral_density, spec.max_frequency, spec.neutral_mass, spec.neutral_temperature,
                    1, spec.max_candidates)
    cfg = SwarmConfig(spec.neutral_density, spec.neutral_temperature, spec.max_frequency, spec.timestep,
                      spec.steps, spec.burn_in_steps, spec.particles,
                      SWARM_BRANCHING if spec.branching else SWARM_FIXED, spec.population_limit,
                      spec.uncertainty_blocks, 0, spec.initial_mean_energy_ev, spec.max_energy_ev, spec.seed,
                      precision)
    return cfg, gas, tabs


def swarm_request(spec: SwarmSpec, td, particles=None, seed=None, steps=None, burn_in_steps=None, tolerance=0.0):
    from . import SWARM_BRANCHING, SWARM_FIXED, SwarmRequest
    return SwarmRequest(td, particles or spec.particles, spec.seed if seed is None else seed, steps or spec.steps,
                        spec.burn_in_steps if burn_in_steps is None else burn_in_steps, spec.uncertainty_blocks,
                        tolerance, SWARM_BRANCHING if spec.branching else SWARM_FIXED, spec.population_limit,
                        spec.initial_mean_energy_ev, spec.max_energy_ev, spec.timestep)
