"""Test infrastructure only: ctypes bindings to the CPU oracle.

Two libraries sit behind this module:

* ``build/libapic_oracle.so`` -- the plain-C restatement of the reference's
  particle step (``apic_oracle.c``), always available once ``make oracle`` ran;
* ``_ref/libapic_ref.so`` -- the reference's own library compiled from its
  sources plus ``ref_harness.cpp``; present only where the reference tree was
  available at build time (it then travels with the repository snapshot).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module.  The product (``aurora-pic_b200``) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "build", "libapic_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libapic_ref.so")

MAX_CHANNELS = 8
MAX_SPECIES = 4
MAX_MODELS = 4

ELASTIC, EXCITATION, IONIZATION, ATTACHMENT, CHARGE_EXCHANGE = range(5)


class Channel(C.Structure):
    _fields_ = [
        ("process", C.c_int), ("angular", C.c_int), ("energy_frame", C.c_int),
        ("threshold_energy", C.c_double),
        ("secondary_species", C.c_int), ("ion_species", C.c_int),
        ("rows", C.c_size_t),
        ("energy", C.POINTER(C.c_double)), ("sigma", C.POINTER(C.c_double)),
        ("mu_rows", C.c_size_t),
        ("mu_energy", C.POINTER(C.c_double)), ("mu", C.POINTER(C.c_double)),
    ]


class MccModel(C.Structure):
    _fields_ = [
        ("species", C.c_int),
        ("neutral_density", C.c_double), ("max_frequency", C.c_double),
        ("neutral_mass", C.c_double), ("neutral_temperature", C.c_double),
        ("si", C.c_int), ("max_candidates", C.c_size_t),
        ("nch", C.c_int), ("ch", Channel * MAX_CHANNELS),
    ]


class SpeciesCfg(C.Structure):
    _fields_ = [
        ("charge", C.c_double), ("mass", C.c_double), ("weight", C.c_double),
        ("particles", C.c_size_t), ("drift", C.c_double), ("thermal", C.c_double),
        ("thermal_y", C.c_double), ("thermal_z", C.c_double),
    ]


class Config1D(C.Structure):
    _fields_ = [
        ("dirichlet", C.c_int), ("vdim", C.c_int), ("si", C.c_int),
        ("nx", C.c_size_t), ("length", C.c_double), ("dt", C.c_double),
        ("phi_left", C.c_double), ("phi_right", C.c_double),
        ("drive_left", C.c_double * 3), ("drive_right", C.c_double * 3),
        ("seed", C.c_uint), ("threads", C.c_int), ("max_particles", C.c_size_t),
        ("nspecies", C.c_int), ("species", SpeciesCfg * MAX_SPECIES),
        ("nmodels", C.c_int), ("models", MccModel * MAX_MODELS),
        ("bgk", C.c_int), ("bgk_frequency", C.c_double), ("bgk_neutral_velocity", C.c_double),
    ]


class CollideStats(C.Structure):
    _fields_ = [
        ("candidates", C.c_uint64), ("null_collisions", C.c_uint64),
        ("channel_collisions", C.c_uint64 * MAX_CHANNELS),
        ("energy_change", C.c_double * MAX_CHANNELS),
        ("nsecondaries", C.c_int),
        ("secondary_channel", C.c_int * 16),
        ("secondary_velocity", (C.c_double * 3) * 16),
        ("secondary_ion_velocity", (C.c_double * 3) * 16),
        ("removed", C.c_int),
        ("draws", C.c_uint64),
    ]


class Rng(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("mt", C.c_void_p), ("key", C.c_uint32 * 2),
        ("ctr", C.c_uint32 * 3), ("index", C.c_uint64),
        ("array", C.POINTER(C.c_uint64)), ("array_len", C.c_uint64), ("overrun", C.c_int),
    ]


class SpatialAverage1D(C.Structure):
    """ora_spatial_average1d (SpatialAverage1DConfig + PhaseEedf1DConfig)."""
    _fields_ = [
        ("interval", C.c_size_t), ("start_step", C.c_size_t), ("end_step", C.c_size_t),
        ("rf_frequency", C.c_double), ("rf_cycles", C.c_size_t), ("phase_bins", C.c_size_t),
        ("eedf_species", C.c_int), ("eedf_bins", C.c_size_t), ("eedf_energy_max", C.c_double),
        ("eedf_regions", C.c_int), ("eedf_x_min", C.c_double * 8), ("eedf_x_max", C.c_double * 8),
    ]


def spatial_average1d(interval=1, start_step=1, end_step=1, rf_frequency=0.0, rf_cycles=0, phase_bins=0,
                      eedf_species=-1, eedf_bins=0, eedf_energy_max=0.0, eedf_regions=()):
    a = SpatialAverage1D()
    a.interval, a.start_step, a.end_step = interval, start_step, end_step
    a.rf_frequency, a.rf_cycles, a.phase_bins = rf_frequency, rf_cycles, phase_bins
    a.eedf_species, a.eedf_bins, a.eedf_energy_max = eedf_species, eedf_bins, eedf_energy_max
    a.eedf_regions = len(eedf_regions)
    for i, (lo, hi) in enumerate(eedf_regions):
        a.eedf_x_min[i], a.eedf_x_max[i] = lo, hi
    return a


# quantities of the spatial sums
SA_DENSITY, SA_VX, SA_VY, SA_VZ, SA_KINETIC, SA_POTENTIAL, SA_ELECTRIC, SA_ELECTRIC2, SA_COLLISION = range(9)


def reference_tree_present() -> bool:
    """Whether the reference's source tree is present on this host (the
    Makefile knows where: APIC_REFERENCE or its default)."""
    try:
        out = subprocess.run(["make", "-s", "-C", HERE, "has-ref"], check=True, capture_output=True, text=True)
    except (OSError, subprocess.CalledProcessError):
        return False
    return out.stdout.strip() == "yes"


def ensure_built() -> None:
    """Build the C restatement (and the reference harness when the reference
    tree is present) with oracle/Makefile."""
    targets = ["oracle"]
    if reference_tree_present():
        targets.append("ref")
    if not os.path.exists(ORACLE_SO) or ("ref" in targets and not os.path.exists(REF_SO)):
        subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


_DP = C.POINTER(C.c_double)
_U8P = C.POINTER(C.c_uint8)
_U64P = C.POINTER(C.c_uint64)


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_DP)


def u8ptr(a: np.ndarray):
    assert a.dtype == np.uint8 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_U8P)


def u64ptr(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_U64P)


_oracle = None
_ref = None


def oracle() -> C.CDLL:
    global _oracle
    if _oracle is None:
        ensure_built()
        L = C.CDLL(ORACLE_SO)
        L.ora_mt64_next.restype = C.c_uint64
        L.ora_draw.restype = C.c_uint64
        L.ora_canonical.restype = C.c_double
        L.ora_uniform01.restype = C.c_double
        L.ora_normal_draw.restype = C.c_double
        L.ora_gather1d.restype = C.c_double
        L.ora_gather1d.argtypes = [_DP, C.c_size_t, C.c_double, C.c_double, C.c_int, C.c_double]
        L.ora_deposit1d.argtypes = [_DP, C.c_size_t, C.c_double, C.c_double, C.c_int, C.c_double,
                                    C.c_double, C.c_size_t, _DP, _U8P]
        L.ora_solve1d.argtypes = [_DP, _DP, _DP, C.c_size_t, C.c_double, C.c_double, C.c_int,
                                  C.c_double, C.c_double, C.c_double]
        L.ora_sim1d_create.restype = C.c_void_p
        L.ora_sim1d_create.argtypes = [C.POINTER(Config1D), C.c_int, C.c_uint64]
        L.ora_sim1d_destroy.argtypes = [C.c_void_p]
        L.ora_sim1d_load.argtypes = [C.c_void_p, C.c_int, C.c_size_t, _DP, _DP, _DP, _DP, _DP, _U8P]
        L.ora_sim1d_initialize_fields.argtypes = [C.c_void_p, C.c_double, C.c_uint64]
        L.ora_sim1d_step.argtypes = [C.c_void_p, C.c_size_t]
        L.ora_sim1d_round_fp32.argtypes = [C.c_void_p]
        L.ora_sim1d_initialize.argtypes = [C.c_void_p]
        L.ora_sim1d_count.restype = C.c_size_t
        L.ora_sim1d_count.argtypes = [C.c_void_p, C.c_int]
        L.ora_sim1d_get.argtypes = [C.c_void_p, C.c_int, _DP, _DP, _DP, _DP, _DP, _U8P]
        L.ora_sim1d_fields.argtypes = [C.c_void_p, _DP, _DP, _DP]
        L.ora_sim1d_time.restype = C.c_double
        L.ora_sim1d_time.argtypes = [C.c_void_p]
        L.ora_sim1d_set_mt.argtypes = [C.c_void_p, _U64P]
        L.ora_sim1d_collisions.argtypes = [C.c_void_p, _U64P, _U64P, _U64P]
        L.ora_sim1d_bgk_energy.restype = C.c_double
        L.ora_sim1d_bgk_energy.argtypes = [C.c_void_p]
        L.ora_sim1d_losses.argtypes = [C.c_void_p, C.c_int, _U64P, _U64P, _DP, _DP]
        L.ora_sim1d_kinetic.restype = C.c_double
        L.ora_sim1d_kinetic.argtypes = [C.c_void_p, C.c_int]
        L.ora_sim1d_electric_work.restype = C.c_double
        L.ora_sim1d_electric_work.argtypes = [C.c_void_p, C.c_int]
        L.ora_sim1d_field_energy.restype = C.c_double
        L.ora_sim1d_field_energy.argtypes = [C.c_void_p]
        L.ora_last_error.restype = C.c_char_p
        L.ora_sim1d_enable_spatial_average.argtypes = [C.c_void_p, C.POINTER(SpatialAverage1D)]
        L.ora_sim1d_spatial_counts.argtypes = [C.c_void_p, _U64P, _U64P, _U64P, _U64P]
        L.ora_sim1d_spatial_sums.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _DP]
        L.ora_sim1d_phase_eedf.argtypes = [C.c_void_p, C.c_int, C.c_int, _U64P, _DP, _DP]
        L.ora_collider_init.argtypes = [C.c_void_p, C.POINTER(MccModel), C.c_double]
        L.ora_collide3.argtypes = [C.c_void_p, _DP, C.c_double, C.POINTER(Rng), C.POINTER(CollideStats)]
        _oracle = L
    return _oracle


def reference_available() -> bool:
    return os.path.exists(REF_SO)


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        ensure_built()
        L = C.CDLL(REF_SO)
        L.ref_last_error.restype = C.c_char_p
        L.ref1d_create.argtypes = [C.POINTER(Config1D), C.c_char_p, C.POINTER(C.c_void_p)]
        L.ref1d_destroy.argtypes = [C.c_void_p]
        L.ref1d_initialize.argtypes = [C.c_void_p]
        L.ref1d_step.argtypes = [C.c_void_p, C.c_size_t]
        L.ref1d_count.restype = C.c_size_t
        L.ref1d_count.argtypes = [C.c_void_p, C.c_int]
        L.ref1d_time.restype = C.c_double
        L.ref1d_time.argtypes = [C.c_void_p]
        L.ref1d_get_particles.argtypes = [C.c_void_p, C.c_int, _DP, _DP, _DP, _DP, _DP, _U8P]
        L.ref1d_get_fields.argtypes = [C.c_void_p, _DP, _DP, _DP]
        L.ref1d_sample.argtypes = [C.c_void_p, _DP, _DP, C.POINTER(C.c_size_t)]
        L.ref1d_collisions.argtypes = [C.c_void_p, _U64P, _U64P, _U64P, C.c_size_t]
        L.ref1d_channel_energy.argtypes = [C.c_void_p, _DP, C.c_size_t]
        L.ref1d_losses.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t), _DP, _DP]
        L.ref1d_rng_state.argtypes = [C.c_void_p, C.c_char_p, _U64P]
        L.ref1d_save_checkpoint.argtypes = [C.c_void_p, C.c_char_p]
        L.ref1d_load_checkpoint.argtypes = [C.c_void_p, C.c_char_p]
        L.ref1d_electric_work.restype = C.c_double
        L.ref1d_electric_work.argtypes = [C.c_void_p, C.c_int]
        L.ref_deposit_solve_gather_1d.argtypes = [
            C.c_int, C.c_size_t, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
            _DP, _DP, C.POINTER(C.c_size_t), C.POINTER(_DP), _DP, _DP, _DP, C.c_size_t, _DP, _DP]
        L.ref_collide3.argtypes = [C.POINTER(MccModel), C.c_double, C.c_char_p, C.c_size_t, _DP, _U64P,
                                   C.c_double, C.POINTER(CollideStats), _U64P, C.c_size_t]
        L.ref1d_create_diag.argtypes = [C.POINTER(Config1D), C.POINTER(SpatialAverage1D), C.c_char_p,
                                        C.POINTER(C.c_void_p)]
        L.ref1d_run_diag.argtypes = [C.POINTER(Config1D), C.POINTER(SpatialAverage1D), C.c_size_t, C.c_char_p]
        L.ref1d_validate_diag.argtypes = [C.POINTER(Config1D), C.POINTER(SpatialAverage1D), C.c_char_p]
        L.ref1d_collision_energy.argtypes = [C.c_void_p, C.c_int, C.c_int, _DP]
        L.ref1d_collision_steps.argtypes = [C.c_void_p, _U64P, _U64P]
        L.ref1d_phase_eedf.argtypes = [C.c_void_p, C.c_int, C.c_int, _U64P, _DP, _DP]
        L.ref_mt64.argtypes = [C.c_uint64, C.c_size_t, _U64P]
        L.ref_dist.argtypes = [C.c_int, C.c_uint64, C.c_size_t, _DP]
        _ref = L
    return _ref


# ---------------------------------------------------------------------------
# Configuration builders shared by tests, smoke() and bench.py.

class TableSet:
    """Keeps the numpy arrays behind ctypes table pointers alive."""

    def __init__(self):
        self.keep = []

    def channel(self, process, energy, sigma, threshold=0.0, secondary=-1, ion=-1,
                angular=0, frame=0, mu_energy=None, mu=None) -> Channel:
        """angular 2 (Henyey-Greenstein) takes a mean-cosine table mu(mu_energy)."""
        e = np.ascontiguousarray(energy, dtype=np.float64)
        s = np.ascontiguousarray(sigma, dtype=np.float64)
        self.keep += [e, s]
        ch = Channel(process, angular, frame, threshold, secondary, ion, len(e), dptr(e), dptr(s))
        if mu is not None:
            me = np.ascontiguousarray(mu_energy, dtype=np.float64)
            mv = np.ascontiguousarray(mu, dtype=np.float64)
            self.keep += [me, mv]
            ch.mu_rows, ch.mu_energy, ch.mu = len(me), dptr(me), dptr(mv)
        return ch


def make_model(species, channels, neutral_density, max_frequency, neutral_mass=0.0,
               neutral_temperature=0.0, si=1, max_candidates=64) -> MccModel:
    m = MccModel()
    m.species = species
    m.neutral_density = neutral_density
    m.max_frequency = max_frequency
    m.neutral_mass = neutral_mass
    m.neutral_temperature = neutral_temperature
    m.si = si
    m.max_candidates = max_candidates
    m.nch = len(channels)
    for i, ch in enumerate(channels):
        m.ch[i] = ch
    return m


def config1d(*, dirichlet, vdim, si, nx, length, dt, species, models=(), phi_left=0.0,
             phi_right=0.0, drive_left=(0, 0, 0), drive_right=(0, 0, 0), seed=12345, threads=0,
             max_particles=0, bgk=None) -> Config1D:
    """bgk: (frequency, neutral_temperature_velocity) enables the legacy BGK model."""
    c = Config1D()
    c.dirichlet, c.vdim, c.si, c.nx, c.length, c.dt = dirichlet, vdim, si, nx, length, dt
    c.phi_left, c.phi_right = phi_left, phi_right
    c.drive_left[:] = list(drive_left)
    c.drive_right[:] = list(drive_right)
    c.seed, c.threads, c.max_particles = seed, threads, max_particles
    c.nspecies = len(species)
    for i, sp in enumerate(species):
        c.species[i] = SpeciesCfg(*sp)
    c.nmodels = len(models)
    for i, m in enumerate(models):
        c.models[i] = m
    if bgk is not None:
        c.bgk, c.bgk_frequency, c.bgk_neutral_velocity = 1, bgk[0], bgk[1]
    return c


class Sim1D:
    """Oracle 1D simulation (mode 0 = reference layout and stream, mode 1 =
    device layout with Philox streams, mode 2 = mode 1 with FP32-stored
    velocities, the device's FP32 particle form)."""

    def __init__(self, cfg: Config1D, mode: int, philox_seed: int = 0):
        L = oracle()
        self.cfg = cfg
        self.h = L.ora_sim1d_create(C.byref(cfg), mode, philox_seed)
        if not self.h:
            raise RuntimeError(L.ora_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            oracle().ora_sim1d_destroy(self.h)
            self.h = None

    def load(self, s, x, v, vh, vy=None, vz=None, alive=None):
        n = len(x)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else np.zeros(n)
                for a in (x, v, vh, vy, vz)]
        al = np.ones(n, np.uint8) if alive is None else np.ascontiguousarray(alive, dtype=np.uint8)
        oracle().ora_sim1d_load(self.h, s, n, *[dptr(a) for a in arrs], u8ptr(al))

    def initialize_fields(self, time=0.0, step=0):
        oracle().ora_sim1d_initialize_fields(self.h, time, step)

    def initialize(self):
        oracle().ora_sim1d_initialize(self.h)

    def set_mt(self, state):
        st = np.ascontiguousarray(state, dtype=np.uint64)
        oracle().ora_sim1d_set_mt(self.h, u64ptr(st))

    def step(self, n=1):
        rc = oracle().ora_sim1d_step(self.h, n)
        if rc:
            raise RuntimeError(oracle().ora_last_error().decode())

    def round_fp32(self):
        """Mode 2: round the stored velocities as a device read-back does."""
        oracle().ora_sim1d_round_fp32(self.h)

    def particles(self, s):
        L = oracle()
        n = L.ora_sim1d_count(self.h, s)
        out = {k: np.zeros(n) for k in ("x", "v", "vh", "vy", "vz")}
        al = np.zeros(n, np.uint8)
        L.ora_sim1d_get(self.h, s, *[dptr(out[k]) for k in ("x", "v", "vh", "vy", "vz")], u8ptr(al))
        out["alive"] = al
        return out

    def fields(self):
        n = self.cfg.nx
        rho, phi, E = np.zeros(n), np.zeros(n), np.zeros(n)
        oracle().ora_sim1d_fields(self.h, dptr(rho), dptr(phi), dptr(E))
        return rho, phi, E

    def collisions(self):
        c, nl = np.zeros(1, np.uint64), np.zeros(1, np.uint64)
        per = np.zeros(MAX_MODELS * MAX_CHANNELS, np.uint64)
        oracle().ora_sim1d_collisions(self.h, u64ptr(c), u64ptr(nl), u64ptr(per))
        return int(c[0]), int(nl[0]), per.reshape(MAX_MODELS, MAX_CHANNELS)

    def bgk_energy(self):
        return oracle().ora_sim1d_bgk_energy(self.h)

    def losses(self, s):
        a, b = np.zeros(1, np.uint64), np.zeros(1, np.uint64)
        ea, eb = np.zeros(1), np.zeros(1)
        oracle().ora_sim1d_losses(self.h, s, u64ptr(a), u64ptr(b), dptr(ea), dptr(eb))
        return int(a[0]), int(b[0]), float(ea[0]), float(eb[0])

    def kinetic(self, s):
        return oracle().ora_sim1d_kinetic(self.h, s)

    def field_energy(self):
        return oracle().ora_sim1d_field_energy(self.h)

    def electric_work(self, s):
        return oracle().ora_sim1d_electric_work(self.h, s)

    def time(self):
        return oracle().ora_sim1d_time(self.h)

    # -- CCP campaign diagnostics --
    def enable_spatial_average(self, sa: "SpatialAverage1D"):
        self.sa = sa
        oracle().ora_sim1d_enable_spatial_average(self.h, C.byref(sa))

    def spatial_counts(self):
        P = max(int(self.sa.phase_bins), 1)
        a, b = np.zeros(1, np.uint64), np.zeros(1, np.uint64)
        pa, pb = np.zeros(P, np.uint64), np.zeros(P, np.uint64)
        oracle().ora_sim1d_spatial_counts(self.h, u64ptr(a), u64ptr(b), u64ptr(pa), u64ptr(pb))
        P = int(self.sa.phase_bins)
        return int(a[0]), int(b[0]), pa[:P], pb[:P]

    def spatial_sums(self, quantity, index=0, phase=-1):
        out = np.zeros(self.cfg.nx)
        if oracle().ora_sim1d_spatial_sums(self.h, quantity, index, phase, dptr(out)):
            raise RuntimeError(oracle().ora_last_error().decode())
        return out

    def phase_eedf(self, phase, region):
        cnt, sums = np.zeros(2, np.uint64), np.zeros(7)
        hist = np.zeros(max(int(self.sa.eedf_bins), 1))
        if oracle().ora_sim1d_phase_eedf(self.h, phase, region, u64ptr(cnt), dptr(sums), dptr(hist)):
            raise RuntimeError(oracle().ora_last_error().decode())
        return cnt, sums, hist[:int(self.sa.eedf_bins)]


class Ref1D:
    """The reference's own Simulation, driven through the harness."""

    def __init__(self, cfg: Config1D, workdir: str, spatial_average=None):
        L = ref()
        self.cfg = cfg
        self.workdir = workdir
        self.sa = spatial_average
        h = C.c_void_p()
        if spatial_average is None:
            rc = L.ref1d_create(C.byref(cfg), workdir.encode(), C.byref(h))
        else:
            rc = L.ref1d_create_diag(C.byref(cfg), C.byref(spatial_average), workdir.encode(), C.byref(h))
        if rc:
            raise RuntimeError(L.ref_last_error().decode())
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            ref().ref1d_destroy(self.h)
            self.h = None

    def _chk(self, rc):
        if rc:
            raise RuntimeError(ref().ref_last_error().decode())

    def initialize(self):
        self._chk(ref().ref1d_initialize(self.h))

    def step(self, n=1):
        self._chk(ref().ref1d_step(self.h, n))

    def particles(self, s):
        L = ref()
        n = L.ref1d_count(self.h, s)
        out = {k: np.zeros(n) for k in ("x", "v", "vh", "vy", "vz")}
        al = np.zeros(n, np.uint8)
        self._chk(L.ref1d_get_particles(self.h, s, *[dptr(out[k]) for k in ("x", "v", "vh", "vy", "vz")],
                                        u8ptr(al)))
        out["alive"] = al
        return out

    def fields(self):
        n = self.cfg.nx
        rho, phi, E = np.zeros(n), np.zeros(n), np.zeros(n)
        ref().ref1d_get_fields(self.h, dptr(rho), dptr(phi), dptr(E))
        return rho, phi, E

    def save_checkpoint(self, path):
        self._chk(ref().ref1d_save_checkpoint(self.h, path.encode()))

    def load_checkpoint(self, path):
        self._chk(ref().ref1d_load_checkpoint(self.h, path.encode()))

    def rng_state(self):
        st = np.zeros(313, np.uint64)
        path = os.path.join(self.workdir, "rng_probe.apc")
        self._chk(ref().ref1d_rng_state(self.h, path.encode(), u64ptr(st)))
        return st

    def collisions(self):
        c, nl = np.zeros(1, np.uint64), np.zeros(1, np.uint64)
        per = np.zeros(64, np.uint64)
        k = ref().ref1d_collisions(self.h, u64ptr(c), u64ptr(nl), u64ptr(per), 64)
        return int(c[0]), int(nl[0]), per[:k]

    def channel_energy(self):
        out = np.zeros(64)
        k = ref().ref1d_channel_energy(self.h, dptr(out), 64)
        return out[:k]

    def losses(self, s):
        a, b = C.c_size_t(), C.c_size_t()
        ea, eb = np.zeros(1), np.zeros(1)
        ref().ref1d_losses(self.h, s, C.byref(a), C.byref(b), dptr(ea), dptr(eb))
        return a.value, b.value, float(ea[0]), float(eb[0])

    def sample(self):
        ns = self.cfg.nspecies
        ke = np.zeros(ns)
        fe = np.zeros(1)
        live = (C.c_size_t * ns)()
        self._chk(ref().ref1d_sample(self.h, dptr(ke), dptr(fe), live))
        return ke, float(fe[0]), list(live)

    def time(self):
        return ref().ref1d_time(self.h)

    def electric_work(self, s):
        return ref().ref1d_electric_work(self.h, s)

    def collision_energy(self, channel, phase=-1):
        out = np.zeros(self.cfg.nx)
        ref().ref1d_collision_energy(self.h, channel, phase, dptr(out))
        return out

    def collision_steps(self):
        a = np.zeros(1, np.uint64)
        P = max(int(self.sa.phase_bins), 1)
        pb = np.zeros(P, np.uint64)
        ref().ref1d_collision_steps(self.h, u64ptr(a), u64ptr(pb))
        return int(a[0]), pb[:int(self.sa.phase_bins)]

    def phase_eedf(self, phase, region):
        cnt, sums = np.zeros(2, np.uint64), np.zeros(7)
        hist = np.zeros(max(int(self.sa.eedf_bins), 1))
        self._chk(ref().ref1d_phase_eedf(self.h, phase, region, u64ptr(cnt), dptr(sums), dptr(hist)))
        return cnt, sums, hist[:int(self.sa.eedf_bins)]


def ref_run_spatial_average(cfg: Config1D, sa: SpatialAverage1D, steps: int, workdir: str) -> str:
    """Simulation::run of the reference over `steps` steps; returns the folder
    holding its spatial-average CSV files."""
    L = ref()
    if L.ref1d_run_diag(C.byref(cfg), C.byref(sa), steps, workdir.encode()):
        raise RuntimeError(L.ref_last_error().decode())
    return os.path.join(workdir, "out")


def ref_validate_spatial_average(cfg: Config1D, sa: SpatialAverage1D, workdir: str):
    """The reference's configuration error for `sa`, or None."""
    L = ref()
    if L.ref1d_validate_diag(C.byref(cfg), C.byref(sa), workdir.encode()):
        return L.ref_last_error().decode()
    return None


def config_from_workload(wl, tables: TableSet, seed=12345, threads=0, particles=None, own_loading=False):
    """The oracle / reference configuration of a workload (apic.workloads.Workload1D).
    own_loading=True gives each species its Maxwellian parameters so that the
    reference loads its own particles (bench.py's CPU timing)."""
    models = []
    for m in wl.models:
        chans = [tables.channel(c.process, c.energy, c.sigma, c.threshold, c.secondary, c.ion) for c in m.channels]
        models.append(make_model(m.species, chans, m.neutral_density, m.max_frequency, m.neutral_mass,
                                 m.neutral_temperature, 1 if wl.si else 0, m.max_candidates))
    species = []
    for s in wl.species:
        n = len(s.x) if particles is None else particles
        if own_loading:
            species.append((s.charge, s.mass, s.weight, n, s.drift, s.thermal, s.thermal, s.thermal))
        else:
            species.append((s.charge, s.mass, s.weight, n, 0.0, 0.0, 0.0, 0.0))
    return config1d(dirichlet=int(wl.dirichlet), vdim=wl.vdim, si=int(wl.si), nx=wl.nx, length=wl.length,
                    dt=wl.dt, species=species, models=models, phi_left=wl.phi_left, phi_right=wl.phi_right,
                    drive_left=wl.drive_left, drive_right=wl.drive_right, seed=seed, threads=threads,
                    max_particles=max(s.capacity for s in wl.species), bgk=getattr(wl, "bgk", None))


# ---------------------------------------------------------------------------
# Structured 2D3V / 3D3V periodic

_SZP = C.POINTER(C.c_size_t)


def _nd_bind():
    L = oracle()
    if getattr(L, "_nd_bound", False):
        return L
    L.ora_solve_nd.argtypes = [_DP, _DP, _DP, C.c_int, _SZP, _DP, C.c_double]
    L.ora_gather_nd.argtypes = [_DP, C.c_int, _SZP, _DP, _DP, _DP]
    L.ora_deposit_nd.argtypes = [_DP, C.c_int, _SZP, _DP, C.c_double, C.c_size_t, _DP]
    L.ora_boris.argtypes = [_DP, _DP, _DP, C.c_double, C.c_double]
    L.ora_simnd_create.restype = C.c_void_p
    L.ora_simnd_create.argtypes = [C.c_int, _SZP, _DP, C.c_double, C.c_double, _DP, C.c_int, _DP, _DP, _DP]
    L.ora_simnd_destroy.argtypes = [C.c_void_p]
    L.ora_simnd_load.argtypes = [C.c_void_p, C.c_int, C.c_size_t, _DP, _DP, _DP]
    L.ora_simnd_initialize_fields.argtypes = [C.c_void_p]
    L.ora_simnd_initialize.argtypes = [C.c_void_p]
    L.ora_simnd_step.argtypes = [C.c_void_p, C.c_size_t]
    L.ora_simnd_get.argtypes = [C.c_void_p, C.c_int, _DP, _DP, _DP]
    L.ora_simnd_fields.argtypes = [C.c_void_p, _DP, _DP, _DP]
    L._nd_bound = True
    return L


def solve_mixed_2d(rho, n, L, periodic_axis, eps, lower, upper):
    """Oracle FieldSolver::solve(Mesh2D&) with one periodic axis: (phi, E[2])."""
    Lb = oracle()
    Lb.ora_solve_mixed_2d.argtypes = [_DP, _DP, _DP, _SZP, _DP, C.c_int, C.c_double, C.c_double, C.c_double]
    rho = np.ascontiguousarray(rho, dtype=np.float64).ravel()
    N = int(n[0] * n[1])
    phi, E = np.zeros(N), np.zeros(2 * N)
    nn = (C.c_size_t * 2)(*[int(v) for v in n])
    Lv = np.ascontiguousarray(L, dtype=np.float64)
    rc = Lb.ora_solve_mixed_2d(dptr(rho), dptr(phi), dptr(E), nn, dptr(Lv), periodic_axis, eps, lower, upper)
    if rc:
        raise RuntimeError(Lb.ora_last_error().decode())
    return phi, E.reshape(2, N)


def solve_dirichlet_nd(rho, n, L, eps, potentials=None):
    """Oracle SOR solve on a fully Dirichlet mesh: (phi, E[dims])."""
    Lb = oracle()
    Lb.ora_solve_dirichlet_nd.argtypes = [_DP, _DP, _DP, C.c_int, _SZP, _DP, C.c_double, _DP]
    dims = len(n)
    N = int(np.prod(n))
    rho = np.ascontiguousarray(rho, dtype=np.float64).ravel()
    phi, E = np.zeros(N), np.zeros(dims * N)
    pot = None if potentials is None else np.ascontiguousarray(potentials, dtype=np.float64)
    rc = Lb.ora_solve_dirichlet_nd(dptr(rho), dptr(phi), dptr(E), dims, sizes3(n), dptr(arr3(L)), eps,
                                   dptr(pot) if pot is not None else None)
    if rc:
        raise RuntimeError(Lb.ora_last_error().decode())
    return phi, E.reshape(dims, N)


def ref_solve_dirichlet_nd(rho, n, L, eps, potentials=(0.0, 0.0, 0.0, 0.0)):
    """The reference's FieldSolver on a fully Dirichlet Mesh2D / Mesh3D."""
    Lb = ref()
    Lb.ref_solve_dirichlet_nd.argtypes = [C.c_int, _SZP, _DP, C.c_double, _DP, _DP, _DP, _DP]
    dims = len(n)
    N = int(np.prod(n))
    rho = np.ascontiguousarray(rho, dtype=np.float64).ravel()
    phi, E = np.zeros(N), np.zeros(dims * N)
    pot = np.ascontiguousarray(potentials, dtype=np.float64)
    if Lb.ref_solve_dirichlet_nd(dims, sizes3(n), dptr(arr3(L)), eps, dptr(pot), dptr(rho), dptr(phi), dptr(E)):
        raise RuntimeError(Lb.ref_last_error().decode())
    return phi, E.reshape(dims, N)


def ref_solve_mixed_2d(rho, n, L, periodic_axis, eps, lower, upper):
    """The reference's own FieldSolver on a mixed Mesh2D, through the harness."""
    Lb = ref()
    Lb.ref_solve_mixed_2d.argtypes = [_SZP, _DP, C.c_int, C.c_double, C.c_double, C.c_double, _DP, _DP, _DP]
    rho = np.ascontiguousarray(rho, dtype=np.float64).ravel()
    N = int(n[0] * n[1])
    phi, E = np.zeros(N), np.zeros(2 * N)
    nn = (C.c_size_t * 2)(*[int(v) for v in n])
    Lv = np.ascontiguousarray(L, dtype=np.float64)
    rc = Lb.ref_solve_mixed_2d(nn, dptr(Lv), periodic_axis, eps, lower, upper, dptr(rho), dptr(phi), dptr(E))
    if rc:
        raise RuntimeError("reference mixed solve failed")
    return phi, E.reshape(2, N)


def ref_aps_write(path, dimension, si, species):
    """The reference's write_external_particle_state; species {name: (pos[3][n],
    vel[3][n])}; returns its signature."""
    Lb = ref()
    Lb.ref_aps_write.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_size_t, C.POINTER(C.c_char_p), _SZP,
                                 C.POINTER(_DP), C.POINTER(_DP), C.POINTER(C.c_uint64)]
    names = list(species)
    keep = [(np.ascontiguousarray(species[k][0], dtype=np.float64), np.ascontiguousarray(species[k][1], dtype=np.float64))
            for k in names]
    nm = (C.c_char_p * len(names))(*[k.encode() for k in names])
    counts = (C.c_size_t * len(names))(*[p.shape[1] for p, _ in keep])
    pp = (_DP * len(names))(*[dptr(p) for p, _ in keep])
    vv = (_DP * len(names))(*[dptr(v) for _, v in keep])
    sig = C.c_uint64()
    if Lb.ref_aps_write(os.fsencode(path), dimension, si, len(names), nm, counts, pp, vv, C.byref(sig)):
        raise RuntimeError(Lb.ref_last_error().decode())
    return sig.value


def ref_aps_read(path, max_particles=1 << 30, capacity=1 << 20):
    """The reference's load_external_particle_state: (signature, [(pos, vel)] by name)."""
    Lb = ref()
    Lb.ref_aps_read.argtypes = [C.c_char_p, C.c_size_t, C.POINTER(C.c_uint64), _SZP, _SZP, _DP, _DP, C.c_size_t]
    sig, ns = C.c_uint64(), C.c_size_t()
    counts = (C.c_size_t * 64)()
    pos, vel = np.zeros(capacity), np.zeros(capacity)
    if Lb.ref_aps_read(os.fsencode(path), max_particles, C.byref(sig), C.byref(ns), counts, dptr(pos), dptr(vel),
                       capacity):
        raise RuntimeError(Lb.ref_last_error().decode())
    out, off = [], 0
    for k in range(ns.value):
        n = counts[k]
        out.append((pos[off: off + 3 * n].reshape(3, n).copy(), vel[off: off + 3 * n].reshape(3, n).copy()))
        off += 3 * n
    return sig.value, out


def sizes3(n):
    n = list(n) + [1] * (3 - len(n))
    return (C.c_size_t * 3)(*n)


def arr3(v):
    v = list(v) + [1.0] * (3 - len(v))
    return np.ascontiguousarray(v, dtype=np.float64)


class SimND:
    """Oracle structured periodic simulation (2D3V or 3D3V)."""

    def __init__(self, dims, n, L, dt, eps, B, species):
        """species: list of (q, m, w_eff)."""
        Lb = _nd_bind()
        self.dims, self.n = dims, list(n)
        self.N = int(np.prod(n))
        self._L = arr3(L)
        self._B = np.ascontiguousarray(B, dtype=np.float64)
        q = np.array([s[0] for s in species]); m = np.array([s[1] for s in species]); w = np.array([s[2] for s in species])
        self.ns = len(species)
        self.h = Lb.ora_simnd_create(dims, sizes3(n), dptr(self._L), dt, eps, dptr(self._B), self.ns, dptr(q),
                                     dptr(m), dptr(w))
        self.np = [0] * self.ns

    def set_profile(self, axis, coordinates, values):
        """magnetic_field_profile: B piecewise linear along `axis`."""
        Lb = _nd_bind()
        Lb.ora_simnd_set_profile.argtypes = [C.c_void_p, C.c_int, C.c_size_t, _DP, _DP]
        self._prof = (np.ascontiguousarray(coordinates, dtype=np.float64),
                      np.ascontiguousarray(values, dtype=np.float64).ravel())
        if Lb.ora_simnd_set_profile(self.h, axis, len(self._prof[0]), dptr(self._prof[0]), dptr(self._prof[1])):
            raise RuntimeError(Lb.ora_last_error().decode())

    def set_walls(self, dirichlet, potentials, particle):
        """2D walls (before load): Dirichlet field axes (x, y), side potentials
        and particle boundaries (left, right, bottom, top: 0 periodic,
        1 absorbing, 2 reflecting)."""
        Lb = _nd_bind()
        Lb.ora_simnd_set_walls.argtypes = [C.c_void_p, C.POINTER(C.c_int), _DP, C.POINTER(C.c_int)]
        d = (C.c_int * 2)(*dirichlet)
        pot = np.ascontiguousarray(potentials, dtype=np.float64)
        pb = (C.c_int * 4)(*particle)
        if Lb.ora_simnd_set_walls(self.h, d, dptr(pot), pb):
            raise RuntimeError(Lb.ora_last_error().decode())

    def set_walls3d(self, particle):
        """3D walls (before load): a Dirichlet mesh with grounded walls on
        every side and particle boundaries (left, right, bottom, top, back,
        front: 0 periodic, 1 absorbing, 2 reflecting)."""
        Lb = _nd_bind()
        Lb.ora_simnd_set_walls3d.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
        if Lb.ora_simnd_set_walls3d(self.h, (C.c_int * 6)(*particle)):
            raise RuntimeError(Lb.ora_last_error().decode())

    def alive_losses(self, k):
        """alive flags and the absorbed counts per side of species k (4 in 2D, 6 in 3D)"""
        Lb = _nd_bind()
        Lb.ora_simnd_alive_losses.argtypes = [C.c_void_p, C.c_int, _U8P, _U64P]
        al = np.zeros(self.np[k], np.uint8)
        lo = np.zeros(6, np.uint64)
        Lb.ora_simnd_alive_losses(self.h, k, u8ptr(al), u64ptr(lo))
        return al, lo[:2 * self.dims]

    def __del__(self):
        if getattr(self, "h", None):
            _nd_bind().ora_simnd_destroy(self.h)
            self.h = None

    def load(self, k, pos, v, vh):
        pos = np.ascontiguousarray(np.asarray(pos, dtype=np.float64).reshape(3, -1))
        v = np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(3, -1))
        vh = np.ascontiguousarray(np.asarray(vh, dtype=np.float64).reshape(3, -1))
        self.np[k] = pos.shape[1]
        _nd_bind().ora_simnd_load(self.h, k, pos.shape[1], dptr(pos), dptr(v), dptr(vh))

    def initialize(self):
        _nd_bind().ora_simnd_initialize(self.h)

    def initialize_fields(self):
        _nd_bind().ora_simnd_initialize_fields(self.h)

    def step(self, k=1):
        _nd_bind().ora_simnd_step(self.h, k)

    def particles(self, k):
        n = self.np[k]
        pos, v, vh = np.zeros((3, n)), np.zeros((3, n)), np.zeros((3, n))
        _nd_bind().ora_simnd_get(self.h, k, dptr(pos), dptr(v), dptr(vh))
        return pos, v, vh

    def fields(self):
        rho, phi, E = np.zeros(self.N), np.zeros(self.N), np.zeros(3 * self.N)
        _nd_bind().ora_simnd_fields(self.h, dptr(rho), dptr(phi), dptr(E))
        return rho, phi, E[: self.dims * self.N].reshape(self.dims, self.N)


def _refnd_bind():
    L = ref()
    if getattr(L, "_nd_bound", False):
        return L
    L.refnd_create.argtypes = [C.c_int, _SZP, _DP, C.c_double, C.c_int, _DP, C.c_int, _DP, _DP, _DP, _SZP, _DP, _DP,
                               C.c_uint, C.c_int, C.POINTER(C.c_void_p)]
    L.refnd_destroy.argtypes = [C.c_void_p]
    L.refnd_initialize.argtypes = [C.c_void_p]
    L.refnd_step.argtypes = [C.c_void_p, C.c_size_t]
    L.refnd_count.restype = C.c_size_t
    L.refnd_count.argtypes = [C.c_void_p, C.c_int]
    L.refnd_get.argtypes = [C.c_void_p, C.c_int, _DP, _DP, _DP]
    L.refnd_fields.argtypes = [C.c_void_p, _DP, _DP, _DP]
    L.refnd_time.restype = C.c_double
    L.refnd_time.argtypes = [C.c_void_p]
    L.ref_solve_nd.argtypes = [C.c_int, _SZP, _DP, C.c_double, _DP, _DP, _DP]
    L._nd_bound = True
    return L


class RefND:
    """The reference's Simulation2D / Simulation3D (periodic) through the harness."""

    def __init__(self, dims, n, L, dt, si, B, species, seed=12345, threads=0, profile=None, walls=None):
        """species: list of (q, m, w, count, drift_x, thermal); profile: optional
        (axis, coordinates, values[rows][3]) magnetic_field_profile; walls:
        optional 2D (dirichlet[2], potentials[4], particle boundaries[4]) or
        3D particle boundaries[6] (a grounded Dirichlet mesh)."""
        Lb = _refnd_bind()
        if walls is not None and dims == 3:
            Lb.refnd_set_walls3d.argtypes = [C.POINTER(C.c_int)]
            Lb.refnd_set_walls3d((C.c_int * 6)(*walls))
        elif walls is not None:
            Lb.refnd_set_walls.argtypes = [C.POINTER(C.c_int), _DP, C.POINTER(C.c_int)]
            self._pot = np.ascontiguousarray(walls[1], dtype=np.float64)
            Lb.refnd_set_walls((C.c_int * 2)(*walls[0]), dptr(self._pot), (C.c_int * 4)(*walls[2]))
        self.dims, self.n, self.N = dims, list(n), int(np.prod(n))
        cols = [np.array([s[i] for s in species], dtype=np.float64) for i in (0, 1, 2, 4, 5)]
        counts = (C.c_size_t * len(species))(*[s[3] for s in species])
        self._keep = cols
        Bv = np.ascontiguousarray(B, dtype=np.float64)
        Lv = arr3(L)
        h = C.c_void_p()
        if profile is None:
            rc = Lb.refnd_create(dims, sizes3(n), dptr(Lv), dt, si, dptr(Bv), len(species), dptr(cols[0]),
                                 dptr(cols[1]), dptr(cols[2]), counts, dptr(cols[3]), dptr(cols[4]), seed, threads,
                                 C.byref(h))
        else:
            ax, pc, pv = profile
            pc = np.ascontiguousarray(pc, dtype=np.float64)
            pv = np.ascontiguousarray(pv, dtype=np.float64).ravel()
            self._keep_prof = (pc, pv)
            Lb.refnd_create_profile.argtypes = [C.c_int, _SZP, _DP, C.c_double, C.c_int, _DP, C.c_int, _DP, _DP, _DP,
                                                _SZP, _DP, _DP, C.c_uint, C.c_int, C.c_int, C.c_size_t, _DP, _DP,
                                                C.POINTER(C.c_void_p)]
            rc = Lb.refnd_create_profile(dims, sizes3(n), dptr(Lv), dt, si, dptr(Bv), len(species), dptr(cols[0]),
                                         dptr(cols[1]), dptr(cols[2]), counts, dptr(cols[3]), dptr(cols[4]), seed,
                                         threads, ax, len(pc), dptr(pc), dptr(pv), C.byref(h))
        if rc:
            raise RuntimeError(Lb.ref_last_error().decode())
        self.h = h
        self.ns = len(species)

    def __del__(self):
        if getattr(self, "h", None):
            _refnd_bind().refnd_destroy(self.h)
            self.h = None

    def initialize(self):
        if _refnd_bind().refnd_initialize(self.h):
            raise RuntimeError(ref().ref_last_error().decode())

    def step(self, k=1):
        if _refnd_bind().refnd_step(self.h, k):
            raise RuntimeError(ref().ref_last_error().decode())

    def particles(self, k):
        n = _refnd_bind().refnd_count(self.h, k)
        pos, v, vh = np.zeros((3, n)), np.zeros((3, n)), np.zeros((3, n))
        _refnd_bind().refnd_get(self.h, k, dptr(pos), dptr(v), dptr(vh))
        return pos, v, vh

    def alive_losses(self, k):
        Lb = _refnd_bind()
        Lb.refnd_alive_losses.argtypes = [C.c_void_p, C.c_int, _U8P, _U64P]
        n = Lb.refnd_count(self.h, k)
        al = np.zeros(n, np.uint8)
        lo = np.zeros(6, np.uint64)
        Lb.refnd_alive_losses(self.h, k, u8ptr(al), u64ptr(lo))
        return al, lo[:2 * self.dims]

    def fields(self):
        rho, phi, E = np.zeros(self.N), np.zeros(self.N), np.zeros(self.dims * self.N)
        _refnd_bind().refnd_fields(self.h, dptr(rho), dptr(phi), dptr(E))
        return rho, phi, E.reshape(self.dims, self.N)

    def time(self):
        return _refnd_bind().refnd_time(self.h)


# ---------------------------------------------------------------------------
# Homogeneous electron swarm (run_field / run_swarm_benchmark)

class SwarmConfig(C.Structure):
    _fields_ = [
        ("neutral_density", C.c_double), ("neutral_temperature", C.c_double),
        ("max_frequency", C.c_double), ("timestep", C.c_double),
        ("steps", C.c_size_t), ("burn_in_steps", C.c_size_t), ("particles", C.c_size_t),
        ("branching", C.c_int), ("population_limit", C.c_size_t), ("uncertainty_blocks", C.c_size_t),
        ("initial_mean_energy_ev", C.c_double), ("max_energy_ev", C.c_double), ("seed", C.c_uint64),
    ]


class SwarmResult(C.Structure):
    _fields_ = [
        ("reduced_field_td", C.c_double), ("electric_field_v_m", C.c_double),
        ("mean_velocity_x", C.c_double), ("mean_velocity_x_se", C.c_double),
        ("drift_velocity", C.c_double), ("reduced_mobility", C.c_double),
        ("mean_energy_ev", C.c_double), ("mean_energy_se_ev", C.c_double),
        ("diffusion_available", C.c_int),
        ("diffusion_longitudinal", C.c_double), ("diffusion_transverse", C.c_double),
        ("max_observed_energy_ev", C.c_double),
        ("initial_weight", C.c_double), ("final_weight", C.c_double),
        ("final_particles", C.c_uint64),
        ("growth_rate", C.c_double), ("growth_rate_se", C.c_double),
        ("ionization_rate", C.c_double), ("ionization_rate_se", C.c_double),
        ("attachment_rate", C.c_double), ("attachment_rate_se", C.c_double),
        ("net_rate", C.c_double), ("net_rate_se", C.c_double),
        ("townsend_available", C.c_int),
        ("townsend_growth", C.c_double), ("townsend_growth_se", C.c_double),
        ("townsend_rate", C.c_double), ("townsend_rate_se", C.c_double),
        ("candidates", C.c_uint64), ("null_collisions", C.c_uint64),
        ("nch", C.c_int),
        ("channel_collisions", C.c_uint64 * MAX_CHANNELS),
        ("channel_rate", C.c_double * MAX_CHANNELS), ("channel_rate_se", C.c_double * MAX_CHANNELS),
    ]

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v)[: self.nch] if name.startswith("channel_") else v
        return d


def swarm_config(*, neutral_density, max_frequency, timestep, steps, burn_in_steps, particles,
                 neutral_temperature=0.0, branching=False, population_limit=0, uncertainty_blocks=10,
                 initial_mean_energy_ev=0.1, max_energy_ev=100.0, seed=12345) -> SwarmConfig:
    return SwarmConfig(neutral_density, neutral_temperature, max_frequency, timestep, steps, burn_in_steps,
                       particles, int(branching), population_limit, uncertainty_blocks, initial_mean_energy_ev,
                       max_energy_ev, seed)


def _swarm_bind(L):
    L.ora_swarm_run_field.argtypes = [C.POINTER(SwarmConfig), C.POINTER(MccModel), C.c_double, C.c_uint64, C.c_int,
                                      C.POINTER(SwarmResult), _DP]
    L.ora_block_mean_and_error.argtypes = [_DP, C.c_size_t, C.c_size_t, _DP, _DP]
    L.ora_block_slope_and_error.argtypes = [_DP, C.c_size_t, C.c_double, C.c_size_t, _DP, _DP]
    L.ora_swarm_population_limit.restype = C.c_size_t
    L.ora_swarm_population_limit.argtypes = [C.POINTER(SwarmConfig)]
    return L


def swarm_run_field(cfg: SwarmConfig, gas: MccModel, td: float, seed: int, mode: int, samples=False):
    """run_field on the oracle; mode 0 reference form, 1 device FP64 form,
    2 device FP32-storage form.  Returns (SwarmResult, samples or None)."""
    L = _swarm_bind(oracle())
    out = SwarmResult()
    ns = cfg.steps - cfg.burn_in_steps
    buf = np.zeros(3 * ns) if samples else None
    rc = L.ora_swarm_run_field(C.byref(cfg), C.byref(gas), td, seed, mode, C.byref(out),
                               dptr(buf) if samples else None)
    if rc:
        raise RuntimeError(L.ora_last_error().decode())
    return out, (buf.reshape(3, ns) if samples else None)


def block_mean_and_error(x, blocks):
    L = _swarm_bind(oracle())
    x = np.ascontiguousarray(x, dtype=np.float64)
    m, e = C.c_double(), C.c_double()
    if L.ora_block_mean_and_error(dptr(x), len(x), blocks, C.byref(m), C.byref(e)):
        raise ValueError(L.ora_last_error().decode())
    return m.value, e.value


def ref_swarm_run(cfg: SwarmConfig, gas: MccModel, fields, workdir):
    """pic::run_swarm_benchmark through the harness: one SwarmResult per field
    (field f runs with seed cfg.seed + f)."""
    L = ref()
    L.ref_swarm_run.argtypes = [C.POINTER(SwarmConfig), C.POINTER(MccModel), _DP, C.c_size_t, C.c_char_p,
                                C.POINTER(SwarmResult)]
    f = np.ascontiguousarray(fields, dtype=np.float64)
    out = (SwarmResult * len(f))()
    if L.ref_swarm_run(C.byref(cfg), C.byref(gas), dptr(f), len(f), workdir.encode(), out):
        raise RuntimeError(L.ref_last_error().decode())
    return list(out)


def swarm_from_spec(spec, tables: TableSet):
    """(SwarmConfig, MccModel) of an apic.workloads.SwarmSpec."""
    chans = [tables.channel(c.process, c.energy, c.sigma, c.threshold, c.secondary, c.ion, angular=c.angular,
                            mu_energy=c.mu_energy, mu=c.mu) for c in spec.channels]
    gas = make_model(0, chans, spec.neutral_density, spec.max_frequency, spec.neutral_mass,
                     spec.neutral_temperature, 1, spec.max_candidates)
    cfg = swarm_config(neutral_density=spec.neutral_density, max_frequency=spec.max_frequency,
                       timestep=spec.timestep, steps=spec.steps, burn_in_steps=spec.burn_in_steps,
                       particles=spec.particles, neutral_temperature=spec.neutral_temperature,
                       branching=spec.branching, population_limit=spec.population_limit,
                       uncertainty_blocks=spec.uncertainty_blocks,
                       initial_mean_energy_ev=spec.initial_mean_energy_ev, max_energy_ev=spec.max_energy_ev,
                       seed=spec.seed)
    return cfg, gas


# Spatial Townsend pass (run_spatial_townsend, src/Swarm.cpp:645-938)

class SpatialConfig(C.Structure):
    _fields_ = [
        ("histories", C.c_size_t), ("length_m", C.c_double), ("bins", C.c_size_t),
        ("fit_begin_bin", C.c_size_t), ("fit_end_bin", C.c_size_t), ("max_steps", C.c_size_t),
        ("work_item_limit", C.c_uint64), ("min_r_squared", C.c_double),
    ]


class SpatialResult(C.Structure):
    _fields_ = [
        ("townsend_1_m", C.c_double), ("townsend_se_1_m", C.c_double), ("fit_r_squared", C.c_double),
        ("histories_completed", C.c_uint64), ("maximum_active_particles", C.c_uint64),
        ("particle_updates", C.c_uint64),
    ]


def spatial_config(*, histories, length_m, bins, fit_begin_bin=0, fit_end_bin=0, max_steps, work_item_limit=0,
                   min_r_squared=0.0) -> SpatialConfig:
    return SpatialConfig(histories, length_m, bins, fit_begin_bin, fit_end_bin, max_steps, work_item_limit,
                         min_r_squared)


def swarm_spatial_townsend(cfg: SwarmConfig, sp: SpatialConfig, gas: MccModel, td: float, seed: int, mode: int,
                           scan_updates: int = 0):
    """run_spatial_townsend on the oracle (mode 0 reference form, 1 device
    form).  Returns (SpatialResult, profile[bins, 3], crossings[histories, bins],
    scan updates after the pass)."""
    L = oracle()
    L.ora_swarm_spatial_townsend.argtypes = [C.POINTER(SwarmConfig), C.POINTER(SpatialConfig), C.POINTER(MccModel),
                                             C.c_double, C.c_uint64, C.c_int, _U64P, C.POINTER(SpatialResult), _DP,
                                             _DP]
    out = SpatialResult()
    prof = np.zeros((sp.bins, 3))
    cross = np.zeros((sp.histories, sp.bins))
    scan = np.array([scan_updates], np.uint64)
    rc = L.ora_swarm_spatial_townsend(C.byref(cfg), C.byref(sp), C.byref(gas), td, seed, mode, u64ptr(scan),
                                      C.byref(out), dptr(prof), dptr(cross))
    if rc:
        raise RuntimeError(L.ora_last_error().decode())
    return out, prof, cross, int(scan[0])


def ref_swarm_run_spatial(cfg: SwarmConfig, sp: SpatialConfig, gas: MccModel, fields, workdir):
    """pic::run_swarm_benchmark with the spatial Townsend controls: per field
    (SwarmResult, SpatialResult, profile[bins, 3])."""
    L = ref()
    L.ref_swarm_run_spatial.argtypes = [C.POINTER(SwarmConfig), C.POINTER(SpatialConfig), C.POINTER(MccModel), _DP,
                                        C.c_size_t, C.c_char_p, C.POINTER(SwarmResult), C.POINTER(SpatialResult),
                                        _DP]
    f = np.ascontiguousarray(fields, dtype=np.float64)
    out = (SwarmResult * len(f))()
    sout = (SpatialResult * len(f))()
    prof = np.zeros((len(f), sp.bins, 3))
    if L.ref_swarm_run_spatial(C.byref(cfg), C.byref(sp), C.byref(gas), dptr(f), len(f), workdir.encode(), out, sout,
                               dptr(prof)):
        raise RuntimeError(L.ref_last_error().decode())
    return [(out[k], sout[k], prof[k]) for k in range(len(f))]
