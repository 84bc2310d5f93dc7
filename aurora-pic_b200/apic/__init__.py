"""Python bindings (ctypes) to libaurorapic_b200.so, the B200-native
electrostatic PIC particle step.

The library is the product; this module only marshals arguments across the
C ABI declared in include/aurorapic_b200.h.  It loads the in-tree library
and fails loudly when it is missing -- there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "lib", "libaurorapic_b200.so")

MAX_SPECIES = 4
MAX_MODELS = 4
MAX_CHANNELS = 8

PERIODIC, DIRICHLET = 0, 1
NORMALIZED, SI = 0, 1
FP64, FP32, FP32_STORAGE = 0, 1, 2
ELASTIC, EXCITATION, IONIZATION, ATTACHMENT, CHARGE_EXCHANGE = range(5)
ISOTROPIC, BACKWARD, HENYEY_GREENSTEIN = 0, 1, 2

STATUS = {
    0: "APIC_OK", 1: "APIC_ERR_INVALID", 2: "APIC_ERR_CUDA", 3: "APIC_ERR_CAPACITY",
    4: "APIC_ERR_MAJORANT", 5: "APIC_ERR_CANDIDATES", 6: "APIC_ERR_NONFINITE",
    7: "APIC_ERR_TIMEOUT", 8: "APIC_ERR_UNSUPPORTED", 9: "APIC_ERR_STATE", 10: "APIC_ERR_NO_DEVICE",
}


class ApicError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class McChannel(C.Structure):
    _fields_ = [
        ("process", C.c_int), ("angular", C.c_int), ("energy_frame", C.c_int),
        ("threshold_energy", C.c_double), ("secondary_species", C.c_int), ("ion_species", C.c_int),
        ("rows", C.c_size_t), ("energy", C.POINTER(C.c_double)), ("sigma", C.POINTER(C.c_double)),
        ("mean_cosine_rows", C.c_size_t), ("mean_cosine_energy", C.POINTER(C.c_double)),
        ("mean_cosine", C.POINTER(C.c_double)),
    ]


class MccModel(C.Structure):
    _fields_ = [
        ("species", C.c_int), ("neutral_density", C.c_double), ("max_frequency", C.c_double),
        ("neutral_mass", C.c_double), ("neutral_temperature", C.c_double), ("gas_units_si", C.c_int),
        ("max_candidates", C.c_size_t), ("nch", C.c_int), ("ch", McChannel * MAX_CHANNELS),
    ]


class VoltageDrive(C.Structure):
    _fields_ = [("amplitude", C.c_double), ("frequency", C.c_double), ("phase", C.c_double)]


class SpeciesCfg(C.Structure):
    _fields_ = [("charge", C.c_double), ("mass", C.c_double), ("weight", C.c_double),
                ("capacity", C.c_size_t)]


class Config1D(C.Structure):
    _fields_ = [
        ("boundary", C.c_int), ("velocity_dimensions", C.c_int), ("units", C.c_int),
        ("relative_permittivity", C.c_double), ("nx", C.c_size_t), ("length", C.c_double),
        ("dt", C.c_double), ("phi_left", C.c_double), ("phi_right", C.c_double),
        ("drive_left", VoltageDrive), ("drive_right", VoltageDrive), ("precision", C.c_int),
        ("seed", C.c_uint64), ("nspecies", C.c_int), ("species", SpeciesCfg * MAX_SPECIES),
        ("nmodels", C.c_int), ("models", MccModel * MAX_MODELS),
        ("bgk_enabled", C.c_int), ("bgk_frequency", C.c_double), ("bgk_neutral_velocity", C.c_double),
    ]


class Sample1D(C.Structure):
    _fields_ = [
        ("step", C.c_uint64), ("time", C.c_double), ("kinetic_energy", C.c_double),
        ("field_energy", C.c_double), ("total_energy", C.c_double), ("charge_l1", C.c_double),
        ("live_particles", C.c_uint64), ("phi_left", C.c_double), ("phi_right", C.c_double),
        ("kinetic_by_species", C.c_double * MAX_SPECIES), ("live_by_species", C.c_uint64 * MAX_SPECIES),
    ]


class CollisionTotals(C.Structure):
    _fields_ = [
        ("candidates", C.c_uint64), ("null_collisions", C.c_uint64),
        ("channel_collisions", (C.c_uint64 * MAX_CHANNELS) * MAX_MODELS),
        ("channel_energy_change", (C.c_double * MAX_CHANNELS) * MAX_MODELS),
    ]


class BoundaryLoss(C.Structure):
    _fields_ = [("absorbed_left", C.c_uint64), ("absorbed_right", C.c_uint64),
                ("kinetic_energy_left", C.c_double), ("kinetic_energy_right", C.c_double)]


class CollideStats(C.Structure):
    _fields_ = [
        ("candidates", C.c_uint64), ("null_collisions", C.c_uint64),
        ("channel_collisions", C.c_uint32 * MAX_CHANNELS), ("energy_change", C.c_double * MAX_CHANNELS),
        ("nsecondaries", C.c_int), ("secondary_channel", C.c_int * 4),
        ("secondary_velocity", (C.c_double * 3) * 4), ("secondary_ion_velocity", (C.c_double * 3) * 4),
        ("removed", C.c_int), ("draws", C.c_uint32),
    ]


MAX_EEDF_REGIONS = 8
SA_DENSITY, SA_VELOCITY_X, SA_VELOCITY_Y, SA_VELOCITY_Z, SA_KINETIC_ENERGY = range(5)
SA_POTENTIAL, SA_ELECTRIC, SA_ELECTRIC_SQUARED, SA_COLLISION_ENERGY = range(5, 9)


class SpatialAverage1D(C.Structure):
    """apic_spatial_average1d: SpatialAverage1DConfig + PhaseEedf1DConfig."""
    _fields_ = [
        ("interval", C.c_size_t), ("start_step", C.c_size_t), ("end_step", C.c_size_t),
        ("rf_frequency", C.c_double), ("rf_cycles", C.c_size_t), ("phase_bins", C.c_size_t),
        ("eedf_species", C.c_int), ("eedf_bins", C.c_size_t), ("eedf_energy_max", C.c_double),
        ("eedf_regions", C.c_int), ("eedf_x_min", C.c_double * MAX_EEDF_REGIONS),
        ("eedf_x_max", C.c_double * MAX_EEDF_REGIONS),
    ]


class PhaseEedf1D(C.Structure):
    _fields_ = [
        ("macro_observations", C.c_uint64), ("overflow_macro_observations", C.c_uint64),
        ("represented_observations", C.c_double), ("overflow_represented_observations", C.c_double),
        ("weighted_energy_sum", C.c_double), ("weighted_energy_squared_sum", C.c_double),
        ("weighted_velocity_x_sum", C.c_double), ("weighted_velocity_y_sum", C.c_double),
        ("weighted_velocity_z_sum", C.c_double),
    ]


def spatial_average1d(interval=1, start_step=1, end_step=1, rf_frequency=0.0, rf_cycles=0, phase_bins=0,
                      eedf_species=-1, eedf_bins=0, eedf_energy_max=0.0, eedf_regions=()) -> SpatialAverage1D:
    """Spatial-average settings of a 1D run (the reference's spatial_average_*
    and phase_eedf_* keys; eedf_regions as (x_min, x_max) pairs)."""
    a = SpatialAverage1D()
    a.interval, a.start_step, a.end_step = interval, start_step, end_step
    a.rf_frequency, a.rf_cycles, a.phase_bins = rf_frequency, rf_cycles, phase_bins
    a.eedf_species, a.eedf_bins, a.eedf_energy_max = eedf_species, eedf_bins, eedf_energy_max
    a.eedf_regions = len(eedf_regions)
    for i, (lo, hi) in enumerate(eedf_regions):
        a.eedf_x_min[i], a.eedf_x_max[i] = lo, hi
    return a


def validate_spatial_average(cfg: "Config1D", sa: SpatialAverage1D):
    """Raises ApicError with the reference's message for an invalid setting
    (host only: no device needed)."""
    rc = lib().apic_spatial_average1d_validate(C.byref(cfg), C.byref(sa))
    if rc != 0:
        raise ApicError(rc, lib().apic_sim1d_last_error(None).decode())


_DP = C.POINTER(C.c_double)
_U8P = C.POINTER(C.c_uint8)
_U64P = C.POINTER(C.c_uint64)
_lib = None


def library_path() -> str:
    return LIB_PATH


def lib() -> C.CDLL:
    """Loads the in-tree library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libaurorapic_b200.so is not built ({LIB_PATH}); run aurora-pic_b200/build.py")
    L = C.CDLL(LIB_PATH)
    L.apic_version.restype = C.c_char_p
    L.apic_status_string.restype = C.c_char_p
    L.apic_sim1d_create.argtypes = [C.POINTER(Config1D), C.POINTER(C.c_void_p)]
    L.apic_sim1d_destroy.argtypes = [C.c_void_p]
    L.apic_sim1d_last_error.restype = C.c_char_p
    L.apic_sim1d_last_error.argtypes = [C.c_void_p]
    L.apic_sim1d_load_particles.argtypes = [C.c_void_p, C.c_int, C.c_size_t, _DP, _DP, _DP, _DP, _DP, _U8P]
    L.apic_sim1d_initialize.argtypes = [C.c_void_p]
    L.apic_sim1d_resume.argtypes = [C.c_void_p, C.c_double, C.c_uint64]
    L.apic_sim1d_step.argtypes = [C.c_void_p, C.c_size_t]
    L.apic_sim1d_synchronize.argtypes = [C.c_void_p]
    L.apic_sim1d_set_wait_limit.argtypes = [C.c_void_p, C.c_double]
    L.apic_sim1d_count.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_size_t)]
    L.apic_sim1d_read_particles.argtypes = [C.c_void_p, C.c_int, C.c_size_t, _DP, _DP, _DP, _DP, _DP,
                                            C.POINTER(C.c_size_t)]
    L.apic_sim1d_read_fields.argtypes = [C.c_void_p, _DP, _DP, _DP]
    L.apic_sim1d_sample.argtypes = [C.c_void_p, C.POINTER(Sample1D)]
    L.apic_sim1d_collision_totals.argtypes = [C.c_void_p, C.POINTER(CollisionTotals)]
    L.apic_sim1d_boundary_losses.argtypes = [C.c_void_p, C.c_int, C.POINTER(BoundaryLoss)]
    L.apic_sim1d_time.restype = C.c_double
    L.apic_sim1d_time.argtypes = [C.c_void_p]
    L.apic_sim1d_step_count.restype = C.c_uint64
    L.apic_sim1d_step_count.argtypes = [C.c_void_p]
    L.apic_sim1d_cuda_stream.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
    L.apic_sim1d_set_kernel_timing.argtypes = [C.c_void_p, C.c_int]
    L.apic_sim1d_kernel_times.argtypes = [C.c_void_p, _DP, _DP, _U64P]
    L.apic_sim1d_enable_power_transfer.argtypes = [C.c_void_p]
    L.apic_sim1d_power_transfer.argtypes = [C.c_void_p, C.c_int, _DP]
    L.apic_spatial_average1d_validate.argtypes = [C.POINTER(Config1D), C.POINTER(SpatialAverage1D)]
    L.apic_sim1d_enable_spatial_average.argtypes = [C.c_void_p, C.POINTER(SpatialAverage1D)]
    L.apic_sim1d_spatial_average_counts.argtypes = [C.c_void_p, _U64P, _U64P, _U64P, _U64P]
    L.apic_sim1d_spatial_sums.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _DP]
    L.apic_sim1d_phase_eedf.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(PhaseEedf1D), _DP]
    L.apic_deposit_solve_gather_1d.argtypes = [
        C.c_int, C.c_size_t, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, _DP, _DP,
        C.POINTER(C.c_size_t), C.POINTER(_DP), _DP, _DP, _DP, C.c_size_t, _DP, _DP]
    L.apic_collide3.argtypes = [C.POINTER(MccModel), C.c_double, C.c_size_t, _DP, C.c_double, _U64P, _U64P,
                                C.c_uint64, C.c_uint64, C.c_uint32, C.POINTER(CollideStats)]
    _lib = L
    return L


def dptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_DP)


def _check(rc: int, handle=None) -> None:
    if rc != 0:
        msg = lib().apic_sim1d_last_error(handle).decode() if handle is not None else ""
        if not msg:
            msg = lib().apic_sim1d_last_error(None).decode()
        raise ApicError(rc, msg)


class Tables:
    """Owns the numpy arrays behind the table pointers of a configuration."""

    def __init__(self):
        self.keep = []

    def channel(self, process, energy, sigma, threshold=0.0, secondary=-1, ion=-1, angular=ISOTROPIC,
                frame=0, mu_energy=None, mu=None) -> McChannel:
        """angular HENYEY_GREENSTEIN takes the mean-cosine table mu(mu_energy)."""
        e = np.ascontiguousarray(energy, dtype=np.float64)
        s = np.ascontiguousarray(sigma, dtype=np.float64)
        self.keep += [e, s]
        ch = McChannel(process, angular, frame, threshold, secondary, ion, len(e), dptr(e), dptr(s))
        if mu is not None:
            me = np.ascontiguousarray(mu_energy, dtype=np.float64)
            mv = np.ascontiguousarray(mu, dtype=np.float64)
            self.keep += [me, mv]
            ch.mean_cosine_rows, ch.mean_cosine_energy, ch.mean_cosine = len(me), dptr(me), dptr(mv)
        return ch


def mcc_model(species, channels, neutral_density, max_frequency, neutral_mass=0.0, neutral_temperature=0.0,
              gas_units_si=1, max_candidates=64) -> MccModel:
    m = MccModel()
    m.species = species
    m.neutral_density = neutral_density
    m.max_frequency = max_frequency
    m.neutral_mass = neutral_mass
    m.neutral_temperature = neutral_temperature
    m.gas_units_si = gas_units_si
    m.max_candidates = max_candidates
    m.nch = len(channels)
    for i, ch in enumerate(channels):
        m.ch[i] = ch
    return m


def config1d(*, boundary, velocity_dimensions, units, nx, length, dt, species, models=(), phi_left=0.0,
             phi_right=0.0, drive_left=(0.0, 0.0, 0.0), drive_right=(0.0, 0.0, 0.0), precision=FP64, seed=1,
             relative_permittivity=1.0, bgk=None) -> Config1D:
    """bgk = (frequency, neutral_temperature_velocity) enables the legacy BGK
    collision model (CollisionConfig with model = bgk)."""
    c = Config1D()
    c.boundary, c.velocity_dimensions, c.units = boundary, velocity_dimensions, units
    c.relative_permittivity = relative_permittivity
    c.nx, c.length, c.dt = nx, length, dt
    c.phi_left, c.phi_right = phi_left, phi_right
    c.drive_left = VoltageDrive(*drive_left)
    c.drive_right = VoltageDrive(*drive_right)
    c.precision, c.seed = precision, seed
    c.nspecies = len(species)
    for i, (q, m, w, cap) in enumerate(species):
        c.species[i] = SpeciesCfg(q, m, w, cap)
    c.nmodels = len(models)
    for i, mm in enumerate(models):
        c.models[i] = mm
    if bgk is not None:
        c.bgk_enabled, c.bgk_frequency, c.bgk_neutral_velocity = 1, bgk[0], bgk[1]
    return c


class Simulation1D:
    """pic::Simulation (1D1V/1D3V) on the device, through the C ABI."""

    def __init__(self, cfg: Config1D, tables: Tables | None = None):
        self.cfg = cfg
        self._tables = tables
        h = C.c_void_p()
        rc = lib().apic_sim1d_create(C.byref(cfg), C.byref(h))
        if rc != 0:
            raise ApicError(rc, lib().apic_sim1d_last_error(None).decode())
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            if _lib is not None:  # the library outlives every handle, except at interpreter exit
                _lib.apic_sim1d_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def load(self, species, x, v, v_half=None, vy=None, vz=None, alive=None):
        n = len(x)
        conv = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        x, v, v_half, vy, vz = map(conv, (x, v, v_half, vy, vz))
        al = None if alive is None else np.ascontiguousarray(alive, dtype=np.uint8)
        _check(lib().apic_sim1d_load_particles(self.h, species, n, dptr(x), dptr(v), dptr(v_half), dptr(vy),
                                               dptr(vz), None if al is None else al.ctypes.data_as(_U8P)), self.h)

    def initialize(self):
        _check(lib().apic_sim1d_initialize(self.h), self.h)

    def resume(self, time, step):
        _check(lib().apic_sim1d_resume(self.h, time, step), self.h)

    def step(self, n=1):
        _check(lib().apic_sim1d_step(self.h, n), self.h)

    def synchronize(self):
        _check(lib().apic_sim1d_synchronize(self.h), self.h)

    def set_wait_limit(self, seconds):
        _check(lib().apic_sim1d_set_wait_limit(self.h, seconds), self.h)

    def count(self, species) -> int:
        n = C.c_size_t()
        _check(lib().apic_sim1d_count(self.h, species, C.byref(n)), self.h)
        return n.value

    def particles(self, species) -> dict:
        n = self.count(species)
        out = {k: np.zeros(n) for k in ("x", "v", "vh", "vy", "vz")}
        got = C.c_size_t()
        _check(lib().apic_sim1d_read_particles(self.h, species, n, *[dptr(out[k]) for k in ("x", "v", "vh", "vy", "vz")],
                                               C.byref(got)), self.h)
        return out

    def fields(self):
        n = self.cfg.nx
        rho, phi, E = np.zeros(n), np.zeros(n), np.zeros(n)
        _check(lib().apic_sim1d_read_fields(self.h, dptr(rho), dptr(phi), dptr(E)), self.h)
        return rho, phi, E

    def sample(self) -> Sample1D:
        s = Sample1D()
        _check(lib().apic_sim1d_sample(self.h, C.byref(s)), self.h)
        return s

    def collision_totals(self) -> CollisionTotals:
        t = CollisionTotals()
        _check(lib().apic_sim1d_collision_totals(self.h, C.byref(t)), self.h)
        return t

    def boundary_losses(self, species) -> BoundaryLoss:
        b = BoundaryLoss()
        _check(lib().apic_sim1d_boundary_losses(self.h, species, C.byref(b)), self.h)
        return b

    def cuda_stream(self) -> int:
        ptr = C.c_void_p()
        _check(lib().apic_sim1d_cuda_stream(self.h, C.byref(ptr)), self.h)
        return ptr.value or 0

    def set_kernel_timing(self, enable: bool):
        _check(lib().apic_sim1d_set_kernel_timing(self.h, int(enable)), self.h)

    def kernel_times(self):
        a, b = C.c_double(), C.c_double()
        n = C.c_uint64()
        _check(lib().apic_sim1d_kernel_times(self.h, C.byref(a), C.byref(b), C.byref(n)), self.h)
        return a.value, b.value, n.value

    # -- CCP campaign diagnostics --
    def enable_power_transfer(self):
        _check(lib().apic_sim1d_enable_power_transfer(self.h), self.h)

    def electric_work(self, species) -> float:
        w = C.c_double()
        _check(lib().apic_sim1d_power_transfer(self.h, species, C.byref(w)), self.h)
        return w.value

    def enable_spatial_average(self, sa: SpatialAverage1D):
        self._sa = sa
        _check(lib().apic_sim1d_enable_spatial_average(self.h, C.byref(sa)), self.h)

    def spatial_counts(self):
        """(samples, collision steps, per-bin samples, per-bin collision steps)"""
        P = int(self._sa.phase_bins)
        a, b = np.zeros(1, np.uint64), np.zeros(1, np.uint64)
        pa, pb = np.zeros(max(P, 1), np.uint64), np.zeros(max(P, 1), np.uint64)
        _check(lib().apic_sim1d_spatial_average_counts(self.h, a.ctypes.data_as(_U64P), b.ctypes.data_as(_U64P),
                                                       pa.ctypes.data_as(_U64P), pb.ctypes.data_as(_U64P)), self.h)
        return int(a[0]), int(b[0]), pa[:P], pb[:P]

    def spatial_sums(self, quantity, index=0, phase=-1):
        out = np.zeros(self.cfg.nx)
        _check(lib().apic_sim1d_spatial_sums(self.h, quantity, index, phase, dptr(out)), self.h)
        return out

    def phase_eedf(self, phase, region):
        """(counts [macro, overflow macro], sums [represented, overflow
        represented, weighted energy, energy^2, v_x, v_y, v_z], histogram)"""
        e = PhaseEedf1D()
        hist = np.zeros(max(int(self._sa.eedf_bins), 1))
        _check(lib().apic_sim1d_phase_eedf(self.h, phase, region, C.byref(e), dptr(hist)), self.h)
        cnt = np.array([e.macro_observations, e.overflow_macro_observations], np.uint64)
        sums = np.array([e.represented_observations, e.overflow_represented_observations, e.weighted_energy_sum,
                         e.weighted_energy_squared_sum, e.weighted_velocity_x_sum, e.weighted_velocity_y_sum,
                         e.weighted_velocity_z_sum])
        return cnt, sums, hist[:int(self._sa.eedf_bins)]

    @property
    def time(self) -> float:
        return lib().apic_sim1d_time(self.h)

    @property
    def step_count(self) -> int:
        return lib().apic_sim1d_step_count(self.h)


def step_group(sims, nsteps=1):
    """Steps several Simulation1D runs together (their work overlaps on the GPU)."""
    arr = (C.c_void_p * len(sims))(*[s.h for s in sims])
    rc = lib().apic_sim1d_step_group(arr, len(sims), nsteps)
    if rc != 0:
        for s in sims:
            msg = lib().apic_sim1d_last_error(s.h)
            if msg:
                raise ApicError(rc, msg.decode())
        raise ApicError(rc, "step_group failed")


def deposit_solve_gather_1d(boundary, nx, length, permittivity, phi_left, phi_right, charges, weights, xs, xq=None):
    ns = len(xs)
    xs = [np.ascontiguousarray(x, dtype=np.float64) for x in xs]
    counts = (C.c_size_t * ns)(*[len(x) for x in xs])
    ptrs = (_DP * ns)(*[dptr(x) for x in xs])
    q = np.ascontiguousarray(charges, dtype=np.float64)
    w = np.ascontiguousarray(weights, dtype=np.float64)
    rho, phi, E = np.zeros(nx), np.zeros(nx), np.zeros(nx)
    xq = np.zeros(0) if xq is None else np.ascontiguousarray(xq, dtype=np.float64)
    eq = np.zeros(len(xq))
    rc = lib().apic_deposit_solve_gather_1d(boundary, nx, length, permittivity, phi_left, phi_right, ns, dptr(q),
                                            dptr(w), counts, ptrs, dptr(rho), dptr(phi), dptr(E), len(xq),
                                            dptr(xq) if len(xq) else None, dptr(eq) if len(xq) else None)
    _check(rc)
    return rho, phi, E, eq


def collide3(model: MccModel, particle_mass, v3, dt, draws=None, offsets=None, seed=0, step=0, stream=0):
    v3 = np.ascontiguousarray(v3, dtype=np.float64).copy()
    n = v3.shape[0]
    stats = (CollideStats * n)()
    if draws is not None:
        draws = np.ascontiguousarray(draws, dtype=np.uint64)
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        dp, op = draws.ctypes.data_as(_U64P), offsets.ctypes.data_as(_U64P)
    else:
        dp = op = None
    _check(lib().apic_collide3(C.byref(model), particle_mass, n, dptr(v3), dt, dp, op, seed, step, stream, stats))
    return v3, stats


# ---------------------------------------------------------------------------
# Structured 2D3V / 3D3V periodic simulation


class ConfigND(C.Structure):
    _fields_ = [
        ("dims", C.c_int), ("n", C.c_size_t * 3), ("length", C.c_double * 3), ("dt", C.c_double),
        ("units", C.c_int), ("relative_permittivity", C.c_double), ("magnetic_field", C.c_double * 3),
        ("out_of_plane_depth", C.c_double), ("precision", C.c_int), ("sort_interval", C.c_size_t),
        ("nspecies", C.c_int), ("species", SpeciesCfg * MAX_SPECIES),
        ("push_items", C.c_int),
        ("species_sort_interval", C.c_size_t * MAX_SPECIES),
        ("profile_axis", C.c_int), ("profile_rows", C.c_size_t),
        ("profile_coordinates", C.POINTER(C.c_double)), ("profile_values", C.POINTER(C.c_double)),
        ("wall_axis", C.c_int * 2), ("wall_potential", C.c_double * 4), ("particle_boundary", C.c_int * 4),
        ("wall_axis_z", C.c_int), ("particle_boundary_z", C.c_int * 2),
    ]


class SampleND(C.Structure):
    _fields_ = [
        ("step", C.c_uint64), ("time", C.c_double), ("kinetic_energy", C.c_double), ("field_energy", C.c_double),
        ("total_energy", C.c_double), ("charge_l1", C.c_double), ("live_particles", C.c_uint64),
        ("kinetic_by_species", C.c_double * MAX_SPECIES),
    ]


_SZP = C.POINTER(C.c_size_t)


def _bind_nd():
    L = lib()
    if getattr(L, "_nd_bound", False):
        return L
    L.apic_simnd_create.argtypes = [C.POINTER(ConfigND), C.POINTER(C.c_void_p)]
    L.apic_simnd_destroy.argtypes = [C.c_void_p]
    L.apic_simnd_last_error.restype = C.c_char_p
    L.apic_simnd_last_error.argtypes = [C.c_void_p]
    L.apic_simnd_load_particles.argtypes = [C.c_void_p, C.c_int, C.c_size_t, _DP, _DP, _DP]
    L.apic_simnd_initialize.argtypes = [C.c_void_p]
    L.apic_simnd_resume.argtypes = [C.c_void_p, C.c_double, C.c_uint64]
    L.apic_simnd_step.argtypes = [C.c_void_p, C.c_size_t]
    L.apic_simnd_synchronize.argtypes = [C.c_void_p]
    L.apic_simnd_count.argtypes = [C.c_void_p, C.c_int, _SZP]
    L.apic_simnd_read_particles.argtypes = [C.c_void_p, C.c_int, C.c_size_t, _DP, _DP, _DP, _SZP]
    L.apic_simnd_read_fields.argtypes = [C.c_void_p, _DP, _DP, _DP]
    L.apic_simnd_sample.argtypes = [C.c_void_p, C.POINTER(SampleND)]
    L.apic_simnd_cuda_stream.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
    L.apic_simnd_set_kernel_timing.argtypes = [C.c_void_p, C.c_int]
    L.apic_simnd_kernel_times.argtypes = [C.c_void_p, _DP, _DP, _DP, _U64P]
    L.apic_field_solve_periodic_nd.argtypes = [C.c_int, _SZP, _DP, C.c_double, _DP, _DP, _DP]
    L._nd_bound = True
    return L


def _check_nd(rc, handle=None):
    if rc != 0:
        msg = _bind_nd().apic_simnd_last_error(handle).decode() if handle is not None else ""
        if not msg:
            msg = _bind_nd().apic_simnd_last_error(None).decode()
        raise ApicError(rc, msg)


def config_nd(*, dims, n, length, dt, species, magnetic_field=(0.0, 0.0, 0.0), units=NORMALIZED,
              relative_permittivity=1.0, out_of_plane_depth=1.0, precision=FP64, sort_interval=16,
              push_items=0, species_sort_interval=None, magnetic_field_profile=None, walls=None) -> ConfigND:
    """magnetic_field_profile: optional (axis, coordinates, values[rows][3]), B
    tabulated along one axis (the arrays are kept on the returned config until
    the simulation is created, which copies them)."""
    c = ConfigND()
    c.dims = dims
    c.n[:] = list(n) + [1] * (3 - len(n))
    c.length[:] = list(length) + [1.0] * (3 - len(length))
    c.dt, c.units, c.relative_permittivity = dt, units, relative_permittivity
    c.magnetic_field[:] = list(magnetic_field)
    c.out_of_plane_depth, c.precision, c.sort_interval = out_of_plane_depth, precision, sort_interval
    c.push_items = push_items
    if species_sort_interval:
        c.species_sort_interval[:] = list(species_sort_interval) + [0] * (MAX_SPECIES - len(species_sort_interval))
    c.nspecies = len(species)
    for i, (q, m, w, cap) in enumerate(species):
        c.species[i] = SpeciesCfg(q, m, w, cap)
    if magnetic_field_profile is not None:
        ax, coords, values = magnetic_field_profile
        pc = np.ascontiguousarray(coords, dtype=np.float64)
        pv = np.ascontiguousarray(values, dtype=np.float64).ravel()
        if pv.size != 3 * pc.size:
            raise ValueError("magnetic_field_profile values must be rows x 3")
        c._profile_keep = (pc, pv)
        c.profile_axis, c.profile_rows = int(ax), int(pc.size)
        c.profile_coordinates = pc.ctypes.data_as(C.POINTER(C.c_double))
        c.profile_values = pv.ctypes.data_as(C.POINTER(C.c_double))
    if walls is not None:
        # (wall axes [x, y(, z)], potentials [left, right, bottom, top] (3D: None,
        #  grounded), particle boundaries [left, right, bottom, top(, back, front)]:
        #  0 auto, 1 absorbing, 2 reflecting, 3 periodic)
        axes, pots, pbs = walls
        for a in range(2):
            c.wall_axis[a] = int(axes[a])
        if len(axes) > 2:
            c.wall_axis_z = int(axes[2])
        for k in range(4):
            c.wall_potential[k] = float(pots[k]) if pots is not None else 0.0
            c.particle_boundary[k] = int(pbs[k])
        for k in range(4, len(pbs)):
            c.particle_boundary_z[k - 4] = int(pbs[k])
    return c


class SimulationND:
    """pic::Simulation2D / Simulation3D (fully periodic) on the device."""

    def __init__(self, cfg: ConfigND):
        self.cfg = cfg
        self.dims = cfg.dims
        self.N = int(np.prod([cfg.n[a] for a in range(cfg.dims)]))
        h = C.c_void_p()
        rc = _bind_nd().apic_simnd_create(C.byref(cfg), C.byref(h))
        if rc != 0:
            raise ApicError(rc, _bind_nd().apic_simnd_last_error(None).decode())
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            _bind_nd().apic_simnd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load(self, species, pos, v, v_half=None):
        pos = np.ascontiguousarray(np.asarray(pos, dtype=np.float64)[: self.dims])
        v = np.ascontiguousarray(v, dtype=np.float64)
        vh = None if v_half is None else np.ascontiguousarray(v_half, dtype=np.float64)
        n = pos.shape[1]
        _check_nd(_bind_nd().apic_simnd_load_particles(self.h, species, n, dptr(pos), dptr(v), dptr(vh)), self.h)

    def initialize(self):
        _check_nd(_bind_nd().apic_simnd_initialize(self.h), self.h)

    def resume(self, time, step):
        _check_nd(_bind_nd().apic_simnd_resume(self.h, time, step), self.h)

    def step(self, n=1):
        _check_nd(_bind_nd().apic_simnd_step(self.h, n), self.h)

    def synchronize(self):
        _check_nd(_bind_nd().apic_simnd_synchronize(self.h), self.h)

    def count(self, species):
        n = C.c_size_t()
        _check_nd(_bind_nd().apic_simnd_count(self.h, species, C.byref(n)), self.h)
        return n.value

    def particles(self, species):
        n = self.count(species)
        pos, v, vh = np.zeros((3, n)), np.zeros((3, n)), np.zeros((3, n))
        got = C.c_size_t()
        _check_nd(_bind_nd().apic_simnd_read_particles(self.h, species, n, dptr(pos), dptr(v), dptr(vh), C.byref(got)),
                  self.h)
        return pos, v, vh

    def alive(self, species):
        n = self.count(species) if hasattr(self, "count") else None
        n = n if n is not None else len(self.particles(species)[0][0])
        out = np.zeros(n, np.uint8)
        L = lib()
        L.apic_simnd_read_alive.argtypes = [C.c_void_p, C.c_int, C.c_size_t, _U8P]
        _check_nd(L.apic_simnd_read_alive(self.h, species, n, out.ctypes.data_as(_U8P)), self.h)
        return out

    def boundary_losses(self, species):
        """absorbed counts of one species per side: left, right, bottom, top
        (, back, front in 3D)"""
        out = np.zeros(2 * self.dims, np.uint64)
        L = lib()
        L.apic_simnd_boundary_losses.argtypes = [C.c_void_p, C.c_int, _U64P]
        _check_nd(L.apic_simnd_boundary_losses(self.h, species, out.ctypes.data_as(_U64P)), self.h)
        return out

    def fields(self):
        rho, phi, E = np.zeros(self.N), np.zeros(self.N), np.zeros(self.dims * self.N)
        _check_nd(_bind_nd().apic_simnd_read_fields(self.h, dptr(rho), dptr(phi), dptr(E)), self.h)
        return rho, phi, E.reshape(self.dims, self.N)

    def sample(self) -> SampleND:
        s = SampleND()
        _check_nd(_bind_nd().apic_simnd_sample(self.h, C.byref(s)), self.h)
        return s

    def cuda_stream(self) -> int:
        ptr = C.c_void_p()
        _check_nd(_bind_nd().apic_simnd_cuda_stream(self.h, C.byref(ptr)), self.h)
        return ptr.value or 0

    def set_kernel_timing(self, enable: bool):
        _check_nd(_bind_nd().apic_simnd_set_kernel_timing(self.h, int(enable)), self.h)

    def kernel_times(self):
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        n = C.c_uint64()
        _check_nd(_bind_nd().apic_simnd_kernel_times(self.h, C.byref(a), C.byref(b), C.byref(c), C.byref(n)), self.h)
        return a.value, b.value, c.value, n.value


def _simnd_launch_count(self):
    n = C.c_uint64()
    L = _bind_nd()
    L.apic_simnd_launch_count.argtypes = [C.c_void_p, C.POINTER(C.c_uint64)]
    _check_nd(L.apic_simnd_launch_count(self.h, C.byref(n)), self.h)
    return n.value


SimulationND.launch_count = _simnd_launch_count


def field_solve_periodic_nd(dims, n, length, permittivity, rho):
    N = int(np.prod(n[:dims]))
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    phi, E = np.zeros(N), np.zeros(dims * N)
    ns = (C.c_size_t * 3)(*(list(n) + [1] * (3 - len(n))))
    Lv = np.ascontiguousarray(list(length) + [1.0] * (3 - len(length)), dtype=np.float64)
    _check_nd(_bind_nd().apic_field_solve_periodic_nd(dims, ns, dptr(Lv), permittivity, dptr(rho), dptr(phi), dptr(E)))
    return phi, E.reshape(dims, N)


def field_solve_dirichlet_nd(n, length, permittivity, rho, side_potentials=None):
    """FieldSolver::solve(Mesh2D&/Mesh3D&) with walls on every side (2D side
    potentials left, right, bottom, top; 3D grounded); returns (phi, E[dims])."""
    L = _bind_nd()
    L.apic_field_solve_dirichlet_nd.argtypes = [C.c_int, C.POINTER(C.c_size_t), C.POINTER(C.c_double), C.c_double,
                                                C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                                C.POINTER(C.c_double)]
    dims = len(n)
    N = int(np.prod(n))
    rho = np.ascontiguousarray(rho, dtype=np.float64).ravel()
    if rho.size != N:
        raise ValueError("rho must hold prod(n) values")
    phi, E = np.zeros(N), np.zeros(dims * N)
    ns = (C.c_size_t * 3)(*(list(n) + [1] * (3 - dims)))
    Lv = np.ascontiguousarray(list(length) + [1.0] * (3 - dims), dtype=np.float64)
    pot = None if side_potentials is None else np.ascontiguousarray(side_potentials, dtype=np.float64)
    _check_nd(L.apic_field_solve_dirichlet_nd(dims, ns, dptr(Lv), permittivity, dptr(pot) if pot is not None else None,
                                              dptr(rho), dptr(phi), dptr(E)))
    return phi, E.reshape(dims, N)


def field_solve_mixed_2d(n, length, periodic_axis, permittivity, lower_potential, upper_potential, rho):
    """FieldSolver::solve(Mesh2D&) with one periodic axis (0: x, 1: y) and wall
    potentials on the other; returns (phi, E[2]) on the nx * ny mesh."""
    L = _bind_nd()
    L.apic_field_solve_mixed_2d.argtypes = [C.POINTER(C.c_size_t), C.POINTER(C.c_double), C.c_int, C.c_double,
                                            C.c_double, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                            C.POINTER(C.c_double)]
    N = int(n[0] * n[1])
    rho = np.ascontiguousarray(rho, dtype=np.float64).ravel()
    if rho.size != N:
        raise ValueError("rho must hold nx * ny values")
    phi, E = np.zeros(N), np.zeros(2 * N)
    ns = (C.c_size_t * 2)(int(n[0]), int(n[1]))
    Lv = np.ascontiguousarray(length, dtype=np.float64)
    _check_nd(L.apic_field_solve_mixed_2d(ns, dptr(Lv), periodic_axis, permittivity, lower_potential,
                                          upper_potential, dptr(rho), dptr(phi), dptr(E)))
    return phi, E.reshape(2, N)


class ApcInfo(C.Structure):
    _fields_ = [
        ("units", C.c_int), ("relative_permittivity", C.c_double), ("permittivity", C.c_double),
        ("velocity_dimensions", C.c_int), ("collisions_enabled", C.c_int), ("collision_signature", C.c_uint64),
        ("candidates", C.c_uint64), ("null_collisions", C.c_uint64), ("nchannels", C.c_size_t),
        ("boundary_loss_origin_step", C.c_uint64), ("power_transfer_origin_step", C.c_uint64),
        ("spatial_average_enabled", C.c_int), ("step", C.c_uint64), ("time", C.c_double), ("nspecies", C.c_size_t),
    ]


def _bind_apc():
    L = lib()
    if getattr(L, "_apc_bound", False):
        return L
    L.apic_apc_last_error.restype = C.c_char_p
    L.apic_apc_read.argtypes = [C.c_char_p, C.POINTER(C.c_void_p)]
    L.apic_apc_free.argtypes = [C.c_void_p]
    L.apic_apc_write.argtypes = [C.c_void_p, C.c_char_p]
    L.apic_apc_get_info.argtypes = [C.c_void_p, C.POINTER(ApcInfo)]
    L.apic_apc_channel.argtypes = [C.c_void_p, C.c_size_t, _U64P, _DP]
    L.apic_apc_species.argtypes = [C.c_void_p, C.c_size_t, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t),
                                   C.POINTER(BoundaryLoss), _DP]
    L.apic_apc_particles.argtypes = [C.c_void_p, C.c_size_t, _DP, _DP, _DP, _DP, _DP, _U8P]
    L.apic_sim1d_load_checkpoint.argtypes = [C.c_void_p, C.c_void_p]
    L.apic_sim1d_save_checkpoint.argtypes = [C.c_void_p, C.c_void_p, C.c_char_p]
    L._apc_bound = True
    return L


class Checkpoint:
    """A 1D3V checkpoint (.apc version 12) read on the host (apic_apc_*)."""

    def __init__(self, path):
        L = _bind_apc()
        h = C.c_void_p()
        rc = L.apic_apc_read(path.encode(), C.byref(h))
        if rc:
            raise ApicError(rc, L.apic_apc_last_error().decode())
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            _bind_apc().apic_apc_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def write(self, path):
        L = _bind_apc()
        rc = L.apic_apc_write(self.h, path.encode())
        if rc:
            raise ApicError(rc, L.apic_apc_last_error().decode())

    def info(self) -> ApcInfo:
        out = ApcInfo()
        _bind_apc().apic_apc_get_info(self.h, C.byref(out))
        return out

    def channel(self, k):
        c, e = C.c_uint64(), C.c_double()
        _bind_apc().apic_apc_channel(self.h, k, C.byref(c), C.byref(e))
        return c.value, e.value

    def species(self, k):
        name = C.create_string_buffer(256)
        n = C.c_size_t()
        loss = BoundaryLoss()
        w = C.c_double()
        _bind_apc().apic_apc_species(self.h, k, name, 256, C.byref(n), C.byref(loss), C.byref(w))
        return name.value.decode(), n.value, loss, w.value

    def particles(self, k):
        n = self.species(k)[1]
        out = {key: np.zeros(n) for key in ("x", "v", "vy", "vz", "vh")}
        alive = np.zeros(n, np.uint8)
        _bind_apc().apic_apc_particles(self.h, k, *[dptr(out[key]) for key in ("x", "v", "vy", "vz", "vh")],
                                       alive.ctypes.data_as(_U8P))
        out["alive"] = alive
        return out


def _sim1d_load_checkpoint(self, checkpoint: Checkpoint):
    _check(_bind_apc().apic_sim1d_load_checkpoint(self.h, checkpoint.h), self.h)


def _sim1d_save_checkpoint(self, meta: Checkpoint, path):
    _check(_bind_apc().apic_sim1d_save_checkpoint(self.h, meta.h, path.encode()), self.h)


Simulation1D.load_checkpoint = _sim1d_load_checkpoint
Simulation1D.save_checkpoint = _sim1d_save_checkpoint


class ParticleState:
    """An AuroraPIC particle-state file (.aps version 1, the reference's
    external initial state), parsed by the library: `species` maps each name
    (sorted) to (pos[3][n], vel[3][n]) arrays ready for the loaders."""

    def __init__(self, path, max_particles=1 << 40):
        L = lib()
        L.apic_aps_read.argtypes = [C.c_char_p, C.c_size_t, C.POINTER(C.c_void_p)]
        L.apic_aps_info.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_size_t),
                                    C.POINTER(C.c_size_t), C.POINTER(C.c_uint64)]
        L.apic_aps_species.argtypes = [C.c_void_p, C.c_size_t, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]
        L.apic_aps_records.argtypes = [C.c_void_p, C.c_size_t, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.apic_aps_free.argtypes = [C.c_void_p]
        L.apic_aps_last_error.restype = C.c_char_p
        h = C.c_void_p()
        rc = L.apic_aps_read(os.fsencode(path), max_particles, C.byref(h))
        if rc:
            raise ApicError(rc, L.apic_aps_last_error().decode())
        try:
            d, u, n, ns, sig = C.c_int(), C.c_int(), C.c_size_t(), C.c_size_t(), C.c_uint64()
            L.apic_aps_info(h, C.byref(d), C.byref(u), C.byref(n), C.byref(ns), C.byref(sig))
            self.dimension, self.units, self.particle_count, self.signature = d.value, u.value, n.value, sig.value
            self.species = {}
            for k in range(ns.value):
                name = C.create_string_buffer(4096)
                cnt = C.c_size_t()
                L.apic_aps_species(h, k, name, 4096, C.byref(cnt))
                pos, vel = np.zeros((3, cnt.value)), np.zeros((3, cnt.value))
                L.apic_aps_records(h, k, dptr(pos), dptr(vel))
                self.species[name.value.decode()] = (pos, vel)
        finally:
            L.apic_aps_free(h)

    @staticmethod
    def write(path, dimension, units, species, overwrite=False):
        """species: {name: (pos[3][n], vel[3][n])}; returns the signature."""
        L = lib()
        L.apic_aps_write.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_size_t, C.POINTER(C.c_char_p),
                                     C.POINTER(C.c_size_t), C.POINTER(C.POINTER(C.c_double)),
                                     C.POINTER(C.POINTER(C.c_double)), C.c_int, C.POINTER(C.c_uint64)]
        L.apic_aps_last_error.restype = C.c_char_p
        names = list(species)
        keep = [(np.ascontiguousarray(species[k][0], dtype=np.float64), np.ascontiguousarray(species[k][1], dtype=np.float64))
                for k in names]
        nm = (C.c_char_p * len(names))(*[k.encode() for k in names])
        counts = (C.c_size_t * len(names))(*[p.shape[1] for p, _ in keep])
        pp = (C.POINTER(C.c_double) * len(names))(*[dptr(p) for p, _ in keep])
        vv = (C.POINTER(C.c_double) * len(names))(*[dptr(v) for _, v in keep])
        sig = C.c_uint64()
        rc = L.apic_aps_write(os.fsencode(path), dimension, units, len(names), nm, counts, pp, vv, int(overwrite),
                              C.byref(sig))
        if rc:
            raise ApicError(rc, L.apic_aps_last_error().decode())
        return sig.value


def _simnd_load_maxwellian(self, species, n, seed, thermal_speed, drift_x=0.0, perturb_axis=0, perturb_amplitude=0.0):
    L = _bind_nd()
    L.apic_simnd_load_maxwellian.argtypes = [C.c_void_p, C.c_int, C.c_size_t, C.c_uint64, C.c_double, C.c_double,
                                             C.c_int, C.c_double]
    _check_nd(L.apic_simnd_load_maxwellian(self.h, species, n, seed, thermal_speed, drift_x, perturb_axis,
                                           perturb_amplitude), self.h)


SimulationND.load_maxwellian = _simnd_load_maxwellian


# ---------------------------------------------------------------------------
# Homogeneous electron swarms (run_swarm_benchmark) and the serving loop

SWARM_FIXED, SWARM_BRANCHING = 0, 1


class SwarmConfig(C.Structure):
    _fields_ = [
        ("neutral_density", C.c_double), ("neutral_temperature", C.c_double),
        ("max_frequency", C.c_double), ("timestep", C.c_double),
        ("steps", C.c_size_t), ("burn_in_steps", C.c_size_t), ("particles", C.c_size_t),
        ("population_model", C.c_int), ("population_limit", C.c_size_t), ("uncertainty_blocks", C.c_size_t),
        ("work_item_limit", C.c_uint64),
        ("initial_mean_energy_ev", C.c_double), ("max_energy_ev", C.c_double), ("seed", C.c_uint64),
        ("precision", C.c_int),
    ]


class SwarmResult(C.Structure):
    _fields_ = [
        ("id", C.c_uint64), ("status", C.c_int), ("message", C.c_char * 256),
        ("steps_done", C.c_uint64), ("converged", C.c_int), ("latency_s", C.c_double), ("queue_s", C.c_double),
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


class SwarmServerConfig(C.Structure):
    _fields_ = [("memory_budget_bytes", C.c_size_t), ("max_runs", C.c_int), ("precision", C.c_int),
                ("steps_per_launch", C.c_size_t)]


class SwarmRequest(C.Structure):
    _fields_ = [
        ("reduced_field_td", C.c_double), ("particles", C.c_size_t), ("seed", C.c_uint64),
        ("steps", C.c_size_t), ("burn_in_steps", C.c_size_t), ("uncertainty_blocks", C.c_size_t),
        ("tolerance", C.c_double), ("population_model", C.c_int), ("population_limit", C.c_size_t),
        ("initial_mean_energy_ev", C.c_double), ("max_energy_ev", C.c_double), ("timestep", C.c_double),
    ]


class SpatialTownsendConfig(C.Structure):
    """apic_spatial_townsend_config: the spatial_* controls of SwarmBenchmarkConfig."""
    _fields_ = [
        ("histories", C.c_size_t), ("length_m", C.c_double), ("bins", C.c_size_t),
        ("fit_begin_bin", C.c_size_t), ("fit_end_bin", C.c_size_t), ("max_steps", C.c_size_t),
        ("work_item_limit", C.c_uint64), ("min_r_squared", C.c_double),
    ]


class SpatialFluxPoint(C.Structure):
    _fields_ = [("distance_m", C.c_double), ("net_crossings_per_injected_electron", C.c_double),
                ("standard_error", C.c_double)]


class SpatialTownsendResult(C.Structure):
    _fields_ = [
        ("townsend_1_m", C.c_double), ("townsend_standard_error_1_m", C.c_double), ("fit_r_squared", C.c_double),
        ("histories_completed", C.c_uint64), ("maximum_active_particles", C.c_uint64),
        ("particle_updates", C.c_uint64),
    ]


def _bind_swarm():
    L = lib()
    if getattr(L, "_swarm_bound", False):
        return L
    P = C.c_void_p
    L.apic_swarm_run.argtypes = [C.POINTER(SwarmConfig), C.POINTER(MccModel), C.POINTER(C.c_double), C.c_size_t,
                                 C.POINTER(SwarmResult)]
    L.apic_swarm_last_error.restype = C.c_char_p
    L.apic_swarm_last_error.argtypes = [P]
    L.apic_swarm_server_create.argtypes = [C.POINTER(SwarmServerConfig), C.POINTER(MccModel), C.POINTER(P)]
    L.apic_swarm_server_destroy.argtypes = [P]
    L.apic_swarm_server_submit.argtypes = [P, C.POINTER(SwarmRequest), C.POINTER(C.c_uint64)]
    L.apic_swarm_server_advance.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.apic_swarm_server_poll.argtypes = [P, C.c_uint64, C.POINTER(SwarmResult), C.POINTER(C.c_int)]
    L.apic_swarm_server_launch.argtypes = [P]
    L.apic_swarm_server_complete.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.apic_swarm_server_stats.argtypes = [P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_size_t)]
    L.apic_swarm_server_cuda_stream.argtypes = [P, C.POINTER(P)]
    L.apic_swarm_server_copy_bytes.argtypes = [P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.apic_swarm_server_set_kernel_timing.argtypes = [P, C.c_int]
    L.apic_swarm_server_kernel_times.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                                 C.POINTER(C.c_uint64), C.POINTER(C.c_double)]
    L.apic_swarm_spatial_townsend.argtypes = [
        C.POINTER(SwarmConfig), C.POINTER(SpatialTownsendConfig), C.POINTER(MccModel), C.c_double, C.c_uint64,
        C.POINTER(C.c_uint64), C.POINTER(SpatialTownsendResult), C.POINTER(SpatialFluxPoint), C.POINTER(C.c_double)]
    L._swarm_bound = True
    return L


def _check_swarm(rc, handle=None):
    if rc != 0:
        raise ApicError(rc, _bind_swarm().apic_swarm_last_error(handle).decode(errors="replace"))


def swarm_run(cfg: SwarmConfig, gas: MccModel, fields_td):
    """run_swarm_benchmark on the device: one SwarmResult per reduced field."""
    L = _bind_swarm()
    f = np.ascontiguousarray(fields_td, dtype=np.float64)
    out = (SwarmResult * len(f))()
    _check_swarm(L.apic_swarm_run(C.byref(cfg), C.byref(gas), f.ctypes.data_as(C.POINTER(C.c_double)), len(f), out))
    return list(out)


def swarm_spatial_townsend(cfg: SwarmConfig, sp: SpatialTownsendConfig, gas: MccModel, reduced_field_td, seed,
                           scan_particle_updates=0, history_crossings=False):
    """run_spatial_townsend on the device for one reduced field.  Returns
    (SpatialTownsendResult, profile[bins, 3] as (distance, mean net crossings,
    standard error), crossings[histories, bins] or None, scan updates after)."""
    L = _bind_swarm()
    out = SpatialTownsendResult()
    prof = (SpatialFluxPoint * max(int(sp.bins), 1))()
    cross = np.zeros((int(sp.histories), int(sp.bins))) if history_crossings else None
    scan = C.c_uint64(scan_particle_updates)
    _check_swarm(L.apic_swarm_spatial_townsend(
        C.byref(cfg), C.byref(sp), C.byref(gas), reduced_field_td, seed, C.byref(scan), C.byref(out), prof,
        None if cross is None else cross.ctypes.data_as(C.POINTER(C.c_double))))
    p = np.array([[q.distance_m, q.net_crossings_per_injected_electron, q.standard_error]
                  for q in prof[:int(sp.bins)]])
    return out, p, cross, scan.value


class SwarmServer:
    """The batched swarm server (admission by memory budget and run slots,
    graph-launched steps, retirement on convergence)."""

    def __init__(self, gas: MccModel, memory_budget_bytes, max_runs=64, precision=FP32, steps_per_launch=64):
        L = _bind_swarm()
        self.conf = SwarmServerConfig(memory_budget_bytes, max_runs, precision, steps_per_launch)
        h = C.c_void_p()
        _check_swarm(L.apic_swarm_server_create(C.byref(self.conf), C.byref(gas), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            _bind_swarm().apic_swarm_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, req: SwarmRequest) -> int:
        i = C.c_uint64()
        _check_swarm(_bind_swarm().apic_swarm_server_submit(self.h, C.byref(req), C.byref(i)), self.h)
        return i.value

    def advance(self):
        a, q = C.c_int(), C.c_int()
        _check_swarm(_bind_swarm().apic_swarm_server_advance(self.h, C.byref(a), C.byref(q)), self.h)
        return a.value, q.value

    def launch(self):
        """First half of advance(): enqueue the batch's steps and return."""
        _check_swarm(_bind_swarm().apic_swarm_server_launch(self.h), self.h)

    def complete(self):
        """Second half: wait, retire finished runs; returns (active, queued)."""
        a, q = C.c_int(), C.c_int()
        _check_swarm(_bind_swarm().apic_swarm_server_complete(self.h, C.byref(a), C.byref(q)), self.h)
        return a.value, q.value

    def poll(self, rid):
        out, done = SwarmResult(), C.c_int()
        _check_swarm(_bind_swarm().apic_swarm_server_poll(self.h, rid, C.byref(out), C.byref(done)), self.h)
        return out if done.value else None

    def stats(self):
        g, p, f = C.c_uint64(), C.c_uint64(), C.c_size_t()
        _check_swarm(_bind_swarm().apic_swarm_server_stats(self.h, C.byref(g), C.byref(p), C.byref(f)), self.h)
        return g.value, p.value, f.value

    def cuda_stream(self) -> int:
        s = C.c_void_p()
        _check_swarm(_bind_swarm().apic_swarm_server_cuda_stream(self.h, C.byref(s)), self.h)
        return s.value or 0

    def copy_bytes(self):
        """(host -> device, device -> host) bytes the server has copied."""
        a, b = C.c_uint64(), C.c_uint64()
        _check_swarm(_bind_swarm().apic_swarm_server_copy_bytes(self.h, C.byref(a), C.byref(b)), self.h)
        return a.value, b.value

    def kernel_launches(self) -> int:
        n = C.c_uint64()
        L = _bind_swarm()
        L.apic_swarm_server_kernel_launches.argtypes = [C.c_void_p, C.POINTER(C.c_uint64)]
        _check_swarm(L.apic_swarm_server_kernel_launches(self.h, C.byref(n)), self.h)
        return n.value

    def set_kernel_timing(self, enable: bool):
        _check_swarm(_bind_swarm().apic_swarm_server_set_kernel_timing(self.h, int(enable)), self.h)

    def kernel_times(self):
        """(push ms, collision ms, steps timed, push algorithmic bytes) since timing was enabled."""
        ms, cms, n, b = C.c_double(), C.c_double(), C.c_uint64(), C.c_double()
        _check_swarm(_bind_swarm().apic_swarm_server_kernel_times(self.h, C.byref(ms), C.byref(cms), C.byref(n),
                                                                  C.byref(b)), self.h)
        return ms.value, cms.value, n.value, b.value
