/*
 * aurorapic_b200.h - C ABI of the B200-native electrostatic PIC particle step.
 *
 * Drop-in boundary for AuroraPIC's structured-grid particle step.  The
 * reference is a C++ library (the headers under include/pic/); each entry point below names
 * the reference interface it replaces.  All entry points:
 *   - take plain pointers and sizes (host memory unless stated otherwise),
 *   - never throw and never retain caller memory after returning,
 *   - return an apic_status; the handle's last-error string explains failures
 *     (reference exceptions become status codes, see apic_status).
 * Calls on one handle are serialised on that handle's CUDA stream; separate
 * handles are independent.  Device memory is owned by the handle.
 */
#ifndef AURORAPIC_B200_H
#define AURORAPIC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define APIC_EXPORT __attribute__((visibility("default")))
#else
#define APIC_EXPORT
#endif

#define APIC_MAX_SPECIES 4
#define APIC_MAX_MODELS 4
#define APIC_MAX_CHANNELS 8

/* Reference exceptions map onto these codes:
 *   std::invalid_argument          -> APIC_ERR_INVALID
 *   MCC "exceeds max_frequency"    -> APIC_ERR_MAJORANT   (src/Collision.cpp:620-623, :680-684)
 *   MCC candidate limit            -> APIC_ERR_CANDIDATES (src/Collision.cpp:938-943)
 *   max_particles_per_species      -> APIC_ERR_CAPACITY   (src/Simulation.cpp:941-964)
 *   non-finite particle state      -> APIC_ERR_NONFINITE  (src/Collision.cpp:910-916)
 */
typedef enum {
    APIC_OK = 0,
    APIC_ERR_INVALID = 1,
    APIC_ERR_CUDA = 2,
    APIC_ERR_CAPACITY = 3,
    APIC_ERR_MAJORANT = 4,
    APIC_ERR_CANDIDATES = 5,
    APIC_ERR_NONFINITE = 6,
    APIC_ERR_TIMEOUT = 7,
    APIC_ERR_UNSUPPORTED = 8,
    APIC_ERR_STATE = 9,
    APIC_ERR_NO_DEVICE = 10
} apic_status;

typedef enum { APIC_PERIODIC = 0, APIC_DIRICHLET = 1 } apic_boundary;
typedef enum { APIC_NORMALIZED = 0, APIC_SI = 1 } apic_units;
/* Particle storage form.  FP64: x and velocities in double, bit-faithful to
 * the reference arithmetic.  FP32: integer cell index + float in-cell offset
 * and float velocities, with the particle arithmetic (gather, push, walls,
 * null-collision loop) in FP32; charge accumulation (64-bit fixed point),
 * field solve and energy ledgers stay FP64.  FP32_STORAGE (1D only): float
 * velocities with an FP64 position and FP64 arithmetic, for runs that want
 * the campaign diagnostics with FP32 velocity storage. */
typedef enum { APIC_FP64 = 0, APIC_FP32 = 1, APIC_FP32_STORAGE = 2 } apic_precision;

/* CollisionProcessKind, include/pic/Config.hpp:42-48 */
typedef enum {
    APIC_ELASTIC = 0,
    APIC_EXCITATION = 1,
    APIC_IONIZATION = 2,
    APIC_ATTACHMENT = 3,
    APIC_CHARGE_EXCHANGE = 4
} apic_process;
/* AngularScatteringKind, include/pic/Config.hpp:33-37 */
typedef enum { APIC_ISOTROPIC = 0, APIC_BACKWARD = 1, APIC_HENYEY_GREENSTEIN = 2 } apic_angular;
/* CollisionEnergyFrame, include/pic/Config.hpp:38-41 */
typedef enum { APIC_FRAME_PROJECTILE = 0, APIC_FRAME_CENTER_OF_MASS = 1 } apic_frame;

/* CollisionChannelConfig + CrossSectionTable, include/pic/Config.hpp:82-98,
 * include/pic/Collision.hpp:15-31.  Energies in joules (SI) or normalized
 * energy units, already multiplied by any energy_scale; strictly increasing. */
typedef struct {
    int process;            /* apic_process */
    int angular;            /* apic_angular */
    int energy_frame;       /* apic_frame */
    double threshold_energy;
    int secondary_species;  /* ionization: species index receiving the secondary */
    int ion_species;        /* ionization: species index receiving the ion */
    size_t rows;
    const double* energy;
    const double* sigma;
    /* Henyey-Greenstein only: MeanCosineTable (include/pic/Collision.hpp:33-48),
     * energies already multiplied by mean_cosine_energy_scale, strictly
     * increasing, covering the cross-section table; mean cosines in (-1, 1). */
    size_t mean_cosine_rows;
    const double* mean_cosine_energy;
    const double* mean_cosine;
} apic_mcc_channel;

/* CollisionConfig (null_collision), include/pic/Config.hpp:110-132 */
typedef struct {
    int species;                /* projectile species index */
    double neutral_density;
    double max_frequency;
    double neutral_mass;
    double neutral_temperature; /* thermal (8-sigma bounded Maxwellian) neutrals when > 0 and gas_units_si */
    int gas_units_si;
    size_t max_candidates;      /* max_candidates_per_particle */
    int nch;
    apic_mcc_channel ch[APIC_MAX_CHANNELS];
} apic_mcc_model;

/* SinusoidalVoltageConfig, include/pic/Config.hpp:139-143 */
typedef struct { double amplitude, frequency, phase; } apic_voltage_drive;

/* SpeciesConfig subset that the particle step reads, include/pic/Config.hpp:16-30 */
typedef struct {
    double charge, mass, weight;
    size_t capacity;            /* max_particles_per_species */
} apic_species;

/* Config subset of the 1D particle step, include/pic/Config.hpp:170-209 */
typedef struct {
    int boundary;               /* apic_boundary */
    int velocity_dimensions;    /* 1 or 3 */
    int units;                  /* apic_units */
    double relative_permittivity;
    size_t nx;
    double length, dt;
    double phi_left, phi_right;
    apic_voltage_drive drive_left, drive_right;
    int precision;              /* apic_precision */
    uint64_t seed;              /* Philox key of the collision streams */
    int nspecies;
    apic_species species[APIC_MAX_SPECIES];
    int nmodels;
    apic_mcc_model models[APIC_MAX_MODELS];
    /* The legacy BGK model (CollisionConfig with model = bgk,
     * src/Simulation.cpp:481-485, :771-834): each step every live particle of
     * every species is replaced, with probability 1 - exp(-frequency dt), by a
     * Maxwellian neutral of standard deviation bgk_neutral_velocity per
     * component, then its half-step velocity is re-initialised.  Its one
     * "bgk" channel is totals entry [0][0].  Excludes MCC models (nmodels = 0);
     * FP64 and FP32 storage forms. */
    int bgk_enabled;
    double bgk_frequency;
    double bgk_neutral_velocity;    /* neutral_temperature_velocity */
} apic_config1d;

/* DiagnosticSample, include/pic/Diagnostics.hpp (Simulation::sample,
 * src/Simulation.cpp:1140-1161). */
typedef struct {
    uint64_t step;
    double time;
    double kinetic_energy;
    double field_energy;
    double total_energy;
    double charge_l1;
    uint64_t live_particles;
    double phi_left, phi_right;
    double kinetic_by_species[APIC_MAX_SPECIES];
    uint64_t live_by_species[APIC_MAX_SPECIES];
} apic_sample1d;

/* CollisionDiagnostics totals, include/pic/Collision.hpp:64-70, laid out
 * [model][channel]. */
typedef struct {
    uint64_t candidates;
    uint64_t null_collisions;
    uint64_t channel_collisions[APIC_MAX_MODELS][APIC_MAX_CHANNELS];
    double channel_energy_change[APIC_MAX_MODELS][APIC_MAX_CHANNELS];
} apic_collision_totals;

/* BoundaryLoss1D, include/pic/Simulation.hpp:20-25 */
typedef struct {
    uint64_t absorbed_left, absorbed_right;
    double kinetic_energy_left, kinetic_energy_right;
} apic_boundary_loss;

/* Per-call collision statistics of one particle (CollisionStepStatistics,
 * include/pic/Collision.hpp:51-62).  Secondaries beyond 4 are counted only. */
typedef struct {
    uint64_t candidates, null_collisions;
    uint32_t channel_collisions[APIC_MAX_CHANNELS];
    double energy_change[APIC_MAX_CHANNELS];
    int nsecondaries;
    int secondary_channel[4];
    double secondary_velocity[4][3];
    double secondary_ion_velocity[4][3];
    int removed;
    uint32_t draws;             /* raw 64-bit draws consumed */
} apic_collide_stats;

typedef struct apic_sim1d apic_sim1d;

/* ---- library ------------------------------------------------------------ */
APIC_EXPORT const char* apic_version(void);
APIC_EXPORT const char* apic_status_string(int status);
/* Number of visible CUDA devices (0 when none). */
APIC_EXPORT int apic_device_count(void);

/* ---- 1D simulation (replaces pic::Simulation, include/pic/Simulation.hpp:56-64) */

/* Simulation::Simulation(Config), src/Simulation.cpp:341-470.  Validates the
 * configuration and allocates device storage for every species' capacity. */
APIC_EXPORT int apic_sim1d_create(const apic_config1d* cfg, apic_sim1d** out);
APIC_EXPORT void apic_sim1d_destroy(apic_sim1d* sim);
APIC_EXPORT const char* apic_sim1d_last_error(const apic_sim1d* sim);

/* Species::particles() mutation (include/pic/Species.hpp:18): replaces the
 * species' particles.  vy/vz may be NULL for 1D1V; v_half may be NULL
 * (then v_half = v, as the external-state loader does, src/Simulation.cpp:751-752);
 * alive may be NULL (all alive).  Dead entries are dropped. */
APIC_EXPORT int apic_sim1d_load_particles(apic_sim1d* sim, int species, size_t n,
                              const double* x, const double* v, const double* v_half,
                              const double* vy, const double* vz, const uint8_t* alive);

/* Simulation::initialize() after loaded particles, src/Simulation.cpp:698-769:
 * deposit_and_solve(0) then initialize_leapfrog_half_step for every particle. */
APIC_EXPORT int apic_sim1d_initialize(apic_sim1d* sim);

/* Restart from a state whose v_half is already set (the state after a
 * reference step() or checkpoint, src/Simulation.cpp:2018-2899): sets
 * time/step and runs deposit_and_solve(time). */
APIC_EXPORT int apic_sim1d_resume(apic_sim1d* sim, double time, uint64_t step);

/* Simulation::step() repeated nsteps times, src/Simulation.cpp:1008-1138.
 * Asynchronous: returns after enqueueing; errors surface at the next
 * synchronising call. */
APIC_EXPORT int apic_sim1d_step(apic_sim1d* sim, size_t nsteps);
/* Steps n independent runs nsteps each, their work overlapping on the GPU:
 * every run has its own stream, and steady steps go out two per CUDA graph
 * launch, round robin over the runs.  No reference counterpart (the
 * reference steps one Simulation at a time); each run's result is the one
 * apic_sim1d_step would give.  Asynchronous, like apic_sim1d_step. */
APIC_EXPORT int apic_sim1d_step_group(apic_sim1d* const* sims, size_t n, size_t nsteps);

/* Waits (bounded) for the handle's stream and returns the device error word. */
APIC_EXPORT int apic_sim1d_synchronize(apic_sim1d* sim);
/* Longest time (seconds, default 600) a synchronising call waits for the
 * handle's device work before it gives up with APIC_ERR_TIMEOUT; the work
 * itself is not cancelled, and a later synchronising call waits again.  No
 * reference counterpart (the reference's step() runs to completion). */
APIC_EXPORT int apic_sim1d_set_wait_limit(apic_sim1d* sim, double seconds);

/* Species::particles() read access.  Brings the state to the reference's
 * post-step() form (time-centred v) before copying. */
APIC_EXPORT int apic_sim1d_count(apic_sim1d* sim, int species, size_t* n);
APIC_EXPORT int apic_sim1d_read_particles(apic_sim1d* sim, int species, size_t capacity,
                              double* x, double* v, double* v_half,
                              double* vy, double* vz, size_t* n);
/* Grid::rho()/phi()/electric(), include/pic/Grid.hpp:15-20 */
APIC_EXPORT int apic_sim1d_read_fields(apic_sim1d* sim, double* rho, double* phi, double* electric);
/* Simulation::sample(), src/Simulation.cpp:1140-1161 */
APIC_EXPORT int apic_sim1d_sample(apic_sim1d* sim, apic_sample1d* out);
/* Simulation::collision_diagnostics(), include/pic/Simulation.hpp:70-72 */
APIC_EXPORT int apic_sim1d_collision_totals(apic_sim1d* sim, apic_collision_totals* out);
/* Simulation::species_boundary_losses(), include/pic/Simulation.hpp:73-76 */
APIC_EXPORT int apic_sim1d_boundary_losses(apic_sim1d* sim, int species, apic_boundary_loss* out);
APIC_EXPORT double apic_sim1d_time(const apic_sim1d* sim);
/* The handle's CUDA stream (cudaStream_t), for callers that order their own
 * work or timing events with the simulation. */
APIC_EXPORT int apic_sim1d_cuda_stream(apic_sim1d* sim, void** stream);
/* Per-kernel timing with CUDA events on the handle's stream: enable resets the
 * totals; kernel_times returns the summed particle-pass and post (field solve)
 * kernel milliseconds and the number of passes timed. */
APIC_EXPORT int apic_sim1d_set_kernel_timing(apic_sim1d* sim, int enable);
/* Speed at or below which model `model` skips the frequency-bound evaluation
 * (the bound provably holds there); above it the exact check runs. */
APIC_EXPORT int apic_sim1d_model_safe_speed(const apic_sim1d* sim, int model, double* speed);
APIC_EXPORT int apic_sim1d_kernel_times(apic_sim1d* sim, double* pass_ms, double* post_ms, uint64_t* passes);
APIC_EXPORT uint64_t apic_sim1d_step_count(const apic_sim1d* sim);

/* ---- 1D CCP campaign diagnostics ------------------------------------------ */

/* Enables the per-species electric-work ledger of Simulation::step (the work
 * term of every synchronisation and wall crossing, src/Simulation.cpp:1047-1056,
 * :1094-1132).  Before initialize()/resume(); initialize() resets it.  Costs one
 * more FP64 array per particle buffer (16 bytes of traffic per particle-step). */
APIC_EXPORT int apic_sim1d_enable_power_transfer(apic_sim1d* sim);
/* species_power_transfer()[species].electric_work, include/pic/Simulation.hpp:77-81 */
APIC_EXPORT int apic_sim1d_power_transfer(apic_sim1d* sim, int species, double* electric_work);

#define APIC_MAX_EEDF_REGIONS 8

/* SpatialAverage1DConfig + PhaseEedf1DConfig (include/pic/Config.hpp:145-168)
 * of an enabled spatial average: the EEDF species by index (-1: no phase
 * EEDF) and its regions by their bounds. */
typedef struct {
    size_t interval, start_step, end_step;
    double rf_frequency;
    size_t rf_cycles, phase_bins;
    int eedf_species;
    size_t eedf_bins;
    double eedf_energy_max;
    int eedf_regions;
    double eedf_x_min[APIC_MAX_EEDF_REGIONS], eedf_x_max[APIC_MAX_EEDF_REGIONS];
} apic_spatial_average1d;

/* PhaseEedfAccumulator1D without its histogram, include/pic/Simulation.hpp:43-54 */
typedef struct {
    uint64_t macro_observations, overflow_macro_observations;
    double represented_observations, overflow_represented_observations;
    double weighted_energy_sum, weighted_energy_squared_sum;
    double weighted_velocity_x_sum, weighted_velocity_y_sum, weighted_velocity_z_sum;
} apic_phase_eedf1d;

/* Quantities of apic_sim1d_spatial_sums: per-node sums over the samples of the
 * represented density, the velocity-weighted densities, the kinetic-energy
 * density (index = species), the potential, the field and its square (index
 * unused), and the spatial collision-energy density (index = channel, numbered
 * across the models in model order). */
enum {
    APIC_SA_DENSITY = 0, APIC_SA_VELOCITY_X = 1, APIC_SA_VELOCITY_Y = 2, APIC_SA_VELOCITY_Z = 3,
    APIC_SA_KINETIC_ENERGY = 4, APIC_SA_POTENTIAL = 5, APIC_SA_ELECTRIC = 6, APIC_SA_ELECTRIC_SQUARED = 7,
    APIC_SA_COLLISION_ENERGY = 8
};

/* validate_spatial_average_1d (src/Config.cpp:1377-1524) against a 1D
 * configuration, with the reference's messages.  Host only: needs no device. */
APIC_EXPORT int apic_spatial_average1d_validate(const apic_config1d* cfg, const apic_spatial_average1d* sa);
/* Enables the spatial average, phase bins, spatial collision energy and phase
 * EEDF of Simulation (accumulate_spatial_average, begin_spatial_collision_step,
 * deposit_spatial_collision_energy, accumulate_phase_eedf,
 * src/Simulation.cpp:1163-1370).  Before initialize()/resume(); sums start at
 * zero.  Sample steps cost one extra particle pass (the collision part of the
 * step is applied before the moments are taken). */
APIC_EXPORT int apic_sim1d_enable_spatial_average(apic_sim1d* sim, const apic_spatial_average1d* sa);
/* spatial_average_samples, spatial_collision_steps and, per phase bin (arrays
 * of phase_bins entries, may be NULL), the bin samples and collision steps
 * (include/pic/Simulation.hpp:31-41, :94-100) */
APIC_EXPORT int apic_sim1d_spatial_average_counts(apic_sim1d* sim, uint64_t* samples, uint64_t* collision_steps,
                                                  uint64_t* phase_samples, uint64_t* collision_phase_steps);
/* nx sums of one quantity; phase -1: the whole window, else that phase bin
 * (include/pic/Simulation.hpp:86-93, the spatial sums of src/Simulation.cpp:543-580) */
APIC_EXPORT int apic_sim1d_spatial_sums(apic_sim1d* sim, int quantity, int index, int phase, double* out);
/* phase_eedf_accumulators()[phase][region], include/pic/Simulation.hpp:101-104;
 * histogram: eedf_bins entries (may be NULL) */
APIC_EXPORT int apic_sim1d_phase_eedf(apic_sim1d* sim, int phase, int region, apic_phase_eedf1d* out,
                                      double* histogram);

/* ---- stateless kernels (host buffers in, host buffers out) --------------- */

/* Species::deposit_charge(Grid&) summed over species + FieldSolver::solve(Grid&,
 * phi_left, phi_right) + interpolate_electric(Grid&, x) at nq query points
 * (src/Species.cpp:161-185, src/FieldSolver.cpp:384-387, :407-440, :733-759,
 * :909-924).  xs[s] holds counts[s] positions of species s. */
APIC_EXPORT int apic_deposit_solve_gather_1d(int boundary, size_t nx, double length, double permittivity,
                                 double phi_left, double phi_right, int nspecies,
                                 const double* charge, const double* weight,
                                 const size_t* counts, const double* const* xs,
                                 double* rho, double* phi, double* electric,
                                 size_t nq, const double* xq, double* eq);

/* NullCollisionModel::collide(Vec3&, dt, rng), src/Collision.cpp:907-993, on n
 * particles in parallel.  Draw source: when draws != NULL, particle i consumes
 * the recorded raw 64-bit values draws[offsets[i] .. offsets[i+1]) (replay of
 * a std::mt19937_64 stream, including libstdc++'s distribution transforms);
 * otherwise a Philox4x32-10 stream keyed on (seed, i, step, stream).
 * v3 is updated in place (3 doubles per particle). */
APIC_EXPORT int apic_collide3(const apic_mcc_model* model, double particle_mass, size_t n, double* v3,
                  double dt, const uint64_t* draws, const uint64_t* offsets,
                  uint64_t seed, uint64_t step, uint32_t stream, apic_collide_stats* stats);

/* ---- structured 2D3V / 3D3V periodic simulation -------------------------- */

/* Simulation2DConfig / Simulation3DConfig subset of the periodic particle
 * step (include/pic/Simulation2D.hpp:118-165, include/pic/Simulation3D.hpp:30-66):
 * fully periodic fields and particle boundaries, uniform magnetic field.
 * Grid sizes must be powers of two (2..1024 per axis). */
typedef struct {
    int dims;                   /* 2 (2D3V) or 3 (3D3V) */
    size_t n[3];                /* cells (= nodes, periodic) per axis */
    double length[3];
    double dt;
    int units;                  /* apic_units */
    double relative_permittivity;
    double magnetic_field[3];   /* uniform B; all zero selects the leapfrog pusher */
    double out_of_plane_depth;  /* 2D only: weight / depth enters the deposit (0 = 1) */
    int precision;              /* apic_precision */
    size_t sort_interval;       /* steps between particle sorts by cell (0 = default 16) */
    int nspecies;
    apic_species species[APIC_MAX_SPECIES];
    int push_items;             /* FP32 form: particles per thread of the step push, 1, 2, 4 or 8
                                   (0 = default: 4 in 2D, 2 in 3D); a tuning knob, no effect on results */
    size_t species_sort_interval[APIC_MAX_SPECIES];  /* per species (0 = sort_interval): slow heavy
                                   species keep their cell order far longer; no effect on results */
    /* magnetic_field_profile (TabulatedVectorField1D, src/PrescribedField.cpp:89-113): B piecewise
       linear along one axis, evaluated at each particle's position in every Boris kick.
       profile_rows = 0 keeps the uniform magnetic_field; otherwise magnetic_field must be zero
       (mutually exclusive, as in the reference), the coordinates strictly increasing and covering
       [0, length] of that axis (a 2D run queries z = 0).  The arrays are copied at create. */
    int profile_axis;                   /* 0 = x, 1 = y, 2 = z */
    size_t profile_rows;
    const double* profile_coordinates;  /* profile_rows values */
    const double* profile_values;       /* profile_rows x (Bx, By, Bz) */
    /* 2D walls (Simulation2DConfig boundary_x / boundary_y, boundary_config, particle_boundary_config,
       include/pic/Simulation2D.hpp:118-135): wall_axis[a] = 1 makes axis a a Dirichlet axis whose n[a]
       counts nodes (spacing length / (n - 1)); one wall axis solves by FFT along the periodic axis and
       a tridiagonal sweep per mode, two by a direct sine-transform solve (extents 2^k + 1).  Sides are
       left, right, bottom, top.  particle_boundary: 0 auto (periodic on a periodic axis, absorbing on
       a wall axis), 1 absorbing, 2 reflecting, 3 periodic.  FP64 form; particles are not re-sorted;
       absorbed particles stay in place, flagged dead (apic_simnd_read_alive). */
    int wall_axis[2];
    double wall_potential[4];
    int particle_boundary[4];
    /* 3D walls (Simulation3DConfig boundary = Dirichlet, particle_boundary_config,
       include/pic/Simulation3D.hpp:30-66): the 3D mesh is periodic or Dirichlet on every axis, so
       wall_axis_z = 1 needs wall_axis[0] = wall_axis[1] = 1 and zero wall_potential (grounded walls);
       extents 2^k + 1 nodes up to 513, solved directly by sine transforms.  particle_boundary then
       holds left, right, bottom, top and particle_boundary_z back, front (same codes).  FP64 form. */
    int wall_axis_z;
    int particle_boundary_z[2];
} apic_config_nd;

/* DiagnosticSample2D / DiagnosticSample3D, src/Diagnostics.cpp:111-137, :205-232 */
typedef struct {
    uint64_t step;
    double time;
    double kinetic_energy;
    double field_energy;
    double total_energy;
    double charge_l1;
    uint64_t live_particles;
    double kinetic_by_species[APIC_MAX_SPECIES];
} apic_sample_nd;

typedef struct apic_sim_nd apic_sim_nd;

/* Simulation2D::Simulation2D / Simulation3D::Simulation3D (periodic). */
APIC_EXPORT int apic_simnd_create(const apic_config_nd* cfg, apic_sim_nd** out);
APIC_EXPORT void apic_simnd_destroy(apic_sim_nd* sim);
APIC_EXPORT const char* apic_simnd_last_error(const apic_sim_nd* sim);
/* Species2D/3D::particles() mutation.  pos is [dims][n] (component-major), v and
 * v_half are [3][n]; v_half may be NULL (then v_half = v). */
APIC_EXPORT int apic_simnd_load_particles(apic_sim_nd* sim, int species, size_t n, const double* pos,
                                          const double* v, const double* v_half);
/* Loads n particles generated on the device (for runs too large to stage on
 * the host): uniform positions displaced by amplitude/k sin(k x) along
 * perturb_axis, or along every axis of the mesh when perturb_axis < 0
 * (amplitude 0: none), Maxwellian velocities of the given thermal
 * speed plus an x drift, v_half = v.  Seeded Philox streams; no reference
 * counterpart (the reference's loaders, src/Species2D.cpp / Species3D.cpp, use
 * its shared engine). */
APIC_EXPORT int apic_simnd_load_maxwellian(apic_sim_nd* sim, int species, size_t n, uint64_t seed,
                                           double thermal_speed, double drift_x, int perturb_axis,
                                           double perturb_amplitude);
/* Simulation2D/3D::initialize after the particles are loaded
 * (src/Simulation2D.cpp:770-781): deposit_and_solve then the Boris or leapfrog
 * half-step initialisation. */
APIC_EXPORT int apic_simnd_initialize(apic_sim_nd* sim);
/* Restart from a state whose v_half is set: deposit_and_solve only. */
APIC_EXPORT int apic_simnd_resume(apic_sim_nd* sim, double time, uint64_t step);
/* Simulation2D::step / Simulation3D::step (src/Simulation2D.cpp:1337-1364,
 * src/Simulation3D.cpp:342-365) nsteps times; asynchronous. */
APIC_EXPORT int apic_simnd_step(apic_sim_nd* sim, size_t nsteps);
APIC_EXPORT int apic_simnd_synchronize(apic_sim_nd* sim);
APIC_EXPORT int apic_simnd_count(apic_sim_nd* sim, int species, size_t* n);
/* Particles in the order they were loaded, with the time-centred v of the
 * reference's synchronize step (src/Pusher.cpp:131-186). */
APIC_EXPORT int apic_simnd_read_particles(apic_sim_nd* sim, int species, size_t capacity, double* pos,
                                          double* v, double* v_half, size_t* n);
/* Mesh2D/Mesh3D rho(), phi(), electric_{x,y,z}() (E is [dims][N]). */
APIC_EXPORT int apic_simnd_read_fields(apic_sim_nd* sim, double* rho, double* phi, double* electric);
/* Particle::alive of a run with walls (1 for every particle without absorbing sides), in the
 * order of apic_simnd_read_particles. */
APIC_EXPORT int apic_simnd_read_alive(apic_sim_nd* sim, int species, size_t capacity, uint8_t* alive);
/* species_boundary_losses()[species] (BoundaryLoss2D, include/pic/Diagnostics.hpp:27-32):
 * absorbed left, right, bottom, top; 3D runs write six counts (BoundaryLoss3D,
 * include/pic/Diagnostics.hpp:34-41: ... back, front), per species here, their sum over the
 * species being the reference's boundary_losses() of the run. */
APIC_EXPORT int apic_simnd_boundary_losses(apic_sim_nd* sim, int species, uint64_t* absorbed);
APIC_EXPORT int apic_simnd_sample(apic_sim_nd* sim, apic_sample_nd* out);
APIC_EXPORT int apic_simnd_cuda_stream(apic_sim_nd* sim, void** stream);
APIC_EXPORT int apic_simnd_set_kernel_timing(apic_sim_nd* sim, int enable);
/* Summed milliseconds of the particle push, the field solve and the sorts,
 * and the number of steps timed. */
APIC_EXPORT int apic_simnd_kernel_times(apic_sim_nd* sim, double* push_ms, double* solve_ms, double* sort_ms,
                                        uint64_t* steps);
/* Number of kernels step() has launched on this handle (pushes, FFT passes,
 * sort passes); no reference counterpart. */
APIC_EXPORT int apic_simnd_launch_count(apic_sim_nd* sim, uint64_t* launches);

/* FieldSolver::solve(Mesh2D&/Mesh3D&) for a fully periodic mesh
 * (src/FieldSolver.cpp:442-499, :659-731): rho (N values) -> phi (N) and
 * E ([dims][N]). */
APIC_EXPORT int apic_field_solve_periodic_nd(int dims, const size_t* n, const double* length, double permittivity,
                                             const double* rho, double* phi, double* electric);

/* FieldSolver::solve(Mesh2D&/Mesh3D&) for a mesh with walls on every side
 * (solve_dirichlet_iterative, src/FieldSolver.cpp:761-907, with
 * apply_dirichlet_boundary_potentials, :267-296): 2D walls at
 * side_potentials = {left, right, bottom, top} (NULL: grounded; corner nodes the
 * mean of their two sides), 3D walls grounded (side_potentials NULL or zero).
 * The reference iterates SOR until the largest update is below 1e-11; this
 * solves the same discrete system directly (discrete sine transforms), so the
 * results agree to the reference's convergence.  Mesh spacing L / (n - 1); every
 * extent 2^k + 1 nodes from 3 to 513 (APIC_ERR_UNSUPPORTED otherwise).  rho,
 * phi: N = prod(n) values (index (k * ny + j) * nx + i); electric: [dims][N]. */
APIC_EXPORT int apic_field_solve_dirichlet_nd(int dims, const size_t* n, const double* length, double permittivity,
                                              const double* side_potentials, const double* rho, double* phi,
                                              double* electric);

/* FieldSolver::solve(Mesh2D&) for a mesh with exactly one periodic axis
 * (solve_mixed_spectral_tridiagonal, src/FieldSolver.cpp:501-657, and
 * compute_electric_field, :298-346): Fourier transform along the periodic axis,
 * one tridiagonal solve per mode across the wall axis, wall potentials on mode
 * 0.  periodic_axis 0: x periodic, walls at y = 0 (lower_potential, the
 * reference's bottom) and y = Ly (upper, top); 1: y periodic, walls at x = 0
 * (left) and x = Lx (right).  Mesh spacings follow Mesh2D (L / n along the
 * periodic axis, L / (n - 1) across the walls).  rho, phi: nx * ny values
 * (index j * nx + i); electric: [2][nx * ny].  The periodic extent must be a
 * power of two up to 1024 (APIC_ERR_UNSUPPORTED otherwise), the wall extent at
 * least 3.  Host arrays; the call returns when the results are copied back. */
APIC_EXPORT int apic_field_solve_mixed_2d(const size_t* n, const double* length, int periodic_axis,
                                          double permittivity, double lower_potential, double upper_potential,
                                          const double* rho, double* phi, double* electric);

/* Allocation-free variant of apic_field_solve_periodic_nd.  No counterpart in
 * the reference: it exists for callers that cannot call cudaMalloc - hosts that
 * manage all device memory through their own pool, and stepping loops that must
 * not trigger cudaMalloc's implicit synchronisation.  d_rho (N values), d_phi
 * (N) and d_electric ([dims][N]) are DEVICE pointers owned by the caller; the
 * FFT work arrays live in a static device array inside the library (about
 * 5.8 MB, kept by every GPU that loads the library until the process exits),
 * so N = nx*ny*nz may not exceed 65536 (APIC_ERR_CAPACITY beyond) and each
 * extent must be a power of two up to 1024.  Buffers that are not device (or
 * managed) memory of the current device are refused with APIC_ERR_INVALID.
 * Every call looks up that array's address in the current device's context;
 * the first call on a device also sets the FFT kernels' shared-memory limit
 * there, so make it before any stream capture.  Work is
 * enqueued on `stream` (a cudaStream_t, NULL for the default stream) and the
 * call returns without waiting.  Every call shares the one array, so calls
 * whose work overlaps on the GPU (different streams, or different host
 * threads on one device) race; serialise them on one stream. */
APIC_EXPORT int apic_field_solve_periodic_nd_noalloc(int dims, const size_t* n, const double* length,
                                                     double permittivity, const double* d_rho, double* d_phi,
                                                     double* d_electric, void* stream);

/* ======================================================================
 * Homogeneous electron swarms (src/Swarm.cpp)
 * ====================================================================== */

/* SwarmPopulationModel, include/pic/Swarm.hpp:14-17 */
typedef enum { APIC_SWARM_FIXED = 0, APIC_SWARM_BRANCHING = 1 } apic_swarm_population;

/* SwarmBenchmarkConfig, include/pic/Swarm.hpp:29-59, minus the file and
 * spatial-Townsend controls.  The gas dataset arrives as an apic_mcc_model
 * (channels with tables in joules / m^2, neutral_mass); its density,
 * temperature and max_frequency are taken from this struct. */
typedef struct {
    double neutral_density, neutral_temperature, max_frequency, timestep;
    size_t steps, burn_in_steps, particles;
    int population_model;          /* apic_swarm_population */
    size_t population_limit;       /* 0: the reference's default (src/Swarm.cpp:237-260) */
    size_t uncertainty_blocks;
    uint64_t work_item_limit;      /* 0: 100000000 */
    double initial_mean_energy_ev, max_energy_ev;
    uint64_t seed;
    int precision;                 /* electron storage: APIC_FP64 or APIC_FP32 */
} apic_swarm_config;

/* SwarmBenchmarkResult, include/pic/Swarm.hpp:73-115, minus the spatial
 * Townsend fields, plus the serving bookkeeping (id .. queue_s). */
typedef struct {
    uint64_t id;
    int status;                    /* APIC_OK or the run's error */
    char message[256];
    uint64_t steps_done;
    int converged;                 /* stopped by the tolerance test */
    double latency_s, queue_s;     /* submit -> result, submit -> admission */
    double reduced_field_td, electric_field_v_m;
    double mean_velocity_x, mean_velocity_x_se, drift_velocity, reduced_mobility;
    double mean_energy_ev, mean_energy_se_ev;
    int diffusion_available;
    double diffusion_longitudinal, diffusion_transverse;
    double max_observed_energy_ev;
    double initial_weight, final_weight;
    uint64_t final_particles;
    double growth_rate, growth_rate_se;
    double ionization_rate, ionization_rate_se, attachment_rate, attachment_rate_se;
    double net_rate, net_rate_se;
    int townsend_available;
    double townsend_growth, townsend_growth_se, townsend_rate, townsend_rate_se;
    uint64_t candidates, null_collisions;
    int nch;
    uint64_t channel_collisions[APIC_MAX_CHANNELS];
    double channel_rate[APIC_MAX_CHANNELS], channel_rate_se[APIC_MAX_CHANNELS];
} apic_swarm_result;

/* run_swarm_benchmark (src/Swarm.cpp:1503-1524) without the spatial Townsend
 * pass: every reduced field runs as one device run (seed cfg->seed + f), all of
 * them at once; results[f] receives field f.  Same validation and messages as
 * validate_config (src/Swarm.cpp:262-518). */
APIC_EXPORT int apic_swarm_run(const apic_swarm_config* cfg, const apic_mcc_model* gas, const double* fields_td,
                               size_t nfields, apic_swarm_result* results);

/* The spatial-Townsend controls of SwarmBenchmarkConfig, include/pic/Swarm.hpp:46-55
 * (work_item_limit 0: 100000000; fit_end_bin 0: bins). */
typedef struct {
    size_t histories;
    double length_m;
    size_t bins, fit_begin_bin, fit_end_bin;
    size_t max_steps;
    uint64_t work_item_limit;
    double min_r_squared;
} apic_spatial_townsend_config;

/* SwarmSpatialFluxPoint, include/pic/Swarm.hpp:66-70 */
typedef struct {
    double distance_m, net_crossings_per_injected_electron, standard_error;
} apic_spatial_flux_point;

/* The spatial-Townsend fields of SwarmBenchmarkResult, include/pic/Swarm.hpp:85-92 */
typedef struct {
    double townsend_1_m, townsend_standard_error_1_m, fit_r_squared;
    uint64_t histories_completed, maximum_active_particles, particle_updates;
} apic_spatial_townsend_result;

/* run_spatial_townsend (src/Swarm.cpp:645-938) for one reduced field: every
 * history's cascade on the device (one warp per history, histories balanced
 * through a global counter; Philox streams per history), the flux profile,
 * log-linear fit and block errors on the host.  FP64.  The reference runs it
 * after run_field with the same seed (cfg->seed + field index).
 * scan_particle_updates: in/out particle updates of the whole scan so far (may
 * be NULL); profile: sp->bins points; history_crossings (may be NULL):
 * histories x bins net crossings.  Same validation and messages as the
 * reference. */
APIC_EXPORT int apic_swarm_spatial_townsend(const apic_swarm_config* cfg, const apic_spatial_townsend_config* sp,
                                            const apic_mcc_model* gas, double reduced_field_td, uint64_t seed,
                                            uint64_t* scan_particle_updates, apic_spatial_townsend_result* out,
                                            apic_spatial_flux_point* profile, double* history_crossings);

/* Serving: a persistent batch of swarm runs on one GPU.  No reference
 * counterpart (the reference runs fields one after another): requests are
 * admitted while run slots and the device memory budget allow, every active
 * run advances steps_per_launch steps per apic_swarm_server_advance (one CUDA
 * graph launch for the whole batch), and runs retire when their steps are done
 * or their drift velocity and mean energy have converged. */
typedef struct apic_swarm_server apic_swarm_server;
/* Message of the last failed call on srv, or of the last failed call without
 * a server (srv NULL: apic_swarm_run, apic_swarm_server_create). */
APIC_EXPORT const char* apic_swarm_last_error(const apic_swarm_server* srv);
typedef struct {
    size_t memory_budget_bytes;    /* device pool for electron state and samples */
    int max_runs;                  /* concurrent run slots */
    int precision;                 /* APIC_FP64 or APIC_FP32 */
    size_t steps_per_launch;       /* steps per advance (graph length) */
} apic_swarm_server_config;

/* One run_field request on the server's gas. */
typedef struct {
    double reduced_field_td;
    size_t particles;
    uint64_t seed;
    size_t steps;                  /* at most this many steps */
    size_t burn_in_steps;
    size_t uncertainty_blocks;
    double tolerance;              /* > 0: stop once the relative block standard errors of drift
                                      velocity and mean energy are <= tolerance (checked after each
                                      advance, at least 4 samples per block) */
    int population_model;
    size_t population_limit;
    double initial_mean_energy_ev, max_energy_ev, timestep;
} apic_swarm_request;

/* gas: channels, neutral_density, neutral_temperature, max_frequency and
 * neutral_mass of every run on this server. */
APIC_EXPORT int apic_swarm_server_create(const apic_swarm_server_config* cfg, const apic_mcc_model* gas,
                                         apic_swarm_server** out);
APIC_EXPORT void apic_swarm_server_destroy(apic_swarm_server* srv);
APIC_EXPORT int apic_swarm_server_submit(apic_swarm_server* srv, const apic_swarm_request* req, uint64_t* id);
/* Admit, step every active run, retire finished runs; waits for the device. */
APIC_EXPORT int apic_swarm_server_advance(apic_swarm_server* srv, int* active, int* queued);
/* advance in two halves: launch admits and enqueues the batch's steps and
 * returns at once; complete waits for them and retires finished runs.  Work
 * the caller enqueues on other streams in between overlaps the batch. */
APIC_EXPORT int apic_swarm_server_launch(apic_swarm_server* srv);
APIC_EXPORT int apic_swarm_server_complete(apic_swarm_server* srv, int* active, int* queued);
/* done = 1 and *out filled (once) when request id has finished. */
APIC_EXPORT int apic_swarm_server_poll(apic_swarm_server* srv, uint64_t id, apic_swarm_result* out, int* done);
APIC_EXPORT int apic_swarm_server_stats(apic_swarm_server* srv, uint64_t* graph_launches, uint64_t* particle_steps,
                                        size_t* pool_bytes_free);
APIC_EXPORT int apic_swarm_server_cuda_stream(apic_swarm_server* srv, void** stream);
/* Bytes the server has copied host -> device (run set-up, chunk tables) and
 * device -> host (samples for the convergence test, finished runs' results)
 * since it was created.  No counterpart in the reference, which has no server. */
APIC_EXPORT int apic_swarm_server_copy_bytes(apic_swarm_server* srv, uint64_t* h2d, uint64_t* d2h);
/* Step kernels the server has launched (inside its graphs included). */
APIC_EXPORT int apic_swarm_server_kernel_launches(apic_swarm_server* srv, uint64_t* launches);
/* Diagnostics: with timing on, advance launches the step kernels one by one
 * (no graph) and times every streaming push and collision launch with CUDA
 * events; kernel_times reports the summed milliseconds of each, the number of
 * steps timed, and the push's algorithmic bytes (electron velocity read +
 * write, plus displacement read + write in sampling steps).  Enabling resets
 * the sums. */
APIC_EXPORT int apic_swarm_server_set_kernel_timing(apic_swarm_server* srv, int enable);
APIC_EXPORT int apic_swarm_server_kernel_times(apic_swarm_server* srv, double* push_ms, double* collide_ms,
                                               uint64_t* push_launches, double* push_bytes);

/* ---- particle-state interchange (.aps version 1) ------------------------------
 * The reference's external initial-state files (load_external_particle_state,
 * write_external_particle_state, external_particle_state_signature,
 * src/ParticleState.cpp:112-262, :541-624): parsed on the host into per-species
 * component arrays for apic_sim1d_load_particles / apic_simnd_load_particles.
 * Species are ordered by name; records of a species keep file order. */
typedef struct apic_aps apic_aps;
APIC_EXPORT const char* apic_aps_last_error(void);
/* Reads and validates a file (the reference's checks and messages); at most
 * max_particles records. */
APIC_EXPORT int apic_aps_read(const char* path, size_t max_particles, apic_aps** out);
APIC_EXPORT void apic_aps_free(apic_aps* state);
/* dimension 1-3, units apic_units, total records, species, and the canonical
 * 64-bit FNV-1a signature (the reference's initial_state_signature). */
APIC_EXPORT int apic_aps_info(const apic_aps* state, int* dimension, int* units, size_t* particle_count,
                              size_t* nspecies, uint64_t* signature);
/* Species k: its name (NUL-terminated, name_capacity bytes available) and
 * record count. */
APIC_EXPORT int apic_aps_species(const apic_aps* state, size_t k, char* name, size_t name_capacity, size_t* count);
/* Species k's records as component-major arrays: pos [3][count], vel [3][count]
 * (either may be NULL). */
APIC_EXPORT int apic_aps_records(const apic_aps* state, size_t k, double* pos, double* vel);
/* Writes species k's count records (pos[k], vel[k]: [3][counts[k]]) in the
 * reference's deterministic form (17 significant digits, species by name);
 * overwrite = 0 refuses an existing file.  *signature (if non-NULL) receives
 * the state's signature. */
APIC_EXPORT int apic_aps_write(const char* path, int dimension, int units, size_t nspecies,
                               const char* const* names, const size_t* counts, const double* const* pos,
                               const double* const* vel, int overwrite, uint64_t* signature);

/* ---- 1D3V checkpoints (.apc version 12) --------------------------------------
 * The restart files of Simulation::save_checkpoint / load_checkpoint
 * (src/Simulation.cpp:1812-2015, :2018-2899), the reference's route for 1D3V
 * state (its .aps files refuse 1D3V, src/Simulation.cpp:358-363).  Read on the
 * host into their parts; written back line for line in the reference's form
 * (numbers at 17 significant digits), so a file read and written again is
 * byte-identical.  Version 12 only (older files: APIC_ERR_UNSUPPORTED). */
typedef struct apic_apc apic_apc;
typedef struct {
    int units;                      /* apic_units */
    double relative_permittivity, permittivity;
    int velocity_dimensions;
    int collisions_enabled;
    uint64_t collision_signature;
    uint64_t candidates, null_collisions;
    size_t nchannels;               /* every model's channels, in model order */
    uint64_t boundary_loss_origin_step, power_transfer_origin_step;
    int spatial_average_enabled;
    uint64_t step;
    double time;
    size_t nspecies;
} apic_apc_info;
APIC_EXPORT const char* apic_apc_last_error(void);
/* load_checkpoint's structural checks and messages (the ones that need no configuration) */
APIC_EXPORT int apic_apc_read(const char* path, apic_apc** out);
APIC_EXPORT void apic_apc_free(apic_apc* checkpoint);
APIC_EXPORT int apic_apc_write(const apic_apc* checkpoint, const char* path);
APIC_EXPORT int apic_apc_get_info(const apic_apc* checkpoint, apic_apc_info* out);
/* collision_totals / collision_energy_totals entry k */
APIC_EXPORT int apic_apc_channel(const apic_apc* checkpoint, size_t k, uint64_t* count, double* energy);
/* species k: name, particle count (dead entries included), boundary losses, electric work */
APIC_EXPORT int apic_apc_species(const apic_apc* checkpoint, size_t k, char* name, size_t name_capacity,
                                 size_t* count, apic_boundary_loss* loss, double* electric_work);
/* species k's particles as arrays of its particle count */
APIC_EXPORT int apic_apc_particles(const apic_apc* checkpoint, size_t k, double* x, double* v, double* vy,
                                   double* vz, double* v_half, uint8_t* alive);
/* Simulation::load_checkpoint on the device: the configuration checks and
 * messages of the reference that apply (units, velocity dimensions, species
 * and channel counts, capacity, a spatial-average contract), then the
 * particles (dead entries dropped), collision totals, boundary losses,
 * electric work (when the ledger is enabled), step and time, and the field of
 * the restored state (deposit_and_solve).  The collision-model signature and
 * the engine state are not checked: the device draws from its own
 * counter-based streams. */
APIC_EXPORT int apic_sim1d_load_checkpoint(apic_sim1d* sim, const apic_apc* checkpoint);
/* Simulation::save_checkpoint of the device run: its particles (time-centred v,
 * as after step()), collision totals, boundary losses, electric work (without
 * the ledger: zero, counted from this step), step and time, with the
 * collision-model line, species names, engine state and disabled
 * campaign-diagnostics block taken from `meta` (a checkpoint of the same
 * configuration, e.g. the one the run was restarted from). */
APIC_EXPORT int apic_sim1d_save_checkpoint(apic_sim1d* sim, const apic_apc* meta, const char* path);

#ifdef __cplusplus
}
#endif
#endif /* AURORAPIC_B200_H */
