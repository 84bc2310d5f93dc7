/* Test infrastructure only: the CPU oracle for the electrostatic PIC particle
 * step.  A plain-C restatement of the reference's algorithm, used by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker.
 * The product never links or calls it.
 *
 * Parity pinning: every function below is checked against golden vectors that
 * the reference library itself produced (tests/golden/make_golden.py, which
 * drives oracle/_ref/libapic_ref.so built from the reference sources). */
#ifndef APIC_ORACLE_H
#define APIC_ORACLE_H
#include "oracle_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- random numbers ----------------------------------------------------- */
typedef struct { uint64_t mt[312]; int mti; } ora_mt64;
void ora_mt64_seed(ora_mt64* g, uint64_t seed);
uint64_t ora_mt64_next(ora_mt64* g);

/* A stream of raw 64-bit draws: an mt19937_64 engine (reference mode), a
 * Philox4x32-10 counter stream (device mode), or a recorded array (replay). */
enum { ORA_SRC_MT64 = 0, ORA_SRC_PHILOX = 1, ORA_SRC_ARRAY = 2 };
typedef struct {
    int kind;
    ora_mt64* mt;
    uint32_t key[2];
    uint32_t ctr[3];       /* particle slot, step, stream word */
    uint64_t index;        /* draws consumed so far */
    const uint64_t* array;
    uint64_t array_len;
    int overrun;
} ora_rng;
uint64_t ora_draw(ora_rng* r);
void ora_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

double ora_canonical(ora_rng* r);           /* generate_canonical<double, 53|64> */
double ora_uniform01(ora_rng* r);           /* uniform_real_distribution(0,1) */
int ora_bit(ora_rng* r);                    /* uniform_int_distribution<int>(0,1) */
typedef struct { int saved_available; double saved; } ora_normal;
double ora_normal_draw(ora_normal* st, ora_rng* r, double mean, double stddev);

/* ---- MCC (NullCollisionModel) ------------------------------------------- */
typedef struct {
    ora_mcc_model m;
    double particle_mass;
    double neutral_stddev;
} ora_collider;
/* returns 0, or an error code: 1 rate above max_frequency, 2 candidate cap,
 * 3 thermal bound above max_frequency, 4 invalid input, 5 draw array overrun */
int ora_collider_init(ora_collider* c, const ora_mcc_model* m, double particle_mass);
int ora_collide3(const ora_collider* c, double v[3], double dt, ora_rng* r, ora_collide_stats* st);
/* NullCollisionModel::collide(double&) (1V): elastic, excitation, charge
 * exchange and attachment with isotropic (random-sign) scattering */
int ora_collide1(const ora_collider* c, double* v, double dt, ora_rng* r, ora_collide_stats* st);

/* ---- 1D grid kernels ---------------------------------------------------- */
double ora_gather1d(const double* E, size_t nx, double length, double dx, int dirichlet, double x);
void ora_deposit1d(double* rho, size_t nx, double length, double dx, int dirichlet,
                   double charge, double weight, size_t n, const double* x, const uint8_t* alive);
void ora_solve1d(double* rho, double* phi, double* E, size_t nx, double length, double dx,
                 int dirichlet, double eps, double phi_left, double phi_right);

/* ---- 1D simulation ------------------------------------------------------ */
typedef struct ora_sim1d ora_sim1d;
/* mode 0: reference layout and one shared mt19937_64 stream (bit-exact with
 *         the reference's Simulation);
 * mode 1: device layout (survivors compacted in order, products appended in
 *         parent order) and per-(seed, species, slot, step) Philox streams;
 * mode 2: mode 1 with v_half, v_y, v_z stored as float (the device's FP32
 *         particle form), see ora_sim1d_round_fp32. */
ora_sim1d* ora_sim1d_create(const ora_config1d* cfg, int mode, uint64_t philox_seed);
void ora_sim1d_destroy(ora_sim1d* s);
int ora_sim1d_load(ora_sim1d* s, int species, size_t n, const double* x, const double* v,
                   const double* vh, const double* vy, const double* vz, const uint8_t* alive);
int ora_sim1d_initialize_fields(ora_sim1d* s, double time, uint64_t step);
int ora_sim1d_initialize(ora_sim1d* s);
int ora_sim1d_step(ora_sim1d* s, size_t steps);
/* mode 2 only: round the stored velocities as the device stores them when its
 * state is read back (a no-op on values already rounded) */
int ora_sim1d_round_fp32(ora_sim1d* s);
size_t ora_sim1d_count(const ora_sim1d* s, int species);
int ora_sim1d_get(const ora_sim1d* s, int species, double* x, double* v, double* vh,
                  double* vy, double* vz, uint8_t* alive);
void ora_sim1d_fields(const ora_sim1d* s, double* rho, double* phi, double* E);
double ora_sim1d_time(const ora_sim1d* s);
/* engine state in std::mersenne_twister_engine's text order: 312 words, index */
void ora_sim1d_set_mt(ora_sim1d* s, const uint64_t* state313);
/* channel_energy_change of the legacy BGK model's "bgk" channel */
double ora_sim1d_bgk_energy(const ora_sim1d* s);
void ora_sim1d_collisions(const ora_sim1d* s, uint64_t* candidates, uint64_t* nulls,
                          uint64_t* per_channel /* [nmodels][ORA_MAX_CHANNELS] */);
void ora_sim1d_losses(const ora_sim1d* s, int species, uint64_t* left, uint64_t* right,
                      double* eleft, double* eright);
double ora_sim1d_kinetic(const ora_sim1d* s, int species);
double ora_sim1d_field_energy(const ora_sim1d* s);
/* species_power_transfer()[species].electric_work since initialize,
 * src/Simulation.cpp:1094-1132 */
double ora_sim1d_electric_work(const ora_sim1d* s, int species);
/* CCP campaign diagnostics (src/Simulation.cpp:1163-1370): spatial averages,
 * phase bins, spatial collision energy and the phase EEDF.  Enable before
 * initialize; the configuration is assumed valid (the device validates it).
 * quantity: 0 density, 1-3 velocity x/y/z density, 4 kinetic-energy density
 * (index = species), 5 potential, 6 electric, 7 electric squared (index
 * ignored), 8 collision-energy density (index = global channel); phase -1 =
 * the whole window. */
int ora_sim1d_enable_spatial_average(ora_sim1d* s, const ora_spatial_average1d* cfg);
void ora_sim1d_spatial_counts(const ora_sim1d* s, uint64_t* samples, uint64_t* collision_steps,
                              uint64_t* phase_samples, uint64_t* collision_phase_steps);
int ora_sim1d_spatial_sums(const ora_sim1d* s, int quantity, int index, int phase, double* out);
/* counts: macro, overflow macro; sums: represented, overflow represented,
 * weighted energy, weighted energy^2, weighted v_x, v_y, v_z */
int ora_sim1d_phase_eedf(const ora_sim1d* s, int phase, int region, uint64_t* counts, double* sums,
                         double* histogram);
const char* ora_last_error(void);

/* ---- structured 2D3V / 3D3V periodic -------------------------------------- */
void ora_solve_nd(const double* rho, double* phi, double* E, int dims, const size_t* n, const double* L,
                  double eps);
/* FieldSolver::solve(Mesh2D&/Mesh3D&) on fully Dirichlet meshes (the reference's
 * SOR); pot: 2D left, right, bottom, top (NULL = grounded); 3D grounded. */
int ora_solve_dirichlet_nd(const double* rho, double* phi, double* E, int dims, const size_t* n, const double* L,
                           double eps, const double* pot);
int ora_solve_dirichlet_nd_warm(const double* rho, double* phi, double* E, int dims, const size_t* n, const double* L,
                                double eps, const double* pot);
/* FieldSolver::solve(Mesh2D&) with exactly one periodic axis (power of two). */
int ora_solve_mixed_2d(const double* rho, double* phi, double* E, const size_t* n, const double* L,
                       int periodic_axis, double eps, double lower, double upper);
void ora_gather_nd(const double* E, int dims, const size_t* n, const double* L, const double* pos, double* out);
void ora_deposit_nd(double* rho, int dims, const size_t* n, const double* L, double q, size_t np,
                    const double* pos);
void ora_boris(double v[3], const double E[3], const double B[3], double qm, double dt);
typedef struct ora_simnd ora_simnd;
/* w_eff: the weight that multiplies the charge in the deposit (2D: weight / depth) */
ora_simnd* ora_simnd_create(int dims, const size_t* n, const double* L, double dt, double eps, const double* B,
                            int nspecies, const double* q, const double* m, const double* w_eff);
void ora_simnd_destroy(ora_simnd* s);
/* 2D walls (before load): Dirichlet field axes [x, y], side potentials and
 * particle boundaries [left, right, bottom, top] (0 periodic, 1 absorbing,
 * 2 reflecting); absorbed particles stay in place with alive = 0 */
int ora_simnd_set_walls(ora_simnd* s, const int* dirichlet, const double* potentials, const int* particle);
/* 3D walls (before load): a Dirichlet mesh with grounded walls on every side
 * and particle boundaries [left, right, bottom, top, back, front] */
int ora_simnd_set_walls3d(ora_simnd* s, const int* particle);
void ora_simnd_alive_losses(const ora_simnd* s, int k, uint8_t* alive, uint64_t* losses);
void ora_simnd_load(ora_simnd* s, int k, size_t np, const double* pos, const double* v, const double* vh);
/* magnetic_field_profile: B piecewise linear along `axis` (values rows x 3) */
int ora_simnd_set_profile(ora_simnd* s, int axis, size_t rows, const double* coords, const double* values);
void ora_simnd_initialize_fields(ora_simnd* s);
void ora_simnd_initialize(ora_simnd* s);
void ora_simnd_step(ora_simnd* s, size_t steps);
void ora_simnd_get(const ora_simnd* s, int k, double* pos, double* v, double* vh);
void ora_simnd_fields(const ora_simnd* s, double* rho, double* phi, double* E);

/* ---- homogeneous electron swarm (src/Swarm.cpp) ---------------------------- */
/* block_mean_and_error, src/Swarm.cpp:103-134; returns 0 or 4 (invalid blocks) */
int ora_block_mean_and_error(const double* x, size_t n, size_t blocks, double* mean, double* se);
/* block_slope_and_error, src/Swarm.cpp:165-197 */
int ora_block_slope_and_error(const double* x, size_t n, double timestep, size_t blocks, double* slope,
                              double* se);
/* effective_population_limit, src/Swarm.cpp:237-260 */
size_t ora_swarm_population_limit(const ora_swarm_config* cfg);
/* run_field, src/Swarm.cpp:940-1250, for one reduced field (Td) on the gas
 * `gas` (channels and neutral_mass; density, temperature and max_frequency come
 * from cfg).
 * mode 0: the reference's particle layout and one shared mt19937_64 stream
 *         seeded with `seed` (bit-exact with run_swarm_benchmark);
 * mode 1: the device form in FP64: per-particle Philox streams keyed on
 *         (seed, slot, step), displacements accumulated from the sampling
 *         start, one weight per run, systematic resampling by index;
 * mode 2: mode 1 with velocities and displacements stored in FP32 between steps.
 * samples (optional): 3 x (steps - burn_in) doubles: velocity, energy, log weight. */
int ora_swarm_run_field(const ora_swarm_config* cfg, const ora_mcc_model* gas, double td, uint64_t seed, int mode,
                        ora_swarm_result* out, double* samples);
/* run_spatial_townsend, src/Swarm.cpp:645-938, for one reduced field.
 * mode 0: one mt19937_64 stream seeded with seed ^ 0x9e3779b97f4a7c15 shared by
 *         every history (bit-exact with run_swarm_benchmark);
 * mode 1: the device form: each history h draws from Philox streams keyed on
 *         seed with stream word 0x80000000 | h (slot 0xFFFFFFFE: injection;
 *         slot = electron index, counter step: collisions; slot 0xFFFFFFFF:
 *         resampling offset); plane crossings counted per step and added as
 *         weight x net count; one weight per history, resampling by index.
 * scan_updates: in/out particle updates of the scan so far (all fields).
 * profile: bins x (plane position, mean net crossings, standard error);
 * history_crossings (optional): histories x bins. */
int ora_swarm_spatial_townsend(const ora_swarm_config* cfg, const ora_spatial_config* sp, const ora_mcc_model* gas,
                               double td, uint64_t seed, int mode, uint64_t* scan_updates, ora_spatial_result* out,
                               double* profile, double* history_crossings);

#ifdef __cplusplus
}
#endif
#endif
