/* Test infrastructure only: plain-C descriptions shared by the reference
 * harness (ref_harness.cpp, which drives the reference's own classes) and the
 * C restatement (apic_oracle.c).  Nothing in the product includes this file. */
#ifndef APIC_ORACLE_TYPES_H
#define APIC_ORACLE_TYPES_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORA_ELASTIC = 0, ORA_EXCITATION = 1, ORA_IONIZATION = 2, ORA_ATTACHMENT = 3, ORA_CHARGE_EXCHANGE = 4 };
enum { ORA_ISOTROPIC = 0, ORA_BACKWARD = 1, ORA_HENYEY_GREENSTEIN = 2 };
enum { ORA_FRAME_PROJECTILE = 0, ORA_FRAME_CENTER_OF_MASS = 1 };

#define ORA_MAX_CHANNELS 8
#define ORA_MAX_SPECIES 4
#define ORA_MAX_MODELS 4

typedef struct {
    int process;
    int angular;
    int energy_frame;
    double threshold_energy;
    int secondary_species; /* ionization only: species receiving the secondary */
    int ion_species;       /* ionization only: species receiving the ion */
    size_t rows;
    const double* energy;  /* strictly increasing */
    const double* sigma;
    size_t mu_rows;        /* Henyey-Greenstein only: MeanCosineTable rows */
    const double* mu_energy;
    const double* mu;
} ora_channel;

typedef struct {
    int species;                 /* projectile species index */
    double neutral_density;
    double max_frequency;
    double neutral_mass;
    double neutral_temperature;  /* thermal neutrals when > 0 and si != 0 */
    int si;
    size_t max_candidates;
    int nch;
    ora_channel ch[ORA_MAX_CHANNELS];
} ora_mcc_model;

typedef struct {
    double charge, mass, weight;
    size_t particles;
    double drift, thermal;       /* x-velocity Maxwellian */
    double thermal_y, thermal_z; /* 1D3V transverse components */
} ora_species;

typedef struct {
    int dirichlet;               /* 0 periodic, 1 Dirichlet */
    int vdim;                    /* 1 or 3 */
    int si;                      /* 0 normalized (eps=1), 1 SI */
    size_t nx;
    double length, dt;
    double phi_left, phi_right;
    double drive_left[3];        /* amplitude, frequency, phase */
    double drive_right[3];
    unsigned seed;
    int threads;                 /* 0: serial, N: OpenMP with N threads */
    size_t max_particles;        /* per species storage bound */
    int nspecies;
    ora_species species[ORA_MAX_SPECIES];
    int nmodels;
    ora_mcc_model models[ORA_MAX_MODELS];
    /* the legacy BGK model (CollisionConfig with model = bgk; one "bgk"
     * channel), src/Simulation.cpp:481-485, :771-834 */
    int bgk;
    double bgk_frequency;
    double bgk_neutral_velocity; /* neutral_temperature_velocity */
} ora_config1d;

/* SpatialAverage1DConfig + PhaseEedf1DConfig, include/pic/Config.hpp:145-168
 * (the EEDF species by index; regions by bounds) */
#define ORA_MAX_EEDF_REGIONS 8
typedef struct {
    size_t interval, start_step, end_step;
    double rf_frequency;
    size_t rf_cycles, phase_bins;
    int eedf_species;            /* -1: no phase EEDF */
    size_t eedf_bins;
    double eedf_energy_max;
    int eedf_regions;
    double eedf_x_min[ORA_MAX_EEDF_REGIONS], eedf_x_max[ORA_MAX_EEDF_REGIONS];
} ora_spatial_average1d;

/* Per-call collision statistics (one particle, one timestep). */
typedef struct {
    uint64_t candidates, null_collisions;
    uint64_t channel_collisions[ORA_MAX_CHANNELS];
    double energy_change[ORA_MAX_CHANNELS];
    int nsecondaries;
    int secondary_channel[16];
    double secondary_velocity[16][3];
    double secondary_ion_velocity[16][3];
    int removed;                 /* attachment removed the projectile */
    uint64_t draws;              /* raw 64-bit draws consumed */
} ora_collide_stats;

/* SwarmBenchmarkConfig subset of one run_field call, include/pic/Swarm.hpp:29-59 */
typedef struct {
    double neutral_density, neutral_temperature, max_frequency, timestep;
    size_t steps, burn_in_steps, particles;
    int branching;               /* 0 fixed_population_no_avalanche, 1 branching_resampled */
    size_t population_limit;     /* 0: the reference's default */
    size_t uncertainty_blocks;
    double initial_mean_energy_ev, max_energy_ev;
    uint64_t seed;
} ora_swarm_config;

/* Spatial-Townsend controls of SwarmBenchmarkConfig, include/pic/Swarm.hpp:46-55 */
typedef struct {
    size_t histories;
    double length_m;
    size_t bins, fit_begin_bin, fit_end_bin; /* fit_end_bin 0: bins */
    size_t max_steps;
    uint64_t work_item_limit;
    double min_r_squared;
} ora_spatial_config;

/* Spatial-Townsend fields of SwarmBenchmarkResult, include/pic/Swarm.hpp:85-92 */
typedef struct {
    double townsend_1_m, townsend_se_1_m, fit_r_squared;
    uint64_t histories_completed, maximum_active_particles, particle_updates;
} ora_spatial_result;

/* SwarmBenchmarkResult subset, include/pic/Swarm.hpp:73-115 */
typedef struct {
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
    uint64_t channel_collisions[ORA_MAX_CHANNELS];
    double channel_rate[ORA_MAX_CHANNELS], channel_rate_se[ORA_MAX_CHANNELS];
} ora_swarm_result;

#ifdef __cplusplus
}
#endif
#endif
