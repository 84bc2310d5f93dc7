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
enum { ORA_ISOTROPIC = 0, ORA_BACKWARD = 1 };
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
} ora_config1d;

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

#ifdef __cplusplus
}
#endif
#endif
