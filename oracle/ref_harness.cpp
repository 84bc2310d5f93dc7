// Test infrastructure only: a C-ABI shim that drives the reference's own
// classes (compiled from the reference sources by oracle/Makefile) so that the
// tests can generate golden vectors from the real reference and bench.py can
// time the reference's CPU step.  It restates no algorithm: every number it
// returns is computed by the reference library.
#include "oracle_types.h"

#include "pic/Collision.hpp"
#include "pic/Config.hpp"
#include "pic/FieldSolver.hpp"
#include "pic/Grid.hpp"
#include "pic/Mesh2D.hpp"
#include "pic/Mesh3D.hpp"
#include "pic/ParticleState.hpp"
#include "pic/Pusher.hpp"
#include "pic/Simulation.hpp"
#include "pic/Simulation2D.hpp"
#include "pic/Simulation3D.hpp"
#include "pic/Species.hpp"
#include "pic/Swarm.hpp"

#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <memory>
#include <random>
#include <sstream>
#include <string>
#include <vector>

namespace {
thread_local std::string g_error;

int fail(const std::exception& e) {
    g_error = e.what();
    return 1;
}

std::string write_table(const std::string& dir, const std::string& stem,
                        size_t rows, const double* e, const double* s) {
    std::filesystem::create_directories(dir);
    const std::string path = dir + "/" + stem + ".dat";
    std::ofstream out(path);
    out << std::setprecision(17);
    for (size_t i = 0; i < rows; ++i) out << e[i] << ' ' << s[i] << '\n';
    if (!out) throw std::runtime_error("cannot write table " + path);
    return path;
}

pic::CollisionProcessKind process_of(int p) {
    switch (p) {
        case ORA_ELASTIC: return pic::CollisionProcessKind::Elastic;
        case ORA_EXCITATION: return pic::CollisionProcessKind::Excitation;
        case ORA_IONIZATION: return pic::CollisionProcessKind::Ionization;
        case ORA_ATTACHMENT: return pic::CollisionProcessKind::Attachment;
        case ORA_CHARGE_EXCHANGE: return pic::CollisionProcessKind::ChargeExchange;
    }
    throw std::invalid_argument("unknown process");
}

std::string species_name(int index) { return "s" + std::to_string(index); }

pic::CollisionConfig collision_config(const ora_mcc_model& m, const std::string& dir,
                                      const std::string& tag) {
    pic::CollisionConfig c;
    c.enabled = true;
    c.model = pic::CollisionModelKind::NullCollision;
    c.neutral_density = m.neutral_density;
    c.max_frequency = m.max_frequency;
    c.neutral_mass = m.neutral_mass;
    c.neutral_temperature = m.neutral_temperature;
    c.species = species_name(m.species);
    c.max_candidates_per_particle = m.max_candidates;
    c.gas_data_units = m.si ? pic::UnitSystem::SI : pic::UnitSystem::Normalized;
    if (m.neutral_temperature > 0.0) c.gas_name = "synthetic";
    for (int i = 0; i < m.nch; ++i) {
        const ora_channel& ch = m.ch[i];
        pic::CollisionChannelConfig cc;
        cc.name = tag + "_ch" + std::to_string(i);
        cc.process = process_of(ch.process);
        cc.threshold_energy = ch.threshold_energy;
        cc.angular_scattering = ch.angular == ORA_BACKWARD
                                    ? pic::AngularScatteringKind::Backward
                                    : ch.angular == ORA_HENYEY_GREENSTEIN
                                    ? pic::AngularScatteringKind::HenyeyGreenstein
                                    : pic::AngularScatteringKind::Isotropic;
        if (ch.angular == ORA_HENYEY_GREENSTEIN)
            cc.mean_cosine_file = write_table(dir, cc.name + "_mu", ch.mu_rows, ch.mu_energy, ch.mu);
        cc.energy_frame = ch.energy_frame == ORA_FRAME_CENTER_OF_MASS
                              ? pic::CollisionEnergyFrame::CenterOfMass
                              : pic::CollisionEnergyFrame::Projectile;
        cc.cross_section_file = write_table(dir, cc.name, ch.rows, ch.energy, ch.sigma);
        if (ch.process == ORA_IONIZATION) {
            cc.secondary_species = species_name(ch.secondary_species);
            cc.ion_species = species_name(ch.ion_species);
        } else if (ch.process == ORA_ATTACHMENT) {
            cc.attachment_species = "attached";
        }
        c.channels.push_back(cc);
    }
    return c;
}

struct Ref1D {
    std::unique_ptr<pic::Simulation> sim;
};

pic::Config make_config_1d(const ora_config1d& in, const std::string& dir) {
    pic::Config c;
    c.units.system = in.si ? pic::UnitSystem::SI : pic::UnitSystem::Normalized;
    c.velocity_dimensions = static_cast<size_t>(in.vdim);
    c.nx = in.nx;
    c.length = in.length;
    c.dt = in.dt;
    c.boundary = in.dirichlet ? pic::Boundary::Dirichlet : pic::Boundary::Periodic;
    c.phi_left = in.phi_left;
    c.phi_right = in.phi_right;
    c.phi_left_drive = {in.drive_left[0], in.drive_left[1], in.drive_left[2]};
    c.phi_right_drive = {in.drive_right[0], in.drive_right[1], in.drive_right[2]};
    c.seed = in.seed;
    c.output_dir = dir + "/out";
    if (in.max_particles) c.max_particles_per_species = in.max_particles;
    if (in.threads > 0) {
        c.runtime.backend = pic::RuntimeBackend::OpenMP;
        c.runtime.threads = static_cast<size_t>(in.threads);
    }
    for (int s = 0; s < in.nspecies; ++s) {
        const ora_species& sp = in.species[s];
        pic::SpeciesConfig sc;
        sc.name = species_name(s);
        sc.charge = sp.charge;
        sc.mass = sp.mass;
        sc.weight = sp.weight;
        sc.particles = sp.particles;
        sc.drift_velocity = sp.drift;
        sc.thermal_velocity = sp.thermal;
        if (in.vdim == 3) {
            sc.initialization.thermal_velocity_y = sp.thermal_y;
            sc.initialization.thermal_velocity_z = sp.thermal_z;
        }
        c.species.push_back(sc);
    }
    if (in.bgk) {
        c.collisions.enabled = true;
        c.collisions.model = pic::CollisionModelKind::BGK;
        c.collisions.frequency = in.bgk_frequency;
        c.collisions.neutral_temperature_velocity = in.bgk_neutral_velocity;
    }
    for (int m = 0; m < in.nmodels; ++m) {
        pic::NamedCollisionConfig named;
        named.name = "model" + std::to_string(m);
        named.config = collision_config(in.models[m], dir, named.name);
        c.collision_models.push_back(named);
    }
    return c;
}
} // namespace

extern "C" {

const char* ref_last_error() { return g_error.c_str(); }

int ref1d_create(const ora_config1d* cfg, const char* workdir, void** out) {
    try {
        auto r = std::make_unique<Ref1D>();
        r->sim = std::make_unique<pic::Simulation>(make_config_1d(*cfg, workdir));
        *out = r.release();
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

void ref1d_destroy(void* h) { delete static_cast<Ref1D*>(h); }

int ref1d_initialize(void* h) {
    try { static_cast<Ref1D*>(h)->sim->initialize(); return 0; }
    catch (const std::exception& e) { return fail(e); }
}

int ref1d_step(void* h, size_t steps) {
    try {
        auto& sim = *static_cast<Ref1D*>(h)->sim;
        for (size_t i = 0; i < steps; ++i) sim.step();
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

size_t ref1d_count(void* h, int species) {
    return static_cast<Ref1D*>(h)->sim->species().at(species).particles().size();
}

double ref1d_time(void* h) { return static_cast<Ref1D*>(h)->sim->time(); }

int ref1d_get_particles(void* h, int species, double* x, double* v, double* vh,
                        double* vy, double* vz, uint8_t* alive) {
    try {
        const auto& ps = static_cast<Ref1D*>(h)->sim->species().at(species).particles();
        for (size_t i = 0; i < ps.size(); ++i) {
            x[i] = ps[i].x; v[i] = ps[i].v; vh[i] = ps[i].v_half;
            vy[i] = ps[i].velocity_y; vz[i] = ps[i].velocity_z;
            alive[i] = ps[i].alive ? 1 : 0;
        }
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

int ref1d_get_fields(void* h, double* rho, double* phi, double* e) {
    const auto& g = static_cast<Ref1D*>(h)->sim->grid();
    std::memcpy(rho, g.rho().data(), g.nx() * sizeof(double));
    std::memcpy(phi, g.phi().data(), g.nx() * sizeof(double));
    std::memcpy(e, g.electric().data(), g.nx() * sizeof(double));
    return 0;
}

// kinetic energy per species, field energy, live counts
int ref1d_sample(void* h, double* kinetic, double* field_energy, size_t* live) {
    try {
        auto& sim = *static_cast<Ref1D*>(h)->sim;
        const auto& sp = sim.species();
        for (size_t s = 0; s < sp.size(); ++s) {
            kinetic[s] = sp[s].kinetic_energy();
            live[s] = sp[s].live_count();
        }
        *field_energy = sim.sample().field_energy;
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

int ref1d_collisions(void* h, uint64_t* candidates, uint64_t* nulls, uint64_t* per_channel,
                     size_t cap) {
    const auto& d = static_cast<Ref1D*>(h)->sim->collision_diagnostics();
    *candidates = d.candidates;
    *nulls = d.null_collisions;
    for (size_t i = 0; i < d.channel_collisions.size() && i < cap; ++i)
        per_channel[i] = d.channel_collisions[i];
    return static_cast<int>(d.channel_collisions.size());
}

int ref1d_channel_energy(void* h, double* energy, size_t cap) {
    const auto& d = static_cast<Ref1D*>(h)->sim->collision_diagnostics();
    for (size_t i = 0; i < d.channel_energy_change.size() && i < cap; ++i)
        energy[i] = d.channel_energy_change[i];
    return static_cast<int>(d.channel_energy_change.size());
}

double ref1d_electric_work(void* h, int species) {
    return static_cast<Ref1D*>(h)->sim->species_power_transfer().at(species).electric_work;
}

int ref1d_losses(void* h, int species, size_t* left, size_t* right, double* eleft,
                 double* eright) {
    const auto& l = static_cast<Ref1D*>(h)->sim->species_boundary_losses().at(species);
    *left = l.absorbed_left; *right = l.absorbed_right;
    *eleft = l.kinetic_energy_left; *eright = l.kinetic_energy_right;
    return 0;
}

// Simulation::save_checkpoint / load_checkpoint of the reference itself.
int ref1d_save_checkpoint(void* h, const char* path) {
    try {
        static_cast<Ref1D*>(h)->sim->save_checkpoint(path);
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

int ref1d_load_checkpoint(void* h, const char* path) {
    try {
        static_cast<Ref1D*>(h)->sim->load_checkpoint(path);
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

// The engine state of Simulation's private rng_, read back through the
// reference's own checkpoint writer (the "rng" line, src/Simulation.cpp:2004).
int ref1d_rng_state(void* h, const char* path, uint64_t* out313) {
    try {
        static_cast<Ref1D*>(h)->sim->save_checkpoint(path);
        std::ifstream in(path);
        std::string line;
        while (std::getline(in, line)) {
            if (line.rfind("rng ", 0) == 0) {
                std::istringstream row(line.substr(4));
                for (int i = 0; i < 313; ++i) row >> out313[i];
                return row ? 0 : 2;
            }
        }
        return 3;
    } catch (const std::exception& e) { return fail(e); }
}

// --- CCP campaign diagnostics (src/Simulation.cpp:1163-1560) ---------------

namespace {
void apply_spatial_average(pic::Config& c, const ora_spatial_average1d& a) {
    c.spatial_average.enabled = true;
    c.spatial_average.interval = a.interval;
    c.spatial_average.start_step = a.start_step;
    c.spatial_average.end_step = a.end_step;
    c.spatial_average.rf_frequency = a.rf_frequency;
    c.spatial_average.rf_cycles = a.rf_cycles;
    c.spatial_average.phase_bins = a.phase_bins;
    c.phase_eedf.enabled = a.eedf_species >= 0;
    if (a.eedf_species >= 0) c.phase_eedf.species = species_name(a.eedf_species);
    c.phase_eedf.energy_bins = a.eedf_bins;
    c.phase_eedf.energy_max = a.eedf_energy_max;
    for (int r = 0; r < a.eedf_regions; ++r)
        c.phase_eedf.regions.push_back({"r" + std::to_string(r), a.eedf_x_min[r], a.eedf_x_max[r]});
}
}  // namespace

int ref1d_create_diag(const ora_config1d* cfg, const ora_spatial_average1d* sa, const char* workdir,
                      void** out) {
    try {
        auto r = std::make_unique<Ref1D>();
        pic::Config c = make_config_1d(*cfg, workdir);
        apply_spatial_average(c, *sa);
        r->sim = std::make_unique<pic::Simulation>(c);
        *out = r.release();
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

// Simulation::run over `steps` steps; the spatial-average CSV files land in workdir/out.
int ref1d_run_diag(const ora_config1d* cfg, const ora_spatial_average1d* sa, size_t steps,
                   const char* workdir) {
    try {
        pic::Config c = make_config_1d(*cfg, workdir);
        apply_spatial_average(c, *sa);
        c.steps = steps;
        c.output_interval = steps;
        pic::Simulation sim(c);
        sim.run();
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

// spatial_collision_energy_sums (phase -1) or the phase slice; returns the channel count
int ref1d_collision_energy(void* h, int channel, int phase, double* out) {
    const auto& sim = *static_cast<Ref1D*>(h)->sim;
    const auto& src = phase < 0 ? sim.spatial_collision_energy_sums()
                                : sim.spatial_collision_phase_energy_sums().at(phase);
    const auto& row = src.at(channel);
    std::memcpy(out, row.data(), row.size() * sizeof(double));
    return static_cast<int>(src.size());
}

void ref1d_collision_steps(void* h, uint64_t* steps, uint64_t* phase_steps) {
    const auto& sim = *static_cast<Ref1D*>(h)->sim;
    *steps = sim.spatial_collision_steps();
    const auto& ps = sim.spatial_collision_phase_steps();
    for (size_t i = 0; i < ps.size(); ++i) phase_steps[i] = ps[i];
}

int ref1d_phase_eedf(void* h, int phase, int region, uint64_t* counts, double* sums, double* hist) {
    try {
        const auto& a = static_cast<Ref1D*>(h)->sim->phase_eedf_accumulators().at(phase).at(region);
        counts[0] = a.macro_observations;
        counts[1] = a.overflow_macro_observations;
        const double v[7] = {a.represented_observations, a.overflow_represented_observations,
                             a.weighted_energy_sum, a.weighted_energy_squared_sum,
                             a.weighted_velocity_x_sum, a.weighted_velocity_y_sum, a.weighted_velocity_z_sum};
        std::memcpy(sums, v, sizeof v);
        std::memcpy(hist, a.histogram.data(), a.histogram.size() * sizeof(double));
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

// Config validation of the spatial average alone (validate_spatial_average_1d,
// src/Config.cpp:1377-1524), through the Simulation constructor.
int ref1d_validate_diag(const ora_config1d* cfg, const ora_spatial_average1d* sa, const char* workdir) {
    try {
        pic::Config c = make_config_1d(*cfg, workdir);
        apply_spatial_average(c, *sa);
        pic::Simulation sim(c);
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

// --- kernel-level entry points --------------------------------------------

// Species::deposit_charge + FieldSolver::solve + interpolate_electric on one grid.
int ref_deposit_solve_gather_1d(int dirichlet, size_t nx, double length, double eps,
                                double phi_left, double phi_right,
                                int nspecies, const double* charge, const double* weight,
                                const size_t* counts, const double* const* xs,
                                double* rho, double* phi, double* e,
                                size_t nq, const double* xq, double* eq) {
    try {
        pic::Grid grid(nx, length, dirichlet ? pic::Boundary::Dirichlet : pic::Boundary::Periodic);
        grid.clear_charge();
        for (int s = 0; s < nspecies; ++s) {
            pic::SpeciesConfig sc;
            sc.charge = charge[s];
            sc.weight = weight[s];
            sc.particles = counts[s];
            pic::Species sp(sc, 1);
            sp.particles().resize(counts[s]);
            for (size_t i = 0; i < counts[s]; ++i) {
                sp.particles()[i].x = xs[s][i];
                sp.particles()[i].alive = true;
            }
            sp.deposit_charge(grid);
        }
        std::memcpy(rho, grid.rho().data(), nx * sizeof(double));
        pic::FieldSolver solver(eps);
        solver.solve(grid, phi_left, phi_right);
        std::memcpy(phi, grid.phi().data(), nx * sizeof(double));
        std::memcpy(e, grid.electric().data(), nx * sizeof(double));
        for (size_t i = 0; i < nq; ++i) eq[i] = pic::interpolate_electric(grid, xq[i]);
        return 0;
    } catch (const std::exception& e2) { return fail(e2); }
}

// NullCollisionModel::collide(Vec3&) with one fresh std::mt19937_64(seed[i])
// per particle.  Records the raw 64-bit draws each call consumed.
int ref_collide3(const ora_mcc_model* model, double particle_mass, const char* workdir,
                 size_t n, double* v, const uint64_t* seeds, double dt,
                 ora_collide_stats* stats, uint64_t* draws, size_t draws_cap) {
    try {
        const pic::NullCollisionModel m(collision_config(*model, workdir, "collide"), particle_mass);
        for (size_t i = 0; i < n; ++i) {
            std::mt19937_64 rng(seeds[i]);
            std::mt19937_64 shadow(seeds[i]);
            pic::Vec3 vel{v[3 * i], v[3 * i + 1], v[3 * i + 2]};
            const auto st = m.collide(vel, dt, rng);
            v[3 * i] = vel.x; v[3 * i + 1] = vel.y; v[3 * i + 2] = vel.z;
            ora_collide_stats& o = stats[i];
            std::memset(&o, 0, sizeof(o));
            o.candidates = st.candidates;
            o.null_collisions = st.null_collisions;
            for (size_t c = 0; c < st.channel_collisions.size() && c < ORA_MAX_CHANNELS; ++c) {
                o.channel_collisions[c] = st.channel_collisions[c];
                o.energy_change[c] = st.channel_projectile_energy_change[c];
            }
            o.nsecondaries = static_cast<int>(st.secondaries.size());
            for (size_t k = 0; k < st.secondaries.size() && k < 16; ++k) {
                o.secondary_channel[k] = static_cast<int>(st.secondaries[k].channel);
                o.secondary_velocity[k][0] = st.secondaries[k].velocity.x;
                o.secondary_velocity[k][1] = st.secondaries[k].velocity.y;
                o.secondary_velocity[k][2] = st.secondaries[k].velocity.z;
                o.secondary_ion_velocity[k][0] = st.secondaries[k].ion_velocity.x;
                o.secondary_ion_velocity[k][1] = st.secondaries[k].ion_velocity.y;
                o.secondary_ion_velocity[k][2] = st.secondaries[k].ion_velocity.z;
            }
            o.removed = st.primary_removal_channel.has_value() ? 1 : 0;
            uint64_t used = 0;
            while (!(shadow == rng)) {
                const uint64_t d = shadow();
                if (draws && used < draws_cap) draws[i * draws_cap + used] = d;
                ++used;
                if (used > 1000000) throw std::runtime_error("draw count runaway");
            }
            o.draws = used;
        }
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

// Raw output of std::mt19937_64(seed): pins the oracle's engine.
void ref_mt64(uint64_t seed, size_t n, uint64_t* out) {
    std::mt19937_64 g(seed);
    for (size_t i = 0; i < n; ++i) out[i] = g();
}

// libstdc++ transforms on a std::mt19937_64(seed) stream, for pinning the
// oracle's restatement: kind 0 uniform_real(0,1), 1 normal(0,1) sequence on one
// object, 2 uniform_int<int>(0,1), 3 generate_canonical<double,64>.
void ref_dist(int kind, uint64_t seed, size_t n, double* out) {
    std::mt19937_64 g(seed);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    std::normal_distribution<double> nd(0.0, 1.0);
    std::uniform_int_distribution<int> b(0, 1);
    for (size_t i = 0; i < n; ++i) {
        switch (kind) {
            case 0: out[i] = u(g); break;
            case 1: out[i] = nd(g); break;
            case 2: out[i] = b(g); break;
            default: out[i] = std::generate_canonical<double, 64>(g); break;
        }
    }
}

} // extern "C"

// --- structured 2D3V / 3D3V periodic ------------------------------------------

namespace {
struct RefND {
    int dims = 2;
    std::unique_ptr<pic::Simulation2D> s2;
    std::unique_ptr<pic::Simulation3D> s3;
};
}  // namespace

extern "C" {

// species: q, m, w, count, drift_x, thermal (isotropic) per species
// 2D walls for the next refnd_create*: mesh boundary per axis (Dirichlet
// when set), side potentials (left, right, bottom, top) and particle
// boundaries per side (0 periodic, 1 absorbing, 2 reflecting).
static struct {
    bool set = false;
    int dirichlet[2];
    double pot[4];
    int pbc[4];
} g_walls;

void refnd_set_walls(const int* dirichlet, const double* pot, const int* pbc) {
    g_walls.set = true;
    for (int a = 0; a < 2; ++a) g_walls.dirichlet[a] = dirichlet[a];
    for (int k = 0; k < 4; ++k) { g_walls.pot[k] = pot[k]; g_walls.pbc[k] = pbc[k]; }
}

// 3D walls for the next refnd_create*: Boundary::Dirichlet (grounded) and the
// particle boundaries left, right, bottom, top, back, front.
static struct {
    bool set = false;
    int pbc[6];
} g_walls3;

void refnd_set_walls3d(const int* pbc) {
    g_walls3.set = true;
    for (int k = 0; k < 6; ++k) g_walls3.pbc[k] = pbc[k];
}

int refnd_create_profile(int dims, const size_t* n, const double* L, double dt, int si, const double* B,
                         int nspecies, const double* q, const double* m, const double* w, const size_t* count,
                         const double* drift, const double* thermal, unsigned seed, int threads, int prof_axis,
                         size_t prof_rows, const double* prof_c, const double* prof_v, void** out) {
    try {
        std::optional<pic::TabulatedVectorField1D> profile;
        if (prof_rows) {
            std::vector<double> cs(prof_c, prof_c + prof_rows);
            std::vector<pic::Vec3> vs(prof_rows);
            for (size_t k = 0; k < prof_rows; ++k) vs[k] = {prof_v[3 * k], prof_v[3 * k + 1], prof_v[3 * k + 2]};
            const pic::CoordinateAxis ax = prof_axis == 0 ? pic::CoordinateAxis::X
                                         : prof_axis == 1 ? pic::CoordinateAxis::Y : pic::CoordinateAxis::Z;
            profile.emplace(ax, std::move(cs), std::move(vs));
        }
        auto r = std::make_unique<RefND>();
        r->dims = dims;
        pic::RuntimePolicy rt;
        if (threads > 0) { rt.backend = pic::RuntimeBackend::OpenMP; rt.threads = (size_t)threads; }
        if (dims == 2) {
            pic::Simulation2DConfig c;
            c.units.system = si ? pic::UnitSystem::SI : pic::UnitSystem::Normalized;
            c.nx = n[0]; c.ny = n[1]; c.length_x = L[0]; c.length_y = L[1];
            c.dt = dt; c.boundary = pic::Boundary::Periodic;
            c.magnetic_field_x = B[0]; c.magnetic_field_y = B[1]; c.magnetic_field_z = B[2];
            c.magnetic_field_profile = profile;
            c.seed = seed; c.runtime = rt;
            c.output_dir = std::filesystem::temp_directory_path() / "apic_ref2d";
            if (g_walls.set) {
                auto bnd = [](int d) { return d ? pic::Boundary::Dirichlet : pic::Boundary::Periodic; };
                auto pb = [](int k) {
                    return k == 1 ? pic::ParticleBoundary::Absorbing
                           : k == 2 ? pic::ParticleBoundary::Reflecting : pic::ParticleBoundary::Periodic;
                };
                c.boundary_x = bnd(g_walls.dirichlet[0]);
                c.boundary_y = bnd(g_walls.dirichlet[1]);
                c.boundary_config.left.potential = g_walls.pot[0];
                c.boundary_config.right.potential = g_walls.pot[1];
                c.boundary_config.bottom.potential = g_walls.pot[2];
                c.boundary_config.top.potential = g_walls.pot[3];
                c.particle_boundary_config.left = pb(g_walls.pbc[0]);
                c.particle_boundary_config.right = pb(g_walls.pbc[1]);
                c.particle_boundary_config.bottom = pb(g_walls.pbc[2]);
                c.particle_boundary_config.top = pb(g_walls.pbc[3]);
                g_walls.set = false;
            }
            size_t mx = 0;
            for (int s = 0; s < nspecies; ++s) {
                pic::Species2DConfig sc;
                sc.name = "s" + std::to_string(s);
                sc.charge = q[s]; sc.mass = m[s]; sc.weight = w[s]; sc.particles = count[s];
                sc.drift_velocity_x = drift[s]; sc.thermal_velocity = thermal[s];
                c.species.push_back(sc);
                mx = std::max(mx, count[s]);
            }
            c.max_particles_per_species = std::max<size_t>(mx, 10);
            r->s2 = std::make_unique<pic::Simulation2D>(c);
        } else {
            pic::Simulation3DConfig c;
            c.units.system = si ? pic::UnitSystem::SI : pic::UnitSystem::Normalized;
            c.nx = n[0]; c.ny = n[1]; c.nz = n[2];
            c.length_x = L[0]; c.length_y = L[1]; c.length_z = L[2];
            c.dt = dt; c.boundary = pic::Boundary::Periodic;
            c.magnetic_field = {B[0], B[1], B[2]};
            c.magnetic_field_profile = profile;
            c.seed = seed; c.runtime = rt;
            c.output_dir = std::filesystem::temp_directory_path() / "apic_ref3d";
            if (g_walls3.set) {
                auto pb = [](int k) {
                    return k == 1 ? pic::ParticleBoundary::Absorbing
                           : k == 2 ? pic::ParticleBoundary::Reflecting : pic::ParticleBoundary::Periodic;
                };
                c.boundary = pic::Boundary::Dirichlet;
                c.particle_boundary_config.left = pb(g_walls3.pbc[0]);
                c.particle_boundary_config.right = pb(g_walls3.pbc[1]);
                c.particle_boundary_config.bottom = pb(g_walls3.pbc[2]);
                c.particle_boundary_config.top = pb(g_walls3.pbc[3]);
                c.particle_boundary_config.back = pb(g_walls3.pbc[4]);
                c.particle_boundary_config.front = pb(g_walls3.pbc[5]);
                g_walls3.set = false;
            }
            for (int s = 0; s < nspecies; ++s) {
                pic::Species3DConfig sc;
                sc.name = "s" + std::to_string(s);
                sc.charge = q[s]; sc.mass = m[s]; sc.weight = w[s]; sc.particles = count[s];
                sc.drift_velocity_x = drift[s]; sc.thermal_velocity = thermal[s];
                c.species.push_back(sc);
            }
            r->s3 = std::make_unique<pic::Simulation3D>(c);
        }
        *out = r.release();
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

int refnd_create(int dims, const size_t* n, const double* L, double dt, int si, const double* B, int nspecies,
                 const double* q, const double* m, const double* w, const size_t* count, const double* drift,
                 const double* thermal, unsigned seed, int threads, void** out) {
    return refnd_create_profile(dims, n, L, dt, si, B, nspecies, q, m, w, count, drift, thermal, seed, threads, 0, 0,
                                nullptr, nullptr, out);
}

void refnd_destroy(void* h) { delete static_cast<RefND*>(h); }

int refnd_initialize(void* h) {
    try {
        auto* r = static_cast<RefND*>(h);
        if (r->dims == 2) r->s2->initialize(); else r->s3->initialize();
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

int refnd_step(void* h, size_t steps) {
    try {
        auto* r = static_cast<RefND*>(h);
        for (size_t i = 0; i < steps; ++i) { if (r->dims == 2) r->s2->step(); else r->s3->step(); }
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

size_t refnd_count(void* h, int s) {
    auto* r = static_cast<RefND*>(h);
    return r->dims == 2 ? r->s2->species().at(s).particles().size() : r->s3->species().at(s).particles().size();
}

// pos, v, vh: [3][count] component-major
int refnd_get(void* h, int s, double* pos, double* v, double* vh) {
    auto* r = static_cast<RefND*>(h);
    const size_t n = refnd_count(h, s);
    if (r->dims == 2) {
        const auto& ps = r->s2->species().at(s).particles();
        for (size_t i = 0; i < n; ++i) {
            pos[i] = ps[i].position.x; pos[n + i] = ps[i].position.y; pos[2 * n + i] = 0.0;
            v[i] = ps[i].velocity.x; v[n + i] = ps[i].velocity.y; v[2 * n + i] = ps[i].velocity_z;
            vh[i] = ps[i].velocity_half.x; vh[n + i] = ps[i].velocity_half.y; vh[2 * n + i] = ps[i].velocity_half_z;
        }
    } else {
        const auto& ps = r->s3->species().at(s).particles();
        for (size_t i = 0; i < n; ++i) {
            pos[i] = ps[i].position.x; pos[n + i] = ps[i].position.y; pos[2 * n + i] = ps[i].position.z;
            v[i] = ps[i].velocity.x; v[n + i] = ps[i].velocity.y; v[2 * n + i] = ps[i].velocity.z;
            vh[i] = ps[i].velocity_half.x; vh[n + i] = ps[i].velocity_half.y; vh[2 * n + i] = ps[i].velocity_half.z;
        }
    }
    return 0;
}

// alive flags and the absorbed counts: 2D species_boundary_losses()[s] (left,
// right, bottom, top); 3D boundary_losses() of the whole run (left, right,
// bottom, top, back, front; the reference keeps no per-species ledger in 3D)
int refnd_alive_losses(void* h, int s, uint8_t* alive, uint64_t* losses) {
    auto* r = static_cast<RefND*>(h);
    if (r->dims == 3) {
        const auto& ps = r->s3->species().at(s).particles();
        for (size_t i = 0; i < ps.size(); ++i) alive[i] = ps[i].alive ? 1 : 0;
        const auto& l = r->s3->boundary_losses();
        losses[0] = l.absorbed_left; losses[1] = l.absorbed_right;
        losses[2] = l.absorbed_bottom; losses[3] = l.absorbed_top;
        losses[4] = l.absorbed_back; losses[5] = l.absorbed_front;
        return 0;
    }
    const auto& ps = r->s2->species().at(s).particles();
    for (size_t i = 0; i < ps.size(); ++i) alive[i] = ps[i].alive ? 1 : 0;
    const auto& l = r->s2->species_boundary_losses().at(s);
    losses[0] = l.absorbed_left; losses[1] = l.absorbed_right;
    losses[2] = l.absorbed_bottom; losses[3] = l.absorbed_top;
    return 0;
}

// rho, phi: N; E: [dims][N]
int refnd_fields(void* h, double* rho, double* phi, double* E) {
    auto* r = static_cast<RefND*>(h);
    if (r->dims == 2) {
        const auto& m = r->s2->mesh();
        const size_t N = m.rho().size();
        std::memcpy(rho, m.rho().data(), N * 8); std::memcpy(phi, m.phi().data(), N * 8);
        std::memcpy(E, m.electric_x().data(), N * 8); std::memcpy(E + N, m.electric_y().data(), N * 8);
    } else {
        const auto& m = r->s3->mesh();
        const size_t N = m.rho().size();
        std::memcpy(rho, m.rho().data(), N * 8); std::memcpy(phi, m.phi().data(), N * 8);
        std::memcpy(E, m.electric_x().data(), N * 8); std::memcpy(E + N, m.electric_y().data(), N * 8);
        std::memcpy(E + 2 * N, m.electric_z().data(), N * 8);
    }
    return 0;
}

double refnd_time(void* h) {
    auto* r = static_cast<RefND*>(h);
    return r->dims == 2 ? r->s2->time() : r->s3->time();
}

// FieldSolver::solve(Mesh2D&/Mesh3D&) on a given charge density (periodic).
/* FieldSolver::solve(Mesh2D&) on a mesh with one periodic axis: periodic_axis
 * 0 = x periodic with walls bottom (lower) / top (upper); 1 = y periodic with
 * walls left (lower) / right (upper). */
int ref_solve_mixed_2d(const size_t* n, const double* L, int periodic_axis, double eps, double lower, double upper,
                       const double* rho, double* phi, double* E) {
    try {
        pic::FieldSolver solver(eps);
        pic::BoundaryConfig2D bc;
        if (periodic_axis == 0) { bc.bottom.potential = lower; bc.top.potential = upper; }
        else { bc.left.potential = lower; bc.right.potential = upper; }
        const pic::Boundary px = periodic_axis == 0 ? pic::Boundary::Periodic : pic::Boundary::Dirichlet;
        const pic::Boundary py = periodic_axis == 0 ? pic::Boundary::Dirichlet : pic::Boundary::Periodic;
        pic::Mesh2D mesh(n[0], n[1], L[0], L[1], px, py, bc);
        const size_t N = n[0] * n[1];
        std::memcpy(mesh.rho().data(), rho, N * 8);
        solver.solve(mesh);
        std::memcpy(phi, mesh.phi().data(), N * 8);
        std::memcpy(E, mesh.electric_x().data(), N * 8);
        std::memcpy(E + N, mesh.electric_y().data(), N * 8);
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

/* write_external_particle_state with species k's records pos[k], vel[k]
 * ([3][counts[k]]); *signature = external_particle_state_signature. */
int ref_aps_write(const char* path, int dimension, int si, size_t nspecies, const char* const* names,
                  const size_t* counts, const double* const* pos, const double* const* vel, uint64_t* signature) {
    try {
        pic::ExternalParticleState st;
        st.spatial_dimension = (size_t)dimension;
        st.unit_system = si ? pic::UnitSystem::SI : pic::UnitSystem::Normalized;
        for (size_t k = 0; k < nspecies; ++k) {
            auto& recs = st.species[names[k]];
            const size_t n = counts[k];
            for (size_t i = 0; i < n; ++i) {
                pic::ExternalParticleRecord r;
                r.position = {pos[k][i], pos[k][n + i], pos[k][2 * n + i]};
                r.velocity = {vel[k][i], vel[k][n + i], vel[k][2 * n + i]};
                recs.push_back(r);
            }
            st.particle_count += n;
        }
        st.signature = pic::external_particle_state_signature(st);
        pic::write_external_particle_state(path, st, true);
        *signature = st.signature;
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

/* load_external_particle_state: signature and, per species in name order,
 * the record count (counts[k]) and records appended to pos/vel as
 * [species][3][count] blocks (capacity values each). */
int ref_aps_read(const char* path, size_t max_particles, uint64_t* signature, size_t* nspecies, size_t* counts,
                 double* pos, double* vel, size_t capacity) {
    try {
        const auto st = pic::load_external_particle_state(path, max_particles);
        *signature = st.signature;
        *nspecies = st.species.size();
        size_t k = 0, off = 0;
        for (const auto& [name, recs] : st.species) {
            (void)name;
            const size_t n = recs.size();
            counts[k++] = n;
            if (off + 3 * n > capacity) throw std::runtime_error("capacity");
            for (size_t i = 0; i < n; ++i) {
                pos[off + i] = recs[i].position.x; pos[off + n + i] = recs[i].position.y;
                pos[off + 2 * n + i] = recs[i].position.z;
                vel[off + i] = recs[i].velocity.x; vel[off + n + i] = recs[i].velocity.y;
                vel[off + 2 * n + i] = recs[i].velocity.z;
            }
            off += 3 * n;
        }
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

/* FieldSolver::solve on a fully Dirichlet Mesh2D (side potentials pot: left,
 * right, bottom, top) or Mesh3D (grounded). */
int ref_solve_dirichlet_nd(int dims, const size_t* n, const double* L, double eps, const double* pot,
                           const double* rho, double* phi, double* E) {
    try {
        pic::FieldSolver solver(eps);
        if (dims == 2) {
            pic::BoundaryConfig2D bc;
            bc.left.potential = pot[0]; bc.right.potential = pot[1];
            bc.bottom.potential = pot[2]; bc.top.potential = pot[3];
            pic::Mesh2D mesh(n[0], n[1], L[0], L[1], pic::Boundary::Dirichlet, pic::Boundary::Dirichlet, bc);
            const size_t N = n[0] * n[1];
            std::memcpy(mesh.rho().data(), rho, N * 8);
            solver.solve(mesh);
            std::memcpy(phi, mesh.phi().data(), N * 8);
            std::memcpy(E, mesh.electric_x().data(), N * 8);
            std::memcpy(E + N, mesh.electric_y().data(), N * 8);
        } else {
            pic::Mesh3D mesh(n[0], n[1], n[2], L[0], L[1], L[2], pic::Boundary::Dirichlet);
            const size_t N = n[0] * n[1] * n[2];
            std::memcpy(mesh.rho().data(), rho, N * 8);
            solver.solve(mesh);
            std::memcpy(phi, mesh.phi().data(), N * 8);
            std::memcpy(E, mesh.electric_x().data(), N * 8);
            std::memcpy(E + N, mesh.electric_y().data(), N * 8);
            std::memcpy(E + 2 * N, mesh.electric_z().data(), N * 8);
        }
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

int ref_solve_nd(int dims, const size_t* n, const double* L, double eps, const double* rho, double* phi, double* E) {
    try {
        pic::FieldSolver solver(eps);
        if (dims == 2) {
            pic::Mesh2D mesh(n[0], n[1], L[0], L[1], pic::Boundary::Periodic);
            std::memcpy(mesh.rho().data(), rho, n[0] * n[1] * 8);
            solver.solve(mesh);
            const size_t N = n[0] * n[1];
            std::memcpy(phi, mesh.phi().data(), N * 8);
            std::memcpy(E, mesh.electric_x().data(), N * 8); std::memcpy(E + N, mesh.electric_y().data(), N * 8);
        } else {
            pic::Mesh3D mesh(n[0], n[1], n[2], L[0], L[1], L[2], pic::Boundary::Periodic);
            const size_t N = n[0] * n[1] * n[2];
            std::memcpy(mesh.rho().data(), rho, N * 8);
            solver.solve(mesh);
            std::memcpy(phi, mesh.phi().data(), N * 8);
            std::memcpy(E, mesh.electric_x().data(), N * 8); std::memcpy(E + N, mesh.electric_y().data(), N * 8);
            std::memcpy(E + 2 * N, mesh.electric_z().data(), N * 8);
        }
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

}  // extern "C"

/* ---- pic::run_swarm_benchmark (src/Swarm.cpp:1503-1524) ------------------ */
namespace {
const char* process_name(int p) {
    switch (p) {
        case ORA_ELASTIC: return "elastic";
        case ORA_EXCITATION: return "excitation";
        case ORA_IONIZATION: return "ionization";
        case ORA_ATTACHMENT: return "attachment";
        default: return "charge_exchange";
    }
}

// A version-2 SI gas dataset (src/GasDataset.cpp:151-460) holding the
// channels of `gas`, with tables in joules and square metres.
std::string write_gas_dataset(const ora_mcc_model& gas, const std::string& dir) {
    std::filesystem::create_directories(dir);
    const std::string path = dir + "/gas.gas";
    std::ofstream out(path);
    out << std::setprecision(17);
    out << "gas_data_version = 2\nunits = si\ngas = synthetic\nneutral_mass = " << gas.neutral_mass
        << "\ndataset_id = oracle.synthetic\ndataset_version = 1\ndata_provenance = oracle harness\n"
        << "citation = none\nretrieved = 2026-01-01\nlicense = synthetic test data\n";
    for (int i = 0; i < gas.nch; ++i) {
        const ora_channel& ch = gas.ch[i];
        const std::string name = "ch" + std::to_string(i);
        out << "\n[collision." << name << "]\ntype = " << process_name(ch.process) << "\n";
        out << "cross_section_file = " << write_table(dir, name, ch.rows, ch.energy, ch.sigma) << "\n";
        if (ch.threshold_energy != 0.0) out << "threshold_energy = " << ch.threshold_energy << "\n";
        if (ch.energy_frame == ORA_FRAME_CENTER_OF_MASS) out << "energy_frame = center_of_mass\n";
        if (ch.angular == ORA_BACKWARD) out << "angular_model = backward\n";
        if (ch.angular == ORA_HENYEY_GREENSTEIN) {
            out << "angular_model = henyey_greenstein\n";
            out << "mean_cosine_file = " << write_table(dir, name + "_mu", ch.mu_rows, ch.mu_energy, ch.mu) << "\n";
        }
    }
    if (!out) throw std::runtime_error("cannot write gas dataset " + path);
    return path;
}
}  // namespace

extern "C" {

// run_swarm_benchmark; with sp, the spatial Townsend pass of every field too
// (sp_out[f], profiles: f x bins x (plane, mean, standard error)).
static int swarm_run_impl(const ora_swarm_config* cfg, const ora_spatial_config* sp, const ora_mcc_model* gas,
                          const double* fields, size_t nfields, const char* workdir, ora_swarm_result* out,
                          ora_spatial_result* sp_out, double* profiles) {
    try {
        pic::SwarmBenchmarkConfig c;
        c.gas_data_file = write_gas_dataset(*gas, workdir);
        c.neutral_density = cfg->neutral_density;
        c.neutral_temperature = cfg->neutral_temperature;
        c.reduced_fields_td.assign(fields, fields + nfields);
        c.max_frequency = cfg->max_frequency;
        c.timestep = cfg->timestep;
        c.steps = cfg->steps;
        c.burn_in_steps = cfg->burn_in_steps;
        c.particles = cfg->particles;
        c.population_model = cfg->branching ? pic::SwarmPopulationModel::BranchingResampled
                                            : pic::SwarmPopulationModel::FixedPopulationNoAvalanche;
        c.population_limit = cfg->population_limit;
        c.uncertainty_blocks = cfg->uncertainty_blocks;
        c.work_item_limit = 1000000000000000000ull;
        c.initial_mean_energy_ev = cfg->initial_mean_energy_ev;
        c.max_energy_ev = cfg->max_energy_ev;
        c.seed = cfg->seed;
        c.output_file = std::string(workdir) + "/swarm.csv";
        if (sp) {
            c.spatial_histories = sp->histories;
            c.spatial_length_m = sp->length_m;
            c.spatial_bins = sp->bins;
            c.spatial_fit_begin_bin = sp->fit_begin_bin;
            c.spatial_fit_end_bin = sp->fit_end_bin;
            c.spatial_max_steps = sp->max_steps;
            if (sp->work_item_limit) c.spatial_work_item_limit = sp->work_item_limit;
            c.spatial_min_r_squared = sp->min_r_squared;
        }
        const auto results = pic::run_swarm_benchmark(c);
        for (size_t f = 0; f < results.size(); ++f) {
            const auto& r = results[f];
            if (sp) {
                ora_spatial_result& q = sp_out[f];
                q.townsend_1_m = r.spatial_flux_townsend_1_m;
                q.townsend_se_1_m = r.spatial_flux_townsend_standard_error_1_m;
                q.fit_r_squared = r.spatial_flux_fit_r_squared;
                q.histories_completed = r.spatial_histories_completed;
                q.maximum_active_particles = r.spatial_maximum_active_particles;
                q.particle_updates = r.spatial_particle_updates;
                for (size_t b = 0; b < r.spatial_flux_profile.size(); ++b) {
                    double* row = profiles + (f * sp->bins + b) * 3;
                    row[0] = r.spatial_flux_profile[b].distance_m;
                    row[1] = r.spatial_flux_profile[b].net_crossings_per_injected_electron;
                    row[2] = r.spatial_flux_profile[b].standard_error;
                }
            }
            ora_swarm_result& o = out[f];
            std::memset(&o, 0, sizeof o);
            o.reduced_field_td = r.reduced_field_td;
            o.electric_field_v_m = r.electric_field_v_m;
            o.mean_velocity_x = r.mean_velocity_x_m_s;
            o.mean_velocity_x_se = r.mean_velocity_x_standard_error_m_s;
            o.drift_velocity = r.electron_drift_velocity_m_s;
            o.reduced_mobility = r.reduced_mobility_1_v_m_s;
            o.mean_energy_ev = r.mean_energy_ev;
            o.mean_energy_se_ev = r.mean_energy_standard_error_ev;
            o.diffusion_available = r.diffusion_available;
            o.diffusion_longitudinal = r.longitudinal_diffusion_m2_s;
            o.diffusion_transverse = r.transverse_diffusion_m2_s;
            o.max_observed_energy_ev = r.maximum_observed_energy_ev;
            o.initial_weight = r.initial_total_electron_weight;
            o.final_weight = r.final_total_electron_weight;
            o.final_particles = r.final_computational_particles;
            o.growth_rate = r.temporal_growth_rate_s;
            o.growth_rate_se = r.temporal_growth_rate_standard_error_s;
            o.ionization_rate = r.ionization_rate_s;
            o.ionization_rate_se = r.ionization_rate_standard_error_s;
            o.attachment_rate = r.attachment_rate_s;
            o.attachment_rate_se = r.attachment_rate_standard_error_s;
            o.net_rate = r.net_creation_rate_s;
            o.net_rate_se = r.net_creation_rate_standard_error_s;
            o.townsend_available = r.townsend_available;
            o.townsend_growth = r.growth_over_flux_drift_townsend_1_m;
            o.townsend_growth_se = r.growth_over_flux_drift_townsend_standard_error_1_m;
            o.townsend_rate = r.rate_balance_effective_townsend_1_m;
            o.townsend_rate_se = r.rate_balance_effective_townsend_standard_error_1_m;
            o.candidates = r.collision_candidates;
            o.null_collisions = r.null_collisions;
            o.nch = static_cast<int>(r.channels.size());
            for (size_t k = 0; k < r.channels.size() && k < ORA_MAX_CHANNELS; ++k) {
                o.channel_collisions[k] = r.channels[k].collisions;
                o.channel_rate[k] = r.channels[k].rate_per_electron_s;
                o.channel_rate_se[k] = r.channels[k].poisson_standard_error_s;
            }
        }
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int ref_swarm_run(const ora_swarm_config* cfg, const ora_mcc_model* gas, const double* fields, size_t nfields,
                  const char* workdir, ora_swarm_result* out) {
    return swarm_run_impl(cfg, nullptr, gas, fields, nfields, workdir, out, nullptr, nullptr);
}

int ref_swarm_run_spatial(const ora_swarm_config* cfg, const ora_spatial_config* sp, const ora_mcc_model* gas,
                          const double* fields, size_t nfields, const char* workdir, ora_swarm_result* out,
                          ora_spatial_result* sp_out, double* profiles) {
    return swarm_run_impl(cfg, sp, gas, fields, nfields, workdir, out, sp_out, profiles);
}

}  // extern "C"
