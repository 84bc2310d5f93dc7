/* C++20 facade over the C ABI of aurorapic_b200.h with the reference's class
 * names and signatures (include/pic/Simulation.hpp:56-64, Simulation2D.hpp,
 * Simulation3D.hpp, Collision.hpp:75-99, Swarm.hpp:120-121), so code written
 * against pic::Simulation / pic::NullCollisionModel / pic::run_swarm_benchmark
 * can switch to the device path by changing a namespace.  Status codes become
 * the reference's exception types: invalid_argument for configuration errors,
 * overflow_error for non-finite state, runtime_error for the rest (MCC
 * frequency and candidate limits, capacity, CUDA).
 *
 * Header only; link with -laurorapic_b200.  Needs C++20. */
#ifndef AURORAPIC_B200_HPP
#define AURORAPIC_B200_HPP

#include <cstddef>
#include <cstdint>
#include <random>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "aurorapic_b200.h"

namespace aurorapic_b200 {

/* ---- errors ---------------------------------------------------------------- */

[[noreturn]] inline void raise(int status, const char* message) {
    const std::string m = message ? message : "";
    switch (status) {
        case APIC_ERR_INVALID:
        case APIC_ERR_UNSUPPORTED:
            throw std::invalid_argument(m);
        case APIC_ERR_NONFINITE:
            throw std::overflow_error(m);
        default:
            throw std::runtime_error(m);
    }
}

/* ---- types of include/pic/Types.hpp ----------------------------------------- */

struct Vec3 {
    double x{0.0}, y{0.0}, z{0.0};
};

struct Particle {  // include/pic/Types.hpp:90-97
    double x{0.0};
    double v{0.0};
    bool alive{true};
    double v_half{0.0};
    double velocity_y{0.0};
    double velocity_z{0.0};
};

struct DiagnosticSample {  // include/pic/Diagnostics.hpp
    std::size_t step{0};
    double time{0.0};
    double kinetic_energy{0.0};
    double field_energy{0.0};
    double total_energy{0.0};
    double charge_l1{0.0};
    std::size_t live_particles{0};
    double phi_left{0.0};
    double phi_right{0.0};
};

/* ---- pic::Simulation (1D) ----------------------------------------------------- */

/* Config is the C struct itself: a reference-side adapter fills it from
 * pic::Config field by field. */
using Config = apic_config1d;

class Simulation {
public:
    explicit Simulation(const Config& cfg) {
        if (int rc = apic_sim1d_create(&cfg, &h_); rc != APIC_OK) raise(rc, apic_sim1d_last_error(nullptr));
        nspecies_ = cfg.nspecies;
        nx_ = cfg.nx;
    }
    Simulation(const Simulation&) = delete;
    Simulation& operator=(const Simulation&) = delete;
    Simulation(Simulation&& o) noexcept : h_(std::exchange(o.h_, nullptr)), nspecies_(o.nspecies_), nx_(o.nx_) {}
    ~Simulation() { apic_sim1d_destroy(h_); }

    /* Species::particles() as loaded before initialize(). */
    void load_particles(int species, const std::vector<Particle>& ps) {
        std::vector<double> x, v, vh, vy, vz;
        std::vector<std::uint8_t> alive;
        for (const auto& p : ps) {
            x.push_back(p.x); v.push_back(p.v); vh.push_back(p.v_half);
            vy.push_back(p.velocity_y); vz.push_back(p.velocity_z); alive.push_back(p.alive ? 1 : 0);
        }
        check(apic_sim1d_load_particles(h_, species, ps.size(), x.data(), v.data(), vh.data(), vy.data(), vz.data(),
                                        alive.data()));
    }
    void initialize() { check(apic_sim1d_initialize(h_)); }
    void step() { check(apic_sim1d_step(h_, 1)); }
    void run(std::size_t steps) { check(apic_sim1d_step(h_, steps)); }
    DiagnosticSample sample() const {
        apic_sample1d s{};
        check(apic_sim1d_sample(h_, &s));
        return {(std::size_t)s.step, s.time, s.kinetic_energy, s.field_energy, s.total_energy, s.charge_l1,
                (std::size_t)s.live_particles, s.phi_left, s.phi_right};
    }
    /* Species::particles() of the current state (read back from the device). */
    std::vector<Particle> particles(int species) const {
        std::size_t n = 0;
        check(apic_sim1d_count(h_, species, &n));
        std::vector<double> x(n), v(n), vh(n), vy(n), vz(n);
        std::size_t got = 0;
        check(apic_sim1d_read_particles(h_, species, n, x.data(), v.data(), vh.data(), vy.data(), vz.data(), &got));
        std::vector<Particle> out(got);
        for (std::size_t i = 0; i < got; ++i) out[i] = {x[i], v[i], true, vh[i], vy[i], vz[i]};
        return out;
    }
    double time() const { return apic_sim1d_time(h_); }
    std::size_t step_count() const { return (std::size_t)apic_sim1d_step_count(h_); }
    apic_sim1d* handle() const { return h_; }

    /* Config::spatial_average / phase_eedf, and the per-species electric-work
     * ledger: both before initialize(). */
    void enable_spatial_average(const apic_spatial_average1d& sa) {
        check(apic_sim1d_enable_spatial_average(h_, &sa));
    }
    void enable_power_transfer() { check(apic_sim1d_enable_power_transfer(h_)); }
    /* species_power_transfer()[s].electric_work, include/pic/Simulation.hpp:77-81 */
    double electric_work(int species) const {
        double w = 0.0;
        check(apic_sim1d_power_transfer(h_, species, &w));
        return w;
    }
    /* spatial_collision_energy_sums()[channel] (phase -1) or its phase slice,
     * include/pic/Simulation.hpp:86-93 */
    std::vector<double> spatial_collision_energy(int channel, int phase = -1) const {
        return spatial_sums(APIC_SA_COLLISION_ENERGY, channel, phase);
    }
    /* the per-node sums behind the spatial-average output (apic_sim1d_spatial_sums) */
    std::vector<double> spatial_sums(int quantity, int index, int phase = -1) const {
        std::vector<double> out(nx_hint());
        check(apic_sim1d_spatial_sums(h_, quantity, index, phase, out.data()));
        return out;
    }
    /* phase_eedf_accumulators()[phase][region] without its histogram */
    apic_phase_eedf1d phase_eedf(int phase, int region, std::vector<double>* histogram = nullptr) const {
        apic_phase_eedf1d e{};
        check(apic_sim1d_phase_eedf(h_, phase, region, &e, histogram ? histogram->data() : nullptr));
        return e;
    }

private:
    void check(int rc) const {
        if (rc != APIC_OK) raise(rc, apic_sim1d_last_error(h_));
    }
    std::size_t nx_hint() const { return nx_; }
    apic_sim1d* h_ = nullptr;
    int nspecies_ = 0;
    std::size_t nx_ = 0;
};

/* ---- pic::Simulation2D / Simulation3D (periodic) ------------------------------- */

class SimulationND {
public:
    explicit SimulationND(const apic_config_nd& cfg) : dims_(cfg.dims) {
        if (int rc = apic_simnd_create(&cfg, &h_); rc != APIC_OK) raise(rc, apic_simnd_last_error(nullptr));
    }
    SimulationND(const SimulationND&) = delete;
    SimulationND& operator=(const SimulationND&) = delete;
    ~SimulationND() { apic_simnd_destroy(h_); }
    /* positions [dims][n], velocities [3][n] (component-major) */
    void load_particles(int species, std::size_t n, const double* pos, const double* v, const double* v_half) {
        check(apic_simnd_load_particles(h_, species, n, pos, v, v_half));
    }
    void initialize() { check(apic_simnd_initialize(h_)); }
    void step() { check(apic_simnd_step(h_, 1)); }
    void run(std::size_t steps) { check(apic_simnd_step(h_, steps)); }
    apic_sample_nd sample() const {
        apic_sample_nd s{};
        check(apic_simnd_sample(h_, &s));
        return s;
    }
    int dims() const { return dims_; }
    apic_sim_nd* handle() const { return h_; }

private:
    void check(int rc) const {
        if (rc != APIC_OK) raise(rc, apic_simnd_last_error(h_));
    }
    apic_sim_nd* h_ = nullptr;
    int dims_ = 0;
};
using Simulation2D = SimulationND;
using Simulation3D = SimulationND;

/* ---- pic::NullCollisionModel ---------------------------------------------------- */

struct CollisionStepStatistics {  // include/pic/Collision.hpp:50-63
    std::uint64_t candidates{0};
    std::uint64_t null_collisions{0};
    std::vector<std::uint64_t> channel_collisions{};
    std::vector<double> channel_projectile_energy_change{};
    struct Secondary {
        std::size_t channel{0};
        Vec3 velocity{};
        Vec3 ion_velocity{};
    };
    std::vector<Secondary> secondaries{};
    bool primary_removed{false};
};

class NullCollisionModel {
public:
    /* model: channels with tables in joules / m^2 (kept by the caller while
     * this object lives), particle_mass in kg. */
    NullCollisionModel(const apic_mcc_model& model, double particle_mass) : m_(model), mass_(particle_mass) {}

    /* collide(Vec3&, dt, std::mt19937_64&), src/Collision.cpp:907-993, on the
     * device with the caller's engine: the draws the loop needs are taken from
     * `rng` and the engine ends exactly where the reference's would. */
    CollisionStepStatistics collide(Vec3& velocity, double timestep, std::mt19937_64& rng) const {
        std::vector<Vec3> v{velocity};
        auto stats = collide(v, timestep, rng);
        velocity = v[0];
        return std::move(stats[0]);
    }

    /* The same for many particles, one after another on one engine (the
     * reference's loop order): one device call per particle, since each
     * particle's draws start where the previous particle's ended.  Bulk work
     * belongs on apic_collide3 with Philox streams. */
    std::vector<CollisionStepStatistics> collide(std::vector<Vec3>& velocities, double timestep,
                                                 std::mt19937_64& rng) const {
        const std::size_t n = velocities.size();
        std::vector<CollisionStepStatistics> out(n);
        if (n == 0) return out;
        // the loop of particle i starts where particle i-1 stopped, so the
        // draws go out in growing windows until every particle is covered
        std::size_t window = 256;
        for (;;) {
            std::mt19937_64 probe = rng;
            std::vector<std::uint64_t> draws(window * n);
            for (auto& d : draws) d = probe();
            std::vector<double> v3(3 * n);
            std::vector<std::uint64_t> offsets(n + 1);
            std::vector<apic_collide_stats> st(n);
            bool fits = true;
            std::size_t used_total = 0;
            // sequential: the offset of particle i is the draws consumed by 0..i-1
            for (std::size_t i = 0; i < n && fits; ++i) {
                double one[3] = {velocities[i].x, velocities[i].y, velocities[i].z};
                std::uint64_t off[2] = {0, (std::uint64_t)(draws.size() - used_total)};
                apic_collide_stats s{};
                const int rc = apic_collide3(&m_, mass_, 1, one, timestep, draws.data() + used_total, off, 0, 0, 0, &s);
                if (rc != APIC_OK) raise(rc, apic_sim1d_last_error(nullptr));
                if (s.draws & 0x80000000u) { fits = false; break; }  // window exhausted: widen
                used_total += s.draws & 0x7FFFFFFFu;
                velocities[i] = {one[0], one[1], one[2]};
                st[i] = s;
            }
            if (!fits) {
                window *= 4;
                continue;
            }
            rng.discard(used_total);
            for (std::size_t i = 0; i < n; ++i) {
                auto& o = out[i];
                o.candidates = st[i].candidates;
                o.null_collisions = st[i].null_collisions;
                o.channel_collisions.assign(st[i].channel_collisions, st[i].channel_collisions + m_.nch);
                o.channel_projectile_energy_change.assign(st[i].energy_change, st[i].energy_change + m_.nch);
                for (int k = 0; k < st[i].nsecondaries && k < 4; ++k)
                    o.secondaries.push_back({(std::size_t)st[i].secondary_channel[k],
                                             {st[i].secondary_velocity[k][0], st[i].secondary_velocity[k][1],
                                              st[i].secondary_velocity[k][2]},
                                             {st[i].secondary_ion_velocity[k][0], st[i].secondary_ion_velocity[k][1],
                                              st[i].secondary_ion_velocity[k][2]}});
                o.primary_removed = st[i].removed != 0;
            }
            return out;
        }
    }

private:
    apic_mcc_model m_;
    double mass_;
};

/* ---- pic::run_swarm_benchmark ----------------------------------------------------- */

using SwarmBenchmarkConfig = apic_swarm_config;
using SwarmBenchmarkResult = apic_swarm_result;

inline std::vector<SwarmBenchmarkResult> run_swarm_benchmark(const SwarmBenchmarkConfig& config,
                                                             const apic_mcc_model& gas,
                                                             const std::vector<double>& reduced_fields_td) {
    std::vector<SwarmBenchmarkResult> out(reduced_fields_td.size());
    if (int rc = apic_swarm_run(&config, &gas, reduced_fields_td.data(), reduced_fields_td.size(), out.data());
        rc != APIC_OK)
        raise(rc, apic_swarm_last_error(nullptr));
    return out;
}

}  // namespace aurorapic_b200

#endif /* AURORAPIC_B200_HPP */
