// Null-collision Monte Carlo collisions on the device.
//
// collide3() follows NullCollisionModel::collide(Vec3&) (src/Collision.cpp:907-993)
// decision for decision: exponential waiting times at the majorant, thermal
// neutral sampling, channel selection against cumulative rates, channel
// kinematics (src/Collision.cpp:762-829) and ionization secondaries.  The
// per-candidate full-table frequency-bound scan of the reference
// (validate_frequency_bound, src/Collision.cpp:627-685) becomes a precomputed
// safe speed: below it the bound provably holds, above it the exact check runs
// and a violation sets APIC_ERR_MAJORANT instead of throwing.
#pragma once
#include "apic_rng.cuh"

namespace apic {

constexpr int kMaxChannels = 8;
constexpr double kThermalSigma = 8.0;  // include/pic/Collision.hpp:139
constexpr double kDblEpsilon = 2.220446049250313080847e-16;

enum : int { kElastic = 0, kExcitation = 1, kIonization = 2, kAttachment = 3, kChargeExchange = 4 };

// Device errors (bit flags in the handle's error word).
enum : unsigned {
    kErrMajorant = 1u << 0,
    kErrCandidates = 1u << 1,
    kErrNonFinite = 1u << 2,
    kErrCapacity = 1u << 3,
    kErrTimeout = 1u << 4,
    kErrReplay = 1u << 5,
    kErrBirths = 1u << 6,
    kErrCandBuffer = 1u << 7,  // collision candidates of one pass beyond the candidate buffer
};

// Bracket index of a table: bin b of a uniform grid in log2(energy) stores the
// first row whose energy exceeds the bin's lower edge, so an upper_bound search
// only has to look between the entries of the neighbouring bins.
struct TableIndex {
    const unsigned* first_gt;  // nbins + 1 entries
    int nbins;
    double lmin, inv_width;    // bin = floor((log2(E) - lmin) * inv_width)
};

struct MccChannelDev {
    int process, angular, frame;
    double threshold;
    int secondary, ion;
    int rows;
    const double* energy;
    const double* sigma;
    TableIndex index;
    int mu_rows;              // Henyey-Greenstein mean-cosine table (0: none)
    const double* mu_energy;
    const double* mu;
};

struct MccModelDev {
    int nch;
    int species;
    double particle_mass, neutral_mass, neutral_density, max_frequency, neutral_stddev;
    double com_mass;      // particle_mass * neutral_mass / (particle_mass + neutral_mass)
    double v_safe;        // |v| <= v_safe passes the frequency-bound check without evaluation
    double v_safe2;       // |v|^2 <= v_safe2 implies |v| <= v_safe (negative: always evaluate)
    unsigned max_candidates;
    int shared_grid;      // every channel uses the same energy rows and the projectile frame
    // speed bins of width 1 / safe_inv_dv whose every speed provably passes the
    // frequency-bound check (1) or may not (0); speeds past the last bin take
    // the exact check
    const unsigned char* safe_bins;
    int nsafe;
    double safe_inv_dv;
    MccChannelDev ch[kMaxChannels];
};

// std::upper_bound(e, e + n, energy) for energy strictly inside the table.
__device__ inline int upper_bound_indexed(const MccChannelDev& c, double energy) {
    const TableIndex& ix = c.index;
    int lo = 0, hi = c.rows;
    if (ix.nbins > 0) {
        const double t = (log2(energy) - ix.lmin) * ix.inv_width;
        // (a NaN energy takes the whole table: the search stays inside it)
        const int b = !(t >= -1.0) ? -1 : (t > (double)ix.nbins ? ix.nbins : (int)floor(t));
        lo = b >= 1 ? (int)__ldg(ix.first_gt + (b - 1)) : 0;
        hi = b + 2 <= ix.nbins ? (int)__ldg(ix.first_gt + (b + 2)) : c.rows;
    }
    const double* e = c.energy;
    while (lo < hi) {
        const int mid = lo + ((hi - lo) >> 1);
        if (__ldg(e + mid) > energy) hi = mid; else lo = mid + 1;
    }
    return lo;
}

// Interpolation of table c at energy with a known bracket (high = upper_bound).
__device__ inline double table_at(const MccChannelDev& c, double energy, int high) {
    const int low = high - 1;
    const double el = __ldg(c.energy + low), eh = __ldg(c.energy + high);
    const double sl = __ldg(c.sigma + low), sh = __ldg(c.sigma + high);
    const double fraction = (energy - el) / (eh - el);
    return sl + fraction * (sh - sl);
}

// CrossSectionTable::evaluate, src/Collision.cpp:221-237
__device__ inline double table_eval(const MccChannelDev& c, double energy) {
    const double* e = c.energy;
    const int n = c.rows;
    if (energy <= __ldg(e)) return __ldg(c.sigma);
    if (energy >= __ldg(e + n - 1)) return __ldg(c.sigma + n - 1);
    return table_at(c, energy, upper_bound_indexed(c, energy));
}

// collision_energy, src/Collision.cpp:579-594
__device__ inline double collision_energy(const MccModelDev& m, const MccChannelDev& c, double rel) {
    const double mass = c.frame == 1 ? m.com_mass : m.particle_mass;
    return 0.5 * mass * rel * rel;
}

// rates_for_speed, src/Collision.cpp:596-625; returns false when the total
// exceeds max_frequency (+64 eps tolerance).
__device__ inline bool rates_for_speed(const MccModelDev& m, double speed, double* rates) {
    double total = 0.0;
    if (m.shared_grid) {
        // one bracket search serves every channel (same rows, same energy)
        const MccChannelDev& c0 = m.ch[0];
        const double energy = 0.5 * m.particle_mass * speed * speed;
        const int n = c0.rows;
        const bool below = energy <= __ldg(c0.energy), above = energy >= __ldg(c0.energy + n - 1);
        const int high = (below || above) ? 0 : upper_bound_indexed(c0, energy);
        for (int i = 0; i < m.nch; ++i) {
            const MccChannelDev& c = m.ch[i];
            double rate = 0.0;
            if (energy >= c.threshold) {
                const double sg = below ? __ldg(c.sigma) : above ? __ldg(c.sigma + n - 1) : table_at(c, energy, high);
                rate = m.neutral_density * sg * speed;
            }
            rates[i] = rate;
            total += rate;
        }
        const double mx = m.max_frequency > total ? m.max_frequency : total;
        return !(total > m.max_frequency + 64.0 * kDblEpsilon * mx);
    }
    for (int i = 0; i < m.nch; ++i) {
        const MccChannelDev& c = m.ch[i];
        const double energy = collision_energy(m, c, speed);
        double rate = 0.0;
        if (energy >= c.threshold) rate = m.neutral_density * table_eval(c, energy) * speed;
        rates[i] = rate;
        total += rate;
    }
    const double mx = m.max_frequency > total ? m.max_frequency : total;
    return !(total > m.max_frequency + 64.0 * kDblEpsilon * mx);
}

// validate_frequency_bound, src/Collision.cpp:627-685 (exact form, run only
// above the precomputed safe speed).
__device__ inline bool frequency_bound_exact(const MccModelDev& m, double speed);

__device__ __forceinline__ bool frequency_bound_binned(const MccModelDev& m, double speed) {
    if (speed <= m.v_safe) return true;
    if (m.safe_bins) {
        const double f = speed * m.safe_inv_dv;
        if (f < (double)m.nsafe && __ldg(m.safe_bins + (int)f)) return true;
    }
    return false;
}

__device__ __forceinline__ bool frequency_bound_ok(const MccModelDev& m, double speed) {
    return frequency_bound_binned(m, speed) || frequency_bound_exact(m, speed);
}

// The same check with the evaluated part out of line, for kernels whose model
// lives in global memory (an out-of-line call on a kernel-parameter model
// would copy it to local memory).
static __device__ __noinline__ bool frequency_bound_exact_far(const MccModelDev& m, double speed) {
    return frequency_bound_exact(m, speed);
}

__device__ __forceinline__ bool frequency_bound_ok_far(const MccModelDev& m, double speed) {
    return frequency_bound_binned(m, speed) || frequency_bound_exact_far(m, speed);
}

// validate_frequency_bound, src/Collision.cpp:627-685, evaluated
__device__ inline bool frequency_bound_exact(const MccModelDev& m, double speed) {
    double rates[kMaxChannels];
    if (m.neutral_stddev == 0.0) return rates_for_speed(m, speed, rates);
    const double limit = kThermalSigma * m.neutral_stddev;
    const double max_rel = speed + limit;
    double bound = 0.0;
    for (int i = 0; i < m.nch; ++i) {
        const MccChannelDev& c = m.ch[i];
        const double max_e = collision_energy(m, c, max_rel);
        if (max_e < c.threshold) continue;
        const double min_rel = speed - limit > 0.0 ? speed - limit : 0.0;
        double min_e = collision_energy(m, c, min_rel);
        if (c.threshold > min_e) min_e = c.threshold;
        double smax = table_eval(c, min_e);
        const double s2 = table_eval(c, max_e);
        if (s2 > smax) smax = s2;
        // rows with min_e <= energy <= max_e: [lower_bound(min_e), upper_bound(max_e))
        const int n = c.rows;
        int k0, k1;
        if (min_e <= __ldg(c.energy)) k0 = 0;
        else if (min_e > __ldg(c.energy + n - 1)) k0 = n;
        else {
            k0 = upper_bound_indexed(c, min_e);
            if (__ldg(c.energy + k0 - 1) == min_e) --k0;  // lower_bound
        }
        if (max_e >= __ldg(c.energy + n - 1)) k1 = n;
        else if (max_e < __ldg(c.energy)) k1 = 0;
        else k1 = upper_bound_indexed(c, max_e);
        for (int k = k0; k < k1; ++k) {
            const double s = __ldg(c.sigma + k);
            if (s > smax) smax = s;
        }
        bound += m.neutral_density * smax * max_rel;
    }
    const double mx = m.max_frequency > bound ? m.max_frequency : bound;
    return !(bound > m.max_frequency + 64.0 * kDblEpsilon * mx);
}

__device__ inline double norm3(double x, double y, double z) { return sqrt(x * x + y * y + z * z); }

// isotropic_velocity, src/Collision.cpp:53-64
template <class S>
__device__ inline void isotropic(double speed, S& s, double out[3]) {
    const double cosine = 2.0 * uniform01(s) - 1.0;
    const double t = 1.0 - cosine * cosine;
    const double sine = sqrt(0.0 > t ? 0.0 : t);
    const double azimuth = 2.0 * 3.141592653589793 * uniform01(s);
    double sn, cs;
    sincos(azimuth, &sn, &cs);
    out[0] = speed * sine * cs;
    out[1] = speed * sine * sn;
    out[2] = speed * cosine;
}

// MeanCosineTable::evaluate, src/Collision.cpp:296-313
__device__ inline double mean_cosine(const MccChannelDev& c, double energy) {
    const double* e = c.mu_energy;
    const int n = c.mu_rows;
    if (energy <= e[0]) return c.mu[0];
    if (energy >= e[n - 1]) return c.mu[n - 1];
    int lo = 0, hi = n;  // upper_bound
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (energy < e[mid]) hi = mid; else lo = mid + 1;
    }
    const int high = lo, low = high - 1;
    const double fraction = (energy - e[low]) / (e[high] - e[low]);
    return c.mu[low] + fraction * (c.mu[high] - c.mu[low]);
}

// angular_velocity: Henyey-Greenstein deflection about the incoming relative
// velocity, src/Collision.cpp:66-129
template <class S>
__device__ inline void angular_velocity(const double in[3], double speed, double g, S& s, double out[3]) {
    const double in_speed = norm3(in[0], in[1], in[2]);
    if (!(in_speed > 0.0)) { isotropic(speed, s, out); return; }
    const double sample = uniform01(s);
    double cosine = 2.0 * sample - 1.0;
    if (g != 0.0) {
        const double numerator = 1.0 - g * g;
        const double denominator = 1.0 - g + 2.0 * g * sample;
        const double ratio = numerator / denominator;
        cosine = (1.0 + g * g - ratio * ratio) / (2.0 * g);
        cosine = cosine < -1.0 ? -1.0 : (cosine > 1.0 ? 1.0 : cosine);
    }
    const double t = 1.0 - cosine * cosine;
    const double sine = sqrt(0.0 > t ? 0.0 : t);
    const double azimuth = 2.0 * 3.141592653589793 * uniform01(s);
    const double d[3] = {in[0] / in_speed, in[1] / in_speed, in[2] / in_speed};
    const bool low = fabs(d[2]) < 0.9;
    const double h[3] = {0.0, low ? 0.0 : 1.0, low ? 1.0 : 0.0};
    double tg[3] = {h[1] * d[2] - h[2] * d[1], h[2] * d[0] - h[0] * d[2], h[0] * d[1] - h[1] * d[0]};
    const double tn = norm3(tg[0], tg[1], tg[2]);
    tg[0] /= tn; tg[1] /= tn; tg[2] /= tn;
    const double bt[3] = {d[1] * tg[2] - d[2] * tg[1], d[2] * tg[0] - d[0] * tg[2], d[0] * tg[1] - d[1] * tg[0]};
    double sn, cs;
    sincos(azimuth, &sn, &cs);
    const double tf = sine * cs, bf = sine * sn;
    for (int k = 0; k < 3; ++k) out[k] = speed * (cosine * d[k] + tf * tg[k] + bf * bt[k]);
}

struct CollideResult {
    unsigned candidates = 0, nulls = 0;
    unsigned channel[kMaxChannels] = {0, 0, 0, 0, 0, 0, 0, 0};
    double energy_change[kMaxChannels] = {0, 0, 0, 0, 0, 0, 0, 0};
    bool removed = false;
    unsigned error = 0;
};

// NullCollisionModel::collide(Vec3&), src/Collision.cpp:907-993.  on_secondary
// receives (channel, secondary velocity[3], ion velocity[3]) per ionization.
// When have_first is set, the caller already ran the first loop iteration's
// bound check and waiting-time draw (the stream continues after them) and
// passes that waiting time.
template <class S, class OnSecondary>
__device__ inline void collide3(const MccModelDev& m, double v[3], double dt, S& s, CollideResult& r,
                                OnSecondary&& on_secondary, bool have_first = false, double first_wait = 0.0) {
    if (!isfinite(v[0]) || !isfinite(v[1]) || !isfinite(v[2])) { r.error |= kErrNonFinite; return; }
    double elapsed = 0.0;
    for (;;) {
        double waiting;
        if (have_first) {
            waiting = first_wait;
            have_first = false;
        } else {
            if (!frequency_bound_ok(m, norm3(v[0], v[1], v[2]))) { r.error |= kErrMajorant; return; }
            // open_unit_interval, src/Collision.cpp:46-51 (bounded for replay arrays)
            double u = uniform01(s);
            for (int guard = 0; !(u > 0.0) && guard < 64 && !s.overrun(); ++guard) u = uniform01(s);
            if (s.overrun()) { r.error |= kErrReplay; return; }
            waiting = -log(u) / m.max_frequency;
        }
        if (!isfinite(waiting) || waiting >= dt - elapsed) break;
        elapsed += waiting;
        ++r.candidates;
        if (r.candidates > m.max_candidates) { r.error |= kErrCandidates; return; }
        // sample_neutral_velocity_3v, src/Collision.cpp:702-715
        double vn[3] = {0.0, 0.0, 0.0};
        if (m.neutral_stddev != 0.0) {
            NormalState ns;
            const double limit = kThermalSigma * m.neutral_stddev;
            int attempt = 0;
            for (; attempt < 1024; ++attempt) {
                vn[0] = normal(ns, s, 0.0, m.neutral_stddev);
                vn[1] = normal(ns, s, 0.0, m.neutral_stddev);
                vn[2] = normal(ns, s, 0.0, m.neutral_stddev);
                if (norm3(vn[0], vn[1], vn[2]) <= limit) break;
            }
            if (attempt == 1024) { r.error |= kErrMajorant; return; }
        }
        double rates[kMaxChannels];
        if (!rates_for_speed(m, norm3(v[0] - vn[0], v[1] - vn[1], v[2] - vn[2]), rates)) {
            r.error |= kErrMajorant;
            return;
        }
        const double selection = canonical(s) * m.max_frequency;
        double cumulative = 0.0;
        bool accepted = false;
        for (int ci = 0; ci < m.nch; ++ci) {
            cumulative += rates[ci];
            if (selection < cumulative) {
                const MccChannelDev& c = m.ch[ci];
                const double before = 0.5 * m.particle_mass * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
                // apply_channel (3V), src/Collision.cpp:762-829
                if (c.process == kAttachment) {
                    v[0] = v[1] = v[2] = 0.0;
                } else if (c.process == kChargeExchange) {
                    v[0] = vn[0]; v[1] = vn[1]; v[2] = vn[2];
                } else {
                    const double rel[3] = {v[0] - vn[0], v[1] - vn[1], v[2] - vn[2]};
                    const double initial_speed = norm3(rel[0], rel[1], rel[2]);
                    double energy = 0.5 * m.particle_mass * initial_speed * initial_speed;
                    if (c.process == kExcitation || c.process == kIonization) {
                        const double e2 = energy - c.threshold;
                        energy = 0.0 > e2 ? 0.0 : e2;
                    }
                    if (c.process == kIonization) energy *= 0.5;
                    const double speed = sqrt(2.0 * energy / m.particle_mass);
                    double sc[3];
                    if (c.angular == 1) { sc[0] = -rel[0]; sc[1] = -rel[1]; sc[2] = -rel[2]; }
                    else if (c.angular == 2 && c.mu_rows)
                        angular_velocity(rel, speed, mean_cosine(c, collision_energy(m, c, initial_speed)), s, sc);
                    else isotropic(speed, s, sc);
                    if (c.process == kElastic && m.neutral_mass > 0.0) {
                        const double total = m.particle_mass + m.neutral_mass;
                        const double rf = m.neutral_mass / total;
                        for (int d = 0; d < 3; ++d)
                            v[d] = (m.particle_mass * v[d] + m.neutral_mass * vn[d]) / total + rf * sc[d];
                    } else {
                        for (int d = 0; d < 3; ++d) v[d] = vn[d] + sc[d];
                    }
                }
                r.energy_change[ci] +=
                    0.5 * m.particle_mass * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) - before;
                if (c.process == kIonization) {
                    const double sspeed = norm3(v[0] - vn[0], v[1] - vn[1], v[2] - vn[2]);
                    double iso[3];
                    isotropic(sspeed, s, iso);
                    const double vs[3] = {vn[0] + iso[0], vn[1] + iso[1], vn[2] + iso[2]};
                    on_secondary(ci, vs, vn);
                }
                ++r.channel[ci];
                if (c.process == kAttachment) r.removed = true;
                accepted = true;
                break;
            }
        }
        if (!accepted) ++r.nulls;
        if (r.removed) break;
    }
    if (s.overrun()) r.error |= kErrReplay;
}

// NullCollisionModel::collide(double&) (1V), src/Collision.cpp:831-905, with
// the scalar sample_neutral_velocity (:687-700) and the 1V apply_channel
// (:717-760): the scattered speed takes a random sign, the top bit of one
// draw (uniform_int_distribution<int>(0, 1) on a 64-bit engine).  The model
// has no ionization and only isotropic channels (checked at create).  Same
// first-iteration convention as collide3.
template <class S>
__device__ inline void collide1(const MccModelDev& m, double& v, double dt, S& s, CollideResult& r,
                                bool have_first = false, double first_wait = 0.0) {
    if (!isfinite(v)) { r.error |= kErrNonFinite; return; }
    double elapsed = 0.0;
    for (;;) {
        double waiting;
        if (have_first) {
            waiting = first_wait;
            have_first = false;
        } else {
            if (!frequency_bound_ok(m, fabs(v))) { r.error |= kErrMajorant; return; }
            double u = uniform01(s);
            for (int guard = 0; !(u > 0.0) && guard < 64 && !s.overrun(); ++guard) u = uniform01(s);
            if (s.overrun()) { r.error |= kErrReplay; return; }
            waiting = -log(u) / m.max_frequency;
        }
        if (!isfinite(waiting) || waiting >= dt - elapsed) break;
        elapsed += waiting;
        ++r.candidates;
        if (r.candidates > m.max_candidates) { r.error |= kErrCandidates; return; }
        double vn = 0.0;
        if (m.neutral_stddev != 0.0) {
            NormalState ns;
            const double limit = kThermalSigma * m.neutral_stddev;
            int attempt = 0;
            for (; attempt < 1024; ++attempt) {
                vn = normal(ns, s, 0.0, m.neutral_stddev);
                if (fabs(vn) <= limit) break;
            }
            if (attempt == 1024) { r.error |= kErrMajorant; return; }
        }
        double rates[kMaxChannels];
        if (!rates_for_speed(m, fabs(v - vn), rates)) {
            r.error |= kErrMajorant;
            return;
        }
        const double selection = canonical(s) * m.max_frequency;
        double cumulative = 0.0;
        bool accepted = false;
        for (int ci = 0; ci < m.nch; ++ci) {
            cumulative += rates[ci];
            if (selection < cumulative) {
                const MccChannelDev& c = m.ch[ci];
                const double before = 0.5 * m.particle_mass * v * v;
                if (c.process == kAttachment) {
                    v = 0.0;
                } else if (c.process == kChargeExchange) {
                    v = vn;
                } else {
                    const double rel = v - vn;
                    double energy = 0.5 * m.particle_mass * rel * rel;
                    if (c.process == kExcitation) {
                        const double e2 = energy - c.threshold;
                        energy = 0.0 < e2 ? e2 : 0.0;  // std::max(0.0, e2)
                    }
                    const double speed = sqrt(2.0 * energy / m.particle_mass);
                    const double scattered = (s.next() >> 63) == 0ull ? -speed : speed;
                    if (c.process == kElastic && m.neutral_mass > 0.0) {
                        const double total = m.particle_mass + m.neutral_mass;
                        v = (m.particle_mass * v + m.neutral_mass * vn) / total + (m.neutral_mass / total) * scattered;
                    } else {
                        v = vn + scattered;
                    }
                }
                r.energy_change[ci] += 0.5 * m.particle_mass * v * v - before;
                ++r.channel[ci];
                if (c.process == kAttachment) r.removed = true;
                accepted = true;
                break;
            }
        }
        if (!accepted) ++r.nulls;
        if (r.removed) break;
    }
    if (s.overrun()) r.error |= kErrReplay;
}

}  // namespace apic
