/* Test infrastructure only: the CPU oracle (a plain-C restatement of the
 * reference's electrostatic PIC particle step).  Each function cites the
 * reference file:line it restates.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load this library, as the checker.
 *
 * Pinned against golden vectors produced by the reference library itself
 * (tests/golden/make_golden.py drives oracle/_ref/libapic_ref.so). */
#include "apic_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static char g_err[256];
const char* ora_last_error(void) { return g_err; }
static int seterr(int code, const char* msg) {
    snprintf(g_err, sizeof g_err, "%s", msg);
    return code;
}

/* ======================================================================= */
/* mt19937_64: Matsumoto & Nishimura's 64-bit Mersenne Twister as specified
 * by ISO C++ [rand.predef] (the reference's engine, include/pic/Simulation.hpp:177). */
void ora_mt64_seed(ora_mt64* g, uint64_t seed) {
    g->mt[0] = seed;
    for (int i = 1; i < 312; ++i)
        g->mt[i] = 6364136223846793005ULL * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + (uint64_t)i;
    g->mti = 312;
}

uint64_t ora_mt64_next(ora_mt64* g) {
    static const uint64_t mag[2] = {0ULL, 0xB5026F5AA96619E9ULL};
    const uint64_t upper = 0xFFFFFFFF80000000ULL, lower = 0x7FFFFFFFULL;
    if (g->mti >= 312) {
        int i;
        for (i = 0; i < 312 - 156; ++i) {
            uint64_t x = (g->mt[i] & upper) | (g->mt[i + 1] & lower);
            g->mt[i] = g->mt[i + 156] ^ (x >> 1) ^ mag[x & 1ULL];
        }
        for (; i < 311; ++i) {
            uint64_t x = (g->mt[i] & upper) | (g->mt[i + 1] & lower);
            g->mt[i] = g->mt[i + (156 - 312)] ^ (x >> 1) ^ mag[x & 1ULL];
        }
        uint64_t x = (g->mt[311] & upper) | (g->mt[0] & lower);
        g->mt[311] = g->mt[155] ^ (x >> 1) ^ mag[x & 1ULL];
        g->mti = 0;
    }
    uint64_t y = g->mt[g->mti++];
    y ^= (y >> 29) & 0x5555555555555555ULL;
    y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
    y ^= (y << 37) & 0xFFF7EEE000000000ULL;
    y ^= y >> 43;
    return y;
}

/* Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11): the device's
 * counter-based stream.  The same function runs in the CUDA kernels. */
void ora_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int round = 0; round < 10; ++round) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

uint64_t ora_draw(ora_rng* r) {
    const uint64_t k = r->index++;
    switch (r->kind) {
        case ORA_SRC_MT64: return ora_mt64_next(r->mt);
        case ORA_SRC_PHILOX: {
            const uint32_t ctr[4] = {(uint32_t)(k >> 1), r->ctr[0], r->ctr[1], r->ctr[2]};
            uint32_t out[4];
            ora_philox4x32_10(ctr, r->key, out);
            return (k & 1) ? ((uint64_t)out[3] << 32 | out[2]) : ((uint64_t)out[1] << 32 | out[0]);
        }
        default:
            if (k >= r->array_len) { r->overrun = 1; return 0; }
            return r->array[k];
    }
}

/* libstdc++ generate_canonical<double, b> on a 64-bit engine (<bits/random.tcc>):
 * one draw, sum / 2^64, values that round to 1 become nextafter(1, 0).  Used for
 * uniform_real_distribution (src/Collision.cpp:46-51) and the channel
 * selection generate_canonical<double, 64> (src/Collision.cpp:948). */
double ora_canonical(ora_rng* r) {
    const double sum = (double)ora_draw(r);
    double ret = sum / 18446744073709551616.0;
    if (ret >= 1.0) ret = nextafter(1.0, 0.0);
    return ret;
}

double ora_uniform01(ora_rng* r) { return ora_canonical(r) * (1.0 - 0.0) + 0.0; }

/* uniform_int_distribution<int>(0, 1) on a 64-bit engine: Lemire's
 * nearly-divisionless reduction (ACM TOMACS 29(1), 2019) with range 2, whose
 * rejection threshold is 0, so it is the draw's top bit (src/Collision.cpp:745). */
int ora_bit(ora_rng* r) { return (int)(ora_draw(r) >> 63); }

/* normal_distribution: Marsaglia's polar method with one saved value, as in
 * libstdc++ (<bits/random.tcc>, normal_distribution::operator()). */
double ora_normal_draw(ora_normal* st, ora_rng* r, double mean, double stddev) {
    double ret;
    if (st->saved_available) {
        st->saved_available = 0;
        ret = st->saved;
    } else {
        double x, y, r2;
        do {
            x = 2.0 * ora_canonical(r) - 1.0;
            y = 2.0 * ora_canonical(r) - 1.0;
            r2 = x * x + y * y;
        } while (r2 > 1.0 || r2 == 0.0);
        const double mult = sqrt(-2 * log(r2) / r2);
        st->saved = x * mult;
        st->saved_available = 1;
        ret = y * mult;
    }
    return ret * stddev + mean;
}

/* ======================================================================= */
/* MCC: NullCollisionModel (src/Collision.cpp). */

static const double kBoltzmann = 1.380649e-23; /* src/Collision.cpp:16 */
static const double kThermalSigma = 8.0;       /* include/pic/Collision.hpp:139 */
static const double kEpsilon = 2.220446049250313080847e-16;

/* CrossSectionTable::evaluate, src/Collision.cpp:221-237 (clamped ends,
 * upper_bound, linear interpolation). */
static double table_eval(const ora_channel* ch, double energy) {
    const double* e = ch->energy;
    const size_t n = ch->rows;
    if (energy <= e[0]) return ch->sigma[0];
    if (energy >= e[n - 1]) return ch->sigma[n - 1];
    size_t lo = 0, hi = n; /* first index with e[i] > energy */
    while (lo < hi) {
        size_t mid = lo + (hi - lo) / 2;
        if (e[mid] > energy) hi = mid; else lo = mid + 1;
    }
    const size_t high = lo, low = high - 1;
    const double fraction = (energy - e[low]) / (e[high] - e[low]);
    return ch->sigma[low] + fraction * (ch->sigma[high] - ch->sigma[low]);
}

int ora_collider_init(ora_collider* c, const ora_mcc_model* m, double particle_mass) {
    memset(c, 0, sizeof *c);
    c->m = *m;
    c->particle_mass = particle_mass;
    /* src/Collision.cpp:348-362: thermal neutrals only with SI gas data */
    if (m->si && m->neutral_temperature > 0.0) {
        c->neutral_stddev = sqrt(kBoltzmann * m->neutral_temperature / m->neutral_mass);
    }
    if (!(m->max_frequency > 0.0) || m->max_candidates == 0 || m->nch <= 0)
        return seterr(4, "invalid MCC model");
    return 0;
}

/* collision_energy, src/Collision.cpp:579-594 */
static double collision_energy(const ora_collider* c, const ora_channel* ch, double rel_speed) {
    double energy_mass = c->particle_mass;
    if (ch->energy_frame == ORA_FRAME_CENTER_OF_MASS)
        energy_mass = c->particle_mass * c->m.neutral_mass / (c->particle_mass + c->m.neutral_mass);
    return 0.5 * energy_mass * rel_speed * rel_speed;
}

/* rates_for_speed, src/Collision.cpp:596-625 */
static int rates_for_speed(const ora_collider* c, double speed, double* rates) {
    double total = 0.0;
    for (int i = 0; i < c->m.nch; ++i) {
        const ora_channel* ch = &c->m.ch[i];
        const double energy = collision_energy(c, ch, speed);
        double rate = 0.0;
        if (energy >= ch->threshold_energy)
            rate = c->m.neutral_density * table_eval(ch, energy) * speed;
        rates[i] = rate;
        total += rate;
    }
    const double mx = c->m.max_frequency > total ? c->m.max_frequency : total;
    const double tolerance = 64.0 * kEpsilon * mx;
    if (total > c->m.max_frequency + tolerance)
        return seterr(1, "MCC total collision frequency exceeds configured max_frequency");
    return 0;
}

/* validate_frequency_bound, src/Collision.cpp:627-685 */
static int validate_bound(const ora_collider* c, double projectile_speed) {
    double rates[ORA_MAX_CHANNELS];
    if (c->neutral_stddev == 0.0) return rates_for_speed(c, projectile_speed, rates);
    const double limit = kThermalSigma * c->neutral_stddev;
    const double max_rel = projectile_speed + limit;
    double bound = 0.0;
    for (int i = 0; i < c->m.nch; ++i) {
        const ora_channel* ch = &c->m.ch[i];
        const double max_e = collision_energy(c, ch, max_rel);
        if (max_e < ch->threshold_energy) continue;
        const double min_rel = projectile_speed - limit > 0.0 ? projectile_speed - limit : 0.0;
        double min_e = collision_energy(c, ch, min_rel);
        if (ch->threshold_energy > min_e) min_e = ch->threshold_energy;
        double smax = table_eval(ch, min_e);
        const double s2 = table_eval(ch, max_e);
        if (s2 > smax) smax = s2;
        for (size_t k = 0; k < ch->rows; ++k) {
            const double e = ch->energy[k];
            if (e >= min_e && e <= max_e && ch->sigma[k] > smax) smax = ch->sigma[k];
        }
        bound += c->m.neutral_density * smax * max_rel;
    }
    const double mx = c->m.max_frequency > bound ? c->m.max_frequency : bound;
    if (bound > c->m.max_frequency + 64.0 * kEpsilon * mx)
        return seterr(3, "MCC thermal-neutral collision-frequency bound exceeds configured max_frequency");
    return 0;
}

/* open_unit_interval, src/Collision.cpp:46-51 */
static double open_unit(ora_rng* r) {
    double value = ora_uniform01(r);
    while (!(value > 0.0)) value = ora_uniform01(r);
    return value;
}

/* isotropic_velocity, src/Collision.cpp:53-64 */
static void isotropic(double speed, ora_rng* r, double out[3]) {
    const double cosine = 2.0 * ora_uniform01(r) - 1.0;
    const double t = 1.0 - cosine * cosine;
    const double sine = sqrt(0.0 > t ? 0.0 : t);
    const double azimuth = 2.0 * acos(-1.0) * ora_uniform01(r);
    out[0] = speed * sine * cos(azimuth);
    out[1] = speed * sine * sin(azimuth);
    out[2] = speed * cosine;
}

static double norm3(const double v[3]) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

/* MeanCosineTable::evaluate, src/Collision.cpp:296-313 */
static double mean_cosine_eval(const ora_channel* ch, double energy) {
    const double* e = ch->mu_energy;
    const size_t n = ch->mu_rows;
    if (energy <= e[0]) return ch->mu[0];
    if (energy >= e[n - 1]) return ch->mu[n - 1];
    size_t lo = 0, hi = n; /* upper_bound */
    while (lo < hi) {
        const size_t mid = lo + (hi - lo) / 2;
        if (energy < e[mid]) hi = mid; else lo = mid + 1;
    }
    const size_t high = lo, low = high - 1;
    const double fraction = (energy - e[low]) / (e[high] - e[low]);
    return ch->mu[low] + fraction * (ch->mu[high] - ch->mu[low]);
}

/* angular_velocity (Henyey-Greenstein about the incoming direction),
 * src/Collision.cpp:66-129 */
static void angular_velocity(const double in[3], double speed, double g, ora_rng* r, double out[3]) {
    const double in_speed = norm3(in);
    if (!(in_speed > 0.0)) { isotropic(speed, r, out); return; }
    const double sample = ora_uniform01(r);
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
    const double azimuth = 2.0 * acos(-1.0) * ora_uniform01(r);
    const double dir[3] = {in[0] / in_speed, in[1] / in_speed, in[2] / in_speed};
    const double h[3] = {0.0, fabs(dir[2]) < 0.9 ? 0.0 : 1.0, fabs(dir[2]) < 0.9 ? 1.0 : 0.0};
    double tg[3] = {h[1] * dir[2] - h[2] * dir[1], h[2] * dir[0] - h[0] * dir[2], h[0] * dir[1] - h[1] * dir[0]};
    const double tn = norm3(tg);
    tg[0] /= tn; tg[1] /= tn; tg[2] /= tn;
    const double bt[3] = {dir[1] * tg[2] - dir[2] * tg[1], dir[2] * tg[0] - dir[0] * tg[2],
                          dir[0] * tg[1] - dir[1] * tg[0]};
    const double tf = sine * cos(azimuth), bf = sine * sin(azimuth);
    for (int d = 0; d < 3; ++d) out[d] = speed * (cosine * dir[d] + tf * tg[d] + bf * bt[d]);
}

/* sample_neutral_velocity_3v, src/Collision.cpp:702-715 (a fresh normal
 * distribution object per call, bounded at 8 sigma) */
static int neutral_3v(const ora_collider* c, ora_rng* r, double out[3]) {
    out[0] = out[1] = out[2] = 0.0;
    if (c->neutral_stddev == 0.0) return 0;
    ora_normal nd = {0, 0.0};
    const double limit = kThermalSigma * c->neutral_stddev;
    for (int attempt = 0; attempt < 1024; ++attempt) {
        out[0] = ora_normal_draw(&nd, r, 0.0, c->neutral_stddev);
        out[1] = ora_normal_draw(&nd, r, 0.0, c->neutral_stddev);
        out[2] = ora_normal_draw(&nd, r, 0.0, c->neutral_stddev);
        if (norm3(out) <= limit) return 0;
    }
    return seterr(6, "thermal-neutral 3V sampler exceeded its rejection limit");
}

/* apply_channel (3V), src/Collision.cpp:762-829 */
static void apply_channel3(const ora_collider* c, int idx, double v[3], const double vn[3], ora_rng* r) {
    const ora_channel* ch = &c->m.ch[idx];
    if (ch->process == ORA_ATTACHMENT) { v[0] = v[1] = v[2] = 0.0; return; }
    if (ch->process == ORA_CHARGE_EXCHANGE) { v[0] = vn[0]; v[1] = vn[1]; v[2] = vn[2]; return; }
    const double rel[3] = {v[0] - vn[0], v[1] - vn[1], v[2] - vn[2]};
    const double initial_speed = norm3(rel);
    double energy = 0.5 * c->particle_mass * initial_speed * initial_speed;
    if (ch->process == ORA_EXCITATION || ch->process == ORA_IONIZATION) {
        const double e2 = energy - ch->threshold_energy;
        energy = 0.0 > e2 ? 0.0 : e2;
    }
    if (ch->process == ORA_IONIZATION) energy *= 0.5;
    const double speed = sqrt(2.0 * energy / c->particle_mass);
    double sc[3];
    if (ch->angular == ORA_BACKWARD) { sc[0] = -rel[0]; sc[1] = -rel[1]; sc[2] = -rel[2]; }
    else if (ch->angular == ORA_HENYEY_GREENSTEIN && ch->mu_rows)
        angular_velocity(rel, speed, mean_cosine_eval(ch, collision_energy(c, ch, initial_speed)), r, sc);
    else isotropic(speed, r, sc);
    if (ch->process == ORA_ELASTIC && c->m.neutral_mass > 0.0) {
        const double total = c->particle_mass + c->m.neutral_mass;
        const double rf = c->m.neutral_mass / total;
        for (int d = 0; d < 3; ++d)
            v[d] = (c->particle_mass * v[d] + c->m.neutral_mass * vn[d]) / total + rf * sc[d];
    } else {
        for (int d = 0; d < 3; ++d) v[d] = vn[d] + sc[d];
    }
}

/* NullCollisionModel::collide(Vec3&), src/Collision.cpp:907-993 */
int ora_collide3(const ora_collider* c, double v[3], double dt, ora_rng* r, ora_collide_stats* st) {
    memset(st, 0, sizeof *st);
    const uint64_t start = r->index;
    if (!isfinite(v[0]) || !isfinite(v[1]) || !isfinite(v[2]))
        return seterr(4, "MCC particle velocity must be finite");
    double elapsed = 0.0;
    int rc;
    for (;;) {
        if ((rc = validate_bound(c, norm3(v)))) return rc;
        const double waiting = -log(open_unit(r)) / c->m.max_frequency;
        if (!isfinite(waiting) || waiting >= dt - elapsed) break;
        elapsed += waiting;
        ++st->candidates;
        if (st->candidates > c->m.max_candidates)
            return seterr(2, "MCC candidate limit exceeded");
        double vn[3];
        if ((rc = neutral_3v(c, r, vn))) return rc;
        const double rel[3] = {v[0] - vn[0], v[1] - vn[1], v[2] - vn[2]};
        double rates[ORA_MAX_CHANNELS];
        if ((rc = rates_for_speed(c, norm3(rel), rates))) return rc;
        const double selection = ora_canonical(r) * c->m.max_frequency;
        double cumulative = 0.0;
        int accepted = 0;
        for (int ch = 0; ch < c->m.nch; ++ch) {
            cumulative += rates[ch];
            if (selection < cumulative) {
                const double before = 0.5 * c->particle_mass * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
                apply_channel3(c, ch, v, vn, r);
                st->energy_change[ch] += 0.5 * c->particle_mass * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) - before;
                if (c->m.ch[ch].process == ORA_IONIZATION) {
                    const double rel2[3] = {v[0] - vn[0], v[1] - vn[1], v[2] - vn[2]};
                    const double sspeed = norm3(rel2);
                    double iso[3];
                    isotropic(sspeed, r, iso);
                    if (st->nsecondaries < 16) {
                        const int k = st->nsecondaries;
                        st->secondary_channel[k] = ch;
                        for (int d = 0; d < 3; ++d) {
                            st->secondary_velocity[k][d] = vn[d] + iso[d];
                            st->secondary_ion_velocity[k][d] = vn[d];
                        }
                    }
                    st->nsecondaries++;
                }
                ++st->channel_collisions[ch];
                if (c->m.ch[ch].process == ORA_ATTACHMENT) st->removed = 1;
                accepted = 1;
                break;
            }
        }
        if (!accepted) ++st->null_collisions;
        if (st->removed) break;
    }
    st->draws = r->index - start;
    if (r->overrun) return seterr(5, "recorded draw array overrun");
    return 0;
}

/* sample_neutral_velocity (scalar), src/Collision.cpp:687-700 (a fresh normal
 * distribution object per call, bounded at 8 sigma) */
static int neutral_1v(const ora_collider* c, ora_rng* r, double* out) {
    *out = 0.0;
    if (c->neutral_stddev == 0.0) return 0;
    ora_normal nd = {0, 0.0};
    const double limit = kThermalSigma * c->neutral_stddev;
    for (int attempt = 0; attempt < 1024; ++attempt) {
        const double value = ora_normal_draw(&nd, r, 0.0, c->neutral_stddev);
        if (fabs(value) <= limit) { *out = value; return 0; }
    }
    return seterr(6, "thermal-neutral scalar sampler exceeded its rejection limit");
}

/* apply_channel (1V), src/Collision.cpp:717-760: the scattered speed along a
 * random sign (uniform_int_distribution<int>(0, 1)) */
static void apply_channel1(const ora_collider* c, int idx, double* v, double vn, ora_rng* r) {
    const ora_channel* ch = &c->m.ch[idx];
    if (ch->process == ORA_ATTACHMENT) { *v = 0.0; return; }
    if (ch->process == ORA_CHARGE_EXCHANGE) { *v = vn; return; }
    const double rel = *v - vn;
    double energy = 0.5 * c->particle_mass * rel * rel;
    if (ch->process == ORA_EXCITATION || ch->process == ORA_IONIZATION) {
        const double e2 = energy - ch->threshold_energy;
        energy = 0.0 < e2 ? e2 : 0.0; /* std::max(0.0, e2) */
    }
    if (ch->process == ORA_IONIZATION) energy *= 0.5;
    const double speed = sqrt(2.0 * energy / c->particle_mass);
    const double scattered = ora_bit(r) == 0 ? -speed : speed;
    if (ch->process == ORA_ELASTIC && c->m.neutral_mass > 0.0) {
        const double total = c->particle_mass + c->m.neutral_mass;
        *v = (c->particle_mass * *v + c->m.neutral_mass * vn) / total + (c->m.neutral_mass / total) * scattered;
    } else {
        *v = vn + scattered;
    }
}

/* NullCollisionModel::collide(double&), src/Collision.cpp:831-905 */
int ora_collide1(const ora_collider* c, double* v, double dt, ora_rng* r, ora_collide_stats* st) {
    memset(st, 0, sizeof *st);
    const uint64_t start = r->index;
    for (int ch = 0; ch < c->m.nch; ++ch)
        if (c->m.ch[ch].process == ORA_IONIZATION || c->m.ch[ch].angular != ORA_ISOTROPIC)
            return seterr(10, "ionization and anisotropic MCC require the 3V collision interface");
    if (!isfinite(dt) || !(dt > 0.0)) return seterr(11, "MCC timestep must be positive and finite");
    double elapsed = 0.0;
    int rc;
    for (;;) {
        if ((rc = validate_bound(c, fabs(*v)))) return rc;
        const double waiting = -log(open_unit(r)) / c->m.max_frequency;
        if (!isfinite(waiting) || waiting >= dt - elapsed) break;
        elapsed += waiting;
        ++st->candidates;
        if (st->candidates > c->m.max_candidates)
            return seterr(2, "MCC candidate limit exceeded");
        double vn;
        if ((rc = neutral_1v(c, r, &vn))) return rc;
        double rates[ORA_MAX_CHANNELS];
        if ((rc = rates_for_speed(c, fabs(*v - vn), rates))) return rc;
        const double selection = ora_canonical(r) * c->m.max_frequency;
        double cumulative = 0.0;
        int accepted = 0;
        for (int ch = 0; ch < c->m.nch; ++ch) {
            cumulative += rates[ch];
            if (selection < cumulative) {
                const double before = 0.5 * c->particle_mass * *v * *v;
                apply_channel1(c, ch, v, vn, r);
                st->energy_change[ch] += 0.5 * c->particle_mass * *v * *v - before;
                ++st->channel_collisions[ch];
                if (c->m.ch[ch].process == ORA_ATTACHMENT) st->removed = 1;
                accepted = 1;
                break;
            }
        }
        if (!accepted) ++st->null_collisions;
        if (st->removed) break;
    }
    st->draws = r->index - start;
    if (r->overrun) return seterr(5, "recorded draw array overrun");
    return 0;
}

/* ======================================================================= */
/* 1D grid kernels. */

/* wrap_periodic, src/FieldSolver.cpp:15-17 (also src/Simulation.cpp:1041-1046) */
static double wrap(double x, double L) { return fmod(fmod(x, L) + L, L); }

/* interpolate_electric(const Grid&), src/FieldSolver.cpp:909-924 */
double ora_gather1d(const double* E, size_t nx, double length, double dx, int dirichlet, double x) {
    if (!dirichlet) {
        const double xp = wrap(x, length);
        const double g = xp / dx;
        const size_t i = (size_t)floor(g);
        const double f = g - (double)i;
        return E[i % nx] * (1.0 - f) + E[(i + 1) % nx] * f;
    }
    const double xp = x < 0.0 ? 0.0 : (x > length ? length : x);
    const double g = xp / dx;
    double fl = floor(g);
    if ((double)(nx - 2) < fl) fl = (double)(nx - 2);
    const size_t i = (size_t)fl;
    const double f = g - (double)i;
    return E[i] * (1.0 - f) + E[i + 1] * f;
}

/* Grid::node_volume, src/Grid.cpp:26-30 */
static double node_volume(size_t i, size_t nx, double dx, int dirichlet) {
    if (!dirichlet) return dx;
    return (i == 0 || i + 1 == nx) ? 0.5 * dx : dx;
}

/* Species::deposit_charge, src/Species.cpp:161-185 */
void ora_deposit1d(double* rho, size_t nx, double length, double dx, int dirichlet,
                   double charge, double weight, size_t n, const double* x, const uint8_t* alive) {
    const double qwdx = charge * weight / dx;
    for (size_t p = 0; p < n; ++p) {
        if (alive && !alive[p]) continue;
        if (!dirichlet) {
            const double xp = wrap(x[p], length);
            const double g = xp / dx;
            const size_t i = (size_t)floor(g);
            const double f = g - (double)i;
            rho[i % nx] += qwdx * (1.0 - f);
            rho[(i + 1) % nx] += qwdx * f;
        } else {
            const double xp = x[p] < 0.0 ? 0.0 : (x[p] > length ? length : x[p]);
            const double g = xp / dx;
            double fl = floor(g);
            if ((double)(nx - 2) < fl) fl = (double)(nx - 2);
            const size_t i = (size_t)fl;
            const double f = g - (double)i;
            rho[i] += charge * weight * (1.0 - f) / node_volume(i, nx, dx, 1);
            rho[i + 1] += charge * weight * f / node_volume(i + 1, nx, dx, 1);
        }
    }
}

/* FieldSolver::solve_periodic_spectral(Grid&), src/FieldSolver.cpp:407-440:
 * mean removal, a direct DFT per mode, phi_k = rho_k/(eps k^2), E_k = -i k phi_k. */
static void solve_periodic(const double* rho, double* phi, double* E, size_t n, double L, double eps) {
    const double twopi = 2.0 * 3.14159265358979323846;
    double mean = 0.0;
    for (size_t j = 0; j < n; ++j) mean += rho[j];
    mean /= (double)n;
    for (size_t j = 0; j < n; ++j) { phi[j] = 0.0; E[j] = 0.0; }
    for (size_t k = 1; k < n; ++k) {
        const double kk = (k <= n / 2) ? (double)k : -(double)(n - k);
        const double wave = twopi * kk / L;
        double re = 0.0, im = 0.0;
        for (size_t j = 0; j < n; ++j) {
            const double angle = -twopi * (double)(k * j) / (double)n;
            const double a = rho[j] - mean;
            /* complex += real * (cos, sin): libstdc++ real*complex is component-wise */
            re += a * cos(angle);
            im += a * sin(angle);
        }
        re /= (double)n;
        im /= (double)n;
        const double den = eps * wave * wave;
        const double pr = re / den, pi = im / den;
        /* Ek = -(0,1) * wave * phik = (wave*pi, -wave*pr) */
        const double ekr = wave * pi, eki = -(wave * pr);
        for (size_t j = 0; j < n; ++j) {
            const double angle = twopi * (double)(k * j) / (double)n;
            const double c = cos(angle), s = sin(angle);
            phi[j] += pr * c - pi * s;
            E[j] += ekr * c - eki * s;
        }
    }
}

/* FieldSolver::solve_dirichlet_tridiagonal, src/FieldSolver.cpp:733-759 */
static void solve_dirichlet(const double* rho, double* phi, double* E, size_t n, double dx,
                            double eps, double phil, double phir) {
    const double dx2 = dx * dx;
    phi[0] = phil;
    phi[n - 1] = phir;
    const size_t m = n - 2;
    double* cp = (double*)calloc(m, sizeof(double));
    double* dp = (double*)calloc(m, sizeof(double));
    double* d = (double*)calloc(m, sizeof(double));
    for (size_t i = 0; i < m; ++i) d[i] = rho[i + 1] * dx2 / eps;
    d[0] += phil;
    d[m - 1] += phir;
    cp[0] = -1.0 / 2.0;
    dp[0] = d[0] / 2.0;
    for (size_t i = 1; i < m; ++i) {
        const double denom = 2.0 + cp[i - 1];
        cp[i] = (i == m - 1) ? 0.0 : -1.0 / denom;
        dp[i] = (d[i] + dp[i - 1]) / denom;
    }
    phi[n - 2] = dp[m - 1];
    for (size_t ii = m - 1; ii-- > 0;) phi[ii + 1] = dp[ii] - cp[ii] * phi[ii + 2];
    for (size_t i = 1; i + 1 < n; ++i) E[i] = -(phi[i + 1] - phi[i - 1]) / (2.0 * dx);
    E[0] = -(phi[1] - phi[0]) / dx;
    E[n - 1] = -(phi[n - 1] - phi[n - 2]) / dx;
    free(cp); free(dp); free(d);
}

void ora_solve1d(double* rho, double* phi, double* E, size_t nx, double length, double dx,
                 int dirichlet, double eps, double phi_left, double phi_right) {
    if (dirichlet) solve_dirichlet(rho, phi, E, nx, dx, eps, phi_left, phi_right);
    else solve_periodic(rho, phi, E, nx, length, eps);
}

/* ======================================================================= */
/* 1D simulation driver: Simulation::step / deposit_and_solve /
 * apply_collisions (src/Simulation.cpp:678-1138). */

typedef struct {
    size_t n, cap;
    double *x, *v, *vh, *vy, *vz;
    uint8_t* alive;
    uint64_t lost_left, lost_right;
    double e_left, e_right;
} ora_store;

typedef struct {
    double x, v[3];
    int species;
} ora_product;

struct ora_sim1d {
    ora_config1d cfg;
    int mode;
    uint64_t philox_seed;
    double dx, eps, time;
    uint64_t step;
    double *rho, *phi, *E;
    ora_store sp[ORA_MAX_SPECIES];
    ora_collider col[ORA_MAX_MODELS];
    ora_mt64 mt;
    uint64_t candidates, nulls, per_channel[ORA_MAX_MODELS][ORA_MAX_CHANNELS];
    double bgk_energy;           /* channel_energy_change of the "bgk" channel */
    ora_product* staged;
    size_t nstaged, staged_cap;
    double electric_work[ORA_MAX_SPECIES]; /* species_power_transfer_, src/Simulation.cpp:1094-1132 */
    struct {
        int on;
        ora_spatial_average1d cfg;
        size_t spc;              /* RF steps per cycle (0: no RF contract) */
        size_t P;                /* phase bins */
        int nch, off[ORA_MAX_MODELS];
        double* tot;             /* [5 moments][species][nx] + [3 fields][nx] */
        double* phase;           /* [P][same block] */
        double* scratch;         /* [5][nx], one species of one sample */
        double* coll;            /* [nch][nx] */
        double* coll_phase;      /* [P][nch][nx] */
        uint64_t samples, coll_steps, *psamples, *pcoll;
        int coll_active;
        size_t coll_phase_id;
        uint64_t* eedf_cnt;      /* [P][R][2] */
        double* eedf_sum;        /* [P][R][7] */
        double* eedf_hist;       /* [P][R][bins] */
    } diag;
};

static void store_reserve(ora_store* s, size_t cap) {
    if (cap <= s->cap) return;
    s->x = realloc(s->x, cap * sizeof(double));
    s->v = realloc(s->v, cap * sizeof(double));
    s->vh = realloc(s->vh, cap * sizeof(double));
    s->vy = realloc(s->vy, cap * sizeof(double));
    s->vz = realloc(s->vz, cap * sizeof(double));
    s->alive = realloc(s->alive, cap);
    s->cap = cap;
}

static double f32_round(double v) { return (double)(float)v; }

static void round_stored(ora_store* st) {
    for (size_t i = 0; i < st->n; ++i) {
        st->vh[i] = f32_round(st->vh[i]);
        st->vy[i] = f32_round(st->vy[i]);
        st->vz[i] = f32_round(st->vz[i]);
    }
}

ora_sim1d* ora_sim1d_create(const ora_config1d* cfg, int mode, uint64_t philox_seed) {
    ora_sim1d* s = calloc(1, sizeof *s);
    s->cfg = *cfg;
    s->mode = mode;
    s->philox_seed = philox_seed;
    s->dx = cfg->length / (double)(cfg->dirichlet ? cfg->nx - 1 : cfg->nx);
    s->eps = cfg->si ? 8.8541878128e-12 : 1.0; /* include/pic/Types.hpp:7-8 */
    s->rho = calloc(cfg->nx, sizeof(double));
    s->phi = calloc(cfg->nx, sizeof(double));
    s->E = calloc(cfg->nx, sizeof(double));
    ora_mt64_seed(&s->mt, cfg->seed);
    /* the collision checks of validate() and the Simulation constructor,
     * src/Simulation.cpp:95-100, :388-392 */
    if (!isfinite(cfg->bgk_frequency) || cfg->bgk_frequency < 0.0) {
        seterr(4, "collision frequency must be non-negative and finite");
        ora_sim1d_destroy(s);
        return NULL;
    }
    if (!isfinite(cfg->bgk_neutral_velocity) || cfg->bgk_neutral_velocity < 0.0) {
        seterr(4, "neutral_temperature_velocity must be non-negative and finite");
        ora_sim1d_destroy(s);
        return NULL;
    }
    if (cfg->bgk && cfg->nmodels > 0) {
        seterr(4, "named collision models cannot be combined with the legacy collision model");
        ora_sim1d_destroy(s);
        return NULL;
    }
    for (int m = 0; m < cfg->nmodels; ++m) {
        const ora_mcc_model* mm = &cfg->models[m];
        if (ora_collider_init(&s->col[m], mm, cfg->species[mm->species].mass)) {
            ora_sim1d_destroy(s);
            return NULL;
        }
    }
    return s;
}

void ora_sim1d_destroy(ora_sim1d* s) {
    if (!s) return;
    for (int i = 0; i < ORA_MAX_SPECIES; ++i) {
        free(s->sp[i].x); free(s->sp[i].v); free(s->sp[i].vh);
        free(s->sp[i].vy); free(s->sp[i].vz); free(s->sp[i].alive);
    }
    free(s->rho); free(s->phi); free(s->E); free(s->staged);
    free(s->diag.tot); free(s->diag.phase); free(s->diag.scratch); free(s->diag.coll);
    free(s->diag.coll_phase); free(s->diag.psamples); free(s->diag.pcoll);
    free(s->diag.eedf_cnt); free(s->diag.eedf_sum); free(s->diag.eedf_hist);
    free(s);
}

int ora_sim1d_load(ora_sim1d* s, int species, size_t n, const double* x, const double* v,
                   const double* vh, const double* vy, const double* vz, const uint8_t* alive) {
    ora_store* st = &s->sp[species];
    store_reserve(st, n + 16);
    st->n = 0;
    for (size_t i = 0; i < n; ++i) {
        if (s->mode != 0 && alive && !alive[i]) continue; /* device layout holds live particles only */
        const size_t k = st->n++;
        st->x[k] = x[i]; st->v[k] = v[i]; st->vh[k] = vh[i];
        st->vy[k] = vy ? vy[i] : 0.0; st->vz[k] = vz ? vz[i] : 0.0;
        st->alive[k] = alive ? alive[i] : 1;
    }
    if (s->mode == 2) round_stored(st);
    return 0;
}

/* Mode 2 (the device's FP32 particle form): v_half, v_y and v_z are stored as
 * float, rounded to nearest each time a particle is stored (load, the end of
 * initialize, after each drift, and whenever the state is read back); the
 * position stays FP64 and all arithmetic is FP64. */
int ora_sim1d_round_fp32(ora_sim1d* s) {
    for (int k = 0; k < s->cfg.nspecies; ++k) round_stored(&s->sp[k]);
    return 0;
}

/* electrode_potential, src/Simulation.cpp:678-685 */
static double electrode(double offset, const double drive[3], double t) {
    return offset + drive[0] * sin(2.0 * 3.14159265358979323846 * drive[1] * t + drive[2]);
}

/* deposit_and_solve, src/Simulation.cpp:687-696 */
static void deposit_and_solve(ora_sim1d* s, double field_time) {
    const ora_config1d* c = &s->cfg;
    memset(s->rho, 0, c->nx * sizeof(double));
    for (int k = 0; k < c->nspecies; ++k)
        ora_deposit1d(s->rho, c->nx, c->length, s->dx, c->dirichlet, c->species[k].charge,
                      c->species[k].weight, s->sp[k].n, s->sp[k].x, s->sp[k].alive);
    ora_solve1d(s->rho, s->phi, s->E, c->nx, c->length, s->dx, c->dirichlet, s->eps,
                electrode(c->phi_left, c->drive_left, field_time),
                electrode(c->phi_right, c->drive_right, field_time));
}

/* Simulation::initialize after the particles are loaded, src/Simulation.cpp:760-767 */
int ora_sim1d_initialize(ora_sim1d* s) {
    s->time = 0.0;
    s->step = 0;
    memset(s->electric_work, 0, sizeof s->electric_work);
    deposit_and_solve(s, 0.0);
    for (int sid = 0; sid < s->cfg.nspecies; ++sid) {
        ora_store* st = &s->sp[sid];
        const double qm = s->cfg.species[sid].charge / s->cfg.species[sid].mass;
        for (size_t i = 0; i < st->n; ++i)
            if (st->alive[i])
                st->vh[i] = st->v[i] - 0.5 * qm * ora_gather1d(s->E, s->cfg.nx, s->cfg.length, s->dx,
                                                              s->cfg.dirichlet, st->x[i]) * s->cfg.dt;
        if (s->mode == 2) round_stored(st);
    }
    return 0;
}

int ora_sim1d_initialize_fields(ora_sim1d* s, double time, uint64_t step) {
    s->time = time;
    s->step = step;
    deposit_and_solve(s, time);
    return 0;
}

static double gather(const ora_sim1d* s, double x) {
    return ora_gather1d(s->E, s->cfg.nx, s->cfg.length, s->dx, s->cfg.dirichlet, x);
}

static int stage_product(ora_sim1d* s, int species, double x, const double v[3]) {
    if (s->nstaged == s->staged_cap) {
        s->staged_cap = s->staged_cap ? 2 * s->staged_cap : 64;
        s->staged = realloc(s->staged, s->staged_cap * sizeof(ora_product));
    }
    ora_product* p = &s->staged[s->nstaged++];
    p->x = x; p->species = species;
    p->v[0] = v[0]; p->v[1] = v[1]; p->v[2] = v[2];
    return 0;
}

/* ---- CCP campaign diagnostics, src/Simulation.cpp:1163-1370 ------------- */

static size_t diag_block(const ora_sim1d* s) { return (5 * (size_t)s->cfg.nspecies + 3) * s->cfg.nx; }

int ora_sim1d_enable_spatial_average(ora_sim1d* s, const ora_spatial_average1d* cfg) {
    const size_t nx = s->cfg.nx;
    s->diag.on = 1;
    s->diag.cfg = *cfg;
    s->diag.spc = cfg->rf_frequency > 0.0 ? (size_t)llround(1.0 / (cfg->rf_frequency * s->cfg.dt)) : 0;
    s->diag.P = cfg->phase_bins;
    s->diag.nch = 0;
    for (int m = 0; m < s->cfg.nmodels; ++m) {
        s->diag.off[m] = s->diag.nch;
        s->diag.nch += s->cfg.models[m].nch;
    }
    if (s->cfg.bgk) s->diag.nch = 1; /* the "bgk" channel */
    const size_t P = s->diag.P, nch = (size_t)s->diag.nch;
    s->diag.tot = calloc(diag_block(s), sizeof(double));
    s->diag.phase = calloc(P * diag_block(s) + 1, sizeof(double));
    s->diag.scratch = calloc(5 * nx, sizeof(double));
    s->diag.coll = calloc(nch * nx + 1, sizeof(double));
    s->diag.coll_phase = calloc(P * nch * nx + 1, sizeof(double));
    s->diag.psamples = calloc(P + 1, sizeof(uint64_t));
    s->diag.pcoll = calloc(P + 1, sizeof(uint64_t));
    if (cfg->eedf_species >= 0) {
        const size_t R = (size_t)cfg->eedf_regions;
        s->diag.eedf_cnt = calloc(P * R * 2 + 1, sizeof(uint64_t));
        s->diag.eedf_sum = calloc(P * R * 7 + 1, sizeof(double));
        s->diag.eedf_hist = calloc(P * R * cfg->eedf_bins + 1, sizeof(double));
    }
    return 0;
}

/* begin_spatial_collision_step, src/Simulation.cpp:1214-1236 */
static void diag_begin_collision_step(ora_sim1d* s) {
    const ora_spatial_average1d* a = &s->diag.cfg;
    const uint64_t cs = s->step + 1;
    s->diag.coll_active = 0;
    s->diag.coll_phase_id = s->diag.P;
    if (!s->diag.on || s->diag.nch == 0 || cs < a->start_step || cs > a->end_step) return;
    s->diag.coll_active = 1;
    ++s->diag.coll_steps;
    if (s->diag.P) {
        const size_t in_cycle = (size_t)(cs - a->start_step) % s->diag.spc;
        s->diag.coll_phase_id = in_cycle * s->diag.P / s->diag.spc;
        ++s->diag.pcoll[s->diag.coll_phase_id];
    }
}

/* The two-node CIC stencil of the diagnostics deposits (periodic wrap, or the
 * clamped Dirichlet form with the half-cell wall volumes),
 * src/Simulation.cpp:1193-1211, src/Species.cpp:314-334 */
static void diag_stencil(const ora_sim1d* s, double x, size_t node[2], double shape[2], double vol[2]) {
    const ora_config1d* c = &s->cfg;
    const double dx = s->dx;
    if (!c->dirichlet) {
        const double coordinate = wrap(x, c->length) / dx;
        const size_t cell = (size_t)floor(coordinate);
        const double f = coordinate - (double)cell;
        node[0] = cell % c->nx; node[1] = (cell + 1) % c->nx;
        shape[0] = 1.0 - f; shape[1] = f;
        vol[0] = vol[1] = dx;
    } else {
        const double bounded = x < 0.0 ? 0.0 : (c->length < x ? c->length : x);
        const double coordinate = bounded / dx;
        double fl = floor(coordinate);
        if ((double)(c->nx - 2) < fl) fl = (double)(c->nx - 2);
        const size_t cell = (size_t)fl;
        const double f = coordinate - (double)cell;
        node[0] = cell; node[1] = cell + 1;
        shape[0] = 1.0 - f; shape[1] = f;
        vol[0] = node_volume(cell, c->nx, dx, 1);
        vol[1] = node_volume(cell + 1, c->nx, dx, 1);
    }
}

/* deposit_spatial_collision_energy, src/Simulation.cpp:1171-1212 */
static void diag_collision_energy(ora_sim1d* s, double x, int channel, double e) {
    if (!s->diag.coll_active) return;
    size_t node[2];
    double shape[2], vol[2];
    diag_stencil(s, x, node, shape, vol);
    const size_t nx = s->cfg.nx;
    for (int k = 0; k < 2; ++k) {
        const double density = e * shape[k] / vol[k];
        s->diag.coll[(size_t)channel * nx + node[k]] += density;
        if (s->diag.coll_phase_id < s->diag.P)
            s->diag.coll_phase[(s->diag.coll_phase_id * (size_t)s->diag.nch + (size_t)channel) * nx + node[k]] +=
                density;
    }
}

/* The stored transverse velocity as the device's moment pass reads it (mode 2:
 * rounded to float, as stored after the collision part). */
static double diag_comp(const ora_sim1d* s, double v) { return s->mode == 2 ? f32_round(v) : v; }

/* accumulate_phase_eedf, src/Simulation.cpp:1238-1285 */
static void diag_eedf(ora_sim1d* s, size_t phase) {
    const ora_spatial_average1d* a = &s->diag.cfg;
    const int sid = a->eedf_species;
    const ora_store* st = &s->sp[sid];
    const double scale = s->cfg.si ? 1.602176634e-19 : 1.0; /* include/pic/Types.hpp:9 */
    const double weight = s->cfg.species[sid].weight, mass = s->cfg.species[sid].mass;
    const size_t R = (size_t)a->eedf_regions;
    for (size_t i = 0; i < st->n; ++i) {
        if (!st->alive[i]) continue;
        const double vy = diag_comp(s, st->vy[i]), vz = diag_comp(s, st->vz[i]);
        const double vsq = st->v[i] * st->v[i] + (s->cfg.vdim == 3 ? vy * vy + vz * vz : 0.0);
        const double energy = 0.5 * mass * vsq / scale;
        for (size_t r = 0; r < R; ++r) {
            if (st->x[i] < a->eedf_x_min[r] || st->x[i] > a->eedf_x_max[r]) continue;
            uint64_t* cnt = s->diag.eedf_cnt + (phase * R + r) * 2;
            double* sum = s->diag.eedf_sum + (phase * R + r) * 7;
            ++cnt[0];
            sum[0] += weight;
            sum[2] += weight * energy;
            sum[3] += weight * energy * energy;
            sum[4] += weight * st->v[i];
            sum[5] += weight * (s->cfg.vdim == 3 ? vy : st->vy[i]);
            sum[6] += weight * (s->cfg.vdim == 3 ? vz : st->vz[i]);
            if (energy >= a->eedf_energy_max) {
                ++cnt[1];
                sum[1] += weight;
            } else {
                size_t bin = (size_t)(energy / a->eedf_energy_max * (double)a->eedf_bins);
                if (bin > a->eedf_bins - 1) bin = a->eedf_bins - 1;
                s->diag.eedf_hist[(phase * R + r) * a->eedf_bins + bin] += weight;
            }
        }
    }
}

/* accumulate_spatial_average, src/Simulation.cpp:1287-1370, with
 * Species::deposit_velocity_moments, src/Species.cpp:285-336 */
static void diag_accumulate(ora_sim1d* s) {
    const ora_spatial_average1d* a = &s->diag.cfg;
    const uint64_t k = s->step;
    if (!s->diag.on || k < a->start_step || k > a->end_step || (k - a->start_step) % a->interval != 0) return;
    const size_t nx = s->cfg.nx, ns = (size_t)s->cfg.nspecies, P = s->diag.P;
    size_t phase = P;
    if (P) {
        const size_t per_cycle = s->diag.spc / a->interval;
        const size_t in_cycle = (size_t)((k - a->start_step) / a->interval) % per_cycle;
        phase = in_cycle * P / per_cycle;
    }
    if (s->mode == 2) ora_sim1d_round_fp32(s); /* the device stores its state here */
    double* bin = phase < P ? s->diag.phase + phase * diag_block(s) : NULL;
    for (size_t sid = 0; sid < ns; ++sid) {
        const ora_store* st = &s->sp[sid];
        const double weight = s->cfg.species[sid].weight, mass = s->cfg.species[sid].mass;
        double* sc = s->diag.scratch;
        memset(sc, 0, 5 * nx * sizeof(double));
        for (size_t i = 0; i < st->n; ++i) {
            if (!st->alive[i]) continue;
            const double v = st->v[i];
            const double vy = s->cfg.vdim == 3 ? diag_comp(s, st->vy[i]) : 0.0;
            const double vz = s->cfg.vdim == 3 ? diag_comp(s, st->vz[i]) : 0.0;
            const double pe = 0.5 * mass * weight * (v * v + vy * vy + vz * vz);
            size_t node[2];
            double shape[2], vol[2];
            diag_stencil(s, st->x[i], node, shape, vol);
            for (int q = 0; q < 2; ++q) {
                const double rd = weight * shape[q] / vol[q];
                sc[0 * nx + node[q]] += rd;
                sc[1 * nx + node[q]] += rd * v;
                sc[2 * nx + node[q]] += rd * vy;
                sc[3 * nx + node[q]] += rd * vz;
                sc[4 * nx + node[q]] += pe * shape[q] / vol[q];
            }
        }
        for (size_t m = 0; m < 5; ++m)
            for (size_t i = 0; i < nx; ++i) {
                s->diag.tot[(m * ns + sid) * nx + i] += sc[m * nx + i];
                if (bin) bin[(m * ns + sid) * nx + i] += sc[m * nx + i];
            }
    }
    double* f = s->diag.tot + 5 * ns * nx;
    for (size_t i = 0; i < nx; ++i) {
        f[i] += s->phi[i];
        f[nx + i] += s->E[i];
        f[2 * nx + i] += s->E[i] * s->E[i];
        if (bin) {
            double* g = bin + 5 * ns * nx;
            g[i] += s->phi[i];
            g[nx + i] += s->E[i];
            g[2 * nx + i] += s->E[i] * s->E[i];
        }
    }
    if (bin) ++s->diag.psamples[phase];
    if (phase < P && a->eedf_species >= 0) diag_eedf(s, phase);
    ++s->diag.samples;
}

void ora_sim1d_spatial_counts(const ora_sim1d* s, uint64_t* samples, uint64_t* collision_steps,
                              uint64_t* phase_samples, uint64_t* collision_phase_steps) {
    if (samples) *samples = s->diag.samples;
    if (collision_steps) *collision_steps = s->diag.coll_steps;
    for (size_t p = 0; p < s->diag.P; ++p) {
        if (phase_samples) phase_samples[p] = s->diag.psamples[p];
        if (collision_phase_steps) collision_phase_steps[p] = s->diag.pcoll[p];
    }
}

int ora_sim1d_spatial_sums(const ora_sim1d* s, int quantity, int index, int phase, double* out) {
    const size_t nx = s->cfg.nx, ns = (size_t)s->cfg.nspecies;
    if (!s->diag.on || phase < -1 || (phase >= 0 && (size_t)phase >= s->diag.P)) return seterr(1, "bad phase");
    const double* src;
    if (quantity == 8) {
        if (index < 0 || index >= s->diag.nch) return seterr(1, "bad channel");
        src = phase < 0 ? s->diag.coll + (size_t)index * nx
                        : s->diag.coll_phase + ((size_t)phase * (size_t)s->diag.nch + (size_t)index) * nx;
    } else {
        const double* blk = phase < 0 ? s->diag.tot : s->diag.phase + (size_t)phase * diag_block(s);
        if (quantity >= 0 && quantity < 5) {
            if (index < 0 || (size_t)index >= ns) return seterr(1, "bad species");
            src = blk + ((size_t)quantity * ns + (size_t)index) * nx;
        } else if (quantity >= 5 && quantity < 8) {
            src = blk + 5 * ns * nx + (size_t)(quantity - 5) * nx;
        } else {
            return seterr(1, "bad quantity");
        }
    }
    memcpy(out, src, nx * sizeof(double));
    return 0;
}

int ora_sim1d_phase_eedf(const ora_sim1d* s, int phase, int region, uint64_t* counts, double* sums,
                         double* histogram) {
    const ora_spatial_average1d* a = &s->diag.cfg;
    if (!s->diag.on || a->eedf_species < 0 || phase < 0 || (size_t)phase >= s->diag.P || region < 0 ||
        region >= a->eedf_regions)
        return seterr(1, "bad phase or region");
    const size_t at = (size_t)phase * (size_t)a->eedf_regions + (size_t)region;
    if (counts) memcpy(counts, s->diag.eedf_cnt + at * 2, 2 * sizeof(uint64_t));
    if (sums) memcpy(sums, s->diag.eedf_sum + at * 7, 7 * sizeof(double));
    if (histogram) memcpy(histogram, s->diag.eedf_hist + at * a->eedf_bins, a->eedf_bins * sizeof(double));
    return 0;
}

/* initialize_leapfrog_half_step, src/Pusher.cpp:66-68 */
static double init_half(double v, double E, double qm, double dt) { return v - 0.5 * qm * E * dt; }

/* The legacy BGK branch of apply_collisions, src/Simulation.cpp:772-834:
 * every live particle of every species relaxes to a fresh neutral Maxwellian
 * with probability 1 - exp(-frequency dt), then re-initialises its half-step
 * velocity.  Mode 0 draws from the shared engine with one normal_distribution
 * (and its saved value) per species; modes 1-2 draw from the particle's
 * (seed, slot, step, species) Philox stream with its own normal state. */
static void apply_bgk(ora_sim1d* s) {
    const ora_config1d* c = &s->cfg;
    const double probability = 1.0 - exp(-c->bgk_frequency * c->dt);
    const double vt = c->bgk_neutral_velocity;
    for (int sid = 0; sid < c->nspecies; ++sid) {
        ora_store* st = &s->sp[sid];
        const double qm = c->species[sid].charge / c->species[sid].mass;
        ora_normal shared_normal = {0, 0.0};
        for (size_t i = 0; i < st->n; ++i) {
            if (!st->alive[i]) continue;
            ora_rng r;
            ora_normal own = {0, 0.0};
            ora_normal* ns = &own;
            memset(&r, 0, sizeof r);
            if (s->mode == 0) { r.kind = ORA_SRC_MT64; r.mt = &s->mt; ns = &shared_normal; }
            else {
                r.kind = ORA_SRC_PHILOX;
                r.key[0] = (uint32_t)s->philox_seed; r.key[1] = (uint32_t)(s->philox_seed >> 32);
                r.ctr[0] = (uint32_t)i; r.ctr[1] = (uint32_t)s->step; r.ctr[2] = (uint32_t)sid;
            }
            if (ora_uniform01(&r) >= probability) continue;
            const double before = 0.5 * c->species[sid].mass * c->species[sid].weight *
                (st->v[i] * st->v[i] + (c->vdim == 3 ? st->vy[i] * st->vy[i] + st->vz[i] * st->vz[i] : 0.0));
            st->v[i] = ora_normal_draw(ns, &r, 0.0, vt);
            if (c->vdim == 3) {
                st->vy[i] = ora_normal_draw(ns, &r, 0.0, vt);
                st->vz[i] = ora_normal_draw(ns, &r, 0.0, vt);
            }
            ++s->candidates;
            ++s->per_channel[0][0];
            const double after = 0.5 * c->species[sid].mass * c->species[sid].weight *
                (st->v[i] * st->v[i] + (c->vdim == 3 ? st->vy[i] * st->vy[i] + st->vz[i] * st->vz[i] : 0.0));
            const double change = after - before;
            s->bgk_energy += change;
            if (s->diag.coll_active) diag_collision_energy(s, st->x[i], 0, change);
            st->vh[i] = init_half(st->v[i], gather(s, st->x[i]), qm, c->dt);
        }
    }
}

/* apply_collisions (named null-collision models), src/Simulation.cpp:835-1006 */
static int apply_collisions(ora_sim1d* s) {
    const ora_config1d* c = &s->cfg;
    s->nstaged = 0;
    if (c->bgk && c->bgk_frequency > 0.0) apply_bgk(s);
    for (int m = 0; m < c->nmodels; ++m) {
        const int sid = c->models[m].species;
        ora_store* st = &s->sp[sid];
        const double qm = c->species[sid].charge / c->species[sid].mass;
        const size_t initial = st->n;
        for (size_t i = 0; i < initial; ++i) {
            if (!st->alive[i]) continue;
            ora_rng r;
            memset(&r, 0, sizeof r);
            if (s->mode == 0) { r.kind = ORA_SRC_MT64; r.mt = &s->mt; }
            else {
                r.kind = ORA_SRC_PHILOX;
                r.key[0] = (uint32_t)s->philox_seed; r.key[1] = (uint32_t)(s->philox_seed >> 32);
                r.ctr[0] = (uint32_t)i; r.ctr[1] = (uint32_t)s->step; r.ctr[2] = (uint32_t)sid;
            }
            ora_collide_stats cs;
            int rc;
            if (c->vdim == 3) {
                double v[3] = {st->v[i], st->vy[i], st->vz[i]};
                rc = ora_collide3(&s->col[m], v, c->dt, &r, &cs);
                st->v[i] = v[0]; st->vy[i] = v[1]; st->vz[i] = v[2];
            } else {
                rc = ora_collide1(&s->col[m], &st->v[i], c->dt, &r, &cs);
            }
            if (rc) return rc;
            s->candidates += cs.candidates;
            s->nulls += cs.null_collisions;
            for (int ch = 0; ch < c->models[m].nch; ++ch) s->per_channel[m][ch] += cs.channel_collisions[ch];
            for (int k = 0; k < cs.nsecondaries && k < 16; ++k) {
                const ora_channel* ch = &c->models[m].ch[cs.secondary_channel[k]];
                stage_product(s, ch->secondary_species, st->x[i], cs.secondary_velocity[k]);
                stage_product(s, ch->ion_species, st->x[i], cs.secondary_ion_velocity[k]);
            }
            if (cs.removed) return seterr(8, "1D MCC produced an unsupported primary removal event");
            if (s->diag.coll_active) {
                /* tracked_energy_change: the weighted projectile change, plus each
                 * product pair's energy in its channel, src/Simulation.cpp:862-923 */
                double tracked[ORA_MAX_CHANNELS];
                const double w = c->species[sid].weight;
                for (int ch = 0; ch < c->models[m].nch; ++ch) tracked[ch] = cs.energy_change[ch] * w;
                for (int k = 0; k < cs.nsecondaries && k < 16; ++k) {
                    const ora_channel* chp = &c->models[m].ch[cs.secondary_channel[k]];
                    const ora_species* A = &c->species[chp->secondary_species];
                    const ora_species* B = &c->species[chp->ion_species];
                    const double* vs = cs.secondary_velocity[k];
                    const double* vi = cs.secondary_ion_velocity[k];
                    tracked[cs.secondary_channel[k]] +=
                        0.5 * A->mass * A->weight * (vs[0] * vs[0] + vs[1] * vs[1] + vs[2] * vs[2]) +
                        0.5 * B->mass * B->weight * (vi[0] * vi[0] + vi[1] * vi[1] + vi[2] * vi[2]);
                }
                for (int ch = 0; ch < c->models[m].nch; ++ch)
                    if (tracked[ch] != 0.0) diag_collision_energy(s, st->x[i], s->diag.off[m] + ch, tracked[ch]);
            }
            st->vh[i] = init_half(st->v[i], gather(s, st->x[i]), qm, c->dt);
        }
    }
    /* capacity preflight, src/Simulation.cpp:929-965 */
    size_t need[ORA_MAX_SPECIES] = {0};
    for (size_t k = 0; k < s->nstaged; ++k) need[s->staged[k].species]++;
    for (int sid = 0; sid < c->nspecies; ++sid) {
        ora_store* st = &s->sp[sid];
        size_t dead = 0;
        for (size_t i = 0; i < st->n; ++i) dead += !st->alive[i];
        const size_t cap = c->max_particles ? c->max_particles : 10000000;
        if (need[sid] > cap - st->n + dead)
            return seterr(9, "reactive collisions exceeded max_particles_per_species");
    }
    /* append_product, src/Simulation.cpp:966-1005 */
    for (size_t k = 0; k < s->nstaged; ++k) {
        const ora_product* p = &s->staged[k];
        ora_store* st = &s->sp[p->species];
        size_t slot = st->n;
        if (s->mode == 0) {
            for (size_t i = 0; i < st->n; ++i)
                if (!st->alive[i]) { slot = i; break; }
        }
        if (slot == st->n) { store_reserve(st, st->n * 2 + 16); st->n++; }
        const double qm = c->species[p->species].charge / c->species[p->species].mass;
        st->x[slot] = p->x;
        st->v[slot] = p->v[0]; st->vy[slot] = p->v[1]; st->vz[slot] = p->v[2];
        st->alive[slot] = 1;
        st->vh[slot] = init_half(st->v[slot], gather(s, p->x), qm, c->dt);
    }
    return 0;
}

/* Simulation::step, src/Simulation.cpp:1008-1138 */
static int step_once(ora_sim1d* s) {
    const ora_config1d* c = &s->cfg;
    double work[ORA_MAX_SPECIES] = {0.0, 0.0, 0.0, 0.0}; /* one chunk per species: the serial runtime */
    for (int sid = 0; sid < c->nspecies; ++sid) {
        ora_store* st = &s->sp[sid];
        const double qm = c->species[sid].charge / c->species[sid].mass;
        const double mw = c->species[sid].mass * c->species[sid].weight;
        size_t out = 0;
        for (size_t i = 0; i < st->n; ++i) {
            if (!st->alive[i]) { if (s->mode == 0) continue; else continue; }
            /* kick_leapfrog + drift_leapfrog, src/Pusher.cpp:70-76 */
            st->vh[i] += qm * gather(s, st->x[i]) * c->dt;
            st->x[i] += st->vh[i] * c->dt;
            if (!c->dirichlet) {
                st->x[i] = wrap(st->x[i], c->length);
            } else if (st->x[i] < 0.0 || st->x[i] > c->length) {
                /* electric work of a wall crossing, src/Simulation.cpp:1047-1056 */
                const double hmw = 0.5 * c->species[sid].mass * c->species[sid].weight;
                work[sid] += hmw * st->vh[i] * st->vh[i] - hmw * st->v[i] * st->v[i];
                const double sp2 = st->vh[i] * st->vh[i] + st->vy[i] * st->vy[i] + st->vz[i] * st->vz[i];
                const double e = 0.5 * c->species[sid].mass * c->species[sid].weight * sp2;
                if (st->x[i] < 0.0) { st->lost_left++; st->e_left += e; }
                else { st->lost_right++; st->e_right += e; }
                st->alive[i] = 0;
            }
            (void)mw;
            if (s->mode == 2 && st->alive[i]) {
                st->vh[i] = f32_round(st->vh[i]);
                st->vy[i] = f32_round(st->vy[i]);
                st->vz[i] = f32_round(st->vz[i]);
            }
            if (s->mode != 0 && st->alive[i]) {
                /* device layout: survivors compacted in order */
                st->x[out] = st->x[i]; st->v[out] = st->v[i]; st->vh[out] = st->vh[i];
                st->vy[out] = st->vy[i]; st->vz[out] = st->vz[i]; st->alive[out] = 1;
                ++out;
            }
        }
        if (s->mode != 0) st->n = out;
    }
    deposit_and_solve(s, s->time + c->dt);
    for (int sid = 0; sid < c->nspecies; ++sid) {
        ora_store* st = &s->sp[sid];
        const double qm = c->species[sid].charge / c->species[sid].mass;
        for (size_t i = 0; i < st->n; ++i) {
            if (!st->alive[i]) continue;
            const double old_velocity = st->v[i];
            /* synchronize_leapfrog, src/Pusher.cpp:78-80 */
            st->v[i] = st->vh[i] + 0.5 * qm * gather(s, st->x[i]) * c->dt;
            /* the electric-work ledger, src/Simulation.cpp:1109-1114 */
            work[sid] += 0.5 * c->species[sid].mass * c->species[sid].weight *
                         (st->v[i] * st->v[i] - old_velocity * old_velocity);
        }
        s->electric_work[sid] += work[sid];
    }
    diag_begin_collision_step(s);
    const int rc = apply_collisions(s);
    if (rc) return rc;
    ++s->step;
    s->time += c->dt;
    diag_accumulate(s);
    return 0;
}

int ora_sim1d_step(ora_sim1d* s, size_t steps) {
    for (size_t i = 0; i < steps; ++i) {
        const int rc = step_once(s);
        if (rc) return rc;
    }
    return 0;
}

size_t ora_sim1d_count(const ora_sim1d* s, int species) { return s->sp[species].n; }

int ora_sim1d_get(const ora_sim1d* s, int species, double* x, double* v, double* vh,
                  double* vy, double* vz, uint8_t* alive) {
    const ora_store* st = &s->sp[species];
    for (size_t i = 0; i < st->n; ++i) {
        if (x) x[i] = st->x[i];
        if (v) v[i] = st->v[i];
        if (vh) vh[i] = st->vh[i];
        if (vy) vy[i] = st->vy[i];
        if (vz) vz[i] = st->vz[i];
        if (alive) alive[i] = st->alive[i];
    }
    return 0;
}

void ora_sim1d_fields(const ora_sim1d* s, double* rho, double* phi, double* E) {
    const size_t n = s->cfg.nx * sizeof(double);
    if (rho) memcpy(rho, s->rho, n);
    if (phi) memcpy(phi, s->phi, n);
    if (E) memcpy(E, s->E, n);
}

double ora_sim1d_time(const ora_sim1d* s) { return s->time; }

void ora_sim1d_set_mt(ora_sim1d* s, const uint64_t* state313) {
    for (int i = 0; i < 312; ++i) s->mt.mt[i] = state313[i];
    s->mt.mti = (int)state313[312];
}

double ora_sim1d_bgk_energy(const ora_sim1d* s) { return s->bgk_energy; }

void ora_sim1d_collisions(const ora_sim1d* s, uint64_t* candidates, uint64_t* nulls, uint64_t* per_channel) {
    *candidates = s->candidates;
    *nulls = s->nulls;
    if (per_channel) memcpy(per_channel, s->per_channel, sizeof s->per_channel);
}

void ora_sim1d_losses(const ora_sim1d* s, int species, uint64_t* left, uint64_t* right,
                      double* eleft, double* eright) {
    const ora_store* st = &s->sp[species];
    *left = st->lost_left; *right = st->lost_right; *eleft = st->e_left; *eright = st->e_right;
}

double ora_sim1d_electric_work(const ora_sim1d* s, int species) { return s->electric_work[species]; }

/* Species::kinetic_energy, src/Species.cpp:338-351 */
double ora_sim1d_kinetic(const ora_sim1d* s, int species) {
    const ora_store* st = &s->sp[species];
    const ora_species* sc = &s->cfg.species[species];
    double e = 0.0;
    for (size_t i = 0; i < st->n; ++i) {
        if (!st->alive[i]) continue;
        double sq = st->v[i] * st->v[i];
        if (s->cfg.vdim == 3) sq += st->vy[i] * st->vy[i] + st->vz[i] * st->vz[i];
        e += 0.5 * sc->mass * sc->weight * sq;
    }
    return e;
}

/* Simulation::sample field energy, src/Simulation.cpp:1149-1155 */
double ora_sim1d_field_energy(const ora_sim1d* s) {
    double fe = 0.0;
    for (size_t i = 0; i < s->cfg.nx; ++i)
        fe += 0.5 * s->eps * s->E[i] * s->E[i] * node_volume(i, s->cfg.nx, s->dx, s->cfg.dirichlet);
    return fe;
}

/* ======================================================================= */
/* Structured 2D3V / 3D3V periodic step: Mesh2D/Mesh3D deposit and gather,
 * Boris/leapfrog pushers, FFT spectral Poisson (Simulation2D::step,
 * src/Simulation2D.cpp:1337-1364; Simulation3D::step, src/Simulation3D.cpp:342-365). */

typedef struct { double re, im; } ora_cplx;

/* fft_radix2, src/FieldSolver.cpp:171-201: bit reversal, butterflies with the
 * twiddle recurrence w *= wlen, 1/n scaling of the inverse. */
static void fft_radix2(ora_cplx* a, size_t n, int inverse) {
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) { ora_cplx t = a[i]; a[i] = a[j]; a[j] = t; }
    }
    const double twopi = 2.0 * 3.14159265358979323846;
    for (size_t len = 2; len <= n; len <<= 1) {
        const double angle = (inverse ? 1.0 : -1.0) * twopi / (double)len;
        const double wr = cos(angle), wi = sin(angle);
        for (size_t i = 0; i < n; i += len) {
            double cr = 1.0, ci = 0.0;
            for (size_t j = 0; j < len / 2; ++j) {
                const ora_cplx u = a[i + j];
                const ora_cplx x = a[i + j + len / 2];
                /* complex<double> multiply: (x.re*cr - x.im*ci, x.re*ci + x.im*cr) */
                const ora_cplx v = {x.re * cr - x.im * ci, x.re * ci + x.im * cr};
                a[i + j].re = u.re + v.re; a[i + j].im = u.im + v.im;
                a[i + j + len / 2].re = u.re - v.re; a[i + j + len / 2].im = u.im - v.im;
                const double nr = cr * wr - ci * wi, ni = cr * wi + ci * wr;
                cr = nr; ci = ni;
            }
        }
    }
    if (inverse) {
        const double scale = 1.0 / (double)n;
        for (size_t i = 0; i < n; ++i) { a[i].re *= scale; a[i].im *= scale; }
    }
}

/* transform_2d / transform_3d, src/FieldSolver.cpp:216-265: lines along x, then y, then z */
static void transform_nd(ora_cplx* v, const size_t* n, int dims, int inverse) {
    const size_t nx = n[0], ny = n[1], nz = dims == 3 ? n[2] : 1;
    size_t mx = nx > ny ? nx : ny; if (nz > mx) mx = nz;
    ora_cplx* line = malloc(mx * sizeof(ora_cplx));
    for (size_t k = 0; k < nz; ++k)
        for (size_t j = 0; j < ny; ++j) {
            for (size_t i = 0; i < nx; ++i) line[i] = v[(k * ny + j) * nx + i];
            fft_radix2(line, nx, inverse);
            for (size_t i = 0; i < nx; ++i) v[(k * ny + j) * nx + i] = line[i];
        }
    for (size_t k = 0; k < nz; ++k)
        for (size_t i = 0; i < nx; ++i) {
            for (size_t j = 0; j < ny; ++j) line[j] = v[(k * ny + j) * nx + i];
            fft_radix2(line, ny, inverse);
            for (size_t j = 0; j < ny; ++j) v[(k * ny + j) * nx + i] = line[j];
        }
    if (dims == 3)
        for (size_t j = 0; j < ny; ++j)
            for (size_t i = 0; i < nx; ++i) {
                for (size_t k = 0; k < nz; ++k) line[k] = v[(k * ny + j) * nx + i];
                fft_radix2(line, nz, inverse);
                for (size_t k = 0; k < nz; ++k) v[(k * ny + j) * nx + i] = line[k];
            }
    free(line);
}

/* solve_periodic_spectral(Mesh2D&/Mesh3D&), src/FieldSolver.cpp:442-499, :659-731.
 * E holds dims components, each of N = prod(n) values. */
void ora_solve_nd(const double* rho, double* phi, double* E, int dims, const size_t* n, const double* L,
                  double eps) {
    const size_t nx = n[0], ny = n[1], nz = dims == 3 ? n[2] : 1;
    const size_t N = nx * ny * nz;
    const double twopi = 2.0 * 3.14159265358979323846;
    double mean = 0.0;
    for (size_t i = 0; i < N; ++i) mean += rho[i];
    mean /= (double)N;
    ora_cplx* rh = malloc(N * sizeof(ora_cplx));
    ora_cplx* out[4];
    for (int c = 0; c <= dims; ++c) out[c] = calloc(N, sizeof(ora_cplx));
    for (size_t i = 0; i < N; ++i) { rh[i].re = rho[i] - mean; rh[i].im = 0.0; }
    transform_nd(rh, n, dims, 0);
    for (size_t kz = 0; kz < nz; ++kz) {
        const double kzm = (kz <= nz / 2) ? (double)kz : -(double)(nz - kz);
        const double kzw = dims == 3 ? twopi * kzm / L[2] : 0.0;
        for (size_t ky = 0; ky < ny; ++ky) {
            const double kym = (ky <= ny / 2) ? (double)ky : -(double)(ny - ky);
            const double kyw = twopi * kym / L[1];
            for (size_t kx = 0; kx < nx; ++kx) {
                if (kx == 0 && ky == 0 && kz == 0) continue;
                const double kxm = (kx <= nx / 2) ? (double)kx : -(double)(nx - kx);
                const double kxw = twopi * kxm / L[0];
                const double k2 = dims == 3 ? kxw * kxw + kyw * kyw + kzw * kzw : kxw * kxw + kyw * kyw;
                const size_t idx = (kz * ny + ky) * nx + kx;
                const double den = eps * k2;
                const double pr = rh[idx].re / den, pi = rh[idx].im / den;
                out[0][idx].re = pr; out[0][idx].im = pi;
                /* -(0,1) * k * phik = (k * pi, -(k * pr)) */
                const double kw[3] = {kxw, kyw, kzw};
                for (int c = 0; c < dims; ++c) {
                    out[1 + c][idx].re = kw[c] * pi;
                    out[1 + c][idx].im = -(kw[c] * pr);
                }
            }
        }
    }
    for (int c = 0; c <= dims; ++c) transform_nd(out[c], n, dims, 1);
    for (size_t i = 0; i < N; ++i) {
        phi[i] = out[0][i].re;
        for (int c = 0; c < dims; ++c) E[c * N + i] = out[1 + c][i].re;
    }
    for (int c = 0; c <= dims; ++c) free(out[c]);
    free(rh);
}

/* solve_mixed_spectral_tridiagonal(Mesh2D&), src/FieldSolver.cpp:501-657, for a
 * power-of-two periodic extent (transform_1d is then fft_radix2), followed by
 * compute_electric_field(Mesh2D&), src/FieldSolver.cpp:298-346.  Mesh index
 * j * nx + i; periodic_axis 0: x periodic, walls along y (bottom = lower,
 * top = upper); 1: y periodic, walls along x (left = lower, right = upper).
 * E holds [2][nx * ny].  Returns nonzero for an unsupported shape. */
int ora_solve_mixed_2d(const double* rho, double* phi, double* E, const size_t* n, const double* L,
                       int periodic_axis, double eps, double lower, double upper) {
    const size_t nx = n[0], ny = n[1];
    const int periodic_y = periodic_axis == 1;
    const size_t nd = periodic_y ? nx : ny;  /* direct (wall) extent */
    const size_t np = periodic_y ? ny : nx;  /* periodic extent */
    if (nd < 3 || np < 2 || (np & (np - 1))) return seterr(1, "mixed solve needs a power-of-two periodic extent");
    /* Mesh2D spacings, src/Mesh2D.cpp:57-60 */
    const double dx = L[0] / (double)(periodic_y ? nx - 1 : nx);
    const double dy = L[1] / (double)(periodic_y ? ny : ny - 1);
    const double hd = periodic_y ? dx : dy, hp = periodic_y ? dy : dx;
    const double inv_dsq = 1.0 / (hd * hd), inv_psq = 1.0 / (hp * hp);
    const size_t ni = nd - 2;
#define MIDX(d, q) (periodic_y ? (q) * nx + (d) : (d) * nx + (q))
    ora_cplx* rho_hat = calloc(nd * np, sizeof(ora_cplx));
    ora_cplx* phi_hat = calloc(nd * np, sizeof(ora_cplx));
    ora_cplx* line = malloc(np * sizeof(ora_cplx));
    double* mu = calloc(ni, sizeof(double)); /* modified_upper: real for real coefficients */
    ora_cplx* mr = calloc(ni, sizeof(ora_cplx));
    for (size_t d = 0; d < nd; ++d) {
        for (size_t q = 0; q < np; ++q) { line[q].re = rho[MIDX(d, q)]; line[q].im = 0.0; }
        fft_radix2(line, np, 0);
        for (size_t m = 0; m < np; ++m) rho_hat[m * nd + d] = line[m];
    }
    const double off = -inv_dsq;
    const double bscale = (double)np;
    for (size_t m = 0; m < np; ++m) {
        const double angle = 3.14159265358979323846 * (double)m / (double)np;
        const double eig = 4.0 * sin(angle) * sin(angle) * inv_psq;
        const double diag = 2.0 * inv_dsq + eig;
        const double lb = m == 0 ? lower * bscale : 0.0, ub = m == 0 ? upper * bscale : 0.0;
        phi_hat[m * nd + 0].re = lb; phi_hat[m * nd + 0].im = 0.0;
        phi_hat[m * nd + nd - 1].re = ub; phi_hat[m * nd + nd - 1].im = 0.0;
        for (size_t k = 0; k < ni; ++k) {
            const ora_cplx rh = rho_hat[m * nd + k + 1];
            double rr = rh.re / eps, ri = rh.im / eps;
            if (k == 0) rr += inv_dsq * lb;  /* the boundary terms are real */
            if (k + 1 == ni) rr += inv_dsq * ub;
            if (k == 0) {
                mu[k] = off / diag;
                mr[k].re = rr / diag; mr[k].im = ri / diag;
            } else {
                const double den = diag - off * mu[k - 1];
                mu[k] = k + 1 == ni ? 0.0 : off / den;
                mr[k].re = (rr - off * mr[k - 1].re) / den;
                mr[k].im = (ri - off * mr[k - 1].im) / den;
            }
        }
        phi_hat[m * nd + nd - 2] = mr[ni - 1];
        for (size_t k = ni - 1; k-- > 0;) {
            const ora_cplx nxt = phi_hat[m * nd + k + 2];
            phi_hat[m * nd + k + 1].re = mr[k].re - mu[k] * nxt.re;
            phi_hat[m * nd + k + 1].im = mr[k].im - mu[k] * nxt.im;
        }
    }
    for (size_t d = 0; d < nd; ++d) {
        for (size_t m = 0; m < np; ++m) line[m] = phi_hat[m * nd + d];
        fft_radix2(line, np, 1);
        for (size_t q = 0; q < np; ++q) phi[MIDX(d, q)] = line[q].re;
    }
#undef MIDX
    /* compute_electric_field(Mesh2D&), src/FieldSolver.cpp:298-346 */
    const size_t N = nx * ny;
    for (size_t j = 0; j < ny; ++j)
        for (size_t i = 0; i < nx; ++i) {
            const size_t idx = j * nx + i;
            double ex, ey;
            if (!periodic_y) ex = -(phi[j * nx + (i + 1) % nx] - phi[j * nx + (i + nx - 1) % nx]) / (2.0 * dx);
            else if (i == 0) ex = -(phi[j * nx + 1] - phi[idx]) / dx;
            else if (i + 1 == nx) ex = -(phi[idx] - phi[j * nx + i - 1]) / dx;
            else ex = -(phi[j * nx + i + 1] - phi[j * nx + i - 1]) / (2.0 * dx);
            if (periodic_y) ey = -(phi[((j + 1) % ny) * nx + i] - phi[((j + ny - 1) % ny) * nx + i]) / (2.0 * dy);
            else if (j == 0) ey = -(phi[nx + i] - phi[idx]) / dy;
            else if (j + 1 == ny) ey = -(phi[idx] - phi[(j - 1) * nx + i]) / dy;
            else ey = -(phi[(j + 1) * nx + i] - phi[(j - 1) * nx + i]) / (2.0 * dy);
            E[idx] = ex;
            E[N + idx] = ey;
        }
    free(rho_hat); free(phi_hat); free(line); free(mu); free(mr);
    return 0;
}

/* solve_dirichlet_iterative(Mesh2D&) / (Mesh3D&), src/FieldSolver.cpp:761-907:
 * fixed wall potentials (2D: left, right, bottom, top, corners the mean of their
 * two sides, apply_dirichlet_boundary_potentials :267-296; 3D: grounded), then
 * lexicographic SOR (omega 1.7 in 2D, 1.65 in 3D) until the largest update is
 * below 1e-11, then E by differences (one-sided at the walls).  Mesh spacing
 * L / (n - 1).  E holds [dims][N].  Returns nonzero when SOR does not converge. */
static int solve_dirichlet_sor(const double* rho, double* phi, double* E, int dims, const size_t* n, const double* L,
                               double eps, const double* pot, int warm);

int ora_solve_dirichlet_nd(const double* rho, double* phi, double* E, int dims, const size_t* n, const double* L,
                           double eps, const double* pot) {
    return solve_dirichlet_sor(rho, phi, E, dims, n, L, eps, pot, 0);
}

/* The same solve started from the potential already in phi: inside a run the
 * mesh keeps its potential between steps, so the reference's SOR starts from
 * the previous step's solution. */
int ora_solve_dirichlet_nd_warm(const double* rho, double* phi, double* E, int dims, const size_t* n, const double* L,
                                double eps, const double* pot) {
    return solve_dirichlet_sor(rho, phi, E, dims, n, L, eps, pot, 1);
}

static int solve_dirichlet_sor(const double* rho, double* phi, double* E, int dims, const size_t* n, const double* L,
                               double eps, const double* pot, int warm) {
    const size_t nx = n[0], ny = n[1], nz = dims == 3 ? n[2] : 1;
    const double dx = L[0] / (double)(nx - 1), dy = L[1] / (double)(ny - 1);
    const double dz = dims == 3 ? L[2] / (double)(nz - 1) : 1.0;
    const size_t N = nx * ny * nz;
    if (!warm)
        for (size_t i = 0; i < N; ++i) phi[i] = 0.0;
    if (dims == 2) {
        const double left = pot ? pot[0] : 0.0, right = pot ? pot[1] : 0.0;
        const double bottom = pot ? pot[2] : 0.0, top = pot ? pot[3] : 0.0;
        for (size_t j = 0; j < ny; ++j) { phi[j * nx] = left; phi[j * nx + nx - 1] = right; }
        for (size_t i = 0; i < nx; ++i) { phi[i] = bottom; phi[(ny - 1) * nx + i] = top; }
        phi[0] = 0.5 * (left + bottom);
        phi[nx - 1] = 0.5 * (right + bottom);
        phi[(ny - 1) * nx] = 0.5 * (left + top);
        phi[(ny - 1) * nx + nx - 1] = 0.5 * (right + top);
    }
    const double idx2 = 1.0 / (dx * dx), idy2 = 1.0 / (dy * dy), idz2 = dims == 3 ? 1.0 / (dz * dz) : 0.0;
    const double diag = dims == 3 ? 2.0 * (idx2 + idy2 + idz2) : 2.0 * (idx2 + idy2);
    const double omega = dims == 3 ? 1.65 : 1.7;
    const size_t maxit = dims == 3 ? (50000 > 150 * N ? 50000 : 150 * N) : (20000 > 100 * N ? 20000 : 100 * N);
    int converged = 0;
    for (size_t it = 0; it < maxit && !converged; ++it) {
        double md = 0.0;
        for (size_t k = (dims == 3 ? 1 : 0); k + (dims == 3 ? 1 : 0) < nz; ++k)
            for (size_t j = 1; j + 1 < ny; ++j)
                for (size_t i = 1; i + 1 < nx; ++i) {
                    const size_t id = (k * ny + j) * nx + i;
                    const double rhs = rho[id] / eps;
                    double up;
                    if (dims == 2)
                        up = ((phi[id - 1] + phi[id + 1]) * idx2 + (phi[id - nx] + phi[id + nx]) * idy2 + rhs) / diag;
                    else
                        up = ((phi[id - 1] + phi[id + 1]) * idx2 + (phi[id - nx] + phi[id + nx]) * idy2 +
                              (phi[id - nx * ny] + phi[id + nx * ny]) * idz2 + rhs) / diag;
                    const double d = omega * (up - phi[id]);
                    phi[id] += d;
                    if (fabs(d) > md) md = fabs(d);
                }
        if (md < 1.0e-11) converged = 1;
    }
    if (!converged) return seterr(1, "Dirichlet Poisson solve did not converge");
    for (size_t k = 0; k < nz; ++k)
        for (size_t j = 0; j < ny; ++j)
            for (size_t i = 0; i < nx; ++i) {
                const size_t id = (k * ny + j) * nx + i;
                double ex, ey;
                if (i == 0) ex = -(phi[id + 1] - phi[id]) / dx;
                else if (i + 1 == nx) ex = -(phi[id] - phi[id - 1]) / dx;
                else ex = -(phi[id + 1] - phi[id - 1]) / (2.0 * dx);
                if (j == 0) ey = -(phi[id + nx] - phi[id]) / dy;
                else if (j + 1 == ny) ey = -(phi[id] - phi[id - nx]) / dy;
                else ey = -(phi[id + nx] - phi[id - nx]) / (2.0 * dy);
                E[id] = ex;
                E[N + id] = ey;
                if (dims == 3) {
                    double ez;
                    if (k == 0) ez = -(phi[id + nx * ny] - phi[id]) / dz;
                    else if (k + 1 == nz) ez = -(phi[id] - phi[id - nx * ny]) / dz;
                    else ez = -(phi[id + nx * ny] - phi[id - nx * ny]) / (2.0 * dz);
                    E[2 * N + id] = ez;
                }
            }
    return 0;
}

/* Periodic CIC stencil of one axis, src/Mesh2D.cpp:96-129, src/FieldSolver.cpp:936-960 */
static void cic_axis(double x, double L, double d, size_t n, size_t* i0, size_t* i1, double* f) {
    const double xp = wrap(x, L);
    const double g = xp / d;
    const size_t i = (size_t)floor(g);
    *f = g - (double)i;
    *i0 = i % n;
    *i1 = (i + 1) % n;
}

/* interpolate_electric(Mesh2D&) / (Mesh3D&), src/FieldSolver.cpp:926-1038 (periodic) */
void ora_gather_nd(const double* E, int dims, const size_t* n, const double* L, const double* pos,
                   double* out) {
    const size_t nx = n[0], ny = n[1], nz = dims == 3 ? n[2] : 1;
    const size_t N = nx * ny * nz;
    size_t ii[3][2];
    double f[3];
    for (int a = 0; a < dims; ++a)
        cic_axis(pos[a], L[a], L[a] / (double)n[a], n[a], &ii[a][0], &ii[a][1], &f[a]);
    if (dims == 2) {
        const double fx = f[0], fy = f[1];
        const double w00 = (1.0 - fx) * (1.0 - fy), w10 = fx * (1.0 - fy), w01 = (1.0 - fx) * fy, w11 = fx * fy;
        const size_t i00 = ii[1][0] * nx + ii[0][0], i10 = ii[1][0] * nx + ii[0][1];
        const size_t i01 = ii[1][1] * nx + ii[0][0], i11 = ii[1][1] * nx + ii[0][1];
        for (int c = 0; c < 2; ++c) {
            const double* e = E + c * N;
            out[c] = e[i00] * w00 + e[i10] * w10 + e[i01] * w01 + e[i11] * w11;
        }
        return;
    }
    const double wx[2] = {1.0 - f[0], f[0]}, wy[2] = {1.0 - f[1], f[1]}, wz[2] = {1.0 - f[2], f[2]};
    out[0] = out[1] = out[2] = 0.0;
    for (int c3 = 0; c3 < 2; ++c3)
        for (int b = 0; b < 2; ++b)
            for (int a = 0; a < 2; ++a) {
                const double shape = wx[a] * wy[b] * wz[c3];
                const size_t idx = (ii[2][c3] * ny + ii[1][b]) * nx + ii[0][a];
                for (int c = 0; c < 3; ++c) out[c] += E[c * N + idx] * shape;
            }
}

/* deposit_charge_cic(Mesh2D&) with q = charge * weight / depth, src/Mesh2D.cpp:90-144,
 * src/Species2D.cpp:160-170; deposit_charge_cic(Mesh3D&), src/Mesh3D.cpp:62-126 (periodic) */
void ora_deposit_nd(double* rho, int dims, const size_t* n, const double* L, double q, size_t np,
                    const double* pos /* dims x np */) {
    const size_t nx = n[0], ny = n[1];
    double d[3];
    for (int a = 0; a < dims; ++a) d[a] = L[a] / (double)n[a];
    const double area = d[0] * d[1];
    const double qv = dims == 3 ? q / (d[0] * d[1] * d[2]) : 0.0;
    for (size_t p = 0; p < np; ++p) {
        size_t ii[3][2];
        double f[3];
        for (int a = 0; a < dims; ++a) cic_axis(pos[a * np + p], L[a], d[a], n[a], &ii[a][0], &ii[a][1], &f[a]);
        if (dims == 2) {
            const double fx = f[0], fy = f[1];
            rho[ii[1][0] * nx + ii[0][0]] += q * (1.0 - fx) * (1.0 - fy) / area;
            rho[ii[1][0] * nx + ii[0][1]] += q * fx * (1.0 - fy) / area;
            rho[ii[1][1] * nx + ii[0][0]] += q * (1.0 - fx) * fy / area;
            rho[ii[1][1] * nx + ii[0][1]] += q * fx * fy / area;
        } else {
            const double wx[2] = {1.0 - f[0], f[0]}, wy[2] = {1.0 - f[1], f[1]}, wz[2] = {1.0 - f[2], f[2]};
            for (int c3 = 0; c3 < 2; ++c3)
                for (int b = 0; b < 2; ++b)
                    for (int a = 0; a < 2; ++a) {
                        const double shape = wx[a] * wy[b] * wz[c3];
                        rho[(ii[2][c3] * ny + ii[1][b]) * nx + ii[0][a]] += qv * shape;
                    }
        }
    }
}

/* boris_advance, src/Pusher.cpp:20-29 */
void ora_boris(double v[3], const double E[3], const double B[3], double qm, double dt) {
    const double h = 0.5 * qm * dt;
    const double vm[3] = {v[0] + h * E[0], v[1] + h * E[1], v[2] + h * E[2]};
    const double t[3] = {h * B[0], h * B[1], h * B[2]};
    const double t2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
    const double sf = 2.0 / (1.0 + t2);
    const double s[3] = {sf * t[0], sf * t[1], sf * t[2]};
    const double vp[3] = {vm[0] + (vm[1] * t[2] - vm[2] * t[1]), vm[1] + (vm[2] * t[0] - vm[0] * t[2]),
                          vm[2] + (vm[0] * t[1] - vm[1] * t[0])};
    const double vq[3] = {vm[0] + (vp[1] * s[2] - vp[2] * s[1]), vm[1] + (vp[2] * s[0] - vp[0] * s[2]),
                          vm[2] + (vp[0] * s[1] - vp[1] * s[0])};
    v[0] = vq[0] + h * E[0];
    v[1] = vq[1] + h * E[1];
    v[2] = vq[2] + h * E[2];
}

struct ora_simnd {
    int dims, nspecies, boris;
    /* magnetic_field_profile (TabulatedVectorField1D): rows > 0 replaces B */
    int prof_axis;
    size_t prof_rows;
    double *prof_c, *prof_v; /* rows, rows x 3 */
    size_t n[3];
    double L[3], d[3], dt, eps, B[3], q[ORA_MAX_SPECIES], m[ORA_MAX_SPECIES], w[ORA_MAX_SPECIES];
    size_t np[ORA_MAX_SPECIES];
    double *pos[ORA_MAX_SPECIES], *v[ORA_MAX_SPECIES], *vh[ORA_MAX_SPECIES]; /* [3][np] each */
    double *rho, *phi, *E;
    double time;
    /* walls: Dirichlet field axes, side potentials (2D) and particle boundaries
     * (left, right, bottom, top, back, front: 0 periodic, 1 absorbing, 2 reflecting) */
    int walls, dir[3], pbc[6];
    double pot[4];
    uint8_t* alive[ORA_MAX_SPECIES];
    uint64_t losses[ORA_MAX_SPECIES][6];
};

ora_simnd* ora_simnd_create(int dims, const size_t* n, const double* L, double dt, double eps, const double* B,
                            int nspecies, const double* q, const double* m, const double* w_eff) {
    ora_simnd* s = calloc(1, sizeof *s);
    s->dims = dims;
    s->nspecies = nspecies;
    size_t N = 1;
    for (int a = 0; a < 3; ++a) {
        s->n[a] = a < dims ? n[a] : 1;
        s->L[a] = a < dims ? L[a] : 1.0;
        s->d[a] = s->L[a] / (double)s->n[a];
        s->B[a] = B[a];
        N *= s->n[a];
    }
    s->boris = B[0] != 0.0 || B[1] != 0.0 || B[2] != 0.0;
    s->dt = dt;
    s->eps = eps;
    for (int k = 0; k < nspecies; ++k) { s->q[k] = q[k]; s->m[k] = m[k]; s->w[k] = w_eff[k]; }
    s->rho = calloc(N, sizeof(double));
    s->phi = calloc(N, sizeof(double));
    s->E = calloc(3 * N, sizeof(double));
    return s;
}

void ora_simnd_destroy(ora_simnd* s) {
    if (!s) return;
    free(s->prof_c); free(s->prof_v);
    for (int k = 0; k < ORA_MAX_SPECIES; ++k) { free(s->pos[k]); free(s->v[k]); free(s->vh[k]); free(s->alive[k]); }
    free(s->rho); free(s->phi); free(s->E); free(s);
}

/* arrays are [3][np] (component-major); for 2D the third position row is ignored */
void ora_simnd_load(ora_simnd* s, int k, size_t np, const double* pos, const double* v, const double* vh) {
    s->np[k] = np;
    free(s->pos[k]); free(s->v[k]); free(s->vh[k]);
    s->pos[k] = malloc(3 * np * sizeof(double));
    s->v[k] = malloc(3 * np * sizeof(double));
    s->vh[k] = malloc(3 * np * sizeof(double));
    memcpy(s->pos[k], pos, 3 * np * sizeof(double));
    memcpy(s->v[k], v, 3 * np * sizeof(double));
    memcpy(s->vh[k], vh, 3 * np * sizeof(double));
    free(s->alive[k]);
    s->alive[k] = malloc(np + 1);
    memset(s->alive[k], 1, np + 1);
}

/* Mesh2D with a boundary per axis (src/Mesh2D.cpp:51-88) and the 2D particle
 * boundaries (src/Simulation2D.cpp:38-97, :1309-1335). */
int ora_simnd_set_walls(ora_simnd* s, const int* dirichlet, const double* potentials, const int* particle) {
    if (s->dims != 2) return seterr(1, "walls are 2D only");
    s->walls = dirichlet[0] || dirichlet[1];
    for (int a = 0; a < 2; ++a) {
        s->dir[a] = dirichlet[a];
        s->d[a] = s->L[a] / (double)(dirichlet[a] ? s->n[a] - 1 : s->n[a]);
    }
    for (int k = 0; k < 4; ++k) { s->pot[k] = potentials[k]; s->pbc[k] = particle[k]; }
    return 0;
}

/* Mesh3D with Boundary::Dirichlet (grounded walls on every side, spacing
 * L / (n - 1), src/Mesh3D.cpp:37-60) and the 3D particle boundaries per side
 * (left, right, bottom, top, back, front; src/Simulation3D.cpp:25-97, :309-340). */
int ora_simnd_set_walls3d(ora_simnd* s, const int* particle) {
    if (s->dims != 3) return seterr(1, "3D walls need a 3D run");
    s->walls = 1;
    for (int a = 0; a < 3; ++a) {
        s->dir[a] = 1;
        s->d[a] = s->L[a] / (double)(s->n[a] - 1);
    }
    for (int k = 0; k < 4; ++k) s->pot[k] = 0.0;
    for (int k = 0; k < 6; ++k) s->pbc[k] = particle[k];
    return 0;
}

/* alive flags and the absorbed counts per side (2D: 4 sides, 3D: 6) of species k */
void ora_simnd_alive_losses(const ora_simnd* s, int k, uint8_t* alive, uint64_t* losses) {
    if (alive) for (size_t i = 0; i < s->np[k]; ++i) alive[i] = s->alive[k] ? s->alive[k][i] : 1;
    if (losses) for (int q = 0; q < 2 * s->dims; ++q) losses[q] = s->losses[k][q];
}

/* One axis of the 2D CIC stencil with a wall or a wrap, src/Mesh2D.cpp:96-129,
 * src/FieldSolver.cpp:926-960 */
static void wall_axis(const ora_simnd* s, int a, double x, size_t* i0, size_t* i1, double* f) {
    const size_t n = s->n[a];
    const double L = s->L[a];
    if (!s->dir[a]) {
        cic_axis(x, L, s->d[a], n, i0, i1, f);
        return;
    }
    const double c = x < 0.0 ? 0.0 : (L < x ? L : x);
    const double g = c / s->d[a];
    size_t i = (size_t)floor(g);
    if (i > n - 2) i = n - 2;
    double fr = g - (double)i;
    *f = fr < 0.0 ? 0.0 : (fr > 1.0 ? 1.0 : fr);
    *i0 = i;
    *i1 = i + 1;
}

/* Mesh2D::node_area, src/Mesh2D.cpp:77-88 */
static double wall_node_area(const ora_simnd* s, size_t i, size_t j) {
    const double wx = !s->dir[0] ? s->d[0] : ((i == 0 || i + 1 == s->n[0]) ? 0.5 * s->d[0] : s->d[0]);
    const double wy = !s->dir[1] ? s->d[1] : ((j == 0 || j + 1 == s->n[1]) ? 0.5 * s->d[1] : s->d[1]);
    return wx * wy;
}

/* Mesh3D::node_volume of a Dirichlet mesh, src/Mesh3D.cpp:52-60 */
static double wall_node_volume(const ora_simnd* s, size_t i, size_t j, size_t k) {
    const double wx = (i == 0 || i + 1 == s->n[0]) ? 0.5 * s->d[0] : s->d[0];
    const double wy = (j == 0 || j + 1 == s->n[1]) ? 0.5 * s->d[1] : s->d[1];
    const double wz = (k == 0 || k + 1 == s->n[2]) ? 0.5 * s->d[2] : s->d[2];
    return wx * wy * wz;
}

static void simnd_deposit_solve(ora_simnd* s) {
    const size_t N = s->n[0] * s->n[1] * s->n[2];
    memset(s->rho, 0, N * sizeof(double));
    if (s->walls && s->dims == 3) {
        /* deposit_charge_cic(Mesh3D&) on a Dirichlet mesh, src/Mesh3D.cpp:62-126:
         * clamped stencil, q shape / node_volume, loops z, y, x */
        const size_t nx = s->n[0], ny = s->n[1];
        for (int k = 0; k < s->nspecies; ++k) {
            const double q = s->q[k] * s->w[k];
            const size_t np = s->np[k];
            for (size_t p = 0; p < np; ++p) {
                if (!s->alive[k][p]) continue;
                size_t ii[2], jj[2], kk[2];
                double fx, fy, fz;
                wall_axis(s, 0, s->pos[k][p], &ii[0], &ii[1], &fx);
                wall_axis(s, 1, s->pos[k][np + p], &jj[0], &jj[1], &fy);
                wall_axis(s, 2, s->pos[k][2 * np + p], &kk[0], &kk[1], &fz);
                const double wx[2] = {1.0 - fx, fx}, wy[2] = {1.0 - fy, fy}, wz[2] = {1.0 - fz, fz};
                for (int c = 0; c < 2; ++c)
                    for (int b = 0; b < 2; ++b)
                        for (int a = 0; a < 2; ++a) {
                            const double shape = wx[a] * wy[b] * wz[c];
                            s->rho[(kk[c] * ny + jj[b]) * nx + ii[a]] +=
                                q * shape / wall_node_volume(s, ii[a], jj[b], kk[c]);
                        }
            }
        }
        /* FieldSolver::solve(Mesh3D&) -> solve_dirichlet_iterative, src/FieldSolver.cpp:399-405,
         * started from the previous step's potential */
        ora_solve_dirichlet_nd_warm(s->rho, s->phi, s->E, 3, s->n, s->L, s->eps, NULL);
        return;
    }
    if (s->walls) {
        /* deposit_charge_cic(Mesh2D&), src/Mesh2D.cpp:90-144 */
        const size_t nx = s->n[0];
        for (int k = 0; k < s->nspecies; ++k) {
            const double q = s->q[k] * s->w[k];
            const size_t np = s->np[k];
            for (size_t p = 0; p < np; ++p) {
                if (!s->alive[k][p]) continue;
                size_t i0, i1, j0, j1;
                double fx, fy;
                wall_axis(s, 0, s->pos[k][p], &i0, &i1, &fx);
                wall_axis(s, 1, s->pos[k][np + p], &j0, &j1, &fy);
                s->rho[j0 * nx + i0] += q * (1.0 - fx) * (1.0 - fy) / wall_node_area(s, i0, j0);
                s->rho[j0 * nx + i1] += q * fx * (1.0 - fy) / wall_node_area(s, i1, j0);
                s->rho[j1 * nx + i0] += q * (1.0 - fx) * fy / wall_node_area(s, i0, j1);
                s->rho[j1 * nx + i1] += q * fx * fy / wall_node_area(s, i1, j1);
            }
        }
        /* FieldSolver::solve(Mesh2D&), src/FieldSolver.cpp:389-397 */
        if (s->dir[0] && s->dir[1]) {
            ora_solve_dirichlet_nd_warm(s->rho, s->phi, s->E, 2, s->n, s->L, s->eps, s->pot);
        } else {
            const int periodic_axis = s->dir[0] ? 1 : 0;
            const double lo = periodic_axis == 1 ? s->pot[0] : s->pot[2];
            const double hi = periodic_axis == 1 ? s->pot[1] : s->pot[3];
            ora_solve_mixed_2d(s->rho, s->phi, s->E, s->n, s->L, periodic_axis, s->eps, lo, hi);
        }
        return;
    }
    for (int k = 0; k < s->nspecies; ++k)
        ora_deposit_nd(s->rho, s->dims, s->n, s->L, s->q[k] * s->w[k], s->np[k], s->pos[k]);
    ora_solve_nd(s->rho, s->phi, s->E, s->dims, s->n, s->L, s->eps);
}

static void simnd_gather(const ora_simnd* s, const double* pos, size_t np, size_t i, double e[3]) {
    double p[3] = {pos[i], pos[np + i], s->dims == 3 ? pos[2 * np + i] : 0.0};
    e[2] = 0.0;
    if (s->walls && s->dims == 3) {
        /* interpolate_electric(Mesh3D&) on a Dirichlet mesh, src/FieldSolver.cpp:978-1038 */
        const size_t nx = s->n[0], ny = s->n[1], N = s->n[0] * s->n[1] * s->n[2];
        size_t ii[2], jj[2], kk[2];
        double fx, fy, fz;
        wall_axis(s, 0, p[0], &ii[0], &ii[1], &fx);
        wall_axis(s, 1, p[1], &jj[0], &jj[1], &fy);
        wall_axis(s, 2, p[2], &kk[0], &kk[1], &fz);
        const double wx[2] = {1.0 - fx, fx}, wy[2] = {1.0 - fy, fy}, wz[2] = {1.0 - fz, fz};
        e[0] = e[1] = e[2] = 0.0;
        for (int c = 0; c < 2; ++c)
            for (int b = 0; b < 2; ++b)
                for (int a = 0; a < 2; ++a) {
                    const double shape = wx[a] * wy[b] * wz[c];
                    const size_t id = (kk[c] * ny + jj[b]) * nx + ii[a];
                    e[0] += s->E[id] * shape;
                    e[1] += s->E[N + id] * shape;
                    e[2] += s->E[2 * N + id] * shape;
                }
        return;
    }
    if (s->walls) {
        /* interpolate_electric(Mesh2D&), src/FieldSolver.cpp:926-975 */
        const size_t nx = s->n[0], N = s->n[0] * s->n[1];
        size_t i0, i1, j0, j1;
        double fx, fy;
        wall_axis(s, 0, p[0], &i0, &i1, &fx);
        wall_axis(s, 1, p[1], &j0, &j1, &fy);
        const double w00 = (1.0 - fx) * (1.0 - fy), w10 = fx * (1.0 - fy), w01 = (1.0 - fx) * fy, w11 = fx * fy;
        for (int c = 0; c < 2; ++c) {
            const double* E = s->E + c * N;
            e[c] = E[j0 * nx + i0] * w00 + E[j0 * nx + i1] * w10 + E[j1 * nx + i0] * w01 + E[j1 * nx + i1] * w11;
        }
        return;
    }
    ora_gather_nd(s->E, s->dims, s->n, s->L, p, e);
}

void ora_simnd_initialize_fields(ora_simnd* s) { simnd_deposit_solve(s); }

/* magnetic_field_profile: B(position) = TabulatedVectorField1D::evaluate,
 * src/PrescribedField.cpp:89-113 (piecewise linear along one axis; the query
 * is the particle position, z = 0 in 2D). */
int ora_simnd_set_profile(ora_simnd* s, int axis, size_t rows, const double* coords, const double* values) {
    if (rows < 2 || axis < 0 || axis > 2) return seterr(1, "tabulated vector field requires at least two rows");
    free(s->prof_c); free(s->prof_v);
    s->prof_c = malloc(rows * sizeof(double));
    s->prof_v = malloc(3 * rows * sizeof(double));
    memcpy(s->prof_c, coords, rows * sizeof(double));
    memcpy(s->prof_v, values, 3 * rows * sizeof(double));
    s->prof_axis = axis;
    s->prof_rows = rows;
    s->boris = 1;
    return 0;
}

static void simnd_b(const ora_simnd* s, const double* pos, size_t np, size_t i, double B[3]) {
    if (!s->prof_rows) { B[0] = s->B[0]; B[1] = s->B[1]; B[2] = s->B[2]; return; }
    const double q = s->prof_axis < s->dims ? pos[s->prof_axis * np + i] : 0.0;
    const double* c = s->prof_c;
    const size_t n = s->prof_rows;
    if (q == c[0]) { for (int a = 0; a < 3; ++a) B[a] = s->prof_v[a]; return; }
    if (q == c[n - 1]) { for (int a = 0; a < 3; ++a) B[a] = s->prof_v[3 * (n - 1) + a]; return; }
    size_t lo = 0, hi = n; /* upper_bound */
    while (lo < hi) { const size_t mid = (lo + hi) / 2; if (q < c[mid]) hi = mid; else lo = mid + 1; }
    const size_t right = lo, left = right - 1;
    const double f = (q - c[left]) / (c[right] - c[left]);
    for (int a = 0; a < 3; ++a) {
        const double l = s->prof_v[3 * left + a], r = s->prof_v[3 * right + a];
        B[a] = l + f * (r - l);
    }
}

/* initialize(): deposit_and_solve + initialize_{boris,leapfrog}_half_step */
void ora_simnd_initialize(ora_simnd* s) {
    simnd_deposit_solve(s);
    for (int k = 0; k < s->nspecies; ++k) {
        const double qm = s->q[k] / s->m[k];
        const size_t np = s->np[k];
        for (size_t i = 0; i < np; ++i) {
            if (s->alive[k] && !s->alive[k][i]) continue;
            double e[3];
            simnd_gather(s, s->pos[k], np, i, e);
            double v[3] = {s->v[k][i], s->v[k][np + i], s->v[k][2 * np + i]};
            if (s->boris) {
                double B[3];
                simnd_b(s, s->pos[k], np, i, B);
                ora_boris(v, e, B, qm, -0.5 * s->dt);
            } else {
                for (int a = 0; a < s->dims; ++a) v[a] = v[a] - 0.5 * qm * e[a] * s->dt;
            }
            for (int a = 0; a < 3; ++a) s->vh[k][a * np + i] = v[a];
        }
    }
}

/* apply_lower/upper_boundary with periodic particle boundaries, src/Simulation2D.cpp:57-97 */
static double wrap_if_outside(double c, double L) { return (c >= 0.0 && c <= L) ? c : wrap(c, L); }

/* reflect_coordinate, src/Simulation2D.cpp:43-54 */
static void reflect_coordinate(double* c, double* v, double L) {
    while (*c < 0.0 || *c > L) {
        if (*c < 0.0) { *c = -*c; *v = -*v; }
        else { *c = 2.0 * L - *c; *v = -*v; }
    }
}

/* Simulation2D::apply_particle_boundaries, src/Simulation2D.cpp:1309-1335, and
 * Simulation3D::apply_particle_boundaries, src/Simulation3D.cpp:309-340: sides
 * in the order left, right, bottom, top (, back, front); returns 0 when the
 * particle is absorbed */
static int apply_walls(ora_simnd* s, int k, double* x, double* v) {
    for (int side = 0; side < 2 * s->dims; ++side) {
        const int a = side >> 1, lower = (side & 1) == 0;
        const double L = s->L[a];
        if (lower ? x[a] >= 0.0 : x[a] <= L) continue;
        if (s->pbc[side] == 1) { s->losses[k][side]++; return 0; }
        if (s->pbc[side] == 2) reflect_coordinate(&x[a], &v[a], L);
        else x[a] = wrap(x[a], L);
    }
    return 1;
}

void ora_simnd_step(ora_simnd* s, size_t steps) {
    for (size_t it = 0; it < steps; ++it) {
        for (int k = 0; k < s->nspecies; ++k) {
            const double qm = s->q[k] / s->m[k];
            const size_t np = s->np[k];
            for (size_t i = 0; i < np; ++i) {
                if (s->alive[k] && !s->alive[k][i]) continue;
                double e[3];
                simnd_gather(s, s->pos[k], np, i, e);
                double v[3] = {s->vh[k][i], s->vh[k][np + i], s->vh[k][2 * np + i]};
                double B[3];
                if (s->boris) simnd_b(s, s->pos[k], np, i, B);
                if (s->boris) ora_boris(v, e, B, qm, s->dt);
                else for (int a = 0; a < s->dims; ++a) v[a] += qm * e[a] * s->dt;
                if (s->walls) {
                    double x[3];
                    for (int a = 0; a < s->dims; ++a) x[a] = s->pos[k][a * np + i] + v[a] * s->dt;
                    if (!apply_walls(s, k, x, v)) s->alive[k][i] = 0;
                    for (int a = 0; a < s->dims; ++a) s->pos[k][a * np + i] = x[a];
                    for (int a = 0; a < 3; ++a) s->vh[k][a * np + i] = v[a];
                    continue;
                }
                for (int a = 0; a < 3; ++a) s->vh[k][a * np + i] = v[a];
                for (int a = 0; a < s->dims; ++a) {
                    double c = s->pos[k][a * np + i] + v[a] * s->dt;
                    s->pos[k][a * np + i] = wrap_if_outside(c, s->L[a]);
                }
            }
        }
        simnd_deposit_solve(s);
        for (int k = 0; k < s->nspecies; ++k) {
            const double qm = s->q[k] / s->m[k];
            const size_t np = s->np[k];
            for (size_t i = 0; i < np; ++i) {
                if (s->alive[k] && !s->alive[k][i]) continue;
                double e[3];
                simnd_gather(s, s->pos[k], np, i, e);
                double v[3] = {s->vh[k][i], s->vh[k][np + i], s->vh[k][2 * np + i]};
                double B[3];
                if (s->boris) simnd_b(s, s->pos[k], np, i, B);
                if (s->boris) ora_boris(v, e, B, qm, 0.5 * s->dt);
                else for (int a = 0; a < s->dims; ++a) v[a] = v[a] + 0.5 * qm * e[a] * s->dt;
                for (int a = 0; a < 3; ++a) s->v[k][a * np + i] = v[a];
            }
        }
        s->time += s->dt;
    }
}

void ora_simnd_get(const ora_simnd* s, int k, double* pos, double* v, double* vh) {
    const size_t np = s->np[k];
    if (pos) memcpy(pos, s->pos[k], 3 * np * sizeof(double));
    if (v) memcpy(v, s->v[k], 3 * np * sizeof(double));
    if (vh) memcpy(vh, s->vh[k], 3 * np * sizeof(double));
}

void ora_simnd_fields(const ora_simnd* s, double* rho, double* phi, double* E) {
    const size_t N = s->n[0] * s->n[1] * s->n[2];
    if (rho) memcpy(rho, s->rho, N * sizeof(double));
    if (phi) memcpy(phi, s->phi, N * sizeof(double));
    if (E) memcpy(E, s->E, 3 * N * sizeof(double));
}

/* ======================================================================== */
/* Homogeneous electron swarm (src/Swarm.cpp)                               */
/* ======================================================================== */

static const double kSwarmElectronMass = 9.1093837139e-31; /* src/Swarm.cpp:23 */
static const double kSwarmEvToJ = 1.602176634e-19;         /* src/Swarm.cpp:24-25 */
static const double kSwarmTownsend = 1.0e-21;              /* src/Swarm.cpp:26 */
static const size_t kSwarmAllocationLimit = 10000000;      /* src/Swarm.cpp:27 */

/* kinetic_energy_ev, src/Swarm.cpp:95-101 */
static double swarm_ke_ev(const double v[3]) {
    const double s2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    return 0.5 * kSwarmElectronMass * s2 / kSwarmEvToJ;
}

int ora_block_mean_and_error(const double* x, size_t n, size_t blocks, double* mean, double* se) {
    if (n == 0 || blocks == 0 || blocks > n)
        return seterr(4, "swarm block statistics require at least one sample per block");
    double* means = (double*)malloc(blocks * sizeof(double));
    for (size_t b = 0; b < blocks; ++b) {
        const size_t begin = b * n / blocks, end = (b + 1) * n / blocks;
        double total = 0.0;
        for (size_t i = begin; i < end; ++i) total += x[i];
        means[b] = total / (double)(end - begin);
    }
    double m = 0.0;
    for (size_t b = 0; b < blocks; ++b) m += means[b];
    m /= (double)blocks;
    double e = 0.0;
    if (blocks > 1) {
        double sq = 0.0;
        for (size_t b = 0; b < blocks; ++b) {
            const double d = means[b] - m;
            sq += d * d;
        }
        e = sqrt(sq / ((double)blocks * (double)(blocks - 1)));
    }
    free(means);
    *mean = m;
    *se = e;
    return 0;
}

/* linear_slope, src/Swarm.cpp:136-163 */
static double swarm_linear_slope(const double* v, size_t begin, size_t end, double timestep) {
    const size_t count = end - begin;
    const double mean_index = 0.5 * (double)(count - 1);
    double covariance = 0.0, index_variance = 0.0, mean_value = 0.0;
    for (size_t i = begin; i < end; ++i) mean_value += v[i];
    mean_value /= (double)count;
    for (size_t l = 0; l < count; ++l) {
        const double ci = (double)l - mean_index;
        covariance += ci * (v[begin + l] - mean_value);
        index_variance += ci * ci;
    }
    return covariance / (index_variance * timestep);
}

int ora_block_slope_and_error(const double* x, size_t n, double timestep, size_t blocks, double* slope,
                              double* se) {
    if (blocks == 0 || n % blocks != 0 || n / blocks < 2)
        return seterr(4, "swarm growth statistics require at least two samples per equal block");
    const size_t bs = n / blocks;
    double* slopes = (double*)malloc(blocks * sizeof(double));
    for (size_t b = 0; b < blocks; ++b) slopes[b] = swarm_linear_slope(x, b * bs, (b + 1) * bs, timestep);
    double m = 0.0;
    for (size_t b = 0; b < blocks; ++b) m += slopes[b];
    m /= (double)blocks;
    double e = 0.0;
    if (blocks > 1) {
        double sq = 0.0;
        for (size_t b = 0; b < blocks; ++b) {
            const double d = slopes[b] - m;
            sq += d * d;
        }
        e = sqrt(sq / ((double)blocks * (double)(blocks - 1)));
    }
    free(slopes);
    *slope = m;
    *se = e;
    return 0;
}

size_t ora_swarm_population_limit(const ora_swarm_config* cfg) {
    if (cfg->population_limit != 0) return cfg->population_limit;
    if (cfg->particles >= kSwarmAllocationLimit) return cfg->particles;
    const size_t source = kSwarmAllocationLimit - cfg->particles;
    const size_t doubled = cfg->particles > source / 2 ? source : 2 * cfg->particles;
    const size_t buffer = source < 1024 ? source : 1024;
    const size_t buffered = cfg->particles > source - buffer ? source : cfg->particles + 1024;
    const size_t mx = doubled > buffered ? doubled : buffered;
    return source < mx ? source : mx;
}

/* One electron of the ensemble.  Mode 0 keeps the reference's SwarmParticle
 * (src/Swarm.cpp:559-565: absolute position and sampling start); modes 1-2
 * keep the displacement since the sampling start in pos[] and no start. */
typedef struct {
    double v[3], pos[3], start[3], w;
    int alive;
} swarm_particle;

static void swarm_round_float(swarm_particle* p) {
    for (int d = 0; d < 3; ++d) {
        p->v[d] = (double)(float)p->v[d];
        p->pos[d] = (double)(float)p->pos[d];
    }
}

static void swarm_philox(ora_rng* r, uint64_t seed, uint32_t slot, uint32_t step, uint32_t stream) {
    memset(r, 0, sizeof *r);
    r->kind = ORA_SRC_PHILOX;
    r->key[0] = (uint32_t)seed;
    r->key[1] = (uint32_t)(seed >> 32);
    r->ctr[0] = slot;
    r->ctr[1] = step;
    r->ctr[2] = stream;
}

int ora_swarm_run_field(const ora_swarm_config* cfg, const ora_mcc_model* gas, double td, uint64_t seed, int mode,
                        ora_swarm_result* out, double* samples) {
    memset(out, 0, sizeof *out);
    /* collision_config, src/Swarm.cpp:520-557 */
    ora_mcc_model model = *gas;
    model.neutral_density = cfg->neutral_density;
    model.max_frequency = cfg->max_frequency;
    model.neutral_temperature = cfg->neutral_temperature;
    model.si = 1;
    if (model.max_candidates == 0) model.max_candidates = 64;
    ora_collider col;
    if (ora_collider_init(&col, &model, kSwarmElectronMass)) return 4;
    if (cfg->steps == 0 || cfg->burn_in_steps >= cfg->steps || cfg->particles == 0)
        return seterr(4, "invalid swarm steps or particles");

    const size_t N = cfg->particles;
    const size_t limit = ora_swarm_population_limit(cfg);
    const size_t cap = cfg->branching ? limit : N;
    swarm_particle* P = (swarm_particle*)calloc(cap, sizeof *P);
    swarm_particle* R = cfg->branching ? (swarm_particle*)calloc(N, sizeof *R) : NULL;
    const size_t ns = cfg->steps - cfg->burn_in_steps;
    double* vs = (double*)malloc(ns * sizeof(double));
    double* es = (double*)malloc(ns * sizeof(double));
    double* ls = (double*)malloc(ns * sizeof(double));
    int rc = 0;

    ora_mt64 mt;
    ora_mt64_seed(&mt, seed);
    ora_rng shared;
    memset(&shared, 0, sizeof shared);
    shared.kind = ORA_SRC_MT64;
    shared.mt = &mt;

    const double sd = sqrt(2.0 * cfg->initial_mean_energy_ev * kSwarmEvToJ / (3.0 * kSwarmElectronMass));
    ora_normal nst = {0, 0.0};
    for (size_t i = 0; i < N; ++i) {
        P[i].w = 1.0;
        P[i].alive = 1;
        if (mode == 0) {
            for (int d = 0; d < 3; ++d) P[i].v[d] = ora_normal_draw(&nst, &shared, 0.0, sd);
        } else {
            ora_rng r;
            swarm_philox(&r, seed, (uint32_t)i, 0xFFFFFFFFu, 2u);
            ora_normal pn = {0, 0.0};
            for (int d = 0; d < 3; ++d) P[i].v[d] = ora_normal_draw(&pn, &r, 0.0, sd);
            if (mode == 2) swarm_round_float(&P[i]);
        }
    }
    size_t M = N;
    double w = 1.0; /* modes 1-2: the one weight of every electron */

    const double E = td * kSwarmTownsend * cfg->neutral_density;
    const double acceleration = -kSwarmEvToJ * E / kSwarmElectronMass;
    const double half_kick = 0.5 * acceleration * cfg->timestep;
    out->reduced_field_td = td;
    out->electric_field_v_m = E;
    out->initial_weight = (double)N;
    out->diffusion_available = !cfg->branching;
    out->nch = model.nch;
    double wcoll[ORA_MAX_CHANNELS] = {0}, wcoll2[ORA_MAX_CHANNELS] = {0};
    double exposure = 0.0;
    size_t si = 0;

    for (size_t step = 0; step < cfg->steps && !rc; ++step) {
        if (mode == 0 && step == cfg->burn_in_steps)
            for (size_t i = 0; i < M; ++i) memcpy(P[i].start, P[i].pos, sizeof P[i].pos);
        const size_t active = M;
        double start_weight;
        if (mode == 0) {
            start_weight = 0.0;
            for (size_t i = 0; i < M; ++i) if (P[i].alive) start_weight += P[i].w;
        } else {
            start_weight = (double)M * w;
        }
        if (step >= cfg->burn_in_steps) exposure += start_weight * cfg->timestep;
        uint64_t step_counts[ORA_MAX_CHANNELS] = {0};
        for (size_t i = 0; i < active && !rc; ++i) {
            swarm_particle* p = &P[i];
            p->v[0] += half_kick;
            const double pre = swarm_ke_ev(p->v);
            if (pre > out->max_observed_energy_ev) out->max_observed_energy_ev = pre;
            if (pre > cfg->max_energy_ev) {
                rc = seterr(7, "swarm particle energy exceeded max_energy_ev before collision lookup");
                break;
            }
            if (mode == 0 || step >= cfg->burn_in_steps)
                for (int d = 0; d < 3; ++d) p->pos[d] += p->v[d] * cfg->timestep;
            ora_rng r;
            if (mode == 0) r = shared;
            else swarm_philox(&r, seed, (uint32_t)i, (uint32_t)step, 0u);
            ora_collide_stats st;
            const int crc = ora_collide3(&col, p->v, cfg->timestep, &r, &st);
            if (mode == 0) shared.index = r.index;
            if (crc) { rc = crc; break; }
            p->v[0] += half_kick;
            const double e = swarm_ke_ev(p->v);
            if (e > out->max_observed_energy_ev) out->max_observed_energy_ev = e;
            if (e > cfg->max_energy_ev) {
                rc = seterr(7, "swarm particle energy exceeded max_energy_ev");
                break;
            }
            if (step >= cfg->burn_in_steps) {
                out->candidates += st.candidates;
                out->null_collisions += st.null_collisions;
                for (int c = 0; c < model.nch; ++c) {
                    out->channel_collisions[c] += st.channel_collisions[c];
                    if (mode == 0) {
                        wcoll[c] += p->w * (double)st.channel_collisions[c];
                        wcoll2[c] += p->w * p->w * (double)st.channel_collisions[c];
                    } else {
                        step_counts[c] += st.channel_collisions[c];
                    }
                }
            }
            if (mode == 2) swarm_round_float(p);
            if (cfg->branching) {
                if (st.nsecondaries > 16) { rc = seterr(8, "more than 16 secondaries in one step"); break; }
                for (int k = 0; k < st.nsecondaries; ++k) {
                    if (M >= limit) {
                        rc = seterr(9, "branching swarm exceeded population_limit before resampling");
                        break;
                    }
                    swarm_particle* q = &P[M++];
                    *q = P[i];
                    q->alive = 1;
                    memcpy(q->v, st.secondary_velocity[k], sizeof q->v);
                    if (mode == 2) swarm_round_float(q);
                }
                if (st.removed) P[i].alive = 0;
            }
        }
        if (rc) break;
        if (mode != 0 && step >= cfg->burn_in_steps)
            for (int c = 0; c < model.nch; ++c) {
                wcoll[c] += w * (double)step_counts[c];
                wcoll2[c] += w * w * (double)step_counts[c];
            }
        if (cfg->branching) {
            size_t k = 0; /* erase_if, stable */
            for (size_t i = 0; i < M; ++i) if (P[i].alive) P[k++] = P[i];
            M = k;
            if (M == 0) { rc = seterr(10, "branching swarm electron ensemble became extinct"); break; }
            if (M != N) {
                /* systematic_resample, src/Swarm.cpp:616-643 */
                if (mode == 0) {
                    double ws = 0.0;
                    for (size_t i = 0; i < M; ++i) ws += P[i].w;
                    const double ow = ws / (double)N;
                    const double offset = ora_uniform01(&shared) * ow;
                    size_t src = 0;
                    double cumulative = P[0].w;
                    for (size_t s = 0; s < N; ++s) {
                        const double threshold = offset + (double)s * ow;
                        while (src + 1 < M && cumulative < threshold) {
                            ++src;
                            cumulative += P[src].w;
                        }
                        R[s] = P[src];
                        R[s].w = ow;
                    }
                } else {
                    /* every electron carries the weight w: the cumulative weight
                     * of the first j+1 is (j+1) w, so sample s takes source
                     * ceil((u + s) M / N) - 1 */
                    ora_rng r;
                    swarm_philox(&r, seed, 0xFFFFFFFFu, (uint32_t)step, 1u);
                    const double u = ora_uniform01(&r);
                    for (size_t s = 0; s < N; ++s) {
                        const double t = (u + (double)s) * (double)M / (double)N;
                        double c = ceil(t) - 1.0;
                        size_t j = c < 0.0 ? 0 : (size_t)c;
                        if (j > M - 1) j = M - 1;
                        R[s] = P[j];
                    }
                    w = (double)M * w / (double)N;
                }
                memcpy(P, R, N * sizeof *P);
                M = N;
            }
        }
        if (step < cfg->burn_in_steps) continue;
        double vsum = 0.0, esum = 0.0, wsum = 0.0;
        if (mode == 0) {
            for (size_t i = 0; i < M; ++i) wsum += P[i].w;
            for (size_t i = 0; i < M; ++i) {
                vsum += P[i].w * P[i].v[0];
                esum += P[i].w * swarm_ke_ev(P[i].v);
            }
            vs[si] = vsum / wsum;
            es[si] = esum / wsum;
            ls[si] = log(wsum);
        } else {
            for (size_t i = 0; i < M; ++i) {
                vsum += P[i].v[0];
                esum += swarm_ke_ev(P[i].v);
            }
            vs[si] = vsum / (double)M;
            es[si] = esum / (double)M;
            ls[si] = log((double)M * w);
        }
        ++si;
    }

    if (!rc) {
        double m, e;
        rc = ora_block_mean_and_error(vs, ns, cfg->uncertainty_blocks, &m, &e);
        out->mean_velocity_x = m;
        out->mean_velocity_x_se = e;
        out->drift_velocity = -m;
        out->reduced_mobility = E == 0.0 ? 0.0 : out->drift_velocity * cfg->neutral_density / E;
        if (!rc) rc = ora_block_mean_and_error(es, ns, cfg->uncertainty_blocks, &m, &e);
        out->mean_energy_ev = m;
        out->mean_energy_se_ev = e;
    }
    if (!rc) {
        const double sampling_time = (double)ns * cfg->timestep;
        if (out->diffusion_available) {
            double mx = 0.0, my = 0.0, mz = 0.0;
            const double count = (double)M;
            for (size_t i = 0; i < M; ++i) {
                const double* a = P[i].pos;
                const double* b = P[i].start; /* zero in modes 1-2 */
                mx += a[0] - b[0];
                my += a[1] - b[1];
                mz += a[2] - b[2];
            }
            mx /= count; my /= count; mz /= count;
            double vx = 0.0, vyz = 0.0;
            for (size_t i = 0; i < M; ++i) {
                const double* a = P[i].pos;
                const double* b = P[i].start;
                const double dx = a[0] - b[0] - mx, dy = a[1] - b[1] - my, dz = a[2] - b[2] - mz;
                vx += dx * dx;
                vyz += dy * dy + dz * dz;
            }
            vx /= count;
            vyz /= count;
            out->diffusion_longitudinal = vx / (2.0 * sampling_time);
            out->diffusion_transverse = vyz / (4.0 * sampling_time);
        }
        for (int c = 0; c < model.nch; ++c) {
            out->channel_rate[c] = wcoll[c] / exposure;
            out->channel_rate_se[c] = sqrt(wcoll2[c]) / exposure;
            if (model.ch[c].process == ORA_IONIZATION) {
                out->ionization_rate += out->channel_rate[c];
                out->ionization_rate_se = hypot(out->ionization_rate_se, out->channel_rate_se[c]);
            } else if (model.ch[c].process == ORA_ATTACHMENT) {
                out->attachment_rate += out->channel_rate[c];
                out->attachment_rate_se = hypot(out->attachment_rate_se, out->channel_rate_se[c]);
            }
        }
        out->net_rate = out->ionization_rate - out->attachment_rate;
        out->net_rate_se = hypot(out->ionization_rate_se, out->attachment_rate_se);
        if (mode == 0) {
            double ws = 0.0;
            for (size_t i = 0; i < M; ++i) ws += P[i].w;
            out->final_weight = ws;
        } else {
            out->final_weight = (double)M * w;
        }
        out->final_particles = M;
        if (cfg->branching) {
            double g, ge;
            rc = ora_block_slope_and_error(ls, ns, cfg->timestep, cfg->uncertainty_blocks, &g, &ge);
            out->growth_rate = g;
            out->growth_rate_se = ge;
            if (!rc && out->drift_velocity > 0.0) {
                const double drift = out->drift_velocity, de = out->mean_velocity_x_se;
                out->townsend_available = 1;
                out->townsend_growth = g / drift;
                out->townsend_growth_se = hypot(ge / drift, g * de / (drift * drift));
                out->townsend_rate = out->net_rate / drift;
                out->townsend_rate_se = hypot(out->net_rate_se / drift, out->net_rate * de / (drift * drift));
            }
        }
        if (samples)
            for (size_t i = 0; i < ns; ++i) {
                samples[i] = vs[i];
                samples[ns + i] = es[i];
                samples[2 * ns + i] = ls[i];
            }
    }
    free(P); free(R); free(vs); free(es); free(ls);
    return rc;
}

/* ---- spatial Townsend pass, src/Swarm.cpp:645-938 ------------------------- */

/* slope_r_squared, src/Swarm.cpp:202-231 */
static double swarm_slope_r_squared(const double* v, size_t begin, size_t end) {
    const size_t count = end - begin;
    double mean = 0.0;
    for (size_t i = begin; i < end; ++i) mean += v[i];
    mean /= (double)count;
    const double mean_index = 0.5 * (double)(count - 1);
    double covariance = 0.0, index_variance = 0.0, value_variance = 0.0;
    for (size_t l = 0; l < count; ++l) {
        const double ci = (double)l - mean_index;
        const double cv = v[begin + l] - mean;
        covariance += ci * cv;
        index_variance += ci * ci;
        value_variance += cv * cv;
    }
    if (value_variance == 0.0) return 1.0;
    double r = covariance * covariance / (index_variance * value_variance);
    return r < 0.0 ? 0.0 : (r > 1.0 ? 1.0 : r);
}

/* std::upper_bound over the plane positions */
static size_t swarm_upper_bound(const double* planes, size_t n, double value) {
    size_t lo = 0, hi = n;
    while (lo < hi) {
        const size_t mid = (lo + hi) / 2;
        if (value < planes[mid]) hi = mid; else lo = mid + 1;
    }
    return lo;
}

typedef struct {
    double v[3], pos[3], w;
    int alive;
} townsend_particle;

int ora_swarm_spatial_townsend(const ora_swarm_config* cfg, const ora_spatial_config* sp, const ora_mcc_model* gas,
                               double td, uint64_t seed, int mode, uint64_t* scan_updates, ora_spatial_result* out,
                               double* profile, double* history_crossings) {
    memset(out, 0, sizeof *out);
    if (sp->histories == 0) return 0;
    ora_mcc_model model = *gas; /* collision_config, src/Swarm.cpp:520-557 */
    model.neutral_density = cfg->neutral_density;
    model.max_frequency = cfg->max_frequency;
    model.neutral_temperature = cfg->neutral_temperature;
    model.si = 1;
    if (model.max_candidates == 0) model.max_candidates = 64;
    ora_collider col;
    if (ora_collider_init(&col, &model, kSwarmElectronMass)) return 4;

    ora_mt64 mt;
    ora_mt64_seed(&mt, seed ^ 0x9e3779b97f4a7c15ULL);
    ora_rng shared;
    memset(&shared, 0, sizeof shared);
    shared.kind = ORA_SRC_MT64;
    shared.mt = &mt;
    const double sd = sqrt(2.0 * cfg->initial_mean_energy_ev * kSwarmEvToJ / (3.0 * kSwarmElectronMass));
    ora_normal nst = {0, 0.0};
    const double E = td * kSwarmTownsend * cfg->neutral_density;
    const double acceleration = -kSwarmEvToJ * E / kSwarmElectronMass;
    const double half_kick = 0.5 * acceleration * cfg->timestep;
    const size_t bins = sp->bins, H = sp->histories, N = cfg->particles;
    const double spacing = sp->length_m / (double)(bins + 1);
    double* planes = (double*)malloc(bins * sizeof(double));
    for (size_t b = 0; b < bins; ++b) planes[b] = (double)(b + 1) * spacing;
    const size_t limit = ora_swarm_population_limit(cfg);
    const uint64_t work_limit = sp->work_item_limit ? sp->work_item_limit : 100000000ull;

    double* crossings = (double*)calloc(H * bins, sizeof(double));
    long long* net = (long long*)calloc(bins, sizeof(long long));
    townsend_particle* P = (townsend_particle*)calloc(limit + 1, sizeof *P);
    townsend_particle* R = (townsend_particle*)calloc(N + 1, sizeof *R);
    uint64_t updates = 0;
    size_t max_active = 0;
    int rc = 0;
    for (size_t h = 0; h < H && !rc; ++h) {
        double* row = crossings + h * bins;
        const uint32_t hs = 0x80000000u | (uint32_t)h;
        size_t M = 1;
        double w = 1.0; /* mode 1: the one weight of the history */
        memset(&P[0], 0, sizeof P[0]);
        P[0].w = 1.0;
        P[0].alive = 1;
        {
            ora_rng src;
            ora_rng* r = &shared;
            ora_normal pn = {0, 0.0};
            ora_normal* ns = &nst;
            if (mode != 0) {
                swarm_philox(&src, seed, 0xFFFFFFFEu, 0u, hs);
                r = &src;
                ns = &pn;
            }
            double unit = ora_canonical(r);
            if (unit < 2.2250738585072014e-308) unit = 2.2250738585072014e-308; /* max(u, DBL_MIN) */
            const double inward = sd * sqrt(-2.0 * log(unit));
            P[0].v[0] = -inward;
            P[0].v[1] = ora_normal_draw(ns, r, 0.0, sd);
            P[0].v[2] = ora_normal_draw(ns, r, 0.0, sd);
        }
        int terminated = 0;
        for (size_t step = 0; step < sp->max_steps; ++step) {
            if (M == 0) { terminated = 1; break; }
            const size_t active = M;
            if (active > max_active) max_active = active;
            if ((uint64_t)active > work_limit - *scan_updates) {
                rc = seterr(9, "spatial Townsend scan exceeded spatial_work_item_limit");
                break;
            }
            *scan_updates += active;
            updates += active;
            if (mode != 0) memset(net, 0, bins * sizeof(long long));
            for (size_t i = 0; i < active && !rc; ++i) {
                townsend_particle* p = &P[i];
                p->v[0] += half_kick;
                if (swarm_ke_ev(p->v) > cfg->max_energy_ev) {
                    rc = seterr(9, "spatial Townsend particle energy exceeded max_energy_ev before collision lookup");
                    break;
                }
                const double old_distance = -p->pos[0];
                p->pos[0] += p->v[0] * cfg->timestep;
                p->pos[1] += p->v[1] * cfg->timestep;
                p->pos[2] += p->v[2] * cfg->timestep;
                const double new_distance = -p->pos[0];
                if (new_distance > old_distance) {
                    const size_t a = swarm_upper_bound(planes, bins, old_distance);
                    const size_t b = swarm_upper_bound(planes, bins, new_distance);
                    for (size_t k = a; k < b; ++k) {
                        if (mode == 0) row[k] += p->w; else ++net[k];
                    }
                } else if (new_distance < old_distance) {
                    const size_t a = swarm_upper_bound(planes, bins, new_distance);
                    const size_t b = swarm_upper_bound(planes, bins, old_distance);
                    for (size_t k = a; k < b; ++k) {
                        if (mode == 0) row[k] -= p->w; else --net[k];
                    }
                }
                if (new_distance < 0.0 || new_distance >= sp->length_m) {
                    p->alive = 0;
                    continue;
                }
                ora_rng cr;
                ora_rng* r = &shared;
                if (mode != 0) {
                    swarm_philox(&cr, seed, (uint32_t)i, (uint32_t)step, hs);
                    r = &cr;
                }
                ora_collide_stats st;
                const int crc = ora_collide3(&col, p->v, cfg->timestep, r, &st);
                if (crc) { rc = crc; break; }
                p->v[0] += half_kick;
                if (swarm_ke_ev(p->v) > cfg->max_energy_ev) {
                    rc = seterr(9, "spatial Townsend particle energy exceeded max_energy_ev");
                    break;
                }
                for (int k = 0; k < st.nsecondaries && k < 16; ++k) {
                    if (M >= limit) {
                        rc = seterr(9, "spatial Townsend branching exceeded population_limit before resampling");
                        break;
                    }
                    townsend_particle* q = &P[M++];
                    p = &P[i];
                    memcpy(q->v, st.secondary_velocity[k], sizeof q->v);
                    memcpy(q->pos, p->pos, sizeof q->pos);
                    q->w = p->w;
                    q->alive = 1;
                }
                if (st.removed) P[i].alive = 0;
            }
            if (rc) break;
            if (mode != 0)
                for (size_t k = 0; k < bins; ++k)
                    if (net[k]) row[k] += w * (double)net[k];
            if (M > max_active) max_active = M;
            size_t kept = 0; /* erase_if, stable */
            for (size_t i = 0; i < M; ++i) if (P[i].alive) P[kept++] = P[i];
            M = kept;
            if (M > N) {
                /* systematic_resample, src/Swarm.cpp:616-643 */
                if (mode == 0) {
                    double ws = 0.0;
                    for (size_t i = 0; i < M; ++i) ws += P[i].w;
                    const double ow = ws / (double)N;
                    const double offset = ora_uniform01(&shared) * ow;
                    size_t src = 0;
                    double cumulative = P[0].w;
                    for (size_t s = 0; s < N; ++s) {
                        const double threshold = offset + (double)s * ow;
                        while (src + 1 < M && cumulative < threshold) {
                            ++src;
                            cumulative += P[src].w;
                        }
                        R[s] = P[src];
                        R[s].w = ow;
                    }
                } else {
                    ora_rng r;
                    swarm_philox(&r, seed, 0xFFFFFFFFu, (uint32_t)step, hs);
                    const double u = ora_uniform01(&r);
                    for (size_t s = 0; s < N; ++s) {
                        const double t = (u + (double)s) * (double)M / (double)N;
                        const double c = ceil(t) - 1.0;
                        size_t j = c < 0.0 ? 0 : (size_t)c;
                        if (j > M - 1) j = M - 1;
                        R[s] = P[j];
                    }
                    w = (double)M * w / (double)N;
                }
                memcpy(P, R, N * sizeof *P);
                M = N;
            }
        }
        if (rc) break;
        if (!terminated && M == 0) terminated = 1;
        if (!terminated) rc = seterr(9, "spatial Townsend history did not terminate within spatial_max_steps");
    }
    if (!rc) {
        double* logf = (double*)calloc(bins, sizeof(double));
        for (size_t b = 0; b < bins; ++b) {
            double sum = 0.0, sq = 0.0;
            for (size_t h = 0; h < H; ++h) {
                const double value = crossings[h * bins + b];
                sum += value;
                sq += value * value;
            }
            const double hist = (double)H;
            const double mean = sum / hist;
            double se = 0.0;
            if (H > 1) {
                const double centered = sq - sum * sum / hist;
                se = sqrt((centered > 0.0 ? centered : 0.0) / (hist * (hist - 1.0)));
            }
            profile[3 * b] = planes[b];
            profile[3 * b + 1] = mean;
            profile[3 * b + 2] = se;
            if (mean > 0.0) logf[b] = log(mean);
        }
        const size_t fb = sp->fit_begin_bin, fe = sp->fit_end_bin == 0 ? bins : sp->fit_end_bin;
        for (size_t b = fb; b < fe && !rc; ++b)
            if (!(profile[3 * b + 1] > 0.0))
                rc = seterr(9, "spatial Townsend fit requires positive net flux at every fit plane; increase "
                               "spatial_histories or adjust the fit range");
        const size_t blocks = cfg->uncertainty_blocks, hpb = H / blocks;
        double* slopes = (double*)calloc(blocks, sizeof(double));
        double* blog = (double*)calloc(bins, sizeof(double));
        for (size_t blk = 0; blk < blocks && !rc; ++blk) {
            for (size_t b = 0; b < bins && !rc; ++b) {
                double sum = 0.0;
                for (size_t l = 0; l < hpb; ++l) sum += crossings[(blk * hpb + l) * bins + b];
                const double flux = sum / (double)hpb;
                if (b >= fb && b < fe && !(flux > 0.0))
                    rc = seterr(9, "spatial Townsend uncertainty block has non-positive fit flux; increase "
                                   "spatial_histories");
                if (flux > 0.0) blog[b] = log(flux);
            }
            slopes[blk] = swarm_linear_slope(blog, fb, fe, spacing);
        }
        if (!rc) {
            double m = 0.0, se = 0.0;
            ora_block_mean_and_error(slopes, blocks, blocks, &m, &se);
            out->townsend_1_m = swarm_linear_slope(logf, fb, fe, spacing);
            out->townsend_se_1_m = se;
            out->fit_r_squared = swarm_slope_r_squared(logf, fb, fe);
            out->histories_completed = H;
            out->maximum_active_particles = max_active;
            out->particle_updates = updates;
            if (out->fit_r_squared < sp->min_r_squared)
                rc = seterr(9, "spatial Townsend log-flux fit did not meet spatial_min_r_squared");
        }
        free(slopes); free(blog); free(logf);
    }
    if (history_crossings) memcpy(history_crossings, crossings, H * bins * sizeof(double));
    free(planes); free(crossings); free(net); free(P); free(R);
    return rc;
}
