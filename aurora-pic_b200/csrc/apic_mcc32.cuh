// Null-collision Monte Carlo collisions in FP32 arithmetic (the FP32 particle
// form).
//
// collide3f() makes the decisions of NullCollisionModel::collide(Vec3&)
// (src/Collision.cpp:907-993) with single-precision arithmetic: exponential
// waiting times at the majorant, thermal neutral sampling (8-sigma bounded
// Maxwellian, src/Collision.cpp:702-715), channel selection against the
// cumulative rates (:596-625), the channel kinematics of apply_channel
// (:762-829: elastic recoil, threshold losses, ionization halving the
// remaining energy, backward and Henyey-Greenstein scattering, resonant charge
// exchange, attachment) and ionization secondaries.  Cross sections are the same tables,
// rounded to float, interpolated linearly in energy between the bracketing
// rows (CrossSectionTable::evaluate, :221-237) found through the FP64 form's
// log-energy bracket index.
//
// Random numbers come from the particle's Philox4x32-10 stream as 32-bit words
// (23-bit uniforms on (0, 1)); results agree with the FP64 form statistically,
// not draw for draw.  The energy ledger of each collision is formed in FP64
// from the float velocities before and after it.
#pragma once
#include "apic_mcc.cuh"

namespace apic {

constexpr float kFltEpsilon = 1.1920928955078125e-7f;

struct MccChannel32 {
    int process, angular, frame;
    float threshold;   // J (or normalized energy units)
    int secondary, ion;
    int rows;
    const float* energy;
    const float* sigma;
    const unsigned* first_gt;  // bracket index of the FP64 form (nbins + 1 entries), or null
    int nbins;
    float lmin, inv_width;
    int mu_rows;
    const float* mu_energy;
    const float* mu;
};

struct MccModel32 {
    int nch;
    int shared_grid;
    float particle_mass, neutral_mass, neutral_density, max_frequency, inv_max_frequency, neutral_stddev;
    float com_mass;
    float v_safe2;         // |v|^2 at or below which the frequency bound provably holds (< 0: never)
    float m_frac, n_frac;  // m / (m + M), M / (m + M) of the elastic recoil
    unsigned max_candidates;
    MccChannel32 ch[kMaxChannels];
};

// 32-bit words of a particle's Philox stream: block k of the FP64 form's
// stream (counter (k, slot, step, stream)) supplies four words.  The first
// 64-bit draw of the FP64 form (words 0 and 1 of block 0) decides the first
// waiting time of both forms.
struct Philox32 {
    uint32_t k0, k1, slot, step, stream;
    uint32_t block = 0;
    uint32_t buf[4];
    int used = 4;
    __device__ Philox32(uint64_t seed, uint32_t slot_, uint32_t step_, uint32_t stream_)
        : k0((uint32_t)seed), k1((uint32_t)(seed >> 32)), slot(slot_), step(step_), stream(stream_) {}
    __device__ uint32_t next() {
        if (used == 4) {
            philox4x32_10(block++, slot, step, stream, k0, k1, buf);
            used = 0;
        }
        return buf[used++];
    }
    // uniform on (0, 1): the word's top 23 bits, centred in their interval
    // (every value and the centre offset are exact in float)
    __device__ float uniform() { return ((float)(next() >> 9) + 0.5f) * 1.1920928955078125e-7f; }
    // continue after the first block's words [0, w)
    __device__ void start_at(uint32_t w) {
        block = 0;
        used = 4;
        for (uint32_t i = 0; i < w; ++i) next();
    }
};

// upper_bound of `energy` (strictly inside the table) through the log-energy index
__device__ inline int upper_bound32(const MccChannel32& c, float energy) {
    int lo = 0, hi = c.rows;
    if (c.nbins > 0) {
        const float t = (__log2f(energy) - c.lmin) * c.inv_width;
        const int b = !(t >= -1.0f) ? -1 : (t > (float)c.nbins ? c.nbins : (int)floorf(t));
        // one bin of slack on each side covers the fast log's error
        lo = b >= 2 ? (int)__ldg(c.first_gt + (b - 2)) : 0;
        hi = b + 3 <= c.nbins ? (int)__ldg(c.first_gt + (b + 3)) : c.rows;
    }
    const float* e = c.energy;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(e + mid) > energy) hi = mid; else lo = mid + 1;
    }
    return lo;
}

__device__ inline float table_at32(const MccChannel32& c, float energy, int high) {
    const int low = high - 1;
    const float el = __ldg(c.energy + low), eh = __ldg(c.energy + high);
    const float sl = __ldg(c.sigma + low), sh = __ldg(c.sigma + high);
    return eh > el ? sl + (energy - el) / (eh - el) * (sh - sl) : sl;
}

__device__ inline float table_eval32(const MccChannel32& c, float energy) {
    if (energy <= __ldg(c.energy)) return __ldg(c.sigma);
    if (energy >= __ldg(c.energy + c.rows - 1)) return __ldg(c.sigma + c.rows - 1);
    return table_at32(c, energy, upper_bound32(c, energy));
}

// rates_for_speed, src/Collision.cpp:596-625, in FP32; false when the total
// exceeds max_frequency beyond single-precision rounding.  The loops are
// unrolled over the channel slots so that `rates` stays in registers.
__device__ inline bool rates32(const MccModel32& m, float speed, float (&rates)[kMaxChannels]) {
    float total = 0.0f;
    if (m.shared_grid) {
        const MccChannel32& c0 = m.ch[0];
        const float energy = 0.5f * m.particle_mass * speed * speed;
        const int n = c0.rows;
        const bool below = energy <= __ldg(c0.energy), above = energy >= __ldg(c0.energy + n - 1);
        int lo = 0, hi = 0;
        float frac = 0.0f;
        if (below) { lo = hi = 0; }
        else if (above) { lo = hi = n - 1; }
        else {
            hi = upper_bound32(c0, energy);
            lo = hi - 1;
            const float el = __ldg(c0.energy + lo), eh = __ldg(c0.energy + hi);
            frac = eh > el ? (energy - el) / (eh - el) : 0.0f;  // rows merged by rounding: the lower one
        }
#pragma unroll
        for (int i = 0; i < kMaxChannels; ++i) {
            float rate = 0.0f;
            if (i < m.nch) {
                const MccChannel32& c = m.ch[i];
                if (energy >= c.threshold) {
                    const float sl = __ldg(c.sigma + lo), sh = __ldg(c.sigma + hi);
                    rate = m.neutral_density * (sl + frac * (sh - sl)) * speed;
                }
            }
            rates[i] = rate;
            total += rate;
        }
    } else {
#pragma unroll
        for (int i = 0; i < kMaxChannels; ++i) {
            float rate = 0.0f;
            if (i < m.nch) {
                const MccChannel32& c = m.ch[i];
                const float mass = c.frame == 1 ? m.com_mass : m.particle_mass;
                const float energy = 0.5f * mass * speed * speed;
                if (energy >= c.threshold) rate = m.neutral_density * table_eval32(c, energy) * speed;
            }
            rates[i] = rate;
            total += rate;
        }
    }
    return !(total > m.max_frequency * (1.0f + 64.0f * kFltEpsilon));
}

// isotropic_velocity, src/Collision.cpp:53-64
template <class R>
__device__ inline void isotropic32(float speed, R& r, float out[3]) {
    const float cosine = 2.0f * r.uniform() - 1.0f;
    const float sine = sqrtf(fmaxf(0.0f, 1.0f - cosine * cosine));
    float sn, cs;
    // azimuth uniform over one turn, taken on [-pi, pi) where the fast sine is accurate
    __sincosf(6.283185307179586f * (r.uniform() - 0.5f), &sn, &cs);
    out[0] = speed * sine * cs;
    out[1] = speed * sine * sn;
    out[2] = speed * cosine;
}

// MeanCosineTable::evaluate, src/Collision.cpp:296-313
__device__ inline float mean_cosine32(const MccChannel32& c, float energy) {
    const float* e = c.mu_energy;
    const int n = c.mu_rows;
    if (energy <= e[0]) return c.mu[0];
    if (energy >= e[n - 1]) return c.mu[n - 1];
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (energy < e[mid]) hi = mid; else lo = mid + 1;
    }
    return c.mu[lo - 1] + (energy - e[lo - 1]) / (e[lo] - e[lo - 1]) * (c.mu[lo] - c.mu[lo - 1]);
}

// Henyey-Greenstein deflection about the incoming relative velocity,
// src/Collision.cpp:66-129
template <class R>
__device__ inline void angular32(const float in[3], float speed, float g, R& r, float out[3]) {
    const float in2 = in[0] * in[0] + in[1] * in[1] + in[2] * in[2];
    if (!(in2 > 0.0f)) { isotropic32(speed, r, out); return; }
    const float inv = rsqrtf(in2);
    const float sample = r.uniform();
    float cosine = 2.0f * sample - 1.0f;
    if (g != 0.0f) {
        const float ratio = (1.0f - g * g) / (1.0f - g + 2.0f * g * sample);
        cosine = fminf(1.0f, fmaxf(-1.0f, (1.0f + g * g - ratio * ratio) / (2.0f * g)));
    }
    const float sine = sqrtf(fmaxf(0.0f, 1.0f - cosine * cosine));
    const float d[3] = {in[0] * inv, in[1] * inv, in[2] * inv};
    const bool low = fabsf(d[2]) < 0.9f;
    const float h1 = low ? 0.0f : 1.0f, h2 = low ? 1.0f : 0.0f;
    float tg[3] = {h1 * d[2] - h2 * d[1], h2 * d[0], -h1 * d[0]};
    const float tinv = rsqrtf(tg[0] * tg[0] + tg[1] * tg[1] + tg[2] * tg[2]);
    tg[0] *= tinv; tg[1] *= tinv; tg[2] *= tinv;
    const float bt[3] = {d[1] * tg[2] - d[2] * tg[1], d[2] * tg[0] - d[0] * tg[2], d[0] * tg[1] - d[1] * tg[0]};
    float sn, cs;
    __sincosf(6.283185307179586f * (r.uniform() - 0.5f), &sn, &cs);
    const float tf = sine * cs, bf = sine * sn;
    for (int k = 0; k < 3; ++k) out[k] = speed * (cosine * d[k] + tf * tg[k] + bf * bt[k]);
}

// one N(0, stddev) pair by the polar method (libstdc++'s normal_distribution
// transform, in FP32)
template <class R>
__device__ inline void normal_pair32(R& r, float stddev, float& a, float& b) {
    float x, y, r2;
    int guard = 0;
    do {
        x = 2.0f * r.uniform() - 1.0f;
        y = 2.0f * r.uniform() - 1.0f;
        r2 = x * x + y * y;
    } while ((r2 > 1.0f || r2 == 0.0f) && ++guard < 64);
    if (r2 > 1.0f || r2 == 0.0f) { x = 0.0f; y = 0.0f; r2 = 0.5f; }
    const float mult = stddev * sqrtf(-2.0f * __logf(r2) / r2);
    a = y * mult;
    b = x * mult;
}

struct CollideResult32 {
    unsigned candidates = 0, nulls = 0;
    unsigned error = 0;
    bool removed = false;  // attachment
};

__device__ __forceinline__ double energy64(double mass, const float v[3]) {
    const double a = v[0], b = v[1], c = v[2];
    return 0.5 * mass * (a * a + b * b + c * c);
}

// NullCollisionModel::collide(Vec3&) in FP32 after the first waiting time
// `first_wait` (already drawn, inside the step).  majorant_ok(speed) runs the
// frequency-bound check of every later iteration; on_collision receives
// (channel, the particle's energy change in FP64) per real collision and
// on_secondary (channel, secondary velocity[3], ion velocity[3]) per
// ionization.
template <class R, class MajorantOk, class OnCollision, class OnSecondary>
__device__ inline void collide3f(const MccModel32& m, float v[3], float dt, float first_wait, R& r,
                                 CollideResult32& res, MajorantOk&& majorant_ok, OnCollision&& on_collision,
                                 OnSecondary&& on_secondary) {
    float elapsed = 0.0f;
    float waiting = first_wait;
    for (;;) {
        if (!(waiting < dt - elapsed)) break;
        elapsed += waiting;
        ++res.candidates;
        if (res.candidates > m.max_candidates) { res.error |= kErrCandidates; return; }
        float vn[3] = {0.0f, 0.0f, 0.0f};
        if (m.neutral_stddev != 0.0f) {
            const float limit2 = (kThermalSigma * kThermalSigma) * m.neutral_stddev * m.neutral_stddev;
            int attempt = 0;
            for (; attempt < 1024; ++attempt) {
                float spare;
                normal_pair32(r, m.neutral_stddev, vn[0], vn[1]);
                normal_pair32(r, m.neutral_stddev, vn[2], spare);
                if (vn[0] * vn[0] + vn[1] * vn[1] + vn[2] * vn[2] <= limit2) break;
            }
            if (attempt == 1024) { res.error |= kErrMajorant; return; }
        }
        const float rel[3] = {v[0] - vn[0], v[1] - vn[1], v[2] - vn[2]};
        const float rel2 = rel[0] * rel[0] + rel[1] * rel[1] + rel[2] * rel[2];
        const float initial_speed = sqrtf(rel2);
        float rates[kMaxChannels];
        if (!rates32(m, initial_speed, rates)) { res.error |= kErrMajorant; return; }
        const float selection = r.uniform() * m.max_frequency;
        float cumulative = 0.0f;
        int ci = -1;
#pragma unroll
        for (int i = 0; i < kMaxChannels; ++i) {
            cumulative += rates[i];
            if (ci < 0 && i < m.nch && selection < cumulative) ci = i;
        }
        if (ci < 0) {
            ++res.nulls;
        } else {
            const MccChannel32& c = m.ch[ci];
            const double before = energy64(m.particle_mass, v);
            if (c.process == kAttachment) {  // the projectile is removed, src/Collision.cpp:770-773
                v[0] = v[1] = v[2] = 0.0f;
                on_collision(ci, energy64(m.particle_mass, v) - before);
                res.removed = true;
                return;
            }
            if (c.process == kChargeExchange) {
                v[0] = vn[0]; v[1] = vn[1]; v[2] = vn[2];
            } else {
                float energy = 0.5f * m.particle_mass * rel2;
                if (c.process == kExcitation || c.process == kIonization) energy = fmaxf(0.0f, energy - c.threshold);
                if (c.process == kIonization) energy *= 0.5f;
                const float speed = sqrtf(2.0f * energy / m.particle_mass);
                float sc[3];
                if (c.angular == 1) { sc[0] = -rel[0]; sc[1] = -rel[1]; sc[2] = -rel[2]; }
                else if (c.angular == 2 && c.mu_rows) {
                    const float mass = c.frame == 1 ? m.com_mass : m.particle_mass;
                    angular32(rel, speed, mean_cosine32(c, 0.5f * mass * rel2), r, sc);
                } else {
                    isotropic32(speed, r, sc);
                }
                if (c.process == kElastic && m.neutral_mass > 0.0f) {
                    for (int d = 0; d < 3; ++d) v[d] = m.m_frac * v[d] + m.n_frac * vn[d] + m.n_frac * sc[d];
                } else {
                    for (int d = 0; d < 3; ++d) v[d] = vn[d] + sc[d];
                }
            }
            on_collision(ci, energy64(m.particle_mass, v) - before);
            if (c.process == kIonization) {
                const float d0 = v[0] - vn[0], d1 = v[1] - vn[1], d2 = v[2] - vn[2];
                float iso[3];
                isotropic32(sqrtf(d0 * d0 + d1 * d1 + d2 * d2), r, iso);
                const float vs[3] = {vn[0] + iso[0], vn[1] + iso[1], vn[2] + iso[2]};
                on_secondary(ci, vs, vn);
            }
        }
        // next waiting time (the frequency-bound check of the loop's next iteration first)
        const float s2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        if (!(s2 <= m.v_safe2) && !majorant_ok(sqrtf(s2))) { res.error |= kErrMajorant; return; }
        waiting = -__logf(r.uniform()) * m.inv_max_frequency;
    }
}

}  // namespace apic
