// Random-number streams for the null-collision MCC kernels.
//
// The reference draws from std::mt19937_64 through libstdc++'s distributions
// (src/Collision.cpp:46-64, :690-712, :745, :948).  On the device each particle
// owns a counter-based Philox4x32-10 stream (Salmon et al., SC'11) keyed on
// (seed) with counter (draw pair, particle slot, step, stream word), and the
// same libstdc++ transforms turn raw 64-bit draws into doubles.  A replay
// stream feeds recorded raw draws instead, which makes the device decisions
// identical to the reference's for the same engine output.
#pragma once
#include <cstdint>

namespace apic {

__host__ __device__ inline void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                              uint32_t k0, uint32_t k1, uint32_t out[4]) {
#pragma unroll
    for (int round = 0; round < 10; ++round) {
#ifdef __CUDA_ARCH__
        const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
#else
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// Raw 64-bit draws k = 0, 1, 2, ... of one particle's stream: draw k is half
// of Philox block k/2 (low pair for even k, high pair for odd k).
struct PhiloxStream {
    uint32_t k0, k1, slot, step, stream;
    uint32_t index = 0;
    uint32_t buf[4];
    __device__ PhiloxStream(uint64_t seed, uint32_t slot_, uint32_t step_, uint32_t stream_)
        : k0((uint32_t)seed), k1((uint32_t)(seed >> 32)), slot(slot_), step(step_), stream(stream_) {}
    __device__ uint64_t next() {
        const uint32_t k = index++;
        if ((k & 1u) == 0u) philox4x32_10(k >> 1, slot, step, stream, k0, k1, buf);
        return (k & 1u) ? ((uint64_t)buf[3] << 32 | buf[2]) : ((uint64_t)buf[1] << 32 | buf[0]);
    }
    __device__ bool overrun() const { return false; }
    // continue a stream that already produced k draws
    __device__ void seek(uint32_t k) {
        index = k;
        if (k & 1u) philox4x32_10(k >> 1, slot, step, stream, k0, k1, buf);
    }
};

struct ReplayStream {
    const uint64_t* draws;
    uint64_t len;
    uint32_t index = 0;
    bool over = false;
    __device__ uint64_t next() {
        const uint32_t k = index++;
        if (k >= len) { over = true; return 0; }
        return draws[k];
    }
    __device__ bool overrun() const { return over; }
};

// generate_canonical<double, 53|64> on a 64-bit engine (libstdc++
// <bits/random.tcc>): one draw, divided by 2^64, results that round to 1
// become nextafter(1, 0).
// generate_canonical of one given 64-bit draw
__device__ inline double canonical_of(uint64_t draw) {
    double ret = (double)draw / 18446744073709551616.0;
    if (ret >= 1.0) ret = 0x1.fffffffffffffp-1;
    return ret;
}

template <class S>
__device__ inline double canonical(S& s) {
    const double sum = (double)s.next();
    double ret = sum / 18446744073709551616.0;
    if (ret >= 1.0) ret = 0x1.fffffffffffffp-1;
    return ret;
}

// uniform_real_distribution<double>(0, 1): canonical * (1 - 0) + 0.
template <class S>
__device__ inline double uniform01(S& s) { return canonical(s); }

// uniform_int_distribution<int>(0, 1): Lemire's nearly-divisionless reduction
// (ACM TOMACS 29(1), 2019) with range 2 has rejection threshold 0, so the
// result is the draw's top bit.
template <class S>
__device__ inline int bit01(S& s) { return (int)(s.next() >> 63); }

// normal_distribution: Marsaglia's polar method keeping one saved value, as
// libstdc++ does; `saved_available` lives in the caller (one object per
// sample_neutral_velocity_3v call, src/Collision.cpp:705).
struct NormalState {
    bool saved_available = false;
    double saved = 0.0;
};

template <class S>
__device__ inline double normal(NormalState& st, S& s, double mean, double stddev) {
    double ret;
    if (st.saved_available) {
        st.saved_available = false;
        ret = st.saved;
    } else {
        double x, y, r2;
        // acceptance is pi/4 per pair; the bound only guards exhausted replay arrays
        int attempts = 0;
        do {
            x = 2.0 * canonical(s) - 1.0;
            y = 2.0 * canonical(s) - 1.0;
            r2 = x * x + y * y;
        } while ((r2 > 1.0 || r2 == 0.0) && !s.overrun() && ++attempts < 4096);
        if (r2 > 1.0 || r2 == 0.0) { x = 0.0; y = 0.0; r2 = 0.5; }
        const double mult = sqrt(-2 * log(r2) / r2);
        st.saved = x * mult;
        st.saved_available = true;
        ret = y * mult;
    }
    return ret * stddev + mean;
}

}  // namespace apic
