// Homogeneous electron swarms on the device: run_field (src/Swarm.cpp:940-1250)
// for many runs at once, and the serving loop that admits, steps and retires
// them.
//
// Layout.  Every run owns structure-of-arrays electron state (velocity and
// displacement since the sampling start, FP64 or FP32) in one device pool.
// Runs are cut into chunks of kChunk electrons; a chunk table (run slot, first
// electron) lists the chunks of every active run back to back, and one
// persistent push kernel walks it, so runs of any size share one launch per
// substep.  Per-chunk partial sums feed a per-run reduction whose summation
// order depends on the run alone: a run's result is bit-identical whether it
// runs alone or among others.
//
// Random numbers.  Philox4x32-10 streams keyed on (seed, electron index, step):
// stream 0 for the collision loop, stream 1 (index 0xFFFFFFFF) for the
// resampling offset, stream 2 (step 0xFFFFFFFF) for the initial Maxwellian.
//
// Per step (src/Swarm.cpp:994-1128): half kick, energy check, drift,
// null-collision MCC, half kick, energy check, tallies; with branching, the
// surviving electrons and the ionization secondaries are compacted in the
// reference's order (survivors in order, then secondaries in parent order) and
// systematically resampled back to the target population.  All electrons of a
// run share one weight, so the resampling source of output s is the electron
// ceil((u + s) M / N) - 1 of the M compacted ones.
#include <cub/block/block_scan.cuh>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "aurorapic_b200.h"
#include "apic_common.cuh"
#include "apic_mcc.cuh"
#include "apic_mcc_host.h"
#include "apic_rng.cuh"

namespace apic {
cudaError_t bounded_wait(cudaStream_t stream, double seconds);

namespace swarm {

constexpr int kThreads = 256;
constexpr int kChunk = 1024;
constexpr int kItems = kChunk / kThreads;
constexpr int kMaxBirthsPerElectron = 8;
constexpr double kElectronMass = 9.1093837139e-31;  // src/Swarm.cpp:23
constexpr double kEvToJ = 1.602176634e-19;          // src/Swarm.cpp:24-25
constexpr double kTownsend = 1.0e-21;               // src/Swarm.cpp:26
constexpr size_t kAllocationLimit = 10000000;        // src/Swarm.cpp:27

enum : unsigned {
    kErrMaxEnergyPre = 1u << 8,
    kErrMaxEnergy = 1u << 9,
    kErrPopulation = 1u << 10,
    kErrExtinct = 1u << 11,
};

struct RunCfg {  // written by the host at admission, read-only on the device
    double half_kick, dt, max_energy_ev, init_sd;
    double vscale, escale;  // fixed-point scales (powers of two) of the v_x and |v|^2 sums
    // kinetic_energy_ev(v) > max_energy_ev exactly when |v|^2 > s2_max (the
    // energy is a monotone function of |v|^2 in floating point)
    double s2_max;
    // -log(u) / max_frequency < dt exactly when the first 64-bit draw is at
    // least cand_draw_min (u = draw / 2^64; a zero draw is redrawn and takes
    // the evaluated path); no_candidates when no draw qualifies
    uint64_t cand_draw_min;
    int no_candidates;
    int pad0;
    uint64_t seed;
    uint32_t n, steps, burn_in, first_chunk, nchunks, limit;
    int branching;
    int pad;
    void* v[3];
    void* d[3];
    void* bv[3];       // compacted population (branching), `limit` electrons
    void* bd[3];
    void* sv[3];       // secondaries staged per chunk (branching), nchunks * kChunk
    uint32_t* skey;    // their keys: parent index within the chunk * 8 + secondary number
    uint8_t* alive;    // survivors of the current step (branching)
    double* samples;   // velocity, energy, log weight per sampling step
};

struct RunState {  // written by the device
    uint32_t step, active;
    unsigned error;
    uint32_t m_prime, survivors, pad;
    double weight, weight_next, u, exposure, max_ev;
    unsigned long long candidates, nulls;
    unsigned long long counts[kMaxChannels];
    double wcoll[kMaxChannels], wcoll2[kMaxChannels];
    double mean_d[3], var_l, var_t;
};

// Per-chunk tallies of one step.  The sums are fixed point (each electron's
// contribution rounded once), so they do not depend on the order in which the
// push and collision kernels add them.
struct ChunkPartial {
    unsigned long long vsum, esum;  // two's-complement fixed point
    unsigned long long emax_bits;   // largest |v|^2 (bits of a non-negative double)
    unsigned long long cand, nulls;
    unsigned counts[kMaxChannels];
    unsigned surv, births, surv_off, birth_off;
};

// An electron whose first waiting time falls inside the step.  Its stored
// velocity is still the one from the start of the step; the collision kernel
// repeats the first half kick and the first draw.
struct Candidate {
    uint32_t particle;  // index within its run
    uint32_t chunk;     // chunk-table position
    uint32_t slot;
    uint32_t pad;
};

struct Batch {
    const RunCfg* cfg;
    RunState* st;
    const uint32_t* chunk_run;
    const uint32_t* chunk_first;
    const uint32_t* nchunks;
    ChunkPartial* part;
    Candidate* queue;
    unsigned* qlen;
    unsigned qcap;
    int max_runs;
    const MccModelDev* model;  // in device memory: the kernels take references into it
    const MccModel32* model32; // the same model in single precision (FP32 form)
};

template <class T>
__device__ __forceinline__ T* arr(void* p) { return static_cast<T*>(p); }

// kinetic_energy_ev, src/Swarm.cpp:95-101
__device__ __forceinline__ double ke_ev(double x, double y, double z) {
    const double s2 = x * x + y * y + z * z;
    return 0.5 * kElectronMass * s2 / kEvToJ;
}

template <class T>
__device__ __forceinline__ T store_as(double x) { return (T)x; }

__device__ __forceinline__ double sq3(double x, double y, double z) { return x * x + y * y + z * z; }

__device__ __forceinline__ unsigned long long to_fixed(double x, double scale) {
    return (unsigned long long)__double2ll_rn(x * scale);
}

// Block-wide sum of one double per thread in a fixed tree order (valid on thread 0).
__device__ double block_sum(double x, double* red) {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = x;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kThreads / 32; ++w) t += red[w];
    return t;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long x) {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long x) {
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long y = __shfl_xor_sync(0xffffffffu, x, o);
        x = y > x ? y : x;
    }
    return x;
}

// ---- initial Maxwellian (src/Swarm.cpp:948-956) --------------------------------

template <class T>
__global__ void __launch_bounds__(kThreads) k_swarm_init(RunCfg R) {
    const uint32_t i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= R.n) return;
    PhiloxStream s(R.seed, i, 0xFFFFFFFFu, 2u);
    NormalState ns;
    for (int a = 0; a < 3; ++a) {
        arr<T>(R.v[a])[i] = store_as<T>(normal(ns, s, 0.0, R.init_sd));
        arr<T>(R.d[a])[i] = store_as<T>(0.0);
    }
}

// Tally destinations of one chunk: shared memory in the push kernel, the
// chunk's global partial in the collision kernel (atomics on generic addresses).
struct Tally {
    unsigned long long* vsum;
    unsigned long long* esum;
    unsigned long long* emax;
    unsigned long long* cand;
    unsigned long long* nulls;
    unsigned* counts;
    unsigned* surv;
    unsigned* births;
    unsigned* err;
};

// The rest of one electron's step after its first waiting time fell inside
// the step: the collision loop (src/Collision.cpp:907-993), the second half
// kick and energy check, the store, and the tallies.
template <class T>
__device__ __forceinline__ void finish_candidate(const MccModelDev& M, const RunCfg& R, uint32_t step,
                                                 uint32_t first, const Candidate& e, const Tally& t) {
    double v[3];
    for (int a = 0; a < 3; ++a) v[a] = (double)arr<T>(R.v[a])[e.particle];
    v[0] += R.half_kick;  // the push kernel's first half kick, repeated
    PhiloxStream rng(R.seed, e.particle, step, 0u);
    double u = uniform01(rng);
    for (int guard = 0; !(u > 0.0) && guard < 64; ++guard) u = uniform01(rng);
    const double first_wait = -log(u) / M.max_frequency;
    CollideResult r;
    unsigned nsec = 0;
    const uint32_t li = e.particle - first;
    const uint32_t local_chunk = first / kChunk;
    unsigned err = 0;
    collide3(M, v, R.dt, rng, r,
             [&](int, const double* vs, const double*) {
                 if (!R.branching) return;  // fixed population: secondaries are not followed
                 if (nsec >= (unsigned)kMaxBirthsPerElectron) { err |= kErrBirths; return; }
                 const unsigned bi = atomicAdd(t.births, 1u);
                 if (bi >= (unsigned)kChunk) { err |= kErrBirths; return; }
                 const size_t at = (size_t)local_chunk * kChunk + bi;
                 for (int a = 0; a < 3; ++a) arr<T>(R.sv[a])[at] = store_as<T>(vs[a]);
                 R.skey[at] = li * kMaxBirthsPerElectron + nsec;
                 ++nsec;
             },
             true, first_wait);
    err |= r.error;
    v[0] += R.half_kick;
    const double s2 = sq3(v[0], v[1], v[2]);
    if (s2 > R.s2_max) err |= kErrMaxEnergy;
    T vs[3];
    for (int a = 0; a < 3; ++a) {
        vs[a] = store_as<T>(v[a]);
        arr<T>(R.v[a])[e.particle] = vs[a];
    }
    if (R.branching) R.alive[e.particle] = r.removed ? 0 : 1;
    atomicMax(t.emax, (unsigned long long)__double_as_longlong(s2));
    atomicAdd(t.cand, (unsigned long long)r.candidates);
    if (r.nulls) atomicAdd(t.nulls, (unsigned long long)r.nulls);
    for (int ch = 0; ch < M.nch; ++ch)
        if (r.channel[ch]) atomicAdd(&t.counts[ch], r.channel[ch]);
    if (!r.removed) atomicAdd(t.surv, 1u);
    atomicAdd(t.vsum, to_fixed((double)vs[0], R.vscale));
    atomicAdd(t.esum, to_fixed(sq3((double)vs[0], (double)vs[1], (double)vs[2]), R.escale));
    if (err) atomicOr(t.err, err);
}

// The FP32 form of finish_candidate: the collision loop in FP32 (collide3f) on
// the float velocity, the first waiting time from the same first 64-bit draw
// that made the electron a candidate (rounded to a 23-bit uniform, kept inside
// the step), the later uniforms from the rest of the electron's Philox stream.
__device__ __forceinline__ void finish_candidate32(const MccModelDev& M, const MccModel32& M32, const RunCfg& R,
                                                   uint32_t step, uint32_t first, const Candidate& e,
                                                   const Tally& t) {
    float v[3];
    for (int a = 0; a < 3; ++a) v[a] = arr<float>(R.v[a])[e.particle];
    const float hk = (float)R.half_kick;
    v[0] += hk;  // the push kernel's first half kick, repeated
    Philox32 rng(R.seed, e.particle, step, 0u);
    const uint32_t w0 = rng.next(), w1 = rng.next();
    const uint64_t d0 = (uint64_t)w1 << 32 | w0;
    const float dt = (float)R.dt;
    const float u0 = ((float)(d0 >> 41) + 0.5f) * 1.1920928955078125e-7f;
    const float first_wait = fminf(-__logf(u0) * M32.inv_max_frequency, dt * (1.0f - kFltEpsilon));
    CollideResult32 r;
    unsigned nsec = 0;
    const uint32_t li = e.particle - first;
    const uint32_t local_chunk = first / kChunk;
    unsigned err = 0;
    collide3f(
        M32, v, dt, first_wait, rng, r, [&](float speed) { return frequency_bound_ok_far(M, (double)speed); },
        [&](int ch, double) { atomicAdd(&t.counts[ch], 1u); },
        [&](int, const float* vs, const float*) {
            if (!R.branching) return;  // fixed population: secondaries are not followed
            if (nsec >= (unsigned)kMaxBirthsPerElectron) { err |= kErrBirths; return; }
            const unsigned bi = atomicAdd(t.births, 1u);
            if (bi >= (unsigned)kChunk) { err |= kErrBirths; return; }
            const size_t at = (size_t)local_chunk * kChunk + bi;
            for (int a = 0; a < 3; ++a) arr<float>(R.sv[a])[at] = vs[a];
            R.skey[at] = li * kMaxBirthsPerElectron + nsec;
            ++nsec;
        });
    err |= r.error;
    v[0] += hk;
    const double s2 = sq3((double)v[0], (double)v[1], (double)v[2]);
    if (s2 > R.s2_max) err |= kErrMaxEnergy;
    for (int a = 0; a < 3; ++a) arr<float>(R.v[a])[e.particle] = v[a];
    if (R.branching) R.alive[e.particle] = r.removed ? 0 : 1;
    atomicMax(t.emax, (unsigned long long)__double_as_longlong(s2));
    atomicAdd(t.cand, (unsigned long long)r.candidates);
    if (r.nulls) atomicAdd(t.nulls, (unsigned long long)r.nulls);
    if (!r.removed) atomicAdd(t.surv, 1u);
    atomicAdd(t.vsum, to_fixed((double)v[0], R.vscale));
    atomicAdd(t.esum, to_fixed(s2, R.escale));
    if (err) atomicOr(t.err, err);
}

// ---- one step, streaming part: every electron of every active run --------------
// Half kick, energy check, drift, first waiting time; electrons without a
// collision candidate finish the step here, the others go to the candidate
// queue (one global reservation per chunk).

template <class T>
__global__ void __launch_bounds__(kThreads, 2) k_swarm_push(Batch b) {
    __shared__ unsigned long long s_vsum, s_esum, s_emax, s_cand, s_nulls;
    __shared__ unsigned s_counts[kMaxChannels];
    __shared__ unsigned s_surv, s_births, s_err, s_ncand, s_base;
    const int tid = threadIdx.x, lane = tid & 31;
    const uint32_t nch_total = *b.nchunks;
    const MccModelDev& M = *b.model;

    for (uint32_t c = blockIdx.x; c < nch_total; c += gridDim.x) {
        const uint32_t slot = b.chunk_run[c];
        const RunCfg& R = b.cfg[slot];
        const RunState& S = b.st[slot];
        if (!S.active) continue;  // uniform over the CTA
        const uint32_t first = b.chunk_first[c];
        const uint32_t cnt = min((uint32_t)kChunk, R.n - first);
        const uint32_t step = S.step;
        const bool sampling = step >= R.burn_in;
        if (tid == 0) {
            s_vsum = s_esum = s_emax = s_cand = s_nulls = 0ull;
            s_surv = s_births = s_err = s_ncand = 0u;
        }
        if (tid < kMaxChannels) s_counts[tid] = 0u;
        __syncthreads();

        unsigned long long vsum = 0ull, esum = 0ull, emax = 0ull;
        unsigned err = 0, surv = 0;
        unsigned cand_mask = 0;
        int qslot[kItems];
        // loads of the thread's electrons, then their first 64-bit draws (four
        // independent Philox chains that run while the loads are in flight)
        T vl[kItems][3], dl[kItems][3];
        uint64_t d0[kItems];
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            const uint32_t li = k * kThreads + tid;
            const uint32_t i = first + li;
            const bool ok = li < cnt;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                vl[k][a] = ok ? arr<T>(R.v[a])[i] : T(0);
                dl[k][a] = ok && sampling ? arr<T>(R.d[a])[i] : T(0);
            }
        }
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            uint32_t o[4];
            philox4x32_10(0u, first + k * kThreads + tid, step, 0u, (uint32_t)R.seed, (uint32_t)(R.seed >> 32), o);
            d0[k] = (uint64_t)o[1] << 32 | o[0];  // PhiloxStream's first draw
        }
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            const uint32_t li = k * kThreads + tid;
            const uint32_t i = first + li;
            qslot[k] = -1;
            if (li >= cnt) continue;
            double v[3];
            for (int a = 0; a < 3; ++a) v[a] = (double)vl[k][a];
            v[0] += R.half_kick;
            const double pre = sq3(v[0], v[1], v[2]);
            emax = max(emax, (unsigned long long)__double_as_longlong(pre));
            if (pre > R.s2_max) err |= kErrMaxEnergyPre;
            if (sampling)
                for (int a = 0; a < 3; ++a) arr<T>(R.d[a])[i] = store_as<T>((double)dl[k][a] + v[a] * R.dt);
            // first iteration of NullCollisionModel::collide, src/Collision.cpp:926-933
            if (!(pre <= M.v_safe2) && !frequency_bound_ok_far(M, sqrt(pre))) err |= kErrMajorant;
            bool candidate;
            if (d0[k] != 0ull) {
                candidate = !R.no_candidates && d0[k] >= R.cand_draw_min;
            } else {  // open_unit_interval draws again
                PhiloxStream rng(R.seed, i, step, 0u);
                double u = 0.0;
                for (int guard = 0; !(u > 0.0) && guard < 64; ++guard) u = uniform01(rng);
                const double wait = -log(u) / M.max_frequency;
                candidate = isfinite(wait) && wait < R.dt;
            }
            if (candidate) {
                cand_mask |= 1u << k;
                qslot[k] = (int)atomicAdd(&s_ncand, 1u);
                continue;
            }
            // no candidate this step: second half kick, check, store, tallies
            v[0] += R.half_kick;
            const double en = sq3(v[0], v[1], v[2]);
            emax = max(emax, (unsigned long long)__double_as_longlong(en));
            if (en > R.s2_max) err |= kErrMaxEnergy;
            T vs[3];
            for (int a = 0; a < 3; ++a) {
                vs[a] = store_as<T>(v[a]);
                arr<T>(R.v[a])[i] = vs[a];
            }
            if (R.branching) R.alive[i] = 1;
            ++surv;
            vsum += to_fixed((double)vs[0], R.vscale);
            esum += to_fixed(sizeof(T) == sizeof(double) ? en : sq3((double)vs[0], (double)vs[1], (double)vs[2]),
                             R.escale);
        }
        vsum = warp_sum_u64(vsum);
        esum = warp_sum_u64(esum);
        emax = warp_max_u64(emax);
        if (lane == 0) {
            atomicAdd(&s_vsum, vsum);
            atomicAdd(&s_esum, esum);
            atomicMax(&s_emax, emax);
        }
        if (surv) atomicAdd(&s_surv, surv);
        if (err) atomicOr(&s_err, err);
        __syncthreads();
        if (tid == 0) s_base = s_ncand ? atomicAdd(b.qlen, s_ncand) : 0u;
        __syncthreads();
        // the queue holds one entry per active electron, so it cannot overflow
#pragma unroll
        for (int k = 0; k < kItems; ++k)
            if (cand_mask >> k & 1u)
                b.queue[s_base + (unsigned)qslot[k]] = Candidate{first + k * kThreads + tid, c, slot, 0u};
        __syncthreads();
        if (tid == 0) {
            ChunkPartial& P = b.part[c];
            P.vsum = s_vsum;
            P.esum = s_esum;
            P.emax_bits = s_emax;
            P.cand = s_cand;
            P.nulls = s_nulls;
            for (int ch = 0; ch < kMaxChannels; ++ch) P.counts[ch] = s_counts[ch];
            P.surv = s_surv;
            P.births = s_births;
            if (s_err) atomicOr(&b.st[slot].error, s_err);
        }
        __syncthreads();
    }
}

// ---- one step, collision part: the queued candidates, packed densely -----------

template <class T>
__global__ void __launch_bounds__(kThreads, 4) k_swarm_collide(Batch b) {
    const unsigned qn = *b.qlen;
    for (unsigned q = blockIdx.x * kThreads + threadIdx.x; q < qn; q += gridDim.x * kThreads) {
        const Candidate e = b.queue[q];
        const RunCfg& R = b.cfg[e.slot];
        RunState& S = b.st[e.slot];
        ChunkPartial& P = b.part[e.chunk];
        const uint32_t first = b.chunk_first[e.chunk];
        const Tally tl{&P.vsum, &P.esum, &P.emax_bits, &P.cand, &P.nulls, P.counts, &P.surv, &P.births, &S.error};
        if constexpr (sizeof(T) == 4)
            finish_candidate32(*b.model, *b.model32, R, S.step, first, e, tl);
        else
            finish_candidate<T>(*b.model, R, S.step, first, e, tl);
    }
}

// ---- branching: scan of survivors and secondaries per run ------------------------

__global__ void __launch_bounds__(kThreads) k_swarm_branch_scan(Batch b) {
    using Scan = cub::BlockScan<unsigned long long, kThreads>;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ unsigned long long s_carry_s, s_carry_b;
    const int slot = blockIdx.x;
    if (slot >= b.max_runs) return;
    const RunCfg& R = b.cfg[slot];
    RunState& S = b.st[slot];
    if (!S.active || !R.branching) return;
    if (threadIdx.x == 0) { s_carry_s = 0; s_carry_b = 0; }
    __syncthreads();
    for (uint32_t base = 0; base < R.nchunks; base += kThreads) {
        const uint32_t lc = base + threadIdx.x;
        const bool ok = lc < R.nchunks;
        ChunkPartial* P = ok ? &b.part[R.first_chunk + lc] : nullptr;
        // survivors and births packed in one 64-bit scan (each < 2^32 per run)
        const unsigned long long x =
            ok ? (((unsigned long long)P->surv << 32) | min(P->births, (unsigned)kChunk)) : 0ull;
        unsigned long long ex, tot;
        Scan(tmp).ExclusiveSum(x, ex, tot);
        if (ok) {
            P->surv_off = (unsigned)(s_carry_s + (ex >> 32));
            P->birth_off = (unsigned)(s_carry_b + (ex & 0xFFFFFFFFull));
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_carry_s += tot >> 32;
            s_carry_b += tot & 0xFFFFFFFFull;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const unsigned long long mp = s_carry_s + s_carry_b;
        S.survivors = (uint32_t)s_carry_s;
        S.m_prime = (uint32_t)min(mp, 0xFFFFFFFFull);
        if (mp > R.limit) atomicOr(&S.error, kErrPopulation);
        if (mp == 0) atomicOr(&S.error, kErrExtinct);
        // systematic_resample, src/Swarm.cpp:616-643: offset and output weight
        PhiloxStream rng(R.seed, 0xFFFFFFFFu, S.step, 1u);
        S.u = uniform01(rng);
        S.weight_next = mp == R.n ? S.weight : (double)mp * S.weight / (double)R.n;
    }
}

// Survivors in order, then the secondaries in parent order, into the
// compacted population.
template <class T>
__global__ void __launch_bounds__(kThreads) k_swarm_branch_compact(Batch b) {
    using Scan = cub::BlockScan<unsigned, kThreads>;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ uint32_t s_key[kChunk];
    __shared__ unsigned s_carry;
    const uint32_t nch_total = *b.nchunks;
    for (uint32_t c = blockIdx.x; c < nch_total; c += gridDim.x) {
        const uint32_t slot = b.chunk_run[c];
        const RunCfg& R = b.cfg[slot];
        const RunState& S = b.st[slot];
        if (!S.active || !R.branching || S.error) continue;
        const ChunkPartial& P = b.part[c];
        const uint32_t first = b.chunk_first[c];
        const uint32_t local_chunk = first / kChunk;
        const uint32_t cnt = min((uint32_t)kChunk, R.n - first);
        if (threadIdx.x == 0) s_carry = 0;
        __syncthreads();
        for (uint32_t base = 0; base < cnt; base += kThreads) {
            const uint32_t li = base + threadIdx.x;
            const unsigned a = li < cnt ? R.alive[first + li] : 0u;
            unsigned ex, tot;
            Scan(tmp).ExclusiveSum(a, ex, tot);
            if (a) {
                const size_t dst = (size_t)P.surv_off + s_carry + ex;
                for (int k = 0; k < 3; ++k) {
                    arr<T>(R.bv[k])[dst] = arr<T>(R.v[k])[first + li];
                    arr<T>(R.bd[k])[dst] = arr<T>(R.d[k])[first + li];
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) s_carry += tot;
            __syncthreads();
        }
        const unsigned nb = min(P.births, (unsigned)kChunk);
        const size_t sbase = (size_t)local_chunk * kChunk;
        for (unsigned j = threadIdx.x; j < nb; j += kThreads) s_key[j] = R.skey[sbase + j];
        __syncthreads();
        for (unsigned j = threadIdx.x; j < nb; j += kThreads) {
            const uint32_t key = s_key[j];
            unsigned rank = 0;
            for (unsigned q = 0; q < nb; ++q) rank += s_key[q] < key ? 1u : 0u;
            const size_t dst = (size_t)S.survivors + P.birth_off + rank;
            const uint32_t parent = first + key / kMaxBirthsPerElectron;
            for (int k = 0; k < 3; ++k) {
                arr<T>(R.bv[k])[dst] = arr<T>(R.sv[k])[sbase + j];
                arr<T>(R.bd[k])[dst] = arr<T>(R.d[k])[parent];
            }
        }
        __syncthreads();
    }
}

// Systematic resampling back to N electrons, and the sample sums of the step.
template <class T>
__global__ void __launch_bounds__(kThreads) k_swarm_branch_resample(Batch b) {
    __shared__ unsigned long long s_vsum, s_esum;
    const uint32_t nch_total = *b.nchunks;
    for (uint32_t c = blockIdx.x; c < nch_total; c += gridDim.x) {
        const uint32_t slot = b.chunk_run[c];
        const RunCfg& R = b.cfg[slot];
        const RunState& S = b.st[slot];
        if (!S.active || !R.branching || S.error) continue;
        const uint32_t first = b.chunk_first[c];
        const uint32_t cnt = min((uint32_t)kChunk, R.n - first);
        const uint32_t mp = S.m_prime;
        if (threadIdx.x == 0) s_vsum = s_esum = 0ull;
        __syncthreads();
        unsigned long long vsum = 0ull, esum = 0ull;
        for (uint32_t li = threadIdx.x; li < cnt; li += kThreads) {
            const uint32_t s = first + li;
            uint32_t j = s;
            if (mp != R.n) {
                const double t = (S.u + (double)s) * (double)mp / (double)R.n;
                const double cj = ceil(t) - 1.0;
                j = cj < 0.0 ? 0u : (uint32_t)cj;
                if (j > mp - 1) j = mp - 1;
            }
            T vs[3];
            for (int k = 0; k < 3; ++k) {
                vs[k] = arr<T>(R.bv[k])[j];
                arr<T>(R.v[k])[s] = vs[k];
                arr<T>(R.d[k])[s] = arr<T>(R.bd[k])[j];
            }
            vsum += to_fixed((double)vs[0], R.vscale);
            esum += to_fixed(sq3((double)vs[0], (double)vs[1], (double)vs[2]), R.escale);
        }
        vsum = warp_sum_u64(vsum);
        esum = warp_sum_u64(esum);
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&s_vsum, vsum);
            atomicAdd(&s_esum, esum);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            b.part[c].vsum = s_vsum;
            b.part[c].esum = s_esum;
        }
        __syncthreads();
    }
}

// ---- per run: tallies and the samples of the step --------------------------------

__global__ void __launch_bounds__(kThreads) k_swarm_reduce(Batch b) {
    __shared__ unsigned long long s_v, s_e, s_m, s_c, s_n;
    __shared__ unsigned long long s_ch[kMaxChannels];
    const int slot = blockIdx.x;
    if (slot == 0 && threadIdx.x == 0) *b.qlen = 0u;  // the candidate queue of the next step starts empty
    if (slot >= b.max_runs) return;
    const RunCfg& R = b.cfg[slot];
    RunState& S = b.st[slot];
    if (!S.active) return;
    const int nch = b.model->nch;
    if (threadIdx.x == 0) s_v = s_e = s_m = s_c = s_n = 0ull;
    if (threadIdx.x < kMaxChannels) s_ch[threadIdx.x] = 0ull;
    __syncthreads();
    unsigned long long v = 0, e = 0, m = 0, cand = 0, nulls = 0, cnt[kMaxChannels] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t lc = threadIdx.x; lc < R.nchunks; lc += kThreads) {
        const ChunkPartial& P = b.part[R.first_chunk + lc];
        v += P.vsum;
        e += P.esum;
        m = max(m, P.emax_bits);
        cand += P.cand;
        nulls += P.nulls;
#pragma unroll
        for (int ch = 0; ch < kMaxChannels; ++ch) cnt[ch] += P.counts[ch];
    }
    v = warp_sum_u64(v);
    e = warp_sum_u64(e);
    m = warp_max_u64(m);
    cand = warp_sum_u64(cand);
    nulls = warp_sum_u64(nulls);
#pragma unroll
    for (int ch = 0; ch < kMaxChannels; ++ch) cnt[ch] = warp_sum_u64(cnt[ch]);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&s_v, v);
        atomicAdd(&s_e, e);
        atomicMax(&s_m, m);
        atomicAdd(&s_c, cand);
        atomicAdd(&s_n, nulls);
        for (int ch = 0; ch < nch; ++ch) atomicAdd(&s_ch[ch], cnt[ch]);
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const uint32_t step = S.step;
    const double w = S.weight;
    // kinetic_energy_ev of the largest |v|^2: the energy is monotone in |v|^2
    S.max_ev = fmax(S.max_ev, 0.5 * kElectronMass * __longlong_as_double((long long)s_m) / kEvToJ);
    if (step >= R.burn_in) {
        S.exposure += (double)R.n * w * R.dt;
        S.candidates += s_c;
        S.nulls += s_n;
        for (int ch = 0; ch < nch; ++ch) {
            S.counts[ch] += s_ch[ch];
            S.wcoll[ch] += w * (double)s_ch[ch];
            S.wcoll2[ch] += w * w * (double)s_ch[ch];
        }
    }
    if (R.branching && !S.error) S.weight = S.weight_next;
    if (step >= R.burn_in) {
        const size_t ns = R.steps - R.burn_in;
        const size_t k = step - R.burn_in;
        R.samples[k] = (double)(long long)s_v / R.vscale / (double)R.n;
        R.samples[ns + k] = 0.5 * kElectronMass * ((double)(long long)s_e / R.escale) / kEvToJ / (double)R.n;
        R.samples[2 * ns + k] = log((double)R.n * S.weight);
    }
    S.step = step + 1;
    if (S.step >= R.steps || S.error) S.active = 0;
}

// ---- per run: displacement statistics for the diffusion coefficients -------------

template <class T>
__global__ void __launch_bounds__(kThreads) k_swarm_moments(RunCfg R, RunState* S) {
    __shared__ double s_red[kThreads / 32];
    __shared__ double s_mean[3];
    double m[3] = {0.0, 0.0, 0.0};
    for (uint32_t i = threadIdx.x; i < R.n; i += kThreads)
        for (int a = 0; a < 3; ++a) m[a] += (double)arr<T>(R.d[a])[i];
    for (int a = 0; a < 3; ++a) {
        const double t = block_sum(m[a], s_red);
        if (threadIdx.x == 0) s_mean[a] = t / (double)R.n;
        __syncthreads();
    }
    double vl = 0.0, vt = 0.0;
    for (uint32_t i = threadIdx.x; i < R.n; i += kThreads) {
        const double dx = (double)arr<T>(R.d[0])[i] - s_mean[0];
        const double dy = (double)arr<T>(R.d[1])[i] - s_mean[1];
        const double dz = (double)arr<T>(R.d[2])[i] - s_mean[2];
        vl += dx * dx;
        vt += dy * dy + dz * dz;
    }
    const double tl = block_sum(vl, s_red);
    const double tt = block_sum(vt, s_red);
    if (threadIdx.x == 0) {
        for (int a = 0; a < 3; ++a) S->mean_d[a] = s_mean[a];
        S->var_l = tl / (double)R.n;
        S->var_t = tt / (double)R.n;
    }
}

// ---- host side -------------------------------------------------------------------

// block_mean_and_error, src/Swarm.cpp:103-134
static bool block_mean_and_error(const double* x, size_t n, size_t blocks, double& mean, double& se) {
    if (n == 0 || blocks == 0 || blocks > n) return false;
    std::vector<double> means(blocks);
    for (size_t b = 0; b < blocks; ++b) {
        const size_t begin = b * n / blocks, end = (b + 1) * n / blocks;
        double total = 0.0;
        for (size_t i = begin; i < end; ++i) total += x[i];
        means[b] = total / (double)(end - begin);
    }
    double m = 0.0;
    for (double v : means) m += v;
    m /= (double)blocks;
    double e = 0.0;
    if (blocks > 1) {
        double sq = 0.0;
        for (double v : means) sq += (v - m) * (v - m);
        e = std::sqrt(sq / ((double)blocks * (double)(blocks - 1)));
    }
    mean = m;
    se = e;
    return true;
}

// block_slope_and_error / linear_slope, src/Swarm.cpp:136-197
static bool block_slope_and_error(const double* x, size_t n, double dt, size_t blocks, double& slope, double& se) {
    if (blocks == 0 || n % blocks != 0 || n / blocks < 2) return false;
    const size_t bs = n / blocks;
    std::vector<double> slopes(blocks);
    for (size_t b = 0; b < blocks; ++b) {
        const size_t begin = b * bs, count = bs;
        const double mean_index = 0.5 * (double)(count - 1);
        double cov = 0.0, iv = 0.0, mv = 0.0;
        for (size_t i = begin; i < begin + count; ++i) mv += x[i];
        mv /= (double)count;
        for (size_t l = 0; l < count; ++l) {
            const double ci = (double)l - mean_index;
            cov += ci * (x[begin + l] - mv);
            iv += ci * ci;
        }
        slopes[b] = cov / (iv * dt);
    }
    double m = 0.0;
    for (double v : slopes) m += v;
    m /= (double)blocks;
    double e = 0.0;
    if (blocks > 1) {
        double sq = 0.0;
        for (double v : slopes) sq += (v - m) * (v - m);
        e = std::sqrt(sq / ((double)blocks * (double)(blocks - 1)));
    }
    slope = m;
    se = e;
    return true;
}

// Largest |v|^2 whose kinetic_energy_ev (0.5 m |v|^2 / e, src/Swarm.cpp:95-101)
// does not exceed e_max: the energy checks of src/Swarm.cpp:1011-1037 become
// comparisons of |v|^2 with this value.
static double s2_threshold(double e_max) {
    auto f = [](double s2) { return 0.5 * kElectronMass * s2 / kEvToJ; };
    uint64_t lo = 0, hi = 0x7FF0000000000000ull;  // f(0) <= e_max < f(inf)
    while (hi - lo > 1) {
        const uint64_t mid = lo + (hi - lo) / 2;
        double x;
        std::memcpy(&x, &mid, 8);
        if (f(x) <= e_max) lo = mid; else hi = mid;
    }
    double r;
    std::memcpy(&r, &lo, 8);
    return r;
}

// effective_population_limit, src/Swarm.cpp:237-260
static size_t population_limit(size_t particles, size_t requested) {
    if (requested != 0) return requested;
    if (particles >= kAllocationLimit) return particles;
    const size_t source = kAllocationLimit - particles;
    const size_t doubled = particles > source / 2 ? source : 2 * particles;
    const size_t buffer = std::min<size_t>(source, 1024);
    const size_t buffered = particles > source - buffer ? source : particles + 1024;
    return std::min(source, std::max(doubled, buffered));
}

// First-fit allocator over one device block (offsets aligned to 256 bytes).
struct Pool {
    char* base = nullptr;
    size_t size = 0;
    std::map<size_t, size_t> free_;  // offset -> length

    void init(char* b, size_t s) {
        base = b;
        size = s;
        free_.clear();
        free_[0] = s;
    }
    static size_t round(size_t x) { return (x + 255) & ~(size_t)255; }
    char* alloc(size_t bytes) {
        bytes = round(std::max<size_t>(bytes, 1));
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= bytes) {
                const size_t off = it->first, len = it->second;
                free_.erase(it);
                if (len > bytes) free_[off + bytes] = len - bytes;
                return base + off;
            }
        }
        return nullptr;
    }
    void release(char* p, size_t bytes) {
        bytes = round(std::max<size_t>(bytes, 1));
        size_t off = (size_t)(p - base);
        auto next = free_.lower_bound(off);
        if (next != free_.end() && off + bytes == next->first) {
            bytes += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                prev->second += bytes;
                return;
            }
        }
        free_[off] = bytes;
    }
};

struct Request {
    uint64_t id;
    apic_swarm_request req;
    double submitted;      // host clock, seconds
};

struct Run {
    bool used = false;
    uint64_t id = 0;
    apic_swarm_request req{};
    RunCfg cfg{};
    std::vector<std::pair<char*, size_t>> blocks;
    size_t last_check_step = 0;
    std::vector<double> hv, he;  // host copies of the velocity and energy samples so far
    double submitted = 0.0;
    double admitted = 0.0;
};

static double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Server {
    apic_swarm_server_config conf{};
    std::string last_error;
    int device = 0;
    cudaStream_t stream = nullptr;
    // host <-> device bytes of the serving loop (run set-up, tables, samples, results)
    uint64_t h2d_bytes = 0, d2h_bytes = 0;
    void copy_h2d(void* dst, const void* src, size_t bytes) {
        APIC_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream));
        h2d_bytes += bytes;
    }
    void copy_d2h(void* dst, const void* src, size_t bytes) {
        APIC_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream));
        d2h_bytes += bytes;
    }
    std::vector<void*> allocations;
    MccModelDev model{};
    double neutral_density = 0.0, max_frequency = 0.0;
    bool fp32 = false;
    Pool pool;
    size_t max_chunks = 0;
    // device tables
    RunCfg* d_cfg = nullptr;
    RunState* d_st = nullptr;
    uint32_t* d_chunk_run = nullptr;
    uint32_t* d_chunk_first = nullptr;
    uint32_t* d_nchunks = nullptr;
    ChunkPartial* d_part = nullptr;
    Candidate* d_queue = nullptr;
    MccModelDev* d_model = nullptr;
    MccModel32* d_model32 = nullptr;
    unsigned* d_qlen = nullptr;
    size_t qcap = 0;
    // host mirrors
    std::vector<Run> runs;
    std::vector<RunState> h_st;
    std::vector<uint32_t> h_chunk_run, h_chunk_first;
    std::deque<Request> queue;
    std::map<uint64_t, apic_swarm_result> done;
    uint64_t next_id = 1;
    bool tables_dirty = true;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int push_grid = 0;
    uint64_t launches = 0;
    uint64_t kernel_launches = 0;  // step kernels launched (graph nodes included)
    uint64_t particle_steps = 0;
    // optional timing of the push kernel (kernels launched one by one, no graph)
    bool timing = false;
    double push_ms = 0.0, collide_ms = 0.0, push_bytes = 0.0;
    uint64_t push_launches = 0;

    ~Server() {
        if (stream) cudaStreamSynchronize(stream);
        if (h_st_pinned) cudaFreeHost(h_st_pinned);
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        if (graph_exec_fixed) cudaGraphExecDestroy(graph_exec_fixed);
        if (graph_fixed) cudaGraphDestroy(graph_fixed);
        for (void* a : allocations) cudaFree(a);
        if (stream) cudaStreamDestroy(stream);
    }

    Batch batch() const {
        Batch b;
        b.cfg = d_cfg;
        b.st = d_st;
        b.chunk_run = d_chunk_run;
        b.chunk_first = d_chunk_first;
        b.nchunks = d_nchunks;
        b.part = d_part;
        b.queue = d_queue;
        b.qlen = d_qlen;
        b.qcap = (unsigned)qcap;
        b.max_runs = conf.max_runs;
        b.model = d_model;
        b.model32 = d_model32;
        return b;
    }

    void create(const apic_swarm_server_config& c, const apic_mcc_model& gas) {
        conf = c;
        require(c.max_runs >= 1 && c.max_runs <= 4096, "max_runs must be between 1 and 4096");
        require(c.memory_budget_bytes >= (size_t)1 << 20, "memory_budget_bytes must be at least 1 MiB");
        require(c.precision == APIC_FP64 || c.precision == APIC_FP32, "unknown precision");
        require(c.steps_per_launch >= 1 && c.steps_per_launch <= 4096, "steps_per_launch must be between 1 and 4096");
        fp32 = c.precision == APIC_FP32;
        APIC_CUDA(cudaGetDevice(&device));
        APIC_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        // collision_config, src/Swarm.cpp:520-557: electrons on the dataset's channels
        require(gas.nch >= 1, "swarm gas dataset has no collision channels");
        bool has_elastic = false;
        for (int i = 0; i < gas.nch && i < kMaxChannels; ++i) {
            require(gas.ch[i].process != APIC_CHARGE_EXCHANGE,
                    "electron swarm benchmark does not support charge-exchange channels");
            require(gas.ch[i].energy_frame == APIC_FRAME_PROJECTILE,
                    "electron swarm benchmark requires projectile-frame cross-section energy");
            has_elastic = has_elastic || gas.ch[i].process == APIC_ELASTIC;
        }
        require(has_elastic, "electron swarm benchmark requires an elastic channel");
        require(std::isfinite(gas.neutral_density) && gas.neutral_density > 0,
                "swarm neutral_density must be positive and finite");
        require(std::isfinite(gas.max_frequency) && gas.max_frequency > 0,
                "swarm max_frequency must be positive and finite");
        require(std::isfinite(gas.neutral_temperature) && gas.neutral_temperature >= 0,
                "swarm neutral_temperature must be finite and non-negative");
        apic_mcc_model m = gas;
        m.species = 0;
        m.gas_units_si = 1;
        if (m.max_candidates == 0) m.max_candidates = 64;
        DeviceArena arena{allocations, stream};
        build_model(m, kElectronMass, arena, model);
        neutral_density = m.neutral_density;
        max_frequency = m.max_frequency;
        d_model = arena.upload(&model, 1);
        MccModel32 model32;
        build_model32(m, arena, model, model32);
        d_model32 = arena.upload(&model32, 1);
        APIC_CUDA(cudaStreamSynchronize(stream));
        // the collision-candidate queue has one entry per electron the pool can
        // hold (every electron of a step may be a candidate)
        const size_t per_electron = 6 * (fp32 ? 4 : 8);
        qcap = std::min<size_t>(c.memory_budget_bytes / (per_electron + sizeof(Candidate)), 0xFFFFFFF0u);
        d_queue = arena.alloc<Candidate>(qcap);
        d_qlen = arena.alloc<unsigned>(1);
        const size_t pool_bytes = c.memory_budget_bytes - qcap * sizeof(Candidate);
        char* pool_base = arena.alloc<char>(pool_bytes);
        pool.init(pool_base, pool_bytes);
        const size_t min_bytes = (fp32 ? 4 : 8) * 6 * (size_t)kChunk;
        max_chunks = pool_bytes / min_bytes + (size_t)c.max_runs + 1;
        d_cfg = arena.alloc<RunCfg>(c.max_runs);
        d_st = arena.alloc<RunState>(c.max_runs);
        d_chunk_run = arena.alloc<uint32_t>(max_chunks);
        d_chunk_first = arena.alloc<uint32_t>(max_chunks);
        d_nchunks = arena.alloc<uint32_t>(1);
        d_part = arena.alloc<ChunkPartial>(max_chunks);
        runs.resize(c.max_runs);
        h_st.resize(c.max_runs);
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        push_grid = sms * 4;
        APIC_CUDA(cudaStreamSynchronize(stream));
    }

    void validate(const apic_swarm_request& r) const {
        auto pf = [](double x) { return std::isfinite(x) && x > 0.0; };
        require(pf(r.timestep), "swarm timestep must be positive and finite");
        require(max_frequency * r.timestep <= 0.1, "swarm max_frequency * timestep must not exceed 0.1");
        require(r.steps > 0 && r.burn_in_steps < r.steps, "swarm steps must exceed burn_in_steps");
        require(r.particles > 0, "swarm particles must be positive");
        require(r.particles <= kAllocationLimit, "swarm particles exceeds the safety limit of 10000000");
        require(r.steps <= 0xFFFFFF00u, "swarm steps out of range");
        const size_t sampling = r.steps - r.burn_in_steps;
        require(r.uncertainty_blocks >= 1 && r.uncertainty_blocks <= sampling,
                "swarm uncertainty_blocks must be between 1 and the number of sampling steps");
        require(sampling % r.uncertainty_blocks == 0, "swarm sampling steps must be divisible by uncertainty_blocks");
        require(r.population_model == APIC_SWARM_FIXED || r.population_model == APIC_SWARM_BRANCHING,
                "unknown swarm population_model");
        bool has_ion = false, has_att = false;
        for (int i = 0; i < model.nch; ++i) {
            has_ion = has_ion || model.ch[i].process == kIonization;
            has_att = has_att || model.ch[i].process == kAttachment;
        }
        if (r.population_model == APIC_SWARM_FIXED) {
            require(r.population_limit == 0,
                    "swarm population_limit is valid only for population_model = branching_resampled");
            require(!has_att, "fixed-population swarm does not support attachment; use population_model = "
                              "branching_resampled");
        } else {
            const size_t lim = population_limit(r.particles, r.population_limit);
            require(lim > r.particles && lim <= kAllocationLimit - r.particles,
                    "branching swarm population_limit must exceed particles and population_limit + particles must "
                    "not exceed the allocation safety limit of 10000000");
            require(sampling / r.uncertainty_blocks >= 2,
                    "branching swarm requires at least two sampling steps per uncertainty block");
            require(has_ion || has_att, "branching swarm requires an ionization or attachment channel");
        }
        require(std::isfinite(r.initial_mean_energy_ev) && r.initial_mean_energy_ev >= 0,
                "swarm initial_mean_energy_ev must be finite and non-negative");
        require(pf(r.max_energy_ev), "swarm max_energy_ev must be positive and finite");
        for (int i = 0; i < model.nch; ++i) {  // src/Swarm.cpp:455-477
            require(!(r.max_energy_ev > host_table_max_[i] / kEvToJ),
                    "swarm max_energy_ev exceeds channel table coverage");
            require(!(host_mu_max_[i] > 0.0 && r.max_energy_ev > host_mu_max_[i] / kEvToJ),
                    "swarm max_energy_ev exceeds channel angular table coverage");
        }
        require(std::isfinite(r.reduced_field_td) && r.reduced_field_td >= 0,
                "swarm reduced fields must be finite and non-negative");
        require(std::isfinite(r.reduced_field_td * kTownsend * neutral_density),
                "swarm reduced field and neutral density overflow the electric field");
        require(std::isfinite(r.tolerance) && r.tolerance >= 0, "swarm tolerance must be finite and non-negative");
    }
    double host_table_max_[kMaxChannels] = {0, 0, 0, 0, 0, 0, 0, 0};
    double host_mu_max_[kMaxChannels] = {0, 0, 0, 0, 0, 0, 0, 0};

    size_t run_bytes(const apic_swarm_request& r) const {
        const size_t es = fp32 ? 4 : 8;
        const size_t n = r.particles;
        const size_t nch = (n + kChunk - 1) / kChunk;
        size_t bytes = Pool::round(6 * n * es) + Pool::round(3 * (r.steps - r.burn_in_steps) * sizeof(double));
        if (r.population_model == APIC_SWARM_BRANCHING) {
            const size_t lim = population_limit(n, r.population_limit);
            bytes += Pool::round(6 * lim * es) + Pool::round(3 * nch * kChunk * es) +
                     Pool::round(nch * kChunk * sizeof(uint32_t)) + Pool::round(n);
        }
        return bytes;
    }

    // Admits queued requests (first that fits, in arrival order) while slots,
    // chunk-table room and pool memory allow.
    int admit() {
        int admitted = 0;
        size_t used_chunks = h_chunk_run.size();
        size_t electrons = 0;  // the candidate queue holds one entry per active electron
        for (int s = 0; s < conf.max_runs; ++s)
            if (runs[s].used) electrons += runs[s].req.particles;
        for (auto it = queue.begin(); it != queue.end();) {
            int slot = -1;
            for (int s = 0; s < conf.max_runs; ++s)
                if (!runs[s].used) { slot = s; break; }
            if (slot < 0) break;
            const apic_swarm_request& r = it->req;
            const size_t nch = (r.particles + kChunk - 1) / kChunk;
            if (used_chunks + nch > max_chunks || electrons + r.particles > qcap) { ++it; continue; }
            if (!place(slot, *it)) { ++it; continue; }
            used_chunks += nch;
            electrons += r.particles;
            it = queue.erase(it);
            ++admitted;
        }
        return admitted;
    }

    bool place(int slot, const Request& q) {
        const apic_swarm_request& r = q.req;
        Run& run = runs[slot];
        const size_t es = fp32 ? 4 : 8;
        const size_t n = r.particles;
        const size_t nch = (n + kChunk - 1) / kChunk;
        const bool br = r.population_model == APIC_SWARM_BRANCHING;
        const size_t lim = br ? population_limit(n, r.population_limit) : n;
        std::vector<std::pair<char*, size_t>> blocks;
        auto take = [&](size_t bytes) -> char* {
            char* p = pool.alloc(bytes);
            if (p) blocks.push_back({p, bytes});
            return p;
        };
        char* a = take(6 * n * es);
        char* smp = take(3 * (r.steps - r.burn_in_steps) * sizeof(double));
        char *bb = nullptr, *sb = nullptr, *kb = nullptr, *al = nullptr;
        if (br) {
            bb = take(6 * lim * es);
            sb = take(3 * nch * kChunk * es);
            kb = take(nch * kChunk * sizeof(uint32_t));
            al = take(n);
        }
        if (!a || !smp || (br && (!bb || !sb || !kb || !al))) {
            for (auto& blk : blocks) pool.release(blk.first, blk.second);
            return false;
        }
        RunCfg& C = run.cfg;
        C = RunCfg{};
        const double E = r.reduced_field_td * kTownsend * neutral_density;
        const double acceleration = -kEvToJ * E / kElectronMass;
        C.half_kick = 0.5 * acceleration * r.timestep;
        // fixed-point scales: |v_x| <= v(max_energy_ev) and energy <= max_energy_ev
        // for every electron of a healthy run, so n such terms stay below 2^61
        const double vmax = std::sqrt(2.0 * r.max_energy_ev * kEvToJ / kElectronMass);
        C.s2_max = s2_threshold(r.max_energy_ev);
        C.vscale = std::ldexp(1.0, (int)std::floor(std::log2(std::ldexp(1.0, 61) / ((double)n * vmax))));
        C.escale = std::ldexp(1.0, (int)std::floor(std::log2(std::ldexp(1.0, 61) / ((double)n * C.s2_max))));
        draw_threshold(max_frequency, r.timestep, C.cand_draw_min, C.no_candidates);
        C.dt = r.timestep;
        C.max_energy_ev = r.max_energy_ev;
        C.init_sd = std::sqrt(2.0 * r.initial_mean_energy_ev * kEvToJ / (3.0 * kElectronMass));
        C.seed = r.seed;
        C.n = (uint32_t)n;
        C.steps = (uint32_t)r.steps;
        C.burn_in = (uint32_t)r.burn_in_steps;
        C.nchunks = (uint32_t)nch;
        C.limit = (uint32_t)lim;
        C.branching = br ? 1 : 0;
        for (int k = 0; k < 3; ++k) {
            C.v[k] = a + (size_t)k * n * es;
            C.d[k] = a + (size_t)(3 + k) * n * es;
            if (br) {
                C.bv[k] = bb + (size_t)k * lim * es;
                C.bd[k] = bb + (size_t)(3 + k) * lim * es;
                C.sv[k] = sb + (size_t)k * nch * kChunk * es;
            }
        }
        C.skey = reinterpret_cast<uint32_t*>(kb);
        C.alive = reinterpret_cast<uint8_t*>(al);
        C.samples = reinterpret_cast<double*>(smp);
        run.used = true;
        run.id = q.id;
        run.req = r;
        run.blocks = std::move(blocks);
        run.last_check_step = 0;
        run.submitted = q.submitted;
        run.admitted = now_s();
        RunState S{};
        S.active = 1;
        S.weight = 1.0;
        h_st[slot] = S;
        copy_h2d(d_st + slot, &h_st[slot], sizeof S);
        if (fp32) k_swarm_init<float><<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, stream>>>(C);
        else k_swarm_init<double><<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, stream>>>(C);
        APIC_CUDA(cudaGetLastError());
        tables_dirty = true;
        return true;
    }

    void rebuild_tables() {
        h_chunk_run.clear();
        h_chunk_first.clear();
        for (int s = 0; s < conf.max_runs; ++s) {
            Run& r = runs[s];
            if (!r.used) continue;
            r.cfg.first_chunk = (uint32_t)h_chunk_run.size();
            for (uint32_t k = 0; k < r.cfg.nchunks; ++k) {
                h_chunk_run.push_back((uint32_t)s);
                h_chunk_first.push_back(k * kChunk);
            }
            copy_h2d(d_cfg + s, &r.cfg, sizeof(RunCfg));
        }
        const uint32_t nc = (uint32_t)h_chunk_run.size();
        if (nc) {
            copy_h2d(d_chunk_run, h_chunk_run.data(), nc * sizeof(uint32_t));
            copy_h2d(d_chunk_first, h_chunk_first.data(), nc * sizeof(uint32_t));
        }
        nchunks_host_ = nc;
        copy_h2d(d_nchunks, &nchunks_host_, sizeof(uint32_t));
        // the host copies above read pageable host memory: wait before it changes
        APIC_CUDA(cudaStreamSynchronize(stream));
        tables_dirty = false;
    }
    uint32_t nchunks_host_ = 0;

    template <class T>
    void enqueue_step(const Batch& b, bool branching) {
        k_swarm_push<T><<<push_grid, kThreads, 0, stream>>>(b);
        k_swarm_collide<T><<<push_grid, kThreads, 0, stream>>>(b);
        if (branching) {
            k_swarm_branch_scan<<<conf.max_runs, kThreads, 0, stream>>>(b);
            k_swarm_branch_compact<T><<<push_grid, kThreads, 0, stream>>>(b);
            k_swarm_branch_resample<T><<<push_grid, kThreads, 0, stream>>>(b);
        }
        k_swarm_reduce<<<conf.max_runs, kThreads, 0, stream>>>(b);
    }

    // Two step graphs: with the branching kernels, for batches holding a
    // branching run, and without them.
    cudaGraph_t graph_fixed = nullptr;
    cudaGraphExec_t graph_exec_fixed = nullptr;

    cudaGraphExec_t ensure_graph(bool branching) {
        cudaGraph_t& g = branching ? graph : graph_fixed;
        cudaGraphExec_t& ge = branching ? graph_exec : graph_exec_fixed;
        if (ge) return ge;
        const Batch b = batch();
        APIC_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        for (size_t k = 0; k < conf.steps_per_launch; ++k) {
            if (fp32) enqueue_step<float>(b, branching);
            else enqueue_step<double>(b, branching);
        }
        APIC_CUDA(cudaStreamEndCapture(stream, &g));
        APIC_CUDA(cudaGraphInstantiate(&ge, g, 0));
        return ge;
    }

    // Finishes a run whose device state says it stopped (steps done, converged
    // or failed): statistics from its samples, diffusion from its displacements.
    void retire(int slot, bool converged) {
        Run& run = runs[slot];
        RunState& S = h_st[slot];
        const apic_swarm_request& r = run.req;
        apic_swarm_result out{};
        out.id = run.id;
        out.reduced_field_td = r.reduced_field_td;
        const double E = r.reduced_field_td * kTownsend * neutral_density;
        out.electric_field_v_m = E;
        out.steps_done = S.step;
        out.converged = converged ? 1 : 0;
        out.initial_weight = (double)r.particles;
        out.diffusion_available = r.population_model == APIC_SWARM_FIXED;
        out.nch = model.nch;
        out.status = APIC_OK;
        if (S.error) {
            out.status = (S.error & (kErrMajorant)) ? APIC_ERR_MAJORANT
                         : (S.error & kErrCandidates) ? APIC_ERR_CANDIDATES
                         : (S.error & (kErrPopulation | kErrBirths)) ? APIC_ERR_CAPACITY
                         : (S.error & kErrNonFinite) ? APIC_ERR_NONFINITE
                                                     : APIC_ERR_INVALID;
            std::string msg;
            if (S.error & kErrMaxEnergyPre) msg += "swarm particle energy exceeded max_energy_ev before collision lookup; ";
            if (S.error & kErrMaxEnergy) msg += "swarm particle energy exceeded max_energy_ev; ";
            if (S.error & kErrMajorant) msg += "MCC total collision frequency exceeds configured max_frequency; ";
            if (S.error & kErrCandidates) msg += "MCC candidate limit exceeded; ";
            if (S.error & kErrPopulation) msg += "branching swarm exceeded population_limit before resampling; ";
            if (S.error & kErrExtinct) msg += "branching swarm electron ensemble became extinct; ";
            if (S.error & kErrBirths) msg += "ionization secondaries exceeded the per-chunk staging buffer; ";
            if (S.error & kErrNonFinite) msg += "electron velocity became non-finite; ";
            std::snprintf(out.message, sizeof out.message, "%s", msg.c_str());
        }
        const size_t steps_done = S.step;
        const size_t ns = steps_done > r.burn_in_steps ? steps_done - r.burn_in_steps : 0;
        const size_t total_ns = r.steps - r.burn_in_steps;
        if (out.status == APIC_OK && ns > 0) {
            std::vector<double> smp(3 * total_ns);
            copy_d2h(smp.data(), run.cfg.samples, smp.size() * sizeof(double));
            if (r.population_model == APIC_SWARM_FIXED) {
                if (fp32) k_swarm_moments<float><<<1, kThreads, 0, stream>>>(run.cfg, d_st + slot);
                else k_swarm_moments<double><<<1, kThreads, 0, stream>>>(run.cfg, d_st + slot);
                APIC_CUDA(cudaGetLastError());
            }
            copy_d2h(&S, d_st + slot, sizeof S);
            APIC_CUDA(cudaStreamSynchronize(stream));
            const double* vs = smp.data();
            const double* es = smp.data() + total_ns;
            const double* ls = smp.data() + 2 * total_ns;
            const size_t blocks = std::min(r.uncertainty_blocks, ns);
            double m = 0, e = 0;
            block_mean_and_error(vs, ns, blocks, m, e);
            out.mean_velocity_x = m;
            out.mean_velocity_x_se = e;
            out.drift_velocity = -m;
            out.reduced_mobility = E == 0.0 ? 0.0 : out.drift_velocity * neutral_density / E;
            block_mean_and_error(es, ns, blocks, m, e);
            out.mean_energy_ev = m;
            out.mean_energy_se_ev = e;
            const double sampling_time = (double)ns * r.timestep;
            if (out.diffusion_available) {
                out.diffusion_longitudinal = S.var_l / (2.0 * sampling_time);
                out.diffusion_transverse = S.var_t / (4.0 * sampling_time);
            }
            for (int c = 0; c < model.nch; ++c) {
                out.channel_collisions[c] = S.counts[c];
                out.channel_rate[c] = S.wcoll[c] / S.exposure;
                out.channel_rate_se[c] = std::sqrt(S.wcoll2[c]) / S.exposure;
                if (model.ch[c].process == kIonization) {
                    out.ionization_rate += out.channel_rate[c];
                    out.ionization_rate_se = std::hypot(out.ionization_rate_se, out.channel_rate_se[c]);
                } else if (model.ch[c].process == kAttachment) {
                    out.attachment_rate += out.channel_rate[c];
                    out.attachment_rate_se = std::hypot(out.attachment_rate_se, out.channel_rate_se[c]);
                }
            }
            out.net_rate = out.ionization_rate - out.attachment_rate;
            out.net_rate_se = std::hypot(out.ionization_rate_se, out.attachment_rate_se);
            out.final_weight = (double)r.particles * S.weight;
            out.final_particles = r.particles;
            if (r.population_model == APIC_SWARM_BRANCHING) {
                double g = 0, ge = 0;
                if (block_slope_and_error(ls, ns, r.timestep, blocks, g, ge)) {
                    out.growth_rate = g;
                    out.growth_rate_se = ge;
                    if (out.drift_velocity > 0.0) {
                        const double drift = out.drift_velocity, de = out.mean_velocity_x_se;
                        out.townsend_available = 1;
                        out.townsend_growth = g / drift;
                        out.townsend_growth_se = std::hypot(ge / drift, g * de / (drift * drift));
                        out.townsend_rate = out.net_rate / drift;
                        out.townsend_rate_se =
                            std::hypot(out.net_rate_se / drift, out.net_rate * de / (drift * drift));
                    }
                }
            }
            out.candidates = S.candidates;
            out.null_collisions = S.nulls;
        }
        out.max_observed_energy_ev = S.max_ev;
        const double t = now_s();
        out.latency_s = t - run.submitted;
        out.queue_s = run.admitted - run.submitted;
        done[run.id] = out;
        for (auto& blk : run.blocks) pool.release(blk.first, blk.second);
        run = Run{};
        RunState off{};
        h_st[slot] = off;
        copy_h2d(d_st + slot, &h_st[slot], sizeof(RunState));
        APIC_CUDA(cudaStreamSynchronize(stream));
        tables_dirty = true;
    }

    // Convergence: the relative block standard errors of drift velocity and
    // mean energy over the samples so far at most `tolerance`.
    bool converged(int slot) {
        const Run& run = runs[slot];
        const apic_swarm_request& r = run.req;
        if (!(r.tolerance > 0.0)) return false;
        const size_t step = h_st[slot].step;
        if (step <= r.burn_in_steps) return false;
        const size_t ns = step - r.burn_in_steps;
        if (ns < 4 * r.uncertainty_blocks) return false;
        const size_t total_ns = r.steps - r.burn_in_steps;
        Run& rw = runs[slot];
        const size_t have = rw.hv.size();
        rw.hv.resize(ns);
        rw.he.resize(ns);
        copy_d2h(rw.hv.data() + have, run.cfg.samples + have, (ns - have) * sizeof(double));
        copy_d2h(rw.he.data() + have, run.cfg.samples + total_ns + have, (ns - have) * sizeof(double));
        APIC_CUDA(cudaStreamSynchronize(stream));
        double mv, sv, me, se;
        block_mean_and_error(rw.hv.data(), ns, r.uncertainty_blocks, mv, sv);
        block_mean_and_error(rw.he.data(), ns, r.uncertainty_blocks, me, se);
        return sv <= r.tolerance * std::fabs(mv) && se <= r.tolerance * std::fabs(me);
    }

    // One serving iteration: admit, run steps_per_launch steps of every active
    // run (one graph launch), read the run states, retire finished runs.
    // advance = launch + complete; between the two the host may queue other
    // work (other streams) that overlaps this batch on the GPU.
    void advance(int* active_out, int* queued_out) {
        launch();
        complete(active_out, queued_out);
    }

    RunState* h_st_pinned = nullptr;  // async read-back target of the run states
    bool launched = false;

    void launch() {
        require(!launched, "launch() while a launched batch has not completed", APIC_ERR_STATE);
        admit();
        if (tables_dirty) rebuild_tables();
        int active = 0;
        for (int s = 0; s < conf.max_runs; ++s) active += runs[s].used ? 1 : 0;
        if (active && timing) {
            // algorithmic bytes of each push: velocity read + write, and the
            // displacement read + write during sampling steps
            const size_t es = fp32 ? 4 : 8;
            const Batch b = batch();
            struct Ev3 { cudaEvent_t first, second, third; };
            std::vector<Ev3> ev(conf.steps_per_launch);
            for (size_t k = 0; k < conf.steps_per_launch; ++k) {
                for (int s = 0; s < conf.max_runs; ++s) {
                    const Run& run = runs[s];
                    if (!run.used || !h_st[s].active) continue;
                    const size_t st = h_st[s].step + k;
                    if (st >= run.req.steps) continue;
                    push_bytes += (double)run.req.particles * es * (st >= run.req.burn_in_steps ? 12 : 6);
                }
                APIC_CUDA(cudaEventCreate(&ev[k].first));
                APIC_CUDA(cudaEventCreate(&ev[k].second));
                APIC_CUDA(cudaEventCreate(&ev[k].third));
                APIC_CUDA(cudaEventRecord(ev[k].first, stream));
                if (fp32) k_swarm_push<float><<<push_grid, kThreads, 0, stream>>>(b);
                else k_swarm_push<double><<<push_grid, kThreads, 0, stream>>>(b);
                APIC_CUDA(cudaEventRecord(ev[k].second, stream));
                if (fp32) k_swarm_collide<float><<<push_grid, kThreads, 0, stream>>>(b);
                else k_swarm_collide<double><<<push_grid, kThreads, 0, stream>>>(b);
                APIC_CUDA(cudaEventRecord(ev[k].third, stream));
                k_swarm_branch_scan<<<conf.max_runs, kThreads, 0, stream>>>(b);
                if (fp32) {
                    k_swarm_branch_compact<float><<<push_grid, kThreads, 0, stream>>>(b);
                    k_swarm_branch_resample<float><<<push_grid, kThreads, 0, stream>>>(b);
                } else {
                    k_swarm_branch_compact<double><<<push_grid, kThreads, 0, stream>>>(b);
                    k_swarm_branch_resample<double><<<push_grid, kThreads, 0, stream>>>(b);
                }
                k_swarm_reduce<<<conf.max_runs, kThreads, 0, stream>>>(b);
                APIC_CUDA(cudaGetLastError());
            }
            APIC_CUDA(cudaStreamSynchronize(stream));
            for (auto& e : ev) {
                float ms = 0.f, ms2 = 0.f;
                APIC_CUDA(cudaEventElapsedTime(&ms, e.first, e.second));
                APIC_CUDA(cudaEventElapsedTime(&ms2, e.second, e.third));
                push_ms += ms;
                collide_ms += ms2;
                ++push_launches;
                cudaEventDestroy(e.first);
                cudaEventDestroy(e.second);
                cudaEventDestroy(e.third);
            }
        }
        if (active) {
            bool branching = false;
            for (int s = 0; s < conf.max_runs; ++s)
                branching = branching || (runs[s].used && runs[s].cfg.branching);
            if (!timing) APIC_CUDA(cudaGraphLaunch(ensure_graph(branching), stream));
            kernel_launches += conf.steps_per_launch * (timing || branching ? 6 : 3);
            ++launches;
            if (!h_st_pinned) APIC_CUDA(cudaMallocHost(&h_st_pinned, h_st.size() * sizeof(RunState)));
            copy_d2h(h_st_pinned, d_st, h_st.size() * sizeof(RunState));
            launched = true;
        }
    }

    void complete(int* active_out, int* queued_out) {
        if (launched) {
            launched = false;
            const cudaError_t w = bounded_wait(stream, 600.0);
            if (w == cudaErrorNotReady) throw Error(APIC_ERR_TIMEOUT, "swarm step did not complete in time");
            APIC_CUDA(w);
            std::memcpy(h_st.data(), h_st_pinned, h_st.size() * sizeof(RunState));
            for (int s = 0; s < conf.max_runs; ++s) {
                Run& run = runs[s];
                if (!run.used) continue;
                const size_t advanced = h_st[s].step - run.last_check_step;
                particle_steps += advanced * run.req.particles;
                run.last_check_step = h_st[s].step;
                if (!h_st[s].active) {
                    retire(s, false);
                } else if (converged(s)) {
                    retire(s, true);
                }
            }
        }
        int active = 0;
        for (int s = 0; s < conf.max_runs; ++s) active += runs[s].used ? 1 : 0;
        if (active_out) *active_out = active;
        if (queued_out) *queued_out = (int)queue.size();
    }

    uint64_t submit(const apic_swarm_request& r) {
        validate(r);
        require(run_bytes(r) <= pool.size && r.particles <= qcap,
                "swarm request does not fit the server's memory budget", APIC_ERR_CAPACITY);
        require((r.particles + kChunk - 1) / kChunk + 1 <= max_chunks, "swarm request exceeds the chunk table",
                APIC_ERR_CAPACITY);
        Request q;
        q.id = next_id++;
        q.req = r;
        q.submitted = now_s();
        queue.push_back(q);
        return q.id;
    }
};

// ---- spatial Townsend pass (run_spatial_townsend, src/Swarm.cpp:645-938) ----------
//
// Each history starts from one electron injected toward the planes and follows
// its cascade until every electron has left [0, L).  One warp owns one history
// at a time and takes the next from a global counter when it is done, so the
// uneven cascades balance across the GPU without host round trips.  The
// history's population lives in three per-warp global buffers (current, next,
// births), structure of arrays (v_x, v_y, v_z, x); per step the lanes walk the
// population 32 at a time: half kick, energy check, drift, plane crossings
// (counted as integers per plane, then added as weight x count once per step,
// so the tally does not depend on the order of the lanes), exit test, MCC,
// half kick.  Survivors keep their order, the secondaries follow in parent
// order, and a population above the target is systematically resampled by
// index (every electron of a history carries one weight).
constexpr int kTownsendWarps = 8;
constexpr unsigned kErrNoTermination = 1u << 12;
constexpr unsigned kErrSecondaries = 1u << 13;
constexpr unsigned kErrWorkLimit = 1u << 14;

struct TownsendParams {
    const MccModelDev* model;
    uint64_t seed;
    double half_kick, dt, sd, max_energy_ev, length;
    const double* planes;  // bins
    unsigned H, bins, N, limit, max_steps;
    double* crossings;     // H x bins
    int* counts;           // warps x bins
    double* pop;           // warps x 3 buffers x 4 components x limit
    double* stage;         // warps x 32 lanes x kMaxBirthsPerElectron x 3
    unsigned long long* updates;  // H
    unsigned* max_active;         // H
    unsigned* next;
    unsigned* error;
    unsigned long long* work_used;  // particle updates of this pass so far
    unsigned long long work_left;   // spatial_work_item_limit minus the scan's earlier updates
};

// std::upper_bound over the plane positions
__device__ __forceinline__ unsigned upper_plane(const double* planes, unsigned n, double value) {
    unsigned lo = 0, hi = n;
    while (lo < hi) {
        const unsigned mid = (lo + hi) >> 1;
        if (value < __ldg(planes + mid)) hi = mid; else lo = mid + 1;
    }
    return lo;
}

__global__ void __launch_bounds__(kTownsendWarps * 32) k_townsend(TownsendParams P) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned warp_slot = blockIdx.x * kTownsendWarps + (threadIdx.x >> 5);
    const MccModelDev& M = *P.model;
    const size_t L = P.limit;
    int* cnt = P.counts + (size_t)warp_slot * P.bins;
    double* base = P.pop + (size_t)warp_slot * 12 * L;
    double* stage = P.stage + ((size_t)warp_slot * 32 + lane) * kMaxBirthsPerElectron * 3;
    const unsigned lt = (1u << lane) - 1u;
    for (;;) {
        unsigned h = 0;
        if (lane == 0) h = atomicAdd(P.next, 1u);
        h = __shfl_sync(full, h, 0);
        if (h >= P.H || *(volatile unsigned*)P.error) break;
        const uint32_t hs = 0x80000000u | h;
        double* cur = base;
        double* nxt = base + 4 * L;
        double* brn = base + 8 * L;
        double* row = P.crossings + (size_t)h * P.bins;
        if (lane == 0) {
            // the injected electron, src/Swarm.cpp:689-696
            PhiloxStream rng(P.seed, 0xFFFFFFFEu, 0u, hs);
            double unit = canonical(rng);
            if (unit < 2.2250738585072014e-308) unit = 2.2250738585072014e-308;
            const double inward = P.sd * sqrt(-2.0 * log(unit));
            NormalState ns;
            cur[0] = -inward;
            cur[L] = normal(ns, rng, 0.0, P.sd);
            cur[2 * L] = normal(ns, rng, 0.0, P.sd);
            cur[3 * L] = 0.0;
        }
        for (unsigned b = lane; b < P.bins; b += 32) {
            cnt[b] = 0;
            row[b] = 0.0;
        }
        __syncwarp();
        unsigned pop = 1, maxa = 0, err = 0;
        unsigned long long upd = 0;
        double w = 1.0;
        bool terminated = false;
        for (unsigned step = 0; step < P.max_steps; ++step) {
            if (pop == 0) {
                terminated = true;
                break;
            }
            const unsigned active = pop;
            maxa = max(maxa, active);
            upd += active;
            // the scan's work-item limit, src/Swarm.cpp:703-711
            unsigned over = 0;
            if (lane == 0) over = atomicAdd(P.work_used, (unsigned long long)active) + active > P.work_left;
            if (__shfl_sync(full, over, 0)) {
                err |= kErrWorkLimit;
                break;
            }
            unsigned ns = 0, nb = 0;
            for (unsigned b0 = 0; b0 < active; b0 += 32) {
                const unsigned i = b0 + lane;
                bool keep = false;
                unsigned births = 0;
                double v[3] = {0.0, 0.0, 0.0}, x = 0.0;
                if (i < active) {
                    v[0] = cur[i];
                    v[1] = cur[L + i];
                    v[2] = cur[2 * L + i];
                    x = cur[3 * L + i];
                    v[0] += P.half_kick;
                    if (ke_ev(v[0], v[1], v[2]) > P.max_energy_ev) {
                        err |= kErrMaxEnergyPre;
                    } else {
                        const double old_d = -x;
                        x += v[0] * P.dt;
                        const double new_d = -x;
                        if (new_d > old_d) {
                            const unsigned a = upper_plane(P.planes, P.bins, old_d);
                            const unsigned e = upper_plane(P.planes, P.bins, new_d);
                            for (unsigned k = a; k < e; ++k) atomicAdd(cnt + k, 1);
                        } else if (new_d < old_d) {
                            const unsigned a = upper_plane(P.planes, P.bins, new_d);
                            const unsigned e = upper_plane(P.planes, P.bins, old_d);
                            for (unsigned k = a; k < e; ++k) atomicAdd(cnt + k, -1);
                        }
                        if (!(new_d < 0.0 || new_d >= P.length)) {
                            PhiloxStream rng(P.seed, i, step, hs);
                            CollideResult r;
                            collide3(M, v, P.dt, rng, r,
                                     [&](int, const double* vs, const double*) {
                                         if (births < (unsigned)kMaxBirthsPerElectron) {
                                             stage[3 * births] = vs[0];
                                             stage[3 * births + 1] = vs[1];
                                             stage[3 * births + 2] = vs[2];
                                         }
                                         ++births;
                                     },
                                     false, 0.0);
                            err |= r.error;
                            v[0] += P.half_kick;
                            if (ke_ev(v[0], v[1], v[2]) > P.max_energy_ev) err |= kErrMaxEnergy;
                            if (births > (unsigned)kMaxBirthsPerElectron) err |= kErrSecondaries;
                            keep = !r.removed;
                        }
                    }
                }
                const unsigned ball = __ballot_sync(full, keep);
                if (keep) {
                    const unsigned o = ns + __popc(ball & lt);
                    nxt[o] = v[0];
                    nxt[L + o] = v[1];
                    nxt[2 * L + o] = v[2];
                    nxt[3 * L + o] = x;
                }
                ns += __popc(ball);
                unsigned incl = births;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const unsigned t = __shfl_up_sync(full, incl, o);
                    if (lane >= o) incl += t;
                }
                const unsigned total = __shfl_sync(full, incl, 31);
                // particles.size() >= population_limit before a push, src/Swarm.cpp:797-802
                if ((unsigned long long)active + nb + total > L) err |= kErrPopulation;
                if (!err && births) {
                    const unsigned at = nb + incl - births;
                    for (unsigned k = 0; k < births; ++k) {
                        brn[at + k] = stage[3 * k];
                        brn[L + at + k] = stage[3 * k + 1];
                        brn[2 * L + at + k] = stage[3 * k + 2];
                        brn[3 * L + at + k] = x;
                    }
                }
                nb += total;
                err = __reduce_or_sync(full, err);
                if (err) break;
            }
            if (err) break;
            __syncwarp();
            for (unsigned b = lane; b < P.bins; b += 32) {
                const int c = cnt[b];
                if (c) {
                    row[b] += w * (double)c;
                    cnt[b] = 0;
                }
            }
            for (unsigned k = lane; k < nb; k += 32) {
                nxt[ns + k] = brn[k];
                nxt[L + ns + k] = brn[L + k];
                nxt[2 * L + ns + k] = brn[2 * L + k];
                nxt[3 * L + ns + k] = brn[3 * L + k];
            }
            maxa = max(maxa, active + nb);
            pop = ns + nb;
            __syncwarp();
            if (pop > P.N) {
                // systematic_resample by index, src/Swarm.cpp:616-643
                double u = 0.0;
                if (lane == 0) {
                    PhiloxStream rng(P.seed, 0xFFFFFFFFu, step, hs);
                    u = uniform01(rng);
                }
                u = __shfl_sync(full, u, 0);
                for (unsigned q = lane; q < P.N; q += 32) {
                    const double t = (u + (double)q) * (double)pop / (double)P.N;
                    const double c = ceil(t) - 1.0;
                    unsigned j = c < 0.0 ? 0u : (unsigned)c;
                    if (j > pop - 1) j = pop - 1;
                    cur[q] = nxt[j];
                    cur[L + q] = nxt[L + j];
                    cur[2 * L + q] = nxt[2 * L + j];
                    cur[3 * L + q] = nxt[3 * L + j];
                }
                w = (double)pop * w / (double)P.N;
                pop = P.N;
                __syncwarp();
            } else {
                double* t = cur;
                cur = nxt;
                nxt = t;
            }
        }
        if (!err && !terminated && pop == 0) terminated = true;
        if (!err && !terminated) err |= kErrNoTermination;
        if (lane == 0) {
            P.updates[h] = upd;
            P.max_active[h] = maxa;
            if (err) atomicOr(P.error, err);
        }
        if (err) break;
    }
}

// validate_config's spatial section, src/Swarm.cpp:380-440
static void validate_spatial(const apic_swarm_config& c, const apic_spatial_townsend_config& sp) {
    if (sp.histories == 0) {
        require(sp.length_m == 0.0 && sp.bins == 0 && sp.fit_begin_bin == 0 && sp.fit_end_bin == 0 &&
                    sp.max_steps == 0 && sp.min_r_squared == 0.0,
                "spatial Townsend controls require positive spatial_histories");
        return;
    }
    require(c.population_model == APIC_SWARM_BRANCHING,
            "spatial Townsend estimation requires population_model = branching_resampled");
    require(std::isfinite(sp.length_m) && sp.length_m > 0.0, "spatial_length_m must be positive and finite");
    require(sp.bins >= 4, "spatial_bins must be at least 4");
    const size_t fit_end = sp.fit_end_bin == 0 ? sp.bins : sp.fit_end_bin;
    require(!(sp.fit_begin_bin >= fit_end || fit_end > sp.bins || fit_end - sp.fit_begin_bin < 3),
            "spatial Townsend fit range must contain at least three valid bins");
    require(sp.max_steps != 0, "spatial_max_steps and spatial_work_item_limit must be positive");
    require(!(sp.histories < c.uncertainty_blocks || c.uncertainty_blocks == 0 ||
              sp.histories % c.uncertainty_blocks != 0),
            "spatial_histories must be divisible by uncertainty_blocks");
    require(sp.histories <= 1000000 / sp.bins, "spatial history-profile allocation exceeds the safety limit");
    require(std::isfinite(sp.min_r_squared) && sp.min_r_squared >= 0.0 && sp.min_r_squared <= 1.0,
            "spatial_min_r_squared must be between 0 and 1");
}

// linear_slope, src/Swarm.cpp:136-163
static double linear_slope(const std::vector<double>& v, size_t begin, size_t end, double step) {
    const size_t count = end - begin;
    const double mean_index = 0.5 * (double)(count - 1);
    double cov = 0.0, iv = 0.0, mv = 0.0;
    for (size_t i = begin; i < end; ++i) mv += v[i];
    mv /= (double)count;
    for (size_t l = 0; l < count; ++l) {
        const double ci = (double)l - mean_index;
        cov += ci * (v[begin + l] - mv);
        iv += ci * ci;
    }
    return cov / (iv * step);
}

// slope_r_squared, src/Swarm.cpp:202-231
static double slope_r_squared(const std::vector<double>& v, size_t begin, size_t end) {
    const size_t count = end - begin;
    double mean = 0.0;
    for (size_t i = begin; i < end; ++i) mean += v[i];
    mean /= (double)count;
    const double mean_index = 0.5 * (double)(count - 1);
    double cov = 0.0, iv = 0.0, vv = 0.0;
    for (size_t l = 0; l < count; ++l) {
        const double ci = (double)l - mean_index, cv = v[begin + l] - mean;
        cov += ci * cv;
        iv += ci * ci;
        vv += cv * cv;
    }
    if (vv == 0.0) return 1.0;
    return std::clamp(cov * cov / (iv * vv), 0.0, 1.0);
}

// One field's spatial Townsend pass on the device; the flux statistics and
// the fit (src/Swarm.cpp:835-938) on the host from the per-history crossings.
static void spatial_townsend(const apic_swarm_config& c, const apic_spatial_townsend_config& sp,
                             const apic_mcc_model& gas, double td, uint64_t seed, uint64_t* scan,
                             apic_spatial_townsend_result* out, apic_spatial_flux_point* profile,
                             double* history_crossings) {
    validate_spatial(c, sp);
    std::memset(out, 0, sizeof *out);
    if (sp.histories == 0) return;
    require(c.particles > 0 && c.timestep > 0 && std::isfinite(c.timestep), "swarm particles and timestep must be positive");
    require(std::isfinite(c.max_energy_ev) && c.max_energy_ev > 0, "swarm max_energy_ev must be positive and finite");
    require(gas.nch >= 1, "swarm gas dataset has no collision channels");
    bool has_elastic = false;
    for (int i = 0; i < gas.nch && i < kMaxChannels; ++i) {
        require(gas.ch[i].process != APIC_CHARGE_EXCHANGE,
                "electron swarm benchmark does not support charge-exchange channels");
        require(gas.ch[i].energy_frame == APIC_FRAME_PROJECTILE,
                "electron swarm benchmark requires projectile-frame cross-section energy");
        has_elastic = has_elastic || gas.ch[i].process == APIC_ELASTIC;
    }
    require(has_elastic, "electron swarm benchmark requires an elastic channel");
    const size_t H = sp.histories, bins = sp.bins, N = c.particles;
    const size_t limit = population_limit(N, c.population_limit);
    require(limit < (1u << 30) && N <= limit, "swarm population limit out of range", APIC_ERR_UNSUPPORTED);

    std::vector<void*> allocations;
    cudaStream_t stream = nullptr;
    APIC_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    struct Release {
        std::vector<void*>& a;
        cudaStream_t s;
        ~Release() {
            cudaStreamSynchronize(s);
            for (void* p : a) cudaFree(p);
            cudaStreamDestroy(s);
        }
    } release{allocations, stream};
    DeviceArena arena{allocations, stream};
    apic_mcc_model m = gas;  // collision_config, src/Swarm.cpp:520-557
    m.species = 0;
    m.gas_units_si = 1;
    m.neutral_density = c.neutral_density;
    m.neutral_temperature = c.neutral_temperature;
    m.max_frequency = c.max_frequency;
    if (m.max_candidates == 0) m.max_candidates = 64;
    MccModelDev model{};
    build_model(m, kElectronMass, arena, model);

    const double spacing = sp.length_m / (double)(bins + 1);
    std::vector<double> planes(bins);
    for (size_t b = 0; b < bins; ++b) planes[b] = (double)(b + 1) * spacing;
    int device = 0, sms = 148;
    APIC_CUDA(cudaGetDevice(&device));
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    size_t free_b = 0, total_b = 0;
    APIC_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t per_warp = 12 * limit * sizeof(double) + bins * sizeof(int) +
                            32 * kMaxBirthsPerElectron * 3 * sizeof(double);
    const size_t budget = std::min<size_t>(free_b / 4, (size_t)8 << 30);
    size_t warps = std::min<size_t>(H, (size_t)sms * 4 * kTownsendWarps);
    warps = std::min(warps, std::max<size_t>(budget / per_warp, 1));
    const size_t blocks = (warps + kTownsendWarps - 1) / kTownsendWarps;
    warps = blocks * kTownsendWarps;
    require(warps * per_warp <= free_b, "spatial Townsend population buffers do not fit in device memory",
            APIC_ERR_CAPACITY);

    TownsendParams P{};
    P.model = arena.upload(&model, 1);
    P.seed = seed;
    const double E = td * kTownsend * c.neutral_density;  // src/Swarm.cpp:662-667
    P.half_kick = 0.5 * (-kEvToJ * E / kElectronMass) * c.timestep;
    P.dt = c.timestep;
    P.sd = std::sqrt(2.0 * c.initial_mean_energy_ev * kEvToJ / (3.0 * kElectronMass));
    P.max_energy_ev = c.max_energy_ev;
    P.length = sp.length_m;
    P.planes = arena.upload(planes.data(), bins);
    P.H = (unsigned)H;
    P.bins = (unsigned)bins;
    P.N = (unsigned)N;
    P.limit = (unsigned)limit;
    P.max_steps = (unsigned)std::min<size_t>(sp.max_steps, 0xFFFFFFFFu);
    P.crossings = arena.alloc<double>(H * bins);
    P.counts = arena.alloc<int>(warps * bins);
    P.pop = arena.alloc<double>(warps * 12 * limit);
    P.stage = arena.alloc<double>(warps * 32 * kMaxBirthsPerElectron * 3);
    P.updates = arena.alloc<unsigned long long>(H);
    P.max_active = arena.alloc<unsigned>(H);
    P.next = arena.alloc<unsigned>(1);
    P.error = arena.alloc<unsigned>(1);
    const uint64_t work_limit = sp.work_item_limit ? sp.work_item_limit : 100000000ull;
    require(*scan <= work_limit, "spatial Townsend scan exceeded spatial_work_item_limit");
    P.work_used = arena.alloc<unsigned long long>(1);
    P.work_left = work_limit - *scan;
    k_townsend<<<(unsigned)blocks, kTownsendWarps * 32, 0, stream>>>(P);
    APIC_CUDA(cudaGetLastError());
    std::vector<double> cross(H * bins);
    std::vector<unsigned long long> upd(H);
    std::vector<unsigned> maxa(H);
    unsigned err = 0;
    APIC_CUDA(cudaMemcpyAsync(cross.data(), P.crossings, H * bins * sizeof(double), cudaMemcpyDeviceToHost, stream));
    APIC_CUDA(cudaMemcpyAsync(upd.data(), P.updates, H * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream));
    APIC_CUDA(cudaMemcpyAsync(maxa.data(), P.max_active, H * sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
    APIC_CUDA(cudaMemcpyAsync(&err, P.error, sizeof err, cudaMemcpyDeviceToHost, stream));
    const cudaError_t we = bounded_wait(stream, 3600.0);
    if (we == cudaErrorNotReady) throw Error(APIC_ERR_TIMEOUT, "spatial Townsend pass did not complete in time");
    APIC_CUDA(we);
    if (err) {
        const int status = (err & kErrMajorant) ? APIC_ERR_MAJORANT
                           : (err & kErrCandidates) ? APIC_ERR_CANDIDATES
                           : (err & (kErrPopulation | kErrSecondaries)) ? APIC_ERR_CAPACITY
                           : (err & kErrNonFinite) ? APIC_ERR_NONFINITE
                                                   : APIC_ERR_INVALID;
        std::string msg;
        if (err & kErrMaxEnergyPre) msg += "spatial Townsend particle energy exceeded max_energy_ev before collision lookup; ";
        if (err & kErrMaxEnergy) msg += "spatial Townsend particle energy exceeded max_energy_ev; ";
        if (err & kErrPopulation) msg += "spatial Townsend branching exceeded population_limit before resampling; ";
        if (err & kErrNoTermination) msg += "spatial Townsend history did not terminate within spatial_max_steps; ";
        if (err & kErrWorkLimit) msg += "spatial Townsend scan exceeded spatial_work_item_limit; ";
        if (err & kErrSecondaries) msg += "more than 8 secondaries of one electron in one step; ";
        if (err & kErrMajorant) msg += "MCC total collision frequency exceeds configured max_frequency; ";
        if (err & kErrCandidates) msg += "MCC candidate limit exceeded; ";
        if (err & kErrNonFinite) msg += "electron velocity became non-finite; ";
        throw Error(status, msg);
    }
    uint64_t total = 0, max_active = 0;
    for (size_t h = 0; h < H; ++h) {
        total += upd[h];
        max_active = std::max<uint64_t>(max_active, maxa[h]);
    }
    *scan += total;
    if (history_crossings) std::memcpy(history_crossings, cross.data(), H * bins * sizeof(double));

    std::vector<double> log_flux(bins, 0.0);
    for (size_t b = 0; b < bins; ++b) {
        double sum = 0.0, sq = 0.0;
        for (size_t h = 0; h < H; ++h) {
            const double value = cross[h * bins + b];
            sum += value;
            sq += value * value;
        }
        const double hist = (double)H;
        const double mean = sum / hist;
        double se = 0.0;
        if (H > 1) se = std::sqrt(std::max(0.0, sq - sum * sum / hist) / (hist * (hist - 1.0)));
        profile[b].distance_m = planes[b];
        profile[b].net_crossings_per_injected_electron = mean;
        profile[b].standard_error = se;
        if (mean > 0.0) log_flux[b] = std::log(mean);
    }
    const size_t fb = sp.fit_begin_bin, fe = sp.fit_end_bin == 0 ? bins : sp.fit_end_bin;
    for (size_t b = fb; b < fe; ++b)
        require(profile[b].net_crossings_per_injected_electron > 0.0,
                "spatial Townsend fit requires positive net flux at every fit plane; increase spatial_histories or "
                "adjust the fit range");
    const size_t nblocks = c.uncertainty_blocks, hpb = H / nblocks;
    std::vector<double> slopes, block_log(bins, 0.0);
    for (size_t blk = 0; blk < nblocks; ++blk) {
        for (size_t b = 0; b < bins; ++b) {
            double sum = 0.0;
            for (size_t l = 0; l < hpb; ++l) sum += cross[(blk * hpb + l) * bins + b];
            const double flux = sum / (double)hpb;
            require(!(b >= fb && b < fe && !(flux > 0.0)),
                    "spatial Townsend uncertainty block has non-positive fit flux; increase spatial_histories");
            if (flux > 0.0) block_log[b] = std::log(flux);
        }
        slopes.push_back(linear_slope(block_log, fb, fe, spacing));
    }
    double mean_slope = 0.0, se_slope = 0.0;
    block_mean_and_error(slopes.data(), slopes.size(), slopes.size(), mean_slope, se_slope);
    out->townsend_1_m = linear_slope(log_flux, fb, fe, spacing);
    out->townsend_standard_error_1_m = se_slope;
    out->fit_r_squared = slope_r_squared(log_flux, fb, fe);
    out->histories_completed = H;
    out->maximum_active_particles = max_active;
    out->particle_updates = total;
    require(!(out->fit_r_squared < sp.min_r_squared), "spatial Townsend log-flux fit did not meet spatial_min_r_squared");
}

}  // namespace swarm
}  // namespace apic

struct apic_swarm_server {
    apic::swarm::Server impl;
};

namespace {
thread_local std::string g_swarm_error;

template <class F>
int guarded_swarm(apic_swarm_server* h, F&& f) {
    try {
        f();
        return APIC_OK;
    } catch (const apic::Error& e) {
        (h ? h->impl.last_error : g_swarm_error) = e.what();
        return e.status;
    } catch (const std::exception& e) {
        (h ? h->impl.last_error : g_swarm_error) = e.what();
        return APIC_ERR_INVALID;
    }
}
}  // namespace

extern "C" {

int apic_swarm_server_create(const apic_swarm_server_config* cfg, const apic_mcc_model* gas,
                             apic_swarm_server** out) {
    if (!cfg || !gas || !out) {
        g_swarm_error = "null argument";
        return APIC_ERR_INVALID;
    }
    *out = nullptr;
    auto h = std::make_unique<apic_swarm_server>();
    const int rc = guarded_swarm(h.get(), [&] {
        h->impl.create(*cfg, *gas);
        for (int i = 0; i < gas->nch && i < apic::kMaxChannels; ++i) {
            h->impl.host_table_max_[i] = gas->ch[i].energy[gas->ch[i].rows - 1];
            if (gas->ch[i].angular == APIC_HENYEY_GREENSTEIN)
                h->impl.host_mu_max_[i] = gas->ch[i].mean_cosine_energy[gas->ch[i].mean_cosine_rows - 1];
        }
    });
    if (rc != APIC_OK) {
        g_swarm_error = h->impl.last_error;
        return rc;
    }
    *out = h.release();
    return APIC_OK;
}

void apic_swarm_server_destroy(apic_swarm_server* srv) { delete srv; }

const char* apic_swarm_last_error(const apic_swarm_server* srv) {
    return srv ? srv->impl.last_error.c_str() : g_swarm_error.c_str();
}

int apic_swarm_server_submit(apic_swarm_server* srv, const apic_swarm_request* req, uint64_t* id) {
    if (!srv || !req || !id) return APIC_ERR_INVALID;
    return guarded_swarm(srv, [&] { *id = srv->impl.submit(*req); });
}

int apic_swarm_server_advance(apic_swarm_server* srv, int* active, int* queued) {
    if (!srv) return APIC_ERR_INVALID;
    return guarded_swarm(srv, [&] { srv->impl.advance(active, queued); });
}

int apic_swarm_server_launch(apic_swarm_server* srv) {
    if (!srv) return APIC_ERR_INVALID;
    return guarded_swarm(srv, [&] { srv->impl.launch(); });
}

int apic_swarm_server_complete(apic_swarm_server* srv, int* active, int* queued) {
    if (!srv) return APIC_ERR_INVALID;
    return guarded_swarm(srv, [&] { srv->impl.complete(active, queued); });
}

int apic_swarm_server_poll(apic_swarm_server* srv, uint64_t id, apic_swarm_result* out, int* done) {
    if (!srv || !out || !done) return APIC_ERR_INVALID;
    return guarded_swarm(srv, [&] {
        auto it = srv->impl.done.find(id);
        *done = it != srv->impl.done.end() ? 1 : 0;
        if (*done) {
            *out = it->second;
            srv->impl.done.erase(it);
        }
    });
}

int apic_swarm_server_copy_bytes(apic_swarm_server* srv, uint64_t* h2d, uint64_t* d2h) {
    if (!srv) return APIC_ERR_INVALID;
    if (h2d) *h2d = srv->impl.h2d_bytes;
    if (d2h) *d2h = srv->impl.d2h_bytes;
    return APIC_OK;
}

int apic_swarm_server_stats(apic_swarm_server* srv, uint64_t* graph_launches, uint64_t* particle_steps,
                            size_t* pool_bytes_free) {
    if (!srv) return APIC_ERR_INVALID;
    return guarded_swarm(srv, [&] {
        if (graph_launches) *graph_launches = srv->impl.launches;
        if (particle_steps) *particle_steps = srv->impl.particle_steps;
        if (pool_bytes_free) {
            size_t f = 0;
            for (auto& kv : srv->impl.pool.free_) f += kv.second;
            *pool_bytes_free = f;
        }
    });
}

int apic_swarm_server_set_kernel_timing(apic_swarm_server* srv, int enable) {
    if (!srv) return APIC_ERR_INVALID;
    return guarded_swarm(srv, [&] {
        srv->impl.timing = enable != 0;
        srv->impl.push_ms = 0.0;
        srv->impl.collide_ms = 0.0;
        srv->impl.push_bytes = 0.0;
        srv->impl.push_launches = 0;
    });
}

int apic_swarm_server_kernel_times(apic_swarm_server* srv, double* push_ms, double* collide_ms,
                                   uint64_t* push_launches, double* push_bytes) {
    if (!srv) return APIC_ERR_INVALID;
    return guarded_swarm(srv, [&] {
        if (push_ms) *push_ms = srv->impl.push_ms;
        if (collide_ms) *collide_ms = srv->impl.collide_ms;
        if (push_launches) *push_launches = srv->impl.push_launches;
        if (push_bytes) *push_bytes = srv->impl.push_bytes;
    });
}

int apic_swarm_server_kernel_launches(apic_swarm_server* srv, uint64_t* launches) {
    if (!srv || !launches) return APIC_ERR_INVALID;
    *launches = srv->impl.kernel_launches;
    return APIC_OK;
}

int apic_swarm_server_cuda_stream(apic_swarm_server* srv, void** stream) {
    if (!srv || !stream) return APIC_ERR_INVALID;
    *stream = srv->impl.stream;
    return APIC_OK;
}

int apic_swarm_run(const apic_swarm_config* cfg, const apic_mcc_model* gas, const double* fields_td, size_t nfields,
                   apic_swarm_result* results) {
    if (!cfg || !gas || !fields_td || !results || nfields == 0) {
        g_swarm_error = "null argument";
        return APIC_ERR_INVALID;
    }
    return guarded_swarm(nullptr, [&] {
        for (size_t a = 0; a < nfields; ++a)
            for (size_t b = a + 1; b < nfields; ++b)
                apic::require(fields_td[a] != fields_td[b], "swarm reduced fields must not contain duplicates");
        const uint64_t limit = cfg->work_item_limit ? cfg->work_item_limit : 100000000ull;
        auto over = [](uint64_t a, uint64_t b, uint64_t lim) { return a != 0 && b > lim / a; };
        apic::require(!over(nfields, cfg->particles, limit) && !over(nfields * cfg->particles, cfg->steps, limit),
                      "swarm scan exceeds work_item_limit; raise it explicitly only on an appropriate compute host");
        apic_mcc_model m = *gas;
        m.neutral_density = cfg->neutral_density;
        m.neutral_temperature = cfg->neutral_temperature;
        m.max_frequency = cfg->max_frequency;
        apic_swarm_request r{};
        r.particles = cfg->particles;
        r.steps = cfg->steps;
        r.burn_in_steps = cfg->burn_in_steps;
        r.uncertainty_blocks = cfg->uncertainty_blocks;
        r.population_model = cfg->population_model;
        r.population_limit = cfg->population_limit;
        r.initial_mean_energy_ev = cfg->initial_mean_energy_ev;
        r.max_energy_ev = cfg->max_energy_ev;
        r.timestep = cfg->timestep;
        r.tolerance = 0.0;
        apic_swarm_server_config sc{};
        sc.max_runs = (int)nfields;
        sc.precision = cfg->precision;
        sc.steps_per_launch = std::min<size_t>(cfg->steps, 64);
        // every field resident at once
        apic::swarm::Server probe;
        probe.fp32 = cfg->precision == APIC_FP32;
        size_t bytes = 0;
        for (size_t f = 0; f < nfields; ++f) bytes += probe.run_bytes(r) + 4096;
        sc.memory_budget_bytes = std::max<size_t>(bytes, (size_t)1 << 20);
        apic_swarm_server* srv = nullptr;
        int rc = apic_swarm_server_create(&sc, &m, &srv);
        if (rc != APIC_OK) throw apic::Error(rc, g_swarm_error);
        std::unique_ptr<apic_swarm_server> hold(srv);
        std::vector<uint64_t> ids(nfields);
        for (size_t f = 0; f < nfields; ++f) {
            r.reduced_field_td = fields_td[f];
            r.seed = cfg->seed + f;  // src/Swarm.cpp:1513-1515
            ids[f] = srv->impl.submit(r);
        }
        int active = 1, queued = 1;
        while (active || queued) srv->impl.advance(&active, &queued);
        for (size_t f = 0; f < nfields; ++f) {
            auto it = srv->impl.done.find(ids[f]);
            apic::require(it != srv->impl.done.end(), "swarm run did not finish");
            results[f] = it->second;
        }
        for (size_t f = 0; f < nfields; ++f)
            if (results[f].status != APIC_OK) throw apic::Error(results[f].status, results[f].message);
    });
}

int apic_swarm_spatial_townsend(const apic_swarm_config* cfg, const apic_spatial_townsend_config* sp,
                                const apic_mcc_model* gas, double reduced_field_td, uint64_t seed,
                                uint64_t* scan_particle_updates, apic_spatial_townsend_result* out,
                                apic_spatial_flux_point* profile, double* history_crossings) {
    if (!cfg || !sp || !gas || !out || (sp->histories && !profile)) {
        g_swarm_error = "null argument";
        return APIC_ERR_INVALID;
    }
    return guarded_swarm(nullptr, [&] {
        uint64_t scan = scan_particle_updates ? *scan_particle_updates : 0;
        apic::swarm::spatial_townsend(*cfg, *sp, *gas, reduced_field_td, seed, &scan, out, profile,
                                      history_crossings);
        if (scan_particle_updates) *scan_particle_updates = scan;
    });
}

}  // extern "C"
