// 1D1V / 1D3V electrostatic PIC particle step on one B200 (FP64 form).
//
// Replaces pic::Simulation's hot loop (src/Simulation.cpp:1008-1138) and the
// routines it calls: interpolate_electric (src/FieldSolver.cpp:909-924), the
// leapfrog kick/drift/synchronize/initialize (src/Pusher.cpp:66-80), the
// periodic wrap / absorbing walls (src/Simulation.cpp:1039-1077),
// Species::deposit_charge (src/Species.cpp:161-185), FieldSolver::solve(Grid&)
// (src/FieldSolver.cpp:384-440, :733-759) and Simulation::apply_collisions
// (src/Simulation.cpp:771-1006).
//
// Device layout: per species, structure-of-arrays x, v_half, v_y, v_z (and a
// time-centred v written only when the state is read back), double-buffered;
// live particles are kept compacted in [0, n).  One step is two launches:
//
//   pass kernel  (persistent grid, one 1024-particle tile per iteration):
//       [synchronize -> MCC -> re-initialise half step]  (the collision part of
//        the previous step, done while the particle is in registers anyway)
//       kick -> drift -> wall/wrap -> CIC deposit into a shared-memory copy of
//       the grid (64-bit fixed point) -> order-preserving compaction of the
//       survivors (decoupled look-back across tiles) -> write.
//   post kernel  (one CTA): sort and append this pass's ionization products
//       (pushed and deposited like everyone else), convert the fixed-point
//       density to FP64, Poisson solve (scan-form Thomas for Dirichlet walls,
//       exact-twiddle DFT for periodic), E field, advance time and step.
//
// This file is compiled with --fmad=false: every FP64 expression is evaluated
// with the reference's operation order and rounding, so a particle's state
// differs from the reference only through the field it sees.
#include <cub/block/block_radix_sort.cuh>
#include <cub/block/block_scan.cuh>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "apc_internal.h"
#include "apic_common.cuh"
#include "apic_mcc.cuh"
#include "apic_mcc32.cuh"
#include "apic_mcc_host.h"
#include "apic_rng.cuh"

namespace apic {

constexpr int kThreads = 256;
constexpr int kItems = 4;
constexpr int kTile = kThreads * kItems;
constexpr int kMinBlocks = 2;  // resident CTAs of k_pass1d per SM (register budget)
constexpr int kWarpCounts = kItems * (kThreads / 32);  // per-(item, warp) survivor counts of a tile
static_assert(kWarpCounts <= 32, "the survivor scan runs in one warp");
constexpr int kMaxSpecies = APIC_MAX_SPECIES;
constexpr int kMaxModels = APIC_MAX_MODELS;
constexpr int kPostThreads = 512;
constexpr int kPostItems = 8;
constexpr int kMaxBirths = kPostThreads * kPostItems;  // products per pass the post kernel sorts
constexpr int kMaxNx1D = 4096;          // Dirichlet grids
constexpr int kMaxNx1DPeriodic = 2048;  // periodic grids (direct DFT with shared-memory spectra)

enum : unsigned {
    kModeSyncMcc = 1u << 0,   // synchronize + collide + re-initialise (pending collision part)
    kModeKickDrift = 1u << 1, // kick + drift + boundary
    kModeDeposit = 1u << 2,   // CIC deposit of the resulting positions
    kModeWriteV = 1u << 3,    // write time-centred v (state read back)
    kModeInitHalf = 1u << 4,  // v_half = v - qm E dt / 2 (Simulation::initialize)
};
enum : unsigned {
    kPostSolve = 1u << 0,
    kPostAdvance = 1u << 1,
    kPostPushBirths = 1u << 2,
};

struct DevState {
    unsigned n[kMaxSpecies];        // live particles (logical count)
    unsigned nranges[kMaxSpecies];  // ranges of the current input layout
    unsigned nbirths;
    unsigned error;
    unsigned holes[kMaxSpecies];    // FP32 cell form: dead slots among [0, n)
    unsigned long long step;
    double time;
    unsigned long long candidates, nulls;
    unsigned long long chan[kMaxModels][kMaxChannels];
    double chan_energy[kMaxModels][kMaxChannels];
    unsigned long long lost[kMaxSpecies][2];
    double lost_energy[kMaxSpecies][2];
    double work[kMaxSpecies];  // electric-work ledger (species_power_transfer), when enabled
};

struct BirthRec {
    unsigned long long key;  // (parent species, parent slot, product index) ordering key
    double x, v[3];
    int species;
    int pad;  // secondary record: the parent's ionization channel
};

struct SpeciesDev {
    double qm, hqm, qw, qwdx, mass, weight;
    int model;
    unsigned capacity;  // slots of a particle buffer
    unsigned nscratch;  // entries of chunk_surv
    unsigned live_cap;  // max_particles_per_species (the FP32 cell form's buffers add room for holes)
    // MCC first waiting time inside the step exactly when the first 64-bit
    // draw is >= cand_draw_min (see draw_threshold); no_candidates: never
    uint64_t cand_draw_min;
    int no_candidates;
    // Layout: the live particles, in logical order, are the concatenation of
    // ranges r = 0..nranges-1 of physical slots [start[r], start[r] + count[r]);
    // lstart[r] is the logical index of a range's first particle.
    unsigned* rstart[2];
    unsigned* rcount[2];
    unsigned* rlstart[2];
    unsigned* chunk_surv;  // survivors of each 1024-particle chunk of a pass
    // [0] = input buffer of this pass, [1] = output buffer
    double* x[2];
    double* vh[2];
    double* vy[2];
    double* vz[2];
    double* v;  // time-centred velocity (valid after a read-back pass)
    // FP32 form: v_half, v_y, v_z stored as float (x stays FP64: the int32
    // cell + FP32 offset pair would take the same 8 bytes); null in FP64 form
    float* vh32[2];
    float* vy32[2];
    float* vz32[2];
    double* stage;  // FP32 forms: FP64 staging for host copies (capacity)
    // FP32 cell form: the position as the index of the cell holding the
    // particle (its left node) and the float offset in [0, 1] inside it; null
    // in the other forms (which keep x in FP64)
    int* cell[2];
    float* off[2];
    // FP32 cell form constants: q/m dt, q/(2m) dt, dt/dx, and the fixed-point
    // charge of a whole particle on one node (q w / dx times the density scale)
    float qmdt32, hqmdt32, dtdx32, dep32;
    // FP32 cell form candidates: P = 1 - exp(-nu dt) of the first waiting time
    // falling inside the step, and 1 / (nu dt) for the geometric gaps
    float cand_p32, inv_nudt32;
    // electric-work ledger: the time-centred v each particle had at the end of
    // its last step (double-buffered like the state); null unless enabled
    double* vold[2];
};

struct CandRec32;

struct Params1D {
    int nspecies, vdim, dirichlet, nx;
    int f32;  // FP32 velocities (both FP32 forms)
    int c32;  // FP32 cell form: int32 cell + float offset positions, FP32 arithmetic
    double L, dx, inv_dx, dt, eps, rho_scale, inv_rho_scale;
    unsigned mode;
    uint64_t seed;
    double phi_left, phi_right;
    apic_voltage_drive drive_left, drive_right;
    SpeciesDev sp[kMaxSpecies];
    MccModelDev model[kMaxModels];
    int bgk;                   // legacy BGK model active
    double bgk_prob, bgk_vt;   // 1 - exp(-frequency dt), neutral_temperature_velocity
    double* E;
    double* rho;
    double* phi;
    unsigned long long* rho_acc;
    const double* tw;       // periodic: twiddles (cos, sin)(2 pi m / n), m < n
    const double* thomas_r; // Dirichlet: 1/denominator of the Thomas forward sweep
    const double* thomas_a; // Dirichlet: -cp of the back substitution
    BirthRec* births;
    unsigned births_cap;
    DevState* st;
    // campaign diagnostics: spatial collision-energy density of the collision
    // part this pass applies ([channel][nx]; null outside the window) and the
    // slice of its RF phase bin (null without phase bins)
    double* coll_acc;
    double* coll_phase_acc;
    int coll_off[kMaxModels];  // first channel of each model in the channel numbering
    int ledger;                // electric-work ledger enabled (SpeciesDev::vold allocated)
    // FP32 cell form: the collision models in single precision, and the FP64
    // models in device memory for the (rare) exact frequency-bound check
    MccModel32 model32[kMaxModels];
    const MccModelDev* gmodel;
    // this step's collision candidates (FP32 cell form): region b of
    // cand_per_region records belongs to CTA b of the pass, which stores its
    // count in cand_count[b]
    CandRec32* cands;
    unsigned* cand_count;
    unsigned cand_regions, cand_per_region;
};

// ---- field gather / deposit (reference arithmetic) ----------------------

// wrap_periodic, src/FieldSolver.cpp:15-17: fmod(fmod(x, L) + L, L).  For
// |x| < 2L every fmod is a single exact subtraction (Sterbenz), so the fast
// branch returns the same bits as the two library fmod calls.
__device__ __forceinline__ double wrap_periodic(double x, double L) {
    if (!(fabs(x) < 2.0 * L)) return fmod(fmod(x, L) + L, L);
    const double r = x >= L ? x - L : (x <= -L ? x + L : x);  // fmod(x, L)
    const double y = r + L;
    return y >= 2.0 * L ? 0.0 : (y >= L ? y - L : y);          // fmod(y, L), 0 < y <= 2L
}

struct Cic {
    int i0, i1;
    double w0, w1;  // (1 - f), f
};

// interpolate_electric / deposit_charge index + fraction, src/FieldSolver.cpp:909-924,
// src/Species.cpp:167-183
__device__ __forceinline__ Cic cic_periodic(double x, double L, double dx, int nx) {
    const double xp = wrap_periodic(x, L);
    const double g = xp / dx;
    const double fl = floor(g);
    const unsigned long long i = (unsigned long long)fl;
    const double f = g - (double)i;
    // i % nx and (i + 1) % nx; i <= nx after the wrap, so the remainders are
    // single subtractions (the 64-bit division only for out-of-range input)
    const unsigned long long n = (unsigned long long)nx;
    const unsigned long long i1 = i + 1;
    Cic c;
    c.i0 = (int)(i < n ? i : (i < 2 * n ? i - n : i % n));
    c.i1 = (int)(i1 < n ? i1 : (i1 < 2 * n ? i1 - n : i1 % n));
    c.w0 = 1.0 - f;
    c.w1 = f;
    return c;
}

__device__ __forceinline__ Cic cic_dirichlet(double x, double L, double dx, int nx) {
    // std::clamp (a NaN position, already flagged as non-finite, lands on the
    // left wall so that every index stays inside the grid)
    const double xp = !(x >= 0.0) ? 0.0 : (L < x ? L : x);
    const double g = xp / dx;
    double fl = floor(g);
    const double lim = (double)(nx - 2);
    if (lim < fl) fl = lim;  // std::min<double>(floor(g), nx - 2)
    const unsigned long long i = (unsigned long long)fl;
    const double f = g - (double)i;
    Cic c;
    c.i0 = (int)i;
    c.i1 = (int)i + 1;
    c.w0 = 1.0 - f;
    c.w1 = f;
    return c;
}

template <bool DIRICHLET>
__device__ __forceinline__ Cic cic(double x, const Params1D& p) {
    return DIRICHLET ? cic_dirichlet(x, p.L, p.dx, p.nx) : cic_periodic(x, p.L, p.dx, p.nx);
}

__device__ __forceinline__ double gather(const double* E, const Cic& c) {
    return E[c.i0] * c.w0 + E[c.i1] * c.w1;
}

// One particle's two fixed-point contributions.
template <bool DIRICHLET>
__device__ __forceinline__ void deposit_contrib(const Cic& c, const SpeciesDev& s, const Params1D& p,
                                                long long& a0, long long& a1) {
    if (!DIRICHLET) {
        a0 = to_fixed(s.qwdx * c.w0, p.rho_scale);
        a1 = to_fixed(s.qwdx * c.w1, p.rho_scale);
    } else {
        // q w (1 - f) / node_volume(i), src/Species.cpp:180-181: the reciprocal
        // volume differs from the division by at most one rounding, far below
        // the fixed-point resolution of the accumulated density
        const double r0 = (c.i0 == 0 || c.i0 + 1 == p.nx) ? 2.0 * p.inv_dx : p.inv_dx;
        const double r1 = (c.i1 == 0 || c.i1 + 1 == p.nx) ? 2.0 * p.inv_dx : p.inv_dx;
        a0 = to_fixed(s.qw * c.w0 * r0, p.rho_scale);
        a1 = to_fixed(s.qw * c.w1 * r1, p.rho_scale);
    }
}

// ---- range-table layout -----------------------------------------------------

// The range holding logical particle `idx`: the last range whose logical
// start is <= idx, by binary search over the ranges' logical starts.
__device__ __forceinline__ unsigned range_of(const unsigned* lstart, unsigned nr, unsigned idx) {
    unsigned lo = 0, hi = nr;
    while (hi - lo > 1) {
        const unsigned mid = (lo + hi) >> 1;
        if (__ldg(lstart + mid) <= idx) lo = mid; else hi = mid;
    }
    return lo;
}

// Physical slot of logical particle `idx`, walking forward from range r0
// (a range at or before the one holding idx): a tile spans few ranges.
__device__ __forceinline__ unsigned physical_slot_from(const unsigned* lstart, const unsigned* start, unsigned nr,
                                                       unsigned r0, unsigned idx) {
    unsigned r = r0;
    while (r + 1 < nr && __ldg(lstart + r + 1) <= idx) ++r;
    return __ldg(start + r) + (idx - __ldg(lstart + r));
}

// ---- campaign diagnostics stencil ---------------------------------------------

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Node volume of the diagnostics deposits: Grid::node_volume, src/Grid.cpp:26-30
template <bool DIRICHLET>
__device__ __forceinline__ double node_volume(const Params1D& p, int i) {
    return (DIRICHLET && (i == 0 || i + 1 == p.nx)) ? 0.5 * p.dx : p.dx;
}

// deposit_spatial_collision_energy, src/Simulation.cpp:1171-1212: the energy
// change as a density on the particle's two nodes (FP64 atomics: the sum's
// rounding depends on the order of the collisions).
template <bool DIRICHLET>
__device__ __forceinline__ void collision_energy_deposit(const Params1D& p, double x, int channel, double e) {
    const Cic d = cic<DIRICHLET>(x, p);
    const double a0 = e * d.w0 / node_volume<DIRICHLET>(p, d.i0);
    const double a1 = e * d.w1 / node_volume<DIRICHLET>(p, d.i1);
    double* row = p.coll_acc + (size_t)channel * p.nx;
    atomicAdd(row + d.i0, a0);
    atomicAdd(row + d.i1, a1);
    if (p.coll_phase_acc) {
        row = p.coll_phase_acc + (size_t)channel * p.nx;
        atomicAdd(row + d.i0, a0);
        atomicAdd(row + d.i1, a1);
    }
}

// ---- the fused particle pass -----------------------------------------------

// A particle whose first exponential waiting time falls inside the step is a
// collision candidate (a few percent of particles).  Its full collision loop
// runs in a second phase of the tile from a shared-memory queue, so that the
// long, branchy loops are packed into few warps instead of diverging inside
// every warp.
struct CandidateEntry {
    double v[3];
    double x;
    double first_wait;
    unsigned slot;
    unsigned draws;
};
constexpr int kQueue = 384;

// Velocity components of the two storage forms: FP64, or FP32 (rounded to
// nearest when stored, widened exactly when loaded; the arithmetic is FP64).
template <bool F32>
__device__ __forceinline__ double ld_comp(const double* d, const float* f, unsigned i) {
    return F32 ? (double)f[i] : d[i];
}
template <bool F32>
__device__ __forceinline__ void st_comp(double* d, float* f, unsigned long long i, double v) {
    if (F32) f[i] = (float)v;
    else d[i] = v;
}

// The legacy BGK branch, src/Simulation.cpp:772-834: with probability
// 1 - exp(-nu dt) the particle relaxes to a neutral Maxwellian of standard
// deviation vt, drawn from its own stream (the one its MCC would use; the two
// models exclude each other), and the run's totals count it.  Returns the
// energy change (hmw = m w / 2) through `change` and whether it relaxed.  Out
// of line, with plain arguments, so that the pass keeps the register
// allocation of runs without it.
template <int VDIM>
__device__ __noinline__ bool bgk_relax(uint64_t seed, unsigned idx, uint32_t step, uint32_t s, double prob, double vt,
                                       double hmw, DevState* st, double& v, double& vy, double& vz, double& change) {
    PhiloxStream rng(seed, idx, step, s);
    if (!(uniform01(rng) < prob)) return false;
    const double before = hmw * (v * v + (VDIM == 3 ? vy * vy + vz * vz : 0.0));
    NormalState ns;
    v = normal(ns, rng, 0.0, vt);
    if (VDIM == 3) {
        vy = normal(ns, rng, 0.0, vt);
        vz = normal(ns, rng, 0.0, vt);
    }
    change = hmw * (v * v + (VDIM == 3 ? vy * vy + vz * vz : 0.0)) - before;
    atomicAdd(&st->candidates, 1ull);
    atomicAdd(&st->chan[0][0], 1ull);
    atomicAdd(&st->chan_energy[0][0], change);
    return true;
}

// DIAG: the instantiation that also deposits the spatial collision energy,
// keeps the electric-work ledger and applies the legacy BGK model (run only
// inside a campaign-diagnostics window, with the ledger or with BGK, so the
// plain pass keeps its register allocation).
template <int VDIM, bool DIRICHLET, bool F32, bool DIAG>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_pass1d(Params1D p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sE = reinterpret_cast<double*>(smem_raw);
    unsigned long long* sRho = reinterpret_cast<unsigned long long*>(sE + p.nx);
    __shared__ unsigned s_cnt[32];
    __shared__ unsigned s_qlen;
    __shared__ CandidateEntry s_queue[kQueue];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned mode = p.mode;
    for (int i = tid; i < p.nx; i += kThreads) {
        sE[i] = p.E[i];
        sRho[i] = 0ull;
    }
    if (tid == 0) s_qlen = 0;
    DevState* st = p.st;
    unsigned tiles_before[kMaxSpecies + 1];
    tiles_before[0] = 0;
    for (int s = 0; s < kMaxSpecies; ++s)
        tiles_before[s + 1] = tiles_before[s] + (s < p.nspecies ? (st->n[s] + kTile - 1) / kTile : 0);
    const unsigned total_tiles = tiles_before[kMaxSpecies];
    const uint32_t mcc_step = (uint32_t)(st->step - 1ull);
    __syncthreads();

    // chunks of kTile logical particles, statically strided over the grid
    for (unsigned t = blockIdx.x; t < total_tiles; t += gridDim.x) {
        int s = 0;
        while (t >= tiles_before[s + 1]) ++s;
        const unsigned tile = t - tiles_before[s];
        const SpeciesDev& S = p.sp[s];
        const unsigned n = st->n[s];
        const unsigned nr = st->nranges[s];
        const unsigned base = tile * kTile;
        const bool mcc = (mode & kModeSyncMcc) && S.model >= 0;
        // one search per warp for the range of its first particle
        const unsigned wfirst = base + (unsigned)(tid & ~31);
        unsigned r0 = 0;
        if (lane == 0 && wfirst < n) r0 = range_of(S.rlstart[0], nr, wfirst);
        r0 = __shfl_sync(0xffffffffu, r0, 0);

        double x[kItems], vh[kItems], vy[kItems], vz[kItems], vc[kItems], Ek[kItems];
        double vo[kItems];  // DIAG with the ledger: v at the end of the particle's last step
        double wsum = 0.0;  // DIAG with the ledger: this thread's electric work
        bool keep[kItems];
        int queued[kItems];
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            const unsigned idx = base + k * kThreads + tid;
            const bool live = idx < n;
            keep[k] = live;
            queued[k] = -1;
            const unsigned ph = live ? physical_slot_from(S.rlstart[0], S.rstart[0], nr, r0, idx) : 0u;
            x[k] = live ? S.x[0][ph] : 0.0;
            vh[k] = live ? ld_comp<F32>(S.vh[0], S.vh32[0], ph) : 0.0;
            vy[k] = (VDIM == 3 && live) ? ld_comp<F32>(S.vy[0], S.vy32[0], ph) : 0.0;
            vz[k] = (VDIM == 3 && live) ? ld_comp<F32>(S.vz[0], S.vz32[0], ph) : 0.0;
            vc[k] = 0.0;
            if ((mode & kModeInitHalf) && live) vc[k] = S.v[ph];
            vo[k] = 0.0;
            if (DIAG && p.ledger && live)
                vo[k] = (mode & (kModeKickDrift | kModeSyncMcc)) ? S.vold[0][ph] : S.v[ph];
        }
        // -- phase A: gather, synchronize, first collision draw --
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            Ek[k] = 0.0;
            if (!keep[k]) continue;
            const unsigned idx = base + k * kThreads + tid;
            const double E = gather(sE, cic<DIRICHLET>(x[k], p));
            Ek[k] = E;
            if (mode & kModeInitHalf) {
                // initialize_leapfrog_half_step, src/Pusher.cpp:66-68
                vh[k] = vc[k] - S.hqm * E * p.dt;
            }
            if (mode & kModeSyncMcc) {
                // synchronize_leapfrog, src/Pusher.cpp:78-80
                vc[k] = vh[k] + S.hqm * E * p.dt;
                // electric-work ledger, src/Simulation.cpp:1109-1114
                if (DIAG && p.ledger) wsum += 0.5 * S.mass * S.weight * (vc[k] * vc[k] - vo[k] * vo[k]);
                double change;
                if (DIAG && p.bgk && bgk_relax<VDIM>(p.seed, idx, mcc_step, (uint32_t)s, p.bgk_prob, p.bgk_vt,
                                             0.5 * S.mass * S.weight, st, vc[k], vy[k], vz[k], change)) {
                    if (DIAG && p.coll_acc) collision_energy_deposit<DIRICHLET>(p, x[k], 0, change);
                    queued[k] = -2;  // re-initialise the half step in phase C
                }
                if (mcc) {
                    const MccModelDev& M = p.model[S.model];
                    // first iteration of NullCollisionModel::collide, src/Collision.cpp:926-933
                    const double s2 = vc[k] * vc[k] + vy[k] * vy[k] + vz[k] * vz[k];
                    if (!isfinite(s2)) {  // NullCollisionModel rejects non-finite velocities, src/Collision.cpp:910-916
                        atomicOr(&st->error, kErrNonFinite);
                        continue;
                    }
                    // validate_frequency_bound at |v| (1V: src/Collision.cpp:856) or at speed(v)
                    if (!(s2 <= M.v_safe2) && !frequency_bound_ok(M, VDIM == 3 ? sqrt(s2) : fabs(vc[k])))
                        atomicOr(&st->error, kErrMajorant);
                    PhiloxStream rng(p.seed, idx, mcc_step, (uint32_t)s);
                    const uint64_t d0 = rng.next();
                    // the raw-draw threshold decides exactly as -log(u)/nu < dt would
                    bool cand = d0 != 0ull ? (!S.no_candidates && d0 >= S.cand_draw_min) : true;
                    double wait = 0.0;
                    if (cand) {
                        double u = d0 != 0ull ? canonical_of(d0) : 0.0;
                        for (int guard = 0; !(u > 0.0) && guard < 64; ++guard) u = uniform01(rng);
                        wait = -log(u) / M.max_frequency;
                        cand = isfinite(wait) && wait < p.dt;
                    }
                    if (cand) {
                        const unsigned q = atomicAdd(&s_qlen, 1u);
                        if (q < (unsigned)kQueue) {
                            CandidateEntry& ce = s_queue[q];
                            ce.v[0] = vc[k]; ce.v[1] = vy[k]; ce.v[2] = vz[k];
                            ce.first_wait = wait;
                            ce.x = x[k];
                            ce.slot = idx;
                            ce.draws = rng.index;
                            queued[k] = (int)q;
                        } else {
                            atomicOr(&st->error, kErrBirths);  // queue sized for > 30% candidates per tile
                        }
                    }
                }
            }
        }
        __syncthreads();
        // -- phase B: full collision loops of the queued candidates --
        if (mcc) {
            const unsigned qlen = min(s_qlen, (unsigned)kQueue);
            const MccModelDev& M = p.model[S.model];
            for (unsigned q = tid; q < qlen; q += kThreads) {
                CandidateEntry& ce = s_queue[q];
                PhiloxStream rng(p.seed, ce.slot, mcc_step, (uint32_t)s);
                rng.seek(ce.draws);
                CollideResult r;
                unsigned nion = 0;
                const unsigned slot = ce.slot;
                const double px = ce.x;
                double vel[3] = {ce.v[0], ce.v[1], ce.v[2]};
                if (VDIM == 1) collide1(M, vel[0], p.dt, rng, r, true, ce.first_wait);
                else collide3(M, vel, p.dt, rng, r,
                         [&](int ch, const double* vs, const double* vi) {
                             const unsigned bslot = atomicAdd(&st->nbirths, 2u);
                             const MccChannelDev& C = M.ch[ch];
                             if (bslot + 2u <= p.births_cap) {
                                 const unsigned long long key =
                                     ((unsigned long long)s << 56) | ((unsigned long long)slot << 16) | (nion << 1);
                                 BirthRec a, b;
                                 a.key = key; a.species = C.secondary; a.pad = DIAG ? ch : 0;
                                 b.key = key | 1ull; b.species = C.ion; b.pad = 0;
                                 a.x = b.x = px;
                                 for (int d = 0; d < 3; ++d) { a.v[d] = vs[d]; b.v[d] = vi[d]; }
                                 p.births[bslot] = a;
                                 p.births[bslot + 1] = b;
                             } else {
                                 atomicOr(&st->error, kErrBirths);
                             }
                             const SpeciesDev& A = p.sp[C.secondary];
                             const SpeciesDev& B = p.sp[C.ion];
                             const double added =
                                 0.5 * A.mass * A.weight * (vs[0] * vs[0] + vs[1] * vs[1] + vs[2] * vs[2]) +
                                 0.5 * B.mass * B.weight * (vi[0] * vi[0] + vi[1] * vi[1] + vi[2] * vi[2]);
                             atomicAdd(&st->chan_energy[S.model][ch], added);
                             ++nion;
                         },
                         true, ce.first_wait);
                if (r.error) atomicOr(&st->error, r.error);
                atomicAdd(&st->candidates, (unsigned long long)r.candidates);
                if (r.nulls) atomicAdd(&st->nulls, (unsigned long long)r.nulls);
                for (int ch = 0; ch < M.nch; ++ch) {
                    if (r.channel[ch]) {
                        atomicAdd(&st->chan[S.model][ch], (unsigned long long)r.channel[ch]);
                        atomicAdd(&st->chan_energy[S.model][ch], r.energy_change[ch] * S.weight);
                    }
                }
                if (DIAG && p.coll_acc) {
                    // tracked_energy_change, src/Simulation.cpp:862-923: the weighted
                    // projectile change per channel, deposited at the particle (the
                    // product pairs' energies follow from the births list in the
                    // post kernel)
                    for (int ch = 0; ch < M.nch; ++ch) {
                        const double t = r.energy_change[ch] * S.weight;
                        if (t != 0.0) collision_energy_deposit<DIRICHLET>(p, px, p.coll_off[S.model] + ch, t);
                    }
                }
                ce.v[0] = vel[0]; ce.v[1] = vel[1]; ce.v[2] = vel[2];
            }
            __syncthreads();
        }
        // -- phase C: re-initialise, kick, drift, walls, deposit --
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            if (!keep[k]) continue;
            const double E = Ek[k];
            if (mcc) {
                if (queued[k] >= 0) {
                    const CandidateEntry& ce = s_queue[queued[k]];
                    vc[k] = ce.v[0]; vy[k] = ce.v[1]; vz[k] = ce.v[2];
                }
                // initialize_leapfrog_half_step after the collision, src/Simulation.cpp:924-926
                vh[k] = vc[k] - S.hqm * E * p.dt;
            } else if (DIAG && queued[k] == -2) {
                // the BGK particle's initialize_leapfrog_half_step, src/Simulation.cpp:829-833
                vh[k] = vc[k] - S.hqm * E * p.dt;
            }
            if (mode & kModeKickDrift) {
                // kick_leapfrog + drift_leapfrog, src/Pusher.cpp:70-76
                vh[k] = vh[k] + S.qm * E * p.dt;
                x[k] = x[k] + vh[k] * p.dt;
                if (!DIRICHLET) {
                    x[k] = wrap_periodic(x[k], p.L);
                } else if (x[k] < 0.0 || x[k] > p.L) {
                    // absorbing walls and loss ledger, src/Simulation.cpp:1047-1077
                    if (DIAG && p.ledger) {
                        const double vp = (mode & (kModeSyncMcc | kModeInitHalf)) ? vc[k] : vo[k];
                        const double hmw = 0.5 * S.mass * S.weight;
                        wsum += hmw * vh[k] * vh[k] - hmw * vp * vp;
                    }
                    const double sp2 = vh[k] * vh[k] + vy[k] * vy[k] + vz[k] * vz[k];
                    const double e = 0.5 * S.mass * S.weight * sp2;
                    const int side = x[k] < 0.0 ? 0 : 1;
                    atomicAdd(&st->lost[s][side], 1ull);
                    atomicAdd(&st->lost_energy[s][side], e);
                    keep[k] = false;
                }
                if (!isfinite(x[k]) || !isfinite(vh[k])) {
                    // flagged and dropped: a non-finite particle deposits nothing
                    atomicOr(&st->error, kErrNonFinite);
                    keep[k] = false;
                }
            }
            if ((mode & kModeDeposit) && keep[k]) {
                const Cic d = cic<DIRICHLET>(x[k], p);
                long long a0, a1;
                deposit_contrib<DIRICHLET>(d, S, p, a0, a1);
                atomicAdd(&sRho[d.i0], (unsigned long long)a0);
                atomicAdd(&sRho[d.i1], (unsigned long long)a1);
            }
        }
        if (DIAG && p.ledger) {
            const double w = warp_sum(wsum);
            if (lane == 0 && w != 0.0) atomicAdd(&st->work[s], w);
        }
        // ---- order-preserving compaction of the survivors ----
        unsigned ballots[kItems];
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            ballots[k] = __ballot_sync(0xffffffffu, keep[k]);
            if (lane == 0) s_cnt[k * (kThreads / 32) + warp] = __popc(ballots[k]);
        }
        __syncthreads();
        if (warp == 0) {
            const unsigned c = lane < kWarpCounts ? s_cnt[lane] : 0u;
            unsigned incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            s_cnt[lane] = incl - c;
            const unsigned total = __shfl_sync(0xffffffffu, incl, 31);
            if (lane == 0) {
                S.chunk_surv[tile] = total;
                s_qlen = 0;
            }
        }
        __syncthreads();
        // survivors of this chunk keep their order at the chunk's own slots
        const unsigned long long out_base = base;
        const unsigned lt = (1u << lane) - 1u;
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            if (!keep[k]) continue;
            const unsigned long long o =
                out_base + s_cnt[k * (kThreads / 32) + warp] + __popc(ballots[k] & lt);
            if (o >= S.capacity) { atomicOr(&st->error, kErrCapacity); continue; }
            S.x[1][o] = x[k];
            st_comp<F32>(S.vh[1], S.vh32[1], o, vh[k]);
            if (VDIM == 3) {
                st_comp<F32>(S.vy[1], S.vy32[1], o, vy[k]);
                st_comp<F32>(S.vz[1], S.vz32[1], o, vz[k]);
            }
            if (mode & (kModeWriteV | kModeInitHalf)) S.v[o] = vc[k];
            if (DIAG && p.ledger) S.vold[1][o] = (mode & (kModeSyncMcc | kModeInitHalf)) ? vc[k] : vo[k];
        }
        __syncthreads();
    }
    if (mode & kModeDeposit) {
        for (int i = tid; i < p.nx; i += kThreads) {
            const unsigned long long a = sRho[i];
            if (a) atomicAdd(&p.rho_acc[i], a);
        }
    }
}

#include "pic1d_c32.cuh"

// ---- post kernel: products, density, field solve -----------------------------

struct Affine {
    double a, b;
};
struct AffineCompose {
    __device__ Affine operator()(const Affine& l, const Affine& r) const {
        return Affine{r.a * l.a, r.a * l.b + r.b};
    }
};

// Inclusive scan of the affine maps map(i), i < count, over a block of
// kPostThreads threads: out(i, F_i(0)) with F_i = f_i o ... o f_0.  Rounds of
// one map per thread; each round is a warp shuffle scan, one warp scanning the
// warps' totals (with the earlier rounds' composition in front) and two
// barriers.  s_wt holds kPostThreads / 32 + 1 maps.
template <class MapF, class OutF>
__device__ __forceinline__ void block_affine_scan(int count, MapF map, OutF out, Affine* s_wt) {
    constexpr int NW = kPostThreads / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const AffineCompose compose;
    Affine carry{1.0, 0.0};
    for (int base = 0; base < count; base += kPostThreads) {
        const int i = base + tid;
        Affine x = i < count ? map(i) : Affine{1.0, 0.0};
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const Affine y{__shfl_up_sync(0xffffffffu, x.a, o), __shfl_up_sync(0xffffffffu, x.b, o)};
            if (lane >= o) x = compose(y, x);
        }
        if (lane == 31) s_wt[warp] = x;
        __syncthreads();
        if (warp == 0) {
            Affine w = lane < NW ? s_wt[lane] : Affine{1.0, 0.0};
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const Affine y{__shfl_up_sync(0xffffffffu, w.a, o), __shfl_up_sync(0xffffffffu, w.b, o)};
                if (lane >= o) w = compose(y, w);
            }
            Affine ex{__shfl_up_sync(0xffffffffu, w.a, 1), __shfl_up_sync(0xffffffffu, w.b, 1)};
            if (lane == 0) ex = Affine{1.0, 0.0};
            if (lane < NW) s_wt[lane] = compose(carry, ex);
            if (lane == NW - 1) s_wt[NW] = compose(carry, w);
        }
        __syncthreads();
        if (i < count) out(i, compose(s_wt[warp], x).b);
        carry = s_wt[NW];
        __syncthreads();
    }
}

__device__ __forceinline__ double electrode(double offset, const apic_voltage_drive& d, double t) {
    // electrode_potential, src/Simulation.cpp:678-685
    return offset + d.amplitude * sin(2.0 * 3.141592653589793 * d.frequency * t + d.phase);
}

// Shared-memory layout of the post kernel (dynamic): the fixed-point density,
// the solver's constant coefficients and, for the periodic solve, the per-mode
// spectra.  Everything the solve needs is loaded in one round trip at entry.
__host__ __device__ inline size_t post_smem_bytes(int nx, bool dirichlet) {
    return (size_t)nx * 8 /* rho_i */ + (size_t)nx * 8 /* rho */ +
           (dirichlet ? (size_t)2 * nx * 8 : (size_t)2 * nx * 8 /* twiddles */ + (size_t)4 * nx * 8 /* spectra */);
}

template <int VDIM, bool DIRICHLET, bool F32, bool C32 = false>
__global__ void __launch_bounds__(kPostThreads) k_post1d(Params1D p, unsigned post) {
    using Sort = cub::BlockRadixSort<unsigned long long, kPostThreads, kPostItems, int>;
    using ScanU = cub::BlockScan<unsigned, kPostThreads>;
    __shared__ union {
        typename Sort::TempStorage sort;
        typename ScanU::TempStorage scan;
    } tmp;
    __shared__ unsigned s_surv[kMaxSpecies], s_kept[kMaxSpecies], s_bstart[kMaxSpecies], s_nch[kMaxSpecies];
    __shared__ double s_red[kPostThreads / 32];
    __shared__ double s_mean;
    __shared__ unsigned s_carry;
    extern __shared__ __align__(16) unsigned char post_raw[];
    const int nx = p.nx;
    unsigned long long* s_rhoi = reinterpret_cast<unsigned long long*>(post_raw);
    double* s_rho = reinterpret_cast<double*>(s_rhoi + nx);
    double* s_c0 = s_rho + nx;                       // Dirichlet: 1/denominators; periodic: twiddles (2 nx)
    double* s_c1 = s_c0 + nx;                        // Dirichlet: -cp
    double* s_spec = s_c0 + 2 * nx;                  // periodic: 4 nx spectra
    DevState* st = p.st;
    const int tid = threadIdx.x;
    const bool solve = (post & kPostSolve) != 0;

    // -- one round trip: density accumulators and solver coefficients --
    if (solve) {
        for (int i = tid; i < nx; i += kPostThreads) {
            s_rhoi[i] = p.rho_acc[i];
            p.rho_acc[i] = 0ull;
            if (DIRICHLET) {
                if (i < nx - 2) { s_c0[i] = p.thomas_r[i]; s_c1[i] = p.thomas_a[i]; }
            } else {
                s_c0[2 * i] = p.tw[2 * i];
                s_c0[2 * i + 1] = p.tw[2 * i + 1];
            }
        }
    }

    // -- output range table: chunk c of the pass kept its survivors at slots
    //    [c * kTile, c * kTile + surv_c); logical starts are their prefix sums
    //    (the FP32 cell form updates its slots in place: products go after n) --
    constexpr unsigned CHUNK = (unsigned)kTile;
    constexpr int OUT = C32 ? 0 : 1;  // buffer receiving the products
    if (C32) {
        if (tid < p.nspecies) {
            s_surv[tid] = st->n[tid];
            s_bstart[tid] = st->n[tid];
            s_nch[tid] = 0;
            s_kept[tid] = 0;
        }
        __syncthreads();
    }
    for (int s = 0; s < (C32 ? 0 : p.nspecies); ++s) {
        const SpeciesDev& S = p.sp[s];
        const unsigned nch = (st->n[s] + CHUNK - 1) / CHUNK;
        if (tid == 0) s_carry = 0;
        __syncthreads();
        for (unsigned b0 = 0; b0 < nch; b0 += kPostThreads * kPostItems) {
            unsigned cnt[kPostItems], pre[kPostItems];
#pragma unroll
            for (int k = 0; k < kPostItems; ++k) {
                const unsigned c = b0 + tid * kPostItems + k;
                cnt[k] = c < nch ? S.chunk_surv[c] : 0u;
            }
            unsigned total;
            ScanU(tmp.scan).ExclusiveSum(cnt, pre, total);
            const unsigned carry = s_carry;
#pragma unroll
            for (int k = 0; k < kPostItems; ++k) {
                const unsigned c = b0 + tid * kPostItems + k;
                if (c < nch) {
                    S.rstart[1][c] = c * CHUNK;
                    S.rcount[1][c] = cnt[k];
                    S.rlstart[1][c] = carry + pre[k];
                }
            }
            __syncthreads();
            if (tid == 0) s_carry = carry + total;
            __syncthreads();
        }
        if (tid == 0) {
            s_surv[s] = s_carry;
            s_nch[s] = nch;
            s_bstart[s] = nch ? (nch - 1) * CHUNK + S.chunk_surv[nch - 1] : 0u;
            s_kept[s] = 0;
        }
        __syncthreads();
    }

    // -- ionization products, in (parent species, parent slot, product) order --
    unsigned nb = st->nbirths;
    if (nb > p.births_cap) nb = p.births_cap;
    if (nb > (unsigned)kMaxBirths) {
        if (tid == 0) atomicOr(&st->error, kErrBirths);
        nb = kMaxBirths;
    }
    if (p.coll_acc) {
        // collision-energy diagnostics: each product pair's energy in its
        // channel at the parent's position (records come in pairs: secondary, ion)
        for (unsigned j = tid; 2 * j + 1 < nb; j += kPostThreads) {
            const BirthRec a = p.births[2 * j], b = p.births[2 * j + 1];
            const SpeciesDev& A = p.sp[a.species];
            const SpeciesDev& B = p.sp[b.species];
            const double added =
                0.5 * A.mass * A.weight * (a.v[0] * a.v[0] + a.v[1] * a.v[1] + a.v[2] * a.v[2]) +
                0.5 * B.mass * B.weight * (b.v[0] * b.v[0] + b.v[1] * b.v[1] + b.v[2] * b.v[2]);
            const int parent = (int)(a.key >> 56);
            collision_energy_deposit<DIRICHLET>(p, a.x, p.coll_off[p.sp[parent].model] + a.pad, added);
        }
    }
    if (nb > 0) {
        int idx[kPostItems];
        // up to one product per thread: rank tid in item 0 (the blocked scans
        // below then still visit the products in rank order); more: the radix
        // sort's blocked layout, ranks tid * kPostItems + k
        const bool one_each = nb <= (unsigned)kPostThreads;
        auto rank_of = [&](int k) -> unsigned {
            return one_each ? (k == 0 ? (unsigned)tid : nb) : (unsigned)(tid * kPostItems + k);
        };
        if (one_each) {
            // a few products (the usual case): each finds its rank by counting
            // the smaller keys, one key per thread
            __shared__ unsigned long long s_keys[kPostThreads];
            __shared__ int s_order[kPostThreads];
            if (tid < (int)nb) s_keys[tid] = p.births[tid].key;
            __syncthreads();
            if (tid < (int)nb) {
                const unsigned long long key = s_keys[tid];
                unsigned r = 0;
                for (unsigned q = 0; q < nb; ++q) {
                    const unsigned long long o = s_keys[q];
                    r += (o < key || (o == key && q < (unsigned)tid)) ? 1u : 0u;
                }
                s_order[r] = tid;
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < kPostItems; ++k) {
                const unsigned rank = rank_of(k);
                idx[k] = rank < nb ? s_order[rank] : 0;
            }
        } else {
            unsigned long long keys[kPostItems];
#pragma unroll
            for (int k = 0; k < kPostItems; ++k) {
                const unsigned i = tid * kPostItems + k;
                keys[k] = i < nb ? p.births[i].key : ~0ull;
                idx[k] = (int)i;
            }
            Sort(tmp.sort).Sort(keys, idx);
        }
        __syncthreads();
        double bx[kPostItems], bvh[kPostItems], bv[kPostItems][3];
        int bs[kPostItems];
        bool keep[kPostItems];
#pragma unroll
        for (int k = 0; k < kPostItems; ++k) {
            keep[k] = false;
            bs[k] = -1;
            const unsigned rank = rank_of(k);
            if (rank >= nb) continue;
            const BirthRec r = p.births[idx[k]];
            const SpeciesDev& S = p.sp[r.species];
            bs[k] = r.species;
            bx[k] = r.x;
            bv[k][0] = r.v[0]; bv[k][1] = r.v[1]; bv[k][2] = r.v[2];
            const double E = gather(p.E, cic<DIRICHLET>(r.x, p));
            // append_product: v_half = v, then initialize_leapfrog_half_step, src/Simulation.cpp:985-1004
            bvh[k] = r.v[0] - S.hqm * E * p.dt;
            keep[k] = true;
            if (post & kPostPushBirths) {
                bvh[k] = bvh[k] + S.qm * E * p.dt;
                bx[k] = bx[k] + bvh[k] * p.dt;
                if (!DIRICHLET) {
                    bx[k] = wrap_periodic(bx[k], p.L);
                } else if (bx[k] < 0.0 || bx[k] > p.L) {
                    if (p.ledger) {  // electric work of a wall crossing, src/Simulation.cpp:1047-1056
                        const double hmw = 0.5 * S.mass * S.weight;
                        atomicAdd(&st->work[r.species], hmw * bvh[k] * bvh[k] - hmw * bv[k][0] * bv[k][0]);
                    }
                    const double sp2 = bvh[k] * bvh[k] + bv[k][1] * bv[k][1] + bv[k][2] * bv[k][2];
                    const int side = bx[k] < 0.0 ? 0 : 1;
                    atomicAdd(&st->lost[r.species][side], 1ull);
                    atomicAdd(&st->lost_energy[r.species][side], 0.5 * S.mass * S.weight * sp2);
                    keep[k] = false;
                }
                if (keep[k] && solve) {
                    const Cic d = cic<DIRICHLET>(bx[k], p);
                    long long a0, a1;
                    deposit_contrib<DIRICHLET>(d, S, p, a0, a1);
                    atomicAdd(&s_rhoi[d.i0], (unsigned long long)a0);
                    atomicAdd(&s_rhoi[d.i1], (unsigned long long)a1);
                }
            }
        }
        for (int s = 0; s < p.nspecies; ++s) {
            unsigned flags[kPostItems], ranks[kPostItems];
#pragma unroll
            for (int k = 0; k < kPostItems; ++k) flags[k] = (keep[k] && bs[k] == s) ? 1u : 0u;
            unsigned total;
            __syncthreads();
            ScanU(tmp.scan).ExclusiveSum(flags, ranks, total);
            const SpeciesDev& S = p.sp[s];
#pragma unroll
            for (int k = 0; k < kPostItems; ++k) {
                if (!flags[k]) continue;
                const unsigned long long o = (unsigned long long)s_bstart[s] + ranks[k];
                if (o >= S.capacity) { atomicOr(&st->error, kErrCapacity); continue; }
                if (C32) {
                    int c;
                    float f;
                    position_to_cell<DIRICHLET>(bx[k], p, c, f);
                    S.cell[OUT][o] = c;
                    S.off[OUT][o] = f;
                } else {
                    S.x[OUT][o] = bx[k];
                }
                st_comp<F32>(S.vh[OUT], S.vh32[OUT], o, bvh[k]);
                if (VDIM == 3) {
                    st_comp<F32>(S.vy[OUT], S.vy32[OUT], o, bv[k][1]);
                    st_comp<F32>(S.vz[OUT], S.vz32[OUT], o, bv[k][2]);
                }
                S.v[o] = bv[k][0];
                if (p.ledger) S.vold[OUT][o] = bv[k][0];
            }
            if (tid == 0) s_kept[s] = total;
        }
        __syncthreads();
    }
    if (tid < p.nspecies) {
        const SpeciesDev& S = p.sp[tid];
        unsigned kept = s_kept[tid];
        if ((unsigned long long)s_bstart[tid] + kept > S.capacity) {
            atomicOr(&st->error, kErrCapacity);
            kept = S.capacity > s_bstart[tid] ? S.capacity - s_bstart[tid] : 0u;
        }
        // the FP32 cell form's slots include holes: the configured capacity
        // bounds the live particles (max_particles_per_species)
        if (C32 && (unsigned long long)(s_surv[tid] - st->holes[tid]) + kept > S.live_cap)
            atomicOr(&st->error, kErrCapacity);
        unsigned nr = s_nch[tid];
        if (kept && !C32) {  // this pass's products form one more range after the last chunk
            S.rstart[1][nr] = s_bstart[tid];
            S.rcount[1][nr] = kept;
            S.rlstart[1][nr] = s_surv[tid];
            ++nr;
        }
        st->nranges[tid] = nr;
        st->n[tid] = s_surv[tid] + kept;
    }
    if (tid == 0) st->nbirths = 0;
    if (!solve) return;
    __syncthreads();

    // -- density: fixed point -> FP64 ---------------------------------------
    double local = 0.0;
    for (int i = tid; i < nx; i += kPostThreads) {
        const double r = (double)(long long)s_rhoi[i] * p.inv_rho_scale;
        s_rho[i] = r;
        p.rho[i] = r;
        local += r;
    }
    const double field_time = (post & kPostAdvance) ? st->time + p.dt : st->time;
    if (!DIRICHLET) {
        // solve_periodic_spectral(Grid&), src/FieldSolver.cpp:407-440
        for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
        if ((tid & 31) == 0) s_red[tid >> 5] = local;
        __syncthreads();
        if (tid == 0) {
            double m = 0.0;
            for (int w = 0; w < kPostThreads / 32; ++w) m += s_red[w];
            s_mean = m / (double)nx;
        }
        __syncthreads();
        const double mean = s_mean;
        const double twopi = 2.0 * 3.141592653589793;
        double* sp_r = s_spec;
        double* sp_i = s_spec + nx;
        double* se_r = s_spec + 2 * nx;
        double* se_i = s_spec + 3 * nx;
        // forward transform: mode k per thread, summed over j in the reference's order,
        // then the per-mode potential and field, src/FieldSolver.cpp:418-428
        for (int k = tid; k < nx; k += kPostThreads) {
            if (k == 0) { sp_r[0] = sp_i[0] = se_r[0] = se_i[0] = 0.0; continue; }
            double re = 0.0, im = 0.0;
            unsigned m = 0;
            for (int j = 0; j < nx; ++j) {
                const double a = s_rho[j] - mean;
                re += a * s_c0[2 * m];
                im += a * (-s_c0[2 * m + 1]);
                m += (unsigned)k;
                if (m >= (unsigned)nx) m -= (unsigned)nx;
            }
            re /= (double)nx;
            im /= (double)nx;
            const double kk = (k <= nx / 2) ? (double)k : -(double)(nx - k);
            const double wave = twopi * kk / p.L;
            const double den = p.eps * wave * wave;
            const double pr = re / den, pi = im / den;
            sp_r[k] = pr;
            sp_i[k] = pi;
            se_r[k] = wave * pi;    // -(0,1) * wave * phik
            se_i[k] = -(wave * pr);
        }
        __syncthreads();
        // inverse: each node j sums its modes in order k = 1 .. n-1
        for (int j = tid; j < nx; j += kPostThreads) {
            double ph = 0.0, ef = 0.0;
            unsigned m = (unsigned)j;
            for (int k = 1; k < nx; ++k) {
                const double cs = s_c0[2 * m], sn = s_c0[2 * m + 1];
                ph += sp_r[k] * cs - sp_i[k] * sn;
                ef += se_r[k] * cs - se_i[k] * sn;
                m += (unsigned)j;
                if (m >= (unsigned)nx) m -= (unsigned)nx;
            }
            p.phi[j] = ph;
            p.E[j] = ef;
        }
    } else {
        __syncthreads();
        // solve_dirichlet_tridiagonal, src/FieldSolver.cpp:733-759, with the
        // forward sweep and the back substitution evaluated as affine scans
        const double phil = electrode(p.phi_left, p.drive_left, field_time);
        const double phir = electrode(p.phi_right, p.drive_right, field_time);
        const int m = nx - 2;
        const double dx2 = p.dx * p.dx;
        __shared__ Affine s_wt[kPostThreads / 32 + 1];
        double* s_dp = reinterpret_cast<double*>(s_rhoi);  // the fixed-point density is converted already
        // forward sweep: dp_i = r_i (d_i + dp_{i-1})
        block_affine_scan(
            m,
            [&](int i) {
                double d = s_rho[i + 1] * dx2 / p.eps;
                if (i == 0) d += phil;
                if (i == m - 1) d += phir;
                const double r = s_c0[i];
                return Affine{r, r * d};
            },
            [&](int i, double v) { s_dp[i] = v; }, s_wt);
        // back substitution in reverse: z_t = a[m-1-t] z_{t-1} + dp[m-1-t]
        double* s_phi = s_c0;  // coefficients no longer needed
        block_affine_scan(
            m, [&](int t) { return Affine{s_c1[m - 1 - t], s_dp[m - 1 - t]}; },
            [&](int t, double v) { s_phi[m - t] = v; }, s_wt);
        if (tid == 0) {
            s_phi[0] = phil;
            s_phi[nx - 1] = phir;
        }
        __syncthreads();
        for (int i = tid; i < nx; i += kPostThreads) {
            double e;
            if (i == 0) e = -(s_phi[1] - s_phi[0]) / p.dx;
            else if (i == nx - 1) e = -(s_phi[nx - 1] - s_phi[nx - 2]) / p.dx;
            else e = -(s_phi[i + 1] - s_phi[i - 1]) / (2.0 * p.dx);
            p.E[i] = e;
            p.phi[i] = s_phi[i];
        }
    }
    if (tid == 0 && (post & kPostAdvance)) {
        st->time = field_time;
        st->step = st->step + 1ull;
    }
}

// FP32 form: host copies go through an FP64 staging array.
__global__ void k_narrow1d(const double* __restrict__ in, float* __restrict__ out, unsigned n) {
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = (float)in[i];
}
__global__ void k_widen1d(const float* __restrict__ in, double* __restrict__ out, unsigned n) {
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = (double)in[i];
}

// ---- campaign diagnostics: moments of a sample ------------------------------

constexpr int kMomThreads = 512;
constexpr int kMaxEedfRegions = APIC_MAX_EEDF_REGIONS;
constexpr size_t kMomentSmemMax = 200 * 1024;  // moment rows (5 nx doubles) + a staged EEDF histogram

struct MomentArgs {
    double* scratch;               // [5][nspecies][nx] moments of this sample (zero on entry)
    int eedf_species;              // -1: no phase EEDF this sample
    int regions;
    double xmin[kMaxEedfRegions], xmax[kMaxEedfRegions];
    unsigned bins;
    double emax, escale;
    unsigned long long* eedf_cnt;  // [regions][2] of the sample's phase bin
    double* eedf_sum;              // [regions][7]
    double* eedf_hist;             // [regions][bins]
    int hist_shared;               // histogram staged in shared memory
};

// Species::deposit_velocity_moments (src/Species.cpp:285-336) of every species
// and accumulate_phase_eedf (src/Simulation.cpp:1238-1285) of the EEDF species,
// on the state right after a step's collision part (time-centred v in S.v, the
// layout dense).  Per CTA the five moment rows live in shared memory (FP64
// atomics), then are added to the sample's scratch rows; the EEDF sums are
// warp-reduced per region.  One CTA per SM.
template <int VDIM, bool DIRICHLET, bool F32>
__global__ void __launch_bounds__(kMomThreads) k_moments1d(Params1D p, MomentArgs a) {
    extern __shared__ __align__(16) unsigned char mom_raw[];
    double* sm = reinterpret_cast<double*>(mom_raw);  // [5][nx]
    double* sh = sm + 5 * p.nx;                       // [regions][bins] when staged
    __shared__ double s_es[kMaxEedfRegions][7];
    __shared__ unsigned long long s_ec[kMaxEedfRegions][2];
    const int tid = threadIdx.x, lane = tid & 31;
    const int nx = p.nx;
    for (int s = 0; s < p.nspecies; ++s) {
        const SpeciesDev& S = p.sp[s];
        const unsigned n = p.st->n[s];
        const bool eedf = s == a.eedf_species;
        const unsigned hist_n = eedf && a.hist_shared ? (unsigned)a.regions * a.bins : 0u;
        for (int i = tid; i < 5 * nx; i += kMomThreads) sm[i] = 0.0;
        for (unsigned i = tid; i < hist_n; i += kMomThreads) sh[i] = 0.0;
        if (tid < kMaxEedfRegions * 7) (&s_es[0][0])[tid] = 0.0;
        if (tid < kMaxEedfRegions * 2) (&s_ec[0][0])[tid] = 0ull;
        __syncthreads();
        const double w = S.weight;
        const double hmw = 0.5 * S.mass * S.weight;
        double* hist = a.hist_shared ? sh : a.eedf_hist;
        for (unsigned base = blockIdx.x * kMomThreads; base < n; base += gridDim.x * kMomThreads) {
            const unsigned i = base + tid;
            const bool live = i < n;
            double x = 0.0, v = 0.0, vy = 0.0, vz = 0.0;
            if (live) {
                x = S.x[0][i];
                v = S.v[i];
                if (VDIM == 3) {
                    vy = ld_comp<F32>(S.vy[0], S.vy32[0], i);
                    vz = ld_comp<F32>(S.vz[0], S.vz32[0], i);
                }
                const Cic d = cic<DIRICHLET>(x, p);
                const double pe = hmw * (v * v + vy * vy + vz * vz);
                const double vol0 = node_volume<DIRICHLET>(p, d.i0), vol1 = node_volume<DIRICHLET>(p, d.i1);
                const double r0 = w * d.w0 / vol0, r1 = w * d.w1 / vol1;
                atomicAdd(sm + d.i0, r0);
                atomicAdd(sm + nx + d.i0, r0 * v);
                atomicAdd(sm + 2 * nx + d.i0, r0 * vy);
                atomicAdd(sm + 3 * nx + d.i0, r0 * vz);
                atomicAdd(sm + 4 * nx + d.i0, pe * d.w0 / vol0);
                atomicAdd(sm + d.i1, r1);
                atomicAdd(sm + nx + d.i1, r1 * v);
                atomicAdd(sm + 2 * nx + d.i1, r1 * vy);
                atomicAdd(sm + 3 * nx + d.i1, r1 * vz);
                atomicAdd(sm + 4 * nx + d.i1, pe * d.w1 / vol1);
            }
            if (eedf) {
                const double vsq = v * v + (VDIM == 3 ? vy * vy + vz * vz : 0.0);
                const double energy = 0.5 * S.mass * vsq / a.escale;
                for (int r = 0; r < a.regions; ++r) {
                    const bool in = live && !(x < a.xmin[r] || x > a.xmax[r]);
                    const bool over = in && energy >= a.emax;
                    const unsigned c0 = __popc(__ballot_sync(0xffffffffu, in));
                    if (c0 == 0) continue;  // warp-uniform
                    const unsigned c1 = __popc(__ballot_sync(0xffffffffu, over));
                    double q[7] = {in ? w : 0.0, over ? w : 0.0, in ? w * energy : 0.0,
                                   in ? w * energy * energy : 0.0, in ? w * v : 0.0, in ? w * vy : 0.0,
                                   in ? w * vz : 0.0};
#pragma unroll
                    for (int k = 0; k < 7; ++k) q[k] = warp_sum(q[k]);
                    if (lane == 0) {
                        atomicAdd(&s_ec[r][0], (unsigned long long)c0);
                        if (c1) atomicAdd(&s_ec[r][1], (unsigned long long)c1);
#pragma unroll
                        for (int k = 0; k < 7; ++k)
                            if (q[k] != 0.0) atomicAdd(&s_es[r][k], q[k]);
                    }
                    if (in && !over) {
                        unsigned long long b = (unsigned long long)(energy / a.emax * (double)a.bins);
                        if (b > a.bins - 1) b = a.bins - 1;
                        atomicAdd(hist + (size_t)r * a.bins + b, w);
                    }
                }
            }
        }
        __syncthreads();
        for (int i = tid; i < 5 * nx; i += kMomThreads) {
            const double val = sm[i];
            if (val != 0.0) {
                const int q = i / nx, j = i - q * nx;
                atomicAdd(a.scratch + ((size_t)q * p.nspecies + s) * nx + j, val);
            }
        }
        if (eedf) {
            for (unsigned i = tid; i < hist_n; i += kMomThreads)
                if (sh[i] != 0.0) atomicAdd(a.eedf_hist + i, sh[i]);
            if (tid < a.regions * 7) {
                const double val = s_es[tid / 7][tid % 7];
                if (val != 0.0) atomicAdd(a.eedf_sum + tid, val);
            }
            if (tid < a.regions * 2) {
                const unsigned long long c = s_ec[tid / 2][tid % 2];
                if (c) atomicAdd(a.eedf_cnt + tid, c);
            }
        }
        __syncthreads();
    }
}

// The sample's moments and the fields (phi, E, E^2) added to the window sums
// and to the sample's phase bin (null: none); the scratch rows are cleared for
// the next sample (src/Simulation.cpp:1335-1361).
__global__ void k_sa_fold1d(Params1D p, double* scratch, double* tot, double* bin) {
    const int nx = p.nx;
    const int moments = 5 * p.nspecies * nx;
    const int total = moments + 3 * nx;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        double v;
        if (i < moments) {
            v = scratch[i];
            scratch[i] = 0.0;
        } else {
            const int f = (i - moments) / nx, j = i - moments - f * nx;
            const double e = p.E[j];
            v = f == 0 ? p.phi[j] : (f == 1 ? e : e * e);
        }
        tot[i] += v;
        if (bin) bin[i] += v;
    }
}

// Simulation::sample reductions (src/Simulation.cpp:1140-1161,
// src/Species.cpp:338-351): per-block partial sums, then the last block adds
// the partials in block order, so the result does not depend on scheduling.
constexpr int kSampleBlocks = 148;
__global__ void __launch_bounds__(256) k_sample1d(Params1D p, double* partial, unsigned* done, double* out) {
    __shared__ double red[8];
    __shared__ bool last;
    const int tid = threadIdx.x;
    for (int s = 0; s < p.nspecies; ++s) {
        const SpeciesDev& S = p.sp[s];
        const unsigned n = p.st->n[s];
        const double hmw = 0.5 * S.mass * S.weight;
        double acc = 0.0;
        for (unsigned i = blockIdx.x * 256 + tid; i < n; i += gridDim.x * 256) {
            if (p.c32 && S.cell[0][i] == kDeadCell) continue;  // a hole of the FP32 cell form
            const double v = S.v[i];
            double sq = v * v;
            if (p.vdim == 3) {
                const double vy = p.f32 ? (double)S.vy32[0][i] : S.vy[0][i];
                const double vz = p.f32 ? (double)S.vz32[0][i] : S.vz[0][i];
                sq += vy * vy + vz * vz;
            }
            acc += hmw * sq;
        }
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if ((tid & 31) == 0) red[tid >> 5] = acc;
        __syncthreads();
        if (tid == 0) {
            double b = 0.0;
            for (int w = 0; w < 8; ++w) b += red[w];
            partial[s * gridDim.x + blockIdx.x] = b;
        }
        __syncthreads();
    }
    if (tid == 0) {
        __threadfence();
        last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || tid != 0) return;
    __threadfence();
    for (int s = 0; s < p.nspecies; ++s) {
        double e = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) e += ((volatile double*)partial)[s * gridDim.x + b];
        out[s] = e;
    }
    double fe = 0.0, l1 = 0.0;
    for (int i = 0; i < p.nx; ++i) {
        const double vol = p.dirichlet ? ((i == 0 || i + 1 == p.nx) ? 0.5 * p.dx : p.dx) : p.dx;
        fe += 0.5 * p.eps * p.E[i] * p.E[i] * vol;
        l1 += fabs(p.rho[i]) * vol;
    }
    out[kMaxSpecies] = fe;
    out[kMaxSpecies + 1] = l1;
    *done = 0;
}

// interpolate_electric(Grid&, x) at query points, src/FieldSolver.cpp:909-924
template <bool DIRICHLET>
__global__ void k_gather_points1d(Params1D p, const double* xq, double* eq, int nq) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nq) return;
    eq[i] = gather(p.E, cic<DIRICHLET>(xq[i], p));
}

// ---- stateless collide (replay or Philox) -----------------------------------

__global__ void k_collide3(MccModelDev m, int n, double* v3, double dt, const uint64_t* draws,
                           const uint64_t* offsets, uint64_t seed, uint32_t step, uint32_t stream,
                           apic_collide_stats* stats) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v[3] = {v3[3 * i], v3[3 * i + 1], v3[3 * i + 2]};
    CollideResult r;
    apic_collide_stats out;
    memset(&out, 0, sizeof out);
    auto on_sec = [&](int ch, const double* vs, const double* vi) {
        const int k = out.nsecondaries++;
        if (k < 4) {
            out.secondary_channel[k] = ch;
            for (int d = 0; d < 3; ++d) {
                out.secondary_velocity[k][d] = vs[d];
                out.secondary_ion_velocity[k][d] = vi[d];
            }
        }
    };
    unsigned used;
    if (draws) {
        ReplayStream s{draws + offsets[i], offsets[i + 1] - offsets[i]};
        collide3(m, v, dt, s, r, on_sec);
        used = s.index;
    } else {
        PhiloxStream s(seed, (uint32_t)i, step, stream);
        collide3(m, v, dt, s, r, on_sec);
        used = s.index;
    }
    v3[3 * i] = v[0]; v3[3 * i + 1] = v[1]; v3[3 * i + 2] = v[2];
    out.candidates = r.candidates;
    out.null_collisions = r.nulls;
    for (int c = 0; c < kMaxChannels; ++c) {
        out.channel_collisions[c] = r.channel[c];
        out.energy_change[c] = r.energy_change[c];
    }
    out.removed = r.removed ? 1 : 0;
    out.draws = used | (r.error ? 0x80000000u : 0u);
    stats[i] = out;
}

// ---- host side ----------------------------------------------------------------

cudaError_t bounded_wait(cudaStream_t stream, double seconds) {
    cudaEvent_t ev;
    cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
    e = cudaEventRecord(ev, stream);
    if (e != cudaSuccess) { cudaEventDestroy(ev); return e; }
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        e = cudaEventQuery(ev);
        if (e != cudaErrorNotReady) break;
        const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > seconds) { e = cudaErrorNotReady; break; }
        std::this_thread::sleep_for(std::chrono::microseconds(el < 0.01 ? 2 : 200));
    }
    cudaEventDestroy(ev);
    return e;
}

int status_from_device(unsigned w) {
    if (w & kErrMajorant) return APIC_ERR_MAJORANT;
    if (w & kErrCandidates) return APIC_ERR_CANDIDATES;
    if (w & kErrNonFinite) return APIC_ERR_NONFINITE;
    if (w & (kErrCapacity | kErrBirths | kErrCandBuffer)) return APIC_ERR_CAPACITY;
    if (w & kErrTimeout) return APIC_ERR_TIMEOUT;
    if (w & kErrReplay) return APIC_ERR_INVALID;
    return APIC_OK;
}

std::string describe_device_error(unsigned w) {
    std::string s;
    if (w & kErrMajorant) s += "MCC total collision frequency exceeds configured max_frequency; ";
    if (w & kErrCandidates) s += "MCC candidate limit exceeded; reduce dt or increase max_candidates_per_particle; ";
    if (w & kErrNonFinite) s += "particle state became non-finite; ";
    if (w & kErrCapacity) s += "reactive collisions exceeded max_particles_per_species; ";
    if (w & kErrBirths) s += "ionization products in one step exceeded the per-step product buffer; ";
    if (w & kErrCandBuffer) s += "collision candidates of one step exceeded the candidate buffer; ";
    if (w & kErrTimeout) s += "device look-back wait timed out; ";
    if (w & kErrReplay) s += "recorded draw array exhausted; ";
    return s;
}

// validate_spatial_average_1d, src/Config.cpp:1377-1524, for an enabled
// spatial average (the EEDF species by index, its regions by bounds).
void validate_spatial_average(const apic_config1d& c, const apic_spatial_average1d& a) {
    if (a.eedf_species < 0) {
        require(a.eedf_bins == 0 && a.eedf_energy_max == 0.0 && a.eedf_regions == 0,
                "disabled phase_eedf cannot configure species, bins, energy maximum, or regions");
    } else {
        require(a.phase_bins != 0, "phase_eedf requires spatial averaging with phase bins");
        require(a.eedf_bins != 0 && a.eedf_bins <= 1000000 && std::isfinite(a.eedf_energy_max) &&
                    a.eedf_energy_max > 0.0 && a.eedf_regions > 0,
                "phase_eedf requires a species, 1..1000000 bins, a positive energy maximum, and at least one region");
        require(a.eedf_species < c.nspecies, "phase_eedf species does not exist: " + std::to_string(a.eedf_species));
        require(a.eedf_regions <= kMaxEedfRegions, "phase_eedf supports at most 8 regions on the device",
                APIC_ERR_UNSUPPORTED);
        for (int r = 0; r < a.eedf_regions; ++r)
            require(std::isfinite(a.eedf_x_min[r]) && std::isfinite(a.eedf_x_max[r]) && a.eedf_x_min[r] >= 0.0 &&
                        a.eedf_x_max[r] <= c.length && a.eedf_x_max[r] > a.eedf_x_min[r],
                    "phase_eedf regions require unique safe names and 0 <= x_min < x_max <= length");
    }
    require(std::isfinite(a.rf_frequency) && a.rf_frequency >= 0.0,
            "spatial_average_rf_frequency must be non-negative and finite");
    require(a.interval != 0, "spatial_average_interval must be positive");
    require(a.start_step != 0 && a.end_step >= a.start_step, "spatial_average requires 1 <= start_step <= end_step");
    if (a.rf_frequency == 0.0) {
        require(a.rf_cycles == 0 && a.phase_bins == 0,
                "spatial_average_rf_cycles requires positive spatial_average_rf_frequency");
        return;
    }
    require(a.rf_cycles != 0, "positive spatial_average_rf_frequency requires positive spatial_average_rf_cycles");
    const double spc_value = 1.0 / (a.rf_frequency * c.dt);
    require(std::isfinite(spc_value) && spc_value <= (double)std::numeric_limits<long long>::max(),
            "spatial-average RF steps per cycle are invalid");
    const size_t spc = (size_t)std::llround(spc_value);
    require(spc != 0 && !(std::fabs(spc_value - (double)spc) > 1e-10 * std::max(1.0, spc_value)),
            "spatial-average RF period must contain an integer number of timesteps");
    require(a.rf_cycles <= std::numeric_limits<size_t>::max() / spc, "spatial-average RF window step count overflows");
    require(a.end_step - a.start_step + 1 == a.rf_cycles * spc,
            "spatial-average step window does not span the configured whole RF cycles");
    require(a.end_step % spc == 0, "spatial-average RF window must end at the time-zero drive phase");
    require(spc % a.interval == 0, "spatial_average_interval must divide RF steps per cycle");
    const size_t per_cycle = spc / a.interval;
    require(!(a.phase_bins > per_cycle || (a.phase_bins != 0 && per_cycle % a.phase_bins != 0)),
            "spatial_average_phase_bins must divide the sampled RF cycle");
    for (const apic_voltage_drive& d : {c.drive_left, c.drive_right}) {
        if (d.amplitude == 0.0) continue;
        require(!(std::fabs(d.frequency - a.rf_frequency) > 1e-12 * std::max(d.frequency, a.rf_frequency)),
                "spatial-average RF frequency does not match the electrode drive");
    }
}

struct Sim1D {
    apic_config1d cfg{};
    std::string last_error;
    cudaStream_t stream = nullptr;
    int device = 0;
    Params1D p{};
    DevState* st = nullptr;
    std::vector<void*> allocations;
    std::vector<std::vector<double>> tables;  // host copies (kept for safe_speed)
    bool fp32 = false;      // FP32 velocities (APIC_FP32 and APIC_FP32_STORAGE)
    bool c32 = false;       // FP32 cell form (APIC_FP32): cell + offset positions, FP32 arithmetic
    bool pending = false;   // collision part of the last step not yet applied
    bool initialized = false;
    int parity = 0;         // which of the two buffers holds the current state
    double time = 0.0;
    uint64_t step = 0;
    double neutral_stddev[kMaxModels] = {0, 0, 0, 0};
    double wait_limit_s = 600.0;  // longest host wait for the handle's stream

    template <class T>
    T* dalloc(size_t count) {
        void* ptr = nullptr;
        APIC_CUDA(cudaMalloc(&ptr, std::max<size_t>(count, 1) * sizeof(T)));
        allocations.push_back(ptr);
        APIC_CUDA(cudaMemsetAsync(ptr, 0, std::max<size_t>(count, 1) * sizeof(T), stream));
        return static_cast<T*>(ptr);
    }

    // ---- campaign diagnostics (spatial average, phase bins, collision energy, phase EEDF) ----
    struct SpatialAvg {
        bool on = false;
        apic_spatial_average1d cfg{};
        size_t spc = 0, P = 0;  // RF steps per cycle, phase bins
        int nch = 0;
        double* tot = nullptr;         // [5][nspecies][nx] moments + [3][nx] fields
        double* phase = nullptr;       // [P][same block]
        double* scratch = nullptr;     // [5][nspecies][nx] of one sample
        double* coll = nullptr;        // [nch][nx]
        double* coll_phase = nullptr;  // [P][nch][nx]
        unsigned long long* eedf_cnt = nullptr;  // [P][regions][2]
        double* eedf_sum = nullptr;              // [P][regions][7]
        double* eedf_hist = nullptr;             // [P][regions][bins]
        bool hist_shared = false;
        uint64_t samples = 0, coll_steps = 0;
        std::vector<uint64_t> psamples, pcoll;
    } sa;

    size_t sa_block() const { return (5 * (size_t)cfg.nspecies + 3) * cfg.nx; }

    void enable_spatial_average(const apic_spatial_average1d& a) {
        require(!initialized, "spatial averaging must be enabled before initialize() or resume()", APIC_ERR_STATE);
        require(!c32, "spatial averaging runs in the FP64 and FP32_STORAGE forms", APIC_ERR_UNSUPPORTED);
        require(!sa.on, "spatial averaging is already enabled", APIC_ERR_STATE);
        validate_spatial_average(cfg, a);
        sa.cfg = a;
        sa.spc = a.rf_frequency > 0.0 ? (size_t)std::llround(1.0 / (a.rf_frequency * cfg.dt)) : 0;
        sa.P = a.phase_bins;
        sa.nch = 0;
        for (int m = 0; m < cfg.nmodels; ++m) {
            p.coll_off[m] = sa.nch;
            sa.nch += cfg.models[m].nch;
        }
        if (cfg.bgk_enabled) sa.nch = 1;  // the "bgk" channel, src/Simulation.cpp:484-485
        const size_t nx = cfg.nx;
        sa.tot = dalloc<double>(sa_block());
        sa.phase = dalloc<double>(sa.P * sa_block());
        sa.scratch = dalloc<double>(5 * (size_t)cfg.nspecies * nx);
        sa.coll = dalloc<double>((size_t)sa.nch * nx);
        sa.coll_phase = dalloc<double>(sa.P * (size_t)sa.nch * nx);
        if (a.eedf_species >= 0) {
            const size_t R = (size_t)a.eedf_regions;
            sa.eedf_cnt = dalloc<unsigned long long>(sa.P * R * 2);
            sa.eedf_sum = dalloc<double>(sa.P * R * 7);
            sa.eedf_hist = dalloc<double>(sa.P * R * a.eedf_bins);
            sa.hist_shared = (5 * nx + R * a.eedf_bins) * sizeof(double) <= kMomentSmemMax;
        }
        sa.psamples.assign(sa.P, 0);
        sa.pcoll.assign(sa.P, 0);
        APIC_CUDA(cudaStreamSynchronize(stream));
        sa.on = true;
        drop_graphs();
    }

    // begin_spatial_collision_step, src/Simulation.cpp:1214-1236: arms the
    // collision-energy deposit of the pass that applies collision step `cs`.
    void arm_collision_step(uint64_t cs) {
        p.coll_acc = nullptr;
        p.coll_phase_acc = nullptr;
        const auto& a = sa.cfg;
        if (!sa.on || sa.nch == 0 || cs < a.start_step || cs > a.end_step) return;
        p.coll_acc = sa.coll;
        ++sa.coll_steps;
        if (sa.P) {
            const size_t bin = (size_t)((cs - a.start_step) % sa.spc) * sa.P / sa.spc;
            p.coll_phase_acc = sa.coll_phase + bin * (size_t)sa.nch * cfg.nx;
            ++sa.pcoll[bin];
        }
    }
    void disarm() {
        p.coll_acc = nullptr;
        p.coll_phase_acc = nullptr;
    }

    // species_power_transfer, src/Simulation.cpp:1094-1132: keeps each
    // particle's end-of-step v (one more FP64 array per buffer, 16 bytes of
    // traffic per particle-step) and runs the diagnostics pass instantiation.
    void enable_power_transfer() {
        require(!c32, "the electric-work ledger runs in the FP64 and FP32_STORAGE forms", APIC_ERR_UNSUPPORTED);
        require(!initialized, "the electric-work ledger must be enabled before initialize() or resume()",
                APIC_ERR_STATE);
        if (p.ledger) return;
        for (int s = 0; s < cfg.nspecies; ++s) {
            p.sp[s].vold[0] = dalloc<double>(cfg.species[s].capacity);
            p.sp[s].vold[1] = dalloc<double>(cfg.species[s].capacity);
        }
        APIC_CUDA(cudaStreamSynchronize(stream));
        p.ledger = 1;
        drop_graphs();
    }

    bool sample_step(uint64_t k) const {
        const auto& a = sa.cfg;
        return sa.on && k >= a.start_step && k <= a.end_step && (k - a.start_step) % a.interval == 0;
    }

    // accumulate_spatial_average (src/Simulation.cpp:1287-1370) after step k:
    // the pending collision part is applied first (one pass that writes the
    // time-centred v), then the moments, the fields and the phase EEDF.
    void take_sample(uint64_t k) {
        if (pending) {
            arm_collision_step(step);
            launch_pass(kModeSyncMcc | kModeWriteV, 0);
            disarm();
            pending = false;
        }
        const auto& a = sa.cfg;
        size_t bin = sa.P;
        if (sa.P) {
            const size_t per_cycle = sa.spc / a.interval;
            bin = (size_t)((k - a.start_step) / a.interval) % per_cycle * sa.P / per_cycle;
        }
        MomentArgs m{};
        m.scratch = sa.scratch;
        m.eedf_species = (bin < sa.P && a.eedf_species >= 0) ? a.eedf_species : -1;
        size_t smem = 5 * cfg.nx * sizeof(double);
        if (m.eedf_species >= 0) {
            const size_t R = (size_t)a.eedf_regions;
            m.regions = a.eedf_regions;
            for (int r = 0; r < a.eedf_regions; ++r) { m.xmin[r] = a.eedf_x_min[r]; m.xmax[r] = a.eedf_x_max[r]; }
            m.bins = (unsigned)a.eedf_bins;
            m.emax = a.eedf_energy_max;
            m.escale = cfg.units == APIC_SI ? 1.602176634e-19 : 1.0;  // include/pic/Types.hpp:9
            m.eedf_cnt = sa.eedf_cnt + bin * R * 2;
            m.eedf_sum = sa.eedf_sum + bin * R * 7;
            m.eedf_hist = sa.eedf_hist + bin * R * a.eedf_bins;
            m.hist_shared = sa.hist_shared ? 1 : 0;
            if (sa.hist_shared) smem += R * a.eedf_bins * sizeof(double);
        }
        const Params1D q = pass_params(0);
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        const bool dir = cfg.boundary == APIC_DIRICHLET;
        const int form = (cfg.velocity_dimensions == 3 ? 4 : 0) | (dir ? 2 : 0) | (fp32 ? 1 : 0);
        switch (form) {
            case 0: k_moments1d<1, false, false><<<sms, kMomThreads, smem, stream>>>(q, m); break;
            case 1: k_moments1d<1, false, true><<<sms, kMomThreads, smem, stream>>>(q, m); break;
            case 2: k_moments1d<1, true, false><<<sms, kMomThreads, smem, stream>>>(q, m); break;
            case 3: k_moments1d<1, true, true><<<sms, kMomThreads, smem, stream>>>(q, m); break;
            case 4: k_moments1d<3, false, false><<<sms, kMomThreads, smem, stream>>>(q, m); break;
            case 5: k_moments1d<3, false, true><<<sms, kMomThreads, smem, stream>>>(q, m); break;
            case 6: k_moments1d<3, true, false><<<sms, kMomThreads, smem, stream>>>(q, m); break;
            default: k_moments1d<3, true, true><<<sms, kMomThreads, smem, stream>>>(q, m); break;
        }
        APIC_CUDA(cudaGetLastError());
        double* bin_blk = bin < sa.P ? sa.phase + bin * sa_block() : nullptr;
        const unsigned fold_blocks = (unsigned)std::min<size_t>((sa_block() + 255) / 256, 1024);
        k_sa_fold1d<<<fold_blocks, 256, 0, stream>>>(q, sa.scratch, sa.tot, bin_blk);
        APIC_CUDA(cudaGetLastError());
        if (bin_blk) ++sa.psamples[bin];
        ++sa.samples;
    }

    // graphs of two steady steps (collision part pending), one per buffer parity
    cudaGraphExec_t pair_exec[2] = {nullptr, nullptr};
    int blocks_cache = 0;

    void drop_graphs() {
        for (auto& g : pair_exec)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    }

    ~Sim1D() {
        if (stream) cudaStreamSynchronize(stream);
        drop_graphs();
        for (void* a : allocations) cudaFree(a);
        if (stream) cudaStreamDestroy(stream);
    }

    void create(const apic_config1d& c) {
        cfg = c;
        require(c.boundary == APIC_PERIODIC || c.boundary == APIC_DIRICHLET, "unknown boundary");
        require(c.velocity_dimensions == 1 || c.velocity_dimensions == 3,
                "simulation velocity_dimensions must be 1 or 3");
        require(c.nx >= 3, "grid nx must be at least 3");
        require(c.nx <= (size_t)(c.boundary == APIC_DIRICHLET ? kMaxNx1D : kMaxNx1DPeriodic),
                "grid nx above the 1D device limit (4096 Dirichlet, 2048 periodic)", APIC_ERR_UNSUPPORTED);
        require(std::isfinite(c.length) && c.length > 0, "domain length must be positive and finite");
        require(std::isfinite(c.dt) && c.dt > 0, "simulation dt must be positive and finite");
        require(c.nspecies >= 1 && c.nspecies <= kMaxSpecies, "species count out of range");
        require(c.nmodels >= 0 && c.nmodels <= kMaxModels, "model count out of range");
        require(c.precision == APIC_FP64 || c.precision == APIC_FP32 || c.precision == APIC_FP32_STORAGE,
                "unknown precision");
        fp32 = c.precision != APIC_FP64;
        c32 = c.precision == APIC_FP32;
        const double rel = c.relative_permittivity == 0.0 ? 1.0 : c.relative_permittivity;
        require(std::isfinite(rel) && rel > 0, "relative_permittivity must be positive and finite");
        // the collision checks of validate() and the Simulation constructor,
        // src/Simulation.cpp:95-100, :388-392
        require(std::isfinite(c.bgk_frequency) && c.bgk_frequency >= 0.0,
                "collision frequency must be non-negative and finite");
        require(std::isfinite(c.bgk_neutral_velocity) && c.bgk_neutral_velocity >= 0.0,
                "neutral_temperature_velocity must be non-negative and finite");
        require(!c.bgk_enabled || c.nmodels == 0,
                "named collision models cannot be combined with the legacy collision model");
        require(!c.bgk_enabled || !c32, "the FP32 cell form does not take the legacy BGK model", APIC_ERR_UNSUPPORTED);
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
            throw Error(APIC_ERR_NO_DEVICE, "no CUDA device is visible");
        APIC_CUDA(cudaGetDevice(&device));
        APIC_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        int least_priority = 0, greatest_priority = 0;
        APIC_CUDA(cudaDeviceGetStreamPriorityRange(&least_priority, &greatest_priority));
        post_priority = greatest_priority;

        const bool dir = c.boundary == APIC_DIRICHLET;
        p.nspecies = c.nspecies;
        p.f32 = fp32 ? 1 : 0;
        p.c32 = c32 ? 1 : 0;
        p.vdim = c.velocity_dimensions;
        p.dirichlet = dir;
        p.nx = (int)c.nx;
        p.L = c.length;
        p.dx = c.length / (double)(dir ? c.nx - 1 : c.nx);  // Grid::Grid, src/Grid.cpp:19-22
        p.inv_dx = 1.0 / p.dx;
        p.dt = c.dt;
        p.eps = (c.units == APIC_SI ? 8.8541878128e-12 : 1.0) * rel;  // include/pic/Types.hpp:17-27
        p.seed = c.seed;
        p.phi_left = c.phi_left;
        p.phi_right = c.phi_right;
        p.drive_left = c.drive_left;
        p.drive_right = c.drive_right;
        // the legacy BGK branch runs when enabled with a positive frequency,
        // src/Simulation.cpp:772-776 (the probability on the host, as there)
        p.bgk = c.bgk_enabled && c.bgk_frequency > 0.0 ? 1 : 0;
        p.bgk_prob = 1.0 - std::exp(-c.bgk_frequency * c.dt);
        p.bgk_vt = c.bgk_neutral_velocity;

        // fixed-point scale: worst-case |rho| bound below 2^62
        double bound = 0.0;
        for (int s = 0; s < c.nspecies; ++s) {
            const auto& sp = c.species[s];
            require(std::isfinite(sp.mass) && sp.mass > 0, "species mass must be positive and finite");
            require(std::isfinite(sp.charge) && std::isfinite(sp.weight), "species charge/weight must be finite");
            require(sp.capacity > 0 && sp.capacity < (1ull << 31), "species capacity out of range");
            bound += (double)sp.capacity * std::fabs(sp.charge * sp.weight) / (dir ? 0.5 * p.dx : p.dx);
        }
        int bits = bound > 0 ? (int)std::floor(61.0 - std::log2(bound)) : 0;
        if (c32) {
            // the FP32 cell form converts one particle's share of a node to a
            // 32-bit integer: a whole particle's charge on an end node (twice
            // q w / dx) stays below 2^30
            double per = 0.0;
            for (int s = 0; s < c.nspecies; ++s)
                per = std::max(per, 2.0 * std::fabs(c.species[s].charge * c.species[s].weight) / p.dx);
            if (per > 0) bits = std::min(bits, (int)std::floor(30.0 - std::log2(per)));
        }
        p.rho_scale = std::ldexp(1.0, bits);
        p.inv_rho_scale = std::ldexp(1.0, -bits);

        st = dalloc<DevState>(1);
        p.st = st;
        for (int s = 0; s < c.nspecies; ++s) {
            const auto& sp = c.species[s];
            SpeciesDev& S = p.sp[s];
            S.qm = sp.charge / sp.mass;
            S.hqm = 0.5 * S.qm;
            S.qw = sp.charge * sp.weight;
            S.qwdx = sp.charge * sp.weight / p.dx;
            S.qmdt32 = (float)(S.qm * c.dt);
            S.hqmdt32 = (float)(S.hqm * c.dt);
            S.dtdx32 = (float)(c.dt / p.dx);
            S.dep32 = (float)(S.qwdx * p.rho_scale);
            S.mass = sp.mass;
            S.weight = sp.weight;
            S.model = -1;
            // the FP32 cell form's buffers also hold the holes left between compactions
            const size_t cap = c32 ? sp.capacity + sp.capacity / 16 + 4096 : sp.capacity;
            require(cap < (1ull << 31), "species capacity out of range");
            S.capacity = (unsigned)cap;
            S.live_cap = (unsigned)sp.capacity;
            // range tables of the pass chunks (FP32 cell form: chunk counts of the compaction)
            const size_t chunk = c32 ? (size_t)kChunk32 : (size_t)kTile;
            const size_t maxr = (cap + chunk - 1) / chunk + 3;
            S.nscratch = (unsigned)maxr;
            for (int b = 0; b < 2; ++b) {
                S.rstart[b] = dalloc<unsigned>(maxr);
                S.rcount[b] = dalloc<unsigned>(maxr);
                S.rlstart[b] = dalloc<unsigned>(maxr);
            }
            S.chunk_surv = dalloc<unsigned>(maxr);
            const bool v3 = c.velocity_dimensions == 3;
            for (int b = 0; b < 2; ++b) {
                if (c32) {
                    S.cell[b] = dalloc<int>(cap);
                    S.off[b] = dalloc<float>(cap);
                } else {
                    S.x[b] = dalloc<double>(cap);
                }
                if (fp32) {
                    S.vh32[b] = dalloc<float>(cap);
                    S.vy32[b] = v3 ? dalloc<float>(cap) : nullptr;
                    S.vz32[b] = v3 ? dalloc<float>(cap) : nullptr;
                } else {
                    S.vh[b] = dalloc<double>(cap);
                    S.vy[b] = v3 ? dalloc<double>(cap) : nullptr;
                    S.vz[b] = v3 ? dalloc<double>(cap) : nullptr;
                }
            }
            S.v = dalloc<double>(cap);
            if (fp32) S.stage = dalloc<double>(cap);
        }
        for (int mi = 0; mi < c.nmodels; ++mi) {
            const apic_mcc_model& m = c.models[mi];
            require(m.species >= 0 && m.species < c.nspecies, "MCC species does not exist");
            require(p.sp[m.species].model < 0, "one MCC model per species is supported", APIC_ERR_UNSUPPORTED);
            require(c.velocity_dimensions == 3 || !c32,
                    "the FP32 cell form's collisions need velocity_dimensions = 3", APIC_ERR_UNSUPPORTED);
            if (c.velocity_dimensions == 1) {
                // NullCollisionModel::collide(double&), src/Collision.cpp:835-846
                for (int ci = 0; ci < m.nch && ci < kMaxChannels; ++ci)
                    require(m.ch[ci].process != APIC_IONIZATION && m.ch[ci].angular == APIC_ISOTROPIC,
                            "ionization and anisotropic MCC require the 3V collision interface");
            }
            for (int ci = 0; ci < m.nch && ci < kMaxChannels; ++ci) {
                const apic_mcc_channel& ch = m.ch[ci];
                require(ch.process != APIC_ATTACHMENT, "1D MCC does not support attachment");
                if (ch.process == APIC_IONIZATION) {
                    require(ch.secondary_species >= 0 && ch.secondary_species < c.nspecies &&
                                ch.ion_species >= 0 && ch.ion_species < c.nspecies,
                            "ionization MCC channel requires secondary and ion species");
                    const auto& tgt = c.species[m.species];
                    const auto& sec = c.species[ch.secondary_species];
                    const auto& ion = c.species[ch.ion_species];
                    require(tgt.charge != 0.0 && tgt.weight == sec.weight && tgt.weight == ion.weight &&
                                tgt.mass == sec.mass && tgt.charge == sec.charge && ion.charge == -tgt.charge,
                            "1D ionization products violate the equal-weight charge-conservation contract");
                }
            }
            DeviceArena arena{allocations, stream};
            build_model(m, c.species[m.species].mass, arena, p.model[mi]);
            neutral_stddev[mi] = p.model[mi].neutral_stddev;
            p.sp[m.species].model = mi;
            draw_threshold(m.max_frequency, c.dt, p.sp[m.species].cand_draw_min, p.sp[m.species].no_candidates);
            if (c32) {
                build_model32(m, arena, p.model[mi], p.model32[mi]);
                const double nudt = m.max_frequency * c.dt;
                p.sp[m.species].cand_p32 = (float)(-std::expm1(-nudt));
                p.sp[m.species].inv_nudt32 = (float)(1.0 / nudt);
            }
            APIC_CUDA(cudaStreamSynchronize(stream));  // host tables may be freed after create
        }
        if (c32 && c.nmodels > 0) {
            // candidate buffer: twice the expected candidates of a step plus
            // room for fluctuations (overflow sets an error, never a fault)
            size_t phys = 0;
            double pmax = 0.0;
            for (int s = 0; s < c.nspecies; ++s) {
                phys += p.sp[s].capacity;
                if (p.sp[s].model >= 0) pmax = std::max(pmax, (double)p.sp[s].cand_p32);
            }
            // one region per CTA of the pass: twice its expected candidates plus slack
            const int regions = grid_blocks();
            require(regions <= kMaxRegions, "pass grid above the collision kernel's region limit", APIC_ERR_UNSUPPORTED);
            const double per_cta = (double)phys / regions;
            const size_t per = (size_t)std::min(std::ceil(per_cta) + 32.0, std::ceil(2.0 * pmax * per_cta) + 256.0);
            p.cands = dalloc<CandRec32>(per * regions);
            p.cand_count = dalloc<unsigned>(regions);
            p.cand_regions = (unsigned)regions;
            p.cand_per_region = (unsigned)per;
            MccModelDev* g = dalloc<MccModelDev>(c.nmodels);
            APIC_CUDA(cudaMemcpyAsync(g, p.model, c.nmodels * sizeof(MccModelDev), cudaMemcpyHostToDevice, stream));
            APIC_CUDA(cudaStreamSynchronize(stream));
            p.gmodel = g;
        }
        p.E = dalloc<double>(c.nx);
        p.rho = dalloc<double>(c.nx);
        p.phi = dalloc<double>(c.nx);
        p.rho_acc = dalloc<unsigned long long>(c.nx);
        if (!dir) {
            std::vector<double> tw(2 * c.nx);
            const double twopi = 2.0 * 3.141592653589793;
            for (size_t m = 0; m < c.nx; ++m) {
                const double a = twopi * (double)m / (double)c.nx;
                tw[2 * m] = std::cos(a);
                tw[2 * m + 1] = std::sin(a);
            }
            double* d = dalloc<double>(tw.size());
            APIC_CUDA(cudaMemcpyAsync(d, tw.data(), tw.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
            p.tw = d;
            APIC_CUDA(cudaStreamSynchronize(stream));
        } else {
            // Thomas coefficients of the constant [-1 2 -1] matrix, src/FieldSolver.cpp:745-752
            const size_t m = c.nx - 2;
            std::vector<double> cp(m), r(m), a(m);
            cp[0] = -1.0 / 2.0;
            r[0] = 0.5;
            for (size_t i = 1; i < m; ++i) {
                const double den = 2.0 + cp[i - 1];
                cp[i] = (i == m - 1) ? 0.0 : -1.0 / den;
                r[i] = 1.0 / den;
            }
            for (size_t i = 0; i < m; ++i) a[i] = -cp[i];
            double* dr = dalloc<double>(m);
            double* da = dalloc<double>(m);
            APIC_CUDA(cudaMemcpyAsync(dr, r.data(), m * sizeof(double), cudaMemcpyHostToDevice, stream));
            APIC_CUDA(cudaMemcpyAsync(da, a.data(), m * sizeof(double), cudaMemcpyHostToDevice, stream));
            p.thomas_r = dr;
            p.thomas_a = da;
            APIC_CUDA(cudaStreamSynchronize(stream));
        }
        size_t cap_total = 0;
        for (int s = 0; s < c.nspecies; ++s) cap_total += c.species[s].capacity;
        p.births_cap = (unsigned)std::min<size_t>(std::max<size_t>(kMaxBirths, cap_total / 64), kMaxBirths);
        p.births = dalloc<BirthRec>(p.births_cap);
        DevState init{};
        APIC_CUDA(cudaMemcpyAsync(st, &init, sizeof init, cudaMemcpyHostToDevice, stream));
        APIC_CUDA(cudaStreamSynchronize(stream));
        static bool attr_done = false;
        if (!attr_done) {
            set_attributes<1, false, false>(); set_attributes<1, true, false>();
            set_attributes<3, false, false>(); set_attributes<3, true, false>();
            set_attributes<1, false, true>(); set_attributes<1, true, true>();
            set_attributes<3, false, true>(); set_attributes<3, true, true>();
            set_attributes_c32<1, false>(); set_attributes_c32<1, true>();
            set_attributes_c32<3, false>(); set_attributes_c32<3, true>();
            attr_done = true;
        }
    }

    // Buffers as seen by the next pass.
    Params1D pass_params(unsigned mode) {
        Params1D q = p;
        q.mode = mode;
        for (int s = 0; s < cfg.nspecies; ++s) {
            SpeciesDev& S = q.sp[s];
            const SpeciesDev& B = p.sp[s];
            const int in = parity, out = parity ^ 1;
            S.x[0] = B.x[in]; S.x[1] = B.x[out];
            S.cell[0] = B.cell[in]; S.cell[1] = B.cell[out];
            S.off[0] = B.off[in]; S.off[1] = B.off[out];
            S.vh[0] = B.vh[in]; S.vh[1] = B.vh[out];
            S.vy[0] = B.vy[in]; S.vy[1] = B.vy[out];
            S.vz[0] = B.vz[in]; S.vz[1] = B.vz[out];
            S.vh32[0] = B.vh32[in]; S.vh32[1] = B.vh32[out];
            S.vy32[0] = B.vy32[in]; S.vy32[1] = B.vy32[out];
            S.vz32[0] = B.vz32[in]; S.vz32[1] = B.vz32[out];
            S.rstart[0] = B.rstart[in]; S.rstart[1] = B.rstart[out];
            S.rcount[0] = B.rcount[in]; S.rcount[1] = B.rcount[out];
            S.rlstart[0] = B.rlstart[in]; S.rlstart[1] = B.rlstart[out];
            S.vold[0] = B.vold[in]; S.vold[1] = B.vold[out];
        }
        return q;
    }

    int grid_blocks() {
        if (blocks_cache) return blocks_cache;
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        size_t tiles = 0;
        for (int s = 0; s < cfg.nspecies; ++s) tiles += (cfg.species[s].capacity + kTile - 1) / kTile;  // 8 warp chunks of c32 per tile
        // one resident wave of the pass kernel: kMinBlocks (kMinBlocks32) CTAs per SM
        blocks_cache = (int)std::max<size_t>(1, std::min<size_t>(tiles, (size_t)sms * (c32 ? kMinBlocks32 : kMinBlocks)));
#ifdef APIC_C32_GRID_DIV
        if (c32) blocks_cache = std::max(1, blocks_cache / APIC_C32_GRID_DIV);
#endif
        return blocks_cache;
    }

    // Optional per-kernel timing (CUDA events on the handle's stream).
    bool timing = false;
    struct EvPair { cudaEvent_t a, b, c; };
    std::vector<EvPair> events;
    double pass_ms = 0.0, post_ms = 0.0;
    uint64_t timed_passes = 0;

    void collect_timing() {
        for (auto& e : events) {
            float t1 = 0.f, t2 = 0.f;
            APIC_CUDA(cudaEventElapsedTime(&t1, e.a, e.b));
            APIC_CUDA(cudaEventElapsedTime(&t2, e.b, e.c));
            pass_ms += t1;
            post_ms += t2;
            ++timed_passes;
            cudaEventDestroy(e.a); cudaEventDestroy(e.b); cudaEventDestroy(e.c);
        }
        events.clear();
    }

    template <int VDIM, bool DIR, bool F32>
    static void set_attributes() {
        const int smem = kMaxNx1D * 16;
        APIC_CUDA(cudaFuncSetAttribute(k_pass1d<VDIM, DIR, F32, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       smem));
        APIC_CUDA(cudaFuncSetAttribute(k_pass1d<VDIM, DIR, F32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       smem));
        const int psm = (int)post_smem_bytes(DIR ? kMaxNx1D : kMaxNx1DPeriodic, DIR);
        APIC_CUDA(cudaFuncSetAttribute(k_post1d<VDIM, DIR, F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, psm));
        APIC_CUDA(cudaFuncSetAttribute(k_moments1d<VDIM, DIR, F32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kMomentSmemMax));
    }

    template <int VDIM, bool DIR>
    static void set_attributes_c32() {
        APIC_CUDA(cudaFuncSetAttribute(k_pass1d_c32<VDIM, DIR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kMaxNx1D * 12));
        const int psm = (int)post_smem_bytes(DIR ? kMaxNx1D : kMaxNx1DPeriodic, DIR);
        APIC_CUDA(cudaFuncSetAttribute(k_post1d<VDIM, DIR, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       psm));
    }

    template <int VDIM, bool DIR>
    void launch_kernels_c32(const Params1D& q, int blocks, size_t post_smem, unsigned post, EvPair& ev) {
        k_pass1d_c32<VDIM, DIR><<<blocks, kThreads, (size_t)cfg.nx * 12, stream>>>(q);
        if (VDIM == 3 && cfg.nmodels > 0 && (q.mode & kModeSyncMcc))
            k_collide1d_c32<VDIM, DIR><<<148 * 4, kCollideThreads, 0, stream>>>(q);
        if (timing) cudaEventRecord(ev.b, stream);
        cudaLaunchConfig_t lc = {};
        lc.gridDim = dim3(1);
        lc.blockDim = dim3(kPostThreads);
        lc.dynamicSmemBytes = post_smem;
        lc.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributePriority;
        attr[0].val.priority = post_priority;
        lc.attrs = attr;
        lc.numAttrs = 1;
        APIC_CUDA(cudaLaunchKernelEx(&lc, k_post1d<VDIM, DIR, true, true>, q, post));
    }

    // The post kernel takes a whole SM's registers (one 512-thread CTA), so
    // when several runs step together on the GPU it is launched at the
    // highest stream priority: the CTA scheduler then gives it the next free
    // SM instead of another run's pass CTA, and no run waits behind the others.
    int post_priority = 0;

    template <int VDIM, bool DIR, bool F32>
    void launch_kernels(const Params1D& q, int blocks, size_t smem, size_t post_smem, unsigned post, EvPair& ev) {
        if (q.coll_acc || q.ledger || q.bgk)
            k_pass1d<VDIM, DIR, F32, true><<<blocks, kThreads, smem, stream>>>(q);
        else
            k_pass1d<VDIM, DIR, F32, false><<<blocks, kThreads, smem, stream>>>(q);
        if (timing) cudaEventRecord(ev.b, stream);
        cudaLaunchConfig_t lc = {};
        lc.gridDim = dim3(1);
        lc.blockDim = dim3(kPostThreads);
        lc.dynamicSmemBytes = post_smem;
        lc.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributePriority;
        attr[0].val.priority = post_priority;
        lc.attrs = attr;
        lc.numAttrs = 1;
        APIC_CUDA(cudaLaunchKernelEx(&lc, k_post1d<VDIM, DIR, F32>, q, post));
    }

    void launch_pass(unsigned mode, unsigned post) {
        const Params1D q = pass_params(mode);
        const int blocks = grid_blocks();
        const size_t smem = (size_t)cfg.nx * 16;
        const bool dir = cfg.boundary == APIC_DIRICHLET;
        const size_t post_smem = post_smem_bytes((int)cfg.nx, dir);
        EvPair ev{};
        if (timing) {
            APIC_CUDA(cudaEventCreate(&ev.a));
            APIC_CUDA(cudaEventCreate(&ev.b));
            APIC_CUDA(cudaEventCreate(&ev.c));
            APIC_CUDA(cudaEventRecord(ev.a, stream));
        }
        const int form = (cfg.velocity_dimensions == 3 ? 4 : 0) | (dir ? 2 : 0) | (fp32 ? 1 : 0);
        if (c32) {
            switch (form & 6) {
                case 0: launch_kernels_c32<1, false>(q, blocks, post_smem, post, ev); break;
                case 2: launch_kernels_c32<1, true>(q, blocks, post_smem, post, ev); break;
                case 4: launch_kernels_c32<3, false>(q, blocks, post_smem, post, ev); break;
                default: launch_kernels_c32<3, true>(q, blocks, post_smem, post, ev); break;
            }
        } else switch (form) {
            case 0: launch_kernels<1, false, false>(q, blocks, smem, post_smem, post, ev); break;
            case 1: launch_kernels<1, false, true>(q, blocks, smem, post_smem, post, ev); break;
            case 2: launch_kernels<1, true, false>(q, blocks, smem, post_smem, post, ev); break;
            case 3: launch_kernels<1, true, true>(q, blocks, smem, post_smem, post, ev); break;
            case 4: launch_kernels<3, false, false>(q, blocks, smem, post_smem, post, ev); break;
            case 5: launch_kernels<3, false, true>(q, blocks, smem, post_smem, post, ev); break;
            case 6: launch_kernels<3, true, false>(q, blocks, smem, post_smem, post, ev); break;
            default: launch_kernels<3, true, true>(q, blocks, smem, post_smem, post, ev); break;
        }
        if (timing) {
            APIC_CUDA(cudaEventRecord(ev.c, stream));
            events.push_back(ev);
        }
        APIC_CUDA(cudaGetLastError());
        if (!c32) parity ^= 1;  // the FP32 cell form updates its buffer in place
    }

    // FP32 cell form: squeezes the holes out of every species' slots, order
    // preserved (into the other buffer, which becomes the current one).
    void compact32() {
        const int sms = 148;
        for (int s = 0; s < cfg.nspecies; ++s) {
            SpeciesDev& B = p.sp[s];
            const int in = parity, out = parity ^ 1;
            unsigned* counts = B.chunk_surv;
            unsigned* n_old = B.chunk_surv + B.nscratch - 1;
            k_c32_count<<<sms * 4, 256, 0, stream>>>(B.cell[in], &st->n[s], counts);
            k_c32_scan<<<1, kScanThreads, 0, stream>>>(counts, &st->n[s], &st->holes[s], n_old);
            C32Arrays a{B.cell[in], B.off[in], B.vh32[in], B.vy32[in], B.vz32[in], B.v};
            // S.v is not carried: it is rewritten by every read-back
            k_c32_scatter<<<sms * 4, 256, 0, stream>>>(a, B.cell[out], B.off[out], B.vh32[out], B.vy32[out],
                                                       B.vz32[out], nullptr, n_old, counts);
        }
        APIC_CUDA(cudaGetLastError());
        parity ^= 1;
    }
    bool compaction_due(uint64_t k) const { return c32 && k % kCompactSteps == 0; }

    // FP32 cell form read-back: one component of the live particles, in slot
    // order, to host doubles (the device layout is left as it is).
    void gather32(int s, int component, double* host, size_t n) {
        SpeciesDev& B = p.sp[s];
        const int in = parity;
        C32Arrays a{B.cell[in], B.off[in], B.vh32[in], B.vy32[in], B.vz32[in], B.v};
        k_c32_gather<<<148 * 4, 256, 0, stream>>>(a, component, p.dx, &st->n[s], B.chunk_surv, B.stage);
        APIC_CUDA(cudaGetLastError());
        APIC_CUDA(cudaMemcpyAsync(host, B.stage, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
    }

    // One velocity component of species s between host doubles and the
    // current device buffer (FP32 form: rounded to nearest on the way in).
    void put_comp(int s, double* d, float* f, const double* host, size_t n) {
        if (n == 0) return;
        if (!fp32) {
            APIC_CUDA(cudaMemcpyAsync(d, host, n * sizeof(double), cudaMemcpyHostToDevice, stream));
            return;
        }
        double* stage = p.sp[s].stage;
        APIC_CUDA(cudaMemcpyAsync(stage, host, n * sizeof(double), cudaMemcpyHostToDevice, stream));
        k_narrow1d<<<(unsigned)std::min<size_t>((n + 255) / 256, 4096), 256, 0, stream>>>(stage, f, (unsigned)n);
        APIC_CUDA(cudaGetLastError());
    }
    void get_comp(int s, const double* d, const float* f, double* host, size_t n) {
        if (n == 0) return;
        if (!fp32) {
            APIC_CUDA(cudaMemcpyAsync(host, d, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
            return;
        }
        double* stage = p.sp[s].stage;
        k_widen1d<<<(unsigned)std::min<size_t>((n + 255) / 256, 4096), 256, 0, stream>>>(f, stage, (unsigned)n);
        APIC_CUDA(cudaGetLastError());
        APIC_CUDA(cudaMemcpyAsync(host, stage, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
    }

    // Positions of species s from host doubles into the current buffer (FP32
    // cell form: through the staging array into cell + offset).
    void put_x(int s, const double* host, size_t n) {
        if (n == 0) return;
        SpeciesDev& B = p.sp[s];
        if (!c32) {
            APIC_CUDA(cudaMemcpyAsync(B.x[parity], host, n * sizeof(double), cudaMemcpyHostToDevice, stream));
            return;
        }
        APIC_CUDA(cudaMemcpyAsync(B.stage, host, n * sizeof(double), cudaMemcpyHostToDevice, stream));
        const unsigned g = (unsigned)std::min<size_t>((n + 255) / 256, 4096);
        if (cfg.boundary == APIC_DIRICHLET)
            k_x_to_cell<true><<<g, 256, 0, stream>>>(B.stage, B.cell[parity], B.off[parity], (unsigned)n, p);
        else
            k_x_to_cell<false><<<g, 256, 0, stream>>>(B.stage, B.cell[parity], B.off[parity], (unsigned)n, p);
        APIC_CUDA(cudaGetLastError());
    }
    void get_x(int s, double* host, size_t n) {
        if (n == 0) return;
        const SpeciesDev& B = p.sp[s];
        if (!c32) {
            APIC_CUDA(cudaMemcpyAsync(host, B.x[parity], n * sizeof(double), cudaMemcpyDeviceToHost, stream));
            return;
        }
        const unsigned g = (unsigned)std::min<size_t>((n + 255) / 256, 4096);
        k_cell_to_x<<<g, 256, 0, stream>>>(B.cell[parity], B.off[parity], B.stage, (unsigned)n, p.dx);
        APIC_CUDA(cudaGetLastError());
        APIC_CUDA(cudaMemcpyAsync(host, B.stage, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
    }

    void load(int s, size_t n, const double* x, const double* v, const double* vh, const double* vy,
              const double* vz, const uint8_t* alive) {
        require(s >= 0 && s < cfg.nspecies, "species index out of range");
        require(x && v, "x and v are required");
        if (!alive && vh && (cfg.velocity_dimensions == 1 || (vy && vz))) {
            // every particle alive: copy straight from the caller's buffers
            require(n <= cfg.species[s].capacity, "initial particle count exceeds max_particles_per_species",
                    APIC_ERR_CAPACITY);
            SpeciesDev& B = p.sp[s];
            const size_t bytes = n * sizeof(double);
            put_x(s, x, n);
            put_comp(s, B.vh[parity], B.vh32[parity], vh, n);
            APIC_CUDA(cudaMemcpyAsync(B.v, v, bytes, cudaMemcpyHostToDevice, stream));
            if (cfg.velocity_dimensions == 3) {
                put_comp(s, B.vy[parity], B.vy32[parity], vy, n);
                put_comp(s, B.vz[parity], B.vz32[parity], vz, n);
            }
            set_single_range(s, (unsigned)n);
            APIC_CUDA(cudaStreamSynchronize(stream));
            initialized = false;
            pending = false;
            return;
        }
        std::vector<double> hx, hv, hvh, hvy, hvz;
        for (size_t i = 0; i < n; ++i) {
            if (alive && !alive[i]) continue;
            hx.push_back(x[i]);
            hv.push_back(v[i]);
            hvh.push_back(vh ? vh[i] : v[i]);
            hvy.push_back(vy ? vy[i] : 0.0);
            hvz.push_back(vz ? vz[i] : 0.0);
        }
        const size_t m = hx.size();
        require(m <= cfg.species[s].capacity, "initial particle count exceeds max_particles_per_species",
                APIC_ERR_CAPACITY);
        APIC_CUDA(cudaStreamSynchronize(stream));
        SpeciesDev& B = p.sp[s];
        const size_t bytes = m * sizeof(double);
        put_x(s, hx.data(), m);
        put_comp(s, B.vh[parity], B.vh32[parity], hvh.data(), m);
        APIC_CUDA(cudaMemcpyAsync(B.v, hv.data(), bytes, cudaMemcpyHostToDevice, stream));
        if (cfg.velocity_dimensions == 3) {
            put_comp(s, B.vy[parity], B.vy32[parity], hvy.data(), m);
            put_comp(s, B.vz[parity], B.vz32[parity], hvz.data(), m);
        }
        set_single_range(s, (unsigned)m);
        APIC_CUDA(cudaStreamSynchronize(stream));
        initialized = false;
        pending = false;
    }

    // The loaded particles are one contiguous range at slot 0.
    unsigned range_host[kMaxSpecies][4];
    void set_single_range(int s, unsigned n) {
        SpeciesDev& B = p.sp[s];
        unsigned* h = range_host[s];
        h[0] = 0; h[1] = n; h[2] = 0; h[3] = n ? 1u : 0u;
        APIC_CUDA(cudaMemcpyAsync(B.rstart[parity], &h[0], sizeof(unsigned), cudaMemcpyHostToDevice, stream));
        APIC_CUDA(cudaMemcpyAsync(B.rcount[parity], &h[1], sizeof(unsigned), cudaMemcpyHostToDevice, stream));
        APIC_CUDA(cudaMemcpyAsync(B.rlstart[parity], &h[2], sizeof(unsigned), cudaMemcpyHostToDevice, stream));
        APIC_CUDA(cudaMemcpyAsync(&st->n[s], &h[1], sizeof(unsigned), cudaMemcpyHostToDevice, stream));
        APIC_CUDA(cudaMemcpyAsync(&st->nranges[s], &h[3], sizeof(unsigned), cudaMemcpyHostToDevice, stream));
        APIC_CUDA(cudaMemsetAsync(&st->holes[s], 0, sizeof(unsigned), stream));
    }

    void set_time(double t, uint64_t k) {
        time = t;
        step = k;
        APIC_CUDA(cudaMemcpyAsync(&st->time, &time, sizeof time, cudaMemcpyHostToDevice, stream));
        APIC_CUDA(cudaMemcpyAsync(&st->step, &step, sizeof step, cudaMemcpyHostToDevice, stream));
    }

    // Simulation::initialize, src/Simulation.cpp:698-769
    void initialize() {
        set_time(0.0, 0);
        APIC_CUDA(cudaMemsetAsync(&st->work[0], 0, sizeof(double) * kMaxSpecies, stream));  // src/Simulation.cpp:706-710
        launch_pass(kModeDeposit, kPostSolve);
        launch_pass(kModeInitHalf, 0);
        pending = false;
        initialized = true;
    }

    void resume(double t, uint64_t k) {
        set_time(t, k);
        launch_pass(kModeDeposit, kPostSolve);
        pending = false;
        initialized = true;
    }

    // Two steps with the collision part of the previous step pending, as one
    // CUDA graph launch (kernel parameters depend only on the buffer parity).
    void steady_pair() {
        if (compaction_due(step + 1) || compaction_due(step + 2)) {
            do_steps(2);
            return;
        }
        const int par = parity;
        if (!pair_exec[par]) {
            const bool t = timing;
            timing = false;
            cudaGraph_t g = nullptr;
            APIC_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            const unsigned mode = kModeSyncMcc | kModeKickDrift | kModeDeposit;
            launch_pass(mode, kPostSolve | kPostAdvance | kPostPushBirths);
            launch_pass(mode, kPostSolve | kPostAdvance | kPostPushBirths);
            timing = t;
            APIC_CUDA(cudaStreamEndCapture(stream, &g));
            const cudaError_t e = cudaGraphInstantiate(&pair_exec[par], g, 0);
            cudaGraphDestroy(g);
            APIC_CUDA(e);
        }
        APIC_CUDA(cudaGraphLaunch(pair_exec[par], stream));
        time += 2.0 * cfg.dt;
        step += 2;
    }

    void do_steps(size_t nsteps) {
        require(initialized, "initialize() or resume() must precede step()", APIC_ERR_STATE);
        for (size_t i = 0; i < nsteps; ++i) {
            const unsigned mode = (pending ? kModeSyncMcc : 0u) | kModeKickDrift | kModeDeposit;
            if (pending) arm_collision_step(step);
            launch_pass(mode, kPostSolve | kPostAdvance | kPostPushBirths);
            disarm();
            pending = true;
            time += cfg.dt;
            ++step;
            if (sample_step(step)) take_sample(step);
            if (compaction_due(step)) compact32();
        }
    }

    // Applies the pending collision part of the last step so the state equals
    // the reference's state after step() returned.
    void finish() {
        if (!initialized) return;
        if (pending) {
            arm_collision_step(step);
            launch_pass(kModeSyncMcc | kModeWriteV, 0);
            disarm();
            pending = false;
        }
    }

    int sync_status() {
        const cudaError_t e = bounded_wait(stream, wait_limit_s);
        if (e == cudaErrorNotReady) throw Error(APIC_ERR_TIMEOUT, "device work did not complete in time");
        APIC_CUDA(e);
        unsigned word = 0;
        APIC_CUDA(cudaMemcpyAsync(&word, &st->error, sizeof word, cudaMemcpyDeviceToHost, stream));
        APIC_CUDA(cudaStreamSynchronize(stream));
        if (word) {
            const int s = status_from_device(word);
            APIC_CUDA(cudaMemsetAsync(&st->error, 0, sizeof(unsigned), stream));
            APIC_CUDA(cudaStreamSynchronize(stream));
            throw Error(s, describe_device_error(word));
        }
        return APIC_OK;
    }

    DevState read_state() {
        sync_status();
        DevState h;
        APIC_CUDA(cudaMemcpyAsync(&h, st, sizeof h, cudaMemcpyDeviceToHost, stream));
        APIC_CUDA(cudaStreamSynchronize(stream));
        return h;
    }

    size_t count(int s) {
        require(s >= 0 && s < cfg.nspecies, "species index out of range");
        finish();
        const DevState h = read_state();
        return h.n[s] - h.holes[s];
    }

    size_t read_particles(int s, size_t cap, double* x, double* v, double* vh, double* vy, double* vz) {
        require(s >= 0 && s < cfg.nspecies, "species index out of range");
        finish();
        const DevState h = read_state();
        const size_t n = h.n[s] - h.holes[s];
        require(cap >= n, "output capacity below the particle count", APIC_ERR_CAPACITY);
        const SpeciesDev& B = p.sp[s];
        const size_t bytes = n * sizeof(double);
        if (c32) {
            // the live particles in slot order, through the staging array
            unsigned* counts = B.chunk_surv;
            k_c32_count<<<148 * 4, 256, 0, stream>>>(B.cell[parity], &st->n[s], counts);
            k_c32_scan<<<1, kScanThreads, 0, stream>>>(counts, &st->n[s], nullptr, counts + B.nscratch - 1);
            APIC_CUDA(cudaGetLastError());
            if (x) gather32(s, 0, x, n);
            if (v) gather32(s, 1, v, n);
            if (vh) gather32(s, 2, vh, n);
            if (cfg.velocity_dimensions == 3) {
                if (vy) gather32(s, 3, vy, n);
                if (vz) gather32(s, 4, vz, n);
            } else {
                if (vy) std::memset(vy, 0, bytes);
                if (vz) std::memset(vz, 0, bytes);
            }
            APIC_CUDA(cudaStreamSynchronize(stream));
            return n;
        }
        if (x) get_x(s, x, n);
        if (v) APIC_CUDA(cudaMemcpyAsync(v, B.v, bytes, cudaMemcpyDeviceToHost, stream));
        if (vh) get_comp(s, B.vh[parity], B.vh32[parity], vh, n);
        if (cfg.velocity_dimensions == 3) {
            if (vy) get_comp(s, B.vy[parity], B.vy32[parity], vy, n);
            if (vz) get_comp(s, B.vz[parity], B.vz32[parity], vz, n);
        } else {
            if (vy) std::memset(vy, 0, bytes);
            if (vz) std::memset(vz, 0, bytes);
        }
        APIC_CUDA(cudaStreamSynchronize(stream));
        return n;
    }

    double* sample_partial = nullptr;
    unsigned* sample_done = nullptr;
    double* sample_out = nullptr;

    DevState sample_device(apic_sample1d* out) {
        if (!sample_partial) {
            sample_partial = dalloc<double>(kSampleBlocks * kMaxSpecies);
            sample_done = dalloc<unsigned>(1);
            sample_out = dalloc<double>(kMaxSpecies + 2);
        }
        Params1D q = pass_params(0);
        k_sample1d<<<kSampleBlocks, 256, 0, stream>>>(q, sample_partial, sample_done, sample_out);
        APIC_CUDA(cudaGetLastError());
        double h[kMaxSpecies + 2];
        APIC_CUDA(cudaMemcpyAsync(h, sample_out, sizeof h, cudaMemcpyDeviceToHost, stream));
        const DevState st_h = read_state();
        for (int s = 0; s < cfg.nspecies; ++s) out->kinetic_by_species[s] = h[s];
        out->field_energy = h[kMaxSpecies];
        out->charge_l1 = h[kMaxSpecies + 1];
        if (cfg.boundary == APIC_DIRICHLET) {
            APIC_CUDA(cudaMemcpyAsync(&out->phi_left, p.phi, sizeof(double), cudaMemcpyDeviceToHost, stream));
            APIC_CUDA(cudaMemcpyAsync(&out->phi_right, p.phi + cfg.nx - 1, sizeof(double), cudaMemcpyDeviceToHost, stream));
            APIC_CUDA(cudaStreamSynchronize(stream));
        }
        return st_h;
    }

    // the diagnostics channels in the reference's numbering, as (model,
    // channel) slots of the device totals: every model's channels in model
    // order, or the legacy BGK model's one "bgk" channel
    std::vector<std::pair<int, int>> channel_slots() const {
        std::vector<std::pair<int, int>> out;
        if (cfg.bgk_enabled) out.emplace_back(0, 0);
        for (int m = 0; m < cfg.nmodels; ++m)
            for (int ch = 0; ch < cfg.models[m].nch; ++ch) out.emplace_back(m, ch);
        return out;
    }

    // Simulation::load_checkpoint, src/Simulation.cpp:2018-2899, for the parts
    // the device holds (see apic_sim1d_load_checkpoint).
    void load_checkpoint(const Apc& c) {
        const double rel = cfg.relative_permittivity == 0.0 ? 1.0 : cfg.relative_permittivity;
        require(c.units == cfg.units && c.relative_permittivity == rel && c.permittivity == p.eps,
                "checkpoint unit system does not match 1D config");
        require(c.velocity_dimensions == cfg.velocity_dimensions,
                "checkpoint velocity dimensions do not match 1D config");
        const auto slots = channel_slots();
        require(c.channel_counts.size() == slots.size(), "checkpoint collision diagnostics do not match 1D config");
        require(c.losses.size() == (size_t)cfg.nspecies,
                "checkpoint boundary-loss species count does not match 1D config");
        require(c.electric_work.size() == (size_t)cfg.nspecies,
                "checkpoint power-transfer species count does not match 1D config");
        require(!c.spatial_average_enabled && !sa.on, "checkpoint spatial-average contract does not match 1D config");
        require(c.species.size() == (size_t)cfg.nspecies, "checkpoint species count does not match config");
        for (int s = 0; s < cfg.nspecies; ++s)
            require(c.species[s].x.size() <= cfg.species[s].capacity,
                    "checkpoint particle count exceeds max_particles_per_species", APIC_ERR_CAPACITY);
        for (int s = 0; s < cfg.nspecies; ++s) {
            const Apc::Species& sp = c.species[s];
            load(s, sp.x.size(), sp.x.data(), sp.v.data(), sp.vh.data(), sp.vy.data(), sp.vz.data(), sp.alive.data());
        }
        // the ledgers continue from the file's totals
        DevState h = read_state();
        h.candidates = c.candidates;
        h.nulls = c.null_collisions;
        for (size_t k = 0; k < slots.size(); ++k) {
            h.chan[slots[k].first][slots[k].second] = c.channel_counts[k];
            h.chan_energy[slots[k].first][slots[k].second] = c.channel_energy[k];
        }
        for (int s = 0; s < cfg.nspecies; ++s) {
            h.lost[s][0] = c.losses[s].left;
            h.lost[s][1] = c.losses[s].right;
            h.lost_energy[s][0] = c.losses[s].energy_left;
            h.lost_energy[s][1] = c.losses[s].energy_right;
        }
        APIC_CUDA(cudaMemcpyAsync(st, &h, sizeof h, cudaMemcpyHostToDevice, stream));
        resume(c.time, c.step);
        if (p.ledger) {  // resume() keeps the ledger; the file's work replaces it
            double w[kMaxSpecies] = {0, 0, 0, 0};
            for (int s = 0; s < cfg.nspecies; ++s) w[s] = c.electric_work[s].second;
            APIC_CUDA(cudaMemcpyAsync(&st->work[0], w, sizeof w, cudaMemcpyHostToDevice, stream));
        }
        APIC_CUDA(cudaStreamSynchronize(stream));
    }

    // Simulation::save_checkpoint, src/Simulation.cpp:1812-2015, of the device
    // run with meta's identity lines (see apic_sim1d_save_checkpoint).
    void save_checkpoint(const Apc& meta, const std::string& path) {
        require(!sa.on, "checkpoints of runs with spatial averaging are written by the FP64 host path only",
                APIC_ERR_UNSUPPORTED);
        require(!meta.spatial_average_enabled && meta.spatial_average_nx == cfg.nx &&
                    meta.species.size() == (size_t)cfg.nspecies,
                "checkpoint metadata does not match 1D config");
        const auto slots = channel_slots();
        require(meta.channel_counts.size() == slots.size(), "checkpoint collision diagnostics do not match 1D config");
        Apc c = meta;
        const double rel = cfg.relative_permittivity == 0.0 ? 1.0 : cfg.relative_permittivity;
        c.units = cfg.units;
        c.relative_permittivity = rel;
        c.permittivity = p.eps;
        c.velocity_dimensions = cfg.velocity_dimensions;
        finish();
        const DevState h = read_state();
        c.candidates = h.candidates;
        c.null_collisions = h.nulls;
        for (size_t k = 0; k < slots.size(); ++k) {
            c.channel_counts[k] = h.chan[slots[k].first][slots[k].second];
            c.channel_energy[k] = h.chan_energy[slots[k].first][slots[k].second];
        }
        c.losses.resize(cfg.nspecies);
        c.electric_work.resize(cfg.nspecies);
        for (int s = 0; s < cfg.nspecies; ++s) {
            c.losses[s].name = meta.species[s].name;
            c.losses[s].left = h.lost[s][0];
            c.losses[s].right = h.lost[s][1];
            c.losses[s].energy_left = h.lost_energy[s][0];
            c.losses[s].energy_right = h.lost_energy[s][1];
            c.electric_work[s] = {meta.species[s].name, p.ledger ? h.work[s] : 0.0};
        }
        if (!p.ledger) c.power_transfer_origin = step;  // counted from here
        c.step = step;
        c.time = time;
        for (int s = 0; s < cfg.nspecies; ++s) {
            Apc::Species& sp = c.species[s];
            sp.name = meta.species[s].name;
            const size_t n = h.n[s] - h.holes[s];
            sp.x.resize(n); sp.v.resize(n); sp.vy.resize(n); sp.vz.resize(n); sp.vh.resize(n);
            sp.alive.assign(n, 1);
            read_particles(s, n, sp.x.data(), sp.v.data(), sp.vh.data(), sp.vy.data(), sp.vz.data());
        }
        apc_write(path, c);
    }

    void read_fields(double* rho, double* phi, double* E) {
        sync_status();
        const size_t bytes = cfg.nx * sizeof(double);
        if (rho) APIC_CUDA(cudaMemcpyAsync(rho, p.rho, bytes, cudaMemcpyDeviceToHost, stream));
        if (phi) APIC_CUDA(cudaMemcpyAsync(phi, p.phi, bytes, cudaMemcpyDeviceToHost, stream));
        if (E) APIC_CUDA(cudaMemcpyAsync(E, p.E, bytes, cudaMemcpyDeviceToHost, stream));
        APIC_CUDA(cudaStreamSynchronize(stream));
    }
};

}  // namespace apic

// ---- C ABI ----------------------------------------------------------------------

using apic::Error;

struct apic_sim1d {
    apic::Sim1D impl;
};

namespace {
thread_local std::string g_error;

template <class F>
int guarded(apic_sim1d* h, F&& f) {
    try {
        f();
        return APIC_OK;
    } catch (const Error& e) {
        if (h) h->impl.last_error = e.what();
        g_error = e.what();
        return e.status;
    } catch (const std::exception& e) {
        if (h) h->impl.last_error = e.what();
        g_error = e.what();
        return APIC_ERR_INVALID;
    }
}
}  // namespace

extern "C" {

const char* apic_version(void) { return "aurora-pic-b200 0.1 (sm_100a)"; }

const char* apic_status_string(int s) {
    switch (s) {
        case APIC_OK: return "ok";
        case APIC_ERR_INVALID: return "invalid argument";
        case APIC_ERR_CUDA: return "CUDA error";
        case APIC_ERR_CAPACITY: return "particle capacity exceeded";
        case APIC_ERR_MAJORANT: return "collision frequency above max_frequency";
        case APIC_ERR_CANDIDATES: return "MCC candidate limit exceeded";
        case APIC_ERR_NONFINITE: return "non-finite particle state";
        case APIC_ERR_TIMEOUT: return "device wait timed out";
        case APIC_ERR_UNSUPPORTED: return "unsupported configuration";
        case APIC_ERR_STATE: return "call out of order";
        case APIC_ERR_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

int apic_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

int apic_sim1d_create(const apic_config1d* cfg, apic_sim1d** out) {
    if (!cfg || !out) return APIC_ERR_INVALID;
    *out = nullptr;
    auto h = std::make_unique<apic_sim1d>();
    const int rc = guarded(h.get(), [&] { h->impl.create(*cfg); });
    if (rc == APIC_OK) *out = h.release();
    return rc;
}

void apic_sim1d_destroy(apic_sim1d* sim) { delete sim; }

const char* apic_sim1d_last_error(const apic_sim1d* sim) {
    return sim ? sim->impl.last_error.c_str() : g_error.c_str();
}

int apic_sim1d_load_particles(apic_sim1d* sim, int species, size_t n, const double* x, const double* v,
                              const double* v_half, const double* vy, const double* vz, const uint8_t* alive) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded(sim, [&] { sim->impl.load(species, n, x, v, v_half, vy, vz, alive); });
}

int apic_sim1d_initialize(apic_sim1d* sim) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded(sim, [&] { sim->impl.initialize(); });
}

int apic_sim1d_resume(apic_sim1d* sim, double time, uint64_t step) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded(sim, [&] { sim->impl.resume(time, step); });
}

int apic_sim1d_step(apic_sim1d* sim, size_t nsteps) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded(sim, [&] { sim->impl.do_steps(nsteps); });
}

int apic_sim1d_step_group(apic_sim1d* const* sims, size_t n, size_t nsteps) {
    if (!sims) return APIC_ERR_INVALID;
    for (size_t i = 0; i < n; ++i)
        if (!sims[i]) return APIC_ERR_INVALID;
    std::vector<size_t> left(n, nsteps);
    // bring every run to the steady state (collision part pending) one step at a time
    for (size_t i = 0; i < n; ++i) {
        if (!left[i] || sims[i]->impl.pending) continue;
        const int rc = guarded(sims[i], [&] { sims[i]->impl.do_steps(1); });
        if (rc != APIC_OK) return rc;
        --left[i];
    }
    // then two steps per graph launch, round robin over the runs' streams
    for (bool more = true; more;) {
        more = false;
        for (size_t i = 0; i < n; ++i) {
            if (left[i] < 2) continue;
            const int rc = guarded(sims[i], [&] {
                apic::Sim1D& S = sims[i]->impl;
                apic::require(S.initialized, "initialize() or resume() must precede step()", APIC_ERR_STATE);
                if (S.timing || S.sa.on) S.do_steps(2); else S.steady_pair();
            });
            if (rc != APIC_OK) return rc;
            left[i] -= 2;
            more = more || left[i] >= 2;
        }
    }
    for (size_t i = 0; i < n; ++i) {
        if (!left[i]) continue;
        const int rc = guarded(sims[i], [&] { sims[i]->impl.do_steps(left[i]); });
        if (rc != APIC_OK) return rc;
    }
    return APIC_OK;
}

int apic_sim1d_synchronize(apic_sim1d* sim) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded(sim, [&] { sim->impl.sync_status(); });
}

int apic_sim1d_set_wait_limit(apic_sim1d* sim, double seconds) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded(sim, [&] {
        apic::require(std::isfinite(seconds) && seconds > 0.0, "wait limit must be positive and finite");
        sim->impl.wait_limit_s = seconds;
    });
}

int apic_sim1d_load_checkpoint(apic_sim1d* sim, const apic_apc* checkpoint) {
    if (!sim || !checkpoint) return APIC_ERR_INVALID;
    return guarded(sim, [&] { sim->impl.load_checkpoint(checkpoint->c); });
}

int apic_sim1d_save_checkpoint(apic_sim1d* sim, const apic_apc* meta, const char* path) {
    if (!sim || !meta || !path) return APIC_ERR_INVALID;
    return guarded(sim, [&] { sim->impl.save_checkpoint(meta->c, path); });
}

int apic_sim1d_count(apic_sim1d* sim, int species, size_t* n) {
    if (!sim || !n) return APIC_ERR_INVALID;
    return guarded(sim, [&] { *n = sim->impl.count(species); });
}

int apic_sim1d_read_particles(apic_sim1d* sim, int species, size_t capacity, double* x, double* v,
                              double* v_half, double* vy, double* vz, size_t* n) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded(sim, [&] {
        const size_t got = sim->impl.read_particles(species, capacity, x, v, v_half, vy, vz);
        if (n) *n = got;
    });
}

int apic_sim1d_read_fields(apic_sim1d* sim, double* rho, double* phi, double* electric) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded(sim, [&] { sim->impl.read_fields(rho, phi, electric); });
}

int apic_sim1d_collision_totals(apic_sim1d* sim, apic_collision_totals* out) {
    if (!sim || !out) return APIC_ERR_INVALID;
    return guarded(sim, [&] {
        sim->impl.finish();
        const apic::DevState h = sim->impl.read_state();
        std::memset(out, 0, sizeof *out);
        out->candidates = h.candidates;
        out->null_collisions = h.nulls;
        for (int m = 0; m < APIC_MAX_MODELS; ++m)
            for (int c = 0; c < APIC_MAX_CHANNELS; ++c) {
                out->channel_collisions[m][c] = h.chan[m][c];
                out->channel_energy_change[m][c] = h.chan_energy[m][c];
            }
    });
}

int apic_sim1d_boundary_losses(apic_sim1d* sim, int species, apic_boundary_loss* out) {
    if (!sim || !out) return APIC_ERR_INVALID;
    return guarded(sim, [&] {
        apic::require(species >= 0 && species < sim->impl.cfg.nspecies, "species index out of range");
        const apic::DevState h = sim->impl.read_state();
        out->absorbed_left = h.lost[species][0];
        out->absorbed_right = h.lost[species][1];
        out->kinetic_energy_left = h.lost_energy[species][0];
        out->kinetic_energy_right = h.lost_energy[species][1];
    });
}

int apic_sim1d_sample(apic_sim1d* sim, apic_sample1d* out) {
    if (!sim || !out) return APIC_ERR_INVALID;
    return guarded(sim, [&] {
        auto& S = sim->impl;
        S.finish();
        std::memset(out, 0, sizeof *out);
        const apic::DevState h = S.sample_device(out);
        for (int s = 0; s < S.cfg.nspecies; ++s) {
            out->live_by_species[s] = h.n[s] - h.holes[s];
            out->kinetic_energy += out->kinetic_by_species[s];
            out->live_particles += h.n[s] - h.holes[s];
        }
        out->total_energy = out->kinetic_energy + out->field_energy;
        out->step = S.step;
        out->time = S.time;
    });
}

int apic_sim1d_model_safe_speed(const apic_sim1d* sim, int model, double* speed) {
    if (!sim || !speed || model < 0 || model >= sim->impl.cfg.nmodels) return APIC_ERR_INVALID;
    *speed = sim->impl.p.model[model].v_safe;
    return APIC_OK;
}

int apic_sim1d_cuda_stream(apic_sim1d* sim, void** stream) {
    if (!sim || !stream) return APIC_ERR_INVALID;
    *stream = (void*)sim->impl.stream;
    return APIC_OK;
}

int apic_sim1d_set_kernel_timing(apic_sim1d* sim, int enable) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded(sim, [&] {
        sim->impl.sync_status();
        sim->impl.collect_timing();
        sim->impl.timing = enable != 0;
        sim->impl.pass_ms = sim->impl.post_ms = 0.0;
        sim->impl.timed_passes = 0;
    });
}

int apic_sim1d_kernel_times(apic_sim1d* sim, double* pass_ms, double* post_ms, uint64_t* passes) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded(sim, [&] {
        sim->impl.sync_status();
        sim->impl.collect_timing();
        if (pass_ms) *pass_ms = sim->impl.pass_ms;
        if (post_ms) *post_ms = sim->impl.post_ms;
        if (passes) *passes = sim->impl.timed_passes;
    });
}

double apic_sim1d_time(const apic_sim1d* sim) { return sim ? sim->impl.time : 0.0; }
uint64_t apic_sim1d_step_count(const apic_sim1d* sim) { return sim ? sim->impl.step : 0; }

int apic_spatial_average1d_validate(const apic_config1d* cfg, const apic_spatial_average1d* sa) {
    if (!cfg || !sa) return APIC_ERR_INVALID;
    return guarded(nullptr, [&] { apic::validate_spatial_average(*cfg, *sa); });
}
int apic_sim1d_enable_spatial_average(apic_sim1d* sim, const apic_spatial_average1d* sa) {
    if (!sim || !sa) return APIC_ERR_INVALID;
    return guarded(sim, [&] { sim->impl.enable_spatial_average(*sa); });
}
int apic_sim1d_enable_power_transfer(apic_sim1d* sim) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded(sim, [&] { sim->impl.enable_power_transfer(); });
}
int apic_sim1d_power_transfer(apic_sim1d* sim, int species, double* electric_work) {
    if (!sim || !electric_work) return APIC_ERR_INVALID;
    return guarded(sim, [&] {
        auto& S = sim->impl;
        apic::require(species >= 0 && species < S.cfg.nspecies, "species index out of range");
        apic::require(S.p.ledger != 0, "the electric-work ledger is not enabled", APIC_ERR_STATE);
        S.finish();
        *electric_work = S.read_state().work[species];
    });
}
int apic_sim1d_spatial_average_counts(apic_sim1d* sim, uint64_t* samples, uint64_t* collision_steps,
                                      uint64_t* phase_samples, uint64_t* collision_phase_steps) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded(sim, [&] {
        auto& S = sim->impl;
        apic::require(S.sa.on, "spatial averaging is not enabled", APIC_ERR_STATE);
        S.finish();
        S.sync_status();
        if (samples) *samples = S.sa.samples;
        if (collision_steps) *collision_steps = S.sa.coll_steps;
        for (size_t b = 0; b < S.sa.P; ++b) {
            if (phase_samples) phase_samples[b] = S.sa.psamples[b];
            if (collision_phase_steps) collision_phase_steps[b] = S.sa.pcoll[b];
        }
    });
}
int apic_sim1d_spatial_sums(apic_sim1d* sim, int quantity, int index, int phase, double* out) {
    if (!sim || !out) return APIC_ERR_INVALID;
    return guarded(sim, [&] {
        auto& S = sim->impl;
        apic::require(S.sa.on, "spatial averaging is not enabled", APIC_ERR_STATE);
        apic::require(phase >= -1 && (phase < 0 || (size_t)phase < S.sa.P), "phase bin out of range");
        const size_t nx = S.cfg.nx, ns = (size_t)S.cfg.nspecies;
        const double* src = nullptr;
        if (quantity == APIC_SA_COLLISION_ENERGY) {
            apic::require(index >= 0 && index < S.sa.nch, "collision channel out of range");
            src = phase < 0 ? S.sa.coll + (size_t)index * nx
                            : S.sa.coll_phase + ((size_t)phase * (size_t)S.sa.nch + (size_t)index) * nx;
        } else {
            const double* blk = phase < 0 ? S.sa.tot : S.sa.phase + (size_t)phase * S.sa_block();
            if (quantity >= APIC_SA_DENSITY && quantity <= APIC_SA_KINETIC_ENERGY) {
                apic::require(index >= 0 && (size_t)index < ns, "species index out of range");
                src = blk + ((size_t)quantity * ns + (size_t)index) * nx;
            } else if (quantity >= APIC_SA_POTENTIAL && quantity <= APIC_SA_ELECTRIC_SQUARED) {
                src = blk + 5 * ns * nx + (size_t)(quantity - APIC_SA_POTENTIAL) * nx;
            } else {
                throw Error(APIC_ERR_INVALID, "unknown spatial-average quantity");
            }
        }
        S.finish();
        S.sync_status();
        APIC_CUDA(cudaMemcpyAsync(out, src, nx * sizeof(double), cudaMemcpyDeviceToHost, S.stream));
        APIC_CUDA(cudaStreamSynchronize(S.stream));
    });
}
int apic_sim1d_phase_eedf(apic_sim1d* sim, int phase, int region, apic_phase_eedf1d* out, double* histogram) {
    if (!sim || !out) return APIC_ERR_INVALID;
    return guarded(sim, [&] {
        auto& S = sim->impl;
        const auto& a = S.sa.cfg;
        apic::require(S.sa.on && a.eedf_species >= 0, "phase EEDF is not enabled", APIC_ERR_STATE);
        apic::require(phase >= 0 && (size_t)phase < S.sa.P && region >= 0 && region < a.eedf_regions,
                      "phase bin or region out of range");
        S.finish();
        S.sync_status();
        const size_t at = (size_t)phase * (size_t)a.eedf_regions + (size_t)region;
        unsigned long long cnt[2];
        double sums[7];
        APIC_CUDA(cudaMemcpyAsync(cnt, S.sa.eedf_cnt + at * 2, sizeof cnt, cudaMemcpyDeviceToHost, S.stream));
        APIC_CUDA(cudaMemcpyAsync(sums, S.sa.eedf_sum + at * 7, sizeof sums, cudaMemcpyDeviceToHost, S.stream));
        if (histogram)
            APIC_CUDA(cudaMemcpyAsync(histogram, S.sa.eedf_hist + at * a.eedf_bins, a.eedf_bins * sizeof(double),
                                      cudaMemcpyDeviceToHost, S.stream));
        APIC_CUDA(cudaStreamSynchronize(S.stream));
        out->macro_observations = cnt[0];
        out->overflow_macro_observations = cnt[1];
        out->represented_observations = sums[0];
        out->overflow_represented_observations = sums[1];
        out->weighted_energy_sum = sums[2];
        out->weighted_energy_squared_sum = sums[3];
        out->weighted_velocity_x_sum = sums[4];
        out->weighted_velocity_y_sum = sums[5];
        out->weighted_velocity_z_sum = sums[6];
    });
}

int apic_deposit_solve_gather_1d(int boundary, size_t nx, double length, double permittivity, double phi_left,
                                 double phi_right, int nspecies, const double* charge, const double* weight,
                                 const size_t* counts, const double* const* xs, double* rho, double* phi,
                                 double* electric, size_t nq, const double* xq, double* eq) {
    return guarded(nullptr, [&] {
        apic::require(nspecies >= 1 && nspecies <= APIC_MAX_SPECIES, "species count out of range");
        apic::require(std::isfinite(permittivity) && permittivity > 0,
                      "field-solver permittivity must be positive and finite");
        apic_config1d c{};
        c.boundary = boundary;
        c.velocity_dimensions = 1;
        c.units = APIC_NORMALIZED;
        c.relative_permittivity = permittivity;
        c.nx = nx;
        c.length = length;
        c.dt = 1.0;
        c.phi_left = phi_left;
        c.phi_right = phi_right;
        c.nspecies = nspecies;
        for (int s = 0; s < nspecies; ++s) {
            c.species[s].charge = charge[s];
            c.species[s].weight = weight[s];
            c.species[s].mass = 1.0;
            c.species[s].capacity = std::max<size_t>(counts[s], 1);
        }
        apic::Sim1D S;
        S.create(c);
        for (int s = 0; s < nspecies; ++s) {
            std::vector<double> zeros(counts[s], 0.0);
            S.load(s, counts[s], xs[s], zeros.data(), zeros.data(), nullptr, nullptr, nullptr);
        }
        S.resume(0.0, 0);
        S.read_fields(rho, phi, electric);
        if (nq > 0) {
            double* dq = S.dalloc<double>(nq);
            double* de = S.dalloc<double>(nq);
            APIC_CUDA(cudaMemcpyAsync(dq, xq, nq * sizeof(double), cudaMemcpyHostToDevice, S.stream));
            const unsigned blocks = (unsigned)((nq + 255) / 256);
            if (boundary == APIC_DIRICHLET)
                apic::k_gather_points1d<true><<<blocks, 256, 0, S.stream>>>(S.p, dq, de, (int)nq);
            else
                apic::k_gather_points1d<false><<<blocks, 256, 0, S.stream>>>(S.p, dq, de, (int)nq);
            APIC_CUDA(cudaGetLastError());
            APIC_CUDA(cudaMemcpyAsync(eq, de, nq * sizeof(double), cudaMemcpyDeviceToHost, S.stream));
            APIC_CUDA(cudaStreamSynchronize(S.stream));
        }
    });
}

int apic_collide3(const apic_mcc_model* model, double particle_mass, size_t n, double* v3, double dt,
                  const uint64_t* draws, const uint64_t* offsets, uint64_t seed, uint64_t step, uint32_t stream,
                  apic_collide_stats* stats) {
    return guarded(nullptr, [&] {
        apic::require(model && v3 && stats, "null argument");
        apic::require(n > 0 && n < (1u << 30), "particle count out of range");
        apic::require(std::isfinite(dt) && dt > 0, "MCC timestep must be positive and finite");
        // a standalone model: every channel kind (attachment and Henyey-Greenstein
        // included); ionization products are reported in stats
        std::vector<void*> allocs;
        cudaStream_t s = nullptr;
        APIC_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        struct Release {
            std::vector<void*>& a;
            cudaStream_t s;
            ~Release() {
                cudaStreamSynchronize(s);
                for (void* p : a) cudaFree(p);
                cudaStreamDestroy(s);
            }
        } release{allocs, s};
        apic::DeviceArena arena{allocs, s};
        apic_mcc_model mm = *model;
        mm.species = 0;
        apic::MccModelDev D{};
        apic::build_model(mm, particle_mass, arena, D);
        double* dv = arena.alloc<double>(3 * n);
        apic_collide_stats* ds = arena.alloc<apic_collide_stats>(n);
        uint64_t* dd = nullptr;
        uint64_t* doff = nullptr;
        if (draws) {
            apic::require(offsets != nullptr, "replay draws need per-particle offsets");
            const uint64_t total = offsets[n];
            dd = arena.alloc<uint64_t>(total);
            doff = arena.alloc<uint64_t>(n + 1);
            APIC_CUDA(cudaMemcpyAsync(dd, draws, total * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
            APIC_CUDA(cudaMemcpyAsync(doff, offsets, (n + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
        }
        APIC_CUDA(cudaMemcpyAsync(dv, v3, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
        apic::k_collide3<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(D, (int)n, dv, dt, dd, doff, seed,
                                                                    (uint32_t)step, stream, ds);
        APIC_CUDA(cudaGetLastError());
        APIC_CUDA(cudaMemcpyAsync(v3, dv, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
        APIC_CUDA(cudaMemcpyAsync(stats, ds, n * sizeof(apic_collide_stats), cudaMemcpyDeviceToHost, s));
        APIC_CUDA(cudaStreamSynchronize(s));
    });
}

}  // extern "C"
