// The fused 1D particle pass in the FP32 cell form (included by pic1d.cu).
//
// Same step as k_pass1d (src/Simulation.cpp:1008-1138: synchronize, collide,
// re-initialise the half step, kick, drift, walls or wrap, CIC deposit) with a
// particle stored as the index of the cell holding it, a float offset in
// [0, 1] inside that cell and float velocities: 20 bytes per 1D3V particle,
// 40 bytes per particle-step.  Every particle operation runs in FP32: the
// gather from a float copy of the field, the kick and the drift in cell units,
// the wall and wrap tests on the cell index, and the null-collision loop
// (collide3f).  FP64 remains for the charge, accumulated in 64-bit fixed point
// (order-independent), for the field solve (the post kernel) and for the
// energy ledgers (collisions, wall losses), summed in FP64.
//
// Layout: the particles of a species occupy slots [0, n) and are updated in
// place; a particle absorbed by a wall leaves a hole (its cell set to
// kDeadCell), as the reference leaves a dead Particle in its vector
// (src/Simulation.cpp:1039-1077), and ionization products are appended after
// slot n.  Holes are squeezed out, order preserved, every kCompactSteps steps
// (k_c32_count / k_c32_scan / k_c32_scatter), so a pass reads its particles at
// their slots with no index lookup.
//
// Position semantics of the reference (src/FieldSolver.cpp:909-924): a
// Dirichlet particle is gathered at its position clamped to [0, L] with the
// cell index capped at nx - 2, absorbed once x < 0 or x > L; a periodic
// particle wraps into [0, L).  Here x = (cell + off) dx; x = L exactly is
// cell nx - 2 with off = 1.
// (Included inside namespace apic, after k_pass1d and its helpers.)
#pragma once

constexpr int kChunk32 = 32 * kItems;  // particles per warp chunk of k_pass1d_c32
constexpr int kDeadCell = -2147483647 - 1;  // cell index of a hole
constexpr unsigned kCompactSteps = 32;      // steps between compactions (at step counts divisible by it)

// resident CTAs of k_pass1d_c32 per SM (register budget of the launch bounds)
#ifndef APIC_C32_MIN_BLOCKS
#define APIC_C32_MIN_BLOCKS 4
#endif
constexpr int kMinBlocks32 = APIC_C32_MIN_BLOCKS;

// a collision candidate handed from the pass to the collision kernel
struct CandRec32 {
    float v[3];  // time-centred velocity after the synchronize half kick
    float E;     // field at the particle
    int cell;
    float off;
    unsigned slot;
    unsigned species;
};

// The gather cell and weight of a stored position: the stored cell inside the
// grid, or the clamped end of a Dirichlet grid for a position outside it.
template <bool DIRICHLET>
__device__ __forceinline__ void cell_weights(int cell, float off, int nx, int& i0, int& i1, float& f) {
    if (DIRICHLET) {
        if (cell < 0) { i0 = 0; f = 0.0f; }
        else if (cell > nx - 2) { i0 = nx - 2; f = 1.0f; }
        else { i0 = cell; f = off; }
        i1 = i0 + 1;
    } else {
        i0 = cell;
        f = off;
        i1 = cell + 1 == nx ? 0 : cell + 1;
    }
}

// FP64 position -> (cell, offset) with the reference's wrap; a Dirichlet
// position keeps its (possibly out-of-range) cell, x = L maps to cell nx - 2
// with offset 1.
template <bool DIRICHLET>
__device__ __forceinline__ void position_to_cell(double x, const Params1D& p, int& cell, float& off) {
    double g;
    if (DIRICHLET) {
        g = x * p.inv_dx;
    } else {
        g = wrap_periodic(x, p.L) * p.inv_dx;
    }
    if (!(g == g)) { cell = 0; off = 0.0f; return; }  // NaN: flagged by the pass that meets it
    double c = floor(g);
    float o = (float)(g - c);
    if (o >= 1.0f) { c += 1.0; o = 0.0f; }  // g just below an integer rounds to a whole cell
    if (!DIRICHLET) {
        if (c >= (double)p.nx) c -= (double)p.nx;
        if (c < 0.0) c = 0.0;
    } else if (c == (double)(p.nx - 1) && o == 0.0f) {
        c = (double)(p.nx - 2);
        o = 1.0f;
    }
    cell = (int)fmax(fmin(c, 2147483000.0), -2147483000.0);
    off = o;
}

template <bool DIRICHLET>
__global__ void k_x_to_cell(const double* __restrict__ x, int* __restrict__ cell, float* __restrict__ off,
                            unsigned n, Params1D p) {
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        position_to_cell<DIRICHLET>(x[i], p, cell[i], off[i]);
}

__global__ void k_cell_to_x(const int* __restrict__ cell, const float* __restrict__ off, double* __restrict__ x,
                            unsigned n, double dx) {
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[i] = ((double)cell[i] + (double)off[i]) * dx;
}

// Each warp streams chunks of kChunk32 slots on its own (no CTA-wide barrier
// inside the loop): gather, synchronize, the frequency-bound check and the
// choice of this step's collision candidates; every particle that is not a
// candidate is then re-initialised, kicked, drifted, tested against the walls,
// deposited into the CTA's shared-memory density and written back to its slot.
// Candidates leave for the collision kernel (k_collide1d_c32) as records in
// the run's candidate buffer, which finishes their step in full warps.
//
// Candidates: a particle's first null-collision waiting time -ln(u)/nu falls
// inside the step with probability P = 1 - exp(-nu dt), independently of every
// other particle.  Instead of one uniform per particle, the warp draws the gaps
// between candidates along the chunk, geometric with parameter P
// (floor(-ln(u) / (nu dt)) particles skipped before each candidate), and each
// candidate draws its first waiting time from the exponential truncated to the
// step, -ln(1 - u P) / nu.  The candidates and their first waiting times then
// have exactly the distribution of the per-particle test, at a cost per
// candidate instead of per particle.
template <int VDIM, bool DIRICHLET>
__global__ void __launch_bounds__(kThreads, kMinBlocks32) k_pass1d_c32(Params1D p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned long long* sRho = reinterpret_cast<unsigned long long*>(smem_raw);
    float* sE = reinterpret_cast<float*>(sRho + p.nx);
    constexpr int kWarps = kThreads / 32;
    __shared__ unsigned s_mask[kWarps][kChunk32 / 32];
    // the CTA's wall-loss tallies, added to the run's totals once at the end
    // (every warp of the GPU adding to the same few counters would serialise)
    __shared__ unsigned long long s_lost[kMaxSpecies][2];
    __shared__ double s_lost_energy[kMaxSpecies][2];
    __shared__ unsigned s_dead[kMaxSpecies];
    __shared__ unsigned s_ncand;  // candidates this CTA handed on (its region of the candidate buffer)

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned mode = p.mode;
    const int nx = p.nx;
    for (int i = tid; i < nx; i += kThreads) {
        sE[i] = (float)p.E[i];
        sRho[i] = 0ull;
    }
    if (tid == 0) s_ncand = 0u;
    CandRec32* region = p.cands ? p.cands + (size_t)blockIdx.x * p.cand_per_region : nullptr;
    if (lane < kChunk32 / 32) s_mask[warp][lane] = 0u;
    if (tid < kMaxSpecies * 2) {
        (&s_lost[0][0])[tid] = 0ull;
        (&s_lost_energy[0][0])[tid] = 0.0;
    }
    if (tid < kMaxSpecies) s_dead[tid] = 0u;
    DevState* st = p.st;
    // chunk counts of the species, and the first chunk of species 1..3
    unsigned b1 = 0, b2 = 0, b3 = 0, total = 0;
#pragma unroll
    for (int s = 0; s < kMaxSpecies; ++s) {
        total += s < p.nspecies ? (st->n[s] + kChunk32 - 1) / kChunk32 : 0u;
        if (s == 0) b1 = total;
        if (s == 1) b2 = total;
        if (s == 2) b3 = total;
    }
    const uint32_t mcc_step = (uint32_t)(st->step - 1ull);
    const int ncell = DIRICHLET ? nx - 1 : nx;
    const uint32_t key0 = (uint32_t)p.seed, key1 = (uint32_t)(p.seed >> 32);
    const unsigned lt = (1u << lane) - 1u;
    __syncthreads();

    for (unsigned c = blockIdx.x * kWarps + warp; c < total; c += gridDim.x * kWarps) {
        const int s = c < b1 ? 0 : (c < b2 ? 1 : (c < b3 ? 2 : 3));
        const unsigned chunk = c - (s == 0 ? 0u : (s == 1 ? b1 : (s == 2 ? b2 : b3)));
        const SpeciesDev& S = p.sp[s];
        const unsigned n = st->n[s];
        const unsigned base = chunk * kChunk32;
        const bool mcc = (mode & kModeSyncMcc) && S.model >= 0 && VDIM == 3;

        int cell[kItems];
        float off[kItems], vh[kItems], vy[kItems], vz[kItems], vc[kItems], Ek[kItems];
        bool keep[kItems];
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            const unsigned idx = base + k * 32 + lane;
            const bool in = idx < n;
            cell[k] = in ? __ldcs(S.cell[0] + idx) : kDeadCell;
            const bool live = cell[k] != kDeadCell;
            keep[k] = live;
            off[k] = live ? __ldcs(S.off[0] + idx) : 0.0f;
            vh[k] = live ? __ldcs(S.vh32[0] + idx) : 0.0f;
            vy[k] = (VDIM == 3 && live && mcc) ? __ldcs(S.vy32[0] + idx) : 0.0f;
            vz[k] = (VDIM == 3 && live && mcc) ? __ldcs(S.vz32[0] + idx) : 0.0f;
            vc[k] = ((mode & kModeInitHalf) && live) ? (float)S.v[idx] : 0.0f;
        }
        // -- gather, synchronize, frequency-bound check --
        bool finite_v[kItems];
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            Ek[k] = 0.0f;
            finite_v[k] = false;
            if (!keep[k]) continue;
            int i0, i1;
            float f;
            cell_weights<DIRICHLET>(cell[k], off[k], nx, i0, i1, f);
            const float E = sE[i0] * (1.0f - f) + sE[i1] * f;
            Ek[k] = E;
            if (mode & kModeInitHalf) vh[k] = vc[k] - S.hqmdt32 * E;  // src/Pusher.cpp:66-68
            if (mode & kModeSyncMcc) {
                vc[k] = vh[k] + S.hqmdt32 * E;  // src/Pusher.cpp:78-80
                if (mcc) {
                    const float s2 = vc[k] * vc[k] + vy[k] * vy[k] + vz[k] * vz[k];
                    if (!isfinite(s2)) {  // src/Collision.cpp:910-916
                        atomicOr(&st->error, kErrNonFinite);
                        continue;
                    }
                    finite_v[k] = true;
                    if (!(s2 <= p.model32[S.model].v_safe2) &&
                        !frequency_bound_ok_far(p.gmodel[S.model], (double)sqrtf(s2)))
                        atomicOr(&st->error, kErrMajorant);
                }
            }
        }
        if (mcc && !S.no_candidates) {
            // -- candidates: geometric gaps along the chunk from the chunk's own stream --
            int covered = 0;  // chunk positions decided so far
            for (uint32_t round = 0; covered < kChunk32 && round < 64; ++round) {
                uint32_t w[4];
                philox4x32_10(round * 8u + (uint32_t)(lane >> 2), chunk, mcc_step, 0x40000000u | (uint32_t)s, key0,
                              key1, w);
                const int wsel = lane & 3;
                const uint32_t word = wsel == 0 ? w[0] : (wsel == 1 ? w[1] : (wsel == 2 ? w[2] : w[3]));
                const float u = ((float)(word >> 9) + 0.5f) * 1.1920928955078125e-7f;
                const float gap = fminf(-__logf(u) * S.inv_nudt32, 1.0e6f);
                int step_len = (int)gap + 1;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, step_len, o);
                    if (lane >= o) step_len += y;
                }
                const int pos = covered + step_len - 1;
                if (pos < kChunk32) atomicOr(&s_mask[warp][pos >> 5], 1u << (pos & 31));
                covered = __shfl_sync(0xffffffffu, covered + step_len, 31);
            }
            __syncwarp();
            // candidates leave this pass: one record each in the candidate buffer
#pragma unroll
            for (int k = 0; k < kItems; ++k) {
                const bool cand = finite_v[k] && ((s_mask[warp][k] >> lane) & 1u);
                const unsigned b = __ballot_sync(0xffffffffu, cand);
                if (!b) continue;
                unsigned q0 = 0;
                if (lane == 0) q0 = atomicAdd(&s_ncand, (unsigned)__popc(b));
                q0 = __shfl_sync(0xffffffffu, q0, 0);
                if (cand) {
                    const unsigned q = q0 + __popc(b & lt);
                    if (q < p.cand_per_region) {
                        CandRec32 r;
                        r.v[0] = vc[k]; r.v[1] = vy[k]; r.v[2] = vz[k];
                        r.E = Ek[k];
                        r.cell = cell[k];
                        r.off = off[k];
                        r.slot = base + k * 32 + lane;
                        r.species = (unsigned)s;
                        region[q] = r;
                    } else {
                        atomicOr(&st->error, kErrCandBuffer);
                    }
                    keep[k] = false;  // finished by the collision kernel
                }
            }
            __syncwarp();
            if (lane < kChunk32 / 32) s_mask[warp][lane] = 0u;
        }
        // -- re-initialise, kick, drift, walls, deposit, write back --
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            if (!keep[k]) continue;
            const unsigned idx = base + k * 32 + lane;
            const float E = Ek[k];
            if (mcc) vh[k] = vc[k] - S.hqmdt32 * E;  // src/Simulation.cpp:924-926
            if (mode & kModeKickDrift) {
                vh[k] = vh[k] + S.qmdt32 * E;  // src/Pusher.cpp:70-76, in cell units
                const float g = off[k] + vh[k] * S.dtdx32;
                if (!isfinite(g)) {  // flagged and dropped: deposits nothing
                    atomicOr(&st->error, kErrNonFinite);
                    atomicAdd(&s_dead[s], 1u);
                    __stcs(S.cell[0] + idx, kDeadCell);
                    continue;
                }
                const float sh = floorf(g);
                int cc = cell[k] + (int)fmaxf(fminf(sh, 1.0e9f), -1.0e9f);
                float o = g - sh;
                if (o >= 1.0f) { ++cc; o = 0.0f; }
                if (!DIRICHLET) {
                    if (cc >= nx || cc < 0) cc = ((cc % nx) + nx) % nx;  // src/FieldSolver.cpp:15-17
                } else if (cc < 0 || cc > ncell || (cc == ncell && o > 0.0f)) {
                    // absorbing walls and loss ledger, src/Simulation.cpp:1047-1077
                    if (!mcc) {
                        vy[k] = __ldcs(S.vy32[0] + idx);
                        vz[k] = __ldcs(S.vz32[0] + idx);
                    }
                    const float w[3] = {vh[k], VDIM == 3 ? vy[k] : 0.0f, VDIM == 3 ? vz[k] : 0.0f};
                    const int side = cc < 0 ? 0 : 1;
                    atomicAdd(&s_lost[s][side], 1ull);
                    atomicAdd(&s_lost_energy[s][side], energy64(S.mass * S.weight, w));
                    atomicAdd(&s_dead[s], 1u);
                    __stcs(S.cell[0] + idx, kDeadCell);
                    continue;
                } else if (cc == ncell) {
                    cc = ncell - 1;  // x = L: the last cell at offset 1
                    o = 1.0f;
                }
                cell[k] = cc;
                off[k] = o;
                __stcs(S.cell[0] + idx, cc);
                __stcs(S.off[0] + idx, o);
            }
            if (mode & kModeDeposit) {
                int i0, i1;
                float f;
                cell_weights<DIRICHLET>(cell[k], off[k], nx, i0, i1, f);
                float q0 = S.dep32 * (1.0f - f), q1 = S.dep32 * f;
                if (DIRICHLET) {  // q w / node_volume: half volumes at the walls, src/Species.cpp:180-181
                    if (i0 == 0) q0 *= 2.0f;
                    if (i1 == nx - 1) q1 *= 2.0f;
                }
                atomicAdd(&sRho[i0], (unsigned long long)(long long)__float2int_rn(q0));
                atomicAdd(&sRho[i1], (unsigned long long)(long long)__float2int_rn(q1));
            }
            __stcs(S.vh32[0] + idx, vh[k]);
            if (mode & (kModeWriteV | kModeInitHalf)) S.v[idx] = (double)vc[k];
        }
    }
    __syncthreads();
    if (mode & kModeDeposit) {
        for (int i = tid; i < nx; i += kThreads) {
            const unsigned long long a = sRho[i];
            if (a) atomicAdd(&p.rho_acc[i], a);
        }
    }
    if (tid < kMaxSpecies * 2) {
        const unsigned long long c = (&s_lost[0][0])[tid];
        if (c) atomicAdd(&st->lost[0][0] + tid, c);
        const double e = (&s_lost_energy[0][0])[tid];
        if (e != 0.0) atomicAdd(&st->lost_energy[0][0] + tid, e);
    }
    if (tid < kMaxSpecies && s_dead[tid]) atomicAdd(&st->holes[tid], s_dead[tid]);
    // (a run without collision models has no candidate buffer)
    if (tid == 0 && p.cand_count) p.cand_count[blockIdx.x] = min(s_ncand, p.cand_per_region);
}

// The collision candidates of the pass, one per thread in full warps: the
// null-collision loop (collide3f), then the rest of the particle's step as in
// the pass (re-initialise, kick, drift, walls, deposit, write back).  The
// pass's regions hold few records each, so every CTA first takes the prefix
// sums of the region counts and numbers the candidates densely.
constexpr int kCollideThreads = 128;
constexpr int kMaxRegions = 2048;  // regions (CTAs of the pass) the dense numbering covers
template <int VDIM, bool DIRICHLET>
__global__ void __launch_bounds__(kCollideThreads) k_collide1d_c32(Params1D p) {
    __shared__ unsigned long long s_cand, s_null, s_chan[kMaxModels][kMaxChannels], s_lost[kMaxSpecies][2];
    __shared__ double s_energy[kMaxModels][kMaxChannels], s_lost_energy[kMaxSpecies][2];
    __shared__ unsigned s_dead[kMaxSpecies];
    __shared__ unsigned s_start[kMaxRegions + 1];  // first dense index of each region
    const int tid = threadIdx.x;
    const unsigned regions = min(p.cand_regions, (unsigned)kMaxRegions);
    {
        // exclusive prefix sums of the region counts, 16 per thread
        using Scan = cub::BlockScan<unsigned, kCollideThreads>;
        __shared__ typename Scan::TempStorage tmp;
        constexpr int PER = kMaxRegions / kCollideThreads;
        unsigned c[PER], o[PER];
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const unsigned r = tid * PER + k;
            c[k] = r < regions ? __ldg(p.cand_count + r) : 0u;
        }
        unsigned total;
        Scan(tmp).ExclusiveSum(c, o, total);
#pragma unroll
        for (int k = 0; k < PER; ++k) s_start[tid * PER + k] = o[k];
        if (tid == 0) s_start[kMaxRegions] = total;
    }
    if (tid < kMaxModels * kMaxChannels) {
        (&s_chan[0][0])[tid] = 0ull;
        (&s_energy[0][0])[tid] = 0.0;
    }
    if (tid < kMaxSpecies * 2) {
        (&s_lost[0][0])[tid] = 0ull;
        (&s_lost_energy[0][0])[tid] = 0.0;
    }
    if (tid < kMaxSpecies) s_dead[tid] = 0u;
    if (tid == 0) s_cand = s_null = 0ull;
    __syncthreads();
    DevState* st = p.st;
    const unsigned mode = p.mode;
    const unsigned ntotal = s_start[kMaxRegions];
    const uint32_t mcc_step = (uint32_t)(st->step - 1ull);
    const float dt = (float)p.dt;
    const float dt_in = dt * (1.0f - kFltEpsilon);  // largest first wait kept inside the step
    const int nx = p.nx;
    const int ncell = DIRICHLET ? nx - 1 : nx;
    for (unsigned d = blockIdx.x * kCollideThreads + tid; d < ntotal; d += gridDim.x * kCollideThreads) {
        // region holding dense index d: the last region whose start is <= d
        unsigned lo = 0, hi = regions;
        while (hi - lo > 1) {
            const unsigned mid = (lo + hi) >> 1;
            if (s_start[mid] <= d) lo = mid; else hi = mid;
        }
        const CandRec32 rec = p.cands[(size_t)lo * p.cand_per_region + (d - s_start[lo])];
        const int s = (int)rec.species;
        const SpeciesDev& S = p.sp[s];
        const MccModel32& M = p.model32[S.model];
        const MccModelDev& G = p.gmodel[S.model];
        const unsigned slot = rec.slot;
        Philox32 rng(p.seed, slot, mcc_step, (uint32_t)s);
        // first waiting time: the exponential truncated to the step
        const float wait = fminf(-log1pf(-rng.uniform() * S.cand_p32) * M.inv_max_frequency, dt_in);
        CollideResult32 r;
        unsigned nion = 0;
        const double px = ((double)rec.cell + (double)rec.off) * p.dx;
        float v[3] = {rec.v[0], rec.v[1], rec.v[2]};
        collide3f(
            M, v, dt, wait, rng, r, [&](float speed) { return frequency_bound_ok_far(G, (double)speed); },
            [&](int ch, double de) {
                atomicAdd(&s_chan[S.model][ch], 1ull);
                atomicAdd(&s_energy[S.model][ch], de * S.weight);
            },
            [&](int ch, const float* vs, const float* vi) {
                const unsigned bslot = atomicAdd(&st->nbirths, 2u);
                const MccChannel32& C = M.ch[ch];
                if (bslot + 2u <= p.births_cap) {
                    const unsigned long long key =
                        ((unsigned long long)s << 56) | ((unsigned long long)slot << 16) | (nion << 1);
                    BirthRec a, b;
                    a.key = key; a.species = C.secondary; a.pad = 0;
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
                atomicAdd(&s_energy[S.model][ch], energy64(A.mass * A.weight, vs) + energy64(B.mass * B.weight, vi));
                ++nion;
            });
        if (r.error) atomicOr(&st->error, r.error);
        atomicAdd(&s_cand, (unsigned long long)r.candidates);
        if (r.nulls) atomicAdd(&s_null, (unsigned long long)r.nulls);
        // the rest of the step, as in the pass
        const float E = rec.E;
        float vh = v[0] - S.hqmdt32 * E;  // src/Simulation.cpp:924-926
        int cell = rec.cell;
        float off = rec.off;
        bool keep = true;
        if (mode & kModeKickDrift) {
            vh = vh + S.qmdt32 * E;
            const float g = off + vh * S.dtdx32;
            if (!isfinite(g)) {
                atomicOr(&st->error, kErrNonFinite);
                keep = false;
            } else {
                const float sh = floorf(g);
                int cc = cell + (int)fmaxf(fminf(sh, 1.0e9f), -1.0e9f);
                float o = g - sh;
                if (o >= 1.0f) { ++cc; o = 0.0f; }
                if (!DIRICHLET) {
                    if (cc >= nx || cc < 0) cc = ((cc % nx) + nx) % nx;
                } else if (cc < 0 || cc > ncell || (cc == ncell && o > 0.0f)) {
                    const float w[3] = {vh, v[1], v[2]};
                    const int side = cc < 0 ? 0 : 1;
                    atomicAdd(&s_lost[s][side], 1ull);
                    atomicAdd(&s_lost_energy[s][side], energy64(S.mass * S.weight, w));
                    keep = false;
                } else if (cc == ncell) {
                    cc = ncell - 1;
                    o = 1.0f;
                }
                cell = cc;
                off = o;
            }
        }
        if (!keep) {
            atomicAdd(&s_dead[s], 1u);
            S.cell[0][slot] = kDeadCell;
            continue;
        }
        if (mode & kModeDeposit) {
            int i0, i1;
            float f;
            cell_weights<DIRICHLET>(cell, off, nx, i0, i1, f);
            float q0 = S.dep32 * (1.0f - f), q1 = S.dep32 * f;
            if (DIRICHLET) {
                if (i0 == 0) q0 *= 2.0f;
                if (i1 == nx - 1) q1 *= 2.0f;
            }
            atomicAdd(&p.rho_acc[i0], (unsigned long long)(long long)__float2int_rn(q0));
            atomicAdd(&p.rho_acc[i1], (unsigned long long)(long long)__float2int_rn(q1));
        }
        S.cell[0][slot] = cell;
        S.off[0][slot] = off;
        S.vh32[0][slot] = vh;
        S.vy32[0][slot] = v[1];
        S.vz32[0][slot] = v[2];
        if (mode & kModeWriteV) S.v[slot] = (double)v[0];
    }
    __syncthreads();
    if (tid < kMaxModels * kMaxChannels) {
        const unsigned long long c = (&s_chan[0][0])[tid];
        if (c) atomicAdd(&st->chan[0][0] + tid, c);
        const double e = (&s_energy[0][0])[tid];
        if (e != 0.0) atomicAdd(&st->chan_energy[0][0] + tid, e);
    }
    if (tid < kMaxSpecies * 2) {
        const unsigned long long c = (&s_lost[0][0])[tid];
        if (c) atomicAdd(&st->lost[0][0] + tid, c);
        const double e = (&s_lost_energy[0][0])[tid];
        if (e != 0.0) atomicAdd(&st->lost_energy[0][0] + tid, e);
    }
    if (tid < kMaxSpecies && s_dead[tid]) atomicAdd(&st->holes[tid], s_dead[tid]);
    if (tid == 0) {
        if (s_cand) atomicAdd(&st->candidates, s_cand);
        if (s_null) atomicAdd(&st->nulls, s_null);
    }
}

// ---- compaction of the holes (FP32 cell form) ----------------------------------

// live particles of each chunk of slots [0, n)
__global__ void k_c32_count(const int* __restrict__ cell, const unsigned* __restrict__ np, unsigned* counts) {
    const unsigned n = *np;
    const unsigned nch = (n + kChunk32 - 1) / kChunk32;
    const int lane = threadIdx.x & 31;
    for (unsigned c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < nch; c += (gridDim.x * blockDim.x) >> 5) {
        unsigned live = 0;
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            const unsigned i = c * kChunk32 + k * 32 + lane;
            live += __popc(__ballot_sync(0xffffffffu, i < n && cell[i] != kDeadCell));
        }
        if (lane == 0) counts[c] = live;
    }
}

// exclusive prefix sums of the chunk counts in place (counts[nch] = total);
// *n_old receives n; with holes non-null (a compaction) *np becomes the total
// and the holes are cleared
constexpr int kScanThreads = 512, kScanItems = 8;
__global__ void __launch_bounds__(kScanThreads) k_c32_scan(unsigned* counts, unsigned* np, unsigned* holes,
                                                           unsigned* n_old) {
    using Scan = cub::BlockScan<unsigned, kScanThreads>;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ unsigned s_carry;
    const unsigned n = *np;
    const unsigned nch = (n + kChunk32 - 1) / kChunk32;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (unsigned b0 = 0; b0 < nch; b0 += kScanThreads * kScanItems) {
        unsigned v[kScanItems], o[kScanItems];
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            const unsigned c = b0 + threadIdx.x * kScanItems + k;
            v[k] = c < nch ? counts[c] : 0u;
        }
        unsigned total;
        Scan(tmp).ExclusiveSum(v, o, total);
        const unsigned carry = s_carry;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            const unsigned c = b0 + threadIdx.x * kScanItems + k;
            if (c < nch) counts[c] = carry + o[k];
        }
        __syncthreads();
        if (threadIdx.x == 0) s_carry = carry + total;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *n_old = n;
        if (holes) {  // compaction: the run continues on the squeezed layout
            *np = s_carry;
            *holes = 0u;
        }
        counts[nch] = s_carry;
    }
}

struct C32Arrays {
    const int* cell;
    const float* off;
    const float* vh;
    const float* vy;
    const float* vz;
    const double* v;
};

// live particles of [0, n) in slot order to dst (order preserved)
__global__ void k_c32_scatter(C32Arrays src, int* cell, float* off, float* vh, float* vy, float* vz, double* v,
                              const unsigned* n_old, const unsigned* offsets) {
    const unsigned n = *n_old;
    const unsigned nch = (n + kChunk32 - 1) / kChunk32;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    for (unsigned c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < nch; c += (gridDim.x * blockDim.x) >> 5) {
        unsigned o = offsets[c];
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            const unsigned i = c * kChunk32 + k * 32 + lane;
            const int cl = i < n ? src.cell[i] : kDeadCell;
            const bool live = cl != kDeadCell;
            const unsigned b = __ballot_sync(0xffffffffu, live);
            if (live) {
                const unsigned d = o + __popc(b & lt);
                cell[d] = cl;
                off[d] = src.off[i];
                vh[d] = src.vh[i];
                if (vy) { vy[d] = src.vy[i]; vz[d] = src.vz[i]; }
                if (v) v[d] = src.v[i];
            }
            o += __popc(b);
        }
    }
}

// one component of the live particles, in slot order, as doubles (read-back)
__global__ void k_c32_gather(C32Arrays src, int component, double dx, const unsigned* np, const unsigned* offsets,
                             double* out) {
    const unsigned n = *np;
    const unsigned nch = (n + kChunk32 - 1) / kChunk32;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    for (unsigned c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < nch; c += (gridDim.x * blockDim.x) >> 5) {
        unsigned o = offsets[c];
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            const unsigned i = c * kChunk32 + k * 32 + lane;
            const int cl = i < n ? src.cell[i] : kDeadCell;
            const bool live = cl != kDeadCell;
            const unsigned b = __ballot_sync(0xffffffffu, live);
            if (live) {
                double x;
                switch (component) {
                    case 0: x = ((double)cl + (double)src.off[i]) * dx; break;
                    case 1: x = src.v[i]; break;
                    case 2: x = (double)src.vh[i]; break;
                    case 3: x = (double)src.vy[i]; break;
                    default: x = (double)src.vz[i]; break;
                }
                out[o + __popc(b & lt)] = x;
            }
            o += __popc(b);
        }
    }
}
