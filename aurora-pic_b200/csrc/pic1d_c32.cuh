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
// Position semantics of the reference (src/FieldSolver.cpp:909-924): a
// Dirichlet particle is gathered at its position clamped to [0, L] with the
// cell index capped at nx - 2, absorbed once x < 0 or x > L; a periodic
// particle wraps into [0, L).  Here x = (cell + off) dx; x = L exactly is
// cell nx - 2 with off = 1.
// (Included inside namespace apic, after k_pass1d and its helpers.)
#pragma once

// resident CTAs of k_pass1d_c32 per SM (register budget of the launch bounds)
#ifndef APIC_C32_MIN_BLOCKS
#define APIC_C32_MIN_BLOCKS 3
#endif
constexpr int kMinBlocks32 = APIC_C32_MIN_BLOCKS;

struct Cand32 {
    float v[3];
    float wait;   // first waiting time, inside the step
    int cell;
    float off;
    unsigned slot;
    unsigned pad;
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

template <int VDIM, bool DIRICHLET>
__global__ void __launch_bounds__(kThreads, kMinBlocks32) k_pass1d_c32(Params1D p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned long long* sRho = reinterpret_cast<unsigned long long*>(smem_raw);
    float* sE = reinterpret_cast<float*>(sRho + p.nx);
    __shared__ unsigned s_cnt[32];
    __shared__ unsigned s_qlen;
    __shared__ Cand32 s_queue[kQueue];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned mode = p.mode;
    const int nx = p.nx;
    for (int i = tid; i < nx; i += kThreads) {
        sE[i] = (float)p.E[i];
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
    const float dt = (float)p.dt;
    const float dt_in = dt * (1.0f - kFltEpsilon);  // largest first wait kept inside the step
    const int ncell = DIRICHLET ? nx - 1 : nx;
    __syncthreads();

    for (unsigned t = blockIdx.x; t < total_tiles; t += gridDim.x) {
        int s = 0;
        while (t >= tiles_before[s + 1]) ++s;
        const unsigned tile = t - tiles_before[s];
        const SpeciesDev& S = p.sp[s];
        const unsigned n = st->n[s];
        const unsigned nr = st->nranges[s];
        const unsigned base = tile * kTile;
        const bool mcc = (mode & kModeSyncMcc) && S.model >= 0 && VDIM == 3;
        const unsigned wfirst = base + (unsigned)(tid & ~31);
        unsigned r0 = 0;
        if (lane == 0 && wfirst < n) r0 = range_of(S.rlstart[0], nr, wfirst);
        r0 = __shfl_sync(0xffffffffu, r0, 0);

        int cell[kItems];
        float off[kItems], vh[kItems], vy[kItems], vz[kItems], vc[kItems], Ek[kItems];
        bool keep[kItems];
        int queued[kItems];
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            const unsigned idx = base + k * kThreads + tid;
            const bool live = idx < n;
            keep[k] = live;
            queued[k] = -1;
            const unsigned ph = live ? physical_slot_from(S.rlstart[0], S.rstart[0], nr, r0, idx) : 0u;
            cell[k] = live ? __ldcs(S.cell[0] + ph) : 0;
            off[k] = live ? __ldcs(S.off[0] + ph) : 0.0f;
            vh[k] = live ? __ldcs(S.vh32[0] + ph) : 0.0f;
            vy[k] = (VDIM == 3 && live) ? __ldcs(S.vy32[0] + ph) : 0.0f;
            vz[k] = (VDIM == 3 && live) ? __ldcs(S.vz32[0] + ph) : 0.0f;
            vc[k] = ((mode & kModeInitHalf) && live) ? (float)S.v[ph] : 0.0f;
        }
        // -- phase A: gather, synchronize, first collision draw --
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            Ek[k] = 0.0f;
            if (!keep[k]) continue;
            const unsigned idx = base + k * kThreads + tid;
            int i0, i1;
            float f;
            cell_weights<DIRICHLET>(cell[k], off[k], nx, i0, i1, f);
            const float E = sE[i0] * (1.0f - f) + sE[i1] * f;
            Ek[k] = E;
            if (mode & kModeInitHalf) vh[k] = vc[k] - S.hqmdt32 * E;  // src/Pusher.cpp:66-68
            if (mode & kModeSyncMcc) {
                vc[k] = vh[k] + S.hqmdt32 * E;  // src/Pusher.cpp:78-80
                if (mcc) {
                    const MccModel32& M = p.model32[S.model];
                    const float s2 = vc[k] * vc[k] + vy[k] * vy[k] + vz[k] * vz[k];
                    if (!isfinite(s2)) {  // src/Collision.cpp:910-916
                        atomicOr(&st->error, kErrNonFinite);
                        continue;
                    }
                    if (!(s2 <= M.v_safe2) && !frequency_bound_ok_far(p.gmodel[S.model], (double)sqrtf(s2)))
                        atomicOr(&st->error, kErrMajorant);
                    uint32_t w[4];
                    philox4x32_10(0u, idx, mcc_step, (uint32_t)s, (uint32_t)p.seed, (uint32_t)(p.seed >> 32), w);
                    const uint64_t d0 = (uint64_t)w[1] << 32 | w[0];
                    // the FP64 form's exact first-wait decision on the raw draw
                    if (d0 != 0ull && !S.no_candidates && d0 >= S.cand_draw_min) {
                        const float u0 = ((float)(d0 >> 41) + 0.5f) * 1.1920928955078125e-7f;
                        const float wait = fminf(-__logf(u0) * M.inv_max_frequency, dt_in);
                        const unsigned q = atomicAdd(&s_qlen, 1u);
                        if (q < (unsigned)kQueue) {
                            Cand32& ce = s_queue[q];
                            ce.v[0] = vc[k]; ce.v[1] = vy[k]; ce.v[2] = vz[k];
                            ce.wait = wait;
                            ce.cell = cell[k];
                            ce.off = off[k];
                            ce.slot = idx;
                            queued[k] = (int)q;
                        } else {
                            atomicOr(&st->error, kErrBirths);
                        }
                    }
                }
            }
        }
        __syncthreads();
        // -- phase B: collision loops of the queued candidates --
        if (mcc) {
            const unsigned qlen = min(s_qlen, (unsigned)kQueue);
            const MccModel32& M = p.model32[S.model];
            const MccModelDev& G = p.gmodel[S.model];
            for (unsigned q = tid; q < qlen; q += kThreads) {
                Cand32& ce = s_queue[q];
                Philox32 rng(p.seed, ce.slot, mcc_step, (uint32_t)s);
                rng.start_at(2);
                CollideResult32 r;
                unsigned nion = 0;
                const unsigned slot = ce.slot;
                const double px = ((double)ce.cell + (double)ce.off) * p.dx;
                float vel[3] = {ce.v[0], ce.v[1], ce.v[2]};
                collide3f(
                    M, vel, dt, ce.wait, rng, r,
                    [&](float speed) { return frequency_bound_ok_far(G, (double)speed); },
                    [&](int ch, double de) {
                        atomicAdd(&st->chan[S.model][ch], 1ull);
                        atomicAdd(&st->chan_energy[S.model][ch], de * S.weight);
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
                        const double added = energy64(A.mass * A.weight, vs) + energy64(B.mass * B.weight, vi);
                        atomicAdd(&st->chan_energy[S.model][ch], added);
                        ++nion;
                    });
                if (r.error) atomicOr(&st->error, r.error);
                atomicAdd(&st->candidates, (unsigned long long)r.candidates);
                if (r.nulls) atomicAdd(&st->nulls, (unsigned long long)r.nulls);
                ce.v[0] = vel[0]; ce.v[1] = vel[1]; ce.v[2] = vel[2];
            }
            __syncthreads();
        }
        // -- phase C: re-initialise, kick, drift, walls, deposit --
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            if (!keep[k]) continue;
            const float E = Ek[k];
            if (mcc) {
                if (queued[k] >= 0) {
                    const Cand32& ce = s_queue[queued[k]];
                    vc[k] = ce.v[0]; vy[k] = ce.v[1]; vz[k] = ce.v[2];
                }
                vh[k] = vc[k] - S.hqmdt32 * E;  // src/Simulation.cpp:924-926
            }
            if (mode & kModeKickDrift) {
                vh[k] = vh[k] + S.qmdt32 * E;  // src/Pusher.cpp:70-76, in cell units
                const float g = off[k] + vh[k] * S.dtdx32;
                if (!isfinite(g)) {  // flagged and dropped: deposits nothing
                    atomicOr(&st->error, kErrNonFinite);
                    keep[k] = false;
                    continue;
                }
                const float sh = floorf(g);
                int c = cell[k] + (int)fmaxf(fminf(sh, 1.0e9f), -1.0e9f);
                float o = g - sh;
                if (o >= 1.0f) { ++c; o = 0.0f; }
                if (!DIRICHLET) {
                    if (c >= nx || c < 0) c = ((c % nx) + nx) % nx;  // src/FieldSolver.cpp:15-17
                } else if (c < 0 || c > ncell || (c == ncell && o > 0.0f)) {
                    // absorbing walls and loss ledger, src/Simulation.cpp:1047-1077
                    const float w[3] = {vh[k], vy[k], vz[k]};
                    const double e = energy64(S.mass * S.weight, w);
                    const int side = c < 0 ? 0 : 1;
                    atomicAdd(&st->lost[s][side], 1ull);
                    atomicAdd(&st->lost_energy[s][side], e);
                    keep[k] = false;
                    continue;
                } else if (c == ncell) {
                    c = ncell - 1;  // x = L: the last cell at offset 1
                    o = 1.0f;
                }
                cell[k] = c;
                off[k] = o;
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
                atomicAdd(&sRho[i0], (unsigned long long)__float2ll_rn(q0));
                atomicAdd(&sRho[i1], (unsigned long long)__float2ll_rn(q1));
            }
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
        const unsigned lt = (1u << lane) - 1u;
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            if (!keep[k]) continue;
            const unsigned long long o = (unsigned long long)base + s_cnt[k * (kThreads / 32) + warp] +
                                         __popc(ballots[k] & lt);
            if (o >= S.capacity) { atomicOr(&st->error, kErrCapacity); continue; }
            __stcs(S.cell[1] + o, cell[k]);
            __stcs(S.off[1] + o, off[k]);
            __stcs(S.vh32[1] + o, vh[k]);
            if (VDIM == 3) {
                __stcs(S.vy32[1] + o, vy[k]);
                __stcs(S.vz32[1] + o, vz[k]);
            }
            if (mode & (kModeWriteV | kModeInitHalf)) S.v[o] = (double)vc[k];
        }
        __syncthreads();
    }
    if (mode & kModeDeposit) {
        for (int i = tid; i < nx; i += kThreads) {
            const unsigned long long a = sRho[i];
            if (a) atomicAdd(&p.rho_acc[i], a);
        }
    }
}
