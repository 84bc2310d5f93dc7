// Structured 2D3V / 3D3V periodic electrostatic PIC step on one B200 (FP64 form).
//
// Replaces Simulation2D::step / Simulation3D::step for fully periodic meshes
// (src/Simulation2D.cpp:1337-1364, src/Simulation3D.cpp:342-365) and what they
// call: interpolate_electric(Mesh2D&/Mesh3D&) (src/FieldSolver.cpp:926-1038),
// kick_boris / kick_leapfrog / drift_leapfrog (src/Pusher.cpp:82-186), the
// periodic particle boundaries (src/Simulation2D.cpp:57-97),
// deposit_charge_cic (src/Mesh2D.cpp:90-144, src/Mesh3D.cpp:62-126) and
// solve_periodic_spectral (src/FieldSolver.cpp:442-499, :659-731).
//
// One step: a push kernel per species (gather from an interleaved E grid,
// Boris or leapfrog kick, drift, periodic wrap, CIC deposit into a 64-bit
// fixed-point density with global atomics), then the spectral solve as line
// FFTs in shared memory: forward along x (reading and clearing the fixed-point
// density), [forward along y,] forward along the last axis fused with the
// k-space multiply and the first inverse transform, [inverse along y,] and an
// inverse along x that writes phi and the interleaved E field.  Particles are
// re-sorted by cell every `sort_interval` steps so gathers and atomics stay
// local.  Compiled with --fmad=false: particle arithmetic follows the
// reference operation by operation.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "apic_common.cuh"
#include "apic_rng.cuh"

namespace apic {
namespace nd {

constexpr int kThreads = 256;
constexpr int kMaxLine = 1024;

struct Cplx {
    double re, im;
};

struct SpeciesND {
    double qm;
    double dep;   // charge * weight (/ depth in 2D) times the inverse cell area/volume
    double hmw;   // 0.5 * mass * weight
    unsigned n;
    double* pos[2][3];
    double* vh[2][3];
    unsigned* id[2];
    double* v[3];
    // FP32 form: packed cell (10 bits per axis), in-cell offsets in [0, 1) and
    // float velocities; the FP64 arrays above then only stage loads/read-backs
    unsigned* cell[2];
    float* off[2][3];
    float* vel[2][3];
    float hqmdt;       // 0.5 * qm * dt
    float qmdt;        // qm * dt
    float tb[3], sb[3];  // Boris t = hqmdt B and s = 2 t / (1 + t^2)
    float drift[3];    // dt / d_a: cell units per unit velocity
    float dep_fixed;   // dep * rho_scale
    uint8_t* alive;    // runs with walls and an absorbing side: Particle::alive (null: all alive)
    int index;         // species index (loss ledger row)
};

struct ParamsND {
    int dims;
    int n[3];
    double L[3], d[3];
    double dt, eps;
    double B[3];
    double rho_scale, inv_rho_scale;
    const double* E;  // interleaved: 2 doubles per node (2D) or 4 (3D)
    const float* E32; // FP32 form: float copy of E
    unsigned long long* rho_acc;
    // magnetic_field_profile: B piecewise linear along prof_axis (prof_rows = 0: uniform B)
    int prof_axis, prof_rows;
    const double* prof_c;  // coordinates
    const double* prof_v;  // rows x 3
    // walls: Dirichlet axes, particle boundaries (left, right, bottom, top,
    // back, front: 0 periodic, 1 absorbing, 2 reflecting) and the absorbed
    // counts [species][6]
    int wall[3];
    int pbc[6];
    unsigned long long* losses;
};

// TabulatedVectorField1D::evaluate, src/PrescribedField.cpp:89-113, at coordinate
// q inside the table (create checks that the table covers the domain).
__device__ __forceinline__ void profile_b(const ParamsND& p, double q, double B[3]) {
    const double* c = p.prof_c;
    const int n = p.prof_rows;
    int right;
    if (q == __ldg(c)) {
        for (int a = 0; a < 3; ++a) B[a] = __ldg(p.prof_v + a);
        return;
    }
    if (q == __ldg(c + n - 1)) {
        for (int a = 0; a < 3; ++a) B[a] = __ldg(p.prof_v + 3 * (n - 1) + a);
        return;
    }
    int lo = 0, hi = n;  // std::upper_bound
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (q < __ldg(c + mid)) hi = mid; else lo = mid + 1;
    }
    right = lo;
    const int left = right - 1;
    const double f = (q - __ldg(c + left)) / (__ldg(c + right) - __ldg(c + left));
    for (int a = 0; a < 3; ++a) {
        const double l = __ldg(p.prof_v + 3 * left + a), r = __ldg(p.prof_v + 3 * right + a);
        B[a] = l + f * (r - l);
    }
}

// magnetic_field(cfg, position), src/Simulation2D.cpp:121-132, src/Simulation3D.cpp:109-118
__device__ __forceinline__ void field_b(const ParamsND& p, const double pos[3], double B[3]) {
    if (!p.prof_rows) {
        B[0] = p.B[0]; B[1] = p.B[1]; B[2] = p.B[2];
        return;
    }
    const int a = p.prof_axis;
    profile_b(p, a < p.dims ? (a == 0 ? pos[0] : (a == 1 ? pos[1] : pos[2])) : 0.0, B);
}

// FP32 form: each CIC weight is rounded to a multiple of 2^-23 and summed per
// species in 64-bit integers (runs of particles in one cell first add theirs in
// 32-bit registers and warp reductions: 8 particles per lane x 32 lanes x 2^23
// stays below 2^32), so the density does not depend on particle order.
constexpr float kWeightScale = 8388608.0f;  // 2^23

// wrap_periodic, src/FieldSolver.cpp:15-17, with the exact fast branch for |x| < 2L
__device__ __forceinline__ double wrap_periodic(double x, double L) {
    if (!(fabs(x) < 2.0 * L)) return fmod(fmod(x, L) + L, L);
    const double r = x >= L ? x - L : (x <= -L ? x + L : x);
    const double y = r + L;
    return y >= 2.0 * L ? 0.0 : (y >= L ? y - L : y);
}

struct Axis {
    int i0, i1;
    double f;
};

// One axis of the periodic CIC stencil, src/Mesh2D.cpp:96-114, src/FieldSolver.cpp:936-960
__device__ __forceinline__ Axis axis(double x, double L, double d, int n) {
    const double xp = wrap_periodic(x, L);
    const double g = xp / d;
    const unsigned long long i = (unsigned long long)floor(g);
    Axis a;
    a.f = g - (double)i;
    a.i0 = (int)(i % (unsigned long long)n);
    a.i1 = (int)((i + 1) % (unsigned long long)n);
    return a;
}

// One axis of the CIC stencil on a wall axis: clamp into [0, L], cell
// min(floor, n - 2), fraction clamped to [0, 1], src/Mesh2D.cpp:96-129,
// src/FieldSolver.cpp:926-960
__device__ __forceinline__ Axis axis_wall(double x, double L, double d, int n) {
    const double c = x < 0.0 ? 0.0 : (L < x ? L : x);
    const double g = c / d;
    unsigned long long i = (unsigned long long)floor(g);
    if (i > (unsigned long long)(n - 2)) i = (unsigned long long)(n - 2);
    double f = g - (double)i;
    f = f < 0.0 ? 0.0 : (f > 1.0 ? 1.0 : f);
    Axis a;
    a.i0 = (int)i;
    a.i1 = (int)i + 1;
    a.f = f;
    return a;
}

template <bool WALLS>
__device__ __forceinline__ Axis axis2(const ParamsND& p, int a, double x) {
    return (WALLS && p.wall[a]) ? axis_wall(x, p.L[a], p.d[a], p.n[a]) : axis(x, p.L[a], p.d[a], p.n[a]);
}

// 1 / node_area (node_volume) relative to an interior node: 2 on each
// wall-axis wall node (Mesh2D::node_area and Mesh3D::node_volume halve the
// cell there, src/Mesh2D.cpp:77-88, src/Mesh3D.cpp:52-60)
template <bool WALLS>
__device__ __forceinline__ double area_factor(const ParamsND& p, int a, int i) {
    return (WALLS && p.wall[a] && (i == 0 || i == p.n[a] - 1)) ? 2.0 : 1.0;
}

template <int DIM, bool WALLS = false>
__device__ __forceinline__ void gather(const ParamsND& p, const double pos[3], double e[3]) {
    const Axis ax = axis2<WALLS>(p, 0, pos[0]);
    const Axis ay = axis2<WALLS>(p, 1, pos[1]);
    const int nx = p.n[0];
    if (DIM == 2) {
        const double fx = ax.f, fy = ay.f;
        const double w00 = (1.0 - fx) * (1.0 - fy), w10 = fx * (1.0 - fy);
        const double w01 = (1.0 - fx) * fy, w11 = fx * fy;
        const double2* E2 = reinterpret_cast<const double2*>(p.E);
        const double2 e00 = __ldg(E2 + ay.i0 * nx + ax.i0), e10 = __ldg(E2 + ay.i0 * nx + ax.i1);
        const double2 e01 = __ldg(E2 + ay.i1 * nx + ax.i0), e11 = __ldg(E2 + ay.i1 * nx + ax.i1);
        e[0] = e00.x * w00 + e10.x * w10 + e01.x * w01 + e11.x * w11;
        e[1] = e00.y * w00 + e10.y * w10 + e01.y * w01 + e11.y * w11;
        e[2] = 0.0;
    } else {
        // interpolate_electric(Mesh3D&), src/FieldSolver.cpp:978-1038: loops z, y, x
        const Axis az = axis2<WALLS>(p, 2, pos[2]);
        const double wx[2] = {1.0 - ax.f, ax.f}, wy[2] = {1.0 - ay.f, ay.f}, wz[2] = {1.0 - az.f, az.f};
        const int ii[2] = {ax.i0, ax.i1}, jj[2] = {ay.i0, ay.i1}, kk[2] = {az.i0, az.i1};
        const double4* E4 = reinterpret_cast<const double4*>(p.E);
        e[0] = e[1] = e[2] = 0.0;
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int a = 0; a < 2; ++a) {
                    const double shape = wx[a] * wy[b] * wz[c];
                    const double4 ev = E4[((size_t)kk[c] * p.n[1] + jj[b]) * nx + ii[a]];
                    e[0] += ev.x * shape;
                    e[1] += ev.y * shape;
                    e[2] += ev.z * shape;
                }
    }
}

// boris_advance, src/Pusher.cpp:20-29
__device__ __forceinline__ void boris(double v[3], const double E[3], const double B[3], double qm, double dt) {
    const double h = 0.5 * qm * dt;
    const double vm0 = v[0] + h * E[0], vm1 = v[1] + h * E[1], vm2 = v[2] + h * E[2];
    const double t0 = h * B[0], t1 = h * B[1], t2v = h * B[2];
    const double t2 = t0 * t0 + t1 * t1 + t2v * t2v;
    const double sf = 2.0 / (1.0 + t2);
    const double s0 = sf * t0, s1 = sf * t1, s2 = sf * t2v;
    const double vp0 = vm0 + (vm1 * t2v - vm2 * t1);
    const double vp1 = vm1 + (vm2 * t0 - vm0 * t2v);
    const double vp2 = vm2 + (vm0 * t1 - vm1 * t0);
    const double vq0 = vm0 + (vp1 * s2 - vp2 * s1);
    const double vq1 = vm1 + (vp2 * s0 - vp0 * s2);
    const double vq2 = vm2 + (vp0 * s1 - vp1 * s0);
    v[0] = vq0 + h * E[0];
    v[1] = vq1 + h * E[1];
    v[2] = vq2 + h * E[2];
}

template <int DIM>
__device__ __forceinline__ void deposit(const ParamsND& p, const SpeciesND& S, const double pos[3]) {
    const Axis ax = axis(pos[0], p.L[0], p.d[0], p.n[0]);
    const Axis ay = axis(pos[1], p.L[1], p.d[1], p.n[1]);
    const int nx = p.n[0];
    if (DIM == 2) {
        // q (1 - fx)(1 - fy) / node_area, src/Mesh2D.cpp:131-142 (reciprocal area inside the fixed-point rounding)
        const double fx = ax.f, fy = ay.f;
        const double c00 = S.dep * (1.0 - fx) * (1.0 - fy), c10 = S.dep * fx * (1.0 - fy);
        const double c01 = S.dep * (1.0 - fx) * fy, c11 = S.dep * fx * fy;
        atomicAdd(p.rho_acc + ay.i0 * nx + ax.i0, (unsigned long long)to_fixed(c00, p.rho_scale));
        atomicAdd(p.rho_acc + ay.i0 * nx + ax.i1, (unsigned long long)to_fixed(c10, p.rho_scale));
        atomicAdd(p.rho_acc + ay.i1 * nx + ax.i0, (unsigned long long)to_fixed(c01, p.rho_scale));
        atomicAdd(p.rho_acc + ay.i1 * nx + ax.i1, (unsigned long long)to_fixed(c11, p.rho_scale));
    } else {
        // q_over_volume * shape, src/Mesh3D.cpp:110-122
        const Axis az = axis(pos[2], p.L[2], p.d[2], p.n[2]);
        const double wx[2] = {1.0 - ax.f, ax.f}, wy[2] = {1.0 - ay.f, ay.f}, wz[2] = {1.0 - az.f, az.f};
        const int ii[2] = {ax.i0, ax.i1}, jj[2] = {ay.i0, ay.i1}, kk[2] = {az.i0, az.i1};
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int a = 0; a < 2; ++a) {
                    const double shape = wx[a] * wy[b] * wz[c];
                    atomicAdd(p.rho_acc + ((size_t)kk[c] * p.n[1] + jj[b]) * nx + ii[a],
                              (unsigned long long)to_fixed(S.dep * shape, p.rho_scale));
                }
    }
}

// CIC deposit of a warp's particles with one atomic per node per run of lanes
// that share a cell: particles are sorted by cell, so neighbouring lanes mostly
// hit the same 2^DIM nodes.  Each lane's fixed-point contributions are summed
// over its run with a segmented shuffle scan (integer, so the total does not
// depend on the order), and the run's last lane commits them.  All 32 lanes
// must call this; `valid` marks lanes that carry a particle.
template <int DIM, bool WALLS = false>
__device__ __forceinline__ void deposit_warp(const ParamsND& p, const SpeciesND& S, const double pos[3], bool valid) {
    constexpr int K = DIM == 2 ? 4 : 8;
    const int lane = threadIdx.x & 31;
    long long a[K];
    size_t node[K];
    unsigned cell = 0xFFFFFFFFu;
    if (valid) {
        const Axis ax = axis2<WALLS>(p, 0, pos[0]);
        const Axis ay = axis2<WALLS>(p, 1, pos[1]);
        const int nx = p.n[0];
        if (DIM == 2 && WALLS) {
            // q shape / node_area over the wall nodes' half cells, src/Mesh2D.cpp:131-142
            const double fx = ax.f, fy = ay.f;
            const double x0 = area_factor<WALLS>(p, 0, ax.i0), x1 = area_factor<WALLS>(p, 0, ax.i1);
            const double y0 = area_factor<WALLS>(p, 1, ay.i0), y1 = area_factor<WALLS>(p, 1, ay.i1);
            a[0] = to_fixed(S.dep * (1.0 - fx) * (1.0 - fy) * (x0 * y0), p.rho_scale);
            a[1] = to_fixed(S.dep * fx * (1.0 - fy) * (x1 * y0), p.rho_scale);
            a[2] = to_fixed(S.dep * (1.0 - fx) * fy * (x0 * y1), p.rho_scale);
            a[3] = to_fixed(S.dep * fx * fy * (x1 * y1), p.rho_scale);
            node[0] = (size_t)ay.i0 * nx + ax.i0;
            node[1] = (size_t)ay.i0 * nx + ax.i1;
            node[2] = (size_t)ay.i1 * nx + ax.i0;
            node[3] = (size_t)ay.i1 * nx + ax.i1;
            cell = (unsigned)node[0];
        } else if (DIM == 2) {
            const double fx = ax.f, fy = ay.f;
            a[0] = to_fixed(S.dep * (1.0 - fx) * (1.0 - fy), p.rho_scale);
            a[1] = to_fixed(S.dep * fx * (1.0 - fy), p.rho_scale);
            a[2] = to_fixed(S.dep * (1.0 - fx) * fy, p.rho_scale);
            a[3] = to_fixed(S.dep * fx * fy, p.rho_scale);
            node[0] = (size_t)ay.i0 * nx + ax.i0;
            node[1] = (size_t)ay.i0 * nx + ax.i1;
            node[2] = (size_t)ay.i1 * nx + ax.i0;
            node[3] = (size_t)ay.i1 * nx + ax.i1;
            cell = (unsigned)node[0];
        } else {
            const Axis az = axis2<WALLS>(p, 2, pos[2]);
            const double wx[2] = {1.0 - ax.f, ax.f}, wy[2] = {1.0 - ay.f, ay.f}, wz[2] = {1.0 - az.f, az.f};
            const int ii[2] = {ax.i0, ax.i1}, jj[2] = {ay.i0, ay.i1}, kk[2] = {az.i0, az.i1};
#pragma unroll
            for (int c = 0; c < 2; ++c)
#pragma unroll
                for (int b = 0; b < 2; ++b)
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        const int k = (c * 2 + b) * 2 + q;
                        if (WALLS) {
                            // q shape / node_volume over the wall nodes' half cells, src/Mesh3D.cpp:110-122
                            const double f = area_factor<WALLS>(p, 0, ii[q]) * area_factor<WALLS>(p, 1, jj[b]) *
                                             area_factor<WALLS>(p, 2, kk[c]);
                            a[k] = to_fixed(S.dep * (wx[q] * wy[b] * wz[c]) * f, p.rho_scale);
                        } else {
                            a[k] = to_fixed(S.dep * (wx[q] * wy[b] * wz[c]), p.rho_scale);
                        }
                        node[k] = ((size_t)kk[c] * p.n[1] + jj[b]) * nx + ii[q];
                    }
            cell = (unsigned)node[0];
        }
    } else {
#pragma unroll
        for (int k = 0; k < K; ++k) { a[k] = 0; node[k] = 0; }
    }
    const unsigned up = __shfl_up_sync(0xffffffffu, cell, 1);
    const bool head = (lane & 7) == 0 || up != cell;  // runs capped at 8 lanes: three scan steps
    const unsigned heads = __ballot_sync(0xffffffffu, head);
    const int start = 31 - __clz(heads & (0xFFFFFFFFu >> (31 - lane)));
    const bool tail = lane == 31 || ((heads >> (lane + 1)) & 1u);
#pragma unroll
    for (int k = 0; k < K; ++k) {
        long long v = a[k];
#pragma unroll
        for (int d = 1; d < 8; d <<= 1) {
            const long long t = __shfl_up_sync(0xffffffffu, v, d);
            if (lane - d >= start) v += t;
        }
        if (tail && valid) atomicAdd(p.rho_acc + node[k], (unsigned long long)v);
    }
}

enum : int { kPushStep = 0, kPushDepositOnly = 1, kPushInitHalf = 2, kPushSync = 3 };

// One particle per thread.  Modes: a full step (kick, drift, wrap, deposit),
// deposit only (initialize/resume), half-step initialisation from v
// (initialize_{boris,leapfrog}_half_step) and synchronisation into v.
// reflect_coordinate, src/Simulation2D.cpp:43-54 (a particle crosses at most a
// few domain lengths per step; the bound only guards against runaway input)
__device__ __forceinline__ void reflect_coordinate(double& c, double& v, double L) {
    for (int guard = 0; guard < (1 << 20) && (c < 0.0 || c > L); ++guard) {
        if (c < 0.0) { c = -c; v = -v; }
        else { c = 2.0 * L - c; v = -v; }
    }
}

// Simulation2D::apply_particle_boundaries, src/Simulation2D.cpp:1309-1335, and
// Simulation3D::apply_particle_boundaries, src/Simulation3D.cpp:309-340, with
// apply_lower/upper_boundary (src/Simulation2D.cpp:57-97, src/Simulation3D.cpp:42-83):
// sides left, right, bottom, top (, back, front); returns the absorbing side, or -1.
template <int DIM>
__device__ __forceinline__ int apply_walls(const ParamsND& p, double x[3], double v[3]) {
#pragma unroll
    for (int side = 0; side < 2 * DIM; ++side) {
        const int a = side >> 1;
        double& c = x[a];
        const double L = p.L[a];
        if ((side & 1) == 0 ? c >= 0.0 : c <= L) continue;
        const int kind = p.pbc[side];
        if (kind == 1) return side;
        if (kind == 2) reflect_coordinate(c, v[a], L);
        else c = wrap_periodic(c, L);
    }
    return -1;
}

template <int DIM, bool BORIS, int MODE, bool WALLS = false>
__global__ void __launch_bounds__(kThreads) k_push(ParamsND p, SpeciesND S, int buf) {
    const unsigned i = blockIdx.x * kThreads + threadIdx.x;
    const bool valid = i < S.n && (!WALLS || !S.alive || S.alive[i]);
    if (MODE == kPushInitHalf || MODE == kPushSync) {
        if (!valid) return;
    } else if (blockIdx.x * kThreads + (threadIdx.x & ~31u) >= S.n) {
        return;  // whole warp past the end
    }
    const unsigned j = valid ? i : 0u;
    double pos[3] = {S.pos[buf][0][j], S.pos[buf][1][j], DIM == 3 ? S.pos[buf][2][j] : 0.0};
    if (MODE == kPushDepositOnly) {
        deposit_warp<DIM, WALLS>(p, S, pos, valid);
        return;
    }
    double e[3];
    gather<DIM, WALLS>(p, pos, e);
    if (MODE == kPushInitHalf) {
        double v[3] = {S.v[0][i], S.v[1][i], S.v[2][i]};
        if (BORIS) {
            double Bp[3];
            field_b(p, pos, Bp);
            boris(v, e, Bp, S.qm, -0.5 * p.dt);
        } else {
            // initialize_leapfrog_half_step, src/Pusher.cpp:88-92, :152-156
            for (int a = 0; a < DIM; ++a) v[a] = v[a] - 0.5 * S.qm * e[a] * p.dt;
        }
        for (int a = 0; a < 3; ++a) S.vh[buf][a][i] = v[a];
        return;
    }
    double vh[3] = {S.vh[buf][0][j], S.vh[buf][1][j], S.vh[buf][2][j]};
    if (MODE == kPushSync) {
        if (BORIS) {
            double Bp[3];
            field_b(p, pos, Bp);
            boris(vh, e, Bp, S.qm, 0.5 * p.dt);
        } else {
            // synchronize_leapfrog, src/Pusher.cpp:131-135, :176-180
            for (int a = 0; a < DIM; ++a) vh[a] = vh[a] + 0.5 * S.qm * e[a] * p.dt;
        }
        for (int a = 0; a < 3; ++a) S.v[a][i] = vh[a];
        return;
    }
    // kick_boris / kick_leapfrog + drift_leapfrog, src/Pusher.cpp:109-128, :162-174
    if (BORIS) {
        double Bp[3];
        field_b(p, pos, Bp);
        boris(vh, e, Bp, S.qm, p.dt);
    } else {
        for (int a = 0; a < DIM; ++a) vh[a] += S.qm * e[a] * p.dt;
    }
    bool absorbed = false;
    if (WALLS) {
        for (int a = 0; a < DIM; ++a) pos[a] = pos[a] + vh[a] * p.dt;
        const int side = valid ? apply_walls<DIM>(p, pos, vh) : -1;
        if (side >= 0) {
            absorbed = true;
            S.alive[i] = 0;
            atomicAdd(p.losses + 6 * S.index + side, 1ull);
        }
    } else {
        for (int a = 0; a < DIM; ++a) {
            const double c = pos[a] + vh[a] * p.dt;
            // periodic particle boundary: wrap only outside [0, L], src/Simulation2D.cpp:57-97
            pos[a] = (c >= 0.0 && c <= p.L[a]) ? c : wrap_periodic(c, p.L[a]);
        }
    }
    if (valid) {
        for (int a = 0; a < DIM; ++a) S.pos[buf][a][i] = pos[a];
        for (int a = 0; a < 3; ++a) S.vh[buf][a][i] = vh[a];
    }
    deposit_warp<DIM, WALLS>(p, S, pos, valid && !absorbed);
}

// walls: fixed-point density to FP64 (the accumulator is cleared for the
// next deposit)
__global__ void k_walls_rho(unsigned long long* __restrict__ acc, double* __restrict__ rho, size_t N,
                            double inv_scale) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        rho[i] = (double)(long long)acc[i] * inv_scale;
        acc[i] = 0ull;
    }
}

// 3D walls: the field planes (Ex | Ey | Ez) into the interleaved layout of the push
__global__ void k_walls_interleave3(const double* __restrict__ planes, double4* __restrict__ E, size_t N) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x)
        E[i] = make_double4(planes[i], planes[N + i], planes[2 * N + i], 0.0);
}

// 2D walls: the field planes (Ex | Ey) into the interleaved layout of the push
__global__ void k_walls_interleave(const double* __restrict__ planes, double* __restrict__ E, size_t N) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        E[2 * i] = planes[i];
        E[2 * i + 1] = planes[N + i];
    }
}

// ---- FP32 particle form ---------------------------------------------------------
//
// A particle is a packed cell index (10 bits per axis), float offsets in
// [0, 1) inside that cell and float velocities: 24 B (2D3V) or 28 B (3D3V) of
// state instead of 40/48 B.  Positions never leave cell units, so the gather and
// the deposit need no division and no wrap; the field solve, the fixed-point
// density and the diagnostics stay FP64.

__device__ __forceinline__ void unpack_cell(unsigned c, int& ix, int& iy, int& iz) {
    ix = (int)(c & 1023u);
    iy = (int)((c >> 10) & 1023u);
    iz = (int)(c >> 20);
}
__device__ __forceinline__ unsigned pack_cell(int ix, int iy, int iz) {
    return (unsigned)ix | ((unsigned)iy << 10) | ((unsigned)iz << 20);
}

template <int DIM>
__device__ __forceinline__ void gather32(const ParamsND& p, int ix, int iy, int iz, const float f[3], float e[3]) {
    const int nx = p.n[0], ny = p.n[1];
    const int ix1 = (ix + 1) & (nx - 1), iy1 = (iy + 1) & (ny - 1);
    const float wx[2] = {1.0f - f[0], f[0]}, wy[2] = {1.0f - f[1], f[1]};
    if (DIM == 2) {
        const float2* E = reinterpret_cast<const float2*>(p.E32);
        const float2 a = __ldg(E + iy * nx + ix), b = __ldg(E + iy * nx + ix1), c = __ldg(E + iy1 * nx + ix),
                     d = __ldg(E + iy1 * nx + ix1);
        const float w00 = wx[0] * wy[0], w10 = wx[1] * wy[0], w01 = wx[0] * wy[1], w11 = wx[1] * wy[1];
        e[0] = fmaf(a.x, w00, fmaf(b.x, w10, fmaf(c.x, w01, d.x * w11)));
        e[1] = fmaf(a.y, w00, fmaf(b.y, w10, fmaf(c.y, w01, d.y * w11)));
        e[2] = 0.0f;
    } else {
        const int iz1 = (iz + 1) & (p.n[2] - 1);
        const float wz[2] = {1.0f - f[2], f[2]};
        const int xx[2] = {ix, ix1}, yy[2] = {iy, iy1}, zz[2] = {iz, iz1};
        const float4* E = reinterpret_cast<const float4*>(p.E32);
        e[0] = e[1] = e[2] = 0.0f;
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                const float wyz = wy[b] * wz[c];
                const size_t row = ((size_t)zz[c] * ny + yy[b]) * nx;
#pragma unroll
                for (int a = 0; a < 2; ++a) {
                    const float w = wx[a] * wyz;
                    const float4 v = __ldg(E + row + xx[a]);
                    e[0] = fmaf(v.x, w, e[0]);
                    e[1] = fmaf(v.y, w, e[1]);
                    e[2] = fmaf(v.z, w, e[2]);
                }
            }
    }
}

// Boris rotation in float (same algebra as boris_advance, src/Pusher.cpp:20-29)
__device__ __forceinline__ void boris32(float v[3], const float e[3], float h, const float t[3], const float s[3]) {
    const float vm0 = fmaf(h, e[0], v[0]), vm1 = fmaf(h, e[1], v[1]), vm2 = fmaf(h, e[2], v[2]);
    const float vp0 = vm0 + fmaf(vm1, t[2], -vm2 * t[1]);
    const float vp1 = vm1 + fmaf(vm2, t[0], -vm0 * t[2]);
    const float vp2 = vm2 + fmaf(vm0, t[1], -vm1 * t[0]);
    v[0] = fmaf(h, e[0], vm0 + fmaf(vp1, s[2], -vp2 * s[1]));
    v[1] = fmaf(h, e[1], vm1 + fmaf(vp2, s[0], -vp0 * s[2]));
    v[2] = fmaf(h, e[2], vm2 + fmaf(vp0, s[1], -vp1 * s[0]));
}

// FP32 form: the Boris rotation vectors t = (q/m dt/2) B and s = 2 t / (1 + t^2)
// of a particle, from its cell and offset when B is tabulated (the species'
// precomputed pair otherwise), in the same FP64 expression as the species' pair.
__device__ __forceinline__ void boris_ts32(const ParamsND& p, const SpeciesND& S, int ix, int iy, int iz,
                                           const float f[3], float tb[3], float sb[3]) {
    if (!p.prof_rows) {
        for (int a = 0; a < 3; ++a) { tb[a] = S.tb[a]; sb[a] = S.sb[a]; }
        return;
    }
    const int a = p.prof_axis;
    double q = 0.0;
    if (a < p.dims) {
        const int cell = a == 0 ? ix : (a == 1 ? iy : iz);
        const float off = a == 0 ? f[0] : (a == 1 ? f[1] : f[2]);
        q = ((double)cell + (double)off) * p.d[a];
    }
    double B[3];
    profile_b(p, q, B);
    const double hq = 0.5 * S.qm * p.dt;
    double t2 = 0.0;
    for (int c = 0; c < 3; ++c) t2 += (hq * B[c]) * (hq * B[c]);
    for (int c = 0; c < 3; ++c) {
        tb[c] = (float)(hq * B[c]);
        sb[c] = (float)(2.0 * hq * B[c] / (1.0 + t2));
    }
}

// Moves one axis by `disp` cells: integer carry into the periodic cell index.
__device__ __forceinline__ void advance(float& f, int& i, float disp, int n) {
    float g = f + disp;
    const float k = floorf(g);
    g -= k;
    int ki = (int)k;
    if (g >= 1.0f) { g -= 1.0f; ki += 1; }
    f = g;
    i = (i + ki) & (n - 1);
}

// Runs of lanes that share a cell (particles are sorted by cell) add their
// 2^-25-quantised weights with a converged segmented shuffle scan; runs are
// capped at SEG lanes (32 x 2^25 < 2^32, so a run's sum fits 32 bits): SEG = 32
// where a warp usually sits in one or two cells (2D, 64 particles per cell),
// 8 where it spans several (3D).  The last lane of each run commits its sums
// with one 64-bit atomic per node.
template <int DIM>
__device__ __forceinline__ void deposit32_warp(const ParamsND& p, unsigned long long* acc, bool valid, int ix, int iy,
                                               int iz, const float f[3]) {
    constexpr int SEG = DIM == 2 ? 32 : 8;
    const int lane = threadIdx.x & 31;
    const int nx = p.n[0], ny = p.n[1];
    const unsigned key = valid ? (((unsigned)iz * ny + iy) * nx + ix) : 0xFFFFFFFFu;
    const unsigned prev = __shfl_up_sync(0xffffffffu, key, 1);
    const bool head = (lane & (SEG - 1)) == 0 || prev != key;
    const unsigned heads = __ballot_sync(0xffffffffu, head);
    const int start = 31 - __clz(heads & (0xFFFFFFFFu >> (31 - lane)));
    const bool tail = lane == 31 || ((heads >> (lane + 1)) & 1u);
    const int ix1 = (ix + 1) & (nx - 1), iy1 = (iy + 1) & (ny - 1);
    const int iz1 = DIM == 3 ? (iz + 1) & (p.n[2] - 1) : 0;
    const int xx[2] = {ix, ix1}, yy[2] = {iy, iy1}, zz[2] = {iz, iz1};
    const float wx[2] = {1.0f - f[0], f[0]}, wy[2] = {1.0f - f[1], f[1]};
    const float wz[2] = {DIM == 3 ? 1.0f - f[2] : 1.0f, DIM == 3 ? f[2] : 0.0f};
#pragma unroll
    for (int c = 0; c < (DIM == 3 ? 2 : 1); ++c)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                unsigned q = valid ? (unsigned)__float2int_rn(wx[a] * wy[b] * wz[c] * kWeightScale) : 0u;
#pragma unroll
                for (int d = 1; d < SEG; d <<= 1) {
                    const unsigned t = __shfl_up_sync(0xffffffffu, q, d);
                    if (lane - d >= start) q += t;
                }
                if (tail && valid && q)
                    atomicAdd(acc + ((size_t)zz[c] * ny + yy[b]) * nx + xx[a], (unsigned long long)q);
            }
}

template <int DIM, bool BORIS, int MODE>
__global__ void __launch_bounds__(kThreads) k_push32(ParamsND p, SpeciesND S, int buf, unsigned long long* acc) {
    const unsigned i = blockIdx.x * kThreads + threadIdx.x;
    const bool valid = i < S.n;
    if ((MODE == kPushStep || MODE == kPushDepositOnly) && blockIdx.x * kThreads + (threadIdx.x & ~31u) >= S.n)
        return;  // whole warp past the end
    int ix = 0, iy = 0, iz = 0;
    float f[3] = {0.0f, 0.0f, 0.0f}, v[3] = {0.0f, 0.0f, 0.0f};
    if (valid) {  // streamed once per step: evict-first, so L1 keeps the field
        unpack_cell(__ldcs(&S.cell[buf][i]), ix, iy, iz);
        for (int a = 0; a < DIM; ++a) f[a] = __ldcs(&S.off[buf][a][i]);
        for (int a = 0; a < 3; ++a) v[a] = __ldcs(&S.vel[buf][a][i]);
    }
    if (MODE == kPushStep || MODE == kPushInitHalf || MODE == kPushSync) {
        float e[3] = {0.0f, 0.0f, 0.0f};
        if (valid) gather32<DIM>(p, ix, iy, iz, f, e);
        if (MODE == kPushInitHalf || MODE == kPushSync) {
            if (!valid) return;
            float w[3] = {(float)S.v[0][i], (float)S.v[1][i], (float)S.v[2][i]};
            float* vv = MODE == kPushInitHalf ? w : v;
            const float h = MODE == kPushInitHalf ? -0.5f * S.hqmdt : 0.5f * S.hqmdt;
            if (BORIS) {
                float t[3], sb[3], tp[3], sp[3];
                boris_ts32(p, S, ix, iy, iz, f, tp, sp);
                float t2 = 0.0f;
                for (int a = 0; a < 3; ++a) { t[a] = tp[a] * (MODE == kPushInitHalf ? -0.5f : 0.5f); t2 = fmaf(t[a], t[a], t2); }
                for (int a = 0; a < 3; ++a) sb[a] = 2.0f * t[a] / (1.0f + t2);
                boris32(vv, e, h, t, sb);
            } else {
                for (int a = 0; a < DIM; ++a) vv[a] = fmaf(2.0f * h, e[a], vv[a]);
            }
            if (MODE == kPushInitHalf) {
                for (int a = 0; a < 3; ++a) S.vel[buf][a][i] = vv[a];
            } else {
                for (int a = 0; a < 3; ++a) S.v[a][i] = (double)vv[a];
            }
            return;
        }
        // kick + drift
        if (BORIS) {
            float tp[3], sp[3];
            boris_ts32(p, S, ix, iy, iz, f, tp, sp);
            boris32(v, e, S.hqmdt, tp, sp);
        } else {
            for (int a = 0; a < DIM; ++a) v[a] = fmaf(S.qmdt, e[a], v[a]);
        }
        int* idx[3] = {&ix, &iy, &iz};
        for (int a = 0; a < DIM; ++a) advance(f[a], *idx[a], v[a] * S.drift[a], p.n[a]);
        if (valid) {
            __stcs(&S.cell[buf][i], pack_cell(ix, iy, iz));
            for (int a = 0; a < DIM; ++a) __stcs(&S.off[buf][a][i], f[a]);
            for (int a = 0; a < 3; ++a) __stcs(&S.vel[buf][a][i], v[a]);
        }
    }
    // ---- deposit ----
    deposit32_warp<DIM>(p, acc, valid, ix, iy, iz, f);
}

// The step push of the FP32 form with ITEMS particles per thread: all of the
// thread's particle loads are issued before the first gather, so each warp
// keeps ITEMS times the bytes in flight (the single-particle form leaves HBM
// latency-bound).  Slice k of the CTA is the contiguous block of kThreads
// particles at base + k * kThreads, so each warp still deposits runs of
// consecutive (cell-sorted) particles.
// PROF: B tabulated along one axis (a separate instantiation, so the uniform-B
// kernels keep their register budget).
template <int DIM, bool BORIS, int ITEMS, bool PROF>
__global__ void __launch_bounds__(kThreads) k_push32_step(ParamsND p, SpeciesND S, int buf, unsigned long long* acc) {
    const unsigned base = blockIdx.x * (ITEMS * kThreads);
    const unsigned tid = threadIdx.x;
    unsigned cl[ITEMS];
    float fo[ITEMS][3], vv[ITEMS][3];
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        const unsigned i = base + k * kThreads + tid;
        const bool ok = i < S.n;
        cl[k] = ok ? __ldcs(&S.cell[buf][i]) : 0u;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            fo[k][a] = (ok && a < DIM) ? __ldcs(&S.off[buf][a][i]) : 0.0f;
            vv[k][a] = ok ? __ldcs(&S.vel[buf][a][i]) : 0.0f;
        }
    }
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        const unsigned i = base + k * kThreads + tid;
        if (base + k * kThreads + (tid & ~31u) >= S.n) continue;  // whole warp past the end
        const bool valid = i < S.n;
        int ix = 0, iy = 0, iz = 0;
        unpack_cell(cl[k], ix, iy, iz);
        float* f = fo[k];
        float* v = vv[k];
        float e[3] = {0.0f, 0.0f, 0.0f};
        if (valid) gather32<DIM>(p, ix, iy, iz, f, e);
        // kick + drift, src/Pusher.cpp:109-128, :162-174
        if (BORIS && PROF) {
            float tp[3], sp[3];
            boris_ts32(p, S, ix, iy, iz, f, tp, sp);
            boris32(v, e, S.hqmdt, tp, sp);
        } else if (BORIS) {
            boris32(v, e, S.hqmdt, S.tb, S.sb);
        } else {
            for (int a = 0; a < DIM; ++a) v[a] = fmaf(S.qmdt, e[a], v[a]);
        }
        int* idx[3] = {&ix, &iy, &iz};
        for (int a = 0; a < DIM; ++a) advance(f[a], *idx[a], v[a] * S.drift[a], p.n[a]);
        if (valid) {
            __stcs(&S.cell[buf][i], pack_cell(ix, iy, iz));
            for (int a = 0; a < DIM; ++a) __stcs(&S.off[buf][a][i], f[a]);
            for (int a = 0; a < 3; ++a) __stcs(&S.vel[buf][a][i], v[a]);
        }
        deposit32_warp<DIM>(p, acc, valid, ix, iy, iz, f);
    }
}

// The step push of the FP32 form with ITEMS consecutive particles per thread
// (loaded and stored as vectors).  Particles are sorted by cell, so a thread's
// particles mostly share a cell: the field at the cell's nodes is fetched once
// per run of equal cells, and the CIC weights of a run are summed in registers
// (the deposit of src/Mesh2D.cpp:90-144 / src/Mesh3D.cpp:62-126 at the pushed
// positions).  A run that ends inside the thread is committed with one 64-bit
// atomic per node; each lane's last run joins a warp-segmented sum over the
// lanes holding the same cell, whose last lane commits it.
// 2D: the CTA's deposit into a box of nodes in shared memory (kDBoxX cells
// along x from x0 and the cell rows y0 .. y0 + 2 around the CTA's middle
// particle), flushed with one 64-bit global atomic per touched node: a
// particle that left its sorted neighbours then adds into shared memory
// instead of committing its own global atomics (which, on the few nodes a CTA
// touches, serialise in L2).  Each node's weight sum is kept as two 32-bit
// halves (native shared atomics; the low half adds at most 2^16 per commit and
// the high half 2^14, so neither overflows for the CTA's particles) and
// reassembled exactly.  Commits outside the box go to global memory as before.
// (In 3D the box around a CTA's 64 cells needs 1552 nodes; zeroing and
// flushing them and the kernel's extra registers cost more than the atomics
// saved, so 3D commits straight to global memory.)
constexpr int kDBoxX = 48;
constexpr int kDBoxNodes = (kDBoxX + 1) * 4;
struct DepositBox {
    unsigned* lo;
    unsigned* hi;
    int x0, y0;
};

template <int DIM, bool BORIS, int ITEMS, bool PROF>
__device__ __forceinline__ void push_run(const ParamsND& p, const SpeciesND& S, int buf, unsigned long long* acc,
                                         const DepositBox& box) {
    constexpr int NN = DIM == 2 ? 4 : 8;  // nodes of a cell
    const unsigned first = (blockIdx.x * kThreads + threadIdx.x) * ITEMS;
    const int lane = threadIdx.x & 31;
    if ((blockIdx.x * kThreads + (threadIdx.x & ~31u)) * ITEMS >= S.n) return;  // whole warp past the end
    const int nx = p.n[0], ny = p.n[1], nz = DIM == 3 ? p.n[2] : 1;
    unsigned cl[ITEMS];
    float fo[ITEMS][3], vv[ITEMS][3];
    const bool full = first + ITEMS <= S.n;
    if (full) {
        if (ITEMS == 4) {
            const uint4 c = __ldcs(reinterpret_cast<const uint4*>(S.cell[buf] + first));
            cl[0] = c.x; cl[1] = c.y; cl[2 % ITEMS] = c.z; cl[3 % ITEMS] = c.w;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (a < DIM) {
                    const float4 f = __ldcs(reinterpret_cast<const float4*>(S.off[buf][a] + first));
                    fo[0][a] = f.x; fo[1][a] = f.y; fo[2 % ITEMS][a] = f.z; fo[3 % ITEMS][a] = f.w;
                } else {
#pragma unroll
                    for (int k = 0; k < ITEMS; ++k) fo[k][a] = 0.0f;
                }
                const float4 v = __ldcs(reinterpret_cast<const float4*>(S.vel[buf][a] + first));
                vv[0][a] = v.x; vv[1][a] = v.y; vv[2 % ITEMS][a] = v.z; vv[3 % ITEMS][a] = v.w;
            }
        } else {
            const uint2 c = __ldcs(reinterpret_cast<const uint2*>(S.cell[buf] + first));
            cl[0] = c.x; cl[1 % ITEMS] = c.y;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (a < DIM) {
                    const float2 f = __ldcs(reinterpret_cast<const float2*>(S.off[buf][a] + first));
                    fo[0][a] = f.x; fo[1 % ITEMS][a] = f.y;
                } else {
                    fo[0][a] = 0.0f; fo[1 % ITEMS][a] = 0.0f;
                }
                const float2 v = __ldcs(reinterpret_cast<const float2*>(S.vel[buf][a] + first));
                vv[0][a] = v.x; vv[1 % ITEMS][a] = v.y;
            }
        }
    } else {
#pragma unroll
        for (int k = 0; k < ITEMS; ++k) {
            const unsigned i = first + k;
            const bool ok = i < S.n;
            cl[k] = ok ? S.cell[buf][i] : 0u;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                fo[k][a] = (ok && a < DIM) ? S.off[buf][a][i] : 0.0f;
                vv[k][a] = ok ? S.vel[buf][a][i] : 0.0f;
            }
        }
    }
    const unsigned kNoCell = 0xFFFFFFFFu;
    // 3D: the field lines of each later new cell in the thread's run are
    // prefetched into L1 before the first push: a cell change inside the run
    // then finds them there instead of waiting a whole L2 round trip between
    // two pushes (no registers are held for them).  The 2D field (8 B a node)
    // mostly sits in L1 already; prefetching it measured within noise.
#pragma unroll
    for (int k = 1; k < ITEMS; ++k) {
        if (DIM == 2 || first + k >= S.n || cl[k] == cl[k - 1]) continue;
        int ix, iy, iz;
        unpack_cell(cl[k], ix, iy, iz);
        const int iy1 = (iy + 1) & (ny - 1);
        {
            const int iz1 = (iz + 1) & (nz - 1);
            const float4* E = reinterpret_cast<const float4*>(p.E32);
            asm volatile("prefetch.global.L1 [%0];" ::"l"(E + ((size_t)iz * ny + iy) * nx + ix));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(E + ((size_t)iz * ny + iy1) * nx + ix));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(E + ((size_t)iz1 * ny + iy) * nx + ix));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(E + ((size_t)iz1 * ny + iy1) * nx + ix));
        }
    }
    unsigned gcell = kNoCell;   // cell whose node fields are cached
    float en[NN][3];            // the field at its nodes
    unsigned rcell = kNoCell;   // cell of the current deposit run
    unsigned racc[NN];          // its summed quantised weights
#pragma unroll
    for (int j = 0; j < NN; ++j) racc[j] = 0u;
    auto commit = [&](unsigned c, const unsigned* w) {
        int ix, iy, iz;
        unpack_cell(c, ix, iy, iz);
        if (DIM == 2) {
            const int bx = (ix - box.x0) & (nx - 1), by = (iy - box.y0) & (ny - 1);
            if (bx < kDBoxX && by < 3) {
                const int b = by * (kDBoxX + 1) + bx;
#pragma unroll
                for (int j = 0; j < NN; ++j) {
                    if (!w[j]) continue;
                    const int q = b + (j & 1) + ((j >> 1) & 1) * (kDBoxX + 1);
                    atomicAdd(box.lo + q, w[j] & 0xFFFFu);
                    atomicAdd(box.hi + q, w[j] >> 16);
                }
                return;
            }
        }
        const int ix1 = (ix + 1) & (nx - 1), iy1 = (iy + 1) & (ny - 1);
        const int iz1 = DIM == 3 ? (iz + 1) & (nz - 1) : 0;
#pragma unroll
        for (int j = 0; j < NN; ++j) {
            if (!w[j]) continue;
            const int xx = (j & 1) ? ix1 : ix, yy = (j & 2) ? iy1 : iy, zz = (j & 4) ? iz1 : iz;
            atomicAdd(acc + ((size_t)zz * ny + yy) * nx + xx, (unsigned long long)w[j]);
        }
    };
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        if (first + k >= S.n) continue;
        int ix, iy, iz;
        unpack_cell(cl[k], ix, iy, iz);
        float* f = fo[k];
        float* v = vv[k];
        if (cl[k] != gcell) {  // the field at the new cell's nodes
            gcell = cl[k];
            const int ix1 = (ix + 1) & (nx - 1), iy1 = (iy + 1) & (ny - 1);
            if (DIM == 2) {
                const float2* E = reinterpret_cast<const float2*>(p.E32);
                const float2 a = __ldg(E + iy * nx + ix), b = __ldg(E + iy * nx + ix1),
                             c = __ldg(E + iy1 * nx + ix), d = __ldg(E + iy1 * nx + ix1);
                en[0][0] = a.x; en[0][1] = a.y; en[1][0] = b.x; en[1][1] = b.y;
                en[2][0] = c.x; en[2][1] = c.y; en[3][0] = d.x; en[3][1] = d.y;
#pragma unroll
                for (int j = 0; j < NN; ++j) en[j][2] = 0.0f;
            } else {
                const int iz1 = (iz + 1) & (nz - 1);
                const float4* E = reinterpret_cast<const float4*>(p.E32);
#pragma unroll
                for (int j = 0; j < NN; ++j) {
                    const int xx = (j & 1) ? ix1 : ix, yy = (j & 2) ? iy1 : iy, zz = (j & 4) ? iz1 : iz;
                    const float4 q = __ldg(E + ((size_t)zz * ny + yy) * nx + xx);
                    en[j][0] = q.x; en[j][1] = q.y; en[j][2] = q.z;
                }
            }
        }
        // bilinear / trilinear gather, src/FieldSolver.cpp:925-1038 (the
        // arithmetic of gather32, so every particles-per-thread choice gives
        // the same bits)
        const float wx[2] = {1.0f - f[0], f[0]}, wy[2] = {1.0f - f[1], f[1]};
        float e[3] = {0.0f, 0.0f, 0.0f};
        if (DIM == 2) {
            const float w00 = wx[0] * wy[0], w10 = wx[1] * wy[0], w01 = wx[0] * wy[1], w11 = wx[1] * wy[1];
            e[0] = fmaf(en[0][0], w00, fmaf(en[1][0], w10, fmaf(en[2][0], w01, en[3][0] * w11)));
            e[1] = fmaf(en[0][1], w00, fmaf(en[1][1], w10, fmaf(en[2][1], w01, en[3][1] * w11)));
        } else {
            const float wz[2] = {1.0f - f[2], f[2]};
#pragma unroll
            for (int j = 0; j < NN; ++j) {
                const float w = wx[j & 1] * (wy[(j >> 1) & 1] * wz[(j >> 2) & 1]);
                e[0] = fmaf(en[j][0], w, e[0]);
                e[1] = fmaf(en[j][1], w, e[1]);
                e[2] = fmaf(en[j][2], w, e[2]);
            }
        }
        // kick + drift, src/Pusher.cpp:109-128, :162-174
        if (BORIS && PROF) {
            float tp[3], sp[3];
            boris_ts32(p, S, ix, iy, iz, f, tp, sp);
            boris32(v, e, S.hqmdt, tp, sp);
        } else if (BORIS) {
            boris32(v, e, S.hqmdt, S.tb, S.sb);
        } else {
            for (int a = 0; a < DIM; ++a) v[a] = fmaf(S.qmdt, e[a], v[a]);
        }
        advance(f[0], ix, v[0] * S.drift[0], nx);
        advance(f[1], iy, v[1] * S.drift[1], ny);
        if (DIM == 3) advance(f[2], iz, v[2] * S.drift[2], nz);
        cl[k] = pack_cell(ix, iy, iz);
        // deposit at the pushed position into the run of its cell
        if (cl[k] != rcell) {
            if (rcell != kNoCell) commit(rcell, racc);
            rcell = cl[k];
#pragma unroll
            for (int j = 0; j < NN; ++j) racc[j] = 0u;
        }
        const float ux[2] = {1.0f - f[0], f[0]}, uy[2] = {1.0f - f[1], f[1]};
        const float uz[2] = {DIM == 3 ? 1.0f - f[2] : 1.0f, DIM == 3 ? f[2] : 0.0f};
#pragma unroll
        for (int j = 0; j < NN; ++j)
            racc[j] += (unsigned)__float2int_rn(ux[j & 1] * uy[(j >> 1) & 1] * uz[(j >> 2) & 1] * kWeightScale);
    }
    // the state back, in place
    if (full) {
        if (ITEMS == 4) {
            __stcs(reinterpret_cast<uint4*>(S.cell[buf] + first), make_uint4(cl[0], cl[1], cl[2 % ITEMS], cl[3 % ITEMS]));
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (a < DIM)
                    __stcs(reinterpret_cast<float4*>(S.off[buf][a] + first),
                           make_float4(fo[0][a], fo[1][a], fo[2 % ITEMS][a], fo[3 % ITEMS][a]));
                __stcs(reinterpret_cast<float4*>(S.vel[buf][a] + first),
                       make_float4(vv[0][a], vv[1][a], vv[2 % ITEMS][a], vv[3 % ITEMS][a]));
            }
        } else {
            __stcs(reinterpret_cast<uint2*>(S.cell[buf] + first), make_uint2(cl[0], cl[1 % ITEMS]));
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (a < DIM)
                    __stcs(reinterpret_cast<float2*>(S.off[buf][a] + first), make_float2(fo[0][a], fo[1 % ITEMS][a]));
                __stcs(reinterpret_cast<float2*>(S.vel[buf][a] + first), make_float2(vv[0][a], vv[1 % ITEMS][a]));
            }
        }
    } else {
#pragma unroll
        for (int k = 0; k < ITEMS; ++k) {
            const unsigned i = first + k;
            if (i >= S.n) continue;
            S.cell[buf][i] = cl[k];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (a < DIM) S.off[buf][a][i] = fo[k][a];
                S.vel[buf][a][i] = vv[k][a];
            }
        }
    }
    // each lane's last run: summed over the lanes that end in the same cell
    // segments of at most 4 lanes in 3D (a cell's run spans about 4 lanes at 8
    // particles per cell) and 8 in 2D: two or three shuffle steps instead of
    // five per node, for a few more commits; measured 5.89 -> 5.69 ms per
    // 256^3 step and 0.371 -> 0.368 ms per 512^2 step
    constexpr int RSEG = DIM == 3 ? 4 : 8;
    const unsigned key = rcell;
    const unsigned prev = __shfl_up_sync(0xffffffffu, key, 1);
    const bool head = (lane & (RSEG - 1)) == 0 || prev != key;
    const unsigned heads = __ballot_sync(0xffffffffu, head);
    const int start = 31 - __clz(heads & (0xFFFFFFFFu >> (31 - lane)));
    const bool tail = lane == 31 || ((heads >> (lane + 1)) & 1u);
#pragma unroll
    for (int j = 0; j < NN; ++j) {
        unsigned q = racc[j];
#pragma unroll
        for (int d = 1; d < RSEG; d <<= 1) {
            const unsigned t = __shfl_up_sync(0xffffffffu, q, d);
            if (lane - d >= start) q += t;
        }
        racc[j] = q;
    }
    if (tail && key != kNoCell) commit(key, racc);
}

template <int DIM, bool BORIS, int ITEMS, bool PROF>
__global__ void __launch_bounds__(kThreads) k_push32_run(ParamsND p, SpeciesND S, int buf, unsigned long long* acc) {
    if constexpr (DIM == 2) {
        __shared__ unsigned s_lo[kDBoxNodes], s_hi[kDBoxNodes];
        __shared__ int s_anchor[2];
        const int nx = p.n[0], ny = p.n[1];
        if (threadIdx.x == 0) {  // the box around the CTA's middle particle, before the push
            const unsigned mid = min(blockIdx.x * kThreads * ITEMS + (unsigned)(kThreads * ITEMS / 2), S.n - 1u);
            int ix, iy, iz;
            unpack_cell(S.cell[buf][mid], ix, iy, iz);
            s_anchor[0] = (ix - kDBoxX / 2) & (nx - 1);
            s_anchor[1] = (iy - 1) & (ny - 1);
        }
        for (int q = threadIdx.x; q < kDBoxNodes; q += kThreads) { s_lo[q] = 0u; s_hi[q] = 0u; }
        __syncthreads();
        const DepositBox box{s_lo, s_hi, s_anchor[0], s_anchor[1]};
        push_run<DIM, BORIS, ITEMS, PROF>(p, S, buf, acc, box);
        __syncthreads();
        for (int q = threadIdx.x; q < kDBoxNodes; q += kThreads) {
            const unsigned long long v = ((unsigned long long)s_hi[q] << 16) + s_lo[q];
            if (!v) continue;
            const int qx = q % (kDBoxX + 1), qy = q / (kDBoxX + 1);
            atomicAdd(acc + (size_t)((box.y0 + qy) & (ny - 1)) * nx + ((box.x0 + qx) & (nx - 1)), v);
        }
    } else {
        push_run<DIM, BORIS, ITEMS, PROF>(p, S, buf, acc, DepositBox{nullptr, nullptr, 0, 0});
    }
}

// FP64 staging <-> FP32 state.  The cell/offset split follows the periodic CIC
// index of the reference (wrap, divide by the cell size, floor).
template <int DIM>
__global__ void k_to_fp32(ParamsND p, SpeciesND S, int buf) {
    const unsigned i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= S.n) return;
    int ii[3] = {0, 0, 0};
    for (int a = 0; a < DIM; ++a) {
        const Axis ax = axis(S.pos[buf][a][i], p.L[a], p.d[a], p.n[a]);
        float f = (float)ax.f;
        int k = ax.i0;
        if (f >= 1.0f) { f = 0.0f; k = ax.i1; }
        ii[a] = k;
        S.off[buf][a][i] = f;
    }
    S.cell[buf][i] = pack_cell(ii[0], ii[1], ii[2]);
    for (int a = 0; a < 3; ++a) S.vel[buf][a][i] = (float)S.vh[buf][a][i];
}

template <int DIM>
__global__ void k_to_fp64(ParamsND p, SpeciesND S, int buf) {
    const unsigned i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= S.n) return;
    int ii[3];
    unpack_cell(S.cell[buf][i], ii[0], ii[1], ii[2]);
    for (int a = 0; a < DIM; ++a) S.pos[buf][a][i] = ((double)ii[a] + (double)S.off[buf][a][i]) * p.d[a];
    for (int a = 0; a < 3; ++a) S.vh[buf][a][i] = (double)S.vel[buf][a][i];
}

__device__ __forceinline__ unsigned linear_cell(const ParamsND& p, unsigned c) {
    int x, y, z;
    unpack_cell(c, x, y, z);
    return ((unsigned)z * p.n[1] + y) * p.n[0] + x;
}

// Lanes of a warp that share a cell (particles are nearly sorted, so a warp
// spans few cells) take one atomic per cell: the group's leader adds the
// group's size and the lanes take consecutive slots in lane order.
__global__ void k_cell_hist32(ParamsND p, SpeciesND S, int buf, unsigned* count) {
    const unsigned i = blockIdx.x * kThreads + threadIdx.x;
    const bool valid = i < S.n;
    const unsigned key = valid ? linear_cell(p, S.cell[buf][i]) : 0xFFFFFFFFu;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    if (valid && (int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(count + key, (unsigned)__popc(peers));
}

// Counting-sort placement of the FP32 form in two passes.  k_cell_rank32 gives
// each particle its slot (lanes of a warp that share a cell take one atomic per
// cell: the group's leader adds the group's size and the lanes take
// consecutive slots in lane order) and records the particle's index there, in
// the id array of the target buffer; k_cell_gather32 then fills every slot
// from that index.  The stores of the second pass are coalesced, and the
// scattered accesses are reads, served mostly from L2 (a particle moves a few
// cells between sorts); a direct scatter instead writes a partial sector per
// field for every particle that changed its row or plane.
__global__ void k_cell_rank32(ParamsND p, SpeciesND S, int from, unsigned* cursor) {
    const unsigned i = blockIdx.x * kThreads + threadIdx.x;
    const bool valid = i < S.n;
    const unsigned key = valid ? linear_cell(p, __ldcs(S.cell[from] + i)) : 0xFFFFFFFFu;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
    unsigned base = 0;
    if (valid && lane == leader) base = atomicAdd(cursor + key, (unsigned)__popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (!valid) return;
    S.id[from ^ 1][base + (unsigned)__popc(peers & ((1u << lane) - 1u))] = i;
}

template <int DIM>
__global__ void k_cell_gather32(SpeciesND S, int from) {
    const unsigned d = blockIdx.x * kThreads + threadIdx.x;
    if (d >= S.n) return;
    const int to = from ^ 1;
    const unsigned i = S.id[to][d];
    const unsigned c = S.cell[from][i], id = S.id[from][i];
    float off[3], vel[3];
#pragma unroll
    for (int a = 0; a < DIM; ++a) off[a] = S.off[from][a][i];
#pragma unroll
    for (int a = 0; a < 3; ++a) vel[a] = S.vel[from][a][i];
    __stcs(S.cell[to] + d, c);
#pragma unroll
    for (int a = 0; a < DIM; ++a) __stcs(S.off[to][a] + d, off[a]);
#pragma unroll
    for (int a = 0; a < 3; ++a) __stcs(S.vel[to][a] + d, vel[a]);
    __stcs(S.id[to] + d, id);
}

// ---- particle sort by cell -------------------------------------------------------

template <int DIM>
__device__ __forceinline__ unsigned cell_of(const ParamsND& p, const double pos[3]) {
    const Axis ax = axis(pos[0], p.L[0], p.d[0], p.n[0]);
    const Axis ay = axis(pos[1], p.L[1], p.d[1], p.n[1]);
    unsigned c = (unsigned)ay.i0 * p.n[0] + ax.i0;
    if (DIM == 3) {
        const Axis az = axis(pos[2], p.L[2], p.d[2], p.n[2]);
        c += (unsigned)az.i0 * p.n[0] * p.n[1];
    }
    return c;
}

template <int DIM>
__global__ void k_cell_hist(ParamsND p, SpeciesND S, int buf, unsigned* count) {
    const unsigned i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= S.n) return;
    const double pos[3] = {S.pos[buf][0][i], S.pos[buf][1][i], DIM == 3 ? S.pos[buf][2][i] : 0.0};
    atomicAdd(count + cell_of<DIM>(p, pos), 1u);
}

// exclusive scan of `count` (n entries) into `offset`, three launches
constexpr int kScanItems = 8;
constexpr int kScanBlock = kThreads * kScanItems;
__global__ void k_scan_local(const unsigned* count, unsigned* offset, unsigned* block_sums, unsigned n) {
    __shared__ unsigned s[kThreads];
    const unsigned base = blockIdx.x * kScanBlock + threadIdx.x * kScanItems;
    unsigned v[kScanItems], sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? count[base + k] : 0u;
        sum += v[k];
    }
    s[threadIdx.x] = sum;
    __syncthreads();
    for (int o = 1; o < kThreads; o <<= 1) {
        const unsigned y = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0u;
        __syncthreads();
        s[threadIdx.x] += y;
        __syncthreads();
    }
    unsigned run = s[threadIdx.x] - sum;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) offset[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == kThreads - 1) block_sums[blockIdx.x] = s[threadIdx.x];
}

__global__ void k_scan_blocks(unsigned* block_sums, unsigned nblocks) {
    // one CTA: exclusive scan in place (nblocks <= kThreads * kScanItems * kThreads handled by a loop)
    __shared__ unsigned s[kThreads];
    __shared__ unsigned carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (unsigned b0 = 0; b0 < nblocks; b0 += kThreads) {
        const unsigned i = b0 + threadIdx.x;
        const unsigned v = i < nblocks ? block_sums[i] : 0u;
        s[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < kThreads; o <<= 1) {
            const unsigned y = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0u;
            __syncthreads();
            s[threadIdx.x] += y;
            __syncthreads();
        }
        const unsigned c = carry;
        if (i < nblocks) block_sums[i] = c + s[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == kThreads - 1) carry = c + s[threadIdx.x];
        __syncthreads();
    }
}

__global__ void k_scan_add(unsigned* offset, const unsigned* block_sums, unsigned n) {
    const unsigned base = blockIdx.x * kScanBlock;
    const unsigned add = block_sums[blockIdx.x];
    for (unsigned k = threadIdx.x; k < (unsigned)kScanBlock; k += kThreads)
        if (base + k < n) offset[base + k] += add;
}

template <int DIM>
__global__ void k_cell_scatter(ParamsND p, SpeciesND S, int from, unsigned* cursor) {
    const unsigned i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= S.n) return;
    const int to = from ^ 1;
    // loads first, stores after: the buffers may alias as far as the compiler
    // knows, so loads placed after stores would each wait for the previous store
    const double pos[3] = {S.pos[from][0][i], S.pos[from][1][i], DIM == 3 ? S.pos[from][2][i] : 0.0};
    const double vh[3] = {S.vh[from][0][i], S.vh[from][1][i], S.vh[from][2][i]};
    const unsigned id = S.id[from][i];
    const unsigned o = atomicAdd(cursor + cell_of<DIM>(p, pos), 1u);
    for (int a = 0; a < DIM; ++a) S.pos[to][a][o] = pos[a];
    for (int a = 0; a < 3; ++a) S.vh[to][a][o] = vh[a];
    S.id[to][o] = id;
}

// Device-side loading for large runs: uniform positions displaced by
// amp/k sin(k x) along `mode_axis` (amp = 0: none) and Maxwellian velocities
// with thermal speed vt and x drift, from a Philox stream per particle
// (Box-Muller on 53-bit uniforms).
__global__ void k_load_maxwellian(SpeciesND S, int buf, int dims, unsigned n, uint64_t seed, double L0, double L1,
                                  double L2, double vt, double drift, int mode_axis, double amp) {
    const unsigned i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    uint32_t r[4], r2[4];
    philox4x32_10(i, 0x5eedu, 0u, 0u, (uint32_t)seed, (uint32_t)(seed >> 32), r);
    philox4x32_10(i, 0x5eedu, 1u, 0u, (uint32_t)seed, (uint32_t)(seed >> 32), r2);
    auto u53 = [](uint32_t a, uint32_t b) {
        return ((double)(((uint64_t)a << 21) ^ (uint64_t)b & 0x1FFFFFull) + 0.5) * 0x1.0p-53;
    };
    const double L[3] = {L0, L1, L2};
    const double u[3] = {u53(r[0], r[1]), u53(r[2], r[3]), u53(r2[0], r2[1])};
    for (int a = 0; a < dims; ++a) {
        double x = u[a] * L[a];
        if (amp != 0.0 && (mode_axis < 0 || a == mode_axis)) {
            const double k = 2.0 * 3.141592653589793 / L[a];
            x = x + amp / k * sin(k * x);
            x = fmod(fmod(x, L[a]) + L[a], L[a]);
        }
        S.pos[buf][a][i] = x;
    }
    uint32_t g1[4], g2[4];
    philox4x32_10(i, 0x5eedu, 2u, 0u, (uint32_t)seed, (uint32_t)(seed >> 32), g1);
    philox4x32_10(i, 0x5eedu, 3u, 0u, (uint32_t)seed, (uint32_t)(seed >> 32), g2);
    const double a1 = u53(g1[0], g1[1]), b1 = u53(g1[2], g1[3]), a2 = u53(g2[0], g2[1]), b2 = u53(g2[2], g2[3]);
    const double r1 = sqrt(-2.0 * log(a1)), r2v = sqrt(-2.0 * log(a2));
    const double twopi = 2.0 * 3.141592653589793;
    const double nv[3] = {r1 * cos(twopi * b1), r1 * sin(twopi * b1), r2v * cos(twopi * b2)};
    for (int a = 0; a < 3; ++a) {
        const double v = vt * nv[a] + (a == 0 ? drift : 0.0);
        S.v[a][i] = v;
        S.vh[buf][a][i] = v;
    }
    S.id[buf][i] = i;
}

// Read-back in load order: dst[id[i]] = src[i].
__global__ void k_unpermute(const unsigned* id, const double* src, double* dst, unsigned n) {
    const unsigned i = blockIdx.x * kThreads + threadIdx.x;
    if (i < n) dst[id[i]] = src[i];
}

// ---- spectral Poisson solve: line FFTs in shared memory -----------------------------

enum : int { kFwdFromRho = 0, kFwdInPlace = 1, kFwdMulInv = 2, kInvInPlace = 3, kInvToFields = 4 };
constexpr int kFftThreads = 256;             // threads per FFT tile
constexpr size_t kFftTileBytes = 100 * 1024;  // shared-memory budget of one tile (lines per tile follow)
// Largest dynamic shared memory of an FFT tile: four line buffers plus the
// twiddles fit the tile budget whenever a tile holds more than one line, and a
// single 1024-point line takes 4 x 16 KB + 16 KB.
constexpr size_t kFftSmemMax = kFftTileBytes > 5 * 1024 * 16 ? kFftTileBytes : 5 * 1024 * 16;

struct FftPass {
    int n, log2n;
    int log2T;              // log2 of T (every extent and T are powers of two)
    long long es, ls;       // element stride, stride between the tile's lines
    int T;                  // lines per tile
    long long tiles_inner;  // tiles per outer slab
    long long outer_stride;
    const Cplx* tw;         // exp(-2 pi i k / n), k < n/2
    int axis;               // axis of the lines (0, 1, 2)
};

struct FieldsND {
    int dims, nx, ny, nz;
    int lnx, lny;  // log2 nx, log2 ny (power-of-two extents)
    double L[3], eps, inv_scale, pack;  // pack: power of two that balances phi and E in one complex array
    unsigned long long* rho_acc;
    const double* rho_in;  // when set, the forward pass reads FP64 rho instead of the accumulator
    double* rho;
    Cplx* W;
    Cplx* A;
    Cplx* B;
    double* phi;
    double* E;
    float* E32;  // FP32 form: interleaved float copy of E (2 or 4 floats per node)
    const double* kvec[3];  // wavenumbers 2 pi m / L per axis and index (m the signed mode), or null
    int nacc;    // FP32 form: per-species weight accumulators
    unsigned long long* acc[APIC_MAX_SPECIES];
    double acc_scale[APIC_MAX_SPECIES];  // charge density per accumulator unit
};

__device__ __forceinline__ unsigned bitrev(unsigned x, int bits) { return __brev(x) >> (32 - bits); }

// W16^k = exp(-2 pi i k / 16): cos and sin of 2 pi k / 16, k < 16.
__device__ __forceinline__ double c16(int k) {
    constexpr double a = 0.92387953251128675613, b = 0.70710678118654752440, c = 0.38268343236508977173;
    switch (k & 15) {
        case 0: return 1.0;  case 1: return a;   case 2: return b;   case 3: return c;
        case 4: return 0.0;  case 5: return -c;  case 6: return -b;  case 7: return -a;
        case 8: return -1.0; case 9: return -a;  case 10: return -b; case 11: return -c;
        case 12: return 0.0; case 13: return c;  case 14: return b;  default: return a;
    }
}
__device__ __forceinline__ double s16(int k) { return c16(k + 12); }  // sin x = cos(x - pi/2)

__device__ __forceinline__ Cplx cadd(Cplx x, Cplx y) { return {x.re + y.re, x.im + y.im}; }
__device__ __forceinline__ Cplx csub(Cplx x, Cplx y) { return {x.re - y.re, x.im - y.im}; }
// x * W16^k (forward) or x * conj(W16^k) (inverse)
__device__ __forceinline__ Cplx cw16(Cplx x, int k, bool inv) {
    const double wr = c16(k), wi = inv ? s16(k) : -s16(k);
    return {x.re * wr - x.im * wi, x.re * wi + x.im * wr};
}

template <int R>
__device__ __forceinline__ void dft_small(Cplx* a, bool inv);

template <>
__device__ __forceinline__ void dft_small<2>(Cplx* a, bool) {
    const Cplx t = a[0];
    a[0] = cadd(t, a[1]);
    a[1] = csub(t, a[1]);
}

template <>
__device__ __forceinline__ void dft_small<4>(Cplx* a, bool inv) {
    const Cplx t0 = cadd(a[0], a[2]), t1 = csub(a[0], a[2]), t2 = cadd(a[1], a[3]);
    const Cplx d = csub(a[1], a[3]);
    const Cplx t3 = inv ? Cplx{-d.im, d.re} : Cplx{d.im, -d.re};  // (+i) d or (-i) d
    a[0] = cadd(t0, t2);
    a[2] = csub(t0, t2);
    a[1] = cadd(t1, t3);
    a[3] = csub(t1, t3);
}

// R = R1 R2 point DFT from two smaller ones (index m = R2 m1 + m2 in, p = p1 + R1 p2 out).
template <int R1, int R2>
__device__ __forceinline__ void dft_split(Cplx* a, bool inv) {
    constexpr int R = R1 * R2;
    Cplx b[R2][R1];
#pragma unroll
    for (int m2 = 0; m2 < R2; ++m2) {
        Cplx t[R1];
#pragma unroll
        for (int m1 = 0; m1 < R1; ++m1) t[m1] = a[R2 * m1 + m2];
        dft_small<R1>(t, inv);
#pragma unroll
        for (int p1 = 0; p1 < R1; ++p1) b[m2][p1] = (p1 * m2 == 0) ? t[p1] : cw16(t[p1], p1 * m2 * (16 / R), inv);
    }
#pragma unroll
    for (int p1 = 0; p1 < R1; ++p1) {
        Cplx t[R2];
#pragma unroll
        for (int m2 = 0; m2 < R2; ++m2) t[m2] = b[m2][p1];
        dft_small<R2>(t, inv);
#pragma unroll
        for (int p2 = 0; p2 < R2; ++p2) a[p1 + R1 * p2] = t[p2];
    }
}

template <>
__device__ __forceinline__ void dft_small<8>(Cplx* a, bool inv) { dft_split<4, 2>(a, inv); }
template <>
__device__ __forceinline__ void dft_small<16>(Cplx* a, bool inv) { dft_split<4, 4>(a, inv); }

template <int R>
__device__ __forceinline__ void dft_reg(Cplx (&a)[R], bool inv) { dft_small<R>(a, inv); }

// One Stockham radix-R stage over `lines` lines of n points (src -> dst):
// butterfly j reads src[j + m n/R], twiddles by w^(k m) with k = j mod L and
// w = exp(-2 pi i / (L R)), and writes dst[(j - k) R + k + p L].
template <int R>
__device__ void stockham_stage(const Cplx* __restrict__ src, Cplx* __restrict__ dst, int lines, int n, int L,
                               const Cplx* tw, bool inv) {
    const int nb = n / R;  // a power of two
    const int lnb = __ffs(nb) - 1;
    const int tstep = n / (L * R);
    for (int b = threadIdx.x; b < lines * nb; b += blockDim.x) {
        const int l = b >> lnb, j = b & (nb - 1);
        const int k = j & (L - 1);
        const Cplx* s = src + l * n;
        Cplx a[R];
#pragma unroll
        for (int m = 0; m < R; ++m) a[m] = s[j + m * nb];
        if (L > 1) {
#pragma unroll
            for (int m = 1; m < R; ++m) {
                Cplx w = tw[k * m * tstep];
                if (inv) w.im = -w.im;
                const Cplx x = a[m];
                a[m] = {x.re * w.re - x.im * w.im, x.re * w.im + x.im * w.re};
            }
        }
        dft_reg<R>(a, inv);
        Cplx* d = dst + l * n;
        const int o = (j - k) * R + k;
#pragma unroll
        for (int p = 0; p < R; ++p) d[o + p * L] = a[p];
    }
    __syncthreads();
}

// Transforms `lines` lines held in buf0 (buf1 is scratch of the same size);
// returns the buffer that holds the result.  Forward uses exp(-2 pi i k/n),
// inverse the conjugate and a 1/n scale per line, as fft_radix2 does
// (src/FieldSolver.cpp:171-201); the twiddles are exact table values.
__device__ Cplx* fft_lines(Cplx* buf0, Cplx* buf1, int lines, int n, const Cplx* tw, bool inv) {
    Cplx* src = buf0;
    Cplx* dst = buf1;
    int L = 1, rem = n;
    while (rem > 1) {
        if (rem % 16 == 0) { stockham_stage<16>(src, dst, lines, n, L, tw, inv); L *= 16; rem /= 16; }
        else if (rem % 8 == 0) { stockham_stage<8>(src, dst, lines, n, L, tw, inv); L *= 8; rem /= 8; }
        else if (rem % 4 == 0) { stockham_stage<4>(src, dst, lines, n, L, tw, inv); L *= 4; rem /= 4; }
        else { stockham_stage<2>(src, dst, lines, n, L, tw, inv); L *= 2; rem /= 2; }
        Cplx* t = src; src = dst; dst = t;
    }
    if (inv) {
        const double sc = 1.0 / (double)n;
        for (int b = threadIdx.x; b < lines * n; b += blockDim.x) {
            src[b].re *= sc;
            src[b].im *= sc;
        }
        __syncthreads();
    }
    return src;
}

__device__ __forceinline__ long long tile_base(const FftPass& f, long long tile) {
    return (tile % f.tiles_inner) * f.T * f.ls + (tile / f.tiles_inner) * f.outer_stride;
}

// element b of the tile: (line l, element e) so that consecutive b are consecutive in memory
__device__ __forceinline__ void tile_elem(const FftPass& f, int b, int& l, int& e) {
    if (f.es == 1) { l = b >> f.log2n; e = b & (f.n - 1); }
    else { e = b >> f.log2T; l = b & (f.T - 1); }
}

// Forward input at node g: the species' fixed-point densities summed (or the
// FP64 rho of a stand-alone solve); the accumulators are cleared and rho kept.
__device__ __forceinline__ double density_at(const FieldsND& F, long long g) {
    double r;
    if (F.rho_in) {
        r = F.rho_in[g];
    } else if (F.nacc) {
        unsigned long long q[APIC_MAX_SPECIES] = {0, 0, 0, 0};
#pragma unroll
        for (int k = 0; k < APIC_MAX_SPECIES; ++k)
            if (k < F.nacc) q[k] = F.acc[k][g];
        r = 0.0;
#pragma unroll
        for (int k = 0; k < APIC_MAX_SPECIES; ++k)
            if (k < F.nacc) {
                r += (double)(long long)q[k] * F.acc_scale[k];
                F.acc[k][g] = 0ull;
            }
    } else {
        r = (double)(long long)F.rho_acc[g] * F.inv_scale;
        F.rho_acc[g] = 0ull;
    }
    F.rho[g] = r;
    return r;
}

// k-space multiply at node g (src/FieldSolver.cpp:470-488, :687-712) into two
// packed spectra A = phi_k + i Ex_k / pack, B = Ey_k / pack + i Ez_k / pack,
// each E component restricted to its Hermitian part (zero on its own Nyquist
// plane) so that both inverse transforms are real pairs
__device__ __forceinline__ void kspace_at(const FieldsND& F, long long g, Cplx r, Cplx& a, Cplx& bb) {
    const double twopi = 2.0 * 3.141592653589793;
    const double ip = 1.0 / F.pack;
    const int ix = (int)(g & (F.nx - 1));
    const int iy = (int)((g >> F.lnx) & (F.ny - 1));
    const int iz = F.dims == 3 ? (int)(g >> (F.lnx + F.lny)) : 0;
    a = {0.0, 0.0};
    bb = {0.0, 0.0};
    if (ix != 0 || iy != 0 || iz != 0) {
        const double mx = ix <= F.nx / 2 ? (double)ix : -(double)(F.nx - ix);
        const double my = iy <= F.ny / 2 ? (double)iy : -(double)(F.ny - iy);
        const double kx = twopi * mx / F.L[0];
        const double ky = twopi * my / F.L[1];
        double kz = 0.0, k2;
        if (F.dims == 3) {
            const double mz = iz <= F.nz / 2 ? (double)iz : -(double)(F.nz - iz);
            kz = twopi * mz / F.L[2];
            k2 = kx * kx + ky * ky + kz * kz;
        } else {
            k2 = kx * kx + ky * ky;
        }
        const double den = F.eps * k2;
        const double pr = r.re / den, pi = r.im / den;
        // -(0,1) k phik = (k pi, -(k pr))
        const bool nyx = (F.nx % 2 == 0) && ix == F.nx / 2;
        const bool nyy = (F.ny % 2 == 0) && iy == F.ny / 2;
        const bool nyz = F.dims == 3 && (F.nz % 2 == 0) && iz == F.nz / 2;
        const double exr = nyx ? 0.0 : kx * pi, exi = nyx ? 0.0 : -(kx * pr);
        const double eyr = nyy ? 0.0 : ky * pi, eyi = nyy ? 0.0 : -(ky * pr);
        const double ezr = nyz ? 0.0 : kz * pi, ezi = nyz ? 0.0 : -(kz * pr);
        a = {pr - exi * ip, pi + exr * ip};
        bb = {eyr * ip - ezi * ip, eyi * ip + ezr * ip};
    }
}

// kspace_at with the wavenumbers read from the per-axis tables (the same
// values, computed on the host) and one correctly rounded reciprocal of
// eps k^2 in place of two divisions
__device__ __forceinline__ void kspace_tab(const FieldsND& F, long long g, Cplx r, Cplx& a, Cplx& bb) {
    const double ip = 1.0 / F.pack;
    const int ix = (int)(g & (F.nx - 1));
    const int iy = (int)((g >> F.lnx) & (F.ny - 1));
    const int iz = F.dims == 3 ? (int)(g >> (F.lnx + F.lny)) : 0;
    a = {0.0, 0.0};
    bb = {0.0, 0.0};
    if (ix != 0 || iy != 0 || iz != 0) {
        const double kx = __ldg(F.kvec[0] + ix), ky = __ldg(F.kvec[1] + iy);
        const double kz = F.dims == 3 ? __ldg(F.kvec[2] + iz) : 0.0;
        const double k2 = F.dims == 3 ? kx * kx + ky * ky + kz * kz : kx * kx + ky * ky;
        const double inv = __drcp_rn(F.eps * k2);
        const double pr = r.re * inv, pi = r.im * inv;
        const bool nyx = ix == F.nx / 2, nyy = iy == F.ny / 2, nyz = F.dims == 3 && iz == F.nz / 2;
        const double exr = nyx ? 0.0 : kx * pi, exi = nyx ? 0.0 : -(kx * pr);
        const double eyr = nyy ? 0.0 : ky * pi, eyi = nyy ? 0.0 : -(ky * pr);
        const double ezr = nyz ? 0.0 : kz * pi, ezi = nyz ? 0.0 : -(kz * pr);
        a = {pr - exi * ip, pi + exr * ip};
        bb = {eyr * ip - ezi * ip, eyi * ip + ezr * ip};
    }
}

// phi and E at node g from the inverse transforms of the packed spectra
__device__ __forceinline__ void store_fields(const FieldsND& F, long long g, Cplx a, Cplx bb) {
    F.phi[g] = a.re;
    if (F.dims == 2) {
        reinterpret_cast<double2*>(F.E)[g] = make_double2(a.im * F.pack, bb.re * F.pack);
        if (F.E32) reinterpret_cast<float2*>(F.E32)[g] = make_float2((float)(a.im * F.pack), (float)(bb.re * F.pack));
    } else {
        reinterpret_cast<double4*>(F.E)[g] = make_double4(a.im * F.pack, bb.re * F.pack, bb.im * F.pack, 0.0);
        if (F.E32)
            reinterpret_cast<float4*>(F.E32)[g] =
                make_float4((float)(a.im * F.pack), (float)(bb.re * F.pack), (float)(bb.im * F.pack), 0.0f);
    }
}

template <int MODE>
__global__ void __launch_bounds__(kFftThreads) k_fft(FieldsND F, FftPass f) {
    extern __shared__ __align__(16) unsigned char fsm[];
    // shared memory: region0 (2 T lines) and region1 (2 T lines), then the
    // n twiddles; a single array ping-pongs inside region0, an (A, B) pair
    // occupies 2 T lines and ping-pongs between the two regions
    const int ld = f.n;
    Cplx* R0 = reinterpret_cast<Cplx*>(fsm);
    Cplx* R1 = R0 + 2 * f.T * ld;
    Cplx* tws = R1 + ((MODE == kFwdFromRho || MODE == kFwdInPlace) ? 0 : 2 * f.T * ld);
    for (int k = threadIdx.x; k < f.n; k += blockDim.x) tws[k] = f.tw[k];
    Cplx* X = R0;
    Cplx* Y = R0 + f.T * ld;  // B lines of a pair, right after the A lines
    const long long base = tile_base(f, blockIdx.x);
    const int total = f.T * f.n;
    // ---- load (bit-reversed within each line) ----
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
        int l, e;
        tile_elem(f, b, l, e);
        const long long g = base + l * f.ls + e * f.es;
        const int s = l * ld + e;
        if (MODE == kFwdFromRho) {
            X[s] = {density_at(F, g), 0.0};
        } else if (MODE == kFwdInPlace || MODE == kFwdMulInv) {
            X[s] = F.W[g];
        } else {
            X[s] = F.A[g];
            Y[s] = F.B[g];
        }
    }
    __syncthreads();
    const bool inverse_first = (MODE == kInvInPlace || MODE == kInvToFields);
    Cplx* res;
    if (inverse_first) res = fft_lines(R0, R1, 2 * f.T, f.n, tws, true);           // A and B together
    else res = fft_lines(X, X + f.T * ld, f.T, f.n, tws, false);                    // ping-pong inside region0
    X = res;
    Y = res + f.T * ld;
    if (MODE == kFwdMulInv) {
        for (int b = threadIdx.x; b < total; b += blockDim.x) {
            int l, e;
            tile_elem(f, b, l, e);
            const long long g = base + l * f.ls + e * f.es;
            Cplx a, bb;
            kspace_at(F, g, X[l * ld + e], a, bb);
            const int s = l * ld + e;
            R1[s] = a;
            R1[f.T * ld + s] = bb;
        }
        __syncthreads();
        Cplx* pair = fft_lines(R1, R0, 2 * f.T, f.n, tws, true);
        X = pair;
        Y = pair + f.T * ld;
    }
    // ---- store ----
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
        int l, e;
        tile_elem(f, b, l, e);
        const long long g = base + l * f.ls + e * f.es;
        const int s = l * ld + e;
        if (MODE == kFwdFromRho || MODE == kFwdInPlace) {
            F.W[g] = X[s];
        } else if (MODE == kFwdMulInv) {
            F.A[g] = X[s];
            F.B[g] = Y[s];
        } else if (MODE == kInvInPlace) {
            F.A[g] = X[s];
            F.B[g] = Y[s];
        } else {
            store_fields(F, g, X[s], Y[s]);
        }
    }
}

// ---- 256-point lines: a four-step FFT in registers ---------------------------------
//
// Lines of 256 = 16 x 16 points, eight lines per CTA and 16 threads per line.
// Thread slot s of a line holds the points s + 16 j (j < 16) in registers:
// a 16-point DFT over j, the twiddles W256^(s k1), one exchange through shared
// memory (thread s then holds column k1 = s), a second 16-point DFT, and the
// thread holds the transform at s + 16 k2, the same positions it loaded, so a
// pass reads and writes each element once and in place.  Lanes run along the
// line on the x pass (16 consecutive points per half warp) and across the
// tile's lines on the strided y / z passes (8 consecutive lines, 128 B), so
// every global access moves whole 128-256 B segments; the registers hold the
// loads in flight (16 or 32 per thread) instead of a shared-memory tile.
constexpr int kF256Lines = 8;
constexpr int kF256Threads = kF256Lines * 16;

template <bool XP>
__device__ __forceinline__ void f256_map(int tid, int& l, int& s) {
    if (XP) { s = tid & 15; l = tid >> 4; }
    else { l = tid & (kF256Lines - 1); s = tid >> 3; }
}

// exchange slot of (line l, row r, column c): written by slot c as row r,
// read by slot r as column c; conflict-free for both lane layouts
template <bool XP>
__device__ __forceinline__ int f256_xi(int l, int r, int c) {
    return XP ? (l * 16 + r) * 17 + c : (r * 16 + c) * kF256Lines + l;
}
template <bool XP>
constexpr int f256_xsize() { return XP ? kF256Lines * 16 * 17 : kF256Lines * 256; }

// forward (inv = false) or inverse transforms of NA lines held as a[k][16]
template <bool XP, int NA>
__device__ __forceinline__ void fft256(Cplx (&a)[NA][16], Cplx* xb, const Cplx* tws, int l, int s, bool inv) {
#pragma unroll
    for (int k = 0; k < NA; ++k) {
        dft_small<16>(a[k], inv);
#pragma unroll
        for (int k1 = 1; k1 < 16; ++k1) {
            Cplx w = tws[(s * k1) & 255];
            if (inv) w.im = -w.im;
            const Cplx x = a[k][k1];
            a[k][k1] = {x.re * w.re - x.im * w.im, x.re * w.im + x.im * w.re};
        }
    }
    __syncthreads();  // earlier readers of the exchange buffers are done
#pragma unroll
    for (int k = 0; k < NA; ++k)
#pragma unroll
        for (int k1 = 0; k1 < 16; ++k1) xb[k * f256_xsize<XP>() + f256_xi<XP>(l, k1, s)] = a[k][k1];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NA; ++k) {
#pragma unroll
        for (int t = 0; t < 16; ++t) a[k][t] = xb[k * f256_xsize<XP>() + f256_xi<XP>(l, s, t)];
        dft_small<16>(a[k], inv);
        if (inv) {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                a[k][j].re *= 1.0 / 256.0;
                a[k][j].im *= 1.0 / 256.0;
            }
        }
    }
}

template <int MODE, bool XP>
__global__ void __launch_bounds__(kF256Threads, 3) k_fft256(FieldsND F, FftPass f) {
    extern __shared__ __align__(16) unsigned char f256_sm[];
    Cplx* tws = reinterpret_cast<Cplx*>(f256_sm);
    Cplx* xb = tws + 256;
    for (int k = threadIdx.x; k < 256; k += blockDim.x) tws[k] = f.tw[k];
    int l, s;
    f256_map<XP>(threadIdx.x, l, s);
    const long long base = tile_base(f, blockIdx.x) + l * f.ls + s * f.es;
    const long long step = 16 * f.es;  // between a thread's points
    constexpr bool PAIR = MODE == kInvInPlace || MODE == kInvToFields;
    Cplx a[PAIR ? 2 : 1][16];
    // ---- load ----
    if constexpr (MODE == kFwdFromRho) {
        // density_at with every load issued before the stores (the arrays may
        // alias as far as the compiler knows); the same sums in species order
        double r[16];
        if (F.rho_in) {
#pragma unroll
            for (int j = 0; j < 16; ++j) r[j] = F.rho_in[base + j * step];
        } else if (F.nacc) {
#pragma unroll
            for (int j = 0; j < 16; ++j) r[j] = 0.0;
            for (int k = 0; k < F.nacc; ++k) {
                unsigned long long q[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) q[j] = F.acc[k][base + j * step];
#pragma unroll
                for (int j = 0; j < 16; ++j) r[j] += (double)(long long)q[j] * F.acc_scale[k];
            }
            for (int k = 0; k < F.nacc; ++k)
#pragma unroll
                for (int j = 0; j < 16; ++j) F.acc[k][base + j * step] = 0ull;
        } else {
            unsigned long long q[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) q[j] = F.rho_acc[base + j * step];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                r[j] = (double)(long long)q[j] * F.inv_scale;
                F.rho_acc[base + j * step] = 0ull;
            }
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            F.rho[base + j * step] = r[j];
            a[0][j] = {r[j], 0.0};
        }
    } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const long long g = base + j * step;
            if (MODE == kFwdInPlace || MODE == kFwdMulInv) a[0][j] = F.W[g];
            else {
                a[0][j] = F.A[g];
                a[PAIR ? 1 : 0][j] = F.B[g];
            }
        }
    }
    __syncthreads();  // the twiddles are staged
    if constexpr (MODE == kFwdMulInv) {
        fft256<XP, 1>(a, xb, tws, l, s, false);
        Cplx ab[2][16];
#pragma unroll
        for (int j = 0; j < 16; ++j) kspace_tab(F, base + j * step, a[0][j], ab[0][j], ab[1][j]);
        fft256<XP, 2>(ab, xb, tws, l, s, true);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const long long g = base + j * step;
            F.A[g] = ab[0][j];
            F.B[g] = ab[1][j];
        }
    } else {
        fft256<XP, PAIR ? 2 : 1>(a, xb, tws, l, s, PAIR);
    // ---- store ----
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const long long g = base + j * step;
        if (MODE == kFwdFromRho || MODE == kFwdInPlace) F.W[g] = a[0][j];
        else if (MODE == kInvInPlace) {
            F.A[g] = a[0][j];
            F.B[g] = a[PAIR ? 1 : 0][j];
        } else {
            store_fields(F, g, a[0][j], a[PAIR ? 1 : 0][j]);
        }
    }
    }
}

// shared memory of a 256-point pass: the twiddles and one exchange buffer per line set
template <bool XP>
constexpr size_t f256_smem(int mode) {
    return (256 + (size_t)((mode == kFwdMulInv || mode == kInvInPlace || mode == kInvToFields) ? 2 : 1) *
                      f256_xsize<XP>()) * sizeof(Cplx);
}

// Simulation2D/3D sample reductions (src/Diagnostics.cpp:111-137, :205-232):
// kinetic energy of v per species and field energy / charge_l1 of the grid;
// per-block partials, the last block adds them in block order.
constexpr int kSampleBlocks = 148;
__global__ void __launch_bounds__(256) k_sample_nd(SpeciesND S, int dims, double* partial, unsigned* done,
                                                   double* out, const double* E, const double* rho,
                                                   long long N, double half_eps_vol, double vol, int species,
                                                   int last_species, int wall_x, int wall_y, int wall_z, int nx,
                                                   int ny, int nz) {
    __shared__ double red[8], red2[8], red3[8];
    __shared__ bool last;
    const int tid = threadIdx.x;
    double ke = 0.0, fe = 0.0, l1 = 0.0;
    for (unsigned i = blockIdx.x * 256 + tid; i < S.n; i += gridDim.x * 256)
        if (!S.alive || S.alive[i])
            ke += S.hmw * (S.v[0][i] * S.v[0][i] + S.v[1][i] * S.v[1][i] + S.v[2][i] * S.v[2][i]);
    if (last_species) {
        for (long long g = blockIdx.x * 256 + tid; g < N; g += gridDim.x * 256) {
            double e2;
            if (dims == 2) {
                const double2 e = reinterpret_cast<const double2*>(E)[g];
                e2 = e.x * e.x + e.y * e.y;
            } else {
                const double4 e = reinterpret_cast<const double4*>(E)[g];
                e2 = e.x * e.x + e.y * e.y + e.z * e.z;
            }
            // Mesh2D::node_area / Mesh3D::node_volume: half cells on the wall
            // nodes, src/Mesh2D.cpp:77-88, src/Mesh3D.cpp:52-60
            const int gi = (int)(g % nx), gj = (int)((g / nx) % ny), gk = (int)(g / ((long long)nx * ny));
            const double f = ((wall_x && (gi == 0 || gi == nx - 1)) ? 0.5 : 1.0) *
                             ((wall_y && (gj == 0 || gj == ny - 1)) ? 0.5 : 1.0) *
                             ((wall_z && (gk == 0 || gk == nz - 1)) ? 0.5 : 1.0);
            fe += half_eps_vol * e2 * f;
            l1 += fabs(rho[g]) * vol * f;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        ke += __shfl_down_sync(0xffffffffu, ke, o);
        fe += __shfl_down_sync(0xffffffffu, fe, o);
        l1 += __shfl_down_sync(0xffffffffu, l1, o);
    }
    if ((tid & 31) == 0) { red[tid >> 5] = ke; red2[tid >> 5] = fe; red3[tid >> 5] = l1; }
    __syncthreads();
    if (tid == 0) {
        double a = 0, b = 0, c = 0;
        for (int w = 0; w < 8; ++w) { a += red[w]; b += red2[w]; c += red3[w]; }
        partial[3 * blockIdx.x] = a;
        partial[3 * blockIdx.x + 1] = b;
        partial[3 * blockIdx.x + 2] = c;
        __threadfence();
        last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || tid != 0) return;
    __threadfence();
    double a = 0, b = 0, c = 0;
    for (unsigned k = 0; k < gridDim.x; ++k) {
        a += ((volatile double*)partial)[3 * k];
        b += ((volatile double*)partial)[3 * k + 1];
        c += ((volatile double*)partial)[3 * k + 2];
    }
    out[species] = a;
    if (last_species) { out[4] = b; out[5] = c; }
    *done = 0;
}

// ---- host ----------------------------------------------------------------------------

static bool pow2(size_t v) { return v >= 2 && (v & (v - 1)) == 0; }
static int ilog2(size_t v) { int k = 0; while ((size_t(1) << k) < v) ++k; return k; }

// Raises the dynamic shared-memory limit of every FFT / wall-solve kernel, once
// per device, to a fixed bound that covers every tile any mesh here uses.  The
// limit is a property of the kernel function shared by every simulation and
// solve in the process, so it is never lowered to one mesh's need (a later
// small mesh would otherwise make an earlier large mesh's launches fail).
void ensure_solver_attributes();

struct Solver {
    FieldsND F{};
    FftPass px{}, py{}, pz{};    // paired passes (four line buffers)
    FftPass pxs{}, pys{};        // single-array forward passes (two line buffers)
    bool use256[3] = {false, false, false};  // axis a runs the 256-point register kernels
    FftPass q256[3]{};
    size_t smem_fwd = 0, smem_pair = 0;
    std::vector<void*>* allocs = nullptr;
    cudaStream_t stream = nullptr;

    template <class T>
    T* alloc(size_t count) {
        void* p = nullptr;
        APIC_CUDA(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
        allocs->push_back(p);
        APIC_CUDA(cudaMemsetAsync(p, 0, std::max<size_t>(count, 1) * sizeof(T), stream));
        return static_cast<T*>(p);
    }

    Cplx* twiddles(int n) {
        std::vector<Cplx> h(n);
        const double twopi = 2.0 * 3.141592653589793;
        for (int k = 0; k < n; ++k) h[k] = {std::cos(twopi * k / n), -std::sin(twopi * k / n)};
        Cplx* d = alloc<Cplx>(h.size());
        APIC_CUDA(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(Cplx), cudaMemcpyHostToDevice, stream));
        APIC_CUDA(cudaStreamSynchronize(stream));
        return d;
    }

    FftPass pass(int ax, int T) const {
        FftPass f{};
        const long long nx = F.nx, ny = F.ny, nz = F.dims == 3 ? F.nz : 1;
        f.axis = ax;
        f.T = T;
        if (ax == 0) {
            f.n = F.nx; f.es = 1; f.ls = nx;
            f.tiles_inner = ny * nz / T; f.outer_stride = 0;
        } else if (ax == 1) {
            f.n = F.ny; f.es = nx; f.ls = 1;
            f.tiles_inner = nx / T; f.outer_stride = nx * ny;
        } else {
            f.n = F.nz; f.es = nx * ny; f.ls = 1;
            f.tiles_inner = nx / T; f.outer_stride = nx;
        }
        f.log2n = ilog2(f.n);
        f.log2T = ilog2(T);
        return f;
    }

    long long tiles(const FftPass& f) const {
        const long long N = (long long)F.nx * F.ny * (F.dims == 3 ? F.nz : 1);
        return N / ((long long)f.T * f.n);
    }

    void setup(int dims, const size_t* n, const double* L, double eps, double inv_scale) {
        F.dims = dims;
        F.nx = (int)n[0]; F.ny = (int)n[1]; F.nz = dims == 3 ? (int)n[2] : 1;
        F.lnx = ilog2(F.nx);
        F.lny = ilog2(F.ny);
        for (int a = 0; a < 3; ++a) F.L[a] = a < dims ? L[a] : 1.0;
        F.eps = eps;
        F.inv_scale = inv_scale;
        double kmax = 0;
        for (int a = 0; a < dims; ++a) kmax = std::max(kmax, 3.141592653589793 * (double)n[a] / L[a]);
        F.pack = std::ldexp(1.0, (int)std::lround(std::log2(kmax)));
        const size_t N = (size_t)F.nx * F.ny * F.nz;
        F.rho_acc = alloc<unsigned long long>(N);
        F.rho = alloc<double>(N);
        F.W = alloc<Cplx>(N);
        F.A = alloc<Cplx>(N);
        F.B = alloc<Cplx>(N);
        F.phi = alloc<double>(N);
        F.E = alloc<double>(N * (dims == 2 ? 2 : 4));
        // lines per tile: up to 8 (128 B rows in the strided passes), bounded
        // so that the paired passes (three line buffers) fit in shared memory
        // lines per tile: up to 8 (128 B rows in the strided passes), bounded
        // so that two CTAs fit on an SM (about 100 KB of shared memory each)
        auto lines = [](int n, long long available, int buffers) {
            int T = 8;
            while (T > 1 && (size_t)buffers * T * n * sizeof(Cplx) + n * sizeof(Cplx) > kFftTileBytes) T >>= 1;
            while (T > 1 && available % T) T >>= 1;
            return T;
        };
        px = pass(0, lines(F.nx, (long long)F.ny * F.nz, 4));
        pxs = pass(0, lines(F.nx, (long long)F.ny * F.nz, 2));
        py = pass(1, lines(F.ny, F.nx, 4));
        pys = pass(1, lines(F.ny, F.nx, 2));
        if (dims == 3) pz = pass(2, lines(F.nz, F.nx, 4));
        px.tw = pxs.tw = twiddles(F.nx);
        py.tw = pys.tw = F.ny == F.nx ? px.tw : twiddles(F.ny);
        if (dims == 3) pz.tw = F.nz == F.nx ? px.tw : (F.nz == F.ny ? py.tw : twiddles(F.nz));
        for (int a = 0; a < dims; ++a) {  // kspace_at's wavenumbers, src/FieldSolver.cpp:687-712
            const int na = a == 0 ? F.nx : (a == 1 ? F.ny : F.nz);
            std::vector<double> kv(na);
            const double twopi = 2.0 * 3.141592653589793;
            for (int i = 0; i < na; ++i) {
                const double m = i <= na / 2 ? (double)i : -(double)(na - i);
                kv[i] = twopi * m / F.L[a];
            }
            double* d = alloc<double>(na);
            APIC_CUDA(cudaMemcpyAsync(d, kv.data(), na * sizeof(double), cudaMemcpyHostToDevice, stream));
            APIC_CUDA(cudaStreamSynchronize(stream));
            F.kvec[a] = d;
        }
        for (int a = 0; a < dims; ++a) {
            const long long lines = a == 0 ? (long long)F.ny * F.nz : F.nx;
            use256[a] = n[a] == 256 && lines % kF256Lines == 0;
            if (use256[a]) {
                q256[a] = pass(a, kF256Lines);
                q256[a].tw = a == 0 ? px.tw : (a == 1 ? py.tw : pz.tw);
            }
        }
        smem_pair = std::max(smem_of(px, kFwdMulInv), smem_of(py, kFwdMulInv));
        if (dims == 3) smem_pair = std::max(smem_pair, smem_of(pz, kFwdMulInv));
        require(smem_pair <= kFftSmemMax, "FFT tile exceeds the shared-memory bound", APIC_ERR_UNSUPPORTED);
        ensure_solver_attributes();
    }

    size_t smem_of(const FftPass& f, int mode) const {
        const size_t line = (size_t)f.T * f.n * sizeof(Cplx);
        const size_t tw = (size_t)f.n * sizeof(Cplx);
        return (mode == kFwdFromRho || mode == kFwdInPlace) ? 2 * line + tw : 4 * line + tw;
    }

    // one pass along `axis`: the 256-point register kernel where the extent
    // allows it, else the shared-memory tile kernel with pass `tile`
    template <int MODE>
    void fft_pass(int axis, const FftPass& tile) {
        if (use256[axis]) {
            const FftPass& q = q256[axis];
            if (axis == 0)
                k_fft256<MODE, true><<<(unsigned)tiles(q), kF256Threads, f256_smem<true>(MODE), stream>>>(F, q);
            else
                k_fft256<MODE, false><<<(unsigned)tiles(q), kF256Threads, f256_smem<false>(MODE), stream>>>(F, q);
        } else {
            k_fft<MODE><<<(unsigned)tiles(tile), kFftThreads, smem_of(tile, MODE), stream>>>(F, tile);
        }
    }

    // rho_acc -> rho, phi, E (the fixed-point accumulator is cleared)
    void solve() {
        if (F.dims == 2) {
            fft_pass<kFwdFromRho>(0, pxs);
            fft_pass<kFwdMulInv>(1, py);
            fft_pass<kInvToFields>(0, px);
        } else {
            fft_pass<kFwdFromRho>(0, pxs);
            fft_pass<kFwdInPlace>(1, pys);
            fft_pass<kFwdMulInv>(2, pz);
            fft_pass<kInvInPlace>(1, py);
            fft_pass<kInvToFields>(0, px);
        }
        APIC_CUDA(cudaGetLastError());
    }
};

// field solves with walls (defined with their stand-alone entry points below)
__global__ void __launch_bounds__(kFftThreads) k_mixed_forward(const double* __restrict__ rho, Cplx* __restrict__ hat,
                                                               int nx, int np, int periodic_y, const Cplx* tw);
__global__ void k_mixed_tridiag(Cplx* __restrict__ hat, double* __restrict__ mu, int nd, int np, double inv_dsq,
                                double inv_psq, double eps, double lower, double upper);
__global__ void k_mixed_coeffs(double* __restrict__ mu, double* __restrict__ inv, int nd, int np, double inv_dsq,
                               double inv_psq);
constexpr int kMixedSweepMaxRows = 4000;  // k_mixed_sweep's shared memory bound: 48 B per interior row
__global__ void __launch_bounds__(32) k_mixed_sweep(Cplx* __restrict__ hat, const double* __restrict__ mu,
                                                    const double* __restrict__ inv, int nd, int np, double inv_dsq,
                                                    double eps, double lower, double upper);
__global__ void __launch_bounds__(kFftThreads) k_mixed_inverse(const Cplx* __restrict__ hat, double* __restrict__ phi,
                                                               int nx, int np, int periodic_y, const Cplx* tw);
__global__ void k_mixed_efield(const double* __restrict__ phi, double* __restrict__ E, int nx, int ny, double dx,
                               double dy, int periodic_x, int periodic_y);
__global__ void k_dir_rhs(const double* __restrict__ rho, double* __restrict__ u, int nx, int ny, int nz3, double eps,
                          double idx2, double idy2, double left, double right, double bottom, double top);
__global__ void __launch_bounds__(kFftThreads) k_dst_lines(double* __restrict__ u, int M, long long stride, int lines_a,
                                                           long long stride_a, long long stride_b, const Cplx* tw);
__global__ void k_dir_divide(double* __restrict__ u, int Mx, int My, int Mz, double idx2, double idy2, double idz2,
                             double scale);
__global__ void k_dir_assemble(const double* __restrict__ u, double* __restrict__ phi, int nx, int ny, int nz3,
                               double left, double right, double bottom, double top);
__global__ void k_dir_efield3(const double* __restrict__ phi, double* __restrict__ E, int nx, int ny, int nz, double dx,
                              double dy, double dz);

namespace {
std::mutex g_attr_mu;
bool g_attr_done[64] = {};
}  // namespace

void ensure_solver_attributes() {
    int dev = 0;
    APIC_CUDA(cudaGetDevice(&dev));
    require(dev >= 0 && dev < 64, "device index out of range");
    std::lock_guard<std::mutex> lock(g_attr_mu);
    if (g_attr_done[dev]) return;
    const int fft = (int)kFftSmemMax;
    APIC_CUDA(cudaFuncSetAttribute(k_fft<kFwdFromRho>, cudaFuncAttributeMaxDynamicSharedMemorySize, fft));
    APIC_CUDA(cudaFuncSetAttribute(k_fft<kFwdInPlace>, cudaFuncAttributeMaxDynamicSharedMemorySize, fft));
    APIC_CUDA(cudaFuncSetAttribute(k_fft<kFwdMulInv>, cudaFuncAttributeMaxDynamicSharedMemorySize, fft));
    APIC_CUDA(cudaFuncSetAttribute(k_fft<kInvInPlace>, cudaFuncAttributeMaxDynamicSharedMemorySize, fft));
    APIC_CUDA(cudaFuncSetAttribute(k_fft<kInvToFields>, cudaFuncAttributeMaxDynamicSharedMemorySize, fft));
    const int f256x = (int)f256_smem<true>(kInvToFields), f256s = (int)f256_smem<false>(kInvToFields);
    APIC_CUDA(cudaFuncSetAttribute(k_fft256<kFwdFromRho, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, f256x));
    APIC_CUDA(cudaFuncSetAttribute(k_fft256<kFwdInPlace, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, f256x));
    APIC_CUDA(cudaFuncSetAttribute(k_fft256<kFwdMulInv, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, f256x));
    APIC_CUDA(cudaFuncSetAttribute(k_fft256<kInvInPlace, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, f256x));
    APIC_CUDA(cudaFuncSetAttribute(k_fft256<kInvToFields, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, f256x));
    APIC_CUDA(cudaFuncSetAttribute(k_fft256<kFwdFromRho, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, f256s));
    APIC_CUDA(cudaFuncSetAttribute(k_fft256<kFwdInPlace, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, f256s));
    APIC_CUDA(cudaFuncSetAttribute(k_fft256<kFwdMulInv, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, f256s));
    APIC_CUDA(cudaFuncSetAttribute(k_fft256<kInvInPlace, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, f256s));
    APIC_CUDA(cudaFuncSetAttribute(k_fft256<kInvToFields, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, f256s));
    const int lines = (int)(3 * kMaxLine * sizeof(Cplx));  // three line buffers of the longest extent
    APIC_CUDA(cudaFuncSetAttribute(k_mixed_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, lines));
    APIC_CUDA(cudaFuncSetAttribute(k_mixed_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, lines));
    APIC_CUDA(cudaFuncSetAttribute(k_dst_lines, cudaFuncAttributeMaxDynamicSharedMemorySize, lines));
    APIC_CUDA(cudaFuncSetAttribute(k_mixed_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize, kMixedSweepMaxRows * 48));
    g_attr_done[dev] = true;
}

struct SimND {
    apic_config_nd cfg{};
    std::string last_error;
    cudaStream_t stream = nullptr;
    std::vector<void*> allocations;
    ParamsND p{};
    SpeciesND sp[APIC_MAX_SPECIES]{};
    int buf[APIC_MAX_SPECIES] = {0, 0, 0, 0};
    Solver solver;
    bool boris = false;
    bool fp32 = false;
    bool initialized = false;
    double time = 0.0;
    uint64_t step_count = 0;
    size_t sort_interval = 16;
    uint64_t launches = 0;  // kernels launched by step()
    size_t steps_since_sort = 0;                   // of the most frequently sorted species
    size_t since_sort[APIC_MAX_SPECIES] = {0, 0, 0, 0};
    size_t species_interval[APIC_MAX_SPECIES] = {16, 16, 16, 16};
    unsigned* cell_count = nullptr;
    unsigned* cell_offset = nullptr;
    unsigned* block_sums = nullptr;
    size_t ncells = 0;
    double* sample_partial = nullptr;
    unsigned* sample_done = nullptr;
    double* sample_out = nullptr;
    bool timing = false;
    double push_ms = 0, solve_ms = 0, sort_ms = 0;
    uint64_t timed_steps = 0;
    struct Ev { cudaEvent_t a, b, c, d; bool sorted; };
    std::vector<Ev> events;

    template <class T>
    T* dalloc(size_t count) {
        void* ptr = nullptr;
        APIC_CUDA(cudaMalloc(&ptr, std::max<size_t>(count, 1) * sizeof(T)));
        allocations.push_back(ptr);
        APIC_CUDA(cudaMemsetAsync(ptr, 0, std::max<size_t>(count, 1) * sizeof(T), stream));
        return static_cast<T*>(ptr);
    }

    ~SimND() {
        if (stream) cudaStreamSynchronize(stream);
        drop_graphs();
        for (auto& e : events) { cudaEventDestroy(e.a); cudaEventDestroy(e.b); cudaEventDestroy(e.c); cudaEventDestroy(e.d); }
        for (void* a : allocations) cudaFree(a);
        if (stream) cudaStreamDestroy(stream);
    }

    void create(const apic_config_nd& c) {
        cfg = c;
        require(c.dims == 2 || c.dims == 3, "dims must be 2 or 3");
        require(c.precision == APIC_FP64 || c.precision == APIC_FP32, "unknown precision");
        fp32 = c.precision == APIC_FP32;
        walls = c.wall_axis[0] != 0 || c.wall_axis[1] != 0 || (c.dims == 3 && c.wall_axis_z != 0);
        if (walls) {
            require(!fp32, "runs with walls use the FP64 particle form", APIC_ERR_UNSUPPORTED);
            for (int k = 0; k < 4; ++k) {
                require(c.particle_boundary[k] >= 0 && c.particle_boundary[k] <= 3, "unknown particle boundary");
                require(std::isfinite(c.wall_potential[k]), "wall potentials must be finite");
            }
            if (c.dims == 3) {
                // Simulation3DConfig has one field boundary for the mesh (src/Mesh3D.cpp:37-48)
                require(c.wall_axis[0] && c.wall_axis[1] && c.wall_axis_z,
                        "3D meshes are periodic or Dirichlet on every axis", APIC_ERR_UNSUPPORTED);
                require(c.wall_potential[0] == 0.0 && c.wall_potential[1] == 0.0 && c.wall_potential[2] == 0.0 &&
                            c.wall_potential[3] == 0.0,
                        "3D Dirichlet walls are grounded");
                for (int k = 0; k < 2; ++k)
                    require(c.particle_boundary_z[k] >= 0 && c.particle_boundary_z[k] <= 3,
                            "unknown particle boundary");
            }
        }
        for (int a = 0; a < c.dims; ++a) {
            require(c.n[a] >= 3, "mesh extents must be at least 3");
            const bool wall = walls && (a < 2 ? c.wall_axis[a] != 0 : c.wall_axis_z != 0);
            if (!wall)
                require(pow2(c.n[a]) && c.n[a] <= (size_t)kMaxLine,
                        "periodic device meshes need power-of-two extents up to 1024", APIC_ERR_UNSUPPORTED);
            else if (c.wall_axis[0] && c.wall_axis[1])
                require(pow2(c.n[a] - 1) && 2 * (c.n[a] - 1) <= (size_t)kMaxLine,
                        "walls on every side need extents of 2^k + 1 nodes up to 513", APIC_ERR_UNSUPPORTED);
            else
                require(c.n[a] <= 65536, "the wall axis allows up to 65536 nodes", APIC_ERR_UNSUPPORTED);
            require(std::isfinite(c.length[a]) && c.length[a] > 0, "domain lengths must be positive and finite");
        }
        require(std::isfinite(c.dt) && c.dt > 0, "simulation dt must be positive and finite");
        require(c.nspecies >= 1 && c.nspecies <= APIC_MAX_SPECIES, "species count out of range");
        require(c.push_items == 0 || c.push_items == 1 || c.push_items == 2 || c.push_items == 4 ||
                    c.push_items == 8,
                "push_items must be 0, 1, 2, 4 or 8");
        const double rel = c.relative_permittivity == 0.0 ? 1.0 : c.relative_permittivity;
        require(std::isfinite(rel) && rel > 0, "relative_permittivity must be positive and finite");
        const double depth = c.out_of_plane_depth == 0.0 ? 1.0 : c.out_of_plane_depth;
        require(std::isfinite(depth) && depth > 0, "2D deposition depth must be positive and finite");
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
            throw Error(APIC_ERR_NO_DEVICE, "no CUDA device is visible");
        APIC_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        sort_interval = c.sort_interval ? c.sort_interval : 16;
        for (int k = 0; k < APIC_MAX_SPECIES; ++k)
            species_interval[k] = c.species_sort_interval[k] ? c.species_sort_interval[k] : sort_interval;

        p.dims = c.dims;
        size_t N = 1;
        double cellvol = 1.0;
        for (int a = 0; a < 3; ++a) {
            p.n[a] = a < c.dims ? (int)c.n[a] : 1;
            p.L[a] = a < c.dims ? c.length[a] : 1.0;
            // Mesh2D/Mesh3D dx: L / n periodic, L / (n - 1) on a wall axis,
            // src/Mesh2D.cpp:57-62, src/Mesh3D.cpp:43-45
            const bool wall_a = walls && a < c.dims && (a < 2 ? c.wall_axis[a] != 0 : c.wall_axis_z != 0);
            p.d[a] = p.L[a] / (double)(wall_a ? p.n[a] - 1 : p.n[a]);
            p.B[a] = c.magnetic_field[a];
            N *= (size_t)p.n[a];
            if (a < c.dims) cellvol *= p.d[a];
        }
        ncells = N;
        boris = c.magnetic_field[0] != 0.0 || c.magnetic_field[1] != 0.0 || c.magnetic_field[2] != 0.0;
        if (c.profile_rows) {
            // Simulation2D / Simulation3D constructor checks, src/Simulation3D.cpp:184-196
            require(!boris, std::string(c.dims == 2 ? "2D" : "3D") +
                                " uniform magnetic_field components and magnetic_field_profile are mutually exclusive");
            require(c.profile_axis >= 0 && c.profile_axis <= 2, "coordinate axis must be x, y, or z");
            require(c.profile_rows >= 2, "tabulated vector field requires at least two rows");
            require(c.profile_coordinates && c.profile_values, "tabulated vector field arrays are required");
            for (size_t k = 0; k < c.profile_rows; ++k) {
                require(std::isfinite(c.profile_coordinates[k]) && std::isfinite(c.profile_values[3 * k]) &&
                            std::isfinite(c.profile_values[3 * k + 1]) && std::isfinite(c.profile_values[3 * k + 2]),
                        "tabulated vector field values must be finite");
                require(k == 0 || c.profile_coordinates[k] > c.profile_coordinates[k - 1],
                        "tabulated vector field coordinates must be strictly increasing");
            }
            const double hi = c.profile_axis < c.dims ? c.length[c.profile_axis] : 0.0;
            require(c.profile_coordinates[0] <= 0.0 && c.profile_coordinates[c.profile_rows - 1] >= hi,
                    "tabulated magnetic field does not cover the simulation domain");
            require(c.profile_rows < (1u << 30), "tabulated vector field too long");
            boris = true;
        }
        p.dt = c.dt;
        p.eps = (c.units == APIC_SI ? 8.8541878128e-12 : 1.0) * rel;
        double bound = 0.0;
        for (int s = 0; s < c.nspecies; ++s) {
            const auto& S = c.species[s];
            require(std::isfinite(S.mass) && S.mass > 0, "species mass must be positive and finite");
            require(S.capacity > 0 && S.capacity < (1ull << 31), "species capacity out of range");
            const double w = c.dims == 2 ? S.weight / depth : S.weight;  // Species2D::deposit_charge
            // a wall node's half cells (a corner's eighth) raise its density by up to 2^dims
            bound += (double)S.capacity * std::fabs(S.charge * w) / cellvol * (walls ? (double)(1 << c.dims) : 1.0);
        }
        const int bits = bound > 0 ? (int)std::floor(61.0 - std::log2(bound)) : 0;
        p.rho_scale = std::ldexp(1.0, bits);
        p.inv_rho_scale = std::ldexp(1.0, -bits);
        for (int s = 0; s < c.nspecies; ++s) {
            const auto& S = c.species[s];
            SpeciesND& D = sp[s];
            D.qm = S.charge / S.mass;
            const double w = c.dims == 2 ? S.weight / depth : S.weight;
            D.dep = S.charge * w / cellvol;
            D.hmw = 0.5 * S.mass * S.weight;
            D.n = 0;
            for (int b = 0; b < 2; ++b) {
                for (int a = 0; a < c.dims; ++a) D.pos[b][a] = dalloc<double>(S.capacity);
                for (int a = 0; a < 3; ++a) D.vh[b][a] = dalloc<double>(S.capacity);
                D.id[b] = dalloc<unsigned>(S.capacity);
            }
            for (int a = 0; a < 3; ++a) D.v[a] = dalloc<double>(S.capacity);
            if (fp32) {
                for (int b = 0; b < 2; ++b) {
                    D.cell[b] = dalloc<unsigned>(S.capacity);
                    for (int a = 0; a < c.dims; ++a) D.off[b][a] = dalloc<float>(S.capacity);
                    for (int a = 0; a < 3; ++a) D.vel[b][a] = dalloc<float>(S.capacity);
                }
            }
            const double hq = 0.5 * D.qm * c.dt;
            D.hqmdt = (float)hq;
            D.qmdt = (float)(D.qm * c.dt);
            double t2 = 0.0;
            for (int a = 0; a < 3; ++a) { D.tb[a] = (float)(hq * c.magnetic_field[a]); t2 += (hq * c.magnetic_field[a]) * (hq * c.magnetic_field[a]); }
            for (int a = 0; a < 3; ++a) D.sb[a] = (float)(2.0 * hq * c.magnetic_field[a] / (1.0 + t2));
            for (int a = 0; a < 3; ++a) D.drift[a] = a < c.dims ? (float)(c.dt / p.d[a]) : 0.0f;
            D.dep_fixed = (float)(D.dep * p.rho_scale);
            D.index = s;
        }
        solver.allocs = &allocations;
        solver.stream = stream;
        if (walls) {
            setup_walls(c);
        } else {
            solver.setup(c.dims, c.n, c.length, p.eps, p.inv_rho_scale);
        }
        p.E = solver.F.E;
        p.rho_acc = solver.F.rho_acc;
        if (c.profile_rows) {  // copied: the caller's arrays may go away after create
            double* pc = dalloc<double>(c.profile_rows);
            double* pv = dalloc<double>(3 * c.profile_rows);
            APIC_CUDA(cudaMemcpyAsync(pc, c.profile_coordinates, c.profile_rows * sizeof(double),
                                      cudaMemcpyHostToDevice, stream));
            APIC_CUDA(cudaMemcpyAsync(pv, c.profile_values, 3 * c.profile_rows * sizeof(double),
                                      cudaMemcpyHostToDevice, stream));
            p.prof_axis = c.profile_axis;
            p.prof_rows = (int)c.profile_rows;
            p.prof_c = pc;
            p.prof_v = pv;
            cfg.profile_coordinates = nullptr;  // not kept
            cfg.profile_values = nullptr;
        }
        if (fp32) {
            solver.F.E32 = dalloc<float>(N * (c.dims == 2 ? 2 : 4));
            p.E32 = solver.F.E32;
            solver.F.nacc = c.nspecies;
            for (int s = 0; s < c.nspecies; ++s) {
                solver.F.acc[s] = dalloc<unsigned long long>(N);
                solver.F.acc_scale[s] = sp[s].dep / (double)kWeightScale;
            }
        }
        cell_count = dalloc<unsigned>(N);
        cell_offset = dalloc<unsigned>(N);
        block_sums = dalloc<unsigned>((N + kScanBlock - 1) / kScanBlock + 1);
        sample_partial = dalloc<double>(3 * kSampleBlocks);
        sample_done = dalloc<unsigned>(1);
        sample_out = dalloc<double>(8);
        APIC_CUDA(cudaStreamSynchronize(stream));
    }

    SpeciesND view(int s) const { return sp[s]; }

    template <int DIM, bool BORIS>
    void launch_step32(int items, const SpeciesND& S, int b, int s) {
        const unsigned g = (unsigned)((S.n + (unsigned)items * kThreads - 1) / ((unsigned)items * kThreads));
        unsigned long long* acc = solver.F.acc[s];
        if (BORIS && p.prof_rows) {
            switch (items) {
                case 1: k_push32_step<DIM, BORIS, 1, true><<<g, kThreads, 0, stream>>>(p, S, b, acc); break;
                case 2: k_push32_step<DIM, BORIS, 2, true><<<g, kThreads, 0, stream>>>(p, S, b, acc); break;
                case 4: k_push32_step<DIM, BORIS, 4, true><<<g, kThreads, 0, stream>>>(p, S, b, acc); break;
                default: k_push32_step<DIM, BORIS, 8, true><<<g, kThreads, 0, stream>>>(p, S, b, acc); break;
            }
            return;
        }
        switch (items) {
            case 1: k_push32_step<DIM, BORIS, 1, false><<<g, kThreads, 0, stream>>>(p, S, b, acc); break;
            case 2: k_push32_run<DIM, BORIS, 2, false><<<g, kThreads, 0, stream>>>(p, S, b, acc); break;
            case 4: k_push32_run<DIM, BORIS, 4, false><<<g, kThreads, 0, stream>>>(p, S, b, acc); break;
            default: k_push32_step<DIM, BORIS, 8, false><<<g, kThreads, 0, stream>>>(p, S, b, acc); break;
        }
    }

    template <int MODE>
    void launch_push(int s) {
        const SpeciesND& S = sp[s];
        if (S.n == 0) return;
        const unsigned blocks = (S.n + kThreads - 1) / kThreads;
        const int b = buf[s];
        if (fp32 && MODE == kPushStep) {
            // particles per thread: configured, else the measured best (4 in 2D, 2 in 3D)
            const int items = cfg.push_items ? cfg.push_items : (cfg.dims == 2 ? 4 : 2);
            if (cfg.dims == 2) {
                if (boris) launch_step32<2, true>(items, S, b, s);
                else launch_step32<2, false>(items, S, b, s);
            } else {
                if (boris) launch_step32<3, true>(items, S, b, s);
                else launch_step32<3, false>(items, S, b, s);
            }
            APIC_CUDA(cudaGetLastError());
            return;
        }
        if (fp32) {
            if (cfg.dims == 2) {
                if (boris) k_push32<2, true, MODE><<<blocks, kThreads, 0, stream>>>(p, S, b, solver.F.acc[s]);
                else k_push32<2, false, MODE><<<blocks, kThreads, 0, stream>>>(p, S, b, solver.F.acc[s]);
            } else {
                if (boris) k_push32<3, true, MODE><<<blocks, kThreads, 0, stream>>>(p, S, b, solver.F.acc[s]);
                else k_push32<3, false, MODE><<<blocks, kThreads, 0, stream>>>(p, S, b, solver.F.acc[s]);
            }
            APIC_CUDA(cudaGetLastError());
            return;
        }
        if (cfg.dims == 2 && walls) {
            if (boris) k_push<2, true, MODE, true><<<blocks, kThreads, 0, stream>>>(p, S, b);
            else k_push<2, false, MODE, true><<<blocks, kThreads, 0, stream>>>(p, S, b);
        } else if (walls) {
            if (boris) k_push<3, true, MODE, true><<<blocks, kThreads, 0, stream>>>(p, S, b);
            else k_push<3, false, MODE, true><<<blocks, kThreads, 0, stream>>>(p, S, b);
        } else if (cfg.dims == 2) {
            if (boris) k_push<2, true, MODE><<<blocks, kThreads, 0, stream>>>(p, S, b);
            else k_push<2, false, MODE><<<blocks, kThreads, 0, stream>>>(p, S, b);
        } else {
            if (boris) k_push<3, true, MODE><<<blocks, kThreads, 0, stream>>>(p, S, b);
            else k_push<3, false, MODE><<<blocks, kThreads, 0, stream>>>(p, S, b);
        }
        APIC_CUDA(cudaGetLastError());
    }

    void sort_species(int s) {
        SpeciesND& S = sp[s];
        if (S.n == 0) return;
        const unsigned blocks = (S.n + kThreads - 1) / kThreads;
        const unsigned nb = (unsigned)((ncells + kScanBlock - 1) / kScanBlock);
        APIC_CUDA(cudaMemsetAsync(cell_count, 0, ncells * sizeof(unsigned), stream));
        if (fp32) k_cell_hist32<<<blocks, kThreads, 0, stream>>>(p, S, buf[s], cell_count);
        else if (cfg.dims == 2) k_cell_hist<2><<<blocks, kThreads, 0, stream>>>(p, S, buf[s], cell_count);
        else k_cell_hist<3><<<blocks, kThreads, 0, stream>>>(p, S, buf[s], cell_count);
        k_scan_local<<<nb, kThreads, 0, stream>>>(cell_count, cell_offset, block_sums, (unsigned)ncells);
        k_scan_blocks<<<1, kThreads, 0, stream>>>(block_sums, nb);
        k_scan_add<<<nb, kThreads, 0, stream>>>(cell_offset, block_sums, (unsigned)ncells);
        if (fp32) {
            k_cell_rank32<<<blocks, kThreads, 0, stream>>>(p, S, buf[s], cell_offset);
            if (cfg.dims == 2) k_cell_gather32<2><<<blocks, kThreads, 0, stream>>>(S, buf[s]);
            else k_cell_gather32<3><<<blocks, kThreads, 0, stream>>>(S, buf[s]);
        } else if (cfg.dims == 2) {
            k_cell_scatter<2><<<blocks, kThreads, 0, stream>>>(p, S, buf[s], cell_offset);
        } else {
            k_cell_scatter<3><<<blocks, kThreads, 0, stream>>>(p, S, buf[s], cell_offset);
        }
        APIC_CUDA(cudaGetLastError());
        buf[s] ^= 1;
    }

    void to_fp32(int s) {
        const SpeciesND& S = sp[s];
        if (!fp32 || S.n == 0) return;
        const unsigned blocks = (S.n + kThreads - 1) / kThreads;
        if (cfg.dims == 2) k_to_fp32<2><<<blocks, kThreads, 0, stream>>>(p, S, buf[s]);
        else k_to_fp32<3><<<blocks, kThreads, 0, stream>>>(p, S, buf[s]);
        APIC_CUDA(cudaGetLastError());
    }

    void to_fp64(int s) {
        const SpeciesND& S = sp[s];
        if (!fp32 || S.n == 0) return;
        const unsigned blocks = (S.n + kThreads - 1) / kThreads;
        if (cfg.dims == 2) k_to_fp64<2><<<blocks, kThreads, 0, stream>>>(p, S, buf[s]);
        else k_to_fp64<3><<<blocks, kThreads, 0, stream>>>(p, S, buf[s]);
        APIC_CUDA(cudaGetLastError());
    }

    void load(int s, size_t n, const double* pos, const double* v, const double* vh) {
        require(s >= 0 && s < cfg.nspecies, "species index out of range");
        require(pos && v, "positions and velocities are required");
        require(n <= cfg.species[s].capacity, "initial particle count exceeds max_particles_per_species",
                APIC_ERR_CAPACITY);
        SpeciesND& S = sp[s];
        if (S.alive && n) APIC_CUDA(cudaMemsetAsync(S.alive, 1, n, stream));
        const int b = buf[s];
        const size_t bytes = n * sizeof(double);
        for (int a = 0; a < cfg.dims; ++a)
            APIC_CUDA(cudaMemcpyAsync(S.pos[b][a], pos + a * n, bytes, cudaMemcpyHostToDevice, stream));
        for (int a = 0; a < 3; ++a) {
            APIC_CUDA(cudaMemcpyAsync(S.v[a], v + a * n, bytes, cudaMemcpyHostToDevice, stream));
            APIC_CUDA(cudaMemcpyAsync(S.vh[b][a], (vh ? vh : v) + a * n, bytes, cudaMemcpyHostToDevice, stream));
        }
        std::vector<unsigned> ids(n);
        for (size_t i = 0; i < n; ++i) ids[i] = (unsigned)i;
        APIC_CUDA(cudaMemcpyAsync(S.id[b], ids.data(), n * sizeof(unsigned), cudaMemcpyHostToDevice, stream));
        APIC_CUDA(cudaStreamSynchronize(stream));
        if (S.n != (unsigned)n) drop_graphs();  // captured launches carry the particle count
        S.n = (unsigned)n;
        to_fp32(s);
        initialized = false;
    }

    void load_maxwellian(int s, size_t n, uint64_t seed, double vt, double drift, int axis, double amp) {
        require(s >= 0 && s < cfg.nspecies, "species index out of range");
        require(n <= cfg.species[s].capacity, "initial particle count exceeds max_particles_per_species",
                APIC_ERR_CAPACITY);
        require(std::isfinite(vt) && vt >= 0 && std::isfinite(drift) && std::isfinite(amp), "invalid loading parameters");
        SpeciesND& S = sp[s];
        const unsigned blocks = (unsigned)((n + kThreads - 1) / kThreads);
        if (n) k_load_maxwellian<<<blocks, kThreads, 0, stream>>>(S, buf[s], cfg.dims, (unsigned)n, seed, p.L[0],
                                                                   p.L[1], p.L[2], vt, drift, axis, amp);
        APIC_CUDA(cudaGetLastError());
        if (S.n != (unsigned)n) drop_graphs();  // captured launches carry the particle count
        S.n = (unsigned)n;
        to_fp32(s);
        initialized = false;
    }

    // ---- walls: persistent solve scratch on the run's stream ----
    bool walls = false;
    int wall_mode = 0;  // 1: one wall axis (mixed solve), 2: walls on every side
    int periodic_axis = 0;
    double* w_planes = nullptr;  // Ex | Ey (| Ez)
    double* w_mu = nullptr;
    double* w_inv = nullptr;  // per-mode pivots' reciprocals (k_mixed_sweep)
    Cplx* w_hat = nullptr;
    Cplx* w_tw = nullptr;
    double* w_u = nullptr;
    Cplx* w_dtw[3] = {nullptr, nullptr, nullptr};

    void setup_walls(const apic_config_nd& c) {
        const int dims = c.dims;
        const size_t N = c.n[0] * c.n[1] * (dims == 3 ? c.n[2] : 1);
        for (int k = 0; k < 2 * dims; ++k) {
            const int kind = k < 4 ? c.particle_boundary[k] : c.particle_boundary_z[k - 4];
            const bool wall = k < 4 ? c.wall_axis[k >> 1] != 0 : c.wall_axis_z != 0;
            // resolve_particle_boundary, src/Simulation2D.cpp:38-41, src/Simulation3D.cpp:25-28
            // (Auto follows the field boundary)
            p.pbc[k] = kind == 0 ? (wall ? 1 : 0) : (kind == 1 ? 1 : (kind == 2 ? 2 : 0));
        }
        p.wall[0] = c.wall_axis[0] != 0;
        p.wall[1] = c.wall_axis[1] != 0;
        p.wall[2] = dims == 3 && c.wall_axis_z != 0;
        p.losses = dalloc<unsigned long long>(6 * APIC_MAX_SPECIES);
        bool absorbing = false;
        for (int k = 0; k < 2 * dims; ++k) absorbing = absorbing || p.pbc[k] == 1;
        for (int s = 0; s < c.nspecies; ++s)
            sp[s].alive = absorbing ? dalloc<uint8_t>(c.species[s].capacity) : nullptr;
        solver.F.dims = dims;
        solver.F.rho_acc = dalloc<unsigned long long>(N);
        solver.F.rho = dalloc<double>(N);
        solver.F.phi = dalloc<double>(N);
        solver.F.E = dalloc<double>((dims == 3 ? 4 : 2) * N);
        w_planes = dalloc<double>((size_t)dims * N);
        const double twopi = 2.0 * 3.141592653589793;
        if (p.wall[0] && p.wall[1]) {
            wall_mode = 2;
            const int M[3] = {(int)c.n[0] - 2, (int)c.n[1] - 2, dims == 3 ? (int)c.n[2] - 2 : 1};
            w_u = dalloc<double>((size_t)M[0] * M[1] * M[2]);
            for (int a = 0; a < dims; ++a) {
                const int L2 = 2 * (M[a] + 1);
                std::vector<Cplx> tw(L2);
                for (int k = 0; k < L2; ++k) tw[k] = {std::cos(twopi * k / L2), -std::sin(twopi * k / L2)};
                w_dtw[a] = dalloc<Cplx>(L2);
                APIC_CUDA(cudaMemcpyAsync(w_dtw[a], tw.data(), L2 * sizeof(Cplx), cudaMemcpyHostToDevice, stream));
            }
            ensure_solver_attributes();
        } else {
            wall_mode = 1;
            periodic_axis = p.wall[0] ? 1 : 0;
            const size_t np = c.n[periodic_axis];
            w_mu = dalloc<double>(N);
            w_hat = dalloc<Cplx>(N);
            {
                const int nd = (int)c.n[periodic_axis ? 0 : 1];
                const double hd = p.d[periodic_axis ? 0 : 1], hp = p.d[periodic_axis];
                if (nd - 2 <= kMixedSweepMaxRows) {
                    w_inv = dalloc<double>(N);
                    k_mixed_coeffs<<<(unsigned)((np + 127) / 128), 128, 0, stream>>>(
                        w_mu, w_inv, nd, (int)np, 1.0 / (hd * hd), 1.0 / (hp * hp));
                    APIC_CUDA(cudaGetLastError());
                }
            }
            std::vector<Cplx> tw(np);
            for (size_t k = 0; k < np; ++k) tw[k] = {std::cos(twopi * k / np), -std::sin(twopi * k / np)};
            w_tw = dalloc<Cplx>(np);
            APIC_CUDA(cudaMemcpyAsync(w_tw, tw.data(), np * sizeof(Cplx), cudaMemcpyHostToDevice, stream));
            ensure_solver_attributes();
        }
        APIC_CUDA(cudaStreamSynchronize(stream));
    }

    // FieldSolver::solve(Mesh3D&) on a Dirichlet mesh, src/FieldSolver.cpp:399-405:
    // the direct sine-transform solve (grounded walls) of the system the
    // reference's SOR iterates on; E by differences, one-sided at the walls.
    void solve_walls3() {
        const int nx = p.n[0], ny = p.n[1], nz = p.n[2];
        const size_t N = (size_t)nx * ny * nz;
        const unsigned g = (unsigned)std::min<size_t>((N + 255) / 256, 4096);
        k_walls_rho<<<g, 256, 0, stream>>>(solver.F.rho_acc, solver.F.rho, N, p.inv_rho_scale);
        const int M[3] = {nx - 2, ny - 2, nz - 2};
        const double idx2 = 1.0 / (p.d[0] * p.d[0]), idy2 = 1.0 / (p.d[1] * p.d[1]), idz2 = 1.0 / (p.d[2] * p.d[2]);
        k_dir_rhs<<<g, 256, 0, stream>>>(solver.F.rho, w_u, nx, ny, nz, p.eps, idx2, idy2, 0.0, 0.0, 0.0, 0.0);
        auto dst_axis = [&](int a) {
            const long long sx = 1, sy = M[0], sz = (long long)M[0] * M[1];
            long long stride, stride_a, stride_b;
            int lines_a;
            size_t lines;
            if (a == 0) { stride = sx; lines_a = M[1]; stride_a = sy; stride_b = sz; lines = (size_t)M[1] * M[2]; }
            else if (a == 1) { stride = sy; lines_a = M[0]; stride_a = sx; stride_b = sz; lines = (size_t)M[0] * M[2]; }
            else { stride = sz; lines_a = M[0]; stride_a = sx; stride_b = sy; lines = (size_t)M[0] * M[1]; }
            const size_t smem = 3 * (size_t)(2 * (M[a] + 1)) * sizeof(Cplx);
            k_dst_lines<<<(unsigned)lines, kFftThreads, smem, stream>>>(w_u, M[a], stride, lines_a, stride_a, stride_b,
                                                                         w_dtw[a]);
        };
        for (int a = 0; a < 3; ++a) dst_axis(a);
        double scale = 1.0;
        for (int a = 0; a < 3; ++a) scale *= 2.0 / (double)(M[a] + 1);
        k_dir_divide<<<g, 256, 0, stream>>>(w_u, M[0], M[1], M[2], idx2, idy2, idz2, scale);
        for (int a = 0; a < 3; ++a) dst_axis(a);
        k_dir_assemble<<<g, 256, 0, stream>>>(w_u, solver.F.phi, nx, ny, nz, 0.0, 0.0, 0.0, 0.0);
        k_dir_efield3<<<g, 256, 0, stream>>>(solver.F.phi, w_planes, nx, ny, nz, p.d[0], p.d[1], p.d[2]);
        k_walls_interleave3<<<g, 256, 0, stream>>>(w_planes, reinterpret_cast<double4*>(solver.F.E), N);
        APIC_CUDA(cudaGetLastError());
    }

    // FieldSolver::solve(Mesh2D&) with walls, src/FieldSolver.cpp:389-397: the
    // mixed spectral-tridiagonal solve, or the direct sine-transform solve of
    // the system the reference's SOR iterates on; E by differences.
    void solve_walls() {
        if (cfg.dims == 3) {
            solve_walls3();
            return;
        }
        const int nx = p.n[0], ny = p.n[1];
        const size_t N = (size_t)nx * ny;
        const unsigned g = (unsigned)std::min<size_t>((N + 255) / 256, 4096);
        const double* pot = cfg.wall_potential;
        k_walls_rho<<<g, 256, 0, stream>>>(solver.F.rho_acc, solver.F.rho, N, p.inv_rho_scale);
        const double dx = p.d[0], dy = p.d[1];
        if (wall_mode == 1) {
            const int py = periodic_axis == 1;
            const int nd = py ? nx : ny, np = py ? ny : nx;
            const double hd = py ? dx : dy, hp = py ? dy : dx;
            const double lo = py ? pot[0] : pot[2], hi = py ? pot[1] : pot[3];
            const size_t smem = 3 * (size_t)np * sizeof(Cplx);
            k_mixed_forward<<<(unsigned)nd, kFftThreads, smem, stream>>>(solver.F.rho, w_hat, nx, np, py, w_tw);
            if (w_inv)
                k_mixed_sweep<<<(unsigned)np, 32, (size_t)(nd - 2) * 48, stream>>>(w_hat, w_mu, w_inv, nd, np,
                                                                                    1.0 / (hd * hd), p.eps, lo, hi);
            else
                k_mixed_tridiag<<<(unsigned)((np + 127) / 128), 128, 0, stream>>>(w_hat, w_mu, nd, np, 1.0 / (hd * hd),
                                                                                  1.0 / (hp * hp), p.eps, lo, hi);
            k_mixed_inverse<<<(unsigned)nd, kFftThreads, smem, stream>>>(w_hat, solver.F.phi, nx, np, py, w_tw);
            k_mixed_efield<<<g, 256, 0, stream>>>(solver.F.phi, w_planes, nx, ny, dx, dy, py ? 0 : 1, py);
        } else {
            const int Mx = nx - 2, My = ny - 2;
            const double idx2 = 1.0 / (dx * dx), idy2 = 1.0 / (dy * dy);
            k_dir_rhs<<<g, 256, 0, stream>>>(solver.F.rho, w_u, nx, ny, 1, p.eps, idx2, idy2, pot[0], pot[1], pot[2],
                                             pot[3]);
            const int M[2] = {Mx, My};
            auto dst_axis = [&](int a) {
                const long long stride = a == 0 ? 1 : Mx, stride_a = a == 0 ? Mx : 1, stride_b = (long long)Mx * My;
                const int lines_a = a == 0 ? My : Mx;
                const size_t smem = 3 * (size_t)(2 * (M[a] + 1)) * sizeof(Cplx);
                k_dst_lines<<<(unsigned)lines_a, kFftThreads, smem, stream>>>(w_u, M[a], stride, lines_a, stride_a,
                                                                               stride_b, w_dtw[a]);
            };
            dst_axis(0);
            dst_axis(1);
            const double scale = (2.0 / (double)(Mx + 1)) * (2.0 / (double)(My + 1));
            k_dir_divide<<<g, 256, 0, stream>>>(w_u, Mx, My, 1, idx2, idy2, 0.0, scale);
            dst_axis(0);
            dst_axis(1);
            k_dir_assemble<<<g, 256, 0, stream>>>(w_u, solver.F.phi, nx, ny, 1, pot[0], pot[1], pot[2], pot[3]);
            k_mixed_efield<<<g, 256, 0, stream>>>(solver.F.phi, w_planes, nx, ny, dx, dy, 0, 0);
        }
        k_walls_interleave<<<g, 256, 0, stream>>>(w_planes, solver.F.E, N);
        APIC_CUDA(cudaGetLastError());
    }

    void solve_fields() {
        if (walls) solve_walls();
        else solver.solve();
    }

    void deposit_and_solve() {
        for (int s = 0; s < cfg.nspecies; ++s) launch_push<kPushDepositOnly>(s);
        solve_fields();
    }

    void initialize() {
        time = 0.0;
        step_count = 0;
        deposit_and_solve();
        for (int s = 0; s < cfg.nspecies; ++s) launch_push<kPushInitHalf>(s);
        initialized = true;
        steps_since_sort = sort_interval;  // sort before the first step
        for (int k = 0; k < APIC_MAX_SPECIES; ++k) since_sort[k] = species_interval[k];
    }

    void resume(double t, uint64_t k) {
        time = t;
        step_count = k;
        deposit_and_solve();
        initialized = true;
        steps_since_sort = sort_interval;
        for (int k = 0; k < APIC_MAX_SPECIES; ++k) since_sort[k] = species_interval[k];
    }

    // One step as a CUDA graph: its kernel parameters depend only on which
    // species are sorted this step and on each species' buffer parity, so the
    // graphs are cached under that key (at most a few per run).
    struct StepGraph {
        unsigned key;
        cudaGraphExec_t exec;
    };
    std::vector<StepGraph> step_graphs;

    void drop_graphs() {
        for (auto& g : step_graphs) cudaGraphExecDestroy(g.exec);
        step_graphs.clear();
    }

    void enqueue_step(unsigned sort_mask) {
        for (int s = 0; s < cfg.nspecies; ++s)
            if (sort_mask >> s & 1u) sort_species(s);
        for (int s = 0; s < cfg.nspecies; ++s) launch_push<kPushStep>(s);
        solve_fields();
    }

    void launch_step_graph(unsigned sort_mask) {
        unsigned key = sort_mask;
        for (int s = 0; s < cfg.nspecies; ++s) key |= (unsigned)buf[s] << (APIC_MAX_SPECIES + s);
        cudaGraphExec_t exec = nullptr;
        for (const auto& g : step_graphs)
            if (g.key == key) exec = g.exec;
        if (!exec) {
            int saved[APIC_MAX_SPECIES];
            for (int s = 0; s < APIC_MAX_SPECIES; ++s) saved[s] = buf[s];
            cudaGraph_t g = nullptr;
            APIC_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            enqueue_step(sort_mask);
            const cudaError_t ce = cudaStreamEndCapture(stream, &g);
            for (int s = 0; s < APIC_MAX_SPECIES; ++s) buf[s] = saved[s];
            APIC_CUDA(ce);
            const cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
            cudaGraphDestroy(g);
            APIC_CUDA(ie);
            step_graphs.push_back({key, exec});
        }
        APIC_CUDA(cudaGraphLaunch(exec, stream));
        for (int s = 0; s < cfg.nspecies; ++s)
            if (sort_mask >> s & 1u) buf[s] ^= 1;
    }

    void do_steps(size_t nsteps) {
        require(initialized, "initialize() or resume() must precede step()", APIC_ERR_STATE);
        for (size_t it = 0; it < nsteps; ++it) {
            unsigned sort_mask = 0;
            for (int s = 0; s < cfg.nspecies; ++s)
                if (!walls && since_sort[s] >= species_interval[s] && sp[s].n) sort_mask |= 1u << s;
            for (int s = 0; s < cfg.nspecies; ++s) {
                if (since_sort[s] < species_interval[s]) continue;
                since_sort[s] = 0;
                if (sp[s].n) launches += fp32 ? 6 : 5;  // histogram, three scan passes, scatter (FP32: rank + gather)
            }
            if (sort_mask) steps_since_sort = 0;
            for (int s = 0; s < cfg.nspecies; ++s)
                if (sp[s].n) ++launches;
            launches += cfg.dims == 2 ? 3 : 5;  // FFT passes
            if (!timing) {
                launch_step_graph(sort_mask);
            } else {
                // kernel by kernel, with events between the phases
                Ev ev{};
                APIC_CUDA(cudaEventCreate(&ev.a)); APIC_CUDA(cudaEventCreate(&ev.b));
                APIC_CUDA(cudaEventCreate(&ev.c)); APIC_CUDA(cudaEventCreate(&ev.d));
                APIC_CUDA(cudaEventRecord(ev.a, stream));
                for (int s = 0; s < cfg.nspecies; ++s)
                    if (sort_mask >> s & 1u) sort_species(s);
                APIC_CUDA(cudaEventRecord(ev.b, stream));
                for (int s = 0; s < cfg.nspecies; ++s) launch_push<kPushStep>(s);
                APIC_CUDA(cudaEventRecord(ev.c, stream));
                solve_fields();
                APIC_CUDA(cudaEventRecord(ev.d, stream));
                ev.sorted = sort_mask != 0;
                events.push_back(ev);
            }
            ++steps_since_sort;
            for (int s = 0; s < cfg.nspecies; ++s) ++since_sort[s];
            time += cfg.dt;
            ++step_count;
        }
    }

    void collect_timing() {
        for (auto& e : events) {
            float t_sort = 0, t_push = 0, t_solve = 0;
            APIC_CUDA(cudaEventElapsedTime(&t_sort, e.a, e.b));
            APIC_CUDA(cudaEventElapsedTime(&t_push, e.b, e.c));
            APIC_CUDA(cudaEventElapsedTime(&t_solve, e.c, e.d));
            sort_ms += t_sort;
            push_ms += t_push;
            solve_ms += t_solve;
            ++timed_steps;
            cudaEventDestroy(e.a); cudaEventDestroy(e.b); cudaEventDestroy(e.c); cudaEventDestroy(e.d);
        }
        events.clear();
    }

    void sync() {
        const cudaError_t e = bounded_wait(stream, 600.0);
        if (e == cudaErrorNotReady) throw Error(APIC_ERR_TIMEOUT, "device work did not complete in time");
        APIC_CUDA(e);
    }

    size_t read_particles(int s, size_t cap, double* pos, double* v, double* vh) {
        require(s >= 0 && s < cfg.nspecies, "species index out of range");
        const SpeciesND& S = sp[s];
        const size_t n = S.n;
        require(cap >= n, "output capacity below the particle count", APIC_ERR_CAPACITY);
        if (fp32) to_fp64(s);
        if (initialized) launch_push<kPushSync>(s);  // time-centred v of the current state
        const int b = buf[s];
        const int o = b ^ 1;
        // un-permute into the other buffer's arrays (free outside a sort)
        double* scratch[7];
        int k = 0;
        for (int a = 0; a < cfg.dims; ++a) scratch[k++] = S.pos[o][a];
        for (int a = 0; a < 3; ++a) scratch[k++] = S.vh[o][a];
        const unsigned blocks = (unsigned)((n + kThreads - 1) / kThreads);
        auto fetch = [&](const double* src, double* host, double* tmp) {
            if (!host || n == 0) return;
            k_unpermute<<<blocks, kThreads, 0, stream>>>(S.id[b], src, tmp, (unsigned)n);
            APIC_CUDA(cudaGetLastError());
            APIC_CUDA(cudaMemcpyAsync(host, tmp, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
            APIC_CUDA(cudaStreamSynchronize(stream));
        };
        for (int a = 0; a < cfg.dims; ++a) fetch(S.pos[b][a], pos ? pos + a * n : nullptr, scratch[0]);
        if (pos && cfg.dims == 2) std::memset(pos + 2 * n, 0, n * sizeof(double));
        for (int a = 0; a < 3; ++a) fetch(S.vh[b][a], vh ? vh + a * n : nullptr, scratch[0]);
        for (int a = 0; a < 3; ++a) fetch(S.v[a], v ? v + a * n : nullptr, scratch[0]);
        sync();
        return n;
    }

    void read_alive(int s, size_t cap, uint8_t* alive) {
        require(s >= 0 && s < cfg.nspecies, "species index out of range");
        const size_t n = sp[s].n;
        require(cap >= n, "output capacity below the particle count", APIC_ERR_CAPACITY);
        sync();
        if (sp[s].alive) APIC_CUDA(cudaMemcpyAsync(alive, sp[s].alive, n, cudaMemcpyDeviceToHost, stream));
        else std::memset(alive, 1, n);
        APIC_CUDA(cudaStreamSynchronize(stream));
    }

    // absorbed counts of species s per side: 4 in 2D, 6 in 3D
    void read_losses(int s, uint64_t* out) {
        require(s >= 0 && s < cfg.nspecies, "species index out of range");
        sync();
        unsigned long long h[6] = {0, 0, 0, 0, 0, 0};
        if (p.losses) APIC_CUDA(cudaMemcpyAsync(h, p.losses + 6 * s, sizeof h, cudaMemcpyDeviceToHost, stream));
        APIC_CUDA(cudaStreamSynchronize(stream));
        for (int k = 0; k < 2 * cfg.dims; ++k) out[k] = h[k];
    }

    void read_fields(double* rho, double* phi, double* E) {
        sync();
        const size_t N = ncells;
        if (rho) APIC_CUDA(cudaMemcpyAsync(rho, solver.F.rho, N * 8, cudaMemcpyDeviceToHost, stream));
        if (phi) APIC_CUDA(cudaMemcpyAsync(phi, solver.F.phi, N * 8, cudaMemcpyDeviceToHost, stream));
        if (E) {
            const int st = cfg.dims == 2 ? 2 : 4;
            std::vector<double> h(N * st);
            APIC_CUDA(cudaMemcpyAsync(h.data(), solver.F.E, N * st * 8, cudaMemcpyDeviceToHost, stream));
            APIC_CUDA(cudaStreamSynchronize(stream));
            for (int c = 0; c < cfg.dims; ++c)
                for (size_t g = 0; g < N; ++g) E[c * N + g] = h[g * st + c];
        }
        APIC_CUDA(cudaStreamSynchronize(stream));
    }

    void sample(apic_sample_nd* out) {
        std::memset(out, 0, sizeof *out);
        double vol = 1.0;
        for (int a = 0; a < cfg.dims; ++a) vol *= p.d[a];
        if (cfg.dims == 2) vol *= (cfg.out_of_plane_depth == 0.0 ? 1.0 : cfg.out_of_plane_depth);
        for (int s = 0; s < cfg.nspecies; ++s) {
            if (initialized) launch_push<kPushSync>(s);
            k_sample_nd<<<kSampleBlocks, 256, 0, stream>>>(sp[s], cfg.dims, sample_partial, sample_done, sample_out,
                                                           solver.F.E, solver.F.rho, (long long)ncells,
                                                           0.5 * p.eps * vol, vol, s, s == cfg.nspecies - 1,
                                                           p.wall[0], p.wall[1], p.wall[2], p.n[0], p.n[1], p.n[2]);
            APIC_CUDA(cudaGetLastError());
        }
        double h[8];
        unsigned long long lost[6 * APIC_MAX_SPECIES] = {};
        APIC_CUDA(cudaMemcpyAsync(h, sample_out, sizeof h, cudaMemcpyDeviceToHost, stream));
        if (p.losses) APIC_CUDA(cudaMemcpyAsync(lost, p.losses, sizeof lost, cudaMemcpyDeviceToHost, stream));
        sync();
        for (int s = 0; s < cfg.nspecies; ++s) {
            out->kinetic_by_species[s] = h[s];
            out->kinetic_energy += h[s];
            // live_count: absorbed particles stay in place, flagged dead, each counted once in the ledger
            uint64_t dead = 0;
            for (int k = 0; k < 6; ++k) dead += lost[6 * s + k];
            out->live_particles += sp[s].n - dead;
        }
        out->field_energy = h[4];
        out->charge_l1 = h[5];
        out->total_energy = out->kinetic_energy + out->field_energy;
        out->step = step_count;
        out->time = time;
    }
};

}  // namespace nd
}  // namespace apic

// ---- 2D solve with one periodic axis ------------------------------------------------
//
// FieldSolver::solve(Mesh2D&) for a mesh with exactly one periodic axis
// (solve_mixed_spectral_tridiagonal, src/FieldSolver.cpp:501-657): every row
// along the periodic axis is Fourier transformed, each mode solves a
// tridiagonal system across the wall axis (discrete eigenvalue
// 4 sin^2(pi m / N) / h^2 of the periodic second difference, wall potentials on
// mode 0 scaled by N), the rows are transformed back, and E follows from the
// finite differences of compute_electric_field (src/FieldSolver.cpp:298-346).
// The spectra are stored wall-row-major (hat[d * np + m]) so that the one
// thread per mode of the tridiagonal kernel reads and writes coalesced rows.

namespace apic {
namespace nd {

__device__ __forceinline__ size_t mixed_index(int d, int q, int nx, int periodic_y) {
    return periodic_y ? (size_t)q * nx + d : (size_t)d * nx + q;
}

__global__ void __launch_bounds__(kFftThreads) k_mixed_forward(const double* __restrict__ rho, Cplx* __restrict__ hat,
                                                               int nx, int np, int periodic_y, const Cplx* tw) {
    extern __shared__ __align__(16) unsigned char msm[];
    Cplx* a = reinterpret_cast<Cplx*>(msm);
    Cplx* b = a + np;
    Cplx* tws = b + np;
    const int d = blockIdx.x;
    for (int q = threadIdx.x; q < np; q += blockDim.x) {
        tws[q] = tw[q];
        a[q] = {rho[mixed_index(d, q, nx, periodic_y)], 0.0};
    }
    __syncthreads();
    const Cplx* r = fft_lines(a, b, 1, np, tws, false);
    for (int m = threadIdx.x; m < np; m += blockDim.x) hat[(size_t)d * np + m] = r[m];
}

// One thread per mode: the forward sweep keeps modified_rhs in place of
// rho_hat and modified_upper (real for these real coefficients) in mu; the
// back substitution leaves phi_hat in hat.
__global__ void k_mixed_tridiag(Cplx* __restrict__ hat, double* __restrict__ mu, int nd, int np, double inv_dsq,
                                double inv_psq, double eps, double lower, double upper) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= np) return;
    const int ni = nd - 2;
    const double angle = 3.141592653589793 * (double)m / (double)np;
    const double eig = 4.0 * sin(angle) * sin(angle) * inv_psq;
    const double diag = 2.0 * inv_dsq + eig;
    const double off = -inv_dsq;
    const double scale = (double)np;
    const double lb = m == 0 ? lower * scale : 0.0, ub = m == 0 ? upper * scale : 0.0;
    double pr = 0.0, pi = 0.0, pu = 0.0;  // modified_rhs and modified_upper of the previous row
    for (int k = 0; k < ni; ++k) {
        const Cplx rh = hat[(size_t)(k + 1) * np + m];
        double rr = rh.re / eps, ri = rh.im / eps;
        if (k == 0) rr += inv_dsq * lb;
        if (k + 1 == ni) rr += inv_dsq * ub;
        double u, xr, xi;
        if (k == 0) {
            u = off / diag;
            xr = rr / diag;
            xi = ri / diag;
        } else {
            const double den = diag - off * pu;
            u = k + 1 == ni ? 0.0 : off / den;
            xr = (rr - off * pr) / den;
            xi = (ri - off * pi) / den;
        }
        hat[(size_t)(k + 1) * np + m] = {xr, xi};
        mu[(size_t)k * np + m] = u;
        pr = xr; pi = xi; pu = u;
    }
    hat[m] = {lb, 0.0};
    hat[(size_t)(nd - 1) * np + m] = {ub, 0.0};
    for (int k = ni - 2; k >= 0; --k) {
        const Cplx nxt = hat[(size_t)(k + 2) * np + m];
        const Cplx cur = hat[(size_t)(k + 1) * np + m];
        const double u = mu[(size_t)k * np + m];
        hat[(size_t)(k + 1) * np + m] = {cur.re - u * nxt.re, cur.im - u * nxt.im};
    }
}

// The elimination coefficients of every mode's system depend on the mode
// only: modified_upper mu[m * ni + k] and the reciprocal of the pivot
// inv[m * ni + k], computed once per mesh with the arithmetic of the sweep above.
__global__ void k_mixed_coeffs(double* __restrict__ mu, double* __restrict__ inv, int nd, int np, double inv_dsq,
                               double inv_psq) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= np) return;
    const int ni = nd - 2;
    const double angle = 3.141592653589793 * (double)m / (double)np;
    const double eig = 4.0 * sin(angle) * sin(angle) * inv_psq;
    const double diag = 2.0 * inv_dsq + eig;
    const double off = -inv_dsq;
    double pu = 0.0;
    for (int k = 0; k < ni; ++k) {
        const double den = k == 0 ? diag : diag - off * pu;
        const double u = k == 0 ? off / diag : (k + 1 == ni ? 0.0 : off / den);
        mu[(size_t)m * ni + k] = u;
        inv[(size_t)m * ni + k] = 1.0 / den;
        pu = u;
    }
}

// One mode's forward elimination and back substitution per CTA, on its column
// staged in shared memory: with the coefficients precomputed, each row is two
// multiply-adds on the chain, and the column's rows are loaded all at once
// instead of one dependent global round trip per row.
__global__ void __launch_bounds__(32) k_mixed_sweep(Cplx* __restrict__ hat, const double* __restrict__ mu,
                                                    const double* __restrict__ inv, int nd, int np, double inv_dsq,
                                                    double eps, double lower, double upper) {
    extern __shared__ __align__(16) unsigned char ssm[];
    const int m = blockIdx.x, ni = nd - 2, tid = threadIdx.x;
    Cplx* R = reinterpret_cast<Cplx*>(ssm);
    Cplx* X = R + ni;
    double* U = reinterpret_cast<double*>(X + ni);
    double* V = U + ni;
    for (int k = tid; k < ni; k += 32) {
        R[k] = hat[(size_t)(k + 1) * np + m];
        U[k] = mu[(size_t)m * ni + k];
        V[k] = inv[(size_t)m * ni + k];
    }
    __syncthreads();
    const double off = -inv_dsq, ieps = 1.0 / eps;
    const double scale = (double)np;
    const double lb = m == 0 ? lower * scale : 0.0, ub = m == 0 ? upper * scale : 0.0;
    if (tid == 0) {
        double pr = 0.0, pi = 0.0;
#pragma unroll 4
        for (int k = 0; k < ni; ++k) {
            const Cplx rh = R[k];
            double rr = rh.re * ieps, ri = rh.im * ieps;
            if (k == 0) rr += inv_dsq * lb;
            if (k + 1 == ni) rr += inv_dsq * ub;
            const double xr = (k == 0 ? rr : rr - off * pr) * V[k];
            const double xi = (k == 0 ? ri : ri - off * pi) * V[k];
            X[k] = {xr, xi};
            pr = xr;
            pi = xi;
        }
        Cplx xn = X[ni - 1];
#pragma unroll 4
        for (int k = ni - 2; k >= 0; --k) {
            const Cplx c = X[k];
            const double u = U[k];
            xn = {c.re - u * xn.re, c.im - u * xn.im};
            X[k] = xn;
        }
    }
    __syncthreads();
    for (int k = tid; k < ni; k += 32) hat[(size_t)(k + 1) * np + m] = X[k];
    if (tid == 0) {
        hat[m] = {lb, 0.0};
        hat[(size_t)(nd - 1) * np + m] = {ub, 0.0};
    }
}

__global__ void __launch_bounds__(kFftThreads) k_mixed_inverse(const Cplx* __restrict__ hat, double* __restrict__ phi,
                                                               int nx, int np, int periodic_y, const Cplx* tw) {
    extern __shared__ __align__(16) unsigned char msm[];
    Cplx* a = reinterpret_cast<Cplx*>(msm);
    Cplx* b = a + np;
    Cplx* tws = b + np;
    const int d = blockIdx.x;
    for (int m = threadIdx.x; m < np; m += blockDim.x) {
        tws[m] = tw[m];
        a[m] = hat[(size_t)d * np + m];
    }
    __syncthreads();
    const Cplx* r = fft_lines(a, b, 1, np, tws, true);
    for (int q = threadIdx.x; q < np; q += blockDim.x) phi[mixed_index(d, q, nx, periodic_y)] = r[q].re;
}

// compute_electric_field(Mesh2D&), src/FieldSolver.cpp:298-346
__global__ void k_mixed_efield(const double* __restrict__ phi, double* __restrict__ E, int nx, int ny, double dx,
                               double dy, int periodic_x, int periodic_y) {
    const size_t N = (size_t)nx * ny;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < N; idx += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(idx % nx), j = (int)(idx / nx);
        const size_t row = (size_t)j * nx;
        double ex, ey;
        if (periodic_x) ex = -(phi[row + (i + 1) % nx] - phi[row + (i + nx - 1) % nx]) / (2.0 * dx);
        else if (i == 0) ex = -(phi[row + 1] - phi[idx]) / dx;
        else if (i + 1 == nx) ex = -(phi[idx] - phi[row + i - 1]) / dx;
        else ex = -(phi[row + i + 1] - phi[row + i - 1]) / (2.0 * dx);
        if (periodic_y) ey = -(phi[(size_t)((j + 1) % ny) * nx + i] - phi[(size_t)((j + ny - 1) % ny) * nx + i]) / (2.0 * dy);
        else if (j == 0) ey = -(phi[(size_t)nx + i] - phi[idx]) / dy;
        else if (j + 1 == ny) ey = -(phi[idx] - phi[row - nx + i]) / dy;
        else ey = -(phi[row + nx + i] - phi[row - nx + i]) / (2.0 * dy);
        E[idx] = ex;
        E[N + idx] = ey;
    }
}

// device arrays and stream of one call, released on every exit path
struct MixedScratch {
    cudaStream_t s = nullptr;
    std::vector<void*> a;
    ~MixedScratch() {
        if (s) cudaStreamSynchronize(s);
        for (void* p : a) cudaFree(p);
        if (s) cudaStreamDestroy(s);
    }
    template <class T>
    T* get(size_t count) {
        void* p = nullptr;
        APIC_CUDA(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
        a.push_back(p);
        return static_cast<T*>(p);
    }
};

static void solve_mixed_2d(const size_t* n, const double* length, int periodic_axis, double permittivity,
                           double lower, double upper, const double* rho, double* phi, double* electric) {
    require(n && length && rho && phi && electric, "null argument");
    require(periodic_axis == 0 || periodic_axis == 1, "periodic_axis must be 0 (x) or 1 (y)");
    require(std::isfinite(permittivity) && permittivity > 0, "field-solver permittivity must be positive and finite");
    require(std::isfinite(lower) && std::isfinite(upper), "wall potentials must be finite");
    const int periodic_y = periodic_axis == 1;
    const size_t nx = n[0], ny = n[1];
    const size_t nd = periodic_y ? nx : ny, np = periodic_y ? ny : nx;
    require(nd >= 3, "the wall axis needs at least 3 nodes");
    require(pow2(np) && np <= (size_t)kMaxLine, "the periodic extent must be a power of two up to 1024",
            APIC_ERR_UNSUPPORTED);
    for (int a = 0; a < 2; ++a)
        require(std::isfinite(length[a]) && length[a] > 0, "domain lengths must be positive and finite");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        throw Error(APIC_ERR_NO_DEVICE, "no CUDA device is visible");
    // Mesh2D spacings, src/Mesh2D.cpp:57-60
    const double dx = length[0] / (double)(periodic_y ? nx - 1 : nx);
    const double dy = length[1] / (double)(periodic_y ? ny : ny - 1);
    const double hd = periodic_y ? dx : dy, hp = periodic_y ? dy : dx;
    const size_t N = nx * ny;
    MixedScratch S;
    APIC_CUDA(cudaStreamCreateWithFlags(&S.s, cudaStreamNonBlocking));
    double* d_rho = S.get<double>(N);
    double* d_phi = S.get<double>(N);
    double* d_E = S.get<double>(2 * N);
    double* d_mu = S.get<double>(N);
    Cplx* d_hat = S.get<Cplx>(N);
    Cplx* d_tw = S.get<Cplx>(np);
    std::vector<Cplx> tw(np);
    const double twopi = 2.0 * 3.141592653589793;
    for (size_t k = 0; k < np; ++k) tw[k] = {std::cos(twopi * k / np), -std::sin(twopi * k / np)};
    APIC_CUDA(cudaMemcpyAsync(d_tw, tw.data(), np * sizeof(Cplx), cudaMemcpyHostToDevice, S.s));
    APIC_CUDA(cudaMemcpyAsync(d_rho, rho, N * sizeof(double), cudaMemcpyHostToDevice, S.s));
    const size_t smem = 3 * np * sizeof(Cplx);
    ensure_solver_attributes();
    k_mixed_forward<<<(unsigned)nd, kFftThreads, smem, S.s>>>(d_rho, d_hat, (int)nx, (int)np, periodic_y, d_tw);
    if (nd - 2 <= (size_t)kMixedSweepMaxRows) {
        double* d_inv = S.get<double>(N);
        k_mixed_coeffs<<<(unsigned)((np + 127) / 128), 128, 0, S.s>>>(d_mu, d_inv, (int)nd, (int)np, 1.0 / (hd * hd),
                                                                        1.0 / (hp * hp));
        k_mixed_sweep<<<(unsigned)np, 32, (nd - 2) * 48, S.s>>>(d_hat, d_mu, d_inv, (int)nd, (int)np, 1.0 / (hd * hd),
                                                                 permittivity, lower, upper);
    } else {
        k_mixed_tridiag<<<(unsigned)((np + 127) / 128), 128, 0, S.s>>>(d_hat, d_mu, (int)nd, (int)np, 1.0 / (hd * hd),
                                                                         1.0 / (hp * hp), permittivity, lower, upper);
    }
    k_mixed_inverse<<<(unsigned)nd, kFftThreads, smem, S.s>>>(d_hat, d_phi, (int)nx, (int)np, periodic_y, d_tw);
    k_mixed_efield<<<(unsigned)std::min<size_t>((N + 255) / 256, 4096), 256, 0, S.s>>>(
        d_phi, d_E, (int)nx, (int)ny, dx, dy, periodic_y ? 0 : 1, periodic_y);
    APIC_CUDA(cudaGetLastError());
    APIC_CUDA(cudaMemcpyAsync(phi, d_phi, N * sizeof(double), cudaMemcpyDeviceToHost, S.s));
    APIC_CUDA(cudaMemcpyAsync(electric, d_E, 2 * N * sizeof(double), cudaMemcpyDeviceToHost, S.s));
    const cudaError_t e = bounded_wait(S.s, 600.0);
    if (e == cudaErrorNotReady) throw Error(APIC_ERR_TIMEOUT, "device work did not complete in time");
    APIC_CUDA(e);
}

// ---- fully Dirichlet 2D / 3D solve --------------------------------------------------
//
// FieldSolver::solve(Mesh2D&/Mesh3D&) on meshes with walls on every side.  The
// reference iterates SOR to a 1e-11 update (solve_dirichlet_iterative,
// src/FieldSolver.cpp:761-907); here the same discrete system is solved directly:
// the discrete sine transform (DST-I) diagonalises the Dirichlet second
// difference of each axis (eigenvalues 4 sin^2(pi m / (2 (M + 1))) / h^2 over the
// M interior nodes), so the interior potential is three DST passes, a division
// and three more DST passes, each DST-I an odd-extended complex FFT of length
// 2 (M + 1).  Wall potentials (2D sides, corners the mean of their two sides;
// 3D grounded) enter the right-hand side of the nodes next to the walls.

// interior right-hand side, compact [Mz][My][Mx]
__global__ void k_dir_rhs(const double* __restrict__ rho, double* __restrict__ u, int nx, int ny, int nz3, double eps,
                          double idx2, double idy2, double left, double right, double bottom, double top) {
    const int Mx = nx - 2, My = ny - 2, Mz = nz3 > 1 ? nz3 - 2 : 1;
    const size_t M = (size_t)Mx * My * Mz;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < M; q += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(q % Mx), j = (int)((q / Mx) % My), k = (int)(q / ((size_t)Mx * My));
        const size_t node = ((size_t)(nz3 > 1 ? k + 1 : 0) * ny + (j + 1)) * nx + (i + 1);
        double b = rho[node] / eps;
        if (nz3 == 1) {  // 2D walls at their potentials; 3D walls are grounded
            if (i == 0) b += left * idx2;
            if (i == Mx - 1) b += right * idx2;
            if (j == 0) b += bottom * idy2;
            if (j == My - 1) b += top * idy2;
        }
        u[q] = b;
    }
}

// DST-I of lines of M values (u[base + k * stride]) in place: one CTA per line,
// X_m = sum_k x_k sin(pi k m / (M + 1)) = -Im(FFT(odd extension))_m / 2.
__global__ void __launch_bounds__(kFftThreads) k_dst_lines(double* __restrict__ u, int M, long long stride, int lines_a,
                                                           long long stride_a, long long stride_b, const Cplx* tw) {
    extern __shared__ __align__(16) unsigned char dsm[];
    const int N = 2 * (M + 1);
    Cplx* a = reinterpret_cast<Cplx*>(dsm);
    Cplx* b = a + N;
    Cplx* tws = b + N;
    const long long l = blockIdx.x;
    const long long base = (l % lines_a) * stride_a + (l / lines_a) * stride_b;
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
        tws[k] = tw[k];
        double v = 0.0;
        if (k >= 1 && k <= M) v = u[base + (long long)(k - 1) * stride];
        else if (k >= M + 2) v = -u[base + (long long)(N - k - 1) * stride];
        a[k] = {v, 0.0};
    }
    __syncthreads();
    const Cplx* r = fft_lines(a, b, 1, N, tws, false);
    for (int m = threadIdx.x + 1; m <= M; m += blockDim.x) u[base + (long long)(m - 1) * stride] = -0.5 * r[m].im;
}

// divide by the eigenvalues of minus the discrete Laplacian; scale folds in the
// inverse-DST normalisation 2 / (M + 1) of every axis
__global__ void k_dir_divide(double* __restrict__ u, int Mx, int My, int Mz, double idx2, double idy2, double idz2,
                             double scale) {
    const size_t M = (size_t)Mx * My * Mz;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < M; q += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(q % Mx), j = (int)((q / Mx) % My), k = (int)(q / ((size_t)Mx * My));
        const double sx = sin(3.141592653589793 * (i + 1) / (2.0 * (Mx + 1)));
        const double sy = sin(3.141592653589793 * (j + 1) / (2.0 * (My + 1)));
        double lam = 4.0 * sx * sx * idx2 + 4.0 * sy * sy * idy2;
        if (Mz > 1 || idz2 > 0.0) {
            const double sz = sin(3.141592653589793 * (k + 1) / (2.0 * (Mz + 1)));
            lam += 4.0 * sz * sz * idz2;
        }
        u[q] *= scale / lam;
    }
}

// the full mesh: wall nodes (apply_dirichlet_boundary_potentials,
// src/FieldSolver.cpp:267-296, or grounded in 3D) and the interior solution
__global__ void k_dir_assemble(const double* __restrict__ u, double* __restrict__ phi, int nx, int ny, int nz3,
                               double left, double right, double bottom, double top) {
    const size_t N = (size_t)nx * ny * nz3;
    const int Mx = nx - 2, My = ny - 2;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < N; q += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(q % nx), j = (int)((q / nx) % ny), k = (int)(q / ((size_t)nx * ny));
        const bool wi = i == 0 || i == nx - 1, wj = j == 0 || j == ny - 1, wk = nz3 > 1 && (k == 0 || k == nz3 - 1);
        double v;
        if (!wi && !wj && !wk) {
            v = u[((size_t)(nz3 > 1 ? k - 1 : 0) * My + (j - 1)) * Mx + (i - 1)];
        } else if (nz3 > 1) {
            v = 0.0;
        } else if (wi && wj) {
            v = 0.5 * ((i == 0 ? left : right) + (j == 0 ? bottom : top));
        } else if (wj) {
            v = j == 0 ? bottom : top;
        } else {
            v = i == 0 ? left : right;
        }
        phi[q] = v;
    }
}

// 3D E by differences, one-sided at the walls (src/FieldSolver.cpp:872-904)
__global__ void k_dir_efield3(const double* __restrict__ phi, double* __restrict__ E, int nx, int ny, int nz, double dx,
                              double dy, double dz) {
    const size_t N = (size_t)nx * ny * nz, sy = nx, sz = (size_t)nx * ny;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < N; q += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(q % nx), j = (int)((q / nx) % ny), k = (int)(q / sz);
        double ex, ey, ez;
        if (i == 0) ex = -(phi[q + 1] - phi[q]) / dx;
        else if (i + 1 == nx) ex = -(phi[q] - phi[q - 1]) / dx;
        else ex = -(phi[q + 1] - phi[q - 1]) / (2.0 * dx);
        if (j == 0) ey = -(phi[q + sy] - phi[q]) / dy;
        else if (j + 1 == ny) ey = -(phi[q] - phi[q - sy]) / dy;
        else ey = -(phi[q + sy] - phi[q - sy]) / (2.0 * dy);
        if (k == 0) ez = -(phi[q + sz] - phi[q]) / dz;
        else if (k + 1 == nz) ez = -(phi[q] - phi[q - sz]) / dz;
        else ez = -(phi[q + sz] - phi[q - sz]) / (2.0 * dz);
        E[q] = ex;
        E[N + q] = ey;
        E[2 * N + q] = ez;
    }
}

static void solve_dirichlet_nd(int dims, const size_t* n, const double* length, double permittivity,
                               const double* pot, const double* rho, double* phi, double* electric) {
    require(dims == 2 || dims == 3, "dims must be 2 or 3");
    require(n && length && rho && phi && electric, "null argument");
    require(std::isfinite(permittivity) && permittivity > 0, "field-solver permittivity must be positive and finite");
    double side[4] = {0.0, 0.0, 0.0, 0.0};
    if (pot) {
        for (int a = 0; a < 4; ++a) {
            require(std::isfinite(pot[a]), "wall potentials must be finite");
            side[a] = pot[a];
        }
        require(dims == 2 || (side[0] == 0.0 && side[1] == 0.0 && side[2] == 0.0 && side[3] == 0.0),
                "3D Dirichlet walls are grounded");
    }
    size_t N = 1, Mtot = 1;
    for (int a = 0; a < dims; ++a) {
        require(n[a] >= 3 && pow2(n[a] - 1) && 2 * (n[a] - 1) <= (size_t)kMaxLine,
                "each extent must be 2^k + 1 nodes, 3 to 513", APIC_ERR_UNSUPPORTED);
        require(std::isfinite(length[a]) && length[a] > 0, "domain lengths must be positive and finite");
        N *= n[a];
        Mtot *= n[a] - 2;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        throw Error(APIC_ERR_NO_DEVICE, "no CUDA device is visible");
    const int nx = (int)n[0], ny = (int)n[1], nz3 = dims == 3 ? (int)n[2] : 1;
    const int Mx = nx - 2, My = ny - 2, Mz = dims == 3 ? nz3 - 2 : 1;
    // Mesh2D / Mesh3D Dirichlet spacing L / (n - 1)
    const double dx = length[0] / (double)(nx - 1), dy = length[1] / (double)(ny - 1);
    const double dz = dims == 3 ? length[2] / (double)(nz3 - 1) : 1.0;
    const double idx2 = 1.0 / (dx * dx), idy2 = 1.0 / (dy * dy), idz2 = dims == 3 ? 1.0 / (dz * dz) : 0.0;
    MixedScratch S;
    APIC_CUDA(cudaStreamCreateWithFlags(&S.s, cudaStreamNonBlocking));
    double* d_rho = S.get<double>(N);
    double* d_phi = S.get<double>(N);
    double* d_E = S.get<double>((size_t)dims * N);
    double* d_u = S.get<double>(Mtot);
    const int M[3] = {Mx, My, Mz};
    Cplx* d_tw[3] = {nullptr, nullptr, nullptr};
    for (int a = 0; a < dims; ++a) {
        const int L2 = 2 * (M[a] + 1);
        std::vector<Cplx> tw(L2);
        const double twopi = 2.0 * 3.141592653589793;
        for (int k = 0; k < L2; ++k) tw[k] = {std::cos(twopi * k / L2), -std::sin(twopi * k / L2)};
        d_tw[a] = S.get<Cplx>(L2);
        APIC_CUDA(cudaMemcpyAsync(d_tw[a], tw.data(), L2 * sizeof(Cplx), cudaMemcpyHostToDevice, S.s));
    }
    APIC_CUDA(cudaMemcpyAsync(d_rho, rho, N * sizeof(double), cudaMemcpyHostToDevice, S.s));
    const unsigned g = (unsigned)std::min<size_t>((N + 255) / 256, 4096);
    k_dir_rhs<<<g, 256, 0, S.s>>>(d_rho, d_u, nx, ny, nz3, permittivity, idx2, idy2, side[0], side[1], side[2],
                                  side[3]);
    ensure_solver_attributes();
    // axis a: element stride, then the two line axes (stride_a over lines_a, stride_b over the rest)
    auto dst_axis = [&](int a) {
        const long long sx = 1, sy = Mx, sz = (long long)Mx * My;
        long long stride, stride_a, stride_b;
        int lines_a;
        size_t lines;
        if (a == 0) { stride = sx; lines_a = My; stride_a = sy; stride_b = sz; lines = (size_t)My * Mz; }
        else if (a == 1) { stride = sy; lines_a = Mx; stride_a = sx; stride_b = sz; lines = (size_t)Mx * Mz; }
        else { stride = sz; lines_a = Mx; stride_a = sx; stride_b = sy; lines = (size_t)Mx * My; }
        const size_t smem = 3 * (size_t)(2 * (M[a] + 1)) * sizeof(Cplx);
        k_dst_lines<<<(unsigned)lines, kFftThreads, smem, S.s>>>(d_u, M[a], stride, lines_a, stride_a, stride_b, d_tw[a]);
    };
    for (int a = 0; a < dims; ++a) dst_axis(a);
    double scale = 1.0;
    for (int a = 0; a < dims; ++a) scale *= 2.0 / (double)(M[a] + 1);
    k_dir_divide<<<g, 256, 0, S.s>>>(d_u, Mx, My, Mz, idx2, idy2, idz2, scale);
    for (int a = 0; a < dims; ++a) dst_axis(a);
    k_dir_assemble<<<g, 256, 0, S.s>>>(d_u, d_phi, nx, ny, nz3, side[0], side[1], side[2], side[3]);
    if (dims == 2) k_mixed_efield<<<g, 256, 0, S.s>>>(d_phi, d_E, nx, ny, dx, dy, 0, 0);
    else k_dir_efield3<<<g, 256, 0, S.s>>>(d_phi, d_E, nx, ny, nz3, dx, dy, dz);
    APIC_CUDA(cudaGetLastError());
    APIC_CUDA(cudaMemcpyAsync(phi, d_phi, N * sizeof(double), cudaMemcpyDeviceToHost, S.s));
    APIC_CUDA(cudaMemcpyAsync(electric, d_E, (size_t)dims * N * sizeof(double), cudaMemcpyDeviceToHost, S.s));
    const cudaError_t e = bounded_wait(S.s, 600.0);
    if (e == cudaErrorNotReady) throw Error(APIC_ERR_TIMEOUT, "device work did not complete in time");
    APIC_CUDA(e);
}

}  // namespace nd
}  // namespace apic

// ---- C ABI ---------------------------------------------------------------------------

struct apic_sim_nd {
    apic::nd::SimND impl;
};

namespace {
thread_local std::string g_nd_error;

template <class F>
int guarded_nd(apic_sim_nd* h, F&& f) {
    try {
        f();
        return APIC_OK;
    } catch (const apic::Error& e) {
        if (h) h->impl.last_error = e.what();
        g_nd_error = e.what();
        return e.status;
    } catch (const std::exception& e) {
        if (h) h->impl.last_error = e.what();
        g_nd_error = e.what();
        return APIC_ERR_INVALID;
    }
}
}  // namespace

extern "C" {

int apic_simnd_create(const apic_config_nd* cfg, apic_sim_nd** out) {
    if (!cfg || !out) return APIC_ERR_INVALID;
    *out = nullptr;
    auto h = std::make_unique<apic_sim_nd>();
    const int rc = guarded_nd(h.get(), [&] { h->impl.create(*cfg); });
    if (rc == APIC_OK) *out = h.release();
    return rc;
}

void apic_simnd_destroy(apic_sim_nd* sim) { delete sim; }

const char* apic_simnd_last_error(const apic_sim_nd* sim) {
    return sim ? sim->impl.last_error.c_str() : g_nd_error.c_str();
}

int apic_simnd_load_particles(apic_sim_nd* sim, int species, size_t n, const double* pos, const double* v,
                              const double* v_half) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded_nd(sim, [&] { sim->impl.load(species, n, pos, v, v_half); });
}

int apic_simnd_load_maxwellian(apic_sim_nd* sim, int species, size_t n, uint64_t seed, double thermal_speed,
                               double drift_x, int perturb_axis, double perturb_amplitude) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded_nd(sim, [&] {
        sim->impl.load_maxwellian(species, n, seed, thermal_speed, drift_x, perturb_axis, perturb_amplitude);
    });
}

int apic_simnd_initialize(apic_sim_nd* sim) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded_nd(sim, [&] { sim->impl.initialize(); });
}

int apic_simnd_resume(apic_sim_nd* sim, double time, uint64_t step) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded_nd(sim, [&] { sim->impl.resume(time, step); });
}

int apic_simnd_step(apic_sim_nd* sim, size_t nsteps) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded_nd(sim, [&] { sim->impl.do_steps(nsteps); });
}

int apic_simnd_synchronize(apic_sim_nd* sim) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded_nd(sim, [&] { sim->impl.sync(); });
}

int apic_simnd_count(apic_sim_nd* sim, int species, size_t* n) {
    if (!sim || !n || species < 0 || species >= sim->impl.cfg.nspecies) return APIC_ERR_INVALID;
    *n = sim->impl.sp[species].n;
    return APIC_OK;
}

int apic_simnd_read_particles(apic_sim_nd* sim, int species, size_t capacity, double* pos, double* v, double* v_half,
                              size_t* n) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded_nd(sim, [&] {
        const size_t got = sim->impl.read_particles(species, capacity, pos, v, v_half);
        if (n) *n = got;
    });
}

int apic_simnd_read_fields(apic_sim_nd* sim, double* rho, double* phi, double* electric) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded_nd(sim, [&] { sim->impl.read_fields(rho, phi, electric); });
}
int apic_simnd_read_alive(apic_sim_nd* sim, int species, size_t capacity, uint8_t* alive) {
    if (!sim || !alive) return APIC_ERR_INVALID;
    return guarded_nd(sim, [&] { sim->impl.read_alive(species, capacity, alive); });
}
int apic_simnd_boundary_losses(apic_sim_nd* sim, int species, uint64_t* absorbed) {
    if (!sim || !absorbed) return APIC_ERR_INVALID;
    return guarded_nd(sim, [&] { sim->impl.read_losses(species, absorbed); });
}

int apic_simnd_sample(apic_sim_nd* sim, apic_sample_nd* out) {
    if (!sim || !out) return APIC_ERR_INVALID;
    return guarded_nd(sim, [&] { sim->impl.sample(out); });
}

int apic_simnd_cuda_stream(apic_sim_nd* sim, void** stream) {
    if (!sim || !stream) return APIC_ERR_INVALID;
    *stream = (void*)sim->impl.stream;
    return APIC_OK;
}

int apic_simnd_set_kernel_timing(apic_sim_nd* sim, int enable) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded_nd(sim, [&] {
        sim->impl.sync();
        sim->impl.collect_timing();
        sim->impl.timing = enable != 0;
        sim->impl.push_ms = sim->impl.solve_ms = sim->impl.sort_ms = 0;
        sim->impl.timed_steps = 0;
    });
}

int apic_simnd_kernel_times(apic_sim_nd* sim, double* push_ms, double* solve_ms, double* sort_ms, uint64_t* steps) {
    if (!sim) return APIC_ERR_INVALID;
    return guarded_nd(sim, [&] {
        sim->impl.sync();
        sim->impl.collect_timing();
        if (push_ms) *push_ms = sim->impl.push_ms;
        if (solve_ms) *solve_ms = sim->impl.solve_ms;
        if (sort_ms) *sort_ms = sim->impl.sort_ms;
        if (steps) *steps = sim->impl.timed_steps;
    });
}

int apic_simnd_launch_count(apic_sim_nd* sim, uint64_t* launches) {
    if (!sim || !launches) return APIC_ERR_INVALID;
    return guarded_nd(sim, [&] { *launches = sim->impl.launches; });
}

int apic_field_solve_periodic_nd(int dims, const size_t* n, const double* length, double permittivity,
                                 const double* rho, double* phi, double* electric) {
    return guarded_nd(nullptr, [&] {
        apic::require(dims == 2 || dims == 3, "dims must be 2 or 3");
        apic::require(std::isfinite(permittivity) && permittivity > 0,
                      "field-solver permittivity must be positive and finite");
        apic_config_nd c{};
        c.dims = dims;
        for (int a = 0; a < dims; ++a) { c.n[a] = n[a]; c.length[a] = length[a]; }
        c.dt = 1.0;
        c.units = APIC_NORMALIZED;
        c.relative_permittivity = permittivity;
        c.nspecies = 1;
        c.species[0] = {1.0, 1.0, 1.0, 1};
        apic::nd::SimND S;
        S.create(c);
        size_t N = 1;
        for (int a = 0; a < dims; ++a) N *= n[a];
        double* d_rho = S.dalloc<double>(N);
        APIC_CUDA(cudaMemcpyAsync(d_rho, rho, N * 8, cudaMemcpyHostToDevice, S.stream));
        S.solver.F.rho_in = d_rho;
        S.solver.solve();
        S.read_fields(nullptr, phi, electric);
    });
}

int apic_field_solve_dirichlet_nd(int dims, const size_t* n, const double* length, double permittivity,
                                  const double* side_potentials, const double* rho, double* phi, double* electric) {
    return guarded_nd(nullptr, [&] {
        apic::nd::solve_dirichlet_nd(dims, n, length, permittivity, side_potentials, rho, phi, electric);
    });
}

int apic_field_solve_mixed_2d(const size_t* n, const double* length, int periodic_axis, double permittivity,
                              double lower_potential, double upper_potential, const double* rho, double* phi,
                              double* electric) {
    return guarded_nd(nullptr, [&] { apic::nd::solve_mixed_2d(n, length, periodic_axis, permittivity,
                                                              lower_potential, upper_potential, rho, phi, electric); });
}

}  // extern "C"

// ---- allocation-free periodic field solve --------------------------------------
//
// Some callers cannot call cudaMalloc: hosts that own every byte of device
// memory through their own pool or arena, and time-stepping loops that must not
// hit cudaMalloc's implicit device synchronisation (or run where allocation is
// not allowed).  apic_field_solve_periodic_nd_noalloc serves them: the caller
// passes device buffers for rho, phi and E, and the FFT work arrays live in the
// file-scope device array below, which every GPU that loads this library keeps
// until the process exits.

namespace apic {
namespace nd {

constexpr size_t kNoAllocMaxPoints = 65536;  // largest mesh (nx * ny * nz) the array serves
constexpr size_t kNoAllocMaxLine = 1024;     // largest extent per axis
// W, A, B (complex), interleaved E (4 doubles), rho copy, and three twiddle tables
constexpr size_t kNoAllocScratchBytes =
    3 * kNoAllocMaxPoints * sizeof(Cplx) + 4 * kNoAllocMaxPoints * sizeof(double) +
    kNoAllocMaxPoints * sizeof(double) + 3 * kNoAllocMaxLine * sizeof(Cplx);

static __device__ __align__(256) unsigned char g_solve_scratch[kNoAllocScratchBytes];

// exp(-2 pi i k / n), k < n
__global__ void k_noalloc_twiddles(Cplx* tw, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double s, c;
    sincospi(2.0 * (double)k / (double)n, &s, &c);
    tw[k] = {c, -s};
}

// interleaved E (2 or 4 doubles per node) -> [dims][N]
__global__ void k_noalloc_deinterleave(const double* E, int dims, long long N, double* out) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= N) return;
    const int st = dims == 2 ? 2 : 4;
    for (int c = 0; c < dims; ++c) out[c * N + g] = E[g * st + c];
}

}  // namespace nd
}  // namespace apic

namespace {
// A caller buffer of the allocation-free solve must be device (or managed)
// memory of the current device: a host pointer would make the kernels fault.
void require_device_buffer(const void* ptr, const char* name) {
    cudaPointerAttributes a{};
    const cudaError_t e = cudaPointerGetAttributes(&a, ptr);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw apic::Error(APIC_ERR_INVALID, std::string(name) + " is not a device pointer");
    }
    apic::require(a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged,
                  std::string(name) + " must be device or managed memory (got a host pointer)");
    if (a.type == cudaMemoryTypeDevice) {
        int dev = 0;
        APIC_CUDA(cudaGetDevice(&dev));
        apic::require(a.device == dev, std::string(name) + " belongs to another device than the current one");
    }
}
}  // namespace

extern "C" int apic_field_solve_periodic_nd_noalloc(int dims, const size_t* n, const double* length,
                                                     double permittivity, const double* d_rho, double* d_phi,
                                                     double* d_electric, void* stream) {
    using namespace apic::nd;
    return guarded_nd(nullptr, [&] {
        apic::require(dims == 2 || dims == 3, "dims must be 2 or 3");
        apic::require(n && length && d_rho && d_phi && d_electric, "null argument");
        apic::require(std::isfinite(permittivity) && permittivity > 0,
                      "field-solver permittivity must be positive and finite");
        size_t N = 1;
        for (int a = 0; a < dims; ++a) {
            apic::require(pow2(n[a]) && n[a] <= kNoAllocMaxLine,
                          "allocation-free solve: extents must be powers of two up to 1024", APIC_ERR_UNSUPPORTED);
            apic::require(std::isfinite(length[a]) && length[a] > 0, "domain lengths must be positive and finite");
            N *= n[a];
        }
        apic::require(N <= kNoAllocMaxPoints,
                      "allocation-free solve: mesh has " + std::to_string(N) + " points, the scratch array holds " +
                          std::to_string(kNoAllocMaxPoints),
                      APIC_ERR_CAPACITY);
        require_device_buffer(d_rho, "d_rho");
        require_device_buffer(d_phi, "d_phi");
        require_device_buffer(d_electric, "d_electric");
        // the scratch array's address in the current device's context, looked
        // up on every call (cheap), so it stays valid after a device reset; and
        // the FFT kernels' fixed shared-memory limit (set once per device)
        void* base = nullptr;
        APIC_CUDA(cudaGetSymbolAddress(&base, g_solve_scratch));
        ensure_solver_attributes();
        unsigned char* bytes = static_cast<unsigned char*>(base);
        Cplx* W = reinterpret_cast<Cplx*>(bytes);
        Cplx* A = W + kNoAllocMaxPoints;
        Cplx* B = A + kNoAllocMaxPoints;
        double* E = reinterpret_cast<double*>(B + kNoAllocMaxPoints);
        double* rho = E + 4 * kNoAllocMaxPoints;
        Cplx* tw = reinterpret_cast<Cplx*>(rho + kNoAllocMaxPoints);
        cudaStream_t s = static_cast<cudaStream_t>(stream);

        Solver S;
        S.stream = s;
        FieldsND& F = S.F;
        F.dims = dims;
        F.nx = (int)n[0];
        F.ny = (int)n[1];
        F.nz = dims == 3 ? (int)n[2] : 1;
        F.lnx = ilog2(F.nx);
        F.lny = ilog2(F.ny);
        for (int a = 0; a < 3; ++a) F.L[a] = a < dims ? length[a] : 1.0;
        F.eps = permittivity;
        F.inv_scale = 1.0;
        double kmax = 0;
        for (int a = 0; a < dims; ++a) kmax = std::max(kmax, 3.141592653589793 * (double)n[a] / length[a]);
        F.pack = std::ldexp(1.0, (int)std::lround(std::log2(kmax)));
        F.rho_in = d_rho;  // every scratch element below is written before it is read
        F.rho = rho;
        F.W = W;
        F.A = A;
        F.B = B;
        F.phi = d_phi;
        F.E = E;
        auto lines = [](int len, long long available, int buffers) {
            int T = 8;
            while (T > 1 && (size_t)buffers * T * len * sizeof(Cplx) + len * sizeof(Cplx) > kFftTileBytes) T >>= 1;
            while (T > 1 && available % T) T >>= 1;
            return T;
        };
        S.px = S.pass(0, lines(F.nx, (long long)F.ny * F.nz, 4));
        S.pxs = S.pass(0, lines(F.nx, (long long)F.ny * F.nz, 2));
        S.py = S.pass(1, lines(F.ny, F.nx, 4));
        S.pys = S.pass(1, lines(F.ny, F.nx, 2));
        if (dims == 3) S.pz = S.pass(2, lines(F.nz, F.nx, 4));
        const int len[3] = {F.nx, F.ny, F.nz};
        for (int a = 0; a < dims; ++a) {
            k_noalloc_twiddles<<<(len[a] + 255) / 256, 256, 0, s>>>(tw + a * kNoAllocMaxLine, len[a]);
        }
        S.px.tw = S.pxs.tw = tw;
        S.py.tw = S.pys.tw = tw + kNoAllocMaxLine;
        if (dims == 3) S.pz.tw = tw + 2 * kNoAllocMaxLine;
        APIC_CUDA(cudaGetLastError());
        S.solve();
        k_noalloc_deinterleave<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(E, dims, (long long)N, d_electric);
        APIC_CUDA(cudaGetLastError());
    });
}
