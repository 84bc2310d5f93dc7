// Host side of the null-collision model: validation of an apic_mcc_model
// against the checks of NullCollisionModel's constructor
// (src/Collision.cpp:315-577), upload of its tables, the bracket index of each
// table and the safe speed of the frequency-bound check.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "aurorapic_b200.h"
#include "apic_common.cuh"
#include "apic_mcc.cuh"
#include "apic_mcc32.cuh"

namespace apic {

// Device allocations of one handle: every buffer is zeroed and recorded for
// release by the handle's destructor.
struct DeviceArena {
    std::vector<void*>& allocations;
    cudaStream_t stream;

    template <class T>
    T* alloc(size_t count) {
        void* ptr = nullptr;
        APIC_CUDA(cudaMalloc(&ptr, std::max<size_t>(count, 1) * sizeof(T)));
        allocations.push_back(ptr);
        APIC_CUDA(cudaMemsetAsync(ptr, 0, std::max<size_t>(count, 1) * sizeof(T), stream));
        return static_cast<T*>(ptr);
    }

    template <class T>
    T* upload(const T* host, size_t count) {
        T* d = alloc<T>(count);
        APIC_CUDA(cudaMemcpyAsync(d, host, count * sizeof(T), cudaMemcpyHostToDevice, stream));
        return d;
    }
};

// Largest speed below which the reference's frequency-bound check
// (validate_frequency_bound, src/Collision.cpp:627-685) cannot fail.  Each
// channel's cross section is piecewise linear in energy and energy is
// quadratic in speed, so between breakpoints the total rate is
// n v (A + B v^2); its maximum per interval is exact.  Thermal neutrals use
// the monotone majorant n (v + 8 sigma) sum_c max_{E <= E(v + 8 sigma)} sigma_c.
inline double safe_speed(const apic_mcc_model& m, double particle_mass, double neutral_stddev) {
    const double margin = 1.0 - 1e-9;
    const double target = m.max_frequency * margin;
    const double com = m.neutral_mass > 0 ? particle_mass * m.neutral_mass / (particle_mass + m.neutral_mass) : 0;
    auto mass_of = [&](const apic_mcc_channel& c) { return c.energy_frame == APIC_FRAME_CENTER_OF_MASS ? com : particle_mass; };
    auto sigma_at = [&](const apic_mcc_channel& c, double e) {
        if (e <= c.energy[0]) return c.sigma[0];
        if (e >= c.energy[c.rows - 1]) return c.sigma[c.rows - 1];
        const double* up = std::upper_bound(c.energy, c.energy + c.rows, e);
        const size_t hi = (size_t)(up - c.energy), lo = hi - 1;
        const double f = (e - c.energy[lo]) / (c.energy[hi] - c.energy[lo]);
        return c.sigma[lo] + f * (c.sigma[hi] - c.sigma[lo]);
    };
    if (neutral_stddev == 0.0) {
        // speed breakpoints of every channel
        std::vector<double> br{0.0};
        for (int i = 0; i < m.nch; ++i) {
            const auto& c = m.ch[i];
            const double ms = mass_of(c);
            for (size_t k = 0; k < c.rows; ++k) br.push_back(std::sqrt(2.0 * c.energy[k] / ms));
            if (c.threshold_energy > 0) br.push_back(std::sqrt(2.0 * c.threshold_energy / ms));
        }
        std::sort(br.begin(), br.end());
        auto total = [&](double v) {
            double t = 0;
            for (int i = 0; i < m.nch; ++i) {
                const auto& c = m.ch[i];
                const double e = 0.5 * mass_of(c) * v * v;
                if (e >= c.threshold_energy) t += m.neutral_density * sigma_at(c, e) * v;
            }
            return t;
        };
        for (size_t k = 0; k + 1 < br.size(); ++k) {
            const double v1 = br[k], v2 = br[k + 1];
            if (!(v2 > v1)) continue;
            // sample the cubic densely enough to bound it (endpoints + interior extremum)
            double mx = std::max(total(v1 * (1 + 1e-12) + 1e-300), total(v2 * (1 - 1e-12)));
            for (int q = 1; q < 16; ++q) mx = std::max(mx, total(v1 + (v2 - v1) * q / 16.0));
            if (mx * (1 + 1e-6) > target) return v1;
        }
        // beyond the last breakpoint every sigma is constant: rate = n v sum sigma_last
        double s_last = 0;
        for (int i = 0; i < m.nch; ++i) s_last += m.ch[i].sigma[m.ch[i].rows - 1];
        if (s_last <= 0) return 1e300;
        return std::min(std::max(br.back(), 0.0) == br.back() ? 1e300 : 0.0,
                        target / (m.neutral_density * s_last) * (1 - 1e-6));
    }
    const double limit = kThermalSigma * neutral_stddev;
    auto majorant = [&](double v) {
        double b = 0;
        for (int i = 0; i < m.nch; ++i) {
            const auto& c = m.ch[i];
            const double emax = 0.5 * mass_of(c) * (v + limit) * (v + limit);
            if (emax < c.threshold_energy) continue;
            double smax = sigma_at(c, 0.0);
            for (size_t k = 0; k < c.rows && c.energy[k] <= emax; ++k) smax = std::max(smax, c.sigma[k]);
            smax = std::max(smax, sigma_at(c, emax));
            b += m.neutral_density * smax * (v + limit);
        }
        return b;
    };
    if (majorant(0.0) * (1 + 1e-6) > target) return -1.0;  // always check exactly
    double lo = 0.0, hi = 1.0;
    while (majorant(hi) * (1 + 1e-6) <= target && hi < 1e12) hi *= 2;
    if (hi >= 1e12) return 1e300;
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (majorant(mid) * (1 + 1e-6) <= target) lo = mid; else hi = mid;
    }
    return lo;
}


// Bracket index over log2(energy) for a strictly increasing table.
inline TableIndex build_index(const double* e, size_t rows, DeviceArena& arena) {
    TableIndex ix{};
    size_t first_pos = 0;
    while (first_pos < rows && !(e[first_pos] > 0.0)) ++first_pos;
    if (first_pos + 1 >= rows) return ix;  // no usable positive range: plain binary search
    const double lmin = std::log2(e[first_pos]);
    const double lmax = std::log2(e[rows - 1]);
    if (!(lmax > lmin)) return ix;
    const int nbins = (int)std::min<size_t>(std::max<size_t>(rows, 256), 8192);
    std::vector<unsigned> first(nbins + 1);
    for (int b = 0; b <= nbins; ++b) {
        const double edge = std::exp2(lmin + (lmax - lmin) * (double)b / (double)nbins);
        first[b] = (unsigned)(std::upper_bound(e, e + rows, edge) - e);
    }
    first[nbins] = (unsigned)rows;
    ix.first_gt = arena.upload(first.data(), first.size());
    APIC_CUDA(cudaStreamSynchronize(arena.stream));
    ix.nbins = nbins;
    ix.lmin = lmin;
    ix.inv_width = (double)nbins / (lmax - lmin);
    return ix;
}

// The first waiting time -log(u) / nu (src/Collision.cpp:926-933) falls inside
// the step (< dt) exactly when u >= u*, and u = draw / 2^64 (libstdc++'s
// generate_canonical on a 64-bit draw, values rounding to 1 replaced by the
// largest double below 1) is at least u* exactly when the draw is at least
// D*.  Both thresholds are found by bisection with the host's log, the one
// the CPU restatement uses.
inline void draw_threshold(double nu, double dt, uint64_t& dmin, int& none) {
    auto wait = [nu](double u) { return -std::log(u) / nu; };
    const double umax = std::nextafter(1.0, 0.0);
    none = 0;
    dmin = 0;
    if (!(wait(umax) < dt)) { none = 1; return; }
    uint64_t lo = 1, hi;  // bit patterns: wait(lo) >= dt > wait(hi)
    std::memcpy(&hi, &umax, 8);
    {
        double x;
        std::memcpy(&x, &lo, 8);
        if (wait(x) < dt) { dmin = 1; return; }
    }
    while (hi - lo > 1) {
        const uint64_t mid = lo + (hi - lo) / 2;
        double x;
        std::memcpy(&x, &mid, 8);
        if (wait(x) < dt) hi = mid; else lo = mid;
    }
    double ustar;
    std::memcpy(&ustar, &hi, 8);
    auto canon = [umax](uint64_t d) {
        double r = (double)d / 18446744073709551616.0;
        return r >= 1.0 ? umax : r;
    };
    uint64_t a = 0, b = ~0ull;  // canon(a) < u* <= canon(b)
    while (b - a > 1) {
        const uint64_t mid = a + (b - a) / 2;
        if (canon(mid) >= ustar) b = mid; else a = mid;
    }
    dmin = b;
}

// Range maxima of a table column in O(1) after an O(n log n) build.
struct SparseMax {
    std::vector<std::vector<double>> t;
    explicit SparseMax(const double* x, size_t n) {
        t.push_back(std::vector<double>(x, x + n));
        for (size_t w = 1; 2 * w <= n; w *= 2) {
            const auto& p = t.back();
            std::vector<double> q(n - 2 * w + 1);
            for (size_t i = 0; i < q.size(); ++i) q[i] = std::max(p[i], p[i + w]);
            t.push_back(std::move(q));
        }
    }
    double max(size_t a, size_t b) const {  // [a, b), a < b
        int k = 0;
        while (((size_t)2 << k) <= b - a) ++k;
        return std::max(t[k][a], t[k][b - ((size_t)1 << k)]);
    }
};

// Speed bins whose every speed passes the frequency-bound check.  For a bin
// [v_a, v_b] the check's value at any speed inside is at most
// n (v_b + 8 sigma) sum_c max{ sigma_c(E) : E(v_a - 8 sigma) <= E <= E(v_b + 8 sigma) }
// (without thermal neutrals: n v_b sum_c max over [E(v_a), E(v_b)]); the
// cross sections are piecewise linear, so that maximum is attained at a table
// row or at an end of the window.  Bins are marked safe when this bound stays
// below max_frequency (1 - 1e-9).
inline void build_safe_bins(const apic_mcc_model& m, double mass, double sd, DeviceArena& arena, MccModelDev& D) {
    const double com = m.neutral_mass > 0 ? mass * m.neutral_mass / (mass + m.neutral_mass) : 0.0;
    double vtop = 0.0;  // speed of the highest table energy, over channels
    for (int i = 0; i < m.nch; ++i) {
        const auto& c = m.ch[i];
        const double ms = c.energy_frame == APIC_FRAME_CENTER_OF_MASS ? com : mass;
        vtop = std::max(vtop, std::sqrt(2.0 * c.energy[c.rows - 1] / ms));
    }
    const int nbins = 16384;
    const double limit = kThermalSigma * sd;
    if (!(vtop > 0.0) || !std::isfinite(vtop)) return;
    const double dv = vtop / nbins;
    std::vector<SparseMax> rm;
    for (int i = 0; i < m.nch; ++i) rm.emplace_back(m.ch[i].sigma, m.ch[i].rows);
    auto sigma_at = [](const apic_mcc_channel& c, double e) {
        if (e <= c.energy[0]) return c.sigma[0];
        if (e >= c.energy[c.rows - 1]) return c.sigma[c.rows - 1];
        const double* up = std::upper_bound(c.energy, c.energy + c.rows, e);
        const size_t hi = (size_t)(up - c.energy), lo = hi - 1;
        const double f = (e - c.energy[lo]) / (c.energy[hi] - c.energy[lo]);
        return c.sigma[lo] + f * (c.sigma[hi] - c.sigma[lo]);
    };
    const double target = m.max_frequency * (1.0 - 1e-9);
    std::vector<unsigned char> safe(nbins, 0);
    for (int b = 0; b < nbins; ++b) {
        const double va = dv * b, vb = dv * (b + 1) * (1.0 + 1e-12);
        const double lo_v = std::max(va - limit, 0.0), hi_v = vb + limit;
        double bound = 0.0;
        for (int i = 0; i < m.nch; ++i) {
            const auto& c = m.ch[i];
            const double ms = c.energy_frame == APIC_FRAME_CENTER_OF_MASS ? com : mass;
            const double e_hi = 0.5 * ms * hi_v * hi_v;
            if (e_hi < c.threshold_energy) continue;
            const double e_lo = std::max(0.5 * ms * lo_v * lo_v, c.threshold_energy);
            double smax = std::max(sigma_at(c, e_lo), sigma_at(c, e_hi));
            const size_t k0 = (size_t)(std::lower_bound(c.energy, c.energy + c.rows, e_lo) - c.energy);
            const size_t k1 = (size_t)(std::upper_bound(c.energy, c.energy + c.rows, e_hi) - c.energy);
            if (k0 < k1) smax = std::max(smax, rm[i].max(k0, k1));
            bound += m.neutral_density * smax * hi_v;
        }
        safe[b] = bound * (1.0 + 1e-9) <= target ? 1 : 0;
    }
    D.safe_bins = arena.upload(safe.data(), safe.size());
    D.nsafe = nbins;
    D.safe_inv_dv = 1.0 / dv;
}

// Validates one model (the checks that do not depend on the caller's species
// layout) and fills D with device copies of its tables.  The host tables may be
// released when this returns.
inline void build_model(const apic_mcc_model& m, double mass, DeviceArena& arena, MccModelDev& D) {
    require(std::isfinite(m.neutral_density) && m.neutral_density > 0, "MCC neutral_density must be positive and finite");
    require(std::isfinite(m.max_frequency) && m.max_frequency > 0, "MCC max_frequency must be positive and finite");
    require(m.max_candidates > 0, "MCC max_candidates_per_particle must be positive");
    require(m.nch >= 1 && m.nch <= kMaxChannels, "MCC requires at least one collision channel");
    require(std::isfinite(mass) && mass > 0, "MCC particle mass must be positive and finite");
    D = MccModelDev{};
    D.nch = m.nch;
    D.species = m.species;
    D.particle_mass = mass;
    D.neutral_mass = m.neutral_mass;
    D.neutral_density = m.neutral_density;
    D.max_frequency = m.max_frequency;
    D.max_candidates = (unsigned)std::min<size_t>(m.max_candidates, 0xFFFFFFFFu);
    D.com_mass = m.neutral_mass > 0 ? mass * m.neutral_mass / (mass + m.neutral_mass) : 0.0;
    double sd = 0.0;
    if (m.gas_units_si && m.neutral_temperature > 0) {
        require(m.neutral_mass > 0, "thermal-neutral MCC requires positive neutral_mass");
        sd = std::sqrt(1.380649e-23 * m.neutral_temperature / m.neutral_mass);
    }
    D.neutral_stddev = sd;
    for (int ci = 0; ci < m.nch; ++ci) {
        const apic_mcc_channel& ch = m.ch[ci];
        require(ch.rows >= 2 && ch.energy && ch.sigma, "collision cross-section table requires at least two rows");
        for (size_t k = 0; k < ch.rows; ++k) {
            require(std::isfinite(ch.energy[k]) && ch.energy[k] >= 0 && std::isfinite(ch.sigma[k]) && ch.sigma[k] >= 0,
                    "collision table values must be finite and non-negative");
            require(k == 0 || ch.energy[k] > ch.energy[k - 1], "collision table energies must be strictly increasing");
        }
        require(ch.angular == APIC_ISOTROPIC || ch.angular == APIC_BACKWARD || ch.angular == APIC_HENYEY_GREENSTEIN,
                "unknown angular scattering model");
        require(ch.angular == APIC_ISOTROPIC || ch.process == APIC_ELASTIC,
                "anisotropic MCC scattering is supported only for elastic channels");
        if (ch.angular == APIC_HENYEY_GREENSTEIN) {
            require(ch.mean_cosine_rows >= 2 && ch.mean_cosine_energy && ch.mean_cosine,
                    "Henyey-Greenstein scattering requires mean_cosine_file");
            for (size_t k = 0; k < ch.mean_cosine_rows; ++k) {
                require(std::isfinite(ch.mean_cosine_energy[k]) && ch.mean_cosine_energy[k] >= 0 &&
                            std::isfinite(ch.mean_cosine[k]) && std::fabs(ch.mean_cosine[k]) < 1.0,
                        "mean-cosine table requires finite non-negative energies and mean cosines strictly between -1 and 1");
                require(k == 0 || ch.mean_cosine_energy[k] > ch.mean_cosine_energy[k - 1],
                        "mean-cosine table energies must be strictly increasing");
            }
            require(ch.mean_cosine_energy[0] <= ch.energy[0] &&
                        ch.mean_cosine_energy[ch.mean_cosine_rows - 1] >= ch.energy[ch.rows - 1],
                    "mean-cosine energy range must cover the cross-section table");
        } else {
            require(ch.mean_cosine_rows == 0, "mean-cosine data requires angular_model = henyey_greenstein");
        }
        if (ch.energy_frame == APIC_FRAME_CENTER_OF_MASS) {
            require(m.neutral_mass > 0, "center-of-mass collision energy requires positive neutral_mass");
            require(ch.process == APIC_ELASTIC || ch.process == APIC_CHARGE_EXCHANGE,
                    "center-of-mass collision energy is supported only for elastic and charge-exchange channels");
        }
        if (ch.process == APIC_CHARGE_EXCHANGE) {
            const double tol = 64.0 * 2.220446049250313e-16 * std::max(mass, m.neutral_mass);
            require(m.neutral_mass > 0 && std::fabs(mass - m.neutral_mass) <= tol,
                    "resonant charge exchange requires projectile mass equal to neutral_mass");
        }
        MccChannelDev& C = D.ch[ci];
        C.process = ch.process;
        C.angular = ch.angular;
        C.frame = ch.energy_frame;
        C.threshold = ch.threshold_energy;
        C.secondary = ch.secondary_species;
        C.ion = ch.ion_species;
        C.rows = (int)ch.rows;
        C.energy = arena.upload(ch.energy, ch.rows);
        C.sigma = arena.upload(ch.sigma, ch.rows);
        C.index = build_index(ch.energy, ch.rows, arena);
        if (ch.angular == APIC_HENYEY_GREENSTEIN) {
            C.mu_rows = (int)ch.mean_cosine_rows;
            C.mu_energy = arena.upload(ch.mean_cosine_energy, ch.mean_cosine_rows);
            C.mu = arena.upload(ch.mean_cosine, ch.mean_cosine_rows);
        }
    }
    D.shared_grid = 1;
    for (int ci = 0; ci < m.nch; ++ci) {
        const apic_mcc_channel& a = m.ch[0];
        const apic_mcc_channel& b = m.ch[ci];
        if (b.energy_frame != APIC_FRAME_PROJECTILE || b.rows != a.rows ||
            std::memcmp(a.energy, b.energy, a.rows * sizeof(double)) != 0)
            D.shared_grid = 0;
    }
    D.v_safe = safe_speed(m, mass, sd);
    D.v_safe2 = D.v_safe < 0.0 ? -1.0 : std::nextafter(D.v_safe * D.v_safe, 0.0);
    build_safe_bins(m, mass, sd, arena, D);
    APIC_CUDA(cudaStreamSynchronize(arena.stream));  // host tables may be freed after this
}

// The single-precision copy of a model built by build_model (FP32 particle
// form): tables rounded to float, the same bracket index, float constants.
inline void build_model32(const apic_mcc_model& m, DeviceArena& arena, const MccModelDev& D, MccModel32& F) {
    F = MccModel32{};
    F.nch = D.nch;
    F.shared_grid = D.shared_grid;
    F.particle_mass = (float)D.particle_mass;
    F.neutral_mass = (float)D.neutral_mass;
    F.neutral_density = (float)D.neutral_density;
    F.max_frequency = (float)D.max_frequency;
    F.inv_max_frequency = (float)(1.0 / D.max_frequency);
    F.neutral_stddev = (float)D.neutral_stddev;
    F.com_mass = (float)D.com_mass;
    // |v|^2 below which the FP64 safe speed holds, rounded down in float
    F.v_safe2 = D.v_safe < 0.0 ? -1.0f : std::nextafter((float)std::min(D.v_safe * D.v_safe, 1e37), 0.0f);
    const double total = D.particle_mass + D.neutral_mass;
    F.m_frac = (float)(D.particle_mass / total);
    F.n_frac = (float)(D.neutral_mass / total);
    F.max_candidates = D.max_candidates;
    auto narrow = [&](const double* x, size_t n) {
        std::vector<float> f(n);
        for (size_t i = 0; i < n; ++i) f[i] = (float)x[i];
        const float* d = arena.upload(f.data(), n);
        APIC_CUDA(cudaStreamSynchronize(arena.stream));  // the host vector dies here
        return d;
    };
    for (int ci = 0; ci < m.nch; ++ci) {
        const apic_mcc_channel& ch = m.ch[ci];
        const MccChannelDev& C = D.ch[ci];
        MccChannel32& G = F.ch[ci];
        G.process = C.process;
        G.angular = C.angular;
        G.frame = C.frame;
        G.threshold = (float)C.threshold;
        G.secondary = C.secondary;
        G.ion = C.ion;
        G.rows = C.rows;
        G.energy = narrow(ch.energy, ch.rows);
        G.sigma = narrow(ch.sigma, ch.rows);
        G.first_gt = C.index.first_gt;
        G.nbins = C.index.nbins;
        G.lmin = (float)C.index.lmin;
        G.inv_width = (float)C.index.inv_width;
        if (C.mu_rows) {
            G.mu_rows = C.mu_rows;
            G.mu_energy = narrow(ch.mean_cosine_energy, ch.mean_cosine_rows);
            G.mu = narrow(ch.mean_cosine, ch.mean_cosine_rows);
        }
    }
}

}  // namespace apic
