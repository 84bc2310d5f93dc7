// AuroraPIC particle-state interchange (.aps version 1): the initial-condition
// files of the reference's campaigns (load_external_particle_state,
// write_external_particle_state, external_particle_state_signature in
// src/ParticleState.cpp).  Host code: a state is parsed into per-species
// component arrays that the device loaders (apic_sim1d_load_particles,
// apic_simnd_load_particles) take as they are, and written back in the
// reference's deterministic text form.
//
// Format: whitespace-delimited, fixed key order
//   AuroraPIC-particle-state-v1 / dimension D / units normalized|si /
//   weighting species_constant / velocity_staggering time_centered /
//   particle_count N / records / N x "particle <species> x y z vx vy vz" / end
// Species are kept sorted by name (std::map order), records of a species in
// file order.  The signature is 64-bit FNV-1a over the magic, version,
// dimension, unit name, particle count, species count, then per species its
// name, record count and the binary64 bit patterns of every record.

#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "aurorapic_b200.h"

namespace {

constexpr const char* kMagic = "AuroraPIC-particle-state-v1";
constexpr uint64_t kFnvOffset = 14695981039346656037ULL;
constexpr uint64_t kFnvPrime = 1099511628211ULL;

thread_local std::string g_aps_error;

struct ApsError : std::runtime_error {
    int status;
    ApsError(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

void fnv_u64(uint64_t& h, uint64_t v) {
    for (unsigned b = 0; b < 8; ++b) {
        h ^= (unsigned char)(v >> (8 * b));
        h *= kFnvPrime;
    }
}

void fnv_str(uint64_t& h, const std::string& s) {
    fnv_u64(h, s.size());
    for (unsigned char c : s) {
        h ^= c;
        h *= kFnvPrime;
    }
}

void fnv_double(uint64_t& h, double d) {
    uint64_t bits;
    std::memcpy(&bits, &d, 8);
    fnv_u64(h, bits);
}

const char* unit_name(int units) { return units == APIC_SI ? "si" : "normalized"; }

}  // namespace

struct apic_aps {
    int dimension = 0;
    int units = APIC_NORMALIZED;
    size_t particle_count = 0;
    // species name -> records, each record x y z vx vy vz
    std::map<std::string, std::vector<double>> species;
    uint64_t signature = 0;
};

namespace {

void validate(const apic_aps& s, const char* context) {
    if (s.dimension < 1 || s.dimension > 3 || s.particle_count == 0)
        throw ApsError(APIC_ERR_INVALID, std::string(context) + " has invalid particle-state metadata");
    size_t count = 0;
    for (const auto& kv : s.species) {
        if (kv.first.empty() || kv.second.empty())
            throw ApsError(APIC_ERR_INVALID, std::string(context) + " has an empty species name or population");
        const size_t n = kv.second.size() / 6;
        count += n;
        for (size_t i = 0; i < n; ++i) {
            const double* r = &kv.second[6 * i];
            for (int k = 0; k < 6; ++k)
                if (!std::isfinite(r[k]))
                    throw ApsError(APIC_ERR_INVALID,
                                   std::string(context) + " has invalid or active out-of-dimension components");
            if ((s.dimension < 3 && r[2] != 0.0) || (s.dimension == 1 && (r[1] != 0.0 || r[4] != 0.0 || r[5] != 0.0)))
                throw ApsError(APIC_ERR_INVALID,
                               std::string(context) + " has invalid or active out-of-dimension components");
        }
    }
    if (count != s.particle_count)
        throw ApsError(APIC_ERR_INVALID, std::string(context) + " particle count does not match its records");
}

// external_particle_state_signature, src/ParticleState.cpp:541-566
uint64_t signature_of(const apic_aps& s) {
    uint64_t h = kFnvOffset;
    fnv_str(h, kMagic);
    fnv_u64(h, 1);
    fnv_u64(h, (uint64_t)s.dimension);
    fnv_str(h, unit_name(s.units));
    fnv_u64(h, s.particle_count);
    fnv_u64(h, s.species.size());
    for (const auto& kv : s.species) {
        fnv_str(h, kv.first);
        fnv_u64(h, kv.second.size() / 6);
        for (double d : kv.second) fnv_double(h, d);
    }
    return h;
}

void expect_key(std::istream& in, const char* key, const std::string& path) {
    std::string k;
    in >> k;
    if (!in || k != key)
        throw ApsError(APIC_ERR_INVALID, "external particle state '" + path + "' expected key '" + key + "'");
}

bool read_double(std::istream& in, double& d) {
    std::string tok;
    if (!(in >> tok)) return false;
    errno = 0;
    char* end = nullptr;
    d = std::strtod(tok.c_str(), &end);  // correctly rounded, as operator>> is
    return end && *end == '\0' && !tok.empty();
}

// load_external_particle_state, src/ParticleState.cpp:112-262
void parse(const std::string& path, size_t max_particles, apic_aps& s) {
    if (max_particles == 0) throw ApsError(APIC_ERR_INVALID, "external particle-state limit must be positive");
    std::ifstream in(path);
    if (!in) throw ApsError(APIC_ERR_INVALID, "cannot open external particle state: " + path);
    std::string magic;
    in >> magic;
    if (magic != kMagic) throw ApsError(APIC_ERR_INVALID, "invalid external particle-state magic in: " + path);
    expect_key(in, "dimension", path);
    long long dim = 0;
    in >> dim;
    if (!in || dim < 1 || dim > 3) throw ApsError(APIC_ERR_INVALID, "external particle state has invalid dimension");
    s.dimension = (int)dim;
    expect_key(in, "units", path);
    std::string units;
    in >> units;
    if (units == "normalized") s.units = APIC_NORMALIZED;
    else if (units == "si") s.units = APIC_SI;
    else throw ApsError(APIC_ERR_INVALID, "external particle state '" + path + "' has invalid units '" + units + "'");
    expect_key(in, "weighting", path);
    std::string w;
    in >> w;
    if (w != "species_constant")
        throw ApsError(APIC_ERR_INVALID, "external particle state supports only weighting species_constant");
    expect_key(in, "velocity_staggering", path);
    in >> w;
    if (w != "time_centered")
        throw ApsError(APIC_ERR_INVALID, "external particle state supports only time_centered velocities");
    expect_key(in, "particle_count", path);
    unsigned long long count = 0;
    in >> count;
    if (!in || count == 0 || count > max_particles)
        throw ApsError(APIC_ERR_CAPACITY,
                       "external particle-state count is zero, invalid, or exceeds the configured limit");
    s.particle_count = (size_t)count;
    expect_key(in, "records", path);
    for (size_t i = 0; i < s.particle_count; ++i) {
        expect_key(in, "particle", path);
        std::string sp;
        in >> sp;
        double r[6];
        bool ok = (bool)in && !sp.empty();
        for (int k = 0; k < 6 && ok; ++k) ok = read_double(in, r[k]) && std::isfinite(r[k]);
        if (!ok)
            throw ApsError(APIC_ERR_INVALID,
                           "invalid external particle record " + std::to_string(i) + " in: " + path);
        if (s.dimension < 3 && r[2] != 0.0)
            throw ApsError(APIC_ERR_INVALID, "external particle state has nonzero inactive z position");
        if (s.dimension == 1 && (r[1] != 0.0 || r[4] != 0.0 || r[5] != 0.0))
            throw ApsError(APIC_ERR_INVALID, "1D1V external particle state has nonzero inactive components");
        auto& v = s.species[sp];
        v.insert(v.end(), r, r + 6);
    }
    expect_key(in, "end", path);
    std::string trailing;
    if (in >> trailing) throw ApsError(APIC_ERR_INVALID, "external particle state contains trailing data: " + path);
    s.signature = signature_of(s);
}

template <class F>
int guarded_aps(F&& f) {
    try {
        f();
        return APIC_OK;
    } catch (const ApsError& e) {
        g_aps_error = e.what();
        return e.status;
    } catch (const std::bad_alloc&) {
        g_aps_error = "out of host memory";
        return APIC_ERR_CAPACITY;
    } catch (const std::exception& e) {
        g_aps_error = e.what();
        return APIC_ERR_INVALID;
    }
}

}  // namespace

extern "C" {

const char* apic_aps_last_error(void) { return g_aps_error.c_str(); }

int apic_aps_read(const char* path, size_t max_particles, apic_aps** out) {
    if (!path || !out) return APIC_ERR_INVALID;
    *out = nullptr;
    auto s = new (std::nothrow) apic_aps();
    if (!s) return APIC_ERR_CAPACITY;
    const int rc = guarded_aps([&] { parse(path, max_particles, *s); });
    if (rc != APIC_OK) {
        delete s;
        return rc;
    }
    *out = s;
    return APIC_OK;
}

void apic_aps_free(apic_aps* s) { delete s; }

int apic_aps_info(const apic_aps* s, int* dimension, int* units, size_t* particle_count, size_t* nspecies,
                  uint64_t* signature) {
    if (!s) return APIC_ERR_INVALID;
    if (dimension) *dimension = s->dimension;
    if (units) *units = s->units;
    if (particle_count) *particle_count = s->particle_count;
    if (nspecies) *nspecies = s->species.size();
    if (signature) *signature = s->signature;
    return APIC_OK;
}

int apic_aps_species(const apic_aps* s, size_t k, char* name, size_t name_capacity, size_t* count) {
    if (!s || k >= s->species.size()) return APIC_ERR_INVALID;
    auto it = s->species.begin();
    std::advance(it, (long)k);
    if (name) {
        if (name_capacity < it->first.size() + 1) return APIC_ERR_CAPACITY;
        std::memcpy(name, it->first.c_str(), it->first.size() + 1);
    }
    if (count) *count = it->second.size() / 6;
    return APIC_OK;
}

int apic_aps_records(const apic_aps* s, size_t k, double* pos, double* vel) {
    if (!s || k >= s->species.size()) return APIC_ERR_INVALID;
    auto it = s->species.begin();
    std::advance(it, (long)k);
    const size_t n = it->second.size() / 6;
    for (size_t i = 0; i < n; ++i) {
        const double* r = &it->second[6 * i];
        for (int a = 0; a < 3; ++a) {
            if (pos) pos[a * n + i] = r[a];
            if (vel) vel[a * n + i] = r[3 + a];
        }
    }
    return APIC_OK;
}

int apic_aps_write(const char* path, int dimension, int units, size_t nspecies, const char* const* names,
                   const size_t* counts, const double* const* pos, const double* const* vel, int overwrite,
                   uint64_t* signature) {
    if (!path || (nspecies && (!names || !counts || !pos || !vel))) return APIC_ERR_INVALID;
    return guarded_aps([&] {
        apic_aps s;
        s.dimension = dimension;
        s.units = units == APIC_SI ? APIC_SI : APIC_NORMALIZED;
        if (units != APIC_SI && units != APIC_NORMALIZED) throw ApsError(APIC_ERR_INVALID, "unknown units");
        for (size_t k = 0; k < nspecies; ++k) {
            if (!names[k]) throw ApsError(APIC_ERR_INVALID, "null species name");
            const std::string nm(names[k]);
            if (nm.find_first_of(" \t\r\n") != std::string::npos)
                throw ApsError(APIC_ERR_INVALID, "species names must not contain whitespace");
            if (s.species.count(nm)) throw ApsError(APIC_ERR_INVALID, "duplicate species name '" + nm + "'");
            auto& v = s.species[nm];
            const size_t n = counts[k];
            v.resize(6 * n);
            for (size_t i = 0; i < n; ++i)
                for (int a = 0; a < 3; ++a) {
                    v[6 * i + a] = pos[k][a * n + i];
                    v[6 * i + 3 + a] = vel[k][a * n + i];
                }
            s.particle_count += n;
        }
        validate(s, "external particle state writer");
        struct stat sb;
        if (!overwrite && stat(path, &sb) == 0)
            throw ApsError(APIC_ERR_INVALID, std::string("external particle-state output already exists: ") + path);
        // write_external_particle_state, src/ParticleState.cpp:583-624: default
        // floating notation with 17 significant digits
        std::FILE* f = std::fopen(path, "w");
        if (!f) throw ApsError(APIC_ERR_INVALID, std::string("cannot write external particle state: ") + path);
        std::string text;
        text.reserve(64 + s.particle_count * 120);
        text += kMagic;
        text += "\ndimension " + std::to_string(s.dimension) + "\nunits " + unit_name(s.units) +
                "\nweighting species_constant\nvelocity_staggering time_centered\nparticle_count " +
                std::to_string(s.particle_count) + "\nrecords\n";
        char buf[40];
        for (const auto& kv : s.species) {
            const size_t n = kv.second.size() / 6;
            for (size_t i = 0; i < n; ++i) {
                text += "particle ";
                text += kv.first;
                for (int c = 0; c < 6; ++c) {
                    std::snprintf(buf, sizeof buf, " %.17g", kv.second[6 * i + c]);
                    text += buf;
                }
                text += '\n';
            }
        }
        text += "end\n";
        const bool ok = std::fwrite(text.data(), 1, text.size(), f) == text.size();
        const bool closed = std::fclose(f) == 0;
        if (!ok || !closed)
            throw ApsError(APIC_ERR_INVALID, std::string("failed while writing external particle state: ") + path);
        if (signature) *signature = signature_of(s);
    });
}

}  // extern "C"
