// AuroraPIC 1D3V checkpoints (.apc, version 12): the restart files of
// Simulation::save_checkpoint / load_checkpoint (src/Simulation.cpp:1812-2015,
// :2018-2899).  Host code.  A checkpoint is read into its parts (unit system,
// collision-model line, collision totals, boundary losses, electric work, the
// campaign-diagnostics block, step, time, the reference's engine state, every
// species' particles) and written back line for line in the reference's form
// (numbers as std::ostream prints them at precision 17, i.e. %.17g), so a file
// read and written again is byte-identical.
//
// The campaign-diagnostics block (spatial_average ... phase_eedf lines) and the
// engine state ("rng" line) are kept as text: the device restores neither (it
// has its own counter-based streams), and they travel unchanged to a file the
// device writes.

#include <cerrno>
#include <cinttypes>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "aurorapic_b200.h"
#include "apc_internal.h"

namespace {

constexpr const char* kMagic12 = "AuroraPIC-checkpoint-v12";

thread_local std::string g_apc_error;

struct ApcError : std::runtime_error {
    int status;
    ApcError(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

void need(bool ok, const std::string& what, int status = APIC_ERR_INVALID) {
    if (!ok) throw ApcError(status, what);
}

std::vector<std::string> tokens(const std::string& line) {
    std::vector<std::string> t;
    std::istringstream in(line);
    std::string w;
    while (in >> w) t.push_back(w);
    return t;
}

uint64_t to_u64(const std::string& s, const std::string& fail) {
    char* end = nullptr;
    errno = 0;
    const unsigned long long v = std::strtoull(s.c_str(), &end, 10);
    need(errno == 0 && end && *end == '\0' && !s.empty() && s[0] != '-', fail);
    return (uint64_t)v;
}

double to_f64(const std::string& s, const std::string& fail) {
    char* end = nullptr;
    const double v = std::strtod(s.c_str(), &end);
    need(end && *end == '\0' && !s.empty(), fail);
    return v;
}

}  // namespace

namespace apic {

std::string fmt17(double v) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.17g", v);
    return buf;
}

// Parses a version-12 checkpoint; the structural checks and messages of
// load_checkpoint that do not depend on the simulation's configuration.
void apc_parse(const std::string& path, Apc& c) {
    std::ifstream in(path);
    need((bool)in, "cannot open checkpoint for reading: " + path);
    const std::string failed = "failed while reading checkpoint: " + path;
    std::string line;
    std::getline(in, line);
    c.magic = line;
    if (line.rfind("AuroraPIC-checkpoint-v", 0) != 0) throw ApcError(APIC_ERR_INVALID, "invalid checkpoint magic in: " + path);
    need(line == kMagic12, "checkpoint version " + line.substr(22) + " is not supported (version 12 only): " + path,
         APIC_ERR_UNSUPPORTED);
    auto next = [&](const char* key) {
        need((bool)std::getline(in, line), failed);
        std::vector<std::string> t = tokens(line);
        need(!t.empty() && t[0] == key, failed);
        return t;
    };
    std::vector<std::string> t = next("dimension");
    need(t.size() == 2 && t[1] == "1", "checkpoint dimension does not match 1D simulation");
    t = next("units");
    need(t.size() == 4 && (t[1] == "si" || t[1] == "normalized"), failed);
    c.units = t[1] == "si" ? APIC_SI : APIC_NORMALIZED;
    c.relative_permittivity = to_f64(t[2], failed);
    c.permittivity = to_f64(t[3], failed);
    t = next("velocity_dimensions");
    need(t.size() == 2, failed);
    c.velocity_dimensions = (int)to_u64(t[1], failed);
    t = next("collision_model");
    need(t.size() == 4, failed);
    c.collision_model = t[1];
    c.collisions_enabled = (int)to_u64(t[2], failed);
    c.collision_signature = to_u64(t[3], failed);
    t = next("collision_totals");
    need(t.size() >= 4, failed);
    c.candidates = to_u64(t[1], failed);
    c.null_collisions = to_u64(t[2], failed);
    const size_t nch = (size_t)to_u64(t[3], failed);
    need(t.size() == 4 + nch, failed);
    c.channel_counts.clear();
    for (size_t k = 0; k < nch; ++k) c.channel_counts.push_back(to_u64(t[4 + k], failed));
    t = next("collision_energy_totals");
    need(t.size() >= 2 && to_u64(t[1], failed) == nch && t.size() == 2 + nch,
         "checkpoint collision energy diagnostics do not match config");
    c.channel_energy.clear();
    for (size_t k = 0; k < nch; ++k) {
        const double e = to_f64(t[2 + k], failed);
        need(std::isfinite(e), "checkpoint collision energy diagnostic is invalid");
        c.channel_energy.push_back(e);
    }
    t = next("boundary_loss_origin_step");
    need(t.size() == 2, "checkpoint is missing the 1D boundary-loss counter origin");
    c.boundary_loss_origin = to_u64(t[1], failed);
    t = next("boundary_loss_count");
    need(t.size() == 2, failed);
    const size_t nloss = (size_t)to_u64(t[1], failed);
    c.losses.clear();
    for (size_t s = 0; s < nloss; ++s) {
        t = next("boundary_loss");
        need(t.size() == 7 && to_u64(t[1], failed) == s, "checkpoint 1D boundary-loss data are invalid");
        Apc::Loss l;
        l.name = t[2];
        l.left = to_u64(t[3], failed);
        l.right = to_u64(t[4], failed);
        l.energy_left = to_f64(t[5], failed);
        l.energy_right = to_f64(t[6], failed);
        need(std::isfinite(l.energy_left) && l.energy_left >= 0.0 && std::isfinite(l.energy_right) &&
                 l.energy_right >= 0.0,
             "checkpoint 1D boundary-loss data are invalid");
        c.losses.push_back(l);
    }
    t = next("power_transfer_origin_step");
    need(t.size() == 2, "checkpoint is missing the 1D power-transfer counter origin");
    c.power_transfer_origin = to_u64(t[1], failed);
    t = next("power_transfer_count");
    need(t.size() == 2, failed);
    const size_t npow = (size_t)to_u64(t[1], failed);
    c.electric_work.clear();
    for (size_t s = 0; s < npow; ++s) {
        t = next("power_transfer");
        need(t.size() == 4 && to_u64(t[1], failed) == s, "checkpoint 1D power-transfer data are invalid");
        const double w = to_f64(t[3], failed);
        need(std::isfinite(w), "checkpoint 1D power-transfer data are invalid");
        c.electric_work.push_back({t[2], w});
    }
    // campaign diagnostics, kept as written, up to the step line
    c.campaign.clear();
    for (;;) {
        need((bool)std::getline(in, line), "checkpoint missing step");
        if (line.rfind("step ", 0) == 0) break;
        c.campaign.push_back(line);
    }
    need(!c.campaign.empty() && c.campaign.front().rfind("spatial_average ", 0) == 0,
         "checkpoint spatial-average contract does not match 1D config");
    {
        const std::vector<std::string> sa = tokens(c.campaign.front());
        need(sa.size() == 10, failed);
        c.spatial_average_enabled = sa[1] == "1";
        c.spatial_average_nx = (size_t)to_u64(sa[9], failed);
    }
    t = tokens(line);
    need(t.size() == 2, "checkpoint missing step");
    c.step = to_u64(t[1], failed);
    t = next("time");
    need(t.size() == 2, "checkpoint missing time");
    c.time = to_f64(t[1], failed);
    t = next("species_count");
    need(t.size() == 2, failed);
    const size_t ns = (size_t)to_u64(t[1], failed);
    need((bool)std::getline(in, line) && line.rfind("rng ", 0) == 0, "checkpoint missing rng state");
    c.rng = line.substr(4);
    c.species.clear();
    for (size_t s = 0; s < ns; ++s) {
        t = next("species");
        need(t.size() == 4 && to_u64(t[1], failed) == s, "checkpoint species metadata does not match config");
        Apc::Species sp;
        sp.name = t[2];
        const size_t n = (size_t)to_u64(t[3], failed);
        sp.x.reserve(n);
        for (size_t i = 0; i < n; ++i) {
            need((bool)std::getline(in, line), failed);
            const std::vector<std::string> r = tokens(line);
            need(r.size() == 6, failed);
            sp.x.push_back(to_f64(r[0], failed));
            sp.v.push_back(to_f64(r[1], failed));
            sp.vy.push_back(to_f64(r[2], failed));
            sp.vz.push_back(to_f64(r[3], failed));
            sp.vh.push_back(to_f64(r[4], failed));
            sp.alive.push_back(to_u64(r[5], failed) != 0 ? 1 : 0);
        }
        c.species.push_back(std::move(sp));
    }
}

// Writes c line for line as save_checkpoint does.
void apc_write(const std::string& path, const Apc& c) {
    std::ofstream out(path);
    need((bool)out, "cannot open checkpoint for writing: " + path);
    std::string s;
    s.reserve(1 << 16);
    auto u = [](uint64_t v) { return std::to_string(v); };
    s += std::string(kMagic12) + "\n";
    s += "dimension 1\n";
    s += std::string("units ") + (c.units == APIC_SI ? "si" : "normalized") + " " + fmt17(c.relative_permittivity) +
         " " + fmt17(c.permittivity) + "\n";
    s += "velocity_dimensions " + u((uint64_t)c.velocity_dimensions) + "\n";
    s += "collision_model " + c.collision_model + " " + u((uint64_t)c.collisions_enabled) + " " +
         u(c.collision_signature) + "\n";
    s += "collision_totals " + u(c.candidates) + " " + u(c.null_collisions) + " " + u(c.channel_counts.size());
    for (uint64_t v : c.channel_counts) s += " " + u(v);
    s += "\ncollision_energy_totals " + u(c.channel_energy.size());
    for (double e : c.channel_energy) s += " " + fmt17(e);
    s += "\nboundary_loss_origin_step " + u(c.boundary_loss_origin) + "\n";
    s += "boundary_loss_count " + u(c.losses.size()) + "\n";
    for (size_t k = 0; k < c.losses.size(); ++k) {
        const Apc::Loss& l = c.losses[k];
        s += "boundary_loss " + u(k) + " " + l.name + " " + u(l.left) + " " + u(l.right) + " " +
             fmt17(l.energy_left) + " " + fmt17(l.energy_right) + "\n";
    }
    s += "power_transfer_origin_step " + u(c.power_transfer_origin) + "\n";
    s += "power_transfer_count " + u(c.electric_work.size()) + "\n";
    for (size_t k = 0; k < c.electric_work.size(); ++k)
        s += "power_transfer " + u(k) + " " + c.electric_work[k].first + " " + fmt17(c.electric_work[k].second) + "\n";
    for (const std::string& l : c.campaign) s += l + "\n";
    s += "step " + u(c.step) + "\n";
    s += "time " + fmt17(c.time) + "\n";
    s += "species_count " + u(c.species.size()) + "\n";
    s += "rng " + c.rng + "\n";
    out << s;
    for (size_t k = 0; k < c.species.size(); ++k) {
        const Apc::Species& sp = c.species[k];
        std::string b = "species " + u(k) + " " + sp.name + " " + u(sp.x.size()) + "\n";
        for (size_t i = 0; i < sp.x.size(); ++i) {
            b += fmt17(sp.x[i]) + " " + fmt17(sp.v[i]) + " " + fmt17(sp.vy[i]) + " " + fmt17(sp.vz[i]) + " " +
                 fmt17(sp.vh[i]) + (sp.alive[i] ? " 1\n" : " 0\n");
        }
        out << b;
    }
    need((bool)out, "failed while writing checkpoint: " + path);
}

}  // namespace apic

namespace {
template <class F>
int apc_guard(F&& f) {
    try {
        f();
        return APIC_OK;
    } catch (const ApcError& e) {
        g_apc_error = e.what();
        return e.status;
    } catch (const std::exception& e) {
        g_apc_error = e.what();
        return APIC_ERR_INVALID;
    }
}
}  // namespace

extern "C" {

const char* apic_apc_last_error(void) { return g_apc_error.c_str(); }

int apic_apc_read(const char* path, apic_apc** out) {
    if (!path || !out) return APIC_ERR_INVALID;
    *out = nullptr;
    auto h = new apic_apc();
    const int rc = apc_guard([&] { apic::apc_parse(path, h->c); });
    if (rc == APIC_OK) *out = h; else delete h;
    return rc;
}

void apic_apc_free(apic_apc* c) { delete c; }

int apic_apc_write(const apic_apc* c, const char* path) {
    if (!c || !path) return APIC_ERR_INVALID;
    return apc_guard([&] { apic::apc_write(path, c->c); });
}

int apic_apc_get_info(const apic_apc* c, apic_apc_info* out) {
    if (!c || !out) return APIC_ERR_INVALID;
    const apic::Apc& a = c->c;
    std::memset(out, 0, sizeof *out);
    out->units = a.units;
    out->relative_permittivity = a.relative_permittivity;
    out->permittivity = a.permittivity;
    out->velocity_dimensions = a.velocity_dimensions;
    out->collisions_enabled = a.collisions_enabled;
    out->collision_signature = a.collision_signature;
    out->candidates = a.candidates;
    out->null_collisions = a.null_collisions;
    out->nchannels = a.channel_counts.size();
    out->boundary_loss_origin_step = a.boundary_loss_origin;
    out->power_transfer_origin_step = a.power_transfer_origin;
    out->spatial_average_enabled = a.spatial_average_enabled ? 1 : 0;
    out->step = a.step;
    out->time = a.time;
    out->nspecies = a.species.size();
    return APIC_OK;
}

int apic_apc_channel(const apic_apc* c, size_t k, uint64_t* count, double* energy) {
    if (!c || k >= c->c.channel_counts.size()) return APIC_ERR_INVALID;
    if (count) *count = c->c.channel_counts[k];
    if (energy) *energy = c->c.channel_energy[k];
    return APIC_OK;
}

int apic_apc_species(const apic_apc* c, size_t k, char* name, size_t name_capacity, size_t* count,
                     apic_boundary_loss* loss, double* electric_work) {
    if (!c || k >= c->c.species.size()) return APIC_ERR_INVALID;
    const apic::Apc::Species& sp = c->c.species[k];
    if (name && name_capacity) {
        std::strncpy(name, sp.name.c_str(), name_capacity - 1);
        name[name_capacity - 1] = '\0';
    }
    if (count) *count = sp.x.size();
    if (loss) {
        std::memset(loss, 0, sizeof *loss);
        if (k < c->c.losses.size()) {
            const apic::Apc::Loss& l = c->c.losses[k];
            loss->absorbed_left = l.left;
            loss->absorbed_right = l.right;
            loss->kinetic_energy_left = l.energy_left;
            loss->kinetic_energy_right = l.energy_right;
        }
    }
    if (electric_work) *electric_work = k < c->c.electric_work.size() ? c->c.electric_work[k].second : 0.0;
    return APIC_OK;
}

int apic_apc_particles(const apic_apc* c, size_t k, double* x, double* v, double* vy, double* vz, double* v_half,
                       uint8_t* alive) {
    if (!c || k >= c->c.species.size()) return APIC_ERR_INVALID;
    const apic::Apc::Species& sp = c->c.species[k];
    const size_t n = sp.x.size();
    if (x) std::memcpy(x, sp.x.data(), n * sizeof(double));
    if (v) std::memcpy(v, sp.v.data(), n * sizeof(double));
    if (vy) std::memcpy(vy, sp.vy.data(), n * sizeof(double));
    if (vz) std::memcpy(vz, sp.vz.data(), n * sizeof(double));
    if (v_half) std::memcpy(v_half, sp.vh.data(), n * sizeof(double));
    if (alive) std::memcpy(alive, sp.alive.data(), n);
    return APIC_OK;
}

}  // extern "C"
