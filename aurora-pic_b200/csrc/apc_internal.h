// The parts of a 1D3V checkpoint (.apc version 12) shared by the file code
// (apc.cu) and the simulation's restart and save (pic1d.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace apic {

struct Apc {
    std::string magic;
    int units = 0;                        // apic_units
    double relative_permittivity = 1.0, permittivity = 1.0;
    int velocity_dimensions = 1;
    std::string collision_model;          // collision_identity() of the writer
    int collisions_enabled = 0;
    uint64_t collision_signature = 0;
    uint64_t candidates = 0, null_collisions = 0;
    std::vector<uint64_t> channel_counts; // every model's channels, in model order
    std::vector<double> channel_energy;
    uint64_t boundary_loss_origin = 0;
    struct Loss {
        std::string name;
        uint64_t left = 0, right = 0;
        double energy_left = 0.0, energy_right = 0.0;
    };
    std::vector<Loss> losses;
    uint64_t power_transfer_origin = 0;
    std::vector<std::pair<std::string, double>> electric_work;
    std::vector<std::string> campaign;    // spatial_average ... phase_eedf lines, as written
    bool spatial_average_enabled = false;
    size_t spatial_average_nx = 0;
    uint64_t step = 0;
    double time = 0.0;
    std::string rng;                      // the writer's engine state (text after "rng ")
    struct Species {
        std::string name;
        std::vector<double> x, v, vy, vz, vh;
        std::vector<uint8_t> alive;
    };
    std::vector<Species> species;
};

void apc_parse(const std::string& path, Apc& c);
void apc_write(const std::string& path, const Apc& c);
std::string fmt17(double v);

}  // namespace apic

struct apic_apc {
    apic::Apc c;
};
