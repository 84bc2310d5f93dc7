// Compiles the C++20 facade against the library and exercises its error
// mapping without a GPU: creation on a host without a device must throw.
#include "aurorapic_b200.hpp"

#include <cstdio>

int main() {
    apic_config1d c{};
    c.boundary = APIC_PERIODIC;
    c.velocity_dimensions = 1;
    c.units = APIC_NORMALIZED;
    c.nx = 16;
    c.length = 1.0;
    c.dt = 0.1;
    c.nspecies = 1;
    c.species[0] = {-1.0, 1.0, 1.0, 64};
    bool device = apic_device_count() > 0;
    try {
        aurorapic_b200::Simulation sim(c);
        std::vector<aurorapic_b200::Particle> ps(8);
        for (int i = 0; i < 8; ++i) ps[i].x = 0.1 * i;
        sim.load_particles(0, ps);
        sim.initialize();
        sim.run(3);
        const auto s = sim.sample();
        std::printf("device step=%zu live=%zu\n", s.step, s.live_particles);
    } catch (const std::runtime_error& e) {
        std::printf("runtime_error: %s\n", e.what());
        if (device) return 1;
    }
    c.dt = -1.0;  // a configuration error keeps the reference's exception type
    try {
        aurorapic_b200::Simulation bad(c);
        return 2;
    } catch (const std::invalid_argument& e) {
        std::printf("invalid_argument: %s\n", e.what());
    } catch (const std::runtime_error& e) {
        std::printf("runtime_error: %s\n", e.what());
        if (device) return 3;
    }
    return 0;
}
