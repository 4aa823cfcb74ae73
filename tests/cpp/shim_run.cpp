// An apps/moldyn_run.cpp-style NVE run written against the reference's C++ API
// (namespace moldyn), compiled against include/moldyn_b200.hpp: fccLattice,
// VerletList, LennardJones::computeForces(sys, verlet) inside the ForceFn, and
// VelocityVerlet::step.  Prints one row per step (U, W, KE), then the final
// positions and velocities, for comparison with the oracle.  Half way through,
// host code zeroes atom 0's velocity through System::setVelocity, which the next
// step must see (host mirror -> device upload).
#include <cstdio>
#include <cstdlib>
#include <exception>

#include "moldyn_b200.hpp"

namespace moldyn = moldyn_b200;

static int run(int argc, char** argv) {
    const int cells = argc > 1 ? std::atoi(argv[1]) : 6;
    const int steps = argc > 2 ? std::atoi(argv[2]) : 100;
    const unsigned long long seed = argc > 3 ? std::strtoull(argv[3], nullptr, 10) : 1;
    moldyn::System sys = moldyn::fccLattice(cells, 0.8442, 0.722, seed);
    moldyn::LennardJones lj(1.0, 1.0, 2.5, moldyn::Truncation::Truncated);
    moldyn::VerletList verlet(sys.box(), 2.5, 0.3);
    verlet.build(sys);
    double energy = 0.0, virial = 0.0;
    auto forces = [&](moldyn::System& s) {
        verlet.rebuildIfNeeded(s);
        const moldyn::EnergyVirial ev = lj.computeForces(s, verlet);
        energy = ev.energy;
        virial = ev.virial;
        return ev.energy;
    };
    forces(sys);
    moldyn::VelocityVerlet vv(0.005);
    for (int k = 0; k < steps; ++k) {
        if (k == steps / 2) sys.setVelocity(0, moldyn::Vec3{0.0, 0.0, 0.0});
        vv.step(sys, forces);
        std::printf("row %.17g %.17g %.17g\n", energy, virial, sys.kineticEnergy());
    }
    for (std::size_t i = 0; i < sys.size(); ++i) {
        const moldyn::Vec3 r = sys.position(i), v = sys.velocity(i);
        std::printf("atom %.17g %.17g %.17g %.17g %.17g %.17g\n", r.x, r.y, r.z, v.x, v.y, v.z);
    }
    std::printf("rebuilds %zu\n", verlet.rebuildCount());
    return 0;
}

int main(int argc, char** argv) {
    try {
        return run(argc, argv);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
}
