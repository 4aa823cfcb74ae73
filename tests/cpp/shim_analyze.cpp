// Analysis written against the reference's C++ API (namespace moldyn), compiled
// against include/moldyn_b200.hpp: an NVE run that accumulates Rdf, Msd and Vacf
// every `every` steps.  Prints each analysed frame's positions ("F x y z" rows),
// then g(r) ("G" rows), the MSD and normalised VACF ("M", "V" rows) and the two
// diffusion coefficients ("D"), for comparison with the oracle.
#include <cstdio>
#include <cstdlib>
#include <exception>

#include "moldyn_b200.hpp"

namespace moldyn = moldyn_b200;

static int run(int argc, char** argv) {
    const int cells = argc > 1 ? std::atoi(argv[1]) : 6;
    const int frames = argc > 2 ? std::atoi(argv[2]) : 6;
    const int every = argc > 3 ? std::atoi(argv[3]) : 10;
    moldyn::System sys = moldyn::fccLattice(cells, 0.8442, 0.722, 5);
    moldyn::LennardJones lj(1.0, 1.0, 2.5, moldyn::Truncation::Truncated);
    moldyn::VerletList verlet(sys.box(), 2.5, 0.3);
    verlet.build(sys);
    auto forces = [&](moldyn::System& s) {
        verlet.rebuildIfNeeded(s);
        return lj.computeForces(s, verlet).energy;
    };
    forces(sys);
    moldyn::VelocityVerlet vv(0.005);
    moldyn::Rdf rdf(3.0, 30);
    moldyn::Msd msd(sys.size(), 4);
    moldyn::Vacf vacf(sys.size(), 4);
    for (int f = 0; f < frames; ++f) {
        for (int k = 0; k < every; ++k) vv.step(sys, forces);
        rdf.accumulate(sys);
        msd.push(sys);
        vacf.push(sys);
        for (std::size_t i = 0; i < sys.size(); ++i) {
            const moldyn::Vec3 r = sys.position(i);
            std::printf("F %.17g %.17g %.17g\n", r.x, r.y, r.z);
        }
    }
    for (double g : rdf.g()) std::printf("G %.17g\n", g);
    for (double m : msd.msd()) std::printf("M %.17g\n", m);
    for (double c : vacf.vacf()) std::printf("V %.17g\n", c);
    std::printf("D %.17g %.17g\n", msd.diffusionCoefficient(0.05, 1, 5),
                vacf.diffusionCoefficient(0.05));
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
