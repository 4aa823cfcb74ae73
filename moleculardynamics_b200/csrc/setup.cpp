// setup.cpp -- host-side initial-state generation (util/lattice.cpp, util/random.hpp).
//
// Setup only, never on the stepping path: the fcc lattice and its Maxwell-Boltzmann
// velocities are drawn on the host with std::mt19937_64 and the same polar
// Box-Muller transform as the reference's Rng, so a given seed yields the
// reference's initial state bit-for-bit on the same standard library.
#include <array>
#include <cmath>
#include <cstdint>
#include <random>

#include "../../include/moldyn_b200.h"
#include "../../include/moldyn_b200_rng.hpp"

namespace {

double fold(double v, double L) { return v - L * std::floor(v / L + 0.5); }

}  // namespace

extern "C" {

// fccLattice(cells, density, temperature, seed) (util/lattice.cpp:15-64): writes
// 4*cells^3 atoms (caller-allocated arrays) and the cubic box.  Returns the atom
// count or MD_ERR_INVALID_ARGUMENT.
int md_fcc_lattice(int cells, double density, double temperature, uint64_t seed, double* x,
                   double* y, double* z, double* vx, double* vy, double* vz, double* mass,
                   double box[3]) {
    if (cells < 1 || !(density > 0.0) || !x || !y || !z || !vx || !vy || !vz || !mass || !box)
        return MD_ERR_INVALID_ARGUMENT;
    const double cells_d = static_cast<double>(cells);
    const int n = 4 * cells * cells * cells;
    const double length = std::cbrt(static_cast<double>(n) / density);
    const double a = length / cells_d;
    static const std::array<std::array<double, 3>, 4> basis = {
        {{0.0, 0.0, 0.0}, {0.0, 0.5, 0.5}, {0.5, 0.0, 0.5}, {0.5, 0.5, 0.0}}};
    box[0] = box[1] = box[2] = length;
    moldyn_b200::Rng rng(seed);
    const double sigma_v = std::sqrt(temperature / 1.0);
    int k = 0;
    for (int ix = 0; ix < cells; ++ix)
        for (int iy = 0; iy < cells; ++iy)
            for (int iz = 0; iz < cells; ++iz)
                for (const auto& b : basis) {
                    x[k] = fold(a * (static_cast<double>(ix) + b[0]) - 0.5 * length, length);
                    y[k] = fold(a * (static_cast<double>(iy) + b[1]) - 0.5 * length, length);
                    z[k] = fold(a * (static_cast<double>(iz) + b[2]) - 0.5 * length, length);
                    vx[k] = sigma_v * rng.normal();
                    vy[k] = sigma_v * rng.normal();
                    vz[k] = sigma_v * rng.normal();
                    mass[k] = 1.0;
                    ++k;
                }
    // system.cpp:147-164 (removeCenterOfMassMotion)
    double total = 0.0;
    for (int i = 0; i < n; ++i) total += mass[i];
    double px = 0.0, py = 0.0, pz = 0.0;
    for (int i = 0; i < n; ++i) {
        px += mass[i] * vx[i];
        py += mass[i] * vy[i];
        pz += mass[i] * vz[i];
    }
    const double cx = px / total, cy = py / total, cz = pz / total;
    for (int i = 0; i < n; ++i) {
        vx[i] -= cx;
        vy[i] -= cy;
        vz[i] -= cz;
    }
    return n;
}

// `count` consecutive Rng(seed).normal() draws (util/random.hpp:37-76), e.g.
// the thermal velocities v_i = sqrt(T / m_i) * (n0, n1, n2) that
// apps/water_rdf.cpp:167-170 draws atom by atom.  Returns count or
// MD_ERR_INVALID_ARGUMENT.
int64_t md_rng_normals(uint64_t seed, int64_t count, double* out) {
    if (count < 0 || (count > 0 && !out)) return MD_ERR_INVALID_ARGUMENT;
    moldyn_b200::Rng rng(seed);
    for (int64_t k = 0; k < count; ++k) out[k] = rng.normal();
    return count;
}

}  // extern "C"
