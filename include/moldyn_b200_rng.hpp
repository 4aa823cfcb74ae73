// moldyn_b200_rng.hpp -- the seeded random stream of the reference's setup code.
//
// Rng (util/random.hpp:37-76): std::mt19937_64, uniform deviates in (0, 1],
// normals by Marsaglia's polar method keeping the spare -- the same stream as the
// reference's for a seed on the same standard library.  One definition, used by
// the library's lattice setup (md_fcc_lattice, md_rng_normals) and by the C++ API.
#pragma once

#include <cmath>
#include <cstdint>
#include <random>

namespace moldyn_b200 {

class Rng {
public:
    explicit Rng(uint64_t seed) : engine_(seed) {}
    double uniform() { return 1.0 - dist_(engine_); }
    double normal() {
        if (have_spare_) {
            have_spare_ = false;
            return spare_;
        }
        double u = 0.0, v = 0.0, s = 0.0;
        do {
            u = 2.0 * uniform() - 1.0;
            v = 2.0 * uniform() - 1.0;
            s = u * u + v * v;
        } while (s >= 1.0 || s == 0.0);
        const double m = std::sqrt(-2.0 * std::log(s) / s);
        spare_ = v * m;
        have_spare_ = true;
        return u * m;
    }

private:
    std::mt19937_64 engine_;
    std::uniform_real_distribution<double> dist_{0.0, 1.0};
    double spare_ = 0.0;
    bool have_spare_ = false;
};

}  // namespace moldyn_b200
