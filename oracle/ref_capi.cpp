// ref_capi.cpp -- extern "C" entry points over the UNMODIFIED moldyn reference
// classes, so Python tests can call the reference itself.
//
// TEST INFRASTRUCTURE, NOT PRODUCT CODE.  oracle/Makefile compiles this file
// together with the reference's own sources (read in place, never copied) into
// oracle/_ref/libmoldyn_ref.so.  It is used to pin the C restatement
// (md_oracle.c) bit-for-bit, to generate tests/golden/ fixtures, and as the
// timed CPU baseline ("kind": "reference").  Nothing in the product links it.
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <exception>
#include <stdexcept>
#include <utility>
#include <vector>

#include "moldyn/analyze/block_average.hpp"
#include "moldyn/analyze/msd.hpp"
#include "moldyn/analyze/rdf.hpp"
#include "moldyn/analyze/vacf.hpp"
#include "moldyn/constrain/rigid_water.hpp"
#include "moldyn/core/box.hpp"
#include "moldyn/core/system.hpp"
#include "moldyn/core/vec3.hpp"
#include "moldyn/forcefield/ewald.hpp"
#include "moldyn/forcefield/lennard_jones.hpp"
#include "moldyn/forcefield/spce_forcefield.hpp"
#include "moldyn/integrate/constrained_velocity_verlet.hpp"
#include "moldyn/integrate/langevin.hpp"
#include "moldyn/integrate/nose_hoover.hpp"
#include "moldyn/integrate/velocity_verlet.hpp"
#include "moldyn/neighbor/cell_list.hpp"
#include "moldyn/neighbor/verlet_list.hpp"
#include "moldyn/util/lattice.hpp"
#include "moldyn/util/random.hpp"

using namespace moldyn;

namespace {

System makeSystem(int64_t n, const double* box, const double* x, const double* y, const double* z,
                  const double* vx, const double* vy, const double* vz, const double* m,
                  const double* q, const int64_t* mol) {
    System sys(Box(Vec3{box[0], box[1], box[2]}));
    sys.reserve(static_cast<std::size_t>(n));
    for (int64_t i = 0; i < n; ++i) {
        const Vec3 r{x[i], y[i], z[i]};
        const Vec3 v = vx ? Vec3{vx[i], vy[i], vz[i]} : Vec3{0.0, 0.0, 0.0};
        const double mass = m ? m[i] : 1.0;
        if (q || mol) {
            sys.addAtom(r, v, mass, q ? q[i] : 0.0,
                        mol ? static_cast<std::size_t>(mol[i]) : static_cast<std::size_t>(i));
        } else {
            sys.addAtom(r, v, mass);
        }
    }
    return sys;
}

void dumpState(const System& sys, double* x, double* y, double* z, double* vx, double* vy,
               double* vz, double* fx, double* fy, double* fz) {
    for (std::size_t i = 0; i < sys.size(); ++i) {
        const Vec3 r = sys.position(i), v = sys.velocity(i), f = sys.force(i);
        if (x) { x[i] = r.x; y[i] = r.y; z[i] = r.z; }
        if (vx) { vx[i] = v.x; vy[i] = v.y; vz[i] = v.z; }
        if (fx) { fx[i] = f.x; fy[i] = f.y; fz[i] = f.z; }
    }
}

Truncation trunc(int t) { return t == 1 ? Truncation::LinearForceShift : Truncation::Truncated; }

}  // namespace

extern "C" {

// mode: 0 computeEnergyVirial (brute), 1 computeForces (brute),
//       2 computeForces(CellList at rc), 3 computeForces(VerletList at rc+skin).
// Returns 0, or -2 for the reference's std::invalid_argument.
int ref_lj_compute(int64_t n, const double* box, const double* x, const double* y,
                   const double* z, double sigma, double eps, double rc, int truncation, int mode,
                   double skin, double* fx, double* fy, double* fz, double* energy,
                   double* virial) {
    System sys = makeSystem(n, box, x, y, z, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    LennardJones lj(sigma, eps, rc, trunc(truncation));
    EnergyVirial ev;
    try {
        if (mode == 0) {
            ev = lj.computeEnergyVirial(sys);
        } else if (mode == 1) {
            ev = lj.computeForces(sys);
        } else if (mode == 2) {
            CellList cells(sys.box(), rc);
            cells.build(sys);
            ev = lj.computeForces(sys, cells);
        } else {
            VerletList verlet(sys.box(), rc, skin);
            verlet.build(sys);
            ev = lj.computeForces(sys, verlet);
        }
    } catch (const std::invalid_argument&) {
        return -2;
    }
    *energy = ev.energy;
    *virial = ev.virial;
    if (mode != 0) dumpState(sys, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, fx, fy, fz);
    return 0;
}

void ref_lj_lrc(int64_t n, const double* box, double sigma, double eps, double rc, int truncation,
                double* u_lrc, double* p_lrc) {
    std::vector<double> zero(static_cast<std::size_t>(n), 0.0);
    System sys = makeSystem(n, box, zero.data(), zero.data(), zero.data(), nullptr, nullptr,
                            nullptr, nullptr, nullptr, nullptr);
    LennardJones lj(sigma, eps, rc, trunc(truncation));
    *u_lrc = lj.longRangeCorrection(sys);
    *p_lrc = lj.longRangeCorrectionPressure(sys);
}

int64_t ref_cells_pairs(int64_t n, const double* box, const double* x, const double* y,
                        const double* z, double cutoff, int64_t* pi, int64_t* pj, int64_t cap,
                        int* dims) {
    System sys = makeSystem(n, box, x, y, z, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    CellList cells(sys.box(), cutoff);
    cells.build(sys);
    for (int d = 0; d < 3; ++d) dims[d] = cells.cellsPerSide(d);
    int64_t count = 0;
    cells.forEachPair([&](std::size_t i, std::size_t j) {
        if (count < cap) {
            pi[count] = static_cast<int64_t>(i);
            pj[count] = static_cast<int64_t>(j);
        }
        ++count;
    });
    return count;
}

int64_t ref_verlet_pairs(int64_t n, const double* box, const double* x, const double* y,
                         const double* z, double cutoff, double skin, int64_t* pi, int64_t* pj,
                         int64_t cap) {
    System sys = makeSystem(n, box, x, y, z, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    VerletList verlet(sys.box(), cutoff, skin);
    verlet.build(sys);
    int64_t count = 0;
    verlet.forEachPair([&](std::size_t i, std::size_t j) {
        if (count < cap) {
            pi[count] = static_cast<int64_t>(i);
            pj[count] = static_cast<int64_t>(j);
        }
        ++count;
    });
    return count;
}

// One VerletList build (verlet_list.cpp:8-42), then computeForces(sys, verlet)
// (lennard_jones.cpp:116-119) and the list's pairs: the moldyn_run ForceFn's
// outputs on one state.  Returns the pair count (pairs beyond cap are counted,
// not stored), or -2 for std::invalid_argument.
int64_t ref_lj_verlet_all(int64_t n, const double* box, const double* x, const double* y,
                          const double* z, double sigma, double eps, double rc, int truncation,
                          double skin, double* fx, double* fy, double* fz, double* energy,
                          double* virial, int64_t* pi, int64_t* pj, int64_t cap) {
    System sys = makeSystem(n, box, x, y, z, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    LennardJones lj(sigma, eps, rc, trunc(truncation));
    EnergyVirial ev;
    VerletList verlet(sys.box(), rc, skin);
    try {
        verlet.build(sys);
        ev = lj.computeForces(sys, verlet);
    } catch (const std::invalid_argument&) {
        return -2;
    }
    *energy = ev.energy;
    *virial = ev.virial;
    dumpState(sys, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, fx, fy, fz);
    int64_t count = 0;
    verlet.forEachPair([&](std::size_t i, std::size_t j) {
        if (count < cap) {
            pi[count] = static_cast<int64_t>(i);
            pj[count] = static_cast<int64_t>(j);
        }
        ++count;
    });
    return count;
}

// Builds at (x0,y0,z0), then asks needsRebuild at (x1,y1,z1).
int ref_verlet_needs_rebuild(int64_t n, const double* box, const double* x0, const double* y0,
                             const double* z0, const double* x1, const double* y1,
                             const double* z1, double cutoff, double skin) {
    System sys = makeSystem(n, box, x0, y0, z0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    VerletList verlet(sys.box(), cutoff, skin);
    verlet.build(sys);
    for (int64_t i = 0; i < n; ++i)
        sys.setPosition(static_cast<std::size_t>(i), Vec3{x1[i], y1[i], z1[i]});
    return verlet.needsRebuild(sys) ? 1 : 0;
}

int ref_fcc_lattice(int cells, double density, double temperature, uint64_t seed, double* x,
                    double* y, double* z, double* vx, double* vy, double* vz, double* mass,
                    double* box) {
    System sys = fccLattice(cells, density, temperature, seed);
    dumpState(sys, x, y, z, vx, vy, vz, nullptr, nullptr, nullptr);
    for (std::size_t i = 0; i < sys.size(); ++i) mass[i] = sys.mass(i);
    const Vec3 l = sys.box().lengths();
    box[0] = l.x;
    box[1] = l.y;
    box[2] = l.z;
    return static_cast<int>(sys.size());
}

void ref_rng_normals(uint64_t seed, double* out, int64_t count) {
    Rng rng(seed);
    for (int64_t i = 0; i < count; ++i) out[i] = rng.normal();
}

// A moldyn_run-style run (apps/moldyn_run.cpp:575-737): VerletList + LJ as the
// ForceFn, primed once, then `steps` steps of the chosen integrator
// (0 VV, 1 BAOAB, 2 NHC).  State arrays are in/out.  info[0..4] receives the
// last energy, last virial, rebuild count, NHC conserved contribution and the
// wall seconds of the stepping loop.
int ref_run(int kind, int64_t n, const double* box, double* x, double* y, double* z, double* vx,
            double* vy, double* vz, double* fx, double* fy, double* fz, const double* m,
            double sigma, double eps, double rc, int truncation, double skin, double dt,
            int64_t steps, double friction, double temperature, uint64_t seed, double tau,
            int chain, int64_t dof, double* info) {
    System sys = makeSystem(n, box, x, y, z, vx, vy, vz, m, nullptr, nullptr);
    LennardJones lj(sigma, eps, rc, trunc(truncation));
    VerletList verlet(sys.box(), rc, skin);
    verlet.build(sys);
    double lastEnergy = 0.0, lastVirial = 0.0;
    auto computeForces = [&](System& s) {
        verlet.rebuildIfNeeded(s);
        const EnergyVirial ev = lj.computeForces(s, verlet);
        lastEnergy = ev.energy;
        lastVirial = ev.virial;
        return ev.energy;
    };
    computeForces(sys);
    double conserved = 0.0;
    const auto t0 = std::chrono::steady_clock::now();
    try {
        if (kind == 0) {
            VelocityVerlet integ(dt);
            for (int64_t k = 0; k < steps; ++k) integ.step(sys, computeForces);
        } else if (kind == 1) {
            LangevinBAOAB integ(dt, friction, temperature, seed);
            for (int64_t k = 0; k < steps; ++k) integ.step(sys, computeForces);
        } else {
            NoseHooverChain integ(dt, temperature, tau, chain, static_cast<std::size_t>(dof));
            for (int64_t k = 0; k < steps; ++k) integ.step(sys, computeForces);
            conserved = integ.conservedQuantityContribution();
        }
    } catch (const std::invalid_argument&) {
        return -2;
    }
    const auto t1 = std::chrono::steady_clock::now();
    dumpState(sys, x, y, z, vx, vy, vz, fx, fy, fz);
    info[0] = lastEnergy;
    info[1] = lastVirial;
    info[2] = static_cast<double>(verlet.rebuildCount());
    info[3] = conserved;
    info[4] = std::chrono::duration<double>(t1 - t0).count();
    return 0;
}

double ref_coulomb_prefactor() { return coulombPrefactorKelvinAngstrom(); }

// mode: 0 computeEnergies, 1 computeForces, 2 accumulateForces (onto fx..fz).
void ref_ewald(int64_t n, const double* box, const double* x, const double* y, const double* z,
               const double* q, const int64_t* mol, double cutoff, int kmax, int mode,
               double* fx, double* fy, double* fz, double* terms) {
    System sys = makeSystem(n, box, x, y, z, nullptr, nullptr, nullptr, nullptr, q, mol);
    if (mode == 2)
        for (int64_t i = 0; i < n; ++i)
            sys.setForce(static_cast<std::size_t>(i), Vec3{fx[i], fy[i], fz[i]});
    Ewald ewald(cutoff, kmax);
    EwaldTerms t;
    if (mode == 0) t = ewald.computeEnergies(sys);
    else if (mode == 1) t = ewald.computeForces(sys);
    else t = ewald.accumulateForces(sys);
    terms[0] = t.real;
    terms[1] = t.reciprocal;
    terms[2] = t.self;
    terms[3] = t.intra;
    if (mode != 0) dumpState(sys, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, fx, fy, fz);
}

// SpceForceField on a full O,H,H system (masses, charges, molecule ids given).
// forces != 0: computeForces (writes fx..fz); else computeEnergy.
double ref_spce(int64_t n, const double* box, const double* x, const double* y, const double* z,
                const double* m, const double* q, const int64_t* mol, double cutoff, int kmax,
                int forces, double* fx, double* fy, double* fz) {
    System sys = makeSystem(n, box, x, y, z, nullptr, nullptr, nullptr, m, q, mol);
    SpceForceField ff(SpceParameters(), cutoff, kmax);
    if (!forces) return ff.computeEnergy(sys);
    const double e = ff.computeForces(sys);
    dumpState(sys, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, fx, fy, fz);
    return e;
}

// RigidWater constrainPositions (which=0, reference positions rx..rz) or
// constrainVelocities (which=1).  Returns iterations, or -1 on the reference's
// std::runtime_error.
int ref_rigid_water(int which, int64_t n, const double* box, const double* m, double* x,
                    double* y, double* z, double* vx, double* vy, double* vz, const double* rx,
                    const double* ry, const double* rz, double oh, double hoh, double tol,
                    int maxit) {
    System sys = makeSystem(n, box, x, y, z, vx, vy, vz, m, nullptr, nullptr);
    RigidWater rw(oh, hoh, tol, maxit);
    int it = 0;
    try {
        if (which == 0) {
            std::vector<Vec3> ref(static_cast<std::size_t>(n));
            for (int64_t i = 0; i < n; ++i) ref[static_cast<std::size_t>(i)] = Vec3{rx[i], ry[i], rz[i]};
            it = rw.constrainPositions(sys, ref);
        } else {
            it = rw.constrainVelocities(sys);
        }
    } catch (const std::runtime_error&) {
        return -1;
    }
    dumpState(sys, x, y, z, vx, vy, vz, nullptr, nullptr, nullptr);
    return it;
}

// ConstrainedVelocityVerlet with SpceForceField forces, `steps` steps, forces
// primed first.  Returns the last potential energy.
double ref_spce_cvv(int64_t n, const double* box, double* x, double* y, double* z, double* vx,
                    double* vy, double* vz, double* fx, double* fy, double* fz, const double* m,
                    const double* q, const int64_t* mol, double cutoff, int kmax, double dt,
                    int64_t steps) {
    System sys = makeSystem(n, box, x, y, z, vx, vy, vz, m, q, mol);
    SpceForceField ff(SpceParameters(), cutoff, kmax);
    const SpceParameters p;
    ConstrainedVelocityVerlet integ(dt, RigidWater(p.rOH, p.angleHOH));
    double pe = ff.computeForces(sys);
    auto forces = [&](System& s) { pe = ff.computeForces(s); };
    for (int64_t k = 0; k < steps; ++k) integ.step(sys, forces);
    dumpState(sys, x, y, z, vx, vy, vz, fx, fy, fz);
    return pe;
}

// Rdf over `frames` frames (pos: frames x (x[n] | y[n] | z[n])): g and the bin
// centres (bins each).  Returns 0, or -2 for std::invalid_argument.
int ref_rdf(int64_t frames, int64_t n, const double* box, const double* pos, double rmax,
            int64_t bins, double* g, double* centres) {
    try {
        Rdf rdf(rmax, static_cast<std::size_t>(bins));
        for (int64_t f = 0; f < frames; ++f) {
            const double* p = pos + f * 3 * n;
            const System sys = makeSystem(n, box, p, p + n, p + 2 * n, nullptr, nullptr, nullptr,
                                          nullptr, nullptr, nullptr);
            rdf.accumulate(sys);
        }
        const std::vector<double> gv = rdf.g(), cv = rdf.binCentres();
        for (int64_t k = 0; k < bins; ++k) {
            g[k] = gv[k];
            centres[k] = cv[k];
        }
        return 0;
    } catch (const std::invalid_argument&) {
        return -2;
    }
}

// Msd over a trajectory of wrapped positions (as ref_rdf): max_lag + 1 values and
// the Einstein diffusion coefficient over [fit_from, fit_to).
void ref_msd(int64_t frames, int64_t n, const double* box, const double* pos, int64_t max_lag,
             double* out, double dt, int64_t fit_from, int64_t fit_to, double* d) {
    Msd msd(static_cast<std::size_t>(n), static_cast<std::size_t>(max_lag));
    for (int64_t f = 0; f < frames; ++f) {
        const double* p = pos + f * 3 * n;
        msd.push(makeSystem(n, box, p, p + n, p + 2 * n, nullptr, nullptr, nullptr, nullptr,
                            nullptr, nullptr));
    }
    const std::vector<double> m = msd.msd();
    for (int64_t k = 0; k <= max_lag; ++k) out[k] = m[k];
    *d = msd.diffusionCoefficient(dt, static_cast<std::size_t>(fit_from),
                                  static_cast<std::size_t>(fit_to));
}

// Vacf over a trajectory of velocities: the normalised values and the Green-Kubo
// diffusion coefficient.
void ref_vacf(int64_t frames, int64_t n, const double* box, const double* vel, int64_t max_lag,
              double* out, double dt, double* d) {
    Vacf vacf(static_cast<std::size_t>(n), static_cast<std::size_t>(max_lag));
    std::vector<double> zero(static_cast<std::size_t>(n), 0.0);
    for (int64_t f = 0; f < frames; ++f) {
        const double* v = vel + f * 3 * n;
        vacf.push(makeSystem(n, box, zero.data(), zero.data(), zero.data(), v, v + n, v + 2 * n,
                             nullptr, nullptr, nullptr));
    }
    const std::vector<double> c = vacf.vacf();
    for (int64_t k = 0; k <= max_lag; ++k) out[k] = c[k];
    *d = vacf.diffusionCoefficient(dt);
}

// blockAverage (analyze/block_average.cpp): out[0..2] = mean, standard error, blocks.
void ref_block_average(int64_t n, const double* samples, double* out) {
    const BlockResult r = blockAverage(std::vector<double>(samples, samples + n));
    out[0] = r.mean;
    out[1] = r.standardError;
    out[2] = static_cast<double>(r.blocks);
}

}  // extern "C"
