// moldyn_b200.hpp -- the reference's C++ API (namespace moldyn) over the C ABI.
//
// Header-only.  The classes keep the names, constructors and methods of the
// reference's hot path (core/system.hpp, core/box.hpp, core/vec3.hpp,
// neighbor/cell_list.hpp, neighbor/verlet_list.hpp, forcefield/*.hpp,
// constrain/rigid_water.hpp, integrate/*.hpp, util/lattice.hpp, util/random.hpp,
// core/units.hpp, io/nist_config.hpp, analyze/*.hpp), so code written against
// them -- apps/moldyn_run.cpp's simulation loop, apps/water_rdf.cpp -- compiles
// against this header with
//
//     #include "moldyn_b200.hpp"
//     namespace moldyn = moldyn_b200;
//
// and runs on the GPU.  The state lives on the device; System keeps a host
// mirror that is downloaded only when host code reads it and uploaded only when
// host code changed it, so a step whose ForceFn calls the force fields below
// moves no data.  Errors come back as the reference's exception types
// (std::invalid_argument, std::runtime_error).  Link libmoldyn_b200.so.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <fstream>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "moldyn_b200.h"
#include "moldyn_b200_rng.hpp"

namespace moldyn_b200 {

namespace detail {

inline void check(int rc) {
    if (rc >= 0) return;  // MD_OK, or a count some entry points return
    const std::string msg = md_last_error() ? md_last_error() : "moldyn_b200 error";
    if (rc == MD_ERR_INVALID_ARGUMENT) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

// One context (stream and scratch) per process on device 0, created on first use.
struct DefaultContext {
    md_context* ctx = nullptr;
    DefaultContext() { check(md_context_create(0, &ctx)); }
    ~DefaultContext() { md_context_destroy(ctx); }
};

inline md_context* context() {
    static DefaultContext c;
    return c.ctx;
}

}  // namespace detail

// ------------------------------------------------------------------ core/vec3.hpp
struct Vec3 {
    double x, y, z;
};
inline constexpr Vec3 operator+(Vec3 a, Vec3 b) { return Vec3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline constexpr Vec3 operator-(Vec3 a, Vec3 b) { return Vec3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline constexpr Vec3 operator*(Vec3 a, double s) { return Vec3{a.x * s, a.y * s, a.z * s}; }
inline constexpr Vec3 operator*(double s, Vec3 a) { return Vec3{a.x * s, a.y * s, a.z * s}; }
inline constexpr Vec3 operator/(Vec3 a, double s) { return Vec3{a.x / s, a.y / s, a.z / s}; }
inline constexpr Vec3& operator+=(Vec3& a, Vec3 b) {
    a.x += b.x;
    a.y += b.y;
    a.z += b.z;
    return a;
}
inline constexpr Vec3& operator-=(Vec3& a, Vec3 b) {
    a.x -= b.x;
    a.y -= b.y;
    a.z -= b.z;
    return a;
}
inline constexpr double dot(Vec3 a, Vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline constexpr double norm2(Vec3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
inline double norm(Vec3 a) { return std::sqrt(norm2(a)); }

// ------------------------------------------------------------------- core/box.hpp
class Box {
public:
    explicit Box(Vec3 lengths) : lengths_(lengths) {}
    // value - L floor(value / L + 1/2) per component (core/box.cpp:12-33)
    Vec3 minimumImage(Vec3 d) const { return Vec3{fold(d.x, lengths_.x), fold(d.y, lengths_.y), fold(d.z, lengths_.z)}; }
    Vec3 wrap(Vec3 r) const { return minimumImage(r); }
    double volume() const { return lengths_.x * lengths_.y * lengths_.z; }
    Vec3 lengths() const { return lengths_; }

private:
    static double fold(double v, double l) { return v - l * std::floor(v / l + 0.5); }
    Vec3 lengths_;
};

// ---------------------------------------------------------------- core/system.hpp
class System {
public:
    explicit System(Box box, md_context* ctx = nullptr)
        : box_(box), ctx_(ctx ? ctx : detail::context()) {}
    System(const System&) = delete;
    System& operator=(const System&) = delete;
    System(System&& o) noexcept { *this = std::move(o); }
    System& operator=(System&& o) noexcept {
        if (this != &o) {
            release();
            box_ = o.box_;
            ctx_ = o.ctx_;
            h_ = std::move(o.h_);
            dev_ = o.dev_;
            dev_n_ = o.dev_n_;
            host_dirty_ = o.host_dirty_;
            device_ahead_ = o.device_ahead_;
            o.dev_ = nullptr;
        }
        return *this;
    }
    ~System() { release(); }

    std::size_t size() const { return h_.mass.size(); }
    const Box& box() const { return box_; }

    void addAtom(Vec3 position, Vec3 velocity, double mass) {
        addAtom(position, velocity, mass, 0.0, size());
    }
    void addAtom(Vec3 position, Vec3 velocity, double mass, double charge, std::size_t moleculeId) {
        pull();
        h_.x.push_back(position.x);
        h_.y.push_back(position.y);
        h_.z.push_back(position.z);
        h_.vx.push_back(velocity.x);
        h_.vy.push_back(velocity.y);
        h_.vz.push_back(velocity.z);
        h_.fx.push_back(0.0);
        h_.fy.push_back(0.0);
        h_.fz.push_back(0.0);
        h_.mass.push_back(mass);
        h_.charge.push_back(charge);
        h_.mol.push_back(static_cast<int64_t>(moleculeId));
        host_dirty_ = true;
    }
    void reserve(std::size_t n) {
        for (auto* v : {&h_.x, &h_.y, &h_.z, &h_.vx, &h_.vy, &h_.vz, &h_.fx, &h_.fy, &h_.fz,
                        &h_.mass, &h_.charge})
            v->reserve(n);
        h_.mol.reserve(n);
    }

    Vec3 position(std::size_t i) const { pull(); return Vec3{h_.x[i], h_.y[i], h_.z[i]}; }
    Vec3 velocity(std::size_t i) const { pull(); return Vec3{h_.vx[i], h_.vy[i], h_.vz[i]}; }
    Vec3 force(std::size_t i) const { pull(); return Vec3{h_.fx[i], h_.fy[i], h_.fz[i]}; }
    double mass(std::size_t i) const { return h_.mass[i]; }
    double charge(std::size_t i) const { return h_.charge[i]; }
    std::size_t moleculeId(std::size_t i) const { return static_cast<std::size_t>(h_.mol[i]); }

    void setPosition(std::size_t i, Vec3 r) { edit(); h_.x[i] = r.x; h_.y[i] = r.y; h_.z[i] = r.z; }
    void setVelocity(std::size_t i, Vec3 v) { edit(); h_.vx[i] = v.x; h_.vy[i] = v.y; h_.vz[i] = v.z; }
    void setForce(std::size_t i, Vec3 f) { edit(); h_.fx[i] = f.x; h_.fy[i] = f.y; h_.fz[i] = f.z; }
    void addForce(std::size_t i, Vec3 f) { edit(); h_.fx[i] += f.x; h_.fy[i] += f.y; h_.fz[i] += f.z; }
    void setCharge(std::size_t i, double q) { edit(); h_.charge[i] = q; }
    void setMoleculeId(std::size_t i, std::size_t m) { edit(); h_.mol[i] = static_cast<int64_t>(m); }

    void zeroForces() {
        if (on_device()) {
            detail::check(md_system_zero_forces(dev_));
            device_ahead_ = true;
        } else {
            std::fill(h_.fx.begin(), h_.fx.end(), 0.0);
            std::fill(h_.fy.begin(), h_.fy.end(), 0.0);
            std::fill(h_.fz.begin(), h_.fz.end(), 0.0);
        }
    }
    double kineticEnergy() const {
        double ke = 0.0;
        detail::check(md_system_kinetic_energy(device(), &ke));
        return ke;
    }
    double temperature(std::size_t dof) const { return 2.0 * kineticEnergy() / static_cast<double>(dof); }
    Vec3 totalMomentum() const {
        double p[3];
        detail::check(md_system_total_momentum(device(), p));
        return Vec3{p[0], p[1], p[2]};
    }
    void removeCenterOfMassMotion() {
        detail::check(md_system_remove_com_motion(device()));
        device_ahead_ = true;
    }
    // Extension: v *= sqrt(target / T), T = 2 KE / dof, when T > 0, on the device
    // (the equilibration rescale of apps/water_rdf.cpp:188-195).
    void rescaleTemperature(std::size_t dof, double target) {
        detail::check(md_system_rescale_temperature(device(), static_cast<int64_t>(dof), target));
        device_ahead_ = true;
    }

    const double* xs() const { pull(); return h_.x.data(); }
    const double* ys() const { pull(); return h_.y.data(); }
    const double* zs() const { pull(); return h_.z.data(); }
    const double* qs() const { return h_.charge.data(); }
    double* fxs() { edit(); return h_.fx.data(); }
    double* fys() { edit(); return h_.fy.data(); }
    double* fzs() { edit(); return h_.fz.data(); }

    // --- device side (used by the force fields and integrators below) ---
    // The device system, uploaded first if host code changed the mirror.
    md_system* device() const {
        if (!dev_ || dev_n_ != size()) {
            if (dev_) md_system_destroy(dev_);
            dev_ = nullptr;
            const Vec3 l = box_.lengths();
            const double b[3] = {l.x, l.y, l.z};
            detail::check(md_system_create(ctx_, static_cast<int64_t>(size()), b, &dev_));
            dev_n_ = size();
            host_dirty_ = true;
        }
        if (host_dirty_) {
            const double* f[11] = {h_.x.data(), h_.y.data(), h_.z.data(), h_.vx.data(),
                                   h_.vy.data(), h_.vz.data(), h_.fx.data(), h_.fy.data(),
                                   h_.fz.data(), h_.mass.data(), h_.charge.data()};
            static const int fields[11] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10};
            if (size()) detail::check(md_system_set_fields(dev_, 11, fields, f));
            if (size()) detail::check(md_system_set_molecule_ids(dev_, h_.mol.data()));
            host_dirty_ = false;
        }
        return dev_;
    }
    // Device kernels moved the state ahead of the host mirror.
    void deviceChanged() const { device_ahead_ = true; }
    md_context* context() const { return ctx_; }

private:
    struct Host {
        std::vector<double> x, y, z, vx, vy, vz, fx, fy, fz, mass, charge;
        std::vector<int64_t> mol;
    };
    bool on_device() const { return dev_ && dev_n_ == size() && !host_dirty_; }
    void pull() const {
        if (!device_ahead_ || !dev_) return;
        double* f[9] = {h_.x.data(), h_.y.data(), h_.z.data(), h_.vx.data(), h_.vy.data(),
                        h_.vz.data(), h_.fx.data(), h_.fy.data(), h_.fz.data()};
        static const int fields[9] = {0, 1, 2, 3, 4, 5, 6, 7, 8};
        if (size()) detail::check(md_system_get_fields(dev_, 9, fields, f));
        device_ahead_ = false;
    }
    void edit() {
        pull();
        host_dirty_ = true;
    }
    void release() {
        if (dev_) md_system_destroy(dev_);
        dev_ = nullptr;
    }

    Box box_{Vec3{1, 1, 1}};
    md_context* ctx_ = nullptr;
    mutable Host h_;
    mutable md_system* dev_ = nullptr;
    mutable std::size_t dev_n_ = 0;
    mutable bool host_dirty_ = true;
    mutable bool device_ahead_ = false;
};

// --------------------------------------------------------------- neighbour lists
namespace detail {
template <class Export, class Fn>
void for_each_exported(Export&& ex, Fn&& fn) {
    int64_t count = 0;
    check(ex(nullptr, nullptr, 0, &count));
    std::vector<int64_t> a(static_cast<std::size_t>(count)), b(static_cast<std::size_t>(count));
    if (count) check(ex(a.data(), b.data(), count, &count));
    for (int64_t k = 0; k < count; ++k) fn(static_cast<std::size_t>(a[k]), static_cast<std::size_t>(b[k]));
}
}  // namespace detail

class CellList {
public:
    CellList(const Box& box, double cutoff, md_context* ctx = nullptr) {
        const Vec3 l = box.lengths();
        const double b[3] = {l.x, l.y, l.z};
        detail::check(md_cells_create(ctx ? ctx : detail::context(), b, cutoff, &h_));
    }
    CellList(const CellList&) = delete;
    CellList& operator=(const CellList&) = delete;
    ~CellList() { md_cells_destroy(h_); }
    void build(const System& sys) { detail::check(md_cells_build(h_, sys.device())); }
    int cellsPerSide(int dim) const {
        int d[3];
        detail::check(md_cells_dims(h_, d));
        return d[dim];
    }
    bool usable() const { return md_cells_usable(h_) == 1; }
    template <class Fn>
    void forEachPair(Fn&& fn) const {
        detail::for_each_exported(
            [&](int64_t* a, int64_t* b, int64_t cap, int64_t* n) { return md_cells_pairs(h_, a, b, cap, n); },
            fn);
    }
    md_cells* handle() const { return h_; }

private:
    md_cells* h_ = nullptr;
};

class VerletList {
public:
    VerletList(const Box& box, double cutoff, double skin, md_context* ctx = nullptr) {
        const Vec3 l = box.lengths();
        const double b[3] = {l.x, l.y, l.z};
        detail::check(md_verlet_create(ctx ? ctx : detail::context(), b, cutoff, skin, &h_));
    }
    VerletList(const VerletList&) = delete;
    VerletList& operator=(const VerletList&) = delete;
    ~VerletList() { md_verlet_destroy(h_); }
    void build(const System& sys) { detail::check(md_verlet_build(h_, sys.device())); }
    bool needsRebuild(const System& sys) const {
        int f = 0;
        detail::check(md_verlet_needs_rebuild(h_, sys.device(), &f));
        return f != 0;
    }
    void rebuildIfNeeded(const System& sys) {
        detail::check(md_verlet_rebuild_if_needed(h_, sys.device(), nullptr));
    }
    std::size_t rebuildCount() const {
        int64_t c = 0;
        detail::check(md_verlet_rebuild_count(h_, &c));
        return static_cast<std::size_t>(c);
    }
    template <class Fn>
    void forEachPair(Fn&& fn) const {
        detail::for_each_exported(
            [&](int64_t* a, int64_t* b, int64_t cap, int64_t* n) { return md_verlet_pairs(h_, a, b, cap, n); },
            fn);
    }
    md_verlet* handle() const { return h_; }

private:
    md_verlet* h_ = nullptr;
};

// ------------------------------------------------------------------ force fields
struct EnergyVirial {
    double energy = 0.0;  // pair sum, no tail correction
    double virial = 0.0;  // raw sum of w(r), not divided by 3
};

// forcefield/forcefield.hpp:17-23: the interface LennardJones implements.
class ForceField {
public:
    virtual ~ForceField() = default;
    virtual EnergyVirial computeEnergyVirial(const System& sys) const = 0;
    virtual double longRangeCorrection(const System& sys) const = 0;
    virtual double longRangeCorrectionPressure(const System& sys) const = 0;
};

enum class Truncation { Truncated = MD_TRUNCATED, LinearForceShift = MD_LINEAR_FORCE_SHIFT };
// Pair arithmetic: the reference's FP64 (default) or FP32 pair terms (extension).
enum class Precision { FP64 = MD_PRECISION_FP64, Mixed = MD_PRECISION_MIXED };

class LennardJones : public ForceField {
public:
    LennardJones(double sigma, double epsilon, double cutoff, Truncation truncation,
                 Precision precision = Precision::FP64)
        : sigma_(sigma), epsilon_(epsilon), cutoff_(cutoff), trunc_(truncation) {
        detail::check(md_lj_create(sigma, epsilon, cutoff, static_cast<int>(truncation),
                                   static_cast<int>(precision), &h_));
    }
    LennardJones(const LennardJones&) = delete;
    LennardJones& operator=(const LennardJones&) = delete;
    ~LennardJones() override { md_lj_destroy(h_); }

    EnergyVirial computeEnergyVirial(const System& sys) const override {
        EnergyVirial ev;
        detail::check(md_lj_energy_virial(h_, sys.device(), &ev.energy, &ev.virial));
        return ev;
    }
    EnergyVirial computeForces(System& sys) const {
        EnergyVirial ev;
        detail::check(md_lj_forces(h_, sys.device(), &ev.energy, &ev.virial));
        sys.deviceChanged();
        return ev;
    }
    EnergyVirial computeForces(System& sys, const CellList& cells) const {
        EnergyVirial ev;
        detail::check(md_lj_forces_cells(h_, sys.device(), cells.handle(), &ev.energy, &ev.virial));
        sys.deviceChanged();
        return ev;
    }
    EnergyVirial computeForces(System& sys, const VerletList& verlet) const {
        EnergyVirial ev;
        detail::check(md_lj_forces_verlet(h_, sys.device(), verlet.handle(), &ev.energy, &ev.virial));
        sys.deviceChanged();
        return ev;
    }
    double longRangeCorrection(const System& sys) const override { return lrc(sys).first; }
    double longRangeCorrectionPressure(const System& sys) const override { return lrc(sys).second; }
    double sigma() const { return sigma_; }
    double epsilon() const { return epsilon_; }
    double cutoff() const { return cutoff_; }
    Truncation truncation() const { return trunc_; }
    md_lj* handle() const { return h_; }

private:
    std::pair<double, double> lrc(const System& sys) const {
        const Vec3 l = sys.box().lengths();
        const double b[3] = {l.x, l.y, l.z};
        double u = 0.0, p = 0.0;
        detail::check(md_lj_lrc(h_, static_cast<int64_t>(sys.size()), b, &u, &p));
        return {u, p};
    }
    md_lj* h_ = nullptr;
    double sigma_, epsilon_, cutoff_;
    Truncation trunc_;
};

struct EwaldTerms {
    double real = 0.0, reciprocal = 0.0, self = 0.0, intra = 0.0;
    double total() const { return real + reciprocal + self + intra; }
};

class Ewald {
public:
    // alpha <= 0: the reference's 5.6 / min(box lengths) (extension: an explicit alpha)
    Ewald(double cutoff, int kmax, double alpha = 0.0, md_context* ctx = nullptr) {
        detail::check(md_ewald_create(ctx ? ctx : detail::context(), cutoff, kmax, alpha, &h_));
    }
    Ewald(const Ewald&) = delete;
    Ewald& operator=(const Ewald&) = delete;
    ~Ewald() { md_ewald_destroy(h_); }
    // Extensions: smooth PME for the reciprocal term (0, 0, 0: the k-vector
    // sums), FP32 real-space pair terms (MD_PRECISION_MIXED).
    void setPme(int kx, int ky, int kz, int order = 6) { detail::check(md_ewald_set_pme(h_, kx, ky, kz, order)); }
    void setPrecision(int precision) { detail::check(md_ewald_set_precision(h_, precision)); }
    EwaldTerms computeEnergies(const System& sys) const { return run(sys, 0); }
    EwaldTerms computeForces(System& sys) const { EwaldTerms t = run(sys, 1); sys.deviceChanged(); return t; }
    EwaldTerms accumulateForces(System& sys) const { EwaldTerms t = run(sys, 2); sys.deviceChanged(); return t; }

private:
    EwaldTerms run(const System& sys, int mode) const {
        double t[4], w;
        detail::check(md_ewald_compute(h_, sys.device(), mode, t, &w));
        return EwaldTerms{t[0], t[1], t[2], t[3]};
    }
    md_ewald* h_ = nullptr;
};

struct SpceParameters {
    double qH = 0.42380;
    double sigmaO = 3.16555789;
    double epsilonO = 78.19743111;
    double rOH = 1.0;
    double angleHOH = 109.47;
    double massOxygen = 15.9994;
    double massHydrogen = 1.008;
};

class SpceForceField {
public:
    explicit SpceForceField(const SpceParameters& params = SpceParameters(), double cutoff = 10.0,
                            int kmax = 5, md_context* ctx = nullptr) {
        detail::check(md_spce_create(ctx ? ctx : detail::context(), params.sigmaO, params.epsilonO,
                                     cutoff, kmax, 0.0, &h_));
    }
    SpceForceField(const SpceForceField&) = delete;
    SpceForceField& operator=(const SpceForceField&) = delete;
    ~SpceForceField() { md_ewald_destroy(h_); }
    double computeForces(System& sys) const {
        double e = 0.0;
        detail::check(md_spce_compute(h_, sys.device(), 1, &e, nullptr));
        sys.deviceChanged();
        return e;
    }
    double computeEnergy(const System& sys) const {
        double e = 0.0;
        detail::check(md_spce_compute(h_, sys.device(), 0, &e, nullptr));
        return e;
    }
    void setPme(int kx, int ky, int kz, int order = 6) { detail::check(md_ewald_set_pme(h_, kx, ky, kz, order)); }
    void setPrecision(int precision) { detail::check(md_ewald_set_precision(h_, precision)); }
    md_ewald* handle() const { return h_; }

private:
    md_ewald* h_ = nullptr;
};

// ------------------------------------------------------------------ rigid water
class RigidWater {
public:
    RigidWater(double ohDistance, double hohAngleDegrees, double tolerance = 1e-12,
               int maxIterations = 500)
        : tolerance_(tolerance), angle_(hohAngleDegrees), max_it_(maxIterations) {
        detail::check(md_rigid_create(ohDistance, hohAngleDegrees, tolerance, maxIterations, &h_));
    }
    RigidWater(const RigidWater& o) { copy(o); }
    RigidWater& operator=(const RigidWater& o) {
        if (this != &o) {
            md_rigid_destroy(h_);
            copy(o);
        }
        return *this;
    }
    ~RigidWater() { md_rigid_destroy(h_); }
    int constrainPositions(System& sys, const std::vector<Vec3>& reference) const {
        std::vector<double> rx(reference.size()), ry(reference.size()), rz(reference.size());
        for (std::size_t i = 0; i < reference.size(); ++i) {
            rx[i] = reference[i].x;
            ry[i] = reference[i].y;
            rz[i] = reference[i].z;
        }
        int it = 0;
        detail::check(md_rigid_constrain_positions(h_, sys.device(), rx.data(), ry.data(), rz.data(), &it));
        sys.deviceChanged();
        return it;
    }
    int constrainVelocities(System& sys) const {
        int it = 0;
        detail::check(md_rigid_constrain_velocities(h_, sys.device(), &it));
        sys.deviceChanged();
        return it;
    }
    // Extension: closed-form SETTLE instead of SHAKE / RATTLE iterations (the same
    // fixed point); integrators created from this constraint afterwards use it.
    void setSettle(bool on) {
        detail::check(md_rigid_set_settle(h_, on ? 1 : 0));
        settle_ = on;
    }
    double ohDistance() const { double oh, hh; md_rigid_distances(h_, &oh, &hh); return oh; }
    double hhDistance() const { double oh, hh; md_rigid_distances(h_, &oh, &hh); return hh; }
    static std::size_t degreesOfFreedom(std::size_t molecules, bool comRemoved) {
        return static_cast<std::size_t>(md_rigid_degrees_of_freedom(static_cast<int64_t>(molecules), comRemoved ? 1 : 0));
    }
    md_rigid* handle() const { return h_; }

private:
    void copy(const RigidWater& o) {
        double oh, hh;
        md_rigid_distances(o.h_, &oh, &hh);
        tolerance_ = o.tolerance_;
        max_it_ = o.max_it_;
        angle_ = o.angle_;
        detail::check(md_rigid_create(oh, o.angle_, o.tolerance_, o.max_it_, &h_));
        settle_ = o.settle_;
        if (settle_) detail::check(md_rigid_set_settle(h_, 1));
    }
    md_rigid* h_ = nullptr;
    double tolerance_ = 1e-12, angle_ = 109.47;
    int max_it_ = 500;
    bool settle_ = false;
};

// ------------------------------------------------------------------- integrators
namespace detail {
// A step split around the ForceFn (called exactly once per step).
class Stepper {
public:
    Stepper(const Stepper&) = delete;
    Stepper& operator=(const Stepper&) = delete;
    ~Stepper() { md_integrator_destroy(h_); }
    md_integrator* handle() const { return h_; }

protected:
    Stepper() = default;
    template <class ForceFn>
    void run_step(System& sys, ForceFn&& computeForces) {
        check(md_integrator_pre_force(h_, sys.device()));
        sys.deviceChanged();
        computeForces(sys);
        check(md_integrator_post_force(h_, sys.device()));
        sys.deviceChanged();
    }
    md_integrator* h_ = nullptr;
};
}  // namespace detail

class VelocityVerlet : public detail::Stepper {
public:
    explicit VelocityVerlet(double dt) : dt_(dt) { detail::check(md_integrator_create_vv(dt, &h_)); }
    template <class ForceFn>
    void step(System& sys, ForceFn&& computeForces) { run_step(sys, computeForces); }
    double dt() const { return dt_; }

private:
    double dt_;
};

class LangevinBAOAB : public detail::Stepper {
public:
    // The O step's normals come from Philox4x32-10 keyed by seed (not mt19937_64).
    LangevinBAOAB(double dt, double friction, double temperature, uint64_t seed) : dt_(dt) {
        detail::check(md_integrator_create_baoab(dt, friction, temperature, seed, &h_));
    }
    template <class ForceFn>
    void step(System& sys, ForceFn&& computeForces) { run_step(sys, computeForces); }
    double dt() const { return dt_; }

private:
    double dt_;
};

class NoseHooverChain : public detail::Stepper {
public:
    NoseHooverChain(double dt, double temperature, double tau, int chainLength, std::size_t dof)
        : dt_(dt) {
        detail::check(md_integrator_create_nhc(dt, temperature, tau, chainLength,
                                               static_cast<int64_t>(dof), &h_));
    }
    template <class ForceFn>
    void step(System& sys, ForceFn&& computeForces) { run_step(sys, computeForces); }
    double conservedQuantityContribution() const {
        double v = 0.0;
        detail::check(md_integrator_conserved(h_, &v));
        return v;
    }
    double dt() const { return dt_; }

private:
    double dt_;
};

class ConstrainedVelocityVerlet : public detail::Stepper {
public:
    ConstrainedVelocityVerlet(double dt, RigidWater constraint) : dt_(dt), rw_(constraint) {
        detail::check(md_integrator_create_rattle(dt, rw_.handle(), &h_));
    }
    template <class ForceFn>
    void step(System& sys, ForceFn&& computeForces) { run_step(sys, computeForces); }
    double dt() const { return dt_; }
    const RigidWater& constraint() const { return rw_; }

private:
    double dt_;
    RigidWater rw_;
};

// Extension: `steps` fused steps of an LJ run with the ForceFn of
// apps/moldyn_run.cpp (rebuildIfNeeded + computeForces(sys, verlet)) on the
// device, the neighbour rebuild decided there too.
template <class Integrator>
void runFused(Integrator& integ, System& sys, VerletList& verlet, const LennardJones& lj,
              int64_t steps, std::vector<double>* thermo = nullptr) {
    if (thermo) thermo->assign(4 * static_cast<std::size_t>(steps), 0.0);
    detail::check(md_run_lj(integ.handle(), sys.device(), verlet.handle(), lj.handle(), steps,
                            thermo ? thermo->data() : nullptr));
    sys.deviceChanged();
}

// ------------------------------------------------------------- util/lattice.hpp
// fccLattice(cells, density, temperature, seed) (util/lattice.cpp:15-64):
// bit-identical positions and velocities to the reference's.
inline System fccLattice(int cells, double density, double temperature, uint64_t seed) {
    const std::size_t n = 4 * static_cast<std::size_t>(cells) * cells * cells;
    std::vector<double> x(n), y(n), z(n), vx(n), vy(n), vz(n), m(n);
    double box[3];
    detail::check(md_fcc_lattice(cells, density, temperature, seed, x.data(), y.data(), z.data(),
                                 vx.data(), vy.data(), vz.data(), m.data(), box));
    System sys(Box(Vec3{box[0], box[1], box[2]}));
    sys.reserve(n);
    for (std::size_t i = 0; i < n; ++i) sys.addAtom(Vec3{x[i], y[i], z[i]}, Vec3{vx[i], vy[i], vz[i]}, m[i]);
    return sys;
}

// analyze/rdf.hpp:16-34 on the device (md_rdf_*).
class Rdf {
public:
    Rdf(double rMax, std::size_t bins, md_context* ctx = nullptr) : bins_(bins) {
        detail::check(md_rdf_create(ctx ? ctx : detail::context(), rMax,
                                    static_cast<int64_t>(bins), &h_));
    }
    Rdf(const Rdf&) = delete;
    Rdf& operator=(const Rdf&) = delete;
    ~Rdf() { md_rdf_destroy(h_); }
    void accumulate(const System& sys) { detail::check(md_rdf_accumulate(h_, sys.device())); }
    // Extension: the atoms first, first + stride, ... alone, as accumulate() of a
    // System holding just those (apps/water_rdf.cpp's gatherOxygens: 0, 3).
    void accumulateSubset(const System& sys, std::size_t first, std::size_t stride) {
        detail::check(md_rdf_accumulate_subset(h_, sys.device(), static_cast<int64_t>(first),
                                               static_cast<int64_t>(stride)));
    }
    md_rdf* handle() const { return h_; }
    std::vector<double> binCentres() const { return vec(md_rdf_bin_centres); }
    std::vector<double> g() const { return vec(md_rdf_g); }
    std::size_t frames() const {
        int64_t f = 0;
        detail::check(md_rdf_frames(h_, &f));
        return static_cast<std::size_t>(f);
    }

private:
    std::vector<double> vec(int (*fn)(const md_rdf*, double*)) const {
        std::vector<double> out(bins_);
        detail::check(fn(h_, out.data()));
        return out;
    }
    std::size_t bins_;
    md_rdf* h_ = nullptr;
};

// analyze/msd.hpp:19-42 on the device (md_msd_*).
class Msd {
public:
    Msd(std::size_t natoms, std::size_t maxLag, md_context* ctx = nullptr) : lags_(maxLag + 1) {
        detail::check(md_msd_create(ctx ? ctx : detail::context(), static_cast<int64_t>(natoms),
                                    static_cast<int64_t>(maxLag), &h_));
    }
    Msd(const Msd&) = delete;
    Msd& operator=(const Msd&) = delete;
    ~Msd() { md_msd_destroy(h_); }
    void push(const System& sys) { detail::check(md_msd_push(h_, sys.device())); }
    std::vector<double> msd() const {
        std::vector<double> out(lags_);
        detail::check(md_msd_values(h_, out.data()));
        return out;
    }
    double diffusionCoefficient(double dt, std::size_t fitFrom, std::size_t fitTo) const {
        double d = 0.0;
        detail::check(md_msd_diffusion(h_, dt, static_cast<int64_t>(fitFrom),
                                       static_cast<int64_t>(fitTo), &d));
        return d;
    }

private:
    std::size_t lags_;
    md_msd* h_ = nullptr;
};

// analyze/vacf.hpp:151-174 on the device (md_vacf_*).
class Vacf {
public:
    Vacf(std::size_t natoms, std::size_t maxLag, md_context* ctx = nullptr) : lags_(maxLag + 1) {
        detail::check(md_vacf_create(ctx ? ctx : detail::context(), static_cast<int64_t>(natoms),
                                     static_cast<int64_t>(maxLag), &h_));
    }
    Vacf(const Vacf&) = delete;
    Vacf& operator=(const Vacf&) = delete;
    ~Vacf() { md_vacf_destroy(h_); }
    void push(const System& sys) { detail::check(md_vacf_push(h_, sys.device())); }
    std::vector<double> vacf() const {
        std::vector<double> out(lags_);
        detail::check(md_vacf_values(h_, 1, out.data()));
        return out;
    }
    double diffusionCoefficient(double dt) const {
        double d = 0.0;
        detail::check(md_vacf_diffusion(h_, dt, &d));
        return d;
    }

private:
    std::size_t lags_;
    md_vacf* h_ = nullptr;
};

// ------------------------------------------------------- analyze/block_average.hpp
// Host-side statistics (no device work): the mean of a time series and its
// standard error by the blocking method of Flyvbjerg and Petersen (J. Chem. Phys.
// 91, 461 (1989)), as analyze/block_average.cpp applies it.  Level 0 is the
// series itself; each further level halves it by averaging neighbouring pairs
// (an odd last sample is dropped) while at least four blocks remain.  At every
// level with n >= 2 blocks the standard error is sqrt(s^2 / n), s^2 the unbiased
// block variance, with its own uncertainty se / sqrt(2 (n - 1)).  The result is
// the first level whose error moved by no more than the previous level's
// uncertainty (the plateau), else the last level.
struct BlockResult {
    double mean;
    double standardError;
    std::size_t blocks;
};

inline BlockResult blockAverage(const std::vector<double>& samples) {
    if (samples.empty()) return BlockResult{0.0, 0.0, 0};
    if (samples.size() == 1) return BlockResult{samples[0], 0.0, 1};
    auto average = [](const std::vector<double>& v) {
        double t = 0.0;
        for (double x : v) t += x;
        return t / static_cast<double>(v.size());
    };
    const double grand = average(samples);
    std::vector<double> se, err;
    std::vector<std::size_t> count;
    std::vector<double> level(samples);
    for (;;) {
        const std::size_t n = level.size();
        const double m = average(level);
        double ss = 0.0;
        for (double x : level) ss += (x - m) * (x - m);
        const double e = std::sqrt(ss / static_cast<double>(n - 1) / static_cast<double>(n));
        se.push_back(e);
        err.push_back(e / std::sqrt(2.0 * static_cast<double>(n - 1)));
        count.push_back(n);
        if (n < 4) break;
        std::vector<double> next(n / 2);
        for (std::size_t k = 0; k < next.size(); ++k) next[k] = 0.5 * (level[2 * k] + level[2 * k + 1]);
        level.swap(next);
    }
    std::size_t pick = se.size() - 1;
    for (std::size_t k = 1; k < se.size(); ++k) {
        if (std::fabs(se[k] - se[k - 1]) <= err[k - 1]) {
            pick = k;
            break;
        }
    }
    return BlockResult{grand, se[pick], count[pick]};
}

// ------------------------------------------------------------------ core/units.hpp
namespace units {
inline constexpr double kTauInPicoseconds = 1.0966875353;  // core/units.hpp:33
inline constexpr double picoseconds(double ps) { return ps / kTauInPicoseconds; }
inline constexpr double femtoseconds(double fs) { return picoseconds(fs * 1.0e-3); }
inline constexpr double toPicoseconds(double tau) { return tau * kTauInPicoseconds; }
}  // namespace units

// ------------------------------------------------------------- util/random.hpp
// Rng lives in moldyn_b200_rng.hpp (the library's lattice setup draws the same
// stream); md_rng_normals gives the same draws from C.

// ------------------------------------------------------------ io/nist_config.hpp
struct NistConfig {
    System system;
    std::vector<std::string> types;
};

// readNistConfig (io/nist_config.cpp:30-86): line 1 the box, line 2 a count that
// is not trusted (the SPC/E files give molecules), then "index x y z [type]" lines
// to the end of the file; blank lines are skipped, every atom gets mass 1 and zero
// velocity.  Throws std::runtime_error on a missing file or a malformed line.
inline NistConfig readNistConfig(const std::string& path) {
    std::ifstream in(path);
    if (!in.is_open()) throw std::runtime_error("readNistConfig: cannot open file " + path);
    std::string line;
    if (!std::getline(in, line)) throw std::runtime_error("readNistConfig: empty file " + path);
    double lx = 0.0, ly = 0.0, lz = 0.0;
    {
        std::istringstream iss(line);
        if (!(iss >> lx >> ly >> lz))
            throw std::runtime_error("readNistConfig: malformed box line in " + path);
    }
    if (!std::getline(in, line)) throw std::runtime_error("readNistConfig: missing count line in " + path);
    {
        std::istringstream iss(line);
        long declared = 0;
        if (!(iss >> declared))
            throw std::runtime_error("readNistConfig: malformed count line in " + path);
    }
    NistConfig cfg{System(Box(Vec3{lx, ly, lz})), {}};
    std::vector<std::string> types;
    bool typed = false;
    while (std::getline(in, line)) {
        if (line.find_first_not_of(" \t\r\n") == std::string::npos) continue;
        std::istringstream iss(line);
        long index = 0;
        double x = 0.0, y = 0.0, z = 0.0;
        if (!(iss >> index >> x >> y >> z))
            throw std::runtime_error("readNistConfig: malformed atom line in " + path);
        std::string type;
        const bool has_type = static_cast<bool>(iss >> type);
        cfg.system.addAtom(Vec3{x, y, z}, Vec3{0.0, 0.0, 0.0}, 1.0);
        types.push_back(has_type ? type : std::string());
        typed = typed || has_type;
    }
    if (typed) cfg.types = std::move(types);
    return cfg;
}

// ------------------------------------------------------------ forcefield/spce.hpp
struct SpceSystem {
    System full;
    System oxygens;
    std::size_t moleculeCount = 0;
};

// buildSpceSystem (forcefield/spce.cpp:8-40): O, H, H triples with the model's
// charges and masses, molecule id = index / 3; `oxygens` holds the O sites alone.
inline SpceSystem buildSpceSystem(const NistConfig& cfg, const SpceParameters& params = SpceParameters()) {
    const std::size_t n = cfg.system.size();
    if (n == 0 || n % 3 != 0)
        throw std::invalid_argument(
            "buildSpceSystem: atom count must be a positive multiple of 3 (O, H, H per molecule)");
    if (cfg.types.size() != n) throw std::invalid_argument("buildSpceSystem: config has no per-atom types");
    const double qO = -2.0 * params.qH;
    SpceSystem out{System(cfg.system.box()), System(cfg.system.box()), n / 3};
    out.full.reserve(n);
    for (std::size_t i = 0; i < n; ++i) {
        const Vec3 r = cfg.system.position(i), v = cfg.system.velocity(i);
        if (cfg.types[i] == "O") {
            out.full.addAtom(r, v, params.massOxygen, qO, i / 3);
            out.oxygens.addAtom(r, v, params.massOxygen);
        } else if (cfg.types[i] == "H") {
            out.full.addAtom(r, v, params.massHydrogen, params.qH, i / 3);
        } else {
            throw std::invalid_argument("buildSpceSystem: unrecognised atom type '" + cfg.types[i] +
                                        "' (expected \"O\" or \"H\")");
        }
    }
    return out;
}

// Extension: the simulation of apps/water_rdf.cpp:186-216 as one device call
// (md_water_rdf_run): `equilibrate` steps rescaled toward `temperature` and
// re-constrained every `rescaleEvery`, then `production` NVE steps with the
// oxygens (atoms 0, 3, 6, ...) accumulated into rdf every `sampleEvery`.
// Returns the mean production temperature.
inline double runWaterRdf(ConstrainedVelocityVerlet& integ, System& sys, const SpceForceField& ff,
                          Rdf& rdf, double temperature, std::size_t dof, int64_t equilibrate,
                          int64_t rescaleEvery, int64_t production, int64_t sampleEvery) {
    double mean = 0.0;
    detail::check(md_water_rdf_run(integ.handle(), sys.device(), ff.handle(), rdf.handle(),
                                   temperature, static_cast<int64_t>(dof), equilibrate, rescaleEvery,
                                   production, sampleEvery, &mean));
    sys.deviceChanged();
    return mean;
}

}  // namespace moldyn_b200
