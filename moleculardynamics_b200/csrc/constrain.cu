// constrain.cu -- rigid three-site water (constrain/rigid_water.cpp) and the
// constrained velocity-Verlet step (integrate/constrained_velocity_verlet.hpp) on
// the device, plus its Nose-Hoover-chain variant (no reference counterpart).
//
// SHAKE/RATTLE run one thread per molecule.  The reference sweeps all molecules
// Gauss-Seidel style until the worst violation over the whole system is below the
// tolerance; molecules share no atoms and a molecule whose three violations are
// already within tolerance is left untouched by every later sweep, so iterating
// each molecule to its own convergence gives identical positions and velocities,
// and the reference's iteration count is the maximum over molecules.  Each update
// uses the reference's operation order, so results are bit-identical to it.
#include <cmath>
#include <limits>
#include <new>

#include "md_device.cuh"
#include "md_internal.cuh"

namespace mdb {
int nhc_pre_async(md_integrator* it, md_context* ctx, const double* ke_now);
int nhc_post_async(md_integrator* it, md_context* ctx, const double* ke_sum);
int nhc_apply_scale_async(md_integrator* it, md_system* sys);
int record_async(md_context* ctx, const double* ev, const double* ke, const NhcState* nhc,
                 double* row);
int ewald_eval_async(md_ewald* ew, md_system* sys, int mode, bool gated);
int system_kinetic_async(md_system* sys, int slot);
int record_at_async(md_context* ctx, const NhcState* nhc, double* rows, int* idx);
}  // namespace mdb

namespace mdb {
namespace {

constexpr int kBlock = 128;
constexpr double kPi = 3.14159265358979323846;
// The constraints' atom pairs (O-H1, O-H2, H1-H2), as compile-time indices so
// that a molecule's coordinates stay in registers in the unrolled sweeps.
__host__ __device__ constexpr int cons_i(int c) { return c == 2 ? 1 : 0; }
__host__ __device__ constexpr int cons_j(int c) { return c == 0 ? 1 : 2; }

struct RigidArgs {
    double target2[3];  // squared O-H, O-H, H-H distances
    // within[c]: the largest x >= 0 whose rounded quotient x / target2[c] is at
    // most the tolerance, so that |s| / d2 <= tolerance (rigid_water.cpp:85-91,
    // 139-146) is decided by |s| <= within[c] without the division
    double within[3];
    double tolerance;
    int max_iterations;
    int settle;         // closed-form SETTLE instead of SHAKE / RATTLE iterations
    double oh, hh;
};

// Largest x >= 0 with RN(x / d2) <= tol (IEEE division on the host, rounded to
// nearest like __ddiv_rn).  x -> RN(x / d2) is non-decreasing, so the set of
// such x is an interval [0, within] and |s| / d2 <= tol exactly when
// |s| <= within; a NaN fails both tests, an infinity fails both.
double tolerance_bound(double d2, double tol) {
    if (!(d2 > 0.0) || !(tol >= 0.0)) return -1.0;  // nothing passes; the division decides
    double x = tol * d2;
    if (!std::isfinite(x)) x = std::numeric_limits<double>::max();
    for (int k = 0; k < 64 && x > 0.0 && x / d2 > tol; ++k) x = std::nextafter(x, 0.0);
    for (int k = 0; k < 64; ++k) {
        const double up = std::nextafter(x, std::numeric_limits<double>::infinity());
        if (!std::isfinite(up) || up / d2 > tol) break;
        x = up;
    }
    return x / d2 <= tol ? x : -1.0;
}

RigidArgs rigid_args(const md_rigid& rw) {
    RigidArgs a;
    a.target2[0] = rw.oh * rw.oh;
    a.target2[1] = rw.oh * rw.oh;
    a.target2[2] = rw.hh * rw.hh;
    for (int c = 0; c < 3; ++c) a.within[c] = tolerance_bound(a.target2[c], rw.tolerance);
    a.tolerance = rw.tolerance;
    a.max_iterations = rw.max_iterations;
    a.settle = rw.settle ? 1 : 0;
    a.oh = rw.oh;
    a.hh = rw.hh;
    return a;
}

__device__ __forceinline__ double dot_exact(double ax, double ay, double az, double bx, double by,
                                            double bz) {
    return __dadd_rn(__dadd_rn(__dmul_rn(ax, bx), __dmul_rn(ay, by)), __dmul_rn(az, bz));
}

struct Mol {
    double x[3], y[3], z[3];
};

// rigid_water.cpp:61-116 for one molecule.  Returns iterations, -1 (no
// convergence) or -2 (singular denominator).
// The reference bond vectors and the inverse-mass sums do not change during the
// iterations; they are formed once, with the same operations, before the sweeps.
__device__ int shake_molecule(Mol& r, const Mol& ref, const double m[3], const RigidArgs& a,
                              const Fold3& f3) {
    double b[3][3], two_inv_mass[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const int i = cons_i(c), j = cons_j(c);
        min_image_wrapped(f3, ref.x[i], ref.y[i], ref.z[i], ref.x[j], ref.y[j], ref.z[j], b[c][0],
                          b[c][1], b[c][2]);
        two_inv_mass[c] = __dmul_rn(2.0, __dadd_rn(__ddiv_rn(1.0, m[i]), __ddiv_rn(1.0, m[j])));
    }
    for (int it = 0; it < a.max_iterations; ++it) {
        bool open = false;  // some violation above the tolerance (worst > tolerance)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int i = cons_i(c), j = cons_j(c);
            const double d2 = a.target2[c];
            double ax, ay, az;
            min_image_wrapped(f3, r.x[i], r.y[i], r.z[i], r.x[j], r.y[j], r.z[j], ax, ay, az);
            const double s = __dsub_rn(norm2_exact(ax, ay, az), d2);
            if (fabs(s) > a.within[c]) open = true;
            if (fabs(s) <= a.within[c]) continue;
            const double bx = b[c][0], by = b[c][1], bz = b[c][2];
            const double denom = __dmul_rn(two_inv_mass[c], dot_exact(ax, ay, az, bx, by, bz));
            if (fabs(denom) < 1e-30) return -2;
            const double g = __ddiv_rn(s, denom);
            const double gi = __ddiv_rn(g, m[i]), gj = __ddiv_rn(g, m[j]);
            r.x[i] = __dsub_rn(r.x[i], __dmul_rn(bx, gi));
            r.y[i] = __dsub_rn(r.y[i], __dmul_rn(by, gi));
            r.z[i] = __dsub_rn(r.z[i], __dmul_rn(bz, gi));
            r.x[j] = __dadd_rn(r.x[j], __dmul_rn(bx, gj));
            r.y[j] = __dadd_rn(r.y[j], __dmul_rn(by, gj));
            r.z[j] = __dadd_rn(r.z[j], __dmul_rn(bz, gj));
        }
        if (!open) return it + 1;
    }
    return -1;
}

// SETTLE (Miyamoto & Kollman, J. Comput. Chem. 13, 952 (1992)): the positions
// SHAKE converges to, in closed form.  The three corrections act along the
// reference bonds, so they lie in the reference molecular plane: in a frame whose
// z axis is that plane's normal the z coordinates keep their unconstrained values,
// which fixes the two tilts (phi about x, psi about y) of the canonical triangle,
// and the in-plane rotation theta makes the corrections' torque vanish,
// alpha sin(theta) + beta cos(theta) = gamma.  Work is local to the molecule
// (bond vectors by minimum image from the oxygen), and the corrections are added
// to the original coordinates as SHAKE's are.  Needs equal hydrogen masses;
// returns 1, or 0 when the configuration has no solution (then SHAKE runs).
__device__ int settle_molecule(Mol& r, const Mol& ref, const double m[3], const RigidArgs& a,
                               const Fold3& f3) {
    if (m[1] != m[2]) return 0;
    const double mo = m[0], mh = m[1], M = mo + 2.0 * mh;
    const double rc = 0.5 * a.hh;
    const double h = sqrt(a.oh * a.oh - rc * rc);  // O above the H-H midpoint
    const double ra = 2.0 * mh * h / M;             // centre of mass to O
    const double rb = h - ra;                       // centre of mass to the H-H midpoint
    // reference bonds from O, and the unconstrained positions relative to O
    double b0[3], c0[3], p1[3][3];
    min_image_wrapped(f3, ref.x[1], ref.y[1], ref.z[1], ref.x[0], ref.y[0], ref.z[0], b0[0], b0[1], b0[2]);
    min_image_wrapped(f3, ref.x[2], ref.y[2], ref.z[2], ref.x[0], ref.y[0], ref.z[0], c0[0], c0[1], c0[2]);
    p1[0][0] = p1[0][1] = p1[0][2] = 0.0;
    min_image_wrapped(f3, r.x[1], r.y[1], r.z[1], r.x[0], r.y[0], r.z[0], p1[1][0], p1[1][1], p1[1][2]);
    min_image_wrapped(f3, r.x[2], r.y[2], r.z[2], r.x[0], r.y[0], r.z[0], p1[2][0], p1[2][1], p1[2][2]);
    double d[3];  // centre of mass of the unconstrained molecule
    for (int k = 0; k < 3; ++k) d[k] = (mh * p1[1][k] + mh * p1[2][k]) / M;
    double A1[3], B1[3], C1[3];
    for (int k = 0; k < 3; ++k) {
        A1[k] = p1[0][k] - d[k];
        B1[k] = p1[1][k] - d[k];
        C1[k] = p1[2][k] - d[k];
    }
    // frame: ez normal to the reference plane, ex perpendicular to ez and A1
    double ez[3] = {b0[1] * c0[2] - b0[2] * c0[1], b0[2] * c0[0] - b0[0] * c0[2],
                    b0[0] * c0[1] - b0[1] * c0[0]};
    double ex[3] = {A1[1] * ez[2] - A1[2] * ez[1], A1[2] * ez[0] - A1[0] * ez[2],
                    A1[0] * ez[1] - A1[1] * ez[0]};
    const double nz = sqrt(ez[0] * ez[0] + ez[1] * ez[1] + ez[2] * ez[2]);
    const double nx = sqrt(ex[0] * ex[0] + ex[1] * ex[1] + ex[2] * ex[2]);
    if (!(nz > 0.0) || !(nx > 0.0)) return 0;
    for (int k = 0; k < 3; ++k) {
        ez[k] /= nz;
        ex[k] /= nx;
    }
    const double ey[3] = {ez[1] * ex[2] - ez[2] * ex[1], ez[2] * ex[0] - ez[0] * ex[2],
                          ez[0] * ex[1] - ez[1] * ex[0]};
    auto px = [&](const double* v) { return v[0] * ex[0] + v[1] * ex[1] + v[2] * ex[2]; };
    auto py = [&](const double* v) { return v[0] * ey[0] + v[1] * ey[1] + v[2] * ey[2]; };
    auto pz = [&](const double* v) { return v[0] * ez[0] + v[1] * ez[1] + v[2] * ez[2]; };
    // tilts from the out-of-plane coordinates
    const double sphi = pz(A1) / ra;
    const double cphi2 = 1.0 - sphi * sphi;
    if (!(cphi2 > 0.0)) return 0;
    const double cphi = sqrt(cphi2);
    const double spsi = (pz(B1) - pz(C1)) / (2.0 * rc * cphi);
    const double cpsi2 = 1.0 - spsi * spsi;
    if (!(cpsi2 > 0.0)) return 0;
    const double cpsi = sqrt(cpsi2);
    // the tilted canonical triangle (O on +y, H1 at -x, H2 at +x), in-plane coordinates
    const double x2[3] = {0.0, -rc * cpsi, rc * cpsi};
    const double y2[3] = {ra * cphi, -rb * cphi - rc * spsi * sphi, -rb * cphi + rc * spsi * sphi};
    // reference (x0, y0) and unconstrained (x1, y1) in-plane coordinates; the torque
    // about any point is the same since the corrections sum to zero
    const double x0[3] = {0.0, px(b0), px(c0)}, y0[3] = {0.0, py(b0), py(c0)};
    const double x1[3] = {px(A1), px(B1), px(C1)}, y1[3] = {py(A1), py(B1), py(C1)};
    double alpha = 0.0, beta = 0.0, gamma = 0.0;
    for (int k = 0; k < 3; ++k) {
        alpha += m[k] * (x0[k] * x2[k] + y0[k] * y2[k]);
        beta += m[k] * (x0[k] * y2[k] - y0[k] * x2[k]);
        gamma += m[k] * (x0[k] * y1[k] - y0[k] * x1[k]);
    }
    const double r2 = alpha * alpha + beta * beta;
    const double disc = r2 - gamma * gamma;
    if (!(r2 > 0.0) || !(disc >= 0.0)) return 0;
    const double sq = sqrt(disc);
    const double sth = (alpha * gamma - beta * sq) / r2;  // the root near theta = 0
    const double cth = (alpha * sq + beta * gamma) / r2;
    // constrained positions relative to the centre of mass, then the corrections
    for (int k = 0; k < 3; ++k) {
        const double x3 = x2[k] * cth - y2[k] * sth;
        const double y3 = x2[k] * sth + y2[k] * cth;
        const double z3 = pz(k == 0 ? A1 : (k == 1 ? B1 : C1));
        const double* q1 = k == 0 ? A1 : (k == 1 ? B1 : C1);
        const double dx = x3 - px(q1), dy = y3 - py(q1), dz = z3 - pz(q1);
        r.x[k] += dx * ex[0] + dy * ey[0] + dz * ez[0];
        r.y[k] += dx * ex[1] + dy * ey[1] + dz * ez[1];
        r.z[k] += dx * ex[2] + dy * ey[2] + dz * ez[2];
    }
    return 1;
}

// The velocity half of SETTLE: the multipliers of the three bond constraints
// solve one 3x3 linear system (RATTLE's fixed point), by Cramer's rule.
// Returns 1, or 0 for a singular system (then RATTLE runs).
__device__ int settle_velocities(const Mol& r, Mol& v, const double m[3], const Fold3& f3) {
    double rab[3], rac[3], rbc[3];
    min_image_wrapped(f3, r.x[0], r.y[0], r.z[0], r.x[1], r.y[1], r.z[1], rab[0], rab[1], rab[2]);
    min_image_wrapped(f3, r.x[0], r.y[0], r.z[0], r.x[2], r.y[2], r.z[2], rac[0], rac[1], rac[2]);
    min_image_wrapped(f3, r.x[1], r.y[1], r.z[1], r.x[2], r.y[2], r.z[2], rbc[0], rbc[1], rbc[2]);
    auto dot3 = [](const double* p, const double* q) { return p[0] * q[0] + p[1] * q[1] + p[2] * q[2]; };
    const double vab[3] = {v.x[0] - v.x[1], v.y[0] - v.y[1], v.z[0] - v.z[1]};
    const double vac[3] = {v.x[0] - v.x[2], v.y[0] - v.y[2], v.z[0] - v.z[2]};
    const double vbc[3] = {v.x[1] - v.x[2], v.y[1] - v.y[2], v.z[1] - v.z[2]};
    const double ia = 1.0 / m[0], ib = 1.0 / m[1], ic = 1.0 / m[2];
    const double abab = dot3(rab, rab), acac = dot3(rac, rac), bcbc = dot3(rbc, rbc);
    const double abac = dot3(rab, rac), abbc = dot3(rab, rbc), acbc = dot3(rac, rbc);
    // rows: (dv_a - dv_b).r_ab, (dv_a - dv_c).r_ac, (dv_b - dv_c).r_bc = -(v_ij . r_ij)
    const double A[3][3] = {{(ia + ib) * abab, ia * abac, -ib * abbc},
                            {ia * abac, (ia + ic) * acac, ic * acbc},
                            {-ib * abbc, ic * acbc, (ib + ic) * bcbc}};
    const double b[3] = {-dot3(vab, rab), -dot3(vac, rac), -dot3(vbc, rbc)};
    const double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                       A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                       A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
    if (!(fabs(det) > 1e-300)) return 0;
    double lam[3];
    for (int c = 0; c < 3; ++c) {
        double Mc[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) Mc[i][j] = j == c ? b[i] : A[i][j];
        lam[c] = (Mc[0][0] * (Mc[1][1] * Mc[2][2] - Mc[1][2] * Mc[2][1]) -
                  Mc[0][1] * (Mc[1][0] * Mc[2][2] - Mc[1][2] * Mc[2][0]) +
                  Mc[0][2] * (Mc[1][0] * Mc[2][1] - Mc[1][1] * Mc[2][0])) / det;
    }
    // dv_a = (l_ab r_ab + l_ac r_ac)/m_a, dv_b = (-l_ab r_ab + l_bc r_bc)/m_b,
    // dv_c = (-l_ac r_ac - l_bc r_bc)/m_c
    const double da[3] = {(lam[0] * rab[0] + lam[1] * rac[0]) * ia, (lam[0] * rab[1] + lam[1] * rac[1]) * ia,
                          (lam[0] * rab[2] + lam[1] * rac[2]) * ia};
    const double db[3] = {(-lam[0] * rab[0] + lam[2] * rbc[0]) * ib, (-lam[0] * rab[1] + lam[2] * rbc[1]) * ib,
                          (-lam[0] * rab[2] + lam[2] * rbc[2]) * ib};
    const double dc[3] = {(-lam[1] * rac[0] - lam[2] * rbc[0]) * ic, (-lam[1] * rac[1] - lam[2] * rbc[1]) * ic,
                          (-lam[1] * rac[2] - lam[2] * rbc[2]) * ic};
    v.x[0] += da[0]; v.y[0] += da[1]; v.z[0] += da[2];
    v.x[1] += db[0]; v.y[1] += db[1]; v.z[1] += db[2];
    v.x[2] += dc[0]; v.y[2] += dc[1]; v.z[2] += dc[2];
    return 1;
}

// Position and velocity constraints of one molecule by the configured method.
__device__ __forceinline__ int constrain_positions(Mol& r, const Mol& ref, const double m[3],
                                                   const RigidArgs& a, const Fold3& f3) {
    if (a.settle && settle_molecule(r, ref, m, a, f3)) return 1;
    return shake_molecule(r, ref, m, a, f3);
}

// rigid_water.cpp:118-161 for one molecule.
// Positions are fixed during the iterations: the bond vectors, their squared
// lengths times the inverse-mass sums, are formed once before the sweeps.
__device__ int rattle_molecule(const Mol& r, Mol& v, const double m[3], const RigidArgs& a,
                               const Fold3& f3) {
    double b[3][3], mass_norm[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const int i = cons_i(c), j = cons_j(c);
        min_image_wrapped(f3, r.x[i], r.y[i], r.z[i], r.x[j], r.y[j], r.z[j], b[c][0], b[c][1],
                          b[c][2]);
        const double inv_mass_sum = __dadd_rn(__ddiv_rn(1.0, m[i]), __ddiv_rn(1.0, m[j]));
        mass_norm[c] = __dmul_rn(inv_mass_sum, norm2_exact(b[c][0], b[c][1], b[c][2]));
    }
    for (int it = 0; it < a.max_iterations; ++it) {
        bool open = false;  // some |r.v| / d2 above the tolerance
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int i = cons_i(c), j = cons_j(c);
            const double ax = b[c][0], ay = b[c][1], az = b[c][2];
            const double ux = __dsub_rn(v.x[i], v.x[j]), uy = __dsub_rn(v.y[i], v.y[j]),
                         uz = __dsub_rn(v.z[i], v.z[j]);
            const double rv = dot_exact(ax, ay, az, ux, uy, uz);
            if (fabs(rv) > a.within[c]) open = true;
            if (fabs(rv) <= a.within[c]) continue;
            const double k = __ddiv_rn(rv, mass_norm[c]);
            const double ki = __ddiv_rn(k, m[i]), kj = __ddiv_rn(k, m[j]);
            v.x[i] = __dsub_rn(v.x[i], __dmul_rn(ax, ki));
            v.y[i] = __dsub_rn(v.y[i], __dmul_rn(ay, ki));
            v.z[i] = __dsub_rn(v.z[i], __dmul_rn(az, ki));
            v.x[j] = __dadd_rn(v.x[j], __dmul_rn(ax, kj));
            v.y[j] = __dadd_rn(v.y[j], __dmul_rn(ay, kj));
            v.z[j] = __dadd_rn(v.z[j], __dmul_rn(az, kj));
        }
        if (!open) return it + 1;
    }
    return -1;
}

struct MolSlots {
    int s[3];
};

__device__ __forceinline__ MolSlots mol_slots(const int* slot, int64_t m) {
    return MolSlots{{slot[3 * m], slot[3 * m + 1], slot[3 * m + 2]}};
}

__device__ __forceinline__ void load_pos(const md_atoms& a, const MolSlots& ms, Mol& r) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double4 p = a.pos[ms.s[k]];
        r.x[k] = p.x;
        r.y[k] = p.y;
        r.z[k] = p.z;
    }
}

__device__ __forceinline__ void store_pos(md_atoms& a, const MolSlots& ms, const Mol& r) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double4 p = a.pos[ms.s[k]];
        p.x = r.x[k];
        p.y = r.y[k];
        p.z = r.z[k];
        a.pos[ms.s[k]] = p;
    }
}

__device__ __forceinline__ void load_vel(const md_atoms& a, const MolSlots& ms, Mol& v) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        v.x[k] = a.vx[ms.s[k]];
        v.y[k] = a.vy[ms.s[k]];
        v.z[k] = a.vz[ms.s[k]];
    }
}

__device__ __forceinline__ void store_vel(md_atoms& a, const MolSlots& ms, const Mol& v) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        a.vx[ms.s[k]] = v.x[k];
        a.vy[ms.s[k]] = v.y[k];
        a.vz[ms.s[k]] = v.z[k];
    }
}

__device__ __forceinline__ void report(int it, int* max_it, uint32_t* status, uint32_t fail_bit) {
    if (it > 0) atomicMax(max_it, it);
    else atomicOr(status, it == -2 ? MD_STATUS_SHAKE_SINGULAR : fail_bit);
}

// constrainPositions with reference positions given in original order.
__global__ void k_shake(md_atoms a, const int* __restrict__ slot, int64_t nmol,
                        const double* __restrict__ rx, const double* __restrict__ ry,
                        const double* __restrict__ rz, RigidArgs ra, Box3 box, int* max_it,
                        uint32_t* status) {
    const int64_t m = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (m >= nmol) return;
    const Fold3 f3 = fold3_of(box);
    const MolSlots ms = mol_slots(slot, m);
    Mol r, ref;
    load_pos(a, ms, r);
    double mass[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        ref.x[k] = rx[3 * m + k];
        ref.y[k] = ry[3 * m + k];
        ref.z[k] = rz[3 * m + k];
        mass[k] = a.mass[ms.s[k]];
    }
    const int it = constrain_positions(r, ref, mass, ra, f3);
    report(it, max_it, status, MD_STATUS_SHAKE_DIVERGED);
    store_pos(a, ms, r);
}

__global__ void k_rattle(md_atoms a, const int* __restrict__ slot, int64_t nmol, RigidArgs ra,
                         Box3 box, int* max_it, uint32_t* status) {
    const int64_t m = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (m >= nmol) return;
    const Fold3 f3 = fold3_of(box);
    const MolSlots ms = mol_slots(slot, m);
    Mol r, v;
    load_pos(a, ms, r);
    load_vel(a, ms, v);
    double mass[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) mass[k] = a.mass[ms.s[k]];
    const int it = ra.settle && settle_velocities(r, v, mass, f3) ? 1 : rattle_molecule(r, v, mass, ra, f3);
    report(it, max_it, status, MD_STATUS_RATTLE_DIVERGED);
    store_vel(a, ms, v);
}

struct CvvArgs {
    double dt, half_dt, inv_dt;
    RigidArgs ra;
    Box3 box;
};

// constrained_velocity_verlet.hpp:31-52: reference = r; kick; drift (no wrap);
// SHAKE along the reference bonds; velocity correction shift / dt.  An NHC
// pending scale (if any) is applied to the velocities first.
__global__ void k_cvv_pre(md_atoms a, const int* __restrict__ slot, int64_t nmol, CvvArgs c,
                          const NhcState* nhc, int* max_it, uint32_t* status) {
    const int64_t m = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (m >= nmol) return;
    const Fold3 f3 = fold3_of(c.box);
    const MolSlots ms = mol_slots(slot, m);
    Mol r, v, ref, unc;
    load_pos(a, ms, r);
    load_vel(a, ms, v);
    ref = r;
    double mass[3];
    const double sc = nhc ? nhc->scale : 1.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int s = ms.s[k];
        mass[k] = a.mass[s];
        if (nhc) {
            v.x[k] = __dmul_rn(v.x[k], sc);
            v.y[k] = __dmul_rn(v.y[k], sc);
            v.z[k] = __dmul_rn(v.z[k], sc);
        }
        const double kc = __ddiv_rn(c.half_dt, mass[k]);  // 0.5 * dt_ / mass
        v.x[k] = __dadd_rn(v.x[k], __dmul_rn(a.fx[s], kc));
        v.y[k] = __dadd_rn(v.y[k], __dmul_rn(a.fy[s], kc));
        v.z[k] = __dadd_rn(v.z[k], __dmul_rn(a.fz[s], kc));
        r.x[k] = __dadd_rn(r.x[k], __dmul_rn(v.x[k], c.dt));
        r.y[k] = __dadd_rn(r.y[k], __dmul_rn(v.y[k], c.dt));
        r.z[k] = __dadd_rn(r.z[k], __dmul_rn(v.z[k], c.dt));
    }
    unc = r;
    const int it = constrain_positions(r, ref, mass, c.ra, f3);
    report(it, max_it, status, MD_STATUS_SHAKE_DIVERGED);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double sx, sy, sz;
        min_image_wrapped(f3, r.x[k], r.y[k], r.z[k], unc.x[k], unc.y[k], unc.z[k], sx, sy, sz);
        v.x[k] = __dadd_rn(v.x[k], __dmul_rn(sx, c.inv_dt));
        v.y[k] = __dadd_rn(v.y[k], __dmul_rn(sy, c.inv_dt));
        v.z[k] = __dadd_rn(v.z[k], __dmul_rn(sz, c.inv_dt));
    }
    store_pos(a, ms, r);
    store_vel(a, ms, v);
}

// constrained_velocity_verlet.hpp:54-56: kick; RATTLE; kinetic-energy sum.
__global__ void __launch_bounds__(kBlock)
k_cvv_post(md_atoms a, const int* __restrict__ slot, int64_t nmol, CvvArgs c, int* max_it,
           uint32_t* status, double* part, unsigned* ticket, double* ke_out) {
    const int64_t m = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    double ke[1] = {0.0};
    if (m < nmol) {
        const Fold3 f3 = fold3_of(c.box);
        const MolSlots ms = mol_slots(slot, m);
        Mol r, v;
        load_pos(a, ms, r);
        load_vel(a, ms, v);
        double mass[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int s = ms.s[k];
            mass[k] = a.mass[s];
            const double kc = __ddiv_rn(c.half_dt, mass[k]);
            v.x[k] = __dadd_rn(v.x[k], __dmul_rn(a.fx[s], kc));
            v.y[k] = __dadd_rn(v.y[k], __dmul_rn(a.fy[s], kc));
            v.z[k] = __dadd_rn(v.z[k], __dmul_rn(a.fz[s], kc));
        }
        const int it = c.ra.settle && settle_velocities(r, v, mass, f3) ? 1 : rattle_molecule(r, v, mass, c.ra, f3);
        report(it, max_it, status, MD_STATUS_RATTLE_DIVERGED);
        store_vel(a, ms, v);
#pragma unroll
        for (int k = 0; k < 3; ++k)
            ke[0] += 0.5 * mass[k] * (v.x[k] * v.x[k] + v.y[k] * v.y[k] + v.z[k] * v.z[k]);
    }
    grid_reduce<1>(ke, part, ticket, ke_out);
}

// SPC/E potential energy from the Ewald result slots (spce_forcefield.cpp:40):
// disp + elrc + (real + reciprocal + self + intra); self = self_coef * sum q^2.
__global__ void k_spce_total(const double* ew, double elrc, double self_coef, double* ev) {
    // ew slots: 0 real, 1 W real, 2 lj, 3 W lj, 4 intra, 5 W intra, 6 recip, 7 W recip, 8 sum q^2
    const double self = self_coef * ew[8];
    ev[0] = ew[2] + elrc + (ew[0] + ew[6] + self + ew[4]);
    ev[1] = ew[1] + ew[3] + ew[5] + ew[7];
}

Box3 box_of(const md_system* sys) {
    Box3 b;
    for (int d = 0; d < 3; ++d) {
        b.L[d] = sys->box[d];
        b.inv[d] = sys->inv_box[d];
    }
    return b;
}

CvvArgs cvv_args(const md_integrator* it, const md_system* sys) {
    CvvArgs c;
    c.dt = it->dt;
    c.half_dt = 0.5 * it->dt;
    c.inv_dt = 1.0 / it->dt;
    c.ra = rigid_args(it->rigid);
    c.box = box_of(sys);
    return c;
}

int check_triples(const md_system* sys, const char* who) {
    if (sys->n % 3 != 0)  // rigid_water.cpp:63-68
        return fail(MD_ERR_RUNTIME, "%s: atom count is not a multiple of 3", who);
    return MD_OK;
}

int ensure_counters(md_integrator* it) {
    if (!it->counters.ptr) {
        MDB_TRY(it->counters.ensure(4 * sizeof(int)));
        MDB_CUDA(cudaMemset(it->counters.ptr, 0, 4 * sizeof(int)));
    }
    return MD_OK;
}

int status_to_error(md_context* ctx) {
    uint32_t st = 0;
    MDB_CUDA(cudaMemcpyAsync(&st, ctx->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    const uint32_t bits = MD_STATUS_SHAKE_DIVERGED | MD_STATUS_RATTLE_DIVERGED | MD_STATUS_SHAKE_SINGULAR;
    if (st & bits) {
        const uint32_t keep = st & ~bits;
        MDB_CUDA(cudaMemcpyAsync(ctx->d_status, &keep, sizeof(uint32_t), cudaMemcpyHostToDevice, ctx->stream));
        MDB_CUDA(cudaStreamSynchronize(ctx->stream));
        // rigid_water.cpp:63-68, 100-104, 114-115, 159-160 throw std::runtime_error
        if (st & MD_STATUS_SHAKE_SINGULAR)
            return fail(MD_ERR_RUNTIME, "RigidWater: constraint became singular (bond rotated ~90 "
                                        "degrees in one step); the timestep is far too large");
        if (st & MD_STATUS_SHAKE_DIVERGED)
            return fail(MD_ERR_RUNTIME, "RigidWater: SHAKE failed to converge");
        return fail(MD_ERR_RUNTIME, "RigidWater: RATTLE failed to converge");
    }
    return MD_OK;
}

// A fused loop of constrained steps with SPC/E forces
// (constrained_velocity_verlet.hpp:27-57, the Ewald sum between the halves),
// every launch on the context's stream and no host synchronisation per step.
struct SpceLoop {
    md_integrator* it = nullptr;
    md_system* sys = nullptr;
    md_ewald* ff = nullptr;
    NhcState* nhc = nullptr;
    int64_t nmol = 0;
    int g = 1;
    double elrc = 0.0, self_coef = 0.0;
};

int spce_loop_begin(md_integrator* it, md_system* sys, md_ewald* ff, const char* who, SpceLoop& L) {
    if (it->kind < 3) return fail(MD_ERR_INVALID_ARGUMENT, "%s: needs a constrained integrator", who);
    MDB_TRY(check_triples(sys, who));
    // Forces are made current on entry; this also builds the force field's
    // neighbour list and topology once, host-side.
    double e0, parts[8];
    MDB_TRY(md_spce_compute(ff, sys, 1, &e0, parts));
    MDB_TRY(ensure_counters(it));
    double alpha = 0.0;
    MDB_TRY(md_ewald_alpha(ff, &alpha));
    L.it = it;
    L.sys = sys;
    L.ff = ff;
    L.elrc = parts[1];
    L.self_coef = -md_coulomb_prefactor() * alpha / std::sqrt(kPi);
    L.nhc = it->kind == 4 ? it->chain_state.as<NhcState>() : nullptr;
    L.nmol = sys->n / 3;
    L.g = grid_for(std::max<int64_t>(L.nmol, 1), kBlock);
    if (L.nhc) MDB_TRY(system_kinetic_async(sys, kResKE));
    return MD_OK;
}

// One step; `first` feeds the chain the entry kinetic energy, `row` (device,
// or null) receives [energy, virial, kinetic, conserved].  The step's kinetic
// energy is left in the kResKE result slot.
int spce_step_async(SpceLoop& L, bool first, double* row) {
    md_system* sys = L.sys;
    md_integrator* it = L.it;
    md_context* ctx = sys->ctx;
    if (L.nhc) MDB_TRY(nhc_pre_async(it, ctx, first ? ctx_result(ctx, kResKE) : nullptr));
    if (L.nmol > 0) {
        k_cvv_pre<<<grid_for(L.nmol, kBlock), kBlock, 0, ctx->stream>>>(
            sys->cur, sys->slot, L.nmol, cvv_args(it, sys), L.nhc, it->counters.as<int>(),
            ctx->d_status);
        ++ctx->launches;
    }
    MDB_TRY(ewald_eval_async(L.ff, sys, 1, true));
    k_spce_total<<<1, 1, 0, ctx->stream>>>(ctx_result(ctx, kResEwald), L.elrc, L.self_coef,
                                           ctx_result(ctx, kResEnergy));
    double* part;  // fetched after the Ewald sum, which may grow the partials
    MDB_TRY(ctx_partials(ctx, static_cast<size_t>(L.g), &part));
    k_cvv_post<<<L.g, kBlock, 0, ctx->stream>>>(sys->cur, sys->slot, L.nmol, cvv_args(it, sys),
                                               it->counters.as<int>() + 1, ctx->d_status, part,
                                               ctx_counter(ctx, 8), ctx_result(ctx, kResKE));
    ctx->launches += 2;
    if (L.nhc) MDB_TRY(nhc_post_async(it, ctx, ctx_result(ctx, kResKE)));
    if (row) MDB_TRY(record_async(ctx, ctx_result(ctx, kResEnergy), ctx_result(ctx, kResKE), L.nhc, row));
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

// apps/water_rdf.cpp:211 summed on the device: acc += 2 KE / dof (system.cpp:133-135),
// one launch per step so the additions run in step order.
__global__ void k_sum_temperature(const double* __restrict__ ke, double dof, double* acc) {
    acc[0] += 2.0 * ke[0] / dof;
}

// A block of work captured once from the context's stream and replayed: the same
// kernels with the same arguments as the eager launches it replaces, so results
// are identical.  Buffers must already have their final sizes (an eager block
// runs first).  launches counts the kernels of one replay.
struct BlockGraph {
    cudaGraphExec_t exec = nullptr;
    int64_t launches = 0;
    ~BlockGraph() {
        if (exec) cudaGraphExecDestroy(exec);
    }
};

template <class F>
int capture_block(md_context* ctx, F&& work, BlockGraph& bg) {
    MDB_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const int64_t l0 = ctx->launches;
    const int rc = work();
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    bg.launches = ctx->launches - l0;
    ctx->launches = l0;
    if (rc != MD_OK || e != cudaSuccess || cudaGraphInstantiate(&bg.exec, graph, 0) != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        bg.exec = nullptr;
        cudaGetLastError();  // no graph: the caller launches eagerly
        return rc != MD_OK ? rc : MD_ERR_CUDA;
    }
    cudaGraphDestroy(graph);
    return MD_OK;
}

int replay(md_context* ctx, const BlockGraph& bg) {
    MDB_CUDA(cudaGraphLaunch(bg.exec, ctx->stream));
    ctx->launches += bg.launches;
    return MD_OK;
}

}  // namespace

int constrained_pre_force(md_integrator* it, md_system* sys) {
    MDB_TRY(check_triples(sys, "ConstrainedVelocityVerlet"));
    MDB_TRY(ensure_counters(it));
    md_context* ctx = sys->ctx;
    const int64_t nmol = sys->n / 3;
    NhcState* nhc = it->kind == 4 ? it->chain_state.as<NhcState>() : nullptr;
    if (nhc) {
        MDB_TRY(system_kinetic_async(sys, kResKE));
        MDB_TRY(nhc_pre_async(it, ctx, ctx_result(ctx, kResKE)));
    }
    if (nmol > 0) {
        k_cvv_pre<<<grid_for(nmol, kBlock), kBlock, 0, ctx->stream>>>(
            sys->cur, sys->slot, nmol, cvv_args(it, sys), nhc, it->counters.as<int>(), ctx->d_status);
        ++ctx->launches;
        MDB_CHECK_LAUNCH();
    }
    return status_to_error(ctx);
}

int constrained_post_force(md_integrator* it, md_system* sys, bool apply_scale) {
    MDB_TRY(ensure_counters(it));
    md_context* ctx = sys->ctx;
    const int64_t nmol = sys->n / 3;
    const int g = grid_for(std::max<int64_t>(nmol, 1), kBlock);
    double* part;
    MDB_TRY(ctx_partials(ctx, static_cast<size_t>(g), &part));
    k_cvv_post<<<g, kBlock, 0, ctx->stream>>>(sys->cur, sys->slot, nmol, cvv_args(it, sys),
                                             it->counters.as<int>() + 1, ctx->d_status, part,
                                             ctx_counter(ctx, 8), ctx_result(ctx, kResKE));
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    if (it->kind == 4) {
        MDB_TRY(nhc_post_async(it, ctx, ctx_result(ctx, kResKE)));
        if (apply_scale) MDB_TRY(nhc_apply_scale_async(it, sys));
    }
    if (apply_scale) return status_to_error(ctx);
    return MD_OK;
}

}  // namespace mdb

using namespace mdb;

extern "C" {

int md_rigid_create(double oh, double hoh_degrees, double tolerance, int max_iterations,
                    md_rigid** out) {
    graph_epoch_bump();
    if (!out) return fail(MD_ERR_INVALID_ARGUMENT, "md_rigid_create: NULL");
    // rigid_water.cpp:38-49
    if (!(oh > 0.0)) return fail(MD_ERR_INVALID_ARGUMENT, "RigidWater: ohDistance must be positive");
    if (!(hoh_degrees > 0.0) || !(hoh_degrees < 180.0))
        return fail(MD_ERR_INVALID_ARGUMENT, "RigidWater: hohAngleDegrees must lie in (0, 180)");
    if (!(tolerance > 0.0)) return fail(MD_ERR_INVALID_ARGUMENT, "RigidWater: tolerance must be positive");
    if (max_iterations < 1)
        return fail(MD_ERR_INVALID_ARGUMENT, "RigidWater: maxIterations must be at least 1");
    md_rigid* rw = new (std::nothrow) md_rigid();
    if (!rw) return fail(MD_ERR_OUT_OF_MEMORY, "md_rigid_create: host allocation");
    rw->oh = oh;
    rw->tolerance = tolerance;
    rw->max_iterations = max_iterations;
    const double half_angle = 0.5 * hoh_degrees * kPi / 180.0;  // rigid_water.cpp:51-52
    rw->hh = 2.0 * oh * std::sin(half_angle);
    *out = rw;
    return MD_OK;
}

int md_rigid_set_settle(md_rigid* rw, int on) {
    graph_epoch_bump();
    if (!rw) return fail(MD_ERR_INVALID_ARGUMENT, "md_rigid_set_settle: NULL");
    rw->settle = on != 0;
    return MD_OK;
}

int md_rigid_destroy(md_rigid* rw) {
    graph_epoch_bump();
    delete rw;
    return MD_OK;
}

int md_rigid_distances(const md_rigid* rw, double* oh, double* hh) {
    if (!rw) return fail(MD_ERR_INVALID_ARGUMENT, "md_rigid_distances: NULL");
    if (oh) *oh = rw->oh;
    if (hh) *hh = rw->hh;
    return MD_OK;
}

int64_t md_rigid_degrees_of_freedom(int64_t molecules, int com_removed) {
    // rigid_water.cpp:55-59
    const int64_t total = 6 * molecules;
    return com_removed ? (total >= 3 ? total - 3 : 0) : total;
}

int md_rigid_constrain_positions(md_rigid* rw, md_system* sys, const double* rx,
                                 const double* ry, const double* rz, int* iterations) {
    if (!rw || !sys || !rx || !ry || !rz)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_rigid_constrain_positions: NULL argument");
    MDB_TRY(check_triples(sys, "RigidWater"));
    md_context* ctx = sys->ctx;
    const int64_t n = sys->n, nmol = n / 3;
    DevBuf ref, cnt;
    MDB_TRY(ref.ensure(3 * sizeof(double) * static_cast<size_t>(n > 0 ? n : 1)));
    MDB_TRY(cnt.ensure(sizeof(int)));
    double* d = ref.as<double>();
    MDB_CUDA(cudaMemcpyAsync(d, rx, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    MDB_CUDA(cudaMemcpyAsync(d + n, ry, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    MDB_CUDA(cudaMemcpyAsync(d + 2 * n, rz, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    MDB_CUDA(cudaMemsetAsync(cnt.ptr, 0, sizeof(int), ctx->stream));
    if (nmol > 0) {
        k_shake<<<grid_for(nmol, kBlock), kBlock, 0, ctx->stream>>>(
            sys->cur, sys->slot, nmol, d, d + n, d + 2 * n, rigid_args(*rw), box_of(sys),
            cnt.as<int>(), ctx->d_status);
        ++ctx->launches;
        MDB_CHECK_LAUNCH();
    }
    int it = 0;
    MDB_CUDA(cudaMemcpyAsync(&it, cnt.ptr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    const int rc = status_to_error(ctx);
    ref.release();
    cnt.release();
    if (rc != MD_OK) return rc;
    if (iterations) *iterations = nmol > 0 ? it : 1;
    return MD_OK;
}

int md_rigid_constrain_velocities(md_rigid* rw, md_system* sys, int* iterations) {
    if (!rw || !sys) return fail(MD_ERR_INVALID_ARGUMENT, "md_rigid_constrain_velocities: NULL");
    MDB_TRY(check_triples(sys, "RigidWater"));
    md_context* ctx = sys->ctx;
    const int64_t nmol = sys->n / 3;
    DevBuf cnt;
    MDB_TRY(cnt.ensure(sizeof(int)));
    MDB_CUDA(cudaMemsetAsync(cnt.ptr, 0, sizeof(int), ctx->stream));
    if (nmol > 0) {
        k_rattle<<<grid_for(nmol, kBlock), kBlock, 0, ctx->stream>>>(
            sys->cur, sys->slot, nmol, rigid_args(*rw), box_of(sys), cnt.as<int>(), ctx->d_status);
        ++ctx->launches;
        MDB_CHECK_LAUNCH();
    }
    int it = 0;
    MDB_CUDA(cudaMemcpyAsync(&it, cnt.ptr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    const int rc = status_to_error(ctx);
    cnt.release();
    if (rc != MD_OK) return rc;
    if (iterations) *iterations = nmol > 0 ? it : 1;
    return MD_OK;
}

int md_integrator_create_rattle(double dt, const md_rigid* rw, md_integrator** out) {
    graph_epoch_bump();
    if (!rw || !out) return fail(MD_ERR_INVALID_ARGUMENT, "md_integrator_create_rattle: NULL");
    md_integrator* it = new (std::nothrow) md_integrator();
    if (!it) return fail(MD_ERR_OUT_OF_MEMORY, "md_integrator_create_rattle: host allocation");
    it->kind = 3;
    it->dt = dt;
    it->rigid = *rw;
    *out = it;
    return MD_OK;
}

int md_integrator_create_rattle_nhc(double dt, const md_rigid* rw, double temperature, double tau,
                                    int chain_length, int64_t dof, md_integrator** out) {
    graph_epoch_bump();
    if (!rw || !out) return fail(MD_ERR_INVALID_ARGUMENT, "md_integrator_create_rattle_nhc: NULL");
    MDB_TRY(md_integrator_create_nhc(dt, temperature, tau, chain_length, dof, out));
    (*out)->kind = 4;
    (*out)->rigid = *rw;
    return MD_OK;
}

int md_integrator_iterations(md_integrator* it, int* shake, int* rattle) {
    if (!it) return fail(MD_ERR_INVALID_ARGUMENT, "md_integrator_iterations: NULL");
    int h[2] = {0, 0};
    if (it->counters.ptr) {
        MDB_CUDA(cudaDeviceSynchronize());
        MDB_CUDA(cudaMemcpy(h, it->counters.ptr, 2 * sizeof(int), cudaMemcpyDeviceToHost));
    }
    if (shake) *shake = h[0];
    if (rattle) *rattle = h[1];
    return MD_OK;
}

// Fused device loop of a constrained integrator with SPC/E forces.
int md_run_spce(md_integrator* it, md_system* sys, md_ewald* ff, int64_t steps, double* thermo) {
    if (!it || !sys || !ff) return fail(MD_ERR_INVALID_ARGUMENT, "md_run_spce: NULL argument");
    if (steps < 0) return fail(MD_ERR_INVALID_ARGUMENT, "md_run_spce: steps < 0");
    SpceLoop L;
    MDB_TRY(spce_loop_begin(it, sys, ff, "md_run_spce", L));
    md_context* ctx = sys->ctx;
    DevBuf rows, idx;
    if (thermo && steps > 0) {
        MDB_TRY(rows.ensure(sizeof(double) * 4 * static_cast<size_t>(steps)));
        MDB_TRY(idx.ensure(sizeof(int)));
        MDB_CUDA(cudaMemsetAsync(idx.ptr, 0, sizeof(int), ctx->stream));
    }
    // One step with its thermo row at a device-held index; after the first (eager)
    // step it is captured once and replayed, unless kernel timing is on.
    auto one_step = [&](bool first) -> int {
        MDB_TRY(spce_step_async(L, first, nullptr));
        if (rows.ptr) MDB_TRY(record_at_async(ctx, L.nhc, rows.as<double>(), idx.as<int>()));
        return MD_OK;
    };
    BlockGraph bg;
    const bool want_graph = ctx->graphs && !ctx->timing && steps >= 4;
    for (int64_t k = 0; k < steps; ++k) {
        // a failed capture leaves no graph: the eager launches then report any error
        if (k == 1 && want_graph) capture_block(ctx, [&] { return one_step(false); }, bg);
        if (bg.exec) MDB_TRY(replay(ctx, bg));
        else MDB_TRY(one_step(k == 0));
    }
    if (L.nhc && steps > 0) MDB_TRY(nhc_apply_scale_async(it, sys));
    if (rows.ptr)
        MDB_CUDA(cudaMemcpyAsync(thermo, rows.ptr, sizeof(double) * 4 * static_cast<size_t>(steps),
                                 cudaMemcpyDeviceToHost, ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    rows.release();
    idx.release();
    MDB_TRY(status_to_error(ctx));
    return ctx_check_status(ctx);
}

int md_water_rdf_run(md_integrator* it, md_system* sys, md_ewald* ff, md_rdf* rdf,
                     double temperature, int64_t dof, int64_t equilibrate, int64_t rescale_every,
                     int64_t production, int64_t sample_every, double* mean_temperature) {
    if (!it || !sys || !ff || !rdf)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_water_rdf_run: NULL argument");
    if (it->kind != 3)
        return fail(MD_ERR_INVALID_ARGUMENT,
                    "md_water_rdf_run: needs a ConstrainedVelocityVerlet integrator");
    if (dof < 1 || equilibrate < 0 || production < 0 || rescale_every < 1 || sample_every < 1)
        return fail(MD_ERR_INVALID_ARGUMENT,
                    "md_water_rdf_run: dof, rescale_every, sample_every >= 1; step counts >= 0");
    SpceLoop L;
    MDB_TRY(spce_loop_begin(it, sys, ff, "md_water_rdf_run", L));
    md_context* ctx = sys->ctx;
    DevBuf acc;
    MDB_TRY(acc.ensure(sizeof(double)));
    MDB_CUDA(cudaMemsetAsync(acc.ptr, 0, sizeof(double), ctx->stream));
    // apps/water_rdf.cpp:188-200: every rescale_every steps the velocities are
    // scaled toward the target and put back on the constraint surface (RATTLE's
    // velocity half, rigid_water.cpp:107-162, as constrainVelocities does).
    auto eq_block = [&](int64_t steps, bool first, bool rescale) -> int {
        for (int64_t k = 0; k < steps; ++k) MDB_TRY(spce_step_async(L, first && k == 0, nullptr));
        if (!rescale) return MD_OK;
        MDB_TRY(md_system_rescale_temperature(sys, dof, temperature));
        if (L.nmol > 0) {
            k_rattle<<<grid_for(L.nmol, kBlock), kBlock, 0, ctx->stream>>>(
                sys->cur, sys->slot, L.nmol, rigid_args(it->rigid), box_of(sys),
                it->counters.as<int>() + 1, ctx->d_status);
            ++ctx->launches;
            MDB_CHECK_LAUNCH();
        }
        return MD_OK;
    };
    // apps/water_rdf.cpp:207-216: NVE production; the temperature of every
    // step is summed, and the oxygens (first site of each O, H, H triple) are
    // binned every sample_every steps.
    auto prod_block = [&](int64_t steps, bool first, bool frame) -> int {
        for (int64_t k = 0; k < steps; ++k) {
            MDB_TRY(spce_step_async(L, first && k == 0, nullptr));
            k_sum_temperature<<<1, 1, 0, ctx->stream>>>(ctx_result(ctx, kResKE),
                                                        static_cast<double>(dof), acc.as<double>());
            ++ctx->launches;
        }
        if (frame) MDB_TRY(rdf_frame_launch(rdf, sys, 0, 3));
        return MD_OK;
    };
    // Whole blocks after the first (eager, it sizes every buffer) replay one
    // captured graph each: the same launches in the same order.
    const bool want_graph = ctx->graphs && !ctx->timing;
    const int64_t eq_blocks = equilibrate / rescale_every;
    BlockGraph ge, gp;
    for (int64_t b = 0; b < eq_blocks; ++b) {
        if (b == 1 && want_graph) capture_block(ctx, [&] { return eq_block(rescale_every, false, true); }, ge);
        if (ge.exec) MDB_TRY(replay(ctx, ge));
        else MDB_TRY(eq_block(rescale_every, b == 0, true));
    }
    MDB_TRY(eq_block(equilibrate % rescale_every, eq_blocks == 0, false));
    const int64_t prod_blocks = production / sample_every;
    for (int64_t b = 0; b < prod_blocks; ++b) {
        if (b == 1 && want_graph) capture_block(ctx, [&] { return prod_block(sample_every, false, true); }, gp);
        if (gp.exec) MDB_TRY(replay(ctx, gp));
        else MDB_TRY(prod_block(sample_every, equilibrate == 0 && b == 0, true));
        rdf_frame_note(rdf, sys, 0, 3);
    }
    MDB_TRY(prod_block(production % sample_every, equilibrate == 0 && prod_blocks == 0, false));
    double sum = 0.0;
    MDB_CUDA(cudaMemcpyAsync(&sum, acc.ptr, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    acc.release();
    if (mean_temperature) *mean_temperature = production > 0 ? sum / static_cast<double>(production) : 0.0;
    MDB_TRY(status_to_error(ctx));
    return ctx_check_status(ctx);
}

}  // extern "C"
