// ewald.cu -- Ewald summation and the SPC/E force field (forcefield/ewald.cpp,
// forcefield/spce_forcefield.cpp) on the device.
//
//   real space   erfc(alpha r)/r over intermolecular pairs with r < cutoff, taken
//                from a Verlet list built at cutoff + skin (the reference scans all
//                i<j pairs; the list holds exactly the pairs that can pass r < rc,
//                and membership uses the reference's exact min-image r^2);
//   self         -C alpha/sqrt(pi) sum q^2;
//   intra        -C q_i q_j erf(alpha r)/r over same-molecule pairs (min image),
//                from per-atom partner lists built once from the molecule ids;
//   reciprocal   S(k) = sum_j q_j exp(i k.r_j) over the half space of k vectors
//                (S(-k) = conj S(k), so energy and force sums double), with the
//                per-axis factors exp(i n a x) built by complex recurrence.
// The SPC/E force field adds O-O Lennard-Jones (oxygens = atoms with original
// index divisible by 3, as SpceForceField::gatherOxygens takes them) in the same
// pass over the real-space list.
#include <algorithm>
#include <climits>
#include <cmath>
#include <new>
#include <unordered_map>
#include <vector>

#include "md_device.cuh"
#include "md_internal.cuh"

namespace mdb {
int verlet_build(md_verlet* v, md_system* sys, bool conditional);
int verlet_check(md_verlet* v, md_system* sys);
int verlet_ensure_ready(md_verlet* v, md_system* sys, const char* who);
}  // namespace mdb

namespace mdb {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kBlock = 256;

// ewald.hpp:10-13, ewald.cpp:17-21
double coulomb_prefactor() {
    const double e = 1.602176565e-19, eps0 = 8.854187817e-12, kB = 1.3806488e-23;
    return (e * e) / (4.0 * kPi * eps0) * 1e10 / kB;
}

struct RealArgs {
    double rc2, alpha, coulomb, two_alpha_over_sqrt_pi, neg_alpha2;
    int spce_lj;            // add O-O LJ (SPC/E)
    double sig2, four_eps, tf_eps;
    int lj_lfs;             // O-O LJ with linear force shift at the cutoff
    double rc, uc, dudrc;
};

// The real-space Coulomb (ewald.cpp:60-68) and O-O LJ (lennard_jones.cpp:62-77)
// terms of one pair at r2, in FP32 (MD_PRECISION_MIXED): returns the force
// coefficient s (F = s d) and adds the energies and virials of the pair.
__device__ __forceinline__ float real_pair_mixed(float r2, float cqq, bool coulomb, bool lj,
                                                 const RealArgs& a, float& er, float& wr,
                                                 float& el, float& wl) {
    float s = 0.0f;
    if (coulomb) {
        const float r = sqrtf(r2);
        const float erfc_ar = erfcf(static_cast<float>(a.alpha) * r);
        const float w = cqq * (static_cast<float>(a.two_alpha_over_sqrt_pi) *
                                   expf(static_cast<float>(a.neg_alpha2) * r2) +
                               erfc_ar / r);
        s = w / r2;
        er = cqq * erfc_ar / r;
        wr = w;
    }
    if (lj) {
        const float s2 = static_cast<float>(a.sig2) / r2;
        const float s6 = s2 * s2 * s2;
        float w = static_cast<float>(a.tf_eps) * (2.0f * s6 * s6 - s6);
        float u = static_cast<float>(a.four_eps) * (s6 * s6 - s6);
        if (a.lj_lfs) {
            const float r = sqrtf(r2);
            u = u - static_cast<float>(a.uc) - (r - static_cast<float>(a.rc)) * static_cast<float>(a.dudrc);
            w = w + r * static_cast<float>(a.dudrc);
        }
        s += w / r2;
        el = u;
        wl = w;
    }
    return s;
}

// Real-space (and SPC/E O-O LJ) pair terms over the Verlet list.  out[0..3]:
// E_real, W_real, E_lj, W_lj.  mode 1 writes forces, mode 2 adds to them.
// MIXED: the displacement, the cutoff test and every sum stay FP64; the pair
// terms (erfc, exp, the LJ powers) are evaluated in FP32.
// 128-thread blocks (kRealBlock); the FP64 variant fits six per SM in 78
// registers without spilling, the FP32 one five.
template <int TPA, bool MIXED>
__global__ void __launch_bounds__(128, MIXED ? 5 : 6)
k_ewald_real(const double4* __restrict__ pos, const double* __restrict__ q,
             const int64_t* __restrict__ mol, const int* __restrict__ nbr,
             const int* __restrict__ count, int stride, int64_t n, Box3 box, RealArgs a,
             int mode, double* fxo, double* fyo, double* fzo, double* part, unsigned* ticket,
             double* out) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const int64_t i = t / TPA;
    const int g = static_cast<int>(t % TPA);
    const Fold3 f3 = fold3_of(box);
    double fx = 0.0, fy = 0.0, fz = 0.0, er = 0.0, wr = 0.0, el = 0.0, wl = 0.0;
    if (i < n) {
        const double4 pi = pos[i];
        const double qi = q[i];
        const int64_t mi = mol[i];
        const bool oxy_i = (static_cast<int64_t>(pi.w) % 3) == 0;
        const int cnt = min(count[i], stride);
        const int* row = nbr + i * static_cast<int64_t>(stride);
        // the neighbour's position, charge and molecule are requested together, so
        // one L2 round trip serves the cutoff test and the pair terms
#pragma unroll 2
        for (int k = g; k < cnt; k += TPA) {
            const int j = __ldg(row + k);
            const double4 pj = ldg4(pos + j);
            const double qj = __ldg(q + j);
            const int64_t mj = __ldg(mol + j);
            const bool lo = pi.w < pj.w;
            // r_lower - r_higher by original index, the reference's pair order; the
            // operands are selected rather than branched on, so a warp runs one fold
            double dx, dy, dz;
            min_image_wrapped(f3, lo ? pi.x : pj.x, lo ? pi.y : pj.y, lo ? pi.z : pj.z,
                              lo ? pj.x : pi.x, lo ? pj.y : pi.y, lo ? pj.z : pi.z, dx, dy, dz);
            const double r2 = norm2_exact(dx, dy, dz);
            if (!(r2 < a.rc2)) continue;
            double s = 0.0;
            if (MIXED) {
                const bool coul = mj != mi;
                const bool lj = a.spce_lj && oxy_i && (static_cast<int>(pj.w) % 3) == 0;
                float per = 0.0f, pwr = 0.0f, pel = 0.0f, pwl = 0.0f;
                s = real_pair_mixed(static_cast<float>(r2),
                                    coul ? static_cast<float>(a.coulomb * (qi * qj)) : 0.0f, coul,
                                    lj, a, per, pwr, pel, pwl);
                if (lo) {
                    er += per;
                    wr += pwr;
                    el += pel;
                    wl += pwl;
                }
                const double sg = lo ? s : -s;
                fx = fma(dx, sg, fx);
                fy = fma(dy, sg, fy);
                fz = fma(dz, sg, fz);
                continue;
            }
            if (mol[j] != mi) {
                // ewald.cpp:60-68
                const double r = __dsqrt_rn(r2);
                const double cqq = a.coulomb * (qi * q[j]);
                const double erfc_ar = erfc(a.alpha * r);
                const double w = cqq * (a.two_alpha_over_sqrt_pi * exp(a.neg_alpha2 * r2) + erfc_ar / r);
                s = w / r2;
                if (lo) {
                    er += cqq * erfc_ar / r;
                    wr += w;
                }
            }
            if (a.spce_lj && oxy_i && (static_cast<int>(pj.w) % 3) == 0) {
                // lennard_jones.cpp:62-70 (Truncated)
                const double s2 = a.sig2 / r2;
                const double s6 = s2 * s2 * s2;
                double w = a.tf_eps * (2.0 * s6 * s6 - s6);
                double u = a.four_eps * (s6 * s6 - s6);
                if (a.lj_lfs) {  // lennard_jones.cpp:73-77
                    const double r = sqrt(r2);
                    u = u - a.uc - (r - a.rc) * a.dudrc;
                    w = w + r * a.dudrc;
                }
                s += w / r2;
                if (lo) {
                    el += u;
                    wl += w;
                }
            }
            const double sg = lo ? s : -s;
            fx = fma(dx, sg, fx);
            fy = fma(dy, sg, fy);
            fz = fma(dz, sg, fz);
        }
    }
#pragma unroll
    for (int o = TPA / 2; o > 0; o >>= 1) {
        fx += __shfl_xor_sync(0xffffffffu, fx, o);
        fy += __shfl_xor_sync(0xffffffffu, fy, o);
        fz += __shfl_xor_sync(0xffffffffu, fz, o);
    }
    if (i < n && g == 0) {
        if (mode == 1) {
            fxo[i] = fx;
            fyo[i] = fy;
            fzo[i] = fz;
        } else {
            fxo[i] += fx;
            fyo[i] += fy;
            fzo[i] += fz;
        }
    }
    double v[4] = {er, wr, el, wl};
    grid_reduce<4>(v, part, ticket, out);
}

// Intramolecular correction (ewald.cpp:79-110) per atom over its molecule partners
// (original indices, CSR); adds to forces.  out[0..1]: E_intra, W_intra.
__global__ void k_ewald_intra(const double4* __restrict__ pos, const double* __restrict__ q,
                              const int* __restrict__ orig, const int* __restrict__ slot,
                              const int* __restrict__ off, const int* __restrict__ partner,
                              int64_t n, Box3 box, RealArgs a, int add_forces, double* fxo,
                              double* fyo, double* fzo, double* part, unsigned* ticket,
                              double* out) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const Fold3 f3 = fold3_of(box);
    double e = 0.0, vir = 0.0;
    if (k < n) {
        const double4 pi = pos[k];
        const int oi = orig[k];
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (int p = off[oi]; p < off[oi + 1]; ++p) {
            const int oj = partner[p];
            const int j = slot[oj];
            const double4 pj = pos[j];
            const bool lo = oi < oj;
            double dx, dy, dz;
            if (lo) min_image_wrapped(f3, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z, dx, dy, dz);
            else min_image_wrapped(f3, pj.x, pj.y, pj.z, pi.x, pi.y, pi.z, dx, dy, dz);
            const double r2 = norm2_exact(dx, dy, dz);
            const double r = __dsqrt_rn(r2);
            const double cqq = a.coulomb * (q[k] * q[j]);
            const double erf_ar = erf(a.alpha * r);
            const double w = cqq * (a.two_alpha_over_sqrt_pi * exp(a.neg_alpha2 * r2) - erf_ar / r);
            const double s = lo ? w / r2 : -(w / r2);
            fx = fma(dx, s, fx);
            fy = fma(dy, s, fy);
            fz = fma(dz, s, fz);
            if (lo) {
                e += -cqq * erf_ar / r;
                vir += w;
            }
        }
        if (add_forces) {
            fxo[k] += fx;
            fyo[k] += fy;
            fzo[k] += fz;
        }
    }
    double v[2] = {e, vir};
    grid_reduce<2>(v, part, ticket, out);
}

__global__ void k_sum_q2(const double* __restrict__ q, int64_t n, double* part, unsigned* ticket,
                         double* out) {
    double v[1] = {0.0};
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        v[0] += q[k] * q[k];
    grid_reduce<1>(v, part, ticket, out);
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

struct KArgs {
    const double4* kvec;  // kx, ky, kz, factor
    const int4* kn;       // nx, ny, nz
    int nk, kmax;
    double a, b, c;       // 2 pi / L per axis
};

constexpr int kSiteTile = 32;

// S(k) partial sums: block (kb, sb) handles k vectors [kb*256, +256) against the
// sites of slice sb; per-site factor tables X[nx], Y[ny], Z[nz] of a tile of sites
// are built in shared memory by complex recurrence.
__global__ void __launch_bounds__(kBlock)
k_structure_factor(const double4* __restrict__ pos, const double* __restrict__ q, int64_t n,
                   KArgs ka, int64_t sites_per_slice, double2* part) {
    extern __shared__ double2 tab[];  // kSiteTile * (kmax+1 + 2*(2kmax+1))
    const int nX = ka.kmax + 1, nY = 2 * ka.kmax + 1;
    const int per = nX + 2 * nY;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int4 kn = k < ka.nk ? ka.kn[k] : make_int4(0, 0, 0, 0);
    const int64_t s0 = blockIdx.y * sites_per_slice;
    const int64_t s1 = min(n, s0 + sites_per_slice);
    double re = 0.0, im = 0.0;
    for (int64_t base = s0; base < s1; base += kSiteTile) {
        __syncthreads();
        // build tables: thread t builds site (t % tile), one axis per 3 groups
        for (int w = threadIdx.x; w < 3 * kSiteTile; w += blockDim.x) {
            const int site = w % kSiteTile, axis = w / kSiteTile;
            const int64_t sidx = base + site;
            double2* T = tab + site * per;
            if (sidx < s1) {
                const double4 p = pos[sidx];
                const double coord = axis == 0 ? p.x : (axis == 1 ? p.y : p.z);
                const double kk = axis == 0 ? ka.a : (axis == 1 ? ka.b : ka.c);
                double sn, cs;
                sincos(kk * coord, &sn, &cs);
                const double2 e1 = make_double2(cs, sn);
                if (axis == 0) {
                    double2 x = make_double2(1.0, 0.0);
                    for (int m = 0; m < nX; ++m) {
                        T[m] = x;
                        x = cmul(x, e1);
                    }
                } else {
                    double2* Y = T + nX + (axis - 1) * nY;
                    double2 y = make_double2(1.0, 0.0);
                    for (int m = 0; m <= ka.kmax; ++m) {
                        Y[ka.kmax + m] = y;
                        Y[ka.kmax - m] = make_double2(y.x, -y.y);
                        y = cmul(y, e1);
                    }
                }
            } else {
                for (int m = 0; m < (axis == 0 ? nX : nY); ++m)
                    (axis == 0 ? T : T + nX + (axis - 1) * nY)[m] = make_double2(0.0, 0.0);
            }
        }
        __syncthreads();
        const int lim = static_cast<int>(s1 - base < kSiteTile ? s1 - base : kSiteTile);
        if (k < ka.nk) {
            for (int site = 0; site < lim; ++site) {
                const double2* T = tab + site * per;
                const double2 e = cmul(cmul(T[kn.x], T[nX + ka.kmax + kn.y]),
                                       T[nX + nY + ka.kmax + kn.z]);
                const double qs = q[base + site];
                re = fma(qs, e.x, re);
                im = fma(qs, e.y, im);
            }
        }
    }
    if (k < ka.nk) part[static_cast<int64_t>(blockIdx.y) * ka.nk + k] = make_double2(re, im);
}

// Sums the partials (slice order), stores S(k) and reduces the reciprocal energy
// and virial: E = sum_half 2 factor |S|^2, W = sum_half 2 factor |S|^2 (1 - k^2/(2 a^2)).
__global__ void k_structure_final(const double2* __restrict__ part, int slices, KArgs ka,
                                  double inv_2alpha2, double2* sk, double* rpart,
                                  unsigned* ticket, double* out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (k < ka.nk) {
        double re = 0.0, im = 0.0;
        for (int s = 0; s < slices; ++s) {
            const double2 p = part[static_cast<int64_t>(s) * ka.nk + k];
            re += p.x;
            im += p.y;
        }
        sk[k] = make_double2(re, im);
        const double4 kv = ka.kvec[k];
        const double k2 = kv.x * kv.x + kv.y * kv.y + kv.z * kv.z;
        const double e = 2.0 * kv.w * (re * re + im * im);
        v[0] = e;
        v[1] = e * (1.0 - k2 * inv_2alpha2);
    }
    grid_reduce<2>(v, rpart, ticket, out);
}

// Reciprocal-space forces (ewald.cpp:163-170), one thread per site, k vectors in
// (nx, ny) lines with exp(i nz c z) stepped along each line.
// k-space forces (or, with CHARGE, dE_recip/dq_s = sum over the half space of
// 4 factor Re(conj(S) e^{i k.r_s})) over a 2-D grid: blockIdx.x picks 256 sites,
// blockIdx.y a slice of the (nx, ny) lines of k vectors, so small systems still
// fill the GPU.  Each slice starts its e^{i nx a x}, e^{i ny b y} factors with
// sincos and continues by complex recurrence along its lines; its partial sums go
// to part[slice][site] and k_recip_sum adds the slices in order (deterministic).
template <bool CHARGE>
__global__ void __launch_bounds__(kBlock)
k_recip_force(const double4* __restrict__ pos, const double* __restrict__ q, int64_t n, KArgs ka,
              const int4* __restrict__ lines, int nlines, int lines_per_slice,
              const double2* __restrict__ sk, double4* __restrict__ part) {
    const int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (s >= n) return;
    const int l0 = blockIdx.y * lines_per_slice;
    const int l1 = min(nlines, l0 + lines_per_slice);
    const double4 p = pos[s];
    const double qs = q[s];
    double sn, cs;
    sincos(ka.a * p.x, &sn, &cs);
    const double2 ex = make_double2(cs, sn);
    sincos(ka.b * p.y, &sn, &cs);
    const double2 ey = make_double2(cs, sn);
    sincos(ka.c * p.z, &sn, &cs);
    const double2 ez = make_double2(cs, sn);
    double fx = 0.0, fy = 0.0, fz = 0.0;
    double2 X = make_double2(1.0, 0.0), Y = make_double2(1.0, 0.0);
    int cur_nx = INT_MIN, cur_ny = INT_MIN;
    for (int l = l0; l < l1; ++l) {
        const int4 L = lines[l];  // nx, ny, nz0, first k index; count in next line's .w
        if (L.x != cur_nx) {
            if (cur_nx != INT_MIN && L.x == cur_nx + 1) {
                X = cmul(X, ex);
            } else {
                sincos(static_cast<double>(L.x) * ka.a * p.x, &sn, &cs);
                X = make_double2(cs, sn);
            }
            cur_nx = L.x;
            cur_ny = INT_MIN;
        }
        if (L.y != cur_ny) {
            if (cur_ny != INT_MIN && L.y == cur_ny + 1) {
                Y = cmul(Y, ey);
            } else {
                sincos(static_cast<double>(L.y) * ka.b * p.y, &sn, &cs);
                Y = make_double2(cs, sn);
            }
            cur_ny = L.y;
        }
        const double2 XY = cmul(X, Y);
        sincos(static_cast<double>(L.z) * ka.c * p.z, &sn, &cs);
        double2 Z = make_double2(cs, sn);
        const int k0 = L.w, k1 = (l + 1 < nlines) ? lines[l + 1].w : ka.nk;
        for (int k = k0; k < k1; ++k) {
            const double2 e = cmul(XY, Z);
            const double4 kv = ka.kvec[k];
            const double2 S = sk[k];
            if (CHARGE) {
                fx += 4.0 * kv.w * (S.x * e.x + S.y * e.y);
            } else {
                // 2 (half space) * factor * 2 * q * (Re S sin - Im S cos)
                const double coeff = 4.0 * kv.w * qs * (S.x * e.y - S.y * e.x);
                fx = fma(coeff, kv.x, fx);
                fy = fma(coeff, kv.y, fy);
                fz = fma(coeff, kv.z, fz);
            }
            Z = cmul(Z, ez);
        }
    }
    part[blockIdx.y * n + s] = make_double4(fx, fy, fz, 0.0);
}

// Adds the slices' partial k-space forces (CHARGE: charge gradients), one warp
// per site: lane l sums slices l, l + 32, ... in order, then the lanes combine
// by a fixed butterfly, so the result does not depend on scheduling.
template <bool CHARGE>
__global__ void k_recip_sum(const double4* __restrict__ part, int slices, int64_t n, double* fxo,
                            double* fyo, double* fzo, double* dq) {
    const int64_t s = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (s >= n) return;  // whole warps leave together
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int k = lane; k < slices; k += 32) {
        const double4 v = part[k * n + s];
        fx += v.x;
        fy += v.y;
        fz += v.z;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        fx += __shfl_xor_sync(0xffffffffu, fx, o);
        fy += __shfl_xor_sync(0xffffffffu, fy, o);
        fz += __shfl_xor_sync(0xffffffffu, fz, o);
    }
    if (lane != 0) return;
    if (CHARGE) {
        dq[s] += fx;
    } else {
        fxo[s] += fx;
        fyo[s] += fy;
        fzo[s] += fz;
    }
}

// Grid of the k-space force pass: enough line slices to give every SM a few
// blocks (one slice for large systems).
int recip_slices(const md_context* ctx, int64_t n, int nlines) {
    const int64_t site_blocks = (n + kBlock - 1) / kBlock;
    int64_t slices = (4 * static_cast<int64_t>(ctx->sm_count) + site_blocks - 1) / site_blocks;
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(slices, nlines)));
}

__global__ void k_to_slot4(const int* __restrict__ slot, int64_t n, const double4* in, double4* out) {
    const int64_t o = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (o < n) out[slot[o]] = in[o];
}

__global__ void k_to_orig4(const int* __restrict__ orig, int64_t n, const double4* in, double4* out) {
    const int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (s < n) out[orig[s]] = in[s];
}

__global__ void k_to_orig1(const int* __restrict__ orig, int64_t n, const double* in, double* out) {
    const int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (s < n) out[orig[s]] = in[s];
}

// Charge gradient of the real-space and intramolecular terms, plus the self
// term, per atom (device order):
//   dE/dq_i = sum_j C q_j erfc(a r)/r (other molecules, r < rc)
//           - sum_j C q_j erf(a r)/r (same molecule) - 2 C a/sqrt(pi) q_i
__global__ void __launch_bounds__(kBlock)
k_ewald_dq(const double4* __restrict__ pos, const double* __restrict__ q,
           const int64_t* __restrict__ mol, const int* __restrict__ nbr,
           const int* __restrict__ count, int stride, const int* __restrict__ orig,
           const int* __restrict__ slot, const int* __restrict__ off,
           const int* __restrict__ partner, int64_t n, Box3 box, RealArgs a, double* dq) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const Fold3 f3 = fold3_of(box);
    const double4 pi = pos[i];
    const int64_t mi = mol[i];
    double acc = 0.0;
    const int cnt = min(count[i], stride);
    const int* row = nbr + i * static_cast<int64_t>(stride);
    for (int k = 0; k < cnt; ++k) {
        const int j = __ldg(row + k);
        if (mol[j] == mi) continue;
        const double4 pj = ldg4(pos + j);
        double dx, dy, dz;
        min_image_wrapped(f3, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z, dx, dy, dz);
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (!(r2 < a.rc2)) continue;
        const double r = sqrt(r2);
        acc += a.coulomb * q[j] * erfc(a.alpha * r) / r;
    }
    const int oi = orig[i];
    for (int p = off[oi]; p < off[oi + 1]; ++p) {
        const int j = slot[partner[p]];
        const double4 pj = pos[j];
        double dx, dy, dz;
        min_image_wrapped(f3, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z, dx, dy, dz);
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        acc -= a.coulomb * q[j] * erf(a.alpha * r) / r;
    }
    acc -= a.coulomb * a.two_alpha_over_sqrt_pi * q[i];  // 2 C a / sqrt(pi) q_i
    dq[i] = acc;
}

// Hessian-vector product of the real-space Coulomb forces (other molecules,
// r < rc): out_i = sum_j [g (u_i - u_j) + 2 g' d (d . (u_i - u_j))] with
// F_i = sum_j g(r^2) d, g = C q_i q_j (A e^{-a^2 r^2}/r^2 + erfc(a r)/r^3), A = 2a/sqrt(pi).
__global__ void __launch_bounds__(kBlock)
k_ewald_real_hvp(const double4* __restrict__ pos, const double* __restrict__ q,
                 const int64_t* __restrict__ mol, const int* __restrict__ nbr,
                 const int* __restrict__ count, int stride, int64_t n, Box3 box, RealArgs a,
                 const double4* __restrict__ u, double4* out) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const Fold3 f3 = fold3_of(box);
    const double4 pi = pos[i], ui = u[i];
    const int64_t mi = mol[i];
    const double qi = q[i];
    const double a3 = a.alpha * a.alpha * a.two_alpha_over_sqrt_pi;  // 2 a^3 / sqrt(pi)
    const double a1 = 1.5 * a.two_alpha_over_sqrt_pi;                 // 3 a / sqrt(pi)
    double hx = 0.0, hy = 0.0, hz = 0.0;
    const int cnt = min(count[i], stride);
    const int* row = nbr + i * static_cast<int64_t>(stride);
    for (int k = 0; k < cnt; ++k) {
        const int j = __ldg(row + k);
        if (mol[j] == mi) continue;
        const double4 pj = ldg4(pos + j);
        double dx, dy, dz;
        min_image_wrapped(f3, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z, dx, dy, dz);
        const double s = dx * dx + dy * dy + dz * dz;
        if (!(s < a.rc2)) continue;
        const double r = sqrt(s);
        const double cqq = a.coulomb * qi * q[j];
        const double ex = exp(a.neg_alpha2 * s), ec = erfc(a.alpha * r);
        const double g = cqq * (a.two_alpha_over_sqrt_pi * ex / s + ec / (s * r));
        const double gs = -cqq * (a3 * ex / s + a1 * ex / (s * s) + 1.5 * ec / (s * s * r));
        const double4 uj = u[j];
        const double ux = ui.x - uj.x, uy = ui.y - uj.y, uz = ui.z - uj.z;
        const double dm = dx * ux + dy * uy + dz * uz;
        hx += g * ux + 2.0 * gs * dx * dm;
        hy += g * uy + 2.0 * gs * dy * dm;
        hz += g * uz + 2.0 * gs * dz * dm;
    }
    out[i] = make_double4(hx, hy, hz, 0.0);
}

// Threads per atom of the real-space pass: the fewest (at least 4) that put
// about a thousand threads on every SM, so that a few thousand sites still
// spread over the whole GPU instead of a dozen SMs; at most a warp.
int real_tpa(const md_context* ctx, int64_t n) {
    const int64_t want = 1024 * static_cast<int64_t>(ctx->sm_count);
    int tpa = 4;
    while (tpa < 32 && n * tpa < want) tpa *= 2;
    return tpa;
}

// 128-thread blocks: six (FP64) or five (FP32 pair terms) fit on an SM, 24 or 20
// warps, where two 256-thread blocks at ~96 registers would give 16.
constexpr int kRealBlock = 128;

template <int TPA, bool MIXED>
void launch_real_t(md_system* sys, md_verlet* v, const RealArgs& a, int mode, double* fx,
                   double* fy, double* fz, double* part, unsigned* ticket, double* out) {
    const int64_t threads = std::max<int64_t>(sys->n * TPA, 1);
    k_ewald_real<TPA, MIXED><<<grid_for(threads, kRealBlock), kRealBlock, 0, sys->ctx->stream>>>(
        sys->cur.pos, sys->cur.charge, sys->cur.mol, v->nbr.as<int>(), v->count.as<int>(),
        v->stride, sys->n, Box3{{sys->box[0], sys->box[1], sys->box[2]},
                                {sys->inv_box[0], sys->inv_box[1], sys->inv_box[2]}},
        a, mode, fx, fy, fz, part, ticket, out);
}

// mode 1 writes (fx, fy, fz), 2 adds to them; part holds 4 doubles per block.
template <bool MIXED>
void launch_real_p(md_system* sys, md_verlet* v, const RealArgs& a, int mode, int tpa, double* fx,
                   double* fy, double* fz, double* part, unsigned* ticket, double* out) {
    switch (tpa) {
        case 32: launch_real_t<32, MIXED>(sys, v, a, mode, fx, fy, fz, part, ticket, out); break;
        case 16: launch_real_t<16, MIXED>(sys, v, a, mode, fx, fy, fz, part, ticket, out); break;
        case 8: launch_real_t<8, MIXED>(sys, v, a, mode, fx, fy, fz, part, ticket, out); break;
        default: launch_real_t<4, MIXED>(sys, v, a, mode, fx, fy, fz, part, ticket, out); break;
    }
}

void launch_real(md_system* sys, md_verlet* v, const RealArgs& a, int mode, int tpa, bool mixed,
                 double* fx, double* fy, double* fz, double* part, unsigned* ticket, double* out) {
    if (mixed) launch_real_p<true>(sys, v, a, mode, tpa, fx, fy, fz, part, ticket, out);
    else launch_real_p<false>(sys, v, a, mode, tpa, fx, fy, fz, part, ticket, out);
}

}  // namespace

}  // namespace mdb

// Result slots inside kResEwald (doubles).
enum {
    kEwReal = 0, kEwRealW, kEwLj, kEwLjW, kEwIntra, kEwIntraW, kEwRecip, kEwRecipW, kEwQ2,
    kEwCount
};

struct md_ewald {
    md_context* ctx = nullptr;
    double cutoff = 10.0;
    int kmax = 5;
    double alpha_in = 0.0;
    double skin = 1.0;
    bool spce = false;
    double sigma_o = 0, epsilon_o = 0;
    int lj_truncation = MD_TRUNCATED;
    md_verlet* list = nullptr;
    double list_box[3] = {0, 0, 0};
    // topology (per original index)
    md_system* topo_sys = nullptr;
    uint64_t topo_version = 0;
    int64_t topo_n = -1;
    mdb::DevBuf partner_off, partner_idx;
    int64_t npartners = 0;
    // k vectors
    double kbox[3] = {0, 0, 0};
    int k_kmax = -1;
    double k_alpha = 0.0;
    mdb::DevBuf kvec, kn, lines, sk, skpart;
    mdb::DevBuf rpart;            // per line slice k-space force partials
    int nk = 0, nlines = 0;
    double last[kEwCount] = {0};
    double alpha = 0.0;
    mdb::PmeState* pme = nullptr;  // reciprocal term by smooth PME instead of k-vector sums
    bool mixed = false;            // FP32 real-space pair terms (MD_PRECISION_MIXED)
};

namespace mdb {

namespace {

int ewald_topology(md_ewald* ew, md_system* sys) {
    if (ew->topo_sys == sys && ew->topo_version == sys->mol_version && ew->topo_n == sys->n)
        return MD_OK;
    const int64_t n = sys->n;
    std::vector<int64_t> mol(static_cast<size_t>(n));
    if (n > 0) MDB_TRY(md_system_get_molecule_ids(sys, mol.data()));
    // group atoms by molecule (index order within each molecule)
    std::unordered_map<int64_t, std::vector<int>> groups;
    groups.reserve(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) groups[mol[i]].push_back(static_cast<int>(i));
    std::vector<int> off(static_cast<size_t>(n + 1), 0), idx;
    for (int64_t i = 0; i < n; ++i) off[i + 1] = static_cast<int>(groups[mol[i]].size()) - 1;
    for (int64_t i = 0; i < n; ++i) off[i + 1] += off[i];
    idx.resize(static_cast<size_t>(off[n]));
    for (int64_t i = 0; i < n; ++i) {
        int at = off[i];
        for (int j : groups[mol[i]])
            if (j != i) idx[at++] = j;
    }
    MDB_TRY(ew->partner_off.ensure(sizeof(int) * (n + 1)));
    MDB_TRY(ew->partner_idx.ensure(sizeof(int) * std::max<size_t>(idx.size(), 1)));
    MDB_CUDA(cudaMemcpy(ew->partner_off.ptr, off.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    if (!idx.empty())
        MDB_CUDA(cudaMemcpy(ew->partner_idx.ptr, idx.data(), sizeof(int) * idx.size(),
                            cudaMemcpyHostToDevice));
    ew->npartners = static_cast<int64_t>(idx.size());
    ew->topo_sys = sys;
    ew->topo_version = sys->mol_version;
    ew->topo_n = n;
    return MD_OK;
}

// k vectors of the half space, grouped in (nx, ny) lines (ewald.cpp:112-172): the
// full set n in [-kmax,kmax]^3, 0 < |n|^2 < kmax^2 + 2, is {k} u {-k} of these.
int ewald_kvectors(md_ewald* ew, const double box[3], double alpha) {
    if (ew->k_kmax == ew->kmax && ew->k_alpha == alpha && ew->kbox[0] == box[0] &&
        ew->kbox[1] == box[1] && ew->kbox[2] == box[2])
        return MD_OK;
    const int kmax = ew->kmax;
    const double volume = box[0] * box[1] * box[2];
    const double kx0 = 2.0 * kPi / box[0], ky0 = 2.0 * kPi / box[1], kz0 = 2.0 * kPi / box[2];
    const int n2max = kmax * kmax + 2;
    const double coulomb = coulomb_prefactor();
    std::vector<double4> kv;
    std::vector<int4> kn, lines;
    for (int nx = 0; nx <= kmax; ++nx) {
        for (int ny = -kmax; ny <= kmax; ++ny) {
            if (nx == 0 && ny < 0) continue;
            int first = -1;
            for (int nz = -kmax; nz <= kmax; ++nz) {
                if (nx == 0 && ny == 0 && nz <= 0) continue;
                const int n2 = nx * nx + ny * ny + nz * nz;
                if (n2 == 0 || n2 >= n2max) continue;
                if (first < 0) first = nz;
                const double kxv = kx0 * static_cast<double>(nx);
                const double kyv = ky0 * static_cast<double>(ny);
                const double kzv = kz0 * static_cast<double>(nz);
                const double k2 = kxv * kxv + kyv * kyv + kzv * kzv;
                const double factor =
                    coulomb * (2.0 * kPi / volume) * std::exp(-k2 / (4.0 * alpha * alpha)) / k2;
                if (first == nz) lines.push_back(make_int4(nx, ny, nz, static_cast<int>(kv.size())));
                kv.push_back(make_double4(kxv, kyv, kzv, factor));
                kn.push_back(make_int4(nx, ny, nz, 0));
            }
        }
    }
    ew->nk = static_cast<int>(kv.size());
    ew->nlines = static_cast<int>(lines.size());
    const size_t nk = std::max<size_t>(kv.size(), 1);
    MDB_TRY(ew->kvec.ensure(sizeof(double4) * nk));
    MDB_TRY(ew->kn.ensure(sizeof(int4) * nk));
    MDB_TRY(ew->lines.ensure(sizeof(int4) * std::max<size_t>(lines.size(), 1)));
    MDB_TRY(ew->sk.ensure(sizeof(double2) * nk));
    if (!kv.empty()) {
        MDB_CUDA(cudaMemcpy(ew->kvec.ptr, kv.data(), sizeof(double4) * kv.size(), cudaMemcpyHostToDevice));
        MDB_CUDA(cudaMemcpy(ew->kn.ptr, kn.data(), sizeof(int4) * kn.size(), cudaMemcpyHostToDevice));
        MDB_CUDA(cudaMemcpy(ew->lines.ptr, lines.data(), sizeof(int4) * lines.size(),
                            cudaMemcpyHostToDevice));
    }
    ew->k_kmax = kmax;
    ew->k_alpha = alpha;
    for (int d = 0; d < 3; ++d) ew->kbox[d] = box[d];
    return MD_OK;
}

int ewald_list_gated(md_ewald* ew, md_system* sys) {
    MDB_TRY(verlet_check(ew->list, sys));
    return verlet_build(ew->list, sys, true);
}

int ewald_list(md_ewald* ew, md_system* sys) {
    if (ew->list && (ew->list_box[0] != sys->box[0] || ew->list_box[1] != sys->box[1] ||
                     ew->list_box[2] != sys->box[2])) {
        md_verlet_destroy(ew->list);
        ew->list = nullptr;
    }
    if (!ew->list) {
        MDB_TRY(md_verlet_create(ew->ctx, sys->box, ew->cutoff, ew->skin, &ew->list));
        for (int d = 0; d < 3; ++d) ew->list_box[d] = sys->box[d];
    }
    md_verlet* v = ew->list;
    if (!v->sys || v->sys != sys || v->n != sys->n || v->epoch != sys->epoch) {
        MDB_TRY(verlet_build(v, sys, false));
        return MD_OK;
    }
    int f = 0;
    MDB_TRY(md_verlet_needs_rebuild(v, sys, &f));
    if (f) MDB_TRY(verlet_build(v, sys, false));
    return MD_OK;
}

}  // namespace

// Everything of one evaluation, asynchronously; results land in kResEwald slots.
// mode: 0 energies only, 1 zero + accumulate forces, 2 accumulate onto forces.
// gated: the neighbour list is maintained by device-decided rebuilds (no host
// synchronisation; the list must already be built for this system).
// k-space forces added to the system's forces (charge = false), or
// dE_recip/dq added to dq (device order); S(k) must be current.
int recip_force_async(md_ewald* ew, md_system* sys, const KArgs& ka, bool charge, double* dq) {
    md_context* ctx = sys->ctx;
    const int64_t n = sys->n;
    if (n == 0 || ew->nk == 0) return MD_OK;
    const int slices = recip_slices(ctx, n, ew->nlines);
    const int per = (ew->nlines + slices - 1) / slices;
    MDB_TRY(ew->rpart.ensure(sizeof(double4) * static_cast<size_t>(slices) * n));
    const dim3 grid(static_cast<unsigned>((n + kBlock - 1) / kBlock), static_cast<unsigned>(slices));
    double4* part = ew->rpart.as<double4>();
    if (charge) {
        k_recip_force<true><<<grid, kBlock, 0, ctx->stream>>>(
            sys->cur.pos, sys->cur.charge, n, ka, ew->lines.as<int4>(), ew->nlines, per,
            ew->sk.as<double2>(), part);
        k_recip_sum<true><<<grid_for(32 * n, kBlock), kBlock, 0, ctx->stream>>>(
            part, slices, n, nullptr, nullptr, nullptr, dq);
    } else {
        k_recip_force<false><<<grid, kBlock, 0, ctx->stream>>>(
            sys->cur.pos, sys->cur.charge, n, ka, ew->lines.as<int4>(), ew->nlines, per,
            ew->sk.as<double2>(), part);
        k_recip_sum<false><<<grid_for(32 * n, kBlock), kBlock, 0, ctx->stream>>>(
            part, slices, n, sys->cur.fx, sys->cur.fy, sys->cur.fz, nullptr);
    }
    ctx->launches += 2;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

RealArgs real_args_of(const md_ewald* ew, double alpha) {
    RealArgs a;
    a.rc2 = ew->cutoff * ew->cutoff;
    a.alpha = alpha;
    a.coulomb = coulomb_prefactor();
    a.two_alpha_over_sqrt_pi = 2.0 * alpha / std::sqrt(kPi);
    a.neg_alpha2 = -alpha * alpha;
    a.spce_lj = ew->spce ? 1 : 0;
    a.sig2 = ew->sigma_o * ew->sigma_o;
    a.four_eps = 4.0 * ew->epsilon_o;
    a.tf_eps = 24.0 * ew->epsilon_o;
    a.lj_lfs = ew->lj_truncation == MD_LINEAR_FORCE_SHIFT ? 1 : 0;
    a.rc = ew->cutoff;
    // lennard_jones.cpp:32-48
    const double s2 = a.sig2 / a.rc2, s6 = s2 * s2 * s2;
    a.uc = 4.0 * ew->epsilon_o * (s6 * s6 - s6);
    a.dudrc = -(24.0 * ew->epsilon_o * (2.0 * s6 * s6 - s6)) / ew->cutoff;
    return a;
}

KArgs kargs_of(md_ewald* ew, const md_system* sys) {
    KArgs ka;
    ka.kvec = ew->kvec.as<double4>();
    ka.kn = ew->kn.as<int4>();
    ka.nk = ew->nk;
    ka.kmax = ew->kmax;
    ka.a = 2.0 * kPi / sys->box[0];
    ka.b = 2.0 * kPi / sys->box[1];
    ka.c = 2.0 * kPi / sys->box[2];
    return ka;
}

int ewald_eval_async(md_ewald* ew, md_system* sys, int mode, bool gated) {
    md_context* ctx = sys->ctx;
    const int64_t n = sys->n;
    double min_len = std::min(sys->box[0], std::min(sys->box[1], sys->box[2]));
    const double alpha = ew->alpha_in > 0.0 ? ew->alpha_in : 5.6 / min_len;  // ewald.cpp:40
    ew->alpha = alpha;
    if (gated) {
        MDB_TRY(ewald_list_gated(ew, sys));
    } else {
        MDB_TRY(ewald_topology(ew, sys));
        if (!ew->pme) MDB_TRY(ewald_kvectors(ew, sys->box, alpha));
        MDB_TRY(ewald_list(ew, sys));
    }
    md_verlet* v = ew->list;
    const RealArgs a = real_args_of(ew, alpha);
    double* res = ctx_result(ctx, kResEwald);
    const Box3 box{{sys->box[0], sys->box[1], sys->box[2]},
                   {sys->inv_box[0], sys->inv_box[1], sys->inv_box[2]}};
    double* part;
    const int tpa = real_tpa(ctx, n);
    const int64_t real_threads = std::max<int64_t>(n * tpa, 1);
    MDB_TRY(ctx_partials(ctx, 4 * static_cast<size_t>(grid_for(real_threads, kRealBlock)), &part));
    // real space (+ O-O LJ): with forces it writes (mode 1) or adds (mode 2); for
    // energies only it writes into the scratch force sink of a zero-force pass.
    ctx_time_begin(ctx, MD_KERNEL_EWALD_REAL);
    if (mode == 0) {
        // energies only: run the pair pass without touching forces by pointing the
        // sink at scratch (never read back)
        double* sink;
        MDB_TRY(ctx_scratch(ctx, 3 * sizeof(double) * static_cast<size_t>(std::max<int64_t>(n, 1)),
                            reinterpret_cast<void**>(&sink)));
        launch_real(sys, v, a, 1, tpa, ew->mixed, sink, sink + n, sink + 2 * n, part,
                    ctx_counter(ctx, 4), res + kEwReal);
    } else {
        launch_real(sys, v, a, mode, tpa, ew->mixed, sys->cur.fx, sys->cur.fy, sys->cur.fz,
                    part, ctx_counter(ctx, 4), res + kEwReal);
    }
    ctx_time_end(ctx, MD_KERNEL_EWALD_REAL);
    // intramolecular correction
    if (n > 0) {
        k_ewald_intra<<<grid_for(n, kBlock), kBlock, 0, ctx->stream>>>(
            sys->cur.pos, sys->cur.charge, sys->cur.orig, sys->slot, ew->partner_off.as<int>(),
            ew->partner_idx.as<int>(), n, box, a, mode != 0 ? 1 : 0, sys->cur.fx, sys->cur.fy,
            sys->cur.fz, part, ctx_counter(ctx, 5), res + kEwIntra);
        const int g = std::min<int>(grid_for(n, kBlock), ctx->sm_count * 4);
        k_sum_q2<<<g, kBlock, 0, ctx->stream>>>(sys->cur.charge, n, part, ctx_counter(ctx, 6),
                                                res + kEwQ2);
    }
    // reciprocal space
    ctx_time_begin(ctx, MD_KERNEL_EWALD_RECIP);
    const KArgs ka = kargs_of(ew, sys);
    if (ew->pme) {
        MDB_TRY(pme_eval_async(ew->pme, sys, alpha, coulomb_prefactor(), mode, res + kEwRecip,
                               ctx_counter(ctx, 12)));
    } else if (ew->nk > 0 && n > 0) {
        const int kblocks = (ew->nk + kBlock - 1) / kBlock;
        // enough site slices to give every SM a few blocks
        int64_t slices = std::max<int64_t>(1, (4 * ctx->sm_count) / kblocks);
        slices = std::min<int64_t>(slices, (n + kSiteTile - 1) / kSiteTile);
        const int64_t per = ((n + slices - 1) / slices + kSiteTile - 1) / kSiteTile * kSiteTile;
        slices = (n + per - 1) / per;
        MDB_TRY(ew->skpart.ensure(sizeof(double2) * static_cast<size_t>(slices) * ew->nk));
        const size_t smem =
            sizeof(double2) * kSiteTile * static_cast<size_t>((ew->kmax + 1) + 2 * (2 * ew->kmax + 1));
        if (smem > 48 * 1024)
            MDB_CUDA(cudaFuncSetAttribute(k_structure_factor,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(smem)));
        k_structure_factor<<<dim3(kblocks, static_cast<unsigned>(slices)), kBlock, smem, ctx->stream>>>(
            sys->cur.pos, sys->cur.charge, n, ka, per, ew->skpart.as<double2>());
        double* rp;
        MDB_TRY(ctx_partials(ctx, 2 * static_cast<size_t>(kblocks), &rp));
        k_structure_final<<<kblocks, kBlock, 0, ctx->stream>>>(
            ew->skpart.as<double2>(), static_cast<int>(slices), ka, 1.0 / (2.0 * alpha * alpha),
            ew->sk.as<double2>(), rp, ctx_counter(ctx, 7), res + kEwRecip);
        if (mode != 0) MDB_TRY(recip_force_async(ew, sys, ka, false, nullptr));
    } else {
        MDB_CUDA(cudaMemsetAsync(res + kEwRecip, 0, 2 * sizeof(double), ctx->stream));
    }
    ctx_time_end(ctx, MD_KERNEL_EWALD_RECIP);
    MDB_CHECK_LAUNCH();
    ctx->launches += 6;
    return MD_OK;
}

int ewald_read(md_ewald* ew, md_context* ctx) {
    MDB_TRY(ctx_read_results(ctx, kResEwald, kEwCount, ew->last));
    return MD_OK;
}

}  // namespace mdb

using namespace mdb;

namespace {

int ewald_new(md_context* ctx, double cutoff, int kmax, double alpha, md_ewald** out) {
    if (!ctx || !out) return fail(MD_ERR_INVALID_ARGUMENT, "md_ewald_create: NULL argument");
    if (!(cutoff > 0.0) || kmax < 0)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_ewald_create: cutoff must be > 0 and kmax >= 0");
    md_ewald* ew = new (std::nothrow) md_ewald();
    if (!ew) return fail(MD_ERR_OUT_OF_MEMORY, "md_ewald_create: host allocation");
    ew->ctx = ctx;
    ew->cutoff = cutoff;
    ew->kmax = kmax;
    ew->alpha_in = alpha;
    *out = ew;
    return MD_OK;
}

void fill_terms(const md_ewald* ew, double terms[4], double* virial) {
    const double coulomb = coulomb_prefactor();
    // ewald.cpp:76: -C alpha / sqrt(pi) * sum q^2
    const double self = -coulomb * ew->alpha / std::sqrt(kPi) * ew->last[kEwQ2];
    if (terms) {
        terms[0] = ew->last[kEwReal];
        terms[1] = ew->last[kEwRecip];
        terms[2] = self;
        terms[3] = ew->last[kEwIntra];
    }
    if (virial) *virial = ew->last[kEwRealW] + ew->last[kEwIntraW] + ew->last[kEwRecipW];
}

}  // namespace

extern "C" {

double md_coulomb_prefactor(void) { return coulomb_prefactor(); }

int md_ewald_create(md_context* ctx, double cutoff, int kmax, double alpha, md_ewald** out) {
    graph_epoch_bump();
    return ewald_new(ctx, cutoff, kmax, alpha, out);
}

int md_ewald_destroy(md_ewald* ew) {
    graph_epoch_bump();
    if (!ew) return MD_OK;
    if (ew->list) md_verlet_destroy(ew->list);
    if (ew->pme) {
        cudaStreamSynchronize(ew->ctx->stream);
        pme_destroy(ew->pme);
    }
    ew->partner_off.release();
    ew->partner_idx.release();
    ew->kvec.release();
    ew->kn.release();
    ew->lines.release();
    ew->rpart.release();
    ew->sk.release();
    ew->skpart.release();
    delete ew;
    return MD_OK;
}

int md_ewald_set_skin(md_ewald* ew, double skin) {
    graph_epoch_bump();
    if (!ew || !(skin >= 0.0)) return fail(MD_ERR_INVALID_ARGUMENT, "md_ewald_set_skin: bad argument");
    ew->skin = skin;
    if (ew->list) {
        md_verlet_destroy(ew->list);
        ew->list = nullptr;
    }
    return MD_OK;
}

int md_ewald_compute(md_ewald* ew, md_system* sys, int mode, double terms[4], double* virial) {
    if (!ew || !sys) return fail(MD_ERR_INVALID_ARGUMENT, "md_ewald_compute: NULL argument");
    if (mode < 0 || mode > 2) return fail(MD_ERR_INVALID_ARGUMENT, "md_ewald_compute: mode %d", mode);
    if (sys->ctx != ew->ctx) return fail(MD_ERR_INVALID_ARGUMENT, "md_ewald_compute: context mismatch");
    MDB_TRY(ewald_eval_async(ew, sys, mode, false));
    MDB_TRY(ewald_read(ew, sys->ctx));
    fill_terms(ew, terms, virial);
    return MD_OK;
}

namespace {

// per-atom vectors between the caller's order (n x 3 host) and device double4
int upload_vec(md_system* sys, const double* u, double4* dev_orig, double4* dev) {
    const int64_t n = sys->n;
    std::vector<double4> h(static_cast<size_t>(n));
    for (int64_t o = 0; o < n; ++o) h[o] = make_double4(u[3 * o], u[3 * o + 1], u[3 * o + 2], 0.0);
    MDB_CUDA(cudaMemcpyAsync(dev_orig, h.data(), sizeof(double4) * n, cudaMemcpyHostToDevice,
                             sys->ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(sys->ctx->stream));
    k_to_slot4<<<grid_for(n, kBlock), kBlock, 0, sys->ctx->stream>>>(sys->slot, n, dev_orig, dev);
    return MD_OK;
}

}  // namespace

int md_ewald_set_pme(md_ewald* ew, int kx, int ky, int kz, int order) {
    graph_epoch_bump();
    if (!ew) return fail(MD_ERR_INVALID_ARGUMENT, "md_ewald_set_pme: NULL");
    if (kx == 0 && ky == 0 && kz == 0) {  // back to the k-vector sums
        if (ew->pme) {
            cudaStreamSynchronize(ew->ctx->stream);
            pme_destroy(ew->pme);
            ew->pme = nullptr;
        }
        return MD_OK;
    }
    if (order != 4 && order != 6 && order != 8)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_ewald_set_pme: order must be 4, 6 or 8");
    const int K[3] = {kx, ky, kz};
    for (int d = 0; d < 3; ++d)
        if (K[d] < 2 * order || K[d] > 4096)
            return fail(MD_ERR_INVALID_ARGUMENT,
                        "md_ewald_set_pme: grid sizes must lie in [2 * order, 4096]");
    mdb::PmeState* s = nullptr;
    MDB_TRY(pme_create(ew->ctx, K, order, &s));
    if (ew->pme) {
        cudaStreamSynchronize(ew->ctx->stream);
        pme_destroy(ew->pme);
    }
    ew->pme = s;
    return MD_OK;
}

int md_ewald_set_precision(md_ewald* ew, int precision) {
    graph_epoch_bump();
    if (!ew || (precision != MD_PRECISION_FP64 && precision != MD_PRECISION_MIXED))
        return fail(MD_ERR_INVALID_ARGUMENT, "md_ewald_set_precision: MD_PRECISION_FP64 or _MIXED");
    ew->mixed = precision == MD_PRECISION_MIXED;
    return MD_OK;
}

int md_ewald_pme_grid(const md_ewald* ew, int k[3], int* order) {
    if (!ew || !k || !order) return fail(MD_ERR_INVALID_ARGUMENT, "md_ewald_pme_grid: NULL");
    if (!ew->pme) {
        k[0] = k[1] = k[2] = 0;
        *order = 0;
        return MD_OK;
    }
    return pme_grid(ew->pme, k, order);
}

int md_ewald_charge_gradient(md_ewald* ew, md_system* sys, double* dedq) {
    if (!ew || !sys || !dedq) return fail(MD_ERR_INVALID_ARGUMENT, "md_ewald_charge_gradient: NULL");
    if (ew->pme)
        return fail(MD_ERR_INVALID_ARGUMENT,
                    "md_ewald_charge_gradient: needs the k-vector reciprocal sum (PME is set)");
    if (sys->ctx != ew->ctx)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_ewald_charge_gradient: context mismatch");
    const int64_t n = sys->n;
    if (n == 0) return MD_OK;
    md_context* ctx = sys->ctx;
    // energies (also builds the list, topology, k vectors and S(k))
    MDB_TRY(ewald_eval_async(ew, sys, 0, false));
    DevBuf buf;
    MDB_TRY(buf.ensure(2 * sizeof(double) * static_cast<size_t>(n)));
    double* dq = buf.as<double>();
    double* dq_o = dq + n;
    const Box3 box{{sys->box[0], sys->box[1], sys->box[2]},
                   {sys->inv_box[0], sys->inv_box[1], sys->inv_box[2]}};
    const RealArgs a = real_args_of(ew, ew->alpha);
    md_verlet* v = ew->list;
    const int g = grid_for(n, kBlock);
    k_ewald_dq<<<g, kBlock, 0, ctx->stream>>>(
        sys->cur.pos, sys->cur.charge, sys->cur.mol, v->nbr.as<int>(), v->count.as<int>(),
        v->stride, sys->cur.orig, sys->slot, ew->partner_off.as<int>(), ew->partner_idx.as<int>(),
        n, box, a, dq);
    MDB_TRY(recip_force_async(ew, sys, kargs_of(ew, sys), true, dq));
    k_to_orig1<<<g, kBlock, 0, ctx->stream>>>(sys->cur.orig, n, dq, dq_o);
    ctx->launches += 3;
    MDB_CHECK_LAUNCH();
    MDB_CUDA(cudaMemcpyAsync(dedq, dq_o, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    buf.release();
    return ctx_check_status(ctx);
}

int md_ewald_real_hvp(md_ewald* ew, md_system* sys, const double* u, double* out) {
    if (!ew || !sys || !u || !out) return fail(MD_ERR_INVALID_ARGUMENT, "md_ewald_real_hvp: NULL");
    if (sys->ctx != ew->ctx) return fail(MD_ERR_INVALID_ARGUMENT, "md_ewald_real_hvp: context mismatch");
    const int64_t n = sys->n;
    if (n == 0) return MD_OK;
    md_context* ctx = sys->ctx;
    MDB_TRY(ewald_eval_async(ew, sys, 0, false));  // list and alpha for this state
    DevBuf buf;
    MDB_TRY(buf.ensure(4 * sizeof(double4) * static_cast<size_t>(n)));
    double4* uo = buf.as<double4>();
    double4* ud = uo + n;
    double4* res = uo + 2 * n;
    double4* res_o = uo + 3 * n;
    MDB_TRY(upload_vec(sys, u, uo, ud));
    const Box3 box{{sys->box[0], sys->box[1], sys->box[2]},
                   {sys->inv_box[0], sys->inv_box[1], sys->inv_box[2]}};
    md_verlet* v = ew->list;
    const int g = grid_for(n, kBlock);
    k_ewald_real_hvp<<<g, kBlock, 0, ctx->stream>>>(sys->cur.pos, sys->cur.charge, sys->cur.mol,
                                                   v->nbr.as<int>(), v->count.as<int>(), v->stride,
                                                   n, box, real_args_of(ew, ew->alpha), ud, res);
    k_to_orig4<<<g, kBlock, 0, ctx->stream>>>(sys->cur.orig, n, res, res_o);
    ctx->launches += 3;
    MDB_CHECK_LAUNCH();
    std::vector<double4> h(static_cast<size_t>(n));
    MDB_CUDA(cudaMemcpyAsync(h.data(), res_o, sizeof(double4) * n, cudaMemcpyDeviceToHost,
                             ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    buf.release();
    for (int64_t o = 0; o < n; ++o) {
        out[3 * o] = h[o].x;
        out[3 * o + 1] = h[o].y;
        out[3 * o + 2] = h[o].z;
    }
    return ctx_check_status(ctx);
}

int md_ewald_alpha(const md_ewald* ew, double* alpha) {
    if (!ew || !alpha) return fail(MD_ERR_INVALID_ARGUMENT, "md_ewald_alpha: NULL");
    *alpha = ew->alpha;
    return MD_OK;
}

int md_ewald_kvector_count(const md_ewald* ew, int* count) {
    if (!ew || !count) return fail(MD_ERR_INVALID_ARGUMENT, "md_ewald_kvector_count: NULL");
    *count = 2 * ew->nk;  // the full set is the half space and its negatives
    return MD_OK;
}

// ------------------------------------------------------------------- SPC/E
int md_spce_create(md_context* ctx, double sigma_o, double epsilon_o, double cutoff, int kmax,
                   double alpha, md_ewald** out) {
    graph_epoch_bump();
    MDB_TRY(ewald_new(ctx, cutoff, kmax, alpha, out));
    (*out)->spce = true;
    (*out)->sigma_o = sigma_o;
    (*out)->epsilon_o = epsilon_o;
    return MD_OK;
}

int md_spce_set_lj_truncation(md_ewald* ew, int truncation) {
    graph_epoch_bump();
    if (!ew || !ew->spce || (truncation != MD_TRUNCATED && truncation != MD_LINEAR_FORCE_SHIFT))
        return fail(MD_ERR_INVALID_ARGUMENT, "md_spce_set_lj_truncation: bad argument");
    ew->lj_truncation = truncation;
    return MD_OK;
}

int md_spce_compute(md_ewald* ew, md_system* sys, int forces, double* energy, double parts[8]) {
    if (!ew || !sys || !ew->spce) return fail(MD_ERR_INVALID_ARGUMENT, "md_spce_compute: not an SPC/E force field");
    if (sys->n % 3 != 0)  // spce_forcefield.cpp:14-17
        return fail(MD_ERR_INVALID_ARGUMENT,
                    "SpceForceField: atom count is not a multiple of 3; expected O,H,H triples");
    MDB_TRY(ewald_eval_async(ew, sys, forces ? 1 : 0, false));
    MDB_TRY(ewald_read(ew, sys->ctx));
    double terms[4], vir;
    fill_terms(ew, terms, &vir);
    // dispersion tail of the oxygen subsystem (lennard_jones.cpp:121-135 with n = N/3)
    const double m = static_cast<double>(sys->n / 3);
    const double rho = m / (sys->box[0] * sys->box[1] * sys->box[2]);
    const double sr = ew->sigma_o / ew->cutoff;
    const double sr3 = sr * sr * sr, sr9 = sr3 * sr3 * sr3;
    const double sig3 = ew->sigma_o * ew->sigma_o * ew->sigma_o;
    const double elrc = ew->lj_truncation == MD_LINEAR_FORCE_SHIFT
                            ? 0.0
                            : (8.0 / 3.0) * kPi * m * rho * ew->epsilon_o * sig3 *
                                  ((1.0 / 3.0) * sr9 - sr3);
    const double disp = ew->last[kEwLj];
    // spce_forcefield.cpp:40: disp + elrc + total()
    const double total = disp + elrc + (terms[0] + terms[1] + terms[2] + terms[3]);
    if (energy) *energy = total;
    if (parts) {
        parts[0] = disp;
        parts[1] = elrc;
        parts[2] = terms[0];
        parts[3] = terms[1];
        parts[4] = terms[2];
        parts[5] = terms[3];
        parts[6] = vir + ew->last[kEwLjW];  // atomic virial, no reference counterpart
        parts[7] = total;
    }
    sys->last_energy = total;
    return MD_OK;
}

}  // extern "C"
