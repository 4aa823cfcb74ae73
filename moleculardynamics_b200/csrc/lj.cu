// lj.cu -- Lennard-Jones pair forces, energy and virial (forcefield/lennard_jones.cpp).
//
// FP64 path: every pair term is computed with the reference's operation order
// (lennard_jones.cpp:56-86) using non-contracting intrinsics, so each pair's
// contribution is bit-identical to the reference's; only the order in which
// per-atom sums are accumulated differs (full neighbour list, no atomics).
// Mixed path: FP64 minimum-image displacement, FP32 r^2, r^-6 and force terms,
// FP64 accumulation of forces, energy and virial.
#include <algorithm>
#include <new>

#include "md_device.cuh"
#include "md_internal.cuh"

namespace mdb {
int verlet_ensure_ready(md_verlet* v, md_system* sys, const char* who);
}

namespace mdb {

namespace {

struct LJArgs {
    double sig2, rc2, rc, uc, dudrc, four_eps, tf_eps;
    float sig2f, rc2f, rcf, ucf, dudrcf, four_epsf, tf_epsf;
    double res[3];  // fixed-point resolution per axis, L / 2^32 (mixed path)
    double band;    // |r^2 - rc^2| below which the mixed path decides exactly
    double res2;    // res^2 (cubic boxes)
    double rc2_lo, rc2_hi;  // rc^2 -/+ band
};

LJArgs make_lj_args(const md_lj* lj) {
    LJArgs a;
    a.sig2 = lj->sigma * lj->sigma;
    a.rc2 = lj->cutoff * lj->cutoff;
    a.rc = lj->cutoff;
    a.uc = lj->u_at_cutoff;
    a.dudrc = lj->dudr_at_cutoff;
    a.four_eps = 4.0 * lj->epsilon;
    a.tf_eps = 24.0 * lj->epsilon;
    a.sig2f = static_cast<float>(a.sig2);
    a.rc2f = static_cast<float>(a.rc2);
    a.rcf = static_cast<float>(a.rc);
    a.ucf = static_cast<float>(a.uc);
    a.dudrcf = static_cast<float>(a.dudrc);
    a.four_epsf = static_cast<float>(a.four_eps);
    a.tf_epsf = static_cast<float>(a.tf_eps);
    a.res[0] = a.res[1] = a.res[2] = 0.0;
    a.band = 0.0;
    a.res2 = 0.0;
    a.rc2_lo = a.rc2_hi = a.rc2;
    return a;
}

// lennard_jones.cpp:62-79 with exact operation order.  Returns false outside rc.
template <bool LFS>
__device__ __forceinline__ bool pair_exact(const LJArgs& a, double r2, double& u, double& w,
                                           double& s) {
    if (!(r2 < a.rc2)) return false;
    const double s2 = __ddiv_rn(a.sig2, r2);
    const double s6 = __dmul_rn(__dmul_rn(s2, s2), s2);
    const double uLJ = __dmul_rn(a.four_eps, __dsub_rn(__dmul_rn(s6, s6), s6));
    const double wLJ = __dmul_rn(a.tf_eps, __dsub_rn(__dmul_rn(__dmul_rn(2.0, s6), s6), s6));
    if (LFS) {
        const double r = __dsqrt_rn(r2);
        u = __dsub_rn(__dsub_rn(uLJ, a.uc), __dmul_rn(__dsub_rn(r, a.rc), a.dudrc));
        w = __dadd_rn(wLJ, __dmul_rn(r, a.dudrc));
    } else {
        u = uLJ;
        w = wLJ;
    }
    s = __ddiv_rn(w, r2);
    return true;
}

// Accumulates the pair (i, j) into atom i's force (FP64 reference arithmetic).
// The displacement is always r_lo - r_hi by original index, as the reference's
// i<j pair sources produce it; atom lo gains +f, atom hi gains -f.
template <bool LFS>
__device__ __forceinline__ void accumulate_exact(const LJArgs& a, const Fold3& f3, double4 pi,
                                                 double4 pj, double& fx, double& fy, double& fz,
                                                 double& e, double& vir) {
    const bool lo = pi.w < pj.w;
    double dx, dy, dz;
    if (lo) min_image_wrapped(f3, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z, dx, dy, dz);
    else min_image_wrapped(f3, pj.x, pj.y, pj.z, pi.x, pi.y, pi.z, dx, dy, dz);
    double u, w, s;
    if (!pair_exact<LFS>(a, norm2_exact(dx, dy, dz), u, w, s)) return;
    const double gx = __dmul_rn(dx, s), gy = __dmul_rn(dy, s), gz = __dmul_rn(dz, s);
    if (lo) {
        fx = __dadd_rn(fx, gx);
        fy = __dadd_rn(fy, gy);
        fz = __dadd_rn(fz, gz);
        e = __dadd_rn(e, u);
        vir = __dadd_rn(vir, w);
    } else {
        fx = __dsub_rn(fx, gx);
        fy = __dsub_rn(fy, gy);
        fz = __dsub_rn(fz, gz);
    }
}

// Mixed precision.  Positions are gathered as int32 fixed point with the box
// length mapped to 2^32 per axis (resolution L / 2^32: 2.5e-8 for the
// 1,048,576-atom liquid's L = 107.5), so the minimum image is the wrap-around of
// an int32 difference and a neighbour is one 16-byte load.  The displacement and
// r^2 are formed in FP64 from the exact integer difference (r^2 is the quantity
// the r^-14 force steepness amplifies, so it is rounded to FP32 once, after it
// is formed); r^-2, r^-6, energy and force magnitude in FP32; the force vector
// assembled and accumulated in FP64.  Energy and virial terms are summed in FP32
// per thread (a few dozen terms; the grid sum is FP64).
__device__ __forceinline__ int wrap_diff(int a, int b) {
    return static_cast<int>(static_cast<unsigned>(a) - static_cast<unsigned>(b));
}

// Exact int32 -> FP64 on the FP64 pipe instead of the conversion unit: the bit
// pattern (0x43300000, x + 2^31) is the double 2^52 + 2^31 + x, and subtracting
// 2^52 + 2^31 from it is exact.
__device__ __forceinline__ double int_to_double(int x) {
    return __hiloint2double(0x43300000, x ^ static_cast<int>(0x80000000u)) - 4503601774854144.0;
}

// The same for the wrapped difference a - b: (a - b + 2^31) mod 2^32 in one add.
__device__ __forceinline__ double diff_to_double(int a, int b) {
    const unsigned biased = static_cast<unsigned>(a) - static_cast<unsigned>(b) + 0x80000000u;
    return __hiloint2double(0x43300000, static_cast<int>(biased)) - 4503601774854144.0;
}

// Reciprocal by the special-function unit alone (PTX rcp.approx, <= 1 ulp).
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// A pair whose fixed-point r^2 lies within a.band of rc^2 could fall on the other
// side of the cutoff than in the FP64 path (a truncated potential jumps there),
// so it is decided by the reference arithmetic on the FP64 positions: the mixed
// path sums exactly the FP64 path's pairs.  The band is several times the
// largest r^2 change the quantisation can cause, so such pairs are rare; the
// main loop only flags them (keeping its register budget) and a second pass
// over the thread's share of the row settles them.
__device__ __forceinline__ bool inside_exact(const LJArgs& a, const Fold3& f3,
                                             const double4* __restrict__ pd, int i, int j) {
    const double4 p = ldg4(pd + i), q = ldg4(pd + j);
    double dx, dy, dz;
    if (p.w < q.w) min_image_wrapped(f3, p.x, p.y, p.z, q.x, q.y, q.z, dx, dy, dz);
    else min_image_wrapped(f3, q.x, q.y, q.z, p.x, p.y, p.z, dx, dy, dz);
    return norm2_exact(dx, dy, dz) < a.rc2;
}

// Main-loop pair term, branch-free: a pair beyond the band contributes zero, a
// pair inside the band contributes zero and flags `near` (settled by
// near_pair below).  Energy and virial take every list entry, so each pair
// twice; the kernels halve them.  CUBIC: one resolution for all axes, so r^2 is
// the integer-unit r^2 scaled once and the force is the integer-unit
// displacement times (F/r) res.
template <bool LFS, bool CUBIC>
__device__ __forceinline__ void pair_mixed(const LJArgs& a, int4 qi, int4 qj, double& fx,
                                           double& fy, double& fz, float& e, float& vir,
                                           bool& near) {
    double dx = diff_to_double(qi.x, qj.x);
    double dy = diff_to_double(qi.y, qj.y);
    double dz = diff_to_double(qi.z, qj.z);
    double r2;
    if constexpr (CUBIC) {
        r2 = fma(dz, dz, fma(dy, dy, dx * dx)) * a.res2;
    } else {
        dx *= a.res[0];
        dy *= a.res[1];
        dz *= a.res[2];
        r2 = fma(dz, dz, fma(dy, dy, dx * dx));
    }
    const bool in_range = r2 < a.rc2_hi;
    const bool in_band = r2 > a.rc2_lo;
    near = near || (in_range && in_band);
    const bool take = in_range && !in_band;
    const float r2f = static_cast<float>(r2);
    const float inv = rcp_approx(r2f);
    const float s2 = a.sig2f * inv;
    const float s6 = s2 * s2 * s2;
    const float t6 = fmaf(s6, s6, -s6);  // s6^2 - s6
    float u = a.four_epsf * t6;
    float w = a.tf_epsf * fmaf(s6, s6, t6);  // 24 eps (2 s6^2 - s6)
    if (LFS) {
        const float r = sqrtf(r2f);
        u = u - a.ucf - (r - a.rcf) * a.dudrcf;
        w = w + r * a.dudrcf;
    }
    float sf = 0.f;
    if (take) {
        sf = w * inv;
        e += u;
        vir += w;
    }
    double sd = static_cast<double>(sf);
    if constexpr (CUBIC) sd *= a.res[0];
    fx = fma(dx, sd, fx);
    fy = fma(dy, sd, fy);
    fz = fma(dz, sd, fz);
}

// A pair next to the cutoff (second pass): decided by the reference arithmetic
// on the FP64 positions, then the same terms as pair_mixed (non-cubic form).
template <bool LFS>
__device__ __forceinline__ void near_pair(const LJArgs& a, const Fold3& f3,
                                          const double4* __restrict__ pd, int i, int j, int4 qi,
                                          int4 qj, double& fx, double& fy, double& fz, float& e,
                                          float& vir) {
    const double dx = int_to_double(wrap_diff(qi.x, qj.x)) * a.res[0];
    const double dy = int_to_double(wrap_diff(qi.y, qj.y)) * a.res[1];
    const double dz = int_to_double(wrap_diff(qi.z, qj.z)) * a.res[2];
    const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
    if (!(r2 < a.rc2_hi) || !(r2 > a.rc2_lo) || !inside_exact(a, f3, pd, i, j)) return;
    const float r2f = static_cast<float>(r2);
    const float inv = rcp_approx(r2f);
    const float s2 = a.sig2f * inv;
    const float s6 = s2 * s2 * s2;
    const float t6 = fmaf(s6, s6, -s6);
    float u = a.four_epsf * t6;
    float w = a.tf_epsf * fmaf(s6, s6, t6);
    if (LFS) {
        const float r = sqrtf(r2f);
        u = u - a.ucf - (r - a.rcf) * a.dudrcf;
        w = w + r * a.dudrcf;
    }
    const double sd = static_cast<double>(w * inv);
    fx = fma(dx, sd, fx);
    fy = fma(dy, sd, fy);
    fz = fma(dz, sd, fz);
    e += u;
    vir += w;
}

constexpr int kBlock = 256;

// Full Verlet list, TPA lanes per atom; rows are nbr[i*stride .. +count[i]).
// Register budget per unroll factor: U gather chains per thread need ~8U more
// registers, traded against resident blocks per SM.  The mixed kernel is bound by
// gather latency, so it takes 5 blocks (48 registers, a few spilled) -- measured
// 0.266 ms against 0.282 ms at 4 blocks on the 1M-atom liquid; 6 blocks spill too
// much (0.390 ms).
template <int U, bool MIXED>
struct UnrollBlocks {
    static constexpr int value = U >= 4 ? 2 : (MIXED ? 5 : 4);
};

// Position source of the pair kernel: FP64 double4 for the reference arithmetic,
// int32 fixed point for the mixed path.
template <bool MIXED>
struct PosOf {
    using T = double4;
    static __device__ __forceinline__ T load(const T* p) { return ldg4(p); }
};
template <>
struct PosOf<true> {
    using T = int4;
    static __device__ __forceinline__ T load(const T* p) { return __ldg(p); }
};

// The Verlet-list force pass of one system, for block `block` of `nblocks`
// (a batched launch gives each system's blocks their own rank and count).  With
// KICK the pass also applies the closing half-kick to each atom once its force is
// summed, and reduces the kinetic energy with the energy and virial (result slots
// 0, 1, 2), so no separate kick pass re-reads the forces and velocities.
template <int TPA, bool MIXED, bool LFS, int U, bool CUBIC, bool KICK = false>
__device__ __forceinline__ void lj_verlet_body(
    const typename PosOf<MIXED>::T* __restrict__ pos, const double4* __restrict__ pd,
    const int* __restrict__ nbr, const int* __restrict__ count, int stride, int64_t n,
    const Box3& box, const LJArgs& a, double* __restrict__ fxo, double* __restrict__ fyo,
    double* __restrict__ fzo, double* part, unsigned* ticket, double* out, unsigned block,
    unsigned nblocks, const KickArgs& kick) {
    using P = PosOf<MIXED>;
    const int64_t t = block * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const int64_t i = t / TPA;
    const int g = static_cast<int>(t % TPA);
    const Fold3 f3 = fold3_of(box);
    double fx = 0.0, fy = 0.0, fz = 0.0, e = 0.0, vir = 0.0;
    float ef = 0.f, vf = 0.f;  // mixed path: energy and virial terms
    bool near = false;
    if (i < n) {
        const typename P::T pi = P::load(pos + i);
        const int cnt = min(count[i], stride);  // an overflowed row is flagged, never over-read
        const int* row = nbr + i * static_cast<int64_t>(stride);
        // U independent index->position gather chains in flight per thread, and
        // the next U list indices are fetched while the current pairs are
        // computed.  Pair terms are accumulated in list order.
        int k = g;
        int jn[U];
#pragma unroll
        for (int u = 0; u < U; ++u) jn[u] = k + u * TPA < cnt ? __ldg(row + k + u * TPA) : 0;
        for (; k + (U - 1) * TPA < cnt; k += U * TPA) {
            int j[U];
            typename P::T pj[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                j[u] = jn[u];
                pj[u] = P::load(pos + j[u]);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int kn = k + (U + u) * TPA;
                jn[u] = kn < cnt ? __ldg(row + kn) : 0;
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if constexpr (MIXED)
                    pair_mixed<LFS, CUBIC>(a, pi, pj[u], fx, fy, fz, ef, vf, near);
                else accumulate_exact<LFS>(a, f3, pi, pj[u], fx, fy, fz, e, vir);
            }
        }
        // fewer than U entries left; their indices are already in jn
#pragma unroll
        for (int u = 0; u < U - 1; ++u) {
            if (k + u * TPA < cnt) {
                const typename P::T pj = P::load(pos + jn[u]);
                if constexpr (MIXED)
                    pair_mixed<LFS, CUBIC>(a, pi, pj, fx, fy, fz, ef, vf, near);
                else accumulate_exact<LFS>(a, f3, pi, pj, fx, fy, fz, e, vir);
            }
        }
        if constexpr (MIXED) {
            if (near) {  // rare: settle the pairs next to the cutoff
                for (int kk = g; kk < cnt; kk += TPA) {
                    const int j = __ldg(row + kk);
                    near_pair<LFS>(a, f3, pd, static_cast<int>(i), j, pi, P::load(pos + j), fx, fy,
                                   fz, ef, vf);
                }
            }
            e = 0.5 * static_cast<double>(ef);  // every pair was taken from both sides
            vir = 0.5 * static_cast<double>(vf);
        }
    }
#pragma unroll
    for (int o = TPA / 2; o > 0; o >>= 1) {
        fx += __shfl_xor_sync(0xffffffffu, fx, o);
        fy += __shfl_xor_sync(0xffffffffu, fy, o);
        fz += __shfl_xor_sync(0xffffffffu, fz, o);
    }
    double ke = 0.0;
    if (i < n && g == 0) {
        fxo[i] = fx;
        fyo[i] = fy;
        fzo[i] = fz;
        if constexpr (KICK) {  // the closing half-kick, as the separate kick kernel does it
            const double c = __dmul_rn(kick.half_dt, kick.inv_mass[i]);
            const double vx = fma(c, fx, kick.vx[i]);
            const double vy = fma(c, fy, kick.vy[i]);
            const double vz = fma(c, fz, kick.vz[i]);
            kick.vx[i] = vx;
            kick.vy[i] = vy;
            kick.vz[i] = vz;
            ke = 0.5 * kick.mass[i] * (vx * vx + vy * vy + vz * vz);
        }
    }
    if constexpr (KICK) {
        double v[3] = {e, vir, ke};
        grid_reduce_at<3>(v, part, ticket, out, kick.status, block, nblocks);
    } else {
        double v[2] = {e, vir};
        grid_reduce_at<2>(v, part, ticket, out, nullptr, block, nblocks);
    }
}

template <int TPA, bool MIXED, bool LFS, int U, bool CUBIC, bool KICK>
__global__ void __launch_bounds__(kBlock, UnrollBlocks<U, MIXED>::value)
k_lj_verlet(const typename PosOf<MIXED>::T* __restrict__ pos, const double4* __restrict__ pd,
            const int* __restrict__ nbr, const int* __restrict__ count, int stride, int64_t n,
            Box3 box, LJArgs a, double* __restrict__ fxo, double* __restrict__ fyo,
            double* __restrict__ fzo, double* part, unsigned* ticket, double* out, KickArgs kick) {
    lj_verlet_body<TPA, MIXED, LFS, U, CUBIC, KICK>(pos, pd, nbr, count, stride, n, box, a, fxo,
                                                    fyo, fzo, part, ticket, out, blockIdx.x,
                                                    gridDim.x, kick);
}

// The gathered kernel shape that also takes the closing half-kick (the default
// shape; other shapes leave the kick to the integrator's own pass).
constexpr bool verlet_kicks(int tpa, int unroll) { return tpa == 2 && unroll == 2; }

// One system's arguments of the batched force pass.
struct BatchForceRep {
    const void* pos;  // int4 fixed-point (mixed) or double4 positions
    const double4* pd;
    const int* nbr;
    const int* count;
    int stride;
    int64_t n;
    Box3 box;
    LJArgs a;
    double *fx, *fy, *fz;
    double* part;
    unsigned* ticket;
    double* out;
    KickArgs kick;  // used by the kernel that takes the closing half-kick
};

// The force pass of many systems in one launch: each block finds its system in
// the block table and runs exactly the blocks a launch of that system alone
// would, so every system's forces and sums equal its solo pass.
template <int TPA, bool MIXED, bool LFS, int U, bool CUBIC, bool KICK>
__global__ void __launch_bounds__(kBlock, UnrollBlocks<U, MIXED>::value)
k_lj_verlet_batch(const BatchForceRep* __restrict__ reps, const int4* __restrict__ blk) {
    // the system's arguments are read from shared memory as the solo kernel reads
    // its parameters, rather than held in registers
    __shared__ BatchForceRep d;
    const int4 e = __ldg(blk + blockIdx.x);
    if (threadIdx.x == 0) d = reps[e.x];
    __syncthreads();
    lj_verlet_body<TPA, MIXED, LFS, U, CUBIC, KICK>(
        static_cast<const typename PosOf<MIXED>::T*>(d.pos), d.pd, d.nbr, d.count, d.stride, d.n,
        d.box, d.a, d.fx, d.fy, d.fz, d.part, d.ticket, d.out, e.y, e.z, d.kick);
}

// One thread's share of a row (entries g, g + TPA, ...): U position loads in
// flight and the next U indices read one iteration ahead; pairs are accumulated
// in row order.  row(k) gives entry k, load(j) the fixed-point position of j.
template <int TPA, int U, class Row, class Load, class Pair>
__device__ __forceinline__ void walk_row(int g, int cnt, Row row, Load load, Pair pair) {
    int k = g;
    int jn[U];
#pragma unroll
    for (int u = 0; u < U; ++u) jn[u] = k + u * TPA < cnt ? row(k + u * TPA) : 0;
    for (; k + (U - 1) * TPA < cnt; k += U * TPA) {
        int4 pj[U];
#pragma unroll
        for (int u = 0; u < U; ++u) pj[u] = load(jn[u]);
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int kn = k + (U + u) * TPA;
            jn[u] = kn < cnt ? row(kn) : 0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) pair(pj[u]);
    }
#pragma unroll
    for (int u = 0; u < U - 1; ++u)
        if (k + u * TPA < cnt) pair(load(jn[u]));
}

// Pair sums of one thread's share of a row (mixed path).
struct PairSums {
    double fx, fy, fz;
    float e, vir;
};

// The rare paths of k_lj_halo, out of line so that the staged main loop keeps its
// registers.  Pairs of a staged row next to the cutoff, decided exactly and
// added in row order to the sums so far:
template <bool LFS>
__device__ __noinline__ PairSums near_pairs_tile(LJArgs a, Box3 box, const double4* pd,
                                                 const uint16_t* row, int cnt, int g, int ii,
                                                 int4 pi, const int4* s_q, const int* s_beg,
                                                 const int* s_base, int nr, PairSums acc) {
    constexpr int TPA = kBlock / kHaloAtoms;
    const Fold3 f3 = fold3_of(box);
    for (int kk = g; kk < cnt; kk += TPA) {
        const int sl = row[kk] >> 4;  // rows hold byte offsets of 16-byte slots
        int lo = 0, hi = nr;  // the last run whose first slot is <= sl
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_base[mid] <= sl) lo = mid;
            else hi = mid;
        }
        near_pair<LFS>(a, f3, pd, ii, s_beg[lo] + (sl - s_base[lo]), pi, s_q[sl], acc.fx, acc.fy,
                       acc.fz, acc.e, acc.vir);
    }
    return acc;
}

// and a whole row of a tile that was not staged, gathered through the int32 row
// exactly as k_lj_verlet's mixed path walks it.
template <bool LFS, bool CUBIC, int U, int TPA>
__device__ __noinline__ PairSums gathered_row(LJArgs a, Box3 box, const double4* pd, const int4* q,
                                              const int* row, int cnt, int g, int ii, int4 pi) {
    PairSums acc = {0.0, 0.0, 0.0, 0.f, 0.f};
    bool near = false;
    walk_row<TPA, U>(g, cnt, [&](int k) { return __ldg(row + k); },
                     [&](int j) { return __ldg(q + j); },
                     [&](int4 pj) {
                         pair_mixed<LFS, CUBIC>(a, pi, pj, acc.fx, acc.fy, acc.fz, acc.e, acc.vir,
                                                near);
                     });
    if (near) {
        const Fold3 f3 = fold3_of(box);
        for (int kk = g; kk < cnt; kk += TPA) {
            const int j = __ldg(row + kk);
            near_pair<LFS>(a, f3, pd, ii, j, pi, __ldg(q + j), acc.fx, acc.fy, acc.fz, acc.e,
                           acc.vir);
        }
    }
    return acc;
}

// Mixed-precision forces over halo tiles (one CTA per tile of kHaloAtoms sorted
// atoms, two threads per atom).  The CTA copies the fixed-point positions of its
// tile's cell runs into shared memory -- contiguous, coalesced reads of an array
// that stays in L2 -- and then reads each row as 16-bit tile slots: a neighbour
// costs a 2-byte list read and a shared-memory load instead of a 4-byte read and
// a gather through L1/L2.  A tile that was not staged (too many cells or atoms
// around it) walks its int32 row with global gathers.  Pair arithmetic, the
// exact decision of pairs next to the cutoff and the accumulation order are
// those of k_lj_verlet's mixed path.
template <bool LFS, int U, bool CUBIC, bool KICK>
__global__ void __launch_bounds__(kBlock, 4)
k_lj_halo(const int4* __restrict__ q, const double4* __restrict__ pd, const int* __restrict__ nbr,
          const uint16_t* __restrict__ nbr16, const int* __restrict__ count, int stride, int64_t n,
          const int2* __restrict__ runs, const int2* __restrict__ meta, Box3 box, LJArgs a,
          double* __restrict__ fxo, double* __restrict__ fyo, double* __restrict__ fzo,
          double* part, unsigned* ticket, double* out, KickArgs kick) {
    constexpr int TPA = kBlock / kHaloAtoms;
    extern __shared__ int4 s_q[];  // kHaloCap slots
    __shared__ int s_beg[kHaloRuns + 1], s_base[kHaloRuns + 1];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int2 m = meta[blockIdx.x];
    const bool staged = m.x > 0;
    if (staged) {
        if (tid < m.x) {
            const int2 r = runs[static_cast<int64_t>(blockIdx.x) * kHaloRuns + tid];
            s_beg[tid] = r.x;
            s_base[tid] = r.y;
        }
        if (tid == 0) s_base[m.x] = m.y;
        __syncthreads();
        // every copy is issued before any is waited on (asynchronous 16-byte
        // global->shared copies through L2), so the tile costs one L2 latency
        for (int t = warp; t < m.x; t += kBlock / 32) {
            const int4* src = q + s_beg[t];
            const int base = s_base[t], len = s_base[t + 1] - base;
            for (int k = lane; k < len; k += 32) {
                const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(s_q + base + k));
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src + k)
                             : "memory");
            }
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        __syncthreads();
    }
    const int64_t i = static_cast<int64_t>(blockIdx.x) * kHaloAtoms + tid / TPA;
    const int g = tid % TPA;
    PairSums acc = {0.0, 0.0, 0.0, 0.f, 0.f};
    if (i < n) {
        const int4 pi = __ldg(q + i);
        const int cnt = min(count[i], stride);  // an overflowed row is flagged, never over-read
        const int ii = static_cast<int>(i);
        if (staged) {
            // eight slots per 16-byte read (rows start 16-byte aligned: the stride is
            // a multiple of 8), the next read issued before the current pairs; this
            // thread takes the entries g, g + 2, ... of each chunk -- the row order
            // of the gathered walk.  Slots are stored as byte offsets into the tile.
            const uint16_t* row = nbr16 + i * stride;
            const uint4* rowv = reinterpret_cast<const uint4*>(row);
            const char* tile = reinterpret_cast<const char*>(s_q);
            const unsigned sel = g ? 0x4432u : 0x4410u;  // this thread's 16-bit halves
            const int nfull = cnt >> 3, nch = (cnt + 7) >> 3;
            bool near = false;
            uint4 cur = nch > 0 ? __ldg(rowv) : make_uint4(0u, 0u, 0u, 0u);
            auto chunk = [&](const uint4& v) {
                const unsigned w4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int t = 0; t < 4; ++t)
                    pair_mixed<LFS, CUBIC>(
                        a, pi, *reinterpret_cast<const int4*>(tile + __byte_perm(w4[t], 0u, sel)),
                        acc.fx, acc.fy, acc.fz, acc.e, acc.vir, near);
            };
            int c = 0;
            for (; c + 1 < nfull; c += 2) {  // two chunks per trip: no register copies
                const uint4 nxt = __ldg(rowv + c + 1);
                chunk(cur);
                cur = c + 2 < nch ? __ldg(rowv + c + 2) : nxt;
                chunk(nxt);
            }
            if (c < nfull) {
                const uint4 nxt = c + 1 < nch ? __ldg(rowv + c + 1) : cur;
                chunk(cur);
                cur = nxt;
            }
            const int rem = cnt & 7;  // the last, partial chunk
            if (rem > g) {
                const unsigned w4[4] = {cur.x, cur.y, cur.z, cur.w};
#pragma unroll
                for (int t = 0; t < 4; ++t)
                    if (g + 2 * t < rem)
                        pair_mixed<LFS, CUBIC>(
                            a, pi,
                            *reinterpret_cast<const int4*>(tile + __byte_perm(w4[t], 0u, sel)),
                            acc.fx, acc.fy, acc.fz, acc.e, acc.vir, near);
            }
            if (near)  // rare: settle the pairs next to the cutoff
                acc = near_pairs_tile<LFS>(a, box, pd, row, cnt, g, ii, pi, s_q, s_beg, s_base, m.x,
                                           acc);
        } else {
            acc = gathered_row<LFS, CUBIC, U, TPA>(a, box, pd, q, nbr + i * stride, cnt, g, ii, pi);
        }
    }
    double fx = acc.fx, fy = acc.fy, fz = acc.fz;
    const double e = 0.5 * static_cast<double>(acc.e);  // every pair was taken from both sides
    const double vir = 0.5 * static_cast<double>(acc.vir);
#pragma unroll
    for (int o = TPA / 2; o > 0; o >>= 1) {
        fx += __shfl_xor_sync(0xffffffffu, fx, o);
        fy += __shfl_xor_sync(0xffffffffu, fy, o);
        fz += __shfl_xor_sync(0xffffffffu, fz, o);
    }
    double ke = 0.0;
    if (i < n && g == 0) {
        fxo[i] = fx;
        fyo[i] = fy;
        fzo[i] = fz;
        if constexpr (KICK) {  // the closing half-kick, as the separate kick kernel does it
            const double c = __dmul_rn(kick.half_dt, kick.inv_mass[i]);
            const double vx = fma(c, fx, kick.vx[i]);
            const double vy = fma(c, fy, kick.vy[i]);
            const double vz = fma(c, fz, kick.vz[i]);
            kick.vx[i] = vx;
            kick.vy[i] = vy;
            kick.vz[i] = vz;
            ke = 0.5 * kick.mass[i] * (vx * vx + vy * vy + vz * vz);
        }
    }
    if constexpr (KICK) {  // energy, virial and kinetic energy (result slots 0, 1, 2)
        double v[3] = {e, vir, ke};
        grid_reduce<3>(v, part, ticket, out, kick.status);
    } else {
        double v[2] = {e, vir};
        grid_reduce<2>(v, part, ticket, out);
    }
}

// ------------------------------------------------------------ k_lj_tile
// Mixed-precision forces over halo tiles, persistent and double-buffered (cubic
// boxes).  Each CTA walks the tiles blockIdx.x, blockIdx.x + gridDim.x, ...: while
// its warps compute one tile from one shared-memory buffer, the bulk-copy engine
// fills the other with the next tile's halo -- one 1-D cp.async.bulk per run of
// cells, completing on the buffer's mbarrier.  The loop has no CTA-wide barrier:
// each warp finishes a tile on its own, and the last warp to finish one queues
// the copies of the tile after next into the buffer it frees.  The source is this
// GPU's own fixed-point position array; no copy is multicast.
//
// Per list entry: one 16-bit slot read out of a row word, one shared-memory load,
// and the arithmetic of the gathered mixed kernel (pair_mixed): the exact integer
// displacement as FP64, r^2 formed in FP64 and rounded to FP32 once, FP32 pair
// terms, the force vector accumulated in FP64.  Rows of staged tiles are padded to
// whole 8-entry chunks with the atom's own slot (r^2 = 0, skipped), so entries are
// read without a count test.  Pairs within the cutoff band are settled by the
// reference arithmetic on the FP64 positions, as in the gathered kernel.
constexpr long long kTileWaitCycles = 2000000000LL;  // ~1 s bound on a tile's copies

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Every lane of the warp waits for the phase of `bar` with the given parity (each
// then sees the copied data); the warp gives up together after ~1 s.
__device__ __forceinline__ bool warp_wait_bounded(uint64_t* bar, unsigned parity) {
    if (__all_sync(0xffffffffu, mbar_try_wait(bar, parity))) return true;
    const long long t0 = clock64();
    for (;;) {
        if (__all_sync(0xffffffffu, mbar_try_wait(bar, parity))) return true;
        const long long el = __shfl_sync(0xffffffffu, clock64() - t0, 0);
        if (el > kTileWaitCycles) return false;
    }
}

__device__ __forceinline__ uint64_t l2_evict_last_policy() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ uint64_t l2_evict_first_policy() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// Global -> shared bulk copy (16-byte aligned ends, size a multiple of 16) that
// completes `bytes` transactions on the mbarrier.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar,
                                         uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint "
        "[%0], [%1], %2, [%3], %4;" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

// A tile kernel with TPA threads per atom reads each 8-entry chunk of a row as TPA
// words of 8 / TPA 16-bit slots: thread g takes entries 8c + (8 / TPA) g + e.
template <int TPA>
struct TileRow;
template <>
struct TileRow<2> {
    static constexpr int EPT = 4;
    using W = uint2;
    static __device__ __forceinline__ W load(const uint16_t* row, int c, int g, uint64_t pol) {
        uint2 v;
        asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;"
                     : "=r"(v.x), "=r"(v.y)
                     : "l"(reinterpret_cast<const uint2*>(row) + 2 * c + g), "l"(pol));
        return v;
    }
    static __device__ __forceinline__ unsigned slot(const W& w, int e) {
        return ((e < 2 ? w.x : w.y) >> (16 * (e & 1))) & 0xffffu;
    }
};
template <>
struct TileRow<4> {
    static constexpr int EPT = 2;
    using W = unsigned;
    static __device__ __forceinline__ W load(const uint16_t* row, int c, int g, uint64_t pol) {
        unsigned v;
        asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;"
                     : "=r"(v)
                     : "l"(reinterpret_cast<const unsigned*>(row) + 4 * c + g), "l"(pol));
        return v;
    }
    static __device__ __forceinline__ unsigned slot(const W& w, int e) {
        return (w >> (16 * e)) & 0xffffu;
    }
};
template <>
struct TileRow<8> {
    static constexpr int EPT = 1;
    using W = unsigned;
    static __device__ __forceinline__ W load(const uint16_t* row, int c, int g, uint64_t pol) {
        unsigned short v;
        asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u16 %0, [%1], %2;"
                     : "=h"(v)
                     : "l"(row + 8 * c + g), "l"(pol));
        return v;
    }
    static __device__ __forceinline__ unsigned slot(const W& w, int) { return w; }
};

// One warp queues the halo of tile t into `dst`: one bulk copy per run (lane r
// takes run r), then lane 0 arrives on `bar` expecting the bytes.  A tile that is
// not staged arrives with none, so every tile completes one phase.
__device__ __forceinline__ void tile_issue(int t, int4* dst, uint64_t* bar, const int4* q,
                                           const int2* __restrict__ runs,
                                           const int2* __restrict__ meta, uint64_t policy) {
    const int lane = threadIdx.x & 31;
    const int2 m = meta[t];
    unsigned bytes = 0;
    for (int r0 = 0; r0 < m.x; r0 += 32) {
        const int r = r0 + lane;
        const int2 cur = r < m.x ? runs[static_cast<int64_t>(t) * kHaloRuns + r] : make_int2(0, m.y);
        int end = __shfl_down_sync(0xffffffffu, cur.y, 1);
        if (lane == 31 && r + 1 < m.x) end = runs[static_cast<int64_t>(t) * kHaloRuns + r + 1].y;
        if (r + 1 >= m.x) end = m.y;
        const int len = r < m.x ? end - cur.y : 0;
        if (len > 0) bulk_g2s(dst + cur.y, q + cur.x, 16u * static_cast<unsigned>(len), bar, policy);
        bytes += 16u * static_cast<unsigned>(len > 0 ? len : 0);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
    __syncwarp();
    if (lane == 0) mbar_arrive_expect_tx(bar, bytes);
}

// One staged entry (pair_mixed's arithmetic, cubic box); r^2 = 0 is the row's
// padding (the atom itself) and contributes nothing.
template <bool LFS>
__device__ __forceinline__ void pair_tile(const LJArgs& a, int4 qi, int4 qj, double& fx,
                                          double& fy, double& fz, float& e, float& vir,
                                          bool& near) {
    const double dx = diff_to_double(qi.x, qj.x);
    const double dy = diff_to_double(qi.y, qj.y);
    const double dz = diff_to_double(qi.z, qj.z);
    const double r2 = fma(dz, dz, fma(dy, dy, dx * dx)) * a.res2;
    const bool in_range = r2 < a.rc2_hi;
    const bool in_band = r2 > a.rc2_lo;
    near = near || (in_range && in_band);
    const bool take = in_range && !in_band && r2 > 0.0;
    const float r2f = static_cast<float>(r2);
    const float inv = rcp_approx(r2f);
    const float s2 = a.sig2f * inv;
    const float s6 = s2 * s2 * s2;
    const float t6 = fmaf(s6, s6, -s6);
    float u = a.four_epsf * t6;
    float w = a.tf_epsf * fmaf(s6, s6, t6);
    if (LFS) {
        const float r = sqrtf(r2f);
        u = u - a.ucf - (r - a.rcf) * a.dudrcf;
        w = w + r * a.dudrcf;
    }
    float sf = 0.f;
    if (take) {
        sf = w * inv;
        e += u;
        vir += w;
    }
    const double sd = static_cast<double>(sf) * a.res[0];
    fx = fma(dx, sd, fx);
    fy = fma(dy, sd, fy);
    fz = fma(dz, sd, fz);
}

template <bool LFS, int TPA>
__global__ void __launch_bounds__(kHaloAtoms * TPA, TPA == 8 ? 1 : 2)
k_lj_tile(const int4* __restrict__ q, const double4* __restrict__ pd, const int* __restrict__ nbr,
          const uint16_t* __restrict__ nbr16, const int* __restrict__ count, int stride, int64_t n,
          int ntiles, const int2* __restrict__ runs, const int2* __restrict__ meta,
          const __grid_constant__ Box3 box, const __grid_constant__ LJArgs a,
          double* __restrict__ fxo, double* __restrict__ fyo, double* __restrict__ fzo,
          double* part, unsigned* ticket, double* out, uint32_t* status) {
    using R = TileRow<TPA>;
    constexpr int EPT = R::EPT;
    constexpr int kWarps = kHaloAtoms * TPA / 32;
    extern __shared__ __align__(128) int4 s_buf[];  // 2 x kHaloCap slots
    __shared__ uint64_t s_bar[2];
    __shared__ int s_done[2];  // warps finished with each buffer's current tile
    const int tid = threadIdx.x, lane = tid & 31;
    const int g = tid & (TPA - 1);
    const uint64_t pol_q = l2_evict_last_policy(), pol_row = l2_evict_first_policy();
    if (tid == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        s_done[0] = s_done[1] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int stride_t = static_cast<int>(gridDim.x);
    if (tid < 32) {
        if (static_cast<int>(blockIdx.x) < ntiles)
            tile_issue(blockIdx.x, s_buf, &s_bar[0], q, runs, meta, pol_q);
        if (static_cast<int>(blockIdx.x) + stride_t < ntiles)
            tile_issue(blockIdx.x + stride_t, s_buf + kHaloCap, &s_bar[1], q, runs, meta, pol_q);
    }
    const Fold3 f3 = fold3_of(box);
    double e_tot = 0.0, w_tot = 0.0;
    bool timed_out = false;
    int k = 0;
    for (int t = blockIdx.x; t < ntiles; t += stride_t, ++k) {
        const int b = k & 1;
        int4* buf = s_buf + b * kHaloCap;
        if (!warp_wait_bounded(&s_bar[b], static_cast<unsigned>((k >> 1) & 1))) {
            timed_out = true;  // the copies never landed: flag it and leave the loop
            break;
        }
        const int2 m = meta[t];
        const int64_t i = static_cast<int64_t>(t) * kHaloAtoms + (tid / TPA);
        const int ii = static_cast<int>(i);
        double fx = 0.0, fy = 0.0, fz = 0.0;
        float e = 0.f, vir = 0.f;
        if (i < n) {
            const int4 pi = __ldg(q + i);
            const int cnt = min(count[i], stride);  // an overflowed row is flagged, never over-read
            if (m.x > 0) {
                const uint16_t* row = nbr16 + i * stride;
                const char* tile = reinterpret_cast<const char*>(buf);
                const int nch = (cnt + 7) >> 3;  // whole chunks: the last one is padded
                bool near = false;
                typename R::W word = nch > 0 ? R::load(row, 0, g, pol_row) : typename R::W{};
                for (int c = 0; c < nch; ++c) {
                    const typename R::W cur = word;
                    if (c + 1 < nch) word = R::load(row, c + 1, g, pol_row);
#pragma unroll
                    for (int h = 0; h < EPT; ++h) {
                        const int4 qj = *reinterpret_cast<const int4*>(tile + R::slot(cur, h));
                        pair_tile<LFS>(a, pi, qj, fx, fy, fz, e, vir, near);
                    }
                }
                if (near) {
                    // rare: the pairs next to the cutoff, decided by the reference
                    // arithmetic on the FP64 positions (the slot maps to its atom
                    // through the tile's runs)
                    const int2* tr = runs + static_cast<int64_t>(t) * kHaloRuns;
                    for (int c = 0; c < nch; ++c) {
#pragma unroll
                        for (int h = 0; h < EPT; ++h) {
                            const int kk = 8 * c + EPT * g + h;
                            if (kk >= cnt) continue;
                            const unsigned off = row[kk];
                            const int sl = static_cast<int>(off >> 4);
                            int lo = 0, hi = m.x;  // the last run whose first slot is <= sl
                            while (hi - lo > 1) {
                                const int mid = (lo + hi) >> 1;
                                if (tr[mid].y <= sl) lo = mid;
                                else hi = mid;
                            }
                            near_pair<LFS>(a, f3, pd, ii, tr[lo].x + (sl - tr[lo].y), pi,
                                           *reinterpret_cast<const int4*>(tile + off), fx, fy, fz,
                                           e, vir);
                        }
                    }
                }
            } else {
                // a tile that is not staged: its int32 row, positions gathered
                const int* row = nbr + i * stride;
                bool near = false;
                for (int kk = g; kk < cnt; kk += TPA)
                    pair_mixed<LFS, true>(a, pi, __ldg(q + __ldg(row + kk)), fx, fy, fz, e, vir,
                                          near);
                if (near) {
                    for (int kk = g; kk < cnt; kk += TPA) {
                        const int j = __ldg(row + kk);
                        near_pair<LFS>(a, f3, pd, ii, j, pi, __ldg(q + j), fx, fy, fz, e, vir);
                    }
                }
            }
        }
#pragma unroll
        for (int o = TPA / 2; o > 0; o >>= 1) {
            fx += __shfl_xor_sync(0xffffffffu, fx, o);
            fy += __shfl_xor_sync(0xffffffffu, fy, o);
            fz += __shfl_xor_sync(0xffffffffu, fz, o);
        }
        if (i < n && g == 0) {
            fxo[i] = fx;
            fyo[i] = fy;
            fzo[i] = fz;
        }
        e_tot += 0.5 * static_cast<double>(e);  // every pair was taken from both sides
        w_tot += 0.5 * static_cast<double>(vir);
        // this warp is done with the buffer; the last warp to finish queues the
        // tile after next into it
        __syncwarp();
        int done = 0;
        if (lane == 0) {
            __threadfence_block();
            done = atomicAdd(&s_done[b], 1) + 1;
        }
        done = __shfl_sync(0xffffffffu, done, 0);
        if (done == kWarps) {
            if (lane == 0) s_done[b] = 0;
            __threadfence_block();
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            if (t + 2 * stride_t < ntiles)
                tile_issue(t + 2 * stride_t, buf, &s_bar[b], q, runs, meta, pol_q);
        }
    }
    if (timed_out) {
        if (lane == 0) atomicOr(status, MD_STATUS_WAIT_TIMEOUT);
        // before the CTA exits, give the copies that may still be queued into its
        // buffers a bounded time to land
        warp_wait_bounded(&s_bar[k & 1], static_cast<unsigned>((k >> 1) & 1));
        warp_wait_bounded(&s_bar[(k + 1) & 1], static_cast<unsigned>(((k + 1) >> 1) & 1));
    }
    double v[2] = {e_tot, w_tot};
    grid_reduce<2>(v, part, ticket, out);
}

// ------------------------------------------------------------ k_lj_tile1
// A single-buffer form of the tile kernel (shape 1): one CTA per tile,
// two threads per atom, four CTAs per SM, so that while one CTA waits for its
// halo the others compute.  Warp 0 queues the halo with one bulk copy per run
// (tile_issue) and every thread waits on the CTA's mbarrier; no thread copies
// data and no CTA barrier precedes the pairs.  Rows are padded to whole 8-entry
// chunks (the atom's own slot), so each thread reads its 4 slots of a chunk with
// one 8-byte load and evaluates them without a count test.  The arithmetic is the
// gathered kernel's in integer units of the fixed-point grid: d exact, r^2 formed
// in FP64 and rounded to FP32 once, FP32 pair terms, the force accumulated in
// FP64 and scaled by 1 / res at the end; pairs in the cutoff band are settled by
// the reference arithmetic as there.
struct UnitConst {
    double lo, hi;        // rc^2 -/+ band in units res^2
    float sig2u;          // sigma^2 in units res^2
    float four_epsf, tf_epsf, ucf, rcf, dudrcf, res_f;
};

template <bool LFS>
__device__ __forceinline__ void pair_unit(const UnitConst& c, int4 qi, int4 qj, double& fx,
                                          double& fy, double& fz, float& e, float& vir,
                                          bool& near) {
    const double dx = diff_to_double(qi.x, qj.x);
    const double dy = diff_to_double(qi.y, qj.y);
    const double dz = diff_to_double(qi.z, qj.z);
    const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));  // exact up to one rounding
    const bool below = r2 < c.lo;
    near = near || (!below && r2 < c.hi);
    const bool pad = !(r2 > 0.0);  // r^2 = 0: the row's padding (the atom itself)
    const float m = (below && !pad) ? 1.f : 0.f;
    // the padding's r^2 is replaced by a far one, so its (masked) terms stay finite
    const float r2f = pad ? 1.0e30f : static_cast<float>(r2);
    const float inv = rcp_approx(r2f);
    const float s2 = c.sig2u * inv;
    const float s6 = s2 * s2 * s2;
    const float t6 = fmaf(s6, s6, -s6);
    float u = c.four_epsf * t6;
    float w = c.tf_epsf * fmaf(s6, s6, t6);
    if (LFS) {
        const float r = sqrtf(r2f) * c.res_f;
        u = u - c.ucf - (r - c.rcf) * c.dudrcf;
        w = w + r * c.dudrcf;
    }
    e = fmaf(u, m, e);
    vir = fmaf(w, m, vir);
    const double sd = static_cast<double>((w * m) * inv);
    fx = fma(dx, sd, fx);
    fy = fma(dy, sd, fy);
    fz = fma(dz, sd, fz);
}

// Word c of a row for thread g of the two an atom has (4 slots), streamed past L1.
__device__ __forceinline__ uint2 row_word2(const uint16_t* row, int c, int g) {
    uint2 v;
    asm volatile("ld.global.nc.L1::no_allocate.v2.u32 {%0, %1}, [%2];"
                 : "=r"(v.x), "=r"(v.y)
                 : "l"(reinterpret_cast<const uint2*>(row) + 2 * c + g));
    return v;
}

template <bool LFS>
__global__ void __launch_bounds__(kHaloAtoms * 2, 4)
k_lj_tile1(const int4* __restrict__ q, const double4* __restrict__ pd, const int* __restrict__ nbr,
           const uint16_t* __restrict__ nbr16, const int* __restrict__ count, int stride, int64_t n,
           const int2* __restrict__ runs, const int2* __restrict__ meta,
           const __grid_constant__ Box3 box, const __grid_constant__ LJArgs a,
           const __grid_constant__ UnitConst uc, double* __restrict__ fxo,
           double* __restrict__ fyo, double* __restrict__ fzo, double* part, unsigned* ticket,
           double* out, uint32_t* status) {
    constexpr int TPA = 2;
    extern __shared__ __align__(128) int4 s_tile[];  // kHaloCap slots
    __shared__ uint64_t s_bar;
    const int tid = threadIdx.x, t = blockIdx.x;
    const int g = tid & 1;
    if (tid == 0) {
        mbar_init(&s_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid < 32) tile_issue(t, s_tile, &s_bar, q, runs, meta, l2_evict_last_policy());
    // the atom's own data and first row word travel while the halo lands
    const int2 m = meta[t];
    const int64_t i = static_cast<int64_t>(t) * kHaloAtoms + (tid >> 1);
    const int ii = static_cast<int>(i);
    int4 pi = make_int4(0, 0, 0, 0);
    int cnt = 0;
    if (i < n) {
        pi = __ldg(q + i);
        cnt = min(count[i], stride);  // an overflowed row is flagged, never over-read
    }
    const uint16_t* row = nbr16 + i * stride;
    const int nch = (i < n && m.x > 0) ? (cnt + 7) >> 3 : 0;
    uint2 word = nch > 0 ? row_word2(row, 0, g) : make_uint2(0u, 0u);
    const bool landed = warp_wait_bounded(&s_bar, 0u);
    double fx = 0.0, fy = 0.0, fz = 0.0;  // grid units in the main loop, then real units
    float e = 0.f, vir = 0.f;
    if (!landed) {
        if ((tid & 31) == 0) atomicOr(status, MD_STATUS_WAIT_TIMEOUT);
    } else if (i < n) {
        const Fold3 f3 = fold3_of(box);
        if (m.x > 0) {
            const char* tile = reinterpret_cast<const char*>(s_tile);
            bool near = false;
            for (int c = 0; c < nch; ++c) {
                const uint2 cur = word;
                if (c + 1 < nch) word = row_word2(row, c + 1, g);
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    const int4 qj = *reinterpret_cast<const int4*>(tile + TileRow<2>::slot(cur, h));
                    pair_unit<LFS>(uc, pi, qj, fx, fy, fz, e, vir, near);
                }
            }
            const double inv_res = 1.0 / a.res[0];
            fx *= inv_res;
            fy *= inv_res;
            fz *= inv_res;
            if (near) {
                // rare: the pairs next to the cutoff, decided by the reference
                // arithmetic on the FP64 positions (the slot maps to its atom
                // through the tile's runs)
                const int2* tr = runs + static_cast<int64_t>(t) * kHaloRuns;
                for (int c = 0; c < nch; ++c) {
                    for (int h = 0; h < 4; ++h) {
                        const int kk = 8 * c + 4 * g + h;
                        if (kk >= cnt) continue;
                        const unsigned off = row[kk];
                        const int sl = static_cast<int>(off >> 4);
                        int lo = 0, hi = m.x;  // the last run whose first slot is <= sl
                        while (hi - lo > 1) {
                            const int mid = (lo + hi) >> 1;
                            if (tr[mid].y <= sl) lo = mid;
                            else hi = mid;
                        }
                        near_pair<LFS>(a, f3, pd, ii, tr[lo].x + (sl - tr[lo].y), pi,
                                       *reinterpret_cast<const int4*>(tile + off), fx, fy, fz, e,
                                       vir);
                    }
                }
            }
        } else {
            // a tile that is not staged: its int32 row, positions gathered
            const int* r32 = nbr + i * stride;
            bool near = false;
            for (int kk = g; kk < cnt; kk += TPA)
                pair_mixed<LFS, true>(a, pi, __ldg(q + __ldg(r32 + kk)), fx, fy, fz, e, vir, near);
            if (near) {
                for (int kk = g; kk < cnt; kk += TPA) {
                    const int j = __ldg(r32 + kk);
                    near_pair<LFS>(a, f3, pd, ii, j, pi, __ldg(q + j), fx, fy, fz, e, vir);
                }
            }
        }
    }
    fx += __shfl_xor_sync(0xffffffffu, fx, 1);
    fy += __shfl_xor_sync(0xffffffffu, fy, 1);
    fz += __shfl_xor_sync(0xffffffffu, fz, 1);
    if (i < n && g == 0) {
        fxo[i] = fx;
        fyo[i] = fy;
        fzo[i] = fz;
    }
    double v[2] = {0.5 * static_cast<double>(e), 0.5 * static_cast<double>(vir)};  // both sides
    grid_reduce<2>(v, part, ticket, out);
}

// Brute force (lennard_jones.cpp:90-97): every atom against every other atom,
// positions staged through shared memory in tiles.
template <bool LFS>
__global__ void __launch_bounds__(kBlock)
k_lj_brute(const double4* __restrict__ pos, int64_t n, Box3 box, LJArgs a, int write_forces,
           double* __restrict__ fxo, double* __restrict__ fyo, double* __restrict__ fzo,
           double* part, unsigned* ticket, double* out) {
    __shared__ double4 tile[kBlock];
    const Fold3 f3 = fold3_of(box);
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    double fx = 0.0, fy = 0.0, fz = 0.0, e = 0.0, vir = 0.0;
    const double4 pi = i < n ? pos[i] : make_double4(0, 0, 0, -1.0);
    for (int64_t base = 0; base < n; base += kBlock) {
        __syncthreads();
        if (base + threadIdx.x < n) tile[threadIdx.x] = pos[base + threadIdx.x];
        __syncthreads();
        const int lim = static_cast<int>(n - base < kBlock ? n - base : kBlock);
        if (i < n) {
            for (int t = 0; t < lim; ++t) {
                if (base + t == i) continue;
                accumulate_exact<LFS>(a, f3, pi, tile[t], fx, fy, fz, e, vir);
            }
        }
    }
    if (i < n && write_forces) {
        fxo[i] = fx;
        fyo[i] = fy;
        fzo[i] = fz;
    }
    double v[2] = {e, vir};
    grid_reduce<2>(v, part, ticket, out);
}

// CellList source (lennard_jones.cpp:99-114): for every atom, the atoms of the 27
// cells around the cell it was binned into at build time.
struct CellArgs {
    int nx, ny, nz, ncells;
    const int* rank_of_cell;
    const int* cell_of_rank;
    const int* start;
    const int* sorted_orig;
    const int* slot;
};

template <bool LFS>
__global__ void __launch_bounds__(kBlock)
k_lj_cells(const double4* __restrict__ pos, int64_t n, Box3 box, LJArgs a, CellArgs c,
           double* __restrict__ fxo, double* __restrict__ fyo, double* __restrict__ fzo,
           double* part, unsigned* ticket, double* out) {
    const int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const Fold3 f3 = fold3_of(box);
    double fx = 0.0, fy = 0.0, fz = 0.0, e = 0.0, vir = 0.0;
    if (s < n) {
        // rank of sorted position s: binary search in start[]
        int lo = 0, hi = c.ncells;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (c.start[mid] <= s) lo = mid;
            else hi = mid;
        }
        const int cell = c.cell_of_rank[lo];
        const int i = c.slot[c.sorted_orig[s]];
        const double4 pi = pos[i];
        const int cx = cell % c.nx, cy = (cell / c.nx) % c.ny, cz = cell / (c.nx * c.ny);
        for (int q = 0; q < 27; ++q) {
            int jx = cx + (q % 3) - 1, jy = cy + ((q / 3) % 3) - 1, jz = cz + (q / 9) - 1;
            jx = jx < 0 ? jx + c.nx : (jx >= c.nx ? jx - c.nx : jx);
            jy = jy < 0 ? jy + c.ny : (jy >= c.ny ? jy - c.ny : jy);
            jz = jz < 0 ? jz + c.nz : (jz >= c.nz ? jz - c.nz : jz);
            const int rr = c.rank_of_cell[jx + c.nx * (jy + c.ny * jz)];
            for (int t = c.start[rr]; t < c.start[rr + 1]; ++t) {
                if (t == s) continue;
                const int j = c.slot[c.sorted_orig[t]];
                accumulate_exact<LFS>(a, f3, pi, pos[j], fx, fy, fz, e, vir);
            }
        }
        fxo[i] = fx;
        fyo[i] = fy;
        fzo[i] = fz;
    }
    double v[2] = {e, vir};
    grid_reduce<2>(v, part, ticket, out);
}

Box3 box_of(const md_system* sys) {
    Box3 b;
    for (int d = 0; d < 3; ++d) {
        b.L[d] = sys->box[d];
        b.inv[d] = sys->inv_box[d];
    }
    return b;
}

template <int TPA, bool MIXED, bool LFS, int U>
bool launch_verlet(md_system* sys, md_verlet* v, const LJArgs& a, double* part, unsigned* ticket,
                   double* out, const KickArgs* kick) {
    const int64_t threads = sys->n * TPA;
    const typename PosOf<MIXED>::T* pos;
    if constexpr (MIXED) pos = sys->qpos.as<int4>();
    else pos = sys->cur.pos;
    const bool cubic = MIXED && a.res[0] == a.res[1] && a.res[0] == a.res[2];
    auto kernel = cubic ? k_lj_verlet<TPA, MIXED, LFS, U, MIXED, false>
                        : k_lj_verlet<TPA, MIXED, LFS, U, false, false>;
    bool kicks = false;
    if constexpr (verlet_kicks(TPA, U)) {
        if (kick) {
            kernel = cubic ? k_lj_verlet<TPA, MIXED, LFS, U, MIXED, true>
                           : k_lj_verlet<TPA, MIXED, LFS, U, false, true>;
            kicks = true;
        }
    }
    kernel<<<grid_for(threads, kBlock), kBlock, 0, sys->ctx->stream>>>(
        pos, sys->cur.pos, v->nbr.as<int>(), v->count.as<int>(), v->stride, sys->n, box_of(sys), a,
        sys->cur.fx, sys->cur.fy, sys->cur.fz, part, ticket, out, kicks ? *kick : KickArgs{});
    return kicks;
}

// Fixed-point positions for the mixed pair kernels (quantize_position), skipped
// when `flag` is given and zero: the step's kick/drift already wrote them and no
// rebuild re-sorted the atoms since.
__global__ void k_quantize(const double4* __restrict__ pos, int64_t n, double sx, double sy,
                           double sz, int4* __restrict__ q, const int* flag) {
    if (flag && *flag == 0) return;
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= n) return;
    q[k] = quantize_position(pos[k], sx, sy, sz);
}

template <bool LFS, int U>
void launch_halo(md_system* sys, md_verlet* v, const LJArgs& a, double* part, unsigned* ticket,
                 double* out, const KickArgs* kick) {
    const unsigned blocks = static_cast<unsigned>(halo_blocks(sys->n));
    const bool cubic = a.res[0] == a.res[1] && a.res[0] == a.res[2];
    auto kernel = kick ? (cubic ? k_lj_halo<LFS, U, true, true> : k_lj_halo<LFS, U, false, true>)
                       : (cubic ? k_lj_halo<LFS, U, true, false> : k_lj_halo<LFS, U, false, false>);
    kernel<<<blocks, kBlock, kHaloCap * sizeof(int4), sys->ctx->stream>>>(
        sys->qpos.as<int4>(), sys->cur.pos, v->nbr.as<int>(), v->nbr16.as<uint16_t>(),
        v->count.as<int>(), v->stride, sys->n, v->halo_runs.as<int2>(), v->halo_meta.as<int2>(),
        box_of(sys), a, sys->cur.fx, sys->cur.fy, sys->cur.fz, part, ticket, out,
        kick ? *kick : KickArgs{});
}

UnitConst unit_const(const LJArgs& a) {
    UnitConst c;
    const double res2 = a.res2;
    c.lo = a.rc2_lo / res2;
    c.hi = a.rc2_hi / res2;
    c.sig2u = static_cast<float>(a.sig2 / res2);
    c.four_epsf = a.four_epsf;
    c.tf_epsf = a.tf_epsf;
    c.ucf = a.ucf;
    c.rcf = a.rcf;
    c.dudrcf = a.dudrcf;
    c.res_f = static_cast<float>(a.res[0]);
    return c;
}

template <bool LFS>
void launch_tile1(md_system* sys, md_verlet* v, const LJArgs& a, double* part, unsigned* ticket,
                  double* out) {
    const unsigned blocks = static_cast<unsigned>(halo_blocks(sys->n));
    const size_t smem = kHaloCap * sizeof(int4);
    k_lj_tile1<LFS><<<blocks, kHaloAtoms * 2, smem, sys->ctx->stream>>>(
        sys->qpos.as<int4>(), sys->cur.pos, v->nbr.as<int>(), v->nbr16.as<uint16_t>(),
        v->count.as<int>(), v->stride, sys->n, v->halo_runs.as<int2>(), v->halo_meta.as<int2>(),
        box_of(sys), a, unit_const(a), sys->cur.fx, sys->cur.fy, sys->cur.fz, part, ticket, out,
        sys->ctx->d_status);
}

template <bool LFS, int TPA>
void launch_tile_k(md_system* sys, md_verlet* v, const LJArgs& a, double* part,
                   unsigned* ticket, double* out) {
    const int ntiles = static_cast<int>(halo_blocks(sys->n));
    auto kernel = k_lj_tile<LFS, TPA>;
    const size_t smem = 2 * kHaloCap * sizeof(int4);
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem));
        attr_set = true;
    }
    const int per_sm = TPA == 8 ? 1 : 2;
    const int grid = std::max(1, std::min(ntiles, per_sm * sys->ctx->sm_count));
    kernel<<<grid, kHaloAtoms * TPA, smem, sys->ctx->stream>>>(
        sys->qpos.as<int4>(), sys->cur.pos, v->nbr.as<int>(), v->nbr16.as<uint16_t>(),
        v->count.as<int>(), v->stride, sys->n, ntiles, v->halo_runs.as<int2>(),
        v->halo_meta.as<int2>(), box_of(sys), a, sys->cur.fx, sys->cur.fy, sys->cur.fz, part,
        ticket, out, sys->ctx->d_status);
}

// tpa: threads per atom of the tile kernel (the tile shape: 2, 4 or 8; 0 = the
// default, 2).
template <bool LFS>
void launch_tile(int tpa, md_system* sys, md_verlet* v, const LJArgs& a, double* part,
                 unsigned* ticket, double* out) {
    switch (tpa) {
        case 4: launch_tile_k<LFS, 4>(sys, v, a, part, ticket, out); break;
        case 8: launch_tile_k<LFS, 8>(sys, v, a, part, ticket, out); break;
        default: launch_tile_k<LFS, 2>(sys, v, a, part, ticket, out); break;
    }
}

template <bool LFS>
void launch_halo_u(int unroll, md_system* sys, md_verlet* v, const LJArgs& a, double* part,
                   unsigned* ticket, double* out, const KickArgs* kick) {
    switch (unroll) {
        case 1: launch_halo<LFS, 1>(sys, v, a, part, ticket, out, kick); break;
        case 4: launch_halo<LFS, 4>(sys, v, a, part, ticket, out, kick); break;
        default: launch_halo<LFS, 2>(sys, v, a, part, ticket, out, kick); break;
    }
}

template <int TPA, bool MIXED, bool LFS>
bool launch_verlet_u(int unroll, md_system* sys, md_verlet* v, const LJArgs& a, double* part,
                     unsigned* ticket, double* out, const KickArgs* kick) {
    switch (unroll) {
        case 1: return launch_verlet<TPA, MIXED, LFS, 1>(sys, v, a, part, ticket, out, kick);
        case 4: return launch_verlet<TPA, MIXED, LFS, 4>(sys, v, a, part, ticket, out, kick);
        default: return launch_verlet<TPA, MIXED, LFS, 2>(sys, v, a, part, ticket, out, kick);
    }
}

template <bool MIXED, bool LFS>
bool launch_verlet_tpa(int tpa, int unroll, md_system* sys, md_verlet* v, const LJArgs& a,
                       double* part, unsigned* ticket, double* out, const KickArgs* kick) {
    switch (tpa) {
        case 1: return launch_verlet_u<1, MIXED, LFS>(unroll, sys, v, a, part, ticket, out, kick);
        case 4: return launch_verlet_u<4, MIXED, LFS>(unroll, sys, v, a, part, ticket, out, kick);
        case 8: return launch_verlet_u<8, MIXED, LFS>(unroll, sys, v, a, part, ticket, out, kick);
        default: return launch_verlet_u<2, MIXED, LFS>(unroll, sys, v, a, part, ticket, out, kick);
    }
}

}  // namespace

int g_lj_tpa = 2;     // threads per atom of the Verlet force kernel (tunable)
int g_lj_unroll = 2;  // independent gather chains per thread (tunable)

namespace {

// The pair-kernel arguments of one system: the potential plus the fixed-point
// resolution and the exact band of the mixed path (box-dependent).
LJArgs verlet_lj_args(const md_lj* lj, const md_system* sys) {
    LJArgs a = make_lj_args(lj);
    double res_max = 0.0;
    for (int d = 0; d < 3; ++d) {
        a.res[d] = sys->box[d] / 4294967296.0;
        res_max = std::max(res_max, a.res[d]);
    }
    // |r^2 error| <= 2 r |d error| + rounding, |d error| <= sqrt(3) res: 4x margin
    a.band = 8.0 * 1.7320508075688772 * a.rc * res_max + 1e-12 * a.rc2;
    a.res2 = a.res[0] * a.res[0];
    a.rc2_lo = a.rc2 - a.band;
    a.rc2_hi = a.rc2 + a.band;
    return a;
}

}  // namespace

int lj_quantize_async(md_lj* lj, md_system* sys, const int* gate) {
    if (lj->precision != MD_PRECISION_MIXED || sys->n == 0) return MD_OK;
    md_context* ctx = sys->ctx;
    MDB_TRY(sys->qpos.ensure(sizeof(int4) * static_cast<size_t>(sys->n)));
    const double two32 = 4294967296.0;
    k_quantize<<<grid_for(sys->n, kBlock), kBlock, 0, ctx->stream>>>(
        sys->cur.pos, sys->n, two32 / sys->box[0], two32 / sys->box[1], two32 / sys->box[2],
        sys->qpos.as<int4>(), gate);
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

int lj_forces_verlet_async(md_lj* lj, md_system* sys, md_verlet* v, const int* q_gate,
                           bool q_current, const KickArgs* kick, bool* kicked) {
    if (kicked) *kicked = false;
    md_context* ctx = sys->ctx;
    const LJArgs a = verlet_lj_args(lj, sys);
    const int tpa = lj->tpa ? lj->tpa : g_lj_tpa, unroll = lj->unroll ? lj->unroll : g_lj_unroll;
    const int64_t threads = std::max<int64_t>(sys->n * tpa, 1);
    const int64_t blocks = std::max<int64_t>(grid_for(threads, kBlock), halo_blocks(sys->n));
    double* part;
    MDB_TRY(ctx_partials(ctx, 3 * static_cast<size_t>(blocks), &part));
    unsigned* ticket = ctx_counter(ctx, 2);
    double* out = ctx_result(ctx, kResEnergy);
    const bool lfs = lj->truncation == MD_LINEAR_FORCE_SHIFT;
    const bool mixed = lj->precision == MD_PRECISION_MIXED;
    if (!q_current) MDB_TRY(lj_quantize_async(lj, sys, q_gate));
    // halo tiles, when the list keeps them (fused runs of large systems turn them on,
    // or md_verlet_set_halo)
    const bool halo = mixed && lj->halo && sys->n > 0 && v->halo_on && v->stride % 8 == 0;
    ctx_time_begin(ctx, MD_KERNEL_LJ_FORCE);
    const bool cubic = a.res[0] == a.res[1] && a.res[0] == a.res[2];
    if (halo && cubic && lj->tile_tpa > 1) {
        if (lfs) launch_tile<true>(lj->tile_tpa, sys, v, a, part, ticket, out);
        else launch_tile<false>(lj->tile_tpa, sys, v, a, part, ticket, out);
    } else if (halo && cubic && lj->tile_tpa == 1) {
        if (lfs) launch_tile1<true>(sys, v, a, part, ticket, out);
        else launch_tile1<false>(sys, v, a, part, ticket, out);
    } else if (halo) {
        // the default halo kernel also takes the closing half-kick when asked
        if (lfs) launch_halo_u<true>(unroll, sys, v, a, part, ticket, out, kick);
        else launch_halo_u<false>(unroll, sys, v, a, part, ticket, out, kick);
        if (kick && kicked) *kicked = true;
    } else {
        // the default gathered shape also takes the closing half-kick when asked
        bool k;
        if (mixed) {
            k = lfs ? launch_verlet_tpa<true, true>(tpa, unroll, sys, v, a, part, ticket, out, kick)
                    : launch_verlet_tpa<true, false>(tpa, unroll, sys, v, a, part, ticket, out, kick);
        } else {
            k = lfs ? launch_verlet_tpa<false, true>(tpa, unroll, sys, v, a, part, ticket, out, kick)
                    : launch_verlet_tpa<false, false>(tpa, unroll, sys, v, a, part, ticket, out, kick);
        }
        if (k && kicked) *kicked = true;
    }
    ctx_time_end(ctx, MD_KERNEL_LJ_FORCE);
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

struct BatchForce {
    DevBuf reps, blk;  // blk: the launch's block table (block_table)
    int nrep = 0, total = 0, tpa = 2;
    bool mixed = false, lfs = false, cubic = false;
    bool kick = false;  // the kernel takes each replica's closing half-kick
};

int batch_force_create(const BatchRepView* v, int nrep, const KickArgs* kicks, BatchForce** out) {
    if (nrep < 1) return fail(MD_ERR_INVALID_ARGUMENT, "batch_force_create: no replicas");
    const md_lj* l0 = v[0].lj;
    const int tpa0 = l0->tpa ? l0->tpa : g_lj_tpa, unroll0 = l0->unroll ? l0->unroll : g_lj_unroll;
    std::vector<BatchForceRep> h(static_cast<size_t>(nrep));
    std::vector<int> off(static_cast<size_t>(nrep) + 1, 0);
    bool cubic = true, any_cubic = false;
    for (int r = 0; r < nrep; ++r) {
        md_lj* lj = v[r].lj;
        md_system* sys = v[r].sys;
        md_verlet* list = v[r].list;
        const int tpa = lj->tpa ? lj->tpa : g_lj_tpa, unroll = lj->unroll ? lj->unroll : g_lj_unroll;
        const bool mixed = lj->precision == MD_PRECISION_MIXED;
        if (lj->precision != l0->precision || lj->truncation != l0->truncation || tpa != tpa0 ||
            unroll != unroll0 || unroll != 2 || (tpa != 1 && tpa != 2 && tpa != 4 && tpa != 8) ||
            (mixed && lj->halo && list->halo_on))
            return fail(MD_ERR_INVALID_ARGUMENT, "batch_force_create: force kernels differ");
        md_context* ctx = sys->ctx;
        const LJArgs a = verlet_lj_args(lj, sys);
        const bool c = a.res[0] == a.res[1] && a.res[0] == a.res[2];
        cubic = cubic && c;
        any_cubic = any_cubic || c;
        const int64_t blocks = grid_for(std::max<int64_t>(sys->n * tpa, 1), kBlock);
        double* part;
        MDB_TRY(ctx_partials(ctx, 3 * static_cast<size_t>(blocks), &part));
        if (mixed) MDB_TRY(sys->qpos.ensure(sizeof(int4) * static_cast<size_t>(sys->n)));
        BatchForceRep& d = h[static_cast<size_t>(r)];
        d.pos = mixed ? static_cast<const void*>(sys->qpos.as<int4>())
                      : static_cast<const void*>(sys->cur.pos);
        d.pd = sys->cur.pos;
        d.nbr = list->nbr.as<int>();
        d.count = list->count.as<int>();
        d.stride = list->stride;
        d.n = sys->n;
        d.box = box_of(sys);
        d.a = a;
        d.fx = sys->cur.fx;
        d.fy = sys->cur.fy;
        d.fz = sys->cur.fz;
        d.part = part;
        d.ticket = ctx_counter(ctx, 2);
        d.out = ctx_result(ctx, kResEnergy);
        d.kick = kicks ? kicks[r] : KickArgs{};
        off[static_cast<size_t>(r) + 1] = off[static_cast<size_t>(r)] + static_cast<int>(blocks);
    }
    // the mixed kernel specialises on a cubic box: one specialisation for all
    if (l0->precision == MD_PRECISION_MIXED && any_cubic && !cubic)
        return fail(MD_ERR_INVALID_ARGUMENT, "batch_force_create: cubic and non-cubic boxes mixed");
    BatchForce* b = new (std::nothrow) BatchForce();
    if (!b) return fail(MD_ERR_OUT_OF_MEMORY, "batch_force_create: host allocation");
    b->nrep = nrep;
    b->total = off.back();
    b->tpa = tpa0;
    b->mixed = l0->precision == MD_PRECISION_MIXED;
    b->lfs = l0->truncation == MD_LINEAR_FORCE_SHIFT;
    b->cubic = b->mixed && cubic;
    b->kick = kicks && verlet_kicks(tpa0, unroll0);  // as each replica's solo pass
    const std::vector<int4> t = block_table(off.data(), nrep);
    int rc = b->reps.ensure(sizeof(BatchForceRep) * h.size());
    if (rc == MD_OK) rc = b->blk.ensure(sizeof(int4) * t.size());
    if (rc == MD_OK &&
        (cudaMemcpy(b->reps.ptr, h.data(), sizeof(BatchForceRep) * h.size(), cudaMemcpyHostToDevice) !=
             cudaSuccess ||
         cudaMemcpy(b->blk.ptr, t.data(), sizeof(int4) * t.size(), cudaMemcpyHostToDevice) !=
             cudaSuccess))
        rc = fail(MD_ERR_CUDA, "batch_force_create: descriptor upload");
    if (rc != MD_OK) {
        batch_force_destroy(b);
        return rc;
    }
    *out = b;
    return MD_OK;
}

namespace {

template <int TPA, bool MIXED, bool LFS, bool CUBIC>
void batch_force_t(BatchForce* b, cudaStream_t s) {
    auto kernel = k_lj_verlet_batch<TPA, MIXED, LFS, 2, CUBIC, false>;
    if constexpr (verlet_kicks(TPA, 2))
        if (b->kick) kernel = k_lj_verlet_batch<TPA, MIXED, LFS, 2, CUBIC, true>;
    kernel<<<b->total, kBlock, 0, s>>>(b->reps.as<BatchForceRep>(), b->blk.as<int4>());
}

template <int TPA>
void batch_force_tpa(BatchForce* b, cudaStream_t s) {
    if (b->mixed) {
        if (b->lfs) b->cubic ? batch_force_t<TPA, true, true, true>(b, s) : batch_force_t<TPA, true, true, false>(b, s);
        else b->cubic ? batch_force_t<TPA, true, false, true>(b, s) : batch_force_t<TPA, true, false, false>(b, s);
    } else {
        if (b->lfs) batch_force_t<TPA, false, true, false>(b, s);
        else batch_force_t<TPA, false, false, false>(b, s);
    }
}

}  // namespace

int batch_force_launch(BatchForce* b, cudaStream_t s, int64_t* launches) {
    switch (b->tpa) {
        case 1: batch_force_tpa<1>(b, s); break;
        case 4: batch_force_tpa<4>(b, s); break;
        case 8: batch_force_tpa<8>(b, s); break;
        default: batch_force_tpa<2>(b, s); break;
    }
    if (launches) ++*launches;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

bool batch_force_kicks(const BatchForce* b) { return b && b->kick; }

void batch_force_destroy(BatchForce* b) {
    if (!b) return;
    b->reps.release();
    b->blk.release();
    delete b;
}

int lj_forces_brute_async(md_lj* lj, md_system* sys, bool forces) {
    md_context* ctx = sys->ctx;
    const LJArgs a = make_lj_args(lj);
    const int blocks = grid_for(std::max<int64_t>(sys->n, 1), kBlock);
    double* part;
    MDB_TRY(ctx_partials(ctx, 2 * static_cast<size_t>(blocks), &part));
    if (lj->truncation == MD_LINEAR_FORCE_SHIFT)
        k_lj_brute<true><<<blocks, kBlock, 0, ctx->stream>>>(
            sys->cur.pos, sys->n, box_of(sys), a, forces ? 1 : 0, sys->cur.fx, sys->cur.fy,
            sys->cur.fz, part, ctx_counter(ctx, 2), ctx_result(ctx, kResEnergy));
    else
        k_lj_brute<false><<<blocks, kBlock, 0, ctx->stream>>>(
            sys->cur.pos, sys->n, box_of(sys), a, forces ? 1 : 0, sys->cur.fx, sys->cur.fy,
            sys->cur.fz, part, ctx_counter(ctx, 2), ctx_result(ctx, kResEnergy));
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

int lj_forces_cells_async(md_lj* lj, md_system* sys, md_cells* cells) {
    md_context* ctx = sys->ctx;
    const LJArgs a = make_lj_args(lj);
    const int blocks = grid_for(std::max<int64_t>(sys->n, 1), kBlock);
    double* part;
    MDB_TRY(ctx_partials(ctx, 2 * static_cast<size_t>(blocks), &part));
    CellArgs c;
    c.nx = cells->grid.nx;
    c.ny = cells->grid.ny;
    c.nz = cells->grid.nz;
    c.ncells = cells->grid.ncells;
    c.rank_of_cell = cells->grid.rank_of_cell;
    c.cell_of_rank = cells->grid.cell_of_rank;
    c.start = cells->start.as<int>();
    c.sorted_orig = cells->sorted_orig.as<int>();
    c.slot = sys->slot;
    if (lj->truncation == MD_LINEAR_FORCE_SHIFT)
        k_lj_cells<true><<<blocks, kBlock, 0, ctx->stream>>>(
            sys->cur.pos, sys->n, box_of(sys), a, c, sys->cur.fx, sys->cur.fy, sys->cur.fz, part,
            ctx_counter(ctx, 2), ctx_result(ctx, kResEnergy));
    else
        k_lj_cells<false><<<blocks, kBlock, 0, ctx->stream>>>(
            sys->cur.pos, sys->n, box_of(sys), a, c, sys->cur.fx, sys->cur.fy, sys->cur.fz, part,
            ctx_counter(ctx, 2), ctx_result(ctx, kResEnergy));
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

}  // namespace mdb

using namespace mdb;

namespace {
int finish_energy(md_system* sys, double* energy, double* virial) {
    double r[2];
    MDB_TRY(ctx_read_results(sys->ctx, kResEnergy, 2, r));
    sys->last_energy = r[0];
    sys->last_virial = r[1];
    if (energy) *energy = r[0];
    if (virial) *virial = r[1];
    return MD_OK;
}
}  // namespace

extern "C" {

int md_lj_create(double sigma, double epsilon, double cutoff, int truncation, int precision,
                 md_lj** out) {
    graph_epoch_bump();
    if (!out) return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_create: out is NULL");
    if (truncation != MD_TRUNCATED && truncation != MD_LINEAR_FORCE_SHIFT)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_create: unknown truncation %d", truncation);
    if (precision != MD_PRECISION_FP64 && precision != MD_PRECISION_MIXED)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_create: unknown precision %d", precision);
    md_lj* lj = new (std::nothrow) md_lj();
    if (!lj) return fail(MD_ERR_OUT_OF_MEMORY, "md_lj_create: host allocation");
    lj->sigma = sigma;
    lj->epsilon = epsilon;
    lj->cutoff = cutoff;
    lj->truncation = truncation;
    lj->precision = precision;
    // lennard_jones.cpp:32-48
    const double sig2 = sigma * sigma;
    const double rc2 = cutoff * cutoff;
    const double s2 = sig2 / rc2;
    const double s6 = s2 * s2 * s2;
    lj->u_at_cutoff = 4.0 * epsilon * (s6 * s6 - s6);
    const double w_at_cutoff = 24.0 * epsilon * (2.0 * s6 * s6 - s6);
    lj->dudr_at_cutoff = -w_at_cutoff / cutoff;
    *out = lj;
    return MD_OK;
}

int md_lj_destroy(md_lj* lj) {
    graph_epoch_bump();
    delete lj;
    return MD_OK;
}

int md_lj_energy_virial(md_lj* lj, md_system* sys, double* energy, double* virial) {
    if (!lj || !sys) return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_energy_virial: NULL argument");
    MDB_TRY(lj_forces_brute_async(lj, sys, false));
    return finish_energy(sys, energy, virial);
}

int md_lj_forces(md_lj* lj, md_system* sys, double* energy, double* virial) {
    if (!lj || !sys) return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_forces: NULL argument");
    MDB_TRY(lj_forces_brute_async(lj, sys, true));
    return finish_energy(sys, energy, virial);
}

int md_lj_forces_cells(md_lj* lj, md_system* sys, md_cells* cells, double* energy,
                       double* virial) {
    if (!lj || !sys || !cells) return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_forces_cells: NULL argument");
    // lennard_jones.cpp:107-111
    if (!cells->grid.usable)
        return fail(MD_ERR_INVALID_ARGUMENT,
                    "LennardJones::computeForces: CellList is not usable (fewer than 3 cells per "
                    "side); fall back to the brute-force overload");
    if (!cells->built || cells->sys != sys || cells->n != sys->n)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_forces_cells: cell list not built for this system");
    MDB_TRY(lj_forces_cells_async(lj, sys, cells));
    return finish_energy(sys, energy, virial);
}

int md_lj_forces_verlet(md_lj* lj, md_system* sys, md_verlet* list, double* energy,
                        double* virial) {
    if (!lj || !sys || !list) return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_forces_verlet: NULL argument");
    MDB_TRY(verlet_ensure_ready(list, sys, "md_lj_forces_verlet"));
    MDB_TRY(lj_forces_verlet_async(lj, sys, list));
    return finish_energy(sys, energy, virial);
}

int md_lj_lrc(const md_lj* lj, int64_t n, const double box[3], double* u_lrc, double* p_lrc) {
    if (!lj || !box) return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_lrc: NULL argument");
    // lennard_jones.cpp:121-151 (host scalars, O(1))
    const double kPi = 3.14159265358979323846;
    if (lj->truncation == MD_LINEAR_FORCE_SHIFT) {
        if (u_lrc) *u_lrc = 0.0;
        if (p_lrc) *p_lrc = 0.0;
        return MD_OK;
    }
    const double nd = static_cast<double>(n);
    const double rho = nd / (box[0] * box[1] * box[2]);
    const double sr = lj->sigma / lj->cutoff;
    const double sr3 = sr * sr * sr;
    const double sr9 = sr3 * sr3 * sr3;
    const double sig3 = lj->sigma * lj->sigma * lj->sigma;
    if (u_lrc) *u_lrc = (8.0 / 3.0) * kPi * nd * rho * lj->epsilon * sig3 * ((1.0 / 3.0) * sr9 - sr3);
    if (p_lrc)
        *p_lrc = (16.0 / 3.0) * kPi * rho * rho * lj->epsilon * sig3 * ((2.0 / 3.0) * sr9 - sr3);
    return MD_OK;
}

// Threads per atom of the Verlet force kernel (1, 2, 4 or 8); autotuning hook.
int md_lj_set_threads_per_atom(int tpa) {
    graph_epoch_bump();
    if (tpa != 1 && tpa != 2 && tpa != 4 && tpa != 8)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_set_threads_per_atom: %d not in {1,2,4,8}", tpa);
    g_lj_tpa = tpa;
    return MD_OK;
}

// Launch shape of one LJ object's Verlet force kernel (0 = the library default).
int md_lj_set_launch(md_lj* lj, int tpa, int unroll) {
    graph_epoch_bump();
    if (!lj) return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_set_launch: NULL");
    if (tpa != 0 && tpa != 1 && tpa != 2 && tpa != 4 && tpa != 8)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_set_launch: tpa %d not in {0,1,2,4,8}", tpa);
    if (unroll != 0 && unroll != 1 && unroll != 2 && unroll != 4)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_set_launch: unroll %d not in {0,1,2,4}", unroll);
    lj->tpa = tpa;
    lj->unroll = unroll;
    return MD_OK;
}

int md_lj_set_tile_threads(md_lj* lj, int tpa) {
    graph_epoch_bump();
    if (!lj || (tpa != 0 && tpa != 1 && tpa != 2 && tpa != 4 && tpa != 8))
        return fail(MD_ERR_INVALID_ARGUMENT,
                    "md_lj_set_tile_threads: threads per atom must be 0, 1, 2, 4 or 8");
    lj->tile_tpa = tpa;
    return MD_OK;
}

int md_lj_set_halo(md_lj* lj, int on) {
    graph_epoch_bump();
    if (!lj) return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_set_halo: NULL");
    lj->halo = on != 0;
    return MD_OK;
}

// Independent neighbour gathers in flight per thread (1, 2 or 4); autotuning hook.
int md_lj_set_unroll(int unroll) {
    graph_epoch_bump();
    if (unroll != 1 && unroll != 2 && unroll != 4)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_set_unroll: %d not in {1,2,4}", unroll);
    g_lj_unroll = unroll;
    return MD_OK;
}

}  // extern "C"
