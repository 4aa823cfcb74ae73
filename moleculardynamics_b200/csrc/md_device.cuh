// md_device.cuh -- device helpers shared by the kernels.
//
// Exact-arithmetic helpers: the FP64 drop-in path must reproduce the reference's
// pair membership bit-for-bit, so every operation that decides whether a pair is
// inside a cutoff is written with explicit round-to-nearest intrinsics (__dmul_rn,
// __dadd_rn, __dsub_rn, __ddiv_rn), which the compiler may not contract into FMAs.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/moldyn_b200.h"

namespace mdb {

// core/box.cpp:12-15: value - L * floor(value / L + 0.5), bit-exact.
// value/L is first approximated by value * (1/L); only when that lands within
// 1e-9 of a rounding boundary of floor(. + 0.5) -- where the one-ulp difference
// between value*(1/L) and value/L could matter -- is the IEEE division used.
__device__ __forceinline__ double fold_exact(double v, double L, double invL) {
    const double s = __dadd_rn(__dmul_rn(v, invL), 0.5);
    double k = floor(s);
    const double frac = __dsub_rn(s, k);
    if (frac < 1e-9 || frac > 1.0 - 1e-9) k = floor(__dadd_rn(__ddiv_rn(v, L), 0.5));
    return __dsub_rn(v, __dmul_rn(L, k));
}

// fold_exact for a difference of two wrapped coordinates (|v| < 1.5 L), with
// the floor replaced by comparisons wherever they provably agree with it:
// floor(v/L + 0.5) is 0 for |v| <= 0.5 L (1 - 2^-40) and sign(v) for
// 0.5 L (1 + 2^-40) <= |v| <= 1.5 L (1 - 2^-40), whatever the rounding of v/L;
// v - L*k with k = +-1 is then v -+ L with the same single rounding.  Only
// values within 2^-41 L of +-L/2 (or beyond) take the reference path.
struct FoldBounds {
    double L, invL, lo, hi, top;
};

__host__ __device__ inline FoldBounds fold_bounds(double L, double invL) {
    const double e = 9.094947017729282e-13;  // 2^-40
    return FoldBounds{L, invL, 0.5 * L * (1.0 - e), 0.5 * L * (1.0 + e), 1.5 * L * (1.0 - e)};
}

__device__ __forceinline__ double fold_wrapped(double v, const FoldBounds& b) {
    const double a = fabs(v);
    if (a <= b.lo) return v;
    if (a >= b.hi && a <= b.top) return v > 0.0 ? __dsub_rn(v, b.L) : __dadd_rn(v, b.L);
    return fold_exact(v, b.L, b.invL);
}

// core/vec3.hpp:59-65: x*x + y*y + z*z, left to right, no contraction.
__device__ __forceinline__ double norm2_exact(double x, double y, double z) {
    return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

struct Box3 {
    double L[3];
    double inv[3];
};

struct Fold3 {
    FoldBounds b[3];
};

__host__ __device__ inline Fold3 fold3_of(const Box3& box) {
    return Fold3{{fold_bounds(box.L[0], box.inv[0]), fold_bounds(box.L[1], box.inv[1]),
                  fold_bounds(box.L[2], box.inv[2])}};
}

// Minimum-image displacement r_a - r_b (reference arithmetic) for wrapped positions.
__device__ __forceinline__ void min_image_wrapped(const Fold3& f, double ax, double ay,
                                                  double az, double bx, double by, double bz,
                                                  double& dx, double& dy, double& dz) {
    dx = fold_wrapped(__dsub_rn(ax, bx), f.b[0]);
    dy = fold_wrapped(__dsub_rn(ay, by), f.b[1]);
    dz = fold_wrapped(__dsub_rn(az, bz), f.b[2]);
}

// Minimum-image displacement r_a - r_b with the reference's operation order.
__device__ __forceinline__ void min_image_exact(const Box3& b, double ax, double ay, double az,
                                                double bx, double by, double bz, double& dx,
                                                double& dy, double& dz) {
    dx = fold_exact(__dsub_rn(ax, bx), b.L[0], b.inv[0]);
    dy = fold_exact(__dsub_rn(ay, by), b.L[1], b.inv[1]);
    dz = fold_exact(__dsub_rn(az, bz), b.L[2], b.inv[2]);
}

// Read-only 32-byte load through the non-coherent path (two 16-byte loads).
__device__ __forceinline__ double4 ldg4(const double4* p) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

// ----------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Fixed-point position for the mixed pair kernels: q = round(x 2^32 / L) taken
// modulo 2^32 (so unwrapped coordinates land on their periodic image), w = the
// original index.
__device__ __forceinline__ int4 quantize_position(const double4& p, double sx, double sy,
                                                  double sz) {
    return make_int4(static_cast<int>(static_cast<unsigned>(llrint(p.x * sx))),
                     static_cast<int>(static_cast<unsigned>(llrint(p.y * sy))),
                     static_cast<int>(static_cast<unsigned>(llrint(p.z * sz))),
                     static_cast<int>(p.w));
}

// Deterministic grid reduction of K doubles per thread.  Each block reduces its
// values with a fixed shuffle tree and writes part[block*K + k]; the last block
// to arrive (atomic ticket) re-reduces all partials in block order and writes
// out[k], then resets the ticket.  With `status`, a non-finite sum (an atom that
// blew up) also sets MD_STATUS_NONFINITE there.  Must be called by every thread
// of the block; blockDim.x must be a multiple of 32 and <= 1024.  Returns true in
// the last block.  The block index and count are explicit: a batched launch that
// runs many systems gives each system's blocks their own rank and count.
template <int K>
__device__ bool grid_reduce_at(double (&v)[K], double* part, unsigned* ticket, double* out,
                               uint32_t* status, unsigned block, unsigned nblocks) {
    __shared__ double sm[K][32];
    __shared__ bool is_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const double s = warp_sum(v[k]);
        if (lane == 0) sm[k][warp] = s;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double s = lane < nw ? sm[k][lane] : 0.0;
            s = warp_sum(s);
            if (lane == 0) part[static_cast<size_t>(block) * K + k] = s;
        }
    }
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned t = atomicAdd(ticket, 1u);
        is_last = (t == nblocks - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    for (unsigned b = threadIdx.x; b < nblocks; b += blockDim.x) {
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] += __ldcg(part + static_cast<size_t>(b) * K + k);
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const double s = warp_sum(acc[k]);
        if (lane == 0) sm[k][warp] = s;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double s = lane < nw ? sm[k][lane] : 0.0;
            s = warp_sum(s);
            if (lane == 0) {
                out[k] = s;
                if (status && !isfinite(s)) atomicOr(status, MD_STATUS_NONFINITE);
            }
        }
    }
    if (threadIdx.x == 0) *ticket = 0u;
    return true;  // this was the last block: `out` holds the sums
}

template <int K>
__device__ bool grid_reduce(double (&v)[K], double* part, unsigned* ticket, double* out,
                            uint32_t* status = nullptr) {
    return grid_reduce_at<K>(v, part, ticket, out, status, blockIdx.x, gridDim.x);
}

// Top-2 of a multiset (verlet_list.cpp:44-63): (a1 >= a2), merge with (b1 >= b2).
__device__ __forceinline__ void top2_merge(double& a1, double& a2, double b1, double b2) {
    if (b1 > a1) {
        a2 = fmax(a1, b2);
        a1 = b1;
    } else {
        a2 = fmax(a2, b1);
    }
}

__device__ __forceinline__ void top2_insert(double& a1, double& a2, double d) {
    if (d > a1) {
        a2 = a1;
        a1 = d;
    } else if (d > a2) {
        a2 = d;
    }
}

// Grid-wide top-2 of per-thread (a1 >= a2) pairs of SQUARED displacements; the last
// block to arrive takes the square roots of the winners (sqrt is monotone and
// correctly rounded, so these equal the top two of the per-atom norms) and
// writes the rebuild flag: criterion 0 -> d1 + d2 > skin (verlet_list.cpp:44-63),
// 1 -> d1 > skin / 2.  Called by every thread; blockDim.x <= 1024.
struct DispArgs {
    const double4* ref;
    double skin;
    int criterion;
    double* part;
    unsigned* ticket;
    int* flag;
    double* top2;
};

__device__ inline void top2_grid_at(double a1, double a2, const DispArgs& d, unsigned block,
                                    unsigned nblocks) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double b1 = __shfl_xor_sync(0xffffffffu, a1, o);
        const double b2 = __shfl_xor_sync(0xffffffffu, a2, o);
        top2_merge(a1, a2, b1, b2);
    }
    __shared__ double s1[32], s2[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) {
        s1[warp] = a1;
        s2[warp] = a2;
    }
    __syncthreads();
    __shared__ bool last;
    if (threadIdx.x == 0) {
        double b1 = s1[0], b2 = s2[0];
        for (int w = 1; w < nw; ++w) top2_merge(b1, b2, s1[w], s2[w]);
        d.part[2 * block] = b1;
        d.part[2 * block + 1] = b2;
        __threadfence();
        last = atomicAdd(d.ticket, 1u) == nblocks - 1;
    }
    __syncthreads();
    if (!last) return;
    // the last block merges all partials with every thread, then a tree
    __threadfence();
    double c1 = 0.0, c2 = 0.0;
    for (unsigned b = threadIdx.x; b < nblocks; b += blockDim.x)
        top2_merge(c1, c2, __ldcg(d.part + 2 * b), __ldcg(d.part + 2 * b + 1));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double b1 = __shfl_xor_sync(0xffffffffu, c1, o);
        const double b2 = __shfl_xor_sync(0xffffffffu, c2, o);
        top2_merge(c1, c2, b1, b2);
    }
    __syncthreads();
    if (lane == 0) {
        s1[warp] = c1;
        s2[warp] = c2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < nw; ++w) top2_merge(c1, c2, s1[w], s2[w]);
        const double r1 = __dsqrt_rn(c1), r2 = __dsqrt_rn(c2);
        d.top2[0] = r1;
        d.top2[1] = r2;
        const int rebuild = (d.criterion == 0 ? (r1 + r2) > d.skin : r1 > 0.5 * d.skin) ? 1 : 0;
        *d.flag = rebuild;
        *d.ticket = 0u;
    }
}

__device__ inline void top2_grid(double a1, double a2, const DispArgs& d) {
    top2_grid_at(a1, a2, d, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------- Philox
// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11), counter-based RNG.
struct U4 {
    uint32_t x, y, z, w;
};

__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
        const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += W0;
        k1 += W1;
    }
    return c;
}

// Uniform in (0, 1] from 53 random bits.
__device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
    const uint64_t v = (static_cast<uint64_t>(a) << 21) ^ static_cast<uint64_t>(b >> 11);
    return (static_cast<double>(v & ((1ull << 53) - 1)) + 1.0) * (1.0 / 9007199254740992.0);
}

// Two standard normals by Box-Muller from one Philox block.
__device__ __forceinline__ void normal2(U4 r, double& n0, double& n1) {
    const double u1 = u53(r.x, r.y);
    const double u2 = u53(r.z, r.w);
    const double rad = sqrt(-2.0 * log(u1));
    double s, c;
    sincospi(2.0 * u2, &s, &c);
    n0 = rad * c;
    n1 = rad * s;
}

}  // namespace mdb
