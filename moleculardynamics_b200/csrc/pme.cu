// pme.cu -- smooth particle-mesh Ewald for the reciprocal-space term.
//
// Essmann, Perera, Berkowitz, Darden, Lee & Pedersen, "A smooth particle mesh
// Ewald method", J. Chem. Phys. 103, 8577 (1995).  The reference sums the
// reciprocal term over k vectors (forcefield/ewald.cpp:112-172) and defers PME
// (its phase-2 plan); this replaces that sum, for large water boxes, by:
//
//   spread   Q(k) = sum_i q_i M_p(u_i1 - k1) M_p(u_i2 - k2) M_p(u_i3 - k3), with
//            u = K x / L the scaled fractional coordinate and M_p the cardinal
//            B-spline of order p.  Contributions are added as 64-bit fixed-point
//            integers (2^-46 e resolution, |Q| up to 2^17 e per grid point), so
//            the grid -- and everything after it -- does not depend on the order
//            in which atoms land.
//   FFT      F(m) = sum_k Q(k) e^{-2 pi i m.k/K} (cuFFT, double, real-to-complex).
//   energy   E = C/(2 pi V) sum_{m != 0} theta(m) |F(m)|^2, theta(m) =
//            exp(-pi^2 |m|^2 / alpha^2) / |m|^2 * B1(m1) B2(m2) B3(m3), |m|^2 over
//            the reciprocal vectors m_d / L_d, B_d = |b_d|^2 the Euler
//            exponential-spline moduli; virial trace sum E(m) (1 - 2 pi^2 |m|^2 / alpha^2)
//            (the same expression as the k-vector sum's, k = 2 pi m).
//   forces   phi = C/(pi V) IFFT(theta F), F_i = -q_i sum_k phi(k) grad_i
//            [M_p M_p M_p](k), with dM_p/du = M_{p-1}(u) - M_{p-1}(u - 1).
//
// The spread and the gather are this file's kernels; the two 3-D transforms are
// plain cuFFT calls on the context's stream.
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "md_device.cuh"
#include "md_internal.cuh"

namespace mdb {

namespace {

constexpr int kBlock = 256;
constexpr double kPi = 3.14159265358979323846;
constexpr double kFixScale = 70368744177664.0;       // 2^46
constexpr double kFixInv = 1.0 / 70368744177664.0;

struct PmeArgs {
    int K[3];
    double L[3], inv[3];
};

// Weights c[j] = M_p(w + j) and derivatives d[j] = M_p'(w + j), j = 0..p-1, of
// the grid points floor(u) - j, by the recursion M_n(x) = (x M_{n-1}(x) +
// (n - x) M_{n-1}(x - 1)) / (n - 1) from M_2(w) = w, M_2(w + 1) = 1 - w.
template <int P>
__device__ __forceinline__ void bspline(double w, double (&c)[P], double (&d)[P]) {
#pragma unroll
    for (int j = 0; j < P; ++j) c[j] = 0.0;
    c[0] = w;
    c[1] = 1.0 - w;
#pragma unroll
    for (int n = 3; n <= P; ++n) {
        if (n == P) {
#pragma unroll
            for (int j = 0; j < P; ++j) d[j] = c[j] - (j > 0 ? c[j - 1] : 0.0);
        }
        const double inv = 1.0 / static_cast<double>(n - 1);
#pragma unroll
        for (int j = n - 1; j >= 0; --j) {
            const double x = w + static_cast<double>(j);
            const double lo = j > 0 ? c[j - 1] : 0.0;
            c[j] = (x * c[j] + (static_cast<double>(n) - x) * lo) * inv;
        }
    }
    if (P == 2) {
        d[0] = 1.0;
        d[1] = -1.0;
    }
}

// Scaled coordinate u = K * frac(x / L) in [0, K): grid origin i0 = floor(u), w = u - i0.
__device__ __forceinline__ void grid_coord(double x, double inv_l, int k, int& i0, double& w) {
    double t = x * inv_l;
    t -= floor(t);
    double u = t * static_cast<double>(k);
    if (u >= static_cast<double>(k)) u -= static_cast<double>(k);
    const double f = floor(u);
    i0 = static_cast<int>(f);
    w = u - f;
}

__device__ __forceinline__ int wrap_index(int i, int k) { return i < 0 ? i + k : i; }

// One thread per (atom, jx, jy): P contributions along z, as fixed-point integers.
template <int P>
__global__ void __launch_bounds__(kBlock)
k_pme_spread(const double4* __restrict__ pos, const double* __restrict__ q, int64_t n,
             PmeArgs a, unsigned long long* grid) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const int64_t i = t / (P * P);
    if (i >= n) return;
    const int jx = static_cast<int>(t % (P * P)) / P, jy = static_cast<int>(t % P);
    const double4 p = pos[i];
    const double qi = q[i];
    int ix, iy, iz;
    double wx, wy, wz;
    grid_coord(p.x, a.inv[0], a.K[0], ix, wx);
    grid_coord(p.y, a.inv[1], a.K[1], iy, wy);
    grid_coord(p.z, a.inv[2], a.K[2], iz, wz);
    double cx[P], cy[P], cz[P], dd[P];
    bspline<P>(wx, cx, dd);
    bspline<P>(wy, cy, dd);
    bspline<P>(wz, cz, dd);
    const int gx = wrap_index(ix - jx, a.K[0]), gy = wrap_index(iy - jy, a.K[1]);
    double cxj = 0.0, cyj = 0.0;  // cx[jx], cy[jy] without dynamic register indexing
#pragma unroll
    for (int j = 0; j < P; ++j) {
        if (j == jx) cxj = cx[j];
        if (j == jy) cyj = cy[j];
    }
    const double qxy = qi * cxj * cyj;
    unsigned long long* row = grid + (static_cast<int64_t>(gx) * a.K[1] + gy) * a.K[2];
#pragma unroll
    for (int jz = 0; jz < P; ++jz) {
        const long long v = __double2ll_rn(qxy * cz[jz] * kFixScale);
        atomicAdd(row + wrap_index(iz - jz, a.K[2]), static_cast<unsigned long long>(v));
    }
}

// Fixed-point grid -> real grid; the integer grid is cleared for the next spread.
__global__ void k_pme_unfix(unsigned long long* __restrict__ grid, double* __restrict__ out,
                            int64_t count) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= count) return;
    out[k] = static_cast<double>(static_cast<long long>(grid[k])) * kFixInv;
    grid[k] = 0ull;
}

// theta(m) F(m) over the half spectrum (K1, K2, K3/2 + 1), with the energy and
// the virial trace summed on the way; planes m3 = 0 (and K3/2 for even K3) count
// once, the others twice (their conjugates are not stored).
__global__ void k_pme_influence(double2* __restrict__ f, PmeArgs a, const double* __restrict__ bmod,
                                double inv_alpha2, double e_coef, double phi_coef, int energy_only,
                                double* part, unsigned* ticket, double* out) {
    const int nz = a.K[2] / 2 + 1;
    const int64_t count = static_cast<int64_t>(a.K[0]) * a.K[1] * nz;
    double v[2] = {0.0, 0.0};
    for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < count;
         idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int z = static_cast<int>(idx % nz);
        const int y = static_cast<int>((idx / nz) % a.K[1]);
        const int x = static_cast<int>(idx / (static_cast<int64_t>(nz) * a.K[1]));
        const int mx = x <= a.K[0] / 2 ? x : x - a.K[0];
        const int my = y <= a.K[1] / 2 ? y : y - a.K[1];
        const double fx = mx * a.inv[0], fy = my * a.inv[1], fz = z * a.inv[2];
        const double m2 = fx * fx + fy * fy + fz * fz;
        double2 g = f[idx];
        if (m2 > 0.0) {
            const double theta = exp(-kPi * kPi * m2 * inv_alpha2) / m2 * bmod[x] *
                                 bmod[a.K[0] + y] * bmod[a.K[0] + a.K[1] + z];
            const double mult = (z == 0 || 2 * z == a.K[2]) ? 1.0 : 2.0;
            const double e = mult * e_coef * theta * (g.x * g.x + g.y * g.y);
            v[0] += e;
            v[1] += e * (1.0 - 2.0 * kPi * kPi * m2 * inv_alpha2);
            g.x *= phi_coef * theta;
            g.y *= phi_coef * theta;
        } else {
            g.x = 0.0;
            g.y = 0.0;
        }
        if (!energy_only) f[idx] = g;
    }
    grid_reduce<2>(v, part, ticket, out);
}

// Forces from the potential grid: 8 lanes per atom, lane jx < P takes the
// (jx, *, *) plane of the stencil; lanes combine by a fixed butterfly.
template <int P>
__global__ void __launch_bounds__(kBlock)
k_pme_gather(const double4* __restrict__ pos, const double* __restrict__ q, int64_t n, PmeArgs a,
             const double* __restrict__ phi, double* fxo, double* fyo, double* fzo) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const int64_t i = t >> 3;
    const int jx = static_cast<int>(t & 7);
    const bool live = i < n;
    double gx = 0.0, gy = 0.0, gz = 0.0, qi = 0.0;
    if (live) {
        const double4 p = pos[i];
        qi = q[i];
        int ix, iy, iz;
        double wx, wy, wz;
        grid_coord(p.x, a.inv[0], a.K[0], ix, wx);
        grid_coord(p.y, a.inv[1], a.K[1], iy, wy);
        grid_coord(p.z, a.inv[2], a.K[2], iz, wz);
        double cx[P], dx[P], cy[P], dy[P], cz[P], dz[P];
        bspline<P>(wx, cx, dx);
        bspline<P>(wy, cy, dy);
        bspline<P>(wz, cz, dz);
        if (jx < P) {
            double cxj = 0.0, dxj = 0.0;
#pragma unroll
            for (int j = 0; j < P; ++j)
                if (j == jx) {
                    cxj = cx[j];
                    dxj = dx[j];
                }
            const int gxi = wrap_index(ix - jx, a.K[0]);
#pragma unroll
            for (int jy = 0; jy < P; ++jy) {
                const double* row =
                    phi + (static_cast<int64_t>(gxi) * a.K[1] + wrap_index(iy - jy, a.K[1])) * a.K[2];
                double sc = 0.0, sd = 0.0;  // sum phi cz, sum phi dz along the row
#pragma unroll
                for (int jz = 0; jz < P; ++jz) {
                    const double ph = __ldg(row + wrap_index(iz - jz, a.K[2]));
                    sc = fma(ph, cz[jz], sc);
                    sd = fma(ph, dz[jz], sd);
                }
                gx = fma(dxj * cy[jy], sc, gx);
                gy = fma(cxj * dy[jy], sc, gy);
                gz = fma(cxj * cy[jy], sd, gz);
            }
        }
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
        gx += __shfl_xor_sync(0xffffffffu, gx, o);
        gy += __shfl_xor_sync(0xffffffffu, gy, o);
        gz += __shfl_xor_sync(0xffffffffu, gz, o);
    }
    if (live && jx == 0) {
        fxo[i] -= qi * gx * (a.K[0] * a.inv[0]);
        fyo[i] -= qi * gy * (a.K[1] * a.inv[1]);
        fzo[i] -= qi * gz * (a.K[2] * a.inv[2]);
    }
}

// |b(m)|^2 = 1 / |sum_{k=0}^{p-2} M_p(k + 1) e^{2 pi i m k / K}|^2 per axis
// (Essmann eq. 4.4); where the sum vanishes (odd p at m = K/2) the neighbours'
// mean is used, as is customary.
std::vector<double> bspline_moduli(int K, int p) {
    // M_p at the integers 1..p-1 by the same recursion as the device
    std::vector<double> m(static_cast<size_t>(p + 1), 0.0);  // m[x] = M_n(x)
    m[1] = 1.0;                                              // M_2(1) = 1
    for (int n = 3; n <= p; ++n) {
        std::vector<double> next(m.size(), 0.0);
        for (int x = 1; x < n; ++x)
            next[x] = (x * m[x] + (n - x) * m[x - 1]) / static_cast<double>(n - 1);
        m = next;
    }
    std::vector<double> out(static_cast<size_t>(K));
    for (int mi = 0; mi < K; ++mi) {
        double re = 0.0, im = 0.0;
        for (int k = 0; k <= p - 2; ++k) {
            const double arg = 2.0 * kPi * mi * k / K;
            re += m[k + 1] * std::cos(arg);
            im += m[k + 1] * std::sin(arg);
        }
        const double mag = re * re + im * im;
        out[mi] = mag > 1e-10 ? 1.0 / mag : 0.0;
    }
    for (int mi = 0; mi < K; ++mi)
        if (out[mi] == 0.0) out[mi] = 0.5 * (out[(mi + K - 1) % K] + out[(mi + 1) % K]);
    return out;
}

}  // namespace

struct PmeState {
    md_context* ctx = nullptr;
    int K[3] = {0, 0, 0};
    int order = 0;
    DevBuf fix, real, spec, bmod, part;
    cufftHandle fwd = 0, inv = 0;
    bool planned = false;

    ~PmeState() {
        if (planned) {
            cufftDestroy(fwd);
            cufftDestroy(inv);
        }
        fix.release();
        real.release();
        spec.release();
        bmod.release();
        part.release();
    }
};

int pme_create(md_context* ctx, const int K[3], int order, PmeState** out) {
    PmeState* s = new (std::nothrow) PmeState();
    if (!s) return fail(MD_ERR_OUT_OF_MEMORY, "md_ewald_set_pme: host allocation");
    s->ctx = ctx;
    for (int d = 0; d < 3; ++d) s->K[d] = K[d];
    s->order = order;
    const int64_t cells = static_cast<int64_t>(K[0]) * K[1] * K[2];
    const int64_t half = static_cast<int64_t>(K[0]) * K[1] * (K[2] / 2 + 1);
    int rc = MD_OK;
    if ((rc = s->fix.ensure(sizeof(unsigned long long) * cells)) != MD_OK ||
        (rc = s->real.ensure(sizeof(double) * cells)) != MD_OK ||
        (rc = s->spec.ensure(sizeof(double2) * half)) != MD_OK ||
        (rc = s->bmod.ensure(sizeof(double) * (K[0] + K[1] + K[2]))) != MD_OK ||
        (rc = s->part.ensure(sizeof(double) * 2 * 4 * static_cast<size_t>(ctx->sm_count))) != MD_OK) {
        delete s;
        return rc;
    }
    std::vector<double> bm;
    for (int d = 0; d < 3; ++d) {
        const std::vector<double> b = bspline_moduli(K[d], order);
        bm.insert(bm.end(), b.begin(), b.end());
    }
    if (cudaMemcpy(s->bmod.ptr, bm.data(), sizeof(double) * bm.size(), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemset(s->fix.ptr, 0, sizeof(unsigned long long) * cells) != cudaSuccess) {
        delete s;
        return fail(MD_ERR_CUDA, "md_ewald_set_pme: grid initialisation");
    }
    if (cufftPlan3d(&s->fwd, K[0], K[1], K[2], CUFFT_D2Z) != CUFFT_SUCCESS) {
        delete s;
        return fail(MD_ERR_CUDA, "md_ewald_set_pme: cuFFT forward plan");
    }
    if (cufftPlan3d(&s->inv, K[0], K[1], K[2], CUFFT_Z2D) != CUFFT_SUCCESS) {
        cufftDestroy(s->fwd);
        delete s;
        return fail(MD_ERR_CUDA, "md_ewald_set_pme: cuFFT inverse plan");
    }
    s->planned = true;
    if (cufftSetStream(s->fwd, ctx->stream) != CUFFT_SUCCESS ||
        cufftSetStream(s->inv, ctx->stream) != CUFFT_SUCCESS) {
        delete s;
        return fail(MD_ERR_CUDA, "md_ewald_set_pme: cuFFT stream");
    }
    *out = s;
    return MD_OK;
}

void pme_destroy(PmeState* s) { delete s; }

int pme_grid(const PmeState* s, int K[3], int* order) {
    for (int d = 0; d < 3; ++d) K[d] = s->K[d];
    *order = s->order;
    return MD_OK;
}

namespace {

template <int P>
void launch_spread(PmeState* s, md_system* sys, const PmeArgs& a) {
    const int64_t threads = std::max<int64_t>(sys->n * P * P, 1);
    k_pme_spread<P><<<grid_for(threads, kBlock), kBlock, 0, s->ctx->stream>>>(
        sys->cur.pos, sys->cur.charge, sys->n, a, s->fix.as<unsigned long long>());
}

template <int P>
void launch_gather(PmeState* s, md_system* sys, const PmeArgs& a) {
    k_pme_gather<P><<<grid_for(std::max<int64_t>(8 * sys->n, 1), kBlock), kBlock, 0, s->ctx->stream>>>(
        sys->cur.pos, sys->cur.charge, sys->n, a, s->real.as<double>(), sys->cur.fx, sys->cur.fy,
        sys->cur.fz);
}

}  // namespace

// The reciprocal energy and virial trace into out[0..1] (device); with forces
// (mode != 0) the k-space forces are added to the system's.
int pme_eval_async(PmeState* s, md_system* sys, double alpha, double coulomb, int mode, double* out,
                   unsigned* ticket) {
    md_context* ctx = s->ctx;
    const int64_t n = sys->n;
    PmeArgs a;
    for (int d = 0; d < 3; ++d) {
        a.K[d] = s->K[d];
        a.L[d] = sys->box[d];
        a.inv[d] = sys->inv_box[d];
    }
    const int64_t cells = static_cast<int64_t>(s->K[0]) * s->K[1] * s->K[2];
    const int64_t half = static_cast<int64_t>(s->K[0]) * s->K[1] * (s->K[2] / 2 + 1);
    if (n > 0) {
        switch (s->order) {
            case 4: launch_spread<4>(s, sys, a); break;
            case 6: launch_spread<6>(s, sys, a); break;
            default: launch_spread<8>(s, sys, a); break;
        }
    }
    k_pme_unfix<<<grid_for(cells, kBlock), kBlock, 0, ctx->stream>>>(
        s->fix.as<unsigned long long>(), s->real.as<double>(), cells);
    ctx->launches += (n > 0 ? 1 : 0) + 1;
    MDB_CHECK_LAUNCH();
    if (cufftExecD2Z(s->fwd, s->real.as<cufftDoubleReal>(), s->spec.as<cufftDoubleComplex>()) !=
        CUFFT_SUCCESS)
        return fail(MD_ERR_CUDA, "PME: forward FFT");
    const double volume = sys->box[0] * sys->box[1] * sys->box[2];
    const int g = static_cast<int>(std::min<int64_t>(grid_for(half, kBlock), 4 * ctx->sm_count));
    MDB_TRY(s->part.ensure(sizeof(double) * 2 * static_cast<size_t>(g)));
    k_pme_influence<<<g, kBlock, 0, ctx->stream>>>(
        s->spec.as<double2>(), a, s->bmod.as<double>(), 1.0 / (alpha * alpha),
        coulomb / (2.0 * kPi * volume), coulomb / (kPi * volume), mode == 0 ? 1 : 0,
        s->part.as<double>(), ticket, out);
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    if (mode == 0 || n == 0) return MD_OK;
    if (cufftExecZ2D(s->inv, s->spec.as<cufftDoubleComplex>(), s->real.as<cufftDoubleReal>()) !=
        CUFFT_SUCCESS)
        return fail(MD_ERR_CUDA, "PME: inverse FFT");
    switch (s->order) {
        case 4: launch_gather<4>(s, sys, a); break;
        case 6: launch_gather<6>(s, sys, a); break;
        default: launch_gather<8>(s, sys, a); break;
    }
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

}  // namespace mdb
