// noalloc.cu -- a Lennard-Jones force entry point that allocates no device memory.
//
// Who needs it: callers that must not call cudaMalloc.  Examples are a host
// framework that owns all device memory through its own pool allocator, and
// latency-critical loops, because cudaMalloc/cudaFree can synchronise the whole
// device.  Such callers can still hand this library device buffers they own.  md_lj_forces_static takes the positions and the output buffers from the
// caller.  Its only working memory (per-block reduction partials and the
// completion ticket) lives in the file-scope array below, which every GPU that
// loads the library holds until the process exits.
#include <mutex>

#include "md_device.cuh"
#include "md_internal.cuh"

namespace mdb {
namespace {

constexpr int kStaticBlock = 256;
constexpr int kStaticMaxBlocks = 1024;  // => at most 262,144 atoms per call
constexpr int64_t kStaticMaxAtoms = static_cast<int64_t>(kStaticMaxBlocks) * kStaticBlock;

// Scratch: 2 doubles of reduction partials per block, then the ticket counter
// (kept as a double-sized slot so the array stays one type).  16,392 bytes.
constexpr int kScratchDoubles = 2 * kStaticMaxBlocks + 1;
static __device__ __align__(256) double g_static_scratch[kScratchDoubles];

// Device address of g_static_scratch for each device, resolved once and kept for
// the life of the process (a cudaDeviceReset unloads the library's device image and
// invalidates it, so the entry point must not be called after one).  The host
// symbol g_static_scratch is only a stand-in for the device array and must never
// be passed to a kernel itself.
constexpr int kMaxDevices = 64;
double* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mutex;

int static_scratch(double** out) {
    int dev = 0;
    MDB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_forces_static: device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p)
            return fail(MD_ERR_CUDA, "md_lj_forces_static: cudaGetSymbolAddress failed: %s",
                        cudaGetErrorString(e));
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return MD_OK;
}

struct StaticLJ {
    double sig2, rc2, rc, uc, dudrc, four_eps, tf_eps;
    int lfs;
};

// Brute-force pair sum (lennard_jones.cpp:50-97) with the reference arithmetic:
// pair (i, j) uses r_lo - r_hi by index; each atom sums its own force, energy and
// virial count each pair once.  Positions are staged through shared memory.
__global__ void __launch_bounds__(kStaticBlock)
k_lj_static(const double* __restrict__ x, const double* __restrict__ y,
            const double* __restrict__ z, int64_t n, Box3 box, StaticLJ p, double* fxo,
            double* fyo, double* fzo, double* scratch, double* ev) {
    __shared__ double3 tile[kStaticBlock];
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const Fold3 f3 = fold3_of(box);
    double fx = 0.0, fy = 0.0, fz = 0.0, e = 0.0, vir = 0.0;
    double xi = 0.0, yi = 0.0, zi = 0.0;
    if (i < n) {
        xi = x[i];
        yi = y[i];
        zi = z[i];
    }
    for (int64_t base = 0; base < n; base += kStaticBlock) {
        __syncthreads();
        if (base + threadIdx.x < n)
            tile[threadIdx.x] = make_double3(x[base + threadIdx.x], y[base + threadIdx.x],
                                             z[base + threadIdx.x]);
        __syncthreads();
        const int lim = static_cast<int>(n - base < kStaticBlock ? n - base : kStaticBlock);
        if (i >= n) continue;
        for (int t = 0; t < lim; ++t) {
            const int64_t j = base + t;
            if (j == i) continue;
            const double3 pj = tile[t];
            const bool lo = i < j;
            double dx, dy, dz;
            if (lo) min_image_wrapped(f3, xi, yi, zi, pj.x, pj.y, pj.z, dx, dy, dz);
            else min_image_wrapped(f3, pj.x, pj.y, pj.z, xi, yi, zi, dx, dy, dz);
            const double r2 = norm2_exact(dx, dy, dz);
            if (!(r2 < p.rc2)) continue;
            const double s2 = __ddiv_rn(p.sig2, r2);
            const double s6 = __dmul_rn(__dmul_rn(s2, s2), s2);
            double u = __dmul_rn(p.four_eps, __dsub_rn(__dmul_rn(s6, s6), s6));
            double w = __dmul_rn(p.tf_eps, __dsub_rn(__dmul_rn(__dmul_rn(2.0, s6), s6), s6));
            if (p.lfs) {
                const double r = __dsqrt_rn(r2);
                u = __dsub_rn(__dsub_rn(u, p.uc), __dmul_rn(__dsub_rn(r, p.rc), p.dudrc));
                w = __dadd_rn(w, __dmul_rn(r, p.dudrc));
            }
            const double s = __ddiv_rn(w, r2);
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
    }
    if (i < n) {
        fxo[i] = fx;
        fyo[i] = fy;
        fzo[i] = fz;
    }
    double v[2] = {e, vir};
    unsigned* ticket = reinterpret_cast<unsigned*>(scratch + 2 * kStaticMaxBlocks);
    grid_reduce<2>(v, scratch, ticket, ev);
}

}  // namespace
}  // namespace mdb

using namespace mdb;

extern "C" {

// See include/moldyn_b200.h for the contract.
int md_lj_forces_static(const double* d_x, const double* d_y, const double* d_z, int64_t n,
                        const double box[3], double sigma, double epsilon, double cutoff,
                        int truncation, double* d_fx, double* d_fy, double* d_fz,
                        double* d_energy_virial, void* stream) {
    if (n < 0)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_forces_static: n = %lld, must be non-negative",
                    static_cast<long long>(n));
    if (n > kStaticMaxAtoms)
        return fail(MD_ERR_INVALID_ARGUMENT,
                    "md_lj_forces_static: n = %lld exceeds the static scratch limit of %lld atoms "
                    "(use md_lj_forces on an md_system for larger systems)",
                    static_cast<long long>(n), static_cast<long long>(kStaticMaxAtoms));
    if (!box || !d_energy_virial || (n > 0 && (!d_x || !d_y || !d_z || !d_fx || !d_fy || !d_fz)))
        return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_forces_static: NULL argument");
    if (truncation != MD_TRUNCATED && truncation != MD_LINEAR_FORCE_SHIFT)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_forces_static: unknown truncation %d", truncation);
    for (int d = 0; d < 3; ++d)
        if (!(box[d] > 0.0))
            return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_forces_static: box lengths must be positive");
    double* scratch = nullptr;
    MDB_TRY(static_scratch(&scratch));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // The ticket must start at zero; a previous call may have left anything there.
    MDB_CUDA(cudaMemsetAsync(scratch + 2 * kStaticMaxBlocks, 0, sizeof(double), s));
    Box3 b;
    for (int d = 0; d < 3; ++d) {
        b.L[d] = box[d];
        b.inv[d] = 1.0 / box[d];
    }
    // lennard_jones.cpp:32-48
    StaticLJ p;
    p.sig2 = sigma * sigma;
    p.rc2 = cutoff * cutoff;
    p.rc = cutoff;
    const double s2 = p.sig2 / p.rc2, s6 = s2 * s2 * s2;
    p.uc = 4.0 * epsilon * (s6 * s6 - s6);
    p.dudrc = -(24.0 * epsilon * (2.0 * s6 * s6 - s6)) / cutoff;
    p.four_eps = 4.0 * epsilon;
    p.tf_eps = 24.0 * epsilon;
    p.lfs = truncation == MD_LINEAR_FORCE_SHIFT ? 1 : 0;
    const int blocks = static_cast<int>(n > 0 ? (n + kStaticBlock - 1) / kStaticBlock : 1);
    k_lj_static<<<blocks, kStaticBlock, 0, s>>>(d_x, d_y, d_z, n, b, p, d_fx, d_fy, d_fz, scratch,
                                               d_energy_virial);
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

}  // extern "C"
