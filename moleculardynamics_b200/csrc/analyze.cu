// analyze.cu -- the reference's analysis consumers on the device: the radial
// distribution function (analyze/rdf.cpp), the mean-squared displacement
// (analyze/msd.cpp) and the velocity autocorrelation function (analyze/vacf.cpp).
//
// RDF: the reference counts every pair i < j of the frame, brute force; here the
// pairs within rMax are found through a cell grid of width >= rMax (27-cell
// stencil, each pair taken from its lower original index), and the distance and
// bin use the reference's arithmetic (minimum image, norm, sqrt, r / width), so
// the integer histogram equals the reference's.  Grids with fewer than 3 cells
// per side fall back to all pairs.
//
// MSD / VACF: per-atom state lives on the device in original atom order (the
// device order changes at every Verlet rebuild): the running unwrapped position,
// the previous wrapped position and a ring of maxLag + 1 frames.  Each push
// forms, for every available lag, the sum over atoms of |u_i(t) - u_i(t - lag)|^2
// (or v_i(t) . v_i(t - lag)) with a fixed-order tree reduction; the host adds the
// per-lag sums into running totals in the reference's order.
#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "md_device.cuh"
#include "md_internal.cuh"

using namespace mdb;

struct md_rdf {
    md_context* ctx = nullptr;
    double rmax = 0.0, width = 0.0;
    int64_t bins = 0;
    DevBuf hist;                 // unsigned long long[bins]: pair counts of every frame so far
    mutable std::vector<double> host;  // host copy of hist (rdf.cpp:73), refreshed on demand
    mutable bool stale = false;        // hist has frames that host does not
    int64_t frames = 0, natoms = 0;
    double sum_rho = 0.0;
    CellGrid grid;
    double grid_box[3] = {0, 0, 0};
    DevBuf sorted, start;
};

struct md_corr {                 // shared state of md_msd and md_vacf
    md_context* ctx = nullptr;
    int64_t n = 0, max_lag = 0, period = 0, pushed = 0;
    DevBuf prev, unwrapped;      // 3n doubles each (x | y | z), MSD only
    DevBuf ring;                 // period * 3n doubles
    DevBuf part, sums;           // per-lag partial sums
    std::vector<double> sum;     // running per-lag totals (msd.cpp:91, vacf.cpp:211)
    std::vector<int64_t> count;  // per-lag sample counts
};
struct md_msd : md_corr {};
struct md_vacf : md_corr {};

namespace {

constexpr int kRdfBlock = 256;
constexpr int kRdfSharedBins = 8192;  // per-block shared histogram up to this many bins

struct RdfArgs {
    Box3 box;
    double rmax, rmax2_hi, width;
    int bins;
    int use_shared;
    int64_t first, stride;  // atoms counted: original index first + k * stride
};

__device__ __forceinline__ bool rdf_selected(const RdfArgs& a, double w) {
    const int64_t o = static_cast<int64_t>(w) - a.first;
    return o >= 0 && o % a.stride == 0;
}

// rdf.cpp:68-74 for the pair (a, b), a holding the lower original index: the bin
// of r = |minimumImage(r_a - r_b)|, or -1 when r >= rMax or past the last bin.
// r^2 above rMax^2 (1 + 1e-12) cannot round to a distance below rMax, so those
// pairs skip the square root and division.
__device__ __forceinline__ int rdf_bin(const RdfArgs& a, const Fold3& f3, const double4& p,
                                       const double4& q) {
    double dx, dy, dz;
    min_image_wrapped(f3, p.x, p.y, p.z, q.x, q.y, q.z, dx, dy, dz);
    const double r2 = norm2_exact(dx, dy, dz);
    if (!(r2 < a.rmax2_hi)) return -1;
    const double r = __dsqrt_rn(r2);
    if (!(r < a.rmax)) return -1;
    const double k = __ddiv_rn(r, a.width);
    return k < static_cast<double>(a.bins) ? static_cast<int>(k) : -1;
}

__device__ __forceinline__ void rdf_count(const RdfArgs& a, unsigned* s_hist,
                                          unsigned long long* hist, int bin) {
    if (bin < 0) return;
    if (a.use_shared) atomicAdd(s_hist + bin, 1u);
    else atomicAdd(hist + bin, 1ull);
}

__device__ __forceinline__ void rdf_flush(const RdfArgs& a, unsigned* s_hist,
                                          unsigned long long* hist) {
    if (!a.use_shared) return;
    __syncthreads();
    for (int k = threadIdx.x; k < a.bins; k += blockDim.x)
        if (s_hist[k]) atomicAdd(hist + k, static_cast<unsigned long long>(s_hist[k]));
}

__device__ __forceinline__ void rdf_zero(const RdfArgs& a, unsigned* s_hist) {
    if (!a.use_shared) return;
    for (int k = threadIdx.x; k < a.bins; k += blockDim.x) s_hist[k] = 0u;
    __syncthreads();
}

struct RdfGrid {
    int nx, ny, nz, ncells;
    const int* rank_of_cell;
    const int* cell_of_rank;
    const int* start;   // ncells + 1, by Morton rank
    const int* sorted;  // sorted position -> device slot
};

// One thread per sorted position: its atom against the atoms of the 27 cells
// around its cell, each pair counted from its lower original index.
__global__ void __launch_bounds__(kRdfBlock)
k_rdf_cells(const double4* __restrict__ pos, int64_t n, RdfGrid g, RdfArgs a,
            unsigned long long* hist) {
    extern __shared__ unsigned s_hist[];
    rdf_zero(a, s_hist);
    const int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (s < n) {
        const Fold3 f3 = fold3_of(a.box);
        int lo = 0, hi = g.ncells;  // the rank whose range holds s
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (g.start[mid] <= s) lo = mid;
            else hi = mid;
        }
        const int cell = g.cell_of_rank[lo];
        const int cx = cell % g.nx, cy = (cell / g.nx) % g.ny, cz = cell / (g.nx * g.ny);
        const double4 p = ldg4(pos + g.sorted[s]);
        if (!rdf_selected(a, p.w)) goto done;
        for (int q = 0; q < 27; ++q) {
            int jx = cx + (q % 3) - 1, jy = cy + ((q / 3) % 3) - 1, jz = cz + (q / 9) - 1;
            jx = jx < 0 ? jx + g.nx : (jx >= g.nx ? jx - g.nx : jx);
            jy = jy < 0 ? jy + g.ny : (jy >= g.ny ? jy - g.ny : jy);
            jz = jz < 0 ? jz + g.nz : (jz >= g.nz ? jz - g.nz : jz);
            const int rr = g.rank_of_cell[jx + g.nx * (jy + g.ny * jz)];
            const int t1 = g.start[rr + 1];
            for (int t = g.start[rr]; t < t1; ++t) {
                const double4 qd = ldg4(pos + g.sorted[t]);
                if (qd.w > p.w && rdf_selected(a, qd.w))
                    rdf_count(a, s_hist, hist, rdf_bin(a, f3, p, qd));
            }
        }
    }
done:
    rdf_flush(a, s_hist, hist);
}

// Small boxes (fewer than 3 cells of width rMax per side): every pair.  Block
// (x, y) pairs the atoms of block x with one span of the other side, staged in
// shared memory; the spans are short enough to give every SM work even for a
// few hundred atoms.
__global__ void __launch_bounds__(kRdfBlock)
k_rdf_brute(const double4* __restrict__ pos, int64_t n, int span, RdfArgs a,
            unsigned long long* hist) {
    extern __shared__ unsigned s_hist[];
    __shared__ double4 tile[kRdfBlock];
    rdf_zero(a, s_hist);
    const Fold3 f3 = fold3_of(a.box);
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const double4 p = i < n ? pos[i] : make_double4(0.0, 0.0, 0.0, 0.0);
    const int64_t base = blockIdx.y * static_cast<int64_t>(span);
    const int lim = static_cast<int>(n - base < span ? n - base : span);
    if (threadIdx.x < lim) tile[threadIdx.x] = pos[base + threadIdx.x];
    __syncthreads();
    if (i < n && rdf_selected(a, p.w))
        for (int t = 0; t < lim; ++t)
            if (tile[t].w > p.w && rdf_selected(a, tile[t].w))
                rdf_count(a, s_hist, hist, rdf_bin(a, f3, p, tile[t]));
    rdf_flush(a, s_hist, hist);
}

// ------------------------------------------------------------------ MSD / VACF
constexpr int kCorrBlock = 256;
constexpr int64_t kCorrChunk = 8192;  // atoms per partial sum

// msd.cpp:69-81: gather atom o's wrapped position from its device slot, fold the
// minimum-image step from the previous wrapped position into the running
// unwrapped position (the first push takes the position itself) and store it in
// the ring slot of this push.
__global__ void k_msd_unwrap(const double4* __restrict__ pos, const int* __restrict__ slot_of,
                             int64_t n, Box3 box, int first, double* prev, double* unw,
                             double* ring_slot) {
    const int64_t o = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (o >= n) return;
    const double4 p = pos[slot_of[o]];
    double ux = p.x, uy = p.y, uz = p.z;
    if (!first) {
        double dx, dy, dz;
        min_image_exact(box, p.x, p.y, p.z, prev[o], prev[n + o], prev[2 * n + o], dx, dy, dz);
        ux = __dadd_rn(unw[o], dx);
        uy = __dadd_rn(unw[n + o], dy);
        uz = __dadd_rn(unw[2 * n + o], dz);
    }
    prev[o] = p.x;
    prev[n + o] = p.y;
    prev[2 * n + o] = p.z;
    unw[o] = ux;
    unw[n + o] = uy;
    unw[2 * n + o] = uz;
    ring_slot[o] = ux;
    ring_slot[n + o] = uy;
    ring_slot[2 * n + o] = uz;
}

// vacf.cpp:196-202: the velocities of this push in original order, into the ring.
__global__ void k_vacf_gather(const double* __restrict__ vx, const double* __restrict__ vy,
                              const double* __restrict__ vz, const int* __restrict__ slot_of,
                              int64_t n, double* ring_slot) {
    const int64_t o = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (o >= n) return;
    const int s = slot_of[o];
    ring_slot[o] = vx[s];
    ring_slot[n + o] = vy[s];
    ring_slot[2 * n + o] = vz[s];
}

// Per (chunk, lag) partial sums over the chunk's atoms: |a_i - b_i|^2 (MSD,
// msd.cpp:88-89) or a_i . b_i (VACF, vacf.cpp:209), a the newest ring slot and b
// the slot `lag` pushes back.  Block sums in a fixed order: deterministic.
template <bool DIFF>
__global__ void __launch_bounds__(kCorrBlock)
k_corr_lags(const double* __restrict__ ring, int64_t n, int64_t period, int64_t slot,
            int64_t chunks, int64_t lag0, double* part) {
    __shared__ double s_sum[kCorrBlock / 32];
    const int64_t lag = lag0 + blockIdx.y, chunk = blockIdx.x;
    const double* a = ring + slot * 3 * n;
    const double* b = ring + ((slot + period - lag) % period) * 3 * n;
    const int64_t i0 = chunk * kCorrChunk, i1 = min(n, i0 + kCorrChunk);
    double acc = 0.0;
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        const double ax = a[i], ay = a[n + i], az = a[2 * n + i];
        const double bx = b[i], by = b[n + i], bz = b[2 * n + i];
        if (DIFF) {
            acc += norm2_exact(__dsub_rn(ax, bx), __dsub_rn(ay, by), __dsub_rn(az, bz));
        } else {
            acc += __dadd_rn(__dadd_rn(__dmul_rn(ax, bx), __dmul_rn(ay, by)), __dmul_rn(az, bz));
        }
    }
    const double w = warp_sum(acc);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_sum[warp] = w;
    __syncthreads();
    if (warp == 0) {
        double t = lane < kCorrBlock / 32 ? s_sum[lane] : 0.0;
        t = warp_sum(t);
        if (lane == 0) part[lag * chunks + chunk] = t;
    }
}

// One warp per lag: the chunk partial sums in chunk order.
__global__ void k_corr_total(const double* __restrict__ part, int64_t chunks, int nlags,
                             double* sums) {
    const int lag = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (lag >= nlags) return;
    double t = 0.0;
    for (int64_t c = lane; c < chunks; c += 32) t += part[lag * chunks + c];
    t = warp_sum(t);
    if (lane == 0) sums[lag] = t;
}

}  // namespace

namespace {

Box3 box_of_system(const md_system* sys) {
    Box3 b;
    for (int d = 0; d < 3; ++d) {
        b.L[d] = sys->box[d];
        b.inv[d] = sys->inv_box[d];
    }
    return b;
}

int corr_create(md_context* ctx, int64_t natoms, int64_t max_lag, bool msd, md_corr* c,
                const char* who) {
    if (!ctx) return fail(MD_ERR_INVALID_ARGUMENT, "%s: NULL context", who);
    if (natoms < 0 || max_lag < 0)
        return fail(MD_ERR_INVALID_ARGUMENT, "%s: natoms and maxLag must be >= 0", who);
    MDB_CUDA(cudaSetDevice(ctx->device));
    c->ctx = ctx;
    c->n = natoms;
    c->max_lag = max_lag;
    c->period = max_lag + 1;  // msd.cpp:59, vacf.cpp:190
    const size_t n3 = 3 * static_cast<size_t>(natoms > 0 ? natoms : 1);
    if (msd) {
        MDB_TRY(c->prev.ensure(sizeof(double) * n3));
        MDB_TRY(c->unwrapped.ensure(sizeof(double) * n3));
    }
    MDB_TRY(c->ring.ensure(sizeof(double) * n3 * static_cast<size_t>(c->period)));
    const int64_t chunks = std::max<int64_t>(1, (natoms + kCorrChunk - 1) / kCorrChunk);
    MDB_TRY(c->part.ensure(sizeof(double) * static_cast<size_t>(chunks * c->period)));
    MDB_TRY(c->sums.ensure(sizeof(double) * static_cast<size_t>(c->period)));
    c->sum.assign(static_cast<size_t>(c->period), 0.0);
    c->count.assign(static_cast<size_t>(c->period), 0);
    return MD_OK;
}

// One push: fill this push's ring slot (MSD: unwrapped positions; VACF:
// velocities), then add every available lag's sum over atoms to the totals
// (msd.cpp:80-95, vacf.cpp:201-215).
int corr_push(md_corr* c, md_system* sys, bool msd, const char* who) {
    if (!sys) return fail(MD_ERR_INVALID_ARGUMENT, "%s: NULL system", who);
    if (sys->n != c->n)
        return fail(MD_ERR_INVALID_ARGUMENT, "%s: the system has %lld atoms, not the %lld it was created for",
                    who, static_cast<long long>(sys->n), static_cast<long long>(c->n));
    if (sys->ctx != c->ctx)
        return fail(MD_ERR_INVALID_ARGUMENT, "%s: the system lives on another context", who);
    md_context* ctx = c->ctx;
    const int64_t n = c->n;
    const int64_t slot = c->pushed % c->period;
    const int64_t nl = std::min(c->pushed, c->max_lag) + 1;
    if (n > 0) {
        double* ring_slot = c->ring.as<double>() + slot * 3 * n;
        if (msd)
            k_msd_unwrap<<<grid_for(n, kCorrBlock), kCorrBlock, 0, ctx->stream>>>(
                sys->cur.pos, sys->slot, n, box_of_system(sys), c->pushed == 0 ? 1 : 0,
                c->prev.as<double>(), c->unwrapped.as<double>(), ring_slot);
        else
            k_vacf_gather<<<grid_for(n, kCorrBlock), kCorrBlock, 0, ctx->stream>>>(
                sys->cur.vx, sys->cur.vy, sys->cur.vz, sys->slot, n, ring_slot);
        const int64_t chunks = (n + kCorrChunk - 1) / kCorrChunk;
        for (int64_t lag0 = 0; lag0 < nl; lag0 += 65535) {  // grid y holds up to 65535 lags
            const dim3 grid(static_cast<unsigned>(chunks),
                            static_cast<unsigned>(std::min<int64_t>(65535, nl - lag0)));
            if (msd)
                k_corr_lags<true><<<grid, kCorrBlock, 0, ctx->stream>>>(
                    c->ring.as<double>(), n, c->period, slot, chunks, lag0, c->part.as<double>());
            else
                k_corr_lags<false><<<grid, kCorrBlock, 0, ctx->stream>>>(
                    c->ring.as<double>(), n, c->period, slot, chunks, lag0, c->part.as<double>());
        }
        k_corr_total<<<grid_for(32 * nl, kCorrBlock), kCorrBlock, 0, ctx->stream>>>(
            c->part.as<double>(), chunks, static_cast<int>(nl), c->sums.as<double>());
        ctx->launches += 3;
        MDB_CHECK_LAUNCH();
        std::vector<double> s(static_cast<size_t>(nl));
        MDB_CUDA(cudaMemcpyAsync(s.data(), c->sums.ptr, sizeof(double) * nl,
                                 cudaMemcpyDeviceToHost, ctx->stream));
        MDB_CUDA(cudaStreamSynchronize(ctx->stream));
        for (int64_t lag = 0; lag < nl; ++lag) c->sum[lag] += s[lag];
    }
    for (int64_t lag = 0; lag < nl; ++lag) c->count[lag] += n;
    ++c->pushed;
    return ctx_check_status(ctx);
}

// Per-lag means (msd.cpp:98-106, vacf.cpp:218-226).
std::vector<double> corr_means(const md_corr* c) {
    std::vector<double> r(static_cast<size_t>(c->period), 0.0);
    for (int64_t lag = 0; lag < c->period; ++lag)
        if (c->count[lag] > 0) r[lag] = c->sum[lag] / static_cast<double>(c->count[lag]);
    return r;
}

}  // namespace

extern "C" {

// ------------------------------------------------------------------------ RDF
int md_rdf_create(md_context* ctx, double rmax, int64_t bins, md_rdf** out) {
    graph_epoch_bump();
    if (!ctx || !out) return fail(MD_ERR_INVALID_ARGUMENT, "md_rdf_create: NULL argument");
    if (bins < 0) return fail(MD_ERR_INVALID_ARGUMENT, "md_rdf_create: bins must be >= 0");
    md_rdf* r = new (std::nothrow) md_rdf;
    if (!r) return fail(MD_ERR_RUNTIME, "md_rdf_create: out of host memory");
    r->ctx = ctx;
    r->rmax = rmax;
    r->bins = bins;
    r->width = rmax / static_cast<double>(bins);  // rdf.cpp:53
    r->host.assign(static_cast<size_t>(bins), 0.0);
    if (bins > 0 && (r->hist.ensure(sizeof(unsigned long long) * static_cast<size_t>(bins)) != MD_OK ||
                     cudaMemsetAsync(r->hist.ptr, 0, sizeof(unsigned long long) * static_cast<size_t>(bins),
                                     ctx->stream) != cudaSuccess)) {
        r->hist.release();
        delete r;
        return fail(MD_ERR_CUDA, "md_rdf_create: device histogram");
    }
    *out = r;
    return MD_OK;
}

int md_rdf_destroy(md_rdf* r) {
    graph_epoch_bump();
    if (!r) return MD_OK;
    if (r->ctx) cudaStreamSynchronize(r->ctx->stream);
    r->hist.release();
    r->sorted.release();
    r->start.release();
    r->grid.release();
    delete r;
    return MD_OK;
}

int md_rdf_accumulate(md_rdf* r, md_system* sys) { return md_rdf_accumulate_subset(r, sys, 0, 1); }

int md_rdf_accumulate_subset(md_rdf* r, md_system* sys, int64_t first, int64_t stride) {
    MDB_TRY(rdf_accumulate_async(r, sys, first, stride));
    return ctx_check_status(r->ctx);
}

int md_rdf_histogram(const md_rdf* r, double* hist) {
    if (!r || (!hist && r->bins > 0)) return fail(MD_ERR_INVALID_ARGUMENT, "md_rdf_histogram: NULL argument");
    MDB_TRY(rdf_sync(r));
    std::copy(r->host.begin(), r->host.end(), hist);
    return MD_OK;
}

}  // extern "C"

namespace mdb {

// One frame's pair counts are added to the device histogram; nothing is read
// back (the host copy is refreshed by rdf_sync when the counts are asked for).
// Counts are integers, so summing them per bin on the device over frames equals
// the reference's running double sum (rdf.cpp:73) exactly.
int rdf_accumulate_async(md_rdf* r, md_system* sys, int64_t first, int64_t stride) {
    MDB_TRY(rdf_frame_launch(r, sys, first, stride));
    rdf_frame_note(r, sys, first, stride);
    return MD_OK;
}

void rdf_frame_note(md_rdf* r, const md_system* sys, int64_t first, int64_t stride) {
    const int64_t n = sys->n;
    const int64_t selected = n > first ? (n - first + stride - 1) / stride : 0;
    if (selected > 1 && r->bins > 0 && r->rmax > 0.0) r->stale = true;
    r->natoms = selected;  // rdf.cpp:79-81
    r->sum_rho += static_cast<double>(selected) / (sys->box[0] * sys->box[1] * sys->box[2]);
    ++r->frames;
}

int rdf_frame_launch(md_rdf* r, md_system* sys, int64_t first, int64_t stride) {
    if (!r || !sys) return fail(MD_ERR_INVALID_ARGUMENT, "md_rdf_accumulate: NULL argument");
    if (first < 0 || stride < 1)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_rdf_accumulate_subset: first >= 0, stride >= 1");
    if (sys->ctx != r->ctx)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_rdf_accumulate: the system lives on another context");
    const double smallest = std::min({sys->box[0], sys->box[1], sys->box[2]});
    if (r->rmax > 0.5 * smallest)  // rdf.cpp:56-63
        return fail(MD_ERR_INVALID_ARGUMENT,
                    "Rdf: rMax exceeds half the smallest box length; minimum-image distances "
                    "beyond that are ambiguous");
    md_context* ctx = r->ctx;
    const int64_t n = sys->n;
    const int64_t selected = n > first ? (n - first + stride - 1) / stride : 0;
    if (selected > 1 && r->bins > 0 && r->rmax > 0.0) {
        RdfArgs a;
        a.box = box_of_system(sys);
        a.rmax = r->rmax;
        a.rmax2_hi = r->rmax * r->rmax * (1.0 + 1e-12);
        a.width = r->width;
        a.bins = static_cast<int>(std::min<int64_t>(r->bins, 0x7fffffff));
        a.use_shared = r->bins <= kRdfSharedBins ? 1 : 0;
        a.first = first;
        a.stride = stride;
        const size_t shm = a.use_shared ? sizeof(unsigned) * static_cast<size_t>(r->bins) : 0;
        if (!r->grid.rank_of_cell || r->grid_box[0] != sys->box[0] ||
            r->grid_box[1] != sys->box[1] || r->grid_box[2] != sys->box[2]) {
            MDB_TRY(r->grid.init(sys->box, r->rmax));  // cells of width >= rMax
            for (int d = 0; d < 3; ++d) r->grid_box[d] = sys->box[d];
        }
        if (r->grid.usable) {
            MDB_TRY(r->sorted.ensure(sizeof(int) * static_cast<size_t>(n)));
            MDB_TRY(r->start.ensure(sizeof(int) * static_cast<size_t>(r->grid.ncells + 1)));
            MDB_TRY(cell_sort(sys, r->grid, r->sorted.as<int>(), r->start.as<int>()));
            RdfGrid g{r->grid.nx, r->grid.ny, r->grid.nz, r->grid.ncells, r->grid.rank_of_cell,
                      r->grid.cell_of_rank, r->start.as<int>(), r->sorted.as<int>()};
            k_rdf_cells<<<grid_for(n, kRdfBlock), kRdfBlock, shm, ctx->stream>>>(
                sys->cur.pos, n, g, a, r->hist.as<unsigned long long>());
        } else {
            // spans of a multiple of 32 atoms, enough of them for two blocks per SM
            const int64_t xblocks = grid_for(n, kRdfBlock);
            const int64_t want = (2 * static_cast<int64_t>(ctx->sm_count) + xblocks - 1) / xblocks;
            int64_t span = (n + want - 1) / want;
            span = std::min<int64_t>(kRdfBlock, std::max<int64_t>(32, (span + 31) / 32 * 32));
            const int64_t spans = (n + span - 1) / span;
            if (spans > 65535)
                return fail(MD_ERR_INVALID_ARGUMENT,
                            "Rdf: %lld atoms in a box under 3 rMax wide exceed the all-pairs pass",
                            static_cast<long long>(n));
            k_rdf_brute<<<dim3(static_cast<unsigned>(xblocks), static_cast<unsigned>(spans)),
                          kRdfBlock, shm, ctx->stream>>>(sys->cur.pos, n, static_cast<int>(span), a,
                                                         r->hist.as<unsigned long long>());
        }
        ++ctx->launches;
        MDB_CHECK_LAUNCH();
    }
    return MD_OK;
}

int rdf_sync(const md_rdf* r) {
    if (!r->stale) return MD_OK;
    std::vector<unsigned long long> h(static_cast<size_t>(r->bins));
    MDB_CUDA(cudaMemcpyAsync(h.data(), r->hist.ptr, sizeof(unsigned long long) * r->bins,
                             cudaMemcpyDeviceToHost, r->ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(r->ctx->stream));
    for (int64_t k = 0; k < r->bins; ++k) r->host[k] = static_cast<double>(h[k]);
    r->stale = false;
    return MD_OK;
}

}  // namespace mdb

extern "C" {

int md_rdf_bin_centres(const md_rdf* r, double* centres) {
    if (!r || (!centres && r->bins > 0))
        return fail(MD_ERR_INVALID_ARGUMENT, "md_rdf_bin_centres: NULL argument");
    for (int64_t k = 0; k < r->bins; ++k)  // rdf.cpp:84-90
        centres[k] = (static_cast<double>(k) + 0.5) * r->width;
    return MD_OK;
}

int md_rdf_g(const md_rdf* r, double* g) {
    if (!r || (!g && r->bins > 0)) return fail(MD_ERR_INVALID_ARGUMENT, "md_rdf_g: NULL argument");
    const double pi = 3.14159265358979323846;
    MDB_TRY(rdf_sync(r));
    for (int64_t k = 0; k < r->bins; ++k) g[k] = 0.0;
    if (r->frames == 0) return MD_OK;
    const double rho = r->sum_rho / static_cast<double>(r->frames);  // rdf.cpp:97-105
    for (int64_t k = 0; k < r->bins; ++k) {
        const double lo = static_cast<double>(k) * r->width;
        const double hi = static_cast<double>(k + 1) * r->width;
        const double shell = (4.0 / 3.0) * pi * (hi * hi * hi - lo * lo * lo);
        const double denom = static_cast<double>(r->frames) * 0.5 *
                             static_cast<double>(r->natoms) * rho * shell;
        g[k] = denom > 0.0 ? r->host[k] / denom : 0.0;
    }
    return MD_OK;
}

int md_rdf_frames(const md_rdf* r, int64_t* frames) {
    if (!r || !frames) return fail(MD_ERR_INVALID_ARGUMENT, "md_rdf_frames: NULL argument");
    *frames = r->frames;
    return MD_OK;
}

// ------------------------------------------------------------------------ MSD
int md_msd_create(md_context* ctx, int64_t natoms, int64_t max_lag, md_msd** out) {
    graph_epoch_bump();
    if (!out) return fail(MD_ERR_INVALID_ARGUMENT, "md_msd_create: NULL argument");
    md_msd* m = new (std::nothrow) md_msd;
    if (!m) return fail(MD_ERR_RUNTIME, "md_msd_create: out of host memory");
    const int rc = corr_create(ctx, natoms, max_lag, true, m, "md_msd_create");
    if (rc != MD_OK) {
        md_msd_destroy(m);
        return rc;
    }
    *out = m;
    return MD_OK;
}

int md_msd_destroy(md_msd* m) {
    graph_epoch_bump();
    if (!m) return MD_OK;
    if (m->ctx) cudaStreamSynchronize(m->ctx->stream);
    m->prev.release();
    m->unwrapped.release();
    m->ring.release();
    m->part.release();
    m->sums.release();
    delete m;
    return MD_OK;
}

int md_msd_push(md_msd* m, md_system* sys) {
    if (!m) return fail(MD_ERR_INVALID_ARGUMENT, "md_msd_push: NULL argument");
    return corr_push(m, sys, true, "md_msd_push");
}

int md_msd_values(const md_msd* m, double* out) {
    if (!m || !out) return fail(MD_ERR_INVALID_ARGUMENT, "md_msd_values: NULL argument");
    const std::vector<double> r = corr_means(m);
    std::copy(r.begin(), r.end(), out);
    return MD_OK;
}

int md_msd_diffusion(const md_msd* m, double dt, int64_t fit_from, int64_t fit_to, double* d) {
    if (!m || !d) return fail(MD_ERR_INVALID_ARGUMENT, "md_msd_diffusion: NULL argument");
    const std::vector<double> v = corr_means(m);  // msd.cpp:108-135
    const int64_t upper = std::min<int64_t>(fit_to, static_cast<int64_t>(v.size()));
    double st = 0.0, sm = 0.0, stt = 0.0, stm = 0.0;
    int64_t cnt = 0;
    for (int64_t k = std::max<int64_t>(fit_from, 0); k < upper; ++k) {
        const double t = static_cast<double>(k) * dt;
        st += t;
        sm += v[k];
        stt += t * t;
        stm += t * v[k];
        ++cnt;
    }
    *d = 0.0;
    if (cnt < 2) return MD_OK;
    const double nd = static_cast<double>(cnt);
    const double denom = nd * stt - st * st;
    if (denom == 0.0) return MD_OK;
    *d = ((nd * stm - st * sm) / denom) / 6.0;
    return MD_OK;
}

// ----------------------------------------------------------------------- VACF
int md_vacf_create(md_context* ctx, int64_t natoms, int64_t max_lag, md_vacf** out) {
    graph_epoch_bump();
    if (!out) return fail(MD_ERR_INVALID_ARGUMENT, "md_vacf_create: NULL argument");
    md_vacf* v = new (std::nothrow) md_vacf;
    if (!v) return fail(MD_ERR_RUNTIME, "md_vacf_create: out of host memory");
    const int rc = corr_create(ctx, natoms, max_lag, false, v, "md_vacf_create");
    if (rc != MD_OK) {
        md_vacf_destroy(v);
        return rc;
    }
    *out = v;
    return MD_OK;
}

int md_vacf_destroy(md_vacf* v) {
    graph_epoch_bump();
    if (!v) return MD_OK;
    if (v->ctx) cudaStreamSynchronize(v->ctx->stream);
    v->ring.release();
    v->part.release();
    v->sums.release();
    delete v;
    return MD_OK;
}

int md_vacf_push(md_vacf* v, md_system* sys) {
    if (!v) return fail(MD_ERR_INVALID_ARGUMENT, "md_vacf_push: NULL argument");
    return corr_push(v, sys, false, "md_vacf_push");
}

int md_vacf_values(const md_vacf* v, int normalised, double* out) {
    if (!v || !out) return fail(MD_ERR_INVALID_ARGUMENT, "md_vacf_values: NULL argument");
    std::vector<double> u = corr_means(v);  // vacf.cpp:218-239
    if (normalised) {
        const double c0 = u.empty() ? 0.0 : u[0];
        for (double& x : u) x = c0 == 0.0 ? 0.0 : x / c0;
    }
    std::copy(u.begin(), u.end(), out);
    return MD_OK;
}

int md_vacf_diffusion(const md_vacf* v, double dt, double* d) {
    if (!v || !d) return fail(MD_ERR_INVALID_ARGUMENT, "md_vacf_diffusion: NULL argument");
    const std::vector<double> u = corr_means(v);  // vacf.cpp:241-261
    int64_t valid = 0;
    for (int64_t lag = 0; lag < v->period; ++lag) {
        if (v->count[lag] == 0) break;
        valid = lag + 1;
    }
    *d = 0.0;
    if (valid < 2) return MD_OK;
    double integral = 0.0;
    for (int64_t lag = 0; lag + 1 < valid; ++lag) integral += 0.5 * (u[lag] + u[lag + 1]) * dt;
    *d = integral / 3.0;
    return MD_OK;
}

}  // extern "C"
