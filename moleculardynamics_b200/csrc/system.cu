// system.cu -- device structure-of-arrays System (core/system.{hpp,cpp}).
#include <new>

#include "md_device.cuh"
#include "md_internal.cuh"

namespace mdb {

namespace {

constexpr int kBlock = 256;

__global__ void k_system_init(md_atoms a, int* slot, int64_t n) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= n) return;
    a.pos[k] = make_double4(0.0, 0.0, 0.0, static_cast<double>(k));
    a.vx[k] = a.vy[k] = a.vz[k] = 0.0;
    a.fx[k] = a.fy[k] = a.fz[k] = 0.0;
    a.mass[k] = 1.0;
    a.inv_mass[k] = 1.0;
    a.charge[k] = 0.0;
    a.mol[k] = k;
    a.orig[k] = static_cast<int>(k);
    slot[k] = static_cast<int>(k);
}

__device__ __forceinline__ double* field_ptr(const md_atoms& a, int field) {
    switch (field) {
        case MD_FIELD_VX: return a.vx;
        case MD_FIELD_VY: return a.vy;
        case MD_FIELD_VZ: return a.vz;
        case MD_FIELD_FX: return a.fx;
        case MD_FIELD_FY: return a.fy;
        case MD_FIELD_FZ: return a.fz;
        case MD_FIELD_MASS: return a.mass;
        default: return a.charge;
    }
}

// dev[k] = staging[orig[k]]  (host order -> device order)
__global__ void k_set_field(md_atoms a, int field, const double* __restrict__ staging, int64_t n) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= n) return;
    const double v = staging[a.orig[k]];
    if (field <= MD_FIELD_Z) {
        double* p = reinterpret_cast<double*>(a.pos + k);
        p[field] = v;
    } else {
        field_ptr(a, field)[k] = v;
        if (field == MD_FIELD_MASS) a.inv_mass[k] = 1.0 / v;  // velocity_verlet.hpp:59
    }
}

// staging[orig[k]] = dev[k]  (device order -> host order)
__global__ void k_get_field(md_atoms a, int field, double* __restrict__ staging, int64_t n) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= n) return;
    double v;
    if (field <= MD_FIELD_Z) {
        const double* p = reinterpret_cast<const double*>(a.pos + k);
        v = p[field];
    } else {
        v = field_ptr(a, field)[k];
    }
    staging[a.orig[k]] = v;
}

__global__ void k_set_mol(md_atoms a, const int64_t* __restrict__ staging, int64_t n) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k < n) a.mol[k] = staging[a.orig[k]];
}

__global__ void k_get_mol(md_atoms a, int64_t* __restrict__ staging, int64_t n) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k < n) staging[a.orig[k]] = a.mol[k];
}

__global__ void k_permute(md_atoms src, md_atoms dst, const int* __restrict__ perm, int* slot,
                          int64_t n) {
    const int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (s >= n) return;
    const int k = perm[s];
    dst.pos[s] = src.pos[k];
    dst.vx[s] = src.vx[k];
    dst.vy[s] = src.vy[k];
    dst.vz[s] = src.vz[k];
    dst.fx[s] = src.fx[k];
    dst.fy[s] = src.fy[k];
    dst.fz[s] = src.fz[k];
    dst.mass[s] = src.mass[k];
    dst.inv_mass[s] = src.inv_mass[k];
    dst.charge[s] = src.charge[k];
    dst.mol[s] = src.mol[k];
    const int o = src.orig[k];
    dst.orig[s] = o;
    slot[o] = static_cast<int>(s);
}

__global__ void k_zero_forces(md_atoms a, int64_t n) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k < n) a.fx[k] = a.fy[k] = a.fz[k] = 0.0;
}

// system.cpp:124-131: sum 0.5*m*v^2, v^2 = vx*vx + vy*vy + vz*vz.
__device__ __forceinline__ void kinetic_body(const md_atoms& a, int64_t n, double* part,
                                             unsigned* ticket, double* out, unsigned block,
                                             unsigned nblocks) {
    double v[1] = {0.0};
    for (int64_t k = block * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<int64_t>(nblocks) * blockDim.x) {
        const double v2 = a.vx[k] * a.vx[k] + a.vy[k] * a.vy[k] + a.vz[k] * a.vz[k];
        v[0] += 0.5 * a.mass[k] * v2;
    }
    grid_reduce_at<1>(v, part, ticket, out, nullptr, block, nblocks);
}

__global__ void k_kinetic(md_atoms a, int64_t n, double* part, unsigned* ticket, double* out) {
    kinetic_body(a, n, part, ticket, out, blockIdx.x, gridDim.x);
}

// The kinetic energy of many systems in one launch: each block sums for the system
// its block table entry names, with that system's solo blocks (reduce_grid).
__global__ void k_batch_kinetic(const BatchKineticRep* __restrict__ reps, const int4* __restrict__ blk) {
    const int4 e = __ldg(blk + blockIdx.x);
    const BatchKineticRep& d = reps[e.x];
    kinetic_body(d.a, d.n, d.part, d.ticket, d.out, e.y, e.z);
}

// system.cpp:137-145 plus the total mass (system.cpp:148-151).
__global__ void k_momentum(md_atoms a, int64_t n, double* part, unsigned* ticket, double* out) {
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double m = a.mass[k];
        v[0] += m * a.vx[k];
        v[1] += m * a.vy[k];
        v[2] += m * a.vz[k];
        v[3] += m;
    }
    grid_reduce<4>(v, part, ticket, out);
}

// system.cpp:153-163: v -= p / M (skipped when M == 0).
__global__ void k_sub_com(md_atoms a, int64_t n, const double* __restrict__ pm) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= n) return;
    const double total = pm[3];
    if (total == 0.0) return;
    a.vx[k] -= pm[0] / total;
    a.vy[k] -= pm[1] / total;
    a.vz[k] -= pm[2] / total;
}

// apps/water_rdf.cpp:186-195: t = 2 KE / dof (system.cpp:133-135); when t > 0,
// v *= sqrt(target / t).  KE comes from the device result slot of k_kinetic,
// so the rescale needs no host round trip.
__global__ void k_rescale_temperature(md_atoms a, int64_t n, const double* __restrict__ ke,
                                      double dof, double target) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= n) return;
    const double t = 2.0 * ke[0] / dof;
    if (!(t > 0.0)) return;
    const double scale = sqrt(target / t);
    a.vx[k] *= scale;
    a.vy[k] *= scale;
    a.vz[k] *= scale;
}

int reduce_grid(md_system* sys) {
    // Enough blocks to fill the GPU, few enough partials to re-reduce cheaply.
    const int64_t want = (sys->n + kBlock - 1) / kBlock;
    const int cap = sys->ctx->sm_count * 8;
    return static_cast<int>(want < 1 ? 1 : (want > cap ? cap : want));
}

}  // namespace

int system_alloc_atoms(md_system* sys, md_atoms* a) {
    const size_t n = static_cast<size_t>(sys->n > 0 ? sys->n : 1);
    MDB_CUDA(cudaMalloc(&a->pos, n * sizeof(double4)));
    double** fields[] = {&a->vx, &a->vy, &a->vz, &a->fx, &a->fy, &a->fz,
                         &a->mass, &a->inv_mass, &a->charge};
    for (double** f : fields) MDB_CUDA(cudaMalloc(f, n * sizeof(double)));
    MDB_CUDA(cudaMalloc(&a->mol, n * sizeof(int64_t)));
    MDB_CUDA(cudaMalloc(&a->orig, n * sizeof(int)));
    return MD_OK;
}

void system_free_atoms(md_atoms* a) {
    void* ptrs[] = {a->pos, a->vx, a->vy, a->vz, a->fx, a->fy, a->fz, a->mass,
                    a->inv_mass, a->charge, a->mol, a->orig};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    *a = md_atoms();
}

int system_permute(md_system* sys, const int* d_perm) {
    if (sys->n == 0) return MD_OK;
    k_permute<<<grid_for(sys->n, kBlock), kBlock, 0, sys->ctx->stream>>>(sys->cur, sys->alt,
                                                                       d_perm, sys->slot, sys->n);
    ++sys->ctx->launches;
    MDB_CHECK_LAUNCH();
    md_atoms t = sys->cur;
    sys->cur = sys->alt;
    sys->alt = t;
    ++sys->epoch;
    graph_epoch_bump();  // the current arrays moved
    return MD_OK;
}

int batch_kinetic_launch(const BatchKineticRep* reps, const int4* blk, int blocks,
                         cudaStream_t stream) {
    if (blocks <= 0) return MD_OK;
    k_batch_kinetic<<<static_cast<unsigned>(blocks), kBlock, 0, stream>>>(reps, blk);
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

int system_kinetic_async(md_system* sys, int slot) {
    md_context* ctx = sys->ctx;
    const int g = reduce_grid(sys);
    double* part;
    MDB_TRY(ctx_partials(ctx, static_cast<size_t>(g), &part));
    k_kinetic<<<g, kBlock, 0, ctx->stream>>>(sys->cur, sys->n, part, ctx_counter(ctx, 0),
                                            ctx_result(ctx, slot));
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

}  // namespace mdb

using namespace mdb;

extern "C" {

int md_system_create(md_context* ctx, int64_t n, const double box[3], md_system** out) {
    graph_epoch_bump();
    if (!ctx || !box || !out) return fail(MD_ERR_INVALID_ARGUMENT, "md_system_create: NULL argument");
    if (n < 0 || n > (int64_t(1) << 31) - 1)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_system_create: n=%lld out of range",
                    static_cast<long long>(n));
    for (int d = 0; d < 3; ++d)
        if (!(box[d] > 0.0))
            return fail(MD_ERR_INVALID_ARGUMENT, "md_system_create: box lengths must be positive");
    MDB_CUDA(cudaSetDevice(ctx->device));
    md_system* sys = new (std::nothrow) md_system();
    if (!sys) return fail(MD_ERR_OUT_OF_MEMORY, "md_system_create: host allocation");
    sys->ctx = ctx;
    sys->n = n;
    for (int d = 0; d < 3; ++d) {
        sys->box[d] = box[d];
        sys->inv_box[d] = 1.0 / box[d];
    }
    int rc = system_alloc_atoms(sys, &sys->cur);
    if (rc == MD_OK) rc = system_alloc_atoms(sys, &sys->alt);
    if (rc == MD_OK) {
        cudaError_t e = cudaMalloc(&sys->slot, static_cast<size_t>(n > 0 ? n : 1) * sizeof(int));
        if (e != cudaSuccess) rc = fail(MD_ERR_OUT_OF_MEMORY, "md_system_create: %s", cudaGetErrorString(e));
    }
    if (rc != MD_OK) {
        md_system_destroy(sys);
        return rc;
    }
    if (n > 0) {
        k_system_init<<<grid_for(n, kBlock), kBlock, 0, ctx->stream>>>(sys->cur, sys->slot, n);
        ++ctx->launches;
        MDB_CHECK_LAUNCH();
    }
    *out = sys;
    return MD_OK;
}

int md_system_destroy(md_system* sys) {
    graph_epoch_bump();
    if (!sys) return MD_OK;
    if (sys->ctx) cudaStreamSynchronize(sys->ctx->stream);
    system_free_atoms(&sys->cur);
    system_free_atoms(&sys->alt);
    if (sys->slot) cudaFree(sys->slot);
    sys->qpos.release();
    delete sys;
    return MD_OK;
}

int64_t md_system_size(const md_system* sys) { return sys ? sys->n : -1; }

int md_system_box(const md_system* sys, double box[3]) {
    if (!sys || !box) return fail(MD_ERR_INVALID_ARGUMENT, "md_system_box: NULL argument");
    for (int d = 0; d < 3; ++d) box[d] = sys->box[d];
    return MD_OK;
}

int md_system_set(md_system* sys, int field, const double* src) {
    if (!sys || !src) return fail(MD_ERR_INVALID_ARGUMENT, "md_system_set: NULL argument");
    if (field < MD_FIELD_X || field > MD_FIELD_CHARGE)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_system_set: unknown field %d", field);
    if (sys->n == 0) return MD_OK;
    md_context* ctx = sys->ctx;
    void* staging;
    MDB_TRY(ctx_scratch(ctx, static_cast<size_t>(sys->n) * sizeof(double), &staging));
    MDB_CUDA(cudaMemcpyAsync(staging, src, static_cast<size_t>(sys->n) * sizeof(double),
                             cudaMemcpyHostToDevice, ctx->stream));
    k_set_field<<<grid_for(sys->n, kBlock), kBlock, 0, ctx->stream>>>(
        sys->cur, field, static_cast<const double*>(staging), sys->n);
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    // The staging buffer is reused by the next call: finish the host copy first.
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    return MD_OK;
}

int md_system_get(md_system* sys, int field, double* dst) {
    if (!sys || !dst) return fail(MD_ERR_INVALID_ARGUMENT, "md_system_get: NULL argument");
    if (field < MD_FIELD_X || field > MD_FIELD_CHARGE)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_system_get: unknown field %d", field);
    if (sys->n == 0) return MD_OK;
    md_context* ctx = sys->ctx;
    void* staging;
    MDB_TRY(ctx_scratch(ctx, static_cast<size_t>(sys->n) * sizeof(double), &staging));
    k_get_field<<<grid_for(sys->n, kBlock), kBlock, 0, ctx->stream>>>(
        sys->cur, field, static_cast<double*>(staging), sys->n);
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    MDB_CUDA(cudaMemcpyAsync(dst, staging, static_cast<size_t>(sys->n) * sizeof(double),
                             cudaMemcpyDeviceToHost, ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    return MD_OK;
}

int md_system_set_fields(md_system* sys, int count, const int* fields, const double* const* src) {
    if (!sys || count < 0 || (count > 0 && (!fields || !src)))
        return fail(MD_ERR_INVALID_ARGUMENT, "md_system_set_fields: NULL argument");
    for (int k = 0; k < count; ++k)
        if (fields[k] < MD_FIELD_X || fields[k] > MD_FIELD_CHARGE || !src[k])
            return fail(MD_ERR_INVALID_ARGUMENT, "md_system_set_fields: bad field %d", k);
    if (sys->n == 0 || count == 0) return MD_OK;
    md_context* ctx = sys->ctx;
    const size_t col = static_cast<size_t>(sys->n);
    void* staging;
    MDB_TRY(ctx_scratch(ctx, col * sizeof(double) * count, &staging));
    double* st = static_cast<double*>(staging);
    // every column's copy is queued before any scatter, so the copy engine
    // streams them back to back; one synchronisation for all
    for (int k = 0; k < count; ++k)
        MDB_CUDA(cudaMemcpyAsync(st + k * col, src[k], col * sizeof(double), cudaMemcpyHostToDevice,
                                 ctx->stream));
    for (int k = 0; k < count; ++k)
        k_set_field<<<grid_for(sys->n, kBlock), kBlock, 0, ctx->stream>>>(sys->cur, fields[k],
                                                                         st + k * col, sys->n);
    ctx->launches += count;
    MDB_CHECK_LAUNCH();
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    return MD_OK;
}

int md_system_get_fields(md_system* sys, int count, const int* fields, double* const* dst) {
    if (!sys || count < 0 || (count > 0 && (!fields || !dst)))
        return fail(MD_ERR_INVALID_ARGUMENT, "md_system_get_fields: NULL argument");
    for (int k = 0; k < count; ++k)
        if (fields[k] < MD_FIELD_X || fields[k] > MD_FIELD_CHARGE || !dst[k])
            return fail(MD_ERR_INVALID_ARGUMENT, "md_system_get_fields: bad field %d", k);
    if (sys->n == 0 || count == 0) return MD_OK;
    md_context* ctx = sys->ctx;
    const size_t col = static_cast<size_t>(sys->n);
    void* staging;
    MDB_TRY(ctx_scratch(ctx, col * sizeof(double) * count, &staging));
    double* st = static_cast<double*>(staging);
    for (int k = 0; k < count; ++k)
        k_get_field<<<grid_for(sys->n, kBlock), kBlock, 0, ctx->stream>>>(sys->cur, fields[k],
                                                                         st + k * col, sys->n);
    ctx->launches += count;
    MDB_CHECK_LAUNCH();
    for (int k = 0; k < count; ++k)
        MDB_CUDA(cudaMemcpyAsync(dst[k], st + k * col, col * sizeof(double), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    return MD_OK;
}

int md_system_set_molecule_ids(md_system* sys, const int64_t* ids) {
    graph_epoch_bump();
    if (!sys || !ids) return fail(MD_ERR_INVALID_ARGUMENT, "md_system_set_molecule_ids: NULL");
    if (sys->n == 0) return MD_OK;
    md_context* ctx = sys->ctx;
    void* staging;
    MDB_TRY(ctx_scratch(ctx, static_cast<size_t>(sys->n) * sizeof(int64_t), &staging));
    MDB_CUDA(cudaMemcpyAsync(staging, ids, static_cast<size_t>(sys->n) * sizeof(int64_t),
                             cudaMemcpyHostToDevice, ctx->stream));
    k_set_mol<<<grid_for(sys->n, kBlock), kBlock, 0, ctx->stream>>>(
        sys->cur, static_cast<const int64_t*>(staging), sys->n);
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    ++sys->mol_version;
    sys->has_molecules = false;
    for (int64_t i = 0; i < sys->n; ++i)
        if (ids[i] != i) {
            sys->has_molecules = true;
            break;
        }
    return MD_OK;
}

int md_system_get_molecule_ids(md_system* sys, int64_t* ids) {
    if (!sys || !ids) return fail(MD_ERR_INVALID_ARGUMENT, "md_system_get_molecule_ids: NULL");
    if (sys->n == 0) return MD_OK;
    md_context* ctx = sys->ctx;
    void* staging;
    MDB_TRY(ctx_scratch(ctx, static_cast<size_t>(sys->n) * sizeof(int64_t), &staging));
    k_get_mol<<<grid_for(sys->n, kBlock), kBlock, 0, ctx->stream>>>(
        sys->cur, static_cast<int64_t*>(staging), sys->n);
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    MDB_CUDA(cudaMemcpyAsync(ids, staging, static_cast<size_t>(sys->n) * sizeof(int64_t),
                             cudaMemcpyDeviceToHost, ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    return MD_OK;
}

int md_system_zero_forces(md_system* sys) {
    if (!sys) return fail(MD_ERR_INVALID_ARGUMENT, "md_system_zero_forces: NULL");
    if (sys->n == 0) return MD_OK;
    k_zero_forces<<<grid_for(sys->n, kBlock), kBlock, 0, sys->ctx->stream>>>(sys->cur, sys->n);
    ++sys->ctx->launches;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

int md_system_kinetic_energy(md_system* sys, double* ke) {
    if (!sys || !ke) return fail(MD_ERR_INVALID_ARGUMENT, "md_system_kinetic_energy: NULL");
    if (sys->n == 0) {
        *ke = 0.0;
        return MD_OK;
    }
    MDB_TRY(system_kinetic_async(sys, kResKE));
    return ctx_read_results(sys->ctx, kResKE, 1, ke);
}

int md_system_total_momentum(md_system* sys, double p[3]) {
    if (!sys || !p) return fail(MD_ERR_INVALID_ARGUMENT, "md_system_total_momentum: NULL");
    if (sys->n == 0) {
        p[0] = p[1] = p[2] = 0.0;
        return MD_OK;
    }
    md_context* ctx = sys->ctx;
    const int g = reduce_grid(sys);
    double* part;
    MDB_TRY(ctx_partials(ctx, static_cast<size_t>(g) * 4, &part));
    k_momentum<<<g, kBlock, 0, ctx->stream>>>(sys->cur, sys->n, part, ctx_counter(ctx, 0),
                                             ctx_result(ctx, kResMomentum));
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    double r[4];
    MDB_TRY(ctx_read_results(ctx, kResMomentum, 4, r));
    p[0] = r[0];
    p[1] = r[1];
    p[2] = r[2];
    return MD_OK;
}

int md_system_remove_com_motion(md_system* sys) {
    if (!sys) return fail(MD_ERR_INVALID_ARGUMENT, "md_system_remove_com_motion: NULL");
    if (sys->n == 0) return MD_OK;
    md_context* ctx = sys->ctx;
    const int g = reduce_grid(sys);
    double* part;
    MDB_TRY(ctx_partials(ctx, static_cast<size_t>(g) * 4, &part));
    k_momentum<<<g, kBlock, 0, ctx->stream>>>(sys->cur, sys->n, part, ctx_counter(ctx, 0),
                                             ctx_result(ctx, kResMomentum));
    k_sub_com<<<grid_for(sys->n, kBlock), kBlock, 0, ctx->stream>>>(sys->cur, sys->n,
                                                                    ctx_result(ctx, kResMomentum));
    ctx->launches += 2;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

int md_system_rescale_temperature(md_system* sys, int64_t dof, double target) {
    if (!sys) return fail(MD_ERR_INVALID_ARGUMENT, "md_system_rescale_temperature: NULL");
    if (dof < 1 || !(target >= 0.0))
        return fail(MD_ERR_INVALID_ARGUMENT, "md_system_rescale_temperature: dof >= 1, target >= 0");
    if (sys->n == 0) return MD_OK;
    MDB_TRY(system_kinetic_async(sys, kResKE));
    k_rescale_temperature<<<grid_for(sys->n, kBlock), kBlock, 0, sys->ctx->stream>>>(
        sys->cur, sys->n, ctx_result(sys->ctx, kResKE), static_cast<double>(dof), target);
    ++sys->ctx->launches;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

int md_system_last_energy(md_system* sys, double* energy, double* virial) {
    if (!sys) return fail(MD_ERR_INVALID_ARGUMENT, "md_system_last_energy: NULL");
    double r[2];
    MDB_TRY(ctx_read_results(sys->ctx, kResEnergy, 2, r));
    sys->last_energy = r[0];
    sys->last_virial = r[1];
    if (energy) *energy = r[0];
    if (virial) *virial = r[1];
    return MD_OK;
}

}  // extern "C"
