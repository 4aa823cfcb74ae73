// batch.cu -- many independent LJ replicas stepped together (no reference
// counterpart: the reference runs one system per process).
//
// Each replica is an ordinary (integrator, system, Verlet list, LJ) tuple on its
// own context, so it has its own stream, reduction partials, last-block tickets
// and result slots.  A batch run captures one fused step of every replica into a
// single CUDA graph: the replicas are independent chains of nodes (each with its
// own conditional rebuild node), so one graph launch per step lets the device
// run all replicas' kernels concurrently instead of one small system after the
// other.  A replica's trajectory is exactly the one md_run_lj gives it alone.
#include <algorithm>
#include <new>
#include <vector>

#include "md_device.cuh"
#include "md_internal.cuh"

namespace mdb {
int verlet_ensure_ready(md_verlet* v, md_system* sys, const char* who);
}

struct md_batch {
    struct Replica {
        md_integrator* it;
        md_system* sys;
        md_verlet* list;
        md_lj* lj;
    };
    std::vector<Replica> reps;
    int device = -1;
};

using namespace mdb;

namespace {

struct Run {
    DevBuf rows, idx;
    int rebuilt0 = 0, rebuilt1 = 0;
};

int check_replica(const md_batch* b, const md_batch::Replica& r) {
    if (!r.it || !r.sys || !r.list || !r.lj)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_batch_add: NULL argument");
    if (r.it->kind != 0 && r.it->kind != 2)
        return fail(MD_ERR_INVALID_ARGUMENT,
                    "md_batch_add: replicas step with velocity Verlet or a Nose-Hoover chain");
    for (const auto& o : b->reps) {
        if (o.sys->ctx == r.sys->ctx)
            return fail(MD_ERR_INVALID_ARGUMENT,
                        "md_batch_add: every replica needs its own context (stream and scratch)");
        if (o.it == r.it || o.sys == r.sys || o.list == r.list)
            return fail(MD_ERR_INVALID_ARGUMENT, "md_batch_add: replica objects must be distinct");
    }
    if (b->device >= 0 && r.sys->ctx->device != b->device)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_batch_add: replicas must share one device");
    return MD_OK;
}

int read_rebuilds(md_verlet* v, cudaStream_t s, int* out) {
    MDB_CUDA(cudaMemcpyAsync(out, v->d_rebuild_total, sizeof(int), cudaMemcpyDeviceToHost, s));
    return MD_OK;
}

}  // namespace

extern "C" {

int md_batch_create(md_batch** out) {
    if (!out) return fail(MD_ERR_INVALID_ARGUMENT, "md_batch_create: NULL");
    md_batch* b = new (std::nothrow) md_batch();
    if (!b) return fail(MD_ERR_OUT_OF_MEMORY, "md_batch_create: host allocation");
    *out = b;
    return MD_OK;
}

int md_batch_destroy(md_batch* b) {
    delete b;
    return MD_OK;
}

int md_batch_add(md_batch* b, md_integrator* it, md_system* sys, md_verlet* list, md_lj* lj,
                 int* index) {
    if (!b) return fail(MD_ERR_INVALID_ARGUMENT, "md_batch_add: NULL batch");
    const md_batch::Replica r{it, sys, list, lj};
    MDB_TRY(check_replica(b, r));
    if (b->device < 0) b->device = sys->ctx->device;
    b->reps.push_back(r);
    if (index) *index = static_cast<int>(b->reps.size()) - 1;
    return MD_OK;
}

int md_batch_size(const md_batch* b) { return b ? static_cast<int>(b->reps.size()) : 0; }

int md_batch_run(md_batch* b, int64_t steps, double* thermo) {
    if (!b) return fail(MD_ERR_INVALID_ARGUMENT, "md_batch_run: NULL batch");
    if (steps < 0) return fail(MD_ERR_INVALID_ARGUMENT, "md_batch_run: steps < 0");
    const size_t nr = b->reps.size();
    if (nr == 0 || steps == 0) return MD_OK;
    for (auto& r : b->reps) {
        MDB_TRY(verlet_ensure_ready(r.list, r.sys, "md_batch_run"));
        if (r.sys->n == 0) return fail(MD_ERR_INVALID_ARGUMENT, "md_batch_run: empty replica");
        verlet_halo_for_run(r.list, r.sys, r.lj, steps);
    }
    MDB_CUDA(cudaSetDevice(b->device));
    std::vector<Run> run(nr);
    // Step 0 of every replica from the host, on the replica's own stream: it sizes
    // every buffer (the captured graph must not allocate) and sums the chains'
    // entry kinetic energies.
    for (size_t k = 0; k < nr; ++k) {
        auto& r = b->reps[k];
        md_context* ctx = r.sys->ctx;
        if (thermo) {
            MDB_TRY(run[k].rows.ensure(sizeof(double) * 4 * static_cast<size_t>(steps)));
            MDB_TRY(run[k].idx.ensure(sizeof(int)));
            MDB_CUDA(cudaMemsetAsync(run[k].idx.ptr, 0, sizeof(int), ctx->stream));
        }
        MDB_TRY(lj_fused_step(r.it, r.sys, r.list, r.lj, run[k].rows.as<double>(),
                              run[k].idx.as<int>(), true));
    }
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t lead = b->reps[0].sys->ctx->stream;
    int rc = MD_OK;
    std::vector<int64_t> main_l(nr, 0), body_l(nr, 0);
    if (steps > 1) {
        if (cudaGraphCreate(&graph, 0) != cudaSuccess) return fail(MD_ERR_CUDA, "cudaGraphCreate");
        for (size_t k = 0; k < nr && rc == MD_OK; ++k) {
            auto& r = b->reps[k];
            rc = capture_lj_step_into(r.it, r.sys, r.list, r.lj, run[k].rows.as<double>(),
                                      run[k].idx.as<int>(), graph, &main_l[k], &body_l[k]);
        }
        if (rc == MD_OK && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
            rc = fail(MD_ERR_CUDA, "md_batch_run: graph instantiation failed");
        // the lead stream replays the graph once every replica's first step is done
        for (size_t k = 0; k < nr && rc == MD_OK; ++k) {
            md_context* ctx = b->reps[k].sys->ctx;
            MDB_CUDA(cudaStreamSynchronize(ctx->stream));
            MDB_TRY(read_rebuilds(b->reps[k].list, ctx->stream, &run[k].rebuilt0));
        }
        for (size_t k = 0; k < nr && rc == MD_OK; ++k)
            MDB_CUDA(cudaStreamSynchronize(b->reps[k].sys->ctx->stream));
        for (int64_t s = 1; s < steps && rc == MD_OK; ++s)
            if (cudaGraphLaunch(exec, lead) != cudaSuccess)
                rc = fail(MD_ERR_CUDA, "md_batch_run: graph launch failed");
        if (rc == MD_OK) MDB_CUDA(cudaStreamSynchronize(lead));
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (rc != MD_OK) return rc;
    for (size_t k = 0; k < nr; ++k) {
        auto& r = b->reps[k];
        md_context* ctx = r.sys->ctx;
        if (steps > 1) {
            MDB_TRY(read_rebuilds(r.list, ctx->stream, &run[k].rebuilt1));
            MDB_CUDA(cudaStreamSynchronize(ctx->stream));
            ctx->launches += (steps - 1) * main_l[k] +
                             static_cast<int64_t>(run[k].rebuilt1 - run[k].rebuilt0) * body_l[k];
        }
        if (r.it->kind == 2) MDB_TRY(nhc_apply_scale_async(r.it, r.sys));
        if (thermo)
            MDB_CUDA(cudaMemcpyAsync(thermo + 4 * steps * static_cast<int64_t>(k), run[k].rows.ptr,
                                     sizeof(double) * 4 * static_cast<size_t>(steps),
                                     cudaMemcpyDeviceToHost, ctx->stream));
    }
    for (size_t k = 0; k < nr; ++k) {
        auto& r = b->reps[k];
        MDB_CUDA(cudaStreamSynchronize(r.sys->ctx->stream));
        run[k].rows.release();
        run[k].idx.release();
        MDB_TRY(ctx_check_status(r.sys->ctx));
        double e[2];
        MDB_TRY(ctx_read_results(r.sys->ctx, kResEnergy, 2, e));
        r.sys->last_energy = e[0];
        r.sys->last_virial = e[1];
    }
    return MD_OK;
}

}  // extern "C"
