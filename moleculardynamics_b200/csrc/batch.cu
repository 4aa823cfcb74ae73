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
int verlet_build(md_verlet* v, md_system* sys, bool conditional);
}

namespace mdb {
// Per replica: its thermo rows (kept across runs, grown by doubling) and the
// device-held row index.
struct BatchRun {
    DevBuf rows, idx;
    int64_t cap = 0;
    int rebuilt0 = 0, rebuilt1 = 0;
};
struct BatchCache;  // the batched step graph kept across runs (below)
void batch_cache_destroy(BatchCache* c);
}  // namespace mdb

struct md_batch {
    struct Replica {
        md_integrator* it;
        md_system* sys;
        md_verlet* list;
        md_lj* lj;
    };
    std::vector<Replica> reps;
    int device = -1;
    int batched = 1;  // batched stage kernels when the replicas allow them
    std::vector<mdb::BatchRun> runs;
    mdb::BatchCache* cache = nullptr;
    ~md_batch() { mdb::batch_cache_destroy(cache); }
};

using namespace mdb;

namespace {

using Run = BatchRun;

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

// Captures work() from `stream` into graph g after deps; leaves (optional) gets
// the last captured nodes.  The stream leaves capture whatever happened.
template <class F>
int capture_to(cudaStream_t stream, cudaGraph_t g, const cudaGraphNode_t* deps, size_t ndeps,
               F&& work, std::vector<cudaGraphNode_t>* leaves) {
    MDB_CUDA(cudaStreamBeginCaptureToGraph(stream, g, deps, nullptr, ndeps,
                                           cudaStreamCaptureModeThreadLocal));
    int rc = work();
    if (rc == MD_OK && leaves) {
        cudaStreamCaptureStatus st;
        const cudaGraphNode_t* out = nullptr;
        size_t nout = 0;
        if (cudaStreamGetCaptureInfo(stream, &st, nullptr, nullptr, &out, &nout) != cudaSuccess)
            rc = fail(MD_ERR_CUDA, "md_batch_run: capture info");
        else leaves->assign(out, out + nout);
    }
    cudaGraph_t captured = nullptr;
    const cudaError_t e = cudaStreamEndCapture(stream, &captured);
    if (rc != MD_OK) return rc;
    if (e != cudaSuccess) return fail(MD_ERR_CUDA, "md_batch_run: capture: %s", cudaGetErrorString(e));
    return MD_OK;
}

// The step graph of batched stage kernels: the chain halves and kick/drift of
// every replica in one launch (with each replica's rebuild test), the gated
// rebuild of every replica as one launch per stage (each replica's blocks leave
// at once unless its own test asked for a rebuild), then the force pass and the
// kick, kinetic energy, chain half and thermo row of every replica in three
// launches: about fifteen kernel nodes and no conditional node.  Per replica the
// work and its order are those of its solo step.
struct BatchedStep {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // the first step of a run (the chains' entry kinetic energies summed afresh)
    cudaGraph_t first_graph = nullptr;
    cudaGraphExec_t first_exec = nullptr;
    int64_t first_launches = 0;
    BatchKick* kick = nullptr;
    BatchForce* force = nullptr;
    BatchRebuild* rebuild = nullptr;
    int64_t lead_launches = 0;
    std::vector<int64_t> body_launches;
    ~BatchedStep() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (first_exec) cudaGraphExecDestroy(first_exec);
        if (first_graph) cudaGraphDestroy(first_graph);
        batch_kick_destroy(kick);
        batch_force_destroy(force);
        batch_rebuild_destroy(rebuild);
    }
};

}  // namespace

// The batched step graph of the last run, replayed by later runs while nothing it
// captured has changed: the process-wide graph epoch (any device buffer moved or
// a launch setting changed), the batched switch and the replica list.
struct mdb::BatchCache {
    BatchedStep step;
    std::vector<cudaEvent_t> ready;  // each replica's first step done, for the lead stream
    uint32_t* h_status = nullptr;    // pinned: each replica's status word after a run
    uint64_t epoch = 0;
    size_t nrep = 0;
    ~BatchCache() {
        for (cudaEvent_t e : ready)
            if (e) cudaEventDestroy(e);
        if (h_status) cudaFreeHost(h_status);
    }
};

void mdb::batch_cache_destroy(BatchCache* c) { delete c; }

namespace {

// Builds the batched step graph, or leaves bs.exec null when the replicas need
// the per-replica graph (kernels that cannot share a launch).
int build_batched_step(md_batch* b, std::vector<Run>& run, BatchedStep& bs) {
    const size_t nr = b->reps.size();
    if (cudaGraphCreate(&bs.graph, 0) != cudaSuccess) return fail(MD_ERR_CUDA, "cudaGraphCreate");
    std::vector<BatchRepView> views(nr);
    for (size_t k = 0; k < nr; ++k) {
        const auto& r = b->reps[k];
        views[k] = BatchRepView{r.it, r.sys, r.list, r.lj, run[k].rows.as<double>(),
                                run[k].idx.as<int>()};
    }
    std::vector<KickArgs> kicks(nr);
    for (size_t k = 0; k < nr; ++k) kicks[k] = integrator_kick_args(b->reps[k].it, b->reps[k].sys);
    if (batch_rebuild_create(views.data(), static_cast<int>(nr), &bs.rebuild) != MD_OK ||
        batch_force_create(views.data(), static_cast<int>(nr), kicks.data(), &bs.force) != MD_OK ||
        batch_kick_create(views.data(), static_cast<int>(nr), &bs.kick) != MD_OK) {
        cudaGetLastError();
        return MD_OK;  // not batchable: the caller uses the per-replica graph
    }
    cudaStream_t lead = b->reps[0].sys->ctx->stream;
    bs.body_launches.assign(nr, 0);
    MDB_TRY(capture_to(lead, bs.graph, nullptr, 0, [&]() -> int {
        MDB_TRY(batch_kick_pre(bs.kick, lead, &bs.lead_launches));
        MDB_TRY(batch_rebuild_launch(bs.rebuild, lead, &bs.lead_launches));
        MDB_TRY(batch_force_launch(bs.force, lead, &bs.lead_launches));
        return batch_kick_post(bs.kick, lead, &bs.lead_launches, batch_force_kicks(bs.force));
    }, nullptr));
    if (cudaGraphInstantiate(&bs.exec, bs.graph, 0) != cudaSuccess) {
        bs.exec = nullptr;
        return fail(MD_ERR_CUDA, "md_batch_run: batched graph instantiation failed");
    }
    if (cudaGraphCreate(&bs.first_graph, 0) != cudaSuccess) return fail(MD_ERR_CUDA, "cudaGraphCreate");
    MDB_TRY(capture_to(lead, bs.first_graph, nullptr, 0, [&]() -> int {
        MDB_TRY(batch_kick_first(bs.kick, lead, &bs.first_launches));
        MDB_TRY(batch_rebuild_launch(bs.rebuild, lead, &bs.first_launches));
        MDB_TRY(batch_force_launch(bs.force, lead, &bs.first_launches));
        return batch_kick_post(bs.kick, lead, &bs.first_launches, batch_force_kicks(bs.force));
    }, nullptr));
    if (cudaGraphInstantiate(&bs.first_exec, bs.first_graph, 0) != cudaSuccess) {
        bs.first_exec = nullptr;
        return fail(MD_ERR_CUDA, "md_batch_run: batched first-step graph instantiation failed");
    }
    return MD_OK;
}

}  // namespace

extern "C" {

int md_batch_create(md_batch** out) {
    graph_epoch_bump();
    if (!out) return fail(MD_ERR_INVALID_ARGUMENT, "md_batch_create: NULL");
    md_batch* b = new (std::nothrow) md_batch();
    if (!b) return fail(MD_ERR_OUT_OF_MEMORY, "md_batch_create: host allocation");
    *out = b;
    return MD_OK;
}

int md_batch_destroy(md_batch* b) {
    graph_epoch_bump();
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
    batch_cache_destroy(b->cache);  // the replica list is part of the cached graph
    b->cache = nullptr;
    if (index) *index = static_cast<int>(b->reps.size()) - 1;
    return MD_OK;
}

int md_batch_size(const md_batch* b) { return b ? static_cast<int>(b->reps.size()) : 0; }

int md_batch_set_batched(md_batch* b, int on) {
    graph_epoch_bump();
    if (!b) return fail(MD_ERR_INVALID_ARGUMENT, "md_batch_set_batched: NULL batch");
    b->batched = on ? 1 : 0;
    return MD_OK;
}

int md_batch_run(md_batch* b, int64_t steps, double* thermo) {
    if (!b) return fail(MD_ERR_INVALID_ARGUMENT, "md_batch_run: NULL batch");
    if (steps < 0) return fail(MD_ERR_INVALID_ARGUMENT, "md_batch_run: steps < 0");
    const size_t nr = b->reps.size();
    if (nr == 0 || steps == 0) return MD_OK;
    for (auto& r : b->reps) {
        MDB_TRY(verlet_ensure_ready(r.list, r.sys, "md_batch_run"));
        if (r.sys->n == 0) return fail(MD_ERR_INVALID_ARGUMENT, "md_batch_run: empty replica");
        verlet_halo_for_run(r.list, r.sys, r.lj);
    }
    MDB_CUDA(cudaSetDevice(b->device));
    if (b->runs.size() != nr) {
        batch_cache_destroy(b->cache);
        b->cache = nullptr;
        b->runs.clear();
        b->runs.resize(nr);
    }
    std::vector<Run>& run = b->runs;
    // Thermo rows persist across runs, grown by doubling (a move invalidates a cached
    // graph through the graph epoch).
    for (size_t k = 0; k < nr; ++k) {
        if (run[k].cap < steps) {
            const int64_t cap = std::max<int64_t>(steps, 2 * run[k].cap);
            MDB_TRY(run[k].rows.ensure(sizeof(double) * 4 * static_cast<size_t>(cap)));
            run[k].cap = cap;
        }
        MDB_TRY(run[k].idx.ensure(sizeof(int)));
    }
    // A run whose batched graphs are cached replays its first step too (that graph
    // sums the chains' entry kinetic energies afresh).  Otherwise step 0 of every
    // replica runs from the host, on the replica's own stream: it sizes every buffer
    // (the captured graphs must not allocate) and sums the chains' entry energies.
    const bool warm = b->batched && b->cache && b->cache->step.exec && b->cache->step.first_exec &&
                      b->cache->epoch == graph_epoch() && b->cache->nrep == nr;
    if (!warm) {
        for (size_t k = 0; k < nr; ++k) {
            auto& r = b->reps[k];
            MDB_CUDA(cudaMemsetAsync(run[k].idx.ptr, 0, sizeof(int), r.sys->ctx->stream));
            MDB_TRY(lj_fused_step(r.it, r.sys, r.list, r.lj, run[k].rows.as<double>(),
                                  run[k].idx.as<int>(), true));
        }
    }
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t lead = b->reps[0].sys->ctx->stream;
    int rc = MD_OK;
    std::vector<int64_t> main_l(nr, 0), body_l(nr, 0);
    bool batched_done = false;
    if ((steps > 1 || warm) && b->batched) {
        // the batched step graph of an earlier run while nothing it captured moved
        BatchCache* c = b->cache;
        if (!warm) {
            batch_cache_destroy(c);
            c = b->cache = new (std::nothrow) BatchCache();
            if (!c) return fail(MD_ERR_OUT_OF_MEMORY, "md_batch_run: host allocation");
            c->nrep = nr;
            MDB_TRY(build_batched_step(b, run, c->step));
            if (c->step.exec) {
                c->ready.assign(nr, nullptr);
                for (size_t k = 0; k < nr; ++k)
                    MDB_CUDA(cudaEventCreateWithFlags(&c->ready[k], cudaEventDisableTiming));
                MDB_CUDA(cudaMallocHost(&c->h_status, sizeof(uint32_t) * nr));
            }
            c->epoch = graph_epoch();
        }
        if (c->step.exec) {
            // the lead stream starts once every replica's stream has caught up
            for (size_t k = 0; k < nr; ++k) {
                MDB_CUDA(cudaEventRecord(c->ready[k], b->reps[k].sys->ctx->stream));
                MDB_CUDA(cudaStreamWaitEvent(lead, c->ready[k], 0));
            }
            md_context* lctx = b->reps[0].sys->ctx;
            MDB_TRY(batch_rebuild_prime(c->step.rebuild, lead, &lctx->launches));
            if (warm) {
                if (cudaGraphLaunch(c->step.first_exec, lead) != cudaSuccess)
                    return fail(MD_ERR_CUDA, "md_batch_run: graph launch failed");
                lctx->launches += c->step.first_launches;
            }
            for (int64_t s = 1; s < steps; ++s)
                if (cudaGraphLaunch(c->step.exec, lead) != cudaSuccess)
                    return fail(MD_ERR_CUDA, "md_batch_run: graph launch failed");
            lctx->launches += (steps - 1) * c->step.lead_launches;
            // The end of the run on the lead stream: the chains' pending scales, then
            // every replica's thermo rows, status word and energy/virial slots read
            // back, one synchronisation for all.
            MDB_TRY(batch_kick_finish(c->step.kick, lead, &lctx->launches));
            for (size_t k = 0; k < nr; ++k) {
                md_context* ctx = b->reps[k].sys->ctx;
                if (thermo)
                    MDB_CUDA(cudaMemcpyAsync(thermo + 4 * steps * static_cast<int64_t>(k),
                                             run[k].rows.ptr,
                                             sizeof(double) * 4 * static_cast<size_t>(steps),
                                             cudaMemcpyDeviceToHost, lead));
                MDB_CUDA(cudaMemcpyAsync(c->h_status + k, ctx->d_status, sizeof(uint32_t),
                                         cudaMemcpyDeviceToHost, lead));
                MDB_CUDA(cudaMemcpyAsync(ctx->h_result + kResEnergy, ctx_result(ctx, kResEnergy),
                                         2 * sizeof(double), cudaMemcpyDeviceToHost, lead));
            }
            MDB_CUDA(cudaStreamSynchronize(lead));
            int st = MD_OK;
            for (size_t k = 0; k < nr; ++k) {
                md_system* sys = b->reps[k].sys;
                if (c->h_status[k] != 0) {  // reported (and cleared) as ctx_check_status does
                    const int e = ctx_check_status(sys->ctx);
                    if (st == MD_OK) st = e;
                    continue;
                }
                sys->last_energy = sys->ctx->h_result[kResEnergy];
                sys->last_virial = sys->ctx->h_result[kResVirial];
            }
            return st;
        }
    }
    if (steps > 1 && !batched_done) {
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
        if (steps > 1 && !batched_done) {
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
        MDB_TRY(ctx_check_status(r.sys->ctx));
        double e[2];
        MDB_TRY(ctx_read_results(r.sys->ctx, kResEnergy, 2, e));
        r.sys->last_energy = e[0];
        r.sys->last_virial = e[1];
    }
    return MD_OK;
}

}  // extern "C"
