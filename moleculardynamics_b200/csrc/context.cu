// context.cu -- error state, device context, scratch management.
#include <atomic>
#include <cstdio>
#include <cstdarg>
#include <cstring>
#include <new>

#include "md_internal.cuh"

namespace mdb {

namespace {
thread_local std::string g_last_error;
std::atomic<uint64_t> g_graph_epoch{1};
}

uint64_t graph_epoch() { return g_graph_epoch.load(std::memory_order_acquire); }
void graph_epoch_bump() { g_graph_epoch.fetch_add(1, std::memory_order_acq_rel); }

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int DevBuf::ensure(size_t want) {
    if (want <= bytes && ptr) return MD_OK;
    graph_epoch_bump();  // a captured graph may hold the old address
    if (ptr) {
        // Work already queued may still read the old buffer.
        cudaDeviceSynchronize();
        cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    size_t alloc = want < 256 ? 256 : want;
    cudaError_t e = cudaMalloc(&ptr, alloc);
    if (e != cudaSuccess) {
        ptr = nullptr;
        cudaGetLastError();
        return fail(MD_ERR_OUT_OF_MEMORY, "cudaMalloc(%zu) failed: %s", alloc,
                    cudaGetErrorString(e));
    }
    bytes = alloc;
    return MD_OK;
}

void DevBuf::release() {
    if (ptr) {
        graph_epoch_bump();
        cudaFree(ptr);
    }
    ptr = nullptr;
    bytes = 0;
}

int ctx_partials(md_context* ctx, size_t doubles, double** out) {
    MDB_TRY(ctx->partials.ensure(doubles * sizeof(double)));
    *out = ctx->partials.as<double>();
    return MD_OK;
}

int ctx_scratch(md_context* ctx, size_t bytes, void** out) {
    MDB_TRY(ctx->scratch.ensure(bytes));
    *out = ctx->scratch.ptr;
    return MD_OK;
}

int ctx_read_results(md_context* ctx, int first, int count, double* out) {
    MDB_CUDA(cudaMemcpyAsync(ctx->h_result + first, ctx->result.as<double>() + first,
                             sizeof(double) * static_cast<size_t>(count), cudaMemcpyDeviceToHost,
                             ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    std::memcpy(out, ctx->h_result + first, sizeof(double) * static_cast<size_t>(count));
    return ctx_check_status(ctx);
}

int ctx_check_status(md_context* ctx) {
    uint32_t st = 0;
    MDB_CUDA(cudaMemcpyAsync(&st, ctx->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                             ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    if (st == 0) return MD_OK;
    // reported once: clear the word so the context can be used again
    MDB_CUDA(cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    return fail(MD_ERR_DEVICE, "device status 0x%x (%s%s%s%s%s%s)", st,
                (st & MD_STATUS_NEIGHBOR_OVERFLOW) ? "neighbour overflow " : "",
                (st & MD_STATUS_SHAKE_DIVERGED) ? "SHAKE diverged " : "",
                (st & MD_STATUS_RATTLE_DIVERGED) ? "RATTLE diverged " : "",
                (st & MD_STATUS_SHAKE_SINGULAR) ? "SHAKE singular " : "",
                (st & MD_STATUS_NONFINITE) ? "non-finite state " : "",
                (st & MD_STATUS_WAIT_TIMEOUT) ? "bounded wait ran out" : "");
}

void ctx_time_begin(md_context* ctx, int kernel) {
    if (!ctx->timing || kernel < 0 || kernel >= kTimedKernels) return;
    KernelTimer& t = ctx->timers[kernel];
    if (static_cast<size_t>(2 * t.used + 2) > t.ev.size()) {
        cudaEvent_t a, b;
        if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return;
        t.ev.push_back(a);
        t.ev.push_back(b);
    }
    cudaEventRecord(t.ev[2 * t.used], ctx->stream);
}

void ctx_time_end(md_context* ctx, int kernel) {
    if (!ctx->timing || kernel < 0 || kernel >= kTimedKernels) return;
    KernelTimer& t = ctx->timers[kernel];
    if (static_cast<size_t>(2 * t.used + 2) > t.ev.size()) return;
    cudaEventRecord(t.ev[2 * t.used + 1], ctx->stream);
    ++t.used;
}

// Folds recorded event pairs into the running totals (synchronises).
static int ctx_collect(md_context* ctx) {
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < kTimedKernels; ++k) {
        KernelTimer& t = ctx->timers[k];
        for (int u = 0; u < t.used; ++u) {
            float ms = 0.0f;
            MDB_CUDA(cudaEventElapsedTime(&ms, t.ev[2 * u], t.ev[2 * u + 1]));
            t.total_ms += ms;
            ++t.launches;
        }
        t.used = 0;
    }
    return MD_OK;
}

}  // namespace mdb

using namespace mdb;

extern "C" {

const char* md_last_error(void) { return g_last_error.c_str(); }

int md_abi_version(void) { return 10000; }

int md_context_create(int device, md_context** out) {
    if (!out) return fail(MD_ERR_INVALID_ARGUMENT, "md_context_create: out is NULL");
    *out = nullptr;
    int count = 0;
    MDB_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_context_create: device %d of %d", device, count);
    MDB_CUDA(cudaSetDevice(device));
    md_context* ctx = new (std::nothrow) md_context();
    if (!ctx) return fail(MD_ERR_OUT_OF_MEMORY, "md_context_create: host allocation");
    ctx->device = device;
    cudaDeviceProp prop;
    MDB_CUDA(cudaGetDeviceProperties(&prop, device));
    ctx->sm_count = prop.multiProcessorCount;
    MDB_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    MDB_CUDA(cudaMalloc(&ctx->d_status, sizeof(uint32_t)));
    MDB_CUDA(cudaMemset(ctx->d_status, 0, sizeof(uint32_t)));
    MDB_CUDA(cudaMalloc(&ctx->d_counter, sizeof(unsigned) * kCounterSlots));
    MDB_CUDA(cudaMemset(ctx->d_counter, 0, sizeof(unsigned) * kCounterSlots));
    MDB_TRY(ctx->result.ensure(sizeof(double) * kMaxResults));
    // Reduction partials sized once for grids up to 256k blocks x 4 values, so the
    // buffer is never reallocated under queued kernels.
    MDB_TRY(ctx->partials.ensure(sizeof(double) * (size_t(1) << 20)));
    MDB_CUDA(cudaMemset(ctx->result.ptr, 0, sizeof(double) * kMaxResults));
    MDB_CUDA(cudaMallocHost(&ctx->h_result, sizeof(double) * kMaxResults));
    MDB_CUDA(cudaDeviceSynchronize());
    graph_epoch_bump();
    *out = ctx;
    return MD_OK;
}

int md_context_destroy(md_context* ctx) {
    if (!ctx) return MD_OK;
    graph_epoch_bump();
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->partials.release();
    ctx->scratch.release();
    ctx->result.release();
    if (ctx->h_result) cudaFreeHost(ctx->h_result);
    if (ctx->d_status) cudaFree(ctx->d_status);
    if (ctx->d_counter) cudaFree(ctx->d_counter);
    for (auto& t : ctx->timers)
        for (cudaEvent_t e : t.ev) cudaEventDestroy(e);
    if (ctx->span_start) cudaEventDestroy(ctx->span_start);
    if (ctx->span_stop) cudaEventDestroy(ctx->span_stop);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return MD_OK;
}

int md_context_synchronize(md_context* ctx) {
    if (!ctx) return fail(MD_ERR_INVALID_ARGUMENT, "md_context_synchronize: NULL context");
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    return ctx_check_status(ctx);
}

int md_context_device_name(const md_context* ctx, char* name, int len) {
    if (!ctx || !name || len < 1) return fail(MD_ERR_INVALID_ARGUMENT, "md_context_device_name: bad argument");
    cudaDeviceProp prop;
    MDB_CUDA(cudaGetDeviceProperties(&prop, ctx->device));
    std::snprintf(name, static_cast<size_t>(len), "%s (%d SMs)", prop.name, prop.multiProcessorCount);
    return MD_OK;
}

int md_context_status(md_context* ctx, uint32_t* status, int clear) {
    if (!ctx || !status) return fail(MD_ERR_INVALID_ARGUMENT, "md_context_status: NULL argument");
    MDB_CUDA(cudaMemcpyAsync(status, ctx->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                             ctx->stream));
    if (clear) MDB_CUDA(cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    return MD_OK;
}

int md_context_set_timing(md_context* ctx, int enable) {
    if (!ctx) return fail(MD_ERR_INVALID_ARGUMENT, "md_context_set_timing: NULL");
    MDB_TRY(ctx_collect(ctx));
    ctx->timing = enable != 0;
    graph_epoch_bump();
    return MD_OK;
}

int md_context_set_graphs(md_context* ctx, int enable) {
    if (!ctx) return fail(MD_ERR_INVALID_ARGUMENT, "md_context_set_graphs: NULL");
    ctx->graphs = enable != 0;
    graph_epoch_bump();
    return MD_OK;
}

int md_context_kernel_time(md_context* ctx, int kernel, int reset, double* total_ms,
                           int64_t* launches) {
    if (!ctx || kernel < 0 || kernel >= kTimedKernels)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_context_kernel_time: bad argument");
    MDB_TRY(ctx_collect(ctx));
    KernelTimer& t = ctx->timers[kernel];
    if (total_ms) *total_ms = t.total_ms;
    if (launches) *launches = t.launches;
    if (reset) {
        t.total_ms = 0.0;
        t.launches = 0;
    }
    return MD_OK;
}

int md_context_span_begin(md_context* ctx) {
    if (!ctx) return fail(MD_ERR_INVALID_ARGUMENT, "md_context_span_begin: NULL");
    if (!ctx->span_start) {
        MDB_CUDA(cudaEventCreate(&ctx->span_start));
        MDB_CUDA(cudaEventCreate(&ctx->span_stop));
    }
    MDB_CUDA(cudaEventRecord(ctx->span_start, ctx->stream));
    return MD_OK;
}

int md_context_span_end(md_context* ctx, double* ms) {
    if (!ctx || !ms || !ctx->span_start)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_context_span_end: no span was begun");
    MDB_CUDA(cudaEventRecord(ctx->span_stop, ctx->stream));
    MDB_CUDA(cudaEventSynchronize(ctx->span_stop));
    float f = 0.0f;
    MDB_CUDA(cudaEventElapsedTime(&f, ctx->span_start, ctx->span_stop));
    *ms = f;
    return MD_OK;
}

void* md_host_alloc(size_t bytes) {
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        set_error("md_host_alloc: cudaMallocHost(%zu) failed", bytes);
        return nullptr;
    }
    return p;
}

int md_host_free(void* p) {
    if (p) MDB_CUDA(cudaFreeHost(p));
    return MD_OK;
}

int md_context_launch_count(md_context* ctx, int64_t* count) {
    if (!ctx || !count) return fail(MD_ERR_INVALID_ARGUMENT, "md_context_launch_count: NULL");
    *count = ctx->launches;
    return MD_OK;
}

int md_context_graph_captures(md_context* ctx, int64_t* count) {
    if (!ctx || !count) return fail(MD_ERR_INVALID_ARGUMENT, "md_context_graph_captures: NULL");
    *count = ctx->graph_captures;
    return MD_OK;
}

}  // extern "C"
