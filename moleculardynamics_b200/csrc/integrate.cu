// integrate.cu -- velocity-Verlet, BAOAB Langevin and Nose-Hoover-chain steps.
//
// Per-atom updates follow the reference's arithmetic exactly (std::fma ->
// fma(), wrap -> bit-exact fold), so one step from the same forces reproduces the
// reference's positions and velocities bit-for-bit.  The Nose-Hoover chain keeps
// its scalars on the device and tracks the kinetic energy analytically through
// the velocity rescalings (KE * s^2) instead of re-summing it after each of the six
// rescalings per step; the rescalings are folded into one factor applied by the
// next kick.
#include <cmath>
#include <new>
#include <vector>

#include "md_device.cuh"
#include "md_internal.cuh"

namespace mdb {
int verlet_ensure_ready(md_verlet* v, md_system* sys, const char* who);
DispArgs disp_args(md_verlet* v, md_context* ctx, double* part);
}  // namespace mdb

namespace mdb {

namespace {

constexpr int kBlock = 256;

struct StepArgs {
    Box3 box;
    double dt, half_dt;
    // BAOAB
    double c1, c2, temperature;
    uint32_t key0, key1;
    uint64_t step;
    const double* noise;  // replayed normals for this step (original order), or null
    uint32_t* status;     // MD_STATUS_NONFINITE when a position stops being finite
    int4* q;              // fixed-point copy of the new positions for the mixed force, or null
    double qs[3];         // 2^32 / L per axis
};

__device__ __forceinline__ void check_finite(const double4& p, uint32_t* status) {
    if (!(isfinite(p.x) && isfinite(p.y) && isfinite(p.z))) atomicOr(status, MD_STATUS_NONFINITE);
}

// Squared min-image displacement of a freshly moved atom from its position at the
// last Verlet build (for the fused rebuild check).
__device__ __forceinline__ double disp2(const Fold3& f3, double4 p, double4 q) {
    double dx, dy, dz;
    min_image_wrapped(f3, p.x, p.y, p.z, q.x, q.y, q.z, dx, dy, dz);
    return norm2_exact(dx, dy, dz);
}

// velocity_verlet.hpp:55-65 (+ an optional NHC pending scale applied first).  With
// CHECK the kernel also reduces the top-2 displacement since the last Verlet build
// and writes the device rebuild flag (verlet_list.cpp:44-63), saving a pass.
// `scaled`: a chain's pending velocity scale `sc` is applied first.  A block moves
// ATOMS * blockDim.x atoms, each thread every blockDim.x-th of them; the top-2
// displacement is exact whatever the blocking.
template <bool CHECK, int ATOMS = 1>
__device__ __forceinline__ void kick_drift_scaled(md_atoms a, int64_t n, const StepArgs& s,
                                                  bool scaled, double sc, const DispArgs& d,
                                                  unsigned block, unsigned nblocks) {
    double a1 = 0.0, a2 = 0.0;
#pragma unroll
    for (int u = 0; u < ATOMS; ++u) {
        const int64_t k = (block * static_cast<int64_t>(ATOMS) + u) * blockDim.x + threadIdx.x;
        if (k < n) {
            double vx = a.vx[k], vy = a.vy[k], vz = a.vz[k];
            if (scaled) {
                vx = __dmul_rn(vx, sc);
                vy = __dmul_rn(vy, sc);
                vz = __dmul_rn(vz, sc);
            }
            const double c = __dmul_rn(s.half_dt, a.inv_mass[k]);
            vx = fma(c, a.fx[k], vx);
            vy = fma(c, a.fy[k], vy);
            vz = fma(c, a.fz[k], vz);
            const Fold3 f3 = fold3_of(s.box);
            double4 p = a.pos[k];
            p.x = fold_wrapped(fma(s.dt, vx, p.x), f3.b[0]);
            p.y = fold_wrapped(fma(s.dt, vy, p.y), f3.b[1]);
            p.z = fold_wrapped(fma(s.dt, vz, p.z), f3.b[2]);
            check_finite(p, s.status);
            a.pos[k] = p;
            a.vx[k] = vx;
            a.vy[k] = vy;
            a.vz[k] = vz;
            if (s.q) s.q[k] = quantize_position(p, s.qs[0], s.qs[1], s.qs[2]);
            if (CHECK) {
                const double x = disp2(f3, p, d.ref[k]);
                if (u == 0) a1 = x;
                else top2_insert(a1, a2, x);
            }
        }
    }
    if (CHECK) top2_grid_at(a1, a2, d, block, nblocks);
}

template <bool CHECK, int ATOMS = 1>
__device__ __forceinline__ void kick_drift_body(md_atoms a, int64_t n, const StepArgs& s,
                                                const NhcState* nhc, const DispArgs& d,
                                                unsigned block, unsigned nblocks) {
    kick_drift_scaled<CHECK, ATOMS>(a, n, s, nhc != nullptr, nhc ? nhc->scale : 1.0, d, block,
                                    nblocks);
}

// At most 48 registers: five 256-thread blocks per SM keep enough loads in flight
// (the kernel streams ~190 bytes per atom and waits on memory, not arithmetic);
// kKickAtoms atoms per thread.
constexpr int kKickAtoms = 2;

template <bool CHECK>
__global__ void __launch_bounds__(kBlock, 5)
k_kick_drift(md_atoms a, int64_t n, StepArgs s, const NhcState* nhc, DispArgs d) {
    kick_drift_body<CHECK, kKickAtoms>(a, n, s, nhc, d, blockIdx.x, gridDim.x);
}

// langevin.hpp:55-80: B, A (wrap), O, A (wrap).
template <bool CHECK>
__global__ void k_baoab_pre(md_atoms a, int64_t n, StepArgs s, DispArgs d) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    double a1 = 0.0;
    if (k < n) {
        const Fold3 f3 = fold3_of(s.box);
        const double c = __dmul_rn(s.half_dt, a.inv_mass[k]);
        double vx = fma(c, a.fx[k], a.vx[k]);
        double vy = fma(c, a.fy[k], a.vy[k]);
        double vz = fma(c, a.fz[k], a.vz[k]);
        double4 p = a.pos[k];
        p.x = fold_wrapped(fma(s.half_dt, vx, p.x), f3.b[0]);
        p.y = fold_wrapped(fma(s.half_dt, vy, p.y), f3.b[1]);
        p.z = fold_wrapped(fma(s.half_dt, vz, p.z), f3.b[2]);
        // O: v = c1*v + (c2*sqrt(T/m)) * xi
        const int o = a.orig[k];
        double x0, x1, x2;
        if (s.noise) {
            x0 = s.noise[3 * static_cast<int64_t>(o) + 0];
            x1 = s.noise[3 * static_cast<int64_t>(o) + 1];
            x2 = s.noise[3 * static_cast<int64_t>(o) + 2];
        } else {
            const U4 r0 = philox4x32_10(U4{static_cast<uint32_t>(o), 0u, static_cast<uint32_t>(s.step),
                                           static_cast<uint32_t>(s.step >> 32)},
                                        s.key0, s.key1);
            const U4 r1 = philox4x32_10(U4{static_cast<uint32_t>(o), 1u, static_cast<uint32_t>(s.step),
                                           static_cast<uint32_t>(s.step >> 32)},
                                        s.key0, s.key1);
            double x3;
            normal2(r0, x0, x1);
            normal2(r1, x2, x3);
        }
        const double sig = __dsqrt_rn(__ddiv_rn(s.temperature, a.mass[k]));
        const double sc = __dmul_rn(s.c2, sig);
        vx = __dadd_rn(__dmul_rn(s.c1, vx), __dmul_rn(x0, sc));
        vy = __dadd_rn(__dmul_rn(s.c1, vy), __dmul_rn(x1, sc));
        vz = __dadd_rn(__dmul_rn(s.c1, vz), __dmul_rn(x2, sc));
        p.x = fold_wrapped(fma(s.half_dt, vx, p.x), f3.b[0]);
        p.y = fold_wrapped(fma(s.half_dt, vy, p.y), f3.b[1]);
        p.z = fold_wrapped(fma(s.half_dt, vz, p.z), f3.b[2]);
        check_finite(p, s.status);
        a.pos[k] = p;
        a.vx[k] = vx;
        a.vy[k] = vy;
        a.vz[k] = vz;
        if (CHECK) a1 = disp2(f3, p, d.ref[k]);
    }
    if (CHECK) top2_grid(a1, 0.0, d);
}

// Second half-kick (velocity_verlet.hpp:70-73), fused with the kinetic-energy sum;
// true in the block that finished the sum.
__device__ __forceinline__ bool kick_ke_body(md_atoms a, int64_t n, const StepArgs& s, double* part,
                                             unsigned* ticket, double* out, uint32_t* status,
                                             unsigned block, unsigned nblocks) {
    double ke[1] = {0.0};
    for (int64_t k = block * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<int64_t>(nblocks) * blockDim.x) {
        const double c = __dmul_rn(s.half_dt, a.inv_mass[k]);
        const double vx = fma(c, a.fx[k], a.vx[k]);
        const double vy = fma(c, a.fy[k], a.vy[k]);
        const double vz = fma(c, a.fz[k], a.vz[k]);
        a.vx[k] = vx;
        a.vy[k] = vy;
        a.vz[k] = vz;
        ke[0] += 0.5 * a.mass[k] * (vx * vx + vy * vy + vz * vz);
    }
    return grid_reduce_at<1>(ke, part, ticket, out, status, block, nblocks);  // a NaN reaches the KE
}

__global__ void k_kick_ke(md_atoms a, int64_t n, StepArgs s, double* part, unsigned* ticket,
                          double* out, uint32_t* status) {
    kick_ke_body(a, n, s, part, ticket, out, status, blockIdx.x, gridDim.x);
}

__global__ void k_scale(md_atoms a, int64_t n, NhcState* nhc) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const double sc = nhc->scale;
    if (k < n) {
        a.vx[k] = __dmul_rn(a.vx[k], sc);
        a.vy[k] = __dmul_rn(a.vy[k], sc);
        a.vz[k] = __dmul_rn(a.vz[k], sc);
    }
}

__global__ void k_reset_scale(NhcState* nhc) { nhc->scale = 1.0; }

struct Weights {
    double w[3];
};

// nose_hoover.cpp:89-108 for link j of a chain in arrays of C slots (m links in use);
// ke is the current kinetic energy.  Explicit round-to-nearest products and sums (no
// contraction into FMAs; the division is IEEE), in the reference's order of
// operations.  Both damping factors of a link use p[j + 1] before the link changes
// p[j], so one exponential serves both.
template <int C>
__device__ __forceinline__ void chain_link(const double (&Q)[C], double (&p)[C], int j, int m,
                                           double d2, double d4, double ke, double dof,
                                           double temp) {
    const int up = j + 1 < C ? j + 1 : j;  // read only when j + 1 < m <= C
    const int dn = j > 0 ? j - 1 : 0;
    const bool next = j < m - 1;
    const double damp = next ? exp(__dmul_rn(-d4, p[up]) / Q[up]) : 1.0;
    if (next) p[j] = __dmul_rn(p[j], damp);
    const double g = j == 0 ? __dsub_rn(__dmul_rn(2.0, ke), __dmul_rn(dof, temp))
                            : __dsub_rn(__dmul_rn(p[dn], p[dn]) / Q[dn], temp);
    p[j] = __dadd_rn(p[j], __dmul_rn(d2, g));
    if (next) p[j] = __dmul_rn(p[j], damp);
}

// integrateChain(delta) (nose_hoover.cpp:59-124) with weights w on the chain of *st.
// With C > 0 the chain has exactly C links, held in registers: every loop unrolls,
// so no array is indexed at run time.  C = 0 takes any length up to kMaxChain, in
// arrays indexed at run time (local memory).  Returns the product of the velocity
// scale factors and updates ke to KE * scale^2.
template <int C>
__device__ double chain_half(NhcState* st, double delta, Weights w, double& ke) {
    constexpr int kSlots = C > 0 ? C : kMaxChain;
    constexpr int kUnroll = C > 0 ? C : 1;  // link loops: whole for C > 0, rolled for C = 0
    const int m = C > 0 ? C : st->chain;
    const double dof = st->dof, temp = st->temperature;
    double Q[kSlots], xi[kSlots], p[kSlots];
#pragma unroll kUnroll
    for (int k = 0; k < m; ++k) {
        Q[k] = st->Q[k];
        xi[k] = st->xi[k];
        p[k] = st->pxi[k];
    }
    double total = 1.0;
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        const double d = __dmul_rn(w.w[s], delta);
        const double d2 = 0.5 * d, d4 = 0.25 * d;
#pragma unroll kUnroll
        for (int j = m - 1; j >= 0; --j) chain_link(Q, p, j, m, d2, d4, ke, dof, temp);
#pragma unroll kUnroll
        for (int k = 0; k < m; ++k) xi[k] = __dadd_rn(xi[k], __dmul_rn(d, p[k]) / Q[k]);
        const double f = exp(__dmul_rn(-d, p[0]) / Q[0]);
        total = __dmul_rn(total, f);
        ke = __dmul_rn(__dmul_rn(ke, f), f);
#pragma unroll kUnroll
        for (int j = 0; j < m; ++j) chain_link(Q, p, j, m, d2, d4, ke, dof, temp);
    }
#pragma unroll kUnroll
    for (int k = 0; k < m; ++k) {
        st->xi[k] = xi[k];
        st->pxi[k] = p[k];
    }
    return total;
}

// The usual three-link chain in registers; other lengths through C = 0.
__device__ __forceinline__ double nhc_half(NhcState* st, double delta, const Weights& w, double& ke) {
    return st->chain == 3 ? chain_half<3>(st, delta, w, ke) : chain_half<0>(st, delta, w, ke);
}

// Start-of-step chain half, from the kinetic energy of the current velocities (ke_now,
// pending scale included) or, with ke_now null, the one the last chain half left.
__device__ __forceinline__ void nhc_pre_body(NhcState* st, const double* ke_now, const Weights& w) {
    const double scale = st->scale;
    double ke = ke_now ? *ke_now * scale * scale : st->ke;
    const double f = nhc_half(st, 0.5 * st->dt, w, ke);
    st->scale = scale * f;
    st->ke = ke;
}

__global__ void k_nhc_pre(NhcState* st, const double* ke_now, Weights w) { nhc_pre_body(st, ke_now, w); }

// End-of-step chain half using the freshly summed KE; leaves its scale pending.
__device__ __forceinline__ void nhc_post_body(NhcState* st, const double* ke_sum, const Weights& w) {
    double ke = *ke_sum;
    st->scale = nhc_half(st, 0.5 * st->dt, w, ke);
    st->ke = ke;
}

__global__ void k_nhc_post(NhcState* st, const double* ke_sum, Weights w) { nhc_post_body(st, ke_sum, w); }

__device__ double nhc_conserved(const NhcState& c) {
    // nose_hoover.cpp:45-54
    double sum = c.dof * c.temperature * c.xi[0];
    for (int k = 1; k < c.chain; ++k) sum += c.temperature * c.xi[k];
    for (int k = 0; k < c.chain; ++k) sum += 0.5 * c.pxi[k] * c.pxi[k] / c.Q[k];
    return sum;
}

// thermo row: energy, virial, kinetic energy, conserved contribution.
__global__ void k_record(const double* ev, const double* ke, const NhcState* nhc, double* row) {
    row[0] = ev[0];
    row[1] = ev[1];
    row[2] = nhc ? nhc->ke : *ke;
    row[3] = nhc ? nhc_conserved(*nhc) : 0.0;
}

__global__ void k_conserved(const NhcState* nhc, double* out) { *out = nhc_conserved(*nhc); }

// Thermo row at a device-held index (graph replays cannot change a pointer).
__global__ void k_record_at(const double* ev, const double* ke, const NhcState* nhc, double* rows,
                            int* idx) {
    double* row = rows + 4 * static_cast<int64_t>(*idx);
    row[0] = ev[0];
    row[1] = ev[1];
    row[2] = nhc ? nhc->ke : *ke;
    row[3] = nhc ? nhc_conserved(*nhc) : 0.0;
    ++*idx;
}

// Opens the rebuild branch of a step graph when the fused check asked for one.
__global__ void k_set_rebuild(cudaGraphConditionalHandle h, const int* flag) {
    cudaGraphSetConditional(h, *flag != 0 ? 1u : 0u);
}

Weights yoshida() {
    // nose_hoover.cpp:15-18
    const double w1 = 1.0 / (2.0 - std::cbrt(2.0));
    return Weights{{w1, 1.0 - 2.0 * w1, w1}};
}

StepArgs step_args(const md_integrator* it, const md_system* sys) {
    StepArgs s{};
    for (int d = 0; d < 3; ++d) {
        s.box.L[d] = sys->box[d];
        s.box.inv[d] = sys->inv_box[d];
    }
    s.dt = it->dt;
    s.half_dt = 0.5 * it->dt;
    s.c1 = std::exp(-it->friction * it->dt);  // langevin.hpp:39-40
    s.c2 = std::sqrt(1.0 - s.c1 * s.c1);
    s.temperature = it->temperature;
    s.key0 = static_cast<uint32_t>(it->seed);
    s.key1 = static_cast<uint32_t>(it->seed >> 32);
    s.step = it->step;
    s.noise = nullptr;
    s.status = sys->ctx->d_status;
    s.q = nullptr;
    return s;
}

int kick_grid(const md_system* sys) {
    const int64_t want = (sys->n + kBlock - 1) / kBlock;
    const int cap = sys->ctx->sm_count * 8;
    return static_cast<int>(want < 1 ? 1 : (want > cap ? cap : want));
}

NhcState* nhc_of(md_integrator* it) {
    return (it->kind == 2 || it->kind == 4) ? it->chain_state.as<NhcState>() : nullptr;
}

// The pre-force half of a step.  With `check` the rebuild test of that Verlet
// list is fused into the position update (fused stepping loops).
// fresh_ke: the chain half of a Nose-Hoover step sums the kinetic energy of the
// current velocities; otherwise it uses the value the chain tracked through the
// previous step's rescalings (fused loops, after their first step).
// q: also write the fixed-point positions for a mixed-precision force (kick/drift
// integrators only; pre_force_quantizes says whether it does).
bool pre_force_quantizes(const md_integrator* it) { return it->kind != 1; }

int pre_force(md_integrator* it, md_system* sys, md_verlet* check, bool fresh_ke = true,
              int4* q = nullptr) {
    md_context* ctx = sys->ctx;
    const int64_t n = sys->n;
    if (n == 0) return MD_OK;
    StepArgs s = step_args(it, sys);
    if (q && pre_force_quantizes(it)) {
        s.q = q;
        for (int d = 0; d < 3; ++d) s.qs[d] = 4294967296.0 / sys->box[d];
    }
    DispArgs d{};
    const int blocks = grid_for(n, kBlock);
    if (check) {
        double* part;
        MDB_TRY(ctx_partials(ctx, 2 * static_cast<size_t>(blocks), &part));
        d = disp_args(check, ctx, part);
    }
    if (it->kind == 1) {
        if (it->noise.ptr) {
            if (it->noise_used + 3 * n > it->noise_count)
                return fail(MD_ERR_INVALID_ARGUMENT, "BAOAB: replayed noise exhausted");
            s.noise = it->noise.as<double>() + it->noise_used;
            it->noise_used += 3 * n;
        }
        if (check) k_baoab_pre<true><<<blocks, kBlock, 0, ctx->stream>>>(sys->cur, n, s, d);
        else k_baoab_pre<false><<<blocks, kBlock, 0, ctx->stream>>>(sys->cur, n, s, d);
        ++it->step;
    } else {
        NhcState* nhc = nhc_of(it);
        if (nhc) {
            // start-of-step chain half (integrateChain(dt/2), nose_hoover.hpp:37-42)
            if (fresh_ke) MDB_TRY(system_kinetic_async(sys, kResKE));
            k_nhc_pre<<<1, 1, 0, ctx->stream>>>(nhc, fresh_ke ? ctx_result(ctx, kResKE) : nullptr,
                                                yoshida());
            ctx->launches += 1;
        }
        ctx_time_begin(ctx, MD_KERNEL_INTEGRATE);
        const int kd = grid_for(n, kKickAtoms * kBlock);
        if (check) k_kick_drift<true><<<kd, kBlock, 0, ctx->stream>>>(sys->cur, n, s, nhc, d);
        else k_kick_drift<false><<<kd, kBlock, 0, ctx->stream>>>(sys->cur, n, s, nhc, d);
        ctx_time_end(ctx, MD_KERNEL_INTEGRATE);
    }
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

// The closing half-kick for a force kernel to apply (the kick of post_force_async).
KickArgs kick_args(const md_integrator* it, md_system* sys) {
    KickArgs k;
    k.vx = sys->cur.vx;
    k.vy = sys->cur.vy;
    k.vz = sys->cur.vz;
    k.mass = sys->cur.mass;
    k.inv_mass = sys->cur.inv_mass;
    k.half_dt = step_args(it, sys).half_dt;
    k.status = sys->ctx->d_status;
    return k;
}

// The step's end: the closing half-kick with the kinetic energy (unless the force
// kernel took it: `kicked`), then the chain half of a Nose-Hoover integrator.
int post_force_async(md_integrator* it, md_system* sys, bool apply_scale, bool kicked = false) {
    md_context* ctx = sys->ctx;
    const int64_t n = sys->n;
    StepArgs s = step_args(it, sys);
    const int g = kick_grid(sys);
    double* part;
    MDB_TRY(ctx_partials(ctx, static_cast<size_t>(g), &part));
    if (n > 0 && !kicked) {
        ctx_time_begin(ctx, MD_KERNEL_INTEGRATE);
        k_kick_ke<<<g, kBlock, 0, ctx->stream>>>(sys->cur, n, s, part, ctx_counter(ctx, 3),
                                                ctx_result(ctx, kResKE), ctx->d_status);
        ctx_time_end(ctx, MD_KERNEL_INTEGRATE);
        ++ctx->launches;
    }
    NhcState* nhc = nhc_of(it);
    if (nhc) {
        k_nhc_post<<<1, 1, 0, ctx->stream>>>(nhc, ctx_result(ctx, kResKE), yoshida());
        ++ctx->launches;
        if (apply_scale) {
            if (n > 0) {
                k_scale<<<grid_for(n, kBlock), kBlock, 0, ctx->stream>>>(sys->cur, n, nhc);
                ++ctx->launches;
            }
            k_reset_scale<<<1, 1, 0, ctx->stream>>>(nhc);
            ++ctx->launches;
        }
    }
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

}  // namespace

KickArgs integrator_kick_args(const md_integrator* it, md_system* sys) { return kick_args(it, sys); }

int verlet_build(md_verlet* v, md_system* sys, bool conditional);
int verlet_build_q(md_verlet* v, md_system* sys, int4* q, bool* quantized);

// ------------------------------------------------------------ step graphs
namespace {

// One fused LJ step captured as a CUDA graph: [chain half,] kick/drift with the
// displacement check, a conditional node whose body is the gated neighbour
// rebuild (opened by k_set_rebuild from the device flag, so steps without a
// rebuild launch none of its kernels), forces, the closing kick and the thermo
// row.  Replaying it runs the same kernels with the same arguments as the host
// loop.
struct StepGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t main_launches = 0;  // kernels outside the rebuild branch
    int64_t body_launches = 0;  // kernels inside it
    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
};

// Captures work() on the context stream into graph g after the given nodes; on
// return the stream is out of capture whatever happened.  leaves (optional)
// receives the last captured nodes.
template <class F>
int capture_into(md_context* ctx, cudaGraph_t g, const cudaGraphNode_t* deps, size_t ndeps,
                 F&& work, std::vector<cudaGraphNode_t>* leaves) {
    MDB_CUDA(cudaStreamBeginCaptureToGraph(ctx->stream, g, deps, nullptr, ndeps,
                                           cudaStreamCaptureModeThreadLocal));
    int rc = work();
    if (rc == MD_OK && leaves) {
        cudaStreamCaptureStatus st;
        const cudaGraphNode_t* out = nullptr;
        size_t nout = 0;
        const cudaError_t e =
            cudaStreamGetCaptureInfo(ctx->stream, &st, nullptr, nullptr, &out, &nout);
        if (e != cudaSuccess) rc = fail(MD_ERR_CUDA, "capture info: %s", cudaGetErrorString(e));
        else leaves->assign(out, out + nout);
    }
    cudaGraph_t captured = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &captured);
    if (rc != MD_OK) return rc;
    if (e != cudaSuccess) return fail(MD_ERR_CUDA, "step graph capture: %s", cudaGetErrorString(e));
    return MD_OK;
}

}  // namespace (the step graph helpers above are private to this file)

int vv_pre_async(md_integrator* it, md_system* sys, md_verlet* check) {
    return pre_force(it, sys, check, true);
}

int vv_post_async(md_integrator* it, md_system* sys) { return post_force_async(it, sys, true); }

int record_at_async(md_context* ctx, const NhcState* nhc, double* rows, int* idx) {
    k_record_at<<<1, 1, 0, ctx->stream>>>(ctx_result(ctx, kResEnergy), ctx_result(ctx, kResKE), nhc,
                                          rows, idx);
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

// The fixed-point position buffer the step's kick/drift fills for a mixed force
// (null when the force is FP64 or the integrator has no kick/drift kernel).
int step_quantize_target(md_integrator* it, md_system* sys, const md_lj* lj, int4** q) {
    *q = nullptr;
    if (lj->precision != MD_PRECISION_MIXED || !pre_force_quantizes(it) || sys->n <= 0)
        return MD_OK;
    MDB_TRY(sys->qpos.ensure(sizeof(int4) * static_cast<size_t>(sys->n)));
    *q = sys->qpos.as<int4>();
    return MD_OK;
}

int lj_fused_step(md_integrator* it, md_system* sys, md_verlet* v, md_lj* lj, double* rows,
                  int* idx, bool first) {
    md_context* ctx = sys->ctx;
    // Kick/drift with the rebuild test of the ForceFn (apps/moldyn_run.cpp:581-587)
    // fused in; the rebuild itself is gated on the device flag.  A mixed force
    // takes the fixed-point positions the kick/drift wrote, re-quantized only after
    // a rebuild re-sorted the atoms.
    int4* q = nullptr;
    MDB_TRY(step_quantize_target(it, sys, lj, &q));
    MDB_TRY(pre_force(it, sys, v, first, q));
    // a rebuild that re-sorts the atoms also re-quantizes them (q stays current)
    bool requantized = false;
    MDB_TRY(verlet_build_q(v, sys, q, &requantized));
    const KickArgs ka = kick_args(it, sys);
    bool kicked = false;
    MDB_TRY(lj_forces_verlet_async(lj, sys, v, q ? v->d_rebuild_flag : nullptr, requantized, &ka,
                                   &kicked));
    MDB_TRY(post_force_async(it, sys, false, kicked));
    if (rows) {
        k_record_at<<<1, 1, 0, ctx->stream>>>(ctx_result(ctx, kResEnergy), ctx_result(ctx, kResKE),
                                              nhc_of(it), rows, idx);
        ++ctx->launches;
    }
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

int capture_lj_step_into(md_integrator* it, md_system* sys, md_verlet* v, md_lj* lj,
                         double* rows, int* idx, cudaGraph_t graph, int64_t* main_launches,
                         int64_t* body_launches) {
    md_context* ctx = sys->ctx;
    NhcState* nhc = nhc_of(it);
    const int64_t l0 = ctx->launches;
    int rc = MD_OK;
    cudaGraphConditionalHandle h;
    if (cudaGraphConditionalHandleCreate(&h, graph, 0, cudaGraphCondAssignDefault) != cudaSuccess)
        return fail(MD_ERR_CUDA, "cudaGraphConditionalHandleCreate failed");
    std::vector<cudaGraphNode_t> leaves;
    int4* q = nullptr;
    MDB_TRY(step_quantize_target(it, sys, lj, &q));  // allocated by the first, eager step
    rc = capture_into(ctx, graph, nullptr, 0, [&]() -> int {
        MDB_TRY(pre_force(it, sys, v, false, q));
        k_set_rebuild<<<1, 1, 0, ctx->stream>>>(h, v->d_rebuild_flag);
        ++ctx->launches;
        MDB_CHECK_LAUNCH();
        return MD_OK;
    }, &leaves);
    const int64_t l1 = ctx->launches;
    cudaGraphNode_t cond = nullptr;
    cudaGraph_t body = nullptr;
    if (rc == MD_OK) {
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        const cudaError_t e = cudaGraphAddNode(&cond, graph, leaves.data(), leaves.size(), &cp);
        if (e != cudaSuccess) rc = fail(MD_ERR_CUDA, "conditional node: %s", cudaGetErrorString(e));
        else body = cp.conditional.phGraph_out[0];
    }
    // the rebuild branch also re-quantizes the re-sorted positions, so that the
    // main path launches no gated no-op
    if (rc == MD_OK)
        rc = capture_into(ctx, body, nullptr, 0, [&]() -> int {
            bool requantized = false;
            MDB_TRY(verlet_build_q(v, sys, q, &requantized));
            if (q && !requantized) MDB_TRY(lj_quantize_async(lj, sys, v->d_rebuild_flag));
            return MD_OK;
        }, nullptr);
    const int64_t l2 = ctx->launches;
    if (rc == MD_OK)
        rc = capture_into(ctx, graph, &cond, 1, [&]() -> int {
            const KickArgs ka = kick_args(it, sys);
            bool kicked = false;
            MDB_TRY(lj_forces_verlet_async(lj, sys, v, q ? v->d_rebuild_flag : nullptr,
                                           q != nullptr, &ka, &kicked));
            MDB_TRY(post_force_async(it, sys, false, kicked));
            if (rows) {
                k_record_at<<<1, 1, 0, ctx->stream>>>(ctx_result(ctx, kResEnergy),
                                                      ctx_result(ctx, kResKE), nhc, rows, idx);
                ++ctx->launches;
            }
            MDB_CHECK_LAUNCH();
            return MD_OK;
        }, nullptr);
    if (main_launches) *main_launches = (l1 - l0) + (ctx->launches - l2);
    if (body_launches) *body_launches = l2 - l1;
    ctx->launches = l0;  // counted per replay by the caller
    return rc;
}

namespace {

int capture_lj_step(md_integrator* it, md_system* sys, md_verlet* v, md_lj* lj, double* rows,
                    int* idx, StepGraph& sg) {
    if (cudaGraphCreate(&sg.graph, 0) != cudaSuccess)
        return fail(MD_ERR_CUDA, "cudaGraphCreate failed");
    int rc = capture_lj_step_into(it, sys, v, lj, rows, idx, sg.graph, &sg.main_launches,
                                  &sg.body_launches);
    if (rc == MD_OK && cudaGraphInstantiate(&sg.exec, sg.graph, 0) != cudaSuccess)
        rc = fail(MD_ERR_CUDA, "step graph instantiation failed");
    if (rc != MD_OK) sg.release();
    return rc;
}

}  // namespace

// Chain-of-thermostats pieces shared with the constrained integrators.
int nhc_pre_async(md_integrator* it, md_context* ctx, const double* ke_now) {
    k_nhc_pre<<<1, 1, 0, ctx->stream>>>(it->chain_state.as<NhcState>(), ke_now, yoshida());
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

int nhc_post_async(md_integrator* it, md_context* ctx, const double* ke_sum) {
    k_nhc_post<<<1, 1, 0, ctx->stream>>>(it->chain_state.as<NhcState>(), ke_sum, yoshida());
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

int nhc_apply_scale_async(md_integrator* it, md_system* sys) {
    md_context* ctx = sys->ctx;
    NhcState* nhc = it->chain_state.as<NhcState>();
    if (sys->n > 0) {
        k_scale<<<grid_for(sys->n, kBlock), kBlock, 0, ctx->stream>>>(sys->cur, sys->n, nhc);
        ++ctx->launches;
    }
    k_reset_scale<<<1, 1, 0, ctx->stream>>>(nhc);
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

int record_async(md_context* ctx, const double* ev, const double* ke, const NhcState* nhc,
                 double* row) {
    k_record<<<1, 1, 0, ctx->stream>>>(ev, ke, nhc, row);
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

int constrained_pre_force(md_integrator* it, md_system* sys);
int constrained_post_force(md_integrator* it, md_system* sys, bool apply_scale);

// ------------------------------------------------------------ batched replicas
// One replica's arguments of the batched kick kernels: what pre_force (no fresh
// kinetic energy, the rebuild test fused in) and post_force_async give its solo
// kernels, plus its thermo row.
// Atoms per thread of the batched kick/drift and chain-scale launches.
constexpr int kBatchKickAtoms = 2;

struct BatchKickRep {
    md_atoms a;
    int64_t n;
    StepArgs s;
    NhcState* nhc;
    DispArgs d;
    double* ke_part;
    unsigned* ke_ticket;
    double* ke_out;
    uint32_t* status;
    const double* ev;
    double* rows;
    int* idx;
};

namespace {

// Start-of-step chain halves, one thread per replica (k_nhc_pre without a fresh KE).
// (The chain half is serial FP64 work, exp-bound; computing it in every kick block
// instead, or both halves in the block that ends the kinetic-energy sum, measured
// slower: each block then waits on that chain before its atoms.)
__global__ void k_batch_nhc_pre(const BatchKickRep* __restrict__ reps, int nrep, Weights w) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nrep && reps[r].nhc) nhc_pre_body(reps[r].nhc, nullptr, w);
}

// The first step of a run: every row index back to 0, and a chain's start-of-step
// half from the kinetic energy summed just before (k_nhc_pre with a fresh KE, as
// the first step of md_run_lj runs it).
__global__ void k_batch_first_pre(const BatchKickRep* __restrict__ reps, int nrep, Weights w) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrep) return;
    const BatchKickRep& d = reps[r];
    if (d.idx) *d.idx = 0;
    if (d.nhc) nhc_pre_body(d.nhc, d.ke_out, w);
}

// Kick/drift with the rebuild test of every replica, kBatchKickAtoms atoms per
// thread: the batch's many small replicas then fill fewer, fuller blocks.
__global__ void k_batch_kick_drift(const BatchKickRep* __restrict__ reps, const int4* __restrict__ blk) {
    const int4 e = __ldg(blk + blockIdx.x);
    const BatchKickRep& d = reps[e.x];
    kick_drift_body<true, kBatchKickAtoms>(d.a, d.n, d.s, d.nhc, d.d, e.y, e.z);
}

__global__ void k_batch_kick_ke(const BatchKickRep* __restrict__ reps, const int4* __restrict__ blk) {
    const int4 e = __ldg(blk + blockIdx.x);
    const BatchKickRep& d = reps[e.x];
    kick_ke_body(d.a, d.n, d.s, d.ke_part, d.ke_ticket, d.ke_out, d.status, e.y, e.z);
}

// End-of-step chain halves and thermo rows (k_nhc_post, k_record_at), one thread per replica.
__global__ void k_batch_nhc_post(const BatchKickRep* __restrict__ reps, int nrep, Weights w) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrep) return;
    const BatchKickRep& d = reps[r];
    if (d.nhc) nhc_post_body(d.nhc, d.ke_out, w);
    if (d.rows) {
        double* row = d.rows + 4 * static_cast<int64_t>(*d.idx);
        row[0] = d.ev[0];
        row[1] = d.ev[1];
        row[2] = d.nhc ? d.nhc->ke : *d.ke_out;
        row[3] = d.nhc ? nhc_conserved(*d.nhc) : 0.0;
        ++*d.idx;
    }
}

// The end of a batched run: every chain's pending velocity scale applied (k_scale)
// and reset (k_reset_scale), two launches for all replicas.
__global__ void k_batch_scale(const BatchKickRep* __restrict__ reps, const int4* __restrict__ blk) {
    const int4 e = __ldg(blk + blockIdx.x);
    const BatchKickRep& d = reps[e.x];
    if (!d.nhc) return;
    const double sc = d.nhc->scale;
#pragma unroll
    for (int u = 0; u < kBatchKickAtoms; ++u) {
        const int64_t k = (e.y * static_cast<int64_t>(kBatchKickAtoms) + u) * blockDim.x + threadIdx.x;
        if (k < d.n) {
            d.a.vx[k] = __dmul_rn(d.a.vx[k], sc);
            d.a.vy[k] = __dmul_rn(d.a.vy[k], sc);
            d.a.vz[k] = __dmul_rn(d.a.vz[k], sc);
        }
    }
}

__global__ void k_batch_reset_scale(const BatchKickRep* __restrict__ reps, int nrep) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nrep && reps[r].nhc) reps[r].nhc->scale = 1.0;
}

}  // namespace

struct BatchKick {
    DevBuf reps, kick_blk, ke_blk;  // block tables (block_table) of the kick launches
    DevBuf kin_reps, kin_blk;  // the chains' entry kinetic energies (first step of a run)
    int nrep = 0, kick_total = 0, ke_total = 0, kin_total = 0;
    bool any_nhc = false, any_rows = false;
};

int batch_kick_create(const BatchRepView* v, int nrep, BatchKick** out) {
    if (nrep < 1) return fail(MD_ERR_INVALID_ARGUMENT, "batch_kick_create: no replicas");
    std::vector<BatchKickRep> h(static_cast<size_t>(nrep));
    std::vector<BatchKineticRep> kh(static_cast<size_t>(nrep));
    std::vector<int> ko(static_cast<size_t>(nrep) + 1, 0), eo(static_cast<size_t>(nrep) + 1, 0),
        kn(static_cast<size_t>(nrep) + 1, 0);
    bool any_nhc = false, any_rows = false;
    for (int r = 0; r < nrep; ++r) {
        md_integrator* it = v[r].it;
        md_system* sys = v[r].sys;
        md_context* ctx = sys->ctx;
        if ((it->kind != 0 && it->kind != 2) || sys->n <= 0)
            return fail(MD_ERR_INVALID_ARGUMENT, "batch_kick_create: velocity Verlet or NHC replicas");
        BatchKickRep& d = h[static_cast<size_t>(r)];
        d.a = sys->cur;
        d.n = sys->n;
        d.s = step_args(it, sys);
        int4* q = nullptr;
        MDB_TRY(step_quantize_target(it, sys, v[r].lj, &q));
        if (q) {
            d.s.q = q;
            for (int k = 0; k < 3; ++k) d.s.qs[k] = 4294967296.0 / sys->box[k];
        }
        const int blocks = grid_for(sys->n, kBlock);
        double* part;
        MDB_TRY(ctx_partials(ctx, 2 * static_cast<size_t>(blocks), &part));
        d.d = disp_args(v[r].list, ctx, part);
        d.nhc = nhc_of(it);
        const int g = kick_grid(sys);
        MDB_TRY(ctx_partials(ctx, static_cast<size_t>(g), &part));
        d.ke_part = part;
        d.ke_ticket = ctx_counter(ctx, 3);
        d.ke_out = ctx_result(ctx, kResKE);
        d.status = ctx->d_status;
        d.ev = ctx_result(ctx, kResEnergy);
        d.rows = v[r].rows;
        d.idx = v[r].idx;
        any_nhc = any_nhc || d.nhc;
        any_rows = any_rows || d.rows;
        ko[static_cast<size_t>(r) + 1] =
            ko[static_cast<size_t>(r)] + grid_for(sys->n, kBatchKickAtoms * kBlock);
        eo[static_cast<size_t>(r) + 1] = eo[static_cast<size_t>(r)] + g;
        // system_kinetic_async's launch for a chain (reduce_grid blocks: kick_grid's count)
        kh[static_cast<size_t>(r)] = BatchKineticRep{sys->cur, sys->n, part, ctx_counter(ctx, 0),
                                                     ctx_result(ctx, kResKE)};
        kn[static_cast<size_t>(r) + 1] = kn[static_cast<size_t>(r)] + (d.nhc ? g : 0);
    }
    BatchKick* b = new (std::nothrow) BatchKick();
    if (!b) return fail(MD_ERR_OUT_OF_MEMORY, "batch_kick_create: host allocation");
    b->nrep = nrep;
    b->kick_total = ko.back();
    b->ke_total = eo.back();
    b->kin_total = kn.back();
    b->any_nhc = any_nhc;
    b->any_rows = any_rows;
    const std::vector<int4> kt = block_table(ko.data(), nrep), et = block_table(eo.data(), nrep),
                            nt = block_table(kn.data(), nrep);
    int rc = b->reps.ensure(sizeof(BatchKickRep) * h.size());
    if (rc == MD_OK) rc = b->kick_blk.ensure(sizeof(int4) * kt.size());
    if (rc == MD_OK) rc = b->ke_blk.ensure(sizeof(int4) * et.size());
    if (rc == MD_OK) rc = b->kin_reps.ensure(sizeof(BatchKineticRep) * kh.size());
    if (rc == MD_OK) rc = b->kin_blk.ensure(sizeof(int4) * std::max<size_t>(nt.size(), 1));
    if (rc == MD_OK &&
        (cudaMemcpy(b->kin_reps.ptr, kh.data(), sizeof(BatchKineticRep) * kh.size(),
                    cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMemcpy(b->kin_blk.ptr, nt.data(), sizeof(int4) * nt.size(), cudaMemcpyHostToDevice) !=
             cudaSuccess))
        rc = fail(MD_ERR_CUDA, "batch_kick_create: upload");
    if (rc == MD_OK &&
        (cudaMemcpy(b->reps.ptr, h.data(), sizeof(BatchKickRep) * h.size(), cudaMemcpyHostToDevice) !=
             cudaSuccess ||
         cudaMemcpy(b->kick_blk.ptr, kt.data(), sizeof(int4) * kt.size(), cudaMemcpyHostToDevice) !=
             cudaSuccess ||
         cudaMemcpy(b->ke_blk.ptr, et.data(), sizeof(int4) * et.size(), cudaMemcpyHostToDevice) !=
             cudaSuccess))
        rc = fail(MD_ERR_CUDA, "batch_kick_create: descriptor upload");
    if (rc != MD_OK) {
        batch_kick_destroy(b);
        return rc;
    }
    *out = b;
    return MD_OK;
}

int batch_kick_pre(BatchKick* b, cudaStream_t stream, int64_t* launches) {
    if (b->any_nhc) {
        k_batch_nhc_pre<<<grid_for(b->nrep, 128), 128, 0, stream>>>(b->reps.as<BatchKickRep>(),
                                                                   b->nrep, yoshida());
        if (launches) ++*launches;
    }
    k_batch_kick_drift<<<b->kick_total, kBlock, 0, stream>>>(b->reps.as<BatchKickRep>(),
                                                             b->kick_blk.as<int4>());
    if (launches) ++*launches;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

int batch_kick_first(BatchKick* b, cudaStream_t stream, int64_t* launches) {
    MDB_TRY(batch_kinetic_launch(b->kin_reps.as<BatchKineticRep>(), b->kin_blk.as<int4>(),
                                 b->kin_total, stream));
    k_batch_first_pre<<<grid_for(b->nrep, 128), 128, 0, stream>>>(b->reps.as<BatchKickRep>(),
                                                                 b->nrep, yoshida());
    k_batch_kick_drift<<<b->kick_total, kBlock, 0, stream>>>(b->reps.as<BatchKickRep>(),
                                                             b->kick_blk.as<int4>());
    if (launches) *launches += (b->kin_total > 0 ? 1 : 0) + 2;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

int batch_kick_post(BatchKick* b, cudaStream_t stream, int64_t* launches, bool kicked) {
    if (!kicked) {
        k_batch_kick_ke<<<b->ke_total, kBlock, 0, stream>>>(b->reps.as<BatchKickRep>(),
                                                            b->ke_blk.as<int4>());
        if (launches) ++*launches;
    }
    if (b->any_nhc || b->any_rows) {
        k_batch_nhc_post<<<grid_for(b->nrep, 128), 128, 0, stream>>>(b->reps.as<BatchKickRep>(),
                                                                    b->nrep, yoshida());
        if (launches) ++*launches;
    }
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

int batch_kick_finish(BatchKick* b, cudaStream_t stream, int64_t* launches) {
    if (!b->any_nhc) return MD_OK;
    k_batch_scale<<<b->kick_total, kBlock, 0, stream>>>(b->reps.as<BatchKickRep>(),
                                                        b->kick_blk.as<int4>());
    k_batch_reset_scale<<<grid_for(b->nrep, 128), 128, 0, stream>>>(b->reps.as<BatchKickRep>(),
                                                                    b->nrep);
    if (launches) *launches += 2;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

void batch_kick_destroy(BatchKick* b) {
    if (!b) return;
    b->reps.release();
    b->kick_blk.release();
    b->ke_blk.release();
    b->kin_reps.release();
    b->kin_blk.release();
    delete b;
}

}  // namespace mdb

using namespace mdb;

extern "C" {

int md_integrator_create_vv(double dt, md_integrator** out) {
    graph_epoch_bump();
    if (!out) return fail(MD_ERR_INVALID_ARGUMENT, "md_integrator_create_vv: NULL");
    md_integrator* it = new (std::nothrow) md_integrator();
    if (!it) return fail(MD_ERR_OUT_OF_MEMORY, "md_integrator_create_vv: host allocation");
    it->kind = 0;
    it->dt = dt;
    *out = it;
    return MD_OK;
}

int md_integrator_create_baoab(double dt, double friction, double temperature, uint64_t seed,
                               md_integrator** out) {
    graph_epoch_bump();
    if (!out) return fail(MD_ERR_INVALID_ARGUMENT, "md_integrator_create_baoab: NULL");
    md_integrator* it = new (std::nothrow) md_integrator();
    if (!it) return fail(MD_ERR_OUT_OF_MEMORY, "md_integrator_create_baoab: host allocation");
    it->kind = 1;
    it->dt = dt;
    it->friction = friction;
    it->temperature = temperature;
    it->seed = seed;
    *out = it;
    return MD_OK;
}

int md_integrator_create_nhc(double dt, double temperature, double tau, int chain_length,
                             int64_t dof, md_integrator** out) {
    graph_epoch_bump();
    if (!out) return fail(MD_ERR_INVALID_ARGUMENT, "md_integrator_create_nhc: NULL");
    if (chain_length < 1)  // nose_hoover.cpp:36-38
        return fail(MD_ERR_INVALID_ARGUMENT, "NoseHooverChain: chainLength must be >= 1");
    if (chain_length > kMaxChain)
        return fail(MD_ERR_INVALID_ARGUMENT, "NoseHooverChain: chainLength must be <= %d", kMaxChain);
    md_integrator* it = new (std::nothrow) md_integrator();
    if (!it) return fail(MD_ERR_OUT_OF_MEMORY, "md_integrator_create_nhc: host allocation");
    it->kind = 2;
    it->dt = dt;
    it->temperature = temperature;
    it->tau = tau;
    it->chain = chain_length;
    it->dof = dof;
    NhcState st{};
    st.chain = chain_length;
    st.dt = dt;
    st.temperature = temperature;
    st.dof = static_cast<double>(dof);
    st.Q[0] = static_cast<double>(dof) * temperature * tau * tau;  // nose_hoover.cpp:39-42
    for (int k = 1; k < chain_length; ++k) st.Q[k] = temperature * tau * tau;
    st.scale = 1.0;
    int rc = it->chain_state.ensure(sizeof(NhcState));
    if (rc == MD_OK && cudaMemcpy(it->chain_state.ptr, &st, sizeof(NhcState),
                                  cudaMemcpyHostToDevice) != cudaSuccess)
        rc = fail(MD_ERR_CUDA, "md_integrator_create_nhc: upload failed");
    if (rc != MD_OK) {
        it->chain_state.release();
        delete it;
        return rc;
    }
    *out = it;
    return MD_OK;
}

int md_integrator_destroy(md_integrator* it) {
    graph_epoch_bump();
    if (!it) return MD_OK;
    cudaDeviceSynchronize();
    if (it->run_graph) {
        StepGraph* sg = static_cast<StepGraph*>(it->run_graph);
        sg->release();
        delete sg;
    }
    it->run_rows.release();
    it->run_idx.release();
    it->conserved.release();
    if (it->h_rebuilt) cudaFreeHost(it->h_rebuilt);
    it->chain_state.release();
    it->noise.release();
    it->mol_state.release();
    it->counters.release();
    delete it;
    return MD_OK;
}

int md_integrator_pre_force(md_integrator* it, md_system* sys) {
    if (!it || !sys) return fail(MD_ERR_INVALID_ARGUMENT, "md_integrator_pre_force: NULL");
    if (it->kind >= 3) return constrained_pre_force(it, sys);
    return pre_force(it, sys, nullptr);
}

int md_integrator_post_force(md_integrator* it, md_system* sys) {
    if (!it || !sys) return fail(MD_ERR_INVALID_ARGUMENT, "md_integrator_post_force: NULL");
    if (it->kind >= 3) return constrained_post_force(it, sys, true);
    return post_force_async(it, sys, true);
}

int md_integrator_conserved(md_integrator* it, double* value) {
    if (!it || !value) return fail(MD_ERR_INVALID_ARGUMENT, "md_integrator_conserved: NULL");
    if (it->kind != 2 && it->kind != 4) {
        *value = 0.0;
        return MD_OK;
    }
    // A tiny read on the default stream after all work on every stream finished.
    MDB_CUDA(cudaDeviceSynchronize());
    MDB_TRY(it->conserved.ensure(sizeof(double)));
    k_conserved<<<1, 1>>>(it->chain_state.as<NhcState>(), it->conserved.as<double>());
    MDB_CUDA(cudaMemcpy(value, it->conserved.ptr, sizeof(double), cudaMemcpyDeviceToHost));
    return MD_OK;
}

int md_integrator_set_noise(md_integrator* it, const double* xi, int64_t count) {
    if (!it) return fail(MD_ERR_INVALID_ARGUMENT, "md_integrator_set_noise: NULL");
    if (it->kind != 1) return fail(MD_ERR_INVALID_ARGUMENT, "md_integrator_set_noise: not BAOAB");
    if (!xi) {
        it->noise.release();
        it->noise_count = it->noise_used = 0;
        return MD_OK;
    }
    MDB_TRY(it->noise.ensure(sizeof(double) * static_cast<size_t>(count)));
    MDB_CUDA(cudaMemcpy(it->noise.ptr, xi, sizeof(double) * static_cast<size_t>(count),
                        cudaMemcpyHostToDevice));
    it->noise_count = count;
    it->noise_used = 0;
    return MD_OK;
}

int md_run_lj(md_integrator* it, md_system* sys, md_verlet* v, md_lj* lj, int64_t steps,
              double* thermo) {
    if (!it || !sys || !v || !lj) return fail(MD_ERR_INVALID_ARGUMENT, "md_run_lj: NULL argument");
    if (steps < 0) return fail(MD_ERR_INVALID_ARGUMENT, "md_run_lj: steps < 0");
    MDB_TRY(verlet_ensure_ready(v, sys, "md_run_lj"));
    if (it->kind >= 3)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_run_lj: constrained integrators run with md_run_spce");
    md_context* ctx = sys->ctx;
    verlet_halo_for_run(v, sys, lj);
    // Thermo rows persist on the integrator (a captured step graph writes them at a
    // device-held index), grown in powers of two so that calls of similar length
    // keep the same buffer.
    if (steps > 0) {
        size_t cap = 1024;
        while (cap < static_cast<size_t>(steps)) cap *= 2;
        MDB_TRY(it->run_rows.ensure(sizeof(double) * 4 * cap));
        MDB_TRY(it->run_idx.ensure(sizeof(int)));
        MDB_CUDA(cudaMemsetAsync(it->run_idx.ptr, 0, sizeof(int), ctx->stream));
        if (!it->h_rebuilt) MDB_CUDA(cudaMallocHost(&it->h_rebuilt, 2 * sizeof(int)));
    }
    double* rows = it->run_rows.as<double>();
    int* idx = it->run_idx.as<int>();
    NhcState* nhc = nhc_of(it);
    // Steps replay one captured step graph when that is possible (BAOAB's noise
    // counter is a host-side launch argument, so it never is).  The graph of an
    // earlier call is replayed while the system, list and force field are the same
    // handles and nothing has been allocated, freed, permuted or reconfigured since
    // (the graph epoch).  Otherwise the first step runs from the host -- it sizes
    // every buffer -- and the step is captured afterwards.  A chain's first step
    // always runs from the host: it sums the entry kinetic energy instead of using
    // the tracked value, which the caller may have changed between calls.
    const bool want_graph = ctx->graphs && !ctx->timing && it->kind != 1 && steps >= 1 && sys->n > 0;
    StepGraph* sg = static_cast<StepGraph*>(it->run_graph);
    const void* key[3] = {sys, v, lj};
    bool cached = want_graph && sg && sg->exec && it->run_epoch == graph_epoch() &&
                  key[0] == it->run_key[0] && key[1] == it->run_key[1] && key[2] == it->run_key[2];
    int64_t k = 0;
    if (steps > 0 && (!cached || nhc)) {
        MDB_TRY(lj_fused_step(it, sys, v, lj, rows, idx, true));
        k = 1;
    }
    if (want_graph && !cached) {
        if (!sg) {
            sg = new (std::nothrow) StepGraph();
            if (!sg) return fail(MD_ERR_OUT_OF_MEMORY, "md_run_lj: host allocation");
            it->run_graph = sg;
        }
        sg->release();
        if (capture_lj_step(it, sys, v, lj, rows, idx, *sg) == MD_OK) {
            ++ctx->graph_captures;
            // anything the first step and the capture allocated is part of the key
            it->run_epoch = graph_epoch();
            for (int q = 0; q < 3; ++q) it->run_key[q] = key[q];
            cached = true;
        } else {
            cudaGetLastError();  // no graph: the remaining steps run from the host
        }
    }
    if (cached && k < steps) {
        const int64_t graph_steps = steps - k;
        MDB_CUDA(cudaMemcpyAsync(it->h_rebuilt, v->d_rebuild_total, sizeof(int),
                                 cudaMemcpyDeviceToHost, ctx->stream));
        for (int64_t g = 0; g < graph_steps; ++g) MDB_CUDA(cudaGraphLaunch(sg->exec, ctx->stream));
        MDB_CUDA(cudaMemcpyAsync(it->h_rebuilt + 1, v->d_rebuild_total, sizeof(int),
                                 cudaMemcpyDeviceToHost, ctx->stream));
        MDB_CUDA(cudaStreamSynchronize(ctx->stream));
        ctx->launches += graph_steps * sg->main_launches +
                         static_cast<int64_t>(it->h_rebuilt[1] - it->h_rebuilt[0]) * sg->body_launches;
        k = steps;
    }
    for (; k < steps; ++k) MDB_TRY(lj_fused_step(it, sys, v, lj, rows, idx, false));
    if (nhc && steps > 0 && sys->n > 0) {
        k_scale<<<grid_for(sys->n, kBlock), kBlock, 0, ctx->stream>>>(sys->cur, sys->n, nhc);
        k_reset_scale<<<1, 1, 0, ctx->stream>>>(nhc);
        ctx->launches += 2;
    }
    if (thermo && steps > 0)
        MDB_CUDA(cudaMemcpyAsync(thermo, rows, sizeof(double) * 4 * static_cast<size_t>(steps),
                                 cudaMemcpyDeviceToHost, ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    MDB_TRY(ctx_check_status(ctx));
    double r[2];
    MDB_TRY(ctx_read_results(ctx, kResEnergy, 2, r));
    sys->last_energy = r[0];
    sys->last_virial = r[1];
    return MD_OK;
}

}  // extern "C"
