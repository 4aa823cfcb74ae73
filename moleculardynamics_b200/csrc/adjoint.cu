// adjoint.cu -- a differentiable velocity-Verlet LJ trajectory (no reference
// counterpart).
//
// Forward: FP64 velocity-Verlet steps with LJ forces, recording U, W and KE after
// every step, and saving the state (positions, velocities, in the caller's atom
// order) every `every` steps.  The Verlet list is rebuilt only at those
// checkpoints, with its own skin, so the atom order is fixed inside a segment;
// the fused displacement check proves every step's list valid (the reference
// criterion), or the forward fails.
//
// Backward (torch.autograd.Function semantics): given dL/d(U_k, W_k, KE_k) for
// every step, the discrete adjoint of the step map is run from the last
// segment to the first.  Each segment is recomputed from its checkpoint (the
// sort, list and forces are pure functions of the state, so the recomputation
// is bit-identical to the forward), its states are kept, and the adjoint walks
// back through them.  One reverse step at state x_k is one pair pass that forms
//   the Hessian-vector product (dF/dx)^T mu (mu = the adjoint of F(x_k)),
//   the direct loss terms dU/dx = -F and dW/dx,
//   and the parameter terms (dF/d(eps, sigma))^T mu + dL/dU dU/dtheta + dL/dW dW/dtheta.
// Velocity Verlet, per atom, with c = (dt/2)/m:
//   v_h = v_k + c F(x_k);  x_{k+1} = x_k + dt v_h;  v_{k+1} = v_h + c F(x_{k+1})
// so with carries lx (adjoint of x_{k+1} from later steps) and lvh (adjoint of
// the next step's half-step velocity), at state k:
//   lv  = lvh + gKE_k m v_k
//   mu  = c (lv + lvh)            (F(x_k) enters v_k and the next v_h)
//   lx += (dF/dx)^T mu + gU_k (-F) + gW_k dW/dx
//   lvh = lv + dt lx              (the half-step velocity of step k-1 -> k)
// and at x_0: mu_0 = c lvh, dL/dx_0 = lx + (dF/dx)^T mu_0, dL/dv_0 = lvh.
#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "md_device.cuh"
#include "md_internal.cuh"

namespace mdb {
int verlet_build(md_verlet* v, md_system* sys, bool conditional);
int verlet_ensure_ready(md_verlet* v, md_system* sys, const char* who);
}

struct md_adjoint {
    md_context* ctx = nullptr;
    md_system* sys = nullptr;
    md_lj lj;                     // parameters of the last forward
    md_verlet* list = nullptr;
    md_integrator* vv = nullptr;
    double dt = 0.0, skin = 0.0;
    int64_t steps = 0, n = 0;
    int every = 0;
    mdb::DevBuf ck;               // checkpoints: (nseg) x n x 2 double4 (pos, vel), caller's order
    mdb::DevBuf snap;             // one segment's states: (every + 1) x n x 2 double4, device order
    mdb::DevBuf carry;            // lx, lvh (n double4 each) + mu, lv (n double4 each)
    mdb::DevBuf carry_orig;       // lx, lvh in the caller's order between segments
    mdb::DevBuf grads;            // dL/d(U, W, KE) per step, uploaded by backward
    mdb::DevBuf theta;            // per reverse pass: 2 doubles (d eps, d sigma)
    mdb::DevBuf flag;             // list validity (OR over the forward's steps)
    bool have_forward = false;
};

using namespace mdb;

namespace {

constexpr int kBlock = 256;

// ---------------------------------------------------------------- state copies
__global__ void k_state_to_orig(md_atoms a, int64_t n, double4* pos, double4* vel) {
    const int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (s >= n) return;
    const int o = a.orig[s];
    pos[o] = a.pos[s];
    vel[o] = make_double4(a.vx[s], a.vy[s], a.vz[s], 0.0);
}

__global__ void k_state_from_orig(md_atoms a, const int* __restrict__ slot, int64_t n,
                                  const double4* __restrict__ pos, const double4* __restrict__ vel) {
    const int64_t o = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (o >= n) return;
    const int s = slot[o];
    a.pos[s] = pos[o];
    a.vx[s] = vel[o].x;
    a.vy[s] = vel[o].y;
    a.vz[s] = vel[o].z;
}

__global__ void k_snapshot(md_atoms a, int64_t n, double4* pos, double4* vel) {
    const int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (s >= n) return;
    pos[s] = a.pos[s];
    vel[s] = make_double4(a.vx[s], a.vy[s], a.vz[s], 0.0);
}

// device order <-> caller's order for per-atom vectors (double4 lanes x, y, z)
__global__ void k_vec_to_orig(const int* __restrict__ orig, int64_t n, const double4* in,
                              double4* out) {
    const int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (s < n) out[orig[s]] = in[s];
}

__global__ void k_vec_from_orig(const int* __restrict__ slot, int64_t n, const double4* in,
                                double4* out) {
    const int64_t o = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (o < n) out[slot[o]] = in[o];
}

__global__ void k_or_flag(const int* flag, int* acc) {
    if (*flag) *acc = 1;
}

__global__ void k_record3(const double* ev, const double* ke, double* rows, int64_t k) {
    rows[3 * k + 0] = ev[0];
    rows[3 * k + 1] = ev[1];
    rows[3 * k + 2] = *ke;
}

// ---------------------------------------------------------------- reverse step
struct AdjLJ {
    double sig2, eps, inv_eps, inv_sigma, rc, rc2;
    int lfs;
    double uc, dudrc, uc_s, dudrc_s;  // LFS shifts and their sigma derivatives
};

// lv = lvh + gKE m v;  mu = c (a lv + lvh), c = (dt/2)/m as in the kick; a = 1
// for a state that ends a step (F enters v_k and the next half kick), a = 0 for
// the initial state (F(x_0) enters the first half kick only).
__global__ void k_adj_mu(int64_t n, const double4* __restrict__ vel, const double* __restrict__ mass,
                         const double* __restrict__ inv_mass, const double4* __restrict__ lvh,
                         double gke, double a, double half_dt, double4* mu, double4* lv) {
    const int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (s >= n) return;
    const double m = mass[s], c = half_dt * inv_mass[s];
    const double4 v = vel[s], h = lvh[s];
    const double4 l = make_double4(h.x + gke * m * v.x, h.y + gke * m * v.y, h.z + gke * m * v.z, 0.0);
    lv[s] = l;
    mu[s] = make_double4(c * (a * l.x + h.x), c * (a * l.y + h.y), c * (a * l.z + h.z), 0.0);
}

// One pair pass at the positions of a state (full Verlet list, one thread per
// atom).  Per atom: out = (dF/dx)^T mu - gU F + gW dW/dx, then the carries
//   lx += out;  lvh = lv + dt lx   (update_carry),
// and the parameter sums reduced into theta_out[0..1] (d eps, d sigma).
__global__ void __launch_bounds__(kBlock)
k_adj_pairs(const double4* __restrict__ pos, const int* __restrict__ nbr,
            const int* __restrict__ count, int stride, int64_t n, Box3 box, AdjLJ p,
            const double4* __restrict__ mu, double gu, double gw, const double4* __restrict__ lv,
            double dt, double4* lx, double4* lvh, int update_carry, double* part,
            unsigned* ticket, double* theta_out) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const Fold3 f3 = fold3_of(box);
    double th_e = 0.0, th_s = 0.0;
    if (i < n) {
        const double4 pi = pos[i], mi = mu[i];
        double hx = 0.0, hy = 0.0, hz = 0.0;     // (dF/dx)^T mu
        double fx = 0.0, fy = 0.0, fz = 0.0;     // F
        double wx = 0.0, wy = 0.0, wz = 0.0;     // dW/dx
        double gs_x = 0.0, gs_y = 0.0, gs_z = 0.0;
        double ue = 0.0, us = 0.0, we = 0.0, ws = 0.0;
        const int cnt = min(count[i], stride);
        const int* row = nbr + i * static_cast<int64_t>(stride);
        for (int k = 0; k < cnt; ++k) {
            const int j = __ldg(row + k);
            const double4 pj = ldg4(pos + j);
            double dx, dy, dz;
            min_image_wrapped(f3, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z, dx, dy, dz);
            const double s = dx * dx + dy * dy + dz * dz;
            if (!(s < p.rc2)) continue;
            const double t = p.sig2 / s, t3 = t * t * t, t6 = t3 * t3;
            double u = 4.0 * p.eps * (t6 - t3);
            double w = 24.0 * p.eps * (2.0 * t6 - t3);
            double w_s = 24.0 * p.eps * (-12.0 * t6 + 3.0 * t3) / s;
            double u_sig = 4.0 * p.eps * (12.0 * t6 - 6.0 * t3) * p.inv_sigma;
            double w_sig = 24.0 * p.eps * (24.0 * t6 - 6.0 * t3) * p.inv_sigma;
            if (p.lfs) {
                const double r = sqrt(s);
                u = u - p.uc - (r - p.rc) * p.dudrc;
                w = w + r * p.dudrc;
                w_s = w_s + 0.5 * p.dudrc / r;
                u_sig = u_sig - p.uc_s - (r - p.rc) * p.dudrc_s;
                w_sig = w_sig + r * p.dudrc_s;
            }
            const double g = w / s, g_s = (w_s - g) / s, g_sig = w_sig / s;
            const double4 mj = mu[j];
            const double ax = mi.x - mj.x, ay = mi.y - mj.y, az = mi.z - mj.z;
            const double dm = dx * ax + dy * ay + dz * az;
            hx += g * ax + 2.0 * g_s * dx * dm;
            hy += g * ay + 2.0 * g_s * dy * dm;
            hz += g * az + 2.0 * g_s * dz * dm;
            fx += g * dx;
            fy += g * dy;
            fz += g * dz;
            wx += 2.0 * w_s * dx;
            wy += 2.0 * w_s * dy;
            wz += 2.0 * w_s * dz;
            gs_x += g_sig * dx;
            gs_y += g_sig * dy;
            gs_z += g_sig * dz;
            ue += u;
            us += u_sig;
            we += w;
            ws += w_sig;
        }
        const double ox = hx - gu * fx + gw * wx;
        const double oy = hy - gu * fy + gw * wy;
        const double oz = hz - gu * fz + gw * wz;
        // sum_i mu_i . dF_i/dtheta, plus the loss's U and W (each pair is in two rows)
        th_e = p.inv_eps * (mi.x * fx + mi.y * fy + mi.z * fz) +  // dF/d eps = F / eps
               0.5 * p.inv_eps * (gu * ue + gw * we);
        th_s = mi.x * gs_x + mi.y * gs_y + mi.z * gs_z + 0.5 * (gu * us + gw * ws);
        double4 x = lx[i];
        x.x += ox;
        x.y += oy;
        x.z += oz;
        lx[i] = x;
        if (update_carry) {
            const double4 l = lv[i];
            lvh[i] = make_double4(l.x + dt * x.x, l.y + dt * x.y, l.z + dt * x.z, 0.0);
        }
    }
    double v[2] = {th_e, th_s};
    grid_reduce<2>(v, part, ticket, theta_out);
}

AdjLJ adj_params(const md_lj& lj) {
    AdjLJ p;
    p.sig2 = lj.sigma * lj.sigma;
    p.eps = lj.epsilon;
    p.inv_eps = 1.0 / lj.epsilon;
    p.inv_sigma = 1.0 / lj.sigma;
    p.rc = lj.cutoff;
    p.rc2 = lj.cutoff * lj.cutoff;
    p.lfs = lj.truncation == MD_LINEAR_FORCE_SHIFT ? 1 : 0;
    const double t = p.sig2 / p.rc2, t3 = t * t * t, t6 = t3 * t3;
    p.uc = 4.0 * lj.epsilon * (t6 - t3);
    const double wc = 24.0 * lj.epsilon * (2.0 * t6 - t3);
    p.dudrc = -wc / lj.cutoff;
    p.uc_s = 4.0 * lj.epsilon * (12.0 * t6 - 6.0 * t3) / lj.sigma;
    p.dudrc_s = -(24.0 * lj.epsilon * (24.0 * t6 - 6.0 * t3) / lj.sigma) / lj.cutoff;
    return p;
}

Box3 adj_box(const md_system* sys) {
    Box3 b;
    for (int d = 0; d < 3; ++d) {
        b.L[d] = sys->box[d];
        b.inv[d] = sys->inv_box[d];
    }
    return b;
}

int64_t segments(const md_adjoint* a) { return (a->steps + a->every - 1) / a->every; }

// Builds the segment's list and forces from the current state (forward and
// recomputation use this same sequence, so they agree bit for bit).
int segment_start(md_adjoint* a) {
    MDB_TRY(verlet_build(a->list, a->sys, false));
    MDB_TRY(lj_forces_verlet_async(&a->lj, a->sys, a->list));
    return MD_OK;
}

int segment_step(md_adjoint* a) {
    MDB_TRY(vv_pre_async(a->vv, a->sys, a->list));
    k_or_flag<<<1, 1, 0, a->ctx->stream>>>(a->list->d_rebuild_flag, a->flag.as<int>());
    ++a->ctx->launches;
    MDB_TRY(lj_forces_verlet_async(&a->lj, a->sys, a->list));
    MDB_TRY(vv_post_async(a->vv, a->sys));
    return MD_OK;
}

}  // namespace

extern "C" {

int md_adjoint_create(md_context* ctx, md_adjoint** out) {
    graph_epoch_bump();
    if (!ctx || !out) return fail(MD_ERR_INVALID_ARGUMENT, "md_adjoint_create: NULL");
    md_adjoint* a = new (std::nothrow) md_adjoint();
    if (!a) return fail(MD_ERR_OUT_OF_MEMORY, "md_adjoint_create: host allocation");
    a->ctx = ctx;
    *out = a;
    return MD_OK;
}

int md_adjoint_destroy(md_adjoint* a) {
    graph_epoch_bump();
    if (!a) return MD_OK;
    if (a->ctx) cudaStreamSynchronize(a->ctx->stream);
    if (a->list) md_verlet_destroy(a->list);
    if (a->vv) md_integrator_destroy(a->vv);
    a->ck.release();
    a->snap.release();
    a->carry.release();
    a->carry_orig.release();
    a->grads.release();
    a->theta.release();
    a->flag.release();
    delete a;
    return MD_OK;
}

int md_adjoint_forward(md_adjoint* a, md_system* sys, const md_lj* lj, double dt, int64_t steps,
                       int every, double skin, double* rows) {
    if (!a || !sys || !lj) return fail(MD_ERR_INVALID_ARGUMENT, "md_adjoint_forward: NULL");
    if (sys->ctx != a->ctx)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_adjoint_forward: system on another context");
    if (steps < 1 || every < 1 || !(dt > 0.0) || !(skin >= 0.0))
        return fail(MD_ERR_INVALID_ARGUMENT, "md_adjoint_forward: need steps >= 1, every >= 1, "
                                             "dt > 0, skin >= 0");
    if (lj->precision != MD_PRECISION_FP64)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_adjoint_forward: the trajectory is FP64");
    md_context* ctx = a->ctx;
    const int64_t n = sys->n;
    if (n == 0) return fail(MD_ERR_INVALID_ARGUMENT, "md_adjoint_forward: empty system");
    const bool same_list = a->list && a->sys == sys && a->skin == skin &&
                           a->lj.cutoff == lj->cutoff && a->list->box[0] == sys->box[0] &&
                           a->list->box[1] == sys->box[1] && a->list->box[2] == sys->box[2];
    if (!same_list) {
        if (a->list) md_verlet_destroy(a->list);
        a->list = nullptr;
        MDB_TRY(md_verlet_create(ctx, sys->box, lj->cutoff, skin, &a->list));
    }
    if (a->vv) md_integrator_destroy(a->vv);
    a->vv = nullptr;
    MDB_TRY(md_integrator_create_vv(dt, &a->vv));
    a->sys = sys;
    a->lj = *lj;
    a->dt = dt;
    a->skin = skin;
    a->steps = steps;
    a->every = every;
    a->n = n;
    a->have_forward = false;
    const int64_t nseg = segments(a);
    const size_t state = 2 * sizeof(double4) * static_cast<size_t>(n);
    MDB_TRY(a->ck.ensure(state * static_cast<size_t>(nseg + 1)));  // + the final state
    MDB_TRY(a->flag.ensure(sizeof(int)));
    DevBuf drows;
    MDB_TRY(drows.ensure(3 * sizeof(double) * static_cast<size_t>(steps)));
    MDB_CUDA(cudaMemsetAsync(a->flag.ptr, 0, sizeof(int), ctx->stream));
    const int g = grid_for(n, kBlock);
    for (int64_t sg = 0; sg < nseg; ++sg) {
        double4* ckp = a->ck.as<double4>() + 2 * n * sg;
        k_state_to_orig<<<g, kBlock, 0, ctx->stream>>>(sys->cur, n, ckp, ckp + n);
        ++ctx->launches;
        MDB_TRY(segment_start(a));
        const int64_t k0 = sg * every, k1 = std::min(steps, k0 + every);
        for (int64_t k = k0; k < k1; ++k) {
            MDB_TRY(segment_step(a));
            k_record3<<<1, 1, 0, ctx->stream>>>(ctx_result(ctx, kResEnergy), ctx_result(ctx, kResKE),
                                                drows.as<double>(), k);
            ++ctx->launches;
        }
        MDB_CHECK_LAUNCH();
    }
    {
        double4* ckp = a->ck.as<double4>() + 2 * n * nseg;
        k_state_to_orig<<<g, kBlock, 0, ctx->stream>>>(sys->cur, n, ckp, ckp + n);
        ++ctx->launches;
    }
    int bad = 0;
    MDB_CUDA(cudaMemcpyAsync(&bad, a->flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    if (rows)
        MDB_CUDA(cudaMemcpyAsync(rows, drows.ptr, 3 * sizeof(double) * static_cast<size_t>(steps),
                                 cudaMemcpyDeviceToHost, ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    drows.release();
    MDB_TRY(ctx_check_status(ctx));
    if (bad)
        return fail(MD_ERR_RUNTIME,
                    "md_adjoint_forward: an atom pair may have entered the cutoff unlisted within "
                    "a segment (the two largest displacements exceeded the skin %.3g); use a "
                    "larger skin or checkpoint more often", skin);
    a->have_forward = true;
    return MD_OK;
}

int md_adjoint_backward(md_adjoint* a, const double* grad_rows, double grad_theta[2],
                        double* grad_x0, double* grad_v0) {
    if (!a || !grad_rows || !grad_theta)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_adjoint_backward: NULL");
    if (!a->have_forward)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_adjoint_backward: no forward to differentiate");
    md_context* ctx = a->ctx;
    md_system* sys = a->sys;
    const int64_t n = a->n, steps = a->steps, every = a->every, nseg = segments(a);
    if (sys->n != n) return fail(MD_ERR_INVALID_ARGUMENT, "md_adjoint_backward: system resized");
    const size_t vec = sizeof(double4) * static_cast<size_t>(n);
    MDB_TRY(a->snap.ensure(2 * vec * static_cast<size_t>(every + 1)));
    MDB_TRY(a->carry.ensure(4 * vec));
    MDB_TRY(a->carry_orig.ensure(2 * vec));
    MDB_TRY(a->grads.ensure(3 * sizeof(double) * static_cast<size_t>(steps)));
    MDB_TRY(a->theta.ensure(2 * sizeof(double) * static_cast<size_t>(steps + 1)));
    MDB_CUDA(cudaMemcpyAsync(a->grads.ptr, grad_rows, 3 * sizeof(double) * static_cast<size_t>(steps),
                             cudaMemcpyHostToDevice, ctx->stream));
    std::vector<double> hg(grad_rows, grad_rows + 3 * steps);
    double4* lx = a->carry.as<double4>();
    double4* lvh = lx + n;
    double4* mu = lx + 2 * n;
    double4* lv = lx + 3 * n;
    double4* lx_o = a->carry_orig.as<double4>();
    double4* lvh_o = lx_o + n;
    MDB_CUDA(cudaMemsetAsync(a->carry_orig.ptr, 0, 2 * vec, ctx->stream));
    const int g = grid_for(n, kBlock);
    const AdjLJ p = adj_params(a->lj);
    const Box3 box = adj_box(sys);
    const double half_dt = 0.5 * a->dt;
    double* part;
    MDB_TRY(ctx_partials(ctx, 2 * static_cast<size_t>(g), &part));
    double* theta = a->theta.as<double>();
    for (int64_t sg = nseg - 1; sg >= 0; --sg) {
        const int64_t k0 = sg * every, k1 = std::min(steps, k0 + every), len = k1 - k0;
        // recompute the segment from its checkpoint, keeping every state
        const double4* ckp = a->ck.as<double4>() + 2 * n * sg;
        k_state_from_orig<<<g, kBlock, 0, ctx->stream>>>(sys->cur, sys->slot, n, ckp, ckp + n);
        MDB_TRY(segment_start(a));
        double4* snap = a->snap.as<double4>();
        k_snapshot<<<g, kBlock, 0, ctx->stream>>>(sys->cur, n, snap, snap + n);
        for (int64_t j = 1; j <= len; ++j) {
            MDB_TRY(segment_step(a));
            k_snapshot<<<g, kBlock, 0, ctx->stream>>>(sys->cur, n, snap + 2 * n * j,
                                                     snap + 2 * n * j + n);
        }
        ctx->launches += 2 + 2 * len;
        // the carries, into this segment's device order
        k_vec_from_orig<<<g, kBlock, 0, ctx->stream>>>(sys->slot, n, lx_o, lx);
        k_vec_from_orig<<<g, kBlock, 0, ctx->stream>>>(sys->slot, n, lvh_o, lvh);
        for (int64_t j = len; j >= 1; --j) {
            const int64_t k = k0 + j;  // state index; its row is k - 1
            const double* gr = hg.data() + 3 * (k - 1);
            const double4* sp = snap + 2 * n * j;
            k_adj_mu<<<g, kBlock, 0, ctx->stream>>>(n, sp + n, sys->cur.mass, sys->cur.inv_mass,
                                                   lvh, gr[2], 1.0, half_dt, mu, lv);
            k_adj_pairs<<<g, kBlock, 0, ctx->stream>>>(
                sp, a->list->nbr.as<int>(), a->list->count.as<int>(), a->list->stride, n, box, p,
                mu, gr[0], gr[1], lv, a->dt, lx, lvh, 1, part, ctx_counter(ctx, 10),
                theta + 2 * k);
            ctx->launches += 2;
        }
        if (sg == 0) {
            // x_0: F(x_0) enters the first half kick only
            k_adj_mu<<<g, kBlock, 0, ctx->stream>>>(n, snap + n, sys->cur.mass, sys->cur.inv_mass,
                                                   lvh, 0.0, 0.0, half_dt, mu, lv);
            k_adj_pairs<<<g, kBlock, 0, ctx->stream>>>(
                snap, a->list->nbr.as<int>(), a->list->count.as<int>(), a->list->stride, n, box,
                p, mu, 0.0, 0.0, lv, a->dt, lx, lvh, 0, part, ctx_counter(ctx, 10), theta);
            ctx->launches += 2;
        }
        k_vec_to_orig<<<g, kBlock, 0, ctx->stream>>>(sys->cur.orig, n, lx, lx_o);
        k_vec_to_orig<<<g, kBlock, 0, ctx->stream>>>(sys->cur.orig, n, lvh, lvh_o);
        ctx->launches += 4;
        MDB_CHECK_LAUNCH();
    }
    {
        // leave the system where the forward left it (forces too)
        const double4* ckp = a->ck.as<double4>() + 2 * n * nseg;
        k_state_from_orig<<<g, kBlock, 0, ctx->stream>>>(sys->cur, sys->slot, n, ckp, ckp + n);
        ++ctx->launches;
        MDB_TRY(verlet_build(a->list, sys, false));
        MDB_TRY(lj_forces_verlet_async(&a->lj, sys, a->list));
    }
    std::vector<double> th(2 * static_cast<size_t>(steps + 1));
    MDB_CUDA(cudaMemcpyAsync(th.data(), theta, th.size() * sizeof(double), cudaMemcpyDeviceToHost,
                             ctx->stream));
    std::vector<double4> hx, hv;
    if (grad_x0) hx.resize(static_cast<size_t>(n));
    if (grad_v0) hv.resize(static_cast<size_t>(n));
    if (grad_x0)
        MDB_CUDA(cudaMemcpyAsync(hx.data(), lx_o, vec, cudaMemcpyDeviceToHost, ctx->stream));
    if (grad_v0)
        MDB_CUDA(cudaMemcpyAsync(hv.data(), lvh_o, vec, cudaMemcpyDeviceToHost, ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    grad_theta[0] = grad_theta[1] = 0.0;
    for (int64_t k = 0; k <= steps; ++k) {
        grad_theta[0] += th[2 * k];
        grad_theta[1] += th[2 * k + 1];
    }
    for (int64_t o = 0; o < n; ++o) {
        if (grad_x0) {
            grad_x0[3 * o] = hx[o].x;
            grad_x0[3 * o + 1] = hx[o].y;
            grad_x0[3 * o + 2] = hx[o].z;
        }
        if (grad_v0) {
            grad_v0[3 * o] = hv[o].x;
            grad_v0[3 * o + 1] = hv[o].y;
            grad_v0[3 * o + 2] = hv[o].z;
        }
    }
    return ctx_check_status(ctx);
}

int md_lj_hvp(const md_lj* lj, md_system* sys, md_verlet* list, const double* u, double* out,
              double dtheta[2]) {
    if (!lj || !sys || !list || !u || !out)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_lj_hvp: NULL argument");
    MDB_TRY(verlet_ensure_ready(list, sys, "md_lj_hvp"));
    md_context* ctx = sys->ctx;
    const int64_t n = sys->n;
    if (n == 0) {
        if (dtheta) dtheta[0] = dtheta[1] = 0.0;
        return MD_OK;
    }
    const size_t vec = sizeof(double4) * static_cast<size_t>(n);
    DevBuf buf;
    MDB_TRY(buf.ensure(4 * vec + 2 * sizeof(double)));
    double4* uo = buf.as<double4>();
    double4* ud = uo + n;
    double4* res = uo + 2 * n;
    double4* res_o = uo + 3 * n;
    double* th = reinterpret_cast<double*>(uo + 4 * n);
    std::vector<double4> h(static_cast<size_t>(n));
    for (int64_t o = 0; o < n; ++o) h[o] = make_double4(u[3 * o], u[3 * o + 1], u[3 * o + 2], 0.0);
    MDB_CUDA(cudaMemcpyAsync(uo, h.data(), vec, cudaMemcpyHostToDevice, ctx->stream));
    MDB_CUDA(cudaMemsetAsync(res, 0, vec, ctx->stream));
    const int g = grid_for(n, kBlock);
    double* part;
    MDB_TRY(ctx_partials(ctx, 2 * static_cast<size_t>(g), &part));
    k_vec_from_orig<<<g, kBlock, 0, ctx->stream>>>(sys->slot, n, uo, ud);
    k_adj_pairs<<<g, kBlock, 0, ctx->stream>>>(sys->cur.pos, list->nbr.as<int>(),
                                              list->count.as<int>(), list->stride, n,
                                              adj_box(sys), adj_params(*lj), ud, 0.0, 0.0, nullptr,
                                              0.0, res, nullptr, 0, part, ctx_counter(ctx, 10), th);
    k_vec_to_orig<<<g, kBlock, 0, ctx->stream>>>(sys->cur.orig, n, res, res_o);
    ctx->launches += 3;
    MDB_CHECK_LAUNCH();
    double t[2];
    MDB_CUDA(cudaMemcpyAsync(h.data(), res_o, vec, cudaMemcpyDeviceToHost, ctx->stream));
    MDB_CUDA(cudaMemcpyAsync(t, th, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    buf.release();
    for (int64_t o = 0; o < n; ++o) {
        out[3 * o] = h[o].x;
        out[3 * o + 1] = h[o].y;
        out[3 * o + 2] = h[o].z;
    }
    if (dtheta) {
        dtheta[0] = t[0];
        dtheta[1] = t[1];
    }
    return ctx_check_status(ctx);
}

}  // extern "C"
