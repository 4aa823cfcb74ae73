// neighbor.cu -- cell binning (CellList) and Verlet lists (VerletList) on the device.
//
// Binning (neighbor/cell_list.cpp:16-43) assigns each atom the reference's cell
// (wrap, floor((r + L/2) / w), clamp) with bit-identical arithmetic, then counting-
// sorts atoms by the Morton rank of their cell and, within a cell, by original
// index, so the resulting order is a pure function of the positions.
//
// Verlet build (neighbor/verlet_list.cpp:8-42): one warp per cell scans the 27
// neighbouring cells (>= 3 cells per side; the stencil then visits every unordered
// cell pair exactly once from each side) or, for smaller boxes, every atom, and
// compacts hits with __ballot_sync into a fixed-stride row per atom.  Membership
// uses the reference's exact min-image r^2 with the pair ordered by original index
// (r_lo - r_hi), so the pair set is bit-identical to the reference's.
#include <algorithm>
#include <climits>
#include <cmath>
#include <new>

#include "md_device.cuh"
#include "md_internal.cuh"

namespace mdb {

namespace {

constexpr int kBlock = 256;
constexpr int kBuildWarps = 4;
constexpr int kMaxCand = 576;    // candidates staged per warp window (even)

__device__ __forceinline__ bool gate(const int* flag) { return flag == nullptr || *flag != 0; }

// Reference cell id of a position (cell_list.cpp:29-39), exact arithmetic.
__device__ __forceinline__ int cell_of(double x, double y, double z, const Box3& b, double wx,
                                       double wy, double wz, int nx, int ny, int nz) {
    const double rx = fold_exact(x, b.L[0], b.inv[0]);
    const double ry = fold_exact(y, b.L[1], b.inv[1]);
    const double rz = fold_exact(z, b.L[2], b.inv[2]);
    int ix = static_cast<int>(floor(__ddiv_rn(__dadd_rn(rx, __dmul_rn(0.5, b.L[0])), wx)));
    int iy = static_cast<int>(floor(__ddiv_rn(__dadd_rn(ry, __dmul_rn(0.5, b.L[1])), wy)));
    int iz = static_cast<int>(floor(__ddiv_rn(__dadd_rn(rz, __dmul_rn(0.5, b.L[2])), wz)));
    ix = ix < 0 ? 0 : (ix >= nx ? nx - 1 : ix);
    iy = iy < 0 ? 0 : (iy >= ny ? ny - 1 : iy);
    iz = iz < 0 ? 0 : (iz >= nz ? nz - 1 : iz);
    return ix + nx * (iy + ny * iz);
}

struct GridArgs {
    Box3 box;
    double wx, wy, wz;
    int nx, ny, nz, ncells;
    const int* rank_of_cell;
    const int* cell_of_rank;
};

// Kernel bodies take their block index (and count) explicitly: a batched launch
// gives each replica's blocks their own rank, and each replica runs exactly the
// blocks of its solo launch.
__device__ __forceinline__ void zero_int_body(int* a, int64_t n, unsigned block, unsigned nblocks) {
    for (int64_t k = block * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<int64_t>(nblocks) * blockDim.x)
        a[k] = 0;
}

__global__ void k_zero_int(int* a, int64_t n, const int* flag) {
    if (!gate(flag)) return;
    zero_int_body(a, n, blockIdx.x, gridDim.x);
}

__device__ __forceinline__ void bin_body(const double4* __restrict__ pos, int64_t n, const GridArgs& g,
                                         int* atom_rank, int* counts, unsigned block) {
    const int64_t k = block * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= n) return;
    const double4 p = pos[k];
    const int c = cell_of(p.x, p.y, p.z, g.box, g.wx, g.wy, g.wz, g.nx, g.ny, g.nz);
    const int r = g.rank_of_cell[c];
    atom_rank[k] = r;
    atomicAdd(counts + r, 1);
}

__global__ void k_bin(const double4* __restrict__ pos, int64_t n, GridArgs g, int* atom_rank,
                      int* counts, const int* flag) {
    if (!gate(flag)) return;
    bin_body(pos, n, g, atom_rank, counts, blockIdx.x);
}

// Exclusive scan of counts[0..m) into start[0..m] (start[m] = total) in three
// passes: each 1024-thread block scans 4096 consecutive counts (coalesced), the
// block totals are scanned by one block, and the block offsets are added back.
constexpr int kScanBlock = 1024, kScanItems = 4;

__device__ __forceinline__ int block_exclusive_scan(int v, int* total) {
    __shared__ int warp_tot[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < (blockDim.x >> 5) ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        warp_tot[lane] = w;
    }
    __syncthreads();
    const int excl = (warp > 0 ? warp_tot[warp - 1] : 0) + x - v;
    *total = warp_tot[(blockDim.x >> 5) - 1];
    __syncthreads();
    return excl;
}

// single: the grid is one block, whose scan is already the whole exclusive scan;
// it then also writes the end sentinel start[m] (k_scan_top and k_scan_add would
// write it and add nothing), saving their launches.
__device__ __forceinline__ void scan_blocks_body(const int* __restrict__ counts, int* start, int m,
                                                 int* bsum, int single, unsigned block) {
    const int base = block * kScanBlock * kScanItems;
    int v[kScanItems];
    int sum = 0;
#pragma unroll
    for (int u = 0; u < kScanItems; ++u) {
        const int i = base + u * kScanBlock + threadIdx.x;  // coalesced
        v[u] = i < m ? counts[i] : 0;
    }
    // scan in item-major order: thread t owns elements base + u*1024 + t
    int run_base = 0;
#pragma unroll
    for (int u = 0; u < kScanItems; ++u) {
        int tot;
        const int ex = block_exclusive_scan(v[u], &tot);
        const int i = base + u * kScanBlock + threadIdx.x;
        if (i < m) start[i] = run_base + ex;
        run_base += tot;
        sum += v[u];
    }
    (void)sum;
    if (threadIdx.x == 0) {
        bsum[block] = run_base;
        if (single) start[m] = run_base;
    }
}

__global__ void __launch_bounds__(kScanBlock) k_scan_blocks(const int* __restrict__ counts,
                                                            int* start, int m, int* bsum,
                                                            const int* flag, int single) {
    if (!gate(flag)) return;
    scan_blocks_body(counts, start, m, bsum, single, blockIdx.x);
}

__device__ __forceinline__ void scan_top_body(int* bsum, int nb, int* start, int m) {
    int carry = 0;
    for (int b0 = 0; b0 < nb; b0 += kScanBlock) {
        const int b = b0 + threadIdx.x;
        const int v = b < nb ? bsum[b] : 0;
        int tot;
        const int ex = block_exclusive_scan(v, &tot);
        if (b < nb) bsum[b] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) start[m] = carry;
}

__global__ void __launch_bounds__(kScanBlock) k_scan_top(int* bsum, int nb, int* start, int m,
                                                         const int* flag) {
    if (!gate(flag)) return;
    scan_top_body(bsum, nb, start, m);
}

__device__ __forceinline__ void scan_add_body(int* start, int m, const int* __restrict__ bsum,
                                              unsigned block) {
    const int base = block * kScanBlock * kScanItems;
    const int off = bsum[block];
#pragma unroll
    for (int u = 0; u < kScanItems; ++u) {
        const int i = base + u * kScanBlock + threadIdx.x;
        if (i < m) start[i] += off;
    }
}

__global__ void __launch_bounds__(kScanBlock) k_scan_add(int* start, int m, const int* __restrict__ bsum,
                                                         const int* flag) {
    if (!gate(flag)) return;
    scan_add_body(start, m, bsum, blockIdx.x);
}

__device__ __forceinline__ void scatter_body(const int* __restrict__ atom_rank, int64_t n,
                                             const int* __restrict__ start, int* fill, int* sorted,
                                             unsigned block) {
    const int64_t k = block * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= n) return;
    const int r = atom_rank[k];
    const int at = atomicAdd(fill + r, 1);
    sorted[start[r] + at] = static_cast<int>(k);
}

__global__ void k_scatter(const int* __restrict__ atom_rank, int64_t n, const int* __restrict__ start,
                          int* fill, int* sorted, const int* flag) {
    if (!gate(flag)) return;
    scatter_body(atom_rank, n, start, fill, sorted, blockIdx.x);
}

// Within each cell, order atoms by original index.  One warp per cell: each atom's
// rank is the number of smaller keys (keys are distinct), taken from registers
// for up to 32 atoms and from shared memory up to kOrderMax; a cell beyond that
// falls back to an insertion sort by lane 0.
constexpr int kOrderWarps = 8;   // k_cell_order runs 256-thread blocks
constexpr int kOrderMax = 512;   // atoms per cell ordered in shared memory

__device__ __forceinline__ void cell_order_body(int* sorted, const int* __restrict__ start, int m,
                                                const int* __restrict__ orig, unsigned block) {
    const int lane = threadIdx.x & 31;
    const int r = static_cast<int>((block * blockDim.x + threadIdx.x) >> 5);
    if (r >= m) return;
    const int s0 = start[r], s1 = start[r + 1], c = s1 - s0;
    if (c <= 1) return;
    if (c <= 32) {
        const int v = lane < c ? sorted[s0 + lane] : 0;
        const int key = lane < c ? orig[v] : 0x7fffffff;
        int rank = 0;
        for (int o = 0; o < c; ++o) rank += (__shfl_sync(0xffffffffu, key, o) < key) ? 1 : 0;
        __syncwarp();
        if (lane < c) sorted[s0 + rank] = v;
        return;
    }
    if (c <= kOrderMax) {
        // rank sort by the warp: stage (key, atom) in shared memory, each lane
        // ranks every 32nd element against all of the cell's keys
        __shared__ int s_key[kOrderWarps][kOrderMax], s_val[kOrderWarps][kOrderMax];
        const int w = threadIdx.x >> 5;
        for (int t = lane; t < c; t += 32) {
            const int v = sorted[s0 + t];
            s_val[w][t] = v;
            s_key[w][t] = orig[v];
        }
        __syncwarp();
        for (int t = lane; t < c; t += 32) {
            const int key = s_key[w][t];
            int rank = 0;
            for (int o = 0; o < c; ++o) rank += s_key[w][o] < key ? 1 : 0;
            sorted[s0 + rank] = s_val[w][t];
        }
        return;
    }
    if (lane != 0) return;  // very crowded cells: insertion sort by one thread
    for (int a = s0 + 1; a < s1; ++a) {
        const int v = sorted[a];
        const int key = orig[v];
        int b = a - 1;
        while (b >= s0 && orig[sorted[b]] > key) {
            sorted[b + 1] = sorted[b];
            --b;
        }
        sorted[b + 1] = v;
    }
}

__global__ void __launch_bounds__(32 * kOrderWarps)
k_cell_order(int* sorted, const int* __restrict__ start, int m,
                             const int* __restrict__ orig, const int* flag) {
    if (!gate(flag)) return;
    cell_order_body(sorted, start, m, orig, blockIdx.x);
}

// Gathers every per-atom array into the new order.  Forces are skipped when the
// caller recomputes them right after the rebuild (fused stepping loops).
__device__ __forceinline__ void permute_body(const md_atoms& src, const md_atoms& dst,
                                             const int* __restrict__ perm, int* slot, int64_t n,
                                             int with_forces, unsigned block) {
    const int64_t s = block * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (s >= n) return;
    const int k = perm[s];
    dst.pos[s] = src.pos[k];
    dst.vx[s] = src.vx[k];
    dst.vy[s] = src.vy[k];
    dst.vz[s] = src.vz[k];
    if (with_forces) {
        dst.fx[s] = src.fx[k];
        dst.fy[s] = src.fy[k];
        dst.fz[s] = src.fz[k];
    }
    dst.mass[s] = src.mass[k];
    dst.inv_mass[s] = src.inv_mass[k];
    dst.charge[s] = src.charge[k];
    dst.mol[s] = src.mol[k];
    const int o = src.orig[k];
    dst.orig[s] = o;
    slot[o] = static_cast<int>(s);
}

__global__ void k_permute_gated(md_atoms src, md_atoms dst, const int* __restrict__ perm,
                                int* slot, int64_t n, const int* flag, int with_forces) {
    if (!gate(flag)) return;
    permute_body(src, dst, perm, slot, n, with_forces, blockIdx.x);
}

__device__ __forceinline__ void copy_atoms_body(const md_atoms& src, const md_atoms& dst, int64_t n,
                                                int with_forces, unsigned block) {
    const int64_t s = block * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (s >= n) return;
    dst.pos[s] = src.pos[s];
    dst.vx[s] = src.vx[s];
    dst.vy[s] = src.vy[s];
    dst.vz[s] = src.vz[s];
    if (with_forces) {
        dst.fx[s] = src.fx[s];
        dst.fy[s] = src.fy[s];
        dst.fz[s] = src.fz[s];
    }
    dst.mass[s] = src.mass[s];
    dst.inv_mass[s] = src.inv_mass[s];
    dst.charge[s] = src.charge[s];
    dst.mol[s] = src.mol[s];
    dst.orig[s] = src.orig[s];
}

// The copy back also writes what the rebuild needs from the same positions after
// the list build: the reference positions of the rebuild test (and the rebuild
// count), and for a mixed force the fixed-point copy (q, or none).
__global__ void k_copy_atoms(md_atoms src, md_atoms dst, int64_t n, const int* flag,
                             int with_forces, double4* ref, int* total, int4* q, double sx,
                             double sy, double sz) {
    if (!gate(flag)) return;
    copy_atoms_body(src, dst, n, with_forces, blockIdx.x);
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k < n) {
        const double4 p = src.pos[k];
        ref[k] = p;
        if (q) q[k] = quantize_position(p, sx, sy, sz);
    }
    if (k == 0 && total) ++*total;
}

// Exact candidate test with the pair ordered by original index.
__device__ __forceinline__ bool within(const Box3& b, double4 pi, double4 pj, double rl2) {
    double dx, dy, dz;
    const Fold3 f = fold3_of(b);
    if (pi.w < pj.w) min_image_wrapped(f, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z, dx, dy, dz);
    else min_image_wrapped(f, pj.x, pj.y, pj.z, pi.x, pi.y, pi.z, dx, dy, dz);
    return norm2_exact(dx, dy, dz) < rl2;
}

// One warp per (Morton-ranked) cell; device order == sorted order, so cell r holds
// atoms [start[r], start[r+1]).  The candidates of the 27 surrounding cells are
// staged in shared memory once per cell as FP32 coordinates relative to the cell
// centre (nearest periodic image); then each lane takes one atom of the cell and
// scans the staged candidates (broadcast reads, two candidates per packed FP32x2
// step), appending hits to its own row.
// A candidate is listed when its FP32 r^2 is below the list cutoff^2 widened by
// 2^-12 -- far more than the FP32 error of these coordinates -- so the rows hold
// every pair the reference lists plus, at most, pairs within a 1.2e-4 relative
// shell outside the list cutoff.  Every consumer tests its own cutoff, which is
// below the list cutoff, so the extra entries never contribute; the exported
// pair set (forEachPair) applies the reference's exact test to the positions of
// the build and is bit-identical to the reference's.
// Rows list candidates in stencil order, atoms of a cell in sorted order.
__device__ __forceinline__ void verlet_cells_body(const double4* __restrict__ pos,
                                                  const int* __restrict__ start, const GridArgs& g,
                                                  double rl2, int* __restrict__ nbr,
                                                  int* __restrict__ count, int stride,
                                                  uint32_t* status, int* max_count, int groups,
                                                  unsigned block) {
    // Candidates in pairs, structure-of-arrays within a pair so that two
    // candidates are tested with one packed FP32x2 instruction per step:
    // s_a[p] = (-x0, -x1, -y0, -y1), s_b[p] = (-z0, -z1, j0, j1).
    __shared__ float4 s_a[kBuildWarps][kMaxCand / 2];
    __shared__ float4 s_b[kBuildWarps][kMaxCand / 2];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // `groups` warps share a crowded cell, each taking every groups-th run of 32 atoms
    const int wid = static_cast<int>(block) * kBuildWarps + warp;
    const int r = wid / groups, grp = wid % groups;
    if (r >= g.ncells) return;
    const int cell = g.cell_of_rank[r];
    const int cx = cell % g.nx, cy = (cell / g.nx) % g.ny, cz = cell / (g.nx * g.ny);
    const double ox = -0.5 * g.box.L[0] + (cx + 0.5) * g.wx;
    const double oy = -0.5 * g.box.L[1] + (cy + 0.5) * g.wy;
    const double oz = -0.5 * g.box.L[2] + (cz + 0.5) * g.wz;
    const float hi_thr = static_cast<float>(rl2 * (1.0 + 1.0 / 4096.0));
    // half widths of the cell's box, widened a little (its atoms were binned with
    // the reference arithmetic, their offsets here are FP64 then FP32)
    const float hwx = static_cast<float>(0.5 * g.wx * (1.0 + 1e-6)) + 1e-6f;
    const float hwy = static_cast<float>(0.5 * g.wy * (1.0 + 1e-6)) + 1e-6f;
    const float hwz = static_cast<float>(0.5 * g.wz * (1.0 + 1e-6)) + 1e-6f;
    // the 27 neighbour cell ranges (lane q holds cell q of the stencil)
    int beg = 0, cnt = 0;
    if (lane < 27) {
        int jx = cx + (lane % 3) - 1, jy = cy + ((lane / 3) % 3) - 1, jz = cz + (lane / 9) - 1;
        jx = jx < 0 ? jx + g.nx : (jx >= g.nx ? jx - g.nx : jx);
        jy = jy < 0 ? jy + g.ny : (jy >= g.ny ? jy - g.ny : jy);
        jz = jz < 0 ? jz + g.nz : (jz >= g.nz ? jz - g.nz : jz);
        const int rr = g.rank_of_cell[jx + g.nx * (jy + g.ny * jz)];
        beg = start[rr];
        cnt = start[rr + 1] - beg;
    }
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    const int excl = incl - cnt;
    const int a0 = start[r], a1 = start[r + 1];
    int local_max = 0;
    for (int wb = 0; wb < total; wb += kMaxCand) {
        const int wlen = min(kMaxCand, total - wb);
        __syncwarp();
        // stage candidates [wb, wb + wlen) cell by cell, keeping only those within
        // the list cutoff of the cell's own box (a quarter of the 27-cell volume is
        // farther from every atom of the cell); order is kept
        int ns = 0;
        for (int q = 0; q < 27; ++q) {
            const int qb = __shfl_sync(0xffffffffu, beg, q);
            const int qo = __shfl_sync(0xffffffffu, excl, q);
            const int qc = __shfl_sync(0xffffffffu, cnt, q);
            const int lo = max(qo, wb), hi = min(qo + qc, wb + wlen);
            for (int gb = lo; gb < hi; gb += 32) {
                const int gt = gb + lane;
                const int j = qb + (gt - qo);
                double vx = 0.0, vy = 0.0, vz = 0.0;
                bool keep = false;
                if (gt < hi) {
                    const double4 pj = ldg4(pos + j);
                    vx = pj.x - ox;
                    vy = pj.y - oy;
                    vz = pj.z - oz;
                    vx -= g.box.L[0] * rint(vx * g.box.inv[0]);
                    vy -= g.box.L[1] * rint(vy * g.box.inv[1]);
                    vz -= g.box.L[2] * rint(vz * g.box.inv[2]);
                    const float ex = fmaxf(fabsf(static_cast<float>(vx)) - hwx, 0.f);
                    const float ey = fmaxf(fabsf(static_cast<float>(vy)) - hwy, 0.f);
                    const float ez = fmaxf(fabsf(static_cast<float>(vz)) - hwz, 0.f);
                    keep = fmaf(ez, ez, fmaf(ey, ey, ex * ex)) < hi_thr;
                }
                const unsigned m = __ballot_sync(0xffffffffu, keep);
                if (keep) {
                    const int tt = ns + __popc(m & ((1u << lane) - 1u)), pr = tt >> 1, h = tt & 1;
                    float* A = reinterpret_cast<float*>(&s_a[warp][pr]);
                    float* B = reinterpret_cast<float*>(&s_b[warp][pr]);
                    A[h] = -static_cast<float>(vx);
                    A[2 + h] = -static_cast<float>(vy);
                    B[h] = -static_cast<float>(vz);
                    B[2 + h] = __int_as_float(j);
                }
                ns += __popc(m);
            }
        }
        if ((ns & 1) && lane == 0) {  // pad the odd slot: infinitely far, no atom
            float* A = reinterpret_cast<float*>(&s_a[warp][ns >> 1]);
            float* B = reinterpret_cast<float*>(&s_b[warp][ns >> 1]);
            A[1] = A[3] = B[1] = 1e30f;
            B[3] = __int_as_float(-1);
        }
        __syncwarp();
        for (int ib = a0 + 32 * grp; ib < a1; ib += 32 * groups) {
            const int i = ib + lane;
            const bool active = i < a1;
            double4 pi = make_double4(0.0, 0.0, 0.0, 0.0);
            float fx = 0.f, fy = 0.f, fz = 0.f;
            int c = 0;
            if (active) {
                pi = pos[i];
                double ux = pi.x - ox, uy = pi.y - oy, uz = pi.z - oz;
                ux -= g.box.L[0] * rint(ux * g.box.inv[0]);
                uy -= g.box.L[1] * rint(uy * g.box.inv[1]);
                uz -= g.box.L[2] * rint(uz * g.box.inv[2]);
                fx = static_cast<float>(ux);
                fy = static_cast<float>(uy);
                fz = static_cast<float>(uz);
                c = wb == 0 ? 0 : count[i];
            }
            int* row = nbr + static_cast<int64_t>(active ? i : 0) * stride;
            // Per candidate pair: packed FP32x2 distances and predicated appends.
            const float2 fx2 = make_float2(fx, fx), fy2 = make_float2(fy, fy),
                         fz2 = make_float2(fz, fz);
            const int npairs = (ns + 1) >> 1;
#pragma unroll 2
            for (int pr = 0; pr < npairs; ++pr) {
                const float4 A = s_a[warp][pr], B = s_b[warp][pr];
                const float2 dx = __fadd2_rn(fx2, make_float2(A.x, A.y));
                const float2 dy = __fadd2_rn(fy2, make_float2(A.z, A.w));
                const float2 dz = __fadd2_rn(fz2, make_float2(B.x, B.y));
                const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
                const int j0 = __float_as_int(B.z), j1 = __float_as_int(B.w);
                const bool h0 = active && r2.x < hi_thr && j0 != i;
                const bool h1 = active && r2.y < hi_thr && j1 != i;
                if (h0 && c < stride) row[c] = j0;
                c += h0 ? 1 : 0;
                if (h1 && c < stride) row[c] = j1;
                c += h1 ? 1 : 0;
            }
            if (active) {
                count[i] = c;
                local_max = max(local_max, c);
            }
        }
    }
    const int mx = __reduce_max_sync(0xffffffffu, local_max);
    if (lane == 0) {
        if (mx > 0) atomicMax(max_count, mx);
        if (mx > stride) atomicOr(status, MD_STATUS_NEIGHBOR_OVERFLOW);
    }
}

__global__ void __launch_bounds__(kBuildWarps * 32)
k_verlet_cells(const double4* __restrict__ pos, const int* __restrict__ start, GridArgs g,
               double rl2, int* __restrict__ nbr, int* __restrict__ count, int stride,
               uint32_t* status, int* max_count, const int* flag, int groups) {
    if (!gate(flag)) return;
    verlet_cells_body(pos, start, g, rl2, nbr, count, stride, status, max_count, groups, blockIdx.x);
}

// Boxes with fewer than 3 cells per side (verlet_list.cpp:26-33): one warp per atom
// scans every other atom.
__device__ __forceinline__ void brute_body(const double4* __restrict__ pos, int64_t n,
                                           const Box3& box, double rl2, int* __restrict__ nbr,
                                           int* __restrict__ count, int stride, uint32_t* status,
                                           int* max_count, unsigned block) {
    const int lane = threadIdx.x & 31;
    const int64_t i = (block * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
    if (i >= n) return;
    const double4 pi = pos[i];
    int base = 0;
    for (int64_t t0 = 0; t0 < n; t0 += 32) {
        const int64_t j = t0 + lane;
        bool hit = false;
        if (j < n && j != i) hit = within(box, pi, ldg4(pos + j), rl2);
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (hit) {
            const int at = base + __popc(m & ((1u << lane) - 1u));
            if (at < stride) nbr[i * stride + at] = static_cast<int>(j);
        }
        base += __popc(m);
    }
    if (lane == 0) {
        count[i] = base;
        atomicMax(max_count, base);
        if (base > stride) atomicOr(status, MD_STATUS_NEIGHBOR_OVERFLOW);
    }
}

__global__ void k_verlet_brute(const double4* __restrict__ pos, int64_t n, Box3 box, double rl2,
                               int* __restrict__ nbr, int* __restrict__ count, int stride,
                               uint32_t* status, int* max_count, const int* flag) {
    if (!gate(flag)) return;
    brute_body(pos, n, box, rl2, nbr, count, stride, status, max_count, blockIdx.x);
}

// ---------------------------------------------------------------- halo tiles
constexpr int kPlanEntries = 512;  // >= kHaloSpan * 27, a power of two

// Ranks of the cells holding sorted atoms a and b (the largest r with
// start[r] <= a), one 16-way search per half warp: four rounds of one coalesced
// probe per lane for 50k cells.  Every lane returns both.
__device__ __forceinline__ int2 cell_ranks_of(const int* __restrict__ start, int m, int64_t a,
                                              int64_t b, int lane) {
    const int half = lane >> 4, hl = lane & 15;
    const int64_t x = half ? b : a;
    int lo = 0, hi = m;  // start[lo] <= x < start[hi] (start[m] = n)
    while (__any_sync(0xffffffffu, hi - lo > 1)) {
        const bool open = hi - lo > 1;
        const int step = (hi - lo + 15) / 16;
        const int p = lo + (hl + 1) * step;
        const bool le = open && p < hi && start[p] <= x;
        const unsigned mask = __ballot_sync(0xffffffffu, le);
        const int k = __popc((mask >> (16 * half)) & 0xffffu);  // probes are monotone
        if (open) {
            hi = min(hi, lo + (k + 1) * step);
            lo += k * step;
        }
    }
    return make_int2(__shfl_sync(0xffffffffu, lo, 0), __shfl_sync(0xffffffffu, lo, 16));
}

// Plan of the halo tiles, one warp per tile (kHaloAtoms consecutive sorted
// atoms): the cell ranks the tile's atoms span, their 27-cell neighbourhoods
// sorted (bitonic, in shared memory) and merged into runs of consecutive ranks --
// each run one contiguous range of sorted atoms -- and each run's first slot in
// the staged tile.  A tile spanning more than kHaloSpan cells, needing more than
// kHaloRuns runs or kHaloCap slots, or lying inside one crowded cell, is not
// staged (meta.x = -1).
constexpr int kPlanWarps = 8;

__global__ void __launch_bounds__(32 * kPlanWarps)
k_halo_plan(const int* __restrict__ start, GridArgs g, int64_t n, int64_t tiles,
            int2* __restrict__ runs, int2* __restrict__ meta, const int* flag) {
    if (!gate(flag)) return;
    __shared__ int s_ent[kPlanWarps][kPlanEntries];
    __shared__ int s_beg[kPlanWarps][kHaloRuns], s_end[kPlanWarps][kHaloRuns];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t b = static_cast<int64_t>(blockIdx.x) * kPlanWarps + warp;
    if (b >= tiles) return;  // the whole warp; no block-wide barrier follows
    const int64_t a0 = b * kHaloAtoms, a1 = min(n, a0 + kHaloAtoms) - 1;
    const int2 rr = cell_ranks_of(start, g.ncells, a0, a1, lane);
    const int r0 = rr.x, r1 = rr.y;
    // inside one cell whose atoms run past both ends of the tile: the list build
    // writes slots for a cell's first and last tile only
    const bool inner = r0 == r1 && start[r0] < a0 && start[r0 + 1] - 1 > a1;
    if (inner || r1 - r0 + 1 > kHaloSpan) {
        if (lane == 0) meta[b] = make_int2(-1, 0);
        return;
    }
    int* ent = s_ent[warp];
    const int ne = (r1 - r0 + 1) * 27;
    const int np2 = ne <= 256 ? 256 : kPlanEntries;  // sort only the filled power of two
#pragma unroll
    for (int k = 0; k < kPlanEntries / 32; ++k) {  // unrolled: the loads go out together
        const int e = lane + 32 * k;
        if (e >= np2) break;
        int v = 0x7fffffff;
        if (e < ne) {
            const int cell = g.cell_of_rank[r0 + e / 27], q = e % 27;
            const int cx = cell % g.nx, cy = (cell / g.nx) % g.ny, cz = cell / (g.nx * g.ny);
            int jx = cx + (q % 3) - 1, jy = cy + ((q / 3) % 3) - 1, jz = cz + (q / 9) - 1;
            jx = jx < 0 ? jx + g.nx : (jx >= g.nx ? jx - g.nx : jx);
            jy = jy < 0 ? jy + g.ny : (jy >= g.ny ? jy - g.ny : jy);
            jz = jz < 0 ? jz + g.nz : (jz >= g.nz ? jz - g.nz : jz);
            v = g.rank_of_cell[jx + g.nx * (jy + g.ny * jz)];
        }
        ent[e] = v;
    }
    __syncwarp();
    for (int k = 2; k <= np2; k <<= 1) {  // bitonic sort, ascending
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int e = lane; e < np2; e += 32) {
                const int p = e ^ j;
                if (p > e) {
                    const int x = ent[e], y = ent[p];
                    if ((x > y) == ((e & k) == 0)) {
                        ent[e] = y;
                        ent[p] = x;
                    }
                }
            }
            __syncwarp();
        }
    }
    // runs of consecutive distinct ranks (duplicates neither open nor close one)
    int nopen = 0, nclose = 0;
    for (int c = 0; c < ne; c += 32) {
        const int e = c + lane;
        const int v = e < ne ? ent[e] : 0;
        const bool opens = e < ne && (e == 0 || v > ent[e - 1] + 1);
        const bool closes = e < ne && (e == ne - 1 || ent[e + 1] > v + 1);
        const unsigned mo = __ballot_sync(0xffffffffu, opens);
        const unsigned mc = __ballot_sync(0xffffffffu, closes);
        const unsigned below = (1u << lane) - 1u;
        const int io = nopen + __popc(mo & below), ic = nclose + __popc(mc & below);
        if (opens && io < kHaloRuns) s_beg[warp][io] = v;   // first rank of a run
        if (closes && ic < kHaloRuns) s_end[warp][ic] = v;  // last rank of a run
        nopen += __popc(mo);
        nclose += __popc(mc);
    }
    __syncwarp();
    const int nr = nopen;
    if (nr > kHaloRuns) {
        if (lane == 0) meta[b] = make_int2(-1, 0);
        return;
    }
    // run atoms [start[first rank], start[last rank + 1]) -> slot bases (exclusive
    // scan, two runs per lane)
    int len[2], beg[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int t = 2 * lane + h;
        beg[h] = t < nr ? start[s_beg[warp][t]] : 0;
        len[h] = t < nr ? start[s_end[warp][t] + 1] - beg[h] : 0;
    }
    const int pair = len[0] + len[1];
    int incl = pair;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    const int base0 = incl - pair;
    int2* out = runs + b * kHaloRuns;
    if (2 * lane < nr) out[2 * lane] = make_int2(beg[0], base0);
    if (2 * lane + 1 < nr) out[2 * lane + 1] = make_int2(beg[1], base0 + len[0]);
    if (lane == 0) meta[b] = make_int2(total <= kHaloCap ? nr : -1, total);
}

// Rows of a planned tile as 16-bit byte offsets of 16-byte slots (slot = base of
// the run holding j + j - the run's first atom; kHaloCap * 16 < 2^16), the last
// 8-entry chunk padded with the atom's own slot (r^2 = 0, which the force kernels
// skip, so they read whole chunks without a count test).  Four threads per atom,
// one 8-entry chunk (two 16-byte loads, one 16-byte store) per step.  A neighbour
// outside the tile's runs (not possible for a list built from the same cells)
// un-stages the tile.
constexpr int kRowsThreads = 4 * kHaloAtoms;

struct HaloRun {
    int shift;  // first atom - first slot: slot = j - shift
    int base;   // first slot
    int len;    // atoms in the run
    int pad;
};

// The run holding j: six fixed steps over first atoms padded with INT_MAX to
// kHaloRuns entries (no bounds test), the position carried as a byte offset so
// that each step is one shared load at a constant offset, one compare and one
// predicated add; then one 16-byte read of the run.  Any j (also one read past
// the row's end, whose result is not used) stays inside the table.
__device__ __forceinline__ unsigned halo_slot(int j, const int* s_beg, const HaloRun* s_run,
                                              bool& ok) {
    const char* sb = reinterpret_cast<const char*>(s_beg);
    unsigned tb = 0u;  // 4 * run index
#pragma unroll
    for (int step = kHaloRuns / 2; step > 0; step >>= 1)
        if (*reinterpret_cast<const int*>(sb + tb + 4 * step) <= j) tb += 4u * step;
    const HaloRun r = *reinterpret_cast<const HaloRun*>(reinterpret_cast<const char*>(s_run) + 4u * tb);
    const int slot = j - r.shift;
    ok = static_cast<unsigned>(slot - r.base) < static_cast<unsigned>(r.len);
    return static_cast<unsigned>(slot) << 4;
}

__global__ void __launch_bounds__(kRowsThreads)
k_halo_rows(const int* __restrict__ nbr, const int* __restrict__ count, int stride, int64_t n,
            const int2* __restrict__ runs, int2* meta, uint16_t* __restrict__ nbr16,
            const int* flag) {
    static_assert(kRowsThreads >= kHaloRuns, "one thread per run");
    if (!gate(flag)) return;
    __shared__ int s_beg[kHaloRuns];
    __shared__ HaloRun s_run[kHaloRuns];
    const int b = blockIdx.x, tid = threadIdx.x;
    const int2 m = meta[b];
    if (m.x <= 0) return;
    const int nr = m.x;
    if (tid < kHaloRuns) {
        const int2* tr = runs + static_cast<int64_t>(b) * kHaloRuns;
        int beg = INT_MAX;
        HaloRun hr{0, 0, 0, 0};
        if (tid < nr) {
            const int2 r = tr[tid];
            const int next = tid + 1 < nr ? tr[tid + 1].y : m.y;
            beg = r.x;
            hr = HaloRun{r.x - r.y, r.y, next - r.y, 0};
        }
        s_beg[tid] = beg;
        s_run[tid] = hr;
    }
    __syncthreads();
    const int64_t i = static_cast<int64_t>(b) * kHaloAtoms + (tid >> 2);
    bool bad = false;
    if (i < n) {  // thread t converts chunks (t & 3), (t & 3) + 4, ... of atom t >> 2
        const int c = min(count[i], stride);
        const int4* src = reinterpret_cast<const int4*>(nbr + i * stride);
        uint4* dst = reinterpret_cast<uint4*>(nbr16 + i * stride);
        bool ok_self;
        const unsigned self = halo_slot(static_cast<int>(i), s_beg, s_run, ok_self);
        bad = !ok_self;
        for (int ch = tid & 3; 8 * ch < c; ch += 4) {
            const int4 a0 = __ldg(src + 2 * ch), a1 = __ldg(src + 2 * ch + 1);
            const int js[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const int rem = c - 8 * ch;  // entries of this chunk inside the row
            unsigned off[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                bool ok;
                const unsigned o = halo_slot(js[k], s_beg, s_run, ok);
                off[k] = k < rem ? o : self;
                bad = bad || (k < rem && !ok);
            }
            dst[ch] = make_uint4(off[0] | (off[1] << 16), off[2] | (off[3] << 16),
                                 off[4] | (off[5] << 16), off[6] | (off[7] << 16));
        }
    }
    if (__syncthreads_or(bad) && tid == 0) meta[b].x = -1;
}

__device__ __forceinline__ void store_ref_body(const double4* __restrict__ pos, double4* ref,
                                               int64_t n, int* total, unsigned block) {
    const int64_t k = block * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k < n) ref[k] = pos[k];
    if (k == 0 && total) ++*total;
}

__global__ void k_store_ref(const double4* __restrict__ pos, double4* ref, int64_t n,
                            const int* flag, int* total) {
    if (!gate(flag)) return;
    store_ref_body(pos, ref, n, total, blockIdx.x);
}

// verlet_list.cpp:44-63: top-2 min-image displacements; decides on device.
__global__ void k_displacement(const double4* __restrict__ pos, int64_t n, Box3 box,
                               DispArgs d) {
    const Fold3 f3 = fold3_of(box);
    double a1 = 0.0, a2 = 0.0;
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double4 p = pos[k], q = d.ref[k];
        double dx, dy, dz;
        min_image_wrapped(f3, p.x, p.y, p.z, q.x, q.y, q.z, dx, dy, dz);
        top2_insert(a1, a2, norm2_exact(dx, dy, dz));
    }
    top2_grid(a1, a2, d);
}

inline uint32_t spread3(uint32_t v) {
    uint32_t x = v & 0x3ffu;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

GridArgs make_args(const CellGrid& gr, const md_system* sys) {
    GridArgs g;
    for (int d = 0; d < 3; ++d) {
        g.box.L[d] = sys->box[d];
        g.box.inv[d] = sys->inv_box[d];
    }
    g.wx = gr.width[0];
    g.wy = gr.width[1];
    g.wz = gr.width[2];
    g.nx = gr.nx;
    g.ny = gr.ny;
    g.nz = gr.nz;
    g.ncells = gr.ncells;
    g.rank_of_cell = gr.rank_of_cell;
    g.cell_of_rank = gr.cell_of_rank;
    return g;
}

Box3 make_box(const md_system* sys) {
    Box3 b;
    for (int d = 0; d < 3; ++d) {
        b.L[d] = sys->box[d];
        b.inv[d] = sys->inv_box[d];
    }
    return b;
}

// Scratch for one sort: atom_rank (n) + counts (m) + fill (m).
int sort_scratch(md_context* ctx, int64_t n, int m, int** atom_rank, int** counts, int** fill) {
    void* p;
    const size_t bsums = static_cast<size_t>(m) / (4096) + 64;  // k_scan block totals
    const size_t bytes = (static_cast<size_t>(n) + 2 * static_cast<size_t>(m) + bsums) * sizeof(int);
    MDB_TRY(ctx_scratch(ctx, bytes, &p));
    *atom_rank = static_cast<int*>(p);
    *counts = *atom_rank + n;
    *fill = *counts + m;
    return MD_OK;
}

// Counting sort (see cell_sort), optionally gated by a device flag.
int cell_sort_gated(md_system* sys, const CellGrid& grid, int* d_sorted, int* d_start,
                    const int* flag) {
    md_context* ctx = sys->ctx;
    const int64_t n = sys->n;
    const int m = grid.ncells;
    int *atom_rank, *counts, *fill;
    MDB_TRY(sort_scratch(ctx, n, m, &atom_rank, &counts, &fill));
    const GridArgs g = make_args(grid, sys);
    const int zb = std::min<int64_t>(grid_for(2 * static_cast<int64_t>(m), kBlock), 4096);
    k_zero_int<<<zb, kBlock, 0, ctx->stream>>>(counts, 2 * static_cast<int64_t>(m), flag);
    if (n > 0)
        k_bin<<<grid_for(n, kBlock), kBlock, 0, ctx->stream>>>(sys->cur.pos, n, g, atom_rank,
                                                               counts, flag);
    const int nb = (m + kScanBlock * kScanItems - 1) / (kScanBlock * kScanItems);
    int* bsum = fill + m;  // scratch tail (sort_scratch reserves it)
    k_scan_blocks<<<nb, kScanBlock, 0, ctx->stream>>>(counts, d_start, m, bsum, flag, nb == 1 ? 1 : 0);
    if (nb > 1) {
        k_scan_top<<<1, kScanBlock, 0, ctx->stream>>>(bsum, nb, d_start, m, flag);
        k_scan_add<<<nb, kScanBlock, 0, ctx->stream>>>(d_start, m, bsum, flag);
        ctx->launches += 2;
    }
    if (n > 0)
        k_scatter<<<grid_for(n, kBlock), kBlock, 0, ctx->stream>>>(atom_rank, n, d_start, fill,
                                                                   d_sorted, flag);
    k_cell_order<<<grid_for(32 * static_cast<int64_t>(m), 256), 256, 0, ctx->stream>>>(
        d_sorted, d_start, m, sys->cur.orig, flag);
    ctx->launches += 3 + (n > 0 ? 2 : 0);
    MDB_CHECK_LAUNCH();
    return MD_OK;
}


// ------------------------------------------------------------ batched rebuilds
// The gated rebuild of many replicas, one launch per stage (the counting sort, the
// re-sort of the system with the reference positions and, for a mixed force, the
// fixed-point copy, the list build).  Each block serves the replica the stage's
// block table assigns it and leaves at once when that replica's rebuild
// flag is clear; a replica's blocks are those of its solo gated rebuild.
struct RebuildRep {
    const int* flag;
    int64_t n;
    int m;       // cells (0 for a brute-force build)
    int groups;  // warps per cell in the list build
    GridArgs g;
    md_atoms cur, alt;
    int* slot;
    int *atom_rank, *counts, *fill;
    int* start;
    int* perm;
    double rl2;
    int* nbr;
    int* count;
    int stride;
    uint32_t* status;
    int* max_count;
    double4* ref;
    int* total;
    int4* q;      // the fixed-point copy for a mixed force, or null
    double qs[3];  // 2^32 / L per axis
};

enum RebuildStage : int {
    kStZero, kStBin, kStScan, kStScatter, kStOrder, kStPermute, kStCopy, kStCells, kStBrute,
    kRebuildStages
};

// The stages on 256-thread blocks.
template <int STAGE>
__global__ void __launch_bounds__(kBlock)
k_batch_rebuild(const RebuildRep* __restrict__ reps, const int4* __restrict__ blk) {
    const int4 e = __ldg(blk + blockIdx.x);
    const RebuildRep& d = reps[e.x];
    if (!gate(d.flag)) return;
    const unsigned b = e.y, nb = e.z;
    if constexpr (STAGE == kStBin) {
        bin_body(d.cur.pos, d.n, d.g, d.atom_rank, d.counts, b);
    } else if constexpr (STAGE == kStScatter) {
        scatter_body(d.atom_rank, d.n, d.start, d.fill, d.perm, b);
    } else if constexpr (STAGE == kStOrder) {
        cell_order_body(d.perm, d.start, d.m, d.cur.orig, b);
        // the counts are used up: cleared here for the next rebuild, and the row
        // maximum for this one's build
        zero_int_body(d.counts, 2 * static_cast<int64_t>(d.m), b, nb);
        if (b == 0 && threadIdx.x == 0) *d.max_count = 0;
    } else if constexpr (STAGE == kStPermute) {
        permute_body(d.cur, d.alt, d.perm, d.slot, d.n, 0, b);
    } else if constexpr (STAGE == kStCopy) {
        // the copy back also writes what the solo rebuild writes from the same
        // positions after the list build: the reference positions of the rebuild
        // test and the fixed-point copy
        copy_atoms_body(d.alt, d.cur, d.n, 0, b);
        const int64_t k = b * static_cast<int64_t>(blockDim.x) + threadIdx.x;
        if (k < d.n) {
            const double4 p = d.alt.pos[k];
            d.ref[k] = p;
            if (d.q) d.q[k] = quantize_position(p, d.qs[0], d.qs[1], d.qs[2]);
        }
        if (k == 0) ++*d.total;
    } else if constexpr (STAGE == kStBrute) {  // no re-sort: one warp per atom
        brute_body(d.cur.pos, d.n, d.g.box, d.rl2, d.nbr, d.count, d.stride, d.status, d.max_count, b);
        const int64_t i = (b * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5;
        if ((threadIdx.x & 31) == 0 && i < d.n) {  // the reference and fixed-point copies
            const double4 p = d.cur.pos[i];
            d.ref[i] = p;
            if (d.q) d.q[i] = quantize_position(p, d.qs[0], d.qs[1], d.qs[2]);
        }
        if (b == 0 && threadIdx.x == 0) ++*d.total;
    }
}

// Once per run, before the first replay: every replica's cell counts cleared (a
// rebuild launched from the host leaves them set; the replays clear them as they
// use them).
__global__ void __launch_bounds__(kBlock)
k_batch_rebuild_prime(const RebuildRep* __restrict__ reps, const int4* __restrict__ blk) {
    const int4 e = __ldg(blk + blockIdx.x);
    const RebuildRep& d = reps[e.x];
    zero_int_body(d.counts, 2 * static_cast<int64_t>(d.m), e.y, e.z);
}

// The cell-count scan, one 1024-thread block per replica over its whole grid:
// chunks of kScanBlock * kScanItems counts scanned in turn with a running carry
// (the same exclusive sums as the solo multi-block scan).
__global__ void __launch_bounds__(kScanBlock)
k_batch_rebuild_scan(const RebuildRep* __restrict__ reps, const int4* __restrict__ blk) {
    const RebuildRep& d = reps[__ldg(blk + blockIdx.x).x];
    if (!gate(d.flag)) return;
    int carry = 0;
    for (int base = 0; base < d.m; base += kScanBlock * kScanItems) {
        int v[kScanItems];
#pragma unroll
        for (int u = 0; u < kScanItems; ++u) {
            const int i = base + u * kScanBlock + threadIdx.x;  // coalesced
            v[u] = i < d.m ? d.counts[i] : 0;
        }
#pragma unroll
        for (int u = 0; u < kScanItems; ++u) {
            int tot;
            const int ex = block_exclusive_scan(v[u], &tot);
            const int i = base + u * kScanBlock + threadIdx.x;
            if (i < d.m) d.start[i] = carry + ex;
            carry += tot;
        }
    }
    if (threadIdx.x == 0) d.start[d.m] = carry;
}

// The list build, on the build's own 128-thread blocks.  (Blocks that each take two
// or four of the solo build's blocks in turn, so that a step in which few replicas
// rebuild places fewer blocks, measured slower: the rebuilding replicas' builds
// lose more parallelism than the skipped blocks cost.)
__global__ void __launch_bounds__(kBuildWarps * 32)
k_batch_rebuild_cells(const RebuildRep* __restrict__ reps, const int4* __restrict__ blk) {
    const int4 e = __ldg(blk + blockIdx.x);
    const RebuildRep& d = reps[e.x];
    if (!gate(d.flag)) return;
    verlet_cells_body(d.cur.pos, d.start, d.g, d.rl2, d.nbr, d.count, d.stride, d.status,
                      d.max_count, d.groups, e.y);
}

}  // namespace

// ------------------------------------------------------------------ CellGrid
int CellGrid::init(const double box[3], double cut) {
    release();
    cutoff = cut;
    // cell_list.cpp:8-14: n = max(1, floor(L / cutoff)), width = L / n.
    int dims[3];
    for (int d = 0; d < 3; ++d) {
        const double f = std::floor(box[d] / cut);
        dims[d] = f < 1.0 ? 1 : (f > 1024.0 ? 1024 : static_cast<int>(f));
        width[d] = box[d] / static_cast<double>(dims[d]);
    }
    nx = dims[0];
    ny = dims[1];
    nz = dims[2];
    ncells = nx * ny * nz;
    usable = nx >= 3 && ny >= 3 && nz >= 3;  // cell_list.cpp:51-53
    // Morton rank of every cell, so sorted atoms of nearby cells sit nearby in HBM.
    std::vector<std::pair<uint32_t, int>> keyed(static_cast<size_t>(ncells));
    for (int c = 0; c < ncells; ++c) {
        const uint32_t ix = c % nx, iy = (c / nx) % ny, iz = c / (nx * ny);
        keyed[c] = {spread3(ix) | (spread3(iy) << 1) | (spread3(iz) << 2), c};
    }
    std::sort(keyed.begin(), keyed.end());
    std::vector<int> rank(static_cast<size_t>(ncells)), cell(static_cast<size_t>(ncells));
    for (int r = 0; r < ncells; ++r) {
        cell[r] = keyed[r].second;
        rank[keyed[r].second] = r;
    }
    MDB_CUDA(cudaMalloc(&rank_of_cell, sizeof(int) * ncells));
    MDB_CUDA(cudaMalloc(&cell_of_rank, sizeof(int) * ncells));
    MDB_CUDA(cudaMemcpy(rank_of_cell, rank.data(), sizeof(int) * ncells, cudaMemcpyHostToDevice));
    MDB_CUDA(cudaMemcpy(cell_of_rank, cell.data(), sizeof(int) * ncells, cudaMemcpyHostToDevice));
    return MD_OK;
}

void CellGrid::release() {
    if (rank_of_cell) cudaFree(rank_of_cell);
    if (cell_of_rank) cudaFree(cell_of_rank);
    rank_of_cell = cell_of_rank = nullptr;
}

int cell_sort(md_system* sys, const CellGrid& grid, int* d_sorted, int* d_start) {
    return cell_sort_gated(sys, grid, d_sorted, d_start, nullptr);
}

// ---------------------------------------------------------------- Verlet
static int verlet_alloc(md_verlet* v, md_system* sys) {
    const int64_t n = sys->n;
    if (v->n != n || !v->count.ptr) {
        MDB_TRY(v->count.ensure(sizeof(int) * static_cast<size_t>(n > 0 ? n : 1)));
        MDB_TRY(v->ref.ensure(sizeof(double4) * static_cast<size_t>(n > 0 ? n : 1)));
        MDB_TRY(v->perm.ensure(sizeof(int) * static_cast<size_t>(n > 0 ? n : 1)));
        v->n = n;
    }
    if (v->stride == 0) {
        // Expected full-list neighbours at this density, doubled, plus slack.
        const double vol = sys->box[0] * sys->box[1] * sys->box[2];
        const double rl = v->cutoff + v->skin;
        const double expect = (n / vol) * 4.18879020478639 * rl * rl * rl;
        int s = static_cast<int>(2.0 * expect) + 48;
        s = std::min<int64_t>(s, std::max<int64_t>(n, 1));
        v->stride = (s + 7) & ~7;
    }
    MDB_TRY(v->nbr.ensure(sizeof(int) * static_cast<size_t>(n > 0 ? n : 1) * v->stride));
    return MD_OK;
}

// Halo tile buffers for the current size and row capacity.
int halo_alloc(md_verlet* v, int64_t n) {
    const int64_t tiles = halo_blocks(n);
    MDB_TRY(v->halo_runs.ensure(sizeof(int2) * static_cast<size_t>(tiles) * kHaloRuns));
    MDB_TRY(v->halo_meta.ensure(sizeof(int2) * static_cast<size_t>(tiles)));
    MDB_TRY(v->nbr16.ensure(sizeof(uint16_t) * static_cast<size_t>(n) * v->stride));
    return MD_OK;
}

void halo_plan(md_verlet* v, md_system* sys, const int* flag) {
    const int64_t n = sys->n, tiles = halo_blocks(n);
    k_halo_plan<<<static_cast<unsigned>((tiles + kPlanWarps - 1) / kPlanWarps), 32 * kPlanWarps, 0,
                  sys->ctx->stream>>>(v->start.as<int>(), make_args(v->grid, sys), n, tiles,
                                      v->halo_runs.as<int2>(), v->halo_meta.as<int2>(), flag);
    ++sys->ctx->launches;
}

// Halo tiles of the current list: plan, then convert its rows (gated by the
// rebuild flag inside fused loops).
int halo_build(md_verlet* v, md_system* sys, const int* flag) {
    md_context* ctx = sys->ctx;
    const int64_t n = sys->n;
    if (v->stride % 8 != 0) {  // rows are converted and read 16 bytes at a time
        v->halo_on = false;
        return MD_OK;
    }
    MDB_TRY(halo_alloc(v, n));
    halo_plan(v, sys, flag);
    k_halo_rows<<<static_cast<unsigned>(halo_blocks(n)), kRowsThreads, 0, ctx->stream>>>(
        v->nbr.as<int>(), v->count.as<int>(), v->stride, n, v->halo_runs.as<int2>(),
        v->halo_meta.as<int2>(), v->nbr16.as<uint16_t>(), flag);
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

int verlet_build_impl(md_verlet* v, md_system* sys, const int* flag, int4* q = nullptr,
                      bool* quantized = nullptr) {
    if (quantized) *quantized = false;
    md_context* ctx = sys->ctx;
    const int64_t n = sys->n;
    const Box3 box = make_box(sys);
    const double rl2 = (v->cutoff + v->skin) * (v->cutoff + v->skin);  // verlet_list.cpp:11
    MDB_CUDA(cudaMemsetAsync(v->d_max_count, 0, sizeof(int), ctx->stream));
    if (v->grid.usable) {
        int* start = v->start.as<int>();
        MDB_TRY(cell_sort_gated(sys, v->grid, v->perm.as<int>(), start, flag));
        // Re-sort the system into cell order: permute into alt, copy back, so the
        // device pointers of the current arrays never change.
        if (n > 0) {
            const int with_forces = flag ? 0 : 1;  // fused loops recompute forces next
            k_permute_gated<<<grid_for(n, kBlock), kBlock, 0, ctx->stream>>>(
                sys->cur, sys->alt, v->perm.as<int>(), sys->slot, n, flag, with_forces);
            k_copy_atoms<<<grid_for(n, kBlock), kBlock, 0, ctx->stream>>>(
                sys->alt, sys->cur, n, flag, with_forces, v->ref.as<double4>(),
                flag ? v->d_rebuild_total : nullptr, q, 4294967296.0 / sys->box[0],
                4294967296.0 / sys->box[1], 4294967296.0 / sys->box[2]);
            ctx->launches += 2;
            if (quantized) *quantized = q != nullptr;
        }
        const GridArgs g = make_args(v->grid, sys);
        // warps per cell from the mean occupancy (crowded cells, e.g. a long cutoff)
        const double mean = static_cast<double>(n) / v->grid.ncells;
        const int groups = static_cast<int>(std::min(16.0, std::max(1.0, std::ceil(1.5 * mean / 32.0))));
        const int64_t warps = static_cast<int64_t>(v->grid.ncells) * groups;
        k_verlet_cells<<<grid_for(warps, kBuildWarps), kBuildWarps * 32, 0, ctx->stream>>>(
            sys->cur.pos, start, g, rl2, v->nbr.as<int>(), v->count.as<int>(), v->stride,
            ctx->d_status, v->d_max_count, flag, groups);
        ++ctx->launches;
        if (v->halo_on && n > 0) MDB_TRY(halo_build(v, sys, flag));
    } else if (n > 0) {
        k_verlet_brute<<<grid_for(n * 32, kBlock), kBlock, 0, ctx->stream>>>(
            sys->cur.pos, n, box, rl2, v->nbr.as<int>(), v->count.as<int>(), v->stride,
            ctx->d_status, v->d_max_count, flag);
        ++ctx->launches;
        // no re-sort: the reference positions straight from the system
        k_store_ref<<<grid_for(n, kBlock), kBlock, 0, ctx->stream>>>(
            sys->cur.pos, v->ref.as<double4>(), n, flag, flag ? v->d_rebuild_total : nullptr);
        ++ctx->launches;
    }
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

int verlet_build(md_verlet* v, md_system* sys, bool conditional) {
    MDB_TRY(verlet_alloc(v, sys));
    if (!conditional) {
        // Host-driven build: retry with a larger stride until no row overflows.
        for (int attempt = 0; attempt < 8; ++attempt) {
            ctx_time_begin(sys->ctx, MD_KERNEL_NEIGHBOR);
            const int rc = verlet_build_impl(v, sys, nullptr);
            ctx_time_end(sys->ctx, MD_KERNEL_NEIGHBOR);
            MDB_TRY(rc);
            int mx = 0;
            MDB_CUDA(cudaMemcpyAsync(&mx, v->d_max_count, sizeof(int), cudaMemcpyDeviceToHost,
                                     sys->ctx->stream));
            MDB_CUDA(cudaStreamSynchronize(sys->ctx->stream));
            if (mx <= v->stride) break;
            uint32_t st = 0;
            md_context_status(sys->ctx, &st, 1);  // clear the overflow bit we resolve here
            if (v->stride_fixed) {
                v->sys = nullptr;
                return fail(MD_ERR_RUNTIME,
                            "VerletList: an atom has %d neighbours within the list cutoff, more "
                            "than the fixed row capacity %d", mx, v->stride);
            }
            v->stride = ((mx + mx / 4 + 16) + 7) & ~7;
            graph_epoch_bump();  // the stride is a captured launch argument
            MDB_TRY(v->nbr.ensure(sizeof(int) * static_cast<size_t>(sys->n) * v->stride));
            // positions are already sorted; the re-sort below is a no-op permutation
        }
        ++v->rebuilds;
        v->epoch = sys->epoch;
        v->sys = sys;
        graph_epoch_bump();
        return MD_OK;
    }
    return verlet_build_impl(v, sys, v->d_rebuild_flag);
}

// The gated (conditional) build of a fused step for a mixed force: the rebuild also
// writes the fixed-point copy q when it re-sorts the system (*quantized then true).
int verlet_build_q(md_verlet* v, md_system* sys, int4* q, bool* quantized) {
    MDB_TRY(verlet_alloc(v, sys));
    return verlet_build_impl(v, sys, v->d_rebuild_flag, q, quantized);
}

bool verlet_halo_ready(md_verlet* v, md_system* sys) {
    if (v->stride % 8 != 0) return false;  // the force kernel reads rows 16 bytes at a time
    if (v->halo_on) return true;
    if (!v->grid.usable || sys->n <= 0 || v->sys != sys) return false;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(sys->ctx->stream, &cs) != cudaSuccess ||
        cs != cudaStreamCaptureStatusNone)
        return false;
    if (halo_build(v, sys, nullptr) != MD_OK) {
        cudaGetLastError();
        return false;
    }
    v->halo_on = true;
    graph_epoch_bump();
    return true;
}

void verlet_halo_for_run(md_verlet* v, md_system* sys, const md_lj* lj) {
    if (lj->precision == MD_PRECISION_MIXED && lj->halo && sys->n >= kHaloMinAtoms)
        verlet_halo_ready(v, sys);
}

DispArgs disp_args(md_verlet* v, md_context* ctx, double* part) {
    DispArgs d;
    d.ref = v->ref.as<double4>();
    d.skin = v->skin;
    d.criterion = v->criterion;
    d.part = part;
    d.ticket = ctx_counter(ctx, 1);
    d.flag = v->d_rebuild_flag;
    d.top2 = ctx_result(ctx, kResTop2);
    return d;
}

int verlet_check(md_verlet* v, md_system* sys) {
    md_context* ctx = sys->ctx;
    const int64_t n = sys->n;
    const int g = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(grid_for(n, kBlock),
                                                                      ctx->sm_count * 8)));
    double* part;
    MDB_TRY(ctx_partials(ctx, 2 * static_cast<size_t>(g), &part));
    k_displacement<<<g, kBlock, 0, ctx->stream>>>(sys->cur.pos, n, make_box(sys),
                                                 disp_args(v, ctx, part));
    ++ctx->launches;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}


// ------------------------------------------------------------ batched rebuilds
struct BatchRebuild {
    DevBuf reps, blk;  // blk: the stages' block tables (block_table), one after another
    int nrep = 0;
    int blocks[kRebuildStages] = {};
    int base[kRebuildStages] = {};  // first entry of each stage's table in blk
};

int batch_rebuild_create(const BatchRepView* v, int nrep, BatchRebuild** out) {
    *out = nullptr;
    if (nrep < 1) return fail(MD_ERR_INVALID_ARGUMENT, "batch_rebuild_create: no replicas");
    std::vector<RebuildRep> h(static_cast<size_t>(nrep));
    std::vector<int> off(static_cast<size_t>(kRebuildStages) * (nrep + 1), 0);
    for (int r = 0; r < nrep; ++r) {
        md_system* sys = v[r].sys;
        md_verlet* lst = v[r].list;
        md_context* ctx = sys->ctx;
        const int64_t n = sys->n;
        const bool cells = lst->grid.usable;
        const int m = cells ? lst->grid.ncells : 0;
        if (lst->halo_on || n <= 0 || (cells && (!lst->start.ptr || !lst->perm.ptr || !sys->alt.pos)))
            return fail(MD_ERR_INVALID_ARGUMENT, "batch_rebuild_create: replica %d rebuilds alone", r);
        RebuildRep& d = h[static_cast<size_t>(r)];
        d.flag = lst->d_rebuild_flag;
        d.n = n;
        d.m = m;
        const double mean = cells ? static_cast<double>(n) / m : 0.0;  // as verlet_build_impl
        d.groups = static_cast<int>(std::min(16.0, std::max(1.0, std::ceil(1.5 * mean / 32.0))));
        d.g = make_args(lst->grid, sys);
        d.cur = sys->cur;
        d.alt = sys->alt;
        d.slot = sys->slot;
        d.atom_rank = d.counts = d.fill = nullptr;
        if (cells) MDB_TRY(sort_scratch(ctx, n, m, &d.atom_rank, &d.counts, &d.fill));
        d.start = lst->start.as<int>();
        d.perm = lst->perm.as<int>();
        d.rl2 = (lst->cutoff + lst->skin) * (lst->cutoff + lst->skin);  // verlet_list.cpp:11
        d.nbr = lst->nbr.as<int>();
        d.count = lst->count.as<int>();
        d.stride = lst->stride;
        d.status = ctx->d_status;
        d.max_count = lst->d_max_count;
        d.ref = lst->ref.as<double4>();
        d.total = lst->d_rebuild_total;
        d.q = nullptr;
        if (v[r].lj->precision == MD_PRECISION_MIXED) {
            MDB_TRY(sys->qpos.ensure(sizeof(int4) * static_cast<size_t>(n)));
            d.q = sys->qpos.as<int4>();
        }
        for (int k = 0; k < 3; ++k) d.qs[k] = 4294967296.0 / sys->box[k];
        // blocks of each stage: those of the solo gated rebuild
        const int nblk = grid_for(n, kBlock), c = cells ? 1 : 0;
        const int per[kRebuildStages] = {
            c * static_cast<int>(std::min<int64_t>(grid_for(2 * static_cast<int64_t>(m), kBlock), 4096)),
            c * nblk, c, c * nblk,
            cells ? grid_for(32 * static_cast<int64_t>(m), 256) : 1,  // + clearing the row maximum
            c * nblk, c * nblk, c * grid_for(static_cast<int64_t>(m) * d.groups, kBuildWarps),
            cells ? 0 : grid_for(n * 32, kBlock)};
        for (int st = 0; st < kRebuildStages; ++st) {
            int* o = off.data() + static_cast<size_t>(st) * (nrep + 1);
            o[r + 1] = o[r] + per[st];
        }
    }
    BatchRebuild* b = new (std::nothrow) BatchRebuild();
    if (!b) return fail(MD_ERR_OUT_OF_MEMORY, "batch_rebuild_create: host allocation");
    b->nrep = nrep;
    std::vector<int4> t;
    for (int st = 0; st < kRebuildStages; ++st) {
        const std::vector<int4> ts = block_table(off.data() + static_cast<size_t>(st) * (nrep + 1), nrep);
        b->blocks[st] = static_cast<int>(ts.size());
        b->base[st] = static_cast<int>(t.size());
        t.insert(t.end(), ts.begin(), ts.end());
    }
    int rc = b->reps.ensure(sizeof(RebuildRep) * h.size());
    if (rc == MD_OK) rc = b->blk.ensure(sizeof(int4) * std::max<size_t>(t.size(), 1));
    if (rc == MD_OK && (cudaMemcpy(b->reps.ptr, h.data(), sizeof(RebuildRep) * h.size(),
                                   cudaMemcpyHostToDevice) != cudaSuccess ||
                        cudaMemcpy(b->blk.ptr, t.data(), sizeof(int4) * t.size(),
                                   cudaMemcpyHostToDevice) != cudaSuccess))
        rc = fail(MD_ERR_CUDA, "batch_rebuild_create: upload");
    if (rc != MD_OK) {
        delete b;
        return rc;
    }
    *out = b;
    return MD_OK;
}

int batch_rebuild_launch(BatchRebuild* b, cudaStream_t stream, int64_t* launches) {
    const RebuildRep* reps = b->reps.as<RebuildRep>();
    auto table = [&](int st) { return b->blk.as<int4>() + b->base[st]; };
    int64_t l = 0;
    auto stage = [&](int st, auto kernel) {
        if (b->blocks[st] == 0) return;
        kernel<<<static_cast<unsigned>(b->blocks[st]), kBlock, 0, stream>>>(reps, table(st));
        ++l;
    };
    stage(kStBin, k_batch_rebuild<kStBin>);
    if (b->blocks[kStScan] > 0) {
        k_batch_rebuild_scan<<<static_cast<unsigned>(b->blocks[kStScan]), kScanBlock, 0, stream>>>(
            reps, table(kStScan));
        ++l;
    }
    stage(kStScatter, k_batch_rebuild<kStScatter>);
    stage(kStOrder, k_batch_rebuild<kStOrder>);
    stage(kStPermute, k_batch_rebuild<kStPermute>);
    stage(kStCopy, k_batch_rebuild<kStCopy>);
    if (b->blocks[kStCells] > 0) {
        k_batch_rebuild_cells<<<static_cast<unsigned>(b->blocks[kStCells]), kBuildWarps * 32, 0,
                                stream>>>(reps, table(kStCells));
        ++l;
    }
    stage(kStBrute, k_batch_rebuild<kStBrute>);
    if (launches) *launches += l;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

int batch_rebuild_prime(BatchRebuild* b, cudaStream_t stream, int64_t* launches) {
    if (b->blocks[kStZero] == 0) return MD_OK;
    k_batch_rebuild_prime<<<static_cast<unsigned>(b->blocks[kStZero]), kBlock, 0, stream>>>(
        b->reps.as<RebuildRep>(), b->blk.as<int4>() + b->base[kStZero]);
    if (launches) ++*launches;
    MDB_CHECK_LAUNCH();
    return MD_OK;
}

void batch_rebuild_destroy(BatchRebuild* b) { delete b; }

}  // namespace mdb

// --------------------------------------------------------------- pair export
namespace mdb {
namespace {

__global__ void k_to_orig(const int* __restrict__ sorted, const int* __restrict__ orig, int* out,
                          int64_t n) {
    const int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (s < n) out[s] = orig[sorted[s]];
}

// The exported pairs: rows entries (i, j) with orig(i) < orig(j) that pass the
// reference's exact test on the positions of the build (`ref`).
__global__ void k_verlet_pair_count(const int* __restrict__ nbr, const int* __restrict__ count,
                                    const double4* __restrict__ ref, int64_t n, int stride,
                                    Box3 box, double rl2, int* out) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const double4 pi = ref[i];
    int c = 0;
    const int cnt = min(count[i], stride);
    for (int k = 0; k < cnt; ++k) {
        const double4 pj = ref[nbr[i * stride + k]];
        if (pj.w > pi.w && within(box, pi, pj, rl2)) ++c;
    }
    out[i] = c;
}

__global__ void k_verlet_pair_write(const int* __restrict__ nbr, const int* __restrict__ count,
                                    const double4* __restrict__ ref, int64_t n, int stride,
                                    Box3 box, double rl2, const int64_t* __restrict__ offset,
                                    int64_t* pi, int64_t* pj) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const double4 p = ref[i];
    int64_t at = offset[i];
    const int cnt = min(count[i], stride);
    for (int k = 0; k < cnt; ++k) {
        const double4 q = ref[nbr[i * stride + k]];
        if (q.w > p.w && within(box, p, q, rl2)) {
            pi[at] = static_cast<int64_t>(p.w);
            pj[at] = static_cast<int64_t>(q.w);
            ++at;
        }
    }
}

// Candidate pairs of a CellList: for each atom (sorted position s) every atom of
// the 27 neighbouring cells with a larger original index.
__device__ __forceinline__ int cells_neighbor_rank(const GridArgs& g, int cell, int q) {
    const int cx = cell % g.nx, cy = (cell / g.nx) % g.ny, cz = cell / (g.nx * g.ny);
    int jx = cx + (q % 3) - 1, jy = cy + ((q / 3) % 3) - 1, jz = cz + (q / 9) - 1;
    jx = jx < 0 ? jx + g.nx : (jx >= g.nx ? jx - g.nx : jx);
    jy = jy < 0 ? jy + g.ny : (jy >= g.ny ? jy - g.ny : jy);
    jz = jz < 0 ? jz + g.nz : (jz >= g.nz ? jz - g.nz : jz);
    return g.rank_of_cell[jx + g.nx * (jy + g.ny * jz)];
}

__global__ void k_cell_pairs(const int* __restrict__ sorted_orig, const int* __restrict__ start,
                             GridArgs g, int64_t n, const int64_t* __restrict__ offset, int* counts,
                             int64_t* pi, int64_t* pj) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= g.ncells) return;
    const int cell = g.cell_of_rank[r];
    int64_t at = offset ? offset[r] : 0;
    int64_t c = 0;
    for (int s = start[r]; s < start[r + 1]; ++s) {
        const int oi = sorted_orig[s];
        for (int q = 0; q < 27; ++q) {
            const int rr = cells_neighbor_rank(g, cell, q);
            for (int t = start[rr]; t < start[rr + 1]; ++t) {
                const int oj = sorted_orig[t];
                if (oj > oi) {
                    if (pi) {
                        pi[at] = oi;
                        pj[at] = oj;
                        ++at;
                    }
                    ++c;
                }
            }
        }
    }
    if (counts) counts[r] = static_cast<int>(c);
}

int exclusive_offsets(const std::vector<int>& counts, std::vector<int64_t>& off) {
    off.resize(counts.size() + 1);
    int64_t acc = 0;
    for (size_t k = 0; k < counts.size(); ++k) {
        off[k] = acc;
        acc += counts[k];
    }
    off[counts.size()] = acc;
    return MD_OK;
}

}  // namespace
}  // namespace mdb

using namespace mdb;

namespace {

int check_box_match(const double a[3], const md_system* sys, const char* who) {
    for (int d = 0; d < 3; ++d)
        if (a[d] != sys->box[d])
            return fail(MD_ERR_INVALID_ARGUMENT, "%s: box differs from the system's box", who);
    return MD_OK;
}

int verlet_ready(md_verlet* v, md_system* sys, const char* who) {
    if (!v->sys) return fail(MD_ERR_INVALID_ARGUMENT, "%s: Verlet list was never built", who);
    if (v->sys != sys || v->n != sys->n)
        return fail(MD_ERR_INVALID_ARGUMENT, "%s: Verlet list was built for another system", who);
    if (v->epoch != sys->epoch)
        return fail(MD_ERR_INVALID_ARGUMENT, "%s: system was re-sorted since this list was built",
                    who);
    return MD_OK;
}

}  // namespace

namespace mdb {
int verlet_ensure_ready(md_verlet* v, md_system* sys, const char* who) {
    return verlet_ready(v, sys, who);
}
}  // namespace mdb

extern "C" {

// ------------------------------------------------------------------ CellList
int md_cells_create(md_context* ctx, const double box[3], double cutoff, md_cells** out) {
    graph_epoch_bump();
    if (!ctx || !box || !out) return fail(MD_ERR_INVALID_ARGUMENT, "md_cells_create: NULL argument");
    if (!(cutoff > 0.0)) return fail(MD_ERR_INVALID_ARGUMENT, "md_cells_create: cutoff must be > 0");
    md_cells* c = new (std::nothrow) md_cells();
    if (!c) return fail(MD_ERR_OUT_OF_MEMORY, "md_cells_create: host allocation");
    c->ctx = ctx;
    for (int d = 0; d < 3; ++d) c->box[d] = box[d];
    const int rc = c->grid.init(box, cutoff);
    if (rc != MD_OK) {
        delete c;
        return rc;
    }
    *out = c;
    return MD_OK;
}

int md_cells_destroy(md_cells* c) {
    graph_epoch_bump();
    if (!c) return MD_OK;
    c->grid.release();
    c->sorted_orig.release();
    c->start.release();
    delete c;
    return MD_OK;
}

int md_cells_dims(const md_cells* c, int dims[3]) {
    if (!c || !dims) return fail(MD_ERR_INVALID_ARGUMENT, "md_cells_dims: NULL argument");
    dims[0] = c->grid.nx;
    dims[1] = c->grid.ny;
    dims[2] = c->grid.nz;
    return MD_OK;
}

int md_cells_usable(const md_cells* c) { return c && c->grid.usable ? 1 : 0; }


int md_cells_build(md_cells* c, md_system* sys) {
    if (!c || !sys) return fail(MD_ERR_INVALID_ARGUMENT, "md_cells_build: NULL argument");
    MDB_TRY(check_box_match(c->box, sys, "md_cells_build"));
    md_context* ctx = sys->ctx;
    const int64_t n = sys->n;
    MDB_TRY(c->sorted_orig.ensure(sizeof(int) * static_cast<size_t>(2 * (n > 0 ? n : 1))));
    MDB_TRY(c->start.ensure(sizeof(int) * static_cast<size_t>(c->grid.ncells + 1)));
    int* sorted = c->sorted_orig.as<int>() + (n > 0 ? n : 1);  // second half: device slots
    MDB_TRY(cell_sort(sys, c->grid, sorted, c->start.as<int>()));
    if (n > 0) {
        k_to_orig<<<grid_for(n, kBlock), kBlock, 0, ctx->stream>>>(sorted, sys->cur.orig,
                                                                   c->sorted_orig.as<int>(), n);
        ++ctx->launches;
        MDB_CHECK_LAUNCH();
    }
    c->sys = sys;
    c->n = n;
    c->built = true;
    return MD_OK;
}

// ---------------------------------------------------------------- VerletList
int md_verlet_create(md_context* ctx, const double box[3], double cutoff, double skin,
                     md_verlet** out) {
    graph_epoch_bump();
    if (!ctx || !box || !out) return fail(MD_ERR_INVALID_ARGUMENT, "md_verlet_create: NULL argument");
    if (!(cutoff > 0.0) || !(skin >= 0.0))
        return fail(MD_ERR_INVALID_ARGUMENT, "md_verlet_create: cutoff must be > 0 and skin >= 0");
    md_verlet* v = new (std::nothrow) md_verlet();
    if (!v) return fail(MD_ERR_OUT_OF_MEMORY, "md_verlet_create: host allocation");
    v->ctx = ctx;
    for (int d = 0; d < 3; ++d) v->box[d] = box[d];
    v->cutoff = cutoff;
    v->skin = skin;
    int rc = v->grid.init(box, cutoff + skin);  // verlet_list.cpp:6: CellList at rc+skin
    if (rc == MD_OK) rc = v->start.ensure(sizeof(int) * static_cast<size_t>(v->grid.ncells + 1));
    if (rc == MD_OK) {
        int* flags = nullptr;
        if (cudaMalloc(&flags, 4 * sizeof(int)) != cudaSuccess ||
            cudaMemset(flags, 0, 4 * sizeof(int)) != cudaSuccess) {
            rc = fail(MD_ERR_OUT_OF_MEMORY, "md_verlet_create: device flags");
        } else {
            v->d_rebuild_flag = flags;
            v->d_rebuild_total = flags + 1;
            v->d_max_count = flags + 2;
        }
    }
    if (rc != MD_OK) {
        md_verlet_destroy(v);
        return rc;
    }
    *out = v;
    return MD_OK;
}

int md_verlet_destroy(md_verlet* v) {
    graph_epoch_bump();
    if (!v) return MD_OK;
    if (v->ctx) cudaStreamSynchronize(v->ctx->stream);
    v->grid.release();
    v->start.release();
    v->perm.release();
    v->nbr.release();
    v->count.release();
    v->ref.release();
    v->halo_runs.release();
    v->halo_meta.release();
    v->nbr16.release();
    if (v->d_rebuild_flag) cudaFree(v->d_rebuild_flag);
    delete v;
    return MD_OK;
}

int md_verlet_build(md_verlet* v, md_system* sys) {
    if (!v || !sys) return fail(MD_ERR_INVALID_ARGUMENT, "md_verlet_build: NULL argument");
    MDB_TRY(check_box_match(v->box, sys, "md_verlet_build"));
    return verlet_build(v, sys, false);
}

int md_verlet_needs_rebuild(md_verlet* v, md_system* sys, int* flag) {
    if (!v || !sys || !flag) return fail(MD_ERR_INVALID_ARGUMENT, "md_verlet_needs_rebuild: NULL");
    MDB_TRY(verlet_ready(v, sys, "md_verlet_needs_rebuild"));
    MDB_TRY(verlet_check(v, sys));
    int f = 0;
    MDB_CUDA(cudaMemcpyAsync(&f, v->d_rebuild_flag, sizeof(int), cudaMemcpyDeviceToHost,
                             sys->ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(sys->ctx->stream));
    *flag = f;
    return MD_OK;
}

int md_verlet_rebuild_if_needed(md_verlet* v, md_system* sys, int* rebuilt) {
    int f = 0;
    MDB_TRY(md_verlet_needs_rebuild(v, sys, &f));
    if (f) MDB_TRY(verlet_build(v, sys, false));
    if (rebuilt) *rebuilt = f;
    return MD_OK;
}

int md_verlet_rebuild_count(md_verlet* v, int64_t* count) {
    if (!v || !count) return fail(MD_ERR_INVALID_ARGUMENT, "md_verlet_rebuild_count: NULL");
    int dev = 0;
    MDB_CUDA(cudaMemcpyAsync(&dev, v->d_rebuild_total, sizeof(int), cudaMemcpyDeviceToHost,
                             v->ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(v->ctx->stream));
    *count = v->rebuilds + dev;
    return MD_OK;
}

int md_verlet_set_capacity(md_verlet* v, int capacity, int fixed) {
    graph_epoch_bump();
    if (!v || capacity < 1) return fail(MD_ERR_INVALID_ARGUMENT, "md_verlet_set_capacity: bad argument");
    if (v->ctx) MDB_CUDA(cudaStreamSynchronize(v->ctx->stream));
    v->stride = capacity;
    v->stride_fixed = fixed != 0;
    v->sys = nullptr;  // rows of the old capacity are no longer readable
    v->halo_on = false;
    return MD_OK;
}

int md_verlet_set_halo(md_verlet* v, int on) {
    graph_epoch_bump();
    if (!v) return fail(MD_ERR_INVALID_ARGUMENT, "md_verlet_set_halo: NULL");
    if (!on) {
        v->halo_on = false;
        return MD_OK;
    }
    if (!v->sys) return fail(MD_ERR_INVALID_ARGUMENT, "md_verlet_set_halo: list was never built");
    MDB_TRY(verlet_ready(v, v->sys, "md_verlet_set_halo"));
    verlet_halo_ready(v, v->sys);  // a list without a cell grid keeps gathering
    return ctx_check_status(v->ctx);
}

int md_verlet_halo_tiles(md_verlet* v, int64_t* staged, int64_t* tiles) {
    if (!v || !staged || !tiles) return fail(MD_ERR_INVALID_ARGUMENT, "md_verlet_halo_tiles: NULL");
    *staged = *tiles = 0;
    if (!v->halo_on || v->n <= 0) return MD_OK;
    const int64_t blocks = halo_blocks(v->n);
    std::vector<int2> meta(static_cast<size_t>(blocks));
    MDB_CUDA(cudaStreamSynchronize(v->ctx->stream));
    MDB_CUDA(cudaMemcpy(meta.data(), v->halo_meta.ptr, sizeof(int2) * meta.size(),
                        cudaMemcpyDeviceToHost));
    for (const int2& m : meta) *staged += m.x > 0 ? 1 : 0;
    *tiles = blocks;
    return MD_OK;
}

int md_verlet_set_criterion(md_verlet* v, int criterion) {
    graph_epoch_bump();
    if (!v || (criterion != 0 && criterion != 1))
        return fail(MD_ERR_INVALID_ARGUMENT, "md_verlet_set_criterion: criterion must be 0 or 1");
    v->criterion = criterion;
    return MD_OK;
}

int md_verlet_set_cell_width(md_verlet* v, double width) {
    graph_epoch_bump();
    if (!v) return fail(MD_ERR_INVALID_ARGUMENT, "md_verlet_set_cell_width: NULL list");
    const double rl = v->cutoff + v->skin;
    if (!(width == 0.0 || width >= rl))
        return fail(MD_ERR_INVALID_ARGUMENT,
                    "md_verlet_set_cell_width: width %g is below the list cutoff %g (0 restores "
                    "the reference's rule)", width, rl);
    if (v->ctx) cudaStreamSynchronize(v->ctx->stream);
    MDB_TRY(v->grid.init(v->box, width == 0.0 ? rl : width));
    MDB_TRY(v->start.ensure(sizeof(int) * static_cast<size_t>(v->grid.ncells + 1)));
    v->cell_width = width;
    v->sys = nullptr;  // the list must be built again on the new grid
    return MD_OK;
}

int md_verlet_cells_per_side(const md_verlet* v, int dims[3]) {
    if (!v || !dims) return fail(MD_ERR_INVALID_ARGUMENT, "md_verlet_cells_per_side: NULL");
    dims[0] = v->grid.nx;
    dims[1] = v->grid.ny;
    dims[2] = v->grid.nz;
    return MD_OK;
}

int md_verlet_displacements(md_verlet* v, md_system* sys, double* largest, double* second) {
    if (!v || !sys) return fail(MD_ERR_INVALID_ARGUMENT, "md_verlet_displacements: NULL");
    MDB_TRY(verlet_ready(v, sys, "md_verlet_displacements"));
    MDB_TRY(verlet_check(v, sys));
    double r[2];
    MDB_TRY(ctx_read_results(sys->ctx, kResTop2, 2, r));
    if (largest) *largest = r[0];
    if (second) *second = r[1];
    return MD_OK;
}

}  // extern "C"


extern "C" {

int md_verlet_pairs(md_verlet* v, int64_t* pi, int64_t* pj, int64_t cap, int64_t* count) {
    if (!v || !count) return fail(MD_ERR_INVALID_ARGUMENT, "md_verlet_pairs: NULL argument");
    md_system* sys = v->sys;
    if (!sys) return fail(MD_ERR_INVALID_ARGUMENT, "md_verlet_pairs: list was never built");
    MDB_TRY(verlet_ready(v, sys, "md_verlet_pairs"));
    md_context* ctx = v->ctx;
    const int64_t n = sys->n;
    if (n == 0) {
        *count = 0;
        return MD_OK;
    }
    DevBuf cnt;
    MDB_TRY(cnt.ensure(sizeof(int) * n));
    const Box3 box = make_box(sys);
    const double rl2 = (v->cutoff + v->skin) * (v->cutoff + v->skin);  // verlet_list.cpp:11
    k_verlet_pair_count<<<grid_for(n, kBlock), kBlock, 0, ctx->stream>>>(
        v->nbr.as<int>(), v->count.as<int>(), v->ref.as<double4>(), n, v->stride, box, rl2,
        cnt.as<int>());
    ++ctx->launches;
    std::vector<int> hc(static_cast<size_t>(n));
    MDB_CUDA(cudaMemcpyAsync(hc.data(), cnt.ptr, sizeof(int) * n, cudaMemcpyDeviceToHost, ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    std::vector<int64_t> off;
    exclusive_offsets(hc, off);
    const int64_t total = off[n];
    *count = total;
    if (pi && pj && cap >= total && total > 0) {
        DevBuf doff, dpi, dpj;
        MDB_TRY(doff.ensure(sizeof(int64_t) * (n + 1)));
        MDB_TRY(dpi.ensure(sizeof(int64_t) * total));
        MDB_TRY(dpj.ensure(sizeof(int64_t) * total));
        MDB_CUDA(cudaMemcpyAsync(doff.ptr, off.data(), sizeof(int64_t) * (n + 1),
                                 cudaMemcpyHostToDevice, ctx->stream));
        k_verlet_pair_write<<<grid_for(n, kBlock), kBlock, 0, ctx->stream>>>(
            v->nbr.as<int>(), v->count.as<int>(), v->ref.as<double4>(), n, v->stride, box, rl2,
            doff.as<int64_t>(), dpi.as<int64_t>(), dpj.as<int64_t>());
        ++ctx->launches;
        MDB_CUDA(cudaMemcpyAsync(pi, dpi.ptr, sizeof(int64_t) * total, cudaMemcpyDeviceToHost, ctx->stream));
        MDB_CUDA(cudaMemcpyAsync(pj, dpj.ptr, sizeof(int64_t) * total, cudaMemcpyDeviceToHost, ctx->stream));
        MDB_CUDA(cudaStreamSynchronize(ctx->stream));
        doff.release();
        dpi.release();
        dpj.release();
        // sort by (i, j) on the host for a canonical export order
        std::vector<std::pair<int64_t, int64_t>> pr(static_cast<size_t>(total));
        for (int64_t k = 0; k < total; ++k) pr[k] = {pi[k], pj[k]};
        std::sort(pr.begin(), pr.end());
        for (int64_t k = 0; k < total; ++k) {
            pi[k] = pr[k].first;
            pj[k] = pr[k].second;
        }
    }
    cnt.release();
    return ctx_check_status(ctx);
}

int md_cells_pairs(md_cells* c, int64_t* pi, int64_t* pj, int64_t cap, int64_t* count) {
    if (!c || !count) return fail(MD_ERR_INVALID_ARGUMENT, "md_cells_pairs: NULL argument");
    if (!c->built) return fail(MD_ERR_INVALID_ARGUMENT, "md_cells_pairs: cell list was never built");
    if (!c->grid.usable)
        return fail(MD_ERR_INVALID_ARGUMENT,
                    "md_cells_pairs: CellList is not usable (fewer than 3 cells per side)");
    md_context* ctx = c->ctx;
    const int m = c->grid.ncells;
    GridArgs g = make_args(c->grid, c->sys);
    DevBuf cnt;
    MDB_TRY(cnt.ensure(sizeof(int) * m));
    k_cell_pairs<<<grid_for(m, 64), 64, 0, ctx->stream>>>(c->sorted_orig.as<int>(),
                                                         c->start.as<int>(), g, c->n, nullptr,
                                                         cnt.as<int>(), nullptr, nullptr);
    ++ctx->launches;
    std::vector<int> hc(static_cast<size_t>(m));
    MDB_CUDA(cudaMemcpyAsync(hc.data(), cnt.ptr, sizeof(int) * m, cudaMemcpyDeviceToHost, ctx->stream));
    MDB_CUDA(cudaStreamSynchronize(ctx->stream));
    std::vector<int64_t> off;
    exclusive_offsets(hc, off);
    const int64_t total = off[m];
    *count = total;
    if (pi && pj && cap >= total && total > 0) {
        DevBuf doff, dpi, dpj;
        MDB_TRY(doff.ensure(sizeof(int64_t) * (m + 1)));
        MDB_TRY(dpi.ensure(sizeof(int64_t) * total));
        MDB_TRY(dpj.ensure(sizeof(int64_t) * total));
        MDB_CUDA(cudaMemcpyAsync(doff.ptr, off.data(), sizeof(int64_t) * (m + 1),
                                 cudaMemcpyHostToDevice, ctx->stream));
        k_cell_pairs<<<grid_for(m, 64), 64, 0, ctx->stream>>>(
            c->sorted_orig.as<int>(), c->start.as<int>(), g, c->n, doff.as<int64_t>(), nullptr,
            dpi.as<int64_t>(), dpj.as<int64_t>());
        ++ctx->launches;
        MDB_CUDA(cudaMemcpyAsync(pi, dpi.ptr, sizeof(int64_t) * total, cudaMemcpyDeviceToHost, ctx->stream));
        MDB_CUDA(cudaMemcpyAsync(pj, dpj.ptr, sizeof(int64_t) * total, cudaMemcpyDeviceToHost, ctx->stream));
        MDB_CUDA(cudaStreamSynchronize(ctx->stream));
        doff.release();
        dpi.release();
        dpj.release();
    }
    cnt.release();
    return ctx_check_status(ctx);
}

}  // extern "C"
