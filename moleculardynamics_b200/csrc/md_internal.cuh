// md_internal.cuh -- shared internals of the moldyn B200 library.
//
// Device layout (one md_system):
//   pos   double4  (x, y, z, original index as a double)  -- gathered by pair kernels
//   vx vy vz fx fy fz mass inv_mass charge   double SoA   -- streamed by integrators
//   mol   int64 molecule id; orig (device slot -> original index), slot (inverse)
// Atoms are stored sorted by Morton-ranked cell (re-sorted at each Verlet rebuild).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/moldyn_b200.h"

namespace mdb {

// ------------------------------------------------------------------ errors
void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);

// Process-wide count of the events that can leave a captured step graph pointing
// at stale memory or parameters: every device buffer allocated, grown or freed,
// every atom permutation that swaps the system's arrays, every handle created,
// destroyed or reconfigured.  A cached graph is replayed only while it is unchanged.
uint64_t graph_epoch();
void graph_epoch_bump();

#define MDB_CUDA(call)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return ::mdb::fail(MD_ERR_CUDA, "%s:%d: %s: %s", __FILE__, __LINE__, #call,  \
                               cudaGetErrorString(e_));                                  \
    } while (0)

#define MDB_CHECK_LAUNCH() MDB_CUDA(cudaGetLastError())

#define MDB_TRY(call)            \
    do {                         \
        int rc_ = (call);        \
        if (rc_ != MD_OK) return rc_; \
    } while (0)

// One entry per block of a batched launch, {system, rank of the block among that
// system's blocks, their count, 0}, from the systems' block offsets off[0..nrep]:
// a block finds its system with one load.
inline std::vector<int4> block_table(const int* off, int nrep) {
    std::vector<int4> t(static_cast<size_t>(off[nrep]));
    for (int r = 0; r < nrep; ++r)
        for (int b = off[r]; b < off[r + 1]; ++b)
            t[static_cast<size_t>(b)] = make_int4(r, b - off[r], off[r + 1] - off[r], 0);
    return t;
}

// ------------------------------------------------------------ device buffers
// Grow-only device allocation (bytes), freed by the owner.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    int ensure(size_t want);
    void release();
    template <class T>
    T* as() const { return static_cast<T*>(ptr); }
};

}  // namespace mdb

// ------------------------------------------------------------------ context
namespace mdb {
// CUDA-event brackets around selected kernel launches (instrumentation only).
struct KernelTimer {
    std::vector<cudaEvent_t> ev;  // pairs: start, stop
    int used = 0;                 // pairs recorded since the last read
    int64_t launches = 0;
    double total_ms = 0.0;
};
constexpr int kTimedKernels = 8;
}  // namespace mdb

struct md_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t* d_status = nullptr;        // device status word
    unsigned* d_counter = nullptr;       // last-block counters (zeroed; reset by the last block)
    mdb::DevBuf partials;                // per-block reduction partials
    mdb::DevBuf scratch;                 // general scratch (staging, scans)
    mdb::DevBuf result;                  // small device results (energy, virial, ...)
    double* h_result = nullptr;          // pinned host mirror of `result`
    int64_t launches = 0;
    int64_t graph_captures = 0;          // step graphs captured by fused loops
    int sm_count = 148;
    bool timing = false;
    bool graphs = true;                  // fused loops replay a captured step graph
    mdb::KernelTimer timers[mdb::kTimedKernels];
    cudaEvent_t span_start = nullptr, span_stop = nullptr;
};

namespace mdb {

constexpr int kMaxResults = 64;      // doubles in context->result
constexpr int kCounterSlots = 64;    // independent last-block counters

// Result slot layout inside ctx->result (doubles).
enum ResultSlot : int {
    kResEnergy = 0,
    kResVirial = 1,
    kResKE = 2,
    kResTop2 = 4,      // 2 doubles: largest, second
    kResMomentum = 8,  // 4 doubles: px, py, pz, total mass
    kResFlag = 12,     // rebuild flag (as double)
    kResEwald = 16,    // 8 doubles: real, recip, self, intra, virial
    kResScratch = 32,
};

int ctx_partials(md_context* ctx, size_t doubles, double** out);
int ctx_scratch(md_context* ctx, size_t bytes, void** out);
int ctx_read_results(md_context* ctx, int first, int count, double* out);  // synchronises
int ctx_check_status(md_context* ctx);  // synchronises; MD_ERR_DEVICE if status set
// Bracket a launch with events when timing is enabled (kernel ids: MD_KERNEL_*).
void ctx_time_begin(md_context* ctx, int kernel);
void ctx_time_end(md_context* ctx, int kernel);
inline unsigned* ctx_counter(md_context* ctx, int slot) { return ctx->d_counter + slot; }
inline double* ctx_result(md_context* ctx, int slot) {
    return ctx->result.as<double>() + slot;
}

inline int grid_for(int64_t threads, int block) {
    int64_t g = (threads + block - 1) / block;
    return static_cast<int>(g < 1 ? 1 : g);
}

}  // namespace mdb

// ------------------------------------------------------------------- system
struct md_atoms {
    double4* pos = nullptr;  // x, y, z, (double) original index
    double *vx = nullptr, *vy = nullptr, *vz = nullptr;
    double *fx = nullptr, *fy = nullptr, *fz = nullptr;
    double *mass = nullptr, *inv_mass = nullptr, *charge = nullptr;
    int64_t* mol = nullptr;
    int* orig = nullptr;
};

struct md_system {
    md_context* ctx = nullptr;
    int64_t n = 0;
    double box[3] = {0, 0, 0};
    double inv_box[3] = {0, 0, 0};
    md_atoms cur, alt;        // current device order and the permutation target
    int* slot = nullptr;      // original index -> device slot
    uint64_t epoch = 1;       // bumped by every re-sort
    bool has_molecules = false;  // molecule ids differ from the atom's own index
    uint64_t mol_version = 1;    // bumped whenever molecule ids are set
    double last_energy = 0.0, last_virial = 0.0;
    // Fixed-point copy of the positions for the mixed-precision pair kernel: per
    // axis the box length maps to 2^32, so x, y, z are int32 (w = original index)
    // and one 16-byte load fetches a neighbour; written before each mixed launch.
    mdb::DevBuf qpos;
};

namespace mdb {

int system_alloc_atoms(md_system* sys, md_atoms* a);
void system_free_atoms(md_atoms* a);
// Applies a gather permutation: new slot s takes old slot perm[s].
int system_permute(md_system* sys, const int* d_perm);

// ------------------------------------------------------------- cell grid
struct CellGrid {
    int nx = 1, ny = 1, nz = 1;
    int ncells = 1;
    double cutoff = 0.0;
    double width[3] = {0, 0, 0};
    bool usable = false;
    int* rank_of_cell = nullptr;   // device: reference cell id -> Morton rank
    int* cell_of_rank = nullptr;   // device: rank -> reference cell id
    int init(const double box[3], double cutoff);
    void release();
};

// Counting sort of the system's atoms by (Morton rank of cell, original index).
// d_sorted receives, for sorted position s, the current device slot; d_start
// (ncells+1) the start of each rank's range.  Pure function of the positions.
int cell_sort(md_system* sys, const CellGrid& grid, int* d_sorted, int* d_start);

// One RDF frame of the atoms first, first + stride, ... added to the device
// histogram, no host synchronisation; rdf_sync refreshes the host counts.
int rdf_accumulate_async(md_rdf* r, md_system* sys, int64_t first, int64_t stride);
int rdf_sync(const md_rdf* r);
// The two halves of rdf_accumulate_async: the device work of a frame (capturable
// into a graph once the first frame has sized every buffer) and the host
// bookkeeping (frame count, density sum) each frame needs.
int rdf_frame_launch(md_rdf* r, md_system* sys, int64_t first, int64_t stride);
void rdf_frame_note(md_rdf* r, const md_system* sys, int64_t first, int64_t stride);

// Replicas stepped by batched kernels: one launch per stage of the step covers
// every replica, each block finding its replica in a per-block table.  The
// per-replica work inside is exactly that replica's solo step.
struct BatchRepView {
    md_integrator* it;
    md_system* sys;
    md_verlet* list;
    md_lj* lj;
    double* rows;                     // thermo rows at a device-held index, or null
    int* idx;
};
// system.cu: the kinetic energy of many systems in one launch, each with the blocks
// of its own system_kinetic_async (reduce_grid), into `out`.
struct BatchKineticRep {
    md_atoms a;
    int64_t n;
    double* part;
    unsigned* ticket;
    double* out;
};
int batch_kinetic_launch(const BatchKineticRep* reps, const int4* blk, int blocks,
                         cudaStream_t stream);
struct KickArgs;
// The closing half-kick of integrator `it` on `sys` for a force kernel to apply.
KickArgs integrator_kick_args(const md_integrator* it, md_system* sys);
struct BatchKick;     // integrate.cu: chain halves, kick/drift (+ rebuild test), kick + KE
struct BatchForce;    // lj.cu: the Verlet-list force pass
struct BatchRebuild;  // neighbor.cu: the gated rebuild of every replica, stage by stage
int batch_kick_create(const BatchRepView* reps, int nrep, BatchKick** out);
int batch_kick_pre(BatchKick* b, cudaStream_t stream, int64_t* launches);
// The first step of a run instead of batch_kick_pre: row indices reset, the chains'
// entry kinetic energies summed afresh, then the same kick/drift.
int batch_kick_first(BatchKick* b, cudaStream_t stream, int64_t* launches);
// The step's end: the closing half-kick with the kinetic energy (unless the force
// kernel took it: `kicked`), then the chain halves and thermo rows.
int batch_kick_post(BatchKick* b, cudaStream_t stream, int64_t* launches, bool kicked);
// After the last step of a batched run: every chain's pending scale applied.
int batch_kick_finish(BatchKick* b, cudaStream_t stream, int64_t* launches);
void batch_kick_destroy(BatchKick* b);
// MD_ERR_INVALID_ARGUMENT when the replicas' force kernels cannot share a launch
// (different precision, truncation, threads per atom or unrolling, halo tiles).
// With `kicks` (one per replica), a force kernel shape that can take the closing
// half-kick does (batch_force_kicks), as each replica's solo pass would.
int batch_force_create(const BatchRepView* reps, int nrep, const KickArgs* kicks, BatchForce** out);
int batch_force_launch(BatchForce* b, cudaStream_t stream, int64_t* launches);
bool batch_force_kicks(const BatchForce* b);
void batch_force_destroy(BatchForce* b);
// MD_ERR_INVALID_ARGUMENT when a replica's rebuild cannot join the batched stages
// (a list with halo tiles).
int batch_rebuild_create(const BatchRepView* reps, int nrep, BatchRebuild** out);
int batch_rebuild_launch(BatchRebuild* b, cudaStream_t stream, int64_t* launches);
// Once per run before the first replay: every replica's cell counts cleared.
int batch_rebuild_prime(BatchRebuild* b, cudaStream_t stream, int64_t* launches);
void batch_rebuild_destroy(BatchRebuild* b);
// Mixed precision: the fixed-point positions (after a rebuild re-sorted the atoms).
int lj_quantize_async(md_lj* lj, md_system* sys, const int* gate);

// Smooth particle-mesh Ewald reciprocal term (pme.cu): grid and cuFFT plans of
// one Ewald handle.  pme_eval_async writes the reciprocal energy and virial trace
// to out[0..1] (device) and, for mode != 0, adds the k-space forces.
struct PmeState;
int pme_create(md_context* ctx, const int K[3], int order, PmeState** out);
void pme_destroy(PmeState* s);
int pme_grid(const PmeState* s, int K[3], int* order);
int pme_eval_async(PmeState* s, md_system* sys, double alpha, double coulomb, int mode, double* out,
                   unsigned* ticket);

}  // namespace mdb

struct md_cells {
    md_context* ctx = nullptr;
    double box[3] = {0, 0, 0};
    mdb::CellGrid grid;
    mdb::DevBuf sorted_orig;  // original index per sorted position
    mdb::DevBuf start;        // ncells + 1
    md_system* sys = nullptr; // system it was last built from
    int64_t n = 0;
    bool built = false;
};

struct md_verlet {
    md_context* ctx = nullptr;
    double box[3] = {0, 0, 0};
    double cutoff = 0.0, skin = 0.0;
    int criterion = 0;            // 0 reference top-2 sum, 1 max > skin/2
    double cell_width = 0.0;      // 0: the reference's cells at the list cutoff
    mdb::CellGrid grid;
    mdb::DevBuf start;            // ncells + 1 (device order == sorted order)
    mdb::DevBuf perm;             // scratch for the sort
    mdb::DevBuf nbr;              // n * stride device indices
    mdb::DevBuf count;            // n neighbour counts
    mdb::DevBuf ref;              // n double4 positions at the last build
    int stride = 0;               // row capacity
    bool stride_fixed = false;    // host builds fail instead of growing it
    int64_t n = 0;
    int64_t rebuilds = 0;
    uint64_t epoch = 0;           // system epoch the list refers to
    md_system* sys = nullptr;
    int* d_rebuild_flag = nullptr; // device: set by the displacement check
    int* d_rebuild_total = nullptr; // device: rebuilds done inside fused loops
    int* d_max_count = nullptr;     // device: largest row seen by the last build
    // Halo tiles (mixed-precision force path): per block of kHaloAtoms sorted
    // atoms, runs of the cells around them and the rows as 16-bit halo slots.
    bool halo_on = false;
    mdb::DevBuf halo_runs;          // blocks * kHaloRuns int2 (first atom, slot base)
    mdb::DevBuf halo_meta;          // blocks int2 (runs or -1 when not staged, atoms)
    mdb::DevBuf nbr16;              // n * stride halo slots
};

namespace mdb {
// A halo tile: kHaloAtoms consecutive sorted atoms (one force block) and every
// atom of the cells around their cells, staged in at most kHaloCap slots of
// shared memory; blocks that span more than kHaloSpan cells or need more runs or
// slots than that keep gathering through the int32 rows.
constexpr int kHaloAtoms = 128;
constexpr int kHaloRuns = 64;
constexpr int kHaloCap = 2560;
constexpr int kHaloSpan = 16;
// Fused runs keep halo tiles for systems of at least this many atoms: below that,
// building the tiles at each rebuild costs more than the faster force kernel saves.
// The choice depends on the list and the force field only, never on the length of
// one call, so short and long runs of the same system step with the same kernels.
constexpr int64_t kHaloMinAtoms = 65536;
inline int64_t halo_blocks(int64_t n) { return (n + kHaloAtoms - 1) / kHaloAtoms; }
// Turns the halo tiles on for this list (built right away from the current list
// unless the stream is capturing); false when they cannot be used.
bool verlet_halo_ready(md_verlet* v, md_system* sys);
// The fused-run policy above, for a mixed-precision LJ force field.
void verlet_halo_for_run(md_verlet* v, md_system* sys, const md_lj* lj);
int verlet_build(md_verlet* v, md_system* sys, bool conditional);
int verlet_check(md_verlet* v, md_system* sys);  // device flag <- needs rebuild
int verlet_ensure_capacity(md_verlet* v, md_system* sys);
}  // namespace mdb

// --------------------------------------------------------------- potentials
struct md_lj {
    double sigma = 1, epsilon = 1, cutoff = 2.5;
    int truncation = MD_TRUNCATED;
    int precision = MD_PRECISION_FP64;
    double u_at_cutoff = 0, dudr_at_cutoff = 0;
    int tpa = 0, unroll = 0;   // launch shape of the Verlet force kernel (0: library default)
    bool halo = true;          // mixed precision: staged halo tiles where the list allows
    int tile_tpa = 0;          // tile kernel shape (0 single-buffer, 1 single-buffer bulk copies, 2/4/8 persistent)
};

namespace mdb {
// Adds one fused LJ step (kick/drift with the displacement check, a conditional
// node holding the gated neighbour rebuild, forces, kick, thermo row at rows +
// 4 * (*idx)) to `graph`, captured on the system's context stream.  The kernel
// counts outside / inside the rebuild branch are returned for launch accounting.
// One fused LJ step launched from the host (first: the chain half sums the
// current kinetic energy instead of using the tracked value).
int lj_fused_step(md_integrator* it, md_system* sys, md_verlet* v, md_lj* lj, double* rows,
                  int* idx, bool first);
int nhc_apply_scale_async(md_integrator* it, md_system* sys);
// The two halves of one host-driven step (pre_force with an optional fused
// displacement check against `check`'s reference positions; post_force).
int vv_pre_async(md_integrator* it, md_system* sys, md_verlet* check);
int vv_post_async(md_integrator* it, md_system* sys);
int capture_lj_step_into(md_integrator* it, md_system* sys, md_verlet* v, md_lj* lj,
                         double* rows, int* idx, cudaGraph_t graph, int64_t* main_launches,
                         int64_t* body_launches);

// Pair-force kernels over the Verlet list; results land in the context result
// slots kResEnergy / kResVirial (device), no synchronisation.
// q_gate: the fixed-point positions were written by the step's kick/drift; they
// are re-quantized only when this device flag says a rebuild re-sorted the atoms
// (null: always quantize).
// q_current: the fixed-point positions are known to be current (a step graph
// re-quantizes inside its rebuild branch), so no quantize launch at all.
// The closing half-kick of a step (velocity_verlet.hpp:70-73) and the kinetic
// energy after it, for a force kernel that applies the kick to each atom as it
// writes the atom's force (the kinetic energy lands in result slot kResKE).
struct KickArgs {
    double *vx = nullptr, *vy = nullptr, *vz = nullptr;
    const double* mass = nullptr;
    const double* inv_mass = nullptr;
    double half_dt = 0.0;
    uint32_t* status = nullptr;  // MD_STATUS_NONFINITE when a sum is not finite
};
// Verlet-list LJ forces, energy and virial.  With `kick`, a force kernel that can
// apply it does, and sets *kicked; otherwise *kicked stays false and the caller
// kicks.
int lj_forces_verlet_async(md_lj* lj, md_system* sys, md_verlet* v,
                           const int* q_gate = nullptr, bool q_current = false,
                           const KickArgs* kick = nullptr, bool* kicked = nullptr);
int lj_forces_brute_async(md_lj* lj, md_system* sys, bool forces);
int lj_forces_cells_async(md_lj* lj, md_system* sys, md_cells* cells);
int system_kinetic_async(md_system* sys, int slot);
}  // namespace mdb

// ------------------------------------------------------------- integrators
struct md_rigid {
    double oh = 1.0, hh = 0.0, tolerance = 1e-12;
    int max_iterations = 500;
    bool settle = false;  // closed-form SETTLE instead of SHAKE / RATTLE iterations
};

struct md_integrator {
    int kind = 0;                 // 0 VV, 1 BAOAB, 2 NHC, 3 constrained VV, 4 constrained VV + NHC
    md_rigid rigid;               // constraint of kinds 3 and 4
    mdb::DevBuf mol_state;        // kinds 3/4: per-molecule scratch (unconstrained positions)
    mdb::DevBuf counters;         // kinds 3/4: device iteration maxima
    double dt = 0.005;
    // BAOAB
    double friction = 1.0, temperature = 1.0;
    uint64_t seed = 0;
    uint64_t step = 0;            // O-step counter for Philox
    mdb::DevBuf noise;            // optional replayed normals (original order)
    int64_t noise_count = 0;
    int64_t noise_used = 0;
    // NHC
    double tau = 0.5;
    int chain = 3;
    int64_t dof = 0;
    mdb::DevBuf chain_state;      // device: NhcState
    md_context* ctx = nullptr;
    // md_run_lj: thermo rows that persist across calls (so a captured step graph
    // keeps its record target) and the last captured step graph with the key it
    // was captured under (system, list, force field, graph epoch).
    mdb::DevBuf run_rows, run_idx;
    mdb::DevBuf conserved;         // md_integrator_conserved's device result
    void* run_graph = nullptr;     // mdb::StepGraph*
    const void* run_key[3] = {nullptr, nullptr, nullptr};
    uint64_t run_epoch = 0;
    int* h_rebuilt = nullptr;      // pinned: device rebuild totals around the replays
};

namespace mdb {
// Chain-of-thermostats state kept on the device (nose_hoover.hpp:63-65).
constexpr int kMaxChain = 16;
struct NhcState {
    double Q[kMaxChain];
    double xi[kMaxChain];
    double pxi[kMaxChain];
    double dt, temperature;
    double dof;
    int chain;
    double scale;       // pending velocity scale (applied by the next kick)
    double ke;          // kinetic energy of the scaled velocities
};
}  // namespace mdb
