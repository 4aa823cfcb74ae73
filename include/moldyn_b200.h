/*
 * moldyn_b200.h -- C ABI of the B200-native moldyn force / neighbour / integrator path.
 *
 * Plain C: opaque handles, plain pointers and sizes, int status codes.  Every
 * entry point names the reference interface it replaces (path:line inside the
 * moldyn project); the C++ drop-in headers (moleculardynamics_b200/include/
 * moldyn/...) wrap these calls behind the reference's own class names.
 *
 * Conventions
 *  - Status: MD_OK (0) on success, a negative MD_ERR_* otherwise; the message is
 *    in md_last_error() (thread-local).  MD_ERR_INVALID_ARGUMENT and
 *    MD_ERR_RUNTIME map to the reference's std::invalid_argument and
 *    std::runtime_error.
 *  - Host arrays are in the caller's atom order ("original order"), one double
 *    per atom per component.  On the device atoms are kept sorted by cell; the
 *    library permutes on the way in and out.
 *  - Each context owns one CUDA stream.  Handles are not thread-safe; distinct
 *    contexts may be used from distinct host threads.
 *  - Device-side failures (neighbour-list overflow, constraint non-convergence,
 *    non-finite forces) are recorded in a per-context status word and reported
 *    at the next call that synchronises.  No kernel traps or waits unboundedly.
 */
#ifndef MOLDYN_B200_H
#define MOLDYN_B200_H

#include <stddef.h>
#include <stdint.h>

/* Only the md_* entry points are exported from libmoldyn_b200.so. */
#if defined(__GNUC__)
#define MD_API __attribute__((visibility("default")))
#else
#define MD_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define MD_OK 0
#define MD_ERR_INVALID_ARGUMENT (-1) /* reference: std::invalid_argument */
#define MD_ERR_RUNTIME (-2)          /* reference: std::runtime_error */
#define MD_ERR_CUDA (-3)             /* CUDA runtime error (no reference counterpart) */
#define MD_ERR_OUT_OF_MEMORY (-4)
#define MD_ERR_DEVICE (-5)           /* device status word set (see md_context_status) */

/* Device status bits (md_context_status). */
#define MD_STATUS_NEIGHBOR_OVERFLOW 0x1u /* a per-atom neighbour row overflowed */
#define MD_STATUS_SHAKE_DIVERGED 0x2u    /* SHAKE did not converge in maxIterations */
#define MD_STATUS_RATTLE_DIVERGED 0x4u   /* RATTLE did not converge in maxIterations */
#define MD_STATUS_SHAKE_SINGULAR 0x8u    /* SHAKE denominator below 1e-30 */
#define MD_STATUS_NONFINITE 0x10u        /* a position or the kinetic energy stopped being finite */
#define MD_STATUS_WAIT_TIMEOUT 0x20u     /* a kernel's bounded wait on its own copies ran out */

/* System fields (core/system.hpp:54-59). */
#define MD_FIELD_X 0
#define MD_FIELD_Y 1
#define MD_FIELD_Z 2
#define MD_FIELD_VX 3
#define MD_FIELD_VY 4
#define MD_FIELD_VZ 5
#define MD_FIELD_FX 6
#define MD_FIELD_FY 7
#define MD_FIELD_FZ 8
#define MD_FIELD_MASS 9
#define MD_FIELD_CHARGE 10

/* Truncation (forcefield/lennard_jones.hpp:11). */
#define MD_TRUNCATED 0
#define MD_LINEAR_FORCE_SHIFT 1

/* Precision of the pair arithmetic. */
#define MD_PRECISION_FP64 0  /* drop-in path: reference arithmetic in FP64 */
#define MD_PRECISION_MIXED 1 /* FP32 pair terms, FP64 displacement and accumulation */

typedef struct md_context md_context;
typedef struct md_system md_system;
typedef struct md_cells md_cells;
typedef struct md_verlet md_verlet;
typedef struct md_lj md_lj;
typedef struct md_integrator md_integrator;
typedef struct md_ewald md_ewald;
typedef struct md_rigid md_rigid;
typedef struct md_batch md_batch;
typedef struct md_adjoint md_adjoint;
typedef struct md_rdf md_rdf;
typedef struct md_msd md_msd;
typedef struct md_vacf md_vacf;
typedef struct md_thermo_csv md_thermo_csv;

/* ------------------------------------------------------------------ library */
/* Message of the last failing call on this thread ("" if none). */
MD_API const char* md_last_error(void);
/* ABI version of this header (major*10000 + minor*100 + patch). */
MD_API int md_abi_version(void);

/* ------------------------------------------------------------------ context */
/* No reference counterpart: the reference is one CPU thread.  One context =
 * one device + one stream + the device status word + reusable scratch. */
MD_API int md_context_create(int device, md_context** out);
MD_API int md_context_destroy(md_context* ctx);
MD_API int md_context_synchronize(md_context* ctx);
/* The device's name and SM count, e.g. for keying tuned launch shapes. */
MD_API int md_context_device_name(const md_context* ctx, char* name, int len);
/* Reads (and with clear != 0, clears) the device status word; synchronises. */
MD_API int md_context_status(md_context* ctx, uint32_t* status, int clear);
/* Number of kernels this context has launched (instrumentation). */
MD_API int md_context_launch_count(md_context* ctx, int64_t* count);
/* Step graphs captured by fused loops on this context (no reference counterpart).
 * md_run_lj replays the step graph of an earlier call while the system, list and
 * force field are the same handles and no device buffer was allocated, freed or
 * permuted and no handle created, destroyed or reconfigured in between; each new
 * capture adds one. */
MD_API int md_context_graph_captures(md_context* ctx, int64_t* count);

/* Instrumentation, no reference counterpart.  With timing enabled, launches of
 * the kernels below are bracketed by CUDA events on the context's stream;
 * md_context_kernel_time returns their summed device time (synchronises). */
#define MD_KERNEL_LJ_FORCE 0     /* Lennard-Jones pair forces over the Verlet list */
#define MD_KERNEL_NEIGHBOR 1     /* cell binning + Verlet build (host-driven builds) */
#define MD_KERNEL_INTEGRATE 2    /* kick / drift / thermostat kernels */
#define MD_KERNEL_EWALD_REAL 3   /* Ewald real-space pairs */
#define MD_KERNEL_EWALD_RECIP 4  /* Ewald structure factors and k-space forces */
MD_API int md_context_set_timing(md_context* ctx, int enable);
/* Fused device loops (md_run_lj) replay one captured CUDA graph per step, the
 * device-decided neighbour rebuild being a conditional node, when enabled
 * (default) and timing is off; 0 launches every kernel from the host instead.
 * Results are identical either way.  No reference counterpart. */
MD_API int md_context_set_graphs(md_context* ctx, int enable);
MD_API int md_context_kernel_time(md_context* ctx, int kernel, int reset, double* total_ms,
                                  int64_t* launches);
/* Device time between two points on the context's stream (CUDA events). */
MD_API int md_context_span_begin(md_context* ctx);
MD_API int md_context_span_end(md_context* ctx, double* ms);
/* Page-locked host memory for fast host<->device copies (NULL on failure). */
MD_API void* md_host_alloc(size_t bytes);
MD_API int md_host_free(void* p);

/* ------------------------------------------------------------------- system */
/* System(Box) + addAtom (core/system.hpp:15-27).  Positions, velocities,
 * forces and charges start at 0, masses at 1, molecule ids at the atom's own
 * index (system.cpp:17-22). */
MD_API int md_system_create(md_context* ctx, int64_t n, const double box[3], md_system** out);
MD_API int md_system_destroy(md_system* sys);
MD_API int64_t md_system_size(const md_system* sys);                  /* system.hpp:17 */
MD_API int md_system_box(const md_system* sys, double box[3]);        /* box.hpp:14-15 */
/* Set or get one field: n doubles in original order (system.hpp:29-43). */
MD_API int md_system_set(md_system* sys, int field, const double* src);
MD_API int md_system_get(md_system* sys, int field, double* dst);
/* Several fields at once (fields[k] <- src[k], dst[k] <- fields[k]): every
 * column's copy is queued before one host synchronisation, where md_system_set
 * and md_system_get synchronise per field.  Pinned host memory (md_host_alloc)
 * lets the copies run as DMA. */
MD_API int md_system_set_fields(md_system* sys, int count, const int* fields, const double* const* src);
MD_API int md_system_get_fields(md_system* sys, int count, const int* fields, double* const* dst);
MD_API int md_system_set_molecule_ids(md_system* sys, const int64_t* ids); /* system.hpp:43 */
MD_API int md_system_get_molecule_ids(md_system* sys, int64_t* ids);       /* system.hpp:34 */
MD_API int md_system_zero_forces(md_system* sys);                          /* system.cpp:116-122 */
MD_API int md_system_kinetic_energy(md_system* sys, double* ke);           /* system.cpp:124-131 */
MD_API int md_system_total_momentum(md_system* sys, double p[3]);          /* system.cpp:137-145 */
MD_API int md_system_remove_com_motion(md_system* sys);                    /* system.cpp:147-164 */
/* Velocity rescale toward `target` on the device, no host round trip:
 * t = 2 KE / dof, and v *= sqrt(target / t) when t > 0 (the equilibration
 * rescale of apps/water_rdf.cpp:186-195, system.cpp:133-135). */
MD_API int md_system_rescale_temperature(md_system* sys, int64_t dof, double target);
/* Potential energy and virial of the last force evaluation on this system. */
MD_API int md_system_last_energy(md_system* sys, double* energy, double* virial);

/* --------------------------------------------------------------- cell list */
/* CellList(box, cutoff) (neighbor/cell_list.hpp:28, cell_list.cpp:8-14). */
MD_API int md_cells_create(md_context* ctx, const double box[3], double cutoff, md_cells** out);
MD_API int md_cells_destroy(md_cells* cells);
MD_API int md_cells_dims(const md_cells* cells, int dims[3]);  /* cell_list.hpp:36 */
MD_API int md_cells_usable(const md_cells* cells);             /* cell_list.hpp:37: 1/0 */
MD_API int md_cells_build(md_cells* cells, md_system* sys);    /* cell_list.cpp:16-43 */
/* forEachPair (cell_list.hpp:55-108) as an exported candidate-pair set: every
 * (i<j), original indices, each unordered pair once, in unspecified order.
 * *count receives the total; at most cap pairs are written.  Requires usable(). */
MD_API int md_cells_pairs(md_cells* cells, int64_t* pi, int64_t* pj, int64_t cap, int64_t* count);

/* ------------------------------------------------------------- Verlet list */
/* VerletList(box, cutoff, skin) (neighbor/verlet_list.hpp:28, verlet_list.cpp:5-6). */
MD_API int md_verlet_create(md_context* ctx, const double box[3], double cutoff, double skin,
                     md_verlet** out);
MD_API int md_verlet_destroy(md_verlet* list);
/* build (verlet_list.cpp:8-42): re-sorts the system's device order by cell. */
MD_API int md_verlet_build(md_verlet* list, md_system* sys);
/* needsRebuild (verlet_list.cpp:44-63): *flag = 1/0. */
MD_API int md_verlet_needs_rebuild(md_verlet* list, md_system* sys, int* flag);
/* rebuildIfNeeded (verlet_list.cpp:65-69).  *rebuilt (nullable) = 1/0. */
MD_API int md_verlet_rebuild_if_needed(md_verlet* list, md_system* sys, int* rebuilt);
MD_API int md_verlet_rebuild_count(md_verlet* list, int64_t* count); /* verlet_list.hpp:32 */
/* forEachPair (verlet_list.hpp:52-57) as an exported set: pairs (i<j), original
 * indices, sorted by (i, j). */
MD_API int md_verlet_pairs(md_verlet* list, int64_t* pi, int64_t* pj, int64_t cap, int64_t* count);
/* Rebuild criterion: 0 = reference (sum of the two largest displacements >
 * skin, verlet_list.cpp:44-63), 1 = largest displacement > skin/2. */
MD_API int md_verlet_set_criterion(md_verlet* list, int criterion);
/* Largest and second-largest displacement since the last build (diagnostics). */
MD_API int md_verlet_displacements(md_verlet* list, md_system* sys, double* largest, double* second);
/* Row capacity (neighbours per atom) of the list; no reference counterpart (the
 * reference's list is a growing vector of pairs).  Host-driven builds grow a row
 * capacity that overflows and build again, unless `fixed` is set, in which case
 * the build fails with MD_ERR_RUNTIME; a rebuild decided on the device inside a
 * fused loop cannot grow it and reports MD_ERR_DEVICE (neighbour overflow).  The
 * list must be built again before its next use. */
MD_API int md_verlet_set_capacity(md_verlet* list, int capacity, int fixed);
/* Width of the cells the list is built from; no reference counterpart (the
 * reference bins at the list cutoff rc + skin, cell_list.cpp:8-14, which 0
 * restores).  Any width >= rc + skin gives the same pair set: wider cells mean
 * more candidates per atom but fewer cells (a tuning axis).  The list must be
 * built again before its next use. */
MD_API int md_verlet_set_cell_width(md_verlet* list, double width);
/* Cells per side of the list's grid (after md_verlet_set_cell_width). */
MD_API int md_verlet_cells_per_side(const md_verlet* list, int dims[3]);

/* ----------------------------------------------------------- Lennard-Jones */
/* LennardJones(sigma, epsilon, cutoff, truncation) (lennard_jones.hpp:26,
 * lennard_jones.cpp:32-48) plus the pair precision. */
MD_API int md_lj_create(double sigma, double epsilon, double cutoff, int truncation, int precision,
                 md_lj** out);
MD_API int md_lj_destroy(md_lj* lj);
/* computeEnergyVirial (lennard_jones.cpp:90-92): brute force, forces untouched. */
MD_API int md_lj_energy_virial(md_lj* lj, md_system* sys, double* energy, double* virial);
/* computeForces(sys) (lennard_jones.cpp:94-97): brute force, zeroes forces first. */
MD_API int md_lj_forces(md_lj* lj, md_system* sys, double* energy, double* virial);
/* computeForces(sys, CellList) (lennard_jones.cpp:99-114): MD_ERR_INVALID_ARGUMENT
 * when the cell list is not usable. */
MD_API int md_lj_forces_cells(md_lj* lj, md_system* sys, md_cells* cells, double* energy,
                       double* virial);
/* computeForces(sys, VerletList) (lennard_jones.cpp:116-119). */
MD_API int md_lj_forces_verlet(md_lj* lj, md_system* sys, md_verlet* list, double* energy,
                        double* virial);
/* longRangeCorrection / longRangeCorrectionPressure (lennard_jones.cpp:121-151). */
MD_API int md_lj_lrc(const md_lj* lj, int64_t n, const double box[3], double* u_lrc, double* p_lrc);
/* Launch shape of the Verlet-list force kernel (process-wide tuning knobs; no
 * reference counterpart -- the reference is scalar): threads per atom 1, 2, 4 or 8
 * (default 2) and independent neighbour gathers in flight per thread 1, 2 or 4
 * (default 2). */
MD_API int md_lj_set_threads_per_atom(int tpa);
MD_API int md_lj_set_unroll(int unroll);
/* Launch shape of this LJ object's Verlet force kernel (threads per atom 1/2/4/8,
 * gathers in flight 1/2/4; 0 = the library default).  Set by the autotuner
 * (moleculardynamics_b200/autotune.py); no reference counterpart. */
MD_API int md_lj_set_launch(md_lj* lj, int tpa, int unroll);
/* Mixed precision only: read neighbours through the list's halo tiles when it
 * keeps them (on = 1, the default) or always gather them through the int32 rows
 * (0).  A halo tile holds a block of 128 cell-sorted atoms and every atom of the
 * cells around them in shared memory; rows then also exist as 16-bit tile slots.
 * Forces are identical either way.  No reference counterpart. */
MD_API int md_lj_set_halo(md_lj* lj, int on);
/* Shape of the mixed tile kernel: 0 (the default) one CTA per tile with two threads
 * per atom, the halo staged by the threads; 1 the same with the halo queued by bulk
 * copies on an mbarrier and the rows read in whole padded chunks; 2, 4 or 8 threads
 * per atom in the persistent double-buffered kernel.  No reference counterpart, a
 * tuning axis.  Every shape sums the
 * same pairs with the same arithmetic, in a different order. */
MD_API int md_lj_set_tile_threads(md_lj* lj, int tpa);
/* Halo tiles of a Verlet list: built now from the current list and again at
 * every rebuild (on = 1), or dropped (0).  md_run_lj and md_batch_run turn them on
 * by themselves for mixed-precision runs of >= 16 steps on >= 65,536 atoms, where
 * the faster force kernel pays for building them.  Lists without a cell grid
 * (fewer than 3 cells per side) keep none.  No reference counterpart. */
MD_API int md_verlet_set_halo(md_verlet* v, int on);
/* How many of a list's halo tiles are staged in shared memory (the rest gather
 * through the int32 rows), out of how many (0, 0 without tiles).  Diagnostics;
 * synchronises. */
MD_API int md_verlet_halo_tiles(md_verlet* v, int64_t* staged, int64_t* tiles);

/* ------------------------------------------------------------------- Ewald */
/* e^2/(4 pi eps0 kB) in K*Angstrom/e^2 (ewald.cpp:17-21). */
MD_API double md_coulomb_prefactor(void);
/* Ewald(cutoff, kmax) (forcefield/ewald.hpp:51) plus alpha: alpha <= 0 selects the
 * reference's 5.6 / min(L) (ewald.cpp:40); the reference has no alpha parameter.
 * Real space runs over an internal Verlet list at cutoff + skin (default 1.0). */
MD_API int md_ewald_create(md_context* ctx, double cutoff, int kmax, double alpha,
                           md_ewald** out);
MD_API int md_ewald_destroy(md_ewald* ew);
MD_API int md_ewald_set_skin(md_ewald* ew, double skin);
/* mode 0 computeEnergies, 1 computeForces (zeroes first), 2 accumulateForces
 * (ewald.cpp:177-188).  terms = EwaldTerms {real, reciprocal, self, intra}
 * (ewald.hpp:24-31).  virial (nullable): atomic virial of the Ewald sum -- no
 * reference counterpart (the reference computes none). */
MD_API int md_ewald_compute(md_ewald* ew, md_system* sys, int mode, double terms[4],
                            double* virial);
MD_API int md_ewald_alpha(const md_ewald* ew, double* alpha);          /* last alpha used */
MD_API int md_ewald_kvector_count(const md_ewald* ew, int* count);     /* full k set */
/* Smooth particle-mesh Ewald (Essmann et al., J. Chem. Phys. 103, 8577 (1995))
 * for the reciprocal term instead of the k-vector sums of ewald.cpp:112-172:
 * a kx x ky x kz charge grid (each in [2 order, 4096]) and cardinal B-splines of
 * order 4, 6 or 8; kx = ky = kz = 0 returns to the k-vector sums.  The
 * reference defers PME (no counterpart); real space, self and intramolecular
 * terms are unchanged.  md_ewald_charge_gradient needs the k-vector sums. */
MD_API int md_ewald_set_pme(md_ewald* ew, int kx, int ky, int kz, int order);
/* Precision of the real-space pair terms (erfc, exp, O-O LJ powers):
 * MD_PRECISION_FP64 (default, the reference's arithmetic) or MD_PRECISION_MIXED
 * (FP32 pair terms; displacements, cutoff test and all sums in FP64). */
MD_API int md_ewald_set_precision(md_ewald* ew, int precision);
/* The PME grid and order, zeros when the k-vector sums are in use. */
MD_API int md_ewald_pme_grid(const md_ewald* ew, int k[3], int* order);

/* SpceForceField(params, cutoff, kmax) (forcefield/spce_forcefield.hpp:31-33):
 * O-O Lennard-Jones (sigma_o, epsilon_o, truncated, with tail) + Ewald, on O,H,H
 * triples.  Returns an md_ewald handle usable with md_spce_compute. */
MD_API int md_spce_create(md_context* ctx, double sigma_o, double epsilon_o, double cutoff,
                          int kmax, double alpha, md_ewald** out);
/* computeForces (forces != 0; zeroes forces first) or computeEnergy
 * (spce_forcefield.cpp:26-48).  parts (nullable, 8 doubles): Edisp, ELRC, Ereal,
 * Efourier, Eself, Eintra, atomic virial, total. */
MD_API int md_spce_compute(md_ewald* ff, md_system* sys, int forces, double* energy,
                           double parts[8]);

/* O-O Lennard-Jones truncation of an SPC/E force field: MD_TRUNCATED (default,
 * with the analytic tail, spce_forcefield.cpp:9) or MD_LINEAR_FORCE_SHIFT (no
 * tail; the continuous force tests/test_rigid_water.cpp:189-190 use). */
MD_API int md_spce_set_lj_truncation(md_ewald* ff, int truncation);

/* ------------------------------------------------------------- rigid water */
/* RigidWater(ohDistance, hohAngleDegrees, tolerance, maxIterations)
 * (constrain/rigid_water.hpp:32-35, rigid_water.cpp:30-53); invalid arguments give
 * MD_ERR_INVALID_ARGUMENT like the reference's std::invalid_argument. */
MD_API int md_rigid_create(double oh, double hoh_degrees, double tolerance, int max_iterations,
                           md_rigid** out);
/* Solve the constraints in closed form (on = 1) with SETTLE (Miyamoto &
 * Kollman 1992) -- the specialisation rigid_water.hpp:20-24 plans -- instead of
 * SHAKE / RATTLE iterations: the same fixed point, reached without iterating
 * (positions agree with SHAKE to its tolerance; molecules with unequal hydrogen
 * masses, or configurations SETTLE cannot solve, still take SHAKE).  Applies to
 * md_rigid_constrain_* and to integrators created from this object afterwards. */
MD_API int md_rigid_set_settle(md_rigid* rw, int on);
MD_API int md_rigid_destroy(md_rigid* rw);
MD_API int md_rigid_distances(const md_rigid* rw, double* oh, double* hh);
/* degreesOfFreedom(molecules, comRemoved) (rigid_water.cpp:55-59). */
MD_API int64_t md_rigid_degrees_of_freedom(int64_t molecules, int com_removed);
/* constrainPositions(sys, reference) (rigid_water.cpp:61-116): reference positions
 * as host arrays in original order.  constrainVelocities (rigid_water.cpp:118-161).
 * *iterations receives the sweep count; non-convergence or a singular constraint
 * returns MD_ERR_RUNTIME (the reference's std::runtime_error). */
MD_API int md_rigid_constrain_positions(md_rigid* rw, md_system* sys, const double* rx,
                                        const double* ry, const double* rz, int* iterations);
MD_API int md_rigid_constrain_velocities(md_rigid* rw, md_system* sys, int* iterations);

/* -------------------------------------------------------------- integrators */
/* VelocityVerlet(dt) (integrate/velocity_verlet.hpp:41). */
MD_API int md_integrator_create_vv(double dt, md_integrator** out);
/* LangevinBAOAB(dt, friction, temperature, seed) (integrate/langevin.hpp:29).
 * The O-step noise is Philox4x32-10 keyed by seed, counter (step, atom). */
MD_API int md_integrator_create_baoab(double dt, double friction, double temperature, uint64_t seed,
                               md_integrator** out);
/* NoseHooverChain(dt, T, tau, chainLength, dof) (integrate/nose_hoover.hpp:27-28);
 * MD_ERR_INVALID_ARGUMENT when chainLength < 1 (nose_hoover.cpp:36-38). */
MD_API int md_integrator_create_nhc(double dt, double temperature, double tau, int chain_length,
                             int64_t dof, md_integrator** out);
/* ConstrainedVelocityVerlet(dt, RigidWater) (integrate/constrained_velocity_verlet.hpp:25-26). */
MD_API int md_integrator_create_rattle(double dt, const md_rigid* rw, md_integrator** out);
/* The Nose-Hoover chain around the constrained step -- no reference counterpart
 * (the reference has no thermostatted rigid-water integrator); dof = 6M - 3 for M
 * molecules with the centre of mass fixed. */
MD_API int md_integrator_create_rattle_nhc(double dt, const md_rigid* rw, double temperature,
                                           double tau, int chain_length, int64_t dof,
                                           md_integrator** out);
/* Largest SHAKE / RATTLE sweep counts seen by a constrained integrator. */
MD_API int md_integrator_iterations(md_integrator* integ, int* shake, int* rattle);
MD_API int md_integrator_destroy(md_integrator* integ);
/* The step is split around the force call so a host ForceFn can run between
 * (velocity_verlet.hpp:43-47: called exactly once per step):
 *   pre_force  -- everything before computeForces (B, A[, O, A] / chain, B, A);
 *   post_force -- everything after it (B[, chain]). */
MD_API int md_integrator_pre_force(md_integrator* integ, md_system* sys);
MD_API int md_integrator_post_force(md_integrator* integ, md_system* sys);
/* conservedQuantityContribution (nose_hoover.cpp:45-54); 0 for VV and BAOAB. */
MD_API int md_integrator_conserved(md_integrator* integ, double* value);
/* BAOAB only: take the O-step normals from xi[3*i + {0,1,2}] (original atom
 * order, n*steps values, one block of 3n per step) instead of Philox.  Lets a
 * test replay the reference's exact mt19937_64 stream.  NULL restores Philox. */
MD_API int md_integrator_set_noise(md_integrator* integ, const double* xi, int64_t count);

/* Fused device loop: `steps` steps of integ with LJ forces on the Verlet list
 * (rebuildIfNeeded + computeForces, apps/moldyn_run.cpp:581-587), without a
 * host synchronisation per step.  Forces must be current on entry.  thermo
 * (nullable, steps*4 doubles) receives per step: pair energy, virial, kinetic
 * energy, conserved-quantity contribution. */
MD_API int md_run_lj(md_integrator* integ, md_system* sys, md_verlet* list, md_lj* lj, int64_t steps,
              double* thermo);

/* Lennard-Jones forces, energy and virial by brute force (the arithmetic of
 * md_lj_forces) for callers that must not allocate device memory -- no counterpart
 * in the reference.  Callers such as a host framework that owns all device memory
 * through its own pool, or latency-critical loops that cannot afford cudaMalloc's
 * device-wide synchronisation, pass their own device buffers: positions
 * d_x/d_y/d_z (n doubles each, atom order; they need not be wrapped into the box:
 * every displacement folds by the reference's minimum image), force
 * outputs d_fx/d_fy/d_fz and d_energy_virial (2 doubles: pair energy, virial),
 * and the CUDA stream to run on (NULL = legacy default stream).  The call
 * allocates nothing: its reduction scratch is a fixed 16 KiB array in the
 * library's device image, held by every GPU that loads the library until the
 * process exits, which limits n to 262,144 atoms (larger n is rejected with
 * MD_ERR_INVALID_ARGUMENT).  The first call on each device looks up the array's
 * device address (cudaGetSymbolAddress), so make that first call before any
 * stream capture.  The address is kept for the life of the process: do not call
 * this after a cudaDeviceReset.  All calls share the array: calls that may overlap
 * on the GPU (different streams, or different host threads on one device) race
 * and must be serialised by the caller.  The call returns once the work is
 * enqueued. */
MD_API int md_lj_forces_static(const double* d_x, const double* d_y, const double* d_z,
                               int64_t n, const double box[3], double sigma, double epsilon,
                               double cutoff, int truncation, double* d_fx, double* d_fy,
                               double* d_fz, double* d_energy_virial, void* stream);

/* -------------------------------------------------------------------- setup */
/* fccLattice(cells, density, temperature, seed) (util/lattice.cpp:15-64), on the
 * host: writes 4*cells^3 atoms into caller arrays (original order) and the cubic
 * box; velocities from std::mt19937_64 with the reference's polar Box-Muller
 * (util/random.hpp:52-69).  Returns the atom count, or MD_ERR_INVALID_ARGUMENT. */
MD_API int md_fcc_lattice(int cells, double density, double temperature, uint64_t seed, double* x,
                   double* y, double* z, double* vx, double* vy, double* vz, double* mass,
                   double box[3]);
/* `count` consecutive normal draws of Rng(seed) (util/random.hpp:37-76):
 * std::mt19937_64 and the polar Box-Muller transform, host-side setup.
 * Returns count or MD_ERR_INVALID_ARGUMENT. */
MD_API int64_t md_rng_normals(uint64_t seed, int64_t count, double* out);

/* ------------------------------------------------------------ replica batches */
/* Many independent LJ replicas stepped together; no reference counterpart (the
 * reference runs one system per moldyn_run process).  Each replica is an
 * integrator (velocity Verlet or Nose-Hoover chain), a system on its own context,
 * its Verlet list (built) and an LJ force field.  md_batch_run advances every
 * replica by `steps` fused steps, replaying one CUDA graph per step that holds
 * all replicas' kernels as independent chains; each replica's trajectory equals
 * the one md_run_lj gives it alone.  thermo (nullable): replicas x steps x 4
 * doubles (potential energy, virial, kinetic energy, chain contribution). */
MD_API int md_batch_create(md_batch** out);
MD_API int md_batch_destroy(md_batch* batch);
MD_API int md_batch_add(md_batch* batch, md_integrator* integ, md_system* sys, md_verlet* list,
                        md_lj* lj, int* index);
MD_API int md_batch_size(const md_batch* batch);
/* Stage kernels shared by all replicas (default, 1): each stage of the step is
 * one launch over every replica through a per-block table of replicas, the
 * rebuild stages gated per replica on the device; 0, or replicas whose force kernels
 * differ (precision, truncation, threads per atom, unrolling, halo tiles, cubic
 * and non-cubic boxes in one mixed batch), replay a graph of per-replica
 * kernels.  Each replica's trajectory is its solo run's either way. */
MD_API int md_batch_set_batched(md_batch* b, int on);
MD_API int md_batch_run(md_batch* batch, int64_t steps, double* thermo);

/* ------------------------------------------------ differentiable trajectories */
/* No reference counterpart.  A velocity-Verlet LJ trajectory (FP64) with a
 * hand-written adjoint, in torch.autograd.Function form: md_adjoint_forward runs
 * `steps` steps from the system's state, saves the state every `every` steps
 * (the save-for-backward) and writes rows (steps x 3: potential energy, virial
 * W = sum of w, kinetic energy after each step).  Its Verlet list (cutoff + skin)
 * is rebuilt only at the saved states; a step whose list the reference rebuild
 * criterion would reject fails the call (MD_ERR_RUNTIME: raise the skin or save
 * more often).  md_adjoint_backward takes dL/d(row) (steps x 3), recomputes each
 * segment from its saved state and returns dL/d(epsilon, sigma), and optionally
 * dL/d(initial positions) and dL/d(initial velocities) (n x 3, caller's order).
 * The system is left where the forward left it.  md_adjoint_backward replays
 * on the system the forward ran on: it must not be destroyed in between. */
MD_API int md_adjoint_create(md_context* ctx, md_adjoint** out);
MD_API int md_adjoint_destroy(md_adjoint* adj);
MD_API int md_adjoint_forward(md_adjoint* adj, md_system* sys, const md_lj* lj, double dt,
                              int64_t steps, int every, double skin, double* rows);
MD_API int md_adjoint_backward(md_adjoint* adj, const double* grad_rows, double grad_theta[2],
                               double* grad_x0, double* grad_v0);
/* Hessian-vector product of the LJ forces: out = (dF/dx)^T u for a per-atom
 * field u (n x 3, caller's order), and dtheta = (u . dF/d epsilon, u . dF/d sigma).
 * FP64, over a built Verlet list.  No reference counterpart. */
MD_API int md_lj_hvp(const md_lj* lj, md_system* sys, md_verlet* list, const double* u, double* out,
                     double dtheta[2]);

/* Derivatives of the Ewald sum (no reference counterpart).  Charge gradient of
 * the Coulomb energy, real + reciprocal + self + intramolecular terms
 * (ewald.cpp:33-175): dedq[i] = dE/dq_i (n, caller's order).  Hessian-vector
 * product of the real-space Coulomb forces: out = (dF_real/dx)^T u (n x 3). */
MD_API int md_ewald_charge_gradient(md_ewald* ff, md_system* sys, double* dedq);
MD_API int md_ewald_real_hvp(md_ewald* ff, md_system* sys, const double* u, double* out);

/* Fused device loop of a constrained integrator with SPC/E forces (the
 * water_rdf-style NVE / NHC production loop): forces are (re)computed on entry,
 * neighbour rebuilds are decided on the device.  thermo (nullable, steps*4):
 * potential energy (K), virial, kinetic energy, conserved contribution. */
MD_API int md_run_spce(md_integrator* integ, md_system* sys, md_ewald* ff, int64_t steps,
                       double* thermo);

/* ---------------------------------------------------------------- analysis */
/* Radial distribution function, analyze/rdf.hpp:16-34 (Rdf(rMax, bins)).
 * md_rdf_accumulate adds one frame (rdf.cpp:55-82): every pair i < j with
 * minimum-image distance r < rMax counted into bin (size_t)(r / (rMax / bins)),
 * MD_ERR_INVALID_ARGUMENT (the reference's std::invalid_argument) when rMax
 * exceeds half the smallest box length.  Pairs are found through a cell grid of
 * width >= rMax on the device; the distance and bin use the reference's
 * arithmetic, so md_rdf_histogram (bins doubles: the raw pair counts) equals the
 * reference's histogram.  md_rdf_g is Rdf::g (rdf.cpp:92-107), md_rdf_bin_centres
 * Rdf::binCentres (rdf.cpp:84-90), md_rdf_frames Rdf::frames. */
MD_API int md_rdf_create(md_context* ctx, double rmax, int64_t bins, md_rdf** out);
MD_API int md_rdf_destroy(md_rdf* rdf);
MD_API int md_rdf_accumulate(md_rdf* rdf, md_system* sys);
/* The frame of the atoms with original index first, first + stride, ... alone,
 * as Rdf::accumulate of a System holding just those atoms in that order (e.g.
 * the oxygens of consecutive O, H, H water molecules: first 0, stride 3, as
 * apps/water_rdf.cpp:90-97 gathers them). */
MD_API int md_rdf_accumulate_subset(md_rdf* rdf, md_system* sys, int64_t first, int64_t stride);
MD_API int md_rdf_histogram(const md_rdf* rdf, double* hist);
MD_API int md_rdf_g(const md_rdf* rdf, double* g);
MD_API int md_rdf_bin_centres(const md_rdf* rdf, double* centres);
MD_API int md_rdf_frames(const md_rdf* rdf, int64_t* frames);

/* The simulation of apps/water_rdf.cpp:159-216 in one call, on the device:
 * forces on entry, `equilibrate` constrained steps with the velocities scaled
 * toward `temperature` (T = 2 KE / dof) and re-constrained every
 * `rescale_every` steps (:188-200), then `production` NVE steps whose
 * temperatures are averaged into *mean_temperature (nullable, :207-211) while
 * the oxygens (atoms 0, 3, 6, ...) are accumulated into `rdf` every
 * `sample_every` steps (:212-215).  `integ` is a ConstrainedVelocityVerlet
 * (md_integrator_create_rattle); the system is O, H, H triples.  One host
 * synchronisation at the end; the histogram is read when rdf is queried. */
MD_API int md_water_rdf_run(md_integrator* integ, md_system* sys, md_ewald* ff, md_rdf* rdf,
                            double temperature, int64_t dof, int64_t equilibrate,
                            int64_t rescale_every, int64_t production, int64_t sample_every,
                            double* mean_temperature);

/* Mean-squared displacement, analyze/msd.hpp:19-42 (Msd(natoms, maxLag)).
 * md_msd_push (msd.cpp:66-96) unwraps incrementally with the minimum image of
 * each step and adds |u_i(t) - u_i(t - lag)|^2 over atoms for every available lag;
 * the ring of maxLag + 1 frames lives on the device (24 bytes per atom per frame).
 * The per-lag sum over atoms is a fixed-order tree sum (the reference sums in atom
 * order), so values agree with the reference to ~1e-13 relative.  The system must
 * have natoms atoms (MD_ERR_INVALID_ARGUMENT otherwise).  md_msd_values writes
 * maxLag + 1 doubles (Msd::msd, msd.cpp:98-106); md_msd_diffusion is
 * Msd::diffusionCoefficient (msd.cpp:108-136). */
MD_API int md_msd_create(md_context* ctx, int64_t natoms, int64_t max_lag, md_msd** out);
MD_API int md_msd_destroy(md_msd* msd);
MD_API int md_msd_push(md_msd* msd, md_system* sys);
MD_API int md_msd_values(const md_msd* msd, double* out);
MD_API int md_msd_diffusion(const md_msd* msd, double dt, int64_t fit_from, int64_t fit_to,
                            double* d);

/* Velocity autocorrelation, analyze/vacf.hpp:151-174 (Vacf(natoms, maxLag)):
 * md_vacf_push as vacf.cpp:195-216 (v_i(t) . v_i(t - lag), same sums as MSD),
 * md_vacf_values(normalised = 1: Vacf::vacf, vacf.cpp:228-239; 0: the
 * unnormalised means), md_vacf_diffusion the Green-Kubo integral
 * (vacf.cpp:241-261). */
MD_API int md_vacf_create(md_context* ctx, int64_t natoms, int64_t max_lag, md_vacf** out);
MD_API int md_vacf_destroy(md_vacf* vacf);
MD_API int md_vacf_push(md_vacf* vacf, md_system* sys);
MD_API int md_vacf_values(const md_vacf* vacf, int normalised, double* out);
MD_API int md_vacf_diffusion(const md_vacf* vacf, double dt, double* d);

/* ----------------------------------------------------------------- formats */
/* moldyn_run's thermo CSV (apps/moldyn_run.cpp:229-245, 600-617): opens path and
 * writes the header -- "# command", "# git_sha" and "# host" carry the caller's
 * strings (revision/host NULL: "unknown"), the units, truncation and
 * temperature_dof lines -- and the column names.  md_thermo_csv_append writes one
 * row per thermo row of md_run_lj (4 doubles: pair energy, virial, kinetic
 * energy, conserved), as StepSampler::record (moldyn_run.cpp:497-511): step =
 * first_step + k * step_stride, time = step * dt, potential energy with the tail
 * correction, temperature 2 KE / dof, pressure rho T + W / (3V) + P_LRC, numbers
 * at std::setprecision(10).  MD_ERR_RUNTIME when the file cannot be written. */
MD_API int md_thermo_csv_open(const char* path, const char* command_line, const char* revision,
                              const char* host, int truncation, int64_t dof_langevin,
                              int64_t dof_nve, md_thermo_csv** out);
MD_API int md_thermo_csv_append(md_thermo_csv* csv, const md_lj* lj, int64_t n,
                                const double box[3], int64_t first_step, int64_t step_stride,
                                double dt, const char* phase, int64_t dof, const double* rows,
                                int64_t count);
MD_API int md_thermo_csv_close(md_thermo_csv* csv);
/* One XYZ trajectory frame appended to path (moldyn_run.cpp:519-533): the atom
 * count, the "step= time= phase= git_sha= host= command=" comment line and one
 * "Ar x y z" line per atom in original order, default stream precision. */
MD_API int md_xyz_append(const char* path, md_system* sys, int64_t step, double time,
                         const char* phase, const char* revision, const char* host,
                         const char* command_line);
/* Restartable binary checkpoint (no reference counterpart): every per-atom field
 * in original order, molecule ids, the box, and -- when integ is given -- the
 * integrator's parameters, step counter (BAOAB's noise stream) and chain state,
 * with a checksum.  md_checkpoint_load creates the system on ctx and, when integ
 * is given, restores it into an integrator of the same kind (MD_ERR_INVALID_ARGUMENT
 * for another kind, a damaged or foreign file).  A run continued from the loaded
 * state after a fresh Verlet build equals the saved run continued after one. */
MD_API int md_checkpoint_save(md_system* sys, const md_integrator* integ, const char* path);
MD_API int md_checkpoint_load(md_context* ctx, const char* path, md_system** sys,
                              md_integrator* integ);

#ifdef __cplusplus
}
#endif

#endif /* MOLDYN_B200_H */
