/*
 * md_oracle.h -- CPU restatement of moldyn's force / neighbour / integrator path.
 *
 * TEST INFRASTRUCTURE, NOT PRODUCT CODE.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline legs load this library, and only as the checker.  The
 * product (moleculardynamics_b200) never links or calls it.
 *
 * Every function restates the reference algorithm operation-for-operation (same
 * operand order, no FMA contraction except where the reference calls std::fma),
 * so that on the same libm it reproduces the reference bit-for-bit.  That claim is
 * pinned by tests/test_oracle.py against the reference itself, compiled from its
 * own sources into oracle/_ref/ (see oracle/Makefile), and against the NIST
 * published values the reference's own tests hold.
 *
 * All arrays are structure-of-arrays in the caller's atom order; indices are
 * int64_t.  Return codes: 0 = ok, <0 = error (see each function).
 */
#ifndef MD_ORACLE_H
#define MD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- core/box.cpp:12-33 ------------------------------------------------ */
double orc_fold(double value, double length);

/* ---- forcefield/lennard_jones.cpp:32-48 (ctor) ------------------------- */
typedef struct {
    double sigma, epsilon, cutoff;
    int truncation;        /* 0 = Truncated, 1 = LinearForceShift */
    double u_at_cutoff;    /* u_LJ(rc) */
    double dudr_at_cutoff; /* du_LJ/dr at rc */
} orc_lj;

void orc_lj_init(orc_lj* lj, double sigma, double epsilon, double cutoff, int truncation);

/* Pair sources for orc_lj_compute (lennard_jones.cpp:50-119). */
enum { ORC_SRC_BRUTE = 0, ORC_SRC_CELLS = 1, ORC_SRC_PAIRS = 2 };

/* Pair sum over the chosen pair source.  accumulate_forces != 0 zeroes fx/fy/fz
 * first and accumulates (computeForces); 0 leaves them untouched
 * (computeEnergyVirial).  For ORC_SRC_CELLS the cell list is built at `cutoff`
 * itself (CellList(box, lj.cutoff)); returns -2 if it is not usable, the
 * reference's std::invalid_argument.  For ORC_SRC_PAIRS (pi, pj, npairs) is the
 * pair list in traversal order. */
int orc_lj_compute(const orc_lj* lj, int64_t n, const double box[3],
                   const double* x, const double* y, const double* z, int source,
                   const int64_t* pi, const int64_t* pj, int64_t npairs,
                   int accumulate_forces, double* fx, double* fy, double* fz,
                   double* energy, double* virial);

/* lennard_jones.cpp:121-151 */
double orc_lj_lrc_energy(const orc_lj* lj, int64_t n, const double box[3]);
double orc_lj_lrc_pressure(const orc_lj* lj, int64_t n, const double box[3]);

/* ---- neighbor/cell_list.cpp:8-53 ---------------------------------------- */
void orc_cells_dims(const double box[3], double cutoff, int dims[3]);
int orc_cells_usable(const int dims[3]);
/* Candidate pairs (i<j) in the reference's forEachPair traversal order
 * (cell_list.hpp:55-108).  Writes at most cap pairs; returns the total count. */
int64_t orc_cells_pairs(int64_t n, const double box[3], const double* x, const double* y,
                        const double* z, double cutoff, int64_t* pi, int64_t* pj, int64_t cap);

/* ---- neighbor/verlet_list.cpp:8-69 -------------------------------------- */
/* Pairs (i<j) with min-image r^2 < (cutoff+skin)^2, in the reference's order
 * (cell traversal if usable, else the brute i<j scan).  Returns the count. */
int64_t orc_verlet_build(int64_t n, const double box[3], const double* x, const double* y,
                         const double* z, double cutoff, double skin, int64_t* pi, int64_t* pj,
                         int64_t cap);
/* Sum of the two largest min-image displacements since (rx,ry,rz) > skin. */
int orc_verlet_needs_rebuild(int64_t n, const double box[3], const double* x, const double* y,
                             const double* z, const double* rx, const double* ry,
                             const double* rz, double skin);
/* The two largest displacements themselves (diagnostics). */
void orc_verlet_top2(int64_t n, const double box[3], const double* x, const double* y,
                     const double* z, const double* rx, const double* ry, const double* rz,
                     double* largest, double* second);

/* ---- util/random.hpp:37-76 ---------------------------------------------- */
typedef struct {
    uint64_t mt[312];
    int index;
    double spare;
    int have_spare;
} orc_rng;

void orc_rng_seed(orc_rng* rng, uint64_t seed);
uint64_t orc_rng_next_u64(orc_rng* rng);
double orc_rng_uniform(orc_rng* rng);
double orc_rng_normal(orc_rng* rng);
/* Fills out[0..count) with successive normal() draws. */
void orc_rng_normals(orc_rng* rng, double* out, int64_t count);

/* ---- util/lattice.cpp:15-64 ------------------------------------------- */
/* Writes 4*cells^3 atoms (caller allocates) and the cubic box length. */
int orc_fcc_lattice(int cells, double density, double temperature, uint64_t seed, double* x,
                    double* y, double* z, double* vx, double* vy, double* vz, double* mass,
                    double box[3]);

/* ---- core/system.cpp:124-164 -------------------------------------------- */
double orc_kinetic_energy(int64_t n, const double* vx, const double* vy, const double* vz,
                          const double* mass);
void orc_remove_com_motion(int64_t n, double* vx, double* vy, double* vz, const double* mass);

/* ---- integrate/velocity_verlet.hpp:48-74, langevin.hpp:36-88 ------------- */
/* The per-atom parts of the steps, so a driver can interleave its own force
 * call exactly where the reference does. */
void orc_half_kick(int64_t n, double dt, const double* mass, const double* fx, const double* fy,
                   const double* fz, double* vx, double* vy, double* vz);
void orc_drift_wrap(int64_t n, const double box[3], double dt, const double* vx,
                    const double* vy, const double* vz, double* x, double* y, double* z);
/* BAOAB O-step: v = c1 v + c2 sqrt(T/m) xi, xi drawn x,y,z per atom from rng. */
void orc_baoab_o(int64_t n, double dt, double friction, double temperature, const double* mass,
                 orc_rng* rng, double* vx, double* vy, double* vz);
/* The same O-step with caller-supplied normals xi[3*i + {0,1,2}]. */
void orc_baoab_o_noise(int64_t n, double dt, double friction, double temperature,
                       const double* mass, const double* xi, double* vx, double* vy,
                       double* vz);

/* ---- integrate/nose_hoover.{hpp,cpp} ------------------------------------- */
#define ORC_NHC_MAX 16
typedef struct {
    double dt, temperature, tau;
    int chain_length;
    int64_t dof;
    double Q[ORC_NHC_MAX], xi[ORC_NHC_MAX], pxi[ORC_NHC_MAX];
} orc_nhc;

int orc_nhc_init(orc_nhc* c, double dt, double temperature, double tau, int chain_length,
                 int64_t dof);
/* integrateChain(delta) on the given velocities (nose_hoover.cpp:59-124). */
void orc_nhc_chain(orc_nhc* c, int64_t n, const double* mass, double* vx, double* vy, double* vz,
                   double delta);
double orc_nhc_conserved(const orc_nhc* c);

/* ---- A complete moldyn_run-style LJ simulation state --------------------- */
/* System + LennardJones + VerletList + integrator, stepping exactly as
 * apps/moldyn_run.cpp:581-737 does (ForceFn = rebuildIfNeeded + computeForces). */
typedef struct orc_sim orc_sim;
orc_sim* orc_sim_create(int64_t n, const double box[3], const double* x, const double* y,
                        const double* z, const double* vx, const double* vy, const double* vz,
                        const double* mass, double sigma, double epsilon, double cutoff,
                        int truncation, double skin);
void orc_sim_destroy(orc_sim* s);
/* Calls the force function once (the "prime" before the first step). */
double orc_sim_prime(orc_sim* s);
/* kind: 0 velocity-Verlet, 1 BAOAB (rng seeded by orc_sim_set_langevin), 2 NHC
 * (configured by orc_sim_set_nhc).  Runs `steps` steps. */
int orc_sim_run(orc_sim* s, int kind, int64_t steps);
void orc_sim_set_langevin(orc_sim* s, double friction, double temperature, uint64_t seed);
int orc_sim_set_nhc(orc_sim* s, double temperature, double tau, int chain_length, int64_t dof);
void orc_sim_set_dt(orc_sim* s, double dt);
void orc_sim_get(const orc_sim* s, double* x, double* y, double* z, double* vx, double* vy,
                 double* vz, double* fx, double* fy, double* fz);
void orc_sim_set_state(orc_sim* s, const double* x, const double* y, const double* z,
                       const double* vx, const double* vy, const double* vz, const double* fx,
                       const double* fy, const double* fz);
double orc_sim_energy(const orc_sim* s);
double orc_sim_virial(const orc_sim* s);
int64_t orc_sim_rebuild_count(const orc_sim* s);
double orc_sim_nhc_conserved(const orc_sim* s);
void orc_sim_remove_com(orc_sim* s);

/* ---- forcefield/ewald.cpp:17-188 ---------------------------------------- */
double orc_coulomb_prefactor(void);
typedef struct {
    double real, reciprocal, self, intra;
} orc_ewald_terms;
/* alpha <= 0 selects the reference's 5.6 / min(L).  mode: 0 energies only,
 * 1 zero forces then accumulate, 2 accumulate onto existing forces.
 * virial (may be NULL) receives the atomic virial sum w(r) of the real and
 * intramolecular terms plus the reciprocal-space virial; it has no reference
 * counterpart (the reference computes no Ewald virial). */
int orc_ewald_compute(int64_t n, const double box[3], const double* x, const double* y,
                      const double* z, const double* q, const int64_t* mol, double cutoff,
                      int kmax, double alpha, int mode, double* fx, double* fy, double* fz,
                      orc_ewald_terms* terms, double* virial);

/* ---- forcefield/spce_forcefield.cpp:26-48 ------------------------------- */
/* Sites are O,H,H triples.  Returns the total potential energy; forces are
 * zeroed and accumulated when fx != NULL.  Parameters as SpceParameters
 * (spce.hpp:16-24) with the given cutoff / kmax / alpha (alpha <= 0 ->
 * 5.6/min L). */
double orc_spce_compute(int64_t n, const double box[3], const double* x, const double* y,
                        const double* z, const double* q, const int64_t* mol, double sigma_o,
                        double epsilon_o, double cutoff, int kmax, double alpha, double* fx,
                        double* fy, double* fz);

/* ---- constrain/rigid_water.cpp:30-161 ------------------------------------ */
typedef struct {
    double oh, hh, tolerance;
    int max_iterations;
} orc_rigid_water;
int orc_rigid_water_init(orc_rigid_water* rw, double oh, double hoh_degrees, double tolerance,
                         int max_iterations);
/* Return the iteration count, or -1 (not converged), -2 (singular), -3 (bad n). */
int orc_rigid_water_positions(const orc_rigid_water* rw, int64_t n, const double box[3],
                              const double* mass, double* x, double* y, double* z,
                              const double* rx, const double* ry, const double* rz);
int orc_rigid_water_velocities(const orc_rigid_water* rw, int64_t n, const double box[3],
                               const double* mass, const double* x, const double* y,
                               const double* z, double* vx, double* vy, double* vz);

/* ---- analyze/ ------------------------------------------------------------ */
/* rdf.cpp:55-82: one frame's pairs i < j into hist (bins doubles, accumulated).
 * Returns -1 (std::invalid_argument) when rmax exceeds half the smallest box
 * length, else 0. */
int orc_rdf_accumulate(int64_t n, const double box[3], const double* x, const double* y,
                       const double* z, double rmax, int64_t bins, double* hist);
/* rdf.cpp:92-107: g(r) from the accumulated histogram. */
void orc_rdf_g(const double* hist, int64_t bins, double rmax, int64_t frames, int64_t natoms,
               double sum_rho, double* g);
/* msd.cpp:66-106 over a whole trajectory: pos holds frames x (x[n] | y[n] | z[n])
 * wrapped positions in atom order; out receives max_lag + 1 values. */
void orc_msd(int64_t frames, int64_t n, const double box[3], const double* pos,
             int64_t max_lag, double* out);
/* vacf.cpp:195-226: vel as pos above; out receives the max_lag + 1 unnormalised
 * means. */
void orc_vacf(int64_t frames, int64_t n, const double* vel, int64_t max_lag, double* out);

#ifdef __cplusplus
}
#endif

#endif /* MD_ORACLE_H */
