/*
 * md_oracle.c -- CPU restatement of moldyn's force / neighbour / integrator path.
 *
 * TEST INFRASTRUCTURE, NOT PRODUCT CODE: only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline legs load it, as the checker.  Built with
 * -ffp-contract=off so every a*b+c below rounds twice, as the reference's ISO C++
 * build (CMAKE_CXX_EXTENSIONS OFF, baseline x86-64) does; fma() appears only where
 * the reference calls std::fma.
 *
 * Reference citations are path:line inside the moldyn project.
 */
#include "md_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static const double kPi = 3.14159265358979323846;

/* core/box.cpp:12-15: value - L * floor(value / L + 0.5). */
double orc_fold(double value, double length) {
    return value - length * floor(value / length + 0.5);
}

/* core/vec3.hpp:59-65: norm2 = x*x + y*y + z*z, left to right. */
static inline double norm2(double x, double y, double z) { return x * x + y * y + z * z; }

/* forcefield/lennard_jones.cpp:32-48 */
void orc_lj_init(orc_lj* lj, double sigma, double epsilon, double cutoff, int truncation) {
    lj->sigma = sigma;
    lj->epsilon = epsilon;
    lj->cutoff = cutoff;
    lj->truncation = truncation;
    const double sig2 = sigma * sigma;
    const double rc2 = cutoff * cutoff;
    const double s2 = sig2 / rc2;
    const double s6 = s2 * s2 * s2;
    lj->u_at_cutoff = 4.0 * epsilon * (s6 * s6 - s6);
    const double w_at_cutoff = 24.0 * epsilon * (2.0 * s6 * s6 - s6);
    lj->dudr_at_cutoff = -w_at_cutoff / cutoff;
}

/* ---- neighbor/cell_list.cpp ---------------------------------------------- */
void orc_cells_dims(const double box[3], double cutoff, int dims[3]) {
    /* cell_list.cpp:8-14 */
    for (int d = 0; d < 3; ++d) {
        int v = (int)floor(box[d] / cutoff);
        dims[d] = v < 1 ? 1 : v;
    }
}

int orc_cells_usable(const int dims[3]) {
    /* cell_list.cpp:51-53 */
    return dims[0] >= 3 && dims[1] >= 3 && dims[2] >= 3;
}

typedef struct {
    int nx, ny, nz;
    int* head;
    int* next;
} cell_list;

static int clamp_index(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }
static int wrap_index(int v, int n) {
    const int m = v % n;
    return m < 0 ? m + n : m;
}

/* cell_list.cpp:16-43 -- head insertion, so each chain lists descending indices. */
static int cell_list_build(cell_list* cl, int64_t n, const double box[3], const double* x,
                           const double* y, const double* z, double cutoff) {
    int dims[3];
    orc_cells_dims(box, cutoff, dims);
    cl->nx = dims[0];
    cl->ny = dims[1];
    cl->nz = dims[2];
    const size_t ncells = (size_t)cl->nx * (size_t)cl->ny * (size_t)cl->nz;
    cl->head = (int*)malloc(ncells * sizeof(int));
    cl->next = (int*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int));
    if (!cl->head || !cl->next) return -1;
    for (size_t c = 0; c < ncells; ++c) cl->head[c] = -1;
    for (int64_t i = 0; i < n; ++i) cl->next[i] = -1;
    const double wx = box[0] / (double)cl->nx;
    const double wy = box[1] / (double)cl->ny;
    const double wz = box[2] / (double)cl->nz;
    for (int64_t i = 0; i < n; ++i) {
        const double rx = orc_fold(x[i], box[0]);
        const double ry = orc_fold(y[i], box[1]);
        const double rz = orc_fold(z[i], box[2]);
        int ix = (int)floor((rx + 0.5 * box[0]) / wx);
        int iy = (int)floor((ry + 0.5 * box[1]) / wy);
        int iz = (int)floor((rz + 0.5 * box[2]) / wz);
        ix = clamp_index(ix, cl->nx);
        iy = clamp_index(iy, cl->ny);
        iz = clamp_index(iz, cl->nz);
        const int cell = ix + cl->nx * (iy + cl->ny * iz);
        cl->next[i] = cl->head[cell];
        cl->head[cell] = (int)i;
    }
    return 0;
}

static void cell_list_free(cell_list* cl) {
    free(cl->head);
    free(cl->next);
}

typedef void (*pair_fn)(void* ctx, int64_t i, int64_t j);

/* cell_list.hpp:55-108: same cell, then the 13 forward neighbours, i<j normalised. */
static void cell_list_for_each_pair(const cell_list* cl, pair_fn fn, void* ctx) {
    static const int kOffsets[13][3] = {
        {1, 0, 0}, {1, 1, 0},  {0, 1, 0},  {-1, 1, 0}, {0, 0, 1},  {1, 0, 1},   {-1, 0, 1},
        {0, 1, 1}, {0, -1, 1}, {1, 1, 1},  {1, -1, 1}, {-1, 1, 1}, {-1, -1, 1},
    };
    for (int ix = 0; ix < cl->nx; ++ix) {
        for (int iy = 0; iy < cl->ny; ++iy) {
            for (int iz = 0; iz < cl->nz; ++iz) {
                const int cell = ix + cl->nx * (iy + cl->ny * iz);
                for (int i = cl->head[cell]; i != -1; i = cl->next[i]) {
                    for (int j = cl->next[i]; j != -1; j = cl->next[j]) {
                        if (i < j) fn(ctx, i, j);
                        else fn(ctx, j, i);
                    }
                }
                for (int o = 0; o < 13; ++o) {
                    const int jx = wrap_index(ix + kOffsets[o][0], cl->nx);
                    const int jy = wrap_index(iy + kOffsets[o][1], cl->ny);
                    const int jz = wrap_index(iz + kOffsets[o][2], cl->nz);
                    const int nb = jx + cl->nx * (jy + cl->ny * jz);
                    for (int i = cl->head[cell]; i != -1; i = cl->next[i]) {
                        for (int j = cl->head[nb]; j != -1; j = cl->next[j]) {
                            if (i < j) fn(ctx, i, j);
                            else fn(ctx, j, i);
                        }
                    }
                }
            }
        }
    }
}

typedef struct {
    int64_t* pi;
    int64_t* pj;
    int64_t cap;
    int64_t count;
} pair_sink;

static void sink_pair(void* ctx, int64_t i, int64_t j) {
    pair_sink* s = (pair_sink*)ctx;
    if (s->count < s->cap) {
        s->pi[s->count] = i;
        s->pj[s->count] = j;
    }
    ++s->count;
}

int64_t orc_cells_pairs(int64_t n, const double box[3], const double* x, const double* y,
                        const double* z, double cutoff, int64_t* pi, int64_t* pj, int64_t cap) {
    cell_list cl;
    if (cell_list_build(&cl, n, box, x, y, z, cutoff) != 0) return -1;
    pair_sink sink = {pi, pj, cap, 0};
    cell_list_for_each_pair(&cl, sink_pair, &sink);
    cell_list_free(&cl);
    return sink.count;
}

/* ---- neighbor/verlet_list.cpp:8-42 ---------------------------------------- */
typedef struct {
    pair_sink sink;
    const double* x;
    const double* y;
    const double* z;
    const double* box;
    double list_cutoff2;
} verlet_ctx;

static void verlet_pair(void* ctx, int64_t i, int64_t j) {
    verlet_ctx* v = (verlet_ctx*)ctx;
    const double dx = orc_fold(v->x[i] - v->x[j], v->box[0]);
    const double dy = orc_fold(v->y[i] - v->y[j], v->box[1]);
    const double dz = orc_fold(v->z[i] - v->z[j], v->box[2]);
    if (norm2(dx, dy, dz) < v->list_cutoff2) sink_pair(&v->sink, i, j);
}

int64_t orc_verlet_build(int64_t n, const double box[3], const double* x, const double* y,
                         const double* z, double cutoff, double skin, int64_t* pi, int64_t* pj,
                         int64_t cap) {
    verlet_ctx v = {{pi, pj, cap, 0}, x, y, z, box, (cutoff + skin) * (cutoff + skin)};
    int dims[3];
    orc_cells_dims(box, cutoff + skin, dims);
    if (orc_cells_usable(dims)) {
        cell_list cl;
        if (cell_list_build(&cl, n, box, x, y, z, cutoff + skin) != 0) return -1;
        cell_list_for_each_pair(&cl, verlet_pair, &v);
        cell_list_free(&cl);
    } else {
        for (int64_t i = 0; i < n; ++i)
            for (int64_t j = i + 1; j < n; ++j) verlet_pair(&v, i, j);
    }
    return v.sink.count;
}

/* verlet_list.cpp:44-63 */
void orc_verlet_top2(int64_t n, const double box[3], const double* x, const double* y,
                     const double* z, const double* rx, const double* ry, const double* rz,
                     double* largest_out, double* second_out) {
    double largest = 0.0, second = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double dx = orc_fold(x[i] - rx[i], box[0]);
        const double dy = orc_fold(y[i] - ry[i], box[1]);
        const double dz = orc_fold(z[i] - rz[i], box[2]);
        const double d = sqrt(norm2(dx, dy, dz));
        if (d > largest) {
            second = largest;
            largest = d;
        } else if (d > second) {
            second = d;
        }
    }
    *largest_out = largest;
    *second_out = second;
}

int orc_verlet_needs_rebuild(int64_t n, const double box[3], const double* x, const double* y,
                             const double* z, const double* rx, const double* ry,
                             const double* rz, double skin) {
    double a, b;
    orc_verlet_top2(n, box, x, y, z, rx, ry, rz, &a, &b);
    return (a + b) > skin;
}

/* ---- forcefield/lennard_jones.cpp:50-88 ------------------------------------ */
typedef struct {
    const orc_lj* lj;
    const double* x;
    const double* y;
    const double* z;
    const double* box;
    double sig2, rc2;
    int accumulate;
    double* fx;
    double* fy;
    double* fz;
    double energy, virial;
} lj_ctx;

static void lj_pair(void* ctx, int64_t i, int64_t j) {
    lj_ctx* c = (lj_ctx*)ctx;
    const double dx = orc_fold(c->x[i] - c->x[j], c->box[0]);
    const double dy = orc_fold(c->y[i] - c->y[j], c->box[1]);
    const double dz = orc_fold(c->z[i] - c->z[j], c->box[2]);
    const double r2 = norm2(dx, dy, dz);
    if (!(r2 < c->rc2)) return;
    const double eps = c->lj->epsilon;
    const double s2 = c->sig2 / r2;
    const double s6 = s2 * s2 * s2;
    const double uLJ = 4.0 * eps * (s6 * s6 - s6);
    const double wLJ = 24.0 * eps * (2.0 * s6 * s6 - s6);
    double u = uLJ, w = wLJ;
    if (c->lj->truncation == 1) {
        const double r = sqrt(r2);
        u = uLJ - c->lj->u_at_cutoff - (r - c->lj->cutoff) * c->lj->dudr_at_cutoff;
        w = wLJ + r * c->lj->dudr_at_cutoff;
    }
    c->energy += u;
    c->virial += w;
    if (c->accumulate) {
        /* f = (w / r2) * d; atom i gains +f, atom j gains -1.0 * f. */
        const double s = w / r2;
        const double fxv = dx * s, fyv = dy * s, fzv = dz * s;
        c->fx[i] += fxv;
        c->fy[i] += fyv;
        c->fz[i] += fzv;
        c->fx[j] += fxv * -1.0;
        c->fy[j] += fyv * -1.0;
        c->fz[j] += fzv * -1.0;
    }
}

int orc_lj_compute(const orc_lj* lj, int64_t n, const double box[3], const double* x,
                   const double* y, const double* z, int source, const int64_t* pi,
                   const int64_t* pj, int64_t npairs, int accumulate_forces, double* fx,
                   double* fy, double* fz, double* energy, double* virial) {
    lj_ctx c;
    c.lj = lj;
    c.x = x;
    c.y = y;
    c.z = z;
    c.box = box;
    c.sig2 = lj->sigma * lj->sigma;
    c.rc2 = lj->cutoff * lj->cutoff;
    c.accumulate = accumulate_forces;
    c.fx = fx;
    c.fy = fy;
    c.fz = fz;
    c.energy = 0.0;
    c.virial = 0.0;
    if (source == ORC_SRC_CELLS) {
        int dims[3];
        orc_cells_dims(box, lj->cutoff, dims);
        if (!orc_cells_usable(dims)) return -2; /* lennard_jones.cpp:107-111 */
    }
    if (accumulate_forces) {
        for (int64_t i = 0; i < n; ++i) fx[i] = fy[i] = fz[i] = 0.0;
    }
    if (source == ORC_SRC_BRUTE) {
        for (int64_t i = 0; i < n; ++i)
            for (int64_t j = i + 1; j < n; ++j) lj_pair(&c, i, j);
    } else if (source == ORC_SRC_CELLS) {
        cell_list cl;
        if (cell_list_build(&cl, n, box, x, y, z, lj->cutoff) != 0) return -1;
        cell_list_for_each_pair(&cl, lj_pair, &c);
        cell_list_free(&cl);
    } else {
        for (int64_t k = 0; k < npairs; ++k) lj_pair(&c, pi[k], pj[k]);
    }
    *energy = c.energy;
    *virial = c.virial;
    return 0;
}

/* lennard_jones.cpp:121-135 */
double orc_lj_lrc_energy(const orc_lj* lj, int64_t n, const double box[3]) {
    if (lj->truncation == 1) return 0.0;
    const double nd = (double)n;
    const double rho = nd / (box[0] * box[1] * box[2]);
    const double sr = lj->sigma / lj->cutoff;
    const double sr3 = sr * sr * sr;
    const double sr9 = sr3 * sr3 * sr3;
    const double sig3 = lj->sigma * lj->sigma * lj->sigma;
    return (8.0 / 3.0) * kPi * nd * rho * lj->epsilon * sig3 * ((1.0 / 3.0) * sr9 - sr3);
}

/* lennard_jones.cpp:137-151 */
double orc_lj_lrc_pressure(const orc_lj* lj, int64_t n, const double box[3]) {
    if (lj->truncation == 1) return 0.0;
    const double nd = (double)n;
    const double rho = nd / (box[0] * box[1] * box[2]);
    const double sr = lj->sigma / lj->cutoff;
    const double sr3 = sr * sr * sr;
    const double sr9 = sr3 * sr3 * sr3;
    const double sig3 = lj->sigma * lj->sigma * lj->sigma;
    return (16.0 / 3.0) * kPi * rho * rho * lj->epsilon * sig3 * ((2.0 / 3.0) * sr9 - sr3);
}

/* ---- util/random.hpp:37-76 -- std::mt19937_64 (Matsumoto & Nishimura 2000) --
 * plus libstdc++'s generate_canonical<double,53> for one 64-bit draw:
 * (double)u / 2^64, clamped below 1.  Rng::uniform returns 1 - that. */
void orc_rng_seed(orc_rng* rng, uint64_t seed) {
    rng->mt[0] = seed;
    for (int i = 1; i < 312; ++i) {
        const uint64_t prev = rng->mt[i - 1];
        rng->mt[i] = 6364136223846793005ULL * (prev ^ (prev >> 62)) + (uint64_t)i;
    }
    rng->index = 312;
    rng->spare = 0.0;
    rng->have_spare = 0;
}

uint64_t orc_rng_next_u64(orc_rng* rng) {
    static const uint64_t kUpper = 0xFFFFFFFF80000000ULL, kLower = 0x7FFFFFFFULL;
    if (rng->index >= 312) {
        for (int i = 0; i < 312; ++i) {
            const uint64_t y = (rng->mt[i] & kUpper) | (rng->mt[(i + 1) % 312] & kLower);
            uint64_t v = rng->mt[(i + 156) % 312] ^ (y >> 1);
            if (y & 1ULL) v ^= 0xB5026F5AA96619E9ULL;
            rng->mt[i] = v;
        }
        rng->index = 0;
    }
    uint64_t z = rng->mt[rng->index++];
    z ^= (z >> 29) & 0x5555555555555555ULL;
    z ^= (z << 17) & 0x71D67FFFEDA60000ULL;
    z ^= (z << 37) & 0xFFF7EEE000000000ULL;
    z ^= z >> 43;
    return z;
}

double orc_rng_uniform(orc_rng* rng) {
    const double sum = (double)orc_rng_next_u64(rng);
    double ret = sum / 18446744073709551616.0; /* 2^64 */
    if (ret >= 1.0) ret = nextafter(1.0, 0.0);
    ret = ret * (1.0 - 0.0) + 0.0;
    return 1.0 - ret;
}

/* random.hpp:52-69: Marsaglia polar method with one cached spare. */
double orc_rng_normal(orc_rng* rng) {
    if (rng->have_spare) {
        rng->have_spare = 0;
        return rng->spare;
    }
    double u, v, s;
    do {
        u = 2.0 * orc_rng_uniform(rng) - 1.0;
        v = 2.0 * orc_rng_uniform(rng) - 1.0;
        s = u * u + v * v;
    } while (s >= 1.0 || s == 0.0);
    const double multiplier = sqrt(-2.0 * log(s) / s);
    rng->spare = v * multiplier;
    rng->have_spare = 1;
    return u * multiplier;
}

void orc_rng_normals(orc_rng* rng, double* out, int64_t count) {
    for (int64_t i = 0; i < count; ++i) out[i] = orc_rng_normal(rng);
}

/* ---- core/system.cpp:124-164 ---------------------------------------------- */
double orc_kinetic_energy(int64_t n, const double* vx, const double* vy, const double* vz,
                          const double* mass) {
    double ke = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double v2 = vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i];
        ke += 0.5 * mass[i] * v2;
    }
    return ke;
}

void orc_remove_com_motion(int64_t n, double* vx, double* vy, double* vz, const double* mass) {
    double total_mass = 0.0;
    for (int64_t i = 0; i < n; ++i) total_mass += mass[i];
    if (total_mass == 0.0) return;
    double px = 0.0, py = 0.0, pz = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        px += mass[i] * vx[i];
        py += mass[i] * vy[i];
        pz += mass[i] * vz[i];
    }
    const double cx = px / total_mass, cy = py / total_mass, cz = pz / total_mass;
    for (int64_t i = 0; i < n; ++i) {
        vx[i] -= cx;
        vy[i] -= cy;
        vz[i] -= cz;
    }
}

/* ---- util/lattice.cpp:15-64 ---------------------------------------------- */
int orc_fcc_lattice(int cells, double density, double temperature, uint64_t seed, double* x,
                    double* y, double* z, double* vx, double* vy, double* vz, double* mass,
                    double box[3]) {
    const double cells_d = (double)cells;
    const int n = 4 * cells * cells * cells;
    const double length = cbrt((double)n / density);
    const double a = length / cells_d;
    static const double basis[4][3] = {
        {0.0, 0.0, 0.0}, {0.0, 0.5, 0.5}, {0.5, 0.0, 0.5}, {0.5, 0.5, 0.0}};
    box[0] = box[1] = box[2] = length;
    orc_rng rng;
    orc_rng_seed(&rng, seed);
    const double sigma_v = sqrt(temperature / 1.0);
    int64_t k = 0;
    for (int ix = 0; ix < cells; ++ix) {
        for (int iy = 0; iy < cells; ++iy) {
            for (int iz = 0; iz < cells; ++iz) {
                for (int b = 0; b < 4; ++b) {
                    const double rx = a * ((double)ix + basis[b][0]) - 0.5 * length;
                    const double ry = a * ((double)iy + basis[b][1]) - 0.5 * length;
                    const double rz = a * ((double)iz + basis[b][2]) - 0.5 * length;
                    x[k] = orc_fold(rx, length);
                    y[k] = orc_fold(ry, length);
                    z[k] = orc_fold(rz, length);
                    vx[k] = sigma_v * orc_rng_normal(&rng);
                    vy[k] = sigma_v * orc_rng_normal(&rng);
                    vz[k] = sigma_v * orc_rng_normal(&rng);
                    mass[k] = 1.0;
                    ++k;
                }
            }
        }
    }
    orc_remove_com_motion(n, vx, vy, vz, mass);
    return n;
}

/* ---- integrate/velocity_verlet.hpp:48-74 --------------------------------- */
void orc_half_kick(int64_t n, double dt, const double* mass, const double* fx, const double* fy,
                   const double* fz, double* vx, double* vy, double* vz) {
    const double half_dt = 0.5 * dt;
    for (int64_t i = 0; i < n; ++i) {
        const double inv_mass = 1.0 / mass[i];
        const double a = half_dt * inv_mass;
        vx[i] = fma(a, fx[i], vx[i]);
        vy[i] = fma(a, fy[i], vy[i]);
        vz[i] = fma(a, fz[i], vz[i]);
    }
}

void orc_drift_wrap(int64_t n, const double box[3], double dt, const double* vx,
                    const double* vy, const double* vz, double* x, double* y, double* z) {
    for (int64_t i = 0; i < n; ++i) {
        x[i] = orc_fold(fma(dt, vx[i], x[i]), box[0]);
        y[i] = orc_fold(fma(dt, vy[i], y[i]), box[1]);
        z[i] = orc_fold(fma(dt, vz[i], z[i]), box[2]);
    }
}

/* ---- integrate/langevin.hpp:64-72 (O step) --------------------------------- */
void orc_baoab_o_noise(int64_t n, double dt, double friction, double temperature,
                       const double* mass, const double* xi, double* vx, double* vy,
                       double* vz) {
    const double c1 = exp(-friction * dt);
    const double c2 = sqrt(1.0 - c1 * c1);
    for (int64_t i = 0; i < n; ++i) {
        const double sigma = sqrt(temperature / mass[i]);
        const double s = c2 * sigma;
        vx[i] = c1 * vx[i] + xi[3 * i + 0] * s;
        vy[i] = c1 * vy[i] + xi[3 * i + 1] * s;
        vz[i] = c1 * vz[i] + xi[3 * i + 2] * s;
    }
}

void orc_baoab_o(int64_t n, double dt, double friction, double temperature, const double* mass,
                 orc_rng* rng, double* vx, double* vy, double* vz) {
    const double c1 = exp(-friction * dt);
    const double c2 = sqrt(1.0 - c1 * c1);
    for (int64_t i = 0; i < n; ++i) {
        const double sigma = sqrt(temperature / mass[i]);
        const double s = c2 * sigma;
        const double xx = orc_rng_normal(rng);
        const double xy = orc_rng_normal(rng);
        const double xz = orc_rng_normal(rng);
        vx[i] = c1 * vx[i] + xx * s;
        vy[i] = c1 * vy[i] + xy * s;
        vz[i] = c1 * vz[i] + xz * s;
    }
}

/* ---- integrate/nose_hoover.cpp ------------------------------------------- */
int orc_nhc_init(orc_nhc* c, double dt, double temperature, double tau, int chain_length,
                 int64_t dof) {
    if (chain_length < 1 || chain_length > ORC_NHC_MAX) return -1; /* nose_hoover.cpp:36-38 */
    memset(c, 0, sizeof(*c));
    c->dt = dt;
    c->temperature = temperature;
    c->tau = tau;
    c->chain_length = chain_length;
    c->dof = dof;
    c->Q[0] = (double)dof * temperature * tau * tau;
    for (int k = 1; k < chain_length; ++k) c->Q[k] = temperature * tau * tau;
    return 0;
}

double orc_nhc_conserved(const orc_nhc* c) {
    /* nose_hoover.cpp:45-54 */
    double sum = (double)c->dof * c->temperature * c->xi[0];
    for (int k = 1; k < c->chain_length; ++k) sum += c->temperature * c->xi[k];
    for (int k = 0; k < c->chain_length; ++k) sum += 0.5 * c->pxi[k] * c->pxi[k] / c->Q[k];
    return sum;
}

static void nhc_link(orc_nhc* c, int64_t n, const double* mass, const double* vx,
                     const double* vy, const double* vz, int j, double delta2, double delta4) {
    /* nose_hoover.cpp:89-108 */
    const int has_next = j < c->chain_length - 1;
    if (has_next) c->pxi[j] *= exp(-delta4 * c->pxi[j + 1] / c->Q[j + 1]);
    double g;
    if (j == 0) {
        g = 2.0 * orc_kinetic_energy(n, vx, vy, vz, mass) - (double)c->dof * c->temperature;
    } else {
        g = c->pxi[j - 1] * c->pxi[j - 1] / c->Q[j - 1] - c->temperature;
    }
    c->pxi[j] += delta2 * g;
    if (has_next) c->pxi[j] *= exp(-delta4 * c->pxi[j + 1] / c->Q[j + 1]);
}

void orc_nhc_chain(orc_nhc* c, int64_t n, const double* mass, double* vx, double* vy, double* vz,
                   double delta) {
    /* nose_hoover.cpp:15-18 (weights), 59-124 */
    const double w1 = 1.0 / (2.0 - cbrt(2.0));
    const double weights[3] = {w1, 1.0 - 2.0 * w1, w1};
    for (int s = 0; s < 3; ++s) {
        const double d = weights[s] * delta;
        const double delta2 = 0.5 * d;
        const double delta4 = 0.25 * d;
        for (int j = c->chain_length - 1; j >= 0; --j) nhc_link(c, n, mass, vx, vy, vz, j, delta2, delta4);
        for (int k = 0; k < c->chain_length; ++k) c->xi[k] += d * c->pxi[k] / c->Q[k];
        const double factor = exp(-d * c->pxi[0] / c->Q[0]);
        for (int64_t i = 0; i < n; ++i) {
            vx[i] = vx[i] * factor;
            vy[i] = vy[i] * factor;
            vz[i] = vz[i] * factor;
        }
        for (int j = 0; j < c->chain_length; ++j) nhc_link(c, n, mass, vx, vy, vz, j, delta2, delta4);
    }
}

/* ---- moldyn_run-style simulation (apps/moldyn_run.cpp:570-737) ------------ */
struct orc_sim {
    int64_t n;
    double box[3];
    double *x, *y, *z, *vx, *vy, *vz, *fx, *fy, *fz, *m;
    orc_lj lj;
    double skin;
    /* VerletList state */
    int64_t *pi, *pj, npairs, cap;
    double *rx, *ry, *rz;
    int64_t rebuilds;
    double energy, virial, dt;
    /* thermostats */
    double friction, lt;
    orc_rng rng;
    orc_nhc nhc;
};

static int sim_build(orc_sim* s) {
    for (;;) {
        const int64_t cnt = orc_verlet_build(s->n, s->box, s->x, s->y, s->z, s->lj.cutoff, s->skin,
                                             s->pi, s->pj, s->cap);
        if (cnt < 0) return -1;
        if (cnt <= s->cap) {
            s->npairs = cnt;
            break;
        }
        free(s->pi);
        free(s->pj);
        s->cap = cnt + cnt / 4 + 16;
        s->pi = (int64_t*)malloc((size_t)s->cap * sizeof(int64_t));
        s->pj = (int64_t*)malloc((size_t)s->cap * sizeof(int64_t));
        if (!s->pi || !s->pj) return -1;
    }
    memcpy(s->rx, s->x, (size_t)s->n * sizeof(double));
    memcpy(s->ry, s->y, (size_t)s->n * sizeof(double));
    memcpy(s->rz, s->z, (size_t)s->n * sizeof(double));
    ++s->rebuilds;
    return 0;
}

orc_sim* orc_sim_create(int64_t n, const double box[3], const double* x, const double* y,
                        const double* z, const double* vx, const double* vy, const double* vz,
                        const double* mass, double sigma, double epsilon, double cutoff,
                        int truncation, double skin) {
    orc_sim* s = (orc_sim*)calloc(1, sizeof(orc_sim));
    if (!s) return NULL;
    s->n = n;
    memcpy(s->box, box, 3 * sizeof(double));
    const size_t bytes = (size_t)(n > 0 ? n : 1) * sizeof(double);
    double** arrays[] = {&s->x, &s->y, &s->z, &s->vx, &s->vy, &s->vz, &s->fx,
                         &s->fy, &s->fz, &s->m, &s->rx, &s->ry, &s->rz};
    for (size_t a = 0; a < sizeof(arrays) / sizeof(arrays[0]); ++a) {
        *arrays[a] = (double*)calloc(1, bytes);
        if (!*arrays[a]) return NULL;
    }
    memcpy(s->x, x, (size_t)n * sizeof(double));
    memcpy(s->y, y, (size_t)n * sizeof(double));
    memcpy(s->z, z, (size_t)n * sizeof(double));
    memcpy(s->vx, vx, (size_t)n * sizeof(double));
    memcpy(s->vy, vy, (size_t)n * sizeof(double));
    memcpy(s->vz, vz, (size_t)n * sizeof(double));
    memcpy(s->m, mass, (size_t)n * sizeof(double));
    orc_lj_init(&s->lj, sigma, epsilon, cutoff, truncation);
    s->skin = skin;
    s->cap = 64 * n + 16;
    s->pi = (int64_t*)malloc((size_t)s->cap * sizeof(int64_t));
    s->pj = (int64_t*)malloc((size_t)s->cap * sizeof(int64_t));
    s->dt = 0.005;
    if (!s->pi || !s->pj || sim_build(s) != 0) return NULL;
    return s;
}

void orc_sim_destroy(orc_sim* s) {
    if (!s) return;
    free(s->x); free(s->y); free(s->z); free(s->vx); free(s->vy); free(s->vz);
    free(s->fx); free(s->fy); free(s->fz); free(s->m); free(s->rx); free(s->ry); free(s->rz);
    free(s->pi); free(s->pj);
    free(s);
}

/* The ForceFn of moldyn_run.cpp:581-587. */
static double sim_forces(orc_sim* s) {
    if (orc_verlet_needs_rebuild(s->n, s->box, s->x, s->y, s->z, s->rx, s->ry, s->rz, s->skin))
        sim_build(s);
    orc_lj_compute(&s->lj, s->n, s->box, s->x, s->y, s->z, ORC_SRC_PAIRS, s->pi, s->pj, s->npairs,
                   1, s->fx, s->fy, s->fz, &s->energy, &s->virial);
    return s->energy;
}

double orc_sim_prime(orc_sim* s) { return sim_forces(s); }

void orc_sim_set_dt(orc_sim* s, double dt) { s->dt = dt; }

void orc_sim_set_langevin(orc_sim* s, double friction, double temperature, uint64_t seed) {
    s->friction = friction;
    s->lt = temperature;
    orc_rng_seed(&s->rng, seed);
}

int orc_sim_set_nhc(orc_sim* s, double temperature, double tau, int chain_length, int64_t dof) {
    return orc_nhc_init(&s->nhc, s->dt, temperature, tau, chain_length, dof);
}

static void sim_vv_core(orc_sim* s) {
    orc_half_kick(s->n, s->dt, s->m, s->fx, s->fy, s->fz, s->vx, s->vy, s->vz);
    orc_drift_wrap(s->n, s->box, s->dt, s->vx, s->vy, s->vz, s->x, s->y, s->z);
    sim_forces(s);
    orc_half_kick(s->n, s->dt, s->m, s->fx, s->fy, s->fz, s->vx, s->vy, s->vz);
}

int orc_sim_run(orc_sim* s, int kind, int64_t steps) {
    for (int64_t k = 0; k < steps; ++k) {
        if (kind == 0) {
            sim_vv_core(s);
        } else if (kind == 1) {
            /* langevin.hpp:36-88: B A O A F B */
            const double half = 0.5 * s->dt;
            orc_half_kick(s->n, s->dt, s->m, s->fx, s->fy, s->fz, s->vx, s->vy, s->vz);
            orc_drift_wrap(s->n, s->box, half, s->vx, s->vy, s->vz, s->x, s->y, s->z);
            orc_baoab_o(s->n, s->dt, s->friction, s->lt, s->m, &s->rng, s->vx, s->vy, s->vz);
            orc_drift_wrap(s->n, s->box, half, s->vx, s->vy, s->vz, s->x, s->y, s->z);
            sim_forces(s);
            orc_half_kick(s->n, s->dt, s->m, s->fx, s->fy, s->fz, s->vx, s->vy, s->vz);
        } else if (kind == 2) {
            /* nose_hoover.hpp:37-42 */
            orc_nhc_chain(&s->nhc, s->n, s->m, s->vx, s->vy, s->vz, 0.5 * s->dt);
            sim_vv_core(s);
            orc_nhc_chain(&s->nhc, s->n, s->m, s->vx, s->vy, s->vz, 0.5 * s->dt);
        } else {
            return -1;
        }
    }
    return 0;
}

void orc_sim_get(const orc_sim* s, double* x, double* y, double* z, double* vx, double* vy,
                 double* vz, double* fx, double* fy, double* fz) {
    const size_t b = (size_t)s->n * sizeof(double);
    if (x) memcpy(x, s->x, b);
    if (y) memcpy(y, s->y, b);
    if (z) memcpy(z, s->z, b);
    if (vx) memcpy(vx, s->vx, b);
    if (vy) memcpy(vy, s->vy, b);
    if (vz) memcpy(vz, s->vz, b);
    if (fx) memcpy(fx, s->fx, b);
    if (fy) memcpy(fy, s->fy, b);
    if (fz) memcpy(fz, s->fz, b);
}

void orc_sim_set_state(orc_sim* s, const double* x, const double* y, const double* z,
                       const double* vx, const double* vy, const double* vz, const double* fx,
                       const double* fy, const double* fz) {
    const size_t b = (size_t)s->n * sizeof(double);
    if (x) memcpy(s->x, x, b);
    if (y) memcpy(s->y, y, b);
    if (z) memcpy(s->z, z, b);
    if (vx) memcpy(s->vx, vx, b);
    if (vy) memcpy(s->vy, vy, b);
    if (vz) memcpy(s->vz, vz, b);
    if (fx) memcpy(s->fx, fx, b);
    if (fy) memcpy(s->fy, fy, b);
    if (fz) memcpy(s->fz, fz, b);
}

double orc_sim_energy(const orc_sim* s) { return s->energy; }
double orc_sim_virial(const orc_sim* s) { return s->virial; }
int64_t orc_sim_rebuild_count(const orc_sim* s) { return s->rebuilds; }
double orc_sim_nhc_conserved(const orc_sim* s) { return orc_nhc_conserved(&s->nhc); }
void orc_sim_remove_com(orc_sim* s) { orc_remove_com_motion(s->n, s->vx, s->vy, s->vz, s->m); }

/* ---- forcefield/ewald.cpp ------------------------------------------------- */
double orc_coulomb_prefactor(void) {
    /* ewald.hpp:10-13, ewald.cpp:17-21 */
    const double e = 1.602176565e-19, eps0 = 8.854187817e-12, kB = 1.3806488e-23;
    return (e * e) / (4.0 * kPi * eps0) * 1e10 / kB;
}

int orc_ewald_compute(int64_t n, const double box[3], const double* x, const double* y,
                      const double* z, const double* q, const int64_t* mol, double cutoff,
                      int kmax, double alpha_in, int mode, double* fx, double* fy, double* fz,
                      orc_ewald_terms* terms, double* virial) {
    /* ewald.cpp:33-175 */
    const int acc = mode != 0;
    if (mode == 1)
        for (int64_t i = 0; i < n; ++i) fx[i] = fy[i] = fz[i] = 0.0;
    double min_length = box[0];
    if (box[1] < min_length) min_length = box[1];
    if (box[2] < min_length) min_length = box[2];
    const double alpha = alpha_in > 0.0 ? alpha_in : 5.6 / min_length;
    const double coulomb = orc_coulomb_prefactor();
    const double rc2 = cutoff * cutoff;
    const double two_alpha_over_sqrt_pi = 2.0 * alpha / sqrt(kPi);
    double real = 0.0, self = 0.0, intra = 0.0, recip = 0.0, vir = 0.0;

    /* real space, ewald.cpp:45-69 */
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t j = i + 1; j < n; ++j) {
            if (mol[i] == mol[j]) continue;
            const double dx = orc_fold(x[i] - x[j], box[0]);
            const double dy = orc_fold(y[i] - y[j], box[1]);
            const double dz = orc_fold(z[i] - z[j], box[2]);
            const double r2 = norm2(dx, dy, dz);
            if (!(r2 < rc2)) continue;
            const double r = sqrt(r2);
            const double qq = q[i] * q[j];
            const double erfc_ar = erfc(alpha * r);
            real += coulomb * qq * erfc_ar / r;
            const double w =
                coulomb * qq * (two_alpha_over_sqrt_pi * exp(-alpha * alpha * r2) + erfc_ar / r);
            vir += w;
            if (acc) {
                const double s = w / r2;
                fx[i] += dx * s; fy[i] += dy * s; fz[i] += dz * s;
                fx[j] += (dx * s) * -1.0; fy[j] += (dy * s) * -1.0; fz[j] += (dz * s) * -1.0;
            }
        }
    }
    /* self, ewald.cpp:71-77 */
    double sum_q2 = 0.0;
    for (int64_t i = 0; i < n; ++i) sum_q2 += q[i] * q[i];
    self = -coulomb * alpha / sqrt(kPi) * sum_q2;

    /* intramolecular correction, ewald.cpp:79-110: atoms of one molecule in index
     * order, pairs (a<b) within it.  Molecules are visited in order of first
     * appearance (the reference's unordered_map order only changes the order of
     * the energy sum, not any per-atom force). */
    {
        int64_t* order = (int64_t*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int64_t));
        char* done = (char*)calloc((size_t)(n > 0 ? n : 1), 1);
        if (!order || !done) return -1;
        for (int64_t i = 0; i < n; ++i) {
            if (done[i]) continue;
            int64_t cnt = 0;
            for (int64_t k = i; k < n; ++k)
                if (!done[k] && mol[k] == mol[i]) {
                    order[cnt++] = k;
                    done[k] = 1;
                }
            for (int64_t a = 0; a < cnt; ++a) {
                for (int64_t b = a + 1; b < cnt; ++b) {
                    const int64_t ii = order[a], jj = order[b];
                    const double dx = orc_fold(x[ii] - x[jj], box[0]);
                    const double dy = orc_fold(y[ii] - y[jj], box[1]);
                    const double dz = orc_fold(z[ii] - z[jj], box[2]);
                    const double r2 = norm2(dx, dy, dz);
                    const double r = sqrt(r2);
                    const double qq = q[ii] * q[jj];
                    const double erf_ar = erf(alpha * r);
                    intra += -coulomb * qq * erf_ar / r;
                    const double w = coulomb * qq *
                                     (two_alpha_over_sqrt_pi * exp(-alpha * alpha * r2) - erf_ar / r);
                    vir += w;
                    if (acc) {
                        const double s = w / r2;
                        fx[ii] += dx * s; fy[ii] += dy * s; fz[ii] += dz * s;
                        fx[jj] += (dx * s) * -1.0; fy[jj] += (dy * s) * -1.0; fz[jj] += (dz * s) * -1.0;
                    }
                }
            }
        }
        free(order);
        free(done);
    }

    /* reciprocal space, ewald.cpp:112-172 */
    const double volume = box[0] * box[1] * box[2];
    const double kx0 = 2.0 * kPi / box[0];
    const double ky0 = 2.0 * kPi / box[1];
    const double kz0 = 2.0 * kPi / box[2];
    const int n2max = kmax * kmax + 2;
    double* cphi = NULL;
    double* sphi = NULL;
    if (acc) {
        cphi = (double*)malloc((size_t)(n > 0 ? n : 1) * sizeof(double));
        sphi = (double*)malloc((size_t)(n > 0 ? n : 1) * sizeof(double));
        if (!cphi || !sphi) return -1;
    }
    for (int nx = -kmax; nx <= kmax; ++nx) {
        for (int ny = -kmax; ny <= kmax; ++ny) {
            for (int nz = -kmax; nz <= kmax; ++nz) {
                const int n2 = nx * nx + ny * ny + nz * nz;
                if (n2 == 0 || n2 >= n2max) continue;
                const double kxv = kx0 * (double)nx;
                const double kyv = ky0 * (double)ny;
                const double kzv = kz0 * (double)nz;
                const double k2 = kxv * kxv + kyv * kyv + kzv * kzv;
                double re = 0.0, im = 0.0;
                for (int64_t i = 0; i < n; ++i) {
                    const double phase = kxv * x[i] + kyv * y[i] + kzv * z[i];
                    const double c = cos(phase);
                    const double s = sin(phase);
                    re += q[i] * c;
                    im += q[i] * s;
                    if (acc) {
                        cphi[i] = c;
                        sphi[i] = s;
                    }
                }
                const double factor =
                    coulomb * (2.0 * kPi / volume) * exp(-k2 / (4.0 * alpha * alpha)) / k2;
                const double s2 = re * re + im * im;
                recip += factor * s2;
                /* d/ds of the scaled sum at fixed alpha: factor |S|^2 (1 - k^2/(2 alpha^2)). */
                vir += factor * s2 * (1.0 - k2 / (2.0 * alpha * alpha));
                if (acc) {
                    for (int64_t i = 0; i < n; ++i) {
                        const double coeff = factor * 2.0 * q[i] * (re * sphi[i] - im * cphi[i]);
                        fx[i] += coeff * kxv;
                        fy[i] += coeff * kyv;
                        fz[i] += coeff * kzv;
                    }
                }
            }
        }
    }
    free(cphi);
    free(sphi);
    terms->real = real;
    terms->reciprocal = recip;
    terms->self = self;
    terms->intra = intra;
    if (virial) *virial = vir;
    return 0;
}

/* ---- forcefield/spce_forcefield.cpp:26-48 ---------------------------------- */
double orc_spce_compute(int64_t n, const double box[3], const double* x, const double* y,
                        const double* z, const double* q, const int64_t* mol, double sigma_o,
                        double epsilon_o, double cutoff, int kmax, double alpha, double* fx,
                        double* fy, double* fz) {
    const int64_t m = n / 3;
    double* ox = (double*)malloc((size_t)(m > 0 ? m : 1) * 6 * sizeof(double));
    if (!ox) return NAN;
    double *oy = ox + m, *oz = ox + 2 * m, *ofx = ox + 3 * m, *ofy = ox + 4 * m, *ofz = ox + 5 * m;
    for (int64_t k = 0; k < m; ++k) {
        ox[k] = x[3 * k];
        oy[k] = y[3 * k];
        oz[k] = z[3 * k];
    }
    orc_lj lj;
    orc_lj_init(&lj, sigma_o, epsilon_o, cutoff, 0);
    double e_disp, w_disp;
    orc_lj_compute(&lj, m, box, ox, oy, oz, ORC_SRC_BRUTE, NULL, NULL, 0, fx != NULL, ofx, ofy,
                   ofz, &e_disp, &w_disp);
    const double elrc = orc_lj_lrc_energy(&lj, m, box);
    orc_ewald_terms t;
    if (fx) {
        for (int64_t i = 0; i < n; ++i) fx[i] = fy[i] = fz[i] = 0.0;
        for (int64_t k = 0; k < m; ++k) {
            fx[3 * k] += ofx[k];
            fy[3 * k] += ofy[k];
            fz[3 * k] += ofz[k];
        }
        orc_ewald_compute(n, box, x, y, z, q, mol, cutoff, kmax, alpha, 2, fx, fy, fz, &t, NULL);
    } else {
        orc_ewald_compute(n, box, x, y, z, q, mol, cutoff, kmax, alpha, 0, NULL, NULL, NULL, &t, NULL);
    }
    free(ox);
    return e_disp + elrc + (t.real + t.reciprocal + t.self + t.intra);
}

/* ---- constrain/rigid_water.cpp ---------------------------------------------- */
int orc_rigid_water_init(orc_rigid_water* rw, double oh, double hoh_degrees, double tolerance,
                         int max_iterations) {
    if (!(oh > 0.0) || !(hoh_degrees > 0.0) || !(hoh_degrees < 180.0) || !(tolerance > 0.0) ||
        max_iterations < 1)
        return -1;
    rw->oh = oh;
    rw->tolerance = tolerance;
    rw->max_iterations = max_iterations;
    const double half_angle = 0.5 * hoh_degrees * kPi / 180.0;
    rw->hh = 2.0 * oh * sin(half_angle);
    return 0;
}

static const int kCons[3][2] = {{0, 1}, {0, 2}, {1, 2}};

int orc_rigid_water_positions(const orc_rigid_water* rw, int64_t n, const double box[3],
                              const double* mass, double* x, double* y, double* z,
                              const double* rx, const double* ry, const double* rz) {
    /* rigid_water.cpp:61-116 */
    if (n % 3 != 0) return -3;
    const double targets[3] = {rw->oh, rw->oh, rw->hh};
    for (int it = 0; it < rw->max_iterations; ++it) {
        double worst = 0.0;
        for (int64_t m = 0; m < n; m += 3) {
            for (int c = 0; c < 3; ++c) {
                const int64_t i = m + kCons[c][0], j = m + kCons[c][1];
                const double d2 = targets[c] * targets[c];
                const double ax = orc_fold(x[i] - x[j], box[0]);
                const double ay = orc_fold(y[i] - y[j], box[1]);
                const double az = orc_fold(z[i] - z[j], box[2]);
                const double s = norm2(ax, ay, az) - d2;
                const double violation = fabs(s) / d2;
                if (violation > worst) worst = violation;
                if (violation <= rw->tolerance) continue;
                const double bx = orc_fold(rx[i] - rx[j], box[0]);
                const double by = orc_fold(ry[i] - ry[j], box[1]);
                const double bz = orc_fold(rz[i] - rz[j], box[2]);
                const double inv_mass_sum = 1.0 / mass[i] + 1.0 / mass[j];
                const double denom = 2.0 * inv_mass_sum * (ax * bx + ay * by + az * bz);
                if (fabs(denom) < 1e-30) return -2;
                const double g = s / denom;
                const double gi = g / mass[i], gj = g / mass[j];
                x[i] = x[i] - bx * gi; y[i] = y[i] - by * gi; z[i] = z[i] - bz * gi;
                x[j] = x[j] + bx * gj; y[j] = y[j] + by * gj; z[j] = z[j] + bz * gj;
            }
        }
        if (worst <= rw->tolerance) return it + 1;
    }
    return -1;
}

int orc_rigid_water_velocities(const orc_rigid_water* rw, int64_t n, const double box[3],
                               const double* mass, const double* x, const double* y,
                               const double* z, double* vx, double* vy, double* vz) {
    /* rigid_water.cpp:118-161 */
    if (n % 3 != 0) return -3;
    const double targets[3] = {rw->oh, rw->oh, rw->hh};
    for (int it = 0; it < rw->max_iterations; ++it) {
        double worst = 0.0;
        for (int64_t m = 0; m < n; m += 3) {
            for (int c = 0; c < 3; ++c) {
                const int64_t i = m + kCons[c][0], j = m + kCons[c][1];
                const double d2 = targets[c] * targets[c];
                const double ax = orc_fold(x[i] - x[j], box[0]);
                const double ay = orc_fold(y[i] - y[j], box[1]);
                const double az = orc_fold(z[i] - z[j], box[2]);
                const double ux = vx[i] - vx[j], uy = vy[i] - vy[j], uz = vz[i] - vz[j];
                const double rv = ax * ux + ay * uy + az * uz;
                const double scaled = fabs(rv) / d2;
                if (scaled > worst) worst = scaled;
                if (scaled <= rw->tolerance) continue;
                const double inv_mass_sum = 1.0 / mass[i] + 1.0 / mass[j];
                const double k = rv / (inv_mass_sum * norm2(ax, ay, az));
                const double ki = k / mass[i], kj = k / mass[j];
                vx[i] = vx[i] - ax * ki; vy[i] = vy[i] - ay * ki; vz[i] = vz[i] - az * ki;
                vx[j] = vx[j] + ax * kj; vy[j] = vy[j] + ay * kj; vz[j] = vz[j] + az * kj;
            }
        }
        if (worst <= rw->tolerance) return it + 1;
    }
    return -1;
}

/* ---- analyze/ ------------------------------------------------------------ */
/* analyze/rdf.cpp:55-82 */
int orc_rdf_accumulate(int64_t n, const double box[3], const double* x, const double* y,
                       const double* z, double rmax, int64_t bins, double* hist) {
    double smallest = box[0];
    if (box[1] < smallest) smallest = box[1];
    if (box[2] < smallest) smallest = box[2];
    if (rmax > 0.5 * smallest) return -1;
    const double width = rmax / (double)bins; /* rdf.cpp:53 */
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t j = i + 1; j < n; ++j) {
            const double dx = orc_fold(x[i] - x[j], box[0]);
            const double dy = orc_fold(y[i] - y[j], box[1]);
            const double dz = orc_fold(z[i] - z[j], box[2]);
            const double r = sqrt(norm2(dx, dy, dz));
            if (r < rmax) {
                const uint64_t bin = (uint64_t)(r / width);
                if (bin < (uint64_t)bins) hist[bin] += 1.0;
            }
        }
    }
    return 0;
}

/* analyze/rdf.cpp:92-107 */
void orc_rdf_g(const double* hist, int64_t bins, double rmax, int64_t frames, int64_t natoms,
               double sum_rho, double* g) {
    const double pi = 3.14159265358979323846;
    const double width = rmax / (double)bins;
    for (int64_t k = 0; k < bins; ++k) g[k] = 0.0;
    if (frames == 0) return;
    const double rho = sum_rho / (double)frames;
    for (int64_t k = 0; k < bins; ++k) {
        const double lo = (double)k * width;
        const double hi = (double)(k + 1) * width;
        const double shell = (4.0 / 3.0) * pi * (hi * hi * hi - lo * lo * lo);
        const double denom = (double)frames * 0.5 * (double)natoms * rho * shell;
        g[k] = denom > 0.0 ? hist[k] / denom : 0.0;
    }
}

/* Shared ring-buffer loop of analyze/msd.cpp:66-106 (DIFF = 1) and
 * analyze/vacf.cpp:195-226 (DIFF = 0). */
static void orc_corr(int64_t frames, int64_t n, const double* a, int64_t max_lag, int diff,
                     double* out) {
    const int64_t period = max_lag + 1;
    double* sum = (double*)calloc((size_t)period, sizeof(double));
    int64_t* count = (int64_t*)calloc((size_t)period, sizeof(int64_t));
    for (int64_t f = 0; f < frames; ++f) {
        const int64_t avail = f < max_lag ? f : max_lag;
        const double* cur = a + f * 3 * n;
        for (int64_t lag = 0; lag <= avail; ++lag) {
            const double* org = a + (f - lag) * 3 * n;
            double s = 0.0;
            for (int64_t i = 0; i < n; ++i) {
                if (diff) {
                    s += norm2(cur[i] - org[i], cur[n + i] - org[n + i],
                               cur[2 * n + i] - org[2 * n + i]);
                } else {
                    s += cur[i] * org[i] + cur[n + i] * org[n + i] + cur[2 * n + i] * org[2 * n + i];
                }
            }
            sum[lag] += s;
            count[lag] += n;
        }
    }
    for (int64_t lag = 0; lag < period; ++lag)
        out[lag] = count[lag] > 0 ? sum[lag] / (double)count[lag] : 0.0;
    free(sum);
    free(count);
}

/* analyze/msd.cpp:66-96: incremental unwrapping by the minimum image of each step,
 * then the ring loop over unwrapped positions. */
void orc_msd(int64_t frames, int64_t n, const double box[3], const double* pos,
             int64_t max_lag, double* out) {
    double* unw = (double*)malloc(sizeof(double) * (size_t)(frames * 3 * n + 1));
    for (int64_t f = 0; f < frames; ++f) {
        const double* p = pos + f * 3 * n;
        double* u = unw + f * 3 * n;
        for (int64_t i = 0; i < n; ++i) {
            for (int d = 0; d < 3; ++d) {
                if (f == 0) {
                    u[d * n + i] = p[d * n + i];
                } else {
                    const double* q = pos + (f - 1) * 3 * n;
                    const double step = orc_fold(p[d * n + i] - q[d * n + i], box[d]);
                    u[d * n + i] = unw[(f - 1) * 3 * n + d * n + i] + step;
                }
            }
        }
    }
    orc_corr(frames, n, unw, max_lag, 1, out);
    free(unw);
}

/* analyze/vacf.cpp:195-226 */
void orc_vacf(int64_t frames, int64_t n, const double* vel, int64_t max_lag, double* out) {
    orc_corr(frames, n, vel, max_lag, 0, out);
}
