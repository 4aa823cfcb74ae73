// io.cu -- the data formats on either side of the path: moldyn_run's thermo CSV
// (apps/moldyn_run.cpp:229-245 header, 497-511 rows, 600-617 column header), its
// XYZ trajectory frames (moldyn_run.cpp:519-533), and a restartable binary
// checkpoint of a system and its integrator (no reference counterpart).
//
// Numbers are written as moldyn_run writes them: the CSV stream with
// std::setprecision(10), the XYZ stream with the default precision (6), both in
// the default float format, so a row of the same values is the same text.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "md_internal.cuh"

using namespace mdb;

struct md_thermo_csv {
    std::ofstream file;
};

namespace {

int io_fail(const char* who, const char* path) {
    return fail(MD_ERR_RUNTIME, "%s: cannot open '%s'", who, path ? path : "(null)");
}

// Host copies of the system's per-atom fields in original atom order.
int fetch(md_system* sys, int field, std::vector<double>& out) {
    out.resize(static_cast<size_t>(sys->n));
    if (sys->n == 0) return MD_OK;
    return md_system_get(sys, field, out.data());
}

}  // namespace

extern "C" {

// ----------------------------------------------------------------- thermo CSV
int md_thermo_csv_open(const char* path, const char* command_line, const char* revision,
                       const char* host, int truncation, int64_t dof_langevin, int64_t dof_nve,
                       md_thermo_csv** out) {
    if (!path || !out) return fail(MD_ERR_INVALID_ARGUMENT, "md_thermo_csv_open: NULL argument");
    md_thermo_csv* c = new (std::nothrow) md_thermo_csv;
    if (!c) return fail(MD_ERR_RUNTIME, "md_thermo_csv_open: out of host memory");
    c->file.open(path);
    if (!c->file.is_open()) {
        delete c;
        return io_fail("md_thermo_csv_open", path);
    }
    std::ofstream& f = c->file;
    // provenance (moldyn_run.cpp:229-234)
    f << "# command: " << (command_line ? command_line : "") << "\n";
    f << "# git_sha: " << (revision ? revision : "unknown") << "\n";
    f << "# host: " << (host ? host : "unknown") << "\n";
    f << "# units: reduced Lennard-Jones units (sigma = epsilon = mass = kB = 1)\n";
    f << std::setprecision(10);
    // truncation and degrees of freedom (moldyn_run.cpp:600-617)
    const bool tail = truncation == MD_TRUNCATED;
    f << "# truncation: " << (tail ? "truncated" : "linear-force-shift") << "\n";
    f << "# pressure_includes_tail_correction: " << (tail ? "yes" : "no") << "\n";
    f << "# potential_energy_includes_tail_correction: " << (tail ? "yes" : "no") << "\n";
    f << "# temperature_dof: 3N=" << dof_langevin
      << " while Langevin drives (equilibration, and Langevin production), 3N-3=" << dof_nve
      << " under the momentum-conserving integrators (NVE, Nose-Hoover), for which the "
         "centre-of-mass momentum is re-zeroed at the equilibration/production boundary\n";
    f << "step,time,phase,potential_energy,kinetic_energy,total_energy,temperature,pressure\n";
    *out = c;
    return f.good() ? MD_OK : io_fail("md_thermo_csv_open", path);
}

// StepSampler::record (moldyn_run.cpp:497-511) for thermo rows of a fused run
// (md_run_lj: pair energy, virial, kinetic energy, conserved contribution).
int md_thermo_csv_append(md_thermo_csv* c, const md_lj* lj, int64_t n, const double box[3],
                         int64_t first_step, int64_t step_stride, double dt, const char* phase,
                         int64_t dof, const double* rows, int64_t count) {
    if (!c || !lj || !box || (!rows && count > 0))
        return fail(MD_ERR_INVALID_ARGUMENT, "md_thermo_csv_append: NULL argument");
    if (dof <= 0) return fail(MD_ERR_INVALID_ARGUMENT, "md_thermo_csv_append: dof must be > 0");
    double u_lrc = 0.0, p_lrc = 0.0;
    MDB_TRY(md_lj_lrc(lj, n, box, &u_lrc, &p_lrc));
    const double volume = box[0] * box[1] * box[2];  // box.cpp volume: x * y * z
    const double density = static_cast<double>(n) / volume;
    std::ofstream& f = c->file;
    for (int64_t k = 0; k < count; ++k) {
        const double* r = rows + 4 * k;
        const long step = static_cast<long>(first_step + k * step_stride);
        const double t = static_cast<double>(step) * dt;
        const double ke = r[2];
        const double temperature = 2.0 * ke / static_cast<double>(dof);  // system.cpp:133-135
        const double pressure = density * temperature + r[1] / (3.0 * volume) + p_lrc;
        const double pe = r[0] + u_lrc;
        const double total = pe + ke;
        f << step << ',' << t << ',' << (phase ? phase : "") << ',' << pe << ',' << ke << ','
          << total << ',' << temperature << ',' << pressure << '\n';
    }
    return f.good() ? MD_OK : fail(MD_ERR_RUNTIME, "md_thermo_csv_append: write failed");
}

int md_thermo_csv_close(md_thermo_csv* c) {
    if (!c) return MD_OK;
    c->file.close();
    const bool ok = !c->file.fail();
    delete c;
    return ok ? MD_OK : fail(MD_ERR_RUNTIME, "md_thermo_csv_close: write failed");
}

// --------------------------------------------------------------- XYZ frames
int md_xyz_append(const char* path, md_system* sys, int64_t step, double time, const char* phase,
                  const char* revision, const char* host, const char* command_line) {
    if (!path || !sys) return fail(MD_ERR_INVALID_ARGUMENT, "md_xyz_append: NULL argument");
    std::vector<double> x, y, z;
    MDB_TRY(fetch(sys, MD_FIELD_X, x));
    MDB_TRY(fetch(sys, MD_FIELD_Y, y));
    MDB_TRY(fetch(sys, MD_FIELD_Z, z));
    std::ostringstream os;  // default precision, as moldyn_run's trajectory stream
    os << sys->n << '\n';
    os << "step=" << static_cast<long>(step) << " time=" << time << " phase="
       << (phase ? phase : "") << " git_sha=" << (revision ? revision : "unknown") << " host=\""
       << (host ? host : "unknown") << "\" command=\"" << (command_line ? command_line : "")
       << "\"" << '\n';
    for (int64_t i = 0; i < sys->n; ++i) os << "Ar " << x[i] << ' ' << y[i] << ' ' << z[i] << '\n';
    std::ofstream f(path, std::ios::app);
    if (!f.is_open()) return io_fail("md_xyz_append", path);
    f << os.str();
    return f.good() ? MD_OK : fail(MD_ERR_RUNTIME, "md_xyz_append: write failed");
}

}  // extern "C"

// ----------------------------------------------------------------- checkpoint
// Layout (little-endian): "MDB2CKP1", u32 version, u32 has_integrator, i64 n,
// f64 box[3], f64 fields [11][n] (x, y, z, vx, vy, vz, fx, fy, fz, mass, charge;
// original atom order), i64 mol[n], then when has_integrator: i32 kind, i32
// chain, f64 dt, friction, temperature, tau, u64 seed, step, i64 dof, u32
// has_chain and the chain state bytes; last, u64 FNV-1a of everything before.
namespace {

constexpr char kMagic[8] = {'M', 'D', 'B', '2', 'C', 'K', 'P', '1'};
constexpr uint32_t kVersion = 1;

struct Writer {
    std::vector<unsigned char> buf;
    template <class T>
    void put(const T& v) {
        const auto* p = reinterpret_cast<const unsigned char*>(&v);
        buf.insert(buf.end(), p, p + sizeof(T));
    }
    void put_bytes(const void* p, size_t n) {
        const auto* c = static_cast<const unsigned char*>(p);
        buf.insert(buf.end(), c, c + n);
    }
};

struct Reader {
    const std::vector<unsigned char>& buf;
    size_t at = 0;
    bool ok = true;
    template <class T>
    T get() {
        T v{};
        get_bytes(&v, sizeof(T));
        return v;
    }
    void get_bytes(void* p, size_t n) {
        if (at + n > buf.size()) {
            ok = false;
            std::memset(p, 0, n);
            return;
        }
        std::memcpy(p, buf.data() + at, n);
        at += n;
    }
};

uint64_t fnv1a(const unsigned char* p, size_t n) {
    uint64_t h = 1469598103934665603ull;
    for (size_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= 1099511628211ull;
    }
    return h;
}

}  // namespace

extern "C" {

int md_checkpoint_save(md_system* sys, const md_integrator* integ, const char* path) {
    if (!sys || !path) return fail(MD_ERR_INVALID_ARGUMENT, "md_checkpoint_save: NULL argument");
    Writer w;
    w.put_bytes(kMagic, sizeof(kMagic));
    w.put(kVersion);
    w.put(static_cast<uint32_t>(integ ? 1 : 0));
    w.put(static_cast<int64_t>(sys->n));
    for (int d = 0; d < 3; ++d) w.put(sys->box[d]);
    std::vector<double> f;
    for (int field = MD_FIELD_X; field <= MD_FIELD_CHARGE; ++field) {
        MDB_TRY(fetch(sys, field, f));
        w.put_bytes(f.data(), sizeof(double) * f.size());
    }
    std::vector<int64_t> mol(static_cast<size_t>(sys->n));
    if (sys->n) MDB_TRY(md_system_get_molecule_ids(sys, mol.data()));
    w.put_bytes(mol.data(), sizeof(int64_t) * mol.size());
    if (integ) {
        w.put(static_cast<int32_t>(integ->kind));
        w.put(static_cast<int32_t>(integ->chain));
        w.put(integ->dt);
        w.put(integ->friction);
        w.put(integ->temperature);
        w.put(integ->tau);
        w.put(static_cast<uint64_t>(integ->seed));
        w.put(static_cast<uint64_t>(integ->step));
        w.put(static_cast<int64_t>(integ->dof));
        const bool chain = integ->chain_state.ptr != nullptr;
        w.put(static_cast<uint32_t>(chain ? 1 : 0));
        if (chain) {
            NhcState st;
            MDB_CUDA(cudaMemcpy(&st, integ->chain_state.ptr, sizeof(st), cudaMemcpyDeviceToHost));
            w.put_bytes(&st, sizeof(st));
        }
    }
    w.put(fnv1a(w.buf.data(), w.buf.size()));
    std::ofstream out(path, std::ios::binary | std::ios::trunc);
    if (!out.is_open()) return io_fail("md_checkpoint_save", path);
    out.write(reinterpret_cast<const char*>(w.buf.data()), static_cast<std::streamsize>(w.buf.size()));
    return out.good() ? MD_OK : fail(MD_ERR_RUNTIME, "md_checkpoint_save: write failed");
}

int md_checkpoint_load(md_context* ctx, const char* path, md_system** out, md_integrator* integ) {
    if (!ctx || !path || !out) return fail(MD_ERR_INVALID_ARGUMENT, "md_checkpoint_load: NULL argument");
    std::ifstream in(path, std::ios::binary);
    if (!in.is_open()) return io_fail("md_checkpoint_load", path);
    const std::vector<unsigned char> buf((std::istreambuf_iterator<char>(in)),
                                         std::istreambuf_iterator<char>());
    if (buf.size() < sizeof(kMagic) + 8 + sizeof(uint64_t) ||
        std::memcmp(buf.data(), kMagic, sizeof(kMagic)) != 0)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_checkpoint_load: '%s' is not a checkpoint", path);
    uint64_t stored;
    std::memcpy(&stored, buf.data() + buf.size() - sizeof(stored), sizeof(stored));
    if (fnv1a(buf.data(), buf.size() - sizeof(stored)) != stored)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_checkpoint_load: '%s' is damaged (checksum)", path);
    Reader r{buf};
    char magic[8];
    r.get_bytes(magic, sizeof(magic));
    if (r.get<uint32_t>() != kVersion)
        return fail(MD_ERR_INVALID_ARGUMENT, "md_checkpoint_load: unsupported version");
    const bool has_integ = r.get<uint32_t>() != 0;
    const int64_t n = r.get<int64_t>();
    double box[3];
    for (double& b : box) b = r.get<double>();
    const size_t need = sizeof(double) * 11 * static_cast<size_t>(n) + sizeof(int64_t) * n;
    if (n < 0 || r.at + need > buf.size())
        return fail(MD_ERR_INVALID_ARGUMENT, "md_checkpoint_load: truncated file");
    md_system* sys = nullptr;
    MDB_TRY(md_system_create(ctx, n, box, &sys));
    std::vector<double> f(static_cast<size_t>(n));
    int rc = MD_OK;
    for (int field = MD_FIELD_X; field <= MD_FIELD_CHARGE && rc == MD_OK; ++field) {
        r.get_bytes(f.data(), sizeof(double) * f.size());
        if (n) rc = md_system_set(sys, field, f.data());
    }
    std::vector<int64_t> mol(static_cast<size_t>(n));
    r.get_bytes(mol.data(), sizeof(int64_t) * mol.size());
    if (rc == MD_OK && n) rc = md_system_set_molecule_ids(sys, mol.data());
    if (rc == MD_OK && integ) {
        if (!has_integ) {
            rc = fail(MD_ERR_INVALID_ARGUMENT, "md_checkpoint_load: the file holds no integrator");
        } else {
            const int32_t kind = r.get<int32_t>();
            const int32_t chain = r.get<int32_t>();
            const double dt = r.get<double>(), friction = r.get<double>();
            const double temperature = r.get<double>(), tau = r.get<double>();
            const uint64_t seed = r.get<uint64_t>(), step = r.get<uint64_t>();
            const int64_t dof = r.get<int64_t>();
            const bool has_chain = r.get<uint32_t>() != 0;
            if (kind != integ->kind || chain != integ->chain ||
                has_chain != (integ->chain_state.ptr != nullptr)) {
                rc = fail(MD_ERR_INVALID_ARGUMENT,
                          "md_checkpoint_load: the integrator is of another kind than the saved one");
            } else {
                integ->dt = dt;
                integ->friction = friction;
                integ->temperature = temperature;
                integ->tau = tau;
                integ->seed = seed;
                integ->step = step;
                integ->dof = dof;
                if (has_chain) {
                    NhcState st;
                    r.get_bytes(&st, sizeof(st));
                    if (cudaMemcpy(integ->chain_state.ptr, &st, sizeof(st),
                                   cudaMemcpyHostToDevice) != cudaSuccess)
                        rc = fail(MD_ERR_CUDA, "md_checkpoint_load: chain state upload failed");
                }
            }
        }
    }
    if (rc == MD_OK && !r.ok) rc = fail(MD_ERR_INVALID_ARGUMENT, "md_checkpoint_load: truncated file");
    if (rc != MD_OK) {
        md_system_destroy(sys);
        return rc;
    }
    *out = sys;
    return MD_OK;
}

}  // extern "C"
