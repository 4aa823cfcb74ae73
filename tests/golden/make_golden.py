"""Generates the golden fixtures in tests/golden/ from the reference itself.

Run in a container that has the reference tree (REF_ROOT, default /root/reference
as in oracle/Makefile) and the reference built by oracle/Makefile
(oracle/_ref/libmoldyn_ref.so and the reference's own apps oracle/_ref/moldyn_run,
oracle/_ref/water_rdf):

    python tests/golden/make_golden.py [REF_ROOT [FIXTURE ...]]

Inputs come from the reference's own data files (data/nist/...), the published
NIST values are read out of the reference's own test sources
(tests/test_nist_lj.cpp, tests/test_nist_spce.cpp), and every computed output
is produced by calling the compiled reference (not the restatement), so the
fixtures pin both the restatement and the GPU path to the reference.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402  (test infrastructure)


def _p(a):
    return O._p(a)


def published_lj(ref_root):
    """kRefs of tests/test_nist_lj.cpp:26-39 and kPressureTailPoints (:67-72)."""
    src = open(os.path.join(ref_root, "tests", "test_nist_lj.cpp")).read()
    rows = re.findall(r"\{(\d),\s*Truncation::(Truncated|LinearForceShift),\s*([-\d.e]+),"
                      r"\s*([-\d.e]+),\s*([-\d.e]+),\s*([-\d.e]+)\s*\}", src)
    table = np.array([[int(c), 0 if t == "Truncated" else 1, float(rc), float(u), float(w),
                       float(l)] for c, t, rc, u, w, l in rows])
    tail = re.findall(r"\{([\d.]+),\s*([\d.]+),\s*(-[\d.]+),\s*(-[\d.]+)\}", src)
    tail = np.array([[float(v) for v in r] for r in tail])
    assert table.shape == (12, 6), table.shape
    assert tail.shape == (4, 4), tail.shape
    return table, tail


def published_spce(ref_root):
    """kRefs of tests/test_nist_spce.cpp:64-69: config, Edisp, ELRC, Ereal,
    Efourier, Eself, Eintra, Etotal (K)."""
    src = open(os.path.join(ref_root, "tests", "test_nist_spce.cpp")).read()
    rows = re.findall(r"\{(\d),((?:\s*-?[\d.]+e-?\d+,?){7})\}", src)
    table = np.array([[int(c)] + [float(v) for v in vals.replace(" ", "").split(",") if v]
                      for c, vals in rows])
    assert table.shape == (4, 8), table.shape
    return table


def _grow(call, n):
    """Calls a pair-enumerating reference entry point until its buffer fits."""
    cap = 64 * n
    while True:
        pi = np.zeros(cap, np.int64)
        pj = np.zeros(cap, np.int64)
        cnt = call(pi, pj, cap)
        if cnt <= cap:
            return np.stack([pi[:cnt], pj[:cnt]], 1)
        cap = int(cnt)


def lj_fixture(ref_root, R):
    out = {}
    table, tail = published_lj(ref_root)
    out["published"] = table
    out["lrc_points"] = tail
    computed = []
    for c in (1, 2, 3, 4):
        box, pos, _ = O.read_nist_config(
            os.path.join(ref_root, "data", "nist", "lj", f"lj_sample_config_periodic{c}.txt"))
        n = len(pos)
        out[f"box{c}"] = box
        out[f"pos{c}"] = pos
        x, y, z = (np.ascontiguousarray(pos[:, k]) for k in range(3))
        for rc, tr in ((3.0, 0), (4.0, 0), (3.0, 1)):
            f = [np.zeros(n) for _ in range(3)]
            e = C.c_double()
            w = C.c_double()
            R.ref_lj_compute(n, _p(box), _p(x), _p(y), _p(z), 1.0, 1.0, rc, tr, 1, 0.0,
                             *[_p(a) for a in f], C.byref(e), C.byref(w))
            ul = C.c_double()
            pl = C.c_double()
            R.ref_lj_lrc(n, _p(box), 1.0, 1.0, rc, tr, C.byref(ul), C.byref(pl))
            computed.append([c, tr, rc, e.value, w.value, ul.value, pl.value])
            tag = f"{c}_{int(rc)}_{tr}"
            out[f"forces{tag}"] = np.stack(f, 1)
        # Verlet pairs at rc=3, skin=0.3 (tests/test_neighbor.cpp:100-104), reference order.
        out[f"verlet{c}"] = _grow(lambda pi, pj, cap: R.ref_verlet_pairs(
            n, _p(box), _p(x), _p(y), _p(z), 3.0, 0.3, _p(pi), _p(pj), cap), n)
        dims = (C.c_int * 3)()
        cells = _grow(lambda pi, pj, cap: R.ref_cells_pairs(
            n, _p(box), _p(x), _p(y), _p(z), 3.0, _p(pi), _p(pj), cap, dims), n)
        out[f"celldims{c}"] = np.array(list(dims))
        out[f"ncellpairs{c}"] = np.array(len(cells))
        if n <= 200:  # keep the fixture small: full candidate lists for the small configs
            out[f"cells{c}"] = cells
    out["computed"] = np.array(computed)
    return out


def spce_fixture(ref_root, R):
    out = {"published": published_spce(ref_root), "coulomb": np.array(R.ref_coulomb_prefactor())}
    qh = 0.42380
    for c in (1, 2, 3, 4):
        box, pos, types = O.read_nist_config(
            os.path.join(ref_root, "data", "nist", "spce", f"spce_sample_config_periodic{c}.txt"))
        n = len(pos)
        q = np.array([-2.0 * qh if t == "O" else qh for t in types])
        m = np.array([15.9994 if t == "O" else 1.008 for t in types])
        mol = np.arange(n, dtype=np.int64) // 3
        out[f"box{c}"] = box
        out[f"pos{c}"] = pos
        out[f"isO{c}"] = np.array([t == "O" for t in types])
        x, y, z = (np.ascontiguousarray(pos[:, k]) for k in range(3))
        f = [np.zeros(n) for _ in range(3)]
        terms = np.zeros(4)
        R.ref_ewald(n, _p(box), _p(x), _p(y), _p(z), _p(q), _p(mol), 10.0, 5, 1,
                    *[_p(a) for a in f], _p(terms))
        out[f"ewald_terms{c}"] = terms
        out[f"ewald_forces{c}"] = np.stack(f, 1)
        f2 = [np.zeros(n) for _ in range(3)]
        e = R.ref_spce(n, _p(box), _p(x), _p(y), _p(z), _p(m), _p(q), _p(mol), 10.0, 5, 1,
                       *[_p(a) for a in f2])
        out[f"spce_energy{c}"] = np.array(e)
        out[f"spce_forces{c}"] = np.stack(f2, 1)
    return out


def fcc_fixture(R):
    """fccLattice states and a short moldyn_run-style VV trajectory (reference)."""
    out = {}
    for tag, (cells, rho, temp, seed) in {"c6": (6, 0.8442, 0.722, 1),
                                          "c3": (3, 0.80, 1.0, 12345)}.items():
        n = 4 * cells ** 3
        arrs = [np.zeros(n) for _ in range(7)]
        box = np.zeros(3)
        R.ref_fcc_lattice(cells, rho, temp, seed, *[_p(a) for a in arrs], _p(box))
        out[f"{tag}_pos"] = np.stack(arrs[0:3], 1)
        out[f"{tag}_vel"] = np.stack(arrs[3:6], 1)
        out[f"{tag}_box"] = box
    # 25 NVE steps of the N=864 drop-in configuration (rc 2.5 Truncated, skin 0.3, dt 0.005).
    n = 864
    st = [np.ascontiguousarray(out["c6_pos"][:, k]) for k in range(3)] + \
         [np.ascontiguousarray(out["c6_vel"][:, k]) for k in range(3)] + [np.zeros(n) for _ in range(3)]
    info = np.zeros(5)
    R.ref_run(0, n, _p(out["c6_box"]), *[_p(a) for a in st], _p(np.ones(n)), 1.0, 1.0, 2.5, 0,
              0.3, 0.005, 25, 0.0, 0.0, 0, 0.0, 1, 0, _p(info))
    out["vv25_pos"] = np.stack(st[0:3], 1)
    out["vv25_vel"] = np.stack(st[3:6], 1)
    out["vv25_frc"] = np.stack(st[6:9], 1)
    out["vv25_info"] = info[:4]
    return out


def water_rdf_fixture(ref_root, R):
    """The reference's recorded water_rdf run (results/water_rdf.csv, written by
    apps/water_rdf.cpp:274-297): its header values and g_OO(r), plus the first
    normals of Rng(7001) (the app's velocity seed) from the compiled reference."""
    head, rows = {}, []
    for line in open(os.path.join(ref_root, "results", "water_rdf.csv")):
        line = line.strip()
        if line.startswith("# "):
            key, _, val = line[2:].partition(": ")
            try:
                head[key] = float(val)
            except ValueError:
                pass
        elif line and line[0].isdigit():
            rows.append([float(v) for v in line.split(",")])
    rows = np.array(rows)
    assert rows.shape == (200, 2), rows.shape
    keys = ["molecules", "box_length_angstrom", "density_g_per_cm3", "target_temperature_K",
            "mean_production_temperature_K", "dt_fs", "equilibration_steps", "production_steps",
            "rdf_frames", "bin_width_angstrom", "first_peak_bin_r_angstrom", "first_peak_bin_g",
            "first_peak_r_angstrom", "first_peak_g", "tail_mean_g_beyond_8.5A", "wall_seconds"]
    normals = np.zeros(2700)
    R.ref_rng_normals(7001, _p(normals), normals.size)
    return {"r": rows[:, 0], "g": rows[:, 1], "keys": np.array(keys),
            "values": np.array([head[k] for k in keys]), "normals7001": normals}


def exp02_fixture(ref_root, R):
    """The reference's recorded experiment 02 (experiments/exp02_energy_conservation.sh):
    moldyn_run NVE velocity Verlet on fcc(3), rho*=0.80, T*=1.0, seed 12345, rc 2.5,
    skin 0.4, linear-force-shift, dt 0.001 / 0.002 / 0.004 / 0.008 to t = 1.  Every
    thermo row (step, time, PE, KE, E, T, P) and the summary (e0, max |E - e0|,
    relative error) as written by the reference (results/exp02_*.csv)."""
    out = {}
    for dt in ("0.001", "0.002", "0.004", "0.008"):
        rows = []
        for line in open(os.path.join(ref_root, "results", f"exp02_thermo_dt{dt}.csv")):
            if line[:1].isdigit():
                f = line.strip().split(",")
                rows.append([float(f[0]), float(f[1])] + [float(v) for v in f[3:8]])
        out["thermo_" + dt] = np.array(rows)
    summary = []
    for line in open(os.path.join(ref_root, "results", "exp02_energy_conservation.csv")):
        if line[:1].isdigit():
            summary.append([float(v) for v in line.strip().split(",")])
    out["summary"] = np.array(summary)
    assert out["summary"].shape == (4, 4)
    return out


def exp03_fixture(ref_root, R):
    """The reference's recorded experiment 03 (experiments/exp03_argon_rdf.sh):
    moldyn_run on fcc(6) (864 atoms), rc 2.5, skin 0.3, dt 0.005, 5000 Langevin
    then 20000 NVE steps with g(r) (200 bins to 0.98 L/2) every production step,
    at the Rahman (0.8177, 0.7880, seed 3001) and Verlet (0.8442, 0.7280, seed
    3002) state points: each g(r) and the summary peak."""
    out = {}
    for label in ("rahman", "verlet"):
        rows = [[float(v) for v in line.strip().split(",")]
                for line in open(os.path.join(ref_root, "results", f"exp03_rdf_{label}.csv"))
                if line[:1].isdigit()]
        out["rdf_" + label] = np.array(rows)
    summ = {}
    for line in open(os.path.join(ref_root, "results", "exp03_argon_rdf.csv")):
        f = line.strip().split(",")
        if f[0] in ("rahman", "verlet"):
            summ[f[0]] = [float(f[1]), float(f[2]), float(f[3]), float(f[4]), float(f[5])]
    out["summary"] = np.array([summ["rahman"], summ["verlet"]])  # rho, T, seed, peak r, peak g
    return out


def exp04_fixture(ref_root, R):
    """The reference's recorded experiment 04 (experiments/exp04_argon_diffusion.sh):
    per replica (8 seeds at the Rahman and Verlet state points) the diffusion
    coefficients from the MSD fit and the VACF integral
    (results/exp04_argon_diffusion.csv): rho, T, seed, D_msd, D_vacf."""
    rows = []
    for line in open(os.path.join(ref_root, "results", "exp04_argon_diffusion.csv")):
        f = line.strip().split(",")
        if f[0] in ("rahman", "verlet"):
            rows.append([0.0 if f[0] == "rahman" else 1.0] + [float(v) for v in f[1:6]])
    rows = np.array(rows)
    assert rows.shape == (16, 6), rows.shape
    return {"replicas": rows}  # state (0 Rahman, 1 Verlet), rho, T, seed, D_msd, D_vacf


def exp05_fixture(ref_root, R):
    """The reference's recorded experiment 05 (experiments/exp05_lj_eos.sh): the LJ
    equation of state on fcc(5) (500 atoms), rc 3.0 with tail corrections, 10000
    Langevin then 20000 Nose-Hoover steps at NIST's temperature per density
    (results/exp05_lj_eos.csv): rho, seed, its T*, U*, p*, NIST's T*, U*, p*."""
    rows = []
    for line in open(os.path.join(ref_root, "results", "exp05_lj_eos.csv")):
        if line[:1].isdigit():
            rows.append([float(v) for v in line.strip().split(",")[:8]])
    rows = np.array(rows)
    assert rows.shape == (6, 8), rows.shape
    return {"rows": rows}


# moldyn_run command lines whose outputs the drop-in build of the same app must
# reproduce: the 864-atom drop-in configuration (velocity Verlet, 1000 steps), the
# same start under the Nose-Hoover chain, and linear-force-shift truncation.
APP_RUNS = {
    "c1_nve": ["--cells", "6", "--density", "0.8442", "--temperature", "0.722", "--cutoff", "2.5",
               "--skin", "0.3", "--dt", "0.005", "--equilibrate", "0", "--production", "1000",
               "--thermostat", "none", "--seed", "1"],
    "c1_nhc": ["--cells", "6", "--density", "0.8442", "--temperature", "0.722", "--cutoff", "2.5",
               "--skin", "0.3", "--dt", "0.005", "--equilibrate", "0", "--production", "500",
               "--thermostat", "nose-hoover", "--seed", "1"],
    "lfs_nve": ["--cells", "5", "--density", "0.8", "--temperature", "1.0", "--cutoff", "2.5",
                "--skin", "0.3", "--dt", "0.005", "--equilibrate", "0", "--production", "500",
                "--thermostat", "none", "--seed", "12345", "--truncation", "linear-force-shift"],
}
WATER_RDF_ARGS = ["--equilibrate", "200", "--production", "100", "--sample-every", "10"]


def parse_csv(path):
    """(comment lines minus the provenance ones that name the binary or host, rows)."""
    comments, rows = [], []
    for line in open(path):
        line = line.rstrip("\n")
        if line.startswith("#"):
            if not line.startswith(("# command:", "# git_sha:", "# host:", "# wall_seconds:")):
                comments.append(line)
        elif line and not line[0].isalpha():
            rows.append(line.split(","))
    return comments, rows


def apps_fixture(ref_root, R):
    """Outputs of the reference's own apps (oracle/_ref/moldyn_run, water_rdf, built
    from its sources by oracle/Makefile): moldyn_run's thermo, g(r) and MSD/VACF
    CSVs for APP_RUNS, its NIST table (--nist-config data/nist/lj), and a short
    water_rdf run (WATER_RDF_ARGS) on data/nist/spce configuration 3."""
    ref = os.path.join(ROOT, "oracle", "_ref")
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, args in APP_RUNS.items():
            files = {k: os.path.join(tmp, f"{name}_{k}.csv") for k in ("thermo", "rdf", "msd")}
            subprocess.run([os.path.join(ref, "moldyn_run"), *args, "--thermo-out", files["thermo"],
                            "--rdf-out", files["rdf"], "--msd-out", files["msd"]], check=True,
                           stdout=subprocess.DEVNULL)
            for k, path in files.items():
                comments, rows = parse_csv(path)
                out[f"{name}_{k}_comments"] = np.array(comments)
                if k == "thermo":
                    out[f"{name}_thermo_phase"] = np.array([r[2] for r in rows])
                    rows = [[r[0], r[1]] + r[3:] for r in rows]
                out[f"{name}_{k}"] = np.array([[float(v) for v in r] for r in rows])
        nist = subprocess.run([os.path.join(ref, "moldyn_run"), "--nist-config",
                               os.path.join(ref_root, "data", "nist", "lj")], check=True,
                              capture_output=True, text=True)
        out["nist_table"] = np.array(nist.stdout)
        csv = os.path.join(tmp, "water_rdf.csv")
        subprocess.run([os.path.join(ref, "water_rdf"), "--data", os.path.join(ref_root, "data"),
                        "--out", csv, *WATER_RDF_ARGS], check=True, stdout=subprocess.DEVNULL)
        comments, rows = parse_csv(csv)
        out["water_rdf_comments"] = np.array(comments)
        out["water_rdf_g"] = np.array([[float(v) for v in r] for r in rows])
    out["app_runs"] = np.array([" ".join(a) for a in APP_RUNS.values()])
    out["app_run_names"] = np.array(list(APP_RUNS))
    out["water_rdf_args"] = np.array(" ".join(WATER_RDF_ARGS))
    return out


FIXTURES = {
    "nist_lj.npz": lambda root, R: lj_fixture(root, R),
    "nist_spce.npz": lambda root, R: spce_fixture(root, R),
    "fcc_lj.npz": lambda root, R: fcc_fixture(R),
    "water_rdf_ref.npz": water_rdf_fixture,
    "exp02_ref.npz": exp02_fixture,
    "exp03_ref.npz": exp03_fixture,
    "exp04_ref.npz": exp04_fixture,
    "exp05_ref.npz": exp05_fixture,
    "apps_ref.npz": apps_fixture,
}


def main():
    """make_golden.py [REF_ROOT [FIXTURE ...]]: every fixture, or the named ones."""
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REF_ROOT", "/root/reference")
    names = sys.argv[2:] or sorted(FIXTURES)
    O.build(ref_root)
    R = O.ref()
    if R is None:
        raise SystemExit("reference library not built (oracle/_ref/libmoldyn_ref.so missing)")
    for name in names:
        np.savez_compressed(os.path.join(HERE, name), **FIXTURES[name](ref_root, R))
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    main()
