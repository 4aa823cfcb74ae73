"""The reference's own apps, compiled unchanged against this library, on the GPU.

moleculardynamics_b200/apps/Makefile compiles the reference's apps/moldyn_run.cpp
and apps/water_rdf.cpp where they lie, with include/ first on the include path:
include/moldyn/ holds the reference's header paths (moldyn/core/system.hpp, ...)
over the GPU library.  The binaries (moleculardynamics_b200/bin/) must write what
the same apps compiled on the reference's own sources write
(tests/golden/apps_ref.npz, made by tests/golden/make_golden.py from
oracle/_ref/moldyn_run and oracle/_ref/water_rdf):

* moldyn_run's thermo CSV (step, time, phase, U + U_LRC, KE, E, T, P), g(r) and
  MSD/VACF CSVs for the 864-atom drop-in configuration (1000 velocity-Verlet
  steps), the same start under the Nose-Hoover chain, and linear-force-shift
  truncation.  Rows agree to the CSV's 10 significant digits (a last-digit
  difference allowed: relative 1e-9), header lines exactly;
* moldyn_run --nist-config: the 12-case NIST table, character for character;
* a short water_rdf run: header values (6 significant digits) and g(r).

The NIST configuration files are written from the golden arrays (every value
printed so that it parses back to the same double), since the reference's data
tree is not on the GPU machine.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "moleculardynamics_b200", "bin")
APPS = load_golden("apps_ref.npz")
PROVENANCE = ("# command:", "# git_sha:", "# host:", "# wall_seconds:")


def parse_csv(path):
    comments, rows = [], []
    for line in open(path):
        line = line.rstrip("\n")
        if line.startswith("#"):
            if not line.startswith(PROVENANCE):
                comments.append(line)
        elif line and not line[0].isalpha():
            rows.append(line.split(","))
    return comments, rows


def app(name):
    path = os.path.join(BIN, name)
    assert os.access(path, os.X_OK), f"{path} is not built (make -C moleculardynamics_b200/apps)"
    return path


def write_nist(path, box, pos, types=None):
    """A NIST sample configuration in the layout readNistConfig parses
    (io/nist_config.cpp:30-86): box lengths, a count line, index x y z [type]."""
    with open(path, "w") as f:
        f.write(" ".join(repr(float(v)) for v in box) + "\n")
        f.write(f"{len(pos)}\n")
        for k, r in enumerate(pos):
            f.write(f"{k + 1} {float(r[0])!r} {float(r[1])!r} {float(r[2])!r}")
            f.write(f" {types[k]}\n" if types is not None else "\n")


@pytest.mark.parametrize("name", [str(n) for n in APPS["app_run_names"]])
def test_moldyn_run_writes_the_reference_csvs(name, tmp_path):
    args = str(APPS["app_runs"][list(APPS["app_run_names"]).index(name)]).split()
    files = {k: str(tmp_path / f"{k}.csv") for k in ("thermo", "rdf", "msd")}
    subprocess.run([app("moldyn_run"), *args, "--thermo-out", files["thermo"], "--rdf-out",
                    files["rdf"], "--msd-out", files["msd"]], check=True,
                   stdout=subprocess.DEVNULL, timeout=600)
    for k, path in files.items():
        comments, rows = parse_csv(path)
        assert comments == [str(c) for c in APPS[f"{name}_{k}_comments"]], k
        if k == "thermo":
            assert [r[2] for r in rows] == [str(p) for p in APPS[f"{name}_thermo_phase"]]
            rows = [[r[0], r[1]] + r[3:] for r in rows]
        got = np.array([[float(v) for v in r] for r in rows])
        ref = APPS[f"{name}_{k}"]
        assert got.shape == ref.shape, k
        # 10 significant digits as printed: equal up to one unit in the last digit;
        # g(r) holds integer pair counts over 1000 frames (one count ~1e-6 of a bin)
        rtol = 1e-5 if k == "rdf" else 1e-9
        bad = ~np.isclose(got, ref, rtol=rtol, atol=1e-12)
        assert not bad.any(), (k, np.argwhere(bad)[:5], got[bad][:5], ref[bad][:5])


def test_moldyn_run_nist_table_is_the_reference_table(tmp_path, golden):
    lj = golden("nist_lj.npz")
    d = tmp_path / "nist_lj"
    d.mkdir()
    for c in range(1, 5):
        write_nist(d / f"lj_sample_config_periodic{c}.txt", lj[f"box{c}"], lj[f"pos{c}"])
    out = subprocess.run([app("moldyn_run"), "--nist-config", str(d)], capture_output=True,
                         text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout == str(APPS["nist_table"])


def test_water_rdf_writes_the_reference_csv(tmp_path, golden):
    sp = golden("nist_spce.npz")
    d = tmp_path / "data" / "nist" / "spce"
    d.mkdir(parents=True)
    types = ["O" if o else "H" for o in sp["isO3"]]
    write_nist(d / "spce_sample_config_periodic3.txt", sp["box3"], sp["pos3"], types)
    csv = str(tmp_path / "water_rdf.csv")
    subprocess.run([app("water_rdf"), "--data", str(tmp_path / "data"), "--out", csv,
                    *str(APPS["water_rdf_args"]).split()], check=True, stdout=subprocess.DEVNULL,
                   timeout=600)
    comments, rows = parse_csv(csv)
    assert comments == [str(c) for c in APPS["water_rdf_comments"]]
    got = np.array([[float(v) for v in r] for r in rows])
    assert np.allclose(got, APPS["water_rdf_g"], rtol=1e-5, atol=1e-9)
