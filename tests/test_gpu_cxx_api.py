"""The reference's C++ API over the C ABI (include/moldyn_b200.hpp): a
moldyn_run-style NVE loop written against namespace moldyn (tests/cpp/shim_run.cpp)
is compiled with g++ and run on the GPU; its per-step energies and final state
follow the oracle's restatement of the same run, including a velocity the host
code changes half way (host mirror -> device)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle as O
from conftest import ROOT

pytestmark = pytest.mark.gpu


def build_and_run(md, cells, steps, seed):
    libdir = os.path.dirname(md.library_path())
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "shim_run")
        subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I",
                        os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "shim_run.cpp"),
                        f"-L{libdir}", "-lmoldyn_b200", f"-Wl,-rpath,{libdir}", "-o", exe],
                       check=True)
        res = subprocess.run([exe, str(cells), str(steps), str(seed)], capture_output=True,
                             text=True)
        assert res.returncode == 0, res.stderr[-2000:]
        out = res.stdout
    rows = np.array([[float(v) for v in l.split()[1:]] for l in out.splitlines() if l.startswith("row")])
    atoms = np.array([[float(v) for v in l.split()[1:]] for l in out.splitlines() if l.startswith("atom")])
    rebuilds = int([l for l in out.splitlines() if l.startswith("rebuilds")][0].split()[1])
    return rows, atoms, rebuilds


def test_cxx_api_run_follows_the_oracle(md):
    cells, steps, seed = 6, 100, 1
    rows, atoms, rebuilds = build_and_run(md, cells, steps, seed)
    st = O.fcc_lattice(cells, 0.8442, 0.722, seed)
    sim = O.Sim(st["pos"], st["vel"], st["mass"], st["box"], rc=2.5, trunc=0, skin=0.3, dt=0.005)
    sim.prime()
    ref = np.zeros((steps, 3))
    for k in range(steps):
        if k == steps // 2:
            p, v, f = sim.state()
            v[0] = 0.0
            sim.set_state(vel=v)
        sim.run("vv", 1)
        _, v, _ = sim.state()
        ref[k] = (sim.energy, sim.virial, 0.5 * np.sum(st["mass"][:, None] * v * v))
    assert rows.shape == ref.shape
    assert np.max(np.abs(rows - ref) / np.abs(ref)) < 1e-10
    p, v, _ = sim.state()
    assert np.max(np.abs(atoms[:, :3] - p)) < 1e-9
    assert np.max(np.abs(atoms[:, 3:] - v)) < 1e-9
    assert rebuilds == sim.rebuild_count


def test_cxx_analysis_classes_follow_the_oracle(md):
    """Rdf, Msd and Vacf of the C++ layer (tests/cpp/shim_analyze.cpp): g(r) over
    the frames it printed equals the oracle's exactly; the MSD follows the oracle
    at 1e-12."""
    libdir = os.path.dirname(md.library_path())
    cells, frames = 6, 6
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "shim_analyze")
        subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I",
                        os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "cpp", "shim_analyze.cpp"),
                        f"-L{libdir}", "-lmoldyn_b200", f"-Wl,-rpath,{libdir}", "-o", exe],
                       check=True)
        res = subprocess.run([exe, str(cells), str(frames), "10"], capture_output=True, text=True)
        assert res.returncode == 0, res.stderr[-2000:]
    lines = res.stdout.splitlines()
    pick = lambda tag: np.array([[float(v) for v in l.split()[1:]] for l in lines if l.startswith(tag + " ")])
    n = 4 * cells ** 3
    pos = pick("F").reshape(frames, n, 3)
    box = O.fcc_lattice(cells, 0.8442, 0.722, 5)["box"]
    _, g = O.rdf(pos, box, 3.0, 30)
    assert np.array_equal(pick("G")[:, 0], g)
    m = O.msd(pos, box, 4)
    mg = pick("M")[:, 0]
    assert mg[0] == 0.0 and np.all(np.abs(mg[1:] - m[1:]) <= 1e-12 * m[1:])
    v = pick("V")[:, 0]
    assert v[0] == 1.0 and len(v) == 5
    d = pick("D")[0]
    assert d[0] > 0.0 and np.isfinite(d[1])
