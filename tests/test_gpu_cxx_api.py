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
