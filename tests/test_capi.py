"""CPU-only checks of the C ABI boundary: the library loads without a GPU and
exports every entry point include/moldyn_b200.h declares; host-side setup code
(md_fcc_lattice) reproduces the reference's lattice bit-for-bit."""
import ctypes as C
import os
import re

import numpy as np

from conftest import ROOT, load_golden

HEADER = os.path.join(ROOT, "include", "moldyn_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(md_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    syms = declared_symbols()
    for required in ("md_context_create", "md_system_create", "md_verlet_build",
                     "md_lj_forces_verlet", "md_run_lj", "md_integrator_create_nhc"):
        assert required in syms


def test_library_exports_every_declared_symbol():
    import moleculardynamics_b200 as md
    lib = C.CDLL(md.library_path())
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_library_hides_internal_symbols():
    # only md_* entry points are visible; kernels and helpers stay hidden
    out = os.popen(f"nm -D --defined-only {__import__('moleculardynamics_b200').library_path()}").read()
    exported = [l.split()[-1] for l in out.splitlines() if " T " in l]
    assert exported and all(s.startswith("md_") for s in exported), exported[:10]


def test_lattice_setup_bit_exact_on_host():
    import moleculardynamics_b200 as md
    fcc = load_golden("fcc_lj.npz")
    st = md.fcc_lattice(6, 0.8442, 0.722, 1)
    assert np.array_equal(st["pos"], fcc["c6_pos"])
    assert np.array_equal(st["vel"], fcc["c6_vel"])
    assert np.array_equal(st["box"], fcc["c6_box"])
    st = md.fcc_lattice(3, 0.80, 1.0, 12345)
    assert np.array_equal(st["pos"], fcc["c3_pos"])


def test_invalid_arguments_map_to_reference_exceptions():
    import moleculardynamics_b200 as md
    import pytest
    with pytest.raises(md.InvalidArgument):
        md.LennardJones(1.0, 1.0, 2.5, truncation=7)
    h = C.c_void_p()
    rc = md.lib().md_integrator_create_nhc(0.002, 1.0, 0.5, 0, 10, C.byref(h))
    assert rc == md.MD_ERR_INVALID_ARGUMENT
    assert b"chainLength" in md.lib().md_last_error()


def test_rigid_water_host_side():
    """RigidWater's constructor checks and target distances (rigid_water.cpp:30-59)
    run on the host: invalid parameters raise InvalidArgument, the H-H target
    and the degrees of freedom match the oracle."""
    import moleculardynamics_b200 as md
    import pytest

    import oracle as O
    for bad in ((0.0, 109.47), (1.0, 0.0), (1.0, 180.0)):
        with pytest.raises(md.InvalidArgument):
            md.RigidWater(*bad)
    with pytest.raises(md.InvalidArgument):
        md.RigidWater(1.0, 109.47, 0.0)
    with pytest.raises(md.InvalidArgument):
        md.RigidWater(1.0, 109.47, 1e-12, 0)
    rw, orw = md.RigidWater(1.0, 109.47), O.rigid_water(1.0, 109.47)
    assert rw.oh_distance() == orw.oh and rw.hh_distance() == orw.hh
    assert md.RigidWater.degrees_of_freedom(100, True) == 597
    assert md.RigidWater.degrees_of_freedom(0, True) == 0


def test_cxx_api_header_compiles_and_links(tmp_path):
    """include/moldyn_b200.hpp (the reference's C++ class API over the C ABI)
    compiles cleanly and links against the library; running it needs a GPU."""
    import subprocess

    import moleculardynamics_b200 as md
    libdir = os.path.dirname(md.library_path())
    exe = tmp_path / "shim_run"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I",
                    os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "shim_run.cpp"),
                    f"-L{libdir}", "-lmoldyn_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)],
                   check=True)
    assert exe.exists()


def test_cxx_header_compiles_cleanly():
    """The reference-shaped C++ API (include/moldyn_b200.hpp) and the programs
    written against it -- the moldyn_run-style shims and the water_rdf app --
    compile with -Wall -Wextra -Werror (syntax and types only; no GPU)."""
    import os
    import subprocess
    from conftest import ROOT
    srcs = [os.path.join(ROOT, "tests", "cpp", f) for f in ("shim_run.cpp", "shim_analyze.cpp")]
    srcs.append(os.path.join(ROOT, "moleculardynamics_b200", "apps", "water_rdf.cpp"))
    for src in srcs:
        res = subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only",
                              "-I", os.path.join(ROOT, "include"), src],
                             capture_output=True, text=True)
        assert res.returncode == 0, (src, res.stderr[-2000:])
