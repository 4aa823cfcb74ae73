"""CPU-only checks of the C ABI boundary: the library loads without a GPU and
exports every entry point include/moldyn_b200.h declares; host-side setup code
(md_fcc_lattice) reproduces the reference's lattice bit-for-bit."""
import ctypes as C
import os
import re

import numpy as np
import pytest

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
    """The reference-shaped C++ API (include/moldyn_b200.hpp) and the moldyn_run-style
    shims written against it compile with -Wall -Wextra -Werror (syntax and types
    only; no GPU)."""
    import os
    import subprocess
    from conftest import ROOT
    srcs = [os.path.join(ROOT, "tests", "cpp", f) for f in ("shim_run.cpp", "shim_analyze.cpp")]
    for src in srcs:
        res = subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only",
                              "-I", os.path.join(ROOT, "include"), src],
                             capture_output=True, text=True)
        assert res.returncode == 0, (src, res.stderr[-2000:])


def test_reference_apps_build_unchanged(tmp_path):
    """The reference's own apps/moldyn_run.cpp and apps/water_rdf.cpp, read where
    they lie and not edited, compile with -Wall -Wextra -Werror against
    include/moldyn/ (the reference's header paths over this library) and link to
    libmoldyn_b200.so, by the recipe that builds the shipped drop-in binaries
    (moleculardynamics_b200/apps/Makefile).  Skipped where the reference tree is
    absent (the recipe then builds nothing)."""
    import os
    import subprocess
    from conftest import ROOT
    res = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "moleculardynamics_b200", "apps"),
                          f"BINDIR={tmp_path}", "CXXFLAGS=-std=c++17 -O0 -Wall -Wextra -Werror"],
                         capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-3000:]
    built = sorted(os.listdir(tmp_path))
    if not built:
        pytest.skip("the reference's apps are not present here")
    assert built == ["moldyn_run", "water_rdf"]




def test_block_average_equals_reference(tmp_path):
    """blockAverage (analyze/block_average.hpp, host-side statistics in the C++ layer)
    gives the reference's mean, standard error and plateau block count bit for bit on
    correlated series of several lengths, and its empty and one-sample answers."""
    import subprocess

    import oracle as O
    R = O.ref()
    if R is None:
        pytest.skip("the compiled reference (oracle/_ref) is not present")
    R.ref_block_average.argtypes = [C.c_int64, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    exe = tmp_path / "block_average"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I",
                    os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp",
                                                                "block_average.cpp"),
                    "-o", str(exe)], check=True)
    rng = np.random.default_rng(11)
    cases = [np.zeros(0), np.array([2.5])]
    for n in (2, 3, 7, 64, 1000, 4097):
        x = np.empty(n)
        x[0] = rng.normal()
        for k in range(1, n):  # AR(1): correlated, so the plateau is not level 0
            x[k] = 0.9 * x[k - 1] + rng.normal()
        cases.append(x)
    for x in cases:
        out = subprocess.run([str(exe)], input=" ".join(repr(float(v)) for v in x),
                             capture_output=True, text=True, check=True).stdout.split()
        ref = np.zeros(3)
        xs = np.ascontiguousarray(x, dtype=np.float64)
        R.ref_block_average(len(xs), xs.ctypes.data_as(C.POINTER(C.c_double)),
                            ref.ctypes.data_as(C.POINTER(C.c_double)))
        assert float(out[0]) == ref[0] and float(out[1]) == ref[1], (len(x), out, ref)
        assert int(out[2]) == int(ref[2]), (len(x), out, ref)
