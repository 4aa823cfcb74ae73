"""GPU parity of the water_rdf driver (apps/water_rdf.cpp:150-267).

- The O-O frames: Rdf.accumulate over atoms 0, 3, 6, ... of the water system
  equals the oracle's Rdf of the gathered oxygens (gatherOxygens,
  apps/water_rdf.cpp:90-97) bin for bin, and the reference's g(r).
- The fused driver (md_water_rdf_run) equals the same protocol composed from
  public calls -- constrained runs, the device rescale, RATTLE's velocity half,
  per-frame accumulation, the host temperature sum -- bit for bit.
- The reference's full protocol (15,000 + 10,000 steps of 2 fs from NIST
  configuration 3 expanded to 0.997 g/cm^3) reproduces the structure of the
  reference's recorded run: the trajectory is chaotic, so the comparison is of
  g(r) and its first peak within statistical tolerances.
"""
import numpy as np
import pytest

import oracle as O
from conftest import load_golden

pytestmark = pytest.mark.gpu

SPCE = load_golden("nist_spce.npz")
WREF = load_golden("water_rdf_ref.npz")
WVAL = dict(zip([str(k) for k in WREF["keys"]], WREF["values"]))


def config3():
    return SPCE["pos3"], ["O" if o else "H" for o in SPCE["isO3"]], SPCE["box3"]


def prepared(md, settle=False, seed=7001):
    """The app's state: rigid expansion, thermal velocities, COM removal,
    constrained velocities (apps/water_rdf.cpp:150-175)."""
    from moleculardynamics_b200 import water_rdf as W
    pos, types, box, molecules = W.state_point(*config3())
    s = md.build_spce_system(pos, types, box)
    rigid = md.RigidWater(1.0, 109.47, settle=settle)
    s.velocities = W.thermal_velocities(s.masses, 298.0, seed)
    s.remove_center_of_mass_motion()
    rigid.constrain_velocities(s)
    dof = md.RigidWater.degrees_of_freedom(molecules, True)
    return s, rigid, dof, box


def test_rescale_temperature(md):
    s, rigid, dof, box = prepared(md)
    v = s.velocities
    m = s.masses
    t = 2.0 * (0.5 * np.sum(m * np.sum(v * v, axis=1))) / dof
    s.rescale_temperature(dof, 350.0)
    assert np.allclose(s.velocities, v * np.sqrt(350.0 / t), rtol=1e-14, atol=0)
    assert s.temperature(dof) == pytest.approx(350.0, rel=1e-13)
    s.velocities = np.zeros_like(v)  # T = 0: left alone (the app's t > 0 test)
    s.rescale_temperature(dof, 350.0)
    assert np.all(s.velocities == 0.0)
    with pytest.raises(md.InvalidArgument):
        s.rescale_temperature(0, 300.0)


@pytest.mark.parametrize("first,stride", [(0, 3), (1, 3), (0, 1), (2, 5)])
def test_subset_rdf_equals_the_gathered_frames(md, first, stride):
    s, rigid, dof, box = prepared(md)
    integ = md.ConstrainedVelocityVerlet(md.units.femtoseconds(2.0), rigid)
    ff = md.SpceForceField()
    rdf = md.Rdf(10.0, 200)
    frames = []
    for _ in range(3):
        integ.run(s, ff, 15)
        rdf.accumulate(s, first, stride)
        frames.append(s.positions[first::stride])
    assert rdf.frames() == 3
    hist, g = O.rdf(frames, box, 10.0, 200)
    assert np.array_equal(rdf.histogram(), hist)
    assert np.array_equal(rdf.g(), g)
    if O.ref_available():
        g_ref, _ = O.ref_rdf(frames, box, 10.0, 200)
        assert np.array_equal(rdf.g(), g_ref)


def test_subset_rdf_rejects_bad_selections(md):
    s, rigid, dof, box = prepared(md)
    rdf = md.Rdf(10.0, 20)
    for first, stride in ((-1, 3), (0, 0)):
        with pytest.raises(md.InvalidArgument):
            rdf.accumulate(s, first, stride)
    rdf.accumulate(s, 899, 3)  # one atom selected: a frame with no pairs
    assert rdf.frames() == 1 and np.all(rdf.histogram() == 0)


def run_driver(md, s, rigid, dof, equil, rescale, prod, sample):
    import ctypes as C
    integ = md.ConstrainedVelocityVerlet(md.units.femtoseconds(2.0), rigid)
    ff = md.SpceForceField()
    rdf = md.Rdf(10.0, 200)
    mean_t = C.c_double()
    md._check(md.lib().md_water_rdf_run(integ.handle, s.handle, ff.handle, rdf.handle, 298.0,
                                        dof, equil, rescale, prod, sample, C.byref(mean_t)))
    return rdf, mean_t.value, integ


def run_composed(md, s, rigid, dof, equil, rescale, prod, sample):
    integ = md.ConstrainedVelocityVerlet(md.units.femtoseconds(2.0), rigid)
    ff = md.SpceForceField()
    rdf = md.Rdf(10.0, 200)
    done = 0
    while done < equil:
        k = min(rescale - done % rescale, equil - done)
        integ.run(s, ff, k)
        done += k
        if done % rescale == 0:
            s.rescale_temperature(dof, 298.0)
            rigid.constrain_velocities(s)
    total = 0.0
    done = 0
    while done < prod:
        k = min(sample - done % sample, prod - done)
        th = integ.run(s, ff, k, thermo=True)
        for ke in th[:, 2]:
            total += 2.0 * ke / dof
        done += k
        if done % sample == 0:
            rdf.accumulate(s, 0, 3)
    return rdf, total / prod


def test_driver_equals_the_composed_protocol(md):
    a = prepared(md)
    rdf_a, t_a, _ = run_driver(md, *a[:3], 130, 50, 45, 10)
    b = prepared(md)
    rdf_b, t_b = run_composed(md, *b[:3], 130, 50, 45, 10)
    sa, sb = a[0], b[0]
    assert np.array_equal(sa.positions, sb.positions)
    assert np.array_equal(sa.velocities, sb.velocities)
    assert rdf_a.frames() == rdf_b.frames() == 4
    assert np.array_equal(rdf_a.histogram(), rdf_b.histogram())
    assert t_a == t_b


def test_driver_rejects_other_integrators_and_bad_counts(md):
    import ctypes as C
    s, rigid, dof, box = prepared(md)
    ff = md.SpceForceField()
    rdf = md.Rdf(10.0, 200)
    L = md.lib()
    nhc = md.ConstrainedNoseHooverChain(0.001, rigid, 298.0, 0.1, 3, dof)
    cvv = md.ConstrainedVelocityVerlet(0.001, rigid)
    with pytest.raises(md.InvalidArgument, match="ConstrainedVelocityVerlet"):
        md._check(L.md_water_rdf_run(nhc.handle, s.handle, ff.handle, rdf.handle, 298.0, dof,
                                     10, 5, 10, 5, None))
    for args in ((0, 10, 5, 10, 5), (dof, 10, 0, 10, 5), (dof, 10, 5, 10, 0), (dof, -1, 5, 10, 5)):
        with pytest.raises(md.InvalidArgument):
            md._check(L.md_water_rdf_run(cvv.handle, s.handle, ff.handle, rdf.handle, 298.0,
                                         *args, None))


@pytest.mark.parametrize("settle", [False, True])
def test_full_protocol_reproduces_the_reference_structure(md, settle, tmp_path):
    """apps/water_rdf.cpp defaults.  The reference recorded the first peak at
    2.7517 A (g 3.0847), a tail mean of 1.00014 and 294.4 K in production; 1000
    frames of 300 oxygens pin the peak to about a hundredth of an angstrom."""
    from moleculardynamics_b200 import water_rdf as W
    res = W.run(*config3(), settle=settle)
    assert res.frames == 1000 and res.molecules == 300
    assert float("%g" % res.box_length) == WVAL["box_length_angstrom"]
    assert abs(res.first_peak_r - WVAL["first_peak_r_angstrom"]) < 0.03
    assert abs(res.first_peak_g - WVAL["first_peak_g"]) < 0.2
    assert abs(res.tail_mean - 1.0) < 0.01
    # NVE production after a crude rescale: the reference saw 294.4 K after 30 ps
    # and 308.8 K after 10 ps of equilibration (apps/water_rdf.cpp:108-113)
    assert abs(res.mean_temperature - 298.0) < 15.0
    r, g = res.r, res.g
    assert np.all(g[r < 2.2] < 0.05)  # excluded volume
    band = (r > 2.0)
    assert np.sqrt(np.mean((g[band] - WREF["g"][band]) ** 2)) < 0.08
    # bonds held through 25,000 steps
    p = res.system.positions
    d = p[0::3] - p[1::3]
    d -= res.box_length * np.floor(d / res.box_length + 0.5)
    assert np.max(np.abs(np.linalg.norm(d, axis=1) - 1.0)) < 1e-9
    W.write_csv(tmp_path / "w.csv", res, "water_rdf", settle=settle)
    lines = (tmp_path / "w.csv").read_text().splitlines()
    assert lines[22] == "r_angstrom,g_oo" and len(lines) == 223


def test_cxx_app_equals_the_python_driver(md, tmp_path):
    """The C++ app (apps/water_rdf.cpp's drop-in on include/moldyn_b200.hpp) and
    the Python driver, on the same NIST file: every CSV line but the provenance
    ones (command, revision, host, wall time) is identical."""
    import os
    import subprocess
    from moleculardynamics_b200 import water_rdf as W
    pos, types, box = config3()
    cfg_dir = tmp_path / "data" / "nist" / "spce"
    cfg_dir.mkdir(parents=True)
    lines = ["%25.12E%25.12E%25.12E" % tuple(box), "%12d" % (len(types) // 3)]
    lines += ["%5d%25.12E%25.12E%25.12E    %s" % (k + 1, *p, t) for k, (p, t) in enumerate(zip(pos, types))]
    (cfg_dir / "spce_sample_config_periodic3.txt").write_text("\n".join(lines) + "\n")
    exe = os.path.join(os.path.dirname(md.library_path()), "bin", "water_rdf")
    args = ["--equilibrate", "150", "--production", "60", "--sample-every", "10"]
    res = subprocess.run([exe, "--data", str(tmp_path / "data"), "--out", str(tmp_path / "cxx.csv"),
                          *args], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-2000:]
    cfg = md.read_nist_config(cfg_dir / "spce_sample_config_periodic3.txt")
    r = W.run(cfg["pos"], cfg["types"], cfg["box"], equilibrate=150, production=60, sample_every=10)
    W.write_csv(tmp_path / "py.csv", r, "water_rdf")
    skip = ("# command", "# git_sha", "# host", "# wall_seconds")
    a = [l for l in (tmp_path / "cxx.csv").read_text().splitlines() if not l.startswith(skip)]
    b = [l for l in (tmp_path / "py.csv").read_text().splitlines() if not l.startswith(skip)]
    assert len(a) == len(b) == 219
    assert a == b


def test_python_cli_writes_the_csv(md, tmp_path, capsys):
    """python -m moleculardynamics_b200.water_rdf with the reference's flags on a
    short protocol: the summary lines and the CSV (header, 200 rows)."""
    from moleculardynamics_b200 import water_rdf as W
    pos, types, box = config3()
    cfg_dir = tmp_path / "data" / "nist" / "spce"
    cfg_dir.mkdir(parents=True)
    lines = ["%25.12E%25.12E%25.12E" % tuple(box), "%12d" % (len(types) // 3)]
    lines += ["%5d%25.12E%25.12E%25.12E    %s" % (k + 1, *p, t) for k, (p, t) in enumerate(zip(pos, types))]
    (cfg_dir / "spce_sample_config_periodic3.txt").write_text("\n".join(lines) + "\n")
    out = tmp_path / "res" / "w.csv"
    rc = W.main(["water_rdf", "--data", str(tmp_path / "data"), "--out", str(out),
                 "--equilibrate", "100", "--production", "50", "--sample-every", "5", "--settle"])
    assert rc == 0
    printed = capsys.readouterr().out
    assert "300 molecules, L = 20.8020 A" in printed and "O-O first peak" in printed
    text = out.read_text().splitlines()
    assert text[3] == "# model: SPC/E, rigid (SETTLE), Ewald alpha=5.6/L kmax=5 rcut=10 A"
    assert text[12] == "# rdf_frames: 10" and text[22] == "r_angstrom,g_oo" and len(text) == 223


def test_graph_replay_equals_host_launches(md):
    """md_water_rdf_run and md_run_spce replay captured blocks as CUDA graphs by
    default; with graphs off every kernel launches from the host.  Both give the
    same positions, velocities, histogram, mean temperature and thermo rows."""
    import ctypes as C
    out = {}
    for graphs in (True, False):
        ctx = md.Context(0)
        ctx.set_graphs(graphs)
        from moleculardynamics_b200 import water_rdf as W
        pos, types, box, molecules = W.state_point(*config3())
        s = md.build_spce_system(pos, types, box, ctx=ctx)
        rigid = md.RigidWater(1.0, 109.47)
        s.velocities = W.thermal_velocities(s.masses, 298.0, 7001)
        s.remove_center_of_mass_motion()
        rigid.constrain_velocities(s)
        dof = md.RigidWater.degrees_of_freedom(molecules, True)
        integ = md.ConstrainedVelocityVerlet(md.units.femtoseconds(2.0), rigid)
        ff = md.SpceForceField(ctx=ctx)
        rdf = md.Rdf(10.0, 200, ctx=ctx)
        mean_t = C.c_double()
        md._check(md.lib().md_water_rdf_run(integ.handle, s.handle, ff.handle, rdf.handle, 298.0,
                                            dof, 120, 50, 45, 10, C.byref(mean_t)))
        th = integ.run(s, ff, 12, thermo=True)
        out[graphs] = (s.positions, s.velocities, rdf.histogram(), mean_t.value, th)
    a, b = out[True], out[False]
    for x, y in zip(a, b):
        assert np.array_equal(np.asarray(x), np.asarray(y))
