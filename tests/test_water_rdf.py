"""Host side of the water_rdf driver (apps/water_rdf.cpp) and the NIST
configuration reader (io/nist_config.cpp), no GPU: the state point, the initial
velocities, the peak analysis and the CSV, each against a restatement with the
reference's own operation order or the reference's recorded run."""
import numpy as np
import pytest

import moleculardynamics_b200 as md
import oracle as O
from conftest import load_golden
from moleculardynamics_b200 import water_rdf as W

SPCE = load_golden("nist_spce.npz")
WREF = load_golden("water_rdf_ref.npz")
WVAL = dict(zip([str(k) for k in WREF["keys"]], WREF["values"]))


def nist_text(pos, box, types=None, count=None):
    """The NIST sample-configuration layout (13 significant digits, as the
    files carry them)."""
    lines = ["%25.12E%25.12E%25.12E" % tuple(box), "%12d" % (count if count is not None else len(pos))]
    for k, p in enumerate(pos):
        t = f"    {types[k]}" if types else ""
        lines.append("%5d%25.12E%25.12E%25.12E%s" % (k + 1, p[0], p[1], p[2], t))
    return "\n".join(lines) + "\n"


def spce_types(c):
    return ["O" if o else "H" for o in SPCE[f"isO{c}"]]


def test_reads_spce_configuration_and_keeps_types(tmp_path):
    """tests/test_nist_config.cpp:27-34 on configuration 3 (900 sites): the
    count line gives molecules, the reader reads atom lines to the end."""
    path = tmp_path / "spce3.txt"
    path.write_text(nist_text(SPCE["pos3"], SPCE["box3"], spce_types(3), count=300))
    cfg = md.read_nist_config(path)
    assert cfg["pos"].shape == (900, 3) and len(cfg["types"]) == 900
    assert np.array_equal(cfg["pos"], SPCE["pos3"]) and np.array_equal(cfg["box"], SPCE["box3"])
    assert cfg["types"][:3] == ["O", "H", "H"]


def test_reads_untyped_configuration_and_skips_blank_lines(tmp_path):
    """tests/test_nist_config.cpp:10-25: no type column -> types empty."""
    pos = SPCE["pos1"][:30]
    text = nist_text(pos, [8.0, 8.0, 8.0]).replace("\n    3", "\n\n   \n    3", 1)
    path = tmp_path / "lj.txt"
    path.write_text(text)
    cfg = md.read_nist_config(path)
    assert cfg["pos"].shape == (30, 3) and cfg["types"] == []
    assert np.array_equal(cfg["pos"], pos) and cfg["box"][0] == 8.0


def test_reader_errors(tmp_path):
    """tests/test_nist_config.cpp:36-38 plus the reader's other throws
    (nist_config.cpp:32-50, 68-70)."""
    with pytest.raises(md.MDError, match="cannot open file"):
        md.read_nist_config(tmp_path / "missing.txt")
    cases = {"empty": ("", "empty file"),
             "box": ("1.0 2.0\n3\n", "malformed box line"),
             "count": ("1 1 1\n", "missing count line"),
             "count2": ("1 1 1\nabc\n", "malformed count line"),
             "atom": ("1 1 1\n1\n1 0.5 0.5\n", "malformed atom line")}
    for name, (text, msg) in cases.items():
        p = tmp_path / name
        p.write_text(text)
        with pytest.raises(md.MDError, match=msg):
            md.read_nist_config(p)


def test_box_length_for_the_state_point():
    """apps/water_rdf.cpp:52-56; the reference's run recorded L = 20.802 A."""
    grams = 300.0 * 18.01528 / 6.02214076e23
    assert W.box_length_for(300, 0.997) == pytest.approx(np.cbrt(grams / 0.997 * 1e24), rel=1e-15)
    assert float("%g" % W.box_length_for(300, 0.997)) == WVAL["box_length_angstrom"]


def rescale_loop(pos, mass, box, new_length):
    """rescaleRigidly (apps/water_rdf.cpp:61-81), Vec3 arithmetic atom by atom."""
    factor = new_length / box[0]
    out = np.zeros_like(pos)
    for m in range(0, len(pos), 3):
        com = [0.0, 0.0, 0.0]
        total = 0.0
        for k in range(3):
            for d in range(3):
                com[d] += pos[m + k][d] * mass[m + k]
            total += mass[m + k]
        inv = 1.0 / total
        shift = [c * inv * (factor - 1.0) for c in com]
        for k in range(3):
            for d in range(3):
                out[m + k][d] = pos[m + k][d] + shift[d]
    return out


def test_rigid_rescale_matches_the_reference_arithmetic():
    pos = SPCE["pos3"]
    types = spce_types(3)
    mass = np.array([15.9994 if t == "O" else 1.008 for t in types])
    L = W.box_length_for(300, 0.997)
    got, box = W.rescale_rigidly(pos, mass, SPCE["box3"], L)
    assert np.array_equal(got, rescale_loop(pos, mass, SPCE["box3"], L))
    assert np.all(box == L)
    # every intramolecular vector is unchanged (rigid translation)
    for a, b in ((0, 1), (0, 2), (1, 2)):
        assert np.allclose(got[a::3] - got[b::3], pos[a::3] - pos[b::3], atol=1e-12)


def test_thermal_velocities_use_the_reference_rng_stream():
    """apps/water_rdf.cpp:166-170 with Rng(7001): the normals equal the compiled
    reference's (fixture) and the oracle's restatement."""
    mass = np.array([15.9994, 1.008, 1.008] * 300)
    v = W.thermal_velocities(mass, 298.0, 7001)
    xi = WREF["normals7001"].reshape(-1, 3)
    assert np.array_equal(v, np.sqrt(298.0 / mass)[:, None] * xi)
    assert np.array_equal(O.rng_normals(7001, 2700), WREF["normals7001"])


def test_peak_and_tail_on_the_reference_run():
    """apps/water_rdf.cpp:223-267 applied to the reference's own g(r)
    reproduces the peak and tail it recorded."""
    r, g = WREF["r"], WREF["g"]
    bin_r, bin_g, pr, pg = W.first_peak(r, g)
    assert bin_r == WVAL["first_peak_bin_r_angstrom"] and bin_g == WVAL["first_peak_bin_g"]
    assert float("%g" % pr) == WVAL["first_peak_r_angstrom"]
    assert float("%g" % pg) == WVAL["first_peak_g"]
    assert float("%g" % W.tail_mean(r, g)) == WVAL["tail_mean_g_beyond_8.5A"]


def test_peak_edge_cases():
    r = (np.arange(10) + 0.5) * 0.5
    assert W.first_peak(r, np.zeros(10)) == (r[0], 0.0, r[0], 0.0)  # nothing above r = 2
    g = np.zeros(10)
    g[9] = 2.0  # peak in the last bin: no refinement
    assert W.first_peak(r, g) == (r[9], 2.0, r[9], 2.0)
    g = np.zeros(10)
    g[5:8] = [1.0, 3.0, 1.0]  # symmetric: refinement keeps the bin centre
    assert W.first_peak(r, g) == (r[6], 3.0, r[6], 3.0)
    assert W.tail_mean(r, np.ones(10), beyond=100.0) == 0.0


def test_csv_layout(tmp_path):
    """apps/water_rdf.cpp:274-297: the header lines in order, default stream
    formatting (6 significant digits), then r,g rows."""
    r, g = WREF["r"], WREF["g"]
    res = W.WaterRdfResult(
        molecules=300, box_length=W.box_length_for(300, 0.997), density=0.997, temperature=298.0,
        mean_temperature=WVAL["mean_production_temperature_K"], dt_fs=2.0, equilibrate=15000,
        production=10000, frames=1000, r=r, g=g, bin_width=float(r[1] - r[0]),
        first_peak_bin_r=2.775, first_peak_bin_g=3.04588, first_peak_r=2.7516712,
        first_peak_g=3.0847091, tail_mean=1.000141, wall_seconds=434.687)
    path = tmp_path / "water_rdf.csv"
    W.write_csv(path, res, "water_rdf --out x", revision="abc", host="Linux x86_64")
    lines = path.read_text().splitlines()
    assert lines[0] == "# command: water_rdf --out x"
    assert lines[3] == "# model: SPC/E, rigid (SHAKE/RATTLE), Ewald alpha=5.6/L kmax=5 rcut=10 A"
    assert lines[5] == "# box_length_angstrom: 20.802"
    assert lines[16] == "# first_peak_r_angstrom: 2.75167"
    assert lines[18:20] == ["# reference_first_peak_r_angstrom: 2.75", "# reference_first_peak_g: 3.0"]
    assert lines[20] == "# tail_mean_g_beyond_8.5A: 1.00014"
    assert lines[22] == "r_angstrom,g_oo"
    assert lines[23] == "0.025,0" and lines[-1] == "9.975,%g" % g[-1]
    assert len(lines) == 23 + 200
    keys = [ln[2:].split(":")[0] for ln in lines[:22]]
    assert keys[4:] == ["molecules", "box_length_angstrom", "density_g_per_cm3",
                        "target_temperature_K", "mean_production_temperature_K", "dt_fs",
                        "equilibration_steps", "production_steps", "rdf_frames",
                        "bin_width_angstrom", "first_peak_bin_r_angstrom", "first_peak_bin_g",
                        "first_peak_r_angstrom", "first_peak_g", "reference_first_peak_r_angstrom",
                        "reference_first_peak_g", "tail_mean_g_beyond_8.5A", "wall_seconds"]


def test_flag_errors(capsys):
    """apps/water_rdf.cpp:120-142: an unknown flag or a missing value exits 1."""
    assert W.main(["water_rdf", "--bogus", "1"]) == 1
    assert "unknown flag --bogus" in capsys.readouterr().err
    assert W.main(["water_rdf", "--seed"]) == 1
    assert "--seed needs a value" in capsys.readouterr().err


def test_units():
    """core/units.hpp:33-40"""
    assert md.units.femtoseconds(2.0) == 2.0e-3 / 1.0966875353
    assert md.units.to_picoseconds(md.units.picoseconds(3.5)) == pytest.approx(3.5, rel=1e-15)


def test_cxx_app_flag_errors():
    """The reference's water_rdf app built unchanged on this library
    (moleculardynamics_b200/bin/water_rdf) rejects flags as apps/water_rdf.cpp:120-142
    does, before touching the device."""
    import os
    import subprocess
    exe = os.path.join(os.path.dirname(md.library_path()), "bin", "water_rdf")
    assert os.path.exists(exe), "build the drop-in apps first (make -C moleculardynamics_b200/apps)"
    res = subprocess.run([exe, "--bogus", "1"], capture_output=True, text=True)
    assert res.returncode == 1 and "unknown flag --bogus" in res.stderr
    res = subprocess.run([exe, "--seed"], capture_output=True, text=True)
    assert res.returncode == 1 and "--seed needs a value" in res.stderr
