"""SPC/E water structure at ambient conditions on the device (apps/water_rdf.cpp).

The reference app builds liquid water at 0.997 g/cm^3 from the 300-molecule NIST
sample configuration 3, expanded rigidly to the target volume; draws thermal
velocities; equilibrates with a velocity rescale toward 298 K every 50 steps;
and then runs NVE production, binning the oxygen-oxygen pairs every 10 steps.
It reports the first peak of g_OO(r) and the mean of g beyond 8.5 A, and writes
a CSV.

Here the state point and the initial velocities are built on the host exactly
as the reference does (same arithmetic, same Rng stream), and the whole
simulation -- every constrained step, every rescale, every O-O frame and the
temperature average -- is one device call, md_water_rdf_run, with one host
synchronisation at its end.  The analysis of the finished histogram and the
CSV follow apps/water_rdf.cpp:218-308.

    python -m moleculardynamics_b200.water_rdf --data DIR [--out PATH] [flags]

takes the reference's flags (apps/water_rdf.cpp:120-142).
"""
from __future__ import annotations

import ctypes as C
import os
import platform
import sys as _sys
import time

import numpy as np

from . import (ConstrainedVelocityVerlet, InvalidArgument, Rdf, RigidWater, SpceForceField,
               SpceParameters, _check, _f64, _ptr, build_spce_system, lib, read_nist_config,
               units)

AVOGADRO = 6.02214076e23        # apps/water_rdf.cpp:48
WATER_MOLAR_MASS = 18.01528     # g/mol, apps/water_rdf.cpp:49
RESCALE_EVERY = 50              # apps/water_rdf.cpp:188
RDF_RMAX = 10.0                 # apps/water_rdf.cpp:205
RDF_BINS = 200
CONFIG_FILE = os.path.join("nist", "spce", "spce_sample_config_periodic3.txt")


def box_length_for(molecules, grams_per_cm3):
    """Box length (A) holding `molecules` of water at the given density
    (apps/water_rdf.cpp:52-56)."""
    grams = float(molecules) * WATER_MOLAR_MASS / AVOGADRO
    cm3 = grams / grams_per_cm3
    return float(np.cbrt(cm3 * 1.0e24))


def rescale_rigidly(pos, mass, box, new_length):
    """Moves each O, H, H triple by its centre of mass times (factor - 1), so
    no bond stretches (apps/water_rdf.cpp:61-81).  Returns the new positions
    and the cubic box."""
    pos = _f64(pos).reshape(-1, 3)
    mass = _f64(mass).reshape(-1)
    if pos.shape[0] % 3 != 0:
        raise InvalidArgument("rescale_rigidly: atom count is not a multiple of 3")
    factor = new_length / float(box[0])
    p = pos.reshape(-1, 3, 3)
    m = mass.reshape(-1, 3)
    # com += p_k * m_k in k order, then com * (1 / mass), as the reference sums
    com = (p[:, 0] * m[:, 0:1] + p[:, 1] * m[:, 1:2]) + p[:, 2] * m[:, 2:3]
    total = (m[:, 0] + m[:, 1]) + m[:, 2]
    com = com * (1.0 / total)[:, None]
    shift = com * (factor - 1.0)
    out = (p + shift[:, None, :]).reshape(-1, 3)
    return out, np.full(3, float(new_length))


def thermal_velocities(mass, temperature, seed):
    """v_i = sqrt(T / m_i) * (n0, n1, n2), three Rng(seed).normal() draws per
    atom in atom order (apps/water_rdf.cpp:166-170)."""
    mass = _f64(mass).reshape(-1)
    xi = np.zeros(3 * mass.size)
    rc = lib().md_rng_normals(int(seed), xi.size, _ptr(xi))
    if rc < 0:
        _check(int(rc))
    s = np.sqrt(temperature / mass)
    return s[:, None] * xi.reshape(-1, 3)


def first_peak(r, g):
    """Tallest bin at r >= 2 and its parabolic refinement
    (apps/water_rdf.cpp:223-255).  Returns (bin r, bin g, refined r, refined g)."""
    peak, peak_g = 0, 0.0
    for k in range(len(g)):
        if r[k] < 2.0:
            continue
        if g[k] > peak_g:
            peak_g, peak = float(g[k]), k
    width = float(r[1] - r[0]) if len(r) > 1 else 0.0
    refined_r, refined_g = float(r[peak]), peak_g
    if 0 < peak < len(g) - 1:
        gm, g0, gp = float(g[peak - 1]), float(g[peak]), float(g[peak + 1])
        denom = gm - 2.0 * g0 + gp
        if abs(denom) > 1e-12:
            offset = 0.5 * (gm - gp) / denom
            refined_r = float(r[peak]) + offset * width
            refined_g = g0 - 0.25 * (gm - gp) * offset
    return float(r[peak]), peak_g, refined_r, refined_g


def tail_mean(r, g, beyond=8.5):
    """Mean of g over bins with r > 8.5 A (apps/water_rdf.cpp:257-267)."""
    total, count = 0.0, 0
    for k in range(len(g)):
        if r[k] > beyond:
            total += float(g[k])
            count += 1
    return total / count if count else 0.0


def state_point(pos, types, box, density=0.997, params=SpceParameters):
    """The reference's starting state: the SPC/E system of (pos, types, box)
    expanded rigidly to `density` (apps/water_rdf.cpp:150-156).  Returns
    (positions, types, box, molecules)."""
    types = list(types)
    m = np.array([params.massOxygen if t == "O" else params.massHydrogen for t in types])
    molecules = len(types) // 3
    length = box_length_for(molecules, density)
    new_pos, new_box = rescale_rigidly(pos, m, box, length)
    return new_pos, types, new_box, molecules


class WaterRdfResult(dict):
    """Everything apps/water_rdf.cpp reports: r, g, frames, temperatures, the
    first peak and the tail mean, timings."""

    __getattr__ = dict.__getitem__


def run(pos, types, box, density=0.997, temperature=298.0, dt_fs=2.0, equilibrate=15000,
        production=10000, sample_every=10, seed=7001, settle=False, ctx=None,
        params=SpceParameters):
    """apps/water_rdf.cpp:150-267 with the simulation on the device.

    (pos, types, box) is the starting configuration (NIST sample configuration
    3 in the reference).  settle=True resets positions and velocities with the
    closed-form SETTLE instead of SHAKE / RATTLE iterations (the same fixed
    point)."""
    pos, types, box, molecules = state_point(pos, types, box, density, params)
    sys = build_spce_system(pos, types, box, params, ctx=ctx)
    rigid = RigidWater(params.rOH, params.angleHOH, settle=settle)
    dt = units.femtoseconds(dt_fs)
    integ = ConstrainedVelocityVerlet(dt, rigid)
    ff = SpceForceField(ctx=ctx)
    dof = RigidWater.degrees_of_freedom(molecules, True)
    sys.velocities = thermal_velocities(sys.masses, temperature, seed)
    sys.remove_center_of_mass_motion()
    rigid.constrain_velocities(sys)
    rdf = Rdf(RDF_RMAX, RDF_BINS, ctx=ctx)
    mean_t = C.c_double()
    t0 = time.perf_counter()
    _check(lib().md_water_rdf_run(integ.handle, sys.handle, ff.handle, rdf.handle,
                                  float(temperature), int(dof), int(equilibrate),
                                  RESCALE_EVERY, int(production), int(sample_every),
                                  C.byref(mean_t)))
    r = rdf.bin_centres()
    g = rdf.g()
    wall = time.perf_counter() - t0
    bin_r, bin_g, peak_r, peak_g = first_peak(r, g)
    return WaterRdfResult(
        molecules=molecules, box_length=float(box[0]), density=density,
        temperature=temperature, mean_temperature=mean_t.value, dt_fs=dt_fs,
        equilibrate=int(equilibrate), production=int(production), frames=rdf.frames(),
        r=r, g=g, histogram=rdf.histogram(), bin_width=float(r[1] - r[0]) if len(r) > 1 else 0.0,
        first_peak_bin_r=bin_r, first_peak_bin_g=bin_g, first_peak_r=peak_r,
        first_peak_g=peak_g, tail_mean=tail_mean(r, g), wall_seconds=wall,
        system=sys, rdf=rdf, integrator=integ)


def _g(x):
    """std::ostream's default formatting of a double (6 significant digits)."""
    return "%g" % x


def write_csv(path, res, command_line="", revision=None, host=None, settle=False):
    """The CSV of apps/water_rdf.cpp:274-297."""
    host = host or f"{platform.system()} {platform.machine()}"
    model = "SETTLE" if settle else "SHAKE/RATTLE"
    lines = [
        f"# command: {command_line}",
        f"# git_sha: {revision or 'unknown'}",
        f"# host: {host}",
        f"# model: SPC/E, rigid ({model}), Ewald alpha=5.6/L kmax=5 rcut=10 A",
        f"# molecules: {res.molecules}",
        f"# box_length_angstrom: {_g(res.box_length)}",
        f"# density_g_per_cm3: {_g(res.density)}",
        f"# target_temperature_K: {_g(res.temperature)}",
        f"# mean_production_temperature_K: {_g(res.mean_temperature)}",
        f"# dt_fs: {_g(res.dt_fs)}",
        f"# equilibration_steps: {res.equilibrate}",
        f"# production_steps: {res.production}",
        f"# rdf_frames: {res.frames}",
        f"# bin_width_angstrom: {_g(res.bin_width)}",
        f"# first_peak_bin_r_angstrom: {_g(res.first_peak_bin_r)}",
        f"# first_peak_bin_g: {_g(res.first_peak_bin_g)}",
        f"# first_peak_r_angstrom: {_g(res.first_peak_r)}",
        f"# first_peak_g: {_g(res.first_peak_g)}",
        "# reference_first_peak_r_angstrom: 2.75",  # literal text in the reference's CSV
        "# reference_first_peak_g: 3.0",
        f"# tail_mean_g_beyond_8.5A: {_g(res.tail_mean)}",
        f"# wall_seconds: {_g(res.wall_seconds)}",
        "r_angstrom,g_oo",
    ]
    lines += [f"{_g(a)},{_g(b)}" for a, b in zip(res.r, res.g)]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def main(argv=None):
    """apps/water_rdf.cpp:104-308: the reference's flags, its printed summary."""
    argv = list(_sys.argv if argv is None else argv)
    opts = dict(data="data", out="results/water_rdf.csv", density=0.997, temperature=298.0,
                dt_fs=2.0, equilibrate=15000, production=10000, sample_every=10, seed=7001)
    kinds = dict(density=float, temperature=float, dt_fs=float, equilibrate=int,
                 production=int, sample_every=int, seed=int)
    settle = False
    i = 1
    while i < len(argv):
        a = argv[i]
        if a == "--settle":
            settle = True
            i += 1
            continue
        key = a[2:].replace("-", "_") if a.startswith("--") else None
        if key not in opts:
            print(f"water_rdf: unknown flag {a}", file=_sys.stderr)
            return 1
        if i + 1 >= len(argv):
            print(f"water_rdf: {a} needs a value", file=_sys.stderr)
            return 1
        opts[key] = kinds.get(key, str)(argv[i + 1])
        i += 2
    cfg = read_nist_config(os.path.join(opts["data"], CONFIG_FILE))
    res = run(cfg["pos"], cfg["types"], cfg["box"], opts["density"], opts["temperature"],
              opts["dt_fs"], opts["equilibrate"], opts["production"], opts["sample_every"],
              opts["seed"], settle=settle)
    print("water_rdf: %d molecules, L = %.4f A, density %.3f g/cm3, dt = %.1f fs"
          % (res.molecules, res.box_length, res.density, res.dt_fs))
    print("water_rdf: mean production temperature %.1f K (target %.1f)"
          % (res.mean_temperature, res.temperature))
    print("water_rdf: O-O first peak at r = %.4f A, g = %.3f (published ~2.75 A, g ~3.0)"
          % (res.first_peak_r, res.first_peak_g))
    print("water_rdf: g(r) tail beyond 8.5 A averages %.4f (must be 1)" % res.tail_mean)
    out_dir = os.path.dirname(opts["out"])
    if out_dir:
        os.makedirs(out_dir, exist_ok=True)
    write_csv(opts["out"], res, " ".join(argv), settle=settle)
    print("water_rdf: wrote %s in %.1f s" % (opts["out"], res.wall_seconds))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
