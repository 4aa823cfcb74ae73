"""Autotuner for the LJ step (no reference counterpart).

`tune_force_kernel` times the Verlet force kernel of an (LennardJones, system,
list) triple over its launch shapes -- threads per atom x independent gathers
in flight -- with CUDA events on the context stream, applies the fastest to the
LennardJones object and remembers it in an on-disk cache keyed by the device,
the system size and density, the cutoff and skin, the truncation and the
precision, so later runs of the same kind skip the search.

`tune_skin` picks the Verlet skin that minimises the time of a fused step (a
larger skin means a longer list but fewer rebuilds) by running a short fused
segment from the same state for each candidate.  `tune_cell_width` does the same
for the width of the cells the list is built from (the reference bins at the
list cutoff; wider cells give the same pairs from more candidates per atom and
fewer, fuller cells, which also reshapes the halo tiles of the mixed kernel).
`tune_tile_shape` times the mixed tile kernel over its threads per atom.

Cache: $MOLDYN_B200_TUNE_CACHE, else ~/.cache/moleculardynamics_b200/autotune.json.
"""
import ctypes as C
import json
import math
import os

import moleculardynamics_b200 as md

SHAPES = [(tpa, u) for tpa in (1, 2, 4, 8) for u in (1, 2, 4)]


def cache_path():
    return os.environ.get("MOLDYN_B200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "moleculardynamics_b200",
                                       "autotune.json"))


def _load(path):
    try:
        with open(path) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(path, table):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as fh:
        json.dump(table, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def problem_key(ctx, sys, lj, verlet_cutoff, skin):
    """Size bucket (powers of two) and density to two figures: launch shapes that
    win on one system win on its neighbours."""
    n = sys.n
    rho = n / sys.volume()
    return "|".join([ctx.device_name(), f"n2^{max(0, int(round(math.log2(max(n, 1)))))}",
                     f"rho{rho:.2g}", f"rc{lj.cutoff:g}", f"skin{skin:g}",
                     f"trunc{lj.truncation}", f"prec{lj.precision}"])


def time_force_kernel(ctx, sys, lj, verlet, repeats=5):
    """Mean device time (ms) of one Verlet force launch, CUDA events."""
    L = md.lib()
    lj.compute_forces(sys, verlet)  # warm-up (module load, buffers)
    md._check(L.md_context_set_timing(ctx.handle, 1))
    md._check(L.md_context_kernel_time(ctx.handle, md.MD_KERNEL_LJ_FORCE, 1, None, None))
    for _ in range(repeats):
        lj.compute_forces(sys, verlet)
    ms, launches = C.c_double(), C.c_int64()
    md._check(L.md_context_kernel_time(ctx.handle, md.MD_KERNEL_LJ_FORCE, 1, C.byref(ms),
                                       C.byref(launches)))
    md._check(L.md_context_set_timing(ctx.handle, 0))
    return ms.value / max(launches.value, 1)


def tune_force_kernel(sys, lj, verlet, skin, shapes=SHAPES, repeats=5, use_cache=True):
    """Applies and returns the fastest (tpa, unroll) for this problem; the dict of
    timings is returned too (empty when the answer came from the cache)."""
    ctx = sys.ctx
    path = cache_path()
    key = problem_key(ctx, sys, lj, lj.cutoff, skin)
    table = _load(path) if use_cache else {}
    if key in table:
        tpa, unroll = table[key]["shape"]
        lj.set_launch(tpa, unroll)
        return (tpa, unroll), {}
    timings = {}
    for tpa, unroll in shapes:
        lj.set_launch(tpa, unroll)
        timings[(tpa, unroll)] = time_force_kernel(ctx, sys, lj, verlet, repeats)
    best = min(timings, key=timings.get)
    lj.set_launch(*best)
    if use_cache:
        table = _load(path)
        table[key] = {"shape": list(best), "ms": timings[best],
                      "all": {f"{t}x{u}": v for (t, u), v in timings.items()}}
        _store(path, table)
    return best, timings


def tune_skin(box, pos, vel, mass, lj, make_integrator, skins=(0.2, 0.3, 0.4, 0.5), steps=100,
              ctx=None):
    """The skin with the shortest fused step over `steps` steps from this state;
    returns (best skin, {skin: ms per step})."""
    ctx = ctx or md.default_context()
    L = md.lib()
    times = {}
    for skin in skins:
        s = md.System.from_arrays(pos, box, vel=vel, mass=mass, ctx=ctx)
        v = md.VerletList(box, lj.cutoff, skin, ctx=ctx)
        v.build(s)
        lj.compute_forces(s, v)
        integ = make_integrator()
        integ.run(s, v, lj, 5)  # warm-up
        ms = C.c_double()
        md._check(L.md_context_span_begin(ctx.handle))
        integ.run(s, v, lj, steps)
        md._check(L.md_context_span_end(ctx.handle, C.byref(ms)))
        times[skin] = ms.value / steps
    return min(times, key=times.get), times


TILE_SHAPES = (0, 1, 2, 4)


def tune_tile_shape(sys, lj, verlet, shapes=TILE_SHAPES, repeats=5):
    """The fastest threads-per-atom of the mixed tile kernel (the tile shape) for a
    list that keeps halo tiles; applies it and returns (best, {tpa: ms})."""
    ctx = sys.ctx
    verlet.set_halo(True)
    timings = {}
    for tpa in shapes:
        lj.set_tile_threads(tpa)
        timings[tpa] = time_force_kernel(ctx, sys, lj, verlet, repeats)
    best = min(timings, key=timings.get)
    lj.set_tile_threads(best)
    return best, timings


def tune_cell_width(box, pos, vel, mass, lj, skin, make_integrator,
                    factors=(1.0, 1.1, 1.25, 1.5), steps=100, ctx=None):
    """The cell width (a factor of the list cutoff rc + skin) with the shortest
    fused step over `steps` steps from this state; returns (best width,
    {width: ms per step}).  Factor 1.0 is the reference's own binning."""
    ctx = ctx or md.default_context()
    L = md.lib()
    rl = lj.cutoff + skin
    times = {}
    for f in factors:
        width = rl * f
        s = md.System.from_arrays(pos, box, vel=vel, mass=mass, ctx=ctx)
        v = md.VerletList(box, lj.cutoff, skin, ctx=ctx)
        if f != 1.0:
            v.set_cell_width(width)
        if min(v.cells_per_side()) < 3:
            continue  # too few cells: the list would be built by brute force
        v.build(s)
        lj.compute_forces(s, v)
        integ = make_integrator()
        integ.run(s, v, lj, 5)  # warm-up
        ms = C.c_double()
        md._check(L.md_context_span_begin(ctx.handle))
        integ.run(s, v, lj, steps)
        md._check(L.md_context_span_end(ctx.handle, C.byref(ms)))
        times[width] = ms.value / steps
    return min(times, key=times.get), times


__all__ = ["SHAPES", "cache_path", "problem_key", "time_force_kernel", "tune_force_kernel",
           "tune_skin", "tune_cell_width", "TILE_SHAPES", "tune_tile_shape"]
