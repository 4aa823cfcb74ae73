"""Benchmark: atom-steps/s of the 1,048,576-atom Lennard-Jones NVE step on one B200,
mixed precision vs FP64, with the reference CPU path beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Workload (per GPU): fcc 64^3 lattice (N = 1,048,576), rho* = 0.8442, T* = 0.722,
rc = 2.5 sigma (truncated), skin 0.3 sigma, dt* = 0.005; seeded Maxwell-Boltzmann
velocities, equilibrated by 2000 BAOAB Langevin steps (gamma* = 1) of the reference's
own code (oracle/make_lj1m_state.py writes that state once; both arms load it), then
NVE velocity-Verlet steps with device-decided Verlet rebuilds.  Outside the timed
region the GPU arm also runs the full 10,000-step NVE window in both precisions and
reports its energy drift per atom.  One "step" = one
velocity-Verlet step over the whole system (kick+drift, displacement check and
any rebuild, LJ forces, kick).  The per-step working set (positions, velocities,
forces, neighbour rows ~ 0.4 GB) exceeds the 126 MB L2, so no L2 flush is used.

Multi-GPU: the path has no exchange step, so N GPUs run N independent replicas
(weak scaling); value = total atom-steps/s over ranks, time = max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom-steps/s, 1M-atom LJ: mixed vs FP64 on 1 B200 at stated force error"
UNIT = "atom-steps/s"
CELLS = 64
RHO, TEMP, RC, SKIN, DT = 0.8442, 0.722, 2.5, 0.3, 0.005
SEED = 2026
TILE_THREADS = 0  # the mixed tile kernel's default shape unless --tile-threads


STATE_FILE = os.path.join(ROOT, "oracle", "_ref", "lj1m_baoab2000.npz")


def reference_state():
    """(box, pos, vel, steps) of the liquid the reference itself equilibrated
    (2000 LangevinBAOAB steps from the seeded lattice, written once by
    oracle/make_lj1m_state.py), or None when that build artefact is absent."""
    try:
        with np.load(STATE_FILE) as z:
            if int(z["cells"]) != CELLS:
                return None
            return (np.array(z["box"]), np.array(z["pos"]), np.array(z["vel"]),
                    int(z["steps"]))
    except (OSError, KeyError, ValueError):
        return None


def equilibration_note(ref_steps, gpu_steps):
    if ref_steps is not None:
        return (f"{ref_steps} LangevinBAOAB steps (gamma*=1, T*=0.722, seed {SEED + 1}) of the "
                f"reference's own code from the seeded lattice, COM momentum removed "
                f"(state file oracle/_ref/lj1m_baoab2000.npz)")
    if gpu_steps is None:
        return "none: the seeded lattice (the reference-equilibrated state file is absent)"
    return (f"{gpu_steps} BAOAB steps (gamma*=1) on the GPU from the seeded lattice "
            f"(the reference-equilibrated state file is absent)")


def config(equilibration):
    return {
        "workload": ("1M-atom LJ NVE velocity-Verlet: " if CELLS == 64 else "LJ NVE velocity-Verlet: ")
                    + f"fcc {CELLS}^3 (N={4 * CELLS ** 3}), rho*=0.8442, "
                    "T*=0.722, rc=2.5 truncated, skin=0.3, dt*=0.005",
        "n_atoms": 4 * CELLS ** 3,
        "equilibration": equilibration,
        "neighbour": "Verlet list rebuilt on device when the two largest displacements "
                     "exceed the skin (reference criterion)",
        "l2_policy": "no flush: per-step working set ~0.4 GB > 126 MB L2",
        "parallelism": "replicas (one independent system per GPU)",
    }


# ----------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None
        # the timed region starts once nvidia-smi has written its first sample (its
        # start-up, not the sampling, is what could delay this process's launches)
        t0 = time.time()
        while self.proc is not None and time.time() - t0 < 5.0:
            if os.path.getsize(self.path) > 0 or self.proc.poll() is not None:
                break
            time.sleep(0.05)
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        except OSError:
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        load = [s for s in sm if s > 0.5 * (max(mx) if mx else 1)] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(load) if load else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ----------------------------------------------------------------------- ranks
def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Group:
    """Host-side barrier and max/sum over ranks (plumbing only: replicas exchange
    no simulation data)."""

    def __init__(self, world):
        self.world = world
        self.dist = None
        if world > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
            self.dist = dist

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def reduce(self, value, op):
        if not self.dist:
            return value
        import torch
        t = torch.tensor([float(value)], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX if op == "max" else self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()


# ----------------------------------------------------------------------- GPU arm
def traffic_per_atom():
    """DRAM bytes per atom of one mixed LJ force launch, from the committed ncu
    summary (profiles/k_lj_halo_mixed_lj1m.txt), or None."""
    path = os.path.join(ROOT, "profiles", "k_lj_halo_mixed_lj1m.txt")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_atom:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def equilibrated_state(md, ctx, equil):
    st = md.fcc_lattice(CELLS, RHO, TEMP, SEED)
    s = md.System.from_arrays(st["pos"], st["box"], vel=st["vel"], mass=st["mass"], ctx=ctx)
    lj = md.LennardJones(1.0, 1.0, RC)
    v = md.VerletList(st["box"], RC, SKIN, ctx=ctx)
    v.build(s)
    lj.compute_forces(s, v)
    if equil > 0:
        md.LangevinBAOAB(DT, 1.0, TEMP, SEED + 1).run(s, v, lj, equil)
    s.remove_center_of_mass_motion()
    lj.compute_forces(s, v)
    return st["box"], s.positions, s.velocities, s.forces


def forces_of(md, ctx, box, pos, vel):
    """FP64 forces of a given state (the first half-kick of the NVE window needs them)."""
    s = md.System.from_arrays(pos, box, vel=vel, ctx=ctx)
    v = md.VerletList(box, RC, SKIN, ctx=ctx)
    v.build(s)
    md.LennardJones(1.0, 1.0, RC).compute_forces(s, v)
    return s.forces


def drift_run(md, ctx, box, pos, vel, frc, precision, steps):
    """The full NVE window (outside the timed region): `steps` fused VV steps from
    the state with thermo rows.  Returns the energy-conservation summary and the
    window's device-timed atom-steps/s (list rebuilds included)."""
    n = pos.shape[0]
    s = md.System.from_arrays(pos, box, vel=vel, ctx=ctx)
    s.forces = frc
    lj = md.LennardJones(1.0, 1.0, RC, precision=precision)
    v = md.VerletList(box, RC, SKIN, ctx=ctx)
    v.build(s)
    e0, _ = lj.compute_forces(s, v)
    ke0 = 0.5 * float(np.sum(vel * vel))
    integ = md.VelocityVerlet(DT)
    L = md.lib()
    md._check(L.md_context_span_begin(ctx.handle))
    rows = integ.run(s, v, lj, steps, thermo=True)
    ms = C.c_double()
    md._check(L.md_context_span_end(ctx.handle, C.byref(ms)))
    etot = (rows[:, 0] + rows[:, 2]) / n
    base = (e0 + ke0) / n
    t = DT * np.arange(1, steps + 1)
    slope = float(np.polyfit(t, etot - base, 1)[0])
    return {"max_abs_dev_per_atom": float(np.max(np.abs(etot - base))),
            "final_dev_per_atom": float(etot[-1] - base),
            "drift_per_atom_per_time": slope,
            "rebuilds": int(v.rebuild_count()),
            "atom_steps_per_s": n * steps / (ms.value * 1e-3)}


def timed_run(md, ctx, box, pos, vel, frc, precision, steps, warmup, group, clocks=None):
    """W warm-up + K timed fused VV steps from the given state.  Returns
    (device ms for K steps (max over ranks), thermo rows, force-kernel ms per launch,
    launches in the timed region, neighbour entries per atom, rebuilds)."""
    s = md.System.from_arrays(pos, box, vel=vel, ctx=ctx)
    s.forces = frc
    lj = md.LennardJones(1.0, 1.0, RC, precision=precision)
    if TILE_THREADS:
        lj.set_tile_threads(TILE_THREADS)
    v = md.VerletList(box, RC, SKIN, ctx=ctx)
    v.build(s)
    lj.compute_forces(s, v)
    integ = md.VelocityVerlet(DT)
    if warmup > 0:
        integ.run(s, v, lj, warmup)
    L = md.lib()
    ctx.synchronize()
    group.barrier()
    launches0 = ctx.launch_count()
    rebuild0 = v.rebuild_count()
    _check = md._check
    sampler = clocks.__enter__() if clocks else None
    _check(L.md_context_span_begin(ctx.handle))
    rows = integ.run(s, v, lj, steps, thermo=True)
    ms = C.c_double()
    _check(L.md_context_span_end(ctx.handle, C.byref(ms)))
    if sampler:
        clocks.__exit__(None, None, None)
    ctx.synchronize()
    group.barrier()
    launches = ctx.launch_count() - launches0
    rebuilds = v.rebuild_count() - rebuild0
    # The force kernel's own duration: CUDA events around each of its launches on
    # the context stream, over a further run of the same loop with per-kernel
    # timing on (that run launches every kernel from the host, so it is not the
    # timed region above).
    _check(L.md_context_set_timing(ctx.handle, 1))
    L.md_context_kernel_time(ctx.handle, md.MD_KERNEL_LJ_FORCE, 1, None, None)
    integ.run(s, v, lj, min(steps, 50))
    kms = C.c_double()
    kl = C.c_int64()
    _check(L.md_context_kernel_time(ctx.handle, md.MD_KERNEL_LJ_FORCE, 1, C.byref(kms), C.byref(kl)))
    _check(L.md_context_set_timing(ctx.handle, 0))
    pairs = v.pairs()
    nbr_per_atom = 2.0 * len(pairs) / s.n
    dev_ms = group.reduce(ms.value, "max")
    per_launch = kms.value / max(kl.value, 1)
    return dev_ms, rows, per_launch, launches, nbr_per_atom, rebuilds


def e2e_run(md, ctx, box, pos, vel, frc, steps, group):
    """The same steps through the public C ABI with host state: every step uploads
    the state from pinned host memory, runs one step and reads back the state and
    its thermo row.  Returns (wall seconds, max over ranks; h2d bytes/step; d2h)."""
    n = pos.shape[0]
    L = md.lib()
    s = md.System(n, box, ctx=ctx)
    s.masses = np.ones(n)
    lj = md.LennardJones(1.0, 1.0, RC, precision=md.PRECISION_MIXED)
    v = md.VerletList(box, RC, SKIN, ctx=ctx)
    integ = md.VelocityVerlet(DT)
    # pinned host buffers for the 9 state columns
    L.md_host_alloc.restype = C.c_void_p
    L.md_host_alloc.argtypes = [C.c_size_t]
    L.md_host_free.argtypes = [C.c_void_p]
    nbytes = n * 8
    ptrs = [L.md_host_alloc(nbytes) for _ in range(9)]
    if not all(ptrs):
        raise MemoryError("md_host_alloc failed")
    cols = [np.ctypeslib.as_array((C.c_double * n).from_address(p)) for p in ptrs]
    for k in range(3):
        cols[k][:] = pos[:, k]
        cols[3 + k][:] = vel[:, k]
        cols[6 + k][:] = frc[:, k]
    thermo = np.zeros(4)
    dp = C.POINTER(C.c_double)
    fields = (C.c_int * 9)(*range(9))
    cols_p = (dp * 9)(*[C.cast(p, dp) for p in ptrs])

    def step():
        md._check(L.md_system_set_fields(s.handle, 9, fields, cols_p))
        md._check(L.md_run_lj(integ.handle, s.handle, v.handle, lj.handle, 1,
                              thermo.ctypes.data_as(dp)))
        md._check(L.md_system_get_fields(s.handle, 9, fields, cols_p))

    # the list is built once from the uploaded state (rebuilds happen on device)
    for f in range(9):
        md._check(L.md_system_set(s.handle, f, C.cast(ptrs[f], dp)))
    v.build(s)
    for _ in range(2):
        step()
    ctx.synchronize()
    group.barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    t1 = time.perf_counter()
    group.barrier()
    for p in ptrs:
        L.md_host_free(p)
    return group.reduce(t1 - t0, "max"), 9 * nbytes, 9 * nbytes + thermo.nbytes


# ----------------------------------------------------------------------- CPU legs
def _ref_worker(args):
    """One single-threaded reference process: moldyn_run's VV loop on its own
    1M-atom system for `steps` steps; returns seconds of the stepping loop."""
    pos, vel, box, steps = args
    sys.path.insert(0, ROOT)
    import oracle as O
    R = O.ref()
    kind = "reference"
    n = pos.shape[0]
    st = [np.ascontiguousarray(pos[:, k]) for k in range(3)] + \
         [np.ascontiguousarray(vel[:, k]) for k in range(3)] + [np.zeros(n) for _ in range(3)]
    info = np.zeros(5)
    if R is not None:
        R.ref_run(0, n, O._p(np.ascontiguousarray(box)), *[O._p(a) for a in st],
                  O._p(np.ones(n)), 1.0, 1.0, RC, 0, SKIN, DT, steps, 0.0, 0.0, 0, 0.0, 1, 0,
                  O._p(info))
        return kind, info[4]
    kind = "port"
    sim = O.Sim(pos, vel, np.ones(n), box, rc=RC, trunc=0, skin=SKIN, dt=DT)
    sim.prime()
    t0 = time.perf_counter()
    sim.run("vv", steps)
    return kind, time.perf_counter() - t0


def cpu_reference(pos, vel, box, steps, procs):
    n = pos.shape[0]
    if procs <= 1:
        kind, sec = _ref_worker((pos, vel, box, steps))
        rates = [n * steps / sec]
    else:
        ctx = mp.get_context("spawn")
        with ctx.Pool(procs) as pool:
            res = pool.map(_ref_worker, [(pos, vel, box, steps)] * procs)
        kind = res[0][0]
        rates = [n * steps / sec for _, sec in res]
    return kind, float(sum(rates)), rates


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def lattice_state():
    """The seeded fcc 64^3 lattice (host setup, bit-identical to the reference's)."""
    import oracle as O
    st = O.fcc_lattice(CELLS, RHO, TEMP, SEED)
    return st["pos"], st["vel"], st["box"]


# ----------------------------------------------------------------------- main
def run_reference_arm(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    import oracle as O
    O.ref()  # the compiled reference, loaded here as well as in the workers
    steps = max(1, min(args.steps, args.ref_steps))
    procs = max(1, min(os.cpu_count() or 1, args.ref_procs))
    rs = reference_state()
    if rs is not None:
        box, pos, vel, ref_steps = rs
        where = "the reference-equilibrated liquid"
    else:
        pos, vel, box = lattice_state()
        ref_steps = None
        where = "the seeded lattice"
    note = equilibration_note(ref_steps, None)
    kind, _, rates = cpu_reference(pos, vel, box, steps, procs)
    n = 4 * CELLS ** 3
    # the processes run concurrently: the batch takes as long as its slowest one
    wall = max(n * steps / r for r in rates)
    ms = 1e3 * wall / steps
    value = procs * n * steps / wall
    sample = (f"{procs} concurrent single-threaded reference processes, each its own copy of "
              f"{where} ({n} atoms), {steps} NVE VV steps after its first Verlet build "
              f"({cpu_model()})")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
        "requested_steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded fcc lattice, Maxwell-Boltzmann velocities, "
                "reference-equilibrated liquid" if rs is not None else
                "synthetic: seeded fcc lattice, Maxwell-Boltzmann velocities",
        "config": config(note), "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": kind,
                         "sample": sample, "per_process": rates},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_gpu_arm(args):
    global CELLS, TILE_THREADS
    TILE_THREADS = args.tile_threads
    if args.cells != CELLS:
        # profiling configuration: a smaller lattice of the same liquid, equilibrated
        # on the GPU (the reference-equilibrated state is the 64^3 one)
        CELLS = args.cells
        args.gpu_equil = True
    world, rank, local = dist_env()
    group = Group(world)
    import moleculardynamics_b200 as md
    ctx = md.Context(local)
    md.set_threads_per_atom(args.tpa)
    md.set_unroll(args.unroll)
    n = 4 * CELLS ** 3
    rs = None if args.gpu_equil else reference_state()
    if rs is not None:
        box, pos, vel, ref_steps = rs
        frc = forces_of(md, ctx, box, pos, vel)
        note = equilibration_note(ref_steps, None)
        data = ("synthetic: seeded fcc lattice, Maxwell-Boltzmann velocities, "
                "reference-equilibrated liquid")
    else:
        box, pos, vel, frc = equilibrated_state(md, ctx, args.equil)
        note = equilibration_note(None, args.equil)
        data = ("synthetic: seeded fcc lattice, Maxwell-Boltzmann velocities, "
                f"{args.equil} BAOAB equilibration steps on the GPU")
    # identical starting state for both precisions
    clocks = ClockSampler(local)
    def one_arm_line(precision, ms, kms, reb):
        # profiling configuration (one precision alone): a short line, not the contract's
        if rank == 0:
            print(json.dumps({"precision": precision, "steps": args.steps,
                              "ms_per_step": ms / args.steps,
                              "atom_steps_per_s": world * n * args.steps / (ms * 1e-3),
                              "force_kernel_ms": kms, "rebuilds": reb}), flush=True)

    if args.precision == "mixed":
        ms, _, kms, _, _, reb = timed_run(md, ctx, box, pos, vel, frc, md.PRECISION_MIXED,
                                          args.steps, args.warmup, group)
        one_arm_line("mixed", ms, kms, reb)
        group.close()
        return 0
    ms64, rows64, k64, launch64, nbr, reb64 = timed_run(md, ctx, box, pos, vel, frc,
                                                        md.PRECISION_FP64, args.steps,
                                                        args.warmup, group)
    if args.precision == "fp64":
        one_arm_line("fp64", ms64, k64, reb64)
        group.close()
        return 0
    msmx, rowsmx, kmx, launchmx, _, rebmx = timed_run(md, ctx, box, pos, vel, frc,
                                                      md.PRECISION_MIXED, args.steps,
                                                      args.warmup, group, clocks)
    clk = clocks.summary()
    value64 = world * n * args.steps / (ms64 * 1e-3)
    valuemx = world * n * args.steps / (msmx * 1e-3)
    # force error of mixed vs FP64 on the same (equilibrated) state
    s = md.System.from_arrays(pos, box, vel=vel, ctx=ctx)
    v = md.VerletList(box, RC, SKIN, ctx=ctx)
    v.build(s)
    e64, w64 = md.LennardJones(1.0, 1.0, RC).compute_forces(s, v)
    f64 = s.forces
    emx, wmx = md.LennardJones(1.0, 1.0, RC, precision=md.PRECISION_MIXED).compute_forces(s, v)
    fmx = s.forces
    rms = float(np.sqrt(np.sum((fmx - f64) ** 2) / np.sum(f64 ** 2)))
    del s, v
    # end to end through the C ABI with host buffers (mixed)
    e2e_steps = max(3, min(args.steps, args.e2e_steps))
    sec, h2d, d2h = e2e_run(md, ctx, box, pos, vel, frc, e2e_steps, group)
    e2e_value = world * n * e2e_steps / sec
    # the full NVE window of the configuration, both precisions, outside the timed region
    drift = None
    drift_steps = 10000 if args.drift_steps is None else args.drift_steps
    if drift_steps > 0:
        d64 = drift_run(md, ctx, box, pos, vel, frc, md.PRECISION_FP64, drift_steps)
        dmx = drift_run(md, ctx, box, pos, vel, frc, md.PRECISION_MIXED, drift_steps)
        ratio = dmx["max_abs_dev_per_atom"] / max(d64["max_abs_dev_per_atom"], 1e-300)
        drift = {"steps": drift_steps, "fp64": d64, "mixed": dmx,
                 "mixed_over_fp64_max_dev": ratio, "within_2x_fp64": bool(ratio <= 2.0),
                 "window_mixed_over_fp64": dmx["atom_steps_per_s"] / d64["atom_steps_per_s"]}

    if rank == 0:
        peaks, peak_src = measured_peaks()
        # algorithmic bytes of one mixed force launch per atom: own fixed-point
        # position (16 B) + force write (24 B) + its row of the full neighbour list
        # as 16-bit halo-tile slots (2 B per entry), and the closing half-kick the
        # kernel applies: velocities read and written (48 B), mass and 1/mass (16 B)
        alg_per_atom = 16.0 + 24.0 + 2.0 * nbr + 48.0 + 16.0
        achieved = alg_per_atom * n / (kmx * 1e-3) / 1e9
        tpa = traffic_per_atom()
        e0_64 = rows64[0, 0] + rows64[0, 2]
        e0_mx = rowsmx[0, 0] + rowsmx[0, 2]
        drift64 = float(np.max(np.abs(rows64[:, 0] + rows64[:, 2] - e0_64)) / n)
        driftmx = float(np.max(np.abs(rowsmx[:, 0] + rowsmx[:, 2] - e0_mx)) / n)
        cpu = None
        if world == 1 and not args.no_cpu:
            kind, cval, _ = cpu_reference(pos, vel, box, args.cpu_steps, 1)
            cpu = {"value": cval, "unit": UNIT, "cores": 1, "kind": kind,
                   "sample": f"{args.cpu_steps} NVE VV steps of the same equilibrated "
                             f"{n}-atom state after the reference's first Verlet build, "
                             f"1 thread ({cpu_model()})"}
        line = {
            "metric": METRIC, "value": valuemx, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": msmx / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 pair terms, f64 displacement/accumulation/integration (mixed)",
            "data": data,
            "config": config(note),
            "fp64": {"value": value64, "ms_per_step": ms64 / args.steps,
                     "force_kernel_ms": k64, "rebuilds": reb64},
            "mixed_over_fp64": valuemx / value64,
            "force_rms_rel_err": rms,
            "energy_rel_err": abs(emx - e64) / abs(e64),
            "virial_rel_err": abs(wmx - w64) / abs(w64),
            "nve_max_energy_dev_per_atom": {"fp64": drift64, "mixed": driftmx,
                                            "steps": args.steps},
            "nve_drift_per_atom": drift,
            "neighbour_entries_per_atom": nbr,
            "rebuilds_in_timed_region": rebmx,
            "gpu_launches": int(launchmx),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "precision": "mixed",
                    "steps": e2e_steps,
                    "path": "md_system_set_fields (9 pinned host columns) + md_run_lj(1 step) + "
                            "md_system_get_fields (9 columns) per step"},
            "roofline": {"bound": "hbm", "kernel": "k_lj_halo (mixed, halo tiles, closing half-kick fused)",
                         "achieved": achieved, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                         "frac": achieved / peaks.get("hbm_gbs", 6650.0),
                         "peak_source": f"hbm_gbs of {peak_src}",
                         "algorithmic_bytes_per_atom": alg_per_atom,
                         "launch_ms": kmx,
                         "traffic": (tpa * n) if tpa else None},
            "clocks": clk,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    ctx.synchronize()
    group.close()
    return 0


# ------------------------------------------------------------------ batch workload
BATCH_METRIC = "aggregate atom-steps/s, 48 LJ replicas (NHC, mixed) on 1 B200"
BATCH_TABLE = os.path.join(ROOT, "moleculardynamics_b200", "data", "replicas_48.json")


def batch_table():
    with open(BATCH_TABLE) as fh:
        return json.load(fh)["replicas"]


def batch_config():
    rows = batch_table()
    return {"workload": "48 independent LJ replicas (table moleculardynamics_b200/data/"
                        "replicas_48.json): fcc n ~ U{4..20}, rho in {0.1..0.9}, T ~ U[1,2]; "
                        "NHC M=3 tau=0.5 dt=0.005, rc=2.5 truncated, skin 0.3, mixed precision",
            "replicas": len(rows), "atoms": sum(r["atoms"] for r in rows),
            "l2_policy": "no flush: replicas hold ~0.2 GB > 126 MB L2",
            "parallelism": "replicas (one CUDA graph per step holds every replica's kernels)"}


def _batch_ref_worker(args):
    """One single-threaded reference process stepping the given replicas with
    NoseHooverChain; returns (kind, atom-steps, seconds)."""
    rows, steps = args
    sys.path.insert(0, ROOT)
    import oracle as O
    R = O.ref()
    done, sec = 0, 0.0
    for r in rows:
        st = O.fcc_lattice(r["cells"], r["density"], r["temperature"], r["seed"])
        pos, vel, box = st["pos"], st["vel"], st["box"]
        n = pos.shape[0]
        cols = [np.ascontiguousarray(pos[:, k]) for k in range(3)] + \
               [np.ascontiguousarray(vel[:, k]) for k in range(3)] + [np.zeros(n) for _ in range(3)]
        info = np.zeros(5)
        if R is None:
            raise RuntimeError("reference library not built")
        R.ref_run(2, n, O._p(np.ascontiguousarray(box)), *[O._p(a) for a in cols],
                  O._p(np.ones(n)), 1.0, 1.0, RC, 0, SKIN, DT, steps, 0.0, r["temperature"], 0,
                  0.5, 3, 3 * n - 3, O._p(info))
        done += n * steps
        sec += info[4]
    return "reference", done, sec


def batch_cpu_reference(steps, procs):
    """The 48 replicas spread over `procs` concurrent single-threaded reference
    processes (largest first, round robin); aggregate = all atom-steps / the
    slowest process's stepping time."""
    rows = sorted(batch_table(), key=lambda r: -r["atoms"])
    shares = [rows[k::procs] for k in range(procs)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_batch_ref_worker, [(sh, steps) for sh in shares])
    total = sum(r[1] for r in res)
    return total / max(r[2] for r in res), procs


def make_batch(md, rows, device, precision, truncation):
    """The replica table as one batch: each replica its own context, lattice,
    list, force field and Nose-Hoover chain."""
    batch = md.Batch()
    parts = []
    for r in rows:
        ctx = md.Context(device)
        st = md.fcc_lattice(r["cells"], r["density"], r["temperature"], r["seed"])
        s = md.System.from_arrays(st["pos"], st["box"], vel=st["vel"], mass=st["mass"], ctx=ctx)
        lj = md.LennardJones(1.0, 1.0, RC, truncation, precision=precision)
        v = md.VerletList(st["box"], RC, SKIN, ctx=ctx)
        v.build(s)
        pe, _ = lj.compute_forces(s, v)
        integ = md.NoseHooverChain(DT, r["temperature"], 0.5, 3, 3 * s.n - 3)
        parts.append((ctx, s, v, lj, integ, pe + s.kinetic_energy()))
        batch.add(integ, s, v, lj)
    return batch, parts


def batch_drift_table(md, rows, device, steps):
    """Extended-Hamiltonian conservation of every replica over `steps` NHC steps
    from its lattice, outside the timed region: mixed and FP64 with the truncated
    potential of the configuration, and mixed with linear-force-shift truncation
    (no energy step when a pair crosses the cutoff) as the control.  Per replica:
    max |H'(t) - H'(0)| / N and the same relative to |H'(0)|."""
    cols = {}
    for name, prec, trunc in (("mixed", md.PRECISION_MIXED, 0), ("fp64", md.PRECISION_FP64, 0),
                              ("mixed_lfs", md.PRECISION_MIXED, 1)):
        batch, parts = make_batch(md, rows, device, prec, trunc)
        th = batch.run(steps, thermo=True)
        h = th[:, :, 0] + th[:, :, 2] + th[:, :, 3]
        h0 = np.array([p[5] for p in parts])  # H' before the first step (chain at rest)
        dev = np.max(np.abs(h - h0[:, None]), axis=1)
        n = np.array([p[1].n for p in parts], dtype=float)
        cols[name] = (dev / n, dev / np.abs(h0))
        del batch, parts
    table = []
    for k, r in enumerate(rows):
        table.append({"atoms": r["atoms"], "density": r["density"],
                      "temperature": r["temperature"],
                      **{f"{name}_per_atom": float(v[0][k]) for name, v in cols.items()},
                      **{f"{name}_relative": float(v[1][k]) for name, v in cols.items()}})
    summary = {name: {"per_atom_max": float(v[0].max()), "per_atom_median": float(np.median(v[0])),
                      "relative_max": float(v[1].max())} for name, v in cols.items()}
    return {"steps": steps, "summary": summary, "replicas": table,
            "mixed_over_fp64_per_atom_max": summary["mixed"]["per_atom_max"] /
            max(summary["fp64"]["per_atom_max"], 1e-300)}


def run_batch_arm(args):
    world, rank, local = dist_env()
    group = Group(world)
    if args.impl == "reference":
        if rank == 0:
            steps = max(1, min(args.steps, args.ref_steps))
            procs = max(1, min(os.cpu_count() or 1, args.ref_procs))
            value, procs = batch_cpu_reference(steps, procs)
            print(json.dumps({
                "metric": BATCH_METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": None,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded fcc lattices)", "config": batch_config(),
                "impl": "reference",
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs,
                                 "kind": "reference",
                                 "sample": f"all 48 replicas over {procs} concurrent single-threaded "
                                           f"reference processes, {steps} NHC steps each "
                                           f"({cpu_model()})"},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}), flush=True)
        group.close()
        return 0
    import moleculardynamics_b200 as md
    rows = batch_table()
    batch, parts = make_batch(md, rows, local, md.PRECISION_MIXED, 0)
    n_atoms = sum(p[1].n for p in parts)
    batch.run(args.warmup)
    lead = parts[0][0]
    L = md.lib()
    launches0 = sum(p[0].launch_count() for p in parts)
    group.barrier()
    clocks = ClockSampler(local)
    clocks.__enter__()
    md._check(L.md_context_span_begin(lead.handle))
    th = batch.run(args.steps, thermo=True)
    ms = C.c_double()
    md._check(L.md_context_span_end(lead.handle, C.byref(ms)))
    clocks.__exit__(None, None, None)
    group.barrier()
    launches = sum(p[0].launch_count() for p in parts) - launches0
    dev_ms = group.reduce(ms.value, "max")
    value = world * n_atoms * args.steps / (dev_ms * 1e-3)
    h = th[:, :, 0] + th[:, :, 2] + th[:, :, 3]
    dev = np.max(np.abs(h - h[:, :1]), axis=1)
    drift = dev / np.abs(h[:, 0])
    per_atom = dev / np.array([p[1].n for p in parts])
    if rank == 0:
        line = {
            "metric": BATCH_METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 pair terms, f64 displacement/accumulation/integration (mixed)",
            "data": "synthetic: seeded fcc lattices, Maxwell-Boltzmann velocities",
            "config": batch_config(), "gpu_launches": int(launches),
            "nhc_extended_energy_drift": {
                "steps": args.steps, "note": "truncated LJ: cutoff crossings step the energy",
                "relative_max": float(drift.max()), "relative_median": float(np.median(drift)),
                "per_atom_max": float(per_atom.max()), "per_atom_median": float(np.median(per_atom))},
            "clocks": clocks.summary(),
        }
        drift_steps = 5000 if args.drift_steps is None else args.drift_steps
        if drift_steps > 0:
            line["nhc_drift_per_replica"] = batch_drift_table(md, rows, local, drift_steps)
        if world == 1 and not args.no_cpu:
            cval, procs = batch_cpu_reference(max(1, args.cpu_steps), args.ref_procs)
            line["cpu_baseline"] = {"value": cval, "unit": UNIT, "cores": procs,
                                    "kind": "reference",
                                    "sample": f"all 48 replicas over {procs} concurrent "
                                              f"single-threaded reference processes, "
                                              f"{max(1, args.cpu_steps)} NHC steps each "
                                              f"({cpu_model()})"}
        print(json.dumps(line), flush=True)
    group.close()
    return 0


# ---------------------------------------------------------------- adjoint workload
ADJ_METRIC = "atom-steps/s of forward + adjoint backward, 32,000-atom LJ trajectory (FP64)"


def adjoint_config(steps, every, skin):
    return {"workload": f"differentiable LJ trajectory: fcc 20^3 (N=32000), rho*=0.8442, "
                        f"T*=0.722, rc=2.5 force-shifted (continuous, so finite differences "
                        f"see no cutoff jumps), {steps} FP64 velocity-Verlet steps, dt*=0.005, "
                        f"states saved every {every} steps, list skin {skin}",
            "loss": "(mean virial pressure - 1)^2 + (mean potential energy per atom + 5)^2",
            "n_atoms": 32000, "parallelism": "one system"}


def adjoint_sweep(md, ctx, pos, vel, mass, box, every, skin, group, rank):
    """Where the adjoint gradient of the trajectory loss stops agreeing with central
    finite differences of the same forward code, as the trajectory grows: for each
    length, d(loss)/d(epsilon) and d(loss)/d(sigma) by the adjoint, against
    [L(p (1 + h)) - L(p (1 - h))] / 2h for h = 1e-5 ... 1e-10 (relative).  The loss
    and the force-shifted potential are the benchmark's."""
    n, vol = pos.shape[0], float(np.prod(box))
    dof = 3 * n - 3

    def loss_rows(rows):
        p = n / vol * 2 * rows[:, 2] / dof + rows[:, 1] / (3 * vol)
        u = rows[:, 0] / n
        return (p.mean() - 1.0) ** 2 + (u.mean() + 5.0) ** 2, p.mean(), u.mean()

    def forward(steps, sigma=1.0, eps=1.0):
        s = md.System.from_arrays(pos, box, vel=vel, mass=mass, ctx=ctx)
        traj = md.AdjointTrajectory(ctx)
        lj = md.LennardJones(sigma, eps, RC, md.Truncation.LinearForceShift)
        rows = traj.forward(s, lj, DT, steps, every, skin)
        return rows, traj

    hs = [1e-5, 1e-6, 1e-7, 1e-8, 1e-9, 1e-10]
    table = []
    for steps in (50, 100, 200, 400, 700, 1000):
        rows, traj = forward(steps)
        loss, pm, um = loss_rows(rows)
        g = np.zeros_like(rows)
        g[:, 0] = 2 * (um + 5.0) / (n * steps)
        g[:, 1] = 2 * (pm - 1.0) / (3 * vol * steps)
        g[:, 2] = 2 * (pm - 1.0) * (n / vol) * 2 / (dof * steps)
        d_eps, d_sig, _, _ = traj.backward(g)
        entry = {"steps": steps, "loss": loss, "d_epsilon": d_eps, "d_sigma": d_sig, "fd": []}
        for h in hs:
            fe = (loss_rows(forward(steps, eps=1 + h)[0])[0] -
                  loss_rows(forward(steps, eps=1 - h)[0])[0]) / (2 * h)
            fs = (loss_rows(forward(steps, sigma=1 + h)[0])[0] -
                  loss_rows(forward(steps, sigma=1 - h)[0])[0]) / (2 * h)
            entry["fd"].append({"h": h, "fd_epsilon": fe, "fd_sigma": fs,
                                "rel_err_epsilon": abs(d_eps - fe) / abs(fe),
                                "rel_err_sigma": abs(d_sig - fs) / abs(fs)})
        entry["best_rel_err_epsilon"] = min(f["rel_err_epsilon"] for f in entry["fd"])
        entry["best_rel_err_sigma"] = min(f["rel_err_sigma"] for f in entry["fd"])
        table.append(entry)
    if rank == 0:
        print(json.dumps({"adjoint_sweep": table, "config": adjoint_config(1000, every, skin)}),
              flush=True)
    group.close()
    return 0


def run_adjoint_arm(args):
    world, rank, local = dist_env()
    group = Group(world)
    steps, every, skin = args.steps, 50, args.adj_skin
    if args.impl == "reference":
        if rank == 0:
            import oracle as O
            st = O.fcc_lattice(20, RHO, TEMP, SEED)
            nsteps = max(1, min(args.steps, args.ref_steps))
            kind, value, _ = cpu_reference(st["pos"], st["vel"], st["box"], nsteps, 1)
            print(json.dumps({
                "metric": ADJ_METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * 32000 / value,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded fcc lattice)",
                "config": adjoint_config(steps, every, skin), "impl": "reference",
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": kind,
                                 "sample": f"{nsteps} reference NVE VV steps (the forward only: "
                                           f"the reference has no backward) of the 32000-atom "
                                           f"lattice, 1 thread ({cpu_model()})"},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}), flush=True)
        group.close()
        return 0
    import moleculardynamics_b200 as md
    ctx = md.Context(local)
    st = md.fcc_lattice(20, RHO, TEMP, SEED)
    pos, vel, mass, box = st["pos"], st["vel"], st["mass"], st["box"]
    n, vol = pos.shape[0], float(np.prod(box))
    dof = 3 * n - 3
    L = md.lib()

    def loss_rows(rows):
        p = n / vol * 2 * rows[:, 2] / dof + rows[:, 1] / (3 * vol)
        u = rows[:, 0] / n
        return (p.mean() - 1.0) ** 2 + (u.mean() + 5.0) ** 2, p.mean(), u.mean()

    def run_forward(sigma=1.0, eps=1.0, timed=False):
        s = md.System.from_arrays(pos, box, vel=vel, mass=mass, ctx=ctx)
        traj = md.AdjointTrajectory(ctx)
        lj = md.LennardJones(sigma, eps, RC, md.Truncation.LinearForceShift)
        ms = C.c_double()
        md._check(L.md_context_span_begin(ctx.handle))
        rows = traj.forward(s, lj, DT, steps, every, skin)
        md._check(L.md_context_span_end(ctx.handle, C.byref(ms)))
        return rows, traj, s, ms.value

    run_forward()  # warm-up: allocations, module load
    if args.adj_sweep:
        return adjoint_sweep(md, ctx, pos, vel, mass, box, every, skin, group, rank)
    rows, traj, s, fwd_ms = run_forward(timed=True)
    loss, pm, um = loss_rows(rows)
    g = np.zeros_like(rows)
    g[:, 0] = 2 * (um + 5.0) / (n * steps)
    g[:, 1] = 2 * (pm - 1.0) / (3 * vol * steps)
    g[:, 2] = 2 * (pm - 1.0) * (n / vol) * 2 / (dof * steps)
    ms = C.c_double()
    md._check(L.md_context_span_begin(ctx.handle))
    d_eps, d_sig, gx, gv = traj.backward(g)
    md._check(L.md_context_span_end(ctx.handle, C.byref(ms)))
    bwd_ms = ms.value
    def fd(h):
        e = (loss_rows(run_forward(eps=1 + h)[0])[0] - loss_rows(run_forward(eps=1 - h)[0])[0]) / (2 * h)
        s_ = (loss_rows(run_forward(sigma=1 + h)[0])[0] -
              loss_rows(run_forward(sigma=1 - h)[0])[0]) / (2 * h)
        return e, s_

    fd_eps, fd_sig = fd(1e-6)
    fd_eps9, fd_sig9 = fd(1e-9)
    total_ms = group.reduce(fwd_ms + bwd_ms, "max")
    value = world * n * steps / (total_ms * 1e-3)
    if rank == 0:
        line = {
            "metric": ADJ_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
            "warmup": 1, "ms_per_step": total_ms / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded fcc lattice, Maxwell-Boltzmann velocities",
            "config": adjoint_config(steps, every, skin),
            "forward_ms": fwd_ms, "backward_ms": bwd_ms, "backward_over_forward": bwd_ms / fwd_ms,
            "loss": loss,
            "grad": {"d_epsilon": d_eps, "d_sigma": d_sig,
                     "fd_epsilon": fd_eps, "fd_sigma": fd_sig,
                     "rel_err_epsilon": abs(d_eps - fd_eps) / abs(fd_eps),
                     "rel_err_sigma": abs(d_sig - fd_sig) / abs(fd_sig),
                     "fd_step": "central, h = 1e-6 relative",
                     "fd_h1e-9": {"fd_epsilon": fd_eps9, "fd_sigma": fd_sig9,
                                  "rel_err_epsilon": abs(d_eps - fd_eps9) / abs(fd_eps9),
                                  "rel_err_sigma": abs(d_sig - fd_sig9) / abs(fd_sig9)},
                     "d_x0_norm": float(np.linalg.norm(gx))},
        }
        if world == 1 and not args.no_cpu:
            kind, cval, _ = cpu_reference(pos, vel, box, max(1, args.cpu_steps) * 4, 1)
            line["cpu_baseline"] = {"value": cval, "unit": UNIT, "cores": 1, "kind": kind,
                                    "sample": f"{max(1, args.cpu_steps) * 4} reference NVE VV "
                                              f"steps (forward only) of the same 32000-atom state, "
                                              f"1 thread ({cpu_model()})"}
        print(json.dumps(line), flush=True)
    group.close()
    return 0


# ---------------------------------------------------------------- water workload
WATER_METRIC = "site-steps/s, 4096 rigid SPC/E molecules, Ewald, Nose-Hoover 298 K, 1 B200"
WATER_ALPHA, WATER_KMAX, WATER_RC, WATER_L = 0.34, 18, 10.0, 49.72
TAU_PS = 1.0966875353  # internal time unit in ps (core/units.hpp:33)


def water_config(steps):
    return {"workload": f"4096 rigid SPC/E molecules (12,288 sites) on a seeded random-orientation "
                        f"lattice at 0.997 g/cm^3, L={WATER_L} A; Ewald rc={WATER_RC} A, "
                        f"alpha={WATER_ALPHA}/A, kmax={WATER_KMAX} (half space |n|^2 < kmax^2+2); "
                        f"O-O LJ truncated + tail; RATTLE velocity Verlet + Nose-Hoover chain "
                        f"(M=3, tau=0.1 ps) at 298 K, dt=2 fs, {steps} steps after equilibration",
            "sites": 12288, "precision": "FP64 (real and reciprocal space)",
            "parallelism": "one system"}


def run_water_arm(args):
    world, rank, local = dist_env()
    group = Group(world)
    import moleculardynamics_b200 as md
    fs = lambda x: x * 1e-3 / TAU_PS
    w = md.water_lattice(16, WATER_L, SEED)
    if args.impl == "reference" or (rank == 0 and not args.no_cpu):
        import oracle as O
        q = np.array([-0.8476 if t == "O" else 0.4238 for t in w["types"]])
        mol = np.arange(len(w["types"])) // 3
        t0 = time.perf_counter()
        O.spce(w["pos"], w["box"], q, mol, cutoff=WATER_RC, kmax=WATER_KMAX, alpha=WATER_ALPHA)
        cpu_sec = time.perf_counter() - t0
        cpu = {"value": 12288 / cpu_sec, "unit": "site-steps/s", "cores": 1, "kind": "port",
               "sample": "one SPC/E force evaluation (the oracle's C restatement of "
                         "SpceForceField with the alpha override, brute-force real space) on the "
                         f"12,288-site lattice, 1 thread ({cpu_model()}); forces only, no step"}
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({
                    "metric": WATER_METRIC, "value": cpu["value"], "unit": "site-steps/s",
                    "n_gpus": args.gpus, "steps": 1, "warmup": 0, "ms_per_step": 1e3 * cpu_sec,
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                    "dtype": "f64", "data": "synthetic water lattice", "config": water_config(1),
                    "impl": "reference", "cpu_baseline": cpu,
                    "e2e": {"value": cpu["value"], "unit": "site-steps/s",
                            "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)
            group.close()
            return 0
    ctx = md.Context(local)
    s = md.build_spce_system(w["pos"], w["types"], w["box"], ctx=ctx)
    m = s.masses
    rng = np.random.default_rng(SEED)
    s.velocities = np.sqrt(298.0 / m)[:, None] * rng.normal(size=(s.n, 3))
    s.remove_center_of_mass_motion()
    rw = md.RigidWater(1.0, 109.47, settle=args.settle)
    rw.constrain_velocities(s)
    ff = md.SpceForceField(cutoff=WATER_RC, kmax=WATER_KMAX, alpha=WATER_ALPHA, ctx=ctx)
    if args.pme > 0:
        ff.set_pme_spacing(w["box"], args.pme, args.pme_order)
    if args.mixed:
        ff.set_precision(md.PRECISION_MIXED)
    recip = ("smooth PME, grid %dx%dx%d, B-spline order %d" % (*ff.pme_grid()[0], args.pme_order)
             if args.pme > 0 else f"Ewald k-vector sums, kmax={WATER_KMAX}")
    dof = md.RigidWater.degrees_of_freedom(4096, True)
    md.ConstrainedNoseHooverChain(fs(0.5), rw, 298.0, fs(50.0), 3, dof).run(s, ff, args.equil_water)
    integ = md.ConstrainedNoseHooverChain(fs(2.0), rw, 298.0, fs(100.0), 3, dof)
    integ.run(s, ff, args.warmup)
    L = md.lib()
    launches0 = ctx.launch_count()
    clocks = ClockSampler(local)
    clocks.__enter__()
    ms = C.c_double()
    md._check(L.md_context_span_begin(ctx.handle))
    th = integ.run(s, ff, args.steps, thermo=True)
    md._check(L.md_context_span_end(ctx.handle, C.byref(ms)))
    clocks.__exit__(None, None, None)
    launches = ctx.launch_count() - launches0
    dev_ms = group.reduce(ms.value, "max")
    value = world * 12288 * args.steps / (dev_ms * 1e-3)
    h = th[:, 0] + th[:, 2] + th[:, 3]
    # reciprocal truncation: forces at kmax against kmax + 8 on the final state
    f_ref = None
    ff.compute_forces(s)
    f_run = s.forces
    md.SpceForceField(cutoff=WATER_RC, kmax=WATER_KMAX + 8, alpha=WATER_ALPHA, ctx=ctx).compute_forces(s)
    f_ref = s.forces
    ferr = float(np.sqrt(np.sum((f_run - f_ref) ** 2) / np.sum(f_ref ** 2)))
    if rank == 0:
        line = {
            "metric": WATER_METRIC, "value": value, "unit": "site-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded rigid-water lattice, Maxwell-Boltzmann velocities, "
                    f"{args.equil_water} NHC steps of 0.5 fs",
            "config": dict(water_config(args.steps),
                           constraints="SETTLE" if args.settle else "SHAKE/RATTLE",
                           reciprocal=recip,
                           precision=("FP32 real-space pair terms, FP64 displacements, "
                                      "reciprocal space and sums" if args.mixed
                                      else "FP64 (real and reciprocal space)")),
            "gpu_launches": int(launches),
            "nhc_extended_energy_drift_K": {"max_abs": float(np.max(np.abs(h - h[0]))),
                                            "relative": float(np.max(np.abs(h - h[0])) / abs(h[0]))},
            "mean_temperature_K": float(np.mean(2 * th[:, 2] / dof)),
            "force_rel_rms_vs_kmax+8": ferr,
            "clocks": clocks.summary(),
        }
        if world == 1 and not args.no_cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    group.close()
    return 0


# ------------------------------------------------------------- water_rdf protocol
WRDF_METRIC = ("site-steps/s, SPC/E water_rdf protocol: 300 rigid molecules (900 sites), "
               "15,000 + 10,000 steps, 1 B200")
WRDF_SITES, WRDF_EQUIL, WRDF_PROD, WRDF_SAMPLE = 900, 15000, 10000, 10
WRDF_PUBLISHED_SEC = 434.687  # the reference's recorded wall time for this protocol


def water_rdf_config(runs, equil=15000, prod=10000):
    return {"workload": "apps/water_rdf.cpp protocol: NIST SPC/E configuration 3 (300 molecules) "
                        "expanded rigidly to 0.997 g/cm^3 (L = 20.802 A); Ewald alpha=5.6/L, "
                        f"kmax=5, rc=10 A; RATTLE velocity Verlet, dt=2 fs; {equil:,} equilibration "
                        f"steps rescaled to 298 K every 50, {prod:,} NVE steps with an O-O RDF "
                        "(10 A, 200 bins) every 10; one bench step = the whole protocol",
            "sites": WRDF_SITES, "protocol_runs": runs, "precision": "FP64",
            "l2_policy": "no flush: the working set (about 2 MB) is L2-resident by design",
            "parallelism": "replicas (one independent system per GPU)"}


def water_rdf_inputs():
    """NIST SPC/E configuration 3 (the reference's data file, carried as a test
    fixture) at the app's state point, with its Rng(7001) velocities."""
    from moleculardynamics_b200 import water_rdf as W
    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden",
                             "nist_spce.npz"))
    types = ["O" if o else "H" for o in d["isO3"]]
    return d["pos3"], types, d["box3"]


def reference_water_rdf_rate(steps):
    """The reference's ConstrainedVelocityVerlet + SpceForceField (compiled from
    its sources) for `steps` steps of the protocol's state point, 1 thread."""
    import oracle as O
    from moleculardynamics_b200 import water_rdf as W
    pos, types, box = water_rdf_inputs()
    pos, types, box, _ = W.state_point(pos, types, box)
    m = np.array([15.9994 if t == "O" else 1.008 for t in types])
    q = np.array([-0.8476 if t == "O" else 0.4238 for t in types])
    vel = W.thermal_velocities(m, 298.0, 7001)
    R = O.ref()
    if R is None:
        return None
    cols = [np.ascontiguousarray(a[:, k]) for a in (pos, vel) for k in range(3)]
    f = [np.zeros(len(m)) for _ in range(3)]
    mol = (np.arange(len(m)) // 3).astype(np.int64)
    p = O._p
    t0 = time.perf_counter()
    R.ref_spce_cvv(len(m), p(box), *[p(c) for c in cols], *[p(c) for c in f], p(m), p(q),
                   mol.ctypes.data_as(C.POINTER(C.c_int64)), 10.0, 5, 2e-3 / TAU_PS, int(steps))
    sec = time.perf_counter() - t0
    return WRDF_SITES * steps / sec, sec


def run_water_rdf_arm(args):
    world, rank, local = dist_env()
    group = Group(world)
    cpu = None
    if args.impl == "reference" or (rank == 0 and world == 1 and not args.no_cpu):
        if rank == 0:
            steps = max(args.ref_steps, 1)
            got = reference_water_rdf_rate(steps)
            if got is not None:
                rate, sec = got
                cpu = {"value": rate, "unit": "site-steps/s", "cores": 1, "kind": "reference",
                       "sample": f"{steps} constrained steps (+1 priming force call) of the "
                                 f"protocol's state point through the reference's "
                                 f"ConstrainedVelocityVerlet and SpceForceField, compiled from "
                                 f"its sources ({sec:.2f} s, 1 thread, {cpu_model()}); no RDF"}
        if args.impl == "reference":
            if rank == 0:
                if cpu is None:
                    print(json.dumps({"impl": "reference",
                                      "unavailable": "reference library not built"}), flush=True)
                else:
                    print(json.dumps({
                        "metric": WRDF_METRIC, "value": cpu["value"], "unit": "site-steps/s",
                        "n_gpus": args.gpus, "steps": 1, "warmup": 0,
                        "ms_per_step": 1e3 * WRDF_SITES * (WRDF_EQUIL + WRDF_PROD) / cpu["value"],
                        "higher_is_better": True, "scaling": "weak",
                        "vs_baseline": cpu["value"] / (WRDF_SITES * (WRDF_EQUIL + WRDF_PROD)
                                                        / WRDF_PUBLISHED_SEC),
                        "dtype": "f64", "data": "NIST SPC/E configuration 3 (reference data)",
                        "config": water_rdf_config(1), "impl": "reference", "cpu_baseline": cpu,
                        "e2e": {"value": cpu["value"], "unit": "site-steps/s",
                                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)
            group.close()
            return 0
    import moleculardynamics_b200 as md
    from moleculardynamics_b200 import water_rdf as W
    equil, prod = args.wrdf_steps
    ctx = md.Context(local)
    pos0, types0, box0 = water_rdf_inputs()
    pos, types, box, molecules = W.state_point(pos0, types0, box0)
    dof = md.RigidWater.degrees_of_freedom(molecules, True)
    s = md.build_spce_system(pos, types, box, ctx=ctx)
    m = s.masses
    v0 = W.thermal_velocities(m, 298.0, 7001)
    rigid = md.RigidWater(1.0, 109.47, settle=args.settle)
    ff = md.SpceForceField(ctx=ctx)
    L = md.lib()
    mean_t = C.c_double()

    def protocol(rdf):
        integ = md.ConstrainedVelocityVerlet(md.units.femtoseconds(2.0), rigid)
        s.positions = pos
        s.velocities = v0
        s.remove_center_of_mass_motion()
        rigid.constrain_velocities(s)
        ctx.synchronize()
        l0 = ctx.launch_count()
        ms = C.c_double()
        md._check(L.md_context_span_begin(ctx.handle))
        md._check(L.md_water_rdf_run(integ.handle, s.handle, ff.handle, rdf.handle, 298.0, dof,
                                     equil, 50, prod, WRDF_SAMPLE, C.byref(mean_t)))
        md._check(L.md_context_span_end(ctx.handle, C.byref(ms)))
        return ms.value, ctx.launch_count() - l0

    for _ in range(args.warmup):
        protocol(md.Rdf(10.0, 200, ctx=ctx))
    ctx.synchronize()
    group.barrier()
    # the timed region: the fused protocol alone (state reset outside it)
    total_ms, launches = 0.0, 0
    clocks = ClockSampler(local)
    clocks.__enter__()
    rdf = md.Rdf(10.0, 200, ctx=ctx)
    for _ in range(args.steps):
        ms, n_launch = protocol(rdf)  # state reset and synchronised before the span
        total_ms += ms
        launches += n_launch
    clocks.__exit__(None, None, None)
    dev_ms = group.reduce(total_ms, "max")
    md_steps = equil + prod
    value = world * WRDF_SITES * md_steps * args.steps / (dev_ms * 1e-3)
    # end to end through the public API: host arrays in, the finished g(r) out
    group.barrier()
    t0 = time.perf_counter()
    res = W.run(pos0, types0, box0, equilibrate=equil, production=prod, settle=args.settle,
                ctx=ctx)
    e2e_sec = group.reduce(time.perf_counter() - t0, "max")
    g = rdf.g()
    r = rdf.bin_centres()
    peak = W.first_peak(r, g)
    if rank == 0:
        peaks, peak_src = measured_peaks()
        us_step = 1e3 * dev_ms / (args.steps * md_steps)
        # algorithmic bytes of a step: each site's position, velocity and force
        # read and position and velocity written by the two halves (5 x 24 B),
        # plus position and charge read by the force pass (32 B)
        alg = 152.0 * WRDF_SITES
        achieved = alg / (us_step * 1e-6) / 1e9
        h2d = sum(a.nbytes for a in (pos0, box0)) + 8 * 900 * 5  # positions, box; m, q, mol, v
        line = {
            "metric": WRDF_METRIC, "value": value, "unit": "site-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": value / world / (WRDF_SITES * (WRDF_EQUIL + WRDF_PROD)
                                            / WRDF_PUBLISHED_SEC),
            "dtype": "f64",
            "data": "NIST SPC/E configuration 3 (reference data file) at the app's state point, "
                    "Rng(7001) velocities",
            "config": dict(water_rdf_config(args.steps, equil, prod),
                           constraints="SETTLE" if args.settle else "SHAKE/RATTLE"),
            "gpu_launches": int(launches), "us_per_md_step": us_step,
            "launches_per_md_step": launches / (args.steps * md_steps),
            "result": {"mean_production_temperature_K": mean_t.value,
                       "first_peak_r_angstrom": peak[2], "first_peak_g": peak[3],
                       "tail_mean_g_beyond_8.5A": W.tail_mean(r, g), "rdf_frames": rdf.frames()},
            "e2e": {"value": world * WRDF_SITES * md_steps / e2e_sec, "unit": "site-steps/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": 8 * 200 * 3,
                    "wall_seconds": e2e_sec,
                    "path": "water_rdf.run: host configuration -> state point -> device system, "
                            "md_water_rdf_run, g(r) read back"},
            "roofline": {"bound": "hbm", "kernel": "whole MD step", "achieved": achieved,
                         "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                         "frac": achieved / peaks.get("hbm_gbs", 6650.0),
                         "peak_source": f"hbm_gbs of {peak_src}",
                         "algorithmic_bytes_per_site": 152.0, "traffic": None,
                         "note": "latency bound: 900 sites, about 2 MB of state and lists held "
                                 "in L2; the step is a chain of dependent launches"},
            "clocks": clocks.summary(),
        }
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    group.close()
    return 0


# ------------------------------------------------------------------ analysis
ANALYSIS_METRIC = "RDF frames/s, 1M-atom LJ liquid (rMax 4.0, 200 bins) on 1 B200"
RDF_RMAX, RDF_BINS, CORR_LAGS = 4.0, 200, 100


def analysis_config(steps):
    return {"workload": "radial distribution function of the equilibrated 1M-atom LJ liquid "
                        f"(fcc 64^3, rho*=0.8442): rMax {RDF_RMAX}, {RDF_BINS} bins, every pair "
                        "i<j counted (analyze/rdf.cpp); MSD and VACF pushes with "
                        f"{CORR_LAGS + 1} lags (analyze/msd.cpp, vacf.cpp)",
            "frames": steps, "n_atoms": 4 * CELLS ** 3,
            "l2_policy": "no flush: positions 32 MB, MSD/VACF rings 2.5 GB each > 126 MB L2",
            "parallelism": "replicas (one independent system per GPU)"}


def reference_rdf_rate(cells=20, frames=1):
    """The reference's Rdf (brute force, all pairs) on one seeded frame of a
    cells^3 fcc liquid, 1 thread: pair evaluations per second."""
    import oracle as O
    st = O.fcc_lattice(cells, RHO, TEMP, SEED)
    n = len(st["pos"])
    t0 = time.perf_counter()
    O.ref_rdf(st["pos"][None], st["box"], RDF_RMAX, RDF_BINS)
    sec = time.perf_counter() - t0
    return frames * n * (n - 1) / 2 / sec, n, sec


def run_analysis_arm(args):
    world, rank, local = dist_env()
    group = Group(world)
    n = 4 * CELLS ** 3
    pairs_1m = n * (n - 1) / 2
    cpu = None
    if args.impl == "reference" or (rank == 0 and world == 1 and not args.no_cpu):
        rate, n_s, sec = reference_rdf_rate()
        cpu = {"value": rate / pairs_1m, "unit": "frames/s", "cores": 1, "kind": "reference",
               "sample": f"the reference's Rdf::accumulate on one {n_s}-atom frame of the same "
                         f"liquid ({sec:.2f} s, {rate:.3g} pair evaluations/s), projected to the "
                         f"{n}-atom frame's {pairs_1m:.3g} pairs; 1 thread ({cpu_model()})"}
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({
                    "metric": ANALYSIS_METRIC, "value": cpu["value"], "unit": "frames/s",
                    "n_gpus": args.gpus, "steps": 1, "warmup": 0,
                    "ms_per_step": 1e3 / cpu["value"], "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                    "data": "synthetic: seeded fcc lattice", "config": analysis_config(1),
                    "impl": "reference", "cpu_baseline": cpu,
                    "e2e": {"value": cpu["value"], "unit": "frames/s", "h2d_bytes_per_step": 0,
                            "d2h_bytes_per_step": 0}}), flush=True)
            group.close()
            return 0
    import moleculardynamics_b200 as md
    ctx = md.Context(local)
    box, pos, vel, frc = equilibrated_state(md, ctx, args.equil)
    s = md.System.from_arrays(pos, box, vel=vel, ctx=ctx)
    L = md.lib()
    rdf = md.Rdf(RDF_RMAX, RDF_BINS, ctx=ctx)
    for _ in range(args.warmup):
        rdf.accumulate(s)
    ctx.synchronize()
    group.barrier()
    launches0 = ctx.launch_count()
    clocks = ClockSampler(local)
    clocks.__enter__()
    ms = C.c_double()
    md._check(L.md_context_span_begin(ctx.handle))
    for _ in range(args.steps):
        rdf.accumulate(s)
    md._check(L.md_context_span_end(ctx.handle, C.byref(ms)))
    clocks.__exit__(None, None, None)
    launches = ctx.launch_count() - launches0
    dev_ms = group.reduce(ms.value, "max")
    value = world * args.steps / (dev_ms * 1e-3)
    # MSD / VACF pushes with every lag available
    msd, vacf = md.Msd(n, CORR_LAGS, ctx=ctx), md.Vacf(n, CORR_LAGS, ctx=ctx)
    for _ in range(CORR_LAGS + 1):
        msd.push(s)
        vacf.push(s)
    t = {}
    for name, obj in (("msd", msd), ("vacf", vacf)):
        md._check(L.md_context_span_begin(ctx.handle))
        for _ in range(10):
            obj.push(s)
        md._check(L.md_context_span_end(ctx.handle, C.byref(ms)))
        t[name] = ms.value / 10
    # end to end through the public C ABI: positions from pinned host memory each
    # frame, the frame accumulated, g(r) read back
    hpos = [np.ascontiguousarray(pos[:, d]) for d in range(3)]
    g = np.zeros(RDF_BINS)
    e2e_frames = max(3, min(args.steps, 10))
    ctx.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_frames):
        for d, f in enumerate((md.FIELD_X, md.FIELD_X + 1, md.FIELD_X + 2)):
            md._check(L.md_system_set(s.handle, f, hpos[d].ctypes.data_as(C.POINTER(C.c_double))))
        md._check(L.md_rdf_accumulate(rdf._h, s.handle))
        md._check(L.md_rdf_g(rdf._h, g.ctypes.data_as(C.POINTER(C.c_double))))
    e2e_sec = group.reduce(time.perf_counter() - t0, "max")
    if rank == 0:
        peaks, peak_src = measured_peaks()
        # algorithmic bytes of a frame: every atom's position read once (32 B)
        achieved = 32.0 * n / (dev_ms / args.steps * 1e-3) / 1e9
        line = {
            "metric": ANALYSIS_METRIC, "value": value, "unit": "frames/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded fcc lattice, Maxwell-Boltzmann velocities, "
                    f"{args.equil} BAOAB equilibration steps",
            "config": analysis_config(args.steps), "gpu_launches": int(launches),
            "pairs_within_rmax_per_frame": float(rdf.histogram().sum() / rdf.frames()),
            "msd_push_ms": t["msd"], "vacf_push_ms": t["vacf"],
            "e2e": {"value": world * e2e_frames / e2e_sec, "unit": "frames/s",
                    "h2d_bytes_per_step": 24 * n, "d2h_bytes_per_step": 8 * RDF_BINS,
                    "path": "md_system_set x3 (host positions) + md_rdf_accumulate + md_rdf_g "
                            "per frame"},
            "roofline": {"bound": "hbm", "kernel": "k_rdf_cells", "achieved": achieved,
                         "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                         "frac": achieved / peaks.get("hbm_gbs", 6650.0),
                         "peak_source": f"hbm_gbs of {peak_src}",
                         "algorithmic_bytes_per_atom": 32.0, "traffic": None,
                         "note": "FP64 pair arithmetic (exact fold, sqrt, divide) bounds it"},
            "clocks": clocks.summary(),
        }
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    group.close()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--workload", default="lj1m",
                    choices=["lj1m", "batch", "adjoint", "water", "analysis", "water_rdf"],
                    help="lj1m: the headline 1M-atom run; batch: 48 NHC replicas; adjoint: "
                         "forward + backward of a 32,000-atom differentiable trajectory "
                         "(--steps is its length)")
    ap.add_argument("--adj-skin", type=float, default=2.0)
    ap.add_argument("--adj-sweep", action="store_true",
                    help="adjoint: the gradient against central differences over trajectory "
                         "lengths and difference steps (a table, not the benchmark line)")
    ap.add_argument("--equil-water", type=int, default=1000)
    ap.add_argument("--settle", action="store_true",
                    help="water: SETTLE instead of SHAKE/RATTLE iterations")
    ap.add_argument("--wrdf-steps", type=int, nargs=2, default=[WRDF_EQUIL, WRDF_PROD],
                    metavar=("EQUIL", "PROD"),
                    help="water_rdf: protocol lengths (profiling configurations only; the "
                         "metric is quoted on the default 15000 10000)")
    ap.add_argument("--pme", type=float, default=0.0, metavar="SPACING",
                    help="water: smooth PME with grid cells of at most SPACING A instead of "
                         "the k-vector sums")
    ap.add_argument("--pme-order", type=int, default=6)
    ap.add_argument("--mixed", action="store_true",
                    help="water: FP32 real-space pair terms (FP64 displacements and sums)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--equil", type=int, default=2000,
                    help="BAOAB steps on the GPU when the reference-equilibrated state is "
                         "absent or --gpu-equil is given")
    ap.add_argument("--cells", type=int, default=CELLS,
                    help="fcc cells per side (profiling configurations only; the metric is "
                         "quoted on 64)")
    ap.add_argument("--tile-threads", type=int, default=0,
                    help="mixed tile kernel shape (md_lj_set_tile_threads; profiling)")
    ap.add_argument("--gpu-equil", action="store_true",
                    help="equilibrate on the GPU instead of loading the reference's state")
    ap.add_argument("--drift-steps", type=int, default=None,
                    help="length of the drift runs after the timed region: the NVE window in "
                         "both precisions (lj1m, default 10000) or the per-replica NHC table "
                         "(batch, default 5000); 0 skips them")
    ap.add_argument("--tpa", type=int, default=2)
    ap.add_argument("--unroll", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--cpu-steps", type=int, default=5)
    ap.add_argument("--ref-steps", type=int, default=10)
    ap.add_argument("--ref-procs", type=int, default=8)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--precision", default="both", choices=["both", "mixed", "fp64"],
                    help="'mixed'/'fp64' run only that timed loop and print nothing "
                         "(profiling configuration)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.workload == "batch":
        return run_batch_arm(args)
    if args.workload == "adjoint":
        return run_adjoint_arm(args)
    if args.workload == "water":
        return run_water_arm(args)
    if args.workload == "analysis":
        return run_analysis_arm(args)
    if args.workload == "water_rdf":
        return run_water_rdf_arm(args)
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
