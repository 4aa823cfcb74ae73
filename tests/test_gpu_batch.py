"""Replica batches: every replica of a batch run follows exactly the trajectory
md_run_lj gives it alone (same kernels, same arguments, replayed as independent
chains of one CUDA graph per step)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (cells, density, temperature, seed, integrator): a 2-cells-per-side replica
# (brute-force list build), a dilute gas, dense liquids, a mixed-precision one
REPLICAS = [(4, 0.9, 1.3, 11, "nhc", 0), (5, 0.1, 1.8, 12, "nhc", 0), (6, 0.8, 1.0, 13, "vv", 0),
            (8, 0.5, 1.5, 14, "nhc", 1), (7, 0.3, 2.0, 15, "vv", 0)]


def replica(md, cells, rho, temp, seed, kind, prec, chain=3):
    ctx = md.Context(0)
    st = md.fcc_lattice(cells, rho, temp, seed)
    s = md.System.from_arrays(st["pos"], st["box"], vel=st["vel"], mass=st["mass"], ctx=ctx)
    lj = md.LennardJones(1.0, 1.0, 2.5, precision=prec)
    v = md.VerletList(st["box"], 2.5, 0.3, ctx=ctx)
    v.build(s)
    lj.compute_forces(s, v)
    integ = (md.NoseHooverChain(0.005, temp, 0.5, chain, 3 * s.n - 3) if kind == "nhc"
             else md.VelocityVerlet(0.005))
    return ctx, s, v, lj, integ


def test_batch_equals_replicas_run_alone(md):
    steps = 80
    alone = []
    for r in REPLICAS:
        ctx, s, v, lj, integ = replica(md, *r)
        th = integ.run(s, v, lj, steps, thermo=True)
        alone.append((s.positions, s.velocities, th, v.rebuild_count()))
    batch = md.Batch()
    parts = [replica(md, *r) for r in REPLICAS]
    for ctx, s, v, lj, integ in parts:
        batch.add(integ, s, v, lj)
    assert len(batch) == len(REPLICAS)
    th = batch.run(steps, thermo=True)
    assert th.shape == (len(REPLICAS), steps, 4)
    for k, (ctx, s, v, lj, integ) in enumerate(parts):
        pos, vel, th_alone, rebuilds = alone[k]
        assert np.array_equal(s.positions, pos), k
        assert np.array_equal(s.velocities, vel), k
        assert np.array_equal(th[k], th_alone), k
        assert v.rebuild_count() == rebuilds, k
    assert sum(alone[k][3] for k in range(len(REPLICAS))) > len(REPLICAS)


def test_batch_rejects_shared_context_and_langevin(md):
    ctx, s, v, lj, integ = replica(md, 4, 0.8, 1.0, 3, "vv", 0)
    batch = md.Batch()
    batch.add(integ, s, v, lj)
    st = md.fcc_lattice(4, 0.8, 1.0, 4)
    s2 = md.System.from_arrays(st["pos"], st["box"], vel=st["vel"], ctx=ctx)
    v2 = md.VerletList(st["box"], 2.5, 0.3, ctx=ctx)
    v2.build(s2)
    with pytest.raises(md.InvalidArgument, match="own context"):
        batch.add(md.VelocityVerlet(0.005), s2, v2, lj)
    ctx3, s3, v3, lj3, _ = replica(md, 4, 0.8, 1.0, 5, "vv", 0)
    with pytest.raises(md.InvalidArgument, match="Nose-Hoover"):
        batch.add(md.LangevinBAOAB(0.005, 1.0, 1.0, 7), s3, v3, lj3)


@pytest.mark.parametrize("prec", [0, 1])
def test_batched_stage_kernels_equal_solo_runs(md, prec):
    """Replicas that share one force kernel (same precision, cubic boxes) step
    through the batched stage kernels -- one launch per stage for all replicas,
    blocks mapped to replicas through a per-block table, the rebuild stages
    gated per replica (here with a brute-force build beside the cell builds).
    Each replica still follows its solo trajectory bit for bit, as with the
    per-replica graph, with a fraction of the launches."""
    reps = [(4, 0.9, 1.3, 21, "nhc", prec), (5, 0.1, 1.8, 22, "nhc", prec),
            (6, 0.8, 1.0, 23, "vv", prec), (7, 0.5, 1.5, 24, "nhc", prec),
            (3, 0.8, 1.0, 25, "vv", prec)]  # the last: 2 cells per side, brute-force builds
    steps = 80
    alone = []
    for r in reps:
        ctx, s, v, lj, integ = replica(md, *r)
        th = integ.run(s, v, lj, steps, thermo=True)
        alone.append((s.positions, s.velocities, th, v.rebuild_count()))
    launches = {}
    for batched in (True, False):
        batch = md.Batch()
        parts = [replica(md, *r) for r in reps]
        for ctx, s, v, lj, integ in parts:
            batch.add(integ, s, v, lj)
        batch.set_batched(batched)
        before = sum(p[0].launch_count() for p in parts)
        th = batch.run(steps, thermo=True)
        launches[batched] = sum(p[0].launch_count() for p in parts) - before
        for k, (ctx, s, v, lj, integ) in enumerate(parts):
            pos, vel, th_alone, rebuilds = alone[k]
            assert np.array_equal(s.positions, pos), (batched, k)
            assert np.array_equal(s.velocities, vel), (batched, k)
            assert np.array_equal(th[k], th_alone), (batched, k)
            assert v.rebuild_count() == rebuilds, (batched, k)
    assert sum(a[3] for a in alone) > len(reps)
    assert launches[True] * 2 < launches[False]


@pytest.mark.parametrize("prec", [0, 1])
def test_batched_rebuild_stages_equal_solo_runs(md, prec):
    """Replicas whose cell grids all have 3 or more cells per side also rebuild
    through batched stage kernels: one launch per stage of the counting sort, the
    re-sort, the list build and the reference positions for every replica, each
    replica's blocks leaving at once unless its own displacement test asked for a
    rebuild -- no conditional node in the step graph.  Each replica still follows
    its solo trajectory bit for bit, rebuilding at the same steps."""
    reps = [(5, 0.8, 1.0, 31, "vv", prec), (5, 0.1, 1.8, 32, "nhc", prec),
            (6, 0.9, 1.3, 33, "nhc", prec), (7, 0.5, 1.5, 34, "nhc", prec),
            (8, 0.8, 1.0, 35, "vv", prec)]
    steps = 80
    alone = []
    for r in reps:
        ctx, s, v, lj, integ = replica(md, *r)
        assert min(v.cells_per_side()) >= 3
        th = integ.run(s, v, lj, steps, thermo=True)
        alone.append((s.positions, s.velocities, th, v.rebuild_count()))
    launches = {}
    for batched in (True, False):
        batch = md.Batch()
        parts = [replica(md, *r) for r in reps]
        for ctx, s, v, lj, integ in parts:
            batch.add(integ, s, v, lj)
        batch.set_batched(batched)
        before = sum(p[0].launch_count() for p in parts)
        th = batch.run(steps, thermo=True)
        launches[batched] = sum(p[0].launch_count() for p in parts) - before
        for k, (ctx, s, v, lj, integ) in enumerate(parts):
            pos, vel, th_alone, rebuilds = alone[k]
            assert np.array_equal(s.positions, pos), (batched, k)
            assert np.array_equal(s.velocities, vel), (batched, k)
            assert np.array_equal(th[k], th_alone), (batched, k)
            assert v.rebuild_count() == rebuilds, (batched, k)
    assert sum(a[3] for a in alone) > len(reps)
    assert launches[True] < launches[False]


def test_batch_graph_kept_across_runs(md):
    """A second run of the same batch replays the step graph the first one built
    (the run's first step still goes from the host, as md_run_lj's does); both
    runs follow the replicas' solo calls bit for bit."""
    reps = [(5, 0.8, 1.0, 41, "vv", 1), (6, 0.1, 1.8, 42, "nhc", 1), (7, 0.9, 1.3, 43, "nhc", 1)]
    alone = []
    for r in reps:
        ctx, s, v, lj, integ = replica(md, *r)
        th1 = integ.run(s, v, lj, 30, thermo=True)
        th2 = integ.run(s, v, lj, 50, thermo=True)
        alone.append((s.positions, s.velocities, th1, th2))
    batch = md.Batch()
    parts = [replica(md, *r) for r in reps]
    for ctx, s, v, lj, integ in parts:
        batch.add(integ, s, v, lj)
    th1 = batch.run(30, thermo=True)
    th2 = batch.run(50, thermo=True)
    for k, (ctx, s, v, lj, integ) in enumerate(parts):
        pos, vel, a1, a2 = alone[k]
        assert np.array_equal(th1[k], a1), k
        assert np.array_equal(th2[k], a2), k
        assert np.array_equal(s.positions, pos), k
        assert np.array_equal(s.velocities, vel), k


def test_batched_chains_of_any_length_equal_solo_runs(md):
    """Nose-Hoover replicas with chains of 1, 3 and 5 links in one batched run (the
    three-link chain's halves run in registers, other lengths through the general
    path), beside a velocity-Verlet replica: each follows its solo trajectory and
    thermo rows bit for bit, over a first run and a second that replays the cached
    graphs."""
    reps = [((5, 0.8, 1.0, 51, "nhc", 1), 1), ((6, 0.3, 1.5, 52, "nhc", 1), 3),
            ((7, 0.9, 1.2, 53, "nhc", 1), 5), ((5, 0.5, 1.8, 54, "vv", 1), 3)]
    alone = []
    for r, chain in reps:
        ctx, s, v, lj, integ = replica(md, *r, chain=chain)
        th1 = integ.run(s, v, lj, 30, thermo=True)
        th2 = integ.run(s, v, lj, 50, thermo=True)
        alone.append((s.positions, s.velocities, th1, th2))
    batch = md.Batch()
    parts = [replica(md, *r, chain=chain) for r, chain in reps]
    for ctx, s, v, lj, integ in parts:
        batch.add(integ, s, v, lj)
    th1 = batch.run(30, thermo=True)
    th2 = batch.run(50, thermo=True)
    for k, (ctx, s, v, lj, integ) in enumerate(parts):
        pos, vel, a1, a2 = alone[k]
        assert np.array_equal(th1[k], a1), k
        assert np.array_equal(th2[k], a2), k
        assert np.array_equal(s.positions, pos), k
        assert np.array_equal(s.velocities, vel), k
