"""Halo tiles of the mixed-precision Verlet force kernel.

Reading a neighbour through a tile staged in shared memory (16-bit slots; in cubic
boxes the persistent double-buffered tile kernel) or gathering it through the
int32 row sums the same pairs -- those next to the cutoff are decided exactly in
both -- with FP32 pair terms, in a different order.  So both paths stay within the
mixed-precision error budget of the FP64 path and agree with each other to FP32
rounding; each is deterministic.  Covered: a liquid where every tile is staged, a
dilute gas where none is (a block of 128 atoms spans more than 16 cells),
two-phase boxes where both kinds occur in one launch (cubic and not), the
linear-force-shift truncation, and a fused run with neighbour rebuilds inside the
replayed step graph, bit-identical to the same steps launched from the host.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def melt(md, cells, rho, seed, steps=100):
    st = md.fcc_lattice(cells, rho, 0.722, seed)
    s = md.System.from_arrays(st["pos"], st["box"], vel=st["vel"], mass=st["mass"])
    lj = md.LennardJones(1.0, 1.0, 2.5)
    v = md.VerletList(st["box"], 2.5, 0.3)
    v.build(s)
    lj.compute_forces(s, v)
    md.LangevinBAOAB(0.005, 1.0, 0.722, seed).run(s, v, lj, steps)
    return s, v, st


def rms_rel(f, ref):
    return float(np.sqrt(np.sum((f - ref) ** 2) / np.sum(ref ** 2)))


def three_ways(md, s, v, trunc=0):
    """(FP64, mixed gathered, mixed over tiles): each (energy, virial, forces)."""
    e64, w64 = md.LennardJones(1.0, 1.0, 2.5, trunc).compute_forces(s, v)
    f64 = s.forces
    on = md.LennardJones(1.0, 1.0, 2.5, trunc, precision=md.PRECISION_MIXED)
    off = md.LennardJones(1.0, 1.0, 2.5, trunc, precision=md.PRECISION_MIXED)
    off.set_halo(False)
    e0, w0 = off.compute_forces(s, v)
    f0 = s.forces
    v.set_halo(True)
    e1, w1 = on.compute_forces(s, v)
    f1 = s.forces
    e2, w2 = on.compute_forces(s, v)  # deterministic: a second launch repeats it
    assert np.array_equal(s.forces, f1) and e2 == e1 and w2 == w1
    return (e64, w64, f64), (e0, w0, f0), (e1, w1, f1)


def check_budget(ref, gathered, tiled, e_tol=1e-7):
    """Forces within 1e-6 RMS of FP64; energy and virial, summed from FP32 terms,
    within e_tol and 3e-6 relative (e_tol is looser for the gas boxes, whose
    overlapping atoms give pair energies of 1e4)."""
    (e64, w64, f64), (e0, w0, f0), (e1, w1, f1) = ref, gathered, tiled
    for e, w, f in ((e0, w0, f0), (e1, w1, f1)):
        assert rms_rel(f, f64) < 1e-6, rms_rel(f, f64)
        assert abs(e - e64) < e_tol * abs(e64) and abs(w - w64) < 3e-6 * abs(w64), (e, e64, w, w64)
    assert rms_rel(f1, f0) < 1e-6
    assert abs(e1 - e0) < e_tol * abs(e64) and abs(w1 - w0) < 3e-6 * abs(w64)


@pytest.mark.parametrize("trunc", [0, 1])
def test_liquid_tiles_staged_within_budget(md, trunc):
    s, v, _ = melt(md, 12, 0.8442, 3)  # 6912 atoms
    ref, gathered, tiled = three_ways(md, s, v, trunc)
    staged, tiles = v.halo_tiles()
    assert tiles == (s.n + 127) // 128 and staged == tiles
    check_budget(ref, gathered, tiled)


def test_dilute_gas_falls_back_within_budget(md):
    st = md.fcc_lattice(10, 0.02, 1.5, 4)  # 4000 atoms, ~0.4 per cell
    s = md.System.from_arrays(st["pos"], st["box"], vel=st["vel"], mass=st["mass"])
    v = md.VerletList(st["box"], 2.5, 0.3)
    v.build(s)
    rng = np.random.default_rng(4)
    s.positions = st["pos"] + rng.normal(0, 0.5, st["pos"].shape)
    v.build(s)
    ref, gathered, tiled = three_ways(md, s, v)
    staged, tiles = v.halo_tiles()
    assert tiles > 0 and staged == 0
    check_budget(ref, gathered, tiled, e_tol=1e-6)


def test_two_phase_box_mixes_staged_and_gathered_tiles(md):
    # a dense slab and a dilute gas in one box (not cubic: the single-buffer kernel)
    st = md.fcc_lattice(12, 0.8442, 0.722, 5)
    pos = st["pos"].copy()
    box = st["box"].copy()
    box[2] *= 3.0
    rng = np.random.default_rng(5)
    gas = rng.uniform(-0.5, 0.5, size=(300, 3)) * box
    gas[:, 2] = np.where(gas[:, 2] > 0, gas[:, 2] * 0.5 + box[2] / 4, gas[:, 2] * 0.5 - box[2] / 4)
    pos = np.concatenate([pos, gas])  # gas at |z| > 0.75 Lz, the slab at |z| < 0.5 Lz
    s = md.System.from_arrays(pos, box, vel=np.zeros_like(pos), mass=np.ones(len(pos)))
    v = md.VerletList(box, 2.5, 0.3)
    v.build(s)
    ref, gathered, tiled = three_ways(md, s, v)
    staged, tiles = v.halo_tiles()
    assert 0 < staged < tiles
    check_budget(ref, gathered, tiled, e_tol=1e-6)


def test_cubic_two_phase_box_mixes_staged_and_gathered_tiles(md):
    # the same in a cubic box: a dense cube in one corner, a dilute gas elsewhere
    st = md.fcc_lattice(10, 0.8442, 0.722, 8)
    box = st["box"] * 2.0
    rng = np.random.default_rng(8)
    gas = rng.uniform(0.0, 0.5, size=(200, 3)) * box  # ~0.17 per unit volume
    pos = np.concatenate([st["pos"] - 0.25 * box, gas])
    s = md.System.from_arrays(pos, box, vel=np.zeros_like(pos), mass=np.ones(len(pos)))
    v = md.VerletList(box, 2.5, 0.3)
    v.build(s)
    ref, gathered, tiled = three_ways(md, s, v)
    staged, tiles = v.halo_tiles()
    assert 0 < staged < tiles
    check_budget(ref, gathered, tiled, e_tol=1e-6)


@pytest.mark.parametrize("tpa", [1, 4, 8])
def test_tile_shapes_within_budget(md, tpa):
    """Every tile shape (threads per atom of the tile kernel) sums the same pairs:
    within the error budget of FP64 and of the default shape, and deterministic."""
    s, v, _ = melt(md, 12, 0.8442, 10)
    ref, gathered, tiled = three_ways(md, s, v)
    lj = md.LennardJones(1.0, 1.0, 2.5, precision=md.PRECISION_MIXED)
    lj.set_tile_threads(tpa)
    e, w = lj.compute_forces(s, v)
    f = s.forces
    e2, w2 = lj.compute_forces(s, v)
    assert np.array_equal(s.forces, f) and e2 == e and w2 == w
    check_budget(ref, gathered, (e, w, f))
    assert rms_rel(f, tiled[2]) < 1e-6
    with pytest.raises(md.InvalidArgument):
        lj.set_tile_threads(3)


def test_fused_run_with_rebuilds_replays_host_steps(md):
    s, v, st = melt(md, 10, 0.8442, 6, steps=50)
    x, vel = s.positions, s.velocities
    ctx = md.default_context()
    out = []
    for graphs in (False, True):
        ctx.set_graphs(graphs)
        try:
            sys_ = md.System.from_arrays(x, st["box"], vel=vel, mass=st["mass"])
            lj = md.LennardJones(1.0, 1.0, 2.5, precision=md.PRECISION_MIXED)
            vl = md.VerletList(st["box"], 2.5, 0.3)
            vl.build(sys_)
            vl.set_halo(True)  # 4000 atoms: below the size fused runs turn tiles on at
            lj.compute_forces(sys_, vl)
            th = md.VelocityVerlet(0.005).run(sys_, vl, lj, 300, thermo=True)
            assert vl.rebuild_count() > 3
            out.append((sys_.positions, sys_.velocities, th, vl.halo_tiles()))
        finally:
            ctx.set_graphs(True)
    assert out[1][3][0] == out[1][3][1] > 0
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])


def test_tile_policy(md):
    """Tiles are kept only where they pay: a fused mixed run of a small system or a
    single force call leaves a list without them; set_halo(False) drops them."""
    s, v, st = melt(md, 8, 0.8442, 7, steps=20)  # 2048 atoms
    lj = md.LennardJones(1.0, 1.0, 2.5, precision=md.PRECISION_MIXED)
    lj.compute_forces(s, v)
    md.VelocityVerlet(0.005).run(s, v, lj, 40)
    assert v.halo_tiles() == (0, 0)
    v.set_halo(True)
    staged, tiles = v.halo_tiles()
    assert tiles == 16 and staged == tiles
    v.set_halo(False)
    assert v.halo_tiles() == (0, 0)


def test_list_with_tiles_serves_other_consumers(md):
    """A list that keeps halo tiles (rebuilt inside a fused run and by host builds)
    still exports the reference's pair set and serves an FP64 force call exactly."""
    s, v, st = melt(md, 10, 0.8442, 8, steps=20)  # 4000 atoms
    lj = md.LennardJones(1.0, 1.0, 2.5, precision=md.PRECISION_MIXED)
    v.set_halo(True)
    lj.compute_forces(s, v)
    md.VelocityVerlet(0.005).run(s, v, lj, 200)
    assert v.rebuild_count() > 3 and v.halo_tiles()[0] > 0
    v.build(s)  # a host build with tiles on
    fresh = md.VerletList(st["box"], 2.5, 0.3)
    fresh.build(s)
    assert np.array_equal(v.pairs(), fresh.pairs())
    v.build(s)
    lj64 = md.LennardJones(1.0, 1.0, 2.5)
    e1, w1 = lj64.compute_forces(s, v)
    f1 = s.forces
    e2, w2 = lj64.compute_forces(s, fresh)
    f2 = s.forces
    assert e1 == e2 and w1 == w2 and np.array_equal(f1, f2)


def test_fused_run_over_staged_and_gathered_tiles(md):
    """A dense slab beside a dilute gas: rebuilds inside the fused run write slot
    rows, int32 rows, or both (cells touching both kinds of tile); the trajectory
    equals the one without tiles.  With tiles the force kernel also takes the
    closing half-kick and sums the kinetic energy in its own block order, so the
    kinetic-energy columns agree to rounding and everything else bit for bit."""
    st = md.fcc_lattice(12, 0.8442, 0.722, 9)
    box = st["box"].copy()
    box[2] *= 3.0
    rng = np.random.default_rng(9)
    gas = rng.uniform(-0.5, 0.5, size=(300, 3)) * box
    gas[:, 2] = np.where(gas[:, 2] > 0, gas[:, 2] * 0.5 + box[2] / 4, gas[:, 2] * 0.5 - box[2] / 4)
    keep = []  # no two gas atoms closer than 1.0 (minimum image)
    for k in range(len(gas)):
        d = gas[keep] - gas[k]
        d -= box * np.round(d / box)
        if not keep or np.min(np.sum(d * d, axis=1)) > 1.0:
            keep.append(k)
    gas = gas[keep]
    pos = np.concatenate([st["pos"], gas])
    vel = np.concatenate([st["vel"], rng.normal(0.0, 0.8, size=gas.shape)])
    out = []
    for halo in (False, True):
        s = md.System.from_arrays(pos, box, vel=vel, mass=np.ones(len(pos)))
        lj = md.LennardJones(1.0, 1.0, 2.5, precision=md.PRECISION_MIXED)
        lj.set_halo(halo)
        v = md.VerletList(box, 2.5, 0.3)
        v.build(s)
        v.set_halo(halo)
        lj.compute_forces(s, v)
        th = md.VelocityVerlet(0.002).run(s, v, lj, 150, thermo=True)
        staged, tiles = v.halo_tiles()
        if halo:
            assert v.rebuild_count() >= 1 and 0 < staged < tiles
        out.append((s.positions, th, v.pairs()))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1][:, :2], out[1][1][:, :2])  # potential energy, virial
    assert np.allclose(out[0][1][:, 2:], out[1][1][:, 2:], rtol=1e-13, atol=0.0)
    assert np.array_equal(out[0][2], out[1][2])
