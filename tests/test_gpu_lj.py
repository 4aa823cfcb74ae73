"""GPU parity of the Lennard-Jones / neighbour path against the oracle and the
reference's golden vectors -- the reference's tests/test_nist_lj.cpp,
test_neighbor.cpp and test_forces.cpp restated against the CUDA path.

Tolerances follow the reference's doctest Approx semantics:
|a - b| < eps * (1 + max(|a|, |b|)), with eps = 1e-12 for neighbour-list parity
(only the summation order differs from the reference).
"""
import math

import numpy as np
import pytest

import oracle as O
from conftest import load_golden

pytestmark = pytest.mark.gpu

LJ = load_golden("nist_lj.npz")
FCC = load_golden("fcc_lj.npz")


def approx_eq(a, b, eps):
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    return np.all(np.abs(a - b) < eps * (1.0 + np.maximum(np.abs(a), np.abs(b))))


def half_width(value, sig_figs=5):
    mag = abs(value)
    return 0.0 if mag == 0 else 0.5 * 10.0 ** (math.floor(math.log10(mag)) - (sig_figs - 1))


def nist_system(md, c):
    return md.System.from_arrays(LJ[f"pos{c}"], LJ[f"box{c}"])


@pytest.mark.parametrize("row", range(12))
def test_nist_lj_table_on_gpu(md, row):
    """tests/test_nist_lj.cpp:113-155 and the golden reference outputs."""
    c, tr, rc, up, wp, ulrc = LJ["published"][row]
    c, tr = int(c), int(tr)
    sys_ = nist_system(md, c)
    lj = md.LennardJones(1.0, 1.0, rc, tr)
    e, w = lj.compute_energy_virial(sys_)
    lrc = lj.long_range_correction(sys_)
    assert abs(e - up) <= half_width(up)
    assert abs(w - wp) <= half_width(wp)
    assert (abs(lrc) <= 1e-12) if ulrc == 0.0 else (abs(lrc - ulrc) <= half_width(ulrc))
    gold = LJ["computed"][row]
    assert approx_eq(e, gold[3], 1e-12) and approx_eq(w, gold[4], 1e-12)
    assert lrc == gold[5]
    assert lj.long_range_correction_pressure(sys_) == gold[6]
    # brute-force forces (computeForces(sys)) against the reference's
    e2, w2 = lj.compute_forces(sys_)
    assert approx_eq(e2, gold[3], 1e-12) and approx_eq(w2, gold[4], 1e-12)
    assert approx_eq(sys_.forces, LJ[f"forces{c}_{int(rc)}_{tr}"], 1e-12)


def test_cell_list_forces_match_brute(md):
    """tests/test_neighbor.cpp:37-61 (config 1, N=800, L=10, rc=3: 3 cells/side)."""
    sys_ = nist_system(md, 1)
    lj = md.LennardJones(1.0, 1.0, 3.0)
    cells = md.CellList(LJ["box1"], 3.0)
    assert cells.usable() and cells.cells_per_side(0) == 3
    cells.build(sys_)
    e, w = lj.compute_forces(sys_, cells)
    gold = LJ["computed"][0]
    assert approx_eq(e, gold[3], 1e-12) and approx_eq(w, gold[4], 1e-12)
    assert approx_eq(sys_.forces, LJ["forces1_3_0"], 1e-12)
    assert abs(e - (-4.3515e3)) <= 0.05 and abs(w - (-5.6867e2)) <= 0.005


def test_cell_candidate_pairs_equal_reference_set(md):
    sys_ = nist_system(md, 1)
    cells = md.CellList(LJ["box1"], 3.0)
    cells.build(sys_)
    got = cells.pairs()
    ref = O.cell_pairs(LJ["pos1"], LJ["box1"], 3.0)
    assert len(got) == int(LJ["ncellpairs1"])
    key = lambda p: np.sort(p[:, 0] * 1_000_003 + p[:, 1])
    assert np.array_equal(key(got), key(ref))


def test_unusable_cell_list_refuses(md):
    """tests/test_neighbor.cpp:77-98"""
    cells = md.CellList([5.0, 5.0, 5.0], 3.0)
    assert not cells.usable()
    sys_ = md.System.from_arrays([[0.0, 0.0, 0.0], [1.1, 0.0, 0.0]], [5.0, 5.0, 5.0])
    cells.build(sys_)
    lj = md.LennardJones(1.0, 1.0, 3.0)
    with pytest.raises(md.InvalidArgument):
        lj.compute_forces(sys_, cells)


@pytest.mark.parametrize("c", [1, 2, 3, 4])
def test_verlet_pair_set_bit_exact(md, c):
    """The Verlet pair set equals the reference's exactly (cells or brute build)."""
    sys_ = nist_system(md, c)
    v = md.VerletList(LJ[f"box{c}"], 3.0, 0.3)
    v.build(sys_)
    got = v.pairs()
    ref = LJ[f"verlet{c}"]
    order = np.lexsort((ref[:, 1], ref[:, 0]))
    assert np.array_equal(got, ref[order])


@pytest.mark.parametrize("cells,skin", [(10, 0.3), (10, 1.5), (12, 0.3)])
def test_verlet_pair_set_bit_exact_liquid(md, cells, skin):
    """Pair sets on disordered states: several cells per side, and (skin 1.5) more
    candidates per cell than one shared-memory staging window holds."""
    st = md.fcc_lattice(cells, 0.8442, 0.722, 11)
    rng = np.random.default_rng(cells)
    pos = st["pos"] + rng.normal(scale=0.15, size=st["pos"].shape)
    box = st["box"]
    pos -= box * np.floor(pos / box + 0.5)
    sys_ = md.System.from_arrays(pos, box)
    v = md.VerletList(box, 2.5, skin)
    v.build(sys_)
    got = v.pairs()
    ref = O.verlet_pairs(pos, box, 2.5, skin)
    order = np.lexsort((ref[:, 1], ref[:, 0]))
    assert np.array_equal(got, ref[order])


def test_verlet_forces_match_brute(md):
    """tests/test_neighbor.cpp:106-128"""
    sys_ = nist_system(md, 1)
    lj = md.LennardJones(1.0, 1.0, 3.0)
    v = md.VerletList(LJ["box1"], 3.0, 0.3)
    v.build(sys_)
    e, w = lj.compute_forces(sys_, v)
    gold = LJ["computed"][0]
    assert approx_eq(e, gold[3], 1e-12) and approx_eq(w, gold[4], 1e-12)
    assert approx_eq(sys_.forces, LJ["forces1_3_0"], 1e-12)


def test_rebuild_trigger(md):
    """tests/test_neighbor.cpp:130-159"""
    skin = 0.3
    sys_ = nist_system(md, 1)
    v = md.VerletList(LJ["box1"], 3.0, skin)
    v.build(sys_)
    p = LJ["pos1"].copy()
    p[0, 0] += 0.3 * skin
    sys_.positions = p
    assert not v.needs_rebuild(sys_)
    p = LJ["pos1"].copy()
    p[0, 0] += 0.6 * skin
    p[1, 1] += 0.6 * skin
    sys_.positions = p
    assert v.needs_rebuild(sys_)
    a, b = v.displacements(sys_)
    ra, rb = O.top2(p, LJ["pos1"], LJ["box1"])
    assert (a, b) == (ra, rb)


def test_verlet_under_dynamics(md):
    """tests/test_neighbor.cpp:161-209: 200 hand-rolled VV steps at dt=2e-3."""
    sys_ = nist_system(md, 1)
    lj = md.LennardJones(1.0, 1.0, 3.0)
    v = md.VerletList(LJ["box1"], 3.0, 0.3)
    v.build(sys_)
    dt = 2e-3
    lj.compute_forces(sys_, v)
    vel = np.zeros((800, 3))
    for _ in range(200):
        f = sys_.forces
        vel = vel + (0.5 * dt) * f
        sys_.positions = sys_.positions + dt * vel
        v.rebuild_if_needed(sys_)
        e, w = lj.compute_forces(sys_, v)
        vel = vel + (0.5 * dt) * sys_.forces
    fast = sys_.forces
    eb, wb = lj.compute_forces(sys_)
    assert approx_eq(eb, e, 1e-12) and approx_eq(wb, w, 1e-12)
    assert approx_eq(sys_.forces, fast, 1e-12)
    assert 0 < v.rebuild_count() < 200
    # the pair set still equals the reference's on the final positions
    ref = O.verlet_pairs(sys_.positions, LJ["box1"], 3.0, 0.3)
    if v.needs_rebuild(sys_):
        v.build(sys_)
    else:
        v.build(sys_)
    got = v.pairs()
    order = np.lexsort((ref[:, 1], ref[:, 0]))
    assert np.array_equal(got, ref[order])


def test_forces_equal_minus_gradient(md):
    """tests/test_forces.cpp:10-71 (FD h=1e-5, tol 1e-8) on the GPU energies."""
    for trunc in (0, 1):
        pos = LJ["pos4"].copy()
        sys_ = md.System.from_arrays(pos, LJ["box4"])
        lj = md.LennardJones(1.0, 1.0, 3.0, trunc)
        lj.compute_forces(sys_)
        f = sys_.forces
        h = 1e-5
        for i in (0, 7, 29):
            for d in range(3):
                p = pos.copy()
                p[i, d] += h
                sys_.positions = p
                up, _ = lj.compute_energy_virial(sys_)
                p[i, d] -= 2 * h
                sys_.positions = p
                um, _ = lj.compute_energy_virial(sys_)
                num = -(up - um) / (2 * h)
                assert approx_eq(f[i, d], num, 1e-8)
        sys_.positions = pos


def test_newton_third_law(md):
    """tests/test_forces.cpp:73-83"""
    sys_ = nist_system(md, 4)
    md.LennardJones(1.0, 1.0, 3.0).compute_forces(sys_)
    assert np.all(np.abs(sys_.forces.sum(0)) < 1e-10)


def test_product_lattice_bit_exact():
    """md_fcc_lattice (host setup) reproduces the reference's fccLattice."""
    import moleculardynamics_b200 as mdb
    st = mdb.fcc_lattice(6, 0.8442, 0.722, 1)
    assert np.array_equal(st["pos"], FCC["c6_pos"]) and np.array_equal(st["vel"], FCC["c6_vel"])
