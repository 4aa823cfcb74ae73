"""The launch-shape autotuner: every shape gives the same forces (to the
summation-order rounding), the winner is applied and cached on disk, and a
second call reads it back without timing."""
import numpy as np
import pytest

import moleculardynamics_b200.autotune as T

pytestmark = pytest.mark.gpu


def test_tune_force_kernel_applies_and_caches(md, tmp_path, monkeypatch):
    monkeypatch.setenv("MOLDYN_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    st = md.fcc_lattice(8, 0.8442, 0.722, 3)
    pos = st["pos"] + np.random.default_rng(3).normal(scale=0.1, size=st["pos"].shape)
    pos -= st["box"] * np.floor(pos / st["box"] + 0.5)
    s = md.System.from_arrays(pos, st["box"], vel=st["vel"])
    v = md.VerletList(st["box"], 2.5, 0.3)
    v.build(s)
    ref_lj = md.LennardJones(1.0, 1.0, 2.5)
    e0, w0 = ref_lj.compute_forces(s, v)
    f0 = s.forces
    for tpa, u in T.SHAPES:
        ref_lj.set_launch(tpa, u)
        e, w = ref_lj.compute_forces(s, v)
        assert abs(e - e0) < 1e-12 * abs(e0) and abs(w - w0) < 1e-12 * abs(w0)
        assert np.max(np.abs(s.forces - f0)) < 1e-12 * np.max(np.abs(f0))
    lj = md.LennardJones(1.0, 1.0, 2.5)
    best, timings = T.tune_force_kernel(s, lj, v, 0.3, repeats=2)
    assert best in T.SHAPES and len(timings) == len(T.SHAPES)
    assert timings[best] == min(timings.values())
    again, t2 = T.tune_force_kernel(s, md.LennardJones(1.0, 1.0, 2.5), v, 0.3)
    assert again == best and t2 == {}
    with pytest.raises(md.InvalidArgument):
        lj.set_launch(3, 1)


def test_cell_width_keeps_the_pair_set_and_forces(md):
    """Cells wider than the list cutoff (the cell-width axis of the tuner) give the
    reference's pair set exactly and the same FP64 forces to summation order; a
    width below the list cutoff is refused; tune_cell_width applies the fastest."""
    st = md.fcc_lattice(10, 0.8442, 0.722, 5)
    rng = np.random.default_rng(5)
    pos = st["pos"] + rng.normal(scale=0.1, size=st["pos"].shape)
    pos -= st["box"] * np.floor(pos / st["box"] + 0.5)
    box = st["box"]
    out = []
    for factor in (0.0, 1.25, 1.6):
        s = md.System.from_arrays(pos, box)
        v = md.VerletList(box, 2.5, 0.3)
        if factor:
            v.set_cell_width(factor * 2.8)
        v.build(s)
        e, w = md.LennardJones(1.0, 1.0, 2.5).compute_forces(s, v)
        out.append((v.cells_per_side(), v.pairs(), e, w, s.forces))
    # L = 16.79: 5 cells of the list cutoff 2.8 per side, 4 of 3.5, 3 of 4.48
    assert out[0][0] == (5, 5, 5) and out[1][0] == (4, 4, 4) and out[2][0] == (3, 3, 3)
    for cells, pairs, e, w, f in out[1:]:
        assert np.array_equal(pairs, out[0][1])
        assert abs(e - out[0][2]) < 1e-12 * abs(out[0][2])
        assert abs(w - out[0][3]) < 1e-12 * abs(out[0][3])
        assert np.max(np.abs(f - out[0][4])) < 1e-12 * np.max(np.abs(out[0][4]))
    with pytest.raises(md.InvalidArgument):
        md.VerletList(box, 2.5, 0.3).set_cell_width(2.7)
    lj = md.LennardJones(1.0, 1.0, 2.5)
    best, times = T.tune_cell_width(box, pos, st["vel"], st["mass"], lj, 0.3,
                                    lambda: md.VelocityVerlet(0.005), factors=(1.0, 1.2),
                                    steps=20)
    assert best in times and times[best] == min(times.values()) and len(times) == 2


def test_tune_tile_shape_applies_the_fastest(md):
    st = md.fcc_lattice(12, 0.8442, 0.722, 6)
    s = md.System.from_arrays(st["pos"], st["box"], vel=st["vel"])
    v = md.VerletList(st["box"], 2.5, 0.3)
    v.build(s)
    lj = md.LennardJones(1.0, 1.0, 2.5, precision=md.PRECISION_MIXED)
    best, times = T.tune_tile_shape(s, lj, v, repeats=2)
    assert best in T.TILE_SHAPES and times[best] == min(times.values())
