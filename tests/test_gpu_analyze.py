"""GPU parity of the analysis consumers (analyze/rdf.cpp, msd.cpp, vacf.cpp).

The RDF histogram is an integer count per bin with the reference's distance and
bin arithmetic, so it must equal the oracle's (and g the reference's) exactly,
on both the all-pairs path (fewer than 3 cells of width rMax per side) and the
cell path.  MSD and VACF sum over atoms in a different order than the
reference, so they are compared at 1e-12 relative.  The trajectories run with
Verlet rebuilds in between, which re-sort the atoms on the device: the analysis
state is kept in original atom order.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def liquid(md, cells, rho, seed, box_scale=None):
    st = md.fcc_lattice(cells, rho, 1.0, seed)
    pos, box = st["pos"], st["box"].copy()
    if box_scale is not None:  # stretch one axis: a non-cubic box
        box = box * np.asarray(box_scale)
        pos = pos * np.asarray(box_scale)
    s = md.System.from_arrays(pos, box, vel=st["vel"], mass=st["mass"])
    lj = md.LennardJones(1.0, 1.0, 2.5)
    v = md.VerletList(box, 2.5, 0.3)
    v.build(s)
    lj.compute_forces(s, v)
    return s, v, lj, box


def frames_of(md, s, v, lj, frames, steps):
    integ = md.VelocityVerlet(0.005)
    pos, vel = [], []
    for _ in range(frames):
        integ.run(s, v, lj, steps)
        pos.append(s.positions)
        vel.append(s.velocities)
    return pos, vel


@pytest.mark.parametrize("cells,rmax,bins,scale", [
    (6, 5.0, 100, None),          # L = 10.08: 2 cells of width rMax per side -> all pairs
    (10, 4.0, 80, None),          # L = 16.8: 4 cells per side -> cell path
    (8, 3.0, 60, (1.0, 1.3, 0.9)),  # non-cubic, cell path
])
def test_rdf_histogram_equals_reference(md, cells, rmax, bins, scale):
    s, v, lj, box = liquid(md, cells, 0.8442, 3, scale)
    rdf = md.Rdf(rmax, bins)
    pos, _ = frames_of(md, s, v, lj, 4, 25)
    for p in pos[:3]:
        s.positions = p  # re-upload the same frame: accumulate reads the device copy
        rdf.accumulate(s)
    assert rdf.frames() == 3
    hist, g = O.rdf(pos[:3], box, rmax, bins)
    assert np.array_equal(rdf.histogram(), hist)
    assert np.array_equal(rdf.g(), g)
    assert np.array_equal(rdf.bin_centres(), (np.arange(bins) + 0.5) * (rmax / bins))
    if O.ref_available():
        g_ref, _ = O.ref_rdf(pos[:3], box, rmax, bins)
        assert np.array_equal(rdf.g(), g_ref)
    # a physical g(r): zero inside the core, first peak near 2^(1/6)
    r = rdf.bin_centres()
    assert np.all(rdf.g()[r < 0.8] == 0.0) and rdf.g().max() > 1.5


def test_rdf_rejects_rmax_beyond_half_box(md):
    s, v, lj, box = liquid(md, 6, 0.8442, 4)
    rdf = md.Rdf(0.51 * box.min(), 10)
    with pytest.raises(md.InvalidArgument, match="rMax exceeds half the smallest box length"):
        rdf.accumulate(s)
    assert rdf.frames() == 0


def test_rdf_frames_follow_the_trajectory(md):
    """Accumulating straight after runs (device state re-sorted by rebuilds)."""
    s, v, lj, box = liquid(md, 10, 0.8442, 5)
    rdf = md.Rdf(4.0, 50)
    integ = md.VelocityVerlet(0.005)
    pos = []
    for _ in range(3):
        integ.run(s, v, lj, 40)
        rdf.accumulate(s)
        pos.append(s.positions)
    assert v.rebuild_count() > 1
    hist, _ = O.rdf(pos, box, 4.0, 50)
    assert np.array_equal(rdf.histogram(), hist)


def rel_close(a, b, tol):
    a, b = np.asarray(a), np.asarray(b)
    return np.all(np.abs(a - b) <= tol * np.maximum(np.abs(b), 1e-300))


def test_msd_and_vacf_match_the_oracle(md):
    s, v, lj, box = liquid(md, 8, 0.8442, 6)  # 2048 atoms
    msd = md.Msd(s.n, 10)
    vacf = md.Vacf(s.n, 10)
    integ = md.VelocityVerlet(0.005)
    pos, vel = [], []
    for _ in range(24):
        integ.run(s, v, lj, 10)
        msd.push(s)
        vacf.push(s)
        pos.append(s.positions)
        vel.append(s.velocities)
    assert v.rebuild_count() > 5
    m_or = O.msd(pos, box, 10)
    u_or = O.vacf_unnormalised(vel, 10)
    assert msd.msd()[0] == 0.0 and rel_close(msd.msd()[1:], m_or[1:], 1e-12)
    assert rel_close(vacf.vacf(normalised=False), u_or, 1e-12)
    assert rel_close(vacf.vacf(), u_or / u_or[0], 1e-12)
    if O.ref_available():
        m_ref, d_ref = O.ref_msd(pos, box, 10, 0.05, 2, 10)
        c_ref, dv_ref = O.ref_vacf(vel, box, 10, 0.05)
        assert rel_close(msd.msd()[1:], m_ref[1:], 1e-12)
        assert rel_close(vacf.vacf(), c_ref, 1e-12)
        assert abs(msd.diffusion_coefficient(0.05, 2, 10) - d_ref) <= 1e-11 * abs(d_ref)
        assert abs(vacf.diffusion_coefficient(0.05) - dv_ref) <= 1e-11 * abs(dv_ref)


def test_msd_unwraps_across_the_boundary(md):
    """A dilute gas moving fast: atoms cross the box several times, and the MSD
    grows as (v t)^2 instead of saturating at the box size."""
    st = md.fcc_lattice(4, 0.05, 1.0, 7)
    s = md.System.from_arrays(st["pos"], st["box"], vel=st["vel"] * 0.0 + np.array([3.0, 0.0, 0.0]),
                              mass=st["mass"])
    lj = md.LennardJones(1.0, 1.0, 2.5)
    v = md.VerletList(st["box"], 2.5, 0.3)
    v.build(s)
    lj.compute_forces(s, v)
    msd = md.Msd(s.n, 5)
    integ = md.VelocityVerlet(0.01)
    for _ in range(12):
        integ.run(s, v, lj, 100)  # 3 length units per push; L = 17.2
        msd.push(s)
    m = msd.msd()
    assert np.allclose(m[1:] / (3.0 * np.arange(1, 6)) ** 2, 1.0, rtol=0.05)


def test_msd_rejects_a_system_of_another_size(md):
    s, v, lj, box = liquid(md, 4, 0.8442, 8)
    msd = md.Msd(s.n + 1, 3)
    with pytest.raises(md.InvalidArgument):
        msd.push(s)


@pytest.mark.parametrize("first,stride", [(1, 2), (5, 7)])
def test_rdf_subset_on_the_cell_path(md, first, stride):
    """A subset frame (atoms first, first + stride, ...) through the cell grid
    (4 cells of width rMax per side) equals the oracle's Rdf of those atoms."""
    s, v, lj, box = liquid(md, 10, 0.8442, 9)
    rdf = md.Rdf(4.0, 80)
    pos, _ = frames_of(md, s, v, lj, 2, 30)
    frames = []
    for p in pos:
        s.positions = p
        rdf.accumulate(s, first, stride)
        frames.append(p[first::stride])
    hist, g = O.rdf(frames, box, 4.0, 80)
    assert np.array_equal(rdf.histogram(), hist)
    assert np.array_equal(rdf.g(), g)
