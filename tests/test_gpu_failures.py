"""Failure detection without a GPU fault: device errors are status bits read at
the next synchronising call, never traps.  A tiny
neighbour-row capacity overflows and is grown (or reported when fixed); SHAKE
non-convergence is tested with the water tests; a NaN in the state is reported;
positions far outside the box fold back (exactly as the reference folds them)."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def liquid(md, cells=6, temp=0.722, seed=2):
    st = md.fcc_lattice(cells, 0.8442, temp, seed)
    pos = st["pos"] + np.random.default_rng(seed).normal(scale=0.1, size=st["pos"].shape)
    pos -= st["box"] * np.floor(pos / st["box"] + 0.5)
    return pos, st["vel"], st["mass"], st["box"]


def test_row_overflow_is_grown_by_host_builds(md):
    pos, vel, mass, box = liquid(md)
    s = md.System.from_arrays(pos, box)
    v = md.VerletList(box, 2.5, 0.3)
    v.set_capacity(8)
    v.build(s)
    ref = O.verlet_pairs(pos, box, 2.5, 0.3)
    assert np.array_equal(v.pairs(), ref[np.lexsort((ref[:, 1], ref[:, 0]))])
    e, w = md.LennardJones(1.0, 1.0, 2.5).compute_forces(s, v)
    fo, eo, wo = O.lj_compute(pos, box, rc=2.5)
    assert abs(e - eo) < 1e-12 * abs(eo) and np.max(np.abs(s.forces - fo)) < 1e-10


def test_fixed_capacity_overflow_is_an_error_and_the_context_recovers(md):
    pos, vel, mass, box = liquid(md)
    s = md.System.from_arrays(pos, box)
    v = md.VerletList(box, 2.5, 0.3)
    v.set_capacity(8, fixed=True)
    with pytest.raises(md.MDError, match="fixed row capacity"):
        v.build(s)
    v.set_capacity(256)
    v.build(s)
    md.LennardJones(1.0, 1.0, 2.5).compute_forces(s, v)
    assert s.ctx.status() == 0


def test_overflow_inside_a_fused_loop_is_reported(md):
    """A hot liquid with a row capacity fixed at the first build's longest row:
    a later rebuild decided on the device overflows, the loop reports it and the
    context is usable afterwards."""
    pos, vel, mass, box = liquid(md, temp=4.0)
    s = md.System.from_arrays(pos, box, vel=vel, mass=mass)
    v = md.VerletList(box, 2.5, 0.3)
    v.build(s)
    longest = int(np.max(np.bincount(v.pairs().ravel(), minlength=s.n)))
    v.set_capacity(longest, fixed=True)
    v.build(s)
    lj = md.LennardJones(1.0, 1.0, 2.5)
    lj.compute_forces(s, v)
    with pytest.raises(md.MDError, match="neighbour overflow"):
        md.VelocityVerlet(0.005).run(s, v, lj, 400)
    assert s.ctx.status() == 0
    v.set_capacity(512)
    v.build(s)
    lj.compute_forces(s, v)


@pytest.mark.parametrize("field", ["velocity", "position"])
def test_non_finite_state_is_reported(md, field):
    pos, vel, mass, box = liquid(md)
    s = md.System.from_arrays(pos, box, vel=vel, mass=mass)
    v = md.VerletList(box, 2.5, 0.3)
    v.build(s)
    lj = md.LennardJones(1.0, 1.0, 2.5)
    lj.compute_forces(s, v)
    if field == "velocity":
        bad = vel.copy()
        bad[5, 1] = np.nan
        s.velocities = bad
    else:
        bad = pos.copy()
        bad[5, 1] = np.inf
        s.positions = bad
    with pytest.raises(md.MDError, match="non-finite"):
        md.VelocityVerlet(0.005).run(s, v, lj, 5)
    assert s.ctx.status() == 0


def test_positions_far_outside_the_box_fold_back(md):
    pos, vel, mass, box = liquid(md)
    shift = np.random.default_rng(1).integers(-1000, 1000, size=pos.shape) * box
    far = pos + shift
    a = md.System.from_arrays(pos, box)
    b = md.System.from_arrays(far, box)
    lj = md.LennardJones(1.0, 1.0, 2.5)
    ea, wa = lj.compute_forces(a)
    eb, wb = lj.compute_forces(b)
    fo, eo, wo = O.lj_compute(far, box, rc=2.5)
    assert abs(eb - eo) < 1e-12 * abs(eo) and np.max(np.abs(b.forces - fo)) < 1e-10
    # the far copies carry the rounding of x + k L (|x| ~ 1e4): same physics to ~1e-8
    assert abs(ea - eb) < 1e-10 * abs(ea)
    assert np.max(np.abs(a.forces - b.forces)) < 1e-6 * np.max(np.abs(a.forces))
