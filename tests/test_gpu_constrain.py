"""GPU parity of rigid-water SHAKE/RATTLE and the constrained velocity-Verlet step
(the reference's tests/test_rigid_water.cpp restated against the CUDA path), plus
the Nose-Hoover chain around the constrained step.

Bit-exact comparisons use the oracle's restatement of constrain/rigid_water.cpp
and a numpy restatement of integrate/constrained_velocity_verlet.hpp:27-57 with
the same operation order; forces handed to both sides are the oracle's, so the
step arithmetic is compared without the libm differences of the Ewald sum."""
import math

import numpy as np
import pytest

import oracle as O
from conftest import load_golden

pytestmark = pytest.mark.gpu

SPCE = load_golden("nist_spce.npz")
TAU_PS = 1.0966875353  # core/units.hpp:33


def femtoseconds(fs):
    return fs * 1.0e-3 / TAU_PS  # core/units.hpp:36-37


def water(md, c=1):
    types = ["O" if o else "H" for o in SPCE[f"isO{c}"]]
    return md.build_spce_system(SPCE[f"pos{c}"], types, SPCE[f"box{c}"])


def fold(d, box):
    """Box::minimumImage (core/box.cpp:12-26), same arithmetic."""
    return d - box * np.floor(d / box + 0.5)


def worst_geometry(pos, box, oh, hh):
    """worstGeometryError (tests/test_rigid_water.cpp:32-46)."""
    targets = (oh, oh, hh)
    worst = 0.0
    for c, (i, j) in enumerate(((0, 1), (0, 2), (1, 2))):
        d = fold(pos[i::3] - pos[j::3], box)
        worst = max(worst, float(np.max(np.abs(np.linalg.norm(d, axis=1) - targets[c]))
                                 / targets[c]))
    return worst


def constraint(md):
    p = md.SpceParameters
    return md.RigidWater(p.rOH, p.angleHOH), O.rigid_water(p.rOH, p.angleHOH)


def oracle_forces(s, box):
    f, _ = O.spce(s["pos"], box, s["q"], s["mol"])
    return f


def state(sys):
    return dict(pos=sys.positions, vel=sys.velocities, m=sys.masses, q=sys.charges,
                mol=sys.molecule_ids)


def thermal_velocities(md, sys, temperature, seed):
    """tests/test_rigid_water.cpp:209-215: v = sqrt(T/m) * normal(), Rng(seed)."""
    m = sys.masses
    xi = O.rng_normals(seed, 3 * sys.n).reshape(-1, 3)
    sys.velocities = np.sqrt(temperature / m)[:, None] * xi


def test_degrees_of_freedom(md):
    assert md.RigidWater.degrees_of_freedom(100, False) == 600
    assert md.RigidWater.degrees_of_freedom(100, True) == 597
    assert md.RigidWater.degrees_of_freedom(1, False) == 6


def test_target_distances(md):
    rw, orw = constraint(md)
    assert rw.oh_distance() == orw.oh
    assert rw.hh_distance() == orw.hh


def test_nist_configuration_is_rigid(md):
    rw, _ = constraint(md)
    s = water(md)
    assert worst_geometry(s.positions, SPCE["box1"], rw.oh_distance(), rw.hh_distance()) < 1e-6


def test_constraining_rigid_molecules_is_idempotent(md):
    """tests/test_rigid_water.cpp:62-78 and bit-exact against the oracle."""
    rw, orw = constraint(md)
    s = water(md)
    before = s.positions
    it = rw.constrain_positions(s, before)
    after = s.positions
    assert np.max(np.linalg.norm(after - before, axis=1)) < 1e-9
    want, oit = O.shake(orw, before, before, s.masses, SPCE["box1"])
    assert np.array_equal(after, want)
    assert it == oit


@pytest.mark.parametrize("c", [1, 2])
def test_shake_bit_exact_and_momentum_conserving(md, c):
    """tests/test_rigid_water.cpp:80-125: displaced sites are put back without
    moving any molecule's centre of mass; positions and the sweep count are
    bit-identical to the reference's Gauss-Seidel SHAKE."""
    rw, orw = constraint(md)
    s = water(md, c)
    box = SPCE[f"box{c}"]
    ref = s.positions
    i = np.arange(s.n)
    sh = 0.01 * (i % 7) - 0.03
    disp = ref + np.stack([sh, -0.5 * sh, 0.25 * sh], 1)
    s.positions = disp
    m = s.masses
    com0 = np.add.reduceat(disp * m[:, None], np.arange(0, s.n, 3)) / np.add.reduceat(
        m, np.arange(0, s.n, 3))[:, None]
    it = rw.constrain_positions(s, ref)
    got = s.positions
    want, oit = O.shake(orw, disp, ref, m, box)
    assert np.array_equal(got, want)
    assert it == oit and it > 1
    com1 = np.add.reduceat(got * m[:, None], np.arange(0, s.n, 3)) / np.add.reduceat(
        m, np.arange(0, s.n, 3))[:, None]
    assert np.max(np.linalg.norm(com1 - com0, axis=1)) < 1e-10
    assert worst_geometry(got, box, rw.oh_distance(), rw.hh_distance()) < 1e-10


def test_rattle_bit_exact(md):
    rw, orw = constraint(md)
    s = water(md)
    thermal_velocities(md, s, 298.0, 7)
    v0 = s.velocities
    it = rw.constrain_velocities(s)
    got = s.velocities
    want, oit = O.rattle(orw, s.positions, v0, s.masses, SPCE["box1"])
    assert np.array_equal(got, want)
    assert it == oit and it > 1
    # no relative velocity along any bond
    r, v = s.positions, got
    for i, j in ((0, 1), (0, 2), (1, 2)):
        d = fold(r[i::3] - r[j::3], SPCE["box1"])
        rv = np.einsum("ij,ij->i", d, v[i::3] - v[j::3])
        assert np.max(np.abs(rv)) < 1e-9


def test_shake_reports_non_convergence(md):
    """rigid_water.cpp:100-104: one sweep is not enough for a violated molecule,
    so the call fails with the reference's runtime error."""
    p = md.SpceParameters
    rw1 = md.RigidWater(p.rOH, p.angleHOH, 1e-12, 1)
    s = water(md)
    ref = s.positions
    s.positions = ref + np.tile([[0.02, 0.0, 0.0], [0.0, 0.0, 0.0], [0.0, 0.01, 0.0]],
                                (s.n // 3, 1))
    with pytest.raises(md.MDError, match="SHAKE failed to converge"):
        rw1.constrain_positions(s, ref)
    # the context stays usable and the status bit was cleared
    rw, _ = constraint(md)
    assert rw.constrain_positions(s, ref) > 0


def test_atom_count_must_be_triples(md):
    rw, _ = constraint(md)
    s = md.System.from_arrays(np.zeros((4, 3)) + 1.0, np.array([20.0, 20.0, 20.0]))
    with pytest.raises(md.MDError, match="multiple of 3"):
        rw.constrain_velocities(s)


def cvv_oracle_step(st, box, dt, orw, forces):
    """constrained_velocity_verlet.hpp:27-57 in numpy with the same operation order."""
    r, v, f, m = st["pos"], st["vel"], st["frc"], st["m"]
    kc = (0.5 * dt) / m
    ref = r.copy()
    v = v + f * kc[:, None]
    r = r + v * dt
    unc = r.copy()
    r, _ = O.shake(orw, r, ref, m, box)
    v = v + fold(r - unc, box) * (1.0 / dt)
    st2 = dict(st, pos=r)
    f = forces(st2)
    v = v + f * kc[:, None]
    v, _ = O.rattle(orw, r, v, m, box)
    return dict(st, pos=r, vel=v, frc=f)


def test_constrained_step_bit_exact_with_given_forces(md):
    """Three ConstrainedVelocityVerlet steps with the oracle's SPC/E forces fed to
    both sides: positions and velocities are bit-identical."""
    rw, orw = constraint(md)
    s = water(md)
    box = SPCE["box1"]
    thermal_velocities(md, s, 298.0, 2026)
    rw.constrain_velocities(s)
    st = state(s)
    st["frc"] = oracle_forces(st, box)
    s.forces = st["frc"]
    dt = femtoseconds(2.0)
    integ = md.ConstrainedVelocityVerlet(dt, rw)

    def gpu_forces(sys):
        sys.forces = oracle_forces(state(sys), box)

    for _ in range(3):
        integ.step(s, gpu_forces)
        st = cvv_oracle_step(st, box, dt, orw, lambda x: oracle_forces(x, box))
        assert np.array_equal(s.positions, st["pos"])
        assert np.array_equal(s.velocities, st["vel"])
    shake_it, rattle_it = integ.iterations()
    assert shake_it > 1 and rattle_it > 1


def test_geometry_held_over_trajectory(md):
    """tests/test_rigid_water.cpp:127-151: 50 steps of 2 fs under full SPC/E
    forces keep every constraint within 1e-10."""
    rw, _ = constraint(md)
    s = water(md)
    ff = md.SpceForceField()
    ff.compute_forces(s)
    integ = md.ConstrainedVelocityVerlet(femtoseconds(2.0), rw)
    worst = 0.0
    for _ in range(50):
        integ.step(s, ff.compute_forces)
        worst = max(worst, worst_geometry(s.positions, SPCE["box1"], rw.oh_distance(),
                                          rw.hh_distance()))
    assert worst < 1e-10


def test_fused_loop_matches_host_loop(md):
    """md_run_spce (device-decided list rebuilds, no host round trips) follows the
    host-driven step loop."""
    rw, _ = constraint(md)
    dt = femtoseconds(2.0)
    a, b = water(md), water(md)
    for sys in (a, b):
        thermal_velocities(md, sys, 298.0, 11)
        rw.constrain_velocities(sys)
    ffa, ffb = md.SpceForceField(), md.SpceForceField()
    ffa.compute_forces(a)
    ia = md.ConstrainedVelocityVerlet(dt, rw)
    for _ in range(40):
        ia.step(a, ffa.compute_forces)
    ib = md.ConstrainedVelocityVerlet(dt, rw)
    rows = ib.run(b, ffb, 40, thermo=True)
    assert np.allclose(b.positions, a.positions, rtol=0, atol=1e-11)
    assert np.allclose(b.velocities, a.velocities, rtol=0, atol=1e-11)
    e_host = ffa.compute_energy(a)
    assert abs(rows[-1, 0] - e_host) < 1e-9 * abs(e_host)
    assert abs(rows[-1, 2] - a.kinetic_energy()) < 1e-10 * a.kinetic_energy()


def continuous_forcefield(md, sys):
    """Oxygen-oxygen LJ with the force shifted to zero at 9 A and no charges
    (tests/test_rigid_water.cpp:189-205)."""
    sys.charges = np.zeros(sys.n)
    return md.SpceForceField(cutoff=9.0, truncation=md.Truncation.LinearForceShift)


def test_energy_error_scales_as_dt_squared(md):
    """tests/test_rigid_water.cpp:153-251 on the fused device loop: the maximum
    energy deviation over 100 fs fits a slope in (1.85, 2.15) against dt."""
    rw, _ = constraint(md)
    log_dt, log_err = [], []
    for fs in (0.5, 1.0, 2.0, 4.0):
        s = water(md)
        ff = continuous_forcefield(md, s)
        thermal_velocities(md, s, 298.0, 2026)
        s.remove_center_of_mass_motion()
        rw.constrain_velocities(s)
        e0 = ff.compute_forces(s) + s.kinetic_energy()
        steps = int(round(100.0 / fs))
        rows = md.ConstrainedVelocityVerlet(femtoseconds(fs), rw).run(s, ff, steps, thermo=True)
        dev = np.max(np.abs(rows[:, 0] + rows[:, 2] - e0))
        log_dt.append(math.log(fs))
        log_err.append(math.log(dev / abs(e0)))
    slope = np.polyfit(log_dt, log_err, 1)[0]
    assert 1.85 < slope < 2.15, (slope, np.exp(log_err))


def test_nhc_constrained_follows_oracle(md):
    """The chain around the constrained step: integrateChain(dt/2), the RATTLE
    step, integrateChain(dt/2) -- against the oracle's chain and the numpy step
    with the same forces.  The device tracks the chain's kinetic energy with
    its own reductions, so agreement is to rounding, not bit-exact."""
    rw, orw = constraint(md)
    s = water(md)
    box = SPCE["box1"]
    thermal_velocities(md, s, 350.0, 5)
    s.remove_center_of_mass_motion()
    rw.constrain_velocities(s)
    st = state(s)
    st["frc"] = oracle_forces(st, box)
    s.forces = st["frc"]
    dt, temp, tau = femtoseconds(1.0), 298.0, femtoseconds(50.0)
    dof = md.RigidWater.degrees_of_freedom(s.n // 3, True)
    integ = md.ConstrainedNoseHooverChain(dt, rw, temp, tau, 3, dof)
    chain = O.nhc(dt, temp, tau, 3, dof)

    def gpu_forces(sys):
        sys.forces = oracle_forces(state(sys), box)

    for _ in range(10):
        integ.step(s, gpu_forces)
        st["vel"] = O.nhc_chain(chain, st["vel"], st["m"], 0.5 * dt)
        st = cvv_oracle_step(st, box, dt, orw, lambda x: oracle_forces(x, box))
        st["vel"] = O.nhc_chain(chain, st["vel"], st["m"], 0.5 * dt)
    assert np.allclose(s.positions, st["pos"], rtol=0, atol=1e-11)
    assert np.allclose(s.velocities, st["vel"], rtol=1e-10, atol=1e-12)
    want = O.nhc_conserved(chain)
    assert abs(integ.conserved_quantity_contribution() - want) < 1e-9 * (1 + abs(want))


def test_nhc_constrained_thermostats_and_conserves(md):
    """A hot start relaxes to the target temperature; the extended energy
    H' = PE + KE + chain contribution stays within 1e-3 (relative) over 4 ps
    with the continuous force field."""
    rw, _ = constraint(md)
    s = water(md)
    ff = continuous_forcefield(md, s)
    thermal_velocities(md, s, 400.0, 3)
    s.remove_center_of_mass_motion()
    rw.constrain_velocities(s)
    dof = md.RigidWater.degrees_of_freedom(s.n // 3, True)
    integ = md.ConstrainedNoseHooverChain(femtoseconds(1.0), rw, 298.0, femtoseconds(50.0), 3,
                                          dof)
    e0 = ff.compute_forces(s) + s.kinetic_energy()
    rows = integ.run(s, ff, 4000, thermo=True)
    h = rows[:, 0] + rows[:, 2] + rows[:, 3]
    assert np.max(np.abs(h - e0)) < 1e-3 * abs(e0), np.max(np.abs(h - e0)) / abs(e0)
    t = 2.0 * rows[2000:, 2] / dof
    assert abs(t.mean() - 298.0) < 0.1 * 298.0, t.mean()
    assert worst_geometry(s.positions, SPCE["box1"], rw.oh_distance(), rw.hh_distance()) < 1e-10


# ----------------------------------------------------------------- SETTLE
def settle_constraint(md):
    p = md.SpceParameters
    return md.RigidWater(p.rOH, p.angleHOH, settle=True)


@pytest.mark.parametrize("c", [1, 2])
def test_settle_positions_are_shakes_fixed_point(md, c):
    """rigid_water.hpp:20-24: SETTLE must reproduce SHAKE to machine precision --
    here to SHAKE's own tolerance (1e-12 relative on r^2) -- on the displaced
    NIST sites, without iterating and without moving any centre of mass."""
    rw = settle_constraint(md)
    _, orw = constraint(md)
    s = water(md, c)
    box = SPCE[f"box{c}"]
    ref = s.positions
    i = np.arange(s.n)
    sh = 0.01 * (i % 7) - 0.03
    disp = ref + np.stack([sh, -0.5 * sh, 0.25 * sh], 1)
    s.positions = disp
    m = s.masses
    it = rw.constrain_positions(s, ref)
    got = s.positions
    want, _ = O.shake(orw, disp, ref, m, box)
    assert it == 1
    assert np.max(np.abs(got - want)) < 1e-11
    assert worst_geometry(got, box, rw.oh_distance(), rw.hh_distance()) < 1e-13
    com = lambda p: np.add.reduceat(p * m[:, None], np.arange(0, s.n, 3)) / np.add.reduceat(
        m, np.arange(0, s.n, 3))[:, None]
    assert np.max(np.linalg.norm(com(got) - com(disp), axis=1)) < 1e-12


def test_settle_velocities_are_rattles_fixed_point(md):
    rw = settle_constraint(md)
    _, orw = constraint(md)
    s = water(md)
    thermal_velocities(md, s, 298.0, 21)
    vel = s.velocities
    it = rw.constrain_velocities(s)
    got = s.velocities
    want, _ = O.rattle(orw, s.positions, vel, s.masses, SPCE["box1"])
    assert it == 1
    assert np.max(np.abs(got - want)) < 1e-10 * np.max(np.abs(want))
    # no velocity left along any bond
    pos = s.positions
    for i, j in ((0, 1), (0, 2), (1, 2)):
        d = fold(pos[i::3] - pos[j::3], SPCE["box1"])
        rel = np.sum((got[i::3] - got[j::3]) * d, axis=1)
        assert np.max(np.abs(rel)) < 1e-12 * np.max(np.abs(got))


def test_settle_trajectory_tracks_shake(md):
    """50 constrained steps of 2 fs under full SPC/E forces: SETTLE and SHAKE/RATTLE
    stay within roundoff of each other over the run, and SETTLE holds the geometry
    to 1e-12."""
    rw_s = settle_constraint(md)
    rw, _ = constraint(md)
    runs = []
    for r in (rw, rw_s):
        s = water(md)
        thermal_velocities(md, s, 298.0, 5)
        r.constrain_velocities(s)
        ff = md.SpceForceField()
        ff.compute_forces(s)
        md.ConstrainedVelocityVerlet(femtoseconds(2.0), r).run(s, ff, 50)
        runs.append(s.positions)
    assert np.max(np.abs(runs[0] - runs[1])) < 1e-6
    assert worst_geometry(runs[1], SPCE["box1"], rw.oh_distance(), rw.hh_distance()) < 1e-12
