"""FP64 parity at the sizes and lengths the configurations name.

* The 1,048,576-atom liquid of the large-system configuration: one FP64
  force / energy / virial evaluation over the Verlet list and the list's pair set
  equal the compiled reference's VerletList::build + LennardJones::computeForces
  (neighbor/verlet_list.cpp:8-42, forcefield/lennard_jones.cpp:50-119) on the same
  state -- forces, energy and virial to 1e-12 relative, pairs exactly.  The state
  is the liquid the reference itself equilibrated (2000 LangevinBAOAB steps,
  oracle/make_lj1m_state.py) when that build artefact is present, else the lattice
  after 100 BAOAB steps on the GPU.  38 cells per side, crowded cells and the
  Morton-ordered cell sort are exercised only at this size.
* The 864-atom drop-in configuration over all 1000 velocity-Verlet steps of its
  run: every step's forces, energy and virial equal the oracle's on the GPU's
  state (1e-12), the pair set at every rebuild equals the oracle's list built from
  the same positions, and the trajectory stays on the compiled reference's.
"""
import os

import numpy as np
import pytest

import oracle as O
from conftest import ROOT

pytestmark = pytest.mark.gpu

STATE = os.path.join(ROOT, "oracle", "_ref", "lj1m_baoab2000.npz")


def approx_eq(a, b, eps):
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    return np.all(np.abs(a - b) < eps * (1.0 + np.maximum(np.abs(a), np.abs(b))))


def pair_keys(pairs, n):
    lo = np.minimum(pairs[:, 0], pairs[:, 1]).astype(np.int64)
    hi = np.maximum(pairs[:, 0], pairs[:, 1]).astype(np.int64)
    return np.sort(lo * n + hi)


def liquid_1m(md):
    if os.path.exists(STATE):
        with np.load(STATE) as z:
            return np.array(z["pos"]), np.array(z["box"]), "reference-equilibrated"
    st = md.fcc_lattice(64, 0.8442, 0.722, 2026)
    s = md.System.from_arrays(st["pos"], st["box"], vel=st["vel"], mass=st["mass"])
    lj = md.LennardJones(1.0, 1.0, 2.5)
    v = md.VerletList(st["box"], 2.5, 0.3)
    v.build(s)
    lj.compute_forces(s, v)
    md.LangevinBAOAB(0.005, 1.0, 0.722, 2027).run(s, v, lj, 100)
    return s.positions, st["box"], "lattice + 100 GPU BAOAB steps"


@pytest.mark.skipif(not O.ref_available(), reason="compiled reference (oracle/_ref) absent")
def test_fp64_1m_liquid_forces_and_pairs_equal_reference(md):
    pos, box, _ = liquid_1m(md)
    n = pos.shape[0]
    assert n == 1048576
    s = md.System.from_arrays(pos, box)
    v = md.VerletList(box, 2.5, 0.3)
    v.build(s)
    e, w = md.LennardJones(1.0, 1.0, 2.5).compute_forces(s, v)
    f = s.forces
    pairs = v.pairs()
    fr, er, wr, pr = O.ref_lj_verlet(pos, box, rc=2.5, skin=0.3, trunc=0)
    assert approx_eq(e, er, 1e-12) and approx_eq(w, wr, 1e-12), (e, er, w, wr)
    assert approx_eq(f, fr, 1e-12), np.max(np.abs(f - fr))
    assert len(pairs) == len(pr) and len(pr) > 35 * n  # ~38 half pairs per atom at rc + skin
    assert np.array_equal(pair_keys(pairs, n), pair_keys(pr, n))


def test_vv_c1_shadowed_over_1000_steps(md):
    """moldyn_run's ForceFn (rebuildIfNeeded + computeForces(sys, verlet)) through
    the integrator's step(System&, ForceFn) for the full drop-in run."""
    st = md.fcc_lattice(6, 0.8442, 0.722, 1)
    box = st["box"]
    s = md.System.from_arrays(st["pos"], box, vel=st["vel"], mass=st["mass"])
    lj = md.LennardJones(1.0, 1.0, 2.5)
    v = md.VerletList(box, 2.5, 0.3)
    v.build(s)
    lj.compute_forces(s, v)
    integ = md.VelocityVerlet(0.005)

    def forces(sys_):
        v.rebuild_if_needed(sys_)
        return lj.compute_forces(sys_, v)[0]

    rebuilds = v.rebuild_count()
    checked = 0
    for _ in range(1000):
        integ.step(s, forces)
        pos = s.positions
        fo, eo, wo = O.lj_compute(pos, box, rc=2.5, trunc=0)
        e, w = s.last_energy_virial()
        assert approx_eq(e, eo, 1e-12) and approx_eq(w, wo, 1e-12)
        assert approx_eq(s.forces, fo, 1e-12)
        if v.rebuild_count() != rebuilds:  # rebuilt from this step's drifted positions
            rebuilds = v.rebuild_count()
            assert np.array_equal(pair_keys(v.pairs(), s.n),
                                  pair_keys(O.verlet_pairs(pos, box, 2.5, 0.3), s.n))
            checked += 1
    assert checked >= 10
    if O.ref_available():
        # the same 1000 steps run by the compiled reference from the same lattice
        R = O.ref()
        n = s.n
        x, y, z = (np.ascontiguousarray(st["pos"][:, k]) for k in range(3))
        vx, vy, vz = (np.ascontiguousarray(st["vel"][:, k]) for k in range(3))
        fr = [np.zeros(n) for _ in range(3)]
        info = np.zeros(5)
        R.ref_run(0, n, O._p(np.ascontiguousarray(box)), *[O._p(a) for a in (x, y, z, vx, vy, vz)],
                  *[O._p(a) for a in fr], O._p(np.ascontiguousarray(st["mass"])), 1.0, 1.0, 2.5,
                  0, 0.3, 0.005, 1000, 0.0, 0.0, 0, 0.0, 1, 0, O._p(info))
        assert int(info[2]) == v.rebuild_count()
        # chaotic growth of round-off over 5 time units stays far below a bin of
        # any observable
        dx = np.max(np.abs(s.positions - np.stack([x, y, z], 1)))
        assert dx < 1e-6, dx
