"""GPU smooth PME (pme.cu) against the oracle's numpy restatement of the same
method (Essmann et al. 1995) and against the Ewald k-vector sum, which is
pinned to the reference (forcefield/ewald.cpp).

The device spreads charges as 64-bit fixed-point integers (2^-46 e) and sums
in other orders than numpy, so energies, virials and forces agree with the
restatement to ~1e-11 relative, not bitwise; repeated evaluations on the device
are bitwise identical."""
import numpy as np
import pytest

import oracle as O
from conftest import load_golden

pytestmark = pytest.mark.gpu

SPCE = load_golden("nist_spce.npz")


def water(md, c):
    types = ["O" if o else "H" for o in SPCE[f"isO{c}"]]
    return md.build_spce_system(SPCE[f"pos{c}"], types, SPCE[f"box{c}"])


def recip_forces(md, s, ew):
    """PME (or k-sum) reciprocal forces: total forces minus the kmax = 0 run
    (identical real-space and intramolecular passes)."""
    t = ew.compute_forces(s)
    f = s.forces
    w = ew.last_virial
    base = md.Ewald(10.0, 0, ew.alpha())
    t0 = base.compute_forces(s)
    return t, f - s.forces, w - base.last_virial


@pytest.mark.parametrize("c,K,order", [(1, 24, 4), (1, 32, 6), (3, 28, 8), (4, 40, 6),
                                       (2, (30, 30, 36), 6)])
def test_pme_equals_the_restatement(md, c, K, order):
    s = water(md, c)
    box = SPCE[f"box{c}"]
    ew = md.Ewald(10.0, 5)
    ew.set_pme(K, order)
    assert ew.pme_grid() == ((K,) * 3 if np.isscalar(K) else tuple(K), order)
    t, f, w = recip_forces(md, s, ew)
    q = s.charges
    e_or, w_or, f_or = O.pme_recip(s.positions, box, q, ew.alpha(), K, order)
    assert t["reciprocal"] == pytest.approx(e_or, rel=1e-11)
    assert w == pytest.approx(w_or, rel=1e-9, abs=1e-9 * abs(e_or))
    scale = np.sqrt(np.mean(f_or ** 2))
    assert np.max(np.abs(f - f_or)) < 1e-9 * scale


def test_pme_in_a_non_cubic_box(md):
    """Configuration 1 stretched by (1, 1.25, 1.1) along the axes (the sites
    scaled with the box): unequal box lengths and grid spacings per axis."""
    scale = np.array([1.0, 1.25, 1.1])
    types = ["O" if o else "H" for o in SPCE["isO1"]]
    box = SPCE["box1"] * scale
    s = md.build_spce_system(SPCE["pos1"] * scale, types, box)
    ew = md.Ewald(10.0, 5, 0.3)
    ew.set_pme((24, 30, 28), 6)
    t, f, w = recip_forces(md, s, ew)
    e_or, w_or, f_or = O.pme_recip(s.positions, box, s.charges, 0.3, (24, 30, 28), 6)
    assert t["reciprocal"] == pytest.approx(e_or, rel=1e-11)
    assert w == pytest.approx(w_or, rel=1e-9, abs=1e-9 * abs(e_or))
    assert np.max(np.abs(f - f_or)) < 1e-9 * np.sqrt(np.mean(f_or ** 2))


def test_pme_converges_to_the_ewald_sum(md):
    s = water(md, 1)
    ew = md.Ewald(10.0, 12)
    t_k, f_k, w_k = recip_forces(md, s, ew)
    errs = []
    for K, order in ((16, 4), (32, 6), (48, 8)):
        pme = md.Ewald(10.0, 5)
        pme.set_pme(K, order)
        t, f, w = recip_forces(md, s, pme)
        errs.append((abs(t["reciprocal"] - t_k["reciprocal"]) / abs(t_k["reciprocal"]),
                     np.sqrt(np.mean((f - f_k) ** 2) / np.mean(f_k ** 2))))
    errs = np.array(errs)
    assert np.all(np.diff(errs, axis=0) < 0)
    assert errs[-1, 0] < 1e-8 and errs[-1, 1] < 1e-7


def test_pme_is_deterministic_and_switches_back(md):
    s = water(md, 4)
    ew = md.Ewald(10.0, 5)
    ref_terms = ew.compute_forces(s)
    ref_forces = s.forces
    ew.set_pme(40, 6)
    a = ew.compute_forces(s)
    fa = s.forces
    b = ew.compute_forces(s)
    assert a == b and np.array_equal(fa, s.forces)
    ew.set_pme(None)
    assert ew.pme_grid() == ((0, 0, 0), 0)
    assert ew.compute_forces(s) == ref_terms and np.array_equal(s.forces, ref_forces)


def test_pme_rejects_bad_grids_and_the_charge_gradient(md):
    s = water(md, 1)
    ew = md.Ewald(10.0, 5)
    for K, order in ((7, 4), (32, 5), (32, 10), ((32, 32, 11), 6)):
        with pytest.raises(md.InvalidArgument):
            ew.set_pme(K, order)
    ew.set_pme(32, 6)
    with pytest.raises(md.InvalidArgument, match="k-vector"):
        ew.charge_gradient(s)


def test_spce_with_pme_conserves_energy(md):
    """A constrained NVE run with PME forces conserves the total energy about
    as well as with the k-vector sum."""
    drift = {}
    for use_pme in (False, True):
        s = water(md, 1)
        s.velocities = np.sqrt(300.0 / s.masses)[:, None] * O.rng_normals(5, 3 * s.n).reshape(-1, 3)
        rw = md.RigidWater(1.0, 109.47)
        rw.constrain_velocities(s)
        ff = md.SpceForceField(kmax=7)
        if use_pme:
            ff.set_pme_spacing(s.box, 0.6, 6)
        integ = md.ConstrainedVelocityVerlet(md.units.femtoseconds(1.0), rw)
        th = integ.run(s, ff, 300, thermo=True)
        h = th[:, 0] + th[:, 2]
        drift[use_pme] = np.max(np.abs(h - h[0])) / np.mean(np.abs(th[:, 2]))
    assert drift[True] < 2e-3 and drift[True] < 3 * drift[False] + 1e-4
