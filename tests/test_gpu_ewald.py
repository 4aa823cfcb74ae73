"""GPU parity of the Ewald sum and the SPC/E force field against the reference's
golden outputs and NIST's published SPC/E values (the reference's
tests/test_nist_spce.cpp restated against the CUDA path)."""
import math

import numpy as np
import pytest

import oracle as O
from conftest import load_golden

pytestmark = pytest.mark.gpu

SPCE = load_golden("nist_spce.npz")


def approx_eq(a, b, eps):
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    return np.all(np.abs(a - b) < eps * (1.0 + np.maximum(np.abs(a), np.abs(b))))


def half_width(value):
    mag = abs(value)
    return 0.0 if mag == 0 else 0.5 * 10.0 ** (math.floor(math.log10(mag)) - 5)


def water(md, c):
    types = ["O" if o else "H" for o in SPCE[f"isO{c}"]]
    return md.build_spce_system(SPCE[f"pos{c}"], types, SPCE[f"box{c}"])


def test_coulomb_prefactor(md):
    assert abs(md.coulomb_prefactor() - 167100.956632) < 1e-9 * 167100.956632
    assert md.coulomb_prefactor() == float(SPCE["coulomb"])


@pytest.mark.parametrize("c", [1, 2, 3, 4])
def test_nist_spce_terms_on_gpu(md, c):
    """tests/test_nist_spce.cpp:93-153: every term within NIST's 6th-figure
    half-width, and within 1e-12 of the reference's own values."""
    s = water(md, c)
    ew = md.Ewald(10.0, 5)
    t = ew.compute_energies(s)
    ref = SPCE[f"ewald_terms{c}"]
    got = np.array([t["real"], t["reciprocal"], t["self"], t["intra"]])
    assert approx_eq(got, ref, 1e-12), (got, ref)
    ff = md.SpceForceField(10.0, 5)
    e = ff.compute_energy(s)
    pub = SPCE["published"][c - 1]
    comps = [ff.parts["disp"], ff.parts["lrc"], ff.parts["real"], ff.parts["reciprocal"],
             ff.parts["self"], ff.parts["intra"]]
    tol_sum = 0.0
    for g, r in zip(comps, pub[1:7]):
        assert abs(g - r) <= half_width(r)
        tol_sum += half_width(r)
    assert abs(e - pub[7]) / abs(pub[7]) <= tol_sum / abs(pub[7])
    assert approx_eq(e, float(SPCE[f"spce_energy{c}"]), 1e-12)


@pytest.mark.parametrize("c", [1, 2, 3, 4])
def test_ewald_and_spce_forces_match_reference(md, c):
    s = water(md, c)
    ew = md.Ewald(10.0, 5)
    ew.compute_forces(s)
    assert approx_eq(s.forces, SPCE[f"ewald_forces{c}"], 1e-11)
    ff = md.SpceForceField(10.0, 5)
    e = ff.compute_forces(s)
    assert approx_eq(s.forces, SPCE[f"spce_forces{c}"], 1e-11)
    assert approx_eq(e, float(SPCE[f"spce_energy{c}"]), 1e-12)


def test_accumulate_adds_onto_existing_forces(md):
    s = water(md, 1)
    f0 = np.random.default_rng(0).normal(size=(s.n, 3))
    s.forces = f0
    md.Ewald(10.0, 5).accumulate_forces(s)
    assert approx_eq(s.forces - f0, SPCE["ewald_forces1"], 1e-10)


def test_ewald_forces_equal_minus_gradient(md):
    """tests/test_nist_spce.cpp:155-204 (FD h=1e-5, tol 1e-7)."""
    s = water(md, 1)
    ew = md.Ewald(10.0, 5)
    ew.compute_forces(s)
    f = s.forces
    pos = SPCE["pos1"].copy()
    h = 1e-5
    for i in (0, 1, 2, 150, 299):
        for d in range(3):
            p = pos.copy()
            p[i, d] += h
            s.positions = p
            up = ew.compute_energies(s).total()
            p[i, d] -= 2 * h
            s.positions = p
            um = ew.compute_energies(s).total()
            num = -(up - um) / (2 * h)
            assert approx_eq(f[i, d], num, 1e-7), (i, d, f[i, d], num)
    s.positions = pos


def test_ewald_newton_third_law(md):
    """tests/test_nist_spce.cpp:206-220"""
    s = water(md, 2)
    md.Ewald(10.0, 5).compute_forces(s)
    assert np.all(np.abs(s.forces.sum(0)) < 1e-8)


def test_ewald_virial_equals_scaling_derivative(md):
    """No reference counterpart: W = -dE/ds for r -> s r, L -> s L at fixed alpha."""
    box = SPCE["box1"]
    alpha = 5.6 / box.min()
    types = ["O" if o else "H" for o in SPCE["isO1"]]
    s = md.build_spce_system(SPCE["pos1"], types, box)
    ew = md.Ewald(9.9, 5, alpha=alpha)
    ew.compute_energies(s)
    w = ew.last_virial
    h = 1e-6
    e = []
    for sc in (1 + h, 1 - h):
        ss = md.build_spce_system(SPCE["pos1"] * sc, types, box * sc)
        e.append(md.Ewald(9.9 * sc, 5, alpha=alpha).compute_energies(ss).total())
    w_fd = -(e[0] - e[1]) / (2 * h)
    assert abs(w - w_fd) <= 1e-6 * abs(w), (w, w_fd)
    _, _, w_orc = O.ewald(SPCE["pos1"], box, np.where(SPCE["isO1"], -0.8476, 0.4238),
                          np.arange(len(types)) // 3, cutoff=9.9, alpha=alpha, forces=False)
    assert abs(w - w_orc) <= 1e-10 * abs(w_orc)


def test_ewald_alpha_override_matches_oracle(md):
    """Tuned alpha / kmax (config-4 style) against the oracle restatement."""
    s = water(md, 3)
    ew = md.Ewald(9.0, 7, alpha=0.3)
    t = ew.compute_energies(s)
    _, ot, _ = O.ewald(SPCE["pos3"], SPCE["box3"], s.charges, np.arange(s.n) // 3, cutoff=9.0,
                       kmax=7, alpha=0.3, forces=False)
    for k in ("real", "reciprocal", "self", "intra"):
        assert approx_eq(t[k], ot[k], 1e-12), (k, t[k], ot[k])


def test_charge_gradient_matches_differences(md):
    """dE/dq_i of the Coulomb energy (real + reciprocal + self + intra) against
    central differences; the energy is quadratic in each charge, so the
    differences are exact up to rounding."""
    s = water(md, 1)
    ew = md.Ewald(10.0, 5)
    dedq = ew.charge_gradient(s)
    q0 = s.charges
    rng = np.random.default_rng(3)
    for i in rng.integers(0, s.n, 6):
        h = 1e-3 * abs(q0[i])
        e = []
        for sign in (1, -1):
            q = q0.copy()
            q[i] += sign * h
            s.charges = q
            e.append(ew.compute_energies(s).total())
        s.charges = q0
        fd = (e[0] - e[1]) / (2 * h)
        assert abs(dedq[i] - fd) < 1e-8 * abs(fd), (i, dedq[i], fd)


def test_real_space_hvp_matches_force_differences(md):
    """With every site its own molecule and no k vectors the Ewald force is the
    real-space force alone; its Hessian-vector product against differences."""
    rng = np.random.default_rng(5)
    pos = SPCE["pos1"][::3].copy()  # oxygens: no two sites closer than ~2.5 A
    n = pos.shape[0]
    box = SPCE["box1"]
    q = rng.choice([-0.8, 0.8], size=n)
    s = md.System.from_arrays(pos, box, charge=q, mol=np.arange(n))
    ew = md.Ewald(8.0, 0)
    u = rng.normal(size=(n, 3))
    hvp = ew.real_space_hvp(s, u)
    h = 1e-5

    def forces(p):
        t = md.System.from_arrays(p, box, charge=q, mol=np.arange(n))
        md.Ewald(8.0, 0).compute_forces(t)
        return t.forces

    fd = (forces(pos + h * u) - forces(pos - h * u)) / (2 * h)
    assert np.max(np.abs(hvp - fd)) < 1e-6 * np.max(np.abs(fd))
