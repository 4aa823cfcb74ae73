"""Pins the CPU oracle (oracle/md_oracle.c) before anything is checked against it.

* against the NIST published values the reference's own tests hold
  (tests/test_nist_lj.cpp:26-39, tests/test_nist_spce.cpp:64-69), at NIST's own
  rounding half-widths, as those tests do;
* against golden outputs of the reference itself (tests/golden/, generated by
  tests/golden/make_golden.py from the compiled reference), bit-for-bit;
* against the compiled reference directly (oracle/_ref), bit-for-bit, when that
  library was built (it needs the reference sources at build time).
"""
import ctypes as C
import math

import numpy as np
import pytest

import oracle as O
from conftest import load_golden

LJ = load_golden("nist_lj.npz")
SPCE = load_golden("nist_spce.npz")
FCC = load_golden("fcc_lj.npz")


def half_width(value, sig_figs):
    """tests/test_nist_lj.cpp:83-90 (5 s.f.) and test_nist_spce.cpp:39-46 (6 s.f.)."""
    mag = abs(value)
    if mag == 0.0:
        return 0.0
    return 0.5 * 10.0 ** (math.floor(math.log10(mag)) - (sig_figs - 1))


def need_ref():
    R = O.ref()
    if R is None:
        pytest.skip("reference library (oracle/_ref) not built here")
    return R


# --------------------------------------------------------------------- NIST LJ
@pytest.mark.parametrize("row", range(12))
def test_nist_lj_within_published_half_width(row):
    c, tr, rc, up, wp, ulrc = LJ["published"][row]
    c, tr = int(c), int(tr)
    _, e, w = O.lj_compute(LJ[f"pos{c}"], LJ[f"box{c}"], rc=rc, trunc=tr, forces=False)
    lrc, _ = O.lj_lrc(len(LJ[f"pos{c}"]), LJ[f"box{c}"], rc=rc, trunc=tr)
    assert abs(e - up) <= half_width(up, 5)
    assert abs(w - wp) <= half_width(wp, 5)
    if ulrc == 0.0:
        assert abs(lrc) <= 1e-12
    else:
        assert abs(lrc - ulrc) <= half_width(ulrc, 5)


@pytest.mark.parametrize("row", range(12))
def test_lj_bit_exact_against_reference_golden(row):
    c, tr, rc, e_ref, w_ref, ul_ref, pl_ref = LJ["computed"][row]
    c, tr = int(c), int(tr)
    f, e, w = O.lj_compute(LJ[f"pos{c}"], LJ[f"box{c}"], rc=rc, trunc=tr)
    assert e == e_ref and w == w_ref
    assert np.array_equal(f, LJ[f"forces{c}_{int(rc)}_{tr}"])
    ul, pl = O.lj_lrc(len(f), LJ[f"box{c}"], rc=rc, trunc=tr)
    assert ul == ul_ref and pl == pl_ref


def test_lrc_pressure_points():
    # tests/test_nist_lj.cpp:157-175: U_LRC/N and P_LRC within 2e-3 (doctest Approx)
    for rho, rc, u_n, p in LJ["lrc_points"]:
        n = 500
        side = (n / rho) ** (1.0 / 3.0)
        ul, pl = O.lj_lrc(n, [side] * 3, rc=rc, trunc=0)
        assert abs(ul / n - u_n) < 2e-3 * (1 + max(abs(ul / n), abs(u_n)))
        assert abs(pl - p) < 2e-3 * (1 + max(abs(pl), abs(p)))


@pytest.mark.parametrize("c", [1, 2, 3, 4])
def test_cell_and_verlet_pairs_match_reference_order(c):
    pos, box = LJ[f"pos{c}"], LJ[f"box{c}"]
    assert tuple(O.cells_dims(box, 3.0)) == tuple(LJ[f"celldims{c}"])
    v = O.verlet_pairs(pos, box, 3.0, 0.3)
    assert np.array_equal(v, LJ[f"verlet{c}"])
    cells = O.cell_pairs(pos, box, 3.0)
    assert len(cells) == int(LJ[f"ncellpairs{c}"])
    if f"cells{c}" in LJ:
        assert np.array_equal(cells, LJ[f"cells{c}"])


def test_verlet_forces_equal_brute_to_1e12():
    # tests/test_neighbor.cpp:100-128
    pos, box = LJ["pos1"], LJ["box1"]
    fb, eb, wb = O.lj_compute(pos, box, rc=3.0)
    fv, ev, wv = O.lj_compute(pos, box, rc=3.0, source="pairs", pairs=O.verlet_pairs(pos, box, 3.0, 0.3))
    fc, ec, wc = O.lj_compute(pos, box, rc=3.0, source="cells")
    for (f, e, w) in ((fv, ev, wv), (fc, ec, wc)):
        assert abs(e - eb) < 1e-12 * (1 + abs(eb))
        assert abs(w - wb) < 1e-12 * (1 + abs(wb))
        assert np.all(np.abs(f - fb) < 1e-12 * (1 + np.maximum(np.abs(f), np.abs(fb))))


def test_unusable_cell_list_raises():
    # tests/test_neighbor.cpp:84-98
    pos = np.array([[0.0, 0.0, 0.0], [1.1, 0.0, 0.0]])
    with pytest.raises(ValueError):
        O.lj_compute(pos, [5.0, 5.0, 5.0], rc=3.0, source="cells")


def test_rebuild_trigger_cases():
    # tests/test_neighbor.cpp:130-159
    pos, box = LJ["pos1"], LJ["box1"]
    skin = 0.3
    moved = pos.copy()
    moved[0, 0] += 0.3 * skin
    assert not O.needs_rebuild(moved, pos, box, skin)
    moved = pos.copy()
    moved[0, 0] += 0.6 * skin
    moved[1, 1] += 0.6 * skin
    assert O.needs_rebuild(moved, pos, box, skin)


# --------------------------------------------------------------- lattice, RNG
@pytest.mark.parametrize("tag,args", [("c6", (6, 0.8442, 0.722, 1)), ("c3", (3, 0.80, 1.0, 12345))])
def test_fcc_lattice_bit_exact(tag, args):
    st = O.fcc_lattice(*args)
    assert np.array_equal(st["pos"], FCC[f"{tag}_pos"])
    assert np.array_equal(st["vel"], FCC[f"{tag}_vel"])
    assert np.array_equal(st["box"], FCC[f"{tag}_box"])


def test_velocity_verlet_trajectory_bit_exact():
    # 25 moldyn_run-style NVE steps (VerletList ForceFn) of the N=864 drop-in config
    s = O.Sim(FCC["c6_pos"], FCC["c6_vel"], np.ones(864), FCC["c6_box"], rc=2.5, trunc=0,
              skin=0.3, dt=0.005)
    s.prime()
    s.run("vv", 25)
    p, v, f = s.state()
    assert np.array_equal(p, FCC["vv25_pos"])
    assert np.array_equal(v, FCC["vv25_vel"])
    assert np.array_equal(f, FCC["vv25_frc"])
    e_ref, w_ref, rebuilds, _ = FCC["vv25_info"]
    assert s.energy == e_ref and s.virial == w_ref and s.rebuild_count == rebuilds


# ------------------------------------------------------------ NIST SPC/E
@pytest.mark.parametrize("c", [1, 2, 3, 4])
def test_nist_spce_terms_within_published_half_width(c):
    pub = SPCE["published"][c - 1]
    pos, box, iso = SPCE[f"pos{c}"], SPCE[f"box{c}"], SPCE[f"isO{c}"]
    n = len(pos)
    q = np.where(iso, -2.0 * 0.42380, 0.42380)
    mol = np.arange(n) // 3
    _, terms, _ = O.ewald(pos, box, q, mol, forces=False)
    ox = pos[iso]
    _, edisp, _ = O.lj_compute(ox, box, sigma=3.16555789, eps=78.19743111, rc=10.0, forces=False)
    elrc, _ = O.lj_lrc(len(ox), box, sigma=3.16555789, eps=78.19743111, rc=10.0)
    got = [edisp, elrc, terms["real"], terms["reciprocal"], terms["self"], terms["intra"]]
    tol_sum = 0.0
    for g, r in zip(got, pub[1:7]):
        assert abs(g - r) <= half_width(r, 6)
        tol_sum += half_width(r, 6)
    assert abs(sum(got) - pub[7]) / abs(pub[7]) <= tol_sum / abs(pub[7])
    assert abs(O.lib().orc_coulomb_prefactor() - 167100.956632) < 1e-9 * 167100.956632


@pytest.mark.parametrize("c", [1, 2])
def test_ewald_and_spce_match_reference_golden(c):
    pos, box, iso = SPCE[f"pos{c}"], SPCE[f"box{c}"], SPCE[f"isO{c}"]
    n = len(pos)
    q = np.where(iso, -2.0 * 0.42380, 0.42380)
    mol = np.arange(n) // 3
    f, terms, _ = O.ewald(pos, box, q, mol)
    ref_terms = SPCE[f"ewald_terms{c}"]
    got = np.array([terms["real"], terms["reciprocal"], terms["self"], terms["intra"]])
    # real/recip/self follow the reference's loop order exactly; the intra sum's
    # order over molecules follows the reference's unordered_map, so allow rounding.
    assert np.array_equal(got[:3], ref_terms[:3])
    assert abs(got[3] - ref_terms[3]) <= 1e-12 * abs(ref_terms[3])
    assert np.array_equal(f, SPCE[f"ewald_forces{c}"])
    fs, e = O.spce(pos, box, q, mol)
    assert abs(e - float(SPCE[f"spce_energy{c}"])) <= 1e-12 * abs(e)
    assert np.array_equal(fs, SPCE[f"spce_forces{c}"])


def test_ewald_virial_equals_scaling_derivative():
    # No reference counterpart: W = -dE/ds at s=1 for r -> s r, L -> s L, fixed alpha.
    pos, box, iso = SPCE["pos1"], SPCE["box1"], SPCE["isO1"]
    q = np.where(iso, -2.0 * 0.42380, 0.42380)
    mol = np.arange(len(pos)) // 3
    alpha = 5.6 / box.min()
    _, _, w = O.ewald(pos, box, q, mol, alpha=alpha, cutoff=9.9, forces=False)
    h = 1e-6
    e = []
    for s in (1 + h, 1 - h):
        _, t, _ = O.ewald(pos * s, box * s, q, mol, alpha=alpha, cutoff=9.9 * s, forces=False)
        e.append(sum(t.values()))
    w_fd = -(e[0] - e[1]) / (2 * h)
    assert abs(w - w_fd) <= 1e-6 * abs(w)


# ----------------------------------------------------------- rigid water
def water_state(c=1):
    pos, box, iso = SPCE[f"pos{c}"], SPCE[f"box{c}"], SPCE[f"isO{c}"]
    m = np.where(iso, 15.9994, 1.008)
    return pos, box, m


def test_shake_conserves_com_and_geometry():
    # tests/test_rigid_water.cpp:94-133
    pos, box, m = water_state()
    rw = O.rigid_water()
    n = len(pos)
    disp = np.array([[0.01 * (i % 7) - 0.03] * 3 for i in range(n)]) * np.array([1.0, -0.5, 0.25])
    moved = pos + disp
    out, it = O.shake(rw, moved, pos, m, box)
    assert it > 0
    com0 = (moved * m[:, None]).reshape(-1, 3, 3).sum(1) / m.reshape(-1, 3).sum(1)[:, None]
    com1 = (out * m[:, None]).reshape(-1, 3, 3).sum(1) / m.reshape(-1, 3).sum(1)[:, None]
    assert np.abs(com1 - com0).max() < 1e-10


def test_shake_rattle_match_reference():
    R = need_ref()
    pos, box, m = water_state()
    n = len(pos)
    rng = np.random.default_rng(7)
    moved = pos + rng.normal(scale=0.01, size=pos.shape)
    vel = rng.normal(scale=1.0, size=pos.shape)
    rw = O.rigid_water()
    mine, it = O.shake(rw, moved, pos, m, box)
    st = [np.ascontiguousarray(moved[:, k]) for k in range(3)] + \
         [np.ascontiguousarray(vel[:, k]) for k in range(3)]
    rc = [np.ascontiguousarray(pos[:, k]) for k in range(3)]
    it_ref = R.ref_rigid_water(0, n, O._p(box), O._p(m), *[O._p(a) for a in st],
                               *[O._p(a) for a in rc], 1.0, 109.47, 1e-12, 500)
    assert it == it_ref
    assert np.array_equal(mine, np.stack(st[:3], 1))
    vmine, it = O.rattle(rw, mine, vel, m, box)
    it_ref = R.ref_rigid_water(1, n, O._p(box), O._p(m), *[O._p(a) for a in st],
                               *[O._p(a) for a in rc], 1.0, 109.47, 1e-12, 500)
    assert it == it_ref
    assert np.array_equal(vmine, np.stack(st[3:6], 1))


# -------------------------------------------- integrators vs the reference run
@pytest.mark.parametrize("kind", ["vv", "baoab", "nhc"])
def test_integrators_bit_exact_against_reference(kind):
    R = need_ref()
    st = O.fcc_lattice(3, 0.80, 1.0, 12345)
    n = len(st["mass"])
    steps = 40
    s = O.Sim(st["pos"], st["vel"], st["mass"], st["box"], rc=2.5, trunc=1, skin=0.3, dt=0.005)
    if kind == "baoab":
        s.set_langevin(1.0, 1.0, 777)
    if kind == "nhc":
        s.set_nhc(1.0, 0.5, 3, 3 * n - 3)
    s.prime()
    s.run(kind, steps)
    p, v, f = s.state()
    arrs = [np.ascontiguousarray(st["pos"][:, k]) for k in range(3)] + \
           [np.ascontiguousarray(st["vel"][:, k]) for k in range(3)] + [np.zeros(n) for _ in range(3)]
    info = np.zeros(5)
    k = {"vv": 0, "baoab": 1, "nhc": 2}[kind]
    R.ref_run(k, n, O._p(st["box"]), *[O._p(a) for a in arrs], O._p(st["mass"]), 1.0, 1.0, 2.5,
              1, 0.3, 0.005, steps, 1.0, 1.0, 777, 0.5, 3, 3 * n - 3, O._p(info))
    assert np.array_equal(p, np.stack(arrs[0:3], 1))
    assert np.array_equal(v, np.stack(arrs[3:6], 1))
    assert np.array_equal(f, np.stack(arrs[6:9], 1))
    assert s.energy == info[0] and s.virial == info[1] and s.rebuild_count == info[2]
    if kind == "nhc":
        assert s.nhc_conserved == info[3]


def test_rng_matches_reference():
    R = need_ref()
    a = O.rng_normals(2026, 5001)
    b = np.zeros(5001)
    R.ref_rng_normals(2026, O._p(b), 5001)
    assert np.array_equal(a, b)


# ------------------------------------------------------------------ analyze/
def random_walk(n, frames, box, step, seed):
    """Seeded wrapped positions and velocities, (frames, n, 3) each; steps of
    `step` per frame cross the periodic boundaries often."""
    rng = np.random.default_rng(seed)
    box = np.asarray(box, dtype=float)
    p = (rng.random((n, 3)) - 0.5) * box
    pos, vel = [], []
    for _ in range(frames):
        v = rng.normal(0.0, 1.0, (n, 3))
        p = p + step * v
        p = p - box * np.floor(p / box + 0.5)
        pos.append(p.copy())
        vel.append(v)
    return np.array(pos), np.array(vel)


def test_rdf_restatement_matches_reference():
    need_ref()
    box = np.array([7.0, 7.5, 8.0])
    pos, _ = random_walk(200, 4, box, 0.3, 11)
    hist, g = O.rdf(pos, box, 3.4, 40)
    g_ref, centres = O.ref_rdf(pos, box, 3.4, 40)
    assert np.array_equal(g, g_ref)
    assert np.array_equal(centres, (np.arange(40) + 0.5) * (3.4 / 40))
    assert hist.sum() > 0 and np.all(hist == np.round(hist))
    with pytest.raises(ValueError):
        O.ref_rdf(pos, box, 3.6, 40)  # rMax > L/2
    with pytest.raises(ValueError):
        O.rdf(pos, box, 3.6, 40)


def test_msd_vacf_restatement_matches_reference():
    need_ref()
    box = np.array([5.0, 5.0, 6.0])
    pos, vel = random_walk(64, 30, box, 0.8, 12)
    m = O.msd(pos, box, 10)
    m_ref, _ = O.ref_msd(pos, box, 10, 0.01, 1, 10)
    assert np.array_equal(m, m_ref)
    u = O.vacf_unnormalised(vel, 10)
    c_ref, _ = O.ref_vacf(vel, box, 10, 0.01)
    assert np.array_equal(u / u[0], c_ref)
    assert m[0] == 0.0 and np.all(m[1:] > 0)
