"""The reference's recorded argon experiment 03 (experiments/exp03_argon_rdf.sh,
results/exp03_*.csv) rerun on the GPU path through the public API, following
moldyn_run's protocol (apps/moldyn_run.cpp:630-735): fcc(6) (864 atoms),
truncated LJ rc 2.5, skin 0.3, dt 0.005, 5000 Langevin BAOAB steps (friction 1),
the centre-of-mass momentum re-zeroed, then 20000 NVE steps with g(r) (200 bins
to 0.98 L/2) accumulated after every step.

The Langevin noise here is Philox, not the reference's Rng, so the trajectory
differs and the comparison is statistical: the first peak sits in the recorded
bin (or a neighbour) with the recorded height to 0.05, and the whole g(r) agrees
with the recorded curve to 0.03 RMS."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

EXP = load_golden("exp03_ref.npz")


@pytest.mark.parametrize("row,label", [(0, "rahman"), (1, "verlet")])
def test_exp03_argon_rdf(md, row, label):
    rho, temp, seed, peak_r, peak_g = EXP["summary"][row]
    ref = EXP["rdf_" + label]
    st = md.fcc_lattice(6, rho, temp, int(seed))
    box = st["box"]
    s = md.System.from_arrays(st["pos"], box, vel=st["vel"], mass=st["mass"])
    lj = md.LennardJones(1.0, 1.0, 2.5)
    v = md.VerletList(box, 2.5, 0.3)
    v.build(s)
    lj.compute_forces(s, v)
    md.LangevinBAOAB(0.005, 1.0, temp, int(seed)).run(s, v, lj, 5000)
    s.remove_center_of_mass_motion()
    rdf = md.Rdf(0.98 * 0.5 * box.min(), 200)
    vv = md.VelocityVerlet(0.005)
    for _ in range(20000):
        vv.run(s, v, lj, 1)
        rdf.accumulate(s)
    r, g = rdf.bin_centres(), rdf.g()
    assert rdf.frames() == 20000
    assert np.allclose(r, ref[:, 0], rtol=1e-9)
    window = (r >= 0.85) & (r <= 1.40)  # the script's peak search window
    k = np.flatnonzero(window)[np.argmax(g[window])]
    k_ref = int(np.argmin(np.abs(ref[:, 0] - peak_r)))
    assert abs(k - k_ref) <= 1
    assert abs(g[k] - peak_g) < 0.05
    assert np.sqrt(np.mean((g - ref[:, 1]) ** 2)) < 0.03


EXP4 = load_golden("exp04_ref.npz")["replicas"]


@pytest.mark.parametrize("state", [0, 1])
def test_exp04_argon_diffusion(md, state):
    """experiments/exp04_argon_diffusion.sh: per state point 8 replicas of fcc(6),
    5000 Langevin steps, the centre-of-mass momentum re-zeroed, 2000 NVE steps
    with MSD and VACF pushed after every step (maxLag 1000); D from the MSD fit
    over lags [250, 751) and from the VACF integral (apps/moldyn_run.cpp:744-766).
    The replica means agree with the reference's recorded means within their
    combined standard errors (x3), the two estimators agree (the experiment's
    tolerance, x2), and at the Rahman point D_msd is within 10% of experiment
    (D* = 0.0452)."""
    ref = EXP4[EXP4[:, 0] == state]
    d_msd, d_vacf = [], []
    for _, rho, temp, seed, _, _ in ref:
        st = md.fcc_lattice(6, rho, temp, int(seed))
        box = st["box"]
        s = md.System.from_arrays(st["pos"], box, vel=st["vel"], mass=st["mass"])
        lj = md.LennardJones(1.0, 1.0, 2.5)
        v = md.VerletList(box, 2.5, 0.3)
        v.build(s)
        lj.compute_forces(s, v)
        md.LangevinBAOAB(0.005, 1.0, temp, int(seed)).run(s, v, lj, 5000)
        s.remove_center_of_mass_motion()
        msd, vacf = md.Msd(s.n, 1000), md.Vacf(s.n, 1000)
        vv = md.VelocityVerlet(0.005)
        for _ in range(2000):
            vv.run(s, v, lj, 1)
            msd.push(s)
            vacf.push(s)
        d_msd.append(msd.diffusion_coefficient(0.005, 250, 751))
        d_vacf.append(vacf.diffusion_coefficient(0.005))

    def mean_se(x):
        x = np.asarray(x)
        return x.mean(), x.std(ddof=1) / np.sqrt(len(x))

    for ours, theirs in ((d_msd, ref[:, 4]), (d_vacf, ref[:, 5])):
        (m1, s1), (m2, s2) = mean_se(ours), mean_se(theirs)
        assert abs(m1 - m2) <= 3.0 * np.hypot(s1, s2)
    (mm, sm), (mv, sv) = mean_se(d_msd), mean_se(d_vacf)
    assert abs(mm - mv) <= 2.0 * (sm + sv)
    if state == 0:
        assert abs(mm - 0.0452) <= 0.10 * 0.0452


EXP5 = load_golden("exp05_ref.npz")["rows"]


@pytest.mark.parametrize("row", range(5))
def test_exp05_lj_equation_of_state(md, row):
    """experiments/exp05_lj_eos.sh: fcc(5) (500 atoms), truncated LJ rc 3.0 with
    tail corrections, skin 0.3, dt 0.005, 10000 Langevin steps then 20000
    Nose-Hoover steps (tau 0.5, chain 3, dof 3N - 3) at NIST's temperature for the
    density.  Production means U* = <PE + U_LRC>/N, p* = <rho T + W/(3V) + P_LRC>,
    T* = <2 KE/(3N - 3)> meet the experiment's own tolerances against NIST
    (|dU| <= 0.1, |dp| <= 0.3, |dT| <= 0.02) and agree with the reference's
    recorded means.  The sixth row (rho* = 0.900) is left out: the reference
    records it as a failure (the liquid crystallises at that state point)."""
    rho, seed, t_ref, u_ref, p_ref, t_nist, u_nist, p_nist = EXP5[row]
    st = md.fcc_lattice(5, rho, t_nist, int(seed))
    box = st["box"]
    s = md.System.from_arrays(st["pos"], box, vel=st["vel"], mass=st["mass"])
    lj = md.LennardJones(1.0, 1.0, 3.0)
    v = md.VerletList(box, 3.0, 0.3)
    v.build(s)
    lj.compute_forces(s, v)
    md.LangevinBAOAB(0.005, 1.0, t_nist, int(seed)).run(s, v, lj, 10000)
    s.remove_center_of_mass_motion()
    n = s.n
    th = md.NoseHooverChain(0.005, t_nist, 0.5, 3, 3 * n - 3).run(s, v, lj, 20000, thermo=True)
    vol = float(np.prod(box))
    temp = 2.0 * th[:, 2] / (3 * n - 3)
    u = np.mean(th[:, 0] + lj.long_range_correction(s)) / n
    p = np.mean(n / vol * temp + th[:, 1] / (3.0 * vol) + lj.long_range_correction_pressure(s))
    t = np.mean(temp)
    assert abs(u - u_nist) <= 0.1 and abs(p - p_nist) <= 0.3 and abs(t - t_nist) <= 0.02
    assert abs(u - u_ref) <= 0.03 and abs(p - p_ref) <= 0.15 and abs(t - t_ref) <= 0.01
