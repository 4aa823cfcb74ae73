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
