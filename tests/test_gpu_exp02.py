"""The GPU path against the reference's recorded experiment 02
(results/exp02_*.csv): the fused FP64 velocity-Verlet loop (md_run_lj with
device-decided Verlet rebuilds) on fcc(3), rho*=0.80, T*=1.0, seed 12345,
rc 2.5, skin 0.4, linear-force-shift, to t = 1 at dt = 0.001 ... 0.008.  Every
thermo row equals the reference's to the CSV's 10 significant digits, and the
relative energy errors reproduce the recorded dt^2 law."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

EXP = load_golden("exp02_ref.npz")
DTS = ("0.001", "0.002", "0.004", "0.008")


def run(md, dt, steps):
    st = md.fcc_lattice(3, 0.80, 1.0, 12345)
    s = md.System.from_arrays(st["pos"], st["box"], vel=st["vel"], mass=st["mass"])
    lj = md.LennardJones(1.0, 1.0, 2.5, md.Truncation.LinearForceShift)
    v = md.VerletList(st["box"], 2.5, 0.4)
    v.build(s)
    e0, w0 = lj.compute_forces(s, v)
    ke0 = s.kinetic_energy()
    th = md.VelocityVerlet(float(dt)).run(s, v, lj, steps, thermo=True)
    pe = np.concatenate([[e0], th[:, 0]])
    w = np.concatenate([[w0], th[:, 1]])
    ke = np.concatenate([[ke0], th[:, 2]])
    n, vol = s.n, float(np.prod(st["box"]))
    t = 2.0 * ke / (3 * n - 3)
    return np.stack([pe, ke, pe + ke, t, n / vol * t + w / (3.0 * vol)], axis=1)


@pytest.mark.parametrize("dt", DTS)
def test_gpu_reproduces_the_recorded_thermo(md, dt):
    ref = EXP["thermo_" + dt]
    got = run(md, dt, len(ref) - 1)
    err = np.abs(got - ref[:, 2:]) / np.abs(ref[:, 2:])
    assert np.max(err) < 1e-9


def test_gpu_energy_error_follows_the_recorded_summary(md):
    rel = []
    for (dt, e0, drift, relerr) in EXP["summary"]:
        got = run(md, "%g" % dt, int(round(1.0 / dt)))
        e = got[:, 2]
        rel.append(np.max(np.abs(e - e[0])) / abs(e[0]))
        assert e[0] == pytest.approx(e0, rel=1e-9)
        assert rel[-1] == pytest.approx(relerr, rel=1e-4)
    slope = np.polyfit(np.log(EXP["summary"][:, 0]), np.log(rel), 1)[0]
    assert 1.85 <= slope <= 2.15
