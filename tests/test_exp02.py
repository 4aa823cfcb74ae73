"""The reference's recorded experiment 02 (experiments/exp02_energy_conservation.sh,
results/exp02_*.csv): moldyn_run NVE velocity Verlet on fcc(3), rho*=0.80,
T*=1.0, seed 12345, rc 2.5, skin 0.4, linear-force-shift, to t = 1 at four
time steps.  The oracle's restatement reproduces every recorded thermo row to
the CSV's 10 significant digits, and the summary's dt^2 slope.  No GPU."""
import numpy as np
import pytest

import oracle as O
from conftest import load_golden

EXP = load_golden("exp02_ref.npz")
DTS = ("0.001", "0.002", "0.004", "0.008")


def thermo_rows(pe, ke, w, n, vol):
    """PE, KE, E, T (3N - 3 dof under NVE), P = rho T + W / (3V) (no tail for
    LFS), as StepSampler::record forms them (apps/moldyn_run.cpp:497-511)."""
    t = 2.0 * ke / (3 * n - 3)
    return np.stack([pe, ke, pe + ke, t, n / vol * t + w / (3.0 * vol)], axis=1)


def rel(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


@pytest.mark.parametrize("dt", DTS)
def test_oracle_reproduces_the_recorded_thermo(dt):
    ref = EXP["thermo_" + dt]
    steps = len(ref) - 1
    st = O.fcc_lattice(3, 0.80, 1.0, 12345)
    n = len(st["mass"])
    sim = O.Sim(st["pos"], st["vel"], st["mass"], st["box"], rc=2.5, trunc=1, skin=0.4,
                dt=float(dt))
    sim.prime()
    out = []
    for k in range(steps + 1):
        if k:
            sim.run("vv", 1)
        _, v, _ = sim.state()
        out.append((sim.energy, 0.5 * np.sum(st["mass"][:, None] * v * v), sim.virial))
    out = np.array(out)
    got = thermo_rows(out[:, 0], out[:, 1], out[:, 2], n, float(np.prod(st["box"])))
    assert np.array_equal(ref[:, 1], np.round(np.arange(steps + 1) * float(dt), 12))
    assert np.max(rel(got, ref[:, 2:])) < 1e-9  # 10 significant digits in the CSV


def test_recorded_summary_is_a_dt_squared_law():
    """exp02's own assertion: the log-log slope of the relative energy error
    against dt lies in [1.85, 2.15]."""
    s = EXP["summary"]
    slope = np.polyfit(np.log(s[:, 0]), np.log(s[:, 3]), 1)[0]
    assert 1.85 <= slope <= 2.15
    for (dt, e0, drift, relerr) in s:
        ref = EXP["thermo_%g" % dt]
        assert e0 == pytest.approx(ref[0, 4], rel=1e-9)
        assert drift == pytest.approx(np.max(np.abs(ref[:, 4] - ref[0, 4])), rel=1e-4)
