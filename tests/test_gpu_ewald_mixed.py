"""FP32 real-space pair terms for Ewald / SPC/E (MD_PRECISION_MIXED) against
the FP64 path, which follows the reference (forcefield/ewald.cpp:60-68,
lennard_jones.cpp:62-77).  Displacements, the cutoff test and every sum stay
FP64; erfc, exp and the LJ powers carry FP32's ~1e-7 relative error, so the
energies agree to 1e-6 and the net forces (sums of ~400 pair forces that
largely cancel) to 1e-5 RMS relative."""
import numpy as np
import pytest

import oracle as O
from conftest import load_golden

pytestmark = pytest.mark.gpu

SPCE = load_golden("nist_spce.npz")


def water(md, c):
    types = ["O" if o else "H" for o in SPCE[f"isO{c}"]]
    return md.build_spce_system(SPCE[f"pos{c}"], types, SPCE[f"box{c}"])


@pytest.mark.parametrize("c", [1, 2, 3, 4])
def test_mixed_real_space_tracks_fp64(md, c):
    s = water(md, c)
    ff = md.SpceForceField()
    e64 = ff.compute_forces(s)
    p64 = dict(ff.parts)
    f64 = s.forces
    ff.set_precision(md.PRECISION_MIXED)
    e32 = ff.compute_forces(s)
    p32 = dict(ff.parts)
    f32 = s.forces
    assert abs(p32["real"] - p64["real"]) <= 1e-6 * abs(p64["real"])
    assert abs(p32["disp"] - p64["disp"]) <= 1e-6 * abs(p64["disp"])
    assert abs(e32 - e64) <= 1e-6 * abs(e64)
    assert p32["reciprocal"] == p64["reciprocal"] and p32["intra"] == p64["intra"]
    assert abs(p32["virial"] - p64["virial"]) <= 1e-6 * abs(p64["virial"])
    rel = np.sqrt(np.mean((f32 - f64) ** 2) / np.mean(f64 ** 2))
    assert rel < 1e-5
    ff.set_precision(md.PRECISION_FP64)
    assert ff.compute_forces(s) == e64 and np.array_equal(s.forces, f64)
    with pytest.raises(md.InvalidArgument):
        ff.set_precision(7)


def test_mixed_real_space_conserves_energy(md):
    drift = {}
    for prec in (md.PRECISION_FP64, md.PRECISION_MIXED):
        s = water(md, 1)
        s.velocities = np.sqrt(300.0 / s.masses)[:, None] * O.rng_normals(9, 3 * s.n).reshape(-1, 3)
        rw = md.RigidWater(1.0, 109.47)
        rw.constrain_velocities(s)
        ff = md.SpceForceField()
        ff.set_precision(prec)
        integ = md.ConstrainedVelocityVerlet(md.units.femtoseconds(1.0), rw)
        th = integ.run(s, ff, 300, thermo=True)
        h = th[:, 0] + th[:, 2]
        drift[prec] = np.max(np.abs(h - h[0])) / np.mean(np.abs(th[:, 2]))
    assert drift[md.PRECISION_MIXED] < 3 * drift[md.PRECISION_FP64] + 1e-4
