"""The launch-shape autotuner: every shape gives the same forces (to the
summation-order rounding), the winner is applied and cached on disk, and a
second call reads it back without timing."""
import numpy as np
import pytest

import moleculardynamics_b200.autotune as T

pytestmark = pytest.mark.gpu


def test_tune_force_kernel_applies_and_caches(md, tmp_path, monkeypatch):
    monkeypatch.setenv("MOLDYN_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    st = md.fcc_lattice(8, 0.8442, 0.722, 3)
    pos = st["pos"] + np.random.default_rng(3).normal(scale=0.1, size=st["pos"].shape)
    pos -= st["box"] * np.floor(pos / st["box"] + 0.5)
    s = md.System.from_arrays(pos, st["box"], vel=st["vel"])
    v = md.VerletList(st["box"], 2.5, 0.3)
    v.build(s)
    ref_lj = md.LennardJones(1.0, 1.0, 2.5)
    e0, w0 = ref_lj.compute_forces(s, v)
    f0 = s.forces
    for tpa, u in T.SHAPES:
        ref_lj.set_launch(tpa, u)
        e, w = ref_lj.compute_forces(s, v)
        assert abs(e - e0) < 1e-12 * abs(e0) and abs(w - w0) < 1e-12 * abs(w0)
        assert np.max(np.abs(s.forces - f0)) < 1e-12 * np.max(np.abs(f0))
    lj = md.LennardJones(1.0, 1.0, 2.5)
    best, timings = T.tune_force_kernel(s, lj, v, 0.3, repeats=2)
    assert best in T.SHAPES and len(timings) == len(T.SHAPES)
    assert timings[best] == min(timings.values())
    again, t2 = T.tune_force_kernel(s, md.LennardJones(1.0, 1.0, 2.5), v, 0.3)
    assert again == best and t2 == {}
    with pytest.raises(md.InvalidArgument):
        lj.set_launch(3, 1)
