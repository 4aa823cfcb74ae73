"""Trajectory frames and checkpoints of device systems.

XYZ frames (apps/moldyn_run.cpp:519-533) carry the positions in original atom
order at the default stream precision.  A checkpoint holds a system and its
integrator: a run continued from the loaded state (after a fresh Verlet build)
equals the saved run continued (after one) bit for bit, for velocity Verlet,
the Nose-Hoover chain and Langevin BAOAB (whose noise stream position is part
of the state).  Damaged files and integrators of another kind are rejected.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def liquid(md, cells=6, seed=2):
    st = md.fcc_lattice(cells, 0.8442, 0.722, seed)
    s = md.System.from_arrays(st["pos"], st["box"], vel=st["vel"], mass=st["mass"])
    lj = md.LennardJones(1.0, 1.0, 2.5)
    v = md.VerletList(st["box"], 2.5, 0.3)
    v.build(s)
    lj.compute_forces(s, v)
    return s, v, lj, st["box"]


def test_xyz_frames(md, tmp_path):
    s, v, lj, box = liquid(md)
    path = tmp_path / "traj.xyz"
    md.VelocityVerlet(0.005).run(s, v, lj, 30)
    md.xyz_append(path, s, 30, 0.15, "production", command_line="run", revision="r1", host="h")
    md.xyz_append(path, s, 31, 0.155, "production")
    lines = path.read_text().splitlines()
    n = s.n
    assert lines[0] == str(n) and lines[n + 2] == str(n)
    assert lines[1] == 'step=30 time=0.15 phase=production git_sha=r1 host="h" command="run"'
    pos = s.positions
    want = ["Ar %s %s %s" % tuple("%g" % c for c in p) for p in pos]
    assert lines[2:n + 2] == want
    assert len(lines) == 2 * (n + 2)


def make_integrator(md, kind, n):
    if kind == "vv":
        return md.VelocityVerlet(0.005)
    if kind == "nhc":
        return md.NoseHooverChain(0.005, 0.9, 0.5, 3, 3 * n - 3)
    return md.LangevinBAOAB(0.005, 1.0, 0.9, 17)


@pytest.mark.parametrize("kind", ["vv", "nhc", "baoab"])
def test_checkpoint_continues_bit_for_bit(md, tmp_path, kind):
    s, v, lj, box = liquid(md)
    integ = make_integrator(md, kind, s.n)
    integ.run(s, v, lj, 60)
    v.build(s)  # both continuations start from a list built from this state
    lj.compute_forces(s, v)
    path = tmp_path / "state.ckpt"
    md.checkpoint_save(s, path, integ)
    integ.run(s, v, lj, 80)
    a = (s.positions, s.velocities)
    integ2 = make_integrator(md, kind, s.n)
    s2 = md.checkpoint_load(path, integ2)
    assert s2.n == s.n and np.array_equal(s2.box, box)
    v2 = md.VerletList(box, 2.5, 0.3)
    v2.build(s2)
    lj.compute_forces(s2, v2)
    integ2.run(s2, v2, lj, 80)
    assert np.array_equal(s2.positions, a[0]) and np.array_equal(s2.velocities, a[1])


def test_checkpoint_rejects_damage_and_other_kinds(md, tmp_path):
    s, v, lj, box = liquid(md, cells=4)
    integ = md.NoseHooverChain(0.005, 0.9, 0.5, 3, 3 * s.n - 3)
    path = tmp_path / "state.ckpt"
    md.checkpoint_save(s, path, integ)
    with pytest.raises(md.InvalidArgument, match="another kind"):
        md.checkpoint_load(path, md.VelocityVerlet(0.005))
    s2 = md.checkpoint_load(path)  # the system alone
    assert np.array_equal(s2.positions, s.positions) and np.array_equal(s2.forces, s.forces)
    raw = bytearray(path.read_bytes())
    raw[200] ^= 0x40
    bad = tmp_path / "bad.ckpt"
    bad.write_bytes(bytes(raw))
    with pytest.raises(md.InvalidArgument, match="damaged"):
        md.checkpoint_load(bad)
    (tmp_path / "other").write_bytes(b"not a checkpoint at all, really")
    with pytest.raises(md.InvalidArgument, match="not a checkpoint"):
        md.checkpoint_load(tmp_path / "other")
