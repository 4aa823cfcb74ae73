"""The hand-written adjoint of the FP64 velocity-Verlet LJ trajectory: the
Hessian-vector product against finite differences of the forces, and trajectory
gradients against central finite differences (h = 1e-6 relative) of the same GPU
code and of the oracle's CPU forward (the reference's arithmetic)."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

DT, STEPS, EVERY, SKIN = 0.005, 60, 20, 1.0


def liquid(md, cells=4, rho=0.8442, temp=0.722, seed=9):
    st = md.fcc_lattice(cells, rho, temp, seed)
    rng = np.random.default_rng(seed)
    pos = st["pos"] + rng.normal(scale=0.05, size=st["pos"].shape)
    box = st["box"]
    pos -= box * np.floor(pos / box + 0.5)
    return pos, st["vel"], st["mass"], box


def rel(a, b):
    return abs(a - b) / max(abs(a), abs(b), 1e-300)


@pytest.mark.parametrize("trunc", [0, 1])
def test_hvp_matches_force_differences(md, trunc):
    pos, vel, mass, box = liquid(md)
    s = md.System.from_arrays(pos, box)
    lj = md.LennardJones(1.0, 1.0, 2.5, trunc)
    v = md.VerletList(box, 2.5, 0.3)
    v.build(s)
    u = np.random.default_rng(1).normal(size=pos.shape)
    hvp, dth = lj.hessian_vector_product(s, v, u)
    h = 1e-6

    def forces(p, sigma=1.0, eps=1.0):
        t = md.System.from_arrays(p, box)
        md.LennardJones(sigma, eps, 2.5, trunc).compute_forces(t)
        return t.forces

    fd = (forces(pos + h * u) - forces(pos - h * u)) / (2 * h)
    assert np.max(np.abs(hvp - fd)) < 1e-6 * np.max(np.abs(fd))
    f_de = (forces(pos, eps=1 + h) - forces(pos, eps=1 - h)) / (2 * h)
    f_ds = (forces(pos, sigma=1 + h) - forces(pos, sigma=1 - h)) / (2 * h)
    assert rel(dth[0], np.sum(u * f_de)) < 1e-6
    assert rel(dth[1], np.sum(u * f_ds)) < 1e-6


def loss_of(rows, n, vol):
    dof = 3 * n - 3
    p = n / vol * 2 * rows[:, 2] / dof + rows[:, 1] / (3 * vol)
    u = rows[:, 0] / n
    return (p.mean() - 1.0) ** 2 + (u.mean() + 5.0) ** 2, p.mean(), u.mean()


def loss_grad_rows(rows, n, vol):
    dof = 3 * n - 3
    _, pm, um = loss_of(rows, n, vol)
    g = np.zeros_like(rows)
    k = rows.shape[0]
    g[:, 0] = 2 * (um + 5.0) / (n * k)
    g[:, 1] = 2 * (pm - 1.0) / (3 * vol * k)
    g[:, 2] = 2 * (pm - 1.0) * (n / vol) * 2 / (dof * k)
    return g


def gpu_loss(md, pos, vel, mass, box, sigma=1.0, eps=1.0, trunc=1):
    s = md.System.from_arrays(pos, box, vel=vel, mass=mass)
    traj = md.AdjointTrajectory()
    rows = traj.forward(s, md.LennardJones(sigma, eps, 2.5, trunc), DT, STEPS, EVERY, SKIN)
    return loss_of(rows, s.n, s.volume())[0], rows, traj, s


def test_adjoint_gradients_match_finite_differences(md):
    """d loss / d(epsilon, sigma, x0, v0) of a 60-step trajectory (force-shifted LJ,
    continuous, so the differences see no cutoff jumps) against central
    differences of the same code."""
    pos, vel, mass, box = liquid(md)
    n, vol = pos.shape[0], float(np.prod(box))
    loss, rows, traj, s = gpu_loss(md, pos, vel, mass, box)
    d_eps, d_sig, gx, gv = traj.backward(loss_grad_rows(rows, n, vol))
    h = 1e-6
    fd_eps = (gpu_loss(md, pos, vel, mass, box, eps=1 + h)[0] -
              gpu_loss(md, pos, vel, mass, box, eps=1 - h)[0]) / (2 * h)
    fd_sig = (gpu_loss(md, pos, vel, mass, box, sigma=1 + h)[0] -
              gpu_loss(md, pos, vel, mass, box, sigma=1 - h)[0]) / (2 * h)
    assert rel(d_eps, fd_eps) < 1e-6, (d_eps, fd_eps)
    assert rel(d_sig, fd_sig) < 1e-6, (d_sig, fd_sig)
    rng = np.random.default_rng(4)
    for a, c in zip(rng.integers(0, n, 3), rng.integers(0, 3, 3)):
        for arr, grad in ((pos, gx), (vel, gv)):
            p, m = arr.copy(), arr.copy()
            p[a, c] += h
            m[a, c] -= h
            args_p = (p, vel) if arr is pos else (pos, p)
            args_m = (m, vel) if arr is pos else (pos, m)
            fd = (gpu_loss(md, *args_p, mass, box)[0] - gpu_loss(md, *args_m, mass, box)[0]) / (2 * h)
            assert abs(grad[a, c] - fd) < 1e-6 * max(abs(fd), np.max(np.abs(grad)) * 1e-2), \
                (a, c, grad[a, c], fd)


def oracle_loss(pos, vel, mass, box, sigma=1.0, eps=1.0):
    sim = O.Sim(pos, vel, mass, box, sigma=sigma, eps=eps, rc=2.5, trunc=1, skin=0.3, dt=DT)
    sim.prime()
    rows = np.zeros((STEPS, 3))
    for k in range(STEPS):
        sim.run("vv", 1)
        _, v, _ = sim.state()
        rows[k] = (sim.energy, sim.virial, 0.5 * np.sum(mass[:, None] * v * v))
    return loss_of(rows, pos.shape[0], float(np.prod(box)))[0]


def test_adjoint_matches_reference_forward_differences(md):
    """The reference gradient assembled from the CPU forward (the oracle's
    restatement of VelocityVerlet + LennardJones(sigma +- h, epsilon +- h))."""
    pos, vel, mass, box = liquid(md, seed=17)
    n, vol = pos.shape[0], float(np.prod(box))
    loss, rows, traj, _ = gpu_loss(md, pos, vel, mass, box)
    assert abs(loss - oracle_loss(pos, vel, mass, box)) < 1e-9 * abs(loss)
    d_eps, d_sig, _, _ = traj.backward(loss_grad_rows(rows, n, vol))
    h = 1e-6
    fd_eps = (oracle_loss(pos, vel, mass, box, eps=1 + h) -
              oracle_loss(pos, vel, mass, box, eps=1 - h)) / (2 * h)
    fd_sig = (oracle_loss(pos, vel, mass, box, sigma=1 + h) -
              oracle_loss(pos, vel, mass, box, sigma=1 - h)) / (2 * h)
    assert rel(d_eps, fd_eps) < 1e-6, (d_eps, fd_eps)
    assert rel(d_sig, fd_sig) < 1e-6, (d_sig, fd_sig)


def test_backward_leaves_forward_state_and_checks_skin(md):
    pos, vel, mass, box = liquid(md)
    s = md.System.from_arrays(pos, box, vel=vel, mass=mass)
    traj = md.AdjointTrajectory()
    rows = traj.forward(s, md.LennardJones(1.0, 1.0, 2.5, 1), DT, STEPS, EVERY, SKIN)
    end_pos, end_vel = s.positions, s.velocities
    traj.backward(np.ones_like(rows))
    assert np.array_equal(s.positions, end_pos) and np.array_equal(s.velocities, end_vel)
    s2 = md.System.from_arrays(pos, box, vel=vel * 3.0, mass=mass)
    with pytest.raises(md.MDError, match="larger skin"):
        md.AdjointTrajectory().forward(s2, md.LennardJones(1.0, 1.0, 2.5, 1), DT, 60, 60, 0.05)


def test_adjoint_long_trajectory_matches_differences(md):
    """A 400-step trajectory of the 32,000-atom lattice (fcc 20^3, force-shifted LJ,
    list skin 2.0, states saved every 50 steps): the adjoint d loss / d(epsilon,
    sigma) against central differences at h = 1e-7.  Longer trajectories diverge
    (the differences themselves stop converging near 1000 steps).  The forward's
    system is not kept by the caller: backward() must still replay on it."""
    import gc
    st = md.fcc_lattice(20, 0.8442, 0.722, 2026)
    pos, vel, mass, box = st["pos"], st["vel"], st["mass"], st["box"]
    n, vol = pos.shape[0], float(np.prod(box))
    steps, every, skin, h = 400, 50, 2.0, 1e-7

    def run(sigma=1.0, eps=1.0):
        traj = md.AdjointTrajectory()
        rows = traj.forward(md.System.from_arrays(pos, box, vel=vel, mass=mass),
                            md.LennardJones(sigma, eps, 2.5, 1), DT, steps, every, skin)
        return rows, traj

    rows, traj = run()
    gc.collect()
    d_eps, d_sig, _, _ = traj.backward(loss_grad_rows(rows, n, vol))
    fd_eps = (loss_of(run(eps=1 + h)[0], n, vol)[0] - loss_of(run(eps=1 - h)[0], n, vol)[0]) / (2 * h)
    fd_sig = (loss_of(run(sigma=1 + h)[0], n, vol)[0] -
              loss_of(run(sigma=1 - h)[0], n, vol)[0]) / (2 * h)
    assert rel(d_eps, fd_eps) < 1e-6, (d_eps, fd_eps)
    assert rel(d_sig, fd_sig) < 1e-6, (d_sig, fd_sig)
