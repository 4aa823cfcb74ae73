"""GPU parity of the integrators: velocity-Verlet, BAOAB and the Nose-Hoover chain
(the reference's tests/test_integrator.cpp and test_thermostat.cpp), plus
step-level shadow parity against the oracle.
"""
import numpy as np
import pytest

import oracle as O
from conftest import load_golden

pytestmark = pytest.mark.gpu

FCC = load_golden("fcc_lj.npz")


def approx_eq(a, b, eps):
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    return np.all(np.abs(a - b) < eps * (1.0 + np.maximum(np.abs(a), np.abs(b))))


def lattice_system(md, cells, rho, temp, seed):
    st = md.fcc_lattice(cells, rho, temp, seed)
    s = md.System.from_arrays(st["pos"], st["box"], vel=st["vel"], mass=st["mass"])
    return s, st


def test_vv_one_step_bit_exact_from_same_forces(md):
    """One VV step from identical state and forces reproduces the oracle's
    positions exactly (fma kick, fma drift, bit-exact wrap)."""
    s, st = lattice_system(md, 6, 0.8442, 0.722, 1)
    lj = md.LennardJones(1.0, 1.0, 2.5)
    lj.compute_forces(s)
    f0 = s.forces
    integ = md.VelocityVerlet(0.005)
    pre = {}

    def forces(sys_):
        pre["pos"] = sys_.positions
        pre["vel"] = sys_.velocities
        return lj.compute_forces(sys_)[0]

    integ.step(s, forces)
    # oracle: same kick and drift from the same (pos, vel, f0)
    n = len(st["mass"])
    vx, vy, vz = (np.ascontiguousarray(st["vel"][:, k]) for k in range(3))
    fx, fy, fz = (np.ascontiguousarray(f0[:, k]) for k in range(3))
    x, y, z = (np.ascontiguousarray(st["pos"][:, k]) for k in range(3))
    L = O.lib()
    L.orc_half_kick(n, 0.005, O._p(st["mass"]), O._p(fx), O._p(fy), O._p(fz), O._p(vx), O._p(vy),
                    O._p(vz))
    L.orc_drift_wrap(n, O._p(st["box"]), 0.005, O._p(vx), O._p(vy), O._p(vz), O._p(x), O._p(y),
                     O._p(z))
    assert np.array_equal(pre["pos"], np.stack([x, y, z], 1))
    assert np.array_equal(pre["vel"], np.stack([vx, vy, vz], 1))


def test_vv_trajectory_shadow_parity(md):
    """25 steps of the N=864 drop-in configuration (moldyn_run ForceFn): each
    step's forces/energy/virial match the oracle evaluated on the GPU's state."""
    s, st = lattice_system(md, 6, 0.8442, 0.722, 1)
    lj = md.LennardJones(1.0, 1.0, 2.5)
    v = md.VerletList(st["box"], 2.5, 0.3)
    v.build(s)
    lj.compute_forces(s, v)
    integ = md.VelocityVerlet(0.005)

    def forces(sys_):
        v.rebuild_if_needed(sys_)
        return lj.compute_forces(sys_, v)[0]

    for _ in range(25):
        integ.step(s, forces)
        pos = s.positions
        fo, eo, wo = O.lj_compute(pos, st["box"], rc=2.5, trunc=0)
        e, w = s.last_energy_virial()
        assert approx_eq(e, eo, 1e-12) and approx_eq(w, wo, 1e-12)
        assert approx_eq(s.forces, fo, 1e-12)
    # and the trajectory stays on the reference's to round-off after 25 steps
    assert np.max(np.abs(s.positions - FCC["vv25_pos"])) < 1e-9
    assert np.max(np.abs(s.velocities - FCC["vv25_vel"])) < 1e-9
    assert v.rebuild_count() == int(FCC["vv25_info"][2])


def test_fused_run_equals_host_loop(md):
    """md_run_lj (device-decided rebuilds, no per-step sync) == host-driven steps."""
    outs = []
    for fused in (False, True):
        s, st = lattice_system(md, 5, 0.8442, 0.722, 3)
        lj = md.LennardJones(1.0, 1.0, 2.5)
        v = md.VerletList(st["box"], 2.5, 0.3)
        v.build(s)
        lj.compute_forces(s, v)
        integ = md.VelocityVerlet(0.005)
        if fused:
            th = integ.run(s, v, lj, 60, thermo=True)
            assert th.shape == (60, 4)
        else:
            def forces(sys_):
                v.rebuild_if_needed(sys_)
                return lj.compute_forces(sys_, v)[0]
            for _ in range(60):
                integ.step(s, forces)
        outs.append((s.positions, s.velocities, v.rebuild_count()))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])
    assert outs[0][2] == outs[1][2]


@pytest.mark.parametrize("kind", ["vv", "nhc"])
def test_step_graph_replay_equals_host_launches(md, kind):
    """md_run_lj replaying the captured step graph (conditional rebuild node) and
    launching every kernel from the host give bit-identical trajectories, thermo
    rows and rebuild counts; 300 steps of a hot liquid rebuild many times."""
    outs = []
    ctx = md.default_context()
    for graphs in (False, True):
        ctx.set_graphs(graphs)
        try:
            s, st = lattice_system(md, 5, 0.8442, 1.5, 7)
            lj = md.LennardJones(1.0, 1.0, 2.5)
            v = md.VerletList(st["box"], 2.5, 0.3)
            v.build(s)
            lj.compute_forces(s, v)
            integ = (md.VelocityVerlet(0.005) if kind == "vv"
                     else md.NoseHooverChain(0.005, 1.0, 0.5, 3, 3 * s.n - 3))
            th = integ.run(s, v, lj, 300, thermo=True)
            outs.append((s.positions, s.velocities, th, v.rebuild_count()))
        finally:
            ctx.set_graphs(True)
    assert outs[0][3] == outs[1][3] and outs[0][3] > 5
    for a, b in zip(outs[0][:3], outs[1][:3]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("kind,cells,precision", [("vv", 5, "fp64"), ("nhc", 5, "fp64"),
                                                 ("vv", 26, "mixed")])
def test_step_graph_cached_across_calls(md, kind, cells, precision):
    """Calls of md_run_lj on the same handles replay the step graph the first call
    captured (one capture in all), and give the same trajectory, thermo rows and
    rebuilds as the same calls with every kernel launched from the host.  A
    velocity-Verlet run split into calls also equals one call of the same length.
    fcc 26^3 (70,304 atoms) in mixed precision runs on halo tiles."""
    ctx = md.default_context()
    lengths = [1, 5, 20, 74, 200]
    prec = md.PRECISION_MIXED if precision == "mixed" else md.PRECISION_FP64

    def run(split, graphs):
        ctx.set_graphs(graphs)
        try:
            s, st = lattice_system(md, cells, 0.8442, 1.5, 7)
            lj = md.LennardJones(1.0, 1.0, 2.5, precision=prec)
            v = md.VerletList(st["box"], 2.5, 0.3)
            v.build(s)
            lj.compute_forces(s, v)
            integ = (md.VelocityVerlet(0.005) if kind == "vv"
                     else md.NoseHooverChain(0.005, 1.0, 0.5, 3, 3 * s.n - 3))
            c0 = ctx.graph_captures()
            rows = []
            for k in (lengths if split else [sum(lengths)]):
                rows.append(integ.run(s, v, lj, k, thermo=True))
            caps = ctx.graph_captures() - c0
            return s.positions, s.velocities, np.concatenate(rows), v.rebuild_count(), caps
        finally:
            ctx.set_graphs(True)

    host = run(True, False)
    cached = run(True, True)
    assert cached[4] == 1 and host[4] == 0
    assert host[3] == cached[3] and host[3] > 3
    for a, b in zip(host[:3], cached[:3]):
        assert np.array_equal(a, b)
    if kind == "vv":
        single = run(False, True)
        assert single[3] == cached[3]
        for a, b in zip(single[:3], cached[:3]):
            assert np.array_equal(a, b)


def test_nhc_fused_run_follows_host_steps(md):
    """The fused Nose-Hoover loop applies integrateChain(dt/2) exactly twice per
    step, as NoseHooverChain::step does (nose_hoover.hpp:37-42): it tracks the
    host-driven steps to round-off (it reuses the chain's tracked kinetic energy
    instead of re-summing it)."""
    outs = []
    for fused in (False, True):
        s, st = lattice_system(md, 4, 0.80, 1.2, 21)
        dof = 3 * s.n - 3
        lj = md.LennardJones(1.0, 1.0, 2.5, md.Truncation.LinearForceShift)
        v = md.VerletList(st["box"], 2.5, 0.3)
        v.build(s)
        lj.compute_forces(s, v)
        integ = md.NoseHooverChain(0.002, 1.0, 0.5, 3, dof)
        if fused:
            integ.run(s, v, lj, 100)
        else:
            def forces(sys_):
                v.rebuild_if_needed(sys_)
                return lj.compute_forces(sys_, v)[0]
            for _ in range(100):
                integ.step(s, forces)
        outs.append((s.positions, s.velocities, integ.conserved_quantity_contribution()))
    assert np.max(np.abs(outs[0][0] - outs[1][0])) < 1e-10
    assert np.max(np.abs(outs[0][1] - outs[1][1])) < 1e-10
    assert abs(outs[0][2] - outs[1][2]) < 1e-10 * (1 + abs(outs[0][2]))


def energy_error_slope(md, use_run):
    dts = [0.001, 0.002, 0.004, 0.008]
    log_dt, log_err = [], []
    for dt in dts:
        s, st = lattice_system(md, 3, 0.80, 1.0, 12345)
        lj = md.LennardJones(1.0, 1.0, 2.5, md.Truncation.LinearForceShift)
        integ = md.VelocityVerlet(dt)
        pe, _ = lj.compute_forces(s)
        e0 = pe + s.kinetic_energy()
        steps = int(round(1.0 / dt))
        max_dev = 0.0
        for _ in range(steps):
            integ.step(s, lambda q: lj.compute_forces(q)[0])
            pe, _ = lj.compute_forces(s)
            max_dev = max(max_dev, abs(pe + s.kinetic_energy() - e0))
        log_dt.append(np.log(dt))
        log_err.append(np.log(max_dev / abs(e0)))
    return np.polyfit(log_dt, log_err, 1)[0]


def test_vv_energy_error_scales_as_dt_squared(md):
    """tests/test_integrator.cpp:10-50"""
    slope = energy_error_slope(md, False)
    assert 1.85 < slope < 2.15, slope


def test_vv_time_reversible(md):
    """tests/test_integrator.cpp:52-83"""
    s, st = lattice_system(md, 3, 0.80, 1.0, 999)
    lj = md.LennardJones(1.0, 1.0, 2.5, md.Truncation.LinearForceShift)
    integ = md.VelocityVerlet(0.002)
    start = s.positions
    lj.compute_forces(s)
    for _ in range(200):
        integ.step(s, lambda q: lj.compute_forces(q)[0])
    s.velocities = -s.velocities
    for _ in range(200):
        integ.step(s, lambda q: lj.compute_forces(q)[0])
    d = s.positions - start
    L = st["box"]
    d -= L * np.floor(d / L + 0.5)
    assert np.max(np.linalg.norm(d, axis=1)) < 1e-8


def test_baoab_replayed_noise_matches_oracle(md):
    """BAOAB with the reference's own mt19937_64 normals replayed: the GPU
    trajectory tracks the oracle's to round-off."""
    cells, rho, temp = 3, 0.80, 1.0
    s, st = lattice_system(md, cells, rho, temp, 42)
    n = len(st["mass"])
    steps = 20
    xi = O.rng_normals(777, 3 * n * steps)
    lj = md.LennardJones(1.0, 1.0, 2.5, md.Truncation.LinearForceShift)
    v = md.VerletList(st["box"], 2.5, 0.3)
    v.build(s)
    lj.compute_forces(s, v)
    integ = md.LangevinBAOAB(0.005, 1.0, temp, 777)
    integ.set_noise(xi)

    def forces(sys_):
        v.rebuild_if_needed(sys_)
        return lj.compute_forces(sys_, v)[0]

    for _ in range(steps):
        integ.step(s, forces)
    sim = O.Sim(st["pos"], st["vel"], st["mass"], st["box"], rc=2.5, trunc=1, skin=0.3, dt=0.005)
    sim.set_langevin(1.0, temp, 777)
    sim.prime()
    sim.run("baoab", steps)
    p, vel, f = sim.state()
    assert np.max(np.abs(s.positions - p)) < 1e-10
    assert np.max(np.abs(s.velocities - vel)) < 1e-10


def ks_normal(sample, sigma):
    """Kolmogorov-Smirnov statistic against N(0, sigma) (tests/test_thermostat.cpp:29-39)."""
    from math import erfc, sqrt
    x = np.sort(np.asarray(sample))
    n = len(x)
    phi = np.array([0.5 * erfc(-v / (sigma * sqrt(2.0))) for v in x])
    k = np.arange(1, n + 1)
    return max(np.max(k / n - phi), np.max(phi - (k - 1) / n))


def test_baoab_noise_is_standard_normal(md):
    """The O-step's Philox normals: from v = 0 and zero force, one BAOAB step leaves
    v = c2 * sqrt(T/m) * xi exactly, so the velocities expose the raw noise."""
    s, st = lattice_system(md, 8, 0.8, 1.0, 4)  # N = 2048
    s.velocities = np.zeros((s.n, 3))
    s.forces = np.zeros((s.n, 3))
    dt, gamma = 0.005, 1.0
    c1 = np.exp(-gamma * dt)
    c2 = np.sqrt(1.0 - c1 * c1)
    integ = md.LangevinBAOAB(dt, gamma, 1.0, 99)
    xs = []
    for _ in range(8):
        s.velocities = np.zeros((s.n, 3))
        integ.step(s, lambda q: 0.0)
        xs.append(s.velocities.ravel() / c2)
    xi = np.concatenate(xs)  # 49152 draws
    assert abs(np.mean(xi)) < 5.0 / np.sqrt(len(xi))
    assert abs(np.var(xi) - 1.0) < 5.0 * np.sqrt(2.0 / len(xi))
    assert ks_normal(xi, 1.0) < 1.63 / np.sqrt(len(xi))
    # consecutive steps and neighbouring atoms are uncorrelated
    a = xs[0].reshape(-1, 3)
    b = xs[1].reshape(-1, 3)
    assert abs(np.corrcoef(a[:, 0], b[:, 0])[0, 1]) < 5.0 / np.sqrt(len(a))
    assert abs(np.corrcoef(a[:-1, 0], a[1:, 0])[0, 1]) < 5.0 / np.sqrt(len(a))


def test_baoab_equipartition(md):
    """tests/test_thermostat.cpp:41-96 with Philox noise (statistical parity).  N=864
    rather than 108 so the +-2% band is ~5 standard errors of the mean wide."""
    s, st = lattice_system(md, 6, 0.80, 1.0, 42)
    lj = md.LennardJones(1.0, 1.0, 2.5, md.Truncation.LinearForceShift)
    v = md.VerletList(st["box"], 2.5, 0.3)
    v.build(s)
    lj.compute_forces(s, v)
    integ = md.LangevinBAOAB(0.005, 1.0, 1.0, 777)
    integ.run(s, v, lj, 3000)
    th = integ.run(s, v, lj, 10000, thermo=True)
    dof = 3 * s.n
    mean_t = np.mean(2.0 * th[:, 2] / dof)
    assert 0.98 < mean_t < 1.02, mean_t


def test_baoab_velocity_distribution_is_maxwell_boltzmann(md):
    """tests/test_thermostat.cpp:98-143: frames 5/gamma apart, KS vs N(0, sqrt(T/m))."""
    s, st = lattice_system(md, 3, 0.80, 1.0, 43)
    lj = md.LennardJones(1.0, 1.0, 2.5, md.Truncation.LinearForceShift)
    v = md.VerletList(st["box"], 2.5, 0.3)
    v.build(s)
    lj.compute_forces(s, v)
    integ = md.LangevinBAOAB(0.005, 1.0, 1.0, 778)
    integ.run(s, v, lj, 3000)
    comps = []
    for _ in range(60):
        integ.run(s, v, lj, 1000)
        comps.append(s.velocities.ravel())
    comps = np.concatenate(comps)
    assert ks_normal(comps, 1.0) < 1.63 / np.sqrt(len(comps))


def test_baoab_relaxes_hot_start(md):
    """tests/test_thermostat.cpp:145-179"""
    s, st = lattice_system(md, 3, 0.80, 3.0, 99)
    lj = md.LennardJones(1.0, 1.0, 2.5, md.Truncation.LinearForceShift)
    v = md.VerletList(st["box"], 2.5, 0.3)
    v.build(s)
    lj.compute_forces(s, v)
    integ = md.LangevinBAOAB(0.005, 1.0, 1.0, 779)
    integ.run(s, v, lj, 3000)
    th = integ.run(s, v, lj, 4000, thermo=True)
    final_t = np.mean(2.0 * th[:, 2] / (3 * s.n))
    assert 0.9 < final_t < 1.1 and final_t < 1.5


@pytest.mark.parametrize("chain,fused", [(3, False), (3, True), (1, True), (5, False), (5, True)])
def test_nhc_matches_oracle_short(md, chain, fused):
    """A few NHC steps, host-driven or one fused run, track the oracle's (analytic
    KE*s^2 vs re-summed KE only changes rounding), for the three-link chain the
    kernels hold in registers and for other lengths."""
    s, st = lattice_system(md, 3, 0.80, 3.0, 55)
    n = len(st["mass"])
    dof = 3 * n - 3
    lj = md.LennardJones(1.0, 1.0, 2.5, md.Truncation.LinearForceShift)
    v = md.VerletList(st["box"], 2.5, 0.3)
    v.build(s)
    lj.compute_forces(s, v)
    integ = md.NoseHooverChain(0.002, 1.0, 0.5, chain, dof)

    def forces(sys_):
        v.rebuild_if_needed(sys_)
        return lj.compute_forces(sys_, v)[0]

    if fused:
        integ.run(s, v, lj, 30)
    else:
        for _ in range(30):
            integ.step(s, forces)
    sim = O.Sim(st["pos"], st["vel"], st["mass"], st["box"], rc=2.5, trunc=1, skin=0.3, dt=0.002)
    sim.set_nhc(1.0, 0.5, chain, dof)
    sim.prime()
    sim.run("nhc", 30)
    p, vel, _ = sim.state()
    assert np.max(np.abs(s.positions - p)) < 1e-10
    assert np.max(np.abs(s.velocities - vel)) < 1e-10
    assert abs(integ.conserved_quantity_contribution() - sim.nhc_conserved) < 1e-9


def test_nhc_conserves_extended_hamiltonian(md):
    """tests/test_thermostat.cpp:222-263 (20,000 steps, max relative drift < 1e-3)."""
    s, st = lattice_system(md, 3, 0.80, 1.0, 56)
    dof = 3 * s.n - 3
    lj = md.LennardJones(1.0, 1.0, 2.5, md.Truncation.LinearForceShift)
    v = md.VerletList(st["box"], 2.5, 0.3)
    v.build(s)
    pe, _ = lj.compute_forces(s, v)
    integ = md.NoseHooverChain(0.002, 1.0, 0.5, 3, dof)
    h0 = pe + s.kinetic_energy() + integ.conserved_quantity_contribution()
    th = integ.run(s, v, lj, 20000, thermo=True)
    h = th[:, 0] + th[:, 2] + th[:, 3]
    drift = np.max(np.abs(h - h0)) / abs(h0)
    assert drift < 1e-3, drift
    mean_t = np.mean(2.0 * th[6000:, 2] / dof)
    assert 0.9 < mean_t < 1.1


def test_mixed_precision_force_error(md):
    """Mixed path: force RMS error against FP64 on identical states."""
    s, st = lattice_system(md, 8, 0.8442, 0.722, 5)
    lj64 = md.LennardJones(1.0, 1.0, 2.5)
    ljmx = md.LennardJones(1.0, 1.0, 2.5, precision=md.PRECISION_MIXED)
    v = md.VerletList(st["box"], 2.5, 0.3)
    v.build(s)
    # melt the lattice a little so forces are non-trivial
    integ = md.LangevinBAOAB(0.005, 1.0, 0.722, 9)
    lj64.compute_forces(s, v)
    integ.run(s, v, lj64, 200)
    e64, w64 = lj64.compute_forces(s, v)
    f64 = s.forces
    emx, wmx = ljmx.compute_forces(s, v)
    fmx = s.forces
    rms = np.sqrt(np.sum((fmx - f64) ** 2) / np.sum(f64 ** 2))
    assert rms < 1e-6, rms
    assert abs(emx - e64) < 1e-6 * abs(e64)
    assert abs(wmx - w64) < 1e-5 * abs(w64)


def test_bulk_field_transfer_equals_per_field(md):
    """md_system_set_fields / md_system_get_fields move the same bytes as one
    md_system_set / md_system_get per field, in original atom order, also after
    a rebuild has re-sorted the device arrays."""
    import ctypes as C
    s, st = lattice_system(md, 6, 0.8442, 0.722, 4)
    lj = md.LennardJones(1.0, 1.0, 2.5)
    v = md.VerletList(st["box"], 2.5, 0.3)
    v.build(s)
    lj.compute_forces(s, v)
    md.VelocityVerlet(0.005).run(s, v, lj, 60)
    assert v.rebuild_count() > 1
    n = s.n
    L = md.lib()
    dp = C.POINTER(C.c_double)
    fields = [md.FIELD_X + k for k in range(9)] + [md.FIELD_X + 9, md.FIELD_X + 10]
    outs = [np.zeros(n) for _ in fields]
    md._check(L.md_system_get_fields(s.handle, len(fields), (C.c_int * len(fields))(*fields),
                                     (dp * len(fields))(*[o.ctypes.data_as(dp) for o in outs])))
    per = [s._get1(f) for f in fields]
    for a, b in zip(outs, per):
        assert np.array_equal(a, b)
    rng = np.random.default_rng(3)
    new = [rng.normal(size=n) for _ in range(6)]
    md._check(L.md_system_set_fields(s.handle, 6, (C.c_int * 6)(*fields[:6]),
                                     (dp * 6)(*[a.ctypes.data_as(dp) for a in new])))
    assert np.array_equal(s.positions, np.stack(new[:3], 1))
    assert np.array_equal(s.velocities, np.stack(new[3:6], 1))
    with pytest.raises(md.InvalidArgument):
        md._check(L.md_system_set_fields(s.handle, 1, (C.c_int * 1)(42),
                                         (dp * 1)(new[0].ctypes.data_as(dp))))
