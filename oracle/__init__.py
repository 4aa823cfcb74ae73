"""CPU oracle for moldyn's force / neighbour / integrator path -- TEST INFRASTRUCTURE.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs import
this package, and only as the checker.  The product (``moleculardynamics_b200``)
never imports it.

Two libraries sit behind it:

* ``_build/libmd_oracle.so`` -- ``md_oracle.c``, a C restatement of the reference
  algorithm (always built by ``oracle/Makefile``);
* ``_ref/libmoldyn_ref.so`` -- the reference itself, compiled from its own sources
  (only where the reference tree was present at build time).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libmd_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmoldyn_ref.so")

_d = C.POINTER(C.c_double)
_i64 = C.POINTER(C.c_int64)


def build(ref_root: str | None = None) -> None:
    """Compile the restatement (and the reference, when its sources exist under
    ref_root, else under oracle/Makefile's REF_ROOT)."""
    env = dict(os.environ)
    if ref_root:
        env["REF_ROOT"] = ref_root
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True, env=env)


def _p(a):
    if a is None:
        return None
    if a.dtype == np.float64:
        return a.ctypes.data_as(_d)
    if a.dtype == np.int64:
        return a.ctypes.data_as(_i64)
    raise TypeError(a.dtype)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class OrcLJ(C.Structure):
    _fields_ = [("sigma", C.c_double), ("epsilon", C.c_double), ("cutoff", C.c_double),
                ("truncation", C.c_int), ("u_at_cutoff", C.c_double),
                ("dudr_at_cutoff", C.c_double)]


class OrcRng(C.Structure):
    _fields_ = [("mt", C.c_uint64 * 312), ("index", C.c_int), ("spare", C.c_double),
                ("have_spare", C.c_int)]


class OrcEwaldTerms(C.Structure):
    _fields_ = [("real", C.c_double), ("reciprocal", C.c_double), ("self", C.c_double),
                ("intra", C.c_double)]


class OrcNhc(C.Structure):
    _fields_ = [("dt", C.c_double), ("temperature", C.c_double), ("tau", C.c_double),
                ("chain_length", C.c_int), ("dof", C.c_int64), ("Q", C.c_double * 16),
                ("xi", C.c_double * 16), ("pxi", C.c_double * 16)]


class OrcRigidWater(C.Structure):
    _fields_ = [("oh", C.c_double), ("hh", C.c_double), ("tolerance", C.c_double),
                ("max_iterations", C.c_int)]


_lib = None
_ref = None


def lib():
    """The restatement library (md_oracle.c)."""
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.orc_fold.restype = C.c_double
        L.orc_fold.argtypes = [C.c_double, C.c_double]
        L.orc_lj_init.argtypes = [C.POINTER(OrcLJ), C.c_double, C.c_double, C.c_double, C.c_int]
        L.orc_lj_compute.restype = C.c_int
        L.orc_lj_compute.argtypes = [C.POINTER(OrcLJ), C.c_int64, _d, _d, _d, _d, C.c_int, _i64,
                                     _i64, C.c_int64, C.c_int, _d, _d, _d, _d, _d]
        L.orc_lj_lrc_energy.restype = C.c_double
        L.orc_lj_lrc_energy.argtypes = [C.POINTER(OrcLJ), C.c_int64, _d]
        L.orc_lj_lrc_pressure.restype = C.c_double
        L.orc_lj_lrc_pressure.argtypes = [C.POINTER(OrcLJ), C.c_int64, _d]
        L.orc_cells_dims.argtypes = [_d, C.c_double, C.POINTER(C.c_int)]
        L.orc_cells_pairs.restype = C.c_int64
        L.orc_cells_pairs.argtypes = [C.c_int64, _d, _d, _d, _d, C.c_double, _i64, _i64, C.c_int64]
        L.orc_verlet_build.restype = C.c_int64
        L.orc_verlet_build.argtypes = [C.c_int64, _d, _d, _d, _d, C.c_double, C.c_double, _i64,
                                       _i64, C.c_int64]
        L.orc_verlet_needs_rebuild.restype = C.c_int
        L.orc_verlet_needs_rebuild.argtypes = [C.c_int64, _d, _d, _d, _d, _d, _d, _d, C.c_double]
        L.orc_verlet_top2.argtypes = [C.c_int64, _d, _d, _d, _d, _d, _d, _d, _d, _d]
        L.orc_rng_seed.argtypes = [C.POINTER(OrcRng), C.c_uint64]
        L.orc_rng_normals.argtypes = [C.POINTER(OrcRng), _d, C.c_int64]
        L.orc_fcc_lattice.restype = C.c_int
        L.orc_fcc_lattice.argtypes = [C.c_int, C.c_double, C.c_double, C.c_uint64] + [_d] * 8
        L.orc_kinetic_energy.restype = C.c_double
        L.orc_kinetic_energy.argtypes = [C.c_int64, _d, _d, _d, _d]
        L.orc_remove_com_motion.argtypes = [C.c_int64, _d, _d, _d, _d]
        L.orc_half_kick.argtypes = [C.c_int64, C.c_double, _d, _d, _d, _d, _d, _d, _d]
        L.orc_drift_wrap.argtypes = [C.c_int64, _d, C.c_double, _d, _d, _d, _d, _d, _d]
        L.orc_baoab_o_noise.argtypes = [C.c_int64, C.c_double, C.c_double, C.c_double, _d, _d,
                                        _d, _d, _d]
        L.orc_sim_create.restype = C.c_void_p
        L.orc_sim_create.argtypes = [C.c_int64, _d] + [_d] * 7 + [C.c_double, C.c_double,
                                                                    C.c_double, C.c_int,
                                                                    C.c_double]
        L.orc_sim_destroy.argtypes = [C.c_void_p]
        L.orc_sim_prime.restype = C.c_double
        L.orc_sim_prime.argtypes = [C.c_void_p]
        L.orc_sim_run.restype = C.c_int
        L.orc_sim_run.argtypes = [C.c_void_p, C.c_int, C.c_int64]
        L.orc_sim_set_langevin.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_uint64]
        L.orc_sim_set_nhc.restype = C.c_int
        L.orc_sim_set_nhc.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_int64]
        L.orc_sim_set_dt.argtypes = [C.c_void_p, C.c_double]
        L.orc_sim_get.argtypes = [C.c_void_p] + [_d] * 9
        L.orc_sim_set_state.argtypes = [C.c_void_p] + [_d] * 9
        for name in ("orc_sim_energy", "orc_sim_virial", "orc_sim_nhc_conserved"):
            getattr(L, name).restype = C.c_double
            getattr(L, name).argtypes = [C.c_void_p]
        L.orc_sim_rebuild_count.restype = C.c_int64
        L.orc_sim_rebuild_count.argtypes = [C.c_void_p]
        L.orc_sim_remove_com.argtypes = [C.c_void_p]
        L.orc_coulomb_prefactor.restype = C.c_double
        L.orc_ewald_compute.restype = C.c_int
        L.orc_ewald_compute.argtypes = [C.c_int64, _d, _d, _d, _d, _d, _i64, C.c_double, C.c_int,
                                        C.c_double, C.c_int, _d, _d, _d,
                                        C.POINTER(OrcEwaldTerms), _d]
        L.orc_spce_compute.restype = C.c_double
        L.orc_spce_compute.argtypes = [C.c_int64, _d, _d, _d, _d, _d, _i64, C.c_double,
                                       C.c_double, C.c_double, C.c_int, C.c_double, _d, _d, _d]
        L.orc_rigid_water_init.restype = C.c_int
        L.orc_rigid_water_init.argtypes = [C.POINTER(OrcRigidWater), C.c_double, C.c_double,
                                           C.c_double, C.c_int]
        L.orc_rigid_water_positions.restype = C.c_int
        L.orc_rigid_water_positions.argtypes = [C.POINTER(OrcRigidWater), C.c_int64, _d, _d, _d,
                                                _d, _d, _d, _d, _d]
        L.orc_rigid_water_velocities.restype = C.c_int
        L.orc_rigid_water_velocities.argtypes = [C.POINTER(OrcRigidWater), C.c_int64, _d, _d,
                                                 _d, _d, _d, _d, _d, _d]
        L.orc_nhc_init.restype = C.c_int
        L.orc_nhc_init.argtypes = [C.POINTER(OrcNhc), C.c_double, C.c_double, C.c_double,
                                   C.c_int, C.c_int64]
        L.orc_nhc_chain.restype = None
        L.orc_nhc_chain.argtypes = [C.POINTER(OrcNhc), C.c_int64, _d, _d, _d, _d, C.c_double]
        L.orc_nhc_conserved.restype = C.c_double
        L.orc_nhc_conserved.argtypes = [C.POINTER(OrcNhc)]
        L.orc_rdf_accumulate.restype = C.c_int
        L.orc_rdf_accumulate.argtypes = [C.c_int64, _d, _d, _d, _d, C.c_double, C.c_int64, _d]
        L.orc_rdf_g.argtypes = [_d, C.c_int64, C.c_double, C.c_int64, C.c_int64, C.c_double, _d]
        L.orc_msd.argtypes = [C.c_int64, C.c_int64, _d, _d, C.c_int64, _d]
        L.orc_vacf.argtypes = [C.c_int64, C.c_int64, _d, C.c_int64, _d]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    """The reference compiled from its own sources (None when absent)."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            return None
        R = C.CDLL(REF_SO)
        R.ref_lj_compute.restype = C.c_int
        R.ref_lj_compute.argtypes = [C.c_int64, _d, _d, _d, _d, C.c_double, C.c_double,
                                     C.c_double, C.c_int, C.c_int, C.c_double, _d, _d, _d, _d, _d]
        R.ref_lj_lrc.argtypes = [C.c_int64, _d, C.c_double, C.c_double, C.c_double, C.c_int, _d, _d]
        R.ref_cells_pairs.restype = C.c_int64
        R.ref_cells_pairs.argtypes = [C.c_int64, _d, _d, _d, _d, C.c_double, _i64, _i64,
                                      C.c_int64, C.POINTER(C.c_int)]
        R.ref_verlet_pairs.restype = C.c_int64
        R.ref_verlet_pairs.argtypes = [C.c_int64, _d, _d, _d, _d, C.c_double, C.c_double, _i64,
                                       _i64, C.c_int64]
        R.ref_lj_verlet_all.restype = C.c_int64
        R.ref_lj_verlet_all.argtypes = ([C.c_int64, _d, _d, _d, _d, C.c_double, C.c_double,
                                         C.c_double, C.c_int, C.c_double, _d, _d, _d, _d, _d,
                                         _i64, _i64, C.c_int64])
        R.ref_verlet_needs_rebuild.restype = C.c_int
        R.ref_verlet_needs_rebuild.argtypes = [C.c_int64, _d, _d, _d, _d, _d, _d, _d, C.c_double,
                                               C.c_double]
        R.ref_fcc_lattice.restype = C.c_int
        R.ref_fcc_lattice.argtypes = [C.c_int, C.c_double, C.c_double, C.c_uint64] + [_d] * 8
        R.ref_rng_normals.argtypes = [C.c_uint64, _d, C.c_int64]
        R.ref_run.restype = C.c_int
        R.ref_run.argtypes = ([C.c_int, C.c_int64, _d] + [_d] * 9 + [_d] +
                              [C.c_double, C.c_double, C.c_double, C.c_int, C.c_double,
                               C.c_double, C.c_int64, C.c_double, C.c_double, C.c_uint64,
                               C.c_double, C.c_int, C.c_int64, _d])
        R.ref_coulomb_prefactor.restype = C.c_double
        R.ref_ewald.argtypes = [C.c_int64, _d, _d, _d, _d, _d, _i64, C.c_double, C.c_int, C.c_int,
                                _d, _d, _d, _d]
        R.ref_spce.restype = C.c_double
        R.ref_spce.argtypes = [C.c_int64, _d, _d, _d, _d, _d, _d, _i64, C.c_double, C.c_int,
                               C.c_int, _d, _d, _d]
        R.ref_rigid_water.restype = C.c_int
        R.ref_rigid_water.argtypes = ([C.c_int, C.c_int64, _d, _d] + [_d] * 6 + [_d] * 3 +
                                      [C.c_double, C.c_double, C.c_double, C.c_int])
        R.ref_spce_cvv.restype = C.c_double
        R.ref_spce_cvv.argtypes = ([C.c_int64, _d] + [_d] * 9 + [_d, _d, _i64] +
                                   [C.c_double, C.c_int, C.c_double, C.c_int64])
        R.ref_rdf.restype = C.c_int
        R.ref_rdf.argtypes = [C.c_int64, C.c_int64, _d, _d, C.c_double, C.c_int64, _d, _d]
        R.ref_msd.argtypes = [C.c_int64, C.c_int64, _d, _d, C.c_int64, _d, C.c_double, C.c_int64,
                              C.c_int64, _d]
        R.ref_vacf.argtypes = [C.c_int64, C.c_int64, _d, _d, C.c_int64, _d, C.c_double, _d]
        _ref = R
    return _ref


def ref_lj_verlet(pos, box, rc=2.5, skin=0.3, trunc=0, sigma=1.0, eps=1.0, cap=None):
    """The compiled reference's moldyn_run ForceFn on one state: VerletList::build,
    LennardJones::computeForces(sys, verlet) and the list's pairs.  Returns
    (forces[N,3], energy, virial, pairs[M,2] in the reference's order)."""
    R = ref()
    if R is None:
        raise RuntimeError("the compiled reference (oracle/_ref/libmoldyn_ref.so) is absent")
    pos = _f64(pos)
    n = pos.shape[0]
    x, y, z = (np.ascontiguousarray(pos[:, k]) for k in range(3))
    box = _f64(box)
    f = [np.zeros(n) for _ in range(3)]
    e, w = C.c_double(), C.c_double()
    cap = cap or max(64, 48 * n)
    while True:
        pi = np.zeros(cap, dtype=np.int64)
        pj = np.zeros(cap, dtype=np.int64)
        m = R.ref_lj_verlet_all(n, _p(box), _p(x), _p(y), _p(z), sigma, eps, rc, trunc, skin,
                                *[_p(a) for a in f], C.byref(e), C.byref(w), _p(pi), _p(pj), cap)
        if m == -2:
            raise ValueError("reference raised std::invalid_argument")
        if m <= cap:
            return np.stack(f, 1), e.value, w.value, np.stack([pi[:m], pj[:m]], 1)
        cap = int(m)


# ---------------------------------------------------------------------------
# Convenience wrappers over the restatement
# ---------------------------------------------------------------------------

def fcc_lattice(cells, density, temperature, seed):
    n = 4 * cells ** 3
    arrs = [np.zeros(n) for _ in range(7)]
    box = np.zeros(3)
    lib().orc_fcc_lattice(cells, density, temperature, seed, *[_p(a) for a in arrs], _p(box))
    x, y, z, vx, vy, vz, m = arrs
    return dict(pos=np.stack([x, y, z], 1), vel=np.stack([vx, vy, vz], 1), mass=m, box=box)


def make_lj(sigma, eps, rc, trunc):
    lj = OrcLJ()
    lib().orc_lj_init(C.byref(lj), sigma, eps, rc, trunc)
    return lj


def lj_compute(pos, box, sigma=1.0, eps=1.0, rc=2.5, trunc=0, source="brute", pairs=None,
               forces=True):
    """Returns (forces[N,3] or None, energy, virial); raises ValueError on an unusable
    cell list (the reference's std::invalid_argument)."""
    pos = _f64(pos)
    n = pos.shape[0]
    x, y, z = (np.ascontiguousarray(pos[:, k]) for k in range(3))
    box = _f64(box)
    lj = make_lj(sigma, eps, rc, trunc)
    f = [np.zeros(n) for _ in range(3)]
    e = C.c_double()
    w = C.c_double()
    src = {"brute": 0, "cells": 1, "pairs": 2}[source]
    pi = pj = None
    np_ = 0
    if pairs is not None:
        pi = np.ascontiguousarray(pairs[:, 0], dtype=np.int64)
        pj = np.ascontiguousarray(pairs[:, 1], dtype=np.int64)
        np_ = pairs.shape[0]
    rc_ = lib().orc_lj_compute(C.byref(lj), n, _p(box), _p(x), _p(y), _p(z), src, _p(pi), _p(pj),
                               np_, 1 if forces else 0, *[_p(a) for a in f], C.byref(e),
                               C.byref(w))
    if rc_ == -2:
        raise ValueError("cell list is not usable (fewer than 3 cells per side)")
    return (np.stack(f, 1) if forces else None), e.value, w.value


def lj_lrc(n, box, sigma=1.0, eps=1.0, rc=2.5, trunc=0):
    lj = make_lj(sigma, eps, rc, trunc)
    box = _f64(box)
    return lib().orc_lj_lrc_energy(C.byref(lj), n, _p(box)), lib().orc_lj_lrc_pressure(
        C.byref(lj), n, _p(box))


def cells_dims(box, cutoff):
    dims = (C.c_int * 3)()
    lib().orc_cells_dims(_p(_f64(box)), cutoff, dims)
    return tuple(dims)


def _pairs_call(fn, pos, box, *extra):
    pos = _f64(pos)
    n = pos.shape[0]
    x, y, z = (np.ascontiguousarray(pos[:, k]) for k in range(3))
    box = _f64(box)
    cap = max(16, 8 * n)
    while True:
        pi = np.zeros(cap, np.int64)
        pj = np.zeros(cap, np.int64)
        cnt = fn(n, _p(box), _p(x), _p(y), _p(z), *extra, _p(pi), _p(pj), cap)
        if cnt < 0:
            raise RuntimeError("oracle pair enumeration failed")
        if cnt <= cap:
            return np.stack([pi[:cnt], pj[:cnt]], 1)
        cap = int(cnt)


def verlet_pairs(pos, box, cutoff, skin):
    """Verlet pairs (i<j) in the reference's traversal order."""
    return _pairs_call(lib().orc_verlet_build, pos, box, cutoff, skin)


def cell_pairs(pos, box, cutoff):
    """Candidate cell-list pairs (i<j) in the reference's traversal order."""
    return _pairs_call(lib().orc_cells_pairs, pos, box, cutoff)


def needs_rebuild(pos, ref_pos, box, skin):
    pos = _f64(pos)
    ref_pos = _f64(ref_pos)
    cols = [np.ascontiguousarray(a[:, k]) for a in (pos, ref_pos) for k in range(3)]
    return bool(lib().orc_verlet_needs_rebuild(pos.shape[0], _p(_f64(box)),
                                                *[_p(c) for c in cols], skin))


def top2(pos, ref_pos, box):
    pos = _f64(pos)
    ref_pos = _f64(ref_pos)
    cols = [np.ascontiguousarray(a[:, k]) for a in (pos, ref_pos) for k in range(3)]
    a = C.c_double()
    b = C.c_double()
    lib().orc_verlet_top2(pos.shape[0], _p(_f64(box)), *[_p(c) for c in cols], C.byref(a),
                          C.byref(b))
    return a.value, b.value


def rng_normals(seed, count):
    rng = OrcRng()
    lib().orc_rng_seed(C.byref(rng), seed)
    out = np.zeros(count)
    lib().orc_rng_normals(C.byref(rng), _p(out), count)
    return out


class Sim:
    """moldyn_run-style LJ simulation on the restatement (VerletList ForceFn)."""

    KINDS = {"vv": 0, "baoab": 1, "nhc": 2}

    def __init__(self, pos, vel, mass, box, sigma=1.0, eps=1.0, rc=2.5, trunc=0, skin=0.3,
                 dt=0.005):
        pos = _f64(pos)
        vel = _f64(vel)
        self.n = pos.shape[0]
        cols = [np.ascontiguousarray(a[:, k]) for a in (pos, vel) for k in range(3)]
        self._h = lib().orc_sim_create(self.n, _p(_f64(box)), *[_p(c) for c in cols],
                                       _p(_f64(mass)), sigma, eps, rc, trunc, skin)
        if not self._h:
            raise MemoryError("orc_sim_create failed")
        lib().orc_sim_set_dt(self._h, dt)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_sim_destroy(self._h)
            self._h = None

    def prime(self):
        return lib().orc_sim_prime(self._h)

    def set_langevin(self, friction, temperature, seed):
        lib().orc_sim_set_langevin(self._h, friction, temperature, seed)

    def set_nhc(self, temperature, tau, chain, dof):
        if lib().orc_sim_set_nhc(self._h, temperature, tau, chain, dof) != 0:
            raise ValueError("NoseHooverChain: chainLength must be >= 1")

    def run(self, kind, steps):
        if lib().orc_sim_run(self._h, self.KINDS[kind], steps) != 0:
            raise ValueError(kind)

    def state(self):
        arrs = [np.zeros(self.n) for _ in range(9)]
        lib().orc_sim_get(self._h, *[_p(a) for a in arrs])
        return (np.stack(arrs[0:3], 1), np.stack(arrs[3:6], 1), np.stack(arrs[6:9], 1))

    def set_state(self, pos=None, vel=None, frc=None):
        cols = []
        for a in (pos, vel, frc):
            if a is None:
                cols += [None] * 3
            else:
                a = _f64(a)
                cols += [np.ascontiguousarray(a[:, k]) for k in range(3)]
        lib().orc_sim_set_state(self._h, *[_p(c) for c in cols])

    energy = property(lambda self: lib().orc_sim_energy(self._h))
    virial = property(lambda self: lib().orc_sim_virial(self._h))
    rebuild_count = property(lambda self: lib().orc_sim_rebuild_count(self._h))
    nhc_conserved = property(lambda self: lib().orc_sim_nhc_conserved(self._h))

    def remove_com(self):
        lib().orc_sim_remove_com(self._h)


def ewald(pos, box, q, mol, cutoff=10.0, kmax=5, alpha=0.0, forces=True):
    """Returns (forces or None, terms dict, virial)."""
    pos = _f64(pos)
    n = pos.shape[0]
    x, y, z = (np.ascontiguousarray(pos[:, k]) for k in range(3))
    f = [np.zeros(n) for _ in range(3)]
    t = OrcEwaldTerms()
    vir = C.c_double()
    rc_ = lib().orc_ewald_compute(n, _p(_f64(box)), _p(x), _p(y), _p(z), _p(_f64(q)),
                                  _p(np.ascontiguousarray(mol, dtype=np.int64)), cutoff, kmax,
                                  alpha, 1 if forces else 0, *[_p(a) for a in f], C.byref(t),
                                  C.byref(vir))
    if rc_ != 0:
        raise RuntimeError("orc_ewald_compute failed")
    terms = dict(real=t.real, reciprocal=t.reciprocal, self=t.self, intra=t.intra)
    return (np.stack(f, 1) if forces else None), terms, vir.value


def spce(pos, box, q, mol, sigma_o=3.16555789, epsilon_o=78.19743111, cutoff=10.0, kmax=5,
         alpha=0.0, forces=True):
    pos = _f64(pos)
    n = pos.shape[0]
    x, y, z = (np.ascontiguousarray(pos[:, k]) for k in range(3))
    f = [np.zeros(n) for _ in range(3)] if forces else [None] * 3
    e = lib().orc_spce_compute(n, _p(_f64(box)), _p(x), _p(y), _p(z), _p(_f64(q)),
                               _p(np.ascontiguousarray(mol, dtype=np.int64)), sigma_o, epsilon_o,
                               cutoff, kmax, alpha, *[_p(a) for a in f])
    return (np.stack(f, 1) if forces else None), e


def rigid_water(oh=1.0, hoh=109.47, tol=1e-12, maxit=500):
    rw = OrcRigidWater()
    if lib().orc_rigid_water_init(C.byref(rw), oh, hoh, tol, maxit) != 0:
        raise ValueError("RigidWater: invalid parameters")
    return rw


def shake(rw, pos, ref_pos, mass, box):
    pos = _f64(pos).copy()
    n = pos.shape[0]
    cols = [np.ascontiguousarray(pos[:, k]) for k in range(3)]
    rcols = [np.ascontiguousarray(_f64(ref_pos)[:, k]) for k in range(3)]
    it = lib().orc_rigid_water_positions(C.byref(rw), n, _p(_f64(box)), _p(_f64(mass)),
                                         *[_p(c) for c in cols], *[_p(c) for c in rcols])
    return np.stack(cols, 1), it


def rattle(rw, pos, vel, mass, box):
    vel = _f64(vel).copy()
    n = vel.shape[0]
    pcols = [np.ascontiguousarray(_f64(pos)[:, k]) for k in range(3)]
    vcols = [np.ascontiguousarray(vel[:, k]) for k in range(3)]
    it = lib().orc_rigid_water_velocities(C.byref(rw), n, _p(_f64(box)), _p(_f64(mass)),
                                          *[_p(c) for c in pcols], *[_p(c) for c in vcols])
    return np.stack(vcols, 1), it


def nhc(dt, temperature, tau, chain_length, dof):
    """NoseHooverChain state (nose_hoover.cpp:15-43)."""
    c = OrcNhc()
    if lib().orc_nhc_init(C.byref(c), dt, temperature, tau, chain_length, dof) != 0:
        raise ValueError("NoseHooverChain: chainLength must be >= 1")
    return c


def nhc_chain(c, vel, mass, delta):
    """integrateChain(delta) (nose_hoover.cpp:59-124) on a copy of vel; returns it."""
    vel = _f64(vel)
    cols = [np.ascontiguousarray(vel[:, k]) for k in range(3)]
    lib().orc_nhc_chain(C.byref(c), vel.shape[0], _p(_f64(mass)), *[_p(a) for a in cols], delta)
    return np.stack(cols, 1)


def nhc_conserved(c):
    return lib().orc_nhc_conserved(C.byref(c))


def read_nist_config(path):
    """io/nist_config.cpp:30-86: box line, count line (not trusted), then
    `index x y z [type]` lines until EOF."""
    with open(path) as fh:
        lines = fh.read().splitlines()
    box = np.array([float(v) for v in lines[0].split()[:3]])
    pos, types = [], []
    for line in lines[2:]:
        f = line.split()
        if not f:
            continue
        pos.append([float(f[1]), float(f[2]), float(f[3])])
        types.append(f[4] if len(f) > 4 else "")
    return box, np.array(pos), types


# ---------------------------------------------------------------------------
# analyze/: RDF, MSD, VACF (restatement, and the reference itself)
# ---------------------------------------------------------------------------

def _frames_soa(frames):
    """(F, N, 3) -> contiguous F x (x[N] | y[N] | z[N])."""
    a = np.asarray(frames, dtype=np.float64)
    return np.ascontiguousarray(np.transpose(a, (0, 2, 1)))


def rdf(frames, box, rmax, bins):
    """rdf.cpp:55-107 over (F, N, 3) wrapped positions: (histogram, g)."""
    a = np.asarray(frames, dtype=np.float64)
    box = _f64(box)
    hist = np.zeros(bins)
    sum_rho = 0.0
    for f in a:
        x, y, z = (np.ascontiguousarray(f[:, d]) for d in range(3))
        if lib().orc_rdf_accumulate(len(f), _p(box), _p(x), _p(y), _p(z), rmax, bins,
                                    _p(hist)) != 0:
            raise ValueError("Rdf: rMax exceeds half the smallest box length")
        sum_rho += len(f) / (box[0] * box[1] * box[2])
    g = np.zeros(bins)
    lib().orc_rdf_g(_p(hist), bins, rmax, len(a), a.shape[1], sum_rho, _p(g))
    return hist, g


def msd(frames, box, max_lag):
    a = _frames_soa(frames)
    out = np.zeros(max_lag + 1)
    lib().orc_msd(a.shape[0], a.shape[2], _p(_f64(box)), _p(a), max_lag, _p(out))
    return out


def vacf_unnormalised(frames, max_lag):
    a = _frames_soa(frames)
    out = np.zeros(max_lag + 1)
    lib().orc_vacf(a.shape[0], a.shape[2], _p(a), max_lag, _p(out))
    return out


def ref_rdf(frames, box, rmax, bins):
    a = _frames_soa(frames)
    g, c = np.zeros(bins), np.zeros(bins)
    rc = ref().ref_rdf(a.shape[0], a.shape[2], _p(_f64(box)), _p(a), rmax, bins, _p(g), _p(c))
    if rc != 0:
        raise ValueError("Rdf: rMax exceeds half the smallest box length")
    return g, c


def ref_msd(frames, box, max_lag, dt, fit_from, fit_to):
    a = _frames_soa(frames)
    out, d = np.zeros(max_lag + 1), np.zeros(1)
    ref().ref_msd(a.shape[0], a.shape[2], _p(_f64(box)), _p(a), max_lag, _p(out), dt, fit_from,
                  fit_to, _p(d))
    return out, d[0]


def ref_vacf(frames, box, max_lag, dt):
    a = _frames_soa(frames)
    out, d = np.zeros(max_lag + 1), np.zeros(1)
    ref().ref_vacf(a.shape[0], a.shape[2], _p(_f64(box)), _p(a), max_lag, _p(out), dt, _p(d))
    return out, d[0]


# ---------------------------------------------------------------------------
# Smooth particle-mesh Ewald, restated in numpy from Essmann et al., J. Chem.
# Phys. 103, 8577 (1995).  The reference has no PME (its phase-2 plan defers
# it); this restatement is pinned by converging to the reference-pinned Ewald
# sum above as the grid is refined, and is the checker of the device PME.
# ---------------------------------------------------------------------------

def _bspline_weights(w, p):
    """c[:, j] = M_p(w + j) and d[:, j] = M_p'(w + j), j = 0..p-1 (cardinal
    B-spline recursion, Essmann eq. 4.1 and 4.2)."""
    w = np.asarray(w, dtype=np.float64)
    c = np.zeros((w.size, p))
    c[:, 0] = w
    c[:, 1] = 1.0 - w
    d = np.zeros((w.size, p))
    if p == 2:
        d[:, 0], d[:, 1] = 1.0, -1.0
    for n in range(3, p + 1):
        if n == p:
            d = c - np.concatenate([np.zeros((w.size, 1)), c[:, :-1]], axis=1)
        new = np.zeros_like(c)
        for j in range(n):
            x = w + j
            lo = c[:, j - 1] if j > 0 else 0.0
            new[:, j] = (x * c[:, j] + (n - x) * lo) / (n - 1)
        c = new
    return c, d


def _bspline_moduli(K, p):
    """|b(m)|^2 = 1 / |sum_{k=0}^{p-2} M_p(k+1) exp(2 pi i m k / K)|^2 (Essmann eq. 4.4)."""
    ints, _ = _bspline_weights(np.array([0.0]), p)  # M_p(j), j = 0..p-1
    mk = ints[0, 1:p]                                # M_p(1..p-1)
    m = np.arange(K)[:, None]
    k = np.arange(p - 1)[None, :]
    s = np.sum(mk[None, :] * np.exp(2j * np.pi * m * k / K), axis=1)
    mag = np.abs(s) ** 2
    out = np.where(mag > 1e-10, 1.0 / np.where(mag > 1e-10, mag, 1.0), 0.0)
    for i in np.nonzero(out == 0.0)[0]:
        out[i] = 0.5 * (out[(i - 1) % K] + out[(i + 1) % K])
    return out


def pme_recip(pos, box, q, alpha, K, order):
    """Reciprocal-space energy, virial trace and forces of smooth PME on a
    K[0] x K[1] x K[2] grid with B-splines of `order`.  Returns (E, W, F)."""
    pos, box, q = _f64(pos).reshape(-1, 3), _f64(box), _f64(q)
    K = [int(k) for k in (K if np.ndim(K) else (K, K, K))]
    n = pos.shape[0]
    coulomb = lib().orc_coulomb_prefactor()
    volume = float(np.prod(box))
    frac = pos / box
    frac = frac - np.floor(frac)
    u = frac * np.array(K)
    u = np.where(u >= np.array(K), u - np.array(K), u)
    i0 = np.floor(u).astype(np.int64)
    w = u - i0
    cs, ds = [], []
    for a in range(3):
        c, d = _bspline_weights(w[:, a], order)
        cs.append(c)
        ds.append(d)
    j = np.arange(order)
    gx = (i0[:, 0:1] - j[None, :]) % K[0]
    gy = (i0[:, 1:2] - j[None, :]) % K[1]
    gz = (i0[:, 2:3] - j[None, :]) % K[2]
    Q = np.zeros(K)
    wts = (q[:, None, None, None] * cs[0][:, :, None, None] * cs[1][:, None, :, None] *
           cs[2][:, None, None, :])
    ix = np.broadcast_to(gx[:, :, None, None], wts.shape)
    iy = np.broadcast_to(gy[:, None, :, None], wts.shape)
    iz = np.broadcast_to(gz[:, None, None, :], wts.shape)
    np.add.at(Q, (ix.ravel(), iy.ravel(), iz.ravel()), wts.ravel())
    F = np.fft.fftn(Q)
    m = [np.fft.fftfreq(K[a], 1.0 / K[a]) / box[a] for a in range(3)]
    m2 = m[0][:, None, None] ** 2 + m[1][None, :, None] ** 2 + m[2][None, None, :] ** 2
    B = [_bspline_moduli(K[a], order) for a in range(3)]
    Bm = B[0][:, None, None] * B[1][None, :, None] * B[2][None, None, :]
    with np.errstate(divide="ignore", invalid="ignore"):
        theta = np.where(m2 > 0, np.exp(-np.pi ** 2 * m2 / alpha ** 2) / m2 * Bm, 0.0)
    em = coulomb / (2.0 * np.pi * volume) * theta * np.abs(F) ** 2
    energy = float(np.sum(em))
    virial = float(np.sum(em * (1.0 - 2.0 * np.pi ** 2 * m2 / alpha ** 2)))
    phi = coulomb / (np.pi * volume) * np.real(np.fft.ifftn(theta * F)) * float(np.prod(K))
    grads = []
    for a in range(3):
        parts = [cs[0], cs[1], cs[2]]
        parts[a] = ds[a]
        stencil = (parts[0][:, :, None, None] * parts[1][:, None, :, None] *
                   parts[2][:, None, None, :])
        vals = phi[ix, iy, iz]
        grads.append(np.sum(stencil * vals, axis=(1, 2, 3)) * K[a] / box[a])
    forces = -q[:, None] * np.stack(grads, axis=1)
    return energy, virial, forces
