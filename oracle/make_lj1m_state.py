"""Equilibrated 1,048,576-atom LJ liquid made by the reference itself -- a build
artefact of the oracle, like ``_ref/libmoldyn_ref.so``.

The state is moldyn_run's protocol for the large LJ system: the seeded fcc 64^3
lattice (rho* = 0.8442, T* = 0.722, seed 2026), then 2000 LangevinBAOAB steps
(gamma* = 1, dt* = 0.005, seed 2027) with the reference's VerletList (rc = 2.5,
skin 0.3, truncated) and LennardJones, run by the reference compiled from its own
sources (``ref_run`` in ``ref_capi.cpp`` over ``integrate/langevin.hpp:36-88``), then
the centre-of-mass momentum removed as ``System::removeCenterOfMassMotion``
(``core/system.cpp``) does for unit masses.  Both arms of the benchmark time their
NVE steps from this one state, so they time the same configuration.

    python oracle/make_lj1m_state.py [--steps 2000] [--out oracle/_ref/lj1m_baoab2000.npz]

About an hour on one core.  The output lies under ``_ref/`` (git-ignored, travels
with the built libraries).
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import oracle as O  # noqa: E402

CELLS, RHO, TEMP, RC, SKIN, DT, SEED = 64, 0.8442, 0.722, 2.5, 0.3, 0.005, 2026
DEFAULT_OUT = os.path.join(HERE, "_ref", "lj1m_baoab2000.npz")


def lattice(cells):
    """The reference's seeded fcc lattice (util/lattice.cpp:15-64)."""
    R = O.ref()
    n = 4 * cells ** 3
    arrs = [np.zeros(n) for _ in range(7)]
    box = np.zeros(3)
    rc = R.ref_fcc_lattice(cells, RHO, TEMP, SEED, *[O._p(a) for a in arrs], O._p(box))
    if rc != n:
        raise RuntimeError("ref_fcc_lattice failed")
    return arrs, box


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--cells", type=int, default=CELLS)
    ap.add_argument("--out", default=DEFAULT_OUT)
    a = ap.parse_args()
    R = O.ref()
    if R is None:
        raise SystemExit("oracle/_ref/libmoldyn_ref.so is missing: run make -C oracle ref")
    (x, y, z, vx, vy, vz, m), box = lattice(a.cells)
    n = x.size
    f = [np.zeros(n) for _ in range(3)]
    info = np.zeros(5)
    t0 = time.time()
    # kind 1 = LangevinBAOAB(dt, gamma, T, seed) over VerletList + LennardJones
    rc = R.ref_run(1, n, O._p(box), *[O._p(v) for v in (x, y, z, vx, vy, vz)],
                   *[O._p(v) for v in f], O._p(m), 1.0, 1.0, RC, 0, SKIN, DT, a.steps, 1.0,
                   TEMP, SEED + 1, 0.0, 0, 0, O._p(info))
    if rc != 0:
        raise RuntimeError(f"ref_run failed ({rc})")
    # centre-of-mass momentum to zero (unit masses: subtract the mean velocity)
    for v in (vx, vy, vz):
        v -= np.sum(v * m) / np.sum(m)
    pos = np.stack([x, y, z], 1)
    vel = np.stack([vx, vy, vz], 1)
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    tmp = a.out + ".tmp.npz"
    np.savez(tmp, pos=pos, vel=vel, box=box, steps=np.int64(a.steps), cells=np.int64(a.cells),
             rebuilds=np.int64(info[2]), seconds=np.float64(info[4]))
    os.replace(tmp, a.out)
    print(f"{a.steps} BAOAB steps of {n} atoms in {time.time() - t0:.1f} s "
          f"({int(info[2])} rebuilds) -> {a.out}")


if __name__ == "__main__":
    main()
