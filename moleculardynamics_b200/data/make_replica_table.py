"""Draws the 48-replica batch workload (fcc cells n ~ U{4..20}, density from
{0.1, 0.3, 0.5, 0.7, 0.8, 0.9}, thermostat temperature ~ U[1, 2], distinct lattice
seeds) with a fixed master seed and writes replicas_48.json beside this file.

    python moleculardynamics_b200/data/make_replica_table.py
"""
import json
import os

import numpy as np

MASTER_SEED = 20261203


def draw(count=48, master_seed=MASTER_SEED):
    rng = np.random.default_rng(master_seed)
    densities = [0.1, 0.3, 0.5, 0.7, 0.8, 0.9]
    rows = []
    for k in range(count):
        cells = int(rng.integers(4, 21))
        rho = float(densities[int(rng.integers(0, len(densities)))])
        temp = float(np.round(rng.uniform(1.0, 2.0), 6))
        rows.append({"replica": k, "cells": cells, "atoms": 4 * cells ** 3, "density": rho,
                     "temperature": temp, "seed": 1000 + k})
    return rows


if __name__ == "__main__":
    table = {"master_seed": MASTER_SEED, "integrator": "NoseHooverChain M=3 tau=0.5 dt=0.005",
             "potential": "LJ sigma=epsilon=1 rc=2.5 truncated, Verlet skin 0.3",
             "replicas": draw()}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "replicas_48.json")
    with open(path, "w") as fh:
        json.dump(table, fh, indent=1)
    print(path, sum(r["atoms"] for r in table["replicas"]), "atoms")
