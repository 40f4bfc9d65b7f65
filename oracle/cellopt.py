"""Test infrastructure (the oracle): a CPU restatement of the reference's cell
optimiser, SteepestDecent (Source/CellOptimizers.f90:107-304) with its inner
density solve (ion method "non": the ions stay at their fractional
coordinates), on the oracle's functional, NTN solver and stress
(oracle/stress.py).  Only tests import it.  Pinned to the reference's own
cell relaxation of test/optCell (tests/golden/ref_cases.json, "cell_relax").
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import ntn
from . import stress as ost
from .md import functional_for

MAX_CELL_STEP = 100   # CellOptimizers.f90: maxCellStep
TOLS = 5.0e-7         # CellOptimizers.f90: tols (Ha/bohr^3)


def steepest_descent(cell, n, opts: ntn.NtnOptions, max_steps=MAX_CELL_STEP, tols=TOLS, axis=0,
                     alpha_=5.0 / 6.0, beta_=5.0 / 6.0, kinetic=None, gamma=2.7):
    """Returns (final lattice, [(energy (Ha), stress, lattice) per cell step]).
    kinetic = KEDF_WGC relaxes with the second-order WGC functional (its
    kernel rebuilt at the new N/V after each move, and WGCStress)."""
    from . import functional as fn
    kinetic = fn.KEDF_WT if kinetic is None else kinetic
    from . import cellsetup as cs
    cell = dataclasses.replace(cell, frac=np.array(cell.frac, dtype=float),
                               lattice=np.array(cell.lattice, dtype=float))
    rho = cs.uniform_density(cell, *n)
    dt = 10.0
    old_energy = 0.0
    trace = []
    i = 0
    while True:
        i += 1
        if i > max_steps:
            break
        f = functional_for(cell, n, alpha_, beta_, kinetic, gamma)  # RefreshCellSetup: kernel (rho0 = N/V), ions, Ewald
        r = ntn.NtnSolver(f, opts).solve(rho)
        rho = r.rho
        energy = float(r.energy[0])
        stress = ost.stress(cell, f, rho, gamma=gamma)
        trace.append((energy, stress.copy(), cell.lattice.copy()))
        if axis in (1, 2, 3):
            keep = stress[axis - 1, axis - 1]
            stress = np.zeros((3, 3))
            stress[axis - 1, axis - 1] = keep
            if abs(stress[axis - 1, axis - 1]) < tols:
                break
        elif np.abs(stress).max() < tols:
            break
        if energy > old_energy:
            dt = dt / 4.0
        else:
            dt = dt * 1.2
        old_energy = energy
        new = cell.lattice - cell.vol * dt * (stress @ np.linalg.inv(cell.lattice).T)
        if axis in (1, 2, 3):
            for j in range(3):
                for k in range(3):
                    if k != axis - 1 or j != axis - 1:
                        new[k, j] = cell.lattice[k, j]
        cell.lattice = new
        rho = rho * (cell.num_electrons / (rho.sum() * cell.vol / rho.size))  # RescaleDensity
    return cell.lattice, trace
