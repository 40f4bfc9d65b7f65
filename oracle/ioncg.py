"""Test infrastructure (the oracle): a CPU restatement of the reference's old
conjugate-gradient ion optimiser, GradientOptimization
(Source/IonOptCON.f90:33-241), on the oracle's functional, NTN solver, forces
and its Dcsrch (oracle/linesearch.py).  Only tests import it.  No run of this
optimiser ships with the reference, so it is pinned only against the engine's
driver (parity unpinned to the reference itself).
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import forces as ofo
from . import ntn
from .linesearch import Dcsrch
from .md import functional_for

FORCE_CUTOFF = float(np.float32(5e-5))


def gradient_optimization(cell, n, opts: ntn.NtnOptions, force_cutoff=FORCE_CUTOFF, max_steps=200,
                          alpha_=5.0 / 6.0, beta_=5.0 / 6.0, rho0=None):
    """Returns (final fractional coordinates, the total energy (Ha) of every
    density solve in order, final forces)."""
    from . import cellsetup as cs
    cell = dataclasses.replace(cell, frac=np.array(cell.frac, dtype=float))
    cart2frac = np.linalg.inv(cell.lattice)
    rho = cs.uniform_density(cell, *n) if rho0 is None else rho0

    def solve(rho):
        r = ntn.NtnSolver(functional_for(cell, n, alpha_, beta_), opts).solve(rho)
        f, _, _ = ofo.total_forces(cell, r.rho)
        return r.rho, float(r.energy[0]), f

    rho, energy, forces = solve(rho)
    trace = [energy]
    max_force = float(np.sqrt((forces ** 2).sum(axis=1)).max())
    stp = 0.0
    step = 1
    checkpt1 = checkpt2 = 0.0
    while True:
        if max_force < force_cutoff or step > max_steps:
            break
        if step == 1:
            dir_next = forces.copy()
            fp = float((-forces * dir_next).sum())
            stp = 5.0
        else:
            gamma = max(float((forces * (forces - g)).sum()) / float((g * g).sum()), 0.0)
            dir_next = forces + gamma * dir_next
            fp_last = fp
            fp = float((-forces * dir_next).sum())
            stp = max(min(stp * fp_last / fp, stp * 2.0), stp * 0.25)
        g = forces.copy()
        orig = cell.frac.copy()
        num_line = 0
        task = "START"
        ls = Dcsrch(0.01, 0.1, 1e-10, 1e-100, 1000.0)
        while True:
            stp, task = ls.step(stp, energy, float((-forces * dir_next).sum()), task)
            if task != "FG":
                break
            if num_line % 5 == 4:
                checkpt2 = checkpt1
                checkpt1 = energy
                if num_line > 10 and abs(checkpt2 - checkpt1) / len(cell.frac) < 1e-9:
                    stp = 1.0
                    g = forces.copy()
                    break
            frac_step = np.array([cart2frac @ (stp * dir_next[i]) for i in range(len(cell.frac))])
            cell.frac = np.mod(orig + frac_step, 1.0)
            rho, energy, forces = solve(rho)
            trace.append(energy)
            max_force = float(np.sqrt((forces ** 2).sum(axis=1)).max())
            num_line += 1
        step += 1
    return cell.frac, trace, forces
