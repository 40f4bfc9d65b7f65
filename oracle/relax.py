"""Test infrastructure (the oracle): a CPU restatement of the reference's
QuickMin ion optimiser, QuickMinOptimization (Source/IonOptQui.f90:33-368),
on the oracle's functional, NTN solver and forces.  Only tests import it.

Each step: every tenth step (step mod 10 = 9) the time step halves if the
largest force grew three-fold since the last check; the ions move by
dt v + dt^2 F / 2 (fractional coordinates wrapped into [0, 1)); the density is
re-solved from the last density; a move that raises the energy (or, from the
first step, turns the force against the velocity) is undone with the time step
cut five-fold and the velocity reset; otherwise the time step doubles and the
velocity becomes its projection on the force plus dt F.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import forces as ofo
from . import ntn
from .md import functional_for

FORCE_CUTOFF = float(np.float32(5e-5))  # Source/IonOptimizers.f90:29 (single-precision literal)


def _max_force(f):
    return float(np.sqrt((f * f).sum(axis=1)).max())


def quickmin(cell, n, opts: ntn.NtnOptions, time_step=0.4, force_cutoff=FORCE_CUTOFF, max_steps=200,
             alpha=5.0 / 6.0, beta=5.0 / 6.0):
    """Returns (final fractional coordinates, energy of the last solve, forces,
    history of (step, energy, max force, time step, undone))."""
    from . import cellsetup as cs
    cell = dataclasses.replace(cell, frac=np.array(cell.frac, dtype=float))
    cart2frac = np.linalg.inv(cell.lattice)
    rho = cs.uniform_density(cell, *n)
    r = ntn.NtnSolver(functional_for(cell, n, alpha, beta), opts).solve(rho)
    rho = r.rho
    old_energy = float(r.energy[0])
    forces, _, _ = ofo.total_forces(cell, rho)
    vel = np.zeros_like(forces)
    max_force = best = min_max = _max_force(forces)
    energy = old_energy
    step = 1
    hist = []
    while True:
        step += 1
        if step > max_steps or max_force < force_cutoff:
            break
        if step % 10 == 9:
            if max_force > min_max * 3.0:
                time_step *= 0.5
            else:
                min_max = max_force
        frac_step = (time_step * vel + 0.5 * time_step ** 2 * forces) @ cart2frac.T
        last = cell.frac.copy()
        cell.frac = np.mod(cell.frac + frac_step, 1.0)
        prev = forces
        r = ntn.NtnSolver(functional_for(cell, n, alpha, beta), opts).solve(rho)
        rho = r.rho
        energy = float(r.energy[0])
        forces, _, _ = ofo.total_forces(cell, rho)
        max_force = _max_force(forces)
        best = min(best, max_force)
        fv = float((forces * vel).sum())
        undone = False
        if fv < 0.0 or energy > old_energy:
            if step == 1 or energy > old_energy:
                undone = True
                time_step /= 5.0
                vel = np.zeros_like(vel)
                forces = prev
                cell.frac = last
            else:
                old_energy = energy
                vel = np.zeros_like(vel)
        else:
            time_step *= 2.0
            old_energy = energy
            vel = fv * forces / float((forces * forces).sum()) + forces * time_step
        hist.append((step, energy, max_force, time_step, undone))
    return cell.frac, energy, forces, hist
