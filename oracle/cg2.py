"""Test infrastructure (the oracle): a CPU restatement of the reference's CG2 ion
optimiser, ConjugateGradient (Source/IonOptCG2.f90:39-505), with its line search
LnSrch (Source/MathLNsrch.f90:32-293), on the oracle's functional, NTN solver
and forces.  Only tests import it.

Defaults as the reference has them: the Hager-Zhang update (cg_type = 2,
Source/IonOptimizers.f90:36), force tolerance 5e-5 Ha/bohr, ftol = 1e-4 and
gtol = 0.1 (single-precision literals there, Source/IonOptCG2.f90), a restart
every 30 steps, and the step bound from the nearest-neighbour distance with
nnDist = 2 bohr (Source/Neighbor.f90:33).  The line-search limit maxLine is an
uninitialised local in the reference; it is taken as unbounded here.
"""
from __future__ import annotations

import dataclasses
import itertools

import numpy as np

from . import forces as ofo
from . import ntn
from .md import functional_for

FORCE_CUTOFF = float(np.float32(5e-5))
FTOL = float(np.float32(1e-4))
GTOL = float(np.float32(1e-1))
XTOL = 1.0e-12


class LineSearch:
    """LnSrch (Source/MathLNsrch.f90:32-293): a secant search on dE/dalpha with
    a left and a right point; task strings as the reference's."""

    def __init__(self):
        self.points = np.full((2, 3), -1.0)   # rows: left, right; columns: alpha, E, dE/dalpha
        self.dsave = np.zeros(2)

    @staticmethod
    def _new_alp(x1, y1, x2, y2, stp_min, stp_max):
        slope = (y1 - y2) / (x1 - x2)
        b = y1 - x1 * slope
        a = -b / slope
        return -1.0 if (a >= stp_max or a <= stp_min) else a

    def step(self, alp, f, g, task, c1, c2, stp_min, stp_max):
        p = self.points
        if task.startswith("START"):
            if g > 0.0:
                return "ERROR: Initial G>0", alp
            p[:] = -1.0
            p[0] = (0.0, f, g)
            self.dsave[:] = (f, g)
            p[1, 0] = -1.0
            return "FG", alp
        if task.startswith("FG") and p[1, 0] > 0.0:
            if f <= self.dsave[0] + c1 * alp * self.dsave[1] and abs(g) <= c2 * abs(self.dsave[1]):
                return "CONV", alp
        if p[1, 0] < 0.0:
            if g < p[0, 2]:
                alp = alp * 5.0 if f < p[0, 1] else (p[0, 0] + alp) / 2.0
                return "WARNING: Need a better second point.", alp
            p[1] = (alp, f, g)
            alp = self._new_alp(p[0, 0], p[0, 2], p[1, 0], p[1, 2], stp_min, stp_max)
            if alp < 0.0 or alp < p[0, 0]:
                if p[1, 1] < p[0, 1]:
                    return "WARNING: Interpolation error, code:-1, energy decreases, step further", 5.0 * p[1, 0]
                return "ERROR: Interpolation error, code:-1", alp
            return "FG", alp
        if g > 0:
            if p[1, 2] > 0.0:
                if p[1, 0] > alp:
                    p[1] = (alp, f, g)
                    alp = self._new_alp(p[0, 0], p[0, 2], p[1, 0], p[1, 2], stp_min, stp_max)
                    if alp < p[0, 0]:
                        return "WARNING: Order flips, code:0", (p[0, 0] + p[1, 0]) / 2.0
                    return "FG", alp
                if f < p[1, 1]:
                    return "WARNINIG: Order flipped, code:1", alp * 5.0
                return "WARNING: Order flipped, code:2", (p[0, 0] + p[1, 0]) / 2.0
            if p[1, 2] < 0.0:
                p[0] = p[1]
                p[1] = (alp, f, g)
                alp = self._new_alp(p[0, 0], p[0, 2], p[1, 0], p[1, 2], stp_min, stp_max)
                if alp < p[0, 0] or alp > p[1, 0]:
                    if p[0, 1] > p[1, 1]:
                        return "WARNING: Interpolation error, code:1, energy decreases", p[1, 0] * 5.0
                    return "WARNING: Interpolation error, code:1", (p[0, 0] + p[1, 0]) / 2.0
                return "FG", alp
        if g < 0.0:
            if p[1, 2] > 0.0:
                p[0] = (alp, f, g)
                alp = self._new_alp(p[0, 0], p[0, 2], p[1, 0], p[1, 2], stp_min, stp_max)
                if alp < p[0, 0] or alp > p[1, 0]:
                    if p[0, 1] > p[1, 1]:
                        return "WARNING: Interpolation, code:2, f decreases, step further", 5.0 * p[1, 0]
                    return "WARNING: Interpolation, code:4", (p[0, 0] + p[1, 0]) / 2.0
                return "FG", alp
            if p[1, 2] < 0.0:
                p[0] = p[1]
                p[1] = (alp, f, g)
                alp = self._new_alp(p[0, 0], p[0, 2], p[1, 0], p[1, 2], stp_min, stp_max)
                if alp < p[1, 0]:
                    if p[0, 1] > p[1, 1]:
                        return "WARNING: Interpolation error: code:3, f decrease", p[1, 0] * 5.0
                    return "ERROR: Interpolation error: code:3", alp
                return "FG", alp
        return task, alp


def min_distance(lattice: np.ndarray, frac: np.ndarray) -> float:
    """Shortest ion-ion distance over the cell and its 26 neighbour images
    (CheckNearestDistanceAtoms, Source/Neighbor.f90:45-400, for cells within
    one neighbour shell)."""
    cart = frac @ lattice.T
    best = np.inf
    n = len(frac)
    for t in itertools.product((-1, 0, 1), repeat=3):
        shift = lattice @ np.array(t, dtype=float)
        d = cart[None, :, :] + shift[None, None, :] - cart[:, None, :]
        r = np.sqrt((d * d).sum(axis=2))
        if t == (0, 0, 0):
            r = r + np.diag(np.full(n, np.inf))
        best = min(best, float(r.min()))
    return best


def hager_zhang(new_grad, old_grad, dir_old):
    y = -new_grad + old_grad
    dy = float((dir_old * y).sum())
    tmp1 = y - 2.0 * dir_old * float((y * y).sum()) / dy
    tmp2 = -new_grad / dy
    gam = float((tmp1 * tmp2).sum())
    return max(gam, -1.0 / (np.sqrt(float((dir_old ** 2).sum())) * min(0.01, np.sqrt(float((old_grad ** 2).sum())))))


def cg2(cell, n, opts: ntn.NtnOptions, max_steps=200, force_cutoff=FORCE_CUTOFF, nn_dist=2.0,
        alpha_=5.0 / 6.0, beta_=5.0 / 6.0, rho0=None):
    """Returns (final fractional coordinates, the total energy (Ha) of every
    density solve in order, final forces)."""
    from . import cellsetup as cs
    cell = dataclasses.replace(cell, frac=np.array(cell.frac, dtype=float))
    L = cell.lattice
    cart2frac = np.linalg.inv(L)
    rho = cs.uniform_density(cell, *n) if rho0 is None else rho0

    def solve(rho):
        r = ntn.NtnSolver(functional_for(cell, n, alpha_, beta_), opts).solve(rho)
        f, _, _ = ofo.total_forces(cell, r.rho)
        return r.rho, float(r.energy[0]), f

    rho, energy, forces = solve(rho)
    trace = [energy]
    alpha = 1.0
    restart = False
    old_grad = np.zeros_like(forces)
    dir_old = np.zeros_like(forces)
    step = 0
    while True:
        step += 1
        if step > max_steps:
            break
        if float(np.sqrt((forces ** 2).sum(axis=1)).max()) < force_cutoff:
            break
        old_cart = cell.frac @ L.T
        new_grad = forces
        if step == 1 or restart or step % 30 == 0:
            gam = 0.0
            restart = False
        else:
            gam = hager_zhang(new_grad, old_grad, dir_old)
        d = new_grad + gam * dir_old
        dir_old = d
        old_grad = new_grad
        grad_alp = -float((forces * d).sum())
        stp_min = 0.0
        if nn_dist > 0:
            stp_max = abs((min_distance(L, cell.frac) - nn_dist) / float(d.max()))
        else:
            stp_max = abs(1.0 / float(d.max()))
        alpha = min(alpha, stp_max)
        ls = LineSearch()
        task = "START"
        n_line = 0
        while True:
            task, alpha = ls.step(alpha, energy, grad_alp, task, FTOL, GTOL, stp_min, stp_max)
            if n_line >= 4 and abs(ls.points[0, 1] - ls.points[1, 1]) < 1e-6:
                break
            if ls.points[0, 0] > 0.0:
                b = (ls.points[0, 0] - ls.points[1, 0]) * d
                if float(np.sqrt((b * b).sum(axis=1)).max()) < 1e-5:
                    break
            if task.startswith("CONV"):
                break
            if task.startswith("ERROR"):
                restart = True
                alpha = 1.0
                break
            if task.startswith("FG") or task.startswith("WARN"):
                cell.frac = np.mod((old_cart + alpha * d) @ cart2frac.T, 1.0)
                rho, energy, forces = solve(rho)
                trace.append(energy)
                grad_alp = -float((forces * d).sum())
                if float(np.sqrt((forces ** 2).sum(axis=1)).max()) < force_cutoff:
                    break
                n_line += 1
    return cell.frac, trace, forces
