"""QuickMin geometry relaxation of many independent cells on one engine.

This is the reference's QuickMin ion optimiser, QuickMinOptimization
(Source/IonOptQui.f90:33-368), run for a batch of cells in lockstep: every
batched step, each cell that is still relaxing takes its own QuickMin move, its ion
terms are refreshed on the device (B-spline ion potential, Ewald sum), and
the densities of all moved cells are re-solved together, warm-started from
each cell's resident density.  Forces then decide, per cell, whether the move
is kept (the time step doubles and the velocity is projected on the force) or
undone (the time step drops five-fold and the velocity is reset).

Defaults follow Source/IonOptimizers.f90:26-41: time step 0.4 a.u., force
tolerance 5e-5 Ha/bohr (a single-precision literal there, kept as such) and
at most 200 steps.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import cell as pcell
from . import native
from .workloads import Cell

FORCE_CUTOFF = float(np.float32(5e-5))  # Source/IonOptimizers.f90:29


@dataclasses.dataclass
class RelaxState:
    cell: Cell
    slot: int
    time_step: float
    vel: np.ndarray = None
    forces: np.ndarray = None
    prev_forces: np.ndarray = None
    last_frac: np.ndarray = None
    min_frac: np.ndarray = None
    f_ewald: np.ndarray = None
    energy: np.ndarray = None
    old_energy: float = 0.0
    max_force: float = 0.0
    initial_max_force: float = 0.0
    best_force: float = 0.0
    min_max_force: float = 0.0
    step: int = 1
    over_step: bool = False
    done: bool = False
    converged: bool = False
    num_solves: int = 0
    history: list = dataclasses.field(default_factory=list)


def _max_force(f: np.ndarray) -> float:
    return float(np.sqrt((f * f).sum(axis=1)).max())


class QuickMin:
    """Relax ``cells`` (each gets one FP64 slot) with QuickMin."""

    def __init__(self, eng: native.Engine, cells, time_step: float = 0.4, force_cutoff: float = FORCE_CUTOFF,
                 max_steps: int = 200, opts=None):
        self.eng = eng
        self.force_cutoff = float(force_cutoff)
        self.max_steps = int(max_steps)
        self.opts = opts or native.ntn_options(conv_check=native.CONV_POT, pot_tol=1.0e-6)
        self.states = []
        try:
            for c in cells:
                c = dataclasses.replace(c, frac=np.array(c.frac, dtype=float))
                s = pcell.setup_slot(eng, c, native.FP64)
                self.states.append(RelaxState(cell=c, slot=s, time_step=float(time_step),
                                              vel=np.zeros((c.nion, 3)), min_frac=c.frac.copy()))
            for st in self.states:
                self._refresh_ewald(st)
                rho = np.full(st.cell.grid, st.cell.num_electrons / st.cell.vol)
                self.eng.start_solve(st.slot, np.asfortranarray(rho), self.opts)
            self._finish(self.states)
            for st in self.states:
                st.old_energy = float(st.energy[0])
                st.max_force = st.best_force = st.min_max_force = _max_force(st.forces)
                st.initial_max_force = st.max_force
        except Exception:
            self.close()
            raise

    def close(self):
        for st in self.states:
            self.eng.slot_destroy(st.slot)
        self.states = []

    def _refresh_ewald(self, st: RelaxState):
        _, st.f_ewald = self.eng.ewald(st.slot, st.cell.nion)

    def _finish(self, states):
        while self.eng.run(8):
            pass
        for st in states:
            _, st.energy, stats = self.eng.result(st.slot, want_rho=False)
            if stats["outcome"] != 0:
                raise native.OfdftError(7, "density solve did not converge (slot %d)" % st.slot)
            st.forces = self.eng.forces(st.slot, st.cell.nion, include_ewald=False) + st.f_ewald
            st.num_solves += 1

    def step(self) -> int:
        """One QuickMin step of every cell still relaxing; returns how many moved."""
        moved = []
        for st in self.states:
            if st.done:
                continue
            st.step += 1
            if st.step > self.max_steps or st.max_force < self.force_cutoff:
                st.done = True
                st.converged = st.max_force < self.force_cutoff
                continue
            if st.step % 10 == 9:
                if st.max_force > st.min_max_force * 3.0:
                    st.time_step *= 0.5
                else:
                    st.min_max_force = st.max_force
            c = st.cell
            dt = st.time_step
            frac_step = (dt * st.vel + 0.5 * dt * dt * st.forces) @ np.linalg.inv(c.lattice).T
            st.last_frac = c.frac.copy()
            c.frac = np.mod(c.frac + frac_step, 1.0)
            st.prev_forces = st.forces
            self.eng.hold_density(st.slot)
            self.eng.build_ion_potential(st.slot, c.frac, c.species_of_ion, c.species)
            self._refresh_ewald(st)
            self.eng.start_solve(st.slot, None, self.opts)
            moved.append(st)
        if not moved:
            return 0
        self._finish(moved)
        for st in moved:
            test_energy = float(st.energy[0])
            st.max_force = _max_force(st.forces)
            if st.max_force < st.best_force:
                st.min_frac = st.cell.frac.copy()
                st.best_force = st.max_force
            fv = float((st.forces * st.vel).sum())
            if fv < 0.0 or test_energy > st.old_energy:
                if st.step == 1 or test_energy > st.old_energy:
                    # undo the move (the density stays that of the undone geometry)
                    st.over_step = True
                    st.time_step /= 5.0
                    st.vel = np.zeros_like(st.vel)
                    st.forces = st.prev_forces
                    st.cell.frac = st.last_frac
                else:
                    st.over_step = False
                    st.old_energy = test_energy
                    st.vel = np.zeros_like(st.vel)
            else:
                st.time_step *= 2.0
                st.old_energy = test_energy
                st.over_step = False
                f = st.forces
                st.vel = fv * f / float((f * f).sum()) + f * st.time_step
            st.history.append({"step": st.step, "energy": test_energy, "max_force": st.max_force,
                               "time_step": st.time_step, "undone": st.over_step})
        return len(moved)

    def run(self):
        while self.step():
            pass
        return self.states


# ---------------------------------------------------------------------------- CG2
FTOL = float(np.float32(1e-4))   # Source/IonOptCG2.f90 (single-precision literals)
GTOL = float(np.float32(1e-1))


class IonLineSearch:
    """LnSrch (Source/MathLNsrch.f90:32-293): secant steps on dE/dalpha between a
    left and a right point (columns alpha, E, dE/dalpha), with the reference's
    task strings and its widening / halving fall-backs."""

    def __init__(self):
        self.points = np.full((2, 3), -1.0)
        self.f0 = 0.0
        self.g0 = 0.0

    @staticmethod
    def _secant(x1, y1, x2, y2, stp_min, stp_max):
        slope = (y1 - y2) / (x1 - x2)
        a = -(y1 - x1 * slope) / slope
        return -1.0 if (a >= stp_max or a <= stp_min) else a

    def step(self, alp, f, g, task, stp_min, stp_max):
        p = self.points
        sec = lambda: self._secant(p[0, 0], p[0, 2], p[1, 0], p[1, 2], stp_min, stp_max)
        if task.startswith("START"):
            if g > 0.0:
                return "ERROR: Initial G>0", alp
            p[:] = -1.0
            p[0] = (0.0, f, g)
            self.f0, self.g0 = f, g
            return "FG", alp
        if task.startswith("FG") and p[1, 0] > 0.0:
            if f <= self.f0 + FTOL * alp * self.g0 and abs(g) <= GTOL * abs(self.g0):
                return "CONV", alp
        if p[1, 0] < 0.0:  # no right point yet
            if g < p[0, 2]:
                return "WARNING: Need a better second point.", (alp * 5.0 if f < p[0, 1] else (p[0, 0] + alp) / 2.0)
            p[1] = (alp, f, g)
            alp = sec()
            if alp < 0.0 or alp < p[0, 0]:
                if p[1, 1] < p[0, 1]:
                    return "WARNING: Interpolation error, code:-1", 5.0 * p[1, 0]
                return "ERROR: Interpolation error, code:-1", alp
            return "FG", alp
        if g > 0:
            if p[1, 2] > 0.0:
                if p[1, 0] > alp:
                    p[1] = (alp, f, g)
                    alp = sec()
                    if alp < p[0, 0]:
                        return "WARNING: Order flips, code:0", (p[0, 0] + p[1, 0]) / 2.0
                    return "FG", alp
                if f < p[1, 1]:
                    return "WARNING: Order flipped, code:1", alp * 5.0
                return "WARNING: Order flipped, code:2", (p[0, 0] + p[1, 0]) / 2.0
            if p[1, 2] < 0.0:
                p[0] = p[1]
                p[1] = (alp, f, g)
                alp = sec()
                if alp < p[0, 0] or alp > p[1, 0]:
                    if p[0, 1] > p[1, 1]:
                        return "WARNING: Interpolation error, code:1", p[1, 0] * 5.0
                    return "WARNING: Interpolation error, code:1", (p[0, 0] + p[1, 0]) / 2.0
                return "FG", alp
        if g < 0.0:
            if p[1, 2] > 0.0:
                p[0] = (alp, f, g)
                alp = sec()
                if alp < p[0, 0] or alp > p[1, 0]:
                    if p[0, 1] > p[1, 1]:
                        return "WARNING: Interpolation, code:2", 5.0 * p[1, 0]
                    return "WARNING: Interpolation, code:4", (p[0, 0] + p[1, 0]) / 2.0
                return "FG", alp
            if p[1, 2] < 0.0:
                p[0] = p[1]
                p[1] = (alp, f, g)
                alp = sec()
                if alp < p[1, 0]:
                    if p[0, 1] > p[1, 1]:
                        return "WARNING: Interpolation error: code:3", p[1, 0] * 5.0
                    return "ERROR: Interpolation error: code:3", alp
                return "FG", alp
        return task, alp


def nearest_distance(lattice: np.ndarray, frac: np.ndarray) -> float:
    """Shortest ion-ion distance (bohr) over the cell and its 26 neighbour images."""
    cart = frac @ lattice.T
    n = len(frac)
    best = np.inf
    for t in np.ndindex(3, 3, 3):
        shift = lattice @ (np.array(t, dtype=float) - 1.0)
        d = cart[None, :, :] + shift[None, None, :] - cart[:, None, :]
        r = np.sqrt((d * d).sum(axis=2))
        if t == (1, 1, 1):
            r = r + np.diag(np.full(n, np.inf))
        best = min(best, float(r.min()))
    return best


def cg2_moves(lattice, frac, energy, forces, force_cutoff=FORCE_CUTOFF, max_steps=200, nn_dist=2.0):
    """The CG2 optimiser (ConjugateGradient, Source/IonOptCG2.f90:226-460) as a
    generator: it yields the fractional coordinates of every geometry whose
    density it needs and receives (total energy, forces) for it.  Hager-Zhang
    updates (cg_type = 2), restarts at step 1, every 30 steps and after a
    line-search error; the step bound comes from the nearest-neighbour
    distance (nnDist = 2 bohr).  Its return value is the final coordinates."""
    cart2frac = np.linalg.inv(lattice)
    alpha, restart = 1.0, False
    old_grad = np.zeros_like(forces)
    dir_old = np.zeros_like(forces)
    step = 0
    while True:
        step += 1
        if step > max_steps or float(np.sqrt((forces ** 2).sum(axis=1)).max()) < force_cutoff:
            return frac
        old_cart = frac @ lattice.T
        if step == 1 or restart or step % 30 == 0:
            gam, restart = 0.0, False
        else:
            y = old_grad - forces
            dy = float((dir_old * y).sum())
            gam = float(((y - 2.0 * dir_old * float((y * y).sum()) / dy) * (-forces / dy)).sum())
            gam = max(gam, -1.0 / (np.sqrt(float((dir_old ** 2).sum())) * min(0.01, np.sqrt(float((old_grad ** 2).sum())))))
        d = forces + gam * dir_old
        dir_old, old_grad = d, forces
        g = -float((forces * d).sum())
        stp_max = abs(((nearest_distance(lattice, frac) - nn_dist) if nn_dist > 0 else 1.0) / float(d.max()))
        alpha = min(alpha, stp_max)
        ls = IonLineSearch()
        task, n_line = "START", 0
        while True:
            task, alpha = ls.step(alpha, energy, g, task, 0.0, stp_max)
            if n_line >= 4 and abs(ls.points[0, 1] - ls.points[1, 1]) < 1e-6:
                break
            if ls.points[0, 0] > 0.0:
                b = (ls.points[0, 0] - ls.points[1, 0]) * d
                if float(np.sqrt((b * b).sum(axis=1)).max()) < 1e-5:
                    break
            if task.startswith("CONV"):
                break
            if task.startswith("ERROR"):
                restart, alpha = True, 1.0
                break
            if task.startswith("FG") or task.startswith("WARN"):
                frac = np.mod((old_cart + alpha * d) @ cart2frac.T, 1.0)
                energy, forces = yield frac
                g = -float((forces * d).sum())
                if float(np.sqrt((forces ** 2).sum(axis=1)).max()) < force_cutoff:
                    break
                n_line += 1


class CG2:
    """Relax ``cells`` (each gets one FP64 slot) with the CG2 optimiser; every
    batched step solves the densities of all cells that asked for one together."""

    def __init__(self, eng: native.Engine, cells, max_steps: int = 200, force_cutoff: float = FORCE_CUTOFF,
                 opts=None, nn_dist: float = 2.0):
        self.eng = eng
        self.opts = opts or native.ntn_options()
        self.states = []
        self.traces = []
        try:
            for c in cells:
                c = dataclasses.replace(c, frac=np.array(c.frac, dtype=float))
                self.states.append(RelaxState(cell=c, slot=pcell.setup_slot(eng, c, native.FP64), time_step=0.0))
            for st in self.states:
                _, st.f_ewald = self.eng.ewald(st.slot, st.cell.nion)
                rho = np.full(st.cell.grid, st.cell.num_electrons / st.cell.vol)
                self.eng.start_solve(st.slot, np.asfortranarray(rho), self.opts)
            self._finish(self.states)
            self.gens = []
            for st in self.states:
                self.traces.append([float(st.energy[0])])
                gen = cg2_moves(st.cell.lattice, st.cell.frac, float(st.energy[0]), st.forces,
                                force_cutoff=force_cutoff, max_steps=max_steps, nn_dist=nn_dist)
                self.gens.append(gen)
                self._advance(st, gen, None)
        except Exception:
            self.close()
            raise

    def close(self):
        for st in self.states:
            self.eng.slot_destroy(st.slot)
        self.states = []

    def _finish(self, states):
        while self.eng.run(8):
            pass
        for st in states:
            _, st.energy, stats = self.eng.result(st.slot, want_rho=False)
            if stats["outcome"] != 0:
                raise native.OfdftError(7, "density solve did not converge (slot %d)" % st.slot)
            st.forces = self.eng.forces(st.slot, st.cell.nion, include_ewald=False) + st.f_ewald
            st.num_solves += 1

    def _advance(self, st, gen, sent):
        """Move the cell's optimiser to its next density request (or its end)."""
        try:
            frac = next(gen) if sent is None else gen.send(sent)
        except StopIteration as stop:
            st.done = True
            st.cell.frac = stop.value
            return
        st.cell.frac = frac
        self.eng.hold_density(st.slot)
        self.eng.build_ion_potential(st.slot, frac, st.cell.species_of_ion, st.cell.species)
        _, st.f_ewald = self.eng.ewald(st.slot, st.cell.nion)
        self.eng.start_solve(st.slot, None, self.opts)

    def step(self) -> int:
        """Solve every pending geometry together and advance each optimiser."""
        pending = [k for k, st in enumerate(self.states) if not st.done]
        if not pending:
            return 0
        self._finish([self.states[k] for k in pending])
        for k in pending:
            st = self.states[k]
            self.traces[k].append(float(st.energy[0]))
            self._advance(st, self.gens[k], (float(st.energy[0]), st.forces))
        return len(pending)

    def run(self):
        while self.step():
            pass
        return self.states
