"""Geometry relaxation of many independent cells on one engine: the
reference's ion optimisers (dispatched at Source/Optimizer.f90:247-260)
QuickMin (method 2), the old conjugate gradient (3, GradientCG), CG2 (4) and
BFGS (5), and its cell optimiser (SteepestDecent, CellRelax).

QuickMinOptimization (Source/IonOptQui.f90:33-368) runs a batch of cells in
lockstep: every
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

import concurrent.futures
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
    """Shortest ion-ion distance (bohr) over the cell and its 26 neighbour images
    (CheckNearestDistanceAtoms, Source/Neighbor.f90:45-400, for cells within one
    neighbour shell).  Candidates come from |a|^2 + |b|^2 - 2 a.b per image (one
    matrix product each); every pair within a relative 1e-9 of the smallest is
    then measured as |R_j + T - R_i|, so the result is that distance's value."""
    cart = np.asarray(frac, dtype=float) @ lattice.T
    n = len(cart)
    c2 = (cart * cart).sum(axis=1)
    cands = []
    best2 = np.inf
    for t in np.ndindex(3, 3, 3):
        shift = lattice @ (np.array(t, dtype=float) - 1.0)
        b = cart + shift
        r2 = c2[:, None] + (b * b).sum(axis=1)[None, :] - 2.0 * (cart @ b.T)
        if t == (1, 1, 1):
            r2[np.diag_indices(n)] = np.inf
        m = float(r2.min())
        cands.append((shift, r2, m))
        best2 = min(best2, m)
    lim = best2 + 1e-9 * abs(best2) + 1e-12
    best = np.inf
    for shift, r2, m in cands:
        if m > lim:
            continue
        for i, j in zip(*np.nonzero(r2 <= lim)):
            d = cart[j] + shift - cart[i]
            best = min(best, float(np.sqrt((d * d).sum())))
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


class _GeneratorRelax:
    """Relax ``cells`` (each gets one FP64 slot) with an optimiser written as a
    generator of geometries (cg2_moves, lbfgs_moves): every batched step
    solves the densities of all cells that asked for one together, warm-started
    from each cell's resident density, and sends each optimiser its energy
    and forces."""

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
                gen = self._moves(st, force_cutoff, max_steps, nn_dist)
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

    @staticmethod
    def _next(gen, sent):
        """The optimiser's next geometry, or (None, final coordinates) at its end."""
        try:
            return (next(gen) if sent is None else gen.send(sent)), None
        except StopIteration as stop:
            return None, stop.value

    def _apply(self, st, nxt):
        """Start the density solve of the cell's next geometry (or mark it done)."""
        frac, final = nxt
        if frac is None:
            st.done = True
            st.cell.frac = final
            return
        st.cell.frac = frac
        self.eng.hold_density(st.slot)
        self.eng.build_ion_potential(st.slot, frac, st.cell.species_of_ion, st.cell.species)
        _, st.f_ewald = self.eng.ewald(st.slot, st.cell.nion)
        self.eng.start_solve(st.slot, None, self.opts)

    def _advance(self, st, gen, sent):
        """Move the cell's optimiser to its next density request (or its end)."""
        self._apply(st, self._next(gen, sent))

    def step(self) -> int:
        """Solve every pending geometry together and advance each optimiser.  The
        optimisers' host work (independent per cell, mostly NumPy) runs on a
        thread pool; the engine calls that follow are made in cell order."""
        pending = [k for k, st in enumerate(self.states) if not st.done]
        if not pending:
            return 0
        self._finish([self.states[k] for k in pending])
        sent = []
        for k in pending:
            st = self.states[k]
            self.traces[k].append(float(st.energy[0]))
            sent.append((float(st.energy[0]), st.forces))
        if len(pending) > 1:
            with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, len(pending))) as ex:
                nxt = list(ex.map(self._next, [self.gens[k] for k in pending], sent))
        else:
            nxt = [self._next(self.gens[pending[0]], sent[0])]
        for k, n in zip(pending, nxt):
            self._apply(self.states[k], n)
        return len(pending)

    def run(self):
        while self.step():
            pass
        return self.states


class CG2(_GeneratorRelax):
    """The CG2 optimiser (ConjugateGradient, Source/IonOptCG2.f90) on batched density solves."""

    def _moves(self, st, force_cutoff, max_steps, nn_dist):
        return cg2_moves(st.cell.lattice, st.cell.frac, float(st.energy[0]), st.forces,
                         force_cutoff=force_cutoff, max_steps=max_steps, nn_dist=nn_dist)


# ---------------------------------------------------------------------------- BFGS
# IonLBFGS (Source/IonOptBFGS.f90:39-290) on Nocedal's limited-memory BFGS
# with the More-Thuente line search (LBFGS / MCSRCH / MCSTEP,
# Source/MathLBFGS.f): 5 corrections, the driver's own force test, at most
# 1000 energy and gradient evaluations.
LBFGS_M = 5                  # corrections kept (IonOptBFGS.f90: M)
LBFGS_EPS = 1.0e-5           # LBFGS's own gradient test (EPS)
LBFGS_XTOL = 1.0e-4          # line-search interval tolerance (XTOL)
LBFGS_FTOL = 1.0e-4          # sufficient decrease (set by LBFGS)
LBFGS_GTOL = 0.9             # curvature condition (the LB2 default)
LBFGS_STPMIN, LBFGS_STPMAX = 1.0e-20, 1.0e20
LBFGS_MAXFEV = 20            # evaluations per line search
LBFGS_MAX_CALLS = 1000       # IonOptBFGS.f90: nMax
MT_P66 = float(np.float32(0.66))  # a single-precision literal in MCSTEP


def mt_step(stx, fx, dx, sty, fy, dy, stp, fp, dp, brackt, stpmin, stpmax):
    """One safeguarded step of the More-Thuente interval search (MCSTEP):
    (stx, fx, dx, sty, fy, dy, stp, brackt, info)."""
    if ((brackt and (stp <= min(stx, sty) or stp >= max(stx, sty))) or dx * (stp - stx) >= 0.0
            or stpmax < stpmin):
        return stx, fx, dx, sty, fy, dy, stp, brackt, 0
    sgnd = dp * (dx / abs(dx))
    if fp > fx:
        info, bound = 1, True
        theta = 3 * (fx - fp) / (stp - stx) + dx + dp
        s = max(abs(theta), abs(dx), abs(dp))
        gamma = s * np.sqrt((theta / s) ** 2 - (dx / s) * (dp / s))
        if stp < stx:
            gamma = -gamma
        r = ((gamma - dx) + theta) / (((gamma - dx) + gamma) + dp)
        stpc = stx + r * (stp - stx)
        stpq = stx + ((dx / ((fx - fp) / (stp - stx) + dx)) / 2) * (stp - stx)
        stpf = stpc if abs(stpc - stx) < abs(stpq - stx) else stpc + (stpq - stpc) / 2
        brackt = True
    elif sgnd < 0.0:
        info, bound = 2, False
        theta = 3 * (fx - fp) / (stp - stx) + dx + dp
        s = max(abs(theta), abs(dx), abs(dp))
        gamma = s * np.sqrt((theta / s) ** 2 - (dx / s) * (dp / s))
        if stp > stx:
            gamma = -gamma
        r = ((gamma - dp) + theta) / (((gamma - dp) + gamma) + dx)
        stpc = stp + r * (stx - stp)
        stpq = stp + (dp / (dp - dx)) * (stx - stp)
        stpf = stpc if abs(stpc - stp) > abs(stpq - stp) else stpq
        brackt = True
    elif abs(dp) < abs(dx):
        info, bound = 3, True
        theta = 3 * (fx - fp) / (stp - stx) + dx + dp
        s = max(abs(theta), abs(dx), abs(dp))
        gamma = s * np.sqrt(max(0.0, (theta / s) ** 2 - (dx / s) * (dp / s)))
        if stp > stx:
            gamma = -gamma
        r = ((gamma - dp) + theta) / ((gamma + (dx - dp)) + gamma)
        if r < 0.0 and gamma != 0.0:
            stpc = stp + r * (stx - stp)
        else:
            stpc = stpmax if stp > stx else stpmin
        stpq = stp + (dp / (dp - dx)) * (stx - stp)
        if brackt:
            stpf = stpc if abs(stp - stpc) < abs(stp - stpq) else stpq
        else:
            stpf = stpc if abs(stp - stpc) > abs(stp - stpq) else stpq
    else:
        info, bound = 4, False
        if brackt:
            theta = 3 * (fp - fy) / (sty - stp) + dy + dp
            s = max(abs(theta), abs(dy), abs(dp))
            gamma = s * np.sqrt((theta / s) ** 2 - (dy / s) * (dp / s))
            if stp > sty:
                gamma = -gamma
            r = ((gamma - dp) + theta) / (((gamma - dp) + gamma) + dy)
            stpf = stp + r * (sty - stp)
        else:
            stpf = stpmax if stp > stx else stpmin
    if fp > fx:
        sty, fy, dy = stp, fp, dp
    else:
        if sgnd < 0.0:
            sty, fy, dy = stx, fx, dx
        stx, fx, dx = stp, fp, dp
    stp = max(stpmin, min(stpmax, stpf))
    if brackt and bound:
        if sty > stx:
            stp = min(stx + MT_P66 * (sty - stx), stp)
        else:
            stp = max(stx + MT_P66 * (sty - stx), stp)
    return stx, fx, dx, sty, fy, dy, stp, brackt, info


class MoreThuente:
    """The line search of MCSRCH along s from x: start() returns the first trial
    point (or None when s is not a descent direction), feed(f, g) the next
    trial point or, once done, None with .info set (1: converged)."""

    def __init__(self, ftol=LBFGS_FTOL, gtol=LBFGS_GTOL, xtol=LBFGS_XTOL, stpmin=LBFGS_STPMIN,
                 stpmax=LBFGS_STPMAX, maxfev=LBFGS_MAXFEV):
        self.ftol, self.gtol, self.xtol = ftol, gtol, xtol
        self.stpmin, self.stpmax, self.maxfev = stpmin, stpmax, maxfev
        self.info = 0

    def start(self, x, f, g, s, stp):
        self.s = s
        self.dginit = float(np.dot(g, s))
        if self.dginit >= 0.0:
            self.info = 0
            return None
        self.brackt, self.stage1, self.nfev, self.infoc = False, True, 0, 1
        self.finit, self.dgtest = f, self.ftol * self.dginit
        self.width = self.stpmax - self.stpmin
        self.width1 = self.width / 0.5
        self.wa = x.copy()
        self.stx, self.fx, self.dgx = 0.0, f, self.dginit
        self.sty, self.fy, self.dgy = 0.0, f, self.dginit
        self.stp = stp
        return self._trial()

    def _trial(self):
        if self.brackt:
            self.stmin, self.stmax = min(self.stx, self.sty), max(self.stx, self.sty)
        else:
            self.stmin, self.stmax = self.stx, self.stp + 4.0 * (self.stp - self.stx)
        self.stp = min(max(self.stp, self.stpmin), self.stpmax)
        if ((self.brackt and (self.stp <= self.stmin or self.stp >= self.stmax)) or self.nfev >= self.maxfev - 1
                or self.infoc == 0 or (self.brackt and self.stmax - self.stmin <= self.xtol * self.stmax)):
            self.stp = self.stx
        return self.wa + self.stp * self.s

    def feed(self, f, g):
        self.nfev += 1
        dg = float(np.dot(g, self.s))
        ftest1 = self.finit + self.stp * self.dgtest
        info = 0
        if (self.brackt and (self.stp <= self.stmin or self.stp >= self.stmax)) or self.infoc == 0:
            info = 6
        if self.stp == self.stpmax and f <= ftest1 and dg <= self.dgtest:
            info = 5
        if self.stp == self.stpmin and (f > ftest1 or dg >= self.dgtest):
            info = 4
        if self.nfev >= self.maxfev:
            info = 3
        if self.brackt and self.stmax - self.stmin <= self.xtol * self.stmax:
            info = 2
        if f <= ftest1 and abs(dg) <= self.gtol * (-self.dginit):
            info = 1
        if info:
            self.info = info
            return None
        if self.stage1 and f <= ftest1 and dg >= min(self.ftol, self.gtol) * self.dginit:
            self.stage1 = False
        if self.stage1 and f <= self.fx and f > ftest1:
            # the modified function psi(stp) = f - stp * dgtest while the step is in stage 1
            t = self.dgtest
            r = mt_step(self.stx, self.fx - self.stx * t, self.dgx - t, self.sty, self.fy - self.sty * t,
                        self.dgy - t, self.stp, f - self.stp * t, dg - t, self.brackt, self.stmin, self.stmax)
            self.stx, fxm, dgxm, self.sty, fym, dgym, self.stp, self.brackt, self.infoc = r
            self.fx, self.fy = fxm + self.stx * t, fym + self.sty * t
            self.dgx, self.dgy = dgxm + t, dgym + t
        else:
            r = mt_step(self.stx, self.fx, self.dgx, self.sty, self.fy, self.dgy, self.stp, f, dg, self.brackt,
                        self.stmin, self.stmax)
            self.stx, self.fx, self.dgx, self.sty, self.fy, self.dgy, self.stp, self.brackt, self.infoc = r
        if self.brackt:
            if abs(self.sty - self.stx) >= 0.66 * self.width1:
                self.stp = self.stx + 0.5 * (self.sty - self.stx)
            self.width1 = self.width
            self.width = abs(self.sty - self.stx)
        return self._trial()


class Lbfgs:
    """Limited-memory BFGS in LBFGS's reverse communication: call(x, f, g,
    iflag) returns the point to evaluate next and the flag (1: evaluate and
    call again, 0: converged by the gradient test, < 0: failed).  Calling
    with iflag 0 (re)starts it from x."""

    def __init__(self, m=LBFGS_M, eps=LBFGS_EPS):
        self.m, self.eps = m, eps

    def _start(self, x, g):
        n = len(x)
        self.s = np.zeros((self.m, n))
        self.y = np.zeros((self.m, n))
        self.rho = np.zeros(self.m)
        self.diag = np.ones(n)
        self.point, self.it = 0, 0
        self.s[0] = -g * self.diag
        self.stp1 = 1.0 / float(np.sqrt(np.dot(g, g)))

    def _iteration(self, x, f, g):
        """Label 80: the next search direction, then the line search's first trial."""
        self.it += 1
        bound = self.it - 1
        if self.it != 1:
            bound = min(bound, self.m)
            last = (self.point - 1) % self.m
            ys = float(np.dot(self.y[last], self.s[last]))
            yy = float(np.dot(self.y[last], self.y[last]))
            self.diag[:] = ys / yy
            self.rho[last] = 1.0 / ys
            q = -g
            alpha = np.zeros(self.m)
            cp = self.point
            for _ in range(bound):  # newest correction first
                cp = (cp - 1) % self.m
                alpha[cp] = self.rho[cp] * float(np.dot(self.s[cp], q))
                q = q - alpha[cp] * self.y[cp]
            q = self.diag * q
            for _ in range(bound):  # oldest first
                beta = self.rho[cp] * float(np.dot(self.y[cp], q))
                q = q + (alpha[cp] - beta) * self.s[cp]
                cp = (cp + 1) % self.m
            self.s[self.point] = q
        self.g_old = g.copy()
        self.ls = MoreThuente()
        xt = self.ls.start(x, f, g, self.s[self.point], self.stp1 if self.it == 1 else 1.0)
        if xt is None:
            return x, -1
        return xt, 1

    def call(self, x, f, g, iflag):
        if iflag == 0:
            self._start(x, g)
            return self._iteration(x, f, g)
        xt = self.ls.feed(f, g)
        if xt is not None:
            return xt, 1
        if self.ls.info != 1:
            return x, -1
        p = self.point
        self.s[p] = self.ls.stp * self.s[p]
        self.y[p] = g - self.g_old
        self.point = (p + 1) % self.m
        if float(np.sqrt(np.dot(g, g))) / max(1.0, float(np.sqrt(np.dot(x, x)))) <= self.eps:
            return x, 0
        return self._iteration(x, f, g)


def lbfgs_moves(lattice, frac, energy, forces, force_cutoff=FORCE_CUTOFF, max_calls=LBFGS_MAX_CALLS):
    """The BFGS optimiser (IonLBFGS) as a generator, like cg2_moves: it yields
    the fractional coordinates of every geometry whose density it needs and
    receives (total energy, forces) for it; its return value is the final
    coordinates.  The unknowns are the Cartesian coordinates, ion by ion
    within each direction (the reference's RESHAPE of cart(numIon, 3)), and
    the gradient is minus the forces."""
    cart2frac = np.linalg.inv(lattice)
    x = (np.asarray(frac) @ lattice.T).ravel(order="F")
    f, g = float(energy), -np.asarray(forces).ravel(order="F")
    lb = Lbfgs()
    iflag, calls = 0, 0
    while True:
        x, iflag = lb.call(x, f, g, iflag)
        frac = x.reshape((-1, 3), order="F") @ cart2frac.T
        energy, forces = yield frac
        f, g = float(energy), -np.asarray(forces).ravel(order="F")
        if _max_force(np.asarray(forces)) < force_cutoff or iflag < 0:
            return frac
        calls += 1
        if calls > max_calls:
            return frac


class BFGS(_GeneratorRelax):
    """The BFGS optimiser (IonLBFGS, Source/IonOptBFGS.f90:39-290) on batched
    density solves; max_steps bounds the energy and gradient evaluations."""

    def _moves(self, st, force_cutoff, max_steps, nn_dist):
        return lbfgs_moves(st.cell.lattice, st.cell.frac, float(st.energy[0]), st.forces,
                           force_cutoff=force_cutoff, max_calls=max_steps)


# ---------------------------------------------------------------- old CG
# GradientOptimization (Source/IonOptCON.f90:33-241, ion method 3): Polak-
# Ribiere-type directions (gamma clipped at 0) with the solver's More-Thuente
# search (Dcsrch with ftol 0.01, gtol 0.1, xtol 1e-10, steps in [1e-100, 1000]);
# the first step is 5, later first trials scale the last step by the ratio of
# directional derivatives within [1/4, 2]; a search whose energy changed by
# less than 1e-9 Ha per ion over its last 5 trials (after more than 10) is
# cut and the next direction restarts along the forces.
GRAD_FTOL, GRAD_GTOL, GRAD_XTOL = 0.01, 0.1, 1.0e-10
GRAD_STPMIN, GRAD_STPMAX = 1.0e-100, 1000.0


def gradient_moves(lib, lattice, frac, energy, forces, force_cutoff=FORCE_CUTOFF, max_steps=200):
    """GradientOptimization as a generator (like cg2_moves); ``lib`` supplies
    the line search.  The reference loops until the force test passes;
    max_steps bounds the outer steps."""
    cart2frac = np.linalg.inv(lattice)
    frac = np.array(frac, dtype=float)
    forces = np.asarray(forces, dtype=float)
    energy = float(energy)
    nion = len(frac)
    max_force = _max_force(forces)
    stp, fp = 0.0, 0.0
    g = dir_next = None
    checkpt1 = checkpt2 = 0.0
    step = 1
    while max_force >= force_cutoff and step <= max_steps:
        if step == 1:
            dir_next = forces.copy()
            fp = float(np.sum(-forces * dir_next))
            stp = 5.0
        else:
            gamma = max(float(np.sum(forces * (forces - g))) / float(np.sum(g * g)), 0.0)
            dir_next = forces + gamma * dir_next
            fp_last = fp
            fp = float(np.sum(-forces * dir_next))
            stp = max(min(stp * fp_last / fp, stp * 2.0), stp * 0.25)
        g = forces.copy()
        orig = frac.copy()
        n_line = 0
        ls = native.Dcsrch(lib, GRAD_FTOL, GRAD_GTOL, GRAD_XTOL, GRAD_STPMIN, GRAD_STPMAX)
        task = native.LS_START
        while True:
            stp, task = ls.step(stp, energy, float(np.sum(-forces * dir_next)), task)
            if task != native.LS_FG:
                break
            if n_line % 5 == 4:
                checkpt2, checkpt1 = checkpt1, energy
                if n_line > 10 and abs(checkpt2 - checkpt1) / nion < 1e-9:
                    stp = 1.0
                    g = forces.copy()  # the next gamma is 0
                    break
            frac = np.mod(orig + (stp * dir_next) @ cart2frac.T, 1.0)
            energy, forces = yield frac
            energy = float(energy)
            forces = np.asarray(forces, dtype=float)
            max_force = _max_force(forces)
            n_line += 1
        step += 1
    return frac


class GradientCG(_GeneratorRelax):
    """The old conjugate-gradient optimiser (GradientOptimization,
    Source/IonOptCON.f90:33-241) on batched density solves."""

    def _moves(self, st, force_cutoff, max_steps, nn_dist):
        return gradient_moves(self.eng.lib, st.cell.lattice, st.cell.frac, float(st.energy[0]), st.forces,
                              force_cutoff=force_cutoff, max_steps=max_steps)


# ---------------------------------------------------------------- cell optimiser
CELL_MAX_STEPS = 100   # Source/CellOptimizers.f90: maxCellStep
CELL_TOLS = 5.0e-7     # Source/CellOptimizers.f90: tols (Ha/bohr^3)


@dataclasses.dataclass
class CellState:
    cell: Cell
    slot: int
    dt: float = 10.0
    old_energy: float = 0.0
    energy: np.ndarray = None
    stress: np.ndarray = None
    steps: int = 0
    done: bool = False
    history: list = dataclasses.field(default_factory=list)


class CellRelax:
    """The reference's cell optimiser, SteepestDecent
    (Source/CellOptimizers.f90:107-304), for a batch of cells: each cell step
    solves the density at fixed fractional ion positions (ion method "non"),
    takes the device stress, and moves the lattice down the stress,
    L <- L - V dt sigma L^-T, with dt 10 at the start, x1.2 after a lower
    energy and /4 after a higher one; it stops when max |sigma| < tols
    (5e-7 Ha/bohr^3) or after max_steps.  axis 1-3 relaxes one diagonal
    component only.  A lattice move runs RefreshCellSetup and RescaleDensity
    on the device (ofdft_slot_set_lattice, the kinetic kernel, ion potential and
    Ewald rebuilt, ofdft_slot_rescale_input), and the next solve starts from
    the held density.  All cells' solves run together.  WT or second-order
    WGC cells (the kernel rebuilt at the new N/V; WTStress or WGCStress)."""

    def __init__(self, eng: native.Engine, cells, max_steps: int = CELL_MAX_STEPS, tols: float = CELL_TOLS,
                 axis: int = 0, opts=None):
        self.eng = eng
        self.opts = opts or native.ntn_options()
        self.max_steps, self.tols, self.axis = int(max_steps), float(tols), int(axis)
        self.states = []
        try:
            for c in cells:
                c = dataclasses.replace(c, frac=np.array(c.frac, dtype=float), lattice=np.array(c.lattice, float))
                self.states.append(CellState(cell=c, slot=pcell.setup_slot(eng, c, native.FP64)))
            for st in self.states:
                rho = np.full(st.cell.grid, st.cell.num_electrons / st.cell.vol)
                self.eng.start_solve(st.slot, np.asfortranarray(rho), self.opts)
        except Exception:
            self.close()
            raise

    def close(self):
        for st in self.states:
            self.eng.slot_destroy(st.slot)
        self.states = []

    def _move(self, st):
        """The cell step after a solve (SteepestDecent's loop body)."""
        c = st.cell
        stress = st.stress
        if self.axis in (1, 2, 3):
            a = self.axis - 1
            keep = stress[a, a]
            stress = np.zeros((3, 3))
            stress[a, a] = keep
            if abs(keep) < self.tols:
                st.done = True
                return
        elif float(np.abs(stress).max()) < self.tols:
            st.done = True
            return
        e = float(st.energy[0])
        st.dt = st.dt / 4.0 if e > st.old_energy else st.dt * 1.2
        st.old_energy = e
        new = c.lattice - c.vol * st.dt * (stress @ np.linalg.inv(c.lattice).T)
        if self.axis in (1, 2, 3):
            a = self.axis - 1
            keep = new[a, a]
            new = c.lattice.copy()
            new[a, a] = keep
        if st.steps >= self.max_steps:  # the reference moves the cell, then stops before its next solve
            c.lattice = new
            st.done = True
            return
        self.eng.hold_density(st.slot)
        c.lattice = new
        rho_avg = c.num_electrons / c.vol
        self.eng.set_lattice(st.slot, new, rho_avg, rho_avg)
        self.eng.rescale_input(st.slot, c.num_electrons)
        pcell.build_kernel(self.eng, st.slot, c)
        self.eng.build_ion_potential(st.slot, c.frac, c.species_of_ion, c.species)
        self.eng.ewald(st.slot, c.nion, want_forces=False)
        self.eng.start_solve(st.slot, None, self.opts)

    def step(self) -> int:
        """Finish the pending solves, take every cell's stress and move its lattice."""
        pending = [st for st in self.states if not st.done]
        if not pending:
            return 0
        while self.eng.run(8):
            pass
        for st in pending:
            _, st.energy, stats = self.eng.result(st.slot, want_rho=False)
            if stats["outcome"] != 0:
                raise native.OfdftError(7, "density solve did not converge (slot %d)" % st.slot)
            st.stress = self.eng.stress(st.slot)
            st.steps += 1
            st.history.append({"energy": float(st.energy[0]), "stress": st.stress.copy(),
                               "lattice": st.cell.lattice.copy()})
        for st in pending:
            self._move(st)
        return len(pending)

    def run(self):
        while self.step():
            pass
        return self.states
