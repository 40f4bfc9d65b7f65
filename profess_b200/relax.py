"""QuickMin geometry relaxation of many independent cells on one engine.

This is the reference's QuickMin ion optimiser, QuickMinOptimization
(Source/IonOptQui.f90:33-368), run for a batch of cells in lockstep: every
round, each cell that is still relaxing takes its own QuickMin move, its ion
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

    def round(self) -> int:
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
        while self.round():
            pass
        return self.states
