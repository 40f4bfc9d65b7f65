"""Electron-number-conserving truncated-Newton density optimiser (NTN), restated.

Follows ``ProjNormRhoMinimization``/``DensityOptimization``/``CheckExit``
(Source/RhoOptN.f90:60-977), ``NewtonDirection`` (Source/RhoDirNew.f90:25-210),
``getNextGradient``/``gradOftheta``/``checkGradient``/``LineSearchTN``
(Source/RhoLineSearch.f90:40-444), ``ChemicalPotential``
(Source/RhoDirBFGS.f90:294-343) and ``InnerProd`` (Source/RhoDirCG.f90:109-142),
spin-unpolarised.  Test infrastructure only.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .consts import MACH_PREC
from .functional import Functional, calculate_potential_plus
from .linesearch import Dcsrch


@dataclasses.dataclass
class NtnOptions:
    max_iter: int = 500        # RhoOptimizers.f90:49
    pot_tol: float = 1.0e-5    # RhoOptimizers.f90:55
    tole: float = 1.0e-6       # RhoOptimizers.f90:56 (Ha)
    conv_check: str = "ENE"    # RhoOptimizers.f90:88
    max_line: int = 200        # RhoLineSearch.f90:34
    ftol: float = 1.0e-4       # RhoOptN.f90:255-258
    gtol: float = 0.2
    xtol: float = 1.0e-12      # RhoOptN.f90:193


@dataclasses.dataclass
class NtnResult:
    rho: np.ndarray
    energy: np.ndarray
    outcome: int               # rhoOutcome: 0 converged, 1 failed / max iterations
    iterations: int
    num_evals: int
    history: list              # per outer iteration: dict(energy, pot_norm, ncg, nline, theta)
    pot_norm: float


def _sign(x: np.ndarray) -> np.ndarray:
    """Fortran SIGN(1._DP, x): +1 for x >= 0, -1 for x < 0."""
    return np.where(x < 0.0, -1.0, 1.0)


class NtnSolver:
    def __init__(self, func: Functional, opts: NtnOptions | None = None, eval_hook=None):
        self.f = func
        self.o = opts or NtnOptions()
        self.num_evals = 0
        self.eval_hook = eval_hook

    # -- helpers ---------------------------------------------------------
    def _eval(self, phi: np.ndarray, want_energy: bool):
        self.num_evals += 1
        pot, et = calculate_potential_plus(self.f, phi * phi, True, want_energy)
        if self.eval_hook is not None:
            self.eval_hook(phi, pot, et)
        return pot, et

    def _inner(self, a, b):
        return float(np.sum(a * b)) * self.f.dv

    def _chem_pot(self, dedphi, phi, tot_ele):
        return self.f.dv * float(np.sum(dedphi * phi)) / (2.0 * tot_ele)

    # -- NewtonDirection (RhoDirNew.f90:25-210) --------------------------
    def newton_direction(self, phi, b, mu0):
        flag = -1
        ry = 0.0
        direction = np.zeros_like(phi)
        r = -b
        rr = float(np.sum(r ** 2))
        criteria = rr
        it = 1
        p = None
        while True:
            y = r
            ry_last = ry
            ry = float(np.sum(r * y))
            p = y.copy() if it == 1 else y + ry / ry_last * p
            s1 = float(np.sum(phi ** 2))
            s2 = float(np.sum(p ** 2))
            eps = 2.0 * math.sqrt(MACH_PREC) * (1.0 + math.sqrt(s1)) / math.sqrt(s2)
            new_phi = phi + eps * p
            ap, _ = self._eval(new_phi, False)
            ap = ap * _sign(new_phi)
            ap = ap - mu0 * 2.0 * new_phi
            ap = (ap - b) / eps
            pap = float(np.sum(p * ap))
            if pap < 0.0:
                if it == 1:
                    direction = -(direction - ry / pap * p)
                flag = -2
                break
            alpha = ry / pap
            direction = direction + alpha * p
            r = r - alpha * ap
            rr_last = rr
            rr = float(np.sum(r ** 2))
            if rr < 0.1 * criteria:
                flag = 0
                break
            if it > 50:
                flag = 1
                break
            if abs(rr - rr_last) / rr < 0.01 and it > 9:
                flag = 2
                break
            it += 1
        return direction, it, flag

    # -- getNextGradient (RhoLineSearch.f90:40-139), numSpin = 1 ----------
    def next_gradient(self, tot_ele, phi, dedphi, theta, direction):
        norm_phi_dir = math.sqrt(self._inner(phi + direction, phi + direction))
        direction = direction - phi * self._inner(phi, direction) / tot_ele
        norm_perp = math.sqrt(self._inner(direction, direction))
        theta = min(theta, norm_perp / norm_phi_dir)
        direction = direction * math.sqrt(tot_ele) / norm_perp
        gradth = self.f.dv * float(np.sum(dedphi * direction))   # gradOftheta at theta = 0
        return theta, gradth, direction

    # -- ProjNormRhoMinimization (RhoOptN.f90:60-545) ---------------------
    def solve(self, rho_in: np.ndarray) -> NtnResult:
        o = self.o
        n_points = float(rho_in.size)
        tot_ele = float(np.sum(rho_in)) * self.f.dv
        theta = 0.2
        phi = np.sqrt(np.abs(rho_in))
        dedphi, energy = self._eval(phi, True)
        dedphi = dedphi * _sign(phi)
        mu0 = self._chem_pot(dedphi, phi, tot_ele)
        dldphi = dedphi - mu0 * 2.0 * phi
        pot_norm = math.sqrt(float(np.sum(dldphi ** 2)) / n_points)
        e = [energy[0], 0.0, 0.0]
        history = [dict(energy=energy[0], pot_norm=pot_norm, ncg=0, nline=0, theta=0.0)]
        outcome = -1
        it = 1
        temp_phi = phi
        while True:
            switch_stp = False
            direction, newton_iter, _ = self.newton_direction(phi, dldphi, mu0)
            while True:
                theta, gradth, direction = self.next_gradient(tot_ele, phi, dedphi, theta, direction)
                # checkGradient (RhoLineSearch.f90:201-309)
                if gradth > 1.0e5:
                    raise RuntimeError("The gradient is too large, the value is %r" % gradth)
                if gradth >= 0.0:
                    if switch_stp:
                        outcome = 1
                        break
                    switch_stp = True
                    direction = -dldphi
                    continue
                break
            if outcome == 1:
                break
            # LineSearchTN (RhoLineSearch.f90:312-444)
            ls = Dcsrch(o.ftol, o.gtol, o.xtol, 0.0, math.pi)
            task = "START"
            nline = 0
            while True:
                theta, task = ls.step(theta, energy[0], gradth, task)
                if task.startswith("CONV") or task.startswith("ERROR") or task.startswith("WARN"):
                    break
                if task.startswith("FG"):
                    temp_phi = phi * math.cos(theta) + direction * math.sin(theta)
                    dedphi, energy = self._eval(temp_phi, True)
                    dedphi = dedphi * _sign(temp_phi)
                    gradth = self.f.dv * float(np.sum(
                        dedphi * (-phi * math.sin(theta) + direction * math.cos(theta))))
                    nline += 1
                    if nline > o.max_line:
                        break
            # StepInformation (RhoOptN.f90:692-758): potNorm with the old mu0
            pot_norm = math.sqrt(float(np.sum((dedphi - 2.0 * temp_phi * mu0) ** 2)) / n_points)
            history.append(dict(energy=energy[0], pot_norm=pot_norm, ncg=newton_iter,
                                nline=nline, theta=theta))
            # CheckExit (RhoOptN.f90:853-977)
            exit_flag = False
            e[2], e[1], e[0] = e[1], e[0], energy[0]
            p_conv = pot_norm < o.pot_tol
            e_conv = it >= 3 and abs(e[0] - e[1]) < o.tole and abs(e[0] - e[2]) < o.tole
            cc = o.conv_check.upper()
            if cc.startswith("ENE") and e_conv:
                outcome, exit_flag = 0, True
            if cc.startswith("POT") and p_conv:
                outcome, exit_flag = 0, True
            if cc.startswith("BOTH") and (p_conv or e_conv):
                outcome, exit_flag = 0, True
            if outcome == 1:
                exit_flag = True
            if it >= o.max_iter:
                outcome, exit_flag = 1, True
            phi = temp_phi
            mu0 = self._chem_pot(dedphi, phi, tot_ele)
            dldphi = dedphi - 2.0 * mu0 * phi
            if exit_flag:
                break
            it += 1
        return NtnResult(rho=phi ** 2, energy=energy, outcome=outcome, iterations=it,
                         num_evals=self.num_evals, history=history, pot_norm=pot_norm)
