"""Test infrastructure (the oracle): a CPU restatement of the reference's BFGS
ion optimiser, IonLBFGS (Source/IonOptBFGS.f90:39-290), on Nocedal's
limited-memory BFGS with the More-Thuente line search (LBFGS, MCSRCH,
MCSTEP in Source/MathLBFGS.f), driven by the oracle's functional, NTN
solver and forces.  Only tests import it.

It keeps the reference's work-array layout: W(1:N) the gradient copy / two-
loop vector, W(N+1:N+M) the rho = 1/(y.s) values, W(N+M+1:N+2M) the alphas,
W(ISPT+1:) the M search steps and W(IYPT+1:) the M gradient differences
(1-based offsets ISPT = N + 2M, IYPT = ISPT + N M), with POINT the slot of
the next correction.  Parameters: M = 5, EPS = 1e-5, XTOL = 1e-4 (set by
IonLBFGS), FTOL = 1e-4 and MAXFEV = 20 (set by LBFGS), GTOL = 0.9,
STPMIN = 1e-20, STPMAX = 1e20 (the LB2 defaults), force tolerance 5e-5
Ha/bohr and at most 1000 evaluations (IonOptimizers, IonOptBFGS).  No BFGS
run ships with the reference, so this restatement is pinned only against
the engine's BFGS driver (parity unpinned to the reference itself).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import forces as ofo
from . import ntn
from .md import functional_for

FORCE_CUTOFF = float(np.float32(5e-5))
M, EPS, XTOL, FTOL, GTOL = 5, 1.0e-5, 1.0e-4, 1.0e-4, 0.9
STPMIN, STPMAX, MAXFEV, NMAX = 1.0e-20, 1.0e20, 20, 1000
P66_REAL = float(np.float32(0.66))   # MCSTEP's literal 0.66 (default REAL)


def _fsqrt(v):
    """Fortran's SQRT under IEEE arithmetic: NaN for a negative argument."""
    return math.sqrt(v) if v >= 0.0 else math.nan


def mcstep(stx, fx, dx, sty, fy, dy, stp, fp, dp, brackt, stpmin, stpmax):
    info = 0
    if (brackt and (stp <= min(stx, sty) or stp >= max(stx, sty))) or dx * (stp - stx) >= 0.0 or stpmax < stpmin:
        return stx, fx, dx, sty, fy, dy, stp, brackt, info
    sgnd = dp * (dx / abs(dx))
    if fp > fx:
        info, bound = 1, True
        theta = 3 * (fx - fp) / (stp - stx) + dx + dp
        s = max(abs(theta), abs(dx), abs(dp))
        gamma = s * _fsqrt((theta / s) ** 2 - (dx / s) * (dp / s))
        if stp < stx:
            gamma = -gamma
        p = (gamma - dx) + theta
        q = ((gamma - dx) + gamma) + dp
        stpc = stx + (p / q) * (stp - stx)
        stpq = stx + ((dx / ((fx - fp) / (stp - stx) + dx)) / 2) * (stp - stx)
        if abs(stpc - stx) < abs(stpq - stx):
            stpf = stpc
        else:
            stpf = stpc + (stpq - stpc) / 2
        brackt = True
    elif sgnd < 0.0:
        info, bound = 2, False
        theta = 3 * (fx - fp) / (stp - stx) + dx + dp
        s = max(abs(theta), abs(dx), abs(dp))
        gamma = s * _fsqrt((theta / s) ** 2 - (dx / s) * (dp / s))
        if stp > stx:
            gamma = -gamma
        p = (gamma - dp) + theta
        q = ((gamma - dp) + gamma) + dx
        stpc = stp + (p / q) * (stx - stp)
        stpq = stp + (dp / (dp - dx)) * (stx - stp)
        stpf = stpc if abs(stpc - stp) > abs(stpq - stp) else stpq
        brackt = True
    elif abs(dp) < abs(dx):
        info, bound = 3, True
        theta = 3 * (fx - fp) / (stp - stx) + dx + dp
        s = max(abs(theta), abs(dx), abs(dp))
        gamma = s * _fsqrt(max(0.0, (theta / s) ** 2 - (dx / s) * (dp / s)))
        if stp > stx:
            gamma = -gamma
        p = (gamma - dp) + theta
        q = (gamma + (dx - dp)) + gamma
        r = p / q
        if r < 0.0 and gamma != 0.0:
            stpc = stp + r * (stx - stp)
        elif stp > stx:
            stpc = stpmax
        else:
            stpc = stpmin
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
            gamma = s * _fsqrt((theta / s) ** 2 - (dy / s) * (dp / s))
            if stp > sty:
                gamma = -gamma
            p = (gamma - dp) + theta
            q = ((gamma - dp) + gamma) + dy
            stpf = stp + (p / q) * (sty - stp)
        elif stp > stx:
            stpf = stpmax
        else:
            stpf = stpmin
    if fp > fx:
        sty, fy, dy = stp, fp, dp
    else:
        if sgnd < 0.0:
            sty, fy, dy = stx, fx, dx
        stx, fx, dx = stp, fp, dp
    stpf = min(stpmax, stpf)
    stpf = max(stpmin, stpf)
    stp = stpf
    if brackt and bound:
        if sty > stx:
            stp = min(stx + P66_REAL * (sty - stx), stp)
        else:
            stp = max(stx + P66_REAL * (sty - stx), stp)
    return stx, fx, dx, sty, fy, dy, stp, brackt, info


class LbfgsRC:
    """LBFGS with MCSRCH in reverse communication, on the reference's work array.
    call(X, F, G, IFLAG) updates X in place and returns the new IFLAG."""

    def __init__(self, n):
        self.n = n
        self.w = np.zeros(n * (2 * M + 1) + 2 * M)
        self.diag = np.ones(n)
        self.ispt = n + 2 * M
        self.iypt = self.ispt + n * M
        self.ls = None

    # ------------------------------------------------------------------ MCSRCH
    def _mcsrch(self, x, f, g, s_off, info):
        n, w, L = self.n, self.w, self.ls
        s = w[s_off:s_off + n]
        if info != -1:
            L["infoc"] = 1
            dginit = float(np.dot(g, s))
            if dginit >= 0.0:
                return 0
            L.update(brackt=False, stage1=True, nfev=0, finit=f, dgtest=FTOL * dginit, width=STPMAX - STPMIN)
            L["width1"] = L["width"] / 0.5
            L["dginit"] = dginit
            self.diag[:] = x  # MCSRCH's WA is LBFGS's DIAG array
            L.update(stx=0.0, fx=f, dgx=dginit, sty=0.0, fy=f, dgy=dginit)
        else:
            L["nfev"] += 1
            dg = float(np.dot(g, s))
            ftest1 = L["finit"] + L["stp"] * L["dgtest"]
            info = 0
            if (L["brackt"] and (L["stp"] <= L["stmin"] or L["stp"] >= L["stmax"])) or L["infoc"] == 0:
                info = 6
            if L["stp"] == STPMAX and f <= ftest1 and dg <= L["dgtest"]:
                info = 5
            if L["stp"] == STPMIN and (f > ftest1 or dg >= L["dgtest"]):
                info = 4
            if L["nfev"] >= MAXFEV:
                info = 3
            if L["brackt"] and L["stmax"] - L["stmin"] <= XTOL * L["stmax"]:
                info = 2
            if f <= ftest1 and abs(dg) <= GTOL * (-L["dginit"]):
                info = 1
            if info != 0:
                return info
            if L["stage1"] and f <= ftest1 and dg >= min(FTOL, GTOL) * L["dginit"]:
                L["stage1"] = False
            if L["stage1"] and f <= L["fx"] and f > ftest1:
                t = L["dgtest"]
                fm, fxm, fym = f - L["stp"] * t, L["fx"] - L["stx"] * t, L["fy"] - L["sty"] * t
                dgm, dgxm, dgym = dg - t, L["dgx"] - t, L["dgy"] - t
                (L["stx"], fxm, dgxm, L["sty"], fym, dgym, L["stp"], L["brackt"], L["infoc"]) = mcstep(
                    L["stx"], fxm, dgxm, L["sty"], fym, dgym, L["stp"], fm, dgm, L["brackt"], L["stmin"],
                    L["stmax"])
                L["fx"], L["fy"] = fxm + L["stx"] * t, fym + L["sty"] * t
                L["dgx"], L["dgy"] = dgxm + t, dgym + t
            else:
                (L["stx"], L["fx"], L["dgx"], L["sty"], L["fy"], L["dgy"], L["stp"], L["brackt"], L["infoc"]) = \
                    mcstep(L["stx"], L["fx"], L["dgx"], L["sty"], L["fy"], L["dgy"], L["stp"], f, dg, L["brackt"],
                           L["stmin"], L["stmax"])
            if L["brackt"]:
                if abs(L["sty"] - L["stx"]) >= 0.66 * L["width1"]:
                    L["stp"] = L["stx"] + 0.5 * (L["sty"] - L["stx"])
                L["width1"] = L["width"]
                L["width"] = abs(L["sty"] - L["stx"])
        # label 30: the next trial step
        if L["brackt"]:
            L["stmin"], L["stmax"] = min(L["stx"], L["sty"]), max(L["stx"], L["sty"])
        else:
            L["stmin"], L["stmax"] = L["stx"], L["stp"] + 4.0 * (L["stp"] - L["stx"])
        L["stp"] = min(max(L["stp"], STPMIN), STPMAX)
        if ((L["brackt"] and (L["stp"] <= L["stmin"] or L["stp"] >= L["stmax"])) or L["nfev"] >= MAXFEV - 1
                or L["infoc"] == 0 or (L["brackt"] and L["stmax"] - L["stmin"] <= XTOL * L["stmax"])):
            L["stp"] = L["stx"]
        x[:] = self.diag + L["stp"] * s
        return -1

    # ------------------------------------------------------------------ LBFGS
    def _label80(self, x, f, g):
        n, w, S = self.n, self.w, self.st
        S["iter"] += 1
        bound = S["iter"] - 1
        if S["iter"] != 1:
            if S["iter"] > M:
                bound = M
            npt = S["npt"]
            ys = float(np.dot(w[self.iypt + npt:self.iypt + npt + n], w[self.ispt + npt:self.ispt + npt + n]))
            yy = float(np.dot(w[self.iypt + npt:self.iypt + npt + n], w[self.iypt + npt:self.iypt + npt + n]))
            self.diag[:] = ys / yy
            cp = S["point"] if S["point"] != 0 else M
            w[n + cp - 1] = 1.0 / ys
            w[0:n] = -g
            cp = S["point"]
            for _ in range(bound):
                cp -= 1
                if cp == -1:
                    cp = M - 1
                sq = float(np.dot(w[self.ispt + cp * n:self.ispt + cp * n + n], w[0:n]))
                inmc = n + M + cp
                w[inmc] = w[n + cp] * sq
                w[0:n] -= w[inmc] * w[self.iypt + cp * n:self.iypt + cp * n + n]
            w[0:n] *= self.diag
            for _ in range(bound):
                yr = float(np.dot(w[self.iypt + cp * n:self.iypt + cp * n + n], w[0:n]))
                beta = w[n + cp] * yr
                beta = w[n + M + cp] - beta
                w[0:n] += beta * w[self.ispt + cp * n:self.ispt + cp * n + n]
                cp += 1
                if cp == M:
                    cp = 0
            w[self.ispt + S["point"] * n:self.ispt + S["point"] * n + n] = w[0:n]
        self.ls = {"stp": 1.0 if S["iter"] != 1 else S["stp1"]}
        w[0:n] = g
        return self._search(x, f, g, 0)

    def _search(self, x, f, g, info):
        info = self._mcsrch(x, f, g, self.ispt + self.st["point"] * self.n, info)
        if info == -1:
            return 1
        if info != 1:
            return -1
        n, w, S = self.n, self.w, self.st
        npt = S["point"] * n
        S["npt"] = npt
        w[self.ispt + npt:self.ispt + npt + n] *= self.ls["stp"]
        w[self.iypt + npt:self.iypt + npt + n] = g - w[0:n]
        S["point"] += 1
        if S["point"] == M:
            S["point"] = 0
        gnorm = math.sqrt(float(np.dot(g, g)))
        xnorm = max(1.0, math.sqrt(float(np.dot(x, x))))
        if gnorm / xnorm <= EPS:
            return 0
        return self._label80(x, f, g)

    def call(self, x, f, g, iflag):
        n = self.n
        if iflag == 0:  # label 10
            self.diag[:] = 1.0
            self.st = {"iter": 0, "point": 0, "npt": 0}
            self.w[self.ispt:self.ispt + n] = -g * self.diag
            self.st["stp1"] = 1.0 / math.sqrt(float(np.dot(g, g)))
            return self._label80(x, f, g)
        return self._search(x, f, g, -1)


def bfgs(cell, n, opts: ntn.NtnOptions, force_cutoff=FORCE_CUTOFF, max_calls=NMAX, alpha_=5.0 / 6.0,
         beta_=5.0 / 6.0, rho0=None, kinetic=None, gamma=2.7):
    """IonLBFGS on the oracle: returns (final fractional coordinates, the total
    energy (Ha) of every density solve in order, final forces).  kinetic =
    KEDF_WGC relaxes with the second-order WGC functional."""
    from . import functional as fn
    kinetic = fn.KEDF_WT if kinetic is None else kinetic
    from . import cellsetup as cs
    cell = dataclasses.replace(cell, frac=np.array(cell.frac, dtype=float))
    L = cell.lattice
    cart2frac = np.linalg.inv(L)
    rho = cs.uniform_density(cell, *n) if rho0 is None else rho0

    def solve(rho):
        r = ntn.NtnSolver(functional_for(cell, n, alpha_, beta_, kinetic, gamma), opts).solve(rho)
        f, _, _ = ofo.total_forces(cell, r.rho)
        return r.rho, float(r.energy[0]), f

    rho, F, forces = solve(rho)
    trace = [F]
    cart = cell.frac @ L.T
    X = cart.ravel(order="F").copy()
    G = -forces.ravel(order="F")
    lb = LbfgsRC(len(X))
    iflag, icall = 0, 0
    while True:
        iflag = lb.call(X, F, G, iflag)
        cell.frac = X.reshape((-1, 3), order="F") @ cart2frac.T
        rho, F, forces = solve(rho)
        trace.append(F)
        G = -forces.ravel(order="F")
        if float(np.sqrt((forces ** 2).sum(axis=1)).max()) < force_cutoff:
            break
        if iflag < 0:
            break
        icall += 1
        if icall > max_calls:
            break
    return cell.frac, trace, forces
