"""Moré-Thuente line search (MINPACK-2 dcsrch/dcstep), restated.

Follows Source/MathDCsrch.f and Source/MathDCstep.f as vendored by the
reference.  The state that the Fortran keeps in isave/dsave is an object here.
Test infrastructure only.
"""
from __future__ import annotations

import math

XTRAPL = 1.1
XTRAPU = 4.0
P5 = 0.5
P66 = 0.66


def dcstep(stx, fx, dx, sty, fy, dy, stp, fp, dp, brackt, stpmin, stpmax):
    """Safeguarded cubic/quadratic step (MathDCstep.f).  Returns the updated
    (stx, fx, dx, sty, fy, dy, stp, brackt)."""
    sgnd = dp * (dx / abs(dx))
    if fp > fx:
        theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp
        s = max(abs(theta), abs(dx), abs(dp))
        gamma = s * math.sqrt((theta / s) ** 2 - (dx / s) * (dp / s))
        if stp < stx:
            gamma = -gamma
        p = (gamma - dx) + theta
        q = ((gamma - dx) + gamma) + dp
        r = p / q
        stpc = stx + r * (stp - stx)
        stpq = stx + ((dx / ((fx - fp) / (stp - stx) + dx)) / 2.0) * (stp - stx)
        if abs(stpc - stx) < abs(stpq - stx):
            stpf = stpc
        else:
            stpf = stpc + (stpq - stpc) / 2.0
        brackt = True
    elif sgnd < 0.0:
        theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp
        s = max(abs(theta), abs(dx), abs(dp))
        gamma = s * math.sqrt((theta / s) ** 2 - (dx / s) * (dp / s))
        if stp > stx:
            gamma = -gamma
        p = (gamma - dp) + theta
        q = ((gamma - dp) + gamma) + dx
        r = p / q
        stpc = stp + r * (stx - stp)
        stpq = stp + (dp / (dp - dx)) * (stx - stp)
        stpf = stpc if abs(stpc - stp) > abs(stpq - stp) else stpq
        brackt = True
    elif abs(dp) < abs(dx):
        theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp
        s = max(abs(theta), abs(dx), abs(dp))
        gamma = s * math.sqrt(max(0.0, (theta / s) ** 2 - (dx / s) * (dp / s)))
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
            stpf = stpc if abs(stpc - stp) < abs(stpq - stp) else stpq
            if stp > stx:
                stpf = min(stp + P66 * (sty - stp), stpf)
            else:
                stpf = max(stp + P66 * (sty - stp), stpf)
        else:
            stpf = stpc if abs(stpc - stp) > abs(stpq - stp) else stpq
            stpf = min(stpmax, stpf)
            stpf = max(stpmin, stpf)
    else:
        if brackt:
            theta = 3.0 * (fp - fy) / (sty - stp) + dy + dp
            s = max(abs(theta), abs(dy), abs(dp))
            gamma = s * math.sqrt((theta / s) ** 2 - (dy / s) * (dp / s))
            if stp > sty:
                gamma = -gamma
            p = (gamma - dp) + theta
            q = ((gamma - dp) + gamma) + dy
            r = p / q
            stpc = stp + r * (sty - stp)
            stpf = stpc
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
    return stx, fx, dx, sty, fy, dy, stpf, brackt


class Dcsrch:
    """Reverse-communication Wolfe search (MathDCsrch.f).  Call ``step`` with
    task "START" first, then with the task it returned while it asks for "FG"."""

    def __init__(self, ftol, gtol, xtol, stpmin, stpmax):
        self.ftol, self.gtol, self.xtol = ftol, gtol, xtol
        self.stpmin, self.stpmax = stpmin, stpmax

    def step(self, stp, f, g, task):
        ftol, gtol, xtol, stpmin, stpmax = self.ftol, self.gtol, self.xtol, self.stpmin, self.stpmax
        if task.startswith("START"):
            if stp < stpmin:
                task = "ERROR: STP .LT. STPMIN"
            if stp > stpmax:
                task = "ERROR: STP .GT. STPMAX"
            if g >= 0.0:
                task = "ERROR: INITIAL G .GE. ZERO"
            if ftol < 0.0:
                task = "ERROR: FTOL .LT. ZERO"
            if gtol < 0.0:
                task = "ERROR: GTOL .LT. ZERO"
            if xtol < 0.0:
                task = "ERROR: XTOL .LT. ZERO"
            if stpmin < 0.0:
                task = "ERROR: STPMIN .LT. ZERO"
            if stpmax < stpmin:
                task = "ERROR: STPMAX .LT. STPMIN"
            if task.startswith("ERROR"):
                return stp, task
            self.brackt = False
            self.stage = 1
            self.finit = f
            self.ginit = g
            self.gtest = ftol * self.ginit
            self.width = stpmax - stpmin
            self.width1 = self.width / P5
            self.stx, self.fx, self.gx = 0.0, self.finit, self.ginit
            self.sty, self.fy, self.gy = 0.0, self.finit, self.ginit
            self.stmin = 0.0
            self.stmax = stp + XTRAPU * stp
            return stp, "FG"
        ftest = self.finit + stp * self.gtest
        if self.stage == 1 and f <= ftest and g >= 0.0:
            self.stage = 2
        if self.brackt and (stp <= self.stmin or stp >= self.stmax):
            task = "WARNING: ROUNDING ERRORS PREVENT PROGRESS"
        if self.brackt and self.stmax - self.stmin <= xtol * self.stmax:
            task = "WARNING: XTOL TEST SATISFIED"
        if stp == stpmax and f <= ftest and g <= self.gtest:
            task = "WARNING: STP = STPMAX"
        if stp == stpmin and (f > ftest or g >= self.gtest):
            task = "WARNING: STP = STPMIN"
        if f <= ftest and abs(g) <= gtol * (-self.ginit):
            task = "CONVERGENCE"
        if task.startswith("WARN") or task.startswith("CONV"):
            return stp, task
        if self.stage == 1 and f <= self.fx and f > ftest:
            fm = f - stp * self.gtest
            fxm = self.fx - self.stx * self.gtest
            fym = self.fy - self.sty * self.gtest
            gm = g - self.gtest
            gxm = self.gx - self.gtest
            gym = self.gy - self.gtest
            (self.stx, fxm, gxm, self.sty, fym, gym, stp, self.brackt) = dcstep(
                self.stx, fxm, gxm, self.sty, fym, gym, stp, fm, gm, self.brackt, self.stmin, self.stmax)
            self.fx = fxm + self.stx * self.gtest
            self.fy = fym + self.sty * self.gtest
            self.gx = gxm + self.gtest
            self.gy = gym + self.gtest
        else:
            (self.stx, self.fx, self.gx, self.sty, self.fy, self.gy, stp, self.brackt) = dcstep(
                self.stx, self.fx, self.gx, self.sty, self.fy, self.gy, stp, f, g, self.brackt,
                self.stmin, self.stmax)
        if self.brackt:
            if abs(self.sty - self.stx) >= P66 * self.width1:
                stp = self.stx + P5 * (self.sty - self.stx)
            self.width1 = self.width
            self.width = abs(self.sty - self.stx)
        if self.brackt:
            self.stmin = min(self.stx, self.sty)
            self.stmax = max(self.stx, self.sty)
        else:
            self.stmin = stp + XTRAPL * (stp - self.stx)
            self.stmax = stp + XTRAPU * (stp - self.stx)
        stp = max(stp, stpmin)
        stp = min(stp, stpmax)
        if (self.brackt and (stp <= self.stmin or stp >= self.stmax)) or \
                (self.brackt and self.stmax - self.stmin <= xtol * self.stmax):
            stp = self.stx
        return stp, "FG"
