// Moré-Thuente line search (MINPACK-2 dcsrch/dcstep) as a device/host state
// machine.  Restates Source/MathDCsrch.f and Source/MathDCstep.f of PROFESS:
// the Fortran isave/dsave arrays become the fields of LineSearch, and the task
// string becomes an integer code.  The optimiser calls ls_step with
// task = LS_START once and then with the previous task while it returns LS_FG.
#pragma once
#include "cx.cuh"

namespace ofdft {

enum LsTask : int { LS_START = 0, LS_FG = 1, LS_CONV = 2, LS_WARN = 3, LS_ERROR = 4 };

struct LineSearch {
  double ftol, gtol, xtol, stpmin, stpmax;
  int brackt, stage;
  double ginit, gtest, gx, gy, finit, fx, fy, stx, sty, stmin, stmax, width, width1;
};

HD double dmax(double a, double b) { return a > b ? a : b; }
HD double dmin(double a, double b) { return a < b ? a : b; }
HD double dabs(double a) { return a < 0 ? -a : a; }

// Safeguarded step (MathDCstep.f).
HDNI inline void dcstep(double& stx, double& fx, double& dx, double& sty, double& fy, double& dy,
                        double& stp, double fp, double dp, int& brackt, double stpmin, double stpmax) {
  const double sgnd = dp * (dx / dabs(dx));
  double stpf, stpc, stpq, theta, s, gamma, p, q, r;
  if (fp > fx) {
    theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
    s = dmax(dmax(dabs(theta), dabs(dx)), dabs(dp));
    gamma = s * sqrt((theta / s) * (theta / s) - (dx / s) * (dp / s));
    if (stp < stx) gamma = -gamma;
    p = (gamma - dx) + theta;
    q = ((gamma - dx) + gamma) + dp;
    r = p / q;
    stpc = stx + r * (stp - stx);
    stpq = stx + ((dx / ((fx - fp) / (stp - stx) + dx)) / 2.0) * (stp - stx);
    if (dabs(stpc - stx) < dabs(stpq - stx))
      stpf = stpc;
    else
      stpf = stpc + (stpq - stpc) / 2.0;
    brackt = 1;
  } else if (sgnd < 0.0) {
    theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
    s = dmax(dmax(dabs(theta), dabs(dx)), dabs(dp));
    gamma = s * sqrt((theta / s) * (theta / s) - (dx / s) * (dp / s));
    if (stp > stx) gamma = -gamma;
    p = (gamma - dp) + theta;
    q = ((gamma - dp) + gamma) + dx;
    r = p / q;
    stpc = stp + r * (stx - stp);
    stpq = stp + (dp / (dp - dx)) * (stx - stp);
    stpf = dabs(stpc - stp) > dabs(stpq - stp) ? stpc : stpq;
    brackt = 1;
  } else if (dabs(dp) < dabs(dx)) {
    theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
    s = dmax(dmax(dabs(theta), dabs(dx)), dabs(dp));
    gamma = s * sqrt(dmax(0.0, (theta / s) * (theta / s) - (dx / s) * (dp / s)));
    if (stp > stx) gamma = -gamma;
    p = (gamma - dp) + theta;
    q = (gamma + (dx - dp)) + gamma;
    r = p / q;
    if (r < 0.0 && gamma != 0.0)
      stpc = stp + r * (stx - stp);
    else if (stp > stx)
      stpc = stpmax;
    else
      stpc = stpmin;
    stpq = stp + (dp / (dp - dx)) * (stx - stp);
    if (brackt) {
      stpf = dabs(stpc - stp) < dabs(stpq - stp) ? stpc : stpq;
      if (stp > stx)
        stpf = dmin(stp + 0.66 * (sty - stp), stpf);
      else
        stpf = dmax(stp + 0.66 * (sty - stp), stpf);
    } else {
      stpf = dabs(stpc - stp) > dabs(stpq - stp) ? stpc : stpq;
      stpf = dmin(stpmax, stpf);
      stpf = dmax(stpmin, stpf);
    }
  } else {
    if (brackt) {
      theta = 3.0 * (fp - fy) / (sty - stp) + dy + dp;
      s = dmax(dmax(dabs(theta), dabs(dy)), dabs(dp));
      gamma = s * sqrt((theta / s) * (theta / s) - (dy / s) * (dp / s));
      if (stp > sty) gamma = -gamma;
      p = (gamma - dp) + theta;
      q = ((gamma - dp) + gamma) + dy;
      r = p / q;
      stpc = stp + r * (sty - stp);
      stpf = stpc;
    } else if (stp > stx) {
      stpf = stpmax;
    } else {
      stpf = stpmin;
    }
  }
  if (fp > fx) {
    sty = stp;
    fy = fp;
    dy = dp;
  } else {
    if (sgnd < 0.0) {
      sty = stx;
      fy = fx;
      dy = dx;
    }
    stx = stp;
    fx = fp;
    dx = dp;
  }
  stp = stpf;
}

// One call of the search (MathDCsrch.f).  Returns the new task; stp is updated.
HDNI inline int ls_step(LineSearch& L, double& stp, double f, double g, int task) {
  const double xtrapl = 1.1, xtrapu = 4.0, p5 = 0.5, p66 = 0.66;
  if (task == LS_START) {
    if (stp < L.stpmin || stp > L.stpmax || g >= 0.0 || L.ftol < 0.0 || L.gtol < 0.0 ||
        L.xtol < 0.0 || L.stpmin < 0.0 || L.stpmax < L.stpmin)
      return LS_ERROR;
    L.brackt = 0;
    L.stage = 1;
    L.finit = f;
    L.ginit = g;
    L.gtest = L.ftol * L.ginit;
    L.width = L.stpmax - L.stpmin;
    L.width1 = L.width / p5;
    L.stx = 0.0; L.fx = L.finit; L.gx = L.ginit;
    L.sty = 0.0; L.fy = L.finit; L.gy = L.ginit;
    L.stmin = 0.0;
    L.stmax = stp + xtrapu * stp;
    return LS_FG;
  }
  const double ftest = L.finit + stp * L.gtest;
  if (L.stage == 1 && f <= ftest && g >= 0.0) L.stage = 2;
  int out = LS_FG;
  if (L.brackt && (stp <= L.stmin || stp >= L.stmax)) out = LS_WARN;
  if (L.brackt && L.stmax - L.stmin <= L.xtol * L.stmax) out = LS_WARN;
  if (stp == L.stpmax && f <= ftest && g <= L.gtest) out = LS_WARN;
  if (stp == L.stpmin && (f > ftest || g >= L.gtest)) out = LS_WARN;
  if (f <= ftest && dabs(g) <= L.gtol * (-L.ginit)) out = LS_CONV;
  if (out != LS_FG) return out;
  if (L.stage == 1 && f <= L.fx && f > ftest) {
    double fm = f - stp * L.gtest;
    double fxm = L.fx - L.stx * L.gtest;
    double fym = L.fy - L.sty * L.gtest;
    double gm = g - L.gtest;
    double gxm = L.gx - L.gtest;
    double gym = L.gy - L.gtest;
    dcstep(L.stx, fxm, gxm, L.sty, fym, gym, stp, fm, gm, L.brackt, L.stmin, L.stmax);
    L.fx = fxm + L.stx * L.gtest;
    L.fy = fym + L.sty * L.gtest;
    L.gx = gxm + L.gtest;
    L.gy = gym + L.gtest;
  } else {
    dcstep(L.stx, L.fx, L.gx, L.sty, L.fy, L.gy, stp, f, g, L.brackt, L.stmin, L.stmax);
  }
  if (L.brackt) {
    if (dabs(L.sty - L.stx) >= p66 * L.width1) stp = L.stx + p5 * (L.sty - L.stx);
    L.width1 = L.width;
    L.width = dabs(L.sty - L.stx);
  }
  if (L.brackt) {
    L.stmin = dmin(L.stx, L.sty);
    L.stmax = dmax(L.stx, L.sty);
  } else {
    L.stmin = stp + xtrapl * (stp - L.stx);
    L.stmax = stp + xtrapu * (stp - L.stx);
  }
  stp = dmax(stp, L.stpmin);
  stp = dmin(stp, L.stpmax);
  if ((L.brackt && (stp <= L.stmin || stp >= L.stmax)) ||
      (L.brackt && L.stmax - L.stmin <= L.xtol * L.stmax))
    stp = L.stx;
  return LS_FG;
}

}  // namespace ofdft
