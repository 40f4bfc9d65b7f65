// The NTN optimiser as a per-slot state machine.
//
// Restates ProjNormRhoMinimization / DensityOptimization / CheckExit
// (Source/RhoOptN.f90:60-977), NewtonDirection (Source/RhoDirNew.f90:25-210),
// getNextGradient / checkGradient / LineSearchTN (Source/RhoLineSearch.f90:40-444)
// and ChemicalPotential (Source/RhoDirBFGS.f90:294-343) for one spin channel.
// The reference's grid loops become device vector ops (VecOp) and potential
// evaluations (EvalMode); this function runs after each of them on one thread
// (the last block to finish a slot's work), reads the slot's reduced sums and
// chooses the next op or evaluation.  Sums arrive un-weighted; dV weighting is
// applied here exactly where InnerProd / gradOftheta / ChemicalPotential do.
#pragma once
#include "slot.cuh"

namespace ofdft {

HD bool bad(double v) { return !(v == v) || v > 1.0e300 || v < -1.0e300; }

// The slot quantities the state machine reads, loaded once before it runs.
struct CtlSlot {
  double dv, ion_ion;
  long long N;
  HistEntry* hist;
};
HD CtlSlot ctl_slot(const SlotDev& s) { return CtlSlot{s.dv, s.ion_ion, s.N, s.hist}; }

HDNI inline void ctl_finish(Ctl& c, int status, int err) {
  c.status = status;
  c.error = err;
  c.op = OP_NONE;
  c.ev = EV_NONE;
}

HDNI inline void ctl_push_hist(Ctl& c, const CtlSlot& s, int ncg, int nline) {
  if (c.hist_n < HIST_MAX && s.hist != nullptr) {
    HistEntry& h = s.hist[c.hist_n];
    h.energy = c.energy[0];
    h.pot_norm = c.pot_norm;
    h.theta = c.theta;
    h.ncg = ncg;
    h.nline = nline;
  }
  c.hist_n++;
}

// Energy table from the reduced energy densities (CalculateEnergy, CalPotential.f90:610-644).
HDNI inline void ctl_energy(Ctl& c, const CtlSlot& s, const double* red) {
  double loc[9] = {0, 0, red[CH_EIE], red[CH_EH], red[CH_EXC], 0, red[CH_ETF], red[CH_EVW], red[CH_ENL]};
  loc[1] = loc[6] + loc[7] + loc[8];
  for (int i = 0; i < 9; ++i) c.energy[i] = loc[i] * s.dv;
  c.energy[5] = s.ion_ion;
  c.energy[0] = c.energy[1] + c.energy[2] + c.energy[3] + c.energy[4] + c.energy[5];
}

HDNI inline void ctl_eval(Ctl& c, int mode, double ca, double cb, int evb) {
  c.ev = mode;
  c.ca = ca;
  c.cb = cb;
  c.evb = evb;
  c.op = OP_NONE;
}

HDNI inline void ctl_op(Ctl& c, int op, double coef) {
  c.op = op;
  c.opc = coef;
  c.ev = EV_NONE;
}

// Finite-difference step of NewtonDirection (RhoDirNew.f90:143-147), then the
// Hessian-vector evaluation at phi + eps p.
HDNI inline void ctl_cg_eval(Ctl& c) {
  c.eps = 2.0 * sqrt(c.macheps) * (1.0 + sqrt(c.phi2)) / sqrt(c.pp);
  ctl_eval(c, EV_CG, 1.0, c.eps, B_P);
}

// getNextGradient first half (RhoLineSearch.f90:88-96) once sum (phi+d)^2 and
// sum phi.d are known.
HDNI inline void ctl_next_gradient(Ctl& c, const CtlSlot& s) {
  c.norm_phi_dir = sqrt(c.s_phid2 * s.dv);
  ctl_op(c, OP_NG2, c.s_phid * s.dv / c.tot_ele);
}

HDNI inline void ctl_ls_trial(Ctl& c) {
  c.st = sin(c.theta);
  c.ct = cos(c.theta);
  ctl_eval(c, EV_LS, c.ct, c.st * c.dscale, B_D);
}

// Accept the line-search result: StepInformation, CheckExit, phi = tempPhi,
// ChemicalPotential and dL/dphi (RhoOptN.f90:603-630).
HDNI inline void ctl_accept(Ctl& c, const CtlSlot& s, const double* red) {
  const double npts = (double)s.N;
  c.pot_norm = sqrt(red[CH_M1] / npts);  // StepInformation uses the old mu
  ctl_push_hist(c, s, c.cg_iter, c.nline);
  // CheckExit (RhoOptN.f90:853-977)
  int exit_flag = 0;
  c.e3[2] = c.e3[1];
  c.e3[1] = c.e3[0];
  c.e3[0] = c.energy[0];
  const int p_conv = c.pot_norm < c.pot_tol;
  const int e_conv = c.iter >= 3 && dabs(c.e3[0] - c.e3[1]) < c.tole && dabs(c.e3[0] - c.e3[2]) < c.tole;
  if (c.conv_check == CONV_ENE && e_conv) { c.outcome = 0; exit_flag = 1; }
  if (c.conv_check == CONV_POT && p_conv) { c.outcome = 0; exit_flag = 1; }
  if (c.conv_check == CONV_BOTH && (p_conv || e_conv)) { c.outcome = 0; exit_flag = 1; }
  if (c.outcome == 1) exit_flag = 1;
  if (c.iter >= c.max_iter) { c.outcome = 1; exit_flag = 1; }
  // phi = tempPhi; dE/dphi at tempPhi becomes the current one
  int t = c.iphi; c.iphi = c.itrial; c.itrial = t;
  t = c.iw0; c.iw0 = c.iw1; c.iw1 = t;
  c.mu = s.dv * red[CH_M2] / (2.0 * c.tot_ele);
  c.phi2 = red[CH_M3];
  for (int k = 0; k < 9; ++k) c.energy_acc[k] = c.energy[k];
  if (exit_flag) {
    ctl_finish(c, ST_DONE, ERR_NONE);
    return;
  }
  c.iter++;
  c.switch_stp = 0;
  ctl_op(c, OP_DLDPHI, c.mu);
}

// Called after a vector op (kid = K_VEC, what = op) or an evaluation
// (kid = K_X5, what = eval mode) with the slot's reduced sums.
HDNI inline void ntn_after(Ctl& c, const CtlSlot& s, const double* red, int kid, int what) {
  for (int i = 0; i < NCH; ++i)
    if (bad(red[i])) { ctl_finish(c, ST_ERROR, ERR_NAN); return; }
  if (kid == K_X5) {
    c.num_evals++;
    switch (what) {
      case EV_RHO:
        ctl_energy(c, s, red);
        ctl_finish(c, ST_DONE, ERR_NONE);
        return;
      case EV_ION:
      case EV_FORCE:
      case EV_STRESS:
        c.num_evals--;
        ctl_finish(c, ST_DONE, ERR_NONE);
        return;
      case EV_PHI:  // first evaluation of ProjNormRhoMinimization (RhoOptN.f90:357-362)
        ctl_energy(c, s, red);
        for (int k = 0; k < 9; ++k) c.energy_acc[k] = c.energy[k];
        c.mu = s.dv * red[CH_M0] / (2.0 * c.tot_ele);
        c.phi2 = red[CH_M1];
        c.iter = 0;
        ctl_op(c, OP_DLDPHI, c.mu);
        return;
      case EV_CG: {  // pAp of the finite-difference Hessian product (RhoDirNew.f90:158-170)
        c.pap = red[CH_M0];
        if (c.pap < 0.0) {
          c.cg_flag = -2;
          if (c.cg_iter == 1)
            ctl_op(c, OP_DIRNEG, c.ry / c.pap);
          else
            ctl_op(c, OP_NG1, 0.0);
          return;
        }
        ctl_op(c, OP_CGSTEP, c.ry / c.pap);
        return;
      }
      case EV_LS: {  // LineSearchTN FG branch (RhoLineSearch.f90:400-415)
        ctl_energy(c, s, red);
        c.gradth = s.dv * red[CH_M0];
        c.nline++;
        c.num_ls++;
        if (c.stall_line > 0 && c.nline > c.stall_line) {
          // precision floor: keep the last accepted density and stop (outcome 2)
          for (int k = 0; k < 9; ++k) c.energy[k] = c.energy_acc[k];
          c.outcome = 2;
          ctl_finish(c, ST_DONE, ERR_NONE);
          return;
        }
        if (c.nline > c.max_line) { ctl_accept(c, s, red); return; }
        double stp = c.theta;
        c.ls_task = ls_step(c.ls, stp, c.energy[0], c.gradth, c.ls_task);
        if (c.ls_task == LS_FG) {
          c.theta = stp;
          ctl_ls_trial(c);
          return;
        }
        if (c.ls_task == LS_ERROR && c.iter > c.max_iter) {
          ctl_finish(c, ST_ERROR, ERR_LINESEARCH);
          return;
        }
        ctl_accept(c, s, red);
        return;
      }
      default:
        ctl_finish(c, ST_ERROR, ERR_NAN);
        return;
    }
  }
  // vector ops
  switch (what) {
    case OP_SQRT_INIT:  // totEleNum = sum(rhoR) * dV; phi = sqrt|rho| (RhoOptN.f90:298-354)
      c.tot_ele = red[0] * s.dv;
      c.theta = 0.2;
      c.e3[0] = c.e3[1] = c.e3[2] = 0.0;
      c.hist_n = 0;
      c.outcome = -1;
      c.switch_stp = 0;
      ctl_eval(c, EV_PHI, 1.0, 0.0, B_P);
      return;
    case OP_DLDPHI: {
      if (c.iter == 0) {  // initial report and the start of DensityOptimization
        c.pot_norm = sqrt(red[0] / (double)s.N);
        c.e3[0] = c.energy[0];
        c.e3[1] = 0.0;
        c.e3[2] = 0.0;
        c.theta = 0.2;
        ctl_push_hist(c, s, 0, 0);
        c.theta = 0.2;
        c.iter = 1;
      }
      // NewtonDirection set-up: r = -b, rr, y = r, ry, p = y (RhoDirNew.f90:99-141)
      c.rr = red[0];
      c.rr_last = 2.0 * c.rr;
      c.criteria = c.rr;
      c.ry_last = 0.0;
      c.ry = c.rr;
      c.cg_iter = 1;
      c.cg_flag = -1;
      c.pp = c.rr;
      c.nline = 0;
      ctl_cg_eval(c);
      return;
    }
    case OP_CGSTEP: {  // RhoDirNew.f90:172-199
      c.num_cg++;
      c.rr_last = c.rr;
      c.rr = red[0];
      c.s_phid2 = red[1];
      c.s_phid = red[2];
      int flag = -1;
      if (c.rr < 0.1 * c.criteria) flag = 0;
      else if (c.cg_iter > 50) flag = 1;
      else if (dabs(c.rr - c.rr_last) / c.rr < 0.01 && c.cg_iter > 9) flag = 2;
      if (flag >= 0) {
        c.cg_flag = flag;
        ctl_next_gradient(c, s);
        return;
      }
      c.cg_iter++;
      c.ry_last = c.ry;
      c.ry = c.rr;
      ctl_op(c, OP_PUPD, c.ry / c.ry_last);
      return;
    }
    case OP_PUPD:
      c.pp = red[0];
      ctl_cg_eval(c);
      return;
    case OP_DIRNEG:
    case OP_NG1:
    case OP_SD:
      c.s_phid2 = red[1];
      c.s_phid = red[2];
      ctl_next_gradient(c, s);
      return;
    case OP_NG2: {  // RhoLineSearch.f90:97-103 then checkGradient (:201-309)
      const double norm_perp = sqrt(red[0] * s.dv);
      c.theta = dmin(c.theta, norm_perp / c.norm_phi_dir);
      c.dscale = sqrt(c.tot_ele) / norm_perp;
      c.gradth = s.dv * c.dscale * red[1];
      if (c.gradth > 1.0e5) { ctl_finish(c, ST_ERROR, ERR_GRAD_TOO_LARGE); return; }
      if (c.gradth >= 0.0) {
        if (c.switch_stp) {
          c.outcome = 1;
          ctl_finish(c, ST_DONE, ERR_NONE);
          return;
        }
        c.switch_stp = 1;
        ctl_op(c, OP_SD, 0.0);
        return;
      }
      // LineSearchTN start (RhoLineSearch.f90:370-380)
      c.ls.ftol = 1.0e-4;
      c.ls.gtol = 0.2;
      c.ls.xtol = 1.0e-12;
      c.ls.stpmin = 0.0;
      c.ls.stpmax = 3.141592653589793238462643;
      c.nline = 0;
      double stp = c.theta;
      c.ls_task = ls_step(c.ls, stp, c.energy[0], c.gradth, LS_START);
      if (c.ls_task != LS_FG) {  // cannot happen with gradth < 0
        ctl_finish(c, ST_ERROR, ERR_LINESEARCH);
        return;
      }
      c.theta = stp;
      ctl_ls_trial(c);
      return;
    }
    default:
      ctl_finish(c, ST_ERROR, ERR_NAN);
      return;
  }
}

}  // namespace ofdft
