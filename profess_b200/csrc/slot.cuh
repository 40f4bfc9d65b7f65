// Per-cell ("slot") descriptors and the NTN controller state.
//
// A slot is one cell being evaluated or solved.  Its grid, lattice, functional
// parameters and device buffers live in a SlotDev record; its optimiser state
// lives in a Ctl record that the last block of every kernel updates for that
// slot.  The real-space arrays of a slot are x-fastest (Fortran order, as the
// reference's rho(n1,n2,n3)); half spectra (k1 = n1/2+1 planes of n2*n3
// complex values) are kx-major, each (y, z) plane contiguous with y fastest.
#pragma once
#include "cx.cuh"
#include "dcsrch.cuh"
#include "fft.cuh"

namespace ofdft {

// ---------------------------------------------------------------- buffers
enum BufId : int {
  B_PHI = 0,    // phi = sqrt(rho) (or rho for the drop-in evaluation)
  B_TRIAL = 1,  // phi of the last line-search trial
  B_W0 = 2,     // dE/dphi at phi (output potential of the drop-in evaluation)
  B_W1 = 3,     // dE/dphi at the trial, or the Hessian-vector product in CG
  B_B = 4,      // dL/dphi = dE/dphi - 2 mu phi
  B_R = 5,      // CG residual
  B_P = 6,      // CG search direction
  B_D = 7,      // Newton direction / line-search direction
  NBUF = 8
};

// ---------------------------------------------------------------- kinetic
enum Kinetic : int { KIN_WT = 4, KIN_WGC = 5 };

// Z-pass field groups (which k-space operator applies to which spectra)
enum GroupKind : int { G_HARTREE = 0, G_VW = 1, G_KMUL = 2, G_WGC3 = 3, G_ION = 4, G_FORCE = 5 };
constexpr int MAX_FIELDS = 8;
constexpr int MAX_GROUPS = 4;

// ---------------------------------------------------------------- modes
// EV_STRESS: the forward spectra of the density's fields only (x, y and z
// forward transforms of rho, rho^beta, sqrt(rho), rho^alpha), left in the
// slot's spectra for the stress reduction; no inverse transforms.
enum EvalMode : int { EV_NONE = 0, EV_RHO = 1, EV_PHI = 2, EV_CG = 3, EV_LS = 4, EV_ION = 5, EV_FORCE = 6, EV_STRESS = 7 };
enum VecOp : int {
  OP_NONE = 0,
  OP_SQRT_INIT = 1,  // phi = sqrt|rho|; sum rho
  OP_DLDPHI = 2,     // b = W0 - 2 mu phi; r = p = -b; d = 0; sum b^2
  OP_CGSTEP = 3,     // d += a p; r -= a W1; sums r^2, (phi+d)^2, phi.d
  OP_PUPD = 4,       // p = r + beta p; sum p^2
  OP_DIRNEG = 5,     // d = c p; sums (phi+d)^2, phi.d
  OP_NG1 = 6,        // sums (phi+d)^2, phi.d
  OP_NG2 = 7,        // d = d - c phi; sums d^2, W0.d
  OP_SD = 8          // d = -b; sums (phi+d)^2, phi.d
};
enum SlotStatus : int { ST_IDLE = 0, ST_RUNNING = 1, ST_DONE = 2, ST_ERROR = 3 };
enum SlotError : int { ERR_NONE = 0, ERR_GRAD_TOO_LARGE = 1, ERR_LINESEARCH = 2, ERR_NAN = 3 };

// reduction channels
constexpr int NCH = 10;
enum Chan : int { CH_EIE = 0, CH_EH = 1, CH_EXC = 2, CH_ETF = 3, CH_EVW = 4, CH_ENL = 5,
                  CH_M0 = 6, CH_M1 = 7, CH_M2 = 8, CH_M3 = 9 };

// kernel ids for per-slot task counts and done counters
enum KernelId : int { K_VEC = 0, K_X5 = 1, NKID = 2 };

constexpr int HIST_MAX = 256;
struct HistEntry {
  double energy, pot_norm, theta;
  int ncg, nline;
};

// Local pseudopotential spline of one species (ReadIonFile.f90:914-976).
struct PspDev {
  int npts;
  int off;  // offset of this species' vqs / pot_dd in the packed table
  double max_g, charge, v0, dq;
};

constexpr int MAX_SPECIES = 4;

// Tables of the ion-electron set-up and forces (EV_ION / EV_FORCE modes).
struct IonAux {
  int nspec;
  PspDev psp[MAX_SPECIES];
  const double* tab;      // packed vqs then pot_dd for every species
  const cx<double>* b1;   // exponential-spline factors, k1 entries
  const cx<double>* b2;   // n2 entries
  const cx<double>* b3;   // n3 entries
};

struct SlotDev {
  int n1, n2, n3, k1;
  long long N, Nc;
  FftPlan px, py, pz;
  double recip[9];  // cellRecip, column-major: recip[3*c + r] = b_c component r
  double dv, inv_n, vol;
  int kinetic, nf, ngroups, alpha_eq_beta;
  int pow56;       // alpha == beta == 5/6: rho^(5/6) = sqrt(rho) * cbrt(rho)
  int rp;          // row pairs per X-pass task
  int group_kind[MAX_GROUPS];
  int group_f0[MAX_GROUPS];
  int group_nf[MAX_GROUPS];
  double lambda, mu, alpha, beta, rho_s, ion_ion;
  void* buf[NBUF];
  void* vion;   // ionPotReal (N)
  void* kern;   // keKernel planes (nplanes * Nc), real
  void* spec;   // nf half spectra (nf * Nc complex)
  IonAux ion;
  double* partials;  // ntask_max * NCH
  int ntask[NKID];
  HistEntry* hist;
};

struct Ctl {
  int status, error, state, op, ev;
  int iphi, itrial, iw0, iw1, evb;
  int opt_sqrt, want_energy;
  int force_rho;  // EV_FORCE input: 1 = rho in buf[B_PHI], 0 = phi in buf[iphi]
  // prologue coefficients: phi_in = ca * buf[iphi] + cb * buf[evb]
  double ca, cb;
  double opc;  // op coefficient
  // optimiser scalars
  double tot_ele, mu, phi2, theta, st, ct, dscale, gradth, eps, macheps;
  double energy[9];
  double energy_acc[9];  // energy table of the last accepted density
  double e3[3];
  double pot_norm;
  int iter, max_iter, conv_check, max_line, switch_stp, outcome, nline;
  int stall_line;  // > 0: stop when one line search needs more trials (precision floor)
  double pot_tol, tole;
  // CG
  int cg_iter, cg_flag;
  double rr, rr_last, ry, ry_last, criteria, pap, pp;
  double s_phid2, s_phid, norm_phi_dir;
  // line search
  LineSearch ls;
  int ls_task;
  // statistics
  int num_evals, num_cg, num_ls, hist_n;
};

enum ConvCheck : int { CONV_ENE = 0, CONV_POT = 1, CONV_BOTH = 2 };

// Generic task record: slot plus three kernel-specific integers.
struct Task {
  int slot, a, b, c;
};

// Tiles of the split y and z passes: ceil(n / tx) tiles of nearly equal width
// over n columns (49 columns in tiles of 16 become 13 + 12 + 12 + 12, not
// 16 + 16 + 16 + 1).  A task's c field holds the first column | (width << 16).
HD int tile_count(int k1, int tx) { return (k1 + tx - 1) / tx; }
HD int tile_code(int k1, int tx, int t) {
  const int nt = tile_count(k1, tx), base = k1 / nt, rem = k1 % nt;
  const int kx0 = t * base + (t < rem ? t : rem);
  return kx0 | ((base + (t < rem ? 1 : 0)) << 16);
}
HD int tile_first(int c) { return c & 0xffff; }
HD int tile_width(int c) { return c >> 16; }

}  // namespace ofdft
