/*
 * profess_b200 — C ABI of the B200 orbital-free DFT density-solve engine.
 *
 * This is the drop-in boundary for the density-solve path of PROFESS: the
 * energy/potential evaluation (module CalPotPlus, CalculatePotentialPlus) and
 * the sqrt-density truncated-Newton optimiser (module RhoOptN, method NTN,
 * ProjNormRhoMinimization).  A Fortran host binds these entry points through
 * iso_c_binding; every argument is a plain pointer or scalar, arrays are
 * Fortran-ordered (x fastest) REAL(DP) buffers exactly as the reference holds
 * them, and every entry point returns an int status (0 = OK; see OFDFT_E*).
 * ofdft_last_error() gives the message of the last failure on this thread.
 *
 * Objects: an engine owns device memory, streams and FFT plans; a slot is one
 * cell (grid, lattice, functional parameters, kernel tables, ion potential and
 * solver state) inside an engine.  One engine may hold many slots, which are
 * then evaluated/solved together (batched, one launch per pass for all slots).
 */
#ifndef PROFESS_B200_H
#define PROFESS_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define OFDFT_OK 0
#define OFDFT_EINVAL 1      /* bad argument */
#define OFDFT_ECUDA 2       /* CUDA runtime failure */
#define OFDFT_ENOMEM 3      /* device memory exhausted */
#define OFDFT_EBUSY 4       /* slot is running */
#define OFDFT_ENAN 5        /* non-finite value in a reduction */
#define OFDFT_EGRAD 6       /* dE/dtheta too large (RhoLineSearch.f90:243-245) */
#define OFDFT_ELINESEARCH 7 /* line search error past maxIter (RhoLineSearch.f90:431-440) */
#define OFDFT_ETIMEOUT 8    /* solve exceeded the caller's tick budget */

/* kinetic functional codes (CellInfo::kinetic) */
#define OFDFT_KEDF_WT 4
#define OFDFT_KEDF_WGC 5

/* precision of a slot */
#define OFDFT_FP64 0
#define OFDFT_FP32 1

/* convergence tests (RhoOptimizers::conv_check) */
#define OFDFT_CONV_ENE 0
#define OFDFT_CONV_POT 1
#define OFDFT_CONV_BOTH 2

typedef struct ofdft_engine ofdft_engine;

/* Cell description: the module state CalculatePotentialPlus reads through USE
 * association (Source/CalPotential.f90:41-116; CellInfo, KEDF_TF, KEDF_VW,
 * KEDF_WTkernel, KEDF_WGCkernel, Sys, Ewald). */
typedef struct ofdft_cell_desc {
  int n1, n2, n3;          /* real-space grid n1G, n2G, n3G */
  double lattice[9];       /* cell%cellReal in bohr, column-major: lattice[3*i+k] = component k of vector i */
  int kinetic;             /* OFDFT_KEDF_WT or OFDFT_KEDF_WGC (second order, WGCT = 2) */
  double lambda, mu;       /* TF and vW coefficients (KEDF_TF::lambda, KEDF_VW::mu) */
  double alpha, beta;      /* nonlocal exponents (KEDF_WTkernel::alpha, beta) */
  double gamma;            /* WGC gamma (KEDF_WGCkernel::gamma); kernel construction only */
  double rho0;             /* Sys::rho0, WT/WGC kernel reference density */
  double rho_s;            /* Sys::rhoS, WGC Taylor expansion density */
  double ion_ion_energy;   /* Ewald::ionIonEnergy (Ha), copied into eTable(6) */
  int precision;           /* OFDFT_FP64 or OFDFT_FP32 */
} ofdft_cell_desc;

/* Options of the NTN solve (RhoOptimizers module state, Source/RhoOptimizers.f90:44-101). */
typedef struct ofdft_ntn_options {
  int max_iter;            /* maxIter, default 500 */
  int conv_check;          /* OFDFT_CONV_*, default ENE */
  double pot_tol;          /* pot_tol, default 1e-5 */
  double tole;             /* tole (Ha), default 1e-6 */
  int max_line;            /* maxLine (Source/RhoLineSearch.f90:34), default 200 */
  int max_ticks;           /* safety bound on engine ticks for the blocking call (0 = 20000) */
  int stall_line;          /* > 0: stop with outcome 2, keeping the last accepted density, when one
                              line search needs more than this many trials (the FP32 precision
                              floor of a mixed-precision solve); 0 = reference behaviour */
} ofdft_ntn_options;

/* Outcome of a solve (rhoOutcome, numEnergyTotal, numPotentialTotal ...). */
typedef struct ofdft_ntn_stats {
  int outcome;             /* rhoOutcome: 0 converged, 1 max iterations / no descent, 2 stalled */
  int iterations;          /* outer NTN iterations */
  int num_evals;           /* potential evaluations (CalculatePotentialPlus calls) */
  int num_cg;              /* inner CG steps in total */
  int num_line;            /* line-search evaluations in total */
  int history_len;         /* entries available from ofdft_slot_history */
  double pot_norm;         /* final potential norm (StepInformation) */
  int error;               /* internal error code (0 none) */
  int ticks;               /* engine ticks the solve took */
} ofdft_ntn_stats;

const char* ofdft_last_error(void);
int ofdft_version(void);

/* ---------------------------------------------------------------- engine */
int ofdft_engine_create(ofdft_engine** out);
int ofdft_engine_destroy(ofdft_engine* e);

/* ---------------------------------------------------------------- slots */
/* Allocate a slot for one cell.  Replaces the module set-up that precedes the
 * first CalculatePotentialPlus call (Source/Initializer.f90, SetupKEDF.f90). */
int ofdft_slot_create(ofdft_engine* e, const ofdft_cell_desc* desc, int* slot);
int ofdft_slot_destroy(ofdft_engine* e, int slot);
/* KEDF_WTkernel::keKernel(k1G,k2G,k3G,nplanes), k1G = n1/2+1 (Source/KEDF_WTkernel.f90:81-208,
 * Source/KEDF_WGCkernel.f90:109-277); nplanes = 1 for WT, 4 for WGC. */
int ofdft_slot_set_kernel(ofdft_engine* e, int slot, const double* kernel, int nplanes);
/* IonElectronSpline::ionPotReal(n1G,n2G,n3G) (Source/RefreshIons.f90:215-221). */
int ofdft_slot_set_ion_potential(ofdft_engine* e, int slot, const double* ion_pot);
/* Ewald energy (Ha) and forces (Ha/bohr, nion x 3, may be NULL) of the slot's
 * ions (the positions of its last ofdft_slot_build_ion_potential), summed on
 * the device (EwaldEnergy / EwaldForces, Source/Ewald.f90:465-1193); the energy
 * also becomes the slot's eTable(6).  Same splitting and cut-offs as ofdft_ewald. */
int ofdft_slot_ewald(ofdft_engine* e, int slot, double* energy, double* forces);
/* The ion-ion (Ewald) energy entered as eTable(6) of the slot's energies,
 * after the ions moved (RefreshIonTerms recomputes it, Source/RefreshIons.f90:125-238). */
int ofdft_slot_set_ion_ion_energy(ofdft_engine* e, int slot, double energy);
/* The WT kernel built on the device from LindG (replaces FillWT, KEDF_WTkernel.f90:81-208). */
int ofdft_slot_build_wt_kernel(ofdft_engine* e, int slot);
/* The WGC kernel planes from radial tables of w, eta*w', eta^2*w'' on the eta
 * grid (Source/KEDF_WGCkernel.f90:166-230); splines are evaluated on the device. */
int ofdft_slot_build_wgc_kernel(ofdft_engine* e, int slot, int ntab, const double* eta,
                                const double* w, const double* w1, const double* w2);
/* The ion-electron potential built on the device by the cardinal B-spline
 * method (IonElectronPotRecipSpline, Source/IonElectronSpline.f90:83-216):
 * frac[3*nion] fractional coordinates, species[nion] 0-based species index;
 * per species s: npts[s] points of the recpot table on [0, max_g[s]] (bohr^-1)
 * with values pot_values (Ha*bohr^3), spline knots vqs and second derivatives
 * pot_dd, packed one species after the other; charge[s] the ionic charge. */
int ofdft_slot_build_ion_potential(ofdft_engine* e, int slot, int nion, const double* frac,
                                   const int* species, int nspecies, const int* npts,
                                   const double* max_g, const double* charge,
                                   const double* pot_values, const double* vqs, const double* pot_dd);

/* Ion forces (Ha/bohr, nion x 3, row i = ion i) on the slot's current density
 * (rho = NULL: the density of the last solve, phi^2) or on the given rho:
 * ion-electron forces by the B-spline method (IonElectronForcesSpline /
 * CalculateSplineForces, Source/IonElectronSpline.f90:219-355,642-753) plus,
 * when include_ewald, the ion-ion Ewald forces (ForcesII_IE,
 * Source/CalForce.f90:134-239).  Needs ofdft_slot_build_ion_potential first. */
int ofdft_slot_forces(ofdft_engine* e, int slot, const double* rho, int include_ewald, double* forces);
/* Autotuner, the planning step of the engine (the reference plans its FFTs
 * with FFTW, PlanFFT in Source/Fourier_v1.f90:103-190): for the slot's kind
 * of cell (grid, precision, functional), times one batched evaluation of
 * every idle slot of that kind holding a resident input density
 * (ofdft_slot_set_input) per candidate launch shape - the radix cap of the
 * x-axis FFT plan, row pairs per x-forward and x-inverse task, and the block
 * size of the fused y-z pass - and keeps the fastest.  The choice is cached
 * in the engine for that kind and applied to every such slot, also to those
 * created later.  ms_default / ms_tuned: the median batched evaluation time
 * before and after; shape[4] (may be NULL): radix cap, x-forward and
 * x-inverse row pairs, y-z threads (0: split y/z path).  No slot may be
 * running; the timed slots' solve records are overwritten. */
int ofdft_engine_tune(ofdft_engine* e, int slot, int iters, double* ms_default, double* ms_tuned, int* shape);
/* Pin the slot's launch shape (the four values ofdft_engine_tune reports, e.g.
 * a shape tuned in an earlier run; radix cap 0 and y-z threads 0 mean the
 * defaults).  OFDFT_EINVAL for a cap without a plan or tasks whose shared
 * memory would not fit. */
int ofdft_slot_set_shape(ofdft_engine* e, int slot, const int* shape);
/* The slot's current launch shape, as ofdft_engine_tune reports it. */
int ofdft_slot_shape(ofdft_engine* e, int slot, int* shape);
/* A new lattice (layout as in ofdft_cell_desc) for the slot, same grid:
 * RefreshLattice (Source/CellInfo.f90) with the kernel reference densities of
 * KEDFRefresh (Source/SetupKEDF.f90:620-680).  RefreshCellSetup
 * (Source/RefreshCell.f90:27-76) then continues with
 * ofdft_slot_build_wt_kernel (or _wgc_kernel), ofdft_slot_build_ion_potential
 * and ofdft_slot_ewald. */
int ofdft_slot_set_lattice(ofdft_engine* e, int slot, const double* lattice, double rho0, double rho_s);
/* RescaleDensity (Source/RefreshIons.f90:33-122) of the held input density
 * (ofdft_slot_hold_density): scaled on the device to num_electrons electrons
 * with the slot's current dV, e.g. after a change of lattice. */
int ofdft_slot_rescale_input(ofdft_engine* e, int slot, double num_electrons);
/* Stress tensor (Ha/bohr^3, stress[9] row-major and symmetric) of the slot's
 * current density (rho = NULL: phi^2 of the last solve) or of the given rho:
 * CalculateStress (Source/CalStress.f90:44-253) with the TF, vW, nonlocal
 * kinetic (WTStress or, for second-order WGC slots, WGCStress), Hartree, LDA
 * and B-spline ion-electron terms plus, when include_ewald, the Ewald term
 * (EwaldStress, Source/Ewald.f90:1857-2535).  terms[7*9] (may be NULL)
 * receives the seven parts in that order.  Runs one
 * energy evaluation and the forward transforms of the density on the device;
 * the slot's solve record, current phi and potential are kept.  Needs
 * ofdft_slot_build_ion_potential first. */
int ofdft_slot_stress(ofdft_engine* e, int slot, const double* rho, int include_ewald, double* stress,
                      double* terms);

/* ---------------------------------------------------------------- host set-up helpers */
/* The More-Thuente line search of the solver (Dcsrch / Dcstep,
 * Source/MathDCsrch.f, Source/MathDCstep.f) in reverse communication, for host
 * optimisers (GradientOptimization, Source/IonOptCON.f90:33-241): the record
 * holds Dcsrch's isave/dsave; set ftol, gtol, xtol, stpmin and stpmax, call
 * with task OFDFT_LS_START, then with OFDFT_LS_FG at each requested point
 * while it returns OFDFT_LS_FG.  Returns the new task (CONV, WARN and ERROR
 * end the search; stp then stays the last step), or -OFDFT_EINVAL for a null
 * argument or another task. */
typedef struct {
  double ftol, gtol, xtol, stpmin, stpmax;
  int brackt, stage;
  double ginit, gtest, gx, gy, finit, fx, fy, stx, sty, stmin, stmax, width, width1;
} ofdft_line_search;
enum { OFDFT_LS_START = 0, OFDFT_LS_FG = 1, OFDFT_LS_CONV = 2, OFDFT_LS_WARN = 3, OFDFT_LS_ERROR = 4 };
int ofdft_dcsrch(ofdft_line_search* ls, double* stp, double f, double g, int task);

/* Ewald ion-ion energy (Ha) and forces (may be NULL) of point charges
 * (EwaldEnergy / EwaldForces, Source/Ewald.f90:465-1193,1196+).  lattice as in
 * ofdft_cell_desc; frac[3*nion]; charges[nion]. */
int ofdft_ewald(const double* lattice, int nion, const double* frac, const double* charges, double* energy,
                double* forces);
/* FFT grid from the kinetic-energy cutoff (Ha): SizeSystem / PadFFTdims
 * (Source/SetupFFT.f90:193-382) with dimType 1 (7-smooth sizes). */
int ofdft_grid_size(double ecut_ha, const double* lattice, int* n);
/* Radial WGC kernel tables (eta, w, eta w', eta^2 w'') on the reference's eta
 * grid from the kernel ODE (makeKernel2, Source/KEDF_KernelODE.f90:254-537).
 * Call with max = 0 to get the table length in *n. */
int ofdft_wgc_radial_tables(double alpha, double beta, double gamma, int max, double* eta, double* w, double* w1,
                            double* w2, int* n);

/* ---------------------------------------------------------------- drop-in calls */
/* CalculatePotentialPlus(rho, optSqrt, potential, eTable) (Source/CalPotential.f90:41-647),
 * numSpin = 1.  rho and potential are (n1,n2,n3) x-fastest; eTable (9 doubles,
 * Report.f90:270-308 order) may be NULL, which skips the energy terms. */
int ofdft_calculate_potential_plus(ofdft_engine* e, int slot, const double* rho, int opt_sqrt,
                                   double* potential, double* etable);
/* ProjNormRhoMinimization(energy, dir_type = 1) (Source/RhoOptN.f90:60-545):
 * rho (n1,n2,n3) is Sys::rhoR on entry and the optimised density on return;
 * energy receives the 9-entry table; opts may be NULL for the defaults. */
int ofdft_proj_norm_rho_minimization(ofdft_engine* e, int slot, double* rho, double* energy,
                                     const ofdft_ntn_options* opts, ofdft_ntn_stats* stats);

/* Allocation-free CalculatePotentialPlus (no counterpart in the reference).
 * For callers that cannot allocate device memory themselves or through this
 * library (a host code running inside a device-memory pool it does not own,
 * or under a memory budget fixed before the solve): all scratch comes from a
 * 12 MiB array compiled into the library, which every GPU that loads the
 * library holds until the process exits.  Supports the FP64 WT functional on
 * 7-smooth grids with dimensions <= 128 and at most 262144 points; larger
 * requests return OFDFT_EINVAL.  rho, kernel (keKernel plane, (n1/2+1,n2,n3)),
 * ion_pot and potential are DEVICE pointers (x-fastest, FP64); etable (9
 * doubles, may be NULL) is host memory; stream is a cudaStream_t or NULL.
 * The first call on a device looks up the array's address on that device:
 * make that first call before any stream capture on the device.  Calls on
 * one GPU share its array, so calls whose work overlaps on that GPU race;
 * the host-side staging of a call belongs to the calling thread, so calls
 * from different host threads on different GPUs do not interfere.  The call
 * returns after its stream has finished. */
int ofdft_calculate_potential_plus_noalloc(const ofdft_cell_desc* desc, const double* rho, const double* kernel,
                                           const double* ion_pot, int opt_sqrt, double* potential, double* etable,
                                           void* stream);

/* ---------------------------------------------------------------- batched / asynchronous */
/* Host arrays (rho, results, downloads) are FP64 whatever the slot's
 * precision.  They are copied straight from / to the caller's memory on the
 * engine's stream (page-locked memory copies fastest); the FP32 conversion and
 * phi^2 run on the device. */
/* Upper bound of the device memory one slot of this description uses (bytes). */
int ofdft_slot_footprint(const ofdft_cell_desc* desc, unsigned long long* bytes);
/* Keep an input density resident on the device; start calls with rho = NULL use it. */
int ofdft_slot_set_input(ofdft_engine* e, int slot, const double* rho);
/* Start a solve from rho (host) or, with rho = NULL, from the resident input. */
int ofdft_slot_start_solve(ofdft_engine* e, int slot, const double* rho, const ofdft_ntn_options* opts);
/* The kernel planes, ion potential and ion-ion energy of slot src_slot,
 * converted on the device into slot `slot` of the same grid and functional
 * (either precision).  No counterpart in the reference: a mixed-precision
 * request sets up its FP64 slot once (ofdft_slot_build_* and ofdft_slot_ewald)
 * and gives its FP32 slot the same tables with this call. */
int ofdft_slot_copy_tables(ofdft_engine* e, int slot, int src_slot);
/* Keep the slot's current density (phi^2 of its last solve) on the device as
 * its resident input, so that a later start with rho = NULL resumes from it
 * (no counterpart in the reference, whose rhoR simply persists between
 * geometry steps): a geometry step calls it before rebuilding the ion
 * potential, which reuses the slot's state arrays. */
int ofdft_slot_hold_density(ofdft_engine* e, int slot);
/* Start a solve from the density already resident in another slot of the same
 * engine (e.g. an FP32 slot's result refined in an FP64 slot); no host copy. */
int ofdft_slot_start_solve_from_slot(ofdft_engine* e, int slot, int src_slot, const ofdft_ntn_options* opts);
int ofdft_slot_start_eval(ofdft_engine* e, int slot, const double* rho, int opt_sqrt, int want_energy);
/* Stop a running solve or evaluation (no counterpart in the reference): the
 * slot goes idle and keeps its buffers; a server drops a request with it.  The
 * blocking calls above do this themselves when they run out of ticks
 * (OFDFT_ETIMEOUT). */
int ofdft_slot_cancel(ofdft_engine* e, int slot);
/* Run up to `ticks` engine ticks over every running slot; *running receives the
 * number of slots still running afterwards. */
int ofdft_engine_run(ofdft_engine* e, int ticks, int* running);
/* 1 if the slot has finished (done or error), 0 if it is running. */
int ofdft_slot_poll(ofdft_engine* e, int slot, int* finished);
/* Results of a finished solve: rho (may be NULL) = phi^2, energy (9, may be NULL), stats. */
int ofdft_slot_result(ofdft_engine* e, int slot, double* rho, double* energy, ofdft_ntn_stats* stats);
/* Per-iteration trajectory (MinimizerReportSteps rows): energy (Ha), potential
 * norm, theta, #CG, #line; up to max entries. */
int ofdft_slot_history(ofdft_engine* e, int slot, int max, double* energy, double* pot_norm,
                       double* theta, int* ncg, int* nline, int* n);
/* Device-resident arrays of a slot: which = 0 phi, 1 dE/dphi, 2 ion potential. */
int ofdft_slot_download(ofdft_engine* e, int slot, int which, double* out);

/* ---------------------------------------------------------------- instrumentation */
/* The CUDA stream (cudaStream_t) the engine launches on. */
int ofdft_engine_stream(ofdft_engine* e, void** stream);
/* Kernel launches and ticks issued so far by this engine. */
int ofdft_engine_counters(ofdft_engine* e, long long* kernel_launches, long long* ticks);
/* Graphs captured so far (the task lists changed between runs) and the host
 * time spent capturing and instantiating them (ms). */
int ofdft_engine_capture_stats(ofdft_engine* e, long long* captures, double* host_ms);
/* Mean device time (ms) of one batched potential evaluation over every idle
 * slot with a resident input density, timed with events on the engine stream. */
int ofdft_engine_time_eval(ofdft_engine* e, int iters, double* ms);

#ifdef __cplusplus
}
#endif
#endif /* PROFESS_B200_H */
