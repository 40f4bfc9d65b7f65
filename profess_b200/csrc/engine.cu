// Host runtime of the density-solve engine and its C ABI.
//
// An Engine owns device memory for its slots, the FFT plan/twiddle tables and
// the per-precision task lists of the six kernels (vector op and the five
// evaluation passes).  One engine tick launches, for each precision with
// running slots, the vector kernel VEC_PER_TICK times and then passes 1-5;
// every running slot advances by at most VEC_PER_TICK vector ops and one
// potential evaluation per tick, decided on the device by the NTN controller.
//
// Built twice from this file: the product library (nvcc, sm_100a) and, with
// OFDFT_EMU defined, a host-only emulation library used by the CPU test suite
// to check the same block functions against the oracle.  The emulation build
// runs each block with one thread; it is never loaded by the product.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "passes.cuh"
#include "profess_b200.h"

#if !defined(OFDFT_EMU)
#include <cuda_runtime.h>
#endif

namespace ofdft {

// ------------------------------------------------------------ errors
static thread_local std::string g_err;
static int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

// ------------------------------------------------------------ memory
#if defined(OFDFT_EMU)
static int dmalloc(void** p, size_t n) {
  *p = calloc(1, n ? n : 1);
  return *p ? OFDFT_OK : fail(OFDFT_ENOMEM, "host allocation failed");
}
static void dfree(void* p) { free(p); }
static int h2d(void* d, const void* h, size_t n) { memcpy(d, h, n); return OFDFT_OK; }
static int d2h(void* h, const void* d, size_t n) { memcpy(h, d, n); return OFDFT_OK; }
static int d2d(void* d, const void* s, size_t n) { memmove(d, s, n); return OFDFT_OK; }
static int dzero(void* d, size_t n) { memset(d, 0, n); return OFDFT_OK; }
static int dsync() { return OFDFT_OK; }
#else
static int cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return OFDFT_OK;
  return fail(e == cudaErrorMemoryAllocation ? OFDFT_ENOMEM : OFDFT_ECUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}
static int dmalloc(void** p, size_t n) {
  int rc = cuda_check(cudaMalloc(p, n ? n : 1), "cudaMalloc");
  if (rc == OFDFT_OK) rc = cuda_check(cudaMemset(*p, 0, n ? n : 1), "cudaMemset");
  return rc;
}
static void dfree(void* p) { if (p) cudaFree(p); }
static int h2d(void* d, const void* h, size_t n) { return cuda_check(cudaMemcpy(d, h, n, cudaMemcpyHostToDevice), "H2D"); }
static int d2h(void* h, const void* d, size_t n) { return cuda_check(cudaMemcpy(h, d, n, cudaMemcpyDeviceToHost), "D2H"); }
static int d2d(void* d, const void* s, size_t n) { return cuda_check(cudaMemcpy(d, s, n, cudaMemcpyDeviceToDevice), "D2D"); }
static int dzero(void* d, size_t n) { return cuda_check(cudaMemset(d, 0, n), "cudaMemset"); }
static int dsync() { return cuda_check(cudaDeviceSynchronize(), "synchronize"); }
#endif

// ------------------------------------------------------------ FFT plans
static bool seven_smooth(int n) {
  if (n < 1) return false;
  for (int p : {2, 3, 5, 7})
    while (n % p == 0) n /= p;
  return n == 1;
}

// Radix sequence of n: as many 8s as possible, then one 4 or 2, then 3, 5, 7.
static std::vector<int> radices(int n) {
  std::vector<int> r;
  int e2 = 0;
  while (n % 2 == 0) { n /= 2; ++e2; }
  while (e2 >= 3) { r.push_back(8); e2 -= 3; }
  if (e2 == 2) r.push_back(4);
  if (e2 == 1) r.push_back(2);
  for (int p : {3, 5, 7})
    while (n % p == 0) { r.push_back(p); n /= p; }
  return r;
}

constexpr int MAX_N = 512;

struct PlanTable {
  std::map<int, FftPlan> plans;
  std::vector<long double> re, im;
  void* d_tw64 = nullptr;
  void* d_tw32 = nullptr;

  int build() {
    for (int n = 1; n <= MAX_N; ++n) {
      if (!seven_smooth(n)) continue;
      FftPlan p;
      memset(&p, 0, sizeof(p));
      p.n = n;
      p.tw_base = (int)re.size();
      std::vector<int> rs = radices(n);
      p.nst = (int)rs.size();
      int ns = 1, off = 0;
      for (int s = 0; s < p.nst; ++s) {
        const int R = rs[s];
        p.R[s] = R;
        p.Ns[s] = ns;
        p.tw[s] = off;
        for (int k = 0; k < ns; ++k)
          for (int m = 1; m < R; ++m) {
            const long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)(m * k) /
                                    (long double)(ns * R);
            re.push_back(cosl(ang));
            im.push_back(sinl(ang));
          }
        off += ns * (R - 1);
        ns *= R;
      }
      plans[n] = p;
    }
    const size_t nt = re.size();
    std::vector<cx<double>> t64(nt);
    std::vector<cx<float>> t32(nt);
    for (size_t i = 0; i < nt; ++i) {
      t64[i] = mk<double>((double)re[i], (double)im[i]);
      t32[i] = mk<float>((float)re[i], (float)im[i]);
    }
    int rc = dmalloc(&d_tw64, nt * sizeof(cx<double>));
    if (rc) return rc;
    rc = dmalloc(&d_tw32, nt * sizeof(cx<float>));
    if (rc) return rc;
    rc = h2d(d_tw64, t64.data(), nt * sizeof(cx<double>));
    if (rc) return rc;
    return h2d(d_tw32, t32.data(), nt * sizeof(cx<float>));
  }
  void release() {
    dfree(d_tw64);
    dfree(d_tw32);
    d_tw64 = d_tw32 = nullptr;
  }
};

// ------------------------------------------------------------ kernels
enum Pass : int { P_VEC = 0, P_X1 = 1, P_Y2 = 2, P_Z3 = 3, P_Y4 = 4, P_X5 = 5, NPASS = 6 };
constexpr int VEC_PER_TICK = 3;
constexpr int VCHUNK = 4096;

#if !defined(OFDFT_EMU)
template <typename T> __global__ void k_vec(Args<T> a) {
  extern __shared__ __align__(16) char sm[];
  vec_block<T>(a, blockIdx.x, threadIdx.x, blockDim.x, sm);
}
template <typename T> __global__ void k_xfwd(Args<T> a) {
  extern __shared__ __align__(16) char sm[];
  xfwd_block<T>(a, blockIdx.x, threadIdx.x, blockDim.x, sm);
}
template <typename T> __global__ void k_ypass(Args<T> a, int dir) {
  extern __shared__ __align__(16) char sm[];
  ypass_block<T>(a, blockIdx.x, threadIdx.x, blockDim.x, sm, dir);
}
template <typename T> __global__ void k_zpass(Args<T> a) {
  extern __shared__ __align__(16) char sm[];
  zpass_block<T>(a, blockIdx.x, threadIdx.x, blockDim.x, sm);
}
template <typename T> __global__ void k_xinv(Args<T> a) {
  extern __shared__ __align__(16) char sm[];
  xinv_block<T>(a, blockIdx.x, threadIdx.x, blockDim.x, sm);
}
#endif

struct LaunchList {
  std::vector<Task> h;
  Task* d = nullptr;
  size_t cap = 0;
  size_t smem = 0;
  int nthr = 128;
};

struct HostSlot {
  bool used = false;
  bool running = false;
  int prec = 0;
  SlotDev sd;
  std::vector<void*> allocs;
  int nrowpairs = 0, rp = 1, tx = 8;
  int nplanes = 0;
};

static size_t elem_size(int prec) { return prec == OFDFT_FP32 ? 4 : 8; }

struct Engine {
  std::vector<HostSlot> slots;
  SlotDev* d_slots = nullptr;
  Ctl* d_ctl = nullptr;
  int cap = 0;
  PlanTable plans;
  LaunchList lists[2][NPASS];
  bool dirty = true;
  std::vector<char> emu_smem;

  int init(int capacity) {
    cap = capacity;
    slots.resize(cap);
    int rc = dmalloc((void**)&d_slots, sizeof(SlotDev) * cap);
    if (rc) return rc;
    rc = dmalloc((void**)&d_ctl, sizeof(Ctl) * cap);
    if (rc) return rc;
    return plans.build();
  }

  void release() {
    for (int i = 0; i < cap; ++i) free_slot(i);
    for (auto& pl : lists)
      for (auto& l : pl) dfree(l.d);
    dfree(d_slots);
    dfree(d_ctl);
    plans.release();
  }

  void free_slot(int i) {
    HostSlot& h = slots[i];
    for (void* p : h.allocs) dfree(p);
    h.allocs.clear();
    h.used = false;
    h.running = false;
    dirty = true;
  }

  int alloc(HostSlot& h, void** p, size_t bytes) {
    int rc = dmalloc(p, bytes);
    if (rc == OFDFT_OK) h.allocs.push_back(*p);
    return rc;
  }

  int upload_slot(int i) { return h2d(d_slots + i, &slots[i].sd, sizeof(SlotDev)); }

  int create_slot(const ofdft_cell_desc* d, int* out) {
    if (!d) return fail(OFDFT_EINVAL, "null descriptor");
    const int ns[3] = {d->n1, d->n2, d->n3};
    for (int k = 0; k < 3; ++k)
      if (ns[k] < 2 || ns[k] > MAX_N || !seven_smooth(ns[k]))
        return fail(OFDFT_EINVAL, "grid dimensions must be 7-smooth and in [2, 512]");
    if (d->kinetic != KIN_WT && d->kinetic != KIN_WGC) return fail(OFDFT_EINVAL, "kinetic must be 4 (WT) or 5 (WGC)");
    if (d->precision != OFDFT_FP64 && d->precision != OFDFT_FP32) return fail(OFDFT_EINVAL, "bad precision");
    int idx = -1;
    for (int i = 0; i < cap; ++i)
      if (!slots[i].used) { idx = i; break; }
    if (idx < 0) return fail(OFDFT_ENOMEM, "engine has no free slot");
    HostSlot& h = slots[idx];
    h = HostSlot();
    h.used = true;
    h.prec = d->precision;
    SlotDev& s = h.sd;
    memset(&s, 0, sizeof(s));
    s.n1 = d->n1; s.n2 = d->n2; s.n3 = d->n3;
    s.k1 = d->n1 / 2 + 1;
    s.N = (long long)d->n1 * d->n2 * d->n3;
    s.Nc = (long long)s.k1 * d->n2 * d->n3;
    s.px = plans.plans[d->n1];
    s.py = plans.plans[d->n2];
    s.pz = plans.plans[d->n3];
    // cellRecip = TRANSPOSE(Inverse(cellReal)) * 2 pi  (CellInfo.f90:281)
    const double* L = d->lattice;  // L[3*i + k] = component k of vector i
    auto A = [&](int r, int c) { return L[3 * c + r]; };
    const double det = A(0, 0) * (A(1, 1) * A(2, 2) - A(1, 2) * A(2, 1)) -
                       A(0, 1) * (A(1, 0) * A(2, 2) - A(1, 2) * A(2, 0)) +
                       A(0, 2) * (A(1, 0) * A(2, 1) - A(1, 1) * A(2, 0));
    if (!(std::fabs(det) > 0)) return fail(OFDFT_EINVAL, "singular lattice");
    double inv[3][3];
    inv[0][0] = (A(1, 1) * A(2, 2) - A(1, 2) * A(2, 1)) / det;
    inv[0][1] = (A(0, 2) * A(2, 1) - A(0, 1) * A(2, 2)) / det;
    inv[0][2] = (A(0, 1) * A(1, 2) - A(0, 2) * A(1, 1)) / det;
    inv[1][0] = (A(1, 2) * A(2, 0) - A(1, 0) * A(2, 2)) / det;
    inv[1][1] = (A(0, 0) * A(2, 2) - A(0, 2) * A(2, 0)) / det;
    inv[1][2] = (A(0, 2) * A(1, 0) - A(0, 0) * A(1, 2)) / det;
    inv[2][0] = (A(1, 0) * A(2, 1) - A(1, 1) * A(2, 0)) / det;
    inv[2][1] = (A(0, 1) * A(2, 0) - A(0, 0) * A(2, 1)) / det;
    inv[2][2] = (A(0, 0) * A(1, 1) - A(0, 1) * A(1, 0)) / det;
    const double twopi = 2.0 * 3.141592653589793238462643;
    // recip matrix R = inv^T * 2pi; column c (vector b_c) component r = R(r,c) = inv[c][r] * 2pi
    for (int c = 0; c < 3; ++c)
      for (int r = 0; r < 3; ++r) s.recip[3 * c + r] = inv[c][r] * twopi;
    s.vol = std::fabs(det);
    s.dv = s.vol / (double)s.N;
    s.inv_n = 1.0 / (double)s.N;
    s.kinetic = d->kinetic;
    s.lambda = d->lambda;
    s.mu = d->mu;
    s.alpha = d->alpha;
    s.beta = d->beta;
    s.rho_s = d->rho_s;
    s.ion_ion = d->ion_ion_energy;
    s.alpha_eq_beta = (d->alpha == d->beta) ? 1 : 0;
    if (s.kinetic == KIN_WT) {
      s.nf = s.alpha_eq_beta ? 3 : 4;
      s.ngroups = s.nf;
      const int kinds[4] = {G_HARTREE, G_KMUL, G_VW, G_KMUL};
      for (int g = 0; g < s.ngroups; ++g) { s.group_kind[g] = kinds[g]; s.group_f0[g] = g; s.group_nf[g] = 1; }
      h.nplanes = 1;
    } else {
      s.nf = 8;
      s.ngroups = 4;
      const int kinds[4] = {G_HARTREE, G_VW, G_WGC3, G_WGC3};
      const int f0[4] = {0, 1, 2, 5};
      const int nfg[4] = {1, 1, 3, 3};
      for (int g = 0; g < 4; ++g) { s.group_kind[g] = kinds[g]; s.group_f0[g] = f0[g]; s.group_nf[g] = nfg[g]; }
      h.nplanes = 4;
    }
    // launch geometry
    const long long nrows = (long long)s.n2 * s.n3;
    h.nrowpairs = (int)((nrows + 1) / 2);
    h.rp = std::max(1, std::min(16, 512 / s.n1));
    h.tx = h.prec == OFDFT_FP32 ? 16 : 8;
    s.ntask[K_VEC] = (int)((s.N + VCHUNK - 1) / VCHUNK);
    s.ntask[K_X5] = (h.nrowpairs + h.rp - 1) / h.rp;
    // buffers
    const size_t es = elem_size(h.prec);
    int rc;
    for (int b = 0; b < NBUF; ++b)
      if ((rc = alloc(h, &s.buf[b], es * s.N))) { free_slot(idx); return rc; }
    if ((rc = alloc(h, &s.vion, es * s.N))) { free_slot(idx); return rc; }
    if ((rc = alloc(h, &s.kern, es * s.Nc * h.nplanes))) { free_slot(idx); return rc; }
    if ((rc = alloc(h, &s.spec, 2 * es * s.Nc * s.nf))) { free_slot(idx); return rc; }
    const int ntmax = std::max(s.ntask[K_VEC], s.ntask[K_X5]);
    if ((rc = alloc(h, (void**)&s.partials, sizeof(double) * NCH * ntmax))) { free_slot(idx); return rc; }
    if ((rc = alloc(h, (void**)&s.done, sizeof(int) * NKID))) { free_slot(idx); return rc; }
    if ((rc = alloc(h, (void**)&s.hist, sizeof(HistEntry) * HIST_MAX))) { free_slot(idx); return rc; }
    if ((rc = upload_slot(idx))) { free_slot(idx); return rc; }
    Ctl c;
    memset(&c, 0, sizeof(c));
    c.status = ST_IDLE;
    if ((rc = h2d(d_ctl + idx, &c, sizeof(Ctl)))) { free_slot(idx); return rc; }
    dirty = true;
    *out = idx;
    return OFDFT_OK;
  }

  int check_slot(int i) {
    if (i < 0 || i >= cap || !slots[i].used) return fail(OFDFT_EINVAL, "invalid slot");
    if (slots[i].running) return fail(OFDFT_EBUSY, "slot is running");
    return OFDFT_OK;
  }

  // Upload a host FP64 array into a device array of the slot's precision.
  int upload_real(int prec, void* dst, const double* src, long long n) {
    if (prec == OFDFT_FP64) return h2d(dst, src, sizeof(double) * n);
    std::vector<float> t(n);
    for (long long i = 0; i < n; ++i) t[i] = (float)src[i];
    return h2d(dst, t.data(), sizeof(float) * n);
  }
  int download_real(int prec, double* dst, const void* src, long long n) {
    if (prec == OFDFT_FP64) return d2h(dst, src, sizeof(double) * n);
    std::vector<float> t(n);
    int rc = d2h(t.data(), src, sizeof(float) * n);
    for (long long i = 0; i < n; ++i) dst[i] = (double)t[i];
    return rc;
  }

  int get_ctl(int i, Ctl& c) { return d2h(&c, d_ctl + i, sizeof(Ctl)); }
  int put_ctl(int i, const Ctl& c) { return h2d(d_ctl + i, &c, sizeof(Ctl)); }

  void base_ctl(Ctl& c, int prec) {
    memset(&c, 0, sizeof(c));
    c.status = ST_RUNNING;
    c.iphi = B_PHI;
    c.itrial = B_TRIAL;
    c.iw0 = B_W0;
    c.iw1 = B_W1;
    c.evb = B_P;
    c.dscale = 1.0;
    c.macheps = prec == OFDFT_FP32 ? 1.1920928955078125e-07 : 2.220446049250313e-16;
  }

  int start_eval(int i, const double* rho, int opt_sqrt, int want_energy) {
    int rc = check_slot(i);
    if (rc) return rc;
    HostSlot& h = slots[i];
    if ((rc = upload_real(h.prec, h.sd.buf[B_PHI], rho, h.sd.N))) return rc;
    Ctl c;
    base_ctl(c, h.prec);
    c.ev = EV_RHO;
    c.opt_sqrt = opt_sqrt ? 1 : 0;
    c.want_energy = want_energy ? 1 : 0;
    if ((rc = put_ctl(i, c))) return rc;
    h.running = true;
    dirty = true;
    return OFDFT_OK;
  }

  void solve_ctl(Ctl& c, int prec, const ofdft_ntn_options* o) {
    base_ctl(c, prec);
    c.op = OP_SQRT_INIT;
    c.max_iter = (o && o->max_iter > 0) ? o->max_iter : 500;
    c.conv_check = o ? o->conv_check : CONV_ENE;
    c.pot_tol = (o && o->pot_tol > 0) ? o->pot_tol : 1.0e-5;
    c.tole = (o && o->tole > 0) ? o->tole : 1.0e-6;
    c.max_line = (o && o->max_line > 0) ? o->max_line : 200;
    c.outcome = -1;
  }

  int start_solve(int i, const double* rho, const ofdft_ntn_options* o) {
    int rc = check_slot(i);
    if (rc) return rc;
    HostSlot& h = slots[i];
    if ((rc = upload_real(h.prec, h.sd.buf[B_PHI], rho, h.sd.N))) return rc;
    Ctl c;
    solve_ctl(c, h.prec, o);
    if ((rc = put_ctl(i, c))) return rc;
    h.running = true;
    dirty = true;
    return OFDFT_OK;
  }

  // ---------------------------------------------------------- task lists
  int build_lists() {
    for (int p = 0; p < 2; ++p)
      for (int k = 0; k < NPASS; ++k) {
        lists[p][k].h.clear();
        lists[p][k].smem = 0;
      }
    for (int i = 0; i < cap; ++i) {
      HostSlot& h = slots[i];
      if (!h.used || !h.running) continue;
      const SlotDev& s = h.sd;
      LaunchList* L = lists[h.prec];
      const size_t cs = 2 * elem_size(h.prec);
      for (int t = 0; t < s.ntask[K_VEC]; ++t) L[P_VEC].h.push_back({i, t, 0, 0});
      L[P_VEC].nthr = 256;
      L[P_VEC].smem = std::max(L[P_VEC].smem, (size_t)(NCH * 256 * sizeof(double) + 16));
      for (int f = 0; f < s.nf; ++f)
        for (int r = 0; r < h.nrowpairs; r += h.rp)
          L[P_X1].h.push_back({i, f, r, std::min(h.rp, h.nrowpairs - r)});
      L[P_X1].nthr = 128;
      L[P_X1].smem = std::max(L[P_X1].smem, 2 * (size_t)h.rp * s.n1 * cs);
      for (int pass : {P_Y2, P_Y4}) {
        for (int f = 0; f < s.nf; ++f)
          for (int z = 0; z < s.n3; ++z)
            for (int kx = 0; kx < s.k1; kx += h.tx) L[pass].h.push_back({i, f, z, kx});
        L[pass].nthr = 128;
        L[pass].smem = std::max(L[pass].smem, 2 * (size_t)h.tx * s.n2 * cs);
      }
      for (int g = 0; g < s.ngroups; ++g)
        for (int ky = 0; ky < s.n2; ++ky)
          for (int kx = 0; kx < s.k1; kx += h.tx) L[P_Z3].h.push_back({i, g, ky, kx});
      L[P_Z3].nthr = 128;
      L[P_Z3].smem = std::max(L[P_Z3].smem, 4 * (size_t)h.tx * s.n3 * cs);
      int ord = 0;
      for (int r = 0; r < h.nrowpairs; r += h.rp) L[P_X5].h.push_back({i, r, std::min(h.rp, h.nrowpairs - r), ord++});
      L[P_X5].nthr = 128;
      L[P_X5].smem = std::max(L[P_X5].smem, (size_t)(s.nf + 1) * h.rp * s.n1 * cs + NCH * 128 * sizeof(double) + 16);
    }
#if defined(OFDFT_EMU)
    for (int p = 0; p < 2; ++p)
      for (int k = 0; k < NPASS; ++k) lists[p][k].nthr = 1;
#endif
    for (int p = 0; p < 2; ++p)
      for (int k = 0; k < NPASS; ++k) {
        LaunchList& l = lists[p][k];
        if (l.h.size() > l.cap) {
          dfree(l.d);
          l.d = nullptr;
          size_t nc = std::max<size_t>(l.h.size(), 2 * l.cap);
          int rc = dmalloc((void**)&l.d, nc * sizeof(Task));
          if (rc) return rc;
          l.cap = nc;
        }
        if (!l.h.empty()) {
          int rc = h2d(l.d, l.h.data(), l.h.size() * sizeof(Task));
          if (rc) return rc;
        }
      }
    dirty = false;
    return OFDFT_OK;
  }

  template <typename T>
  Args<T> args(int prec, int pass) {
    Args<T> a;
    a.slots = d_slots;
    a.ctl = d_ctl;
    a.tasks = lists[prec][pass].d;
    a.tw = (const cx<T>*)(prec == OFDFT_FP32 ? plans.d_tw32 : plans.d_tw64);
    a.tx = prec == OFDFT_FP32 ? 16 : 8;
    a.vchunk = VCHUNK;
    return a;
  }

#if defined(OFDFT_EMU)
  template <typename T>
  int launch_prec(int prec) {
    auto run = [&](int pass, auto fn) {
      LaunchList& l = lists[prec][pass];
      if (l.h.empty()) return;
      if (emu_smem.size() < l.smem + 64) emu_smem.assign(l.smem + 64, 0);
      Args<T> a = args<T>(prec, pass);
      for (int b = 0; b < (int)l.h.size(); ++b) fn(a, b, emu_smem.data());
    };
    for (int v = 0; v < VEC_PER_TICK; ++v)
      run(P_VEC, [](Args<T>& a, int b, char* sm) { vec_block<T>(a, b, 0, 1, sm); });
    run(P_X1, [](Args<T>& a, int b, char* sm) { xfwd_block<T>(a, b, 0, 1, sm); });
    run(P_Y2, [](Args<T>& a, int b, char* sm) { ypass_block<T>(a, b, 0, 1, sm, -1); });
    run(P_Z3, [](Args<T>& a, int b, char* sm) { zpass_block<T>(a, b, 0, 1, sm); });
    run(P_Y4, [](Args<T>& a, int b, char* sm) { ypass_block<T>(a, b, 0, 1, sm, 1); });
    run(P_X5, [](Args<T>& a, int b, char* sm) { xinv_block<T>(a, b, 0, 1, sm); });
    return OFDFT_OK;
  }
#else
  template <typename T, typename K, typename... X>
  int launch_one(int prec, int pass, K kern, X... extra) {
    LaunchList& l = lists[prec][pass];
    if (l.h.empty()) return OFDFT_OK;
    if (l.smem > 48 * 1024) {
      int rc = cuda_check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)l.smem),
                          "cudaFuncSetAttribute");
      if (rc) return rc;
    }
    kern<<<(unsigned)l.h.size(), l.nthr, l.smem>>>(args<T>(prec, pass), extra...);
    return cuda_check(cudaGetLastError(), "kernel launch");
  }
  template <typename T>
  int launch_prec(int prec) {
    int rc;
    for (int v = 0; v < VEC_PER_TICK; ++v)
      if ((rc = launch_one<T>(prec, P_VEC, k_vec<T>))) return rc;
    if ((rc = launch_one<T>(prec, P_X1, k_xfwd<T>))) return rc;
    if ((rc = launch_one<T>(prec, P_Y2, k_ypass<T>, -1))) return rc;
    if ((rc = launch_one<T>(prec, P_Z3, k_zpass<T>))) return rc;
    if ((rc = launch_one<T>(prec, P_Y4, k_ypass<T>, 1))) return rc;
    return launch_one<T>(prec, P_X5, k_xinv<T>);
  }
#endif

  int tick() {
    int rc;
    if (dirty && (rc = build_lists())) return rc;
    if ((rc = launch_prec<double>(OFDFT_FP64))) return rc;
    return launch_prec<float>(OFDFT_FP32);
  }

  // Run ticks; after every `check` ticks read the slots' status and retire
  // finished slots from the task lists.
  int run(int ticks, int* running_out, int check = 8) {
    int running = 0;
    for (int t = 0; t < ticks;) {
      int n = std::min(check, ticks - t);
      for (int k = 0; k < n; ++k) {
        int rc = tick();
        if (rc) return rc;
      }
      t += n;
      int rc = dsync();
      if (rc) return rc;
      running = 0;
      for (int i = 0; i < cap; ++i) {
        if (!slots[i].used || !slots[i].running) continue;
        Ctl c;
        if ((rc = get_ctl(i, c))) return rc;
        if (c.status == ST_RUNNING) {
          ++running;
        } else {
          slots[i].running = false;
          dirty = true;
        }
      }
      if (running == 0) break;
    }
    if (running_out) *running_out = running;
    return OFDFT_OK;
  }
};

static int status_code(const Ctl& c) {
  if (c.status == ST_ERROR) {
    switch (c.error) {
      case ERR_GRAD_TOO_LARGE: return fail(OFDFT_EGRAD, "The gradient is too large (dE/dtheta > 1e5)");
      case ERR_LINESEARCH: return fail(OFDFT_ELINESEARCH, "line search error past maxIter");
      default: return fail(OFDFT_ENAN, "non-finite value in a reduction");
    }
  }
  return OFDFT_OK;
}

}  // namespace ofdft

using namespace ofdft;

struct ofdft_engine {
  Engine eng;
};

extern "C" {

const char* ofdft_last_error(void) { return g_err.c_str(); }
int ofdft_version(void) { return 1; }

int ofdft_engine_create(ofdft_engine** out) {
  if (!out) return fail(OFDFT_EINVAL, "null output");
  ofdft_engine* e = new ofdft_engine();
  int rc = e->eng.init(64);
  if (rc) {
    e->eng.release();
    delete e;
    return rc;
  }
  *out = e;
  return OFDFT_OK;
}

int ofdft_engine_destroy(ofdft_engine* e) {
  if (!e) return OFDFT_OK;
  dsync();
  e->eng.release();
  delete e;
  return OFDFT_OK;
}

int ofdft_slot_create(ofdft_engine* e, const ofdft_cell_desc* d, int* slot) {
  if (!e || !slot) return fail(OFDFT_EINVAL, "null argument");
  return e->eng.create_slot(d, slot);
}

int ofdft_slot_destroy(ofdft_engine* e, int slot) {
  if (!e || slot < 0 || slot >= e->eng.cap) return fail(OFDFT_EINVAL, "invalid slot");
  dsync();
  e->eng.free_slot(slot);
  return OFDFT_OK;
}

int ofdft_slot_set_kernel(ofdft_engine* e, int slot, const double* kernel, int nplanes) {
  if (!e || !kernel) return fail(OFDFT_EINVAL, "null argument");
  int rc = e->eng.check_slot(slot);
  if (rc) return rc;
  HostSlot& h = e->eng.slots[slot];
  if (nplanes != h.nplanes) return fail(OFDFT_EINVAL, "kernel plane count does not match the functional");
  return e->eng.upload_real(h.prec, h.sd.kern, kernel, h.sd.Nc * nplanes);
}

int ofdft_slot_set_ion_potential(ofdft_engine* e, int slot, const double* v) {
  if (!e || !v) return fail(OFDFT_EINVAL, "null argument");
  int rc = e->eng.check_slot(slot);
  if (rc) return rc;
  HostSlot& h = e->eng.slots[slot];
  return e->eng.upload_real(h.prec, h.sd.vion, v, h.sd.N);
}

int ofdft_slot_start_eval(ofdft_engine* e, int slot, const double* rho, int opt_sqrt, int want_energy) {
  if (!e || !rho) return fail(OFDFT_EINVAL, "null argument");
  return e->eng.start_eval(slot, rho, opt_sqrt, want_energy);
}

int ofdft_slot_start_solve(ofdft_engine* e, int slot, const double* rho, const ofdft_ntn_options* o) {
  if (!e || !rho) return fail(OFDFT_EINVAL, "null argument");
  return e->eng.start_solve(slot, rho, o);
}

int ofdft_engine_run(ofdft_engine* e, int ticks, int* running) {
  if (!e) return fail(OFDFT_EINVAL, "null engine");
  return e->eng.run(ticks, running);
}

int ofdft_slot_poll(ofdft_engine* e, int slot, int* finished) {
  if (!e || !finished || slot < 0 || slot >= e->eng.cap || !e->eng.slots[slot].used)
    return fail(OFDFT_EINVAL, "invalid slot");
  *finished = e->eng.slots[slot].running ? 0 : 1;
  return OFDFT_OK;
}

int ofdft_slot_result(ofdft_engine* e, int slot, double* rho, double* energy, ofdft_ntn_stats* st) {
  if (!e) return fail(OFDFT_EINVAL, "null engine");
  int rc = e->eng.check_slot(slot);
  if (rc) return rc;
  Engine& g = e->eng;
  HostSlot& h = g.slots[slot];
  Ctl c;
  if ((rc = g.get_ctl(slot, c))) return rc;
  if (rho) {
    if ((rc = g.download_real(h.prec, rho, h.sd.buf[c.iphi], h.sd.N))) return rc;
    for (long long i = 0; i < h.sd.N; ++i) rho[i] = rho[i] * rho[i];  // rhoR = phi**2 (RhoOptN.f90:495)
  }
  if (energy)
    for (int k = 0; k < 9; ++k) energy[k] = c.energy[k];
  if (st) {
    st->outcome = c.outcome;
    st->iterations = c.iter;
    st->num_evals = c.num_evals;
    st->num_cg = c.num_cg;
    st->num_line = c.num_ls;
    st->history_len = std::min(c.hist_n, HIST_MAX);
    st->pot_norm = c.pot_norm;
    st->error = c.error;
  }
  return status_code(c);
}

int ofdft_slot_history(ofdft_engine* e, int slot, int max, double* energy, double* pot_norm, double* theta,
                       int* ncg, int* nline, int* n) {
  if (!e || !n) return fail(OFDFT_EINVAL, "null argument");
  int rc = e->eng.check_slot(slot);
  if (rc) return rc;
  Engine& g = e->eng;
  Ctl c;
  if ((rc = g.get_ctl(slot, c))) return rc;
  const int m = std::min(std::min(c.hist_n, HIST_MAX), max);
  std::vector<HistEntry> hs(HIST_MAX);
  if ((rc = d2h(hs.data(), g.slots[slot].sd.hist, sizeof(HistEntry) * HIST_MAX))) return rc;
  for (int i = 0; i < m; ++i) {
    if (energy) energy[i] = hs[i].energy;
    if (pot_norm) pot_norm[i] = hs[i].pot_norm;
    if (theta) theta[i] = hs[i].theta;
    if (ncg) ncg[i] = hs[i].ncg;
    if (nline) nline[i] = hs[i].nline;
  }
  *n = m;
  return OFDFT_OK;
}

int ofdft_slot_download(ofdft_engine* e, int slot, int which, double* out) {
  if (!e || !out) return fail(OFDFT_EINVAL, "null argument");
  int rc = e->eng.check_slot(slot);
  if (rc) return rc;
  Engine& g = e->eng;
  HostSlot& h = g.slots[slot];
  Ctl c;
  if ((rc = g.get_ctl(slot, c))) return rc;
  const void* src = which == 0 ? h.sd.buf[c.iphi] : which == 1 ? h.sd.buf[c.iw0] : h.sd.vion;
  if (which < 0 || which > 2) return fail(OFDFT_EINVAL, "which must be 0, 1 or 2");
  return g.download_real(h.prec, out, src, h.sd.N);
}

int ofdft_calculate_potential_plus(ofdft_engine* e, int slot, const double* rho, int opt_sqrt, double* potential,
                                   double* etable) {
  if (!e || !rho || !potential) return fail(OFDFT_EINVAL, "null argument");
  Engine& g = e->eng;
  int rc = g.start_eval(slot, rho, opt_sqrt, etable != nullptr);
  if (rc) return rc;
  int running = 1;
  if ((rc = g.run(8, &running, 1))) return rc;
  if (g.slots[slot].running) return fail(OFDFT_ETIMEOUT, "evaluation did not finish");
  Ctl c;
  if ((rc = g.get_ctl(slot, c))) return rc;
  if ((rc = status_code(c))) return rc;
  HostSlot& h = g.slots[slot];
  if ((rc = g.download_real(h.prec, potential, h.sd.buf[c.iw0], h.sd.N))) return rc;
  if (etable)
    for (int k = 0; k < 9; ++k) etable[k] = c.energy[k];
  return OFDFT_OK;
}

int ofdft_proj_norm_rho_minimization(ofdft_engine* e, int slot, double* rho, double* energy,
                                     const ofdft_ntn_options* o, ofdft_ntn_stats* st) {
  if (!e || !rho) return fail(OFDFT_EINVAL, "null argument");
  Engine& g = e->eng;
  int rc = g.start_solve(slot, rho, o);
  if (rc) return rc;
  const int max_ticks = (o && o->max_ticks > 0) ? o->max_ticks : 20000;
  int running = 1;
  if ((rc = g.run(max_ticks, &running, 8))) return rc;
  if (g.slots[slot].running) return fail(OFDFT_ETIMEOUT, "solve exceeded the tick budget");
  return ofdft_slot_result(e, slot, rho, energy, st);
}

int ofdft_slot_start_solve_from_slot(ofdft_engine*, int, int, const ofdft_ntn_options*) {
  return fail(OFDFT_EINVAL, "not available yet");
}
int ofdft_slot_build_wt_kernel(ofdft_engine*, int) { return fail(OFDFT_EINVAL, "not available yet"); }
int ofdft_slot_build_wgc_kernel(ofdft_engine*, int, int, const double*, const double*, const double*,
                                const double*) {
  return fail(OFDFT_EINVAL, "not available yet");
}
int ofdft_slot_build_ion_potential(ofdft_engine*, int, int, const double*, const int*, int, const int*,
                                   const double*, const double*, const double*, const double*, const double*) {
  return fail(OFDFT_EINVAL, "not available yet");
}

}  // extern "C"
