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
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "setup.cuh"
#include "ewald.cuh"
#include "stress.cuh"
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
static int dsync() { return cuda_check(cudaDeviceSynchronize(), "synchronize"); }
#endif

// Row pairs per x-pass block.  The x passes keep their nf*rp complex columns
// interleaved in shared memory ([x][column]), and their prologue and epilogue
// walk x across the threads of a warp, so consecutive threads are nf*rp
// complex values apart.  In FP64 an even count puts 2, 4 or 8 threads of a
// quarter-warp on the same banks (8-way at nf*rp = 24); an odd count spreads
// them over all 32 banks.  With an odd field count, one row pair fewer makes
// the count odd: -2 % FP64 evaluation time at 96^3.  (In FP32 the same
// change costs 2 %: the x passes there are bound by issue, not by banks.)
static int odd_columns(int nf, int rp, size_t csz) {
  return (csz == 16 && (nf & 1) && !(rp & 1) && rp > 1) ? rp - 1 : rp;
}

// Launch shape of a slot's passes: row pairs per x-forward task (*rp1) and
// per x-inverse task (s.rp), up to OFDFT_XPASS_POINTS / n1 of them, whose
// transform buffers (every field or ion species; the x-forward pass adds its
// staged input rows) fit OFDFT_XFWD_KB32 / OFDFT_XINV_KB32 (FP32) or
// OFDFT_XPASS_KB64 (FP64) KB of shared memory; and the tiles of the split y/z
// path: z columns per y-pass task (*ty: columns of n2 values at an odd row
// pitch) and y columns per z-pass task (*tz: a group of gmax fields of n3
// values each), each in about 48 KB, at least 32 columns when n allows.
// s needs n1..n3, k1, nf and kinetic; csz is the size of one complex value.
#ifndef OFDFT_XFWD_KB32
#define OFDFT_XFWD_KB32 48
#endif
#ifndef OFDFT_XINV_KB32
#define OFDFT_XINV_KB32 48
#endif
#ifndef OFDFT_XPASS_KB64
#define OFDFT_XPASS_KB64 72
#endif
#ifndef OFDFT_XPASS_POINTS
#define OFDFT_XPASS_POINTS 2048
#endif
static void launch_shape(SlotDev& s, size_t csz, int nfx, int* rp1, int* ty, int* tz) {
  const size_t esz = csz / 2;
  const size_t fkb = (size_t)(csz == 8 ? OFDFT_XFWD_KB32 : OFDFT_XPASS_KB64) * 1024;
  const size_t ikb = (size_t)(csz == 8 ? OFDFT_XINV_KB32 : OFDFT_XPASS_KB64) * 1024;
  *rp1 = std::max(1, std::min(32, OFDFT_XPASS_POINTS / s.n1));
  while (*rp1 > 1 && xfwd_smem(s.n1, nfx, *rp1, esz) > fkb) (*rp1)--;
  s.rp = std::max(1, std::min(32, OFDFT_XPASS_POINTS / s.n1));
  while (s.rp > 1 && xinv_smem(s.n1, s.nf, s.rp, esz) > ikb) s.rp--;
  *rp1 = odd_columns(s.nf, *rp1, csz);
  s.rp = odd_columns(s.nf, s.rp, csz);
  const int gmax = s.kinetic == KIN_WGC ? 3 : 1;
  const size_t ycol = (size_t)(s.n2 | 1) * csz, zcol = (size_t)gmax * s.n3 * csz;
  *ty = (int)std::max<size_t>(1, std::min<size_t>(s.n3, std::max<size_t>(48 * 1024 / ycol, 32)));
  *tz = (int)std::max<size_t>(1, std::min<size_t>(s.n2, std::max<size_t>(48 * 1024 / zcol, 32)));
  while (*ty > 1 && *ty * ycol > 160 * 1024) (*ty)--;
  while (*tz > 1 && *tz * zcol > 160 * 1024) (*tz)--;
}

// Shared memory of the fused y-z pass of one plane (rows of odd pitch), and
// the largest plane it takes (one block of up to 226 KB per SM: fused at
// 222 KB, a WGC 96^3 FP32 group ran 8 % faster than on the split path);
// bigger planes run the split y/z path.
static size_t yz_smem(const SlotDev& s, size_t csz) { return (size_t)s.n3 * (s.n2 | 1) * csz; }
// A WGC slot's fused pass holds the three planes of a WGC group at once
// (interleaved along y, odd pitch of 3*n2).
static size_t yz_smem_slot(const SlotDev& s, size_t csz) {
  return s.kinetic == KIN_WGC ? (size_t)s.n3 * ((3 * s.n2) | 1) * csz : yz_smem(s, csz);
}
constexpr size_t YZ_SMEM_MAX = 226 * 1024;
// Planes up to this size run 256-thread blocks (three per SM up to 75 KB, two
// up to 112 KB), larger ones one 512-thread block per SM.  Two 256-thread
// blocks beat one 512-thread block on 84-99 KB plane sets (WT 72^3 FP64,
// 108^3 FP32, WGC 64^3 FP32: 9-11 % faster evaluations).
constexpr size_t YZ_SMEM_SMALL = 112 * 1024;

// ------------------------------------------------------------ FFT plans
static bool seven_smooth(int n) {
  if (n < 1) return false;
  for (int p : {2, 3, 5, 7})
    while (n % p == 0) n /= p;
  return n == 1;
}

constexpr int MAX_N = 512;

// Radix caps the tuner may give an x-axis plan (the first is the default).
static const int kCaps[2][3] = {{12, 8, 0}, {16, 12, 8}};  // [0] FP64, [1] FP32

struct PlanTable {
  std::map<int, FftPlan> plans[2];  // [0] FP64 (OFDFT_FP64), [1] FP32: default radix cap
  std::map<int, FftPlan> capped[2];  // key cap * 1024 + n: the plans of the other caps
  void* d_tw64 = nullptr;           // exp(-2 pi i e / n), e < n, for every 7-smooth n <= MAX_N
  void* d_tw32 = nullptr;
  int* d_idx = nullptr;             // perm and iperm of every plan

  int build() {
    std::vector<long double> re, im;
    std::map<int, int> root_off;
    for (int n = 1; n <= MAX_N; ++n) {
      if (!seven_smooth(n)) continue;
      root_off[n] = (int)re.size();
      for (int e = 0; e < n; ++e) {
        const long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)e / (long double)n;
        re.push_back(cosl(ang));
        im.push_back(sinl(ang));
      }
    }
    std::vector<int> idx;
    for (int pi = 0; pi < 2; ++pi)
      for (int n = 1; n <= MAX_N; ++n) {
        if (!seven_smooth(n)) continue;
        for (int ci = 0; ci < 3 && kCaps[pi][ci]; ++ci) {
          int rad[FFT_MAX_STAGES];
          const int nst = fft_radices(n, kCaps[pi][ci], rad);
          FftPlan p;
          memset(&p, 0, sizeof(p));
          std::vector<int> perm(n), iperm(n);
          fft_plan_fill(p, n, rad, nst, perm.data(), iperm.data());
          p.root = root_off[n];
          p.perm = (int)idx.size();
          idx.insert(idx.end(), perm.begin(), perm.end());
          p.iperm = (int)idx.size();
          idx.insert(idx.end(), iperm.begin(), iperm.end());
          if (ci == 0) plans[pi][n] = p;
          else capped[pi][kCaps[pi][ci] * 1024 + n] = p;
        }
      }
    const size_t nt = re.size();
    std::vector<cx<double>> t64(nt);
    std::vector<cx<float>> t32(nt);
    for (size_t i = 0; i < nt; ++i) {
      t64[i] = mk<double>((double)re[i], (double)im[i]);
      t32[i] = mk<float>((float)re[i], (float)im[i]);
    }
    int rc = dmalloc(&d_tw64, nt * sizeof(cx<double>));
    if (!rc) rc = dmalloc(&d_tw32, nt * sizeof(cx<float>));
    if (!rc) rc = dmalloc((void**)&d_idx, idx.size() * sizeof(int));
    if (!rc) rc = h2d(d_tw64, t64.data(), nt * sizeof(cx<double>));
    if (!rc) rc = h2d(d_tw32, t32.data(), nt * sizeof(cx<float>));
    if (!rc) rc = h2d(d_idx, idx.data(), idx.size() * sizeof(int));
    return rc;
  }
  // The plan of length n with radix cap cap (0 or the default cap: the default plan).
  const FftPlan& get(int pi, int n, int cap) const {
    auto it = capped[pi].find(cap * 1024 + n);
    return it == capped[pi].end() ? plans[pi].at(n) : it->second;
  }
  void release() {
    dfree(d_tw64);
    dfree(d_tw32);
    dfree(d_idx);
    d_tw64 = d_tw32 = nullptr;
    d_idx = nullptr;
  }
};

// ------------------------------------------------------------ kernels
// Launch lists of one tick.  Passes 1, 3 and 5 have one list for the WT slots
// (P_X1, P_Z3, P_X5) and one for the WGC slots (P_X1G, P_Z3G, P_X5G), each
// launched with the kernel instantiated for that functional.  A slot takes
// either the fused y-z pass (P_YZ, or P_YZB for planes above YZ_SMEM_SMALL;
// P_YZG / P_YZBG for WGC slots, whose three-field groups share one task)
// or the split path (P_Y2, P_Z3/P_Z3G, P_Y4).
enum Pass : int { P_VEC = 0, P_X1 = 1, P_Y2 = 2, P_Z3 = 3, P_Y4 = 4, P_X5 = 5, P_CTL = 6,
                  P_X1G = 7, P_Z3G = 8, P_X5G = 9, P_YZ = 10, P_YZB = 11, P_YZG = 12, P_YZBG = 13,
                  NPASS = 14 };
constexpr int VEC_PER_TICK = 2;
constexpr int VCHUNK = 4096;

// Minimum resident 256-thread blocks per SM of the x and split y/z pass
// kernels per precision (it caps their registers at 65536 / (256 * minb)).
#ifndef OFDFT_MINB_FP32
#define OFDFT_MINB_FP32 4
#endif
#ifndef OFDFT_MINB_FP64
#define OFDFT_MINB_FP64 3
#endif
template <typename T> struct PassMinBlocks { static constexpr int value = OFDFT_MINB_FP32; };
template <> struct PassMinBlocks<double> { static constexpr int value = OFDFT_MINB_FP64; };
// The x-inverse pass (transform, then the real-space epilogue of two points
// per work item) separately: its FP64 epilogue needs more registers.
#ifndef OFDFT_XINV_MINB_FP64
#define OFDFT_XINV_MINB_FP64 3
#endif
#ifndef OFDFT_XINV_MINB_FP32
#define OFDFT_XINV_MINB_FP32 OFDFT_MINB_FP32
#endif
template <typename T> struct XinvMinBlocks { static constexpr int value = OFDFT_XINV_MINB_FP32; };
template <> struct XinvMinBlocks<double> { static constexpr int value = OFDFT_XINV_MINB_FP64; };

#if !defined(OFDFT_EMU)
template <typename T> __global__ void __launch_bounds__(256) k_vec(Args<T> a) {
  extern __shared__ __align__(16) char sm[];
  vec_block<T>(a, blockIdx.x, threadIdx.x, blockDim.x, sm);
}
template <typename T, int KS> __global__ void __launch_bounds__(256, PassMinBlocks<T>::value) k_xfwd(Args<T> a) {
  extern __shared__ __align__(16) char sm[];
  xfwd_block<T, KS>(a, blockIdx.x, threadIdx.x, blockDim.x, sm);
}
template <typename T> __global__ void __launch_bounds__(256, PassMinBlocks<T>::value) k_ypass(Args<T> a, int dir) {
  extern __shared__ __align__(16) char sm[];
  ypass_block<T>(a, blockIdx.x, threadIdx.x, blockDim.x, sm, dir);
}
template <typename T, int KS> __global__ void __launch_bounds__(256, PassMinBlocks<T>::value) k_zpass(Args<T> a) {
  extern __shared__ __align__(16) char sm[];
  zpass_block<T, KS>(a, blockIdx.x, threadIdx.x, blockDim.x, sm);
}
// Fused y-z pass: 256-thread blocks, up to three per SM, for planes up to
// YZ_SMEM_SMALL; 512-thread blocks, one per SM, for larger planes.
template <typename T, int NT, int KS>
__global__ void __launch_bounds__(NT, NT == 256 ? 3 : 1) k_yzpass(Args<T> a) {
  extern __shared__ __align__(16) char sm[];
  yzpass_block<T, KS>(a, blockIdx.x, threadIdx.x, blockDim.x, sm);
}
template <typename T, int KS> __global__ void __launch_bounds__(256, XinvMinBlocks<T>::value) k_xinv(Args<T> a) {
  extern __shared__ __align__(16) char sm[];
  xinv_block<T, KS>(a, blockIdx.x, threadIdx.x, blockDim.x, sm);
}
// keKernel planes from the reference layout (k1, n2, n3), x fastest, into
// the engine's kx-major digit-reversed layout.
template <typename T> __global__ void __launch_bounds__(256) k_permute_kernel(const SlotDev* sd, const int* idx,
                                                                             const double* src, int nplanes) {
  const SlotDev& s = *sd;
  const long long total = s.Nc * nplanes;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
    ((T*)s.kern)[i] = (T)src[kernel_source_index(s, idx, i)];
}
// keKernel planes of a slot back into the reference layout (FP64).
template <typename T> __global__ void __launch_bounds__(256) k_unpermute_kernel(const SlotDev* sd, const int* idx,
                                                                               double* dst, int nplanes) {
  const SlotDev& s = *sd;
  const long long total = s.Nc * nplanes;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
    dst[kernel_source_index(s, idx, i)] = (double)((const T*)s.kern)[i];
}
template <typename T> __global__ void __launch_bounds__(256) k_fill_kernel(const SlotDev* sd, const int* idx,
                                                                          KernArgs ka, int kind) {
  const SlotDev& s = *sd;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (int)s.Nc; i += gridDim.x * blockDim.x)
    fill_kernel_point<T>(s, idx, ka, kind, i);
}
template <typename T> __global__ void __launch_bounds__(256) k_spread(const SlotDev* sd, const IonStencil* st) {
  for (int w = threadIdx.x; w < SPLINE_ORDER * SPLINE_ORDER * SPLINE_ORDER; w += blockDim.x)
    spread_ion<T>(*sd, st[blockIdx.x], w);
}
template <typename T> __global__ void __launch_bounds__(256) k_force_gather(const SlotDev* sd, const IonStencil* st,
                                                                           double* out) {
  __shared__ double red[3][256];
  double f3[3] = {0, 0, 0};
  for (int w = threadIdx.x; w < SPLINE_ORDER * SPLINE_ORDER * SPLINE_ORDER; w += blockDim.x)
    force_term<T>(*sd, st[blockIdx.x], w, f3);
  for (int k = 0; k < 3; ++k) red[k][threadIdx.x] = f3[k];
  __syncthreads();
  for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
    if ((int)threadIdx.x < stride)
      for (int k = 0; k < 3; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + stride];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) out[3 * blockIdx.x + k] = red[k][0];
}
template <typename S, typename D> __global__ void __launch_bounds__(256) k_square_copy(const S* src, D* dst, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = (double)src[i];
    dst[i] = (D)(v * v);
  }
}
template <typename S, typename D> __global__ void __launch_bounds__(256) k_convert(const S* src, D* dst, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = (D)src[i];
}
template <typename T> __global__ void __launch_bounds__(64) k_ctl(Args<T> a, int kid) {
  __shared__ double sm[CTL_SMEM_BYTES / sizeof(double)];
  ctl_block(a.slots, a.ctl, a.tasks, kid, blockIdx.x, threadIdx.x, blockDim.x, (char*)sm);
}
#endif

struct LaunchList {
  std::vector<Task> h;
  Task* d = nullptr;  // its part of the engine's packed device array
  size_t smem = 0;
  int nthr = 128;
};

struct HostSlot {
  bool used = false;
  bool running = false;
  int prec = 0;
  SlotDev sd;
  std::vector<std::pair<void*, size_t>> allocs;  // device blocks and their sizes
  int nrowpairs = 0, rp1 = 1;
  int ty = 1, tz = 1;           // z columns per y-pass task and y columns per z-pass task (split path)
  int xcap = 0;                 // radix cap of the x-axis plan (0: the default)
  int yzt = 0;                  // threads of the fused y-z pass (0: by plane size)
  bool setup_pass = false;      // running an ion-potential or force pass (split path)
  int nplanes = 0;
  int nion = 0;                 // ions of the last ion-potential build
  IonStencil* d_stencil = nullptr;
  std::vector<IonStencil> stencils;
  double cell_inv_t[9];         // TRANSPOSE(Inverse(cellReal)), row-major
  double lattice[9];
  double rho0 = 0, gamma = 2.7;
  std::vector<double> frac, zion;
  void* input = nullptr;        // device-resident input density (ofdft_slot_set_input)
  size_t input_bytes = 0, stencil_bytes = 0;  // pooled sizes of input and d_stencil
  // pseudopotential tables and B-spline factors of the last ion-potential build
  // (device copy, and the host copy they were uploaded from)
  void* ion_aux = nullptr;
  size_t ion_aux_bytes = 0, ion_aux_cap = 0;  // bytes in use, pooled size
  std::vector<double> ion_tab;
  IonAux ion_ax;
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
  long long n_launches = 0, n_ticks = 0;
  int num_sms = 1;
  long long launches_per_tick() const {
    long long n = 0;
    for (int p = 0; p < 2; ++p)
      for (int k = 0; k < NPASS; ++k)
        if (!lists[p][k].h.empty()) n += (k == P_VEC ? VEC_PER_TICK : k == P_CTL ? VEC_PER_TICK + 1 : 1);
    return n;
  }
#if defined(OFDFT_EMU)
  int d2h_stream(void* h, const void* d, size_t n) { return d2h(h, d, n); }
#else
  cudaStream_t stream = nullptr;
  // A captured graph of ticks with running slots of both precisions forks
  // into an FP64 and an FP32 branch (the two share no slot, task list or
  // table they write): stream2 carries the FP32 branch during the capture,
  // and lstream is the stream the tick launches go to.
  cudaStream_t stream2 = nullptr;
  cudaStream_t lstream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  int graph_ticks = 0;
  int d2h_stream(void* h, const void* d, size_t n) {
    int rc = cuda_check(cudaMemcpyAsync(h, d, n, cudaMemcpyDeviceToHost, stream), "D2H async");
    if (rc) return rc;
    return cuda_check(cudaStreamSynchronize(stream), "stream synchronize");
  }
  // The engine's copies, fills and zeroed allocations go through its own
  // (non-blocking) stream and return once they are complete.  Plain
  // cudaMemcpy/cudaMemset run on the legacy default stream, which a
  // non-blocking stream does not wait for: a kernel launched right after them
  // could read the old contents (a device-to-device copy or a memset returns
  // to the host before it has run).
  int on_stream(cudaError_t e, const char* what) {
    int rc = cuda_check(e, what);
    return rc ? rc : cuda_check(cudaStreamSynchronize(stream), "stream synchronize");
  }
  int h2d(void* d, const void* h, size_t n) {
    return on_stream(cudaMemcpyAsync(d, h, n, cudaMemcpyHostToDevice, stream), "H2D");
  }
  int d2h(void* h, const void* d, size_t n) {
    return on_stream(cudaMemcpyAsync(h, d, n, cudaMemcpyDeviceToHost, stream), "D2H");
  }
  int d2d(void* d, const void* s, size_t n) {
    return on_stream(cudaMemcpyAsync(d, s, n, cudaMemcpyDeviceToDevice, stream), "D2D");
  }
  int dzero(void* d, size_t n) { return on_stream(cudaMemsetAsync(d, 0, n, stream), "cudaMemsetAsync"); }
  int dmalloc(void** p, size_t n) {
    int rc = cuda_check(cudaMalloc(p, n ? n : 1), "cudaMalloc");
    if (rc) {
      cudaGetLastError();  // a failed allocation must not show up as a later launch error
      return rc;
    }
    return dzero(*p, n ? n : 1);
  }
#endif

  int init(int capacity) {
    cap = capacity;
    slots.resize(cap);
#if !defined(OFDFT_EMU)
    int rs = cuda_check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream create");
    if (rs) return rs;
    if ((rs = cuda_check(cudaStreamCreateWithFlags(&stream2, cudaStreamNonBlocking), "stream create"))) return rs;
    if ((rs = cuda_check(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming), "event create"))) return rs;
    if ((rs = cuda_check(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming), "event create"))) return rs;
    lstream = stream;
    int dev = 0;
    if ((rs = cuda_check(cudaGetDevice(&dev), "get device"))) return rs;
    if ((rs = cuda_check(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev), "SM count"))) return rs;
#endif
    int rc = dmalloc((void**)&d_slots, sizeof(SlotDev) * cap);
    if (rc) return rc;
    rc = dmalloc((void**)&d_ctl, sizeof(Ctl) * cap);
    if (rc) return rc;
    if ((rc = plans.build())) return rc;
#if !defined(OFDFT_EMU)
    if ((rc = preload_kernels())) return rc;
#endif
    return dsync();  // the plan tables were copied on the legacy stream
  }

  void release() {
#if !defined(OFDFT_EMU)
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    graph_exec = nullptr;
    if (stream) cudaStreamSynchronize(stream);
#endif
    for (int i = 0; i < cap; ++i) free_slot(i);
    pool_flush();
    dfree(d_tasks);
    d_tasks = nullptr;
    dfree(d_slots);
    dfree(d_ctl);
    plans.release();
#if !defined(OFDFT_EMU)
    dfree(d_io);
    d_io = nullptr;
    if (stream) cudaStreamDestroy(stream);
    if (stream2) cudaStreamDestroy(stream2);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    stream = stream2 = lstream = nullptr;
    ev_fork = ev_join = nullptr;
#endif
  }

  // Device memory of destroyed slots, kept for reuse: a serving engine creates
  // and destroys slots all the time, and cudaMalloc / cudaFree (which
  // synchronises the device) cost far more than reuse.  A request takes the
  // smallest pooled block of at least its size and at most twice it; the
  // bytes it needs are zeroed like a new block's.  The pool is released when
  // an allocation fails, and holds at most POOL_MAX bytes.
  std::multimap<size_t, void*> pool;
  size_t pool_bytes = 0;
  static constexpr size_t POOL_MAX = size_t(32) << 30;
  int pmalloc(void** p, size_t n, size_t* got) {
    n = n ? n : 1;
    auto it = pool.lower_bound(n);  // the smallest pooled block that holds n bytes, if at most 2n
    if (it != pool.end() && it->first <= 2 * n) {
      *p = it->second;
      *got = it->first;
      pool_bytes -= it->first;
      pool.erase(it);
      return dzero(*p, n);
    }
    *got = n;
    int rc = dmalloc(p, n);
    if (rc == OFDFT_ENOMEM && !pool.empty()) {
      pool_flush();
      rc = dmalloc(p, n);
    }
    return rc;
  }
  void pfree(void* p, size_t n) {
    if (!p) return;
    n = n ? n : 1;
    if (pool_bytes + n > POOL_MAX) {
      dfree(p);
      return;
    }
    pool.emplace(n, p);
    pool_bytes += n;
  }
  void pool_flush() {
    for (auto& kv : pool) dfree(kv.second);
    pool.clear();
    pool_bytes = 0;
  }

  void free_slot(int i) {
    HostSlot& h = slots[i];
    for (auto& a : h.allocs) pfree(a.first, a.second);
    h.allocs.clear();
    pfree(h.d_stencil, h.stencil_bytes);
    h.d_stencil = nullptr;
    h.stencil_bytes = 0;
    h.nion = 0;
    pfree(h.input, h.input_bytes);
    h.input = nullptr;
    h.input_bytes = 0;
    pfree(h.ion_aux, h.ion_aux_cap);
    h.ion_aux = nullptr;
    h.ion_aux_bytes = h.ion_aux_cap = 0;
    h.ion_tab.clear();
    h.used = false;
    h.running = false;
    dirty = true;
  }

  int alloc(HostSlot& h, void** p, size_t bytes) {
    size_t got = 0;
    int rc = pmalloc(p, bytes, &got);
    if (rc == OFDFT_OK) h.allocs.push_back({*p, got});
    return rc;
  }
  // A block of the pool for a slot's single buffers (input density, ion
  // stencils, ion tables): its pooled size is kept in *size.
  int palloc(void** p, size_t bytes, size_t* size) { return pmalloc(p, bytes, size); }

  int upload_slot(int i) { return h2d(d_slots + i, &slots[i].sd, sizeof(SlotDev)); }

  // Lattice-dependent fields of a slot: cellRecip = TRANSPOSE(Inverse(cellReal))
  // * 2 pi (CellInfo.f90:281), volume, dV, and the inverse for the forces.
  static int set_geometry(HostSlot& h, const double* L) {  // L[3*i + k] = component k of vector i
    SlotDev& s = h.sd;
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
    for (int k = 0; k < 9; ++k) h.lattice[k] = L[k];
    for (int r = 0; r < 3; ++r)
      for (int c2 = 0; c2 < 3; ++c2) h.cell_inv_t[3 * r + c2] = inv[c2][r];
    return OFDFT_OK;
  }

  // A new lattice for slot i (RefreshLattice, Source/CellInfo.f90, with the
  // reference densities of KEDFRefresh, Source/SetupKEDF.f90:620-680): the
  // kernel, ion potential and Ewald energy must be rebuilt after it.
  int set_lattice(int i, const double* L, double rho0, double rho_s) {
    int rc = check_slot(i);
    if (rc) return rc;
    HostSlot& h = slots[i];
    HostSlot saved = h;
    if ((rc = set_geometry(h, L))) {
      h = saved;
      return rc;
    }
    h.rho0 = rho0;
    h.sd.rho_s = rho_s;
    return upload_slot(i);
  }

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
    const int pi = d->precision == OFDFT_FP32 ? 1 : 0;
    s.px = plans.plans[pi][d->n1];
    s.py = plans.plans[pi][d->n2];
    s.pz = plans.plans[pi][d->n3];
    if (int rc = set_geometry(h, d->lattice)) {
      h.used = false;
      return rc;
    }
    h.rho0 = d->rho0;
    h.gamma = d->gamma;
    s.inv_n = 1.0 / (double)s.N;
    s.kinetic = d->kinetic;
    s.lambda = d->lambda;
    s.mu = d->mu;
    s.alpha = d->alpha;
    s.beta = d->beta;
    s.rho_s = d->rho_s;
    s.ion_ion = d->ion_ion_energy;
    s.alpha_eq_beta = (d->alpha == d->beta) ? 1 : 0;
    s.pow56 = (s.alpha_eq_beta && std::fabs(d->alpha - 5.0 / 6.0) < 1e-15) ? 1 : 0;
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
    const size_t csz = 2 * elem_size(h.prec);
    launch_shape(s, csz, std::max(s.nf, MAX_SPECIES), &h.rp1, &h.ty, &h.tz);
    s.ntask[K_VEC] = (int)((s.N + VCHUNK - 1) / VCHUNK);
    s.ntask[K_X5] = (h.nrowpairs + s.rp - 1) / s.rp;
    // buffers
    const size_t es = elem_size(h.prec);
    int rc;
    for (int b = 0; b < NBUF; ++b)
      if ((rc = alloc(h, &s.buf[b], es * s.N))) { free_slot(idx); return rc; }
    if ((rc = alloc(h, &s.vion, es * s.N))) { free_slot(idx); return rc; }
    if ((rc = alloc(h, &s.kern, es * s.Nc * h.nplanes))) { free_slot(idx); return rc; }
    if ((rc = alloc(h, &s.spec, 2 * es * s.Nc * s.nf))) { free_slot(idx); return rc; }
    const int ntmax = std::max(s.ntask[K_VEC], h.nrowpairs);  // any x-inverse task size the tuner picks
    if ((rc = alloc(h, (void**)&s.partials, sizeof(double) * NCH * ntmax))) { free_slot(idx); return rc; }
    if ((rc = alloc(h, (void**)&s.hist, sizeof(HistEntry) * HIST_MAX))) { free_slot(idx); return rc; }
    auto tuned = tune_cache.find(tune_key(h));
    if (tuned != tune_cache.end()) set_shape(h, tuned->second);
    if ((rc = upload_slot(idx))) { free_slot(idx); return rc; }
    Ctl c;
    memset(&c, 0, sizeof(c));
    c.status = ST_IDLE;
    if ((rc = h2d(d_ctl + idx, &c, sizeof(Ctl)))) { free_slot(idx); return rc; }
    dirty = true;
    *out = idx;
    return OFDFT_OK;
  }

  // ---------------------------------------------------------- set-up on the device
  int sync_stream() {
#if defined(OFDFT_EMU)
    return OFDFT_OK;
#else
    return cuda_check(cudaStreamSynchronize(stream), "stream synchronize");
#endif
  }

  int launch_fill(int i, const KernArgs& ka, int kind) {
    HostSlot& h = slots[i];
#if defined(OFDFT_EMU)
    for (int idx = 0; idx < (int)h.sd.Nc; ++idx) {
      if (h.prec == OFDFT_FP32) fill_kernel_point<float>(h.sd, plans.d_idx, ka, kind, idx);
      else fill_kernel_point<double>(h.sd, plans.d_idx, ka, kind, idx);
    }
    return OFDFT_OK;
#else
    const int blocks = (int)std::min<long long>(4096, (h.sd.Nc + 255) / 256);
    if (h.prec == OFDFT_FP32) k_fill_kernel<float><<<blocks, 256, 0, stream>>>(d_slots + i, plans.d_idx, ka, kind);
    else k_fill_kernel<double><<<blocks, 256, 0, stream>>>(d_slots + i, plans.d_idx, ka, kind);
    int rc = cuda_check(cudaGetLastError(), "fill kernel launch");
    return rc ? rc : sync_stream();
#endif
  }

  int build_wt_kernel(int i) {
    int rc = check_slot(i);
    if (rc) return rc;
    HostSlot& h = slots[i];
    const SlotDev& s = h.sd;
    if (s.kinetic != KIN_WT) return fail(OFDFT_EINVAL, "the slot's functional is not WT");
    if (!(h.rho0 > 0)) return fail(OFDFT_EINVAL, "rho0 must be positive to build the WT kernel");
    KernArgs ka;
    memset(&ka, 0, sizeof(ka));
    lind_series(ka.ser);
    ka.lam = s.lambda;
    ka.mu = s.mu;
    ka.coef = 5.0 / (9.0 * s.alpha * s.beta * std::pow(h.rho0, s.alpha + s.beta - 5.0 / 3.0));
    ka.tkf = 2.0 * std::pow(3.0 * h.rho0 * PI_D * PI_D, 1.0 / 3.0);
    return launch_fill(i, ka, KIN_WT);
  }

  int build_wgc_kernel(int i, int ntab, const double* eta, const double* w, const double* w1, const double* w2) {
    int rc = check_slot(i);
    if (rc) return rc;
    HostSlot& h = slots[i];
    const SlotDev& s = h.sd;
    if (s.kinetic != KIN_WGC) return fail(OFDFT_EINVAL, "the slot's functional is not WGC");
    if (!(s.rho_s > 0)) return fail(OFDFT_EINVAL, "rho_s must be positive to build the WGC kernel");
    std::vector<double> te, tw, tw1, tw2;
    if (ntab > 1 && eta && w && w1 && w2) {
      te.assign(eta, eta + ntab);
      tw.assign(w, w + ntab);
      tw1.assign(w1, w1 + ntab);
      tw2.assign(w2, w2 + ntab);
    } else if (wgc_radial_tables(s.alpha, s.beta, h.gamma, te, tw, tw1, tw2)) {
      return fail(OFDFT_EINVAL, "WGC kernel ODE did not converge");
    }
    const int n = (int)te.size();
    std::vector<double> tab(7 * (size_t)n);
    std::vector<double> pp = spline_cubic_set(te, tw, 0, 0.0, 0, 0.0);
    std::vector<double> pp1 = spline_cubic_set(te, tw1, 0, 0.0, 0, 0.0);
    std::vector<double> pp2 = spline_cubic_set(te, tw2, 0, 0.0, 0, 0.0);
    for (int k = 0; k < n; ++k) {
      tab[k] = te[k]; tab[n + k] = tw[k]; tab[2 * n + k] = tw1[k]; tab[3 * n + k] = tw2[k];
      tab[4 * n + k] = pp[k]; tab[5 * n + k] = pp1[k]; tab[6 * n + k] = pp2[k];
    }
    double* dtab = nullptr;
    if ((rc = dmalloc((void**)&dtab, sizeof(double) * tab.size()))) return rc;
    if ((rc = h2d(dtab, tab.data(), sizeof(double) * tab.size()))) { dfree(dtab); return rc; }
    KernArgs ka;
    memset(&ka, 0, sizeof(ka));
    ka.rho_s = s.rho_s;
    ka.gamma = h.gamma;
    ka.tkf = 2.0 * std::pow(3.0 * PI_D * PI_D * s.rho_s, 1.0 / 3.0);
    ka.ntab = n;
    ka.tab = dtab;
    rc = launch_fill(i, ka, KIN_WGC);
    dfree(dtab);
    return rc;
  }

  int build_ion_potential(int i, int nion, const double* frac, const int* species, int nspec, const int* npts,
                          const double* max_g, const double* charge, const double* pot_values, const double* vqs,
                          const double* pot_dd) {
    int rc = check_slot(i);
    if (rc) return rc;
    HostSlot& h = slots[i];
    SlotDev& s = h.sd;
    if (nion < 1 || nspec < 1 || nspec > MAX_SPECIES || nspec > s.nf)
      return fail(OFDFT_EINVAL, "bad ion or species count for this slot");
    std::vector<double> tab;
    IonAux ax;
    memset(&ax, 0, sizeof(ax));
    ax.nspec = nspec;
    int off_in = 0;
    for (int sp = 0; sp < nspec; ++sp) {
      if (npts[sp] < 4) return fail(OFDFT_EINVAL, "pseudopotential table too short");
      PspDev& p = ax.psp[sp];
      p.npts = npts[sp];
      p.off = (int)tab.size();
      p.max_g = max_g[sp];
      p.charge = charge[sp];
      p.v0 = pot_values[off_in];
      p.dq = max_g[sp] / (double)(npts[sp] - 1);
      tab.insert(tab.end(), vqs + off_in, vqs + off_in + npts[sp]);
      tab.insert(tab.end(), pot_dd + off_in, pot_dd + off_in + npts[sp]);
      off_in += npts[sp];
    }
    for (int k = 0; k < nion; ++k)
      if (species[k] < 0 || species[k] >= nspec) return fail(OFDFT_EINVAL, "ion species index out of range");
    // The tables go to the device once per species set: a geometry step that
    // only moves the ions reuses them (and their device buffer).
    const bool same_tables = h.ion_aux && h.ion_tab == tab && h.ion_ax.nspec == nspec &&
                             memcmp(h.ion_ax.psp, ax.psp, sizeof(ax.psp)) == 0;
    if (same_tables) {
      ax = h.ion_ax;
    } else {
      const std::vector<cx<double>> b1 = bspline_b(s.k1, s.n1), b2 = bspline_b(s.n2, s.n2), b3 = bspline_b(s.n3, s.n3);
      const size_t bytes = sizeof(double) * tab.size() + sizeof(cx<double>) * (b1.size() + b2.size() + b3.size());
      if (h.ion_aux_bytes != bytes) {
        pfree(h.ion_aux, h.ion_aux_cap);
        h.ion_aux = nullptr;
        h.ion_aux_bytes = h.ion_aux_cap = 0;
        if ((rc = palloc(&h.ion_aux, bytes, &h.ion_aux_cap))) return rc;
        h.ion_aux_bytes = bytes;
      }
      char* cur = (char*)h.ion_aux;
      if ((rc = h2d(cur, tab.data(), sizeof(double) * tab.size()))) return rc;
      ax.tab = (const double*)cur;
      cur += sizeof(double) * tab.size();
      if ((rc = h2d(cur, b1.data(), sizeof(cx<double>) * b1.size()))) return rc;
      ax.b1 = (const cx<double>*)cur;
      cur += sizeof(cx<double>) * b1.size();
      if ((rc = h2d(cur, b2.data(), sizeof(cx<double>) * b2.size()))) return rc;
      ax.b2 = (const cx<double>*)cur;
      cur += sizeof(cx<double>) * b2.size();
      if ((rc = h2d(cur, b3.data(), sizeof(cx<double>) * b3.size()))) return rc;
      ax.b3 = (const cx<double>*)cur;
      h.ion_tab = tab;
      h.ion_ax = ax;
    }
    s.ion = ax;
    if ((rc = upload_slot(i))) return rc;
    // ion stencils (kept for the forces)
    const int nn[3] = {s.n1, s.n2, s.n3};
    h.stencils.clear();
    h.frac.assign(frac, frac + 3 * nion);
    h.zion.resize(nion);
    for (int k = 0; k < nion; ++k) {
      h.stencils.push_back(ion_stencil(frac + 3 * k, species[k], nn));
      h.zion[k] = charge[species[k]];
    }
    if (h.nion != nion) {
      pfree(h.d_stencil, h.stencil_bytes);
      h.d_stencil = nullptr;
      h.stencil_bytes = 0;
      h.nion = 0;
      if ((rc = palloc((void**)&h.d_stencil, sizeof(IonStencil) * nion, &h.stencil_bytes))) return rc;
      h.nion = nion;
    }
    if ((rc = h2d(h.d_stencil, h.stencils.data(), sizeof(IonStencil) * nion))) return rc;
    const size_t es = elem_size(h.prec);
    for (int sp = 0; sp < nspec; ++sp)
      if ((rc = dzero(s.buf[B_PHI + sp], es * s.N))) return rc;
#if defined(OFDFT_EMU)
    for (int k = 0; k < nion; ++k)
      for (int w = 0; w < SPLINE_ORDER * SPLINE_ORDER * SPLINE_ORDER; ++w) {
        if (h.prec == OFDFT_FP32) spread_ion<float>(s, h.stencils[k], w);
        else spread_ion<double>(s, h.stencils[k], w);
      }
#else
    if (h.prec == OFDFT_FP32) k_spread<float><<<nion, 256, 0, stream>>>(d_slots + i, h.d_stencil);
    else k_spread<double><<<nion, 256, 0, stream>>>(d_slots + i, h.d_stencil);
    if ((rc = cuda_check(cudaGetLastError(), "spread launch"))) return rc;
    if ((rc = sync_stream())) return rc;
#endif
    Ctl c;
    base_ctl(c, h.prec);
    c.ev = EV_ION;
    if ((rc = put_ctl(i, c))) return rc;
    return run_one(i);
  }

  // Stop a running slot: its controller goes idle and it leaves the task lists.
  int cancel(int i) {
    if (i < 0 || i >= cap || !slots[i].used) return fail(OFDFT_EINVAL, "invalid slot");
    if (!slots[i].running) return OFDFT_OK;
    Ctl c;
    int rc = get_ctl(i, c);
    if (rc) return rc;
    c.status = ST_IDLE;
    if ((rc = put_ctl(i, c))) return rc;
    slots[i].running = false;
    dirty = true;
    return OFDFT_OK;
  }

  // Run a slot that needs a single evaluation tick (the ion-potential and
  // force set-up passes, which take the split y/z path).  The tick advances
  // every running slot; it is repeated (up to 4 times) only while this slot
  // has not finished, so the other solves are not held in un-graphed ticks.
  int run_one(int i) {
    slots[i].running = true;
    slots[i].setup_pass = true;
    dirty = true;
    int running = 0;
    int rc = OFDFT_OK;
    for (int t = 0; t < 4 && slots[i].running && rc == OFDFT_OK; ++t) rc = run(1, &running, 1);
    slots[i].setup_pass = false;
    dirty = true;
    if (rc) return rc;
    if (slots[i].running) return fail(OFDFT_ETIMEOUT, "set-up pass did not finish");
    Ctl c;
    if ((rc = get_ctl(i, c))) return rc;
    return c.status == ST_DONE ? OFDFT_OK : fail(OFDFT_ENAN, "set-up pass failed");
  }

  int forces(int i, const double* rho, int include_ewald, double* out) {
    int rc = check_slot(i);
    if (rc) return rc;
    HostSlot& h = slots[i];
    SlotDev& s = h.sd;
    if (h.nion < 1 || s.ion.nspec < 1) return fail(OFDFT_EINVAL, "build the ion potential before the forces");
    Ctl c;
    if ((rc = get_ctl(i, c))) return rc;
    const int iphi = c.iphi;  // the current phi (a new slot's record is zero: B_PHI)
    base_ctl(c, h.prec);
    c.iphi = iphi;
    c.ev = EV_FORCE;
    c.ca = 1.0;
    c.cb = 0.0;
    if (rho) {
      if ((rc = upload_real(h.prec, s.buf[B_PHI], rho, s.N))) return rc;
      c.iphi = B_PHI;
      c.force_rho = 1;
    }
    if ((rc = put_ctl(i, c))) return rc;
    if ((rc = run_one(i))) return rc;
    std::vector<double> q(3 * (size_t)h.nion, 0.0);
#if defined(OFDFT_EMU)
    for (int k = 0; k < h.nion; ++k)
      for (int w = 0; w < SPLINE_ORDER * SPLINE_ORDER * SPLINE_ORDER; ++w) {
        if (h.prec == OFDFT_FP32) force_term<float>(s, h.stencils[k], w, &q[3 * k]);
        else force_term<double>(s, h.stencils[k], w, &q[3 * k]);
      }
#else
    double* dq = nullptr;
    if ((rc = dmalloc((void**)&dq, sizeof(double) * q.size()))) return rc;
    if (h.prec == OFDFT_FP32) k_force_gather<float><<<h.nion, 256, 0, stream>>>(d_slots + i, h.d_stencil, dq);
    else k_force_gather<double><<<h.nion, 256, 0, stream>>>(d_slots + i, h.d_stencil, dq);
    rc = cuda_check(cudaGetLastError(), "force gather launch");
    if (!rc) rc = sync_stream();
    if (!rc) rc = d2h(q.data(), dq, sizeof(double) * q.size());
    dfree(dq);
    if (rc) return rc;
#endif
    // F_ie = -cellInv * sum(qIonDeriv * Factor) (CalculateSplineForces)
    for (int k = 0; k < h.nion; ++k)
      for (int r = 0; r < 3; ++r)
        out[3 * k + r] = -(h.cell_inv_t[3 * r] * q[3 * k] + h.cell_inv_t[3 * r + 1] * q[3 * k + 1] +
                           h.cell_inv_t[3 * r + 2] * q[3 * k + 2]);
    if (include_ewald) {  // ion-ion forces summed on the device
      std::vector<double> fii(3 * (size_t)h.nion);
      if ((rc = ewald_device(i, nullptr, fii.data()))) return rc;
      for (size_t k = 0; k < fii.size(); ++k) out[k] += fii[k];
    }
    return OFDFT_OK;
  }

  // Stress tensor (Ha/bohr^3, out[9] row-major, symmetric) of rho (host, FP64)
  // or, with rho NULL, of the slot's current density phi^2; terms[7*9] (may be
  // NULL) gets the TF, vW, nonlocal (WT or WGC), Hartree, LDA, ion-electron
  // and Ewald parts.
  // The energies come from one evaluation of the density; the spectral sums
  // from the EV_STRESS transforms and the stress reduction (stress.cuh).  The
  // slot's control record, current phi and potential are left as they were.
  int stress(int i, const double* rho, int include_ewald, double* out, double* terms) {
    int rc = check_slot(i);
    if (rc) return rc;
    HostSlot& h = slots[i];
    SlotDev& s = h.sd;
    const bool wgc = s.kinetic == KIN_WGC;
    if (h.nion < 1 || s.ion.nspec < 1) return fail(OFDFT_EINVAL, "build the ion potential before the stress");
    if (!(h.rho0 > 0) || (wgc && !(s.rho_s > 0))) return fail(OFDFT_EINVAL, "rho0 (and rho* for WGC) must be positive");
    Ctl saved;
    if ((rc = get_ctl(i, saved))) return rc;
    // two work buffers that hold neither the current phi nor its potential
    int spare[2], ns = 0;
    for (int b = 0; b < NBUF && ns < 2; ++b)
      if (b != saved.iphi && b != saved.iw0) spare[ns++] = b;
    const int ib = spare[0], iw = spare[1];
    if (rho) {
      if ((rc = upload_real(h.prec, s.buf[ib], rho, s.N))) return rc;
    } else {
      const void* sp = s.buf[saved.iphi];
#if defined(OFDFT_EMU)
      for (long long k = 0; k < s.N; ++k) {
        if (h.prec == OFDFT_FP32) ((float*)s.buf[ib])[k] = ((const float*)sp)[k] * ((const float*)sp)[k];
        else ((double*)s.buf[ib])[k] = ((const double*)sp)[k] * ((const double*)sp)[k];
      }
#else
      if (h.prec == OFDFT_FP32)
        k_square_copy<float, float><<<io_blocks(s.N), 256, 0, stream>>>((const float*)sp, (float*)s.buf[ib], s.N);
      else
        k_square_copy<double, double><<<io_blocks(s.N), 256, 0, stream>>>((const double*)sp, (double*)s.buf[ib], s.N);
      if ((rc = cuda_check(cudaGetLastError(), "square copy launch"))) return rc;
#endif
    }
    // the energy terms of the density
    Ctl c;
    base_ctl(c, h.prec);
    c.ev = EV_RHO;
    c.iphi = ib;
    c.iw0 = iw;
    c.want_energy = 1;
    if ((rc = put_ctl(i, c))) return rc;
    if ((rc = run_one(i))) return rc;
    if ((rc = get_ctl(i, c))) return rc;
    double et[9];
    for (int k = 0; k < 9; ++k) et[k] = c.energy[k];
    // the density's forward spectra
    base_ctl(c, h.prec);
    c.ev = EV_STRESS;
    c.iphi = ib;
    if ((rc = put_ctl(i, c))) return rc;
    if ((rc = run_one(i))) return rc;
    // the spectral sums
    const int nion = h.nion, L = s.k1 + s.n2 + s.n3;
    std::vector<int> species(nion);
    for (int k = 0; k < nion; ++k) species[k] = h.stencils[k].species;
    StressArgs sa;
    sa.nion = nion;
    sa.kf = std::cbrt(3.0 * PI_D * PI_D * (wgc ? s.rho_s : h.rho0));
    sa.ki = 20.0 * std::pow(h.rho0, 5.0 / 3.0 - (s.alpha + s.beta));
    sa.gamma = h.gamma;
    const int nblk = (int)std::max<long long>(1, std::min<long long>(2 * (long long)num_sms, (s.Nc + 127) / 128));
    std::vector<double> part((size_t)NSC * nblk);
#if defined(OFDFT_EMU)
    std::vector<cx<double>> sf((size_t)nion * L);
    for (int k = 0; k < nion; ++k)
      for (int w = 0; w < L; ++w) sf[(size_t)k * L + w] = stress_sf_entry(s, h.stencils[k], w);
    sa.permy = plans.d_idx + s.py.perm;
    sa.permz = plans.d_idx + s.pz.perm;
    sa.sf = sf.data();
    sa.species = species.data();
    double red[NSC];
    for (int b = 0; b < nblk; ++b) {
      if (h.prec == OFDFT_FP32) stress_block<float>(s, sa, b, nblk, 0, 1, red, &part[(size_t)NSC * b]);
      else stress_block<double>(s, sa, b, nblk, 0, 1, red, &part[(size_t)NSC * b]);
    }
#else
    const size_t sf_bytes = sizeof(cx<double>) * (size_t)nion * L;
    const size_t part_bytes = sizeof(double) * part.size();
    char* scratch = nullptr;
    if ((rc = dmalloc((void**)&scratch, sf_bytes + part_bytes + sizeof(int) * (size_t)nion))) return rc;
    cx<double>* dsf = (cx<double>*)scratch;
    double* dpart = (double*)(scratch + sf_bytes);
    int* dspec = (int*)(scratch + sf_bytes + part_bytes);
    rc = h2d(dspec, species.data(), sizeof(int) * (size_t)nion);
    if (!rc) {
      sa.permy = plans.d_idx + s.py.perm;
      sa.permz = plans.d_idx + s.pz.perm;
      sa.sf = dsf;
      sa.species = dspec;
      k_stress_sf<<<nion, 128, 0, stream>>>(d_slots + i, h.d_stencil, dsf);
      if (h.prec == OFDFT_FP32) k_stress<float><<<nblk, 128, 0, stream>>>(d_slots + i, sa, dpart);
      else k_stress<double><<<nblk, 128, 0, stream>>>(d_slots + i, sa, dpart);
      rc = cuda_check(cudaGetLastError(), "stress launch");
    }
    if (!rc) rc = d2h(part.data(), dpart, part_bytes);
    dfree(scratch);
    if (rc) return rc;
#endif
    double acc[NSC] = {0};
    for (int b = 0; b < nblk; ++b)
      for (int k = 0; k < NSC; ++k) acc[k] += part[(size_t)NSC * b + k];
    if ((rc = put_ctl(i, saved))) return rc;
    // assembly (CalculateStress): six components per term, then the diagonal terms
    const double vol = s.vol;
    double T6[7][6] = {{0}};
    // the kinetic nonlocal term: WT (WTStress) or WGC (WGCStress, x 2 cTF)
    const double wtc = wgc ? 2.0 * C_TF
                           : PI_D * PI_D / (s.alpha * s.beta * sa.kf * std::pow(h.rho0, s.alpha + s.beta - 2.0));
    for (int k = 0; k < 6; ++k) {
      T6[1][k] = -s.mu * acc[SC_VW + k];
      T6[2][k] = wtc * acc[SC_WT + k];
      T6[3][k] = 8.0 * PI_D * acc[SC_H + k];
      T6[5][k] = -2.0 * (double)s.N * acc[SC_IE + k] / vol;
    }
    double sxc = 0.0;
    if ((rc = rho_vxc(i, ib, &sxc))) return rc;
    const int diag[3] = {0, 3, 5};
    for (int d : diag) {
      T6[0][d] += -2.0 / 3.0 * et[6] / vol;
      T6[2][d] += wgc ? wtc * acc[SC_WTTR] : -wtc * acc[SC_WTTR] / 3.0 - 2.0 / 3.0 * et[8] / vol;
      T6[3][d] += -et[3] / vol;
      T6[4][d] += et[4] / vol - sxc;
      T6[5][d] += -et[2] / vol;
    }
    if (include_ewald && (rc = ewald_stress(i, T6[6]))) return rc;
    const int ab[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
    for (int k = 0; k < 9; ++k) {
      out[k] = 0.0;
      for (int t = 0; t < 7; ++t) out[k] += T6[t][ab[k]];
    }
    if (terms)
      for (int t = 0; t < 7; ++t)
        for (int k = 0; k < 9; ++k) terms[9 * t + k] = T6[t][ab[k]];
    return OFDFT_OK;
  }

  // RescaleDensity (Source/RefreshIons.f90:33-122) of the held input density:
  // scaled to num_electrons with the slot's current dV.
  int rescale_input(int i, double num_electrons) {
    int rc = check_slot(i);
    if (rc) return rc;
    HostSlot& h = slots[i];
    const SlotDev& s = h.sd;
    if (!h.input) return fail(OFDFT_EINVAL, "no held input density to rescale");
    const int nblk = (int)std::max<long long>(1, std::min<long long>(2 * (long long)num_sms, (s.N + 255) / 256));
    std::vector<double> part(nblk);
#if defined(OFDFT_EMU)
    double red[1];
    for (int k = 0; k < nblk; ++k) {
      if (h.prec == OFDFT_FP32) sum_block<float>((const float*)h.input, s.N, k, nblk, 0, 1, red, &part[k]);
      else sum_block<double>((const double*)h.input, s.N, k, nblk, 0, 1, red, &part[k]);
    }
#else
    double* dp = nullptr;
    if ((rc = dmalloc((void**)&dp, sizeof(double) * nblk))) return rc;
    if (h.prec == OFDFT_FP32) k_sum<float><<<nblk, 256, 0, stream>>>((const float*)h.input, s.N, dp);
    else k_sum<double><<<nblk, 256, 0, stream>>>((const double*)h.input, s.N, dp);
    rc = cuda_check(cudaGetLastError(), "sum launch");
    if (!rc) rc = d2h(part.data(), dp, sizeof(double) * nblk);
    dfree(dp);
    if (rc) return rc;
#endif
    double sum = 0.0;
    for (int k = 0; k < nblk; ++k) sum += part[k];
    sum *= s.dv;
    if (!(sum > 0)) return fail(OFDFT_EINVAL, "held density has no electrons");
    const double f = num_electrons / sum;
#if defined(OFDFT_EMU)
    for (long long k = 0; k < s.N; ++k) {
      if (h.prec == OFDFT_FP32) ((float*)h.input)[k] = (float)((double)((float*)h.input)[k] * f);
      else ((double*)h.input)[k] *= f;
    }
    return OFDFT_OK;
#else
    if (h.prec == OFDFT_FP32) k_scale<float><<<io_blocks(s.N), 256, 0, stream>>>((float*)h.input, s.N, f);
    else k_scale<double><<<io_blocks(s.N), 256, 0, stream>>>((double*)h.input, s.N, f);
    if ((rc = cuda_check(cudaGetLastError(), "scale launch"))) return rc;
    return sync_stream();
#endif
  }

  // <rho v_xc> over the grid (the mean of rho times the LDA potential) of the
  // density held in buffer b.
  int rho_vxc(int i, int b, double* out) {
    HostSlot& h = slots[i];
    const SlotDev& s = h.sd;
    const int nblk = (int)std::max<long long>(1, std::min<long long>(2 * (long long)num_sms, (s.N + 255) / 256));
    std::vector<double> part(nblk);
#if defined(OFDFT_EMU)
    double red[1];
    for (int k = 0; k < nblk; ++k) {
      if (h.prec == OFDFT_FP32) rho_vxc_block<float>((const float*)s.buf[b], s.N, k, nblk, 0, 1, red, &part[k]);
      else rho_vxc_block<double>((const double*)s.buf[b], s.N, k, nblk, 0, 1, red, &part[k]);
    }
#else
    double* dp = nullptr;
    int rc = dmalloc((void**)&dp, sizeof(double) * nblk);
    if (rc) return rc;
    if (h.prec == OFDFT_FP32) k_rho_vxc<float><<<nblk, 256, 0, stream>>>((const float*)s.buf[b], s.N, dp);
    else k_rho_vxc<double><<<nblk, 256, 0, stream>>>((const double*)s.buf[b], s.N, dp);
    rc = cuda_check(cudaGetLastError(), "rho vxc launch");
    if (!rc) rc = d2h(part.data(), dp, sizeof(double) * nblk);
    dfree(dp);
    if (rc) return rc;
#endif
    double sum = 0.0;
    for (int k = 0; k < nblk; ++k) sum += part[k];
    *out = sum / (double)s.N;
    return OFDFT_OK;
  }

  // Ewald stress (six upper components, Ha/bohr^3) of the slot's ions.
  int ewald_stress(int i, double* out6) {
    HostSlot& h = slots[i];
    const int nion = h.nion;
    const EwaldPar p = ewald_par(h.lattice, nion);
    const int npl = ewald_planes(p);
    std::vector<double> pos(3 * (size_t)nion);
    for (int k = 0; k < nion; ++k)
      for (int r = 0; r < 3; ++r)
        pos[3 * k + r] = p.A[r][0] * h.frac[3 * k] + p.A[r][1] * h.frac[3 * k + 1] + p.A[r][2] * h.frac[3 * k + 2];
    std::vector<double> real7(7 * (size_t)nion), plane7(7 * (size_t)npl);
#if defined(OFDFT_EMU)
    double red[7];
    for (int k = 0; k < nion; ++k) ewald_real_stress_block(p, pos.data(), h.zion.data(), k, 0, 1, red, &real7[7 * k]);
    for (int m = 0; m < npl; ++m)
      ewald_plane_stress_block(p, h.frac.data(), h.zion.data(), m, 0, 1, red, &plane7[7 * m]);
#else
    const size_t nd = 3 * (size_t)nion * 2 + nion + 7 * (size_t)nion + 7 * (size_t)npl;
    double* dbuf = nullptr;
    int rc = dmalloc((void**)&dbuf, sizeof(double) * nd);
    if (rc) return rc;
    double *dpos = dbuf, *dfrac = dpos + 3 * nion, *dz = dfrac + 3 * nion, *dreal = dz + nion, *dplane = dreal + 7 * nion;
    rc = h2d(dpos, pos.data(), sizeof(double) * 3 * nion);
    if (!rc) rc = h2d(dfrac, h.frac.data(), sizeof(double) * 3 * nion);
    if (!rc) rc = h2d(dz, h.zion.data(), sizeof(double) * nion);
    if (!rc) {
      k_ewald_real_stress<<<nion, 128, 0, stream>>>(p, dpos, dz, dreal);
      k_ewald_plane_stress<<<npl, 128, 0, stream>>>(p, dfrac, dz, dplane);
      rc = cuda_check(cudaGetLastError(), "Ewald stress launch");
    }
    if (!rc) rc = d2h(real7.data(), dreal, sizeof(double) * 7 * nion);
    if (!rc) rc = d2h(plane7.data(), dplane, sizeof(double) * 7 * npl);
    dfree(dbuf);
    if (rc) return rc;
#endif
    double qsum = 0.0, e_rec = 0.0, s6[6] = {0};
    for (int k = 0; k < nion; ++k) {
      qsum += h.zion[k];
      for (int c = 0; c < 6; ++c) s6[c] += real7[7 * k + 1 + c];
    }
    double r6[6] = {0};
    for (int m = 0; m < npl; ++m) {
      e_rec += plane7[7 * m];
      for (int c = 0; c < 6; ++c) r6[c] += plane7[7 * m + 1 + c];
    }
    const double e_bg = -0.5 * PI_D / (p.eta * p.eta) / p.vol * qsum * qsum;
    for (int c = 0; c < 6; ++c) {
      double v = s6[c] + r6[c];
      if (c == 0 || c == 3 || c == 5) v -= e_rec + e_bg;
      out6[c] = v / p.vol;
    }
    return OFDFT_OK;
  }

  int check_slot(int i) {
    if (i < 0 || i >= cap || !slots[i].used) return fail(OFDFT_EINVAL, "invalid slot");
    if (slots[i].running) return fail(OFDFT_EBUSY, "slot is running");
    return OFDFT_OK;
  }

  // Host <-> device copies of the caller's FP64 arrays into/out of device
  // arrays of the slot's precision.  The copies go straight from/to the
  // caller's (pageable) buffer on the engine stream; a change of precision and
  // the squaring of phi run on the device, through a device scratch array of
  // n doubles, so the host does no per-point work.
#if defined(OFDFT_EMU)
  int upload_real(int prec, void* dst, const double* src, long long n) {
    if (prec == OFDFT_FP64) return h2d(dst, src, sizeof(double) * (size_t)n);
    float* f = (float*)dst;
    for (long long i = 0; i < n; ++i) f[i] = (float)src[i];
    return OFDFT_OK;
  }
  int download_real(int prec, double* dst, const void* src, long long n, bool square = false) {
    for (long long i = 0; i < n; ++i) {
      const double v = prec == OFDFT_FP32 ? (double)((const float*)src)[i] : ((const double*)src)[i];
      dst[i] = square ? v * v : v;
    }
    return OFDFT_OK;
  }
#else
  void* d_io = nullptr;
  size_t io_bytes = 0;
  int io_scratch(size_t bytes, void** p) {
    if (io_bytes < bytes) {
      dfree(d_io);
      d_io = nullptr;
      io_bytes = 0;
      int rc = cuda_check(cudaMalloc(&d_io, bytes), "cudaMalloc");
      if (rc) return rc;
      io_bytes = bytes;
    }
    *p = d_io;
    return OFDFT_OK;
  }
  static unsigned io_blocks(long long n) { return (unsigned)std::min<long long>(4 * 148, (n + 255) / 256); }
  int upload_real(int prec, void* dst, const double* src, long long n) {
    const size_t bytes = sizeof(double) * (size_t)n;
    if (prec == OFDFT_FP64) return h2d(dst, src, bytes);
    void* io = nullptr;
    int rc = io_scratch(bytes, &io);
    if (rc) return rc;
    if ((rc = cuda_check(cudaMemcpyAsync(io, src, bytes, cudaMemcpyHostToDevice, stream), "H2D async"))) return rc;
    k_convert<double, float><<<io_blocks(n), 256, 0, stream>>>((const double*)io, (float*)dst, n);
    if ((rc = cuda_check(cudaGetLastError(), "convert launch"))) return rc;
    return sync_stream();
  }
  int download_real(int prec, double* dst, const void* src, long long n, bool square = false) {
    const size_t bytes = sizeof(double) * (size_t)n;
    if (prec == OFDFT_FP64 && !square) return d2h(dst, src, bytes);
    void* io = nullptr;
    int rc = io_scratch(bytes, &io);
    if (rc) return rc;
    if (prec == OFDFT_FP64)
      k_square_copy<double, double><<<io_blocks(n), 256, 0, stream>>>((const double*)src, (double*)io, n);
    else if (square)
      k_square_copy<float, double><<<io_blocks(n), 256, 0, stream>>>((const float*)src, (double*)io, n);
    else
      k_convert<float, double><<<io_blocks(n), 256, 0, stream>>>((const float*)src, (double*)io, n);
    if ((rc = cuda_check(cudaGetLastError(), "convert launch"))) return rc;
    return d2h(dst, io, bytes);
  }
#endif

  // keKernel(k1G, k2G, k3G, nplanes) from the host (reference layout, FP64)
  // into the slot's kernel planes (kx-major, digit-reversed, slot precision).
  int set_kernel(int i, const double* kernel) {
    HostSlot& h = slots[i];
    const long long n = h.sd.Nc * h.nplanes;
#if defined(OFDFT_EMU)
    for (long long k = 0; k < n; ++k) {
      const double v = kernel[kernel_source_index(h.sd, plans.d_idx, k)];
      if (h.prec == OFDFT_FP32) ((float*)h.sd.kern)[k] = (float)v;
      else ((double*)h.sd.kern)[k] = v;
    }
    return OFDFT_OK;
#else
    void* io = nullptr;
    int rc = io_scratch(sizeof(double) * (size_t)n, &io);
    if (rc) return rc;
    if ((rc = cuda_check(cudaMemcpyAsync(io, kernel, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, stream),
                         "H2D async")))
      return rc;
    if (h.prec == OFDFT_FP32)
      k_permute_kernel<float><<<io_blocks(n), 256, 0, stream>>>(d_slots + i, plans.d_idx, (const double*)io, h.nplanes);
    else
      k_permute_kernel<double><<<io_blocks(n), 256, 0, stream>>>(d_slots + i, plans.d_idx, (const double*)io, h.nplanes);
    if ((rc = cuda_check(cudaGetLastError(), "kernel permute launch"))) return rc;
    return sync_stream();
#endif
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

  // rho on the host, or NULL for the slot's device-resident input density.
  int load_density(int i, const double* rho) {
    HostSlot& h = slots[i];
    if (rho) return upload_real(h.prec, h.sd.buf[B_PHI], rho, h.sd.N);
    if (!h.input) return fail(OFDFT_EINVAL, "no device-resident input density (ofdft_slot_set_input)");
    return d2d(h.sd.buf[B_PHI], h.input, elem_size(h.prec) * h.sd.N);
  }

  int set_input(int i, const double* rho) {
    int rc = check_slot(i);
    if (rc) return rc;
    HostSlot& h = slots[i];
    if (!h.input && (rc = palloc(&h.input, elem_size(h.prec) * h.sd.N, &h.input_bytes))) return rc;
    return upload_real(h.prec, h.input, rho, h.sd.N);
  }

  int start_eval(int i, const double* rho, int opt_sqrt, int want_energy) {
    int rc = check_slot(i);
    if (rc) return rc;
    HostSlot& h = slots[i];
    if ((rc = load_density(i, rho))) return rc;
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
    c.stall_line = (o && o->stall_line > 0) ? o->stall_line : 0;
    c.outcome = -1;
  }

  int start_solve(int i, const double* rho, const ofdft_ntn_options* o) {
    int rc = check_slot(i);
    if (rc) return rc;
    HostSlot& h = slots[i];
    if ((rc = load_density(i, rho))) return rc;
    Ctl c;
    solve_ctl(c, h.prec, o);
    if ((rc = put_ctl(i, c))) return rc;
    h.running = true;
    dirty = true;
    return OFDFT_OK;
  }

  // Ewald energy and forces (Ha, Ha/bohr; forces may be NULL) of the slot's
  // ions, summed on the device.
  int ewald_device(int i, double* energy, double* forces) {
    int rc = OFDFT_OK;
    HostSlot& h = slots[i];
    const int nion = h.nion;
    if (nion < 1) return fail(OFDFT_EINVAL, "build the ion potential before the Ewald sum");
    const EwaldPar p = ewald_par(h.lattice, nion);
    const int npl = ewald_planes(p), plane = ewald_plane_size(p);
    std::vector<double> pos(3 * (size_t)nion);
    for (int k = 0; k < nion; ++k)
      for (int r = 0; r < 3; ++r)
        pos[3 * k + r] = p.A[r][0] * h.frac[3 * k] + p.A[r][1] * h.frac[3 * k + 1] + p.A[r][2] * h.frac[3 * k + 2];
    std::vector<double> real4(4 * (size_t)nion), plane4(4 * (size_t)npl), rec4(4 * (size_t)nion);
#if defined(OFDFT_EMU)
    std::vector<cx<double>> sfac((size_t)npl * plane);
    double red[4];
    for (int k = 0; k < nion; ++k) ewald_real_block(p, pos.data(), h.zion.data(), k, 0, 1, red, &real4[4 * k]);
    for (int m = 0; m < npl; ++m) ewald_plane_block(p, h.frac.data(), h.zion.data(), m, 0, 1, red, sfac.data(), &plane4[4 * m]);
    if (forces)
      for (int k = 0; k < nion; ++k)
        ewald_recip_force_block(p, h.frac.data(), h.zion.data(), sfac.data(), k, 0, 1, red, &rec4[4 * k]);
#else
    // one scratch array (the engine's transfer scratch): pos, frac, z, the three
    // 4-value outputs, S(G)
    const size_t nd = 3 * (size_t)nion * 2 + nion + 4 * (size_t)nion * 2 + 4 * (size_t)npl;
    double* dbuf = nullptr;
    if ((rc = io_scratch(sizeof(double) * nd + sizeof(cx<double>) * (size_t)npl * plane, (void**)&dbuf))) return rc;
    double *dpos = dbuf, *dfrac = dpos + 3 * nion, *dz = dfrac + 3 * nion, *dreal = dz + nion, *drec = dreal + 4 * nion,
           *dplane = drec + 4 * nion;
    cx<double>* dsf = (cx<double>*)(dbuf + nd);
    rc = h2d(dpos, pos.data(), sizeof(double) * 3 * nion);
    if (!rc) rc = h2d(dfrac, h.frac.data(), sizeof(double) * 3 * nion);
    if (!rc) rc = h2d(dz, h.zion.data(), sizeof(double) * nion);
    if (!rc) {
      k_ewald_real<<<nion, 256, 0, stream>>>(p, dpos, dz, dreal);
      k_ewald_plane<<<npl, 256, 0, stream>>>(p, dfrac, dz, dsf, dplane);
      if (forces) k_ewald_recip_force<<<nion, 256, 0, stream>>>(p, dfrac, dz, dsf, drec);
      rc = cuda_check(cudaGetLastError(), "Ewald launch");
    }
    if (!rc) rc = d2h(real4.data(), dreal, sizeof(double) * 4 * nion);
    if (!rc) rc = d2h(plane4.data(), dplane, sizeof(double) * 4 * npl);
    if (!rc && forces) rc = d2h(rec4.data(), drec, sizeof(double) * 4 * nion);
    if (rc) return rc;
#endif
    double qsum = 0.0, q2 = 0.0, e_real = 0.0, e_rec = 0.0;
    for (int k = 0; k < nion; ++k) {
      qsum += h.zion[k];
      q2 += h.zion[k] * h.zion[k];
      e_real += real4[4 * k];
    }
    for (int m = 0; m < npl; ++m) e_rec += plane4[4 * m];
    const double e_self = -p.eta / std::sqrt(PI_D) * q2;
    const double e_bg = -0.5 * PI_D / (p.eta * p.eta) / p.vol * qsum * qsum;
    const double e = e_real + e_self + e_rec + e_bg;
    if (forces)
      for (int k = 0; k < nion; ++k)
        for (int r = 0; r < 3; ++r) forces[3 * k + r] = real4[4 * k + 1 + r] + rec4[4 * k + 1 + r];
    if (energy) *energy = e;
    return OFDFT_OK;
  }
  // The same, with the energy made the slot's eTable(6).
  int slot_ewald(int i, double* energy, double* forces) {
    int rc = check_slot(i);
    if (rc) return rc;
    double e = 0.0;
    if ((rc = ewald_device(i, &e, forces))) return rc;
    if (energy) *energy = e;
    slots[i].sd.ion_ion = e;
    return upload_slot(i);
  }

  // The kinetic kernel planes, the ion potential and the ion-ion energy of
  // slot src, converted into slot i (same grid and functional; either
  // precision) on the device: a mixed-precision request sets up its FP64
  // slot once and gives its FP32 slot the same tables without a second
  // set-up.
  int copy_tables(int i, int src) {
    int rc = check_slot(i);
    if (rc) return rc;
    if ((rc = check_slot(src))) return rc;
    HostSlot& h = slots[i];
    const HostSlot& g = slots[src];
    if (h.sd.n1 != g.sd.n1 || h.sd.n2 != g.sd.n2 || h.sd.n3 != g.sd.n3 || h.sd.kinetic != g.sd.kinetic ||
        h.nplanes != g.nplanes)
      return fail(OFDFT_EINVAL, "the slots differ in grid or functional");
    // the kernel planes are stored in the digit-reversed order of the slot's
    // own transforms (FP32 and FP64 plans may differ): go through the
    // reference layout
    const long long nk = h.sd.Nc * h.nplanes, nv = h.sd.N;
#if defined(OFDFT_EMU)
    std::vector<double> ref(nk);
    for (long long k = 0; k < nk; ++k) {
      const long long r = kernel_source_index(g.sd, plans.d_idx, k);
      ref[r] = g.prec == OFDFT_FP32 ? (double)((const float*)g.sd.kern)[k] : ((const double*)g.sd.kern)[k];
    }
    if ((rc = set_kernel(i, ref.data()))) return rc;
    for (long long k = 0; k < nv; ++k) {
      const double v = g.prec == OFDFT_FP32 ? (double)((const float*)g.sd.vion)[k] : ((const double*)g.sd.vion)[k];
      if (h.prec == OFDFT_FP32) ((float*)h.sd.vion)[k] = (float)v;
      else ((double*)h.sd.vion)[k] = v;
    }
#else
    double* io = nullptr;
    if ((rc = io_scratch(sizeof(double) * (size_t)std::max(nk, nv), (void**)&io))) return rc;
    if (g.prec == OFDFT_FP32)
      k_unpermute_kernel<float><<<io_blocks(nk), 256, 0, stream>>>(d_slots + src, plans.d_idx, io, h.nplanes);
    else
      k_unpermute_kernel<double><<<io_blocks(nk), 256, 0, stream>>>(d_slots + src, plans.d_idx, io, h.nplanes);
    if (h.prec == OFDFT_FP32)
      k_permute_kernel<float><<<io_blocks(nk), 256, 0, stream>>>(d_slots + i, plans.d_idx, io, h.nplanes);
    else
      k_permute_kernel<double><<<io_blocks(nk), 256, 0, stream>>>(d_slots + i, plans.d_idx, io, h.nplanes);
    if (g.prec == OFDFT_FP64 && h.prec == OFDFT_FP32)
      k_convert<double, float><<<io_blocks(nv), 256, 0, stream>>>((const double*)g.sd.vion, (float*)h.sd.vion, nv);
    else if (g.prec == OFDFT_FP32 && h.prec == OFDFT_FP64)
      k_convert<float, double><<<io_blocks(nv), 256, 0, stream>>>((const float*)g.sd.vion, (double*)h.sd.vion, nv);
    else if (g.prec == OFDFT_FP32)
      k_convert<float, float><<<io_blocks(nv), 256, 0, stream>>>((const float*)g.sd.vion, (float*)h.sd.vion, nv);
    else
      k_convert<double, double><<<io_blocks(nv), 256, 0, stream>>>((const double*)g.sd.vion, (double*)h.sd.vion, nv);
    if ((rc = cuda_check(cudaGetLastError(), "table copy launch"))) return rc;
    if ((rc = sync_stream())) return rc;
#endif
    h.sd.ion_ion = g.sd.ion_ion;
    return upload_slot(i);
  }

  // Keep the slot's current density phi^2 as its resident input (device to
  // device), so that a later start with rho = NULL resumes from it after
  // passes that reuse the state arrays (the ion-potential build does).
  int hold_density(int i) {
    int rc = check_slot(i);
    if (rc) return rc;
    HostSlot& h = slots[i];
    Ctl c;
    if ((rc = get_ctl(i, c))) return rc;
    if (!h.input && (rc = palloc(&h.input, elem_size(h.prec) * h.sd.N, &h.input_bytes))) return rc;
    const void* sp = h.sd.buf[c.iphi];  // the current phi, also after a cancel
    const long long n = h.sd.N;
#if defined(OFDFT_EMU)
    for (long long k = 0; k < n; ++k) {
      if (h.prec == OFDFT_FP32) ((float*)h.input)[k] = ((const float*)sp)[k] * ((const float*)sp)[k];
      else ((double*)h.input)[k] = ((const double*)sp)[k] * ((const double*)sp)[k];
    }
    return OFDFT_OK;
#else
    if (h.prec == OFDFT_FP32)
      k_square_copy<float, float><<<io_blocks(n), 256, 0, stream>>>((const float*)sp, (float*)h.input, n);
    else
      k_square_copy<double, double><<<io_blocks(n), 256, 0, stream>>>((const double*)sp, (double*)h.input, n);
    if ((rc = cuda_check(cudaGetLastError(), "square copy launch"))) return rc;
    return sync_stream();
#endif
  }

  // Start a solve in slot i from the density phi^2 held by slot src (same grid).
  int start_solve_from(int i, int src, const ofdft_ntn_options* o) {
    int rc = check_slot(i);
    if (rc) return rc;
    if ((rc = check_slot(src))) return rc;
    HostSlot& h = slots[i];
    HostSlot& g = slots[src];
    if (h.sd.N != g.sd.N || h.sd.n1 != g.sd.n1 || h.sd.n2 != g.sd.n2)
      return fail(OFDFT_EINVAL, "source slot has a different grid");
    Ctl cs;
    if ((rc = get_ctl(src, cs))) return rc;
    const void* sp = g.sd.buf[cs.iphi];
    void* dp = h.sd.buf[B_PHI];
    const long long n = h.sd.N;
#if defined(OFDFT_EMU)
    for (long long k = 0; k < n; ++k) {
      const double v = g.prec == OFDFT_FP32 ? (double)((const float*)sp)[k] : ((const double*)sp)[k];
      if (h.prec == OFDFT_FP32) ((float*)dp)[k] = (float)(v * v);
      else ((double*)dp)[k] = v * v;
    }
#else
    const int blocks = (int)std::min<long long>(2048, (n + 255) / 256);
    if (g.prec == OFDFT_FP32 && h.prec == OFDFT_FP64)
      k_square_copy<float, double><<<blocks, 256, 0, stream>>>((const float*)sp, (double*)dp, n);
    else if (g.prec == OFDFT_FP64 && h.prec == OFDFT_FP64)
      k_square_copy<double, double><<<blocks, 256, 0, stream>>>((const double*)sp, (double*)dp, n);
    else if (g.prec == OFDFT_FP32 && h.prec == OFDFT_FP32)
      k_square_copy<float, float><<<blocks, 256, 0, stream>>>((const float*)sp, (float*)dp, n);
    else
      k_square_copy<double, float><<<blocks, 256, 0, stream>>>((const double*)sp, (float*)dp, n);
    if ((rc = cuda_check(cudaGetLastError(), "square copy launch"))) return rc;
    if ((rc = sync_stream())) return rc;
#endif
    Ctl c;
    solve_ctl(c, h.prec, o);
    if ((rc = put_ctl(i, c))) return rc;
    h.running = true;
    dirty = true;
    return OFDFT_OK;
  }

  // Back-to-back potential evaluations of every slot that has a resident
  // input density; returns the mean device time of one batched evaluation
  // (passes 1-5 and the controller kernel), timed with events on the engine stream.
  // ---------------------------------------------------------- autotuning
  // The launch shape a tuner may change, per slot: the radix cap of the x-axis
  // FFT plan, row pairs per x-forward and per x-inverse task, and the block
  // size of the fused y-z pass (256 or 512 threads; 0 = by plane size).  The
  // y and z plans stay fixed: the kernel planes are stored in their order.
  struct Shape {
    int xcap, rp1, rp, yzt;
  };
  std::map<std::vector<long long>, Shape> tune_cache;  // by grid, precision and functional
  static std::vector<long long> tune_key(const HostSlot& h) {
    const SlotDev& s = h.sd;
    return {s.n1, s.n2, s.n3, h.prec, s.kinetic, s.nf};
  }
  Shape shape_of(const HostSlot& h) const { return {h.xcap, h.rp1, h.sd.rp, h.yzt}; }
  bool shape_ok(const HostSlot& h, const Shape& c) const {
    const SlotDev& s = h.sd;
    const size_t esz = elem_size(h.prec);
    if (c.rp1 < 1 || c.rp1 > 32 || c.rp < 1 || c.rp > 32) return false;
    if (xfwd_smem(s.n1, std::max(s.nf, MAX_SPECIES), c.rp1, esz) > 200 * 1024) return false;
    if (xinv_smem(s.n1, std::max(s.nf, MAX_SPECIES), c.rp, esz) > 200 * 1024) return false;
    if (c.yzt != 0 && c.yzt != 256 && c.yzt != 512) return false;
    return true;
  }
  void set_shape(HostSlot& h, const Shape& c) {
    SlotDev& s = h.sd;
    const int pi = h.prec == OFDFT_FP32 ? 1 : 0;
    h.xcap = c.xcap;
    s.px = plans.get(pi, s.n1, c.xcap);
    h.rp1 = c.rp1;
    s.rp = c.rp;
    s.ntask[K_X5] = (h.nrowpairs + s.rp - 1) / s.rp;
    h.yzt = c.yzt;
    dirty = true;
  }

  // Median time (ms) of `iters` one-tick evaluations of the slots ids, each
  // from its resident input density.
  int time_ids(const std::vector<int>& ids, int iters, double* ms_out) {
    int rc;
    auto start_all = [&]() -> int {
      for (int i : ids) {
        int r = start_eval(i, nullptr, 1, 1);
        if (r) return r;
      }
      return OFDFT_OK;
    };
    if ((rc = start_all())) return rc;
    int running = 0;
    if ((rc = run(2, &running, 1))) return rc;  // warm-up and graph capture for one tick
#if defined(OFDFT_EMU)
    *ms_out = 0.0;
    (void)iters;
    return OFDFT_OK;
#else
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<float> t;
    for (int it = 0; it < iters; ++it) {
      if ((rc = start_all())) break;
      if (dirty && (rc = build_lists())) break;
      if ((rc = capture(1))) break;
      cudaEventRecord(e0, stream);
      if ((rc = cuda_check(cudaGraphLaunch(graph_exec, stream), "graph launch"))) break;
      cudaEventRecord(e1, stream);
      if ((rc = sync_stream())) break;
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      t.push_back(ms);
      n_ticks += 1;
      n_launches += launches_per_tick();
      for (int i : ids) slots[i].running = false;
      dirty = true;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    std::sort(t.begin(), t.end());
    *ms_out = t.empty() ? 0.0 : (double)t[t.size() / 2];
    return OFDFT_OK;
#endif
  }

  // Tune the launch shape of slot i's kind of cell (grid, precision and
  // functional) by timing one batched evaluation, per candidate, of every idle
  // slot of that kind that holds a resident input density - the batch the
  // shape will serve, since a lone slot leaves most SMs idle and favours other
  // shapes.  Coordinate descent over the x radix cap, the x-forward and
  // x-inverse task sizes and the y-z block size; a candidate must be 1 %
  // faster to replace the incumbent.  The result is cached for the kind and
  // applied to every slot of it, now and at creation.  The timed slots' solve
  // records are overwritten.
  int tune(int i, int iters, double* ms_default, double* ms_tuned, int* shape_out) {
    int rc = check_slot(i);
    if (rc) return rc;
    HostSlot& h = slots[i];
    if (!h.input) return fail(OFDFT_EINVAL, "tuning needs a resident input density (ofdft_slot_set_input)");
    for (int k = 0; k < cap; ++k)
      if (slots[k].used && slots[k].running) return fail(OFDFT_EBUSY, "tune while no slot is running");
    iters = std::max(iters, 3);
    std::vector<int> ids;
    for (int k = 0; k < cap; ++k)
      if (slots[k].used && slots[k].input && tune_key(slots[k]) == tune_key(h)) ids.push_back(k);
    auto apply = [&](const Shape& c) -> int {
      for (int k : ids) {
        set_shape(slots[k], c);
        const int r = upload_slot(k);
        if (r) return r;
      }
      return OFDFT_OK;
    };
    Shape best = shape_of(h);
    if ((rc = apply(best))) return rc;
    double tbest = 0.0;
    if ((rc = time_ids(ids, iters, &tbest))) return rc;
    *ms_default = tbest;
    auto trial = [&](Shape c) -> int {
      if (!shape_ok(h, c)) return OFDFT_OK;
      double t = 0.0;
      int r = apply(c);
      if (!r) r = time_ids(ids, iters, &t);
      if (r) {
        apply(best);
        return r;
      }
      if (t < 0.99 * tbest) {
        tbest = t;
        best = c;
      }
      return apply(best);
    };
    const int pi = h.prec == OFDFT_FP32 ? 1 : 0;
    const SlotDev& s = h.sd;
    const size_t csz = 2 * elem_size(h.prec);
    for (int ci = 1; ci < 3 && kCaps[pi][ci]; ++ci) {
      Shape c = best;
      c.xcap = kCaps[pi][ci];
      if ((rc = trial(c))) return rc;
    }
    const int base1 = best.rp1, base5 = best.rp;
    for (int r : {base1 / 2, (3 * base1) / 4, (3 * base1) / 2, 2 * base1}) {
      Shape c = best;
      c.rp1 = odd_columns(s.nf, std::max(1, r), csz);
      if (c.rp1 != best.rp1 && (rc = trial(c))) return rc;
    }
    for (int r : {base5 / 2, (3 * base5) / 4, (3 * base5) / 2, 2 * base5}) {
      Shape c = best;
      c.rp = odd_columns(s.nf, std::max(1, r), csz);
      if (c.rp != best.rp && (rc = trial(c))) return rc;
    }
    if (uses_yz(h))
      for (int t : {256, 512}) {
        Shape c = best;
        c.yzt = t;
        if ((rc = trial(c))) return rc;
      }
    *ms_tuned = tbest;
    tune_cache[tune_key(h)] = best;
    for (int k = 0; k < cap; ++k)
      if (slots[k].used && tune_key(slots[k]) == tune_key(h)) {
        set_shape(slots[k], best);
        if ((rc = upload_slot(k))) return rc;
      }
    return shape_out ? get_shape(i, shape_out) : OFDFT_OK;
  }

  // Pin slot i's launch shape (cap, x-forward and x-inverse row pairs, y-z
  // threads; 0 keeps the default for the cap and the y-z threads).
  int pin_shape(int i, const int* v) {
    int rc = check_slot(i);
    if (rc) return rc;
    HostSlot& h = slots[i];
    const int pi = h.prec == OFDFT_FP32 ? 1 : 0;
    bool cap_ok = v[0] == 0;
    for (int ci = 0; ci < 3; ++ci) cap_ok = cap_ok || (kCaps[pi][ci] && v[0] == kCaps[pi][ci]);
    const Shape c{v[0] == kCaps[pi][0] ? 0 : v[0], v[1], v[2], v[3]};
    if (!cap_ok || !shape_ok(h, c)) return fail(OFDFT_EINVAL, "launch shape out of range");
    set_shape(h, c);
    return upload_slot(i);
  }

  int get_shape(int i, int* v) {
    if (i < 0 || i >= cap || !slots[i].used) return fail(OFDFT_EINVAL, "invalid slot");
    const HostSlot& h = slots[i];
    const int pi = h.prec == OFDFT_FP32 ? 1 : 0;
    const size_t csz = 2 * elem_size(h.prec);
    v[0] = h.xcap ? h.xcap : kCaps[pi][0];
    v[1] = h.rp1;
    v[2] = h.sd.rp;
    v[3] = uses_yz(h) ? (h.yzt ? h.yzt : (yz_smem_slot(h.sd, csz) <= YZ_SMEM_SMALL ? 256 : 512)) : 0;
    return OFDFT_OK;
  }

  int time_eval(int iters, double* ms_out) {
    int rc;
    std::vector<int> ids;
    for (int i = 0; i < cap; ++i)
      if (slots[i].used && !slots[i].running && slots[i].input) ids.push_back(i);
    if (ids.empty()) return fail(OFDFT_EINVAL, "no slot with a resident input density");
    auto start_all = [&]() -> int {
      for (int i : ids) {
        int r = start_eval(i, nullptr, 1, 1);
        if (r) return r;
      }
      return OFDFT_OK;
    };
    if ((rc = start_all())) return rc;
    int running = 0;
    if ((rc = run(2, &running, 1))) return rc;  // warm-up and graph capture for one tick
#if defined(OFDFT_EMU)
    *ms_out = 0.0;
    (void)iters;
    return OFDFT_OK;
#else
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float total = 0.0f;
    for (int it = 0; it < iters; ++it) {
      if ((rc = start_all())) break;
      if (dirty && (rc = build_lists())) break;
      if ((rc = capture(1))) break;
      cudaEventRecord(e0, stream);
      if ((rc = cuda_check(cudaGraphLaunch(graph_exec, stream), "graph launch"))) break;
      cudaEventRecord(e1, stream);
      if ((rc = sync_stream())) break;
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      total += ms;
      n_ticks += 1;
      n_launches += launches_per_tick();
      for (int i : ids) slots[i].running = false;
      dirty = true;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    *ms_out = total / (double)iters;
    return OFDFT_OK;
#endif
  }

  // ---------------------------------------------------------- task lists
  // Whether a running slot takes the fused y-z pass: WT slots whose (y, z)
  // plane fits shared memory, outside the set-up passes.
  bool uses_yz(const HostSlot& h) const {
    return !h.setup_pass && yz_smem_slot(h.sd, 2 * elem_size(h.prec)) <= YZ_SMEM_MAX;
  }

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
      L[P_VEC].smem = std::max(L[P_VEC].smem, (size_t)(NCH * 33 * sizeof(double) + 16));
      const bool wgc = s.kinetic == KIN_WGC;
      const int px1 = wgc ? P_X1G : P_X1, pz3 = wgc ? P_Z3G : P_Z3, px5 = wgc ? P_X5G : P_X5;
      for (int r = 0; r < h.nrowpairs; r += h.rp1)
        L[px1].h.push_back({i, 0, r, std::min(h.rp1, h.nrowpairs - r)});
      L[px1].nthr = 256;
      L[px1].smem = std::max(L[px1].smem, xfwd_smem(s.n1, std::max(s.nf, s.ion.nspec), h.rp1, cs / 2));
      if (uses_yz(h)) {  // fused y-z pass: one task per (field, kx)
        const size_t sm = yz_smem_slot(s, cs);
        const bool big = h.yzt == 256 ? false : h.yzt == 512 ? true : sm > YZ_SMEM_SMALL;
        const int pyz = wgc ? (big ? P_YZBG : P_YZG) : (big ? P_YZB : P_YZ);
        for (int g = 0; g < s.ngroups; ++g)
          for (int kx = 0; kx < s.k1; ++kx) L[pyz].h.push_back({i, g, kx, 0});
        L[pyz].nthr = big ? 512 : 256;
        L[pyz].smem = std::max(L[pyz].smem, sm);
      } else {  // split path: y forward, z with the operator, y inverse
        for (int pass : {P_Y2, P_Y4}) {
          for (int f = 0; f < s.nf; ++f)
            for (int kx = 0; kx < s.k1; ++kx)
              for (int t = 0; t < tile_count(s.n3, h.ty); ++t)
                L[pass].h.push_back({i, f, kx, tile_code(s.n3, h.ty, t)});
          L[pass].nthr = 256;
          L[pass].smem = std::max(L[pass].smem, (size_t)h.ty * (s.n2 | 1) * cs);
        }
        const int gmax = s.kinetic == KIN_WGC ? 3 : 1;
        for (int g = 0; g < s.ngroups; ++g)
          for (int kx = 0; kx < s.k1; ++kx)
            for (int t = 0; t < tile_count(s.n2, h.tz); ++t)
              L[pz3].h.push_back({i, g, kx, tile_code(s.n2, h.tz, t)});
        L[pz3].nthr = 256;
        L[pz3].smem = std::max(L[pz3].smem, (size_t)std::max(gmax, s.ion.nspec) * h.tz * s.n3 * cs);
      }
      int ord = 0;
      for (int r = 0; r < h.nrowpairs; r += s.rp) L[px5].h.push_back({i, r, std::min(s.rp, h.nrowpairs - r), ord++});
      L[P_CTL].h.push_back({i, 0, 0, 0});
      L[P_CTL].nthr = 64;
      L[P_CTL].smem = 0;
      L[px5].nthr = 256;
      L[px5].smem = std::max(L[px5].smem, xinv_smem(s.n1, std::max(s.nf, s.ion.nspec), s.rp, cs / 2));
    }
#if defined(OFDFT_EMU)
    for (int p = 0; p < 2; ++p)
      for (int k = 0; k < NPASS; ++k) lists[p][k].nthr = 1;
#endif
    // every list packed into one device array, uploaded with one copy
    packed.clear();
    size_t off[2][NPASS];
    for (int p = 0; p < 2; ++p)
      for (int k = 0; k < NPASS; ++k) {
        off[p][k] = packed.size();
        packed.insert(packed.end(), lists[p][k].h.begin(), lists[p][k].h.end());
      }
    if (packed.size() > tasks_cap) {
      dfree(d_tasks);
      d_tasks = nullptr;
      tasks_cap = 0;
      const size_t nc = std::max<size_t>(packed.size(), 2 * tasks_cap + 1024);
      int rc = dmalloc((void**)&d_tasks, nc * sizeof(Task));
      if (rc) return rc;
      tasks_cap = nc;
    }
    for (int p = 0; p < 2; ++p)
      for (int k = 0; k < NPASS; ++k) lists[p][k].d = d_tasks + off[p][k];
    if (!packed.empty()) {
      int rc = h2d(d_tasks, packed.data(), packed.size() * sizeof(Task));
      if (rc) return rc;
    }
    dirty = false;
    return OFDFT_OK;
  }
  std::vector<Task> packed;  // host copy of the packed task lists
  Task* d_tasks = nullptr;
  size_t tasks_cap = 0;

  template <typename T>
  Args<T> args(int prec, int pass) {
    Args<T> a;
    a.slots = d_slots;
    a.ctl = d_ctl;
    a.tasks = lists[prec][pass].d;
    a.tw = (const cx<T>*)(prec == OFDFT_FP32 ? plans.d_tw32 : plans.d_tw64);
    a.idx = plans.d_idx;
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
    static double ctl_sm[CTL_SMEM_BYTES / sizeof(double)];
    for (int v = 0; v < VEC_PER_TICK; ++v) {
      run(P_VEC, [](Args<T>& a, int b, char* sm) { vec_block<T>(a, b, 0, 1, sm); });
      run(P_CTL, [](Args<T>& a, int b, char*) { ctl_block(a.slots, a.ctl, a.tasks, K_VEC, b, 0, 1, (char*)ctl_sm); });
    }
    run(P_X1, [](Args<T>& a, int b, char* sm) { xfwd_block<T, KS_WT>(a, b, 0, 1, sm); });
    run(P_X1G, [](Args<T>& a, int b, char* sm) { xfwd_block<T, KS_WGC>(a, b, 0, 1, sm); });
    run(P_Y2, [](Args<T>& a, int b, char* sm) { ypass_block<T>(a, b, 0, 1, sm, -1); });
    run(P_Z3, [](Args<T>& a, int b, char* sm) { zpass_block<T, KS_WT>(a, b, 0, 1, sm); });
    run(P_Z3G, [](Args<T>& a, int b, char* sm) { zpass_block<T, KS_WGC>(a, b, 0, 1, sm); });
    run(P_Y4, [](Args<T>& a, int b, char* sm) { ypass_block<T>(a, b, 0, 1, sm, 1); });
    run(P_YZ, [](Args<T>& a, int b, char* sm) { yzpass_block<T, KS_WT>(a, b, 0, 1, sm); });
    run(P_YZB, [](Args<T>& a, int b, char* sm) { yzpass_block<T, KS_WT>(a, b, 0, 1, sm); });
    run(P_YZG, [](Args<T>& a, int b, char* sm) { yzpass_block<T, KS_WGC>(a, b, 0, 1, sm); });
    run(P_YZBG, [](Args<T>& a, int b, char* sm) { yzpass_block<T, KS_WGC>(a, b, 0, 1, sm); });
    run(P_X5, [](Args<T>& a, int b, char* sm) { xinv_block<T, KS_WT>(a, b, 0, 1, sm); });
    run(P_X5G, [](Args<T>& a, int b, char* sm) { xinv_block<T, KS_WGC>(a, b, 0, 1, sm); });
    run(P_CTL, [](Args<T>& a, int b, char*) { ctl_block(a.slots, a.ctl, a.tasks, K_X5, b, 0, 1, (char*)ctl_sm); });
    return OFDFT_OK;
  }
#else
  template <typename T, typename K, typename... X>
  int launch_one(int prec, int pass, K kern, X... extra) {
    LaunchList& l = lists[prec][pass];
    if (l.h.empty()) return OFDFT_OK;
    kern<<<(unsigned)l.h.size(), l.nthr, l.smem, lstream>>>(args<T>(prec, pass), extra...);
    return cuda_check(cudaGetLastError(), "kernel launch");
  }
  template <typename T>
  int launch_prec(int prec) {
    int rc;
    for (int v = 0; v < VEC_PER_TICK; ++v) {
      if ((rc = launch_one<T>(prec, P_VEC, k_vec<T>))) return rc;
      if ((rc = launch_one<T>(prec, P_CTL, k_ctl<T>, (int)K_VEC))) return rc;
    }
    if ((rc = launch_one<T>(prec, P_X1, k_xfwd<T, KS_WT>))) return rc;
    if ((rc = launch_one<T>(prec, P_X1G, k_xfwd<T, KS_WGC>))) return rc;
    if ((rc = launch_one<T>(prec, P_YZ, k_yzpass<T, 256, KS_WT>))) return rc;
    if ((rc = launch_one<T>(prec, P_YZB, k_yzpass<T, 512, KS_WT>))) return rc;
    if ((rc = launch_one<T>(prec, P_YZG, k_yzpass<T, 256, KS_WGC>))) return rc;
    if ((rc = launch_one<T>(prec, P_YZBG, k_yzpass<T, 512, KS_WGC>))) return rc;
    if ((rc = launch_one<T>(prec, P_Y2, k_ypass<T>, -1))) return rc;
    if ((rc = launch_one<T>(prec, P_Z3, k_zpass<T, KS_WT>))) return rc;
    if ((rc = launch_one<T>(prec, P_Z3G, k_zpass<T, KS_WGC>))) return rc;
    if ((rc = launch_one<T>(prec, P_Y4, k_ypass<T>, 1))) return rc;
    if ((rc = launch_one<T>(prec, P_X5, k_xinv<T, KS_WT>))) return rc;
    if ((rc = launch_one<T>(prec, P_X5G, k_xinv<T, KS_WGC>))) return rc;
    return launch_one<T>(prec, P_CTL, k_ctl<T>, (int)K_X5);
  }
#endif

  int tick() {
    int rc;
    if ((rc = launch_prec<double>(OFDFT_FP64))) return rc;
    return launch_prec<float>(OFDFT_FP32);
  }
  bool has_work(int prec) const {
    for (int k = 0; k < NPASS; ++k)
      if (!lists[prec][k].h.empty()) return true;
    return false;
  }

#if !defined(OFDFT_EMU)
  // Load every kernel of the library now: with CUDA's lazy module loading the
  // first launch of each kernel would otherwise pay its load (10-30 ms), which
  // a serving engine would see as latency on its first requests.
  template <typename T>
  int preload_prec() {
    cudaFuncAttributes fa;
    int rc = OFDFT_OK;
    auto load = [&](auto kern) {
      if (!rc) rc = cuda_check(cudaFuncGetAttributes(&fa, kern), "kernel load");
    };
    load(k_vec<T>);
    load(k_ctl<T>);
    load(k_xfwd<T, KS_WT>);
    load(k_xfwd<T, KS_WGC>);
    load(k_ypass<T>);
    load(k_zpass<T, KS_WT>);
    load(k_zpass<T, KS_WGC>);
    load(k_yzpass<T, 256, KS_WT>);
    load(k_yzpass<T, 512, KS_WT>);
    load(k_yzpass<T, 256, KS_WGC>);
    load(k_yzpass<T, 512, KS_WGC>);
    load(k_xinv<T, KS_WT>);
    load(k_xinv<T, KS_WGC>);
    load(k_permute_kernel<T>);
    load(k_unpermute_kernel<T>);
    load(k_fill_kernel<T>);
    load(k_spread<T>);
    load(k_force_gather<T>);
    load(k_square_copy<T, T>);
    load(k_square_copy<T, double>);
    load(k_convert<double, T>);
    load(k_convert<T, double>);
    load(k_stress<T>);
    load(k_rho_vxc<T>);
    load(k_sum<T>);
    load(k_scale<T>);
    return rc;
  }
  int preload_kernels() {
    cudaFuncAttributes fa;
    int rc = preload_prec<float>();
    if (!rc) rc = preload_prec<double>();
    for (const void* k : {(const void*)k_ewald_real, (const void*)k_ewald_plane, (const void*)k_ewald_recip_force,
                          (const void*)k_ewald_real_stress, (const void*)k_ewald_plane_stress, (const void*)k_stress_sf})
      if (!rc) rc = cuda_check(cudaFuncGetAttributes(&fa, k), "kernel load");
    return rc;
  }

  // Kernels whose dynamic shared memory exceeds the default 48 KB need the
  // opt-in attribute; it must be set outside stream capture.
  template <typename T>
  int set_smem_attrs(int prec) {
    int rc;
    auto attr = [&](auto kern, int pass) -> int {
      const size_t sm = lists[prec][pass].smem;
      if (sm <= 48 * 1024) return OFDFT_OK;
      return cuda_check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm),
                        "cudaFuncSetAttribute");
    };
    if ((rc = attr(k_vec<T>, P_VEC))) return rc;
    if ((rc = attr(k_xfwd<T, KS_WT>, P_X1))) return rc;
    if ((rc = attr(k_xfwd<T, KS_WGC>, P_X1G))) return rc;
    if ((rc = attr(k_zpass<T, KS_WGC>, P_Z3G))) return rc;
    if ((rc = attr(k_xinv<T, KS_WGC>, P_X5G))) return rc;
    if ((rc = attr(k_ypass<T>, lists[prec][P_Y2].smem >= lists[prec][P_Y4].smem ? P_Y2 : P_Y4))) return rc;
    if ((rc = attr(k_yzpass<T, 256, KS_WT>, P_YZ))) return rc;
    if ((rc = attr(k_yzpass<T, 512, KS_WT>, P_YZB))) return rc;
    if ((rc = attr(k_yzpass<T, 256, KS_WGC>, P_YZG))) return rc;
    if ((rc = attr(k_yzpass<T, 512, KS_WGC>, P_YZBG))) return rc;
    if ((rc = attr(k_zpass<T, KS_WT>, P_Z3))) return rc;
    return attr(k_xinv<T, KS_WT>, P_X5);
  }

  // Capture `nticks` ticks into one CUDA graph (re-captured when the set of
  // running slots changes).
  long long n_captures = 0;
  double capture_ms = 0.0;  // host time spent capturing and instantiating graphs
  int capture(int nticks) {
    const auto t0 = std::chrono::steady_clock::now();
    const int rc0 = capture_graph(nticks);
    capture_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    ++n_captures;
    return rc0;
  }
  int capture_graph(int nticks) {
    if (graph_exec) {
      cudaGraphExecDestroy(graph_exec);
      graph_exec = nullptr;
    }
    int rc = set_smem_attrs<double>(OFDFT_FP64);
    if (!rc) rc = set_smem_attrs<float>(OFDFT_FP32);
    if (rc) return rc;
    if ((rc = cuda_check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture")))
      return rc;
    if (!(has_work(OFDFT_FP64) && has_work(OFDFT_FP32))) {
      for (int k = 0; k < nticks && rc == OFDFT_OK; ++k) rc = tick();
    } else {  // one branch per precision
      rc = cuda_check(cudaEventRecord(ev_fork, stream), "event record");
      if (!rc) rc = cuda_check(cudaStreamWaitEvent(stream2, ev_fork, 0), "stream wait");
      if (!rc) {
        for (int k = 0; k < nticks && rc == OFDFT_OK; ++k) rc = launch_prec<double>(OFDFT_FP64);
        lstream = stream2;
        for (int k = 0; k < nticks && rc == OFDFT_OK; ++k) rc = launch_prec<float>(OFDFT_FP32);
        lstream = stream;
        const int rj = cuda_check(cudaEventRecord(ev_join, stream2), "event record");
        const int rw = cuda_check(cudaStreamWaitEvent(stream, ev_join, 0), "stream wait");
        if (!rc) rc = rj ? rj : rw;
      }
    }
    cudaGraph_t g = nullptr;
    const int rc2 = cuda_check(cudaStreamEndCapture(stream, &g), "end capture");
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (rc2) return rc2;
    rc = cuda_check(cudaGraphInstantiate(&graph_exec, g, 0), "graph instantiate");
    cudaGraphDestroy(g);
    graph_ticks = nticks;
    return rc;
  }
#endif

  // Launch `n` ticks.  Several ticks go through a captured graph (captured
  // again when the task lists changed); a single tick (set-up passes, forces,
  // lone evaluations) is launched directly, since capturing and instantiating
  // a graph for one tick costs more than it saves.
  bool graph_stale = true;  // the task lists changed since the graph and the shared-memory limits were set
  bool attrs_stale = true;
  int launch_ticks(int n) {
    int rc;
    if (dirty) {
      if ((rc = build_lists())) return rc;
      graph_stale = true;
      attrs_stale = true;
    }
    n_ticks += n;
    n_launches += (long long)n * launches_per_tick();
#if !defined(OFDFT_EMU)
    if (n > 1) {
      if (graph_stale || !graph_exec || graph_ticks != n) {
        if ((rc = capture(n))) return rc;
        graph_stale = false;
        attrs_stale = false;
      }
      return cuda_check(cudaGraphLaunch(graph_exec, stream), "graph launch");
    }
    if (attrs_stale) {
      if ((rc = set_smem_attrs<double>(OFDFT_FP64)) || (rc = set_smem_attrs<float>(OFDFT_FP32))) return rc;
      attrs_stale = false;
    }
#endif
    for (int k = 0; k < n; ++k)
      if ((rc = tick())) return rc;
    return OFDFT_OK;
  }

  // Run ticks; after every `check` ticks read the slots' status and retire
  // finished slots from the task lists.
  int run(int ticks, int* running_out, int check = 8) {
    int running = 0;
    std::vector<Ctl> cs(cap);
    for (int t = 0; t < ticks;) {
      int n = std::min(check, ticks - t);
      int rc = launch_ticks(n);
      if (rc) return rc;
      t += n;
      if ((rc = d2h_stream(cs.data(), d_ctl, sizeof(Ctl) * cap))) return rc;
      running = 0;
      for (int i = 0; i < cap; ++i) {
        if (!slots[i].used || !slots[i].running) continue;
        if (cs[i].status == ST_RUNNING) {
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
  int rc = e->eng.init(256);
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
  int rc = e->eng.sync_stream();  // every use of the slot's memory is on the engine stream
  if (rc) return rc;
  e->eng.free_slot(slot);
  return OFDFT_OK;
}

int ofdft_slot_set_kernel(ofdft_engine* e, int slot, const double* kernel, int nplanes) {
  if (!e || !kernel) return fail(OFDFT_EINVAL, "null argument");
  int rc = e->eng.check_slot(slot);
  if (rc) return rc;
  HostSlot& h = e->eng.slots[slot];
  if (nplanes != h.nplanes) return fail(OFDFT_EINVAL, "kernel plane count does not match the functional");
  return e->eng.set_kernel(slot, kernel);
}

int ofdft_slot_set_ion_potential(ofdft_engine* e, int slot, const double* v) {
  if (!e || !v) return fail(OFDFT_EINVAL, "null argument");
  int rc = e->eng.check_slot(slot);
  if (rc) return rc;
  HostSlot& h = e->eng.slots[slot];
  return e->eng.upload_real(h.prec, h.sd.vion, v, h.sd.N);
}

int ofdft_slot_ewald(ofdft_engine* e, int slot, double* energy, double* forces) {
  if (!e) return fail(OFDFT_EINVAL, "null engine");
  return e->eng.slot_ewald(slot, energy, forces);
}

int ofdft_slot_copy_tables(ofdft_engine* e, int slot, int src_slot) {
  if (!e) return fail(OFDFT_EINVAL, "null engine");
  return e->eng.copy_tables(slot, src_slot);
}

int ofdft_slot_hold_density(ofdft_engine* e, int slot) {
  if (!e) return fail(OFDFT_EINVAL, "null engine");
  return e->eng.hold_density(slot);
}

int ofdft_slot_set_ion_ion_energy(ofdft_engine* e, int slot, double energy) {
  if (!e) return fail(OFDFT_EINVAL, "null engine");
  int rc = e->eng.check_slot(slot);
  if (rc) return rc;
  e->eng.slots[slot].sd.ion_ion = energy;
  return e->eng.upload_slot(slot);
}

int ofdft_slot_start_eval(ofdft_engine* e, int slot, const double* rho, int opt_sqrt, int want_energy) {
  if (!e) return fail(OFDFT_EINVAL, "null argument");
  return e->eng.start_eval(slot, rho, opt_sqrt, want_energy);
}

int ofdft_slot_start_solve(ofdft_engine* e, int slot, const double* rho, const ofdft_ntn_options* o) {
  if (!e) return fail(OFDFT_EINVAL, "null argument");
  return e->eng.start_solve(slot, rho, o);
}

int ofdft_slot_footprint(const ofdft_cell_desc* d, unsigned long long* bytes) {
  if (!d || !bytes) return fail(OFDFT_EINVAL, "null argument");
  const long long N = (long long)d->n1 * d->n2 * d->n3;
  const long long Nc = (long long)(d->n1 / 2 + 1) * d->n2 * d->n3;
  const long long es = d->precision == OFDFT_FP32 ? 4 : 8;
  const long long nf = d->kinetic == KIN_WGC ? 8 : (d->alpha == d->beta ? 3 : 4);
  const long long planes = d->kinetic == KIN_WGC ? 4 : 1;
  // NBUF state arrays, ion potential, resident input, kernel planes, spectra, partials
  *bytes = (unsigned long long)(es * N * (NBUF + 2) + es * Nc * planes + 2 * es * Nc * nf +
                                8LL * NCH * (N / VCHUNK + 1 + d->n2 * (long long)d->n3) + (1 << 20));
  return OFDFT_OK;
}

int ofdft_slot_set_input(ofdft_engine* e, int slot, const double* rho) {
  if (!e || !rho) return fail(OFDFT_EINVAL, "null argument");
  return e->eng.set_input(slot, rho);
}

int ofdft_engine_stream(ofdft_engine* e, void** stream) {
  if (!e || !stream) return fail(OFDFT_EINVAL, "null argument");
#if defined(OFDFT_EMU)
  *stream = nullptr;
#else
  *stream = (void*)e->eng.stream;
#endif
  return OFDFT_OK;
}

int ofdft_engine_counters(ofdft_engine* e, long long* kernel_launches, long long* ticks) {
  if (!e) return fail(OFDFT_EINVAL, "null engine");
  if (kernel_launches) *kernel_launches = e->eng.n_launches;
  if (ticks) *ticks = e->eng.n_ticks;
  return OFDFT_OK;
}

int ofdft_engine_capture_stats(ofdft_engine* e, long long* captures, double* host_ms) {
  if (!e) return fail(OFDFT_EINVAL, "null engine");
#if defined(OFDFT_EMU)
  if (captures) *captures = 0;
  if (host_ms) *host_ms = 0.0;
#else
  if (captures) *captures = e->eng.n_captures;
  if (host_ms) *host_ms = e->eng.capture_ms;
#endif
  return OFDFT_OK;
}

int ofdft_engine_time_eval(ofdft_engine* e, int iters, double* ms) {
  if (!e || !ms || iters < 1) return fail(OFDFT_EINVAL, "bad argument");
  return e->eng.time_eval(iters, ms);
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
    // rhoR = phi**2 (RhoOptN.f90:495), squared on the device
    if ((rc = g.download_real(h.prec, rho, h.sd.buf[c.iphi], h.sd.N, true))) return rc;
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
  if (g.slots[slot].running) {
    g.cancel(slot);
    return fail(OFDFT_ETIMEOUT, "evaluation did not finish");
  }
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
  if (g.slots[slot].running) {
    g.cancel(slot);  // the slot is idle again and can take a new solve
    return fail(OFDFT_ETIMEOUT, "solve exceeded the tick budget");
  }
  return ofdft_slot_result(e, slot, rho, energy, st);
}

int ofdft_slot_cancel(ofdft_engine* e, int slot) {
  if (!e) return fail(OFDFT_EINVAL, "null engine");
  return e->eng.cancel(slot);
}

int ofdft_slot_start_solve_from_slot(ofdft_engine* e, int slot, int src_slot, const ofdft_ntn_options* o) {
  if (!e) return fail(OFDFT_EINVAL, "null engine");
  return e->eng.start_solve_from(slot, src_slot, o);
}
int ofdft_slot_build_wt_kernel(ofdft_engine* e, int slot) {
  if (!e) return fail(OFDFT_EINVAL, "null engine");
  return e->eng.build_wt_kernel(slot);
}

int ofdft_slot_build_wgc_kernel(ofdft_engine* e, int slot, int ntab, const double* eta, const double* w,
                                const double* w1, const double* w2) {
  if (!e) return fail(OFDFT_EINVAL, "null engine");
  return e->eng.build_wgc_kernel(slot, ntab, eta, w, w1, w2);
}

int ofdft_slot_build_ion_potential(ofdft_engine* e, int slot, int nion, const double* frac, const int* species,
                                   int nspecies, const int* npts, const double* max_g, const double* charge,
                                   const double* pot_values, const double* vqs, const double* pot_dd) {
  if (!e || !frac || !species || !npts || !max_g || !charge || !pot_values || !vqs || !pot_dd)
    return fail(OFDFT_EINVAL, "null argument");
  return e->eng.build_ion_potential(slot, nion, frac, species, nspecies, npts, max_g, charge, pot_values, vqs,
                                    pot_dd);
}

int ofdft_slot_forces(ofdft_engine* e, int slot, const double* rho, int include_ewald, double* forces) {
  if (!e || !forces) return fail(OFDFT_EINVAL, "null argument");
  return e->eng.forces(slot, rho, include_ewald, forces);
}

int ofdft_engine_tune(ofdft_engine* e, int slot, int iters, double* ms_default, double* ms_tuned, int* shape) {
  if (!e || !ms_default || !ms_tuned) return fail(OFDFT_EINVAL, "null argument");
  return e->eng.tune(slot, iters, ms_default, ms_tuned, shape);
}

int ofdft_slot_shape(ofdft_engine* e, int slot, int* shape) {
  if (!e || !shape) return fail(OFDFT_EINVAL, "null argument");
  return e->eng.get_shape(slot, shape);
}

int ofdft_slot_set_shape(ofdft_engine* e, int slot, const int* shape) {
  if (!e || !shape) return fail(OFDFT_EINVAL, "null argument");
  return e->eng.pin_shape(slot, shape);
}

int ofdft_slot_set_lattice(ofdft_engine* e, int slot, const double* lattice, double rho0, double rho_s) {
  if (!e || !lattice) return fail(OFDFT_EINVAL, "null argument");
  return e->eng.set_lattice(slot, lattice, rho0, rho_s);
}

int ofdft_slot_rescale_input(ofdft_engine* e, int slot, double num_electrons) {
  if (!e) return fail(OFDFT_EINVAL, "null engine");
  return e->eng.rescale_input(slot, num_electrons);
}

int ofdft_slot_stress(ofdft_engine* e, int slot, const double* rho, int include_ewald, double* stress,
                      double* terms) {
  if (!e || !stress) return fail(OFDFT_EINVAL, "null argument");
  return e->eng.stress(slot, rho, include_ewald, stress, terms);
}

static_assert(sizeof(ofdft_line_search) == sizeof(LineSearch), "line-search record layout");

int ofdft_dcsrch(ofdft_line_search* ls, double* stp, double f, double g, int task) {
  if (!ls || !stp) return -fail(OFDFT_EINVAL, "null argument");
  if (task < OFDFT_LS_START || task > OFDFT_LS_FG) return -fail(OFDFT_EINVAL, "task must be START or FG");
  LineSearch L;
  memcpy(&L, ls, sizeof(L));
  const int out = ls_step(L, *stp, f, g, task);
  memcpy(ls, &L, sizeof(L));
  return out;
}

int ofdft_ewald(const double* lattice, int nion, const double* frac, const double* charges, double* energy,
                double* forces) {
  if (!lattice || !frac || !charges || !energy || nion < 1) return fail(OFDFT_EINVAL, "bad argument");
  *energy = ewald(lattice, nion, frac, charges, forces);
  return OFDFT_OK;
}

int ofdft_grid_size(double ecut_ha, const double* lattice, int* n) {
  if (!lattice || !n || !(ecut_ha > 0)) return fail(OFDFT_EINVAL, "bad argument");
  // SizeSystem / PadFFTdims (SetupFFT.f90:193-382), dimType 1
  const double qmax = std::sqrt(ecut_ha * 2.0);
  for (int a = 0; a < 3; ++a) {
    const double len = std::sqrt(lattice[3 * a] * lattice[3 * a] + lattice[3 * a + 1] * lattice[3 * a + 1] +
                                 lattice[3 * a + 2] * lattice[3 * a + 2]);
    const double r = qmax * len / PI_D;
    const double eps = 1.0e-14, lr = std::log(r);
    const int p2 = (int)(lr / std::log(2.0) - eps + 1), p3 = (int)(lr / std::log(3.0) - eps + 1);
    const int p5 = (int)(lr / std::log(5.0) - eps + 1), p7 = (int)(lr / std::log(7.0) - eps + 1);
    long long best = 1;
    for (int k = 0; k < p7; ++k) best *= 7;
    for (int i7 = 0; i7 <= p7; ++i7)
      for (int i5 = 0; i5 <= p5; ++i5)
        for (int i3 = 0; i3 <= p3; ++i3)
          for (int i2 = 0; i2 <= p2; ++i2) {
            long long t = 1;
            for (int k = 0; k < i7; ++k) t *= 7;
            for (int k = 0; k < i5; ++k) t *= 5;
            for (int k = 0; k < i3; ++k) t *= 3;
            for (int k = 0; k < i2; ++k) t *= 2;
            if ((double)t >= r) {
              if (t < best) best = t;
              break;
            }
          }
    n[a] = (int)best;
  }
  return OFDFT_OK;
}

int ofdft_wgc_radial_tables(double alpha, double beta, double gamma, int max, double* eta, double* w, double* w1,
                            double* w2, int* n) {
  if (!n) return fail(OFDFT_EINVAL, "null argument");
  std::vector<double> te, tw, tw1, tw2;
  if (wgc_radial_tables(alpha, beta, gamma, te, tw, tw1, tw2)) return fail(OFDFT_EINVAL, "ODE did not converge");
  *n = (int)te.size();
  if (max < (int)te.size()) return OFDFT_OK;  // size query
  for (size_t k = 0; k < te.size(); ++k) {
    if (eta) eta[k] = te[k];
    if (w) w[k] = tw[k];
    if (w1) w1[k] = tw1[k];
    if (w2) w2[k] = tw2[k];
  }
  return OFDFT_OK;
}

}  // extern "C"

// ------------------------------------------------------------ allocation-free evaluation
// For callers that must not allocate device memory (for example a host code
// that runs inside a memory pool it does not own, or under a device-memory
// budget fixed before the solve starts): one CalculatePotentialPlus-style
// evaluation whose scratch (slot descriptor, controller record, FFT
// twiddles, spectra, reduction partials and task lists) lives in the
// file-scope device array below.  Every GPU that loads this library holds
// the array until the process exits.  Calls share it, so two calls whose
// work overlaps on the same GPU race; each call rewrites everything it reads.
// The host-side staging (task lists, twiddles, controller record) belongs to
// the calling thread, so calls from different host threads on different
// GPUs are independent.
#if !defined(OFDFT_EMU)
namespace noalloc {
constexpr size_t SCRATCH_BYTES = size_t(12) << 20;  // 12 MiB
constexpr long long MAX_POINTS = 262144;             // 64^3 grid points
constexpr int MAX_DIM = 128;
constexpr int MAX_TASKS = 12288;
constexpr int MAX_DEVICES = 128;
static __device__ __align__(256) unsigned char g_scratch[SCRATCH_BYTES];
static void* g_addr[MAX_DEVICES];  // device address of g_scratch per device ordinal
static std::mutex g_addr_mu;       // guards the first look-up on each device
static thread_local Task t_tasks[MAX_TASKS];  // this thread's staging of the task lists

// The device address of g_scratch on the current device (looked up once per
// device, with that device current).
static int scratch_address(int dev, char** base) {
  std::lock_guard<std::mutex> lock(g_addr_mu);
  if (!g_addr[dev]) {
    void* a = nullptr;
    const int rc = cuda_check(cudaGetSymbolAddress(&a, g_scratch), "cudaGetSymbolAddress");
    if (rc) return rc;
    g_addr[dev] = a;
  }
  *base = (char*)g_addr[dev];
  return OFDFT_OK;
}

static size_t up256(size_t x) { return (x + 255) & ~size_t(255); }

// Plan of length n (the engine's FP64 radix rule) with its roots of unity
// appended to tw at *toff and its digit-reversal tables to idx at *ioff (no
// heap use).
static void make_plan(int n, FftPlan& p, cx<double>* tw, int* toff, int* idx, int* ioff) {
  memset(&p, 0, sizeof(p));
  int rad[FFT_MAX_STAGES];
  const int nst = fft_radices(n, FftMaxRadix<double>::value, rad);
  fft_plan_fill(p, n, rad, nst, idx + *ioff, idx + *ioff + n);
  p.root = *toff;
  p.perm = *ioff;
  p.iperm = *ioff + n;
  for (int e = 0; e < n; ++e) {
    const long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)e / (long double)n;
    tw[*toff + e] = mk<double>((double)cosl(a), (double)sinl(a));
  }
  *toff += n;
  *ioff += 2 * n;
}
}  // namespace noalloc
#endif

extern "C" int ofdft_calculate_potential_plus_noalloc(const ofdft_cell_desc* d, const double* rho,
                                                      const double* kernel, const double* ion_pot, int opt_sqrt,
                                                      double* potential, double* etable, void* stream_ptr) {
#if defined(OFDFT_EMU)
  (void)d; (void)rho; (void)kernel; (void)ion_pot; (void)opt_sqrt; (void)potential; (void)etable; (void)stream_ptr;
  return fail(OFDFT_EINVAL, "the allocation-free evaluation needs the CUDA build");
#else
  using namespace noalloc;
  if (!d || !rho || !kernel || !ion_pot || !potential) return fail(OFDFT_EINVAL, "null argument");
  if (d->kinetic != KIN_WT || d->precision != OFDFT_FP64)
    return fail(OFDFT_EINVAL, "the allocation-free evaluation supports the FP64 WT functional only");
  const int ns[3] = {d->n1, d->n2, d->n3};
  for (int k = 0; k < 3; ++k)
    if (ns[k] < 2 || ns[k] > MAX_DIM || !seven_smooth(ns[k]))
      return fail(OFDFT_EINVAL, "grid dimensions must be 7-smooth and in [2, 128]");
  const long long N = (long long)d->n1 * d->n2 * d->n3;
  if (N > MAX_POINTS)
    return fail(OFDFT_EINVAL, "grid too large for the allocation-free evaluation (at most 262144 points)");
  // Host planning first (descriptor, plans, task lists, scratch layout): a
  // grid the fixed scratch cannot hold is refused before any CUDA call.
  // slot descriptor (as ofdft_slot_create fills it) pointing at the caller's buffers
  SlotDev s;
  memset(&s, 0, sizeof(s));
  s.n1 = d->n1; s.n2 = d->n2; s.n3 = d->n3;
  s.k1 = d->n1 / 2 + 1;
  s.N = N;
  s.Nc = (long long)s.k1 * d->n2 * d->n3;
  cx<double> tw[3 * MAX_DIM];  // roots of unity of the three plans
  int ptab[6 * MAX_DIM];        // their digit-reversal tables
  int twoff = 0, poff = 0;
  make_plan(d->n1, s.px, tw, &twoff, ptab, &poff);
  make_plan(d->n2, s.py, tw, &twoff, ptab, &poff);
  make_plan(d->n3, s.pz, tw, &twoff, ptab, &poff);
  const double* L = d->lattice;
  auto A = [&](int r, int c) { return L[3 * c + r]; };
  const double det = A(0, 0) * (A(1, 1) * A(2, 2) - A(1, 2) * A(2, 1)) - A(0, 1) * (A(1, 0) * A(2, 2) - A(1, 2) * A(2, 0)) +
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
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) s.recip[3 * c + r] = inv[c][r] * 2.0 * 3.141592653589793238462643;
  s.vol = std::fabs(det);
  s.dv = s.vol / (double)N;
  s.inv_n = 1.0 / (double)N;
  s.kinetic = KIN_WT;
  s.lambda = d->lambda; s.mu = d->mu; s.alpha = d->alpha; s.beta = d->beta;
  s.rho_s = d->rho_s; s.ion_ion = d->ion_ion_energy;
  s.alpha_eq_beta = d->alpha == d->beta ? 1 : 0;
  s.pow56 = (s.alpha_eq_beta && std::fabs(d->alpha - 5.0 / 6.0) < 1e-15) ? 1 : 0;
  s.nf = s.alpha_eq_beta ? 3 : 4;
  s.ngroups = s.nf;
  const int kinds[4] = {G_HARTREE, G_KMUL, G_VW, G_KMUL};
  for (int g = 0; g < s.ngroups; ++g) { s.group_kind[g] = kinds[g]; s.group_f0[g] = g; s.group_nf[g] = 1; }
  const size_t cs = sizeof(cx<double>);
  const int nrows = s.n2 * s.n3, nrp = (nrows + 1) / 2;
  int rp1 = 1, ty = 1, tz = 1;
  launch_shape(s, cs, s.nf, &rp1, &ty, &tz);  // the engine's own launch shape
  s.ntask[K_X5] = (nrp + s.rp - 1) / s.rp;
  s.buf[B_PHI] = (void*)rho;         // the input density (read only in EV_RHO mode)
  s.buf[B_W0] = (void*)potential;    // the output potential
  s.vion = (void*)ion_pot;
  // the engine's passes: the fused y-z pass when the plane fits, else the split path
  const size_t yzsm = yz_smem(s, cs);
  const bool fused = yzsm <= YZ_SMEM_MAX;
  const int yzthr = yzsm <= YZ_SMEM_SMALL ? 256 : 512;
  // task lists, packed one pass after the other: x forward, y forward (or
  // y-z), z, y inverse, x inverse, controller
  int nt[6] = {0, 0, 0, 0, 0, 0}, ntot = 0;
  auto push = [&](int pass, Task t) -> bool {
    if (ntot >= MAX_TASKS) return false;
    t_tasks[ntot++] = t;
    nt[pass]++;
    return true;
  };
  bool ok = true;
  for (int r = 0; r < nrp && ok; r += rp1) ok = push(0, {0, 0, r, std::min(rp1, nrp - r)});
  if (fused) {
    for (int g = 0; g < s.ngroups && ok; ++g)
      for (int kx = 0; kx < s.k1 && ok; ++kx) ok = push(1, {0, g, kx, 0});
  } else {
    for (int f = 0; f < s.nf && ok; ++f)
      for (int kx = 0; kx < s.k1 && ok; ++kx)
        for (int t = 0; t < tile_count(s.n3, ty) && ok; ++t) ok = push(1, {0, f, kx, tile_code(s.n3, ty, t)});
    for (int g = 0; g < s.ngroups && ok; ++g)
      for (int kx = 0; kx < s.k1 && ok; ++kx)
        for (int t = 0; t < tile_count(s.n2, tz) && ok; ++t) ok = push(2, {0, g, kx, tile_code(s.n2, tz, t)});
  }
  int ord = 0;
  for (int r = 0; r < nrp && ok; r += s.rp) ok = push(3, {0, r, std::min(s.rp, nrp - r), ord++});
  if (ok) ok = push(4, {0, 0, 0, 0});
  if (!ok) return fail(OFDFT_EINVAL, "grid needs more tasks than the allocation-free evaluation holds");
  // scratch layout
  size_t o = 0;
  const size_t o_slot = o; o = up256(o + sizeof(SlotDev));
  const size_t o_ctl = o; o = up256(o + sizeof(Ctl));
  const size_t o_tw = o; o = up256(o + cs * (size_t)twoff);
  const size_t o_idx = o; o = up256(o + sizeof(int) * (size_t)poff);
  const size_t o_part = o; o = up256(o + sizeof(double) * NCH * (size_t)s.ntask[K_X5]);
  const size_t o_task = o; o = up256(o + sizeof(Task) * (size_t)ntot);
  const size_t o_kern = o; o = up256(o + sizeof(double) * (size_t)s.Nc);
  const size_t o_spec = o; o = up256(o + cs * (size_t)s.nf * (size_t)s.Nc);
  if (o > SCRATCH_BYTES) return fail(OFDFT_EINVAL, "grid needs more scratch than the allocation-free evaluation holds");
  cudaStream_t st = (cudaStream_t)stream_ptr;
  int dev = 0;
  int rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (rc) return rc;
  if (dev < 0 || dev >= MAX_DEVICES) return fail(OFDFT_EINVAL, "device ordinal out of range");
  char* base = nullptr;
  if ((rc = scratch_address(dev, &base))) return rc;
  s.partials = (double*)(base + o_part);
  s.spec = (void*)(base + o_spec);
  s.kern = (void*)(base + o_kern);  // the caller's keKernel, permuted into the engine's layout below
  Ctl ctl;
  memset(&ctl, 0, sizeof(ctl));
  ctl.status = ST_RUNNING;
  ctl.iphi = B_PHI; ctl.itrial = B_TRIAL; ctl.iw0 = B_W0; ctl.iw1 = B_W1; ctl.evb = B_P;
  ctl.ev = EV_RHO;
  ctl.opt_sqrt = opt_sqrt ? 1 : 0;
  ctl.want_energy = etable ? 1 : 0;
  ctl.dscale = 1.0;
  if ((rc = cuda_check(cudaMemcpyAsync(base + o_slot, &s, sizeof(SlotDev), cudaMemcpyHostToDevice, st), "H2D")))
    return rc;
  if ((rc = cuda_check(cudaMemcpyAsync(base + o_ctl, &ctl, sizeof(Ctl), cudaMemcpyHostToDevice, st), "H2D")))
    return rc;
  if ((rc = cuda_check(cudaMemcpyAsync(base + o_tw, tw, cs * (size_t)twoff, cudaMemcpyHostToDevice, st), "H2D")))
    return rc;
  if ((rc = cuda_check(cudaMemcpyAsync(base + o_idx, ptab, sizeof(int) * (size_t)poff, cudaMemcpyHostToDevice, st),
                       "H2D")))
    return rc;
  if ((rc = cuda_check(cudaMemcpyAsync(base + o_task, t_tasks, sizeof(Task) * (size_t)ntot, cudaMemcpyHostToDevice,
                                       st), "H2D")))
    return rc;
  const int* didx = (const int*)(base + o_idx);
  k_permute_kernel<double><<<(unsigned)std::min<long long>(4 * 148, (s.Nc + 255) / 256), 256, 0, st>>>(
      (const SlotDev*)(base + o_slot), didx, kernel, 1);
  // launches: the passes and the controller kernel, as one engine tick does
  Args<double> a;
  a.slots = (SlotDev*)(base + o_slot);
  a.ctl = (Ctl*)(base + o_ctl);
  a.tw = (const cx<double>*)(base + o_tw);
  a.idx = didx;
  a.vchunk = VCHUNK;
  const size_t sm1 = xfwd_smem(s.n1, s.nf, rp1, cs / 2);
  const size_t sm2 = (size_t)ty * (s.n2 | 1) * cs;
  const size_t sm3 = (size_t)tz * s.n3 * cs;
  const size_t sm5 = xinv_smem(s.n1, s.nf, s.rp, cs / 2);
  auto attr = [&](auto kern, size_t sm) -> int {
    if (sm <= 48 * 1024) return OFDFT_OK;
    return cuda_check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm),
                      "cudaFuncSetAttribute");
  };
  if ((rc = attr(k_xfwd<double, KS_WT>, sm1)) || (rc = attr(k_xinv<double, KS_WT>, sm5)))
    return rc;
  if (fused && (rc = yzthr == 256 ? attr(k_yzpass<double, 256, KS_WT>, yzsm) : attr(k_yzpass<double, 512, KS_WT>, yzsm)))
    return rc;
  if (!fused && ((rc = attr(k_ypass<double>, sm2)) || (rc = attr(k_zpass<double, KS_WT>, sm3))))
    return rc;
  const Task* tb = (const Task*)(base + o_task);
  a.tasks = tb;
  k_xfwd<double, KS_WT><<<nt[0], 256, sm1, st>>>(a);
  a.tasks = tb + nt[0];
  if (fused) {
    if (yzthr == 256) k_yzpass<double, 256, KS_WT><<<nt[1], 256, yzsm, st>>>(a);
    else k_yzpass<double, 512, KS_WT><<<nt[1], 512, yzsm, st>>>(a);
  } else {
    k_ypass<double><<<nt[1], 256, sm2, st>>>(a, -1);
    a.tasks = tb + nt[0] + nt[1];
    k_zpass<double, KS_WT><<<nt[2], 256, sm3, st>>>(a);
    a.tasks = tb + nt[0];
    k_ypass<double><<<nt[1], 256, sm2, st>>>(a, 1);
  }
  a.tasks = tb + nt[0] + nt[1] + nt[2];
  k_xinv<double, KS_WT><<<nt[3], 256, sm5, st>>>(a);
  a.tasks = tb + nt[0] + nt[1] + nt[2] + nt[3];
  k_ctl<double><<<1, 64, 0, st>>>(a, (int)K_X5);
  if ((rc = cuda_check(cudaGetLastError(), "kernel launch"))) return rc;
  if ((rc = cuda_check(cudaMemcpyAsync(&ctl, base + o_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st), "D2H")))
    return rc;
  if ((rc = cuda_check(cudaStreamSynchronize(st), "stream synchronize"))) return rc;
  if ((rc = status_code(ctl))) return rc;
  if (etable)
    for (int k = 0; k < 9; ++k) etable[k] = ctl.energy[k];
  return OFDFT_OK;
#endif
}

