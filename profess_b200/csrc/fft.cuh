// Batched mixed-radix Stockham FFT over shared memory.
//
// A transform of length n = R_0 * R_1 * ... runs as one Stockham stage per
// radix.  The radices are 2, 3, 4, 5, 7, 8 and the compound radices 6, 9, 10,
// 12, 14, 15, 16, whose R-point DFTs run in registers as an A x B
// Cooley-Tukey split of the small DFTs with compile-time twiddles, so most
// lengths up to 256 take two stages.  Each stage reads R points at stride n/R,
// multiplies by the stage twiddles, does the R-point DFT in registers and
// writes the R outputs in self-sorting order, ping-ponging between two shared
// buffers; the caller reads the result from whichever buffer fft_batch
// returns.  Many independent transforms of the same length are done together:
// element i of transform b lives at buf[b + i*si].  Work items (b, butterfly)
// are spread over the block's threads with b fastest, so consecutive threads
// touch consecutive shared-memory words; the index arithmetic uses
// multiply-high divisions by constants prepared on the host.  The direction
// (DIR = -1 forward, +1 inverse) is a template parameter.
//
// Twiddles are precomputed on the host in long double and stored per plan:
// stage s with span Ns (product of the earlier radices) and radix R uses
// tw[off_s + k*(R-1) + (m-1)] = exp(-2*pi*i*m*k/(Ns*R)), k = 0..Ns-1.
// The inverse transform uses the conjugates.  No scaling is applied here.
#pragma once
#include "cx.cuh"

namespace ofdft {

constexpr int FFT_MAX_STAGES = 12;
constexpr int FFT_MAX_RADIX = 16;

// Largest radix of the FP32 and FP64 plans.  An R-point DFT holds R complex
// values in registers; only the radices up to the limit are compiled into a
// precision's kernels, so the limit also bounds their register use.
#ifndef OFDFT_RMAX_FP32
#define OFDFT_RMAX_FP32 8
#endif
#ifndef OFDFT_RMAX_FP64
#define OFDFT_RMAX_FP64 8
#endif
template <typename T> struct FftMaxRadix { static constexpr int value = OFDFT_RMAX_FP32; };
template <> struct FftMaxRadix<double> { static constexpr int value = OFDFT_RMAX_FP64; };

struct FftPlan {
  int n;
  int nst;
  int R[FFT_MAX_STAGES];
  int Ns[FFT_MAX_STAGES];
  int tw[FFT_MAX_STAGES];  // offset of the stage's twiddles in the plan table
  unsigned ns_magic[FFT_MAX_STAGES];  // ceil(2^20 / Ns): j / Ns == (j * magic) >> 20 for j < 2048
  int tw_base;             // offset of this plan in the global twiddle table
  int root;                // offset of exp(-2 pi i e / n), e = 0..n-1, in that table; -1: none
};

// Exact quotient j / d for 0 <= j < 2048 and 1 <= d <= 512 from magic = ceil(2^20 / d).
HD int magic_div(int j, unsigned magic) { return (int)(((unsigned)j * magic) >> 20); }

// Exact quotient w / d for 0 <= w < 2^24 and 1 <= d <= 4096 from m32 = ceil(2^32 / d)
// (d = 1 is encoded as m32 = 0).
HD int magic_div32(int w, unsigned m32) {
#if defined(__CUDA_ARCH__)
  const int q = (int)__umulhi((unsigned)w, m32);
#else
  const int q = (int)(((unsigned long long)(unsigned)w * m32) >> 32);
#endif
  return m32 == 0u ? w : q;
}
HD unsigned magic32(int d) {
  return d <= 1 ? 0u : (unsigned)((0x100000000ULL + (unsigned long long)d - 1) / (unsigned long long)d);
}

// cos/sin of 2*pi*k/R for the odd radices (mathematical constants).
#define OFDFT_S3 0.8660254037844386467637232
#define OFDFT_C51 0.3090169943749474241022934
#define OFDFT_C52 -0.8090169943749474241022934
#define OFDFT_S51 0.9510565162951535721164393
#define OFDFT_S52 0.5877852522924731291687060
#define OFDFT_C71 0.6234898018587335305250049
#define OFDFT_C72 -0.2225209339563144042889026
#define OFDFT_C73 -0.9009688679024191262361023
#define OFDFT_S71 0.7818314824680298087084445
#define OFDFT_S72 0.9749279121818236070181317
#define OFDFT_S73 0.4338837391175581204757683
#define OFDFT_R2 0.7071067811865475244008444

template <typename T>
HD void dft2(cx<T>* v) {
  cx<T> a = v[0], b = v[1];
  v[0] = a + b;
  v[1] = a - b;
}

template <typename T>
HD void dft3(cx<T>* v, int dir) {
  const T s = T(OFDFT_S3);
  cx<T> t1 = v[1] + v[2];
  cx<T> t2 = v[0] - t1 * T(0.5);
  cx<T> t3 = mul_i(v[1] - v[2], dir) * s;
  v[0] = v[0] + t1;
  v[1] = t2 + t3;
  v[2] = t2 - t3;
}

template <typename T>
HD void dft4(cx<T>* v, int dir) {
  cx<T> a = v[0] + v[2], b = v[0] - v[2];
  cx<T> c = v[1] + v[3], d = mul_i(v[1] - v[3], dir);
  v[0] = a + c;
  v[2] = a - c;
  v[1] = b + d;
  v[3] = b - d;
}

template <typename T>
HD void dft5(cx<T>* v, int dir) {
  const T c1 = T(OFDFT_C51), c2 = T(OFDFT_C52), s1 = T(OFDFT_S51), s2 = T(OFDFT_S52);
  cx<T> t1 = v[1] + v[4], t2 = v[2] + v[3], t3 = v[1] - v[4], t4 = v[2] - v[3];
  cx<T> a1 = v[0] + t1 * c1 + t2 * c2;
  cx<T> a2 = v[0] + t1 * c2 + t2 * c1;
  cx<T> b1 = mul_i(t3 * s1 + t4 * s2, dir);
  cx<T> b2 = mul_i(t3 * s2 - t4 * s1, dir);
  v[0] = v[0] + t1 + t2;
  v[1] = a1 + b1;
  v[4] = a1 - b1;
  v[2] = a2 + b2;
  v[3] = a2 - b2;
}

template <typename T>
HD void dft7(cx<T>* v, int dir) {
  const T c[4] = {T(1), T(OFDFT_C71), T(OFDFT_C72), T(OFDFT_C73)};
  const T s[4] = {T(0), T(OFDFT_S71), T(OFDFT_S72), T(OFDFT_S73)};
  cx<T> tp[4], tm[4];
#pragma unroll
  for (int k = 1; k <= 3; ++k) {
    tp[k] = v[k] + v[7 - k];
    tm[k] = v[k] - v[7 - k];
  }
  cx<T> y[7];
  y[0] = v[0] + tp[1] + tp[2] + tp[3];
#pragma unroll
  for (int j = 1; j <= 3; ++j) {
    cx<T> a = v[0], b = mk<T>(T(0), T(0));
#pragma unroll
    for (int k = 1; k <= 3; ++k) {
      int m = (j * k) % 7;
      T cc = m <= 3 ? c[m] : c[7 - m];
      T ss = m <= 3 ? s[m] : -s[7 - m];
      a = a + tp[k] * cc;
      b = b + tm[k] * ss;
    }
    cx<T> ib = mul_i(b, dir);
    y[j] = a + ib;
    y[7 - j] = a - ib;
  }
#pragma unroll
  for (int k = 0; k < 7; ++k) v[k] = y[k];
}

template <typename T>
HD void dft8(cx<T>* v, int dir) {
  cx<T> e[4] = {v[0], v[2], v[4], v[6]};
  cx<T> o[4] = {v[1], v[3], v[5], v[7]};
  dft4(e, dir);
  dft4(o, dir);
  const T r = T(OFDFT_R2);
  // t_k = w8^k o_k with w8 = exp(dir*2*pi*i/8)
  cx<T> t0 = o[0];
  cx<T> t1 = (o[1] + mul_i(o[1], dir)) * r;
  cx<T> t2 = mul_i(o[2], dir);
  cx<T> t3 = (mul_i(o[3], dir) - o[3]) * r;
  v[0] = e[0] + t0; v[4] = e[0] - t0;
  v[1] = e[1] + t1; v[5] = e[1] - t1;
  v[2] = e[2] + t2; v[6] = e[2] - t2;
  v[3] = e[3] + t3; v[7] = e[3] - t3;
}

// cos(2 pi e / R) (want_sin = 0) or sin(2 pi e / R) for the compound radices
// (mathematical constants), evaluated at compile time.
HDC double root_cs(int R, int e, int want_sin) {
  switch (R) {
    case 6: {
      const double c[6] = {1.0, 0.5, -0.5, -1.0, -0.5, 0.5};
      const double s[6] = {0.0, 0.8660254037844386467637232, 0.8660254037844386467637232, 0.0, -0.8660254037844386467637232, -0.8660254037844386467637232};
      return want_sin ? s[e] : c[e];
    }
    case 9: {
      const double c[9] = {1.0, 0.7660444431189780352023927, 0.1736481776669303488517166, -0.5, -0.9396926207859083840541093, -0.9396926207859083840541093, -0.5, 0.1736481776669303488517166, 0.7660444431189780352023927};
      const double s[9] = {0.0, 0.6427876096865393263226434, 0.984807753012208059366743, 0.8660254037844386467637232, 0.3420201433256687330440996, -0.3420201433256687330440996, -0.8660254037844386467637232, -0.984807753012208059366743, -0.6427876096865393263226434};
      return want_sin ? s[e] : c[e];
    }
    case 10: {
      const double c[10] = {1.0, 0.8090169943749474241022934, 0.3090169943749474241022934, -0.3090169943749474241022934, -0.8090169943749474241022934, -1.0, -0.8090169943749474241022934, -0.3090169943749474241022934, 0.3090169943749474241022934, 0.8090169943749474241022934};
      const double s[10] = {0.0, 0.587785252292473129168706, 0.9510565162951535721164393, 0.9510565162951535721164393, 0.587785252292473129168706, 0.0, -0.587785252292473129168706, -0.9510565162951535721164393, -0.9510565162951535721164393, -0.587785252292473129168706};
      return want_sin ? s[e] : c[e];
    }
    case 12: {
      const double c[12] = {1.0, 0.8660254037844386467637232, 0.5, 0.0, -0.5, -0.8660254037844386467637232, -1.0, -0.8660254037844386467637232, -0.5, 0.0, 0.5, 0.8660254037844386467637232};
      const double s[12] = {0.0, 0.5, 0.8660254037844386467637232, 1.0, 0.8660254037844386467637232, 0.5, 0.0, -0.5, -0.8660254037844386467637232, -1.0, -0.8660254037844386467637232, -0.5};
      return want_sin ? s[e] : c[e];
    }
    case 14: {
      const double c[14] = {1.0, 0.9009688679024191262361023, 0.6234898018587335305250049, 0.2225209339563144042889026, -0.2225209339563144042889026, -0.6234898018587335305250049, -0.9009688679024191262361023, -1.0, -0.9009688679024191262361023, -0.6234898018587335305250049, -0.2225209339563144042889026, 0.2225209339563144042889026, 0.6234898018587335305250049, 0.9009688679024191262361023};
      const double s[14] = {0.0, 0.4338837391175581204757683, 0.7818314824680298087084445, 0.9749279121818236070181317, 0.9749279121818236070181317, 0.7818314824680298087084445, 0.4338837391175581204757683, 0.0, -0.4338837391175581204757683, -0.7818314824680298087084445, -0.9749279121818236070181317, -0.9749279121818236070181317, -0.7818314824680298087084445, -0.4338837391175581204757683};
      return want_sin ? s[e] : c[e];
    }
    case 15: {
      const double c[15] = {1.0, 0.9135454576426008955021276, 0.6691306063588582138262733, 0.3090169943749474241022934, -0.1045284632676534713998342, -0.5, -0.8090169943749474241022934, -0.9781476007338056379285667, -0.9781476007338056379285667, -0.8090169943749474241022934, -0.5, -0.1045284632676534713998342, 0.3090169943749474241022934, 0.6691306063588582138262733, 0.9135454576426008955021276};
      const double s[15] = {0.0, 0.406736643075800207753986, 0.743144825477394235014697, 0.9510565162951535721164393, 0.9945218953682733369226919, 0.8660254037844386467637232, 0.587785252292473129168706, 0.2079116908177593371017423, -0.2079116908177593371017423, -0.587785252292473129168706, -0.8660254037844386467637232, -0.9945218953682733369226919, -0.9510565162951535721164393, -0.743144825477394235014697, -0.406736643075800207753986};
      return want_sin ? s[e] : c[e];
    }
    case 16: {
      const double c[16] = {1.0, 0.9238795325112867561281832, 0.7071067811865475244008444, 0.38268343236508977172846, 0.0, -0.38268343236508977172846, -0.7071067811865475244008444, -0.9238795325112867561281832, -1.0, -0.9238795325112867561281832, -0.7071067811865475244008444, -0.38268343236508977172846, 0.0, 0.38268343236508977172846, 0.7071067811865475244008444, 0.9238795325112867561281832};
      const double s[16] = {0.0, 0.38268343236508977172846, 0.7071067811865475244008444, 0.9238795325112867561281832, 1.0, 0.9238795325112867561281832, 0.7071067811865475244008444, 0.38268343236508977172846, 0.0, -0.38268343236508977172846, -0.7071067811865475244008444, -0.9238795325112867561281832, -1.0, -0.9238795325112867561281832, -0.7071067811865475244008444, -0.38268343236508977172846};
      return want_sin ? s[e] : c[e];
    }
    default:
      return 0.0;
  }
}

// x * exp(DIR * 2 pi i E / R), with the trivial angles special-cased.
template <typename T, int R, int E, int DIR>
HD cx<T> twiddle_const(cx<T> x) {
  constexpr int e = E % R;
  if constexpr (e == 0) {
    return x;
  } else if constexpr (2 * e == R) {
    return mk<T>(-x.x, -x.y);
  } else if constexpr (4 * e == R) {
    return mul_i(x, DIR);
  } else if constexpr (4 * e == 3 * R) {
    return mul_i(x, -DIR);
  } else {
    constexpr double c = root_cs(R, e, 0);
    constexpr double s = root_cs(R, e, 1);
    return cmul(x, mk<T>(T(c), T(DIR * s)));
  }
}

template <typename T, int R, int DIR> struct Dft;
template <typename T, int A, int B, int DIR> HD void dft_ab(cx<T>* v);

template <typename T, int DIR> struct Dft<T, 2, DIR> { static HD void run(cx<T>* v) { dft2(v); } };
template <typename T, int DIR> struct Dft<T, 3, DIR> { static HD void run(cx<T>* v) { dft3(v, DIR); } };
template <typename T, int DIR> struct Dft<T, 4, DIR> { static HD void run(cx<T>* v) { dft4(v, DIR); } };
template <typename T, int DIR> struct Dft<T, 5, DIR> { static HD void run(cx<T>* v) { dft5(v, DIR); } };
template <typename T, int DIR> struct Dft<T, 7, DIR> { static HD void run(cx<T>* v) { dft7(v, DIR); } };
template <typename T, int DIR> struct Dft<T, 8, DIR> { static HD void run(cx<T>* v) { dft8(v, DIR); } };
template <typename T, int DIR> struct Dft<T, 6, DIR> { static HD void run(cx<T>* v) { dft_ab<T, 3, 2, DIR>(v); } };
template <typename T, int DIR> struct Dft<T, 9, DIR> { static HD void run(cx<T>* v) { dft_ab<T, 3, 3, DIR>(v); } };
template <typename T, int DIR> struct Dft<T, 10, DIR> { static HD void run(cx<T>* v) { dft_ab<T, 5, 2, DIR>(v); } };
template <typename T, int DIR> struct Dft<T, 12, DIR> { static HD void run(cx<T>* v) { dft_ab<T, 4, 3, DIR>(v); } };
template <typename T, int DIR> struct Dft<T, 14, DIR> { static HD void run(cx<T>* v) { dft_ab<T, 7, 2, DIR>(v); } };
template <typename T, int DIR> struct Dft<T, 15, DIR> { static HD void run(cx<T>* v) { dft_ab<T, 5, 3, DIR>(v); } };
template <typename T, int DIR> struct Dft<T, 16, DIR> { static HD void run(cx<T>* v) { dft_ab<T, 4, 4, DIR>(v); } };

// R = A*B point DFT in registers (natural order in and out): with
// j = B*j1 + j2 and k = k1 + A*k2,
//   X[k1 + A k2] = sum_j2 W_B^{j2 k2} W_R^{j2 k1} sum_j1 W_A^{j1 k1} x[B j1 + j2],
// W_M = exp(DIR * 2 pi i / M).  The loops over j2 and k1 are template
// recursions, so every index and twiddle angle is a compile-time constant and
// the arrays stay in registers.
template <typename T, int A, int B, int DIR, int J2, int K1>
struct DftAbTwiddle {  // y[k1*B + J2] = W_R^{J2 k1} u[k1] for k1 = K1 .. A-1
  static HD void run(const cx<T>* u, cx<T>* y) {
    if constexpr (K1 < A) {
      y[K1 * B + J2] = twiddle_const<T, A * B, J2 * K1, DIR>(u[K1]);
      DftAbTwiddle<T, A, B, DIR, J2, K1 + 1>::run(u, y);
    }
  }
};
template <typename T, int A, int B, int DIR, int J2>
struct DftAbFirst {  // A-point DFTs over j1 for j2 = J2 .. B-1, with twiddles
  static HD void run(const cx<T>* v, cx<T>* y) {
    if constexpr (J2 < B) {
      cx<T> u[A];
#pragma unroll
      for (int j1 = 0; j1 < A; ++j1) u[j1] = v[B * j1 + J2];
      Dft<T, A, DIR>::run(u);
      DftAbTwiddle<T, A, B, DIR, J2, 0>::run(u, y);
      DftAbFirst<T, A, B, DIR, J2 + 1>::run(v, y);
    }
  }
};

template <typename T, int A, int B, int DIR>
HD void dft_ab(cx<T>* v) {
  cx<T> y[A * B];
  DftAbFirst<T, A, B, DIR, 0>::run(v, y);
#pragma unroll
  for (int k1 = 0; k1 < A; ++k1) {
    cx<T> u[B];
#pragma unroll
    for (int j2 = 0; j2 < B; ++j2) u[j2] = y[k1 * B + j2];
    Dft<T, B, DIR>::run(u);
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = u[k2];
  }
}

// One Stockham stage of radix R over nb transforms: src -> dst.  Element i of
// transform b is at [b + i*si] (si >= nb); mnb = magic32(nb).
template <typename T, int R, int DIR>
HD void fft_stage_r(const cx<T>* __restrict__ src, cx<T>* __restrict__ dst, int nb, unsigned mnb, int si, int n,
                    int Ns, unsigned magic, const cx<T>* __restrict__ tw, int tid, int nthr) {
  const int nbf = n / R;  // butterflies per transform
  const int total = nbf * nb;
  for (int w = tid; w < total; w += nthr) {
    const int j = magic_div32(w, mnb);
    const int b = w - j * nb;
    const int jq = magic_div(j, magic);
    const int kmod = j - jq * Ns;
    cx<T> v[R];
    const cx<T>* s = src + b;
#pragma unroll
    for (int m = 0; m < R; ++m) v[m] = s[(j + m * nbf) * si];
    if (Ns > 1) {
      const cx<T>* t = tw + kmod * (R - 1);
#pragma unroll
      for (int m = 1; m < R; ++m) {
        cx<T> f = t[m - 1];
        if (DIR > 0) f.y = -f.y;
        v[m] = cmul(v[m], f);
      }
    }
    Dft<T, R, DIR>::run(v);
    cx<T>* d = dst + b;
    const int base = jq * Ns * R + kmod;
#pragma unroll
    for (int m = 0; m < R; ++m) d[(base + m * Ns) * si] = v[m];
  }
}

template <typename T, int DIR>
HD void fft_stage(const cx<T>* src, cx<T>* dst, int nb, unsigned mnb, int si, int n, int R, int Ns, unsigned magic,
                  const cx<T>* tw, int tid, int nthr) {
  constexpr int RM = FftMaxRadix<T>::value;
#define OFDFT_STAGE_CASE(r)                                                                 \
  case r:                                                                                   \
    if constexpr (r <= RM) fft_stage_r<T, r, DIR>(src, dst, nb, mnb, si, n, Ns, magic, tw, tid, nthr); \
    break;
  switch (R) {
    OFDFT_STAGE_CASE(2)
    OFDFT_STAGE_CASE(3)
    OFDFT_STAGE_CASE(4)
    OFDFT_STAGE_CASE(5)
    OFDFT_STAGE_CASE(6)
    OFDFT_STAGE_CASE(7)
    OFDFT_STAGE_CASE(8)
    OFDFT_STAGE_CASE(9)
    OFDFT_STAGE_CASE(10)
    OFDFT_STAGE_CASE(12)
    OFDFT_STAGE_CASE(14)
    OFDFT_STAGE_CASE(15)
    OFDFT_STAGE_CASE(16)
    default: break;
  }
#undef OFDFT_STAGE_CASE
}

// Full transform of nb sequences held in buf (tmp is scratch of the same
// layout), element i of sequence b at [b + i*si].  DIR = -1 forward, +1
// inverse.  Returns the buffer (buf or tmp) holding the result.  Must be
// called by every thread of the block.
template <typename T, int DIR>
HD cx<T>* fft_batch(cx<T>* buf, cx<T>* tmp, int nb, int si, const FftPlan& p, const cx<T>* twtab, int tid,
                    int nthr) {
  cx<T>* a = buf;
  cx<T>* b = tmp;
  const unsigned mnb = magic32(nb);
  const int nst = p.nst, n = p.n;
  for (int s = 0; s < nst; ++s) {
    fft_stage<T, DIR>(a, b, nb, mnb, si, n, p.R[s], p.Ns[s], p.ns_magic[s], twtab + p.tw_base + p.tw[s], tid, nthr);
    BLOCK_SYNC();
    cx<T>* t = a;
    a = b;
    b = t;
  }
  return a;
}

// Runtime direction: dir = -1 forward, +1 inverse.
template <typename T>
HD cx<T>* fft_batch(cx<T>* buf, cx<T>* tmp, int nb, int si, const FftPlan& p, const cx<T>* twtab, int dir,
                    int tid, int nthr) {
  return dir < 0 ? fft_batch<T, -1>(buf, tmp, nb, si, p, twtab, tid, nthr)
                 : fft_batch<T, 1>(buf, tmp, nb, si, p, twtab, tid, nthr);
}

// ------------------------------------------------------------ transforms between accessors
// Element i of column b of a batch held in shared memory at p[b + i*si].
template <typename T>
struct SmemIO {
  cx<T>* p;
  int si;
  HD cx<T> ld(int i, int b) const { return p[b + i * si]; }
  HD void st(int i, int b, cx<T> v) const { p[b + i * si] = v; }
};

// One Stockham stage of radix R whose inputs come from src.ld(i, b) and whose
// outputs go to dst.st(i, b, v) (same work split as fft_stage_r).
template <typename T, int R, int DIR, class Src, class Dst>
HD void fft_stage_io(const Src& src, const Dst& dst, int nb, unsigned mnb, int n, int Ns, unsigned magic,
                     const cx<T>* __restrict__ tw, int tid, int nthr) {
  const int nbf = n / R;
  const int total = nbf * nb;
  for (int w = tid; w < total; w += nthr) {
    const int j = magic_div32(w, mnb);
    const int b = w - j * nb;
    const int jq = magic_div(j, magic);
    const int kmod = j - jq * Ns;
    cx<T> v[R];
#pragma unroll
    for (int m = 0; m < R; ++m) v[m] = src.ld(j + m * nbf, b);
    if (Ns > 1) {
      const cx<T>* t = tw + kmod * (R - 1);
#pragma unroll
      for (int m = 1; m < R; ++m) {
        cx<T> f = t[m - 1];
        if (DIR > 0) f.y = -f.y;
        v[m] = cmul(v[m], f);
      }
    }
    Dft<T, R, DIR>::run(v);
    const int base = jq * Ns * R + kmod;
#pragma unroll
    for (int m = 0; m < R; ++m) dst.st(base + m * Ns, b, v[m]);
  }
}

template <typename T, int DIR, class Src, class Dst>
HD void fft_stage_io_any(const Src& src, const Dst& dst, int nb, unsigned mnb, int n, int R, int Ns, unsigned magic,
                         const cx<T>* tw, int tid, int nthr) {
  constexpr int RM = FftMaxRadix<T>::value;
#define OFDFT_IO_CASE(r)                                                                           \
  case r:                                                                                          \
    if constexpr (r <= RM) fft_stage_io<T, r, DIR>(src, dst, nb, mnb, n, Ns, magic, tw, tid, nthr); \
    break;
  switch (R) {
    OFDFT_IO_CASE(2)
    OFDFT_IO_CASE(3)
    OFDFT_IO_CASE(4)
    OFDFT_IO_CASE(5)
    OFDFT_IO_CASE(6)
    OFDFT_IO_CASE(7)
    OFDFT_IO_CASE(8)
    OFDFT_IO_CASE(9)
    OFDFT_IO_CASE(10)
    OFDFT_IO_CASE(12)
    OFDFT_IO_CASE(14)
    OFDFT_IO_CASE(15)
    OFDFT_IO_CASE(16)
    default: break;
  }
#undef OFDFT_IO_CASE
}

// Full transform of nb columns: stage 0 reads src, stage s (0 <= s < nst-1)
// writes buffer A (s even) or B (s odd), the last stage writes dst.  src may
// be A's or B's storage only if it is not the buffer stage 0 writes (A).
// When dst is shared memory it must be fft_out_buffer(nst, A, B), the buffer
// the last stage does not read.  No barrier after the last stage.
template <typename T, int DIR, class Src, class Dst>
HD void fft_run(const Src& src, const Dst& dst, cx<T>* A, cx<T>* B, int nb, const FftPlan& p, const cx<T>* twtab,
                int tid, int nthr) {
  const unsigned mnb = magic32(nb);
  const int nst = p.nst, n = p.n;
  const cx<T>* tw0 = twtab + p.tw_base;
  if (nst == 1) {
    fft_stage_io_any<T, DIR>(src, dst, nb, mnb, n, p.R[0], p.Ns[0], p.ns_magic[0], tw0 + p.tw[0], tid, nthr);
    return;
  }
  const SmemIO<T> a{A, nb}, b{B, nb};
  fft_stage_io_any<T, DIR>(src, a, nb, mnb, n, p.R[0], p.Ns[0], p.ns_magic[0], tw0 + p.tw[0], tid, nthr);
  BLOCK_SYNC();
  for (int s = 1; s < nst - 1; ++s) {
    if (s & 1) fft_stage_io_any<T, DIR>(a, b, nb, mnb, n, p.R[s], p.Ns[s], p.ns_magic[s], tw0 + p.tw[s], tid, nthr);
    else fft_stage_io_any<T, DIR>(b, a, nb, mnb, n, p.R[s], p.Ns[s], p.ns_magic[s], tw0 + p.tw[s], tid, nthr);
    BLOCK_SYNC();
  }
  const int sl = nst - 1;
  if (sl & 1) fft_stage_io_any<T, DIR>(a, dst, nb, mnb, n, p.R[sl], p.Ns[sl], p.ns_magic[sl], tw0 + p.tw[sl], tid, nthr);
  else fft_stage_io_any<T, DIR>(b, dst, nb, mnb, n, p.R[sl], p.Ns[sl], p.ns_magic[sl], tw0 + p.tw[sl], tid, nthr);
}

// The buffer of fft_run that the last stage does not read (A or B).
template <typename T>
HD cx<T>* fft_out_buffer(int nst, cx<T>* A, cx<T>* B) { return ((nst - 1) & 1) ? B : A; }

// ------------------------------------------------------------ two-step register FFT
// A transform of length n = R1 * R2 (both compile-time) over NC columns, with
// one shared-memory exchange: with j = t + R2*j1 and k = k1 + R1*k2,
//   X[k1 + R1 k2] = sum_t W_R2^{t k2} W_n^{t k1} sum_j1 W_R1^{j1 k1} x[t + R2 j1],
// W_m = exp(DIR * 2 pi i / m).  Step 1 (one work item per column and t)
// loads its R1 inputs from src.ld(i, c) straight into registers, does the
// R1-point DFT and the twiddles W_n^{t k1} = roots[t*k1] (t*k1 < n), and
// writes the exchange buffer X (NC * n values); step 2 (one work item per
// column and k1) does the R2-point DFT and writes the outputs with
// dst.st(k, c, v).  Consecutive threads take consecutive columns.  src may be
// the same memory as dst: every input is read before the barrier between the
// steps and every output is written after it.
template <typename T, int R1, int R2, int DIR, class Src, class Dst>
HD void fft2_tile(const Src& src, const Dst& dst, cx<T>* __restrict__ X, int NC, const cx<T>* __restrict__ roots,
                  int tid, int nthr) {
  const unsigned mnc = magic32(NC);
  for (int w = tid; w < NC * R2; w += nthr) {
    const int t = magic_div32(w, mnc), c = w - t * NC;
    cx<T> v[R1], f[R1];
#pragma unroll
    for (int j1 = 0; j1 < R1; ++j1) v[j1] = src.ld(t + R2 * j1, c);
    // the twiddles are loaded while the data loads are in flight
#pragma unroll
    for (int k1 = 1; k1 < R1; ++k1) f[k1] = roots[t * k1];
    Dft<T, R1, DIR>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < R1; ++k1) {
      if (DIR > 0) f[k1].y = -f[k1].y;
      v[k1] = cmul(v[k1], f[k1]);
    }
    cx<T>* x = X + c + NC * t;
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) x[NC * R2 * k1] = v[k1];
  }
  BLOCK_SYNC();
  for (int w = tid; w < NC * R1; w += nthr) {
    const int k1 = magic_div32(w, mnc), c = w - k1 * NC;
    cx<T> v[R2];
    const cx<T>* x = X + c + NC * R2 * k1;
#pragma unroll
    for (int t = 0; t < R2; ++t) v[t] = x[NC * t];
    Dft<T, R2, DIR>::run(v);
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) dst.st(k1 + R1 * k2, c, v[k2]);
  }
}

// Largest step-2 radix of the two-step transforms per precision (R2 complex
// values stay in registers).
template <typename T> struct Fft2MaxRadix { static constexpr int value = 16; };
template <> struct Fft2MaxRadix<double> { static constexpr int value = 12; };

// The lengths with a two-step transform and their factors (R1 <= R2).
#define OFDFT_FFT2_SIZES(X) \
  X(32, 4, 8)               \
  X(48, 6, 8)               \
  X(64, 8, 8)               \
  X(72, 8, 9)               \
  X(80, 8, 10)              \
  X(96, 8, 12)              \
  X(120, 10, 12)            \
  X(128, 8, 16)             \
  X(144, 12, 12)            \
  X(160, 10, 16)            \
  X(192, 12, 16)            \
  X(240, 15, 16)            \
  X(256, 16, 16)

// Second-step radix R2 of the two-step transform of length n (0: none).
HD int fft2_r2(int n) {
  switch (n) {
#define OFDFT_FFT2_R2(N, A, B) \
  case N:                      \
    return B;
    OFDFT_FFT2_SIZES(OFDFT_FFT2_R2)
#undef OFDFT_FFT2_R2
    default:
      return 0;
  }
}

// Whether length n has a two-step transform in precision T.
template <typename T>
HD bool fft2_supported(const FftPlan& p) {
  if (p.root < 0) return false;
  switch (p.n) {
#define OFDFT_FFT2_CASE(N, A, B) \
  case N:                        \
    return B <= Fft2MaxRadix<T>::value;
    OFDFT_FFT2_SIZES(OFDFT_FFT2_CASE)
#undef OFDFT_FFT2_CASE
    default:
      return false;
  }
}

// Two-step transform of length p.n (fft2_supported must hold).
template <typename T, int DIR, class Src, class Dst>
HD void fft2_run(const Src& src, const Dst& dst, cx<T>* X, int NC, const FftPlan& p, const cx<T>* twtab, int tid,
                 int nthr) {
  const cx<T>* roots = twtab + p.root;
  switch (p.n) {
#define OFDFT_FFT2_CASE(N, A, B)                                                       \
  case N:                                                                              \
    if constexpr (B <= Fft2MaxRadix<T>::value)                                         \
      fft2_tile<T, A, B, DIR>(src, dst, X, NC, roots, tid, nthr);                      \
    break;
    OFDFT_FFT2_SIZES(OFDFT_FFT2_CASE)
#undef OFDFT_FFT2_CASE
    default:
      break;
  }
}

}  // namespace ofdft
