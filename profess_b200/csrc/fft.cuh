// Batched in-place mixed-radix FFT over shared memory.
//
// A transform of length n = R_0 * R_1 * ... * R_{S-1} runs as one stage per
// radix, in place: the forward transform is a decimation in frequency
// (natural order in, digit-reversed order out), the inverse a decimation in
// time (digit-reversed order in, natural order out), so a forward transform,
// a pointwise operator in k-space and the inverse need neither a second
// buffer nor a reordering pass.  Stage s works on blocks of length
// L_s = n / (R_0 ... R_{s-1}) with stride m_s = L_s / R_s: the butterfly
// (block b, offset j0 < m_s) reads the R_s points b L_s + j0 + m_s j1, does
// the R_s-point DFT in registers and, going forward, multiplies output r by
// W_{L_s}^{j0 r} (W_M = exp(-2 pi i / M)) and stores it at b L_s + j0 + m_s r;
// the inverse stage undoes that with the conjugate twiddles first and the
// inverse DFT second, stages in reverse order.  After the forward transform,
// position q holds frequency perm[q], with perm built by
// perm(q) = r + R_0 perm'(q - r m_0), r = q / m_0, over the remaining
// radices; iperm is its inverse.
//
// The radices are 2, 3, 4, 5, 7, 8 and the compound 6, 9, 10, 12, 14, 15, 16,
// whose DFTs run in registers as an A x B Cooley-Tukey split with
// compile-time twiddles.  Many columns of the same length are transformed
// together: element i of column c lives at buf[c*cs + i*es]; work items
// (column, butterfly) are spread over the block's threads with the column
// fastest, so consecutive threads touch consecutive columns (conflict-free
// shared-memory access when cs = 1, or when cs is odd).  The twiddles are
// the n-th roots of unity exp(-2 pi i e / n), e < n, computed on the host in
// long double; W_{L_s}^{e} is root[e n / L_s].  No scaling is applied.
#pragma once
#include "cx.cuh"

namespace ofdft {

constexpr int FFT_MAX_STAGES = 12;
constexpr int FFT_MAX_RADIX = 16;

// Largest radix of the FP32 and FP64 plans: an R-point DFT holds R complex
// values in registers, and only the radices up to the limit are compiled
// into a precision's kernels.
template <typename T> struct FftMaxRadix { static constexpr int value = 16; };
template <> struct FftMaxRadix<double> { static constexpr int value = 12; };

struct FftPlan {
  int n;
  int nst;
  int R[FFT_MAX_STAGES];
  int L[FFT_MAX_STAGES];               // block length of stage s, n / (R_0 ... R_{s-1})
  unsigned m_magic[FFT_MAX_STAGES];    // magic32(L[s] / R[s])
  int root;                            // offset of exp(-2 pi i e / n), e < n, in the twiddle table
  int perm;                            // offset of perm (position -> frequency) in the index table
  int iperm;                           // offset of iperm (frequency -> position)
};

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

// One in-place stage of radix R over ncols columns (mcols = magic32(ncols)):
// DIR = -1 forward (DFT, then twiddles), +1 inverse (conjugate twiddles,
// then inverse DFT).  tstep = n / L.
template <typename T, int R, int DIR>
HD void ip_stage_r(cx<T>* __restrict__ buf, int ncols, unsigned mcols, int cs, int es, int n, int L, unsigned mm,
                   const cx<T>* __restrict__ roots, int tid, int nthr) {
  const int m = L / R;
  const int total = (n / R) * ncols;
  const int tstep = n / L;
  const int ms = m * es;
  for (int w = tid; w < total; w += nthr) {
    const int bf = magic_div32(w, mcols), c = w - bf * ncols;
    const int blk = magic_div32(bf, mm), j0 = bf - blk * m;
    cx<T>* p = buf + c * cs + (blk * L + j0) * es;
    cx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = p[r * ms];
    const int e = j0 * tstep;
    if (DIR > 0 && m > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], conj(roots[r * e]));
    }
    Dft<T, R, DIR>::run(v);
    if (DIR < 0 && m > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], roots[r * e]);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) p[r * ms] = v[r];
  }
}

template <typename T, int DIR>
HD void ip_stage(cx<T>* buf, int ncols, unsigned mcols, int cs, int es, const FftPlan& p, int s, const cx<T>* roots,
                 int tid, int nthr) {
  constexpr int RM = FftMaxRadix<T>::value;
  const int n = p.n, L = p.L[s];
  const unsigned mm = p.m_magic[s];
#define OFDFT_IP_CASE(r)                                                                          \
  case r:                                                                                         \
    if constexpr (r <= RM) ip_stage_r<T, r, DIR>(buf, ncols, mcols, cs, es, n, L, mm, roots, tid, nthr); \
    break;
  switch (p.R[s]) {
    OFDFT_IP_CASE(2)
    OFDFT_IP_CASE(3)
    OFDFT_IP_CASE(4)
    OFDFT_IP_CASE(5)
    OFDFT_IP_CASE(6)
    OFDFT_IP_CASE(7)
    OFDFT_IP_CASE(8)
    OFDFT_IP_CASE(9)
    OFDFT_IP_CASE(10)
    OFDFT_IP_CASE(12)
    OFDFT_IP_CASE(14)
    OFDFT_IP_CASE(15)
    OFDFT_IP_CASE(16)
    default: break;
  }
#undef OFDFT_IP_CASE
}

// One stage whose inputs come from src.ld(c, i) and whose outputs go to
// dst.st(c, i, v) (column c, position i), with the butterfly work split of
// ip_stage_r: a first forward stage can load straight from global memory, a
// last inverse stage store straight to it.
template <typename T, int R, int DIR, class Src, class Dst>
HD void ip_stage_io(const Src& src, const Dst& dst, int ncols, unsigned mcols, int n, int L, unsigned mm,
                    const cx<T>* __restrict__ roots, int tid, int nthr) {
  const int m = L / R;
  const int total = (n / R) * ncols;
  const int tstep = n / L;
  for (int w = tid; w < total; w += nthr) {
    const int bf = magic_div32(w, mcols), c = w - bf * ncols;
    const int blk = magic_div32(bf, mm), j0 = bf - blk * m;
    const int base = blk * L + j0;
    cx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src.ld(c, base + r * m);
    const int e = j0 * tstep;
    if (DIR > 0 && m > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], conj(roots[r * e]));
    }
    Dft<T, R, DIR>::run(v);
    if (DIR < 0 && m > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], roots[r * e]);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) dst.st(c, base + r * m, v[r]);
  }
}

// Stage s of plan p through accessors (a switch over the radix).
template <typename T, int DIR, class Src, class Dst>
HD void ip_stage_acc(const Src& src, const Dst& dst, int ncols, unsigned mcols, const FftPlan& p, int s,
                     const cx<T>* roots, int tid, int nthr) {
  constexpr int RM = FftMaxRadix<T>::value;
  const int n = p.n, L = p.L[s];
  const unsigned mm = p.m_magic[s];
#define OFDFT_IO_CASE(r)                                                                              \
  case r:                                                                                             \
    if constexpr (r <= RM) ip_stage_io<T, r, DIR>(src, dst, ncols, mcols, n, L, mm, roots, tid, nthr); \
    break;
  switch (p.R[s]) {
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

// The last forward stage (block length R, stride 1: no twiddles), a real
// pointwise factor op(c, q) at every position q, and the first inverse stage
// (the same butterflies) in registers, in place: one shared-memory round trip
// for a forward transform's end, a k-space operator and an inverse
// transform's start.
template <typename T, int R, class Op>
HD void ip_stage_op_r(cx<T>* __restrict__ buf, int ncols, unsigned mcols, int cs, int es, int n, const Op& op,
                      int tid, int nthr) {
  const int total = (n / R) * ncols;
  for (int w = tid; w < total; w += nthr) {
    const int blk = magic_div32(w, mcols), c = w - blk * ncols;
    cx<T>* p = buf + c * cs + blk * R * es;
    cx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = p[r * es];
    Dft<T, R, -1>::run(v);
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = v[r] * op(c, blk * R + r);
    Dft<T, R, 1>::run(v);
#pragma unroll
    for (int r = 0; r < R; ++r) p[r * es] = v[r];
  }
}

template <typename T, class Op>
HD void ip_stage_op(cx<T>* buf, int ncols, unsigned mcols, int cs, int es, const FftPlan& p, const Op& op, int tid,
                    int nthr) {
  constexpr int RM = FftMaxRadix<T>::value;
  const int n = p.n;
#define OFDFT_OP_CASE(r)                                                                  \
  case r:                                                                                 \
    if constexpr (r <= RM) ip_stage_op_r<T, r>(buf, ncols, mcols, cs, es, n, op, tid, nthr); \
    break;
  switch (p.R[p.nst - 1]) {
    OFDFT_OP_CASE(2)
    OFDFT_OP_CASE(3)
    OFDFT_OP_CASE(4)
    OFDFT_OP_CASE(5)
    OFDFT_OP_CASE(6)
    OFDFT_OP_CASE(7)
    OFDFT_OP_CASE(8)
    OFDFT_OP_CASE(9)
    OFDFT_OP_CASE(10)
    OFDFT_OP_CASE(12)
    OFDFT_OP_CASE(14)
    OFDFT_OP_CASE(15)
    OFDFT_OP_CASE(16)
    default: break;
  }
#undef OFDFT_OP_CASE
}

// Full in-place transform of ncols columns (element i of column c at
// buf[c*cs + i*es]).  DIR = -1: forward, natural -> digit-reversed; DIR = +1:
// inverse, digit-reversed -> natural.  Every thread of the block must call
// it; the data must be complete in shared memory on entry (the caller's
// barrier), and the block synchronises after every stage, so the result is
// complete on return.
template <typename T, int DIR>
HD void fft_inplace(cx<T>* buf, int ncols, int cs, int es, const FftPlan& p, const cx<T>* twtab, int tid, int nthr) {
  const unsigned mcols = magic32(ncols);
  const cx<T>* roots = twtab + p.root;
  if (DIR < 0) {
    for (int s = 0; s < p.nst; ++s) {
      ip_stage<T, -1>(buf, ncols, mcols, cs, es, p, s, roots, tid, nthr);
      BLOCK_SYNC();
    }
  } else {
    for (int s = p.nst - 1; s >= 0; --s) {
      ip_stage<T, 1>(buf, ncols, mcols, cs, es, p, s, roots, tid, nthr);
      BLOCK_SYNC();
    }
  }
}

// ------------------------------------------------------------ host planning
// Radix sequence of n (7-smooth, n <= 512): the fewest stages with radices
// up to rmax, then the smallest largest radix; largest radix first.  No heap
// use (the allocation-free entry point plans with it too).  Returns the
// number of stages, 0 if n has no such factorisation.
inline int fft_radices(int n, int rmax, int* out) {
  static const int kR[] = {16, 15, 14, 12, 10, 9, 8, 7, 6, 5, 4, 3, 2};
  int st[513], big[513], first[513];
  for (int m = 0; m <= n; ++m) { st[m] = 1 << 20; big[m] = 1 << 20; first[m] = 0; }
  st[1] = 0;
  big[1] = 0;
  for (int m = 2; m <= n; ++m) {
    if (n % m) continue;
    for (int R : kR) {
      if (R > rmax || m % R || st[m / R] >= (1 << 20)) continue;
      const int cs = st[m / R] + 1, cb = R > big[m / R] ? R : big[m / R];
      if (cs < st[m] || (cs == st[m] && cb < big[m])) { st[m] = cs; big[m] = cb; first[m] = R; }
    }
  }
  if (st[n] >= (1 << 20)) return 0;
  int k = 0;
  for (int m = n; m > 1; m /= first[m]) out[k++] = first[m];
  for (int a = 0; a < k; ++a)  // largest first
    for (int b = a + 1; b < k; ++b)
      if (out[b] > out[a]) { const int t = out[a]; out[a] = out[b]; out[b] = t; }
  return k;
}

// Fill plan p of length n from its radix sequence (stage block lengths and
// magic numbers; the table offsets are the caller's), and the digit-reversal
// tables: perm[q] = frequency at position q after the forward transform,
// iperm[k] = position of frequency k.  No heap use.
inline void fft_plan_fill(FftPlan& p, int n, const int* radix, int nst, int* perm, int* iperm) {
  p.n = n;
  p.nst = nst;
  int L = n;
  for (int s = 0; s < nst; ++s) {
    p.R[s] = radix[s];
    p.L[s] = L;
    p.m_magic[s] = magic32(L / radix[s]);
    L /= radix[s];
  }
  for (int q = 0; q < n; ++q) {
    int k = 0, mult = 1, rem = q, len = n;
    for (int s = 0; s < nst; ++s) {
      const int m = len / radix[s];
      const int r = rem / m;
      k += mult * r;
      mult *= radix[s];
      rem -= r * m;
      len = m;
    }
    perm[q] = k;
    iperm[k] = q;
  }
}

}  // namespace ofdft
