// Batched mixed-radix Stockham FFT over shared memory.
//
// A transform of length n = R_0 * R_1 * ... (radices 2, 3, 4, 5, 7, 8) runs as
// one Stockham stage per radix.  Each stage reads R points at stride n/R,
// multiplies by the stage twiddles, does a radix-R butterfly in registers and
// writes the R outputs in self-sorting order, ping-ponging between two shared
// buffers; the caller reads the result from whichever buffer fft_batch
// returns.  Many independent transforms of the same length are done together:
// element i of transform b lives at buf[b + i*si].  Work items (b, butterfly)
// are spread over the block's threads with b fastest, so consecutive threads
// touch consecutive shared-memory words; the index arithmetic uses
// multiply-high divisions by constants prepared on the host.
//
// Twiddles are precomputed on the host in long double and stored per plan:
// stage s with span Ns (product of the earlier radices) and radix R uses
// tw[off_s + k*(R-1) + (m-1)] = exp(-2*pi*i*m*k/(Ns*R)), k = 0..Ns-1.
// The inverse transform uses the conjugates.  No scaling is applied here.
#pragma once
#include "cx.cuh"

namespace ofdft {

constexpr int FFT_MAX_STAGES = 12;
constexpr int FFT_MAX_RADIX = 8;

struct FftPlan {
  int n;
  int nst;
  int R[FFT_MAX_STAGES];
  int Ns[FFT_MAX_STAGES];
  int tw[FFT_MAX_STAGES];  // offset of the stage's twiddles in the plan table
  unsigned ns_magic[FFT_MAX_STAGES];  // ceil(2^20 / Ns): j / Ns == (j * magic) >> 20 for j < 2048
  int tw_base;             // offset of this plan in the global twiddle table
};

// Exact quotient j / d for 0 <= j < 2048 and 1 <= d <= 512 from magic = ceil(2^20 / d).
HD int magic_div(int j, unsigned magic) { return (int)(((unsigned)j * magic) >> 20); }

// Exact quotient w / d for 0 <= w < 2^24 and 1 <= d <= 4096 from m32 = ceil(2^32 / d)
// (d = 1 is encoded as m32 = 0).
HD int magic_div32(int w, unsigned m32) {
  if (m32 == 0u) return w;
#if defined(__CUDA_ARCH__)
  return (int)__umulhi((unsigned)w, m32);
#else
  return (int)(((unsigned long long)(unsigned)w * m32) >> 32);
#endif
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
  for (int k = 1; k <= 3; ++k) {
    tp[k] = v[k] + v[7 - k];
    tm[k] = v[k] - v[7 - k];
  }
  cx<T> y[7];
  y[0] = v[0] + tp[1] + tp[2] + tp[3];
  for (int j = 1; j <= 3; ++j) {
    cx<T> a = v[0], b = mk<T>(T(0), T(0));
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

template <typename T, int R> struct Dft;
template <typename T> struct Dft<T, 2> { static HD void run(cx<T>* v, int) { dft2(v); } };
template <typename T> struct Dft<T, 3> { static HD void run(cx<T>* v, int d) { dft3(v, d); } };
template <typename T> struct Dft<T, 4> { static HD void run(cx<T>* v, int d) { dft4(v, d); } };
template <typename T> struct Dft<T, 5> { static HD void run(cx<T>* v, int d) { dft5(v, d); } };
template <typename T> struct Dft<T, 7> { static HD void run(cx<T>* v, int d) { dft7(v, d); } };
template <typename T> struct Dft<T, 8> { static HD void run(cx<T>* v, int d) { dft8(v, d); } };

// One Stockham stage of radix R over nb transforms: src -> dst.  Element i of
// transform b is at [b + i*si] (si >= nb); mnb = magic32(nb).
template <typename T, int R>
HD void fft_stage_r(const cx<T>* __restrict__ src, cx<T>* __restrict__ dst, int nb, unsigned mnb, int si, int n,
                    int Ns, unsigned magic, const cx<T>* __restrict__ tw, int dir, int tid, int nthr) {
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
        if (dir > 0) f.y = -f.y;
        v[m] = cmul(v[m], f);
      }
    }
    Dft<T, R>::run(v, dir);
    cx<T>* d = dst + b;
    const int base = jq * Ns * R + kmod;
#pragma unroll
    for (int m = 0; m < R; ++m) d[(base + m * Ns) * si] = v[m];
  }
}

template <typename T>
HD void fft_stage(const cx<T>* src, cx<T>* dst, int nb, unsigned mnb, int si, int n, int R, int Ns, unsigned magic,
                  const cx<T>* tw, int dir, int tid, int nthr) {
  switch (R) {
    case 2: fft_stage_r<T, 2>(src, dst, nb, mnb, si, n, Ns, magic, tw, dir, tid, nthr); break;
    case 3: fft_stage_r<T, 3>(src, dst, nb, mnb, si, n, Ns, magic, tw, dir, tid, nthr); break;
    case 4: fft_stage_r<T, 4>(src, dst, nb, mnb, si, n, Ns, magic, tw, dir, tid, nthr); break;
    case 5: fft_stage_r<T, 5>(src, dst, nb, mnb, si, n, Ns, magic, tw, dir, tid, nthr); break;
    case 7: fft_stage_r<T, 7>(src, dst, nb, mnb, si, n, Ns, magic, tw, dir, tid, nthr); break;
    case 8: fft_stage_r<T, 8>(src, dst, nb, mnb, si, n, Ns, magic, tw, dir, tid, nthr); break;
    default: break;
  }
}

// Full transform of nb sequences held in buf (tmp is scratch of the same
// layout), element i of sequence b at [b + i*si].  dir = -1 forward, +1
// inverse.  Returns the buffer (buf or tmp) holding the result.  Must be
// called by every thread of the block.
template <typename T>
HD cx<T>* fft_batch(cx<T>* buf, cx<T>* tmp, int nb, int si, const FftPlan& p,
                    const cx<T>* twtab, int dir, int tid, int nthr) {
  cx<T>* a = buf;
  cx<T>* b = tmp;
  const unsigned mnb = magic32(nb);
  for (int s = 0; s < p.nst; ++s) {
    fft_stage(a, b, nb, mnb, si, p.n, p.R[s], p.Ns[s], p.ns_magic[s], twtab + p.tw_base + p.tw[s], dir, tid,
              nthr);
    BLOCK_SYNC();
    cx<T>* t = a;
    a = b;
    b = t;
  }
  return a;
}

}  // namespace ofdft
