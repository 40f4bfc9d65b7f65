// Stress tensor of a density on the device (CalculateStress,
// Source/CalStress.f90:44-253) for the WT and second-order WGC functionals
// with LDA exchange-correlation, the B-spline ion-electron term and the
// Ewald sum.
//
// The density's forward spectra (rho, rho^beta, sqrt(rho), rho^alpha) come
// from the engine's own transforms (EV_STRESS passes: x, y and z forward, in
// the kx-major, digit-reversed layout of the slot's spectra).  One reduction
// kernel then visits every stored frequency once and adds, in FP64,
//   vW        <d_a sqrt(rho) d_b sqrt(rho)> by Parseval over the full
//             spectrum (weight 2 off the kx = 0 and x-Nyquist planes; on
//             those planes, whose imaginary parts the c2r transform drops,
//             the derivative of a Nyquist index is that of index 0)
//                                                  (VWStress, KEDF_VW.f90:365-449)
//   WT        -eta G'(eta) Re(F[rho^a] F[rho^b]*) (q_a q_b / q^2, and its trace)
//                                                  (WTStress, KEDF_WT.f90:263-394)
//   WGC       the kernel-derivative sums of F[rho^x], x = a, b, a+1, b+1, a+2,
//             b+2 (stress_wgc_point)               (WGCStress, KEDF_WGC.f90:519-745)
//   Hartree   |rho(q)|^2 q_a q_b / q^4                (JStress, Hartree.f90:173-247)
//   ion-elec. Re(rho(q) S_s(q)) V_s'(q) q_a q_b / q, S_s the B-spline
//             structure factor of species s       (IonElectronStressSpline,
//                                                   IonElectronSpline.f90:359-534)
// over the half spectrum of qMask (PlaneWave.f90:255-296) for all but vW.
// The structure factor is the DFT of FillQIonTable's spread charges, taken
// ion by ion as a product of three 1D sums of the stencil weights
// (A_d(ion, k) = sum_i M_d[i] exp(-2 pi i k (i - floor_d) / n_d)), so no
// charge grid is built.  The Ewald stress adds the strain derivatives of the
// real- and reciprocal-space sums of ewald.cuh (EwaldStress,
// Ewald.f90:1857-2535) with the same splitting.  Sums run in a fixed order
// (per-thread, a fixed tree per block, blocks in index order on the host), so
// results do not depend on scheduling.
#pragma once

#include "cx.cuh"
#include "ewald.cuh"
#include "setup.cuh"

namespace ofdft {

// Accumulator channels of the spectral reduction: six upper-triangle
// components (xx, xy, xz, yy, yz, zz) per tensor term.
enum StressChannel : int { SC_VW = 0, SC_WT = 6, SC_WTTR = 12, SC_H = 13, SC_IE = 19, NSC = 25 };

struct StressArgs {
  const int* permy;          // digit-reversed position -> natural ky
  const int* permz;          // -> natural kz
  const cx<double>* sf;      // A_d(ion, k): per ion k1 + n2 + n3 entries (x, then y, then z)
  const int* species;        // species of each ion
  int nion;
  double kf;                 // (3 pi^2 rho0)^(1/3) (WT), (3 pi^2 rho*)^(1/3) (WGC)
  double ki, gamma;          // WGC: 20 rho0^(5/3 - alpha - beta), the kernel's gamma
};

// qMask (PlaneWave.f90:255-296) at natural indices (kx < k1, ky, kz): the
// half of the r2c spectrum without the conjugate partners on the kx = 0 and
// x-Nyquist planes and without their self-conjugate points.
HD bool stress_mask(int kx, int ky, int kz, int n1, int n2, int n3) {
  const bool h2 = ky >= 1 && ky <= (n2 - 1) / 2;
  const bool h3 = kz >= 1 && kz <= (n3 - 1) / 2;
  const bool plane = h2 || (ky == 0 && h3) || ((n2 % 2) == 0 && ky == n2 / 2 && h3);
  if (n1 % 2 == 1) {
    if (kx >= 1) return true;
  } else if (kx >= 1 && kx < n1 / 2) {
    return true;
  }
  if (kx == 0) return plane;
  return (n1 % 2) == 0 && kx == n1 / 2 && plane;
}

// dLindG/deta (GPrime, MathFunctions.f90:531-578) with the vW coefficient mu.
HD double wt_g_prime(double e, double mu) {
  if (e < 0.0) return 0.0;
  if (e < 1e-10) return 2.0 * e * (1.0 / 3.0 - 3.0 * mu);
  if (dabs(e - 1.0) < 1e-10) return 40.0;
  const double l1 = log(dabs((1.0 + e) / (1.0 - e)));
  const double l2 = log((1.0 + e) / dabs(1.0 - e));
  const double den = 0.5 + 0.25 * (1.0 - e * e) * l2 / e;
  return ((e * e + 1.0) * 0.25 / (e * e) * l1 - 0.5 / e) / (den * den) - 6.0 * e * mu;
}

// dV_loc/dq by the same index-knot spline as psp_value (PseudoPotDiffLookup,
// LocalPseudoPot.f90:207-276), plus the derivative of the -4 pi Z / q^2 tail.
HD double psp_diff(const IonAux& x, int sp, double q) {
  const PspDev& p = x.psp[sp];
  if (!(q > 0.0) || q > p.max_g) return 0.0;
  const double pos = q / p.dq + 1.0;
  int left = (int)floor(pos);
  if (left < 1) left = 1;
  if (left > p.npts - 1) left = p.npts - 1;
  const double dt = pos - (double)left;
  const double* vqs = x.tab + p.off;
  const double* pdd = x.tab + p.off + p.npts;
  const double yl = vqs[left - 1], yr = vqs[left];
  const double pl = pdd[left - 1], pr = pdd[left];
  const double yp = (yr - yl) - (pr / 6.0 + pl / 3.0) + dt * (pl + dt * 0.5 * (pr - pl));
  return yp / p.dq + 8.0 * PI_D * p.charge / (q * q * q);
}

// sin and cos of 2 pi t / n (0 <= t < n).
HD void sincos_turn(long long t, int n, double* sn, double* cs) {
#if defined(__CUDA_ARCH__)
  sincospi(2.0 * (double)t / (double)n, sn, cs);
#else
  const double a = 2.0 * PI_D * (double)t / (double)n;
  *sn = std::sin(a);
  *cs = std::cos(a);
#endif
}

// Entry w of ion i's table: A_d(i, k) for axis d (w < k1: x; then n2 y
// entries; then n3 z entries).  The phase k (j - floor) is reduced modulo
// n_d in integers first.
HD cx<double> stress_sf_entry(const SlotDev& s, const IonStencil& st, int w) {
  int d = 0, k = w, n = s.n1;
  if (w >= s.k1 + s.n2) {
    d = 2;
    k = w - s.k1 - s.n2;
    n = s.n3;
  } else if (w >= s.k1) {
    d = 1;
    k = w - s.k1;
    n = s.n2;
  }
  double re = 0.0, im = 0.0;
  for (int j = 0; j < SPLINE_ORDER; ++j) {
    long long t = ((long long)k * (long long)(j - st.fl[d])) % n;
    if (t < 0) t += n;
    double sn, cs;
    sincos_turn(t, n, &sn, &cs);
    re += st.M[d][j] * cs;
    im -= st.M[d][j] * sn;
  }
  return mk<double>(re, im);
}

HD void sym_add(double* a, const double* g, double w) {
  a[0] += w * g[0] * g[0];
  a[1] += w * g[0] * g[1];
  a[2] += w * g[0] * g[2];
  a[3] += w * g[1] * g[1];
  a[4] += w * g[1] * g[2];
  a[5] += w * g[2] * g[2];
}

template <typename T>
HD cx<double> spec_at(const SlotDev& s, int f, long long p) {
  const cx<T> v = ((const cx<T>*)s.spec)[(size_t)f * (size_t)s.Nc + (size_t)p];
  return mk<double>((double)v.x * s.inv_n, (double)v.y * s.inv_n);
}

// Re(conj(a) b).
HD double re_cb(cx<double> a, cx<double> b) { return a.x * b.x + a.y * b.y; }

// The WGC kinetic terms of one masked frequency (WGCStress, KEDF_WGC.f90:
// 519-745, WGCT = 2, rho0 and rho* refreshed with the cell): acc[SC_WTTR]
// gets the diagonal sum (diago + offdia diff), acc[SC_WT..] offdia q_a q_b / q^2;
// both are scaled by 2 cTF on the host.  F[rho^(x+1)] and F[rho^(x+2)] come
// from the evaluation's fields rho^x, theta rho^x, theta^2 rho^x / 2 (theta =
// rho - rho*) by linearity.
template <typename T>
HD void stress_wgc_point(const SlotDev& s, const StressArgs& sa, long long p, const double* g, double q2,
                         double eta, double* acc) {
  const double a = s.alpha, b = s.beta, rs = s.rho_s, gm = sa.gamma;
  const cx<double> A = spec_at<T>(s, 2, p), At = spec_at<T>(s, 3, p), Ah = spec_at<T>(s, 4, p);
  const cx<double> B = spec_at<T>(s, 5, p), Bt = spec_at<T>(s, 6, p), Bh = spec_at<T>(s, 7, p);
  const cx<double> A1 = mk<double>(At.x + rs * A.x, At.y + rs * A.y);
  const cx<double> B1 = mk<double>(Bt.x + rs * B.x, Bt.y + rs * B.y);
  const cx<double> A2 = mk<double>(2.0 * Ah.x + 2.0 * rs * At.x + rs * rs * A.x, 2.0 * Ah.y + 2.0 * rs * At.y + rs * rs * A.y);
  const cx<double> B2 = mk<double>(2.0 * Bh.x + 2.0 * rs * Bt.x + rs * rs * B.x, 2.0 * Bh.y + 2.0 * rs * Bt.y + rs * rs * B.y);
  const T* kern = (const T*)s.kern;
  const double K1 = (double)kern[p], K2 = (double)kern[s.Nc + p], K3 = (double)kern[2 * s.Nc + p],
               K4 = (double)kern[3 * s.Nc + p];
  // hold0 = holdS = .FALSE.
  const double c001 = -2.0 / 3.0, c002 = rs * 4.0 / 3.0, c003 = -rs * rs * 2.0 / 3.0;
  const double c011 = -5.0 / 3.0 + 1.0, c012 = rs * 5.0 / 3.0 - rs, c021 = -4.0 / 3.0 + 1.0, c111 = -8.0 / 3.0 + 2.0;
  const double diff = -1.0 / 3.0;
  const double c00 = c001 * K1 + c002 * K2 + c003 * (K3 + K4);
  const double c01 = c011 * K2 + c012 * (K3 + K4);
  const double c02 = c021 * K3;
  const double c11 = c111 * K4;
  const double p00 = re_cb(A, B), p10 = re_cb(A1, B), p01 = re_cb(A, B1), p20 = re_cb(A2, B), p02 = re_cb(A, B2),
               p11 = re_cb(A1, B1);
  const double diago = c00 * p00 + c01 * (p10 + p01) + c02 * (p20 + p02) + c11 * p11;
  const double gp = wt_g_prime(eta, s.mu);
  const double d11 = -sa.ki * eta / (36.0 * rs * rs) * gp - K4 * 6.0 * (a + b) - K2 * (gm * (a + b) + 6.0 * a * b) / rs;
  const double d02 = -sa.ki * eta / (72.0 * rs * rs) * gp - K4 * (3.0 * (a + b + 1.0) - gm) -
                     K2 * (3.0 * gm * (a + b + 1.0) - gm * gm + 18.0 * a * b) / (6.0 * rs);
  double d01 = K4 * 6.0 * rs + K2 * gm;
  const double d00 = 6.0 * rs * K2 - 2.0 * rs * d01 + rs * rs * (2.0 * d02 + d11);
  d01 = -rs * (d11 + 2.0 * d02) + d01;
  const double offdia = d00 * p00 + d01 * (p10 + p01) + d02 * (p20 + p02) + d11 * p11;
  acc[SC_WTTR] += diago + offdia * diff;
  sym_add(acc + SC_WT, g, offdia / q2);
}

// The terms of stored frequency p (kx-major position) added to acc[NSC].
template <typename T>
HD void stress_point(const SlotDev& s, const StressArgs& sa, long long p, double* acc) {
  const int n1 = s.n1, n2 = s.n2, n3 = s.n3, nrows = n2 * n3;
  const int kx = (int)(p / nrows), j = (int)(p - (long long)kx * nrows);
  const int zi = j / n2, yi = j - zi * n2;
  const int ky = sa.permy[yi], kz = sa.permz[zi];
  const int m2 = signed_freq(ky, n2), m3 = signed_freq(kz, n3);
  const double* R = s.recip;
  double g[3], ge[3];
  for (int r = 0; r < 3; ++r) g[r] = R[r] * kx + R[3 + r] * m2 + R[6 + r] * m3;
  const bool wgc = s.kinetic == KIN_WGC;  // WGC fields: rho, sqrt(rho), then the alpha and beta triples
  const cx<double> F0 = spec_at<T>(s, 0, p), Fs = spec_at<T>(s, wgc ? 1 : 2, p);
  // vW
  const bool edge = kx == 0 || ((n1 % 2) == 0 && kx == n1 / 2);
  if (edge) {
    const int e1 = 0;
    const int e2 = ((n2 % 2) == 0 && ky == n2 / 2) ? 0 : m2;
    const int e3 = ((n3 % 2) == 0 && kz == n3 / 2) ? 0 : m3;
    for (int r = 0; r < 3; ++r) ge[r] = R[r] * e1 + R[3 + r] * e2 + R[6 + r] * e3;
  } else {
    for (int r = 0; r < 3; ++r) ge[r] = g[r];
  }
  sym_add(acc + SC_VW, ge, (edge ? 1.0 : 2.0) * (Fs.x * Fs.x + Fs.y * Fs.y));
  if (!stress_mask(kx, ky, kz, n1, n2, n3)) return;
  const double q2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
  const double q = sqrt(q2);
  // Hartree
  sym_add(acc + SC_H, g, (F0.x * F0.x + F0.y * F0.y) / (q2 * q2));
  const double eta = q / (2.0 * sa.kf);
  if (wgc) {
    stress_wgc_point<T>(s, sa, p, g, q2, eta, acc);
  } else {  // WT
    const cx<double> Fb = spec_at<T>(s, 1, p);
    const cx<double> Fa = s.nf > 3 ? spec_at<T>(s, 3, p) : Fb;
    const double diff = -eta * wt_g_prime(eta, s.mu) * (Fa.x * Fb.x + Fa.y * Fb.y);
    sym_add(acc + SC_WT, g, diff / q2);
    acc[SC_WTTR] += diff;
  }
  // ion-electron
  if (sa.nion > 0) {
    double vp[MAX_SPECIES];
    for (int sp = 0; sp < s.ion.nspec; ++sp) vp[sp] = psp_diff(s.ion, sp, q) / q;
    const int L = s.k1 + n2 + n3;
    double tr = 0.0, ti = 0.0;
    for (int i = 0; i < sa.nion; ++i) {
      const cx<double>* A = sa.sf + (size_t)i * L;
      const cx<double> a = cmul(cmul(A[kx], A[s.k1 + ky]), A[s.k1 + n2 + kz]);
      const double v = vp[sa.species[i]];
      tr += a.x * v;
      ti += a.y * v;
    }
    const cx<double> bb = cmul(cmul(s.ion.b1[kx], s.ion.b2[ky]), s.ion.b3[kz]);
    const cx<double> sf = cmul(bb, mk<double>(tr * s.inv_n, ti * s.inv_n));
    sym_add(acc + SC_IE, g, F0.x * sf.x - F0.y * sf.y);
  }
}

// Fixed-order sum of K values per thread over the block; thread 0 writes
// out[0..K-1].  red holds K * nthr doubles.
template <int K>
HD void block_sum(double* red, const double* v, int tid, int nthr, double* out) {
  for (int k = 0; k < K; ++k) red[K * tid + k] = v[k];
  BLOCK_SYNC();
  for (int st = 1; st < nthr; st *= 2) {
    if ((tid % (2 * st)) == 0 && tid + st < nthr)
      for (int k = 0; k < K; ++k) red[K * tid + k] += red[K * (tid + st) + k];
    BLOCK_SYNC();
  }
  if (tid == 0)
    for (int k = 0; k < K; ++k) out[k] = red[k];
}

// Block b of nblk: frequencies p = b*nthr + tid + r*nblk*nthr.
template <typename T>
HD void stress_block(const SlotDev& s, const StressArgs& sa, int b, int nblk, int tid, int nthr, double* red,
                     double* out) {
  double acc[NSC];
  for (int k = 0; k < NSC; ++k) acc[k] = 0.0;
  const long long stride = (long long)nblk * nthr;
  for (long long p = (long long)b * nthr + tid; p < s.Nc; p += stride) stress_point<T>(s, sa, p, acc);
  block_sum<NSC>(red, acc, tid, nthr, out);
}

// Sum of rho * v_xc (Perdew-Zunger LDA, in FP64) over the points of block b
// of nblk; thread 0 writes out[0].
template <typename T>
HD void rho_vxc_block(const T* rho, long long n, int b, int nblk, int tid, int nthr, double* red, double* out) {
  double acc = 0.0;
  const long long stride = (long long)nblk * nthr;
  for (long long k = (long long)b * nthr + tid; k < n; k += stride) {
    const double r = (double)rho[k];
    const double r13 = cbrt(r);
    double vxc, exc;
    lda_point<double>(r, r13, 0.62035049089940009 / r13, vxc, exc);
    acc += r * vxc;
  }
  block_sum<1>(red, &acc, tid, nthr, out);
}

// Sum of v over block b of nblk (strided like rho_vxc_block); thread 0 writes out[0].
template <typename T>
HD void sum_block(const T* v, long long n, int b, int nblk, int tid, int nthr, double* red, double* out) {
  double acc = 0.0;
  const long long stride = (long long)nblk * nthr;
  for (long long k = (long long)b * nthr + tid; k < n; k += stride) acc += (double)v[k];
  block_sum<1>(red, &acc, tid, nthr, out);
}

// ---------------------------------------------------------------- Ewald stress
// out7 = (0, the six components of sum 0.5 z_i z_j f'(r)/r d_a d_b) over the
// images and partners of ion i, f(r) = erfc(eta r)/r.
HD void ewald_real_stress_block(const EwaldPar& p, const double* pos, const double* z, int i, int tid, int nthr,
                                double* red, double* out7) {
  const int na = 2 * p.nimg[0] + 1, nb = 2 * p.nimg[1] + 1, nc = 2 * p.nimg[2] + 1;
  const long long total = (long long)na * nb * nc * p.nion;
  const double rc2 = p.rcut * p.rcut, eta = p.eta;
  const double c2 = 2.0 * eta / sqrt(PI_D);
  const double xi = pos[3 * i], yi = pos[3 * i + 1], zi_ = pos[3 * i + 2];
  double v[7] = {0, 0, 0, 0, 0, 0, 0};
  for (long long w = tid; w < total; w += nthr) {
    const int j = (int)(w % p.nion);
    long long img = w / p.nion;
    const int c = (int)(img % nc) - p.nimg[2];
    img /= nc;
    const int b = (int)(img % nb) - p.nimg[1];
    const int a = (int)(img / nb) - p.nimg[0];
    double d[3];
    d[0] = pos[3 * j] + p.A[0][0] * a + p.A[0][1] * b + p.A[0][2] * c - xi;
    d[1] = pos[3 * j + 1] + p.A[1][0] * a + p.A[1][1] * b + p.A[1][2] * c - yi;
    d[2] = pos[3 * j + 2] + p.A[2][0] * a + p.A[2][1] * b + p.A[2][2] * c - zi_;
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    if (r2 < 1e-24 || r2 >= rc2) continue;
    const double r = sqrt(r2);
    const double ec = erfc(eta * r) / r;
    const double fp = -ec / r - c2 * exp(-eta * eta * r2) / r;
    sym_add(v + 1, d, 0.5 * z[i] * z[j] * fp / r);
  }
  block_sum<7>(red, v, tid, nthr, out7);
}

// out7 = (plane m's reciprocal energy, the six components of
// sum (2 pi / vol) exp(-G^2/4eta^2)/G^2 |S(G)|^2 2 (1/4eta^2 + 1/G^2) G_a G_b).
HD void ewald_plane_stress_block(const EwaldPar& p, const double* frac, const double* z, int m, int tid, int nthr,
                                 double* red, double* out7) {
  const int nm3 = 2 * p.ng[2] + 1, plane = ewald_plane_size(p);
  const int m1 = m - p.ng[0];
  const double gc2 = p.gcut * p.gcut, e4 = 4.0 * p.eta * p.eta;
  double v[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int w = tid; w < plane; w += nthr) {
    const int m2 = w / nm3 - p.ng[1], m3 = w % nm3 - p.ng[2];
    double G[3];
    const double g2 = ewald_g(p, m1, m2, m3, G);
    if ((m1 == 0 && m2 == 0 && m3 == 0) || g2 > gc2) continue;
    double sr = 0.0, si = 0.0;
    for (int i = 0; i < p.nion; ++i) {
      const double ph = 2.0 * PI_D * (m1 * frac[3 * i] + m2 * frac[3 * i + 1] + m3 * frac[3 * i + 2]);
      sr += z[i] * cos(ph);
      si += z[i] * sin(ph);
    }
    const double c = 2.0 * PI_D / p.vol * exp(-g2 / e4) / g2 * (sr * sr + si * si);
    v[0] += c;
    sym_add(v + 1, G, c * 2.0 * (1.0 / e4 + 1.0 / g2));
  }
  block_sum<7>(red, v, tid, nthr, out7);
}

#if !defined(OFDFT_EMU)
__global__ void __launch_bounds__(128) k_stress_sf(const SlotDev* sd, const IonStencil* st, cx<double>* sf) {
  const SlotDev& s = *sd;
  const int L = s.k1 + s.n2 + s.n3;
  for (int w = threadIdx.x; w < L; w += blockDim.x)
    sf[(size_t)blockIdx.x * L + w] = stress_sf_entry(s, st[blockIdx.x], w);
}
template <typename T>
__global__ void __launch_bounds__(128) k_stress(const SlotDev* sd, StressArgs sa, double* out) {
  __shared__ double red[NSC * 128];
  stress_block<T>(*sd, sa, blockIdx.x, gridDim.x, threadIdx.x, blockDim.x, red, out + (size_t)NSC * blockIdx.x);
}
template <typename T>
__global__ void __launch_bounds__(256) k_rho_vxc(const T* rho, long long n, double* out) {
  __shared__ double red[256];
  rho_vxc_block<T>(rho, n, blockIdx.x, gridDim.x, threadIdx.x, blockDim.x, red, out + blockIdx.x);
}
template <typename T>
__global__ void __launch_bounds__(256) k_sum(const T* v, long long n, double* out) {
  __shared__ double red[256];
  sum_block<T>(v, n, blockIdx.x, gridDim.x, threadIdx.x, blockDim.x, red, out + blockIdx.x);
}
template <typename T>
__global__ void __launch_bounds__(256) k_scale(T* v, long long n, double f) {
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    v[k] = (T)((double)v[k] * f);
}
__global__ void __launch_bounds__(128) k_ewald_real_stress(EwaldPar p, const double* pos, const double* z,
                                                           double* out7) {
  __shared__ double red[7 * 128];
  ewald_real_stress_block(p, pos, z, blockIdx.x, threadIdx.x, blockDim.x, red, out7 + 7 * blockIdx.x);
}
__global__ void __launch_bounds__(128) k_ewald_plane_stress(EwaldPar p, const double* frac, const double* z,
                                                            double* out7) {
  __shared__ double red[7 * 128];
  ewald_plane_stress_block(p, frac, z, blockIdx.x, threadIdx.x, blockDim.x, red, out7 + 7 * blockIdx.x);
}
#endif

}  // namespace ofdft
