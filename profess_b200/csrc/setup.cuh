// Set-up of the tables a slot's evaluation reads, and the post-solve forces.
//
// Host side (once per cell or per species): cardinal B-spline weights of each
// ion (GetCardinalBSpline, Source/CBSpline.f90:42-98), the exponential-spline
// factors b1 b2 b3 (FillB, Source/CBSpline.f90:101-194), the large-eta series
// of the inverse Lindhard function, the WGC kernel ODE
// (Source/KEDF_KernelODE.f90:254-537), cubic-spline second derivatives
// (spline_cubic_set, Source/MathSplines.f90:178-393) and the Ewald ion-ion
// energy and forces (Source/Ewald.f90:465-1193).
//
// Device side (data-parallel over the grid or the ions): the WT kernel table
// (FillWT, Source/KEDF_WTkernel.f90:81-208), the WGC kernel planes
// (Source/KEDF_WGCkernel.f90:166-230), the B-spline charge spread of the
// ion-electron potential (FillQIonTable, Source/IonElectronSpline.f90:537-638;
// the transform, V_loc(G) b(G) product and inverse run through the
// evaluation passes in EV_ION mode) and the B-spline force gather
// (CalculateSplineForces, Source/IonElectronSpline.f90:642-753).
#pragma once
#include <cmath>
#include <vector>

#include "passes.cuh"

namespace ofdft {

constexpr int SPLINE_ORDER = 10;  // Source/CBSpline.f90:36

// B-spline stencil of one ion: floor of the grid coordinate and the weights
// M_n(x + i) (and the derivative weights) along each axis.
struct IonStencil {
  int fl[3];
  int species;
  double M[3][SPLINE_ORDER];
  double D[3][SPLINE_ORDER];
};

// ---------------------------------------------------------------- host helpers
// Cardinal B-spline values M_n(x + i - 1), i = 1..order, in s[1..order]; s[0] = 0.
inline void cardinal_bspline(double* s, int order, double x) {
  for (int i = 0; i <= order; ++i) s[i] = 0.0;
  s[1] = x;
  s[2] = 1.0 - x;
  for (int n = 3; n <= order; ++n)
    for (int k = 0; k < n; ++k)
      s[n - k] = ((x + (double)(n - k - 1)) * s[n - k] + ((double)(k + 1) - x) * s[n - k - 1]) / (double)(n - 1);
}

inline IonStencil ion_stencil(const double* frac, int species, const int* n) {
  IonStencil st;
  st.species = species;
  double s[SPLINE_ORDER + 1], t[SPLINE_ORDER + 1];
  for (int ax = 0; ax < 3; ++ax) {
    const double g = frac[ax] * (double)n[ax];
    const double f = std::floor(g);
    st.fl[ax] = (int)f;
    cardinal_bspline(s, SPLINE_ORDER, g - f);
    cardinal_bspline(t, SPLINE_ORDER - 1, g - f);  // t[SPLINE_ORDER] stays 0
    for (int i = 0; i < SPLINE_ORDER; ++i) {
      st.M[ax][i] = s[i + 1];
      st.D[ax][i] = (t[i + 1] - t[i]) * (double)n[ax];
    }
  }
  return st;
}

// b(m) = exp(2 pi i (order-1) m / N) / sum_k M(k+1) exp(2 pi i m k / N), m = 0..size-1.
inline std::vector<cx<double>> bspline_b(int size, int total) {
  double M[SPLINE_ORDER + 1];
  cardinal_bspline(M, SPLINE_ORDER, 1.0);
  std::vector<cx<double>> b(size);
  const long double tp = 2.0L * 3.141592653589793238462643383279502884L;
  for (int m = 0; m < size; ++m) {
    long double dr = 0, di = 0;
    for (int k = 0; k <= SPLINE_ORDER - 2; ++k) {
      const long double a = tp * (long double)m * (long double)k / (long double)total;
      dr += M[k + 1] * cosl(a);
      di += M[k + 1] * sinl(a);
    }
    const long double a = tp * (long double)(SPLINE_ORDER - 1) * (long double)m / (long double)total;
    const long double nr = cosl(a), ni = sinl(a);
    const long double den = dr * dr + di * di;
    b[m] = mk<double>((double)((nr * dr + ni * di) / den), (double)((ni * dr - nr * di) / den));
  }
  return b;
}

// Coefficients of the large-eta expansion of the inverse Lindhard function:
// with u = 1/eta^2, 1/2 + (1-eta^2)/(4 eta) ln|(1+eta)/(1-eta)| = sum_{k>=1}
// u^k / ((2k-1)(2k+1)); inverting the series, 1/F = 3 eta^2 (1 + s1 u + ...).
// out[j] = 3 s_{j+1}, j = 0..15.
inline void lind_series(double* out) {
  long double c[18], s[17];
  for (int k = 1; k <= 17; ++k) c[k] = 3.0L / ((2.0L * k - 1.0L) * (2.0L * k + 1.0L));
  s[0] = 1.0L;
  for (int j = 1; j <= 16; ++j) {
    // the coefficient of u^i in 3D/u is c[i + 1]
    long double acc = 0.0L;
    for (int i = 1; i <= j; ++i) acc += c[i + 1] * s[j - i];
    s[j] = -acc;
  }
  for (int j = 0; j < 16; ++j) out[j] = (double)(3.0L * s[j + 1]);
}

// Second derivatives of the interpolating cubic spline with the reference's
// boundary flags (0: quadratic end interval, 1: given slope, 2: given second
// derivative), by the tridiagonal (Thomas) algorithm.
inline std::vector<double> spline_cubic_set(const std::vector<double>& t, const std::vector<double>& y, int ibcbeg,
                                            double ybcbeg, int ibcend, double ybcend) {
  const int n = (int)t.size();
  std::vector<double> sub(n, 0.0), diag(n, 0.0), sup(n, 0.0), r(n, 0.0);
  if (ibcbeg == 0) { r[0] = 0.0; diag[0] = 1.0; sup[0] = -1.0; }
  else if (ibcbeg == 1) { r[0] = (y[1] - y[0]) / (t[1] - t[0]) - ybcbeg; diag[0] = (t[1] - t[0]) / 3.0; sup[0] = (t[1] - t[0]) / 6.0; }
  else { r[0] = ybcbeg; diag[0] = 1.0; sup[0] = 0.0; }
  for (int i = 1; i < n - 1; ++i) {
    r[i] = (y[i + 1] - y[i]) / (t[i + 1] - t[i]) - (y[i] - y[i - 1]) / (t[i] - t[i - 1]);
    sub[i] = (t[i] - t[i - 1]) / 6.0;
    diag[i] = (t[i + 1] - t[i - 1]) / 3.0;
    sup[i] = (t[i + 1] - t[i]) / 6.0;
  }
  if (ibcend == 0) { r[n - 1] = 0.0; sub[n - 1] = -1.0; diag[n - 1] = 1.0; }
  else if (ibcend == 1) { r[n - 1] = ybcend - (y[n - 1] - y[n - 2]) / (t[n - 1] - t[n - 2]); sub[n - 1] = (t[n - 1] - t[n - 2]) / 6.0; diag[n - 1] = (t[n - 1] - t[n - 2]) / 3.0; }
  else { r[n - 1] = ybcend; sub[n - 1] = 0.0; diag[n - 1] = 1.0; }
  // forward elimination / back substitution
  std::vector<double> cp(n), dp(n), x(n);
  cp[0] = sup[0] / diag[0];
  dp[0] = r[0] / diag[0];
  for (int i = 1; i < n; ++i) {
    const double m = diag[i] - sub[i] * cp[i - 1];
    cp[i] = i < n - 1 ? sup[i] / m : 0.0;
    dp[i] = (r[i] - sub[i] * dp[i - 1]) / m;
  }
  x[n - 1] = dp[n - 1];
  for (int i = n - 2; i >= 0; --i) x[i] = dp[i] - cp[i] * x[i + 1];
  return x;
}

// ---------------------------------------------------------------- device kernels
// keKernel = LindG(|G| / 2kF) * coef (FillWT_ReciprocalSpace, KEDF_WTkernel.f90:139-208).
template <typename T>
HD double lind_g(double eta, double lam, double mu, const double* ser) {
  if (eta < 0.0) return 0.0;
  if (eta < 1e-10) return 1.0 - lam + eta * eta * (1.0 / 3.0 - 3.0 * mu);
  if (dabs(eta - 1.0) < 1e-10) return 2.0 - lam - 3.0 * mu + 20.0 * (eta - 1.0);
  if (eta > 3.65) {
    const double e2 = eta * eta, u = 1.0 / e2;
    double poly = 0.0;
    for (int j = 15; j >= 1; --j) poly = (poly + ser[j]) * u;
    return 3.0 * (1.0 - mu) * e2 - lam + ser[0] + poly;
  }
  return 1.0 / (0.5 + 0.25 * (1.0 - eta * eta) * log((1.0 + eta) / dabs(1.0 - eta)) / eta) - 3.0 * mu * eta * eta - lam;
}

struct KernArgs {
  double ser[16];
  double lam, mu, coef, tkf, rho_s, gamma;
  int ntab;
  const double* tab;  // eta, w, w1, w2, wpp, w1pp, w2pp (7 * ntab)
};

HD double qnorm_at(const SlotDev& s, int m1, int ky, int kz) {
  const int m2 = ky > s.n2 / 2 ? ky - s.n2 : ky;
  const int m3 = kz > s.n3 / 2 ? kz - s.n3 : kz;
  const double gx = s.recip[0] * m1 + s.recip[3] * m2 + s.recip[6] * m3;
  const double gy = s.recip[1] * m1 + s.recip[4] * m2 + s.recip[7] * m3;
  const double gz = s.recip[2] * m1 + s.recip[5] * m2 + s.recip[8] * m3;
  return sqrt(gx * gx + gy * gy + gz * gz);
}

// spline_cubic_val (MathSplines.f90:395-496) on the eta table, bracketing by bisection.
HD double spline_val(const double* t, const double* y, const double* ypp, int n, double tv) {
  int lo = 0, hi = n - 1;
  if (tv <= t[0]) hi = 1;
  else if (tv >= t[n - 1]) lo = n - 2;
  else {
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (t[mid] <= tv) lo = mid; else hi = mid;
    }
  }
  if (hi != lo + 1) hi = lo + 1;
  const double dt = tv - t[lo], h = t[hi] - t[lo];
  const double tmp1 = (y[hi] - y[lo]) / h;
  const double tmp2 = -(ypp[hi] / 6.0 + ypp[lo] / 3.0) * h;
  const double tmp3 = ypp[hi] - ypp[lo];
  return y[lo] + dt * (tmp1 + tmp2 + dt * (0.5 * ypp[lo] + dt * (tmp3 / (6.0 * h))));
}

// Frequencies (kx, ky, kz) of element i of a kernel plane in the engine's
// layout: kx-major planes of n2*n3 values in the digit-reversed order of
// the slot's y and z transforms (idx: the plan index table).
HD void kernel_freq(const SlotDev& s, const int* idx, long long i, int& kx, int& ky, int& kz) {
  const int nrows = s.n2 * s.n3;
  kx = (int)(i / nrows);
  const int rem = (int)(i - (long long)kx * nrows);
  const int qz = rem / s.n2, qy = rem - qz * s.n2;
  ky = idx[s.py.perm + qy];
  kz = idx[s.pz.perm + qz];
}

// Index in the reference layout keKernel(k1G, k2G, k3G, plane) of element i
// (of all planes) in the engine's layout.
HD long long kernel_source_index(const SlotDev& s, const int* idx, long long i) {
  const long long p = i / s.Nc, e = i - p * s.Nc;
  int kx, ky, kz;
  kernel_freq(s, idx, e, kx, ky, kz);
  return p * s.Nc + kx + (long long)s.k1 * (ky + (long long)s.n2 * kz);
}

template <typename T>
HDNI void fill_kernel_point(const SlotDev& s, const int* idxtab, const KernArgs& ka, int kind, int idx) {
  int m1, ky, kz;
  kernel_freq(s, idxtab, idx, m1, ky, kz);
  const double q = qnorm_at(s, m1, ky, kz);
  T* kern = (T*)s.kern;
  if (kind == KIN_WT) {
    kern[idx] = (T)(lind_g<T>(q / ka.tkf, ka.lam, ka.mu, ka.ser) * ka.coef);
    return;
  }
  // WGC planes (KEDF_WGCkernel.f90:213-230)
  const int n = ka.ntab;
  const double* et = ka.tab;
  const double eta = q / ka.tkf;
  const double w = spline_val(et, ka.tab + n, ka.tab + 4 * n, n, eta);
  const double w1 = spline_val(et, ka.tab + 2 * n, ka.tab + 5 * n, n, eta);
  const double w2 = spline_val(et, ka.tab + 3 * n, ka.tab + 6 * n, n, eta);
  const double rs = ka.rho_s;
  kern[idx] = (T)w;
  kern[s.Nc + idx] = (T)(-w1 / (6.0 * rs));
  kern[2 * s.Nc + idx] = (T)((w2 + (7.0 - ka.gamma) * w1) / (36.0 * rs * rs));
  kern[3 * s.Nc + idx] = (T)((w2 + (1.0 + ka.gamma) * w1) / (36.0 * rs * rs));
}

// Spread one ion's B-spline stencil at -R into Q_species (FillQIonTable).
template <typename T>
HDNI void spread_ion(const SlotDev& s, const IonStencil& st, int w) {
  const int i3 = w / (SPLINE_ORDER * SPLINE_ORDER), r = w % (SPLINE_ORDER * SPLINE_ORDER);
  const int i2 = r / SPLINE_ORDER, i1 = r % SPLINE_ORDER;
  int l1 = (-st.fl[0] + i1) % s.n1; if (l1 < 0) l1 += s.n1;
  int l2 = (-st.fl[1] + i2) % s.n2; if (l2 < 0) l2 += s.n2;
  int l3 = (-st.fl[2] + i3) % s.n3; if (l3 < 0) l3 += s.n3;
  T* q = (T*)s.buf[B_PHI + st.species];
  const T v = (T)(st.M[0][i1] * st.M[1][i2] * st.M[2][i3]);
#if defined(__CUDA_ARCH__)
  atomicAdd(q + (l3 * s.n2 + l2) * s.n1 + l1, v);
#else
  q[(l3 * s.n2 + l2) * s.n1 + l1] += v;
#endif
}

// One term of -cellInv * qIonDeriv * Factor for stencil point w of an ion
// (CalculateSplineForces).  Factor_s is buf[B_B + species].
template <typename T>
HD void force_term(const SlotDev& s, const IonStencil& st, int w, double* f3) {
  const int iz = w / (SPLINE_ORDER * SPLINE_ORDER), r = w % (SPLINE_ORDER * SPLINE_ORDER);
  const int iy = r / SPLINE_ORDER, ix = r % SPLINE_ORDER;
  int l1 = (st.fl[0] - ix) % s.n1; if (l1 < 0) l1 += s.n1;
  int l2 = (st.fl[1] - iy) % s.n2; if (l2 < 0) l2 += s.n2;
  int l3 = (st.fl[2] - iz) % s.n3; if (l3 < 0) l3 += s.n3;
  const T* fac = (const T*)s.buf[B_B + st.species];
  const double F = (double)fac[(l3 * s.n2 + l2) * s.n1 + l1];
  const double q1 = st.M[1][iy] * st.M[2][iz] * st.D[0][ix];
  const double q2 = st.M[0][ix] * st.M[2][iz] * st.D[1][iy];
  const double q3 = st.M[0][ix] * st.M[1][iy] * st.D[2][iz];
  f3[0] += q1 * F;
  f3[1] += q2 * F;
  f3[2] += q3 * F;
}

}  // namespace ofdft

namespace ofdft {

// ---------------------------------------------------------------- WGC kernel ODE
// The eta grid of makeKernel2 (Source/KEDF_KernelODE.f90:298-330): step 1e-3
// from 1e-3 to 3, then step 1e-2 to 100.
inline std::vector<double> wgc_eta_grid() {
  const double ts1 = 1.0e-3, te1 = 3.0, dt1 = 1.0e-3;
  const double ts2 = te1 + dt1, te2 = 100.0, dt2 = dt1 * 10.0;
  const int n1 = (int)std::floor((te1 - ts1) / dt1) - 1;
  const int n2 = (int)std::floor((te2 - ts2) / dt2) - 1;
  std::vector<double> e;
  for (int i = 0; i < n1; ++i) e.push_back(ts1 + (double)i * dt1);
  for (int i = 0; i < n2; ++i) e.push_back(ts2 + (double)i * dt2);
  return e;
}

// Right-hand side of the WGC kernel equation (WGC, KEDF_KernelODE.f90:481-537):
// y1' = y2, y2' = [20 (F_Lind - 3 eta^2 - 1) - (gamma - 9) eta y2 - 36 (5/3 - beta) beta y1] / eta^2.
inline void wgc_rhs(double eta, const double* y, double* yp, double beta, double gamma) {
  double fl;
  if (eta == 1.0) fl = 2.0;
  else if (eta == 0.0) fl = 1.0;
  else fl = 1.0 / (0.5 + (1.0 - eta * eta) / (4.0 * eta) * std::log(std::fabs((1.0 + eta) / (1.0 - eta))));
  yp[0] = y[1];
  yp[1] = (20.0 * (fl - 3.0 * eta * eta - 1.0) - (gamma + 1.0 - 6.0 * 5.0 / 3.0) * eta * y[1] -
           36.0 * (5.0 / 3.0 - beta) * beta * y[0]) / (eta * eta);
}

// Integrate inward from eta = 100 with w = w_inf, w' = 0 (makeKernel2) using an
// adaptive Dormand-Prince 5(4) pair stepping exactly onto every grid point.
// Returns eta, w, eta w', eta^2 w'' as FillWGC_ReciprocalSpace splines them;
// the reference stores zeros at the starting point (KEDF_KernelODE.f90:351-353).
inline int wgc_radial_tables(double alpha, double beta, double gamma, std::vector<double>& eta, std::vector<double>& w,
                             std::vector<double>& w1, std::vector<double>& w2) {
  eta = wgc_eta_grid();
  const int n = (int)eta.size();
  w.assign(n, 0.0);
  w1.assign(n, 0.0);
  w2.assign(n, 0.0);
  double y[2] = {-1.6 * 20.0 / (36.0 * alpha * beta), 0.0};
  double t = eta[n - 1];
  double h = -1.0e-4;
  const double rtol = 1.0e-10, atol = 1.0e-13;
  static const double a21 = 1.0 / 5, a31 = 3.0 / 40, a32 = 9.0 / 40, a41 = 44.0 / 45, a42 = -56.0 / 15, a43 = 32.0 / 9,
                      a51 = 19372.0 / 6561, a52 = -25360.0 / 2187, a53 = 64448.0 / 6561, a54 = -212.0 / 729,
                      a61 = 9017.0 / 3168, a62 = -355.0 / 33, a63 = 46732.0 / 5247, a64 = 49.0 / 176,
                      a65 = -5103.0 / 18656, b1 = 35.0 / 384, b3 = 500.0 / 1113, b4 = 125.0 / 192,
                      b5 = -2187.0 / 6784, b6 = 11.0 / 84, e1 = 71.0 / 57600, e3 = -71.0 / 16695, e4 = 71.0 / 1920,
                      e5 = -17253.0 / 339200, e6 = 22.0 / 525, e7 = -1.0 / 40;
  long long steps = 0;
  for (int L = n - 2; L >= 0; --L) {
    const double target = eta[L];
    while (t > target) {
      if (++steps > 200000000LL) return -1;
      if (t + h < target) h = target - t;
      double k1[2], k2[2], k3[2], k4[2], k5[2], k6[2], k7[2], yt[2], y5[2];
      wgc_rhs(t, y, k1, beta, gamma);
      for (int i = 0; i < 2; ++i) yt[i] = y[i] + h * a21 * k1[i];
      wgc_rhs(t + h / 5, yt, k2, beta, gamma);
      for (int i = 0; i < 2; ++i) yt[i] = y[i] + h * (a31 * k1[i] + a32 * k2[i]);
      wgc_rhs(t + 3 * h / 10, yt, k3, beta, gamma);
      for (int i = 0; i < 2; ++i) yt[i] = y[i] + h * (a41 * k1[i] + a42 * k2[i] + a43 * k3[i]);
      wgc_rhs(t + 4 * h / 5, yt, k4, beta, gamma);
      for (int i = 0; i < 2; ++i) yt[i] = y[i] + h * (a51 * k1[i] + a52 * k2[i] + a53 * k3[i] + a54 * k4[i]);
      wgc_rhs(t + 8 * h / 9, yt, k5, beta, gamma);
      for (int i = 0; i < 2; ++i) yt[i] = y[i] + h * (a61 * k1[i] + a62 * k2[i] + a63 * k3[i] + a64 * k4[i] + a65 * k5[i]);
      wgc_rhs(t + h, yt, k6, beta, gamma);
      for (int i = 0; i < 2; ++i) y5[i] = y[i] + h * (b1 * k1[i] + b3 * k3[i] + b4 * k4[i] + b5 * k5[i] + b6 * k6[i]);
      wgc_rhs(t + h, y5, k7, beta, gamma);
      double err = 0.0;
      for (int i = 0; i < 2; ++i) {
        const double e = h * (e1 * k1[i] + e3 * k3[i] + e4 * k4[i] + e5 * k5[i] + e6 * k6[i] + e7 * k7[i]);
        const double sc = atol + rtol * std::max(std::fabs(y[i]), std::fabs(y5[i]));
        err = std::max(err, std::fabs(e) / sc);
      }
      if (err <= 1.0) {
        t += h;
        y[0] = y5[0];
        y[1] = y5[1];
        if (std::fabs(t - target) < 1e-15 * std::max(1.0, std::fabs(target))) t = target;
      }
      const double fac = err > 0 ? 0.9 * std::pow(err, -0.2) : 5.0;
      h *= std::min(5.0, std::max(0.2, fac));
      if (std::fabs(h) < 1e-14) h = -1e-14;
    }
    double yp[2];
    wgc_rhs(target, y, yp, beta, gamma);
    w[L] = y[0];
    w1[L] = target * y[1];
    w2[L] = target * target * yp[1];
    h = h < -1e-3 ? h : std::min(h, -1e-6);
  }
  return 0;
}

// ---------------------------------------------------------------- Ewald
// E = real-space sum + self term + reciprocal sum + average-potential term
// (EwaldEnergy, Source/Ewald.f90:465-520, 1150-1190), evaluated directly with
// splitting eta = sqrt(pi) (N / V^2)^(1/6) and both sums converged to ~1e-14
// relative; forces are -dE/dR (Ha/bohr).
// Splitting, cut-offs and image / reciprocal-plane ranges of the Ewald sum,
// shared by the host sum below and the device sum (ewald.cuh).
struct EwaldPar {
  double A[3][3];    // A[k][i] = component k of lattice vector i
  double inv[3][3];  // inverse of A
  double vol, eta, rcut, gcut;
  int nimg[3], ng[3];
  int nion;
};

inline EwaldPar ewald_par(const double* L, int nion) {
  // L[3*i + k] = component k of lattice vector i
  EwaldPar p;
  double (&A)[3][3] = p.A;
  double (&inv)[3][3] = p.inv;
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) A[k][i] = L[3 * i + k];
  const double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                     A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
  p.vol = std::fabs(det);
  inv[0][0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]) / det;
  inv[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) / det;
  inv[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) / det;
  inv[1][0] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) / det;
  inv[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) / det;
  inv[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) / det;
  inv[2][0] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) / det;
  inv[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) / det;
  inv[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) / det;
  const double pi = PI_D;
  p.eta = std::sqrt(pi) * std::pow((double)std::max(nion, 1) / (p.vol * p.vol), 1.0 / 6.0);
  p.rcut = 7.0 / p.eta;
  p.gcut = 2.0 * p.eta * 7.0;
  // image ranges: heights of the cell along each reciprocal direction
  for (int a = 0; a < 3; ++a) {
    const double hr = 1.0 / std::sqrt(inv[a][0] * inv[a][0] + inv[a][1] * inv[a][1] + inv[a][2] * inv[a][2]);
    p.nimg[a] = (int)std::ceil(p.rcut / hr) + 1;
    // reciprocal vector a has length 2 pi |row a of inv|; plane spacing in G space
    double la = 0;
    for (int k = 0; k < 3; ++k) la += A[k][a] * A[k][a];
    p.ng[a] = (int)std::ceil(p.gcut * std::sqrt(la) / (2.0 * pi)) + 1;
  }
  p.nion = nion;
  return p;
}

inline double ewald(const double* L, int nion, const double* frac, const double* z, double* forces) {
  const EwaldPar p = ewald_par(L, nion);
  const double(&A)[3][3] = p.A;
  const double(&inv)[3][3] = p.inv;
  const double vol = p.vol, eta = p.eta, rcut = p.rcut, gcut = p.gcut;
  const int* nimg = p.nimg;
  const int* ng = p.ng;
  const double pi = PI_D;
  std::vector<double> pos(3 * nion);
  for (int i = 0; i < nion; ++i)
    for (int k = 0; k < 3; ++k) pos[3 * i + k] = A[k][0] * frac[3 * i] + A[k][1] * frac[3 * i + 1] + A[k][2] * frac[3 * i + 2];
  if (forces)
    for (int i = 0; i < 3 * nion; ++i) forces[i] = 0.0;
  // Every partial sum lands in its own slot and the slots are added in a fixed
  // order afterwards, so the result does not depend on the thread schedule.
  std::vector<double> e_real_i(nion, 0.0);
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = 0; i < nion; ++i) {
    double e_i = 0.0;
    double fi[3] = {0, 0, 0};
    for (int a = -nimg[0]; a <= nimg[0]; ++a)
      for (int b = -nimg[1]; b <= nimg[1]; ++b)
        for (int c = -nimg[2]; c <= nimg[2]; ++c) {
          double tr[3];
          for (int k = 0; k < 3; ++k) tr[k] = A[k][0] * a + A[k][1] * b + A[k][2] * c;
          for (int j = 0; j < nion; ++j) {
            const double dx = pos[3 * j] + tr[0] - pos[3 * i];
            const double dy = pos[3 * j + 1] + tr[1] - pos[3 * i + 1];
            const double dz = pos[3 * j + 2] + tr[2] - pos[3 * i + 2];
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 < 1e-24 || r2 >= rcut * rcut) continue;
            const double r = std::sqrt(r2);
            const double ec = std::erfc(eta * r) / r;
            e_i += 0.5 * z[i] * z[j] * ec;
            if (forces) {
              const double dterm = -ec / r - 2.0 * eta / std::sqrt(pi) * std::exp(-eta * eta * r2) / r;
              const double g = z[i] * z[j] * dterm / r;
              fi[0] += g * dx;
              fi[1] += g * dy;
              fi[2] += g * dz;
            }
          }
        }
    if (forces)
      for (int k = 0; k < 3; ++k) forces[3 * i + k] += fi[k];
    e_real_i[i] = e_i;
  }
  double e_real = 0.0;
  for (int i = 0; i < nion; ++i) e_real += e_real_i[i];
  double qsum = 0.0, q2 = 0.0;
  for (int i = 0; i < nion; ++i) { qsum += z[i]; q2 += z[i] * z[i]; }
  const double e_self = -eta / std::sqrt(pi) * q2;
  const double e_bg = -0.5 * pi / (eta * eta) / vol * qsum * qsum;
  // reciprocal sum over G = m1 b1 + m2 b2 + m3 b3, b_a = 2 pi (row a of inv)
  const int n_m1 = 2 * ng[0] + 1;
  const size_t nf3 = forces ? 3 * (size_t)nion : 0;
  std::vector<double> fr_m1(nf3 * n_m1, 0.0), e_rec_m1(n_m1, 0.0);
#pragma omp parallel for schedule(dynamic, 1)
  for (int m1 = -ng[0]; m1 <= ng[0]; ++m1) {
    double* floc = fr_m1.data() + nf3 * (size_t)(m1 + ng[0]);
    double e_m = 0.0;
    for (int m2 = -ng[1]; m2 <= ng[1]; ++m2)
      for (int m3 = -ng[2]; m3 <= ng[2]; ++m3) {
        if (m1 == 0 && m2 == 0 && m3 == 0) continue;
        double G[3];
        for (int k = 0; k < 3; ++k) G[k] = 2.0 * pi * (inv[0][k] * m1 + inv[1][k] * m2 + inv[2][k] * m3);
        const double g2 = G[0] * G[0] + G[1] * G[1] + G[2] * G[2];
        if (g2 > gcut * gcut) continue;
        double sr = 0.0, si = 0.0;
        for (int i = 0; i < nion; ++i) {
          const double ph = 2.0 * pi * (m1 * frac[3 * i] + m2 * frac[3 * i + 1] + m3 * frac[3 * i + 2]);
          sr += z[i] * std::cos(ph);
          si += z[i] * std::sin(ph);
        }
        const double fg = std::exp(-g2 / (4.0 * eta * eta)) / g2;
        e_m += 2.0 * pi / vol * fg * (sr * sr + si * si);
        if (forces) {
          for (int i = 0; i < nion; ++i) {
            const double ph = 2.0 * pi * (m1 * frac[3 * i] + m2 * frac[3 * i + 1] + m3 * frac[3 * i + 2]);
            // Im(conj(S) e^{i G R_i})
            const double im = sr * std::sin(ph) - si * std::cos(ph);
            const double c = 4.0 * pi / vol * z[i] * fg * im;
            for (int k = 0; k < 3; ++k) floc[3 * i + k] += c * G[k];
          }
        }
      }
    e_rec_m1[m1 + ng[0]] = e_m;
  }
  double e_rec = 0.0;
  for (int k = 0; k < n_m1; ++k) {
    e_rec += e_rec_m1[k];
    for (size_t i = 0; i < nf3; ++i) forces[i] += fr_m1[nf3 * (size_t)k + i];
  }
  return e_real + e_self + e_rec + e_bg;
}

}  // namespace ofdft
