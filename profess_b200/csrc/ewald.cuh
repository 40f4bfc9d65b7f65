// Ewald sum of point charges on the device (EwaldEnergy / EwaldForces,
// Source/Ewald.f90:465-1193): the splitting and cut-offs of the host sum
// (ewald_par in setup.cuh), evaluated as block tasks:
//   real space  - block i: every image and partner of ion i (its energy share
//                 and the force on it);
//   reciprocal  - block m: the structure factor S(G) of every G of plane
//                 m1 = m - ng[0] inside the cut-off, and the plane's energy;
//   rec. forces - block i: the force on ion i from every stored S(G).
// Each block adds its threads' partials in a fixed tree and the host adds the
// blocks in index order, so the result does not depend on scheduling.
#pragma once

#include "cx.cuh"
#include "setup.cuh"

namespace ofdft {

// Fixed-order tree sum of four values over the block's threads; thread 0
// writes them to out[0..3].  red holds 4 * nthr doubles.
HD void ewald_reduce4(double* red, int tid, int nthr, double v0, double v1, double v2, double v3, double* out) {
  red[4 * tid] = v0;
  red[4 * tid + 1] = v1;
  red[4 * tid + 2] = v2;
  red[4 * tid + 3] = v3;
  BLOCK_SYNC();
  for (int s = 1; s < nthr; s *= 2) {
    if ((tid % (2 * s)) == 0 && tid + s < nthr)
      for (int k = 0; k < 4; ++k) red[4 * tid + k] += red[4 * (tid + s) + k];
    BLOCK_SYNC();
  }
  if (tid == 0)
    for (int k = 0; k < 4; ++k) out[k] = red[k];
}

// out4 = (energy share of ion i, force on ion i) from the real-space sum.
HD void ewald_real_block(const EwaldPar& p, const double* pos, const double* z, int i, int tid, int nthr,
                         double* red, double* out4) {
  const int na = 2 * p.nimg[0] + 1, nb = 2 * p.nimg[1] + 1, nc = 2 * p.nimg[2] + 1;
  const long long total = (long long)na * nb * nc * p.nion;
  const double rc2 = p.rcut * p.rcut, eta = p.eta;
  const double c2 = 2.0 * eta / sqrt(PI_D);
  const double xi = pos[3 * i], yi = pos[3 * i + 1], zi_ = pos[3 * i + 2];
  double e = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
  for (long long w = tid; w < total; w += nthr) {
    const int j = (int)(w % p.nion);
    long long img = w / p.nion;
    const int c = (int)(img % nc) - p.nimg[2];
    img /= nc;
    const int b = (int)(img % nb) - p.nimg[1];
    const int a = (int)(img / nb) - p.nimg[0];
    const double dx = pos[3 * j] + p.A[0][0] * a + p.A[0][1] * b + p.A[0][2] * c - xi;
    const double dy = pos[3 * j + 1] + p.A[1][0] * a + p.A[1][1] * b + p.A[1][2] * c - yi;
    const double dz = pos[3 * j + 2] + p.A[2][0] * a + p.A[2][1] * b + p.A[2][2] * c - zi_;
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 < 1e-24 || r2 >= rc2) continue;
    const double r = sqrt(r2);
    const double ec = erfc(eta * r) / r;
    const double zz = z[i] * z[j];
    e += 0.5 * zz * ec;
    const double g = zz * (-ec / r - c2 * exp(-eta * eta * r2) / r) / r;
    fx += g * dx;
    fy += g * dy;
    fz += g * dz;
  }
  ewald_reduce4(red, tid, nthr, e, fx, fy, fz, out4);
}

HD int ewald_planes(const EwaldPar& p) { return 2 * p.ng[0] + 1; }
HD int ewald_plane_size(const EwaldPar& p) { return (2 * p.ng[1] + 1) * (2 * p.ng[2] + 1); }

// G of reciprocal index (m1, m2, m3) and |G|^2.
HD double ewald_g(const EwaldPar& p, int m1, int m2, int m3, double* G) {
  for (int k = 0; k < 3; ++k) G[k] = 2.0 * PI_D * (p.inv[0][k] * m1 + p.inv[1][k] * m2 + p.inv[2][k] * m3);
  return G[0] * G[0] + G[1] * G[1] + G[2] * G[2];
}

// Plane m: S(G) = sum_i z_i exp(i G.R_i) into sfac[m * plane + w] (zero outside
// the cut-off and at G = 0), and out4[0] = the plane's reciprocal energy.
HD void ewald_plane_block(const EwaldPar& p, const double* frac, const double* z, int m, int tid, int nthr,
                          double* red, cx<double>* sfac, double* out4) {
  const int nm3 = 2 * p.ng[2] + 1, plane = ewald_plane_size(p);
  const int m1 = m - p.ng[0];
  const double gc2 = p.gcut * p.gcut, e4 = 4.0 * p.eta * p.eta;
  double e = 0.0;
  for (int w = tid; w < plane; w += nthr) {
    const int m2 = w / nm3 - p.ng[1], m3 = w % nm3 - p.ng[2];
    double G[3];
    const double g2 = ewald_g(p, m1, m2, m3, G);
    double sr = 0.0, si = 0.0;
    if (!(m1 == 0 && m2 == 0 && m3 == 0) && g2 <= gc2) {
      for (int i = 0; i < p.nion; ++i) {
        const double ph = 2.0 * PI_D * (m1 * frac[3 * i] + m2 * frac[3 * i + 1] + m3 * frac[3 * i + 2]);
        sr += z[i] * cos(ph);
        si += z[i] * sin(ph);
      }
      e += 2.0 * PI_D / p.vol * exp(-g2 / e4) / g2 * (sr * sr + si * si);
    }
    sfac[(size_t)m * plane + w] = mk<double>(sr, si);
  }
  ewald_reduce4(red, tid, nthr, e, 0.0, 0.0, 0.0, out4);
}

// out4[1..3] = reciprocal-space force on ion i from the stored S(G).
HD void ewald_recip_force_block(const EwaldPar& p, const double* frac, const double* z, const cx<double>* sfac, int i,
                                int tid, int nthr, double* red, double* out4) {
  const int nm3 = 2 * p.ng[2] + 1, plane = ewald_plane_size(p);
  const int total = ewald_planes(p) * plane;
  const double gc2 = p.gcut * p.gcut, e4 = 4.0 * p.eta * p.eta;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  for (int w = tid; w < total; w += nthr) {
    const int m = w / plane, r = w % plane;
    const int m1 = m - p.ng[0], m2 = r / nm3 - p.ng[1], m3 = r % nm3 - p.ng[2];
    double G[3];
    const double g2 = ewald_g(p, m1, m2, m3, G);
    if ((m1 == 0 && m2 == 0 && m3 == 0) || g2 > gc2) continue;
    const cx<double> S = sfac[w];
    const double ph = 2.0 * PI_D * (m1 * frac[3 * i] + m2 * frac[3 * i + 1] + m3 * frac[3 * i + 2]);
    // Im(conj(S) e^{i G R_i})
    const double im = S.x * sin(ph) - S.y * cos(ph);
    const double c = 4.0 * PI_D / p.vol * z[i] * exp(-g2 / e4) / g2 * im;
    fx += c * G[0];
    fy += c * G[1];
    fz += c * G[2];
  }
  ewald_reduce4(red, tid, nthr, 0.0, fx, fy, fz, out4);
}

#if !defined(OFDFT_EMU)
__global__ void __launch_bounds__(256) k_ewald_real(EwaldPar p, const double* pos, const double* z, double* out4) {
  __shared__ double red[4 * 256];
  ewald_real_block(p, pos, z, blockIdx.x, threadIdx.x, blockDim.x, red, out4 + 4 * blockIdx.x);
}
__global__ void __launch_bounds__(256) k_ewald_plane(EwaldPar p, const double* frac, const double* z, cx<double>* sfac,
                                                     double* out4) {
  __shared__ double red[4 * 256];
  ewald_plane_block(p, frac, z, blockIdx.x, threadIdx.x, blockDim.x, red, sfac, out4 + 4 * blockIdx.x);
}
__global__ void __launch_bounds__(256) k_ewald_recip_force(EwaldPar p, const double* frac, const double* z,
                                                           const cx<double>* sfac, double* out4) {
  __shared__ double red[4 * 256];
  ewald_recip_force_block(p, frac, z, sfac, blockIdx.x, threadIdx.x, blockDim.x, red, out4 + 4 * blockIdx.x);
}
#endif

}  // namespace ofdft
