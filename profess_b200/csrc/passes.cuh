// Block functions of the engine: the vector-op kernel and the five passes of
// one potential evaluation (CalculatePotentialPlus):
//
//   pass 1  X forward : prologue (phi_in, rho and the functional's fields) and
//                       the x-direction real-to-complex FFT of row pairs
//   pass 2  Y forward : complex FFT along y on (field, z, kx-tile) tiles
//   pass 3  Z         : complex FFT along z, the k-space operator of each field
//                       group (Hartree 4pi/G^2, vW G^2, WT/WGC kernels, with the
//                       1/N forward scaling), inverse FFT along z
//   pass 4  Y inverse
//   pass 5  X inverse : complex-to-real FFT of all fields of a row pair and the
//                       real-space epilogue (potential, chain rule, energies and
//                       the optimiser's fused sums)
//
// Every block processes one task.  Blocks that finish a slot's work in the
// vector kernel or in pass 5 add their per-channel partial sums to the slot's
// partials; the last of them reduces the partials in a fixed order (the result
// does not depend on block scheduling) and runs the NTN controller.
#pragma once
#include "ntn_ctl.cuh"

namespace ofdft {

#if defined(__CUDA_ARCH__)
HD int atomic_inc(int* p) { return atomicAdd(p, 1); }
HD void fence() { __threadfence(); }
#else
HD int atomic_inc(int* p) { int v = *p; *p = v + 1; return v; }
HD void fence() {}
#endif

constexpr double PI_D = 3.141592653589793238462643;
constexpr double C_TF = 2.87123400018819;  // Source/KEDF_TF.f90:42

template <typename T>
struct Args {
  SlotDev* slots;
  Ctl* ctl;
  const Task* tasks;
  const cx<T>* tw;
  int tx;      // kx tile width of the Y/Z passes
  int vchunk;  // points per task of the vector kernel
};

// ------------------------------------------------------------ reductions
// Reduce acc[NCH] over the block into sred[0*nthr], sred[1*nthr], ...
HDNI inline void block_reduce(double* sred, const double* acc, int tid, int nthr) {
  for (int ch = 0; ch < NCH; ++ch) sred[ch * nthr + tid] = acc[ch];
  BLOCK_SYNC();
  for (int stride = nthr / 2; stride > 0; stride >>= 1) {
    for (int w = tid; w < NCH * stride; w += nthr) {
      const int ch = w / stride, i = w % stride;
      sred[ch * nthr + i] += sred[ch * nthr + i + stride];
    }
    BLOCK_SYNC();
  }
}

// Store this task's partials; the last task of the slot reduces them and runs
// the controller.  kid selects the done counter; what is the op / eval mode.
HDNI inline void slot_finish(SlotDev& s, Ctl& c, int kid, int what, int task_idx, const double* acc,
                             double* sred, int* sflag, int tid, int nthr) {
  block_reduce(sred, acc, tid, nthr);
  for (int ch = tid; ch < NCH; ch += nthr) s.partials[(long long)task_idx * NCH + ch] = sred[ch * nthr];
  BLOCK_SYNC();
  if (tid == 0) {
    fence();
    const int prev = atomic_inc(&s.done[kid]);
    *sflag = (prev == s.ntask[kid] - 1) ? 1 : 0;
  }
  BLOCK_SYNC();
  if (*sflag == 0) return;
  fence();
  const int nt = s.ntask[kid];
  double part[NCH];
  for (int ch = 0; ch < NCH; ++ch) part[ch] = 0.0;
  for (int t = tid; t < nt; t += nthr)
    for (int ch = 0; ch < NCH; ++ch) part[ch] += s.partials[(long long)t * NCH + ch];
  block_reduce(sred, part, tid, nthr);
  if (tid == 0) {
    double red[NCH];
    for (int ch = 0; ch < NCH; ++ch) red[ch] = sred[ch * nthr];
    s.done[kid] = 0;
    ntn_after(c, s, red, kid, what);
  }
  BLOCK_SYNC();
}

// ------------------------------------------------------------ vector ops
template <typename T>
HDNI void vec_block(const Args<T>& a, int bid, int tid, int nthr, char* smem) {
  const Task t = a.tasks[bid];
  SlotDev& s = a.slots[t.slot];
  Ctl& c = a.ctl[t.slot];
  const int op = c.op;
  if (c.status != ST_RUNNING || op == OP_NONE) return;
  T* phi = (T*)s.buf[c.iphi];
  T* w0 = (T*)s.buf[c.iw0];
  T* w1 = (T*)s.buf[c.iw1];
  T* bb = (T*)s.buf[B_B];
  T* r = (T*)s.buf[B_R];
  T* p = (T*)s.buf[B_P];
  T* d = (T*)s.buf[B_D];
  const T k = (T)c.opc;
  const long long i0 = (long long)t.a * a.vchunk;
  long long i1 = i0 + a.vchunk;
  if (i1 > s.N) i1 = s.N;
  double acc[NCH];
  for (int ch = 0; ch < NCH; ++ch) acc[ch] = 0.0;
  for (long long i = i0 + tid; i < i1; i += nthr) {
    switch (op) {
      case OP_SQRT_INIT: {
        const T rho = phi[i];
        acc[0] += (double)rho;
        phi[i] = m_sqrt(rho < T(0) ? -rho : rho);
        break;
      }
      case OP_DLDPHI: {
        const T v = w0[i] - k * T(2) * phi[i];
        bb[i] = v;
        r[i] = -v;
        p[i] = -v;
        d[i] = T(0);
        acc[0] += (double)v * (double)v;
        break;
      }
      case OP_CGSTEP: {
        const T dn = d[i] + k * p[i];
        const T rn = r[i] - k * w1[i];
        d[i] = dn;
        r[i] = rn;
        const T f = phi[i];
        const T pd = f + dn;
        acc[0] += (double)rn * (double)rn;
        acc[1] += (double)pd * (double)pd;
        acc[2] += (double)f * (double)dn;
        break;
      }
      case OP_PUPD: {
        const T pn = r[i] + k * p[i];
        p[i] = pn;
        acc[0] += (double)pn * (double)pn;
        break;
      }
      case OP_DIRNEG:
      case OP_NG1:
      case OP_SD: {
        T dn;
        if (op == OP_DIRNEG) dn = -(d[i] - k * p[i]);
        else if (op == OP_SD) dn = -bb[i];
        else dn = d[i];
        if (op != OP_NG1) d[i] = dn;
        const T f = phi[i];
        const T pd = f + dn;
        acc[1] += (double)pd * (double)pd;
        acc[2] += (double)f * (double)dn;
        break;
      }
      case OP_NG2: {
        const T dn = d[i] - phi[i] * k;
        d[i] = dn;
        acc[0] += (double)dn * (double)dn;
        acc[1] += (double)w0[i] * (double)dn;
        break;
      }
      default:
        break;
    }
  }
  double* sred = (double*)smem;
  int* sflag = (int*)(sred + NCH * nthr);
  slot_finish(s, c, K_VEC, op, t.a, acc, sred, sflag, tid, nthr);
}

// ------------------------------------------------------------ fields
// phi_in of the current evaluation at point i, and rho = phi_in^2.
template <typename T>
HD void phi_in_at(const SlotDev& s, const Ctl& c, long long i, T& phin, T& rho) {
  const T* A = (const T*)s.buf[c.iphi];
  if (c.ev == EV_RHO) {
    rho = A[i];
    phin = m_sqrt(rho);
    return;
  }
  const T* B = (const T*)s.buf[c.evb];
  phin = (T)c.ca * A[i] + (T)c.cb * B[i];
  rho = phin * phin;
}

// Value of forward field f (see the field tables in the header comment of
// SlotDev setup) at density rho.
template <typename T>
HD T field_value(const SlotDev& s, int f, T rho) {
  if (s.kinetic == KIN_WT) {
    switch (f) {
      case 0: return rho;
      case 1: return m_pow(rho, (T)s.beta);
      case 2: return m_sqrt(rho);
      default: return m_pow(rho, (T)s.alpha);
    }
  }
  switch (f) {
    case 0: return rho;
    case 1: return m_sqrt(rho);
    default: break;
  }
  const T ex = f < 5 ? (T)s.alpha : (T)s.beta;
  const int k = (f - 2) % 3;
  const T rx = m_pow(rho, ex);
  const T th = rho - (T)s.rho_s;
  if (k == 0) return rx;
  if (k == 1) return th * rx;
  return th * th * rx / T(2);
}

// ------------------------------------------------------------ pass 1
template <typename T>
HDNI void xfwd_block(const Args<T>& a, int bid, int tid, int nthr, char* smem) {
  const Task t = a.tasks[bid];
  SlotDev& s = a.slots[t.slot];
  const Ctl& c = a.ctl[t.slot];
  if (c.status != ST_RUNNING || c.ev == EV_NONE) return;
  const int f = t.a, rp0 = t.b, nb = t.c;
  const int n1 = s.n1, k1 = s.k1;
  const long long nrows = (long long)s.n2 * s.n3;
  cx<T>* buf = (cx<T>*)smem;
  cx<T>* tmp = buf + (size_t)nb * n1;
  for (int w = tid; w < nb * n1; w += nthr) {
    const int b = w / n1, i = w % n1;
    const long long j0 = 2LL * (rp0 + b), j1 = j0 + 1;
    T phin, rho;
    phi_in_at(s, c, j0 * n1 + i, phin, rho);
    const T v0 = field_value(s, f, rho);
    T v1 = T(0);
    if (j1 < nrows) {
      phi_in_at(s, c, j1 * n1 + i, phin, rho);
      v1 = field_value(s, f, rho);
    }
    buf[b + i * nb] = mk<T>(v0, v1);
  }
  BLOCK_SYNC();
  fft_batch(buf, tmp, nb, 1, nb, s.px, a.tw, -1, tid, nthr);
  cx<T>* out = (cx<T>*)s.spec + (long long)f * s.Nc;
  for (int w = tid; w < nb * k1; w += nthr) {
    const int b = w / k1, k = w % k1;
    const long long j0 = 2LL * (rp0 + b), j1 = j0 + 1;
    const cx<T> z = buf[b + k * nb];
    const cx<T> zc = conj(buf[b + ((n1 - k) % n1) * nb]);
    const cx<T> sum = z + zc, dif = z - zc;
    out[j0 * k1 + k] = mk<T>(sum.x * T(0.5), sum.y * T(0.5));
    if (j1 < nrows) out[j1 * k1 + k] = mk<T>(dif.y * T(0.5), -dif.x * T(0.5));
  }
}

// ------------------------------------------------------------ passes 2, 4
template <typename T>
HDNI void ypass_block(const Args<T>& a, int bid, int tid, int nthr, char* smem, int dir) {
  const Task t = a.tasks[bid];
  SlotDev& s = a.slots[t.slot];
  const Ctl& c = a.ctl[t.slot];
  if (c.status != ST_RUNNING || c.ev == EV_NONE) return;
  const int f = t.a, z = t.b, kx0 = t.c;
  const int n2 = s.n2, k1 = s.k1, TX = a.tx;
  const int nb = (k1 - kx0) < TX ? (k1 - kx0) : TX;
  cx<T>* buf = (cx<T>*)smem;
  cx<T>* tmp = buf + (size_t)TX * n2;
  cx<T>* sp = (cx<T>*)s.spec + (long long)f * s.Nc + (long long)z * n2 * k1 + kx0;
  for (int w = tid; w < nb * n2; w += nthr) {
    const int i = w / nb, b = w % nb;
    buf[b + i * TX] = sp[(long long)i * k1 + b];
  }
  BLOCK_SYNC();
  fft_batch(buf, tmp, nb, 1, TX, s.py, a.tw, dir, tid, nthr);
  for (int w = tid; w < nb * n2; w += nthr) {
    const int i = w / nb, b = w % nb;
    sp[(long long)i * k1 + b] = buf[b + i * TX];
  }
}

// ------------------------------------------------------------ pass 3
template <typename T>
HDNI void zpass_block(const Args<T>& a, int bid, int tid, int nthr, char* smem) {
  const Task t = a.tasks[bid];
  SlotDev& s = a.slots[t.slot];
  const Ctl& c = a.ctl[t.slot];
  if (c.status != ST_RUNNING || c.ev == EV_NONE) return;
  const int g = t.a, ky = t.b, kx0 = t.c;
  const int n2 = s.n2, n3 = s.n3, k1 = s.k1, TX = a.tx;
  const int nb = (k1 - kx0) < TX ? (k1 - kx0) : TX;
  const int kind = s.group_kind[g], f0 = s.group_f0[g], gn = s.group_nf[g];
  const long long plane = (long long)n2 * k1;
  cx<T>* fb[3];
  for (int q = 0; q < 3; ++q) fb[q] = (cx<T>*)smem + (size_t)q * TX * n3;
  cx<T>* tmp = (cx<T>*)smem + (size_t)3 * TX * n3;
  for (int w = tid; w < gn * nb * n3; w += nthr) {
    const int q = w / (nb * n3), rem = w % (nb * n3);
    const int i = rem / nb, b = rem % nb;
    const cx<T>* sp = (const cx<T>*)s.spec + (long long)(f0 + q) * s.Nc;
    fb[q][b + i * TX] = sp[(long long)i * plane + (long long)ky * k1 + kx0 + b];
  }
  BLOCK_SYNC();
  for (int q = 0; q < gn; ++q) fft_batch(fb[q], tmp, nb, 1, TX, s.pz, a.tw, -1, tid, nthr);
  const int m2 = ky > n2 / 2 ? ky - n2 : ky;
  const T* kern = (const T*)s.kern;
  for (int w = tid; w < nb * n3; w += nthr) {
    const int i = w / nb, b = w % nb;
    const int m1 = kx0 + b;
    const int m3 = i > n3 / 2 ? i - n3 : i;
    const double gx = s.recip[0] * m1 + s.recip[3] * m2 + s.recip[6] * m3;
    const double gy = s.recip[1] * m1 + s.recip[4] * m2 + s.recip[7] * m3;
    const double gz = s.recip[2] * m1 + s.recip[5] * m2 + s.recip[8] * m3;
    const double q = sqrt(gx * gx + gy * gy + gz * gz);
    const double q2 = q * q;
    const long long idx = (long long)i * plane + (long long)ky * k1 + m1;
    const int e = b + i * TX;
    const T sc = (T)s.inv_n;
    switch (kind) {
      case G_HARTREE: {
        const T m = (m1 == 0 && ky == 0 && i == 0) ? T(0) : (T)(4.0 * PI_D / q2) * sc;
        fb[0][e] = fb[0][e] * m;
        break;
      }
      case G_VW:
        fb[0][e] = fb[0][e] * ((T)q2 * sc);
        break;
      case G_KMUL:
        fb[0][e] = fb[0][e] * (kern[idx] * sc);
        break;
      default: {  // second-order WGC triple (KEDF_WGC.f90:219-236)
        const T K1 = kern[idx], K2 = kern[s.Nc + idx], K3 = kern[2 * s.Nc + idx], K4 = kern[3 * s.Nc + idx];
        const cx<T> F0 = fb[0][e], F1 = fb[1][e], F2 = fb[2][e];
        fb[0][e] = (F0 * K1 + F1 * K2 + F2 * K3) * sc;
        fb[1][e] = (F0 * K2 + F1 * K4) * sc;
        fb[2][e] = F0 * (K3 * sc);
        break;
      }
    }
  }
  BLOCK_SYNC();
  for (int q = 0; q < gn; ++q) fft_batch(fb[q], tmp, nb, 1, TX, s.pz, a.tw, 1, tid, nthr);
  for (int w = tid; w < gn * nb * n3; w += nthr) {
    const int q = w / (nb * n3), rem = w % (nb * n3);
    const int i = rem / nb, b = rem % nb;
    cx<T>* sp = (cx<T>*)s.spec + (long long)(f0 + q) * s.Nc;
    sp[(long long)i * plane + (long long)ky * k1 + kx0 + b] = fb[q][b + i * TX];
  }
}

// ------------------------------------------------------------ pass 5
// Perdew-Zunger LDA potential and energy density (XC_LDA.f90:51-310), with
// r13 = rho^(1/3).
template <typename T>
HD void lda_point(T rho, T r13, T& vxc, T& exc) {
  const T cXp = T(-0.98474502184269641), cXe = T(-0.73855876638202234), cC = T(0.62035049089940009);
  const T rs = cC / r13;
  if (rs < T(1)) {
    const T lr = m_log(rs);
    vxc = cXp * r13 + lr * (T(3.11e-2) + T(1.33333333333333333e-3) * rs) + T(-5.83666666666666666e-2) +
          T(-8.4e-3) * rs;
    exc = cXe * rho * r13 + rho * (lr * (T(3.11e-2) + T(2e-3) * rs) + T(-4.8e-2) + T(-1.16e-2) * rs);
  } else {
    const T sr = m_sqrt(rs);
    const T den = T(1) + T(1.0529) * sr + T(3.334e-1) * rs;
    vxc = cXp * r13 + (T(-1.423e-1) + T(-0.174798948333333333) * sr + T(-6.325709333333333333e-2) * rs) / (den * den);
    exc = cXe * rho * r13 + rho * (T(-1.423e-1) / den);
  }
}

template <typename T>
HDNI void xinv_block(const Args<T>& a, int bid, int tid, int nthr, char* smem) {
  const Task t = a.tasks[bid];
  SlotDev& s = a.slots[t.slot];
  Ctl& c = a.ctl[t.slot];
  const int ev = c.ev;
  if (c.status != ST_RUNNING || ev == EV_NONE) return;
  const int rp0 = t.a, nb = t.b, ordinal = t.c;
  const int n1 = s.n1, k1 = s.k1, nf = s.nf;
  const long long nrows = (long long)s.n2 * s.n3;
  cx<T>* fb = (cx<T>*)smem;  // nf buffers of nb*n1
  cx<T>* tmp = fb + (size_t)nf * nb * n1;
  const bool even = (n1 % 2) == 0;
  for (int f = 0; f < nf; ++f) {
    const cx<T>* sp = (const cx<T>*)s.spec + (long long)f * s.Nc;
    cx<T>* bf = fb + (size_t)f * nb * n1;
    for (int w = tid; w < nb * n1; w += nthr) {
      const int b = w / n1, k = w % n1;
      const long long j0 = 2LL * (rp0 + b), j1 = j0 + 1;
      cx<T> A, B;
      if (k < k1) {
        A = sp[j0 * k1 + k];
        B = j1 < nrows ? sp[j1 * k1 + k] : mk<T>(T(0), T(0));
        if (k == 0 || (even && k == n1 / 2)) {  // c2r ignores these imaginary parts
          A.y = T(0);
          B.y = T(0);
        }
      } else {
        const int kk = n1 - k;
        A = conj(sp[j0 * k1 + kk]);
        B = j1 < nrows ? conj(sp[j1 * k1 + kk]) : mk<T>(T(0), T(0));
      }
      bf[b + k * nb] = mk<T>(A.x - B.y, A.y + B.x);
    }
  }
  BLOCK_SYNC();
  for (int f = 0; f < nf; ++f) fft_batch(fb + (size_t)f * nb * n1, tmp, nb, 1, nb, s.px, a.tw, 1, tid, nthr);

  const T* vion = (const T*)s.vion;
  T* phi = (T*)s.buf[c.iphi];
  T* w0 = (T*)s.buf[c.iw0];
  T* w1 = (T*)s.buf[c.iw1];
  T* trial = (T*)s.buf[c.itrial];
  const T* bb = (const T*)s.buf[B_B];
  const T* p = (const T*)s.buf[B_P];
  const T* d = (const T*)s.buf[B_D];
  const bool energy = (ev != EV_CG) && (ev != EV_RHO || c.want_energy);
  const T lam = (T)s.lambda, muv = (T)s.mu, al = (T)s.alpha, be = (T)s.beta, cTF = (T)C_TF;
  const T mu0 = (T)c.mu, eps = (T)c.eps, st = (T)c.st, ctd = (T)(c.ct * c.dscale);
  double acc[NCH];
  for (int ch = 0; ch < NCH; ++ch) acc[ch] = 0.0;
  for (int w = tid; w < nb * 2 * n1; w += nthr) {
    const int b = w / (2 * n1), rem = w % (2 * n1);
    const int half = rem / n1, i = rem % n1;
    const long long j = 2LL * (rp0 + b) + half;
    if (j >= nrows) continue;
    const long long idx = j * n1 + i;
    T o[MAX_FIELDS];
    for (int f = 0; f < nf; ++f) {
      const cx<T> z = fb[(size_t)f * nb * n1 + b + i * nb];
      o[f] = half == 0 ? z.x : z.y;
    }
    T phin, rho;
    phi_in_at(s, c, idx, phin, rho);
    const T sq = m_sqrt(rho);
    const T r13 = m_cbrt(rho);
    const T r23 = r13 * r13;
    T vxc, exc;
    lda_point(rho, r13, vxc, exc);
    T vnl, enl, lap;
    if (s.kinetic == KIN_WT) {
      const T rb = m_pow(rho, be);
      const T ra = s.alpha_eq_beta ? rb : m_pow(rho, al);
      const T pa = nf > 3 ? o[3] : o[1];
      vnl = cTF * (al * (ra / rho) * o[1] + be * (rb / rho) * pa);
      enl = cTF * ra * o[1];
      lap = o[2];
    } else {
      const T th = rho - (T)s.rho_s;
      const T ra = m_pow(rho, al), rb = m_pow(rho, be);
      vnl = cTF * ((rb / rho) * (be * o[2] + (rho + be * th) * o[3] + th * (rho + be * th / T(2)) * o[4]) +
                   (ra / rho) * (al * o[5] + (rho + al * th) * o[6] + th * (rho + al * th / T(2)) * o[7]));
      enl = cTF * rb * (o[2] + th * o[3] + th * th / T(2) * o[4]);
      lap = o[1];
    }
    const T vi = vion[idx];
    const T potr = vi + o[0] + vxc + (T(5) / T(3) * cTF * lam) * r23 + vnl;
    T pot;
    if (ev == EV_RHO && !c.opt_sqrt)
      pot = potr + muv * lap / (T(2) * sq);
    else
      pot = T(2) * sq * potr + muv * lap;
    if (energy) {
      acc[CH_EIE] += (double)rho * (double)vi;
      acc[CH_EH] += 0.5 * (double)o[0] * (double)rho;
      acc[CH_EXC] += (double)exc;
      acc[CH_ETF] += (double)(lam * cTF) * (double)(rho * r23);
      acc[CH_EVW] += 0.5 * (double)muv * (double)sq * (double)lap;
      acc[CH_ENL] += (double)enl;
    }
    const T sg = phin < T(0) ? T(-1) : T(1);
    switch (ev) {
      case EV_RHO:
        w0[idx] = pot;
        break;
      case EV_PHI: {
        const T gg = pot * sg;
        w0[idx] = gg;
        acc[CH_M0] += (double)gg * (double)phin;
        acc[CH_M1] += (double)phin * (double)phin;
        break;
      }
      case EV_CG: {
        const T gg = pot * sg;
        const T ap = ((gg - mu0 * T(2) * phin) - bb[idx]) / eps;
        w1[idx] = ap;
        acc[CH_M0] += (double)p[idx] * (double)ap;
        break;
      }
      default: {  // EV_LS
        const T gg = pot * sg;
        w1[idx] = gg;
        trial[idx] = phin;
        const T dir = -phi[idx] * st + d[idx] * ctd;
        const T dl = gg - T(2) * phin * mu0;
        acc[CH_M0] += (double)gg * (double)dir;
        acc[CH_M1] += (double)dl * (double)dl;
        acc[CH_M2] += (double)gg * (double)phin;
        acc[CH_M3] += (double)phin * (double)phin;
        break;
      }
    }
  }
  double* sred = (double*)(tmp + (size_t)nb * n1);
  int* sflag = (int*)(sred + NCH * nthr);
  slot_finish(s, c, K_X5, ev, ordinal, acc, sred, sflag, tid, nthr);
}

}  // namespace ofdft
