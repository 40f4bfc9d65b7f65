// Block functions of the engine: the vector-op kernel and the passes of one
// potential evaluation (CalculatePotentialPlus).
//
// Spectrum layout: field f of a slot is a half spectrum of k1 = n1/2 + 1
// planes, kx-major: element (kx, row j = y + n2 z) at spec[f*Nc + kx*nrows +
// j], so that every (y, z) plane of one kx is contiguous.  Between the
// forward and the inverse transforms along y and z the plane is in the
// digit-reversed order of the in-place FFT (position q holds frequency
// perm[q]); the kernel planes are stored in that order.
//
//   pass 1  X forward : prologue (phi_in, rho and the functional's fields) and
//                       the x-direction real-to-complex FFT of row pairs,
//                       stored kx-major
//   pass YZ           : one (y, z) plane of one field in shared memory:
//                       forward FFT along y and z, the k-space operator
//                       (Hartree 4pi/G^2, vW G^2, the WT kernel, with the 1/N
//                       forward scaling), inverse FFT along z and y
//   (planes that do not fit shared memory, the WGC groups and the set-up
//    modes run the same work as three passes: Y forward, Z with the
//    operator, Y inverse)
//   pass 5  X inverse : complex-to-real FFT of all fields of a row pair and the
//                       real-space epilogue (potential, chain rule, energies and
//                       the optimiser's fused sums)
//
// Every block processes one task.  The block functions are force-inlined into
// their kernels: each kernel calls one, and a non-inlined call puts the
// functions' small structs and arrays in local memory.  Blocks of the vector kernel and of pass 5
// store their per-channel sums in the slot's partials; a controller kernel
// that follows (one block per slot) reduces them in a fixed order (the result
// does not depend on block scheduling) and runs the NTN controller.
#pragma once
#include "ntn_ctl.cuh"

namespace ofdft {

constexpr double PI_D = 3.141592653589793238462643;
constexpr double C_TF = 2.87123400018819;  // Source/KEDF_TF.f90:42

// Kernel instantiations per kinetic functional: the WT kernels carry at most
// 4 fields and no WGC code, so their register allocation is not set by the
// 8-field WGC paths.
enum KinSel : int { KS_WT = 0, KS_WGC = 1 };
template <int KS> struct KinFields { static constexpr int value = KS == KS_WT ? 4 : MAX_FIELDS; };

template <typename T>
struct Args {
  SlotDev* slots;
  Ctl* ctl;
  const Task* tasks;
  const cx<T>* tw;   // roots of unity of every plan length
  const int* idx;    // digit-reversal tables (FftPlan::perm, iperm)
  int vchunk;        // points per task of the vector kernel
};

// Shared memory of an x-inverse task with nfb transformed fields (or ion
// species) and nb row pairs, elements of esz bytes: the transform buffer,
// then the reduction scratch.
HD size_t align16(size_t x) { return (x + 15) & ~size_t(15); }
HD size_t xinv_smem(int n1, int nfb, int nb, size_t esz) {
  return align16((size_t)nfb * nb * n1 * 2 * esz) + NCH * 33 * sizeof(double);
}

// Shared memory of an x-forward task: the transform buffer, then the task's
// rows of the two evaluation inputs.
HD size_t xfwd_stage_offset(int n1, int nfb, int nb, size_t esz) {
  return align16((size_t)nfb * nb * n1 * 2 * esz);
}
HD size_t xfwd_smem(int n1, int nfb, int nb, size_t esz) {
  return xfwd_stage_offset(n1, nfb, nb, esz) + 2 * align16((size_t)2 * nb * n1 * esz);
}

// V_loc(|q|) by the index-knot cubic spline (PspRecipCubicSpline, LocalPseudoPot.f90:92-202).
HD double psp_value(const IonAux& x, int sp, double q) {
  const PspDev& p = x.psp[sp];
  if (q == 0.0) return p.v0;
  if (q >= p.max_g) return 0.0;
  const double pos = q / p.dq + 1.0;
  const int left = (int)floor(pos);
  const double dt = pos - (double)left;
  const double* vqs = x.tab + p.off;
  const double* pdd = x.tab + p.off + p.npts;
  const double yl = vqs[left - 1], yr = vqs[left];
  const double pl = pdd[left - 1], pr = pdd[left];
  const double yval = yl + dt * (yr - yl - (pr / 6.0 + pl / 3.0) + dt * (0.5 * pl + dt * ((pr - pl) / 6.0)));
  return yval - 4.0 * PI_D * p.charge / (q * q);
}

// ------------------------------------------------------------ reductions
// Reduce channels [LO, HI) of acc[NCH] over the block; the block totals end
// up in sred[LO..HI-1] and the other channels of sred[0..NCH-1] are zero.  On
// the device: warp shuffles, then one warp over the per-warp sums (sred needs
// NCH * 33 doubles).  In the host emulation the block has one thread.  Passes
// whose sums use few channels (a CG evaluation one, the vector operations
// three) reduce only those.
template <int LO = 0, int HI = NCH>
HDNI inline void block_reduce(double* sred, const double* acc, int tid, int nthr) {
#if defined(__CUDA_ARCH__)
  const int lane = tid & 31, warp = tid >> 5, nw = (nthr + 31) >> 5;
  double v[NCH];
#pragma unroll
  for (int ch = LO; ch < HI; ++ch) {
    double x = acc[ch];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    v[ch] = x;
  }
  if (lane == 0) {
#pragma unroll
    for (int ch = LO; ch < HI; ++ch) sred[NCH + ch * 32 + warp] = v[ch];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int ch = 0; ch < NCH; ++ch) {
      if (ch < LO || ch >= HI) {
        if (lane == 0) sred[ch] = 0.0;
        continue;
      }
      double x = lane < nw ? sred[NCH + ch * 32 + lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane == 0) sred[ch] = x;
    }
  }
  __syncthreads();
#else
  (void)tid;
  (void)nthr;
  for (int ch = 0; ch < NCH; ++ch) sred[ch] = (ch >= LO && ch < HI) ? acc[ch] : 0.0;
#endif
}

// Store this task's per-channel sums (channels [LO, HI), the rest zero) in
// the slot's partials.
template <int LO = 0, int HI = NCH>
HDNI inline void store_partials(SlotDev& s, int task_idx, const double* acc, double* sred, int tid, int nthr) {
  block_reduce<LO, HI>(sred, acc, tid, nthr);
  if (tid == 0) {
#pragma unroll
    for (int ch = 0; ch < NCH; ++ch) s.partials[(size_t)task_idx * NCH + ch] = sred[ch];
  }
}

// Shared memory of the controller block: the reduction scratch, then a copy
// of the slot's controller record.
constexpr size_t CTL_SRED_BYTES = (NCH * 33 + 2) * sizeof(double);
constexpr size_t CTL_SMEM_BYTES = CTL_SRED_BYTES + sizeof(Ctl);
static_assert(sizeof(Ctl) % 8 == 0, "the controller record is copied as 8-byte words");

// Copy nbytes (a multiple of 8) as 8-byte words spread over the block.
HDNI inline void copy_words(void* dst, const void* src, size_t nbytes, int tid, int nthr) {
  unsigned long long* d = (unsigned long long*)dst;
  const unsigned long long* s = (const unsigned long long*)src;
  for (int w = tid; w < (int)(nbytes / 8); w += nthr) d[w] = s[w];
}

// Controller kernel body, one block per running slot: reduce the partials
// of the work kernel that just ran (in a fixed order, independent of block
// scheduling) and advance the slot's NTN state machine.  kid = K_VEC after the
// vector kernel, K_X5 after pass 5.  The block copies the controller record
// into shared memory with all its threads; the one thread that runs the
// state machine reads and writes only the fields it needs there, and the
// block writes the record back.
HDNI inline void ctl_block(SlotDev* slots, Ctl* ctls, const Task* tasks, int kid, int bid, int tid, int nthr,
                           char* smem) {
  const int si = tasks[bid].slot;
  SlotDev& s = slots[si];
  Ctl& c = ctls[si];
  if (c.status != ST_RUNNING) return;
  const int what = kid == K_VEC ? c.op : c.ev;
  if (what == 0) return;
  double* sred = (double*)smem;
  Ctl* cs = (Ctl*)(smem + CTL_SRED_BYTES);
  copy_words(cs, &c, sizeof(Ctl), tid, nthr);
  const CtlSlot sl = ctl_slot(s);
  const int nt = s.ntask[kid];
  double part[NCH];
#pragma unroll
  for (int ch = 0; ch < NCH; ++ch) part[ch] = 0.0;
  for (int t = tid; t < nt; t += nthr) {
#pragma unroll
    for (int ch = 0; ch < NCH; ++ch) part[ch] += s.partials[(size_t)t * NCH + ch];
  }
  block_reduce(sred, part, tid, nthr);  // its barriers also publish the copy
  if (tid == 0) {
    double red[NCH];
#pragma unroll
    for (int ch = 0; ch < NCH; ++ch) red[ch] = sred[ch];
    ntn_after(*cs, sl, red, kid, what);
  }
  BLOCK_SYNC();
  copy_words(&c, cs, sizeof(Ctl), tid, nthr);
}

// ------------------------------------------------------------ vector ops
// 16-byte packs (4 floats or 2 doubles): the vector operations stream their
// arrays with one 16-byte load or store per pack and array.
template <typename T> struct Pack { static constexpr int n = 16 / (int)sizeof(T); };
template <typename T>
HD void ld_pack(T* v, const T* p) {
#if defined(__CUDA_ARCH__)
  if constexpr (sizeof(T) == 4) {
    const float4 x = *(const float4*)p;
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
  } else {
    const double2 x = *(const double2*)p;
    v[0] = x.x; v[1] = x.y;
  }
#else
  for (int l = 0; l < Pack<T>::n; ++l) v[l] = p[l];
#endif
}
template <typename T>
HD void st_pack(T* p, const T* v) {
#if defined(__CUDA_ARCH__)
  if constexpr (sizeof(T) == 4) *(float4*)p = make_float4(v[0], v[1], v[2], v[3]);
  else *(double2*)p = make_double2(v[0], v[1]);
#else
  for (int l = 0; l < Pack<T>::n; ++l) p[l] = v[l];
#endif
}

// One task of a vector operation over points [i0, i1) of a slot: packs of
// Pack<T>::n points first (i0 is a multiple of the chunk size, so packs are
// 16-byte aligned), then the points after the last full pack one at a time.
template <typename T>
HD void vec_block(const Args<T>& a, int bid, int tid, int nthr, char* smem) {
  const Task t = a.tasks[bid];
  SlotDev& s = a.slots[t.slot];
  Ctl& c = a.ctl[t.slot];
  const int op = c.op;
  if (c.status != ST_RUNNING || op == OP_NONE) return;
  T* __restrict__ phi = (T*)s.buf[c.iphi];
  const T* __restrict__ w0 = (const T*)s.buf[c.iw0];
  const T* __restrict__ w1 = (const T*)s.buf[c.iw1];
  T* __restrict__ bb = (T*)s.buf[B_B];
  T* __restrict__ r = (T*)s.buf[B_R];
  T* __restrict__ p = (T*)s.buf[B_P];
  T* __restrict__ d = (T*)s.buf[B_D];
  const T k = (T)c.opc;
  const int i0 = t.a * a.vchunk;
  const int n = (int)s.N;
  const int i1 = i0 + a.vchunk < n ? i0 + a.vchunk : n;
  constexpr int VP = Pack<T>::n;
  const int npk = (i1 - i0) / VP;  // full packs
  const int it = i0 + npk * VP;    // first point after them
  double acc[NCH];
#pragma unroll
  for (int ch = 0; ch < NCH; ++ch) acc[ch] = 0.0;
  switch (op) {
    case OP_SQRT_INIT:
      for (int q = tid; q < npk; q += nthr) {
        const int i = i0 + q * VP;
        T v[VP];
        ld_pack(v, phi + i);
#pragma unroll
        for (int l = 0; l < VP; ++l) {
          acc[0] += (double)v[l];
          v[l] = m_sqrt(v[l] < T(0) ? -v[l] : v[l]);
        }
        st_pack(phi + i, v);
      }
      for (int i = it + tid; i < i1; i += nthr) {
        const T rho = phi[i];
        acc[0] += (double)rho;
        phi[i] = m_sqrt(rho < T(0) ? -rho : rho);
      }
      break;
    case OP_DLDPHI:
      for (int q = tid; q < npk; q += nthr) {
        const int i = i0 + q * VP;
        T wv[VP], fv[VP], bv[VP], rv[VP], zv[VP];
        ld_pack(wv, w0 + i);
        ld_pack(fv, phi + i);
#pragma unroll
        for (int l = 0; l < VP; ++l) {
          const T v = wv[l] - k * T(2) * fv[l];
          bv[l] = v;
          rv[l] = -v;
          zv[l] = T(0);
          acc[0] += (double)v * (double)v;
        }
        st_pack(bb + i, bv);
        st_pack(r + i, rv);
        st_pack(p + i, rv);
        st_pack(d + i, zv);
      }
      for (int i = it + tid; i < i1; i += nthr) {
        const T v = w0[i] - k * T(2) * phi[i];
        bb[i] = v;
        r[i] = -v;
        p[i] = -v;
        d[i] = T(0);
        acc[0] += (double)v * (double)v;
      }
      break;
    case OP_CGSTEP:
      for (int q = tid; q < npk; q += nthr) {
        const int i = i0 + q * VP;
        T dv[VP], pv[VP], rv[VP], wv[VP], fv[VP];
        ld_pack(dv, d + i);
        ld_pack(pv, p + i);
        ld_pack(rv, r + i);
        ld_pack(wv, w1 + i);
        ld_pack(fv, phi + i);
#pragma unroll
        for (int l = 0; l < VP; ++l) {
          const T dn = dv[l] + k * pv[l];
          const T rn = rv[l] - k * wv[l];
          dv[l] = dn;
          rv[l] = rn;
          const T pd = fv[l] + dn;
          acc[0] += (double)rn * (double)rn;
          acc[1] += (double)pd * (double)pd;
          acc[2] += (double)fv[l] * (double)dn;
        }
        st_pack(d + i, dv);
        st_pack(r + i, rv);
      }
      for (int i = it + tid; i < i1; i += nthr) {
        const T dn = d[i] + k * p[i];
        const T rn = r[i] - k * w1[i];
        d[i] = dn;
        r[i] = rn;
        const T f = phi[i];
        const T pd = f + dn;
        acc[0] += (double)rn * (double)rn;
        acc[1] += (double)pd * (double)pd;
        acc[2] += (double)f * (double)dn;
      }
      break;
    case OP_PUPD:
      for (int q = tid; q < npk; q += nthr) {
        const int i = i0 + q * VP;
        T rv[VP], pv[VP];
        ld_pack(rv, r + i);
        ld_pack(pv, p + i);
#pragma unroll
        for (int l = 0; l < VP; ++l) {
          pv[l] = rv[l] + k * pv[l];
          acc[0] += (double)pv[l] * (double)pv[l];
        }
        st_pack(p + i, pv);
      }
      for (int i = it + tid; i < i1; i += nthr) {
        const T pn = r[i] + k * p[i];
        p[i] = pn;
        acc[0] += (double)pn * (double)pn;
      }
      break;
    case OP_DIRNEG:
    case OP_NG1:
    case OP_SD:
      for (int q = tid; q < npk; q += nthr) {
        const int i = i0 + q * VP;
        T dv[VP], fv[VP], xv[VP];
        if (op == OP_DIRNEG) {
          ld_pack(dv, d + i);
          ld_pack(xv, p + i);
        } else if (op == OP_SD) {
          ld_pack(xv, bb + i);
        } else {
          ld_pack(dv, d + i);
        }
        ld_pack(fv, phi + i);
#pragma unroll
        for (int l = 0; l < VP; ++l) {
          T dn;
          if (op == OP_DIRNEG) dn = -(dv[l] - k * xv[l]);
          else if (op == OP_SD) dn = -xv[l];
          else dn = dv[l];
          dv[l] = dn;
          const T pd = fv[l] + dn;
          acc[1] += (double)pd * (double)pd;
          acc[2] += (double)fv[l] * (double)dn;
        }
        if (op != OP_NG1) st_pack(d + i, dv);
      }
      for (int i = it + tid; i < i1; i += nthr) {
        T dn;
        if (op == OP_DIRNEG) dn = -(d[i] - k * p[i]);
        else if (op == OP_SD) dn = -bb[i];
        else dn = d[i];
        if (op != OP_NG1) d[i] = dn;
        const T f = phi[i];
        const T pd = f + dn;
        acc[1] += (double)pd * (double)pd;
        acc[2] += (double)f * (double)dn;
      }
      break;
    case OP_NG2:
      for (int q = tid; q < npk; q += nthr) {
        const int i = i0 + q * VP;
        T dv[VP], fv[VP], wv[VP];
        ld_pack(dv, d + i);
        ld_pack(fv, phi + i);
        ld_pack(wv, w0 + i);
#pragma unroll
        for (int l = 0; l < VP; ++l) {
          const T dn = dv[l] - fv[l] * k;
          dv[l] = dn;
          acc[0] += (double)dn * (double)dn;
          acc[1] += (double)wv[l] * (double)dn;
        }
        st_pack(d + i, dv);
      }
      for (int i = it + tid; i < i1; i += nthr) {
        const T dn = d[i] - phi[i] * k;
        d[i] = dn;
        acc[0] += (double)dn * (double)dn;
        acc[1] += (double)w0[i] * (double)dn;
      }
      break;
    default:
      break;
  }
  store_partials<0, 3>(s, t.a, acc, (double*)smem, tid, nthr);  // vector ops use channels 0-2
}

// ------------------------------------------------------------ evaluation inputs
// phi_in = ca * A + cb * B of the current evaluation (or rho itself for the
// drop-in evaluation), held in registers for a whole block.
template <typename T>
struct EvalIn {
  const T* __restrict__ A;
  const T* __restrict__ B;
  T ca, cb;
  int rho_mode;
  HD void at(int i, T& phin, T& rho, T& sq) const {
    if (rho_mode) {
      rho = A[i];
      sq = m_sqrt(rho);
      phin = sq;
    } else {
      phin = cb == T(0) ? ca * A[i] : ca * A[i] + cb * B[i];
      rho = phin * phin;
      sq = phin < T(0) ? -phin : phin;  // sqrt(rho) = |phi_in|
    }
  }
};

template <typename T>
HD EvalIn<T> eval_in(const SlotDev& s, const Ctl& c) {
  EvalIn<T> e;
  e.A = (const T*)s.buf[c.iphi];
  e.B = (const T*)s.buf[c.evb];
  e.ca = (T)c.ca;
  e.cb = (T)c.cb;
  e.rho_mode = (c.ev == EV_RHO || c.ev == EV_STRESS || (c.ev == EV_FORCE && c.force_rho)) ? 1 : 0;
  return e;
}

// Functional parameters of the real-space stages, in registers.
template <typename T>
struct FieldPar {
  int wt, pow56, aeqb, sum53;
  T alpha, beta, rho_s;
};

template <typename T>
HD FieldPar<T> field_par(const SlotDev& s) {
  FieldPar<T> f;
  f.wt = s.kinetic == KIN_WT;
  f.pow56 = s.pow56;
  f.aeqb = s.alpha_eq_beta;
  f.sum53 = (s.alpha + s.beta - 5.0 / 3.0) < 1e-14 && (s.alpha + s.beta - 5.0 / 3.0) > -1e-14;
  f.alpha = (T)s.alpha;
  f.beta = (T)s.beta;
  f.rho_s = (T)s.rho_s;
  return f;
}

// ------------------------------------------------------------ pass 1
// All forward fields of one point (WT: rho, rho^beta, sqrt(rho) and, when
// alpha != beta, rho^alpha; WGC: rho, sqrt(rho), then for x = alpha and
// x = beta: rho^x, theta rho^x, theta^2 rho^x / 2 with theta = rho - rho*),
// with each power computed once.
template <typename T, int KS>
HD void field_values(const FieldPar<T>& fp, int nf, T rho, T sq, T* v) {
  v[0] = rho;
  if constexpr (KS == KS_WT) {
    v[1] = fp.pow56 ? sq * m_cbrt(rho) : m_pow(rho, fp.beta);
    v[2] = sq;
    if (nf > 3) v[3] = m_pow(rho, fp.alpha);
    return;
  }
  v[1] = sq;
  const T th = rho - fp.rho_s;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const T rx = m_pow(rho, h == 0 ? fp.alpha : fp.beta);
    v[2 + 3 * h] = rx;
    v[3 + 3 * h] = th * rx;
    v[4 + 3 * h] = th * th * rx / T(2);
  }
}

// Every field of a range of row pairs in one block: the inputs of a point are
// read and its field values computed once, and the nf * nb x-transforms run
// as one batch, column f*nb + b, element i at buf[(f*nb + b) + i*NB].
template <typename T, int KS>
HD void xfwd_block(const Args<T>& a, int bid, int tid, int nthr, char* smem) {
  constexpr int NFM = KinFields<KS>::value;
  const Task t = a.tasks[bid];
  const SlotDev& s = a.slots[t.slot];
  const Ctl& c = a.ctl[t.slot];
  if (c.status != ST_RUNNING || c.ev == EV_NONE) return;
  const int rp0 = t.b, nb = t.c;
  const int ev = c.ev;
  const int nfe = ev == EV_ION ? s.ion.nspec : ev == EV_FORCE ? 1 : s.nf;
  const int NB = nfe * nb;
  const int n1 = s.n1, k1 = s.k1;
  const int nrows = s.n2 * s.n3;
  const long long Nc = s.Nc;
  EvalIn<T> in = eval_in<T>(s, c);
  const FieldPar<T> fp = field_par<T>(s);
  const FftPlan& px = s.px;
  cx<T>* buf = (cx<T>*)smem;
  // the task's rows of the evaluation inputs, staged with asynchronous copies
  // (local row r at [r*n1 + i])
  const int rows = nrows - 2 * rp0 < 2 * nb ? nrows - 2 * rp0 : 2 * nb;
  if (ev != EV_ION) {
    const size_t rbytes = (size_t)rows * n1 * sizeof(T), goff = (size_t)2 * rp0 * n1;
    T* sa = (T*)(smem + xfwd_stage_offset(n1, nfe, nb, sizeof(T)));
    T* sb = (T*)((char*)sa + align16((size_t)2 * nb * n1 * sizeof(T)));
    cp_async_block(sa, in.A + goff, rbytes, (int)sizeof(T), tid, nthr);
    if (!in.rho_mode && in.cb != T(0)) cp_async_block(sb, in.B + goff, rbytes, (int)sizeof(T), tid, nthr);
    in.A = sa;
    in.B = sb;
    cp_async_wait();
    BLOCK_SYNC();
  }
  const unsigned mn1 = magic32(n1);
  for (int w = tid; w < nb * n1; w += nthr) {
    const int b = magic_div32(w, mn1), i = w - b * n1;
    const int j0 = 2 * (rp0 + b), j1 = j0 + 1;
    const bool has1 = j1 < nrows;
    cx<T>* d = buf + b + i * NB;
    if (ev == EV_ION) {  // B-spline charge of each species (FillQIonTable)
      for (int f = 0; f < nfe; ++f) {
        const T* __restrict__ q = (const T*)s.buf[B_PHI + f];
        d[f * nb] = mk<T>(q[j0 * n1 + i], has1 ? q[j1 * n1 + i] : T(0));
      }
      continue;
    }
    T v0[NFM], v1[NFM];
    T phin, rho, sq;
    in.at(2 * b * n1 + i, phin, rho, sq);
    if (ev == EV_FORCE) v0[0] = rho;
    else field_values<T, KS>(fp, nfe, rho, sq, v0);
#pragma unroll
    for (int f = 0; f < NFM; ++f) v1[f] = T(0);
    if (has1) {
      in.at((2 * b + 1) * n1 + i, phin, rho, sq);
      if (ev == EV_FORCE) v1[0] = rho;
      else field_values<T, KS>(fp, nfe, rho, sq, v1);
    }
#pragma unroll
    for (int f = 0; f < NFM; ++f)
      if (f < nfe) d[f * nb] = mk<T>(v0[f], v1[f]);
  }
  BLOCK_SYNC();
  fft_inplace<T, -1>(buf, NB, 1, NB, px, a.tw, tid, nthr);
  // split the two real rows' spectra: Z = X[k], Zc = conj(X[n1 - k]) (read at
  // their digit-reversed positions); row j0 gets (Z + Zc) / 2, row j1
  // (Z - Zc) / 2i, stored kx-major (consecutive threads, consecutive row pairs)
  const int* __restrict__ ip = a.idx + px.iperm;
  const unsigned mnb = magic32(nb), mk1 = magic32(k1);
  for (int w = tid; w < NB * k1; w += nthr) {
    const int rest = magic_div32(w, mnb), b = w - rest * nb;
    const int f = magic_div32(rest, mk1), k = rest - f * k1;
    const int col = f * nb + b;
    const int j0 = 2 * (rp0 + b), j1 = j0 + 1;
    const cx<T> z = buf[col + ip[k] * NB];
    const cx<T> zc = conj(buf[col + ip[k == 0 ? 0 : n1 - k] * NB]);
    const cx<T> sum = z + zc, dif = z - zc;
    cx<T>* __restrict__ out = (cx<T>*)s.spec + (size_t)f * (size_t)Nc + (size_t)k * nrows;
    out[j0] = mk<T>(sum.x * T(0.5), sum.y * T(0.5));
    if (j1 < nrows) out[j1] = mk<T>(dif.y * T(0.5), -dif.x * T(0.5));
  }
}

// ------------------------------------------------------------ k-space operators
HD int signed_freq(int k, int n) { return k > n / 2 ? k - n : k; }

// Real factor of the single-field operators at the frequency (m1, m2, m3)
// (signed): Hartree 4 pi / |G|^2 (0 at G = 0) and vW |G|^2, each times the
// 1/N forward scale; |G|^2 in the slot's precision.
template <typename T>
struct GFactor {
  T rt[9];
  T sc, c4;
  HD void init(const SlotDev& s) {
#pragma unroll
    for (int q = 0; q < 9; ++q) rt[q] = (T)s.recip[q];
    sc = (T)s.inv_n;
    c4 = (T)(4.0 * PI_D * s.inv_n);
  }
  HD T operator()(int kind, int m1, int m2, int m3) const {
    const T tx = rt[0] * (T)m1 + rt[3] * (T)m2 + rt[6] * (T)m3;
    const T ty = rt[1] * (T)m1 + rt[4] * (T)m2 + rt[7] * (T)m3;
    const T tz = rt[2] * (T)m1 + rt[5] * (T)m2 + rt[8] * (T)m3;
    const T g2 = tx * tx + ty * ty + tz * tz;
    if (kind == G_VW) return g2 * sc;
    return (m1 == 0 && m2 == 0 && m3 == 0) ? T(0) : c4 / g2;
  }
};

// The operator of one z-pass tile: res[i*NB + q*nb + b] holds field q of
// the group at z position i (frequency kz = permz[i]) and y position y0 + b
// (ky = permy[y0 + b]), for kx; the results replace the inputs.
template <typename T, int KS>
HD void zpass_operator(const SlotDev& s, int kind, int gn, bool setup_mode, cx<T>* res, int NB, int nb, int kx,
                       int y0, const int* __restrict__ permy, const int* __restrict__ permz, int tid, int nthr) {
  const int n2 = s.n2, n3 = s.n3, nrows = n2 * n3;
  const long long Nc = s.Nc;
  const unsigned mnb = magic32(nb);
  const T* __restrict__ kern = (const T*)s.kern + (size_t)kx * nrows + y0;
  const T sc = (T)s.inv_n;
  GFactor<T> gf;
  gf.init(s);
  for (int w = tid; w < nb * n3; w += nthr) {
    const int i = magic_div32(w, mnb), b = w - i * nb;
    const int ky = permy[y0 + b], kz = permz[i];
    const int m2 = signed_freq(ky, n2), m3 = signed_freq(kz, n3);
    const int kidx = i * n2 + b;
    cx<T>* e = res + i * NB + b;
    if (kind == G_HARTREE || kind == G_VW) {
      e[0] = e[0] * gf(kind, kx, m2, m3);
      continue;
    }
    double q = 0.0;
    if (setup_mode) {
      const double gx = s.recip[0] * kx + s.recip[3] * m2 + s.recip[6] * m3;
      const double gy = s.recip[1] * kx + s.recip[4] * m2 + s.recip[7] * m3;
      const double gz = s.recip[2] * kx + s.recip[5] * m2 + s.recip[8] * m3;
      q = sqrt(gx * gx + gy * gy + gz * gz);
    }
    switch (kind) {
      case G_KMUL:
        e[0] = e[0] * (kern[kidx] * sc);
        break;
      case G_WGC3: {  // second-order WGC triple (KEDF_WGC.f90:219-236)
        if constexpr (KS == KS_WGC) {
          const T K1 = kern[kidx], K2 = kern[Nc + kidx], K3 = kern[2 * Nc + kidx], K4 = kern[3 * Nc + kidx];
          const cx<T> F0 = e[0], F1 = e[nb], F2 = e[2 * nb];
          e[0] = (F0 * K1 + F1 * K2 + F2 * K3) * sc;
          e[nb] = (F0 * K2 + F1 * K4) * sc;
          e[2 * nb] = F0 * (K3 * sc);
        }
        break;
      }
      case G_ION: {  // conj(sum_s V_s(|G|) b1 b2 b3 S_s) N / vol, times the 1/N forward scale
        // (IonElectronPotRecipSpline, IonElectronSpline.f90:180-203)
        const cx<double> bb = cmul(cmul(s.ion.b1[kx], s.ion.b2[ky]), s.ion.b3[kz]);
        double yr = 0.0, yi = 0.0;
        for (int sp = 0; sp < gn; ++sp) {
          const double v = psp_value(s.ion, sp, q);
          const cx<T> F = e[sp * nb];
          yr += v * (double)F.x;
          yi += v * (double)F.y;
        }
        const double pr = yr * bb.x - yi * bb.y, pim = yr * bb.y + yi * bb.x;
        e[0] = mk<T>((T)(pr / s.vol), (T)(-pim / s.vol));
        break;
      }
      default: {  // G_FORCE: rho(G) V_s(|G|) b1 b2 b3 per species, G = 0 excluded
        // (IonElectronForcesSpline, IonElectronSpline.f90:300-330)
        const cx<double> bb = cmul(cmul(s.ion.b1[kx], s.ion.b2[ky]), s.ion.b3[kz]);
        const cx<T> F = e[0];
        const bool g0 = kx == 0 && ky == 0 && kz == 0;
        for (int sp = gn - 1; sp >= 0; --sp) {
          const double v = g0 ? 0.0 : psp_value(s.ion, sp, q) * s.inv_n;
          const double fr = (double)F.x * v, fi = (double)F.y * v;
          e[sp * nb] = mk<T>((T)(fr * bb.x - fi * bb.y), (T)(fr * bb.y + fi * bb.x));
        }
        break;
      }
    }
  }
}

// Odd row pitch of a plane or tile held in shared memory with y fastest:
// transforms along y then take columns at an odd stride (conflict-free).
HD int odd_pitch(int n) { return n | 1; }

// ------------------------------------------------------------ Y passes (split path)
// Task (field f, kx, z tile): nz columns of n2 contiguous values (one per
// z), transformed along y in place: forward (dir < 0) natural -> digit
// reversed, inverse (dir > 0) back.
template <typename T>
HD void ypass_block(const Args<T>& a, int bid, int tid, int nthr, char* smem, int dir) {
  const Task t = a.tasks[bid];
  const SlotDev& s = a.slots[t.slot];
  const Ctl& c = a.ctl[t.slot];
  if (c.status != ST_RUNNING || c.ev == EV_NONE) return;
  const int f = t.a, kx = t.b, z0 = tile_first(t.c), nz = tile_width(t.c);
  if (c.ev == EV_ION && f >= (dir < 0 ? s.ion.nspec : 1)) return;
  if (c.ev == EV_FORCE && f >= (dir < 0 ? 1 : s.ion.nspec)) return;
  if (c.ev == EV_STRESS && dir > 0) return;  // forward spectra only
  const int n2 = s.n2, P = odd_pitch(n2);
  cx<T>* buf = (cx<T>*)smem;
  cx<T>* __restrict__ sp =
      (cx<T>*)s.spec + (size_t)f * (size_t)s.Nc + (size_t)kx * (n2 * s.n3) + (size_t)z0 * n2;
  const unsigned mn2 = magic32(n2);
  for (int w = tid; w < nz * n2; w += nthr) {
    const int zc = magic_div32(w, mn2), y = w - zc * n2;
    buf[zc * P + y] = sp[w];
  }
  BLOCK_SYNC();
  if (dir < 0) fft_inplace<T, -1>(buf, nz, P, 1, s.py, a.tw, tid, nthr);
  else fft_inplace<T, 1>(buf, nz, P, 1, s.py, a.tw, tid, nthr);
  for (int w = tid; w < nz * n2; w += nthr) {
    const int zc = magic_div32(w, mn2), y = w - zc * n2;
    sp[w] = buf[zc * P + y];
  }
}

// ------------------------------------------------------------ Z pass (split path)
// Task (group g, kx, y tile): the group's gn fields at ny consecutive y
// positions, all n3 z values, as gn*ny columns [z][q*ny + b]: forward FFT
// along z, the group's operator, inverse FFT along z.
template <typename T, int KS>
HD void zpass_block(const Args<T>& a, int bid, int tid, int nthr, char* smem) {
  const Task t = a.tasks[bid];
  const SlotDev& s = a.slots[t.slot];
  const Ctl& c = a.ctl[t.slot];
  if (c.status != ST_RUNNING || c.ev == EV_NONE) return;
  const int g = t.a, kx = t.b, y0 = tile_first(t.c), nb = tile_width(t.c);
  const int ev = c.ev;
  const bool setup_mode = ev == EV_ION || ev == EV_FORCE;
  if (setup_mode && g != 0) return;
  const int n2 = s.n2, n3 = s.n3, nrows = n2 * n3;
  const int kind = ev == EV_ION ? G_ION : ev == EV_FORCE ? G_FORCE : s.group_kind[g];
  const int gn = setup_mode ? s.ion.nspec : s.group_nf[g];
  const int gin = ev == EV_FORCE ? 1 : gn;  // fields loaded
  const int gout = ev == EV_ION ? 1 : gn;   // fields stored
  const int NB = gn * nb;
  const long long Nc = s.Nc;
  cx<T>* __restrict__ spec =
      (cx<T>*)s.spec + (size_t)(setup_mode ? 0 : s.group_f0[g]) * (size_t)Nc + (size_t)kx * nrows + y0;
  cx<T>* buf = (cx<T>*)smem;
  const unsigned mNB = magic32(NB), mnb = magic32(nb);
  for (int w = tid; w < NB * n3; w += nthr) {
    const int i = magic_div32(w, mNB), qb = w - i * NB;
    const int q = magic_div32(qb, mnb), b = qb - q * nb;
    buf[w] = q < gin ? spec[(size_t)q * Nc + i * n2 + b] : mk<T>(T(0), T(0));
  }
  BLOCK_SYNC();
  fft_inplace<T, -1>(buf, NB, 1, NB, s.pz, a.tw, tid, nthr);
  if (ev == EV_STRESS) {  // keep the forward spectra
    for (int w = tid; w < NB * n3; w += nthr) {
      const int i = magic_div32(w, mNB), qb = w - i * NB;
      const int q = magic_div32(qb, mnb), b = qb - q * nb;
      spec[(size_t)q * Nc + i * n2 + b] = buf[w];
    }
    return;
  }
  zpass_operator<T, KS>(s, kind, gn, setup_mode, buf, NB, nb, kx, y0, a.idx + s.py.perm, a.idx + s.pz.perm, tid,
                        nthr);
  BLOCK_SYNC();
  fft_inplace<T, 1>(buf, NB, 1, NB, s.pz, a.tw, tid, nthr);
  for (int w = tid; w < NB * n3; w += nthr) {
    const int i = magic_div32(w, mNB), qb = w - i * NB;
    const int q = magic_div32(qb, mnb), b = qb - q * nb;
    if (q < gout) spec[(size_t)q * Nc + i * n2 + b] = buf[w];
  }
}

// ------------------------------------------------------------ YZ pass (fused path)
// Accessors of the fused pass: the plane in global memory (y fastest, row
// length n2) and in shared memory (rows of odd pitch P); column c is y,
// position i is z.
template <typename T>
struct PlaneIO {
  cx<T>* p;
  int pitch;
  HD cx<T> ld(int y, int z) const { return p[z * pitch + y]; }
  HD void st(int y, int z, cx<T> v) const { p[z * pitch + y] = v; }
};

// Operator factors at (column z, y position q) of the fused pass: the WT
// kernel plane (stored in the transforms' digit-reversed order) times the
// 1/N forward scale, or the Hartree / vW factor of the frequencies there.
template <typename T>
struct KernOp {
  const T* __restrict__ kern;
  T sc;
  int n2;
  HD T operator()(int z, int q) const { return kern[z * n2 + q] * sc; }
};
template <typename T>
struct GOp {
  GFactor<T> gf;
  int kind, kx, n2, n3;
  const int* __restrict__ permy;
  const int* __restrict__ permz;
  HD T operator()(int z, int q) const {
    return gf(kind, kx, signed_freq(permy[q], n2), signed_freq(permz[z], n3));
  }
};

// The (y, z) planes at kx of the three fields of a WGC group in the spectra
// (field p at base + p*Nc), seen as 3*n2 columns c = p*n2 + y of n3
// positions z.
template <typename T>
struct Planes3IO {
  cx<T>* base;
  long long Nc;
  int n2;
  unsigned mn2;
  HD size_t at(int c, int z) const {
    const int p = magic_div32(c, mn2), y = c - p * n2;
    return (size_t)p * (size_t)Nc + (size_t)z * n2 + y;
  }
  HD cx<T> ld(int c, int z) const { return base[at(c, z)]; }
  HD void st(int c, int z, cx<T> v) const { base[at(c, z)] = v; }
};

// The last forward y stage (radix R, stride 1) of the three planes of a WGC
// group, the second-order WGC operator (the same sums as the split z pass:
// G_WGC3 in zpass_operator, KEDF_WGC.f90:219-236) and the first inverse y
// stage, in registers.  Plane p of column z starts at buf + z*cs + p*n2; the
// kernel planes K1..K4 of this kx are kern + j*Nc, indexed z*n2 + y.
template <typename T, int R>
HD void ip_stage_wgc3_r(cx<T>* __restrict__ buf, int n3, unsigned mn3, int cs, int n2,
                        const T* __restrict__ kern, long long Nc, T sc, int tid, int nthr) {
  const int total = (n2 / R) * n3;
  for (int w = tid; w < total; w += nthr) {
    const int blk = magic_div32(w, mn3), z = w - blk * n3;
    cx<T>* p0 = buf + z * cs + blk * R;
    cx<T> v0[R], v1[R], v2[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      v0[r] = p0[r];
      v1[r] = p0[n2 + r];
      v2[r] = p0[2 * n2 + r];
    }
    Dft<T, R, -1>::run(v0);
    Dft<T, R, -1>::run(v1);
    Dft<T, R, -1>::run(v2);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int kidx = z * n2 + blk * R + r;
      const T K1 = kern[kidx], K2 = kern[Nc + kidx], K3 = kern[2 * Nc + kidx], K4 = kern[3 * Nc + kidx];
      const cx<T> F0 = v0[r], F1 = v1[r], F2 = v2[r];
      v0[r] = (F0 * K1 + F1 * K2 + F2 * K3) * sc;
      v1[r] = (F0 * K2 + F1 * K4) * sc;
      v2[r] = F0 * (K3 * sc);
    }
    Dft<T, R, 1>::run(v0);
    Dft<T, R, 1>::run(v1);
    Dft<T, R, 1>::run(v2);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      p0[r] = v0[r];
      p0[n2 + r] = v1[r];
      p0[2 * n2 + r] = v2[r];
    }
  }
}

template <typename T>
HD void ip_stage_wgc3(cx<T>* buf, int n3, unsigned mn3, int cs, const FftPlan& py, const T* kern, long long Nc,
                      T sc, int tid, int nthr) {
  constexpr int RM = FftMaxRadix<T>::value;
  const int n2 = py.n;
#define OFDFT_W3_CASE(r)                                                                              \
  case r:                                                                                             \
    if constexpr (r <= RM) ip_stage_wgc3_r<T, r>(buf, n3, mn3, cs, n2, kern, Nc, sc, tid, nthr);     \
    break;
  switch (py.R[py.nst - 1]) {
    OFDFT_W3_CASE(2)
    OFDFT_W3_CASE(3)
    OFDFT_W3_CASE(4)
    OFDFT_W3_CASE(5)
    OFDFT_W3_CASE(6)
    OFDFT_W3_CASE(7)
    OFDFT_W3_CASE(8)
    OFDFT_W3_CASE(9)
    OFDFT_W3_CASE(10)
    OFDFT_W3_CASE(12)
    OFDFT_W3_CASE(14)
    OFDFT_W3_CASE(15)
    OFDFT_W3_CASE(16)
    default: break;
  }
#undef OFDFT_W3_CASE
}

// Task (WGC group g, kx): the three fields' (y, z) planes at kx together in
// shared memory, interleaved along y (field p, y, z at z*P3 + p*n2 + y, P3 =
// odd pitch of 3*n2), since the WGC operator mixes the three at each
// frequency.  The z transforms run over all 3*n2 columns at once, the y
// transforms plane by plane, and the last forward y stage, the operator and
// the first inverse y stage run in registers for the three planes together.
// As the single-field task, one read and one write of each plane in HBM.
template <typename T>
HD void yz_wgc3_block(const Args<T>& a, const SlotDev& s, int g, int kx, cx<T>* buf, int tid, int nthr) {
  const int n2 = s.n2, n3 = s.n3, nrows = n2 * n3, nc = 3 * n2, P3 = odd_pitch(nc);
  const long long Nc = s.Nc;
  const FftPlan& py = s.py;
  const FftPlan& pz = s.pz;
  const cx<T>* ry = a.tw + py.root;
  const cx<T>* rz = a.tw + pz.root;
  const unsigned mnc = magic32(nc), mn3 = magic32(n3);
  const Planes3IO<T> glob{(cx<T>*)s.spec + (size_t)s.group_f0[g] * (size_t)Nc + (size_t)kx * nrows, Nc, n2,
                          magic32(n2)};
  const PlaneIO<T> rows{buf, P3};
  ip_stage_acc<T, -1>(glob, rows, nc, mnc, pz, 0, rz, tid, nthr);
  BLOCK_SYNC();
  for (int st = 1; st < pz.nst; ++st) {
    ip_stage<T, -1>(buf, nc, mnc, 1, P3, pz, st, rz, tid, nthr);
    BLOCK_SYNC();
  }
  for (int st = 0; st < py.nst - 1; ++st) {
    for (int p = 0; p < 3; ++p) ip_stage<T, -1>(buf + p * n2, n3, mn3, P3, 1, py, st, ry, tid, nthr);
    BLOCK_SYNC();
  }
  ip_stage_wgc3<T>(buf, n3, mn3, P3, py, (const T*)s.kern + (size_t)kx * nrows, Nc, (T)s.inv_n, tid, nthr);
  BLOCK_SYNC();
  for (int st = py.nst - 2; st >= 0; --st) {
    for (int p = 0; p < 3; ++p) ip_stage<T, 1>(buf + p * n2, n3, mn3, P3, 1, py, st, ry, tid, nthr);
    BLOCK_SYNC();
  }
  for (int st = pz.nst - 1; st >= 1; --st) {
    ip_stage<T, 1>(buf, nc, mnc, 1, P3, pz, st, rz, tid, nthr);
    BLOCK_SYNC();
  }
  ip_stage_acc<T, 1>(rows, glob, nc, mnc, pz, 0, rz, tid, nthr);
}

// Task (group g, kx) of a single-field group: the whole (y, z) plane of the
// field at kx (n2*n3 contiguous values) in shared memory, rows of odd pitch
// P.  The forward FFT along z loads its first stage straight from the
// spectra (consecutive threads, consecutive y); then the forward FFT along y;
// its last stage, the operator and the first inverse stage run in registers
// in one pass; then the inverse along y and z, whose last stage stores
// straight to the spectra.  One read and one write of the plane in HBM.
// KS = KS_WGC also takes the three-field WGC groups (yz_wgc3_block); the WT
// instantiation carries none of their code.
template <typename T, int KS>
HD void yzpass_block(const Args<T>& a, int bid, int tid, int nthr, char* smem) {
  const Task t = a.tasks[bid];
  const SlotDev& s = a.slots[t.slot];
  const Ctl& c = a.ctl[t.slot];
  const int ev = c.ev;
  if (c.status != ST_RUNNING || ev == EV_NONE || ev == EV_ION || ev == EV_FORCE || ev == EV_STRESS) return;
  const int g = t.a, kx = t.b;
  if constexpr (KS == KS_WGC) {
    if (s.group_kind[g] == G_WGC3) {
      yz_wgc3_block<T>(a, s, g, kx, (cx<T>*)smem, tid, nthr);
      return;
    }
  }
  const int n2 = s.n2, n3 = s.n3, nrows = n2 * n3, P = odd_pitch(n2);
  const int kind = s.group_kind[g];
  cx<T>* plane = (cx<T>*)s.spec + (size_t)s.group_f0[g] * (size_t)s.Nc + (size_t)kx * nrows;
  cx<T>* buf = (cx<T>*)smem;
  const FftPlan& py = s.py;
  const FftPlan& pz = s.pz;
  const cx<T>* ry = a.tw + py.root;
  const cx<T>* rz = a.tw + pz.root;
  const unsigned mn2 = magic32(n2), mn3 = magic32(n3);
  const PlaneIO<T> glob{plane, n2}, rows{buf, P};
  ip_stage_acc<T, -1>(glob, rows, n2, mn2, pz, 0, rz, tid, nthr);
  BLOCK_SYNC();
  for (int st = 1; st < pz.nst; ++st) {
    ip_stage<T, -1>(buf, n2, mn2, 1, P, pz, st, rz, tid, nthr);
    BLOCK_SYNC();
  }
  for (int st = 0; st < py.nst - 1; ++st) {
    ip_stage<T, -1>(buf, n3, mn3, P, 1, py, st, ry, tid, nthr);
    BLOCK_SYNC();
  }
  if (kind == G_KMUL) {
    const KernOp<T> op{(const T*)s.kern + (size_t)kx * nrows, (T)s.inv_n, n2};
    ip_stage_op<T>(buf, n3, mn3, P, 1, py, op, tid, nthr);
  } else {
    GOp<T> op;
    op.gf.init(s);
    op.kind = kind;
    op.kx = kx;
    op.n2 = n2;
    op.n3 = n3;
    op.permy = a.idx + py.perm;
    op.permz = a.idx + pz.perm;
    ip_stage_op<T>(buf, n3, mn3, P, 1, py, op, tid, nthr);
  }
  BLOCK_SYNC();
  for (int st = py.nst - 2; st >= 0; --st) {
    ip_stage<T, 1>(buf, n3, mn3, P, 1, py, st, ry, tid, nthr);
    BLOCK_SYNC();
  }
  for (int st = pz.nst - 1; st >= 1; --st) {
    ip_stage<T, 1>(buf, n2, mn2, 1, P, pz, st, rz, tid, nthr);
    BLOCK_SYNC();
  }
  ip_stage_acc<T, 1>(rows, glob, n2, mn2, pz, 0, rz, tid, nthr);
}

// ------------------------------------------------------------ pass 5
// Perdew-Zunger LDA potential and energy density (XC_LDA.f90:51-310) from
// rho, r13 = rho^(1/3) and rs = cC / r13.
template <typename T>
HD void lda_point(T rho, T r13, T rs, T& vxc, T& exc) {
  const T cXp = T(-0.98474502184269641), cXe = T(-0.73855876638202234);
  if (rs < T(1)) {
    const T lr = m_log(rs);
    vxc = cXp * r13 + lr * (T(3.11e-2) + T(1.33333333333333333e-3) * rs) + T(-5.83666666666666666e-2) +
          T(-8.4e-3) * rs;
    exc = cXe * rho * r13 + rho * (lr * (T(3.11e-2) + T(2e-3) * rs) + T(-4.8e-2) + T(-1.16e-2) * rs);
  } else {
    const T sr = m_sqrt(rs);
    const T den = T(1) + T(1.0529) * sr + T(3.334e-1) * rs;
    const T iden = T(1) / den;
    vxc = cXp * r13 + (T(-1.423e-1) + T(-0.174798948333333333) * sr + T(-6.325709333333333333e-2) * rs) *
                          (iden * iden);
    exc = cXe * rho * r13 + rho * (T(-1.423e-1) * iden);
  }
}

// All nf fields of a row-pair range are transformed as one batch of nf*nb
// sequences laid out [i][f*nb + b]; then every point of the rows gets the
// real-space epilogue.
// Inputs of the real-space epilogue of pass 5 (one task).
template <typename T>
struct XinvEpi {
  EvalIn<T> in;
  FieldPar<T> fp;
  const T* vion;
  T* w0;
  T* w1;
  T* trial;
  const T* bb;
  const cx<T>* res;  // the c2r outputs, column f*nb + b, element i at res[i*NB + f*nb + b]
  int NB, nb, nf, n1, nrows, rp0;
  bool opt_sqrt;
  T lam, muv, al, be, cTF, mu0, ieps, st, ctd, ctf53;
};

// The epilogue of one point: its potential (stored to the mode's output
// arrays at idx) and its terms of the mode's sums, added to sums[] in the
// slot precision.  o[f] are the point's field outputs of the inverse
// transforms; vi, aa, bx, ex, ey its ion potential and optimiser inputs.
template <typename T, int KS, int EV, bool ENERGY>
HD void epi_point(const XinvEpi<T>& e, const T* o, T vi, T aa, T bx, T ex, T ey, int idx, T* sums) {
  constexpr bool RHO = EV == EV_RHO;  // the input is rho itself
  const FieldPar<T> fp = e.fp;
  const T cC = T(0.62035049089940009);
  T phin, rho, sq;
  if (RHO) {
    rho = aa;
    sq = m_sqrt(rho);
    phin = sq;
  } else {
    phin = e.in.ca * aa + e.in.cb * bx;
    rho = phin * phin;
    sq = phin < T(0) ? -phin : phin;
  }
  const T x = m_rcbrt(rho);        // rho^(-1/3)
  const T r13 = rho * x * x;       // rho^(1/3)
  const T r23 = r13 * r13;
  const T rinv = x * x * x;        // 1/rho
  T vxc, exc;
  lda_point(rho, r13, cC * x, vxc, exc);
  T vnl, enl, lap;
  const T al = e.al, be = e.be, cTF = e.cTF;
  if constexpr (KS == KS_WT) {
    const T rbeta = fp.pow56 ? sq * r13 : m_pow(rho, be);
    const T ralpha = fp.aeqb ? rbeta : m_pow(rho, al);
    const T pa = e.nf > 3 ? o[3] : o[1];
    vnl = cTF * (al * (ralpha * rinv) * o[1] + be * (rbeta * rinv) * pa);
    enl = cTF * ralpha * o[1];
    lap = o[2];
  } else {
    const T th = rho - fp.rho_s;
    const T ralpha = m_pow(rho, al);
    const T rbeta = fp.sum53 ? rho * r23 / ralpha : m_pow(rho, be);
    vnl = cTF * ((rbeta * rinv) * (be * o[2] + (rho + be * th) * o[3] + th * (rho + be * th * T(0.5)) * o[4]) +
                 (ralpha * rinv) * (al * o[5] + (rho + al * th) * o[6] + th * (rho + al * th * T(0.5)) * o[7]));
    enl = cTF * rbeta * (o[2] + th * o[3] + th * th * T(0.5) * o[4]);
    lap = o[1];
  }
  const T potr = vi + o[0] + vxc + e.ctf53 * r23 + vnl;
  const T muv = e.muv;
  const T pot = e.opt_sqrt ? T(2) * sq * potr + muv * lap : potr + muv * lap * (T(0.5) * sq * rinv);
  if constexpr (ENERGY) {
    sums[CH_EIE] += rho * vi;
    sums[CH_EH] += T(0.5) * o[0] * rho;
    sums[CH_EXC] += exc;
    sums[CH_ETF] += e.lam * cTF * (rho * r23);
    sums[CH_EVW] += T(0.5) * muv * sq * lap;
    sums[CH_ENL] += enl;
  }
  const T sg = phin < T(0) ? T(-1) : T(1);
  if constexpr (EV == EV_RHO) {
    e.w0[idx] = pot;
  } else if constexpr (EV == EV_PHI) {
    const T gg = pot * sg;
    e.w0[idx] = gg;
    sums[CH_M0] += gg * phin;
    sums[CH_M1] += phin * phin;
  } else if constexpr (EV == EV_CG) {
    const T gg = pot * sg;
    const T ap = ((gg - e.mu0 * T(2) * phin) - ex) * e.ieps;
    e.w1[idx] = ap;
    sums[CH_M0] += ey * ap;
  } else {  // EV_LS
    const T gg = pot * sg;
    e.w1[idx] = gg;
    e.trial[idx] = phin;
    const T dir = -ex * e.st + ey * e.ctd;
    const T dl = gg - T(2) * phin * e.mu0;
    sums[CH_M0] += gg * dir;
    sums[CH_M1] += dl * dl;
    sums[CH_M2] += gg * phin;
    sums[CH_M3] += phin * phin;
  }
}

// The epilogue over every point of the task, compiled per evaluation mode EV
// (ENERGY: the six energy channels are summed), so that each loop keeps only
// its own inputs and accumulators live.  A work item is one complex output
// of the inverse transforms: x index i of row pair b, whose real and
// imaginary parts are the two rows' points (consecutive threads take
// consecutive i, so every global access is coalesced).  The two points'
// terms are added in the slot precision, then accumulated in FP64; the sums
// go to acc_out[NCH].
template <typename T, int KS, int EV, bool ENERGY>
HD void xinv_points(const XinvEpi<T>& e, double* acc_out, int tid, int nthr) {
  constexpr int NFM = KinFields<KS>::value;
  const T* __restrict__ vion = e.vion;
  const T* __restrict__ A = e.in.A;
  const T* __restrict__ B = e.in.B;
  const T* __restrict__ bb = e.bb;
  const int NB = e.NB, nb = e.nb, nf = e.nf, n1 = e.n1, nrows = e.nrows, rp0 = e.rp0;
  double acc[NCH];
#pragma unroll
  for (int ch = 0; ch < NCH; ++ch) acc[ch] = 0.0;
  const unsigned mn1 = magic32(n1);
  for (int w = tid; w < nb * n1; w += nthr) {
    const int b = magic_div32(w, mn1), i = w - b * n1;
    const int j0 = 2 * (rp0 + b);
    const bool has1 = j0 + 1 < nrows;
    const int idx0 = j0 * n1 + i, idx1 = has1 ? idx0 + n1 : idx0;
    // every global load of both points first
    const T vi0 = vion[idx0], vi1 = vion[idx1];
    const T aa0 = A[idx0], aa1 = A[idx1];
    // the second input (p in CG evaluations, d in line searches; the first
    // evaluation of a solve has none: its coefficient is 0)
    constexpr bool HASB = EV == EV_CG || EV == EV_LS;
    const T bx0 = HASB ? B[idx0] : T(0), bx1 = HASB ? B[idx1] : T(0);
    // the CG evaluation's second input is p, the line search's are phi and d
    const T ex0 = EV == EV_CG ? bb[idx0] : EV == EV_LS ? aa0 : T(0);
    const T ex1 = EV == EV_CG ? bb[idx1] : EV == EV_LS ? aa1 : T(0);
    T o0[NFM], o1[NFM];
    const cx<T>* rv = e.res + i * NB + b;
#pragma unroll
    for (int f = 0; f < NFM; ++f) {
      const cx<T> z = f < nf ? rv[f * nb] : mk<T>(T(0), T(0));
      o0[f] = z.x;
      o1[f] = z.y;
    }
    T sums[NCH];
#pragma unroll
    for (int ch = 0; ch < NCH; ++ch) sums[ch] = T(0);
    epi_point<T, KS, EV, ENERGY>(e, o0, vi0, aa0, bx0, ex0, bx0, idx0, sums);
    if (has1) epi_point<T, KS, EV, ENERGY>(e, o1, vi1, aa1, bx1, ex1, bx1, idx1, sums);
#pragma unroll
    for (int ch = 0; ch < NCH; ++ch) acc[ch] += (double)sums[ch];
  }
#pragma unroll
  for (int ch = 0; ch < NCH; ++ch) acc_out[ch] = acc[ch];
}

template <typename T, int KS>
HD void xinv_block(const Args<T>& a, int bid, int tid, int nthr, char* smem) {
  const Task t = a.tasks[bid];
  SlotDev& s = a.slots[t.slot];
  Ctl& c = a.ctl[t.slot];
  const int ev = c.ev;
  if (c.status != ST_RUNNING || ev == EV_NONE) return;
  const int rp0 = t.a, nb = t.b, ordinal = t.c;
  const bool setup_mode = ev == EV_ION || ev == EV_FORCE;
  const int n1 = s.n1, k1 = s.k1;
  const int nf = ev == EV_ION ? 1 : ev == EV_FORCE ? s.ion.nspec : s.nf;
  const int NB = nf * nb;
  const int nrows = s.n2 * s.n3;
  const long long Nc = s.Nc;
  const cx<T>* __restrict__ spec = (const cx<T>*)s.spec;
  cx<T>* buf = (cx<T>*)smem;
  if (ev == EV_STRESS) {  // the spectra stay; no sums
    double zero[NCH];
#pragma unroll
    for (int ch = 0; ch < NCH; ++ch) zero[ch] = 0.0;
    store_partials<0, 0>(s, ordinal, zero, (double*)(buf + NB * n1), tid, nthr);
    return;
  }
  const int nyq = (n1 % 2) == 0 ? n1 / 2 : -1;
  // gather: consecutive threads read the consecutive row pairs of one kx
  // (kx-major spectra); the packed complex sequence Z = A + i B of the two
  // rows' spectra goes to the digit-reversed positions the inverse
  // transform takes, Z[k] from the stored k < k1 and Z[n1 - k] from its
  // conjugate symmetry
  const int* __restrict__ ip = a.idx + s.px.iperm;
  const unsigned mnb = magic32(nb), mk1 = magic32(k1);
  for (int w = tid; w < NB * k1; w += nthr) {
    const int rest = magic_div32(w, mnb), b = w - rest * nb;
    const int f = magic_div32(rest, mk1), k = rest - f * k1;
    const cx<T>* sp = spec + (size_t)f * Nc + (size_t)k * nrows;
    const int j0 = 2 * (rp0 + b), j1 = j0 + 1;
    cx<T> A = sp[j0];
    cx<T> B = j1 < nrows ? sp[j1] : mk<T>(T(0), T(0));
    const int col = f * nb + b;
    if (k == 0 || k == nyq) {  // c2r ignores these imaginary parts
      buf[ip[k] * NB + col] = mk<T>(A.x, B.x);
    } else {
      buf[ip[k] * NB + col] = mk<T>(A.x - B.y, A.y + B.x);
      buf[ip[n1 - k] * NB + col] = mk<T>(A.x + B.y, B.x - A.y);
    }
  }
  BLOCK_SYNC();
  fft_inplace<T, 1>(buf, NB, 1, NB, s.px, a.tw, tid, nthr);
  const cx<T>* res = buf;
  if (setup_mode) {
    // EV_ION: ionPotReal; EV_FORCE: the per-species Factor arrays in buf[B_B + s]
    const unsigned m2n1s = magic32(2 * n1);
    for (int w = tid; w < nb * 2 * n1; w += nthr) {
      const int b = magic_div32(w, m2n1s), rem = w - b * 2 * n1;
      const int half = rem >= n1 ? 1 : 0, i = rem - half * n1;
      const int j = 2 * (rp0 + b) + half;
      if (j >= nrows) continue;
      for (int f = 0; f < nf; ++f) {
        const cx<T> z = res[i * NB + f * nb + b];
        T* dst = ev == EV_ION ? (T*)s.vion : (T*)s.buf[B_B + f];
        dst[j * n1 + i] = half == 0 ? z.x : z.y;
      }
    }
    double zero[NCH];
#pragma unroll
    for (int ch = 0; ch < NCH; ++ch) zero[ch] = 0.0;
    store_partials<0, 0>(s, ordinal, zero, (double*)(buf + NB * n1), tid, nthr);
    return;
  }

  XinvEpi<T> e;
  e.in = eval_in<T>(s, c);
  e.fp = field_par<T>(s);
  e.vion = (const T*)s.vion;
  e.w0 = (T*)s.buf[c.iw0];
  e.w1 = (T*)s.buf[c.iw1];
  e.trial = (T*)s.buf[c.itrial];
  e.bb = (const T*)s.buf[B_B];
  e.res = res;
  e.NB = NB;
  e.nb = nb;
  e.nf = nf;
  e.n1 = n1;
  e.nrows = nrows;
  e.rp0 = rp0;
  e.opt_sqrt = c.opt_sqrt != 0 || ev != EV_RHO;
  e.lam = (T)s.lambda;
  e.muv = (T)s.mu;
  e.al = e.fp.alpha;
  e.be = e.fp.beta;
  e.cTF = (T)C_TF;
  e.mu0 = (T)c.mu;
  e.ieps = (T)(ev == EV_CG ? 1.0 / c.eps : 0.0);
  e.st = (T)c.st;
  e.ctd = (T)(c.ct * c.dscale);
  e.ctf53 = T(5) / T(3) * e.cTF * e.lam;
  double acc[NCH];
  switch (ev) {
    case EV_CG:
      xinv_points<T, KS, EV_CG, false>(e, acc, tid, nthr);
      break;
    case EV_LS:
      xinv_points<T, KS, EV_LS, true>(e, acc, tid, nthr);
      break;
    case EV_PHI:
      xinv_points<T, KS, EV_PHI, true>(e, acc, tid, nthr);
      break;
    default:
      if (c.want_energy) xinv_points<T, KS, EV_RHO, true>(e, acc, tid, nthr);
      else xinv_points<T, KS, EV_RHO, false>(e, acc, tid, nthr);
      break;
  }
  if (ev == EV_CG) store_partials<CH_M0, CH_M0 + 1>(s, ordinal, acc, (double*)(buf + NB * n1), tid, nthr);
  else store_partials(s, ordinal, acc, (double*)(buf + NB * n1), tid, nthr);
}

}  // namespace ofdft
