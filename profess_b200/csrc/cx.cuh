// Basic device helpers shared by all kernels of the density-solve engine.
//
// Every kernel body is written as a "block function": a __host__ __device__
// function that receives the block index, the thread index and the block size
// explicitly and synchronises only through BLOCK_SYNC().  On the device it runs
// inside a __global__ wrapper; in the host-emulation build (OFDFT_EMU, a test
// harness) the same body runs once per block with a single thread, so the block
// function must do all per-thread work in strided loops and keep no per-thread
// register state across a BLOCK_SYNC().
#pragma once
#include <cstdint>
#include <cmath>
#include <cstring>

#if defined(__CUDACC__)
#define HD __host__ __device__ __forceinline__
#define HDNI __host__ __device__
#define HDC __host__ __device__ constexpr
#else
#define HD inline
#define HDNI
#define HDC constexpr
#endif

#if defined(__CUDA_ARCH__)
#define BLOCK_SYNC() __syncthreads()
#else
#define BLOCK_SYNC() ((void)0)
#endif

namespace ofdft {

template <typename T>
struct alignas(2 * sizeof(T)) cx {
  T x, y;
};

template <typename T> HD cx<T> mk(T a, T b) { cx<T> r; r.x = a; r.y = b; return r; }
template <typename T> HD cx<T> operator+(cx<T> a, cx<T> b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <typename T> HD cx<T> operator-(cx<T> a, cx<T> b) { return mk<T>(a.x - b.x, a.y - b.y); }
template <typename T> HD cx<T> operator*(cx<T> a, T s) { return mk<T>(a.x * s, a.y * s); }
template <typename T> HD cx<T> cmul(cx<T> a, cx<T> b) {
  return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T> HD cx<T> conj(cx<T> a) { return mk<T>(a.x, -a.y); }
// multiply by dir * i  (dir = +1 or -1)
template <typename T> HD cx<T> mul_i(cx<T> a, int dir) {
  return dir > 0 ? mk<T>(-a.y, a.x) : mk<T>(a.y, -a.x);
}

// Precision-generic math wrappers (float versions map to the float library calls).
HD double m_sqrt(double v) { return sqrt(v); }
HD float m_sqrt(float v) { return sqrtf(v); }
HD double m_cbrt(double v) { return cbrt(v); }
HD float m_cbrt(float v) { return cbrtf(v); }
HD double m_pow(double a, double b) { return pow(a, b); }
HD float m_pow(float a, float b) { return powf(a, b); }
HD double m_log(double v) { return log(v); }
HD float m_log(float v) { return logf(v); }
#if defined(__CUDA_ARCH__)
HD double m_rcbrt(double v) { return rcbrt(v); }
HD float m_rcbrt(float v) { return rcbrtf(v); }
HD double m_rsqrt(double v) { return rsqrt(v); }
HD float m_rsqrt(float v) { return rsqrtf(v); }
#else
HD double m_rcbrt(double v) { return 1.0 / cbrt(v); }
HD float m_rcbrt(float v) { return 1.0f / cbrtf(v); }
HD double m_rsqrt(double v) { return 1.0 / sqrt(v); }
HD float m_rsqrt(float v) { return 1.0f / sqrtf(v); }
#endif

// ------------------------------------------------------------ async staging
// Asynchronous global -> shared copies (cp.async) of n bytes by the threads of
// a block: 16-byte copies when both addresses are 16-byte aligned and n is a
// multiple of 16, else copies of the element size (4 or 8 bytes, which must
// divide both addresses and n).  They put a block's input rows in flight at
// once instead of one dependent load per work item.  cp_async_wait() waits
// for the calling thread's copies; a block barrier after it makes every
// thread's copies visible.  The host emulation copies at once.
HD void cp_async_block(void* dst, const void* src, size_t n, int elem, int tid, int nthr) {
#if defined(__CUDA_ARCH__)
  const unsigned sdst = (unsigned)__cvta_generic_to_shared(dst);
  const char* g = (const char*)src;
  if (((((size_t)g) | sdst | n) & 15) == 0) {
    for (size_t o = (size_t)tid * 16; o < n; o += (size_t)nthr * 16)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sdst + (unsigned)o), "l"(g + o) : "memory");
  } else if (elem == 8) {
    for (size_t o = (size_t)tid * 8; o < n; o += (size_t)nthr * 8)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sdst + (unsigned)o), "l"(g + o) : "memory");
  } else {
    for (size_t o = (size_t)tid * 4; o < n; o += (size_t)nthr * 4)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sdst + (unsigned)o), "l"(g + o) : "memory");
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
#else
  (void)elem;
  (void)nthr;
  if (tid == 0) memcpy(dst, src, n);
#endif
}

// One asynchronous copy of U = 4, 8 or 16 bytes (both addresses U-aligned);
// cp_async_commit() closes the calling thread's group of copies.
template <int U>
HD void cp_async_unit(void* dst, const void* src) {
#if defined(__CUDA_ARCH__)
  const unsigned sdst = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (U == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sdst), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sdst), "l"(src), "n"(U) : "memory");
#else
  memcpy(dst, src, U);
#endif
}

HD void cp_async_commit() {
#if defined(__CUDA_ARCH__)
  asm volatile("cp.async.commit_group;\n" ::: "memory");
#endif
}

HD void cp_async_wait() {
#if defined(__CUDA_ARCH__)
  asm volatile("cp.async.wait_all;\n" ::: "memory");
#endif
}

}  // namespace ofdft
