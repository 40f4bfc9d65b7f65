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

}  // namespace ofdft
