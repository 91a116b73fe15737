// Common device helpers for the west_b200 response-operator kernels.
//
// Complex numbers are double2 (x = real, y = imaginary), the layout of
// Fortran COMPLEX(DP), so host arrays from WEST map onto device arrays
// without repacking.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define WB_DEV __device__ __forceinline__

namespace wb {

// Complex helpers for double2 (FP64) and float2 (FP32 inner solves).
template <class C> struct RealOf;
template <> struct RealOf<double2> { using type = double; };
template <> struct RealOf<float2> { using type = float; };
template <class C> using real_t = typename RealOf<C>::type;

template <class C> WB_DEV C mkc(real_t<C> x, real_t<C> y);
template <> WB_DEV double2 mkc<double2>(double x, double y) { return make_double2(x, y); }
template <> WB_DEV float2 mkc<float2>(float x, float y) { return make_float2(x, y); }

template <class C> WB_DEV C cadd(C a, C b) { return mkc<C>(a.x + b.x, a.y + b.y); }
template <class C> WB_DEV C csub(C a, C b) { return mkc<C>(a.x - b.x, a.y - b.y); }
// FP32 complex add and subtract as one paired instruction (sm_100 f32x2; same
// rounding as two scalar adds)
WB_DEV unsigned long long f2_bits(float2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
WB_DEV float2 bits_f2(unsigned long long r) {
  float2 a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
template <> WB_DEV float2 cadd<float2>(float2 a, float2 b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return bits_f2(r);
}
template <> WB_DEV float2 csub<float2>(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return bits_f2(r);
}
template <class C> WB_DEV C cmul(C a, C b) {
  return mkc<C>(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
template <class C> WB_DEV C cscale(C a, real_t<C> s) { return mkc<C>(a.x * s, a.y * s); }
template <class C> WB_DEV C cconj(C a) { return mkc<C>(a.x, -a.y); }
// multiply by (i * sign), sign = +1 or -1
template <int S, class C>
WB_DEV C cmul_i(C a) {
  return S > 0 ? mkc<C>(-a.y, a.x) : mkc<C>(a.y, -a.x);
}
// twiddle with direction: DIR = +1 uses w, DIR = -1 uses conj(w)
template <int DIR, class C>
WB_DEV C ctw(C a, C w) {
  if (DIR > 0) return cmul(a, w);
  return mkc<C>(fma(a.x, w.x, a.y * w.y), fma(a.y, w.x, -a.x * w.y));
}

// Work units of a launch: the host count, or, when dn is given (launches
// replayed from a CUDA graph), the count an earlier kernel left in device
// memory; PAIRS rounds half of it up (two bands per Gamma FFT).
template <bool PAIRS = false>
WB_DEV int dev_count(const int* dn, int host) {
  if (!dn) return host;
  const int n = *dn;
  return PAIRS ? (n + 1) / 2 : n;
}

// Block-wide sum of one double per thread; result valid in every thread.
template <int NT>
WB_DEV double block_sum(double v, double* red /* >= NT/32 doubles */) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < NT / 32; ++i) s += red[i];
  return s;
}

// Two sums at once.
template <int NT>
WB_DEV double2 block_sum2(double a, double b, double* red /* >= NT/16 doubles */) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) { red[2 * w] = a; red[2 * w + 1] = b; }
  __syncthreads();
  double sa = 0.0, sb = 0.0;
#pragma unroll
  for (int i = 0; i < NT / 32; ++i) { sa += red[2 * i]; sb += red[2 * i + 1]; }
  return make_double2(sa, sb);
}

}  // namespace wb
