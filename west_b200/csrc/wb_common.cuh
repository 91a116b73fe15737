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

WB_DEV double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
WB_DEV double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
WB_DEV double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
WB_DEV double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
WB_DEV double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
// multiply by (i * sign), sign = +1 or -1
template <int S>
WB_DEV double2 cmul_i(double2 a) {
  return S > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}
// twiddle with direction: DIR = +1 uses w, DIR = -1 uses conj(w)
template <int DIR>
WB_DEV double2 ctw(double2 a, double2 w) {
  if (DIR > 0) return cmul(a, w);
  return make_double2(fma(a.x, w.x, a.y * w.y), fma(a.y, w.x, -a.x * w.y));
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
