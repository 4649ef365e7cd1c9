// Shared device helpers for the vFLIP B200 kernels.
//
// Layout: every grid is a dense linear array, index = i + ni*(j + nj*k)
// (i fastest), the same order the reference uses for its pressure vector
// (Smoke_Solver/Smoke_solver3D.cpp:993).  A level's 7-point operator is
// symmetric and stored as four arrays: diag, xp, yp, zp (the +x/+y/+z
// couplings); the -x coupling of cell c is xp[c-1], and so on.
//
// The library is compiled with -fmad=false: every a*b+c is rounded twice, as
// the reference's x86-64 build does, so kernels that follow the reference's
// order of operations reproduce its FP64/FP32 results bit for bit.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#define VFLIP_HD __host__ __device__ __forceinline__

namespace vflip {

constexpr int kWarp = 32;

VFLIP_HD size_t lin3(int i, int j, int k, int ni, int nj) {
  return (size_t)i + (size_t)ni * ((size_t)j + (size_t)nj * (size_t)k);
}

// Storage-type conversions: stencils and vectors may be stored as double,
// float or bf16 (coarse levels of the mixed-precision mode); arithmetic uses
// Acc (double for the FP64 path, float otherwise).
template <typename T> struct Num;
template <> struct Num<double> {
  using Acc = double;
  static __device__ __forceinline__ double ld(const double* p) { return __ldg(p); }
  static __device__ __forceinline__ double ldv(const double* p) { return *p; }
  static __device__ __forceinline__ double to(double v) { return v; }
};
template <> struct Num<float> {
  using Acc = float;
  static __device__ __forceinline__ float ld(const float* p) { return __ldg(p); }
  static __device__ __forceinline__ float ldv(const float* p) { return *p; }
  static __device__ __forceinline__ float to(float v) { return v; }
};
template <> struct Num<__nv_bfloat16> {
  using Acc = float;
  static __device__ __forceinline__ float ld(const __nv_bfloat16* p) { return __bfloat162float(__ldg(p)); }
  static __device__ __forceinline__ float ldv(const __nv_bfloat16* p) { return __bfloat162float(*p); }
  static __device__ __forceinline__ __nv_bfloat16 to(float v) { return __float2bfloat16_rn(v); }
};

template <typename T> __device__ __forceinline__ typename Num<T>::Acc ldg(const T* p) { return Num<T>::ld(p); }
template <typename T> __device__ __forceinline__ typename Num<T>::Acc ldv(const T* p) { return Num<T>::ldv(p); }
template <typename T, typename A> __device__ __forceinline__ T cvt(A v) { return Num<T>::to(v); }

// Gauss-Seidel division: IEEE in FP64 (reproduces the reference's
// smoother bit for bit), the hardware fast division (2 ulp) in FP32, whose
// smoother is not bit-exact with the FP64 reference in any case.
// One term of a Gauss-Seidel row sum, sum + c x.  FP64 keeps the two
// roundings of the reference's x86-64 build (its order of operations is the
// parity bar); FP32 smoothers, which approximate the FP64 V-cycle to a
// tolerance, take one fused multiply-add - every FP32 smoother uses this same
// form, so they stay bit-identical to one another.
__device__ __forceinline__ double gs_madd(double sum, double c, double x) { return sum + c * x; }
__device__ __forceinline__ float gs_madd(float sum, float c, float x) { return __fmaf_rn(c, x, sum); }
__device__ __forceinline__ double gs_div(double a, double b) { return a / b; }
__device__ __forceinline__ float gs_div(float a, float b) { return __fdividef(a, b); }

// (i, j, k) of the linear index e of an nx x ny x . grid in 32-bit unsigned
// arithmetic: every grid here has fewer than 2^31 elements (the host checks),
// and a 64-bit division costs several times a 32-bit one.
__device__ __forceinline__ void decode3(size_t e, int nx, int ny, int& i, int& j, int& k) {
  const unsigned ue = (unsigned)e, row = ue / (unsigned)nx;
  i = (int)(ue - row * (unsigned)nx);
  j = (int)(row % (unsigned)ny);
  k = (int)(row / (unsigned)ny);
}

__device__ __forceinline__ int linear_tid() {
  return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
}

// Block-wide sum of one double per thread (1-, 2- or 3-D blocks of BLOCK
// threads); result valid in linear thread 0.  Fixed order: warp shuffle
// tree, then warps in index order.
template <int BLOCK>
__device__ __forceinline__ double block_sum(double v, double* smem /* >= BLOCK/32 */) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int tid = linear_tid();
  int lane = tid & 31, wid = tid >> 5;
  if (lane == 0) smem[wid] = v;
  __syncthreads();
  double s = 0;
  if (tid == 0) {
    for (int w = 0; w < BLOCK / 32; ++w) s += smem[w];
  }
  __syncthreads();
  return s;
}

// Block-wide max of |v| ignoring NaN (the reference's abs_max never lets a
// NaN win, Smoke_Solver/blas_wrapper.h:25-37); result valid in thread 0.
template <int BLOCK>
__device__ __forceinline__ double block_absmax(double v, double* smem) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  const int tid = linear_tid();
  int lane = tid & 31, wid = tid >> 5;
  if (lane == 0) smem[wid] = v;
  __syncthreads();
  double s = 0;
  if (tid == 0) {
    for (int w = 0; w < BLOCK / 32; ++w) s = fmax(s, smem[w]);
  }
  __syncthreads();
  return s;
}

}  // namespace vflip
