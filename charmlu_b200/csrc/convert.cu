// Precision conversions and vector kernels of the mixed-precision path and
// of iterative refinement (no reference counterpart: charmlu is FP64 only).
#include <cuda_bf16.h>
#include <type_traits>
#include <cuda_fp16.h>

#include "common.cuh"
#include "kernels.h"

namespace lub {
namespace {

__global__ void f64_to_f32_kernel(const double* __restrict__ src, int64_t lds, float* __restrict__ dst, int64_t ldd,
                                  int rows, int cols) {
  for (int r = blockIdx.y; r < rows; r += gridDim.y)
  for (int c = (blockIdx.x * blockDim.x + threadIdx.x) * 2; c < cols; c += gridDim.x * blockDim.x * 2) {
    if (c + 1 < cols && !(lds & 1) && !(ldd & 1)) {
      const double2 v = __ldcs(reinterpret_cast<const double2*>(src + (int64_t)r * lds + c));
      *reinterpret_cast<float2*>(dst + (int64_t)r * ldd + c) = make_float2((float)v.x, (float)v.y);
    } else {
      dst[(int64_t)r * ldd + c] = (float)src[(int64_t)r * lds + c];
      if (c + 1 < cols) dst[(int64_t)r * ldd + c + 1] = (float)src[(int64_t)r * lds + c + 1];
    }
  }
}

template <typename OUT>
__device__ __forceinline__ OUT to_lp(float v);
template <>
__device__ __forceinline__ __nv_bfloat16 to_lp<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <>
__device__ __forceinline__ __half to_lp<__half>(float v) { return __float2half_rn(v); }
__device__ __forceinline__ float from_lp(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float from_lp(__half v) { return __half2float(v); }

__device__ __forceinline__ float scale_of(const unsigned* amax, int which) {
  return amax ? pow2_scale_of(__uint_as_float(amax[which])) : 1.f;
}

// dst[r][p*ps + k] = part p of src[r][k] * scale (hi, or lo = rest after
// hi); part p occupies [p*ps, p*ps + ps), zero past K (ps >= K)
template <typename OUT>
__global__ void split_rows_kernel(const float* __restrict__ src, int64_t lds, OUT* __restrict__ dst, int64_t ldd,
                                  int rows, int K, int ps, int nparts, unsigned lo_mask, const unsigned* amax,
                                  int which) {
  const int r = blockIdx.y * blockDim.y + threadIdx.y;
  if (r >= rows) return;
  const float sc = scale_of(amax, which);
  for (int k = threadIdx.x; k < ps; k += blockDim.x) {
    const float v = k < K ? src[(int64_t)r * lds + k] * sc : 0.f;
    const OUT hi = to_lp<OUT>(v);
    const OUT lo = to_lp<OUT>(v - from_lp(hi));
    for (int p = 0; p < nparts; p++) dst[(int64_t)r * ldd + (int64_t)p * ps + k] = ((lo_mask >> p) & 1) ? lo : hi;
  }
}

// dst[n][p*ps + k] = part p of src[k][n] * scale: src is K x N, dst
// N x (nparts*ps), zero past K in each part (ps >= K)
template <typename OUT>
__global__ void split_transpose_kernel(const float* __restrict__ src, int64_t lds, OUT* __restrict__ dst, int64_t ldd,
                                       int K, int ps, int N, int nparts, unsigned lo_mask, const unsigned* amax,
                                       int which) {
  __shared__ float t[32][33];
  const int k0 = blockIdx.y * 32, n0 = blockIdx.x * 32;
  const float sc = scale_of(amax, which);
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int k = k0 + i, n = n0 + threadIdx.x;
    t[i][threadIdx.x] = (k < K && n < N) ? src[(int64_t)k * lds + n] * sc : 0.f;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int n = n0 + i, k = k0 + threadIdx.x;
    if (n < N && k < ps) {
      const float v = t[threadIdx.x][i];  // zero past K (staged above)
      const OUT hi = to_lp<OUT>(v);
      const OUT lo = to_lp<OUT>(v - from_lp(hi));
      for (int p = 0; p < nparts; p++) dst[(int64_t)n * ldd + (int64_t)p * ps + k] = ((lo_mask >> p) & 1) ? lo : hi;
    }
  }
}

// max |P| over a rows x cols row-major block: warps take segments of up to
// 2048 columns of one row (one division per segment), lanes read float4 when
// the block allows 16-byte loads
__device__ __forceinline__ float absmax_block(const float* __restrict__ P, int64_t ld, int rows, int cols, int gw,
                                             int nw, int lane) {
  constexpr int SEG = 2048;
  float m = 0.f;
  if (rows <= 0 || cols <= 0) return m;
  const int nseg = (cols + SEG - 1) / SEG;
  const int64_t units = (int64_t)rows * nseg;
  const bool vec = ((reinterpret_cast<uintptr_t>(P) & 15) == 0) && ((ld & 3) == 0) && ((cols & 3) == 0);
  for (int64_t u = gw; u < units; u += nw) {
    const int64_t r = u / nseg;
    const int c0 = (int)(u - r * nseg) * SEG, c1 = min(cols, c0 + SEG);
    const float* row = P + r * ld;
    if (vec) {
#pragma unroll 4
      for (int c = c0 + 4 * lane; c < c1; c += 128) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(row + c));
        m = fmaxf(m, fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w))));
      }
    } else {
#pragma unroll 4
      for (int c = c0 + lane; c < c1; c += 32) m = fmaxf(m, fabsf(row[c]));
    }
  }
  return m;
}

// amax[0] = max |L| (rows x K), or *lmax_from when given; amax[1] = max |U|
// (K x N); float bit patterns (non-negative floats order as unsigned)
__global__ void panel_absmax_kernel(const float* __restrict__ L, int64_t ldl, int rows, int K,
                                    const float* __restrict__ U, int64_t ldu, int N, unsigned* amax,
                                    const unsigned* lmax_from) {
  const int lane = threadIdx.x & 31;
  const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nw = (int)((gridDim.x * blockDim.x) >> 5);
  float mL = lmax_from ? 0.f : absmax_block(L, ldl, rows, K, gw, nw, lane);
  float mU = absmax_block(U, ldu, K, N, gw, nw, lane);
  for (int o = 16; o > 0; o >>= 1) {
    mL = fmaxf(mL, __shfl_xor_sync(0xffffffffu, mL, o));
    mU = fmaxf(mU, __shfl_xor_sync(0xffffffffu, mU, o));
  }
  if (lane == 0) {
    if (lmax_from) {
      if (gw == 0) atomicMax(&amax[0], *lmax_from);
    } else {
      atomicMax(&amax[0], __float_as_uint(mL));
    }
    atomicMax(&amax[1], __float_as_uint(mU));
  }
}

__device__ __forceinline__ double rnorm_of(const ResidualAccum* acc) {
  const double r = __longlong_as_double((long long)acc->rmax);
  return (r > 0.0 && isfinite(r)) ? r : 1.0;
}

// r32[i] = r64[perm[i]] / ||r||inf  (permuted, scaled into FP32 range)
__global__ void ir_prep_kernel(const double* __restrict__ r64, const int32_t* __restrict__ perm, float* __restrict__ r32,
                               int n, const ResidualAccum* acc) {
  const double inv = 1.0 / rnorm_of(acc);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r32[i] = (float)(r64[perm[i]] * inv);
}
// x[i] += d32[i] * ||r||inf
__global__ void ir_update_kernel(double* __restrict__ x, const float* __restrict__ d32, int n,
                                 const ResidualAccum* acc) {
  const double sc = rnorm_of(acc);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = fma((double)d32[i], sc, x[i]);
}
// y32[i] = v64[perm[i]] (no scaling) and back
__global__ void gather_f64_to_f32_kernel(const double* __restrict__ v, const int32_t* __restrict__ perm,
                                         float* __restrict__ y, int n, double scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = (float)(v[perm[i]] * scale);
}
__global__ void gather_f64_kernel(const double* __restrict__ v, const int32_t* __restrict__ perm,
                                  double* __restrict__ y, int n, double scale, const ResidualAccum* acc) {
  const double sc = acc ? 1.0 / rnorm_of(acc) : scale;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = v[perm[i]] * sc;
}
__global__ void f32_to_f64_kernel(const float* __restrict__ y, double* __restrict__ x, int n, double scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = (double)y[i] * scale;
}

constexpr int kDotBlocks = 128;

// part[j * kDotBlocks + b] = sum over block b's slice of V_j . w (fixed order)
__global__ void __launch_bounds__(256) multi_dot_part_kernel(const double* __restrict__ V, const double* __restrict__ w,
                                                             int n, double* __restrict__ part) {
  __shared__ double red[8];
  const int j = blockIdx.y, b = blockIdx.x;
  const int per = (n + kDotBlocks - 1) / kDotBlocks;
  const int lo = b * per, hi = min(n, lo + per);
  const double* v = V + (int64_t)j * n;
  double acc = 0.0;
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) acc = fma(v[i], w[i], acc);
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < 8; q++) t += red[q];
    part[j * kDotBlocks + b] = t;
  }
}
__global__ void multi_dot_final_kernel(const double* __restrict__ part, int k, double* __restrict__ out) {
  for (int j = threadIdx.x; j < k; j += blockDim.x) {
    double t = 0.0;
    for (int b = 0; b < kDotBlocks; b++) t += part[j * kDotBlocks + b];
    out[j] = t;
  }
}
// w += sign * sum_j h[j] V_j
__global__ void multi_axpy_kernel(double* __restrict__ w, const double* __restrict__ V, int k,
                                  const double* __restrict__ h, int n, double sign) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double t = 0.0;
  for (int j = 0; j < k; j++) t = fma(h[j], V[(int64_t)j * n + i], t);
  w[i] = fma(sign, t, w[i]);
}
// y = a * x
__global__ void scale_vec_kernel(const double* __restrict__ x, double* __restrict__ y, int n, double a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = a * x[i];
}
// dst = src / sqrt(*sq)  (sq = squared norm)
__global__ void scale_copy_kernel(const double* __restrict__ src, double* __restrict__ dst, int n,
                                  const double* __restrict__ sq) {
  const double nr = sqrt(*sq);
  const double inv = nr > 0.0 ? 1.0 / nr : 0.0;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[i] * inv;
}

}  // namespace

int launch_multi_dot(const double* V, int k, const double* w, int n, double* part, double* out, cudaStream_t s) {
  if (k <= 0) return LU_OK;
  multi_dot_part_kernel<<<dim3(kDotBlocks, k), 256, 0, s>>>(V, w, n, part);
  LUB_LAUNCH_CHECK();
  multi_dot_final_kernel<<<1, 256, 0, s>>>(part, k, out);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}
int launch_multi_axpy(double* w, const double* V, int k, const double* h, int n, double sign, cudaStream_t s) {
  if (k <= 0) return LU_OK;
  multi_axpy_kernel<<<ceil_div(n, 256), 256, 0, s>>>(w, V, k, h, n, sign);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}
int launch_scale_vec(const double* x, double* y, int n, double a, cudaStream_t s) {
  if (n <= 0) return LU_OK;
  scale_vec_kernel<<<ceil_div(n, 256), 256, 0, s>>>(x, y, n, a);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}
int launch_scale_copy(const double* src, double* dst, int n, const double* sq, cudaStream_t s) {
  scale_copy_kernel<<<ceil_div(n, 256), 256, 0, s>>>(src, dst, n, sq);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

int launch_f64_to_f32(const double* src, int64_t lds, float* dst, int64_t ldd, int rows, int cols, cudaStream_t s) {
  if (rows <= 0 || cols <= 0) return LU_OK;
  dim3 grid(std::max(1, std::min(ceil_div(cols, 512), 8)), std::min(rows, 32768));
  f64_to_f32_kernel<<<grid, 256, 0, s>>>(src, lds, dst, ldd, rows, cols);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

template <typename OUT>
int launch_split_rows(const float* src, int64_t lds, OUT* dst, int64_t ldd, int rows, int K, int nparts,
                      unsigned lo_mask, const unsigned* amax, int which, cudaStream_t s, int part_stride) {
  if (rows <= 0 || K <= 0) return LU_OK;
  const int ps = part_stride > 0 ? part_stride : K;
  if (ps < K) return LU_ERR_ARG;
  dim3 block(128, 4);
  dim3 grid(1, ceil_div(rows, 4));
  split_rows_kernel<OUT><<<grid, block, 0, s>>>(src, lds, dst, ldd, rows, K, ps, nparts, lo_mask, amax, which);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}
template <typename OUT>
int launch_split_transpose(const float* src, int64_t lds, OUT* dst, int64_t ldd, int K, int N, int nparts,
                           unsigned lo_mask, const unsigned* amax, int which, cudaStream_t s, int part_stride) {
  if (K <= 0 || N <= 0) return LU_OK;
  const int ps = part_stride > 0 ? part_stride : K;
  if (ps < K) return LU_ERR_ARG;
  dim3 block(32, 8);
  dim3 grid(ceil_div(N, 32), ceil_div(ps, 32));
  split_transpose_kernel<OUT><<<grid, block, 0, s>>>(src, lds, dst, ldd, K, ps, N, nparts, lo_mask, amax, which);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}
template int launch_split_rows<__nv_bfloat16>(const float*, int64_t, __nv_bfloat16*, int64_t, int, int, int, unsigned,
                                              const unsigned*, int, cudaStream_t, int);
template int launch_split_rows<__half>(const float*, int64_t, __half*, int64_t, int, int, int, unsigned,
                                       const unsigned*, int, cudaStream_t, int);
template int launch_split_transpose<__nv_bfloat16>(const float*, int64_t, __nv_bfloat16*, int64_t, int, int, int,
                                                   unsigned, const unsigned*, int, cudaStream_t, int);
template int launch_split_transpose<__half>(const float*, int64_t, __half*, int64_t, int, int, int, unsigned,
                                            const unsigned*, int, cudaStream_t, int);

int launch_panel_absmax(const float* L, int64_t ldl, int rows, int K, const float* U, int64_t ldu, int N,
                        unsigned* amax, cudaStream_t s, const unsigned* lmax_from) {
  LUB_CUDA(cudaMemsetAsync(amax, 0, 2 * sizeof(unsigned), s));
  const int64_t tot = std::max(lmax_from ? 0 : (int64_t)rows * K, (int64_t)K * N);
  const int blocks = (int)std::min<int64_t>(std::max<int64_t>(1, tot / 4096), 4 * kNumSMsB200);
  panel_absmax_kernel<<<blocks, 256, 0, s>>>(L, ldl, rows, K, U, ldu, N, amax, lmax_from);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

int launch_ir_prep(const double* r64, const int32_t* perm, float* r32, int n, const ResidualAccum* acc,
                   cudaStream_t s) {
  ir_prep_kernel<<<ceil_div(n, 256), 256, 0, s>>>(r64, perm, r32, n, acc);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}
int launch_ir_update(double* x, const float* d32, int n, const ResidualAccum* acc, cudaStream_t s) {
  ir_update_kernel<<<ceil_div(n, 256), 256, 0, s>>>(x, d32, n, acc);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}
int launch_gather_f64_to_f32(const double* v, const int32_t* perm, float* y, int n, double scale, cudaStream_t s) {
  gather_f64_to_f32_kernel<<<ceil_div(n, 256), 256, 0, s>>>(v, perm, y, n, scale);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}
int launch_gather_f64(const double* v, const int32_t* perm, double* y, int n, double scale, const ResidualAccum* acc,
                      cudaStream_t s) {
  gather_f64_kernel<<<ceil_div(n, 256), 256, 0, s>>>(v, perm, y, n, scale, acc);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}
int launch_f32_to_f64(const float* y, double* x, int n, double scale, cudaStream_t s) {
  f32_to_f64_kernel<<<ceil_div(n, 256), 256, 0, s>>>(y, x, n, scale);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

}  // namespace lub
