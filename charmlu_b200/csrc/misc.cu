// Residual check, generators and permutation helpers.
//
// Residual: restates the validation pass (benchmark.C:462-573): r = b - A x
// with the ORIGINAL A, plus the maxima the scaled residual needs
// (max |a_ij| as in infNorm, benchmark.C:476-483; also the true row-sum
// ||A||inf).  One warp per row, 16-byte loads; HBM-bound (8 n^2 bytes).
#include "common.cuh"
#include "kernels.h"

namespace lub {
namespace {

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* p, double v) {
  atomicMax(p, (unsigned long long)__double_as_longlong(v));
}

// Rows row0 .. row0 + rows - 1 of the system; A points at row row0 (a
// device-resident matrix, or a chunk of a host matrix staged on the device).
__global__ void __launch_bounds__(256) residual_f64_kernel(const double* A, int64_t lda, int rows, int row0, int n,
                                                           const double* x, const double* b, double* r,
                                                           ResidualAccum* acc) {
  __shared__ double s_m[8], s_rs[8], s_r[8], s_b[8], s_x[8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lrow = blockIdx.x * 8 + warp;
  const int row = row0 + lrow;
  double m = 0.0, rs = 0.0, ra = 0.0, bb = 0.0, xx = 0.0;
  if (lrow < rows) {
    const double* ar = A + (int64_t)lrow * lda;
    double s0 = 0.0, s1 = 0.0;
    const bool vec = ((lda & 1) == 0) && ((reinterpret_cast<uintptr_t>(A) & 15) == 0);
    if (vec) {
      const int n2 = n & ~1;
      for (int j = lane * 2; j < n2; j += 64) {
        const double2 a = __ldcs(reinterpret_cast<const double2*>(ar + j));
        const double2 xv = *reinterpret_cast<const double2*>(x + j);
        s0 = fma(a.x, xv.x, s0);
        s1 = fma(a.y, xv.y, s1);
        rs += fabs(a.x) + fabs(a.y);
        m = fmax(m, fmax(fabs(a.x), fabs(a.y)));
      }
      if ((n & 1) && lane == 0) {
        const double a = ar[n - 1];
        s0 = fma(a, x[n - 1], s0);
        rs += fabs(a);
        m = fmax(m, fabs(a));
      }
    } else {
      for (int j = lane; j < n; j += 32) {
        const double a = ar[j];
        s0 = fma(a, x[j], s0);
        rs += fabs(a);
        m = fmax(m, fabs(a));
      }
    }
    double s = s0 + s1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s += __shfl_xor_sync(0xffffffffu, s, o);
      rs += __shfl_xor_sync(0xffffffffu, rs, o);
      m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    const double ri = b[row] - s;
    if (lane == 0 && r) r[row] = ri;
    ra = fabs(ri);
    bb = fabs(b[row]);
    xx = fabs(x[row]);
    if (isnan(ri)) ra = ri;
  }
  if (lane == 0) { s_m[warp] = m; s_rs[warp] = rs; s_r[warp] = ra; s_b[warp] = bb; s_x[warp] = xx; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < 8; w++) {
      s_m[0] = fmax(s_m[0], s_m[w]);
      s_rs[0] = fmax(s_rs[0], s_rs[w]);
      s_r[0] = (isnan(s_r[w]) || s_r[w] > s_r[0]) ? s_r[w] : s_r[0];
      s_b[0] = fmax(s_b[0], s_b[w]);
      s_x[0] = fmax(s_x[0], s_x[w]);
    }
    atomic_max_nonneg(&acc->amax, s_m[0]);
    atomic_max_nonneg(&acc->anorm, s_rs[0]);
    atomic_max_nonneg(&acc->rmax, isnan(s_r[0]) ? __longlong_as_double(0x7ff8000000000000LL) : s_r[0]);
    atomic_max_nonneg(&acc->bmax, s_b[0]);
    atomic_max_nonneg(&acc->xmax, s_x[0]);
  }
}

// In-place transpose of the n x n matrix A (row pitch lda) by 32 x 32
// tiles: the CTA of tile (bi, bj), bi <= bj, reads it and tile (bj, bi)
// into shared memory and writes each back transposed into the other's
// place (a diagonal tile is transposed in place). 32 x 8 threads.
__global__ void __launch_bounds__(256) transpose_inplace_kernel(double* A, int64_t lda, int n) {
  __shared__ double t1[32][33], t2[32][33];
  const int bi = blockIdx.x, bj = blockIdx.y;
  if (bi > bj) return;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int k = ty; k < 32; k += 8) {
    int r = bi * 32 + k, c = bj * 32 + tx;
    if (r < n && c < n) t1[k][tx] = A[(int64_t)r * lda + c];
    r = bj * 32 + k;
    c = bi * 32 + tx;
    if (bi != bj && r < n && c < n) t2[k][tx] = A[(int64_t)r * lda + c];
  }
  __syncthreads();
  for (int k = ty; k < 32; k += 8) {
    int r = bj * 32 + k, c = bi * 32 + tx;  // tile (bj, bi) <- tile (bi, bj)^T
    if (r < n && c < n) A[(int64_t)r * lda + c] = t1[tx][k];
    r = bi * 32 + k;
    c = bj * 32 + tx;  // tile (bi, bj) <- tile (bj, bi)^T
    if (bi != bj && r < n && c < n) A[(int64_t)r * lda + c] = t2[tx][k];
  }
}

// y[i] -= A[i, :] . x for i < m (one warp per row; k columns)
__global__ void __launch_bounds__(256) gemv_sub_kernel(const double* A, int64_t lda, int m, int k, const double* x,
                                                       double* y) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * 8 + warp;
  if (row >= m) return;
  const double* ar = A + (int64_t)row * lda;
  double s0 = 0.0, s1 = 0.0;
  const bool vec = ((lda & 1) == 0) && ((reinterpret_cast<uintptr_t>(A) & 15) == 0) &&
                   ((reinterpret_cast<uintptr_t>(x) & 15) == 0);
  if (vec) {
    const int k2 = k & ~1;
    for (int j = lane * 2; j < k2; j += 64) {
      const double2 a = *reinterpret_cast<const double2*>(ar + j);
      const double2 xv = *reinterpret_cast<const double2*>(x + j);
      s0 = fma(a.x, xv.x, s0);
      s1 = fma(a.y, xv.y, s1);
    }
    if ((k & 1) && lane == 0) s0 = fma(ar[k - 1], x[k - 1], s0);
  } else {
    for (int j = lane; j < k; j += 32) s0 = fma(ar[j], x[j], s0);
  }
  double s = s0 + s1;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) y[row] -= s;
}

__global__ void gen_uniform_kernel(double* d, int64_t rows, int64_t cols, int64_t ld, uint64_t key) {
  const int64_t total = rows * cols;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx / cols, j = idx - i * cols;
    d[i * ld + j] = uniform_at(key, (uint64_t)idx);
  }
}

__global__ void gather_perm_kernel(const double* b, const int32_t* perm, double* y, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = b[perm[i]];
}
__global__ void scatter_perm_kernel(const double* y, const int32_t* perm, double* b, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[perm[i]] = y[i];
}
__global__ void iota_kernel(int32_t* p, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = i;
}

}  // namespace

int launch_residual_f64(const double* A, int64_t lda, int n, const double* x, const double* b, double* r,
                        ResidualAccum* acc, cudaStream_t s) {
  LUB_CUDA(cudaMemsetAsync(acc, 0, sizeof(ResidualAccum), s));
  if (n <= 0) return LU_OK;
  residual_f64_kernel<<<ceil_div(n, 8), 256, 0, s>>>(A, lda, n, 0, n, x, b, r, acc);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

int launch_transpose_inplace(double* A, int64_t lda, int n, cudaStream_t s) {
  if (n <= 1) return LU_OK;
  const int nt = ceil_div(n, 32);
  if (nt > 65535) return LU_ERR_UNSUPPORTED;
  transpose_inplace_kernel<<<dim3(nt, nt), dim3(32, 8), 0, s>>>(A, lda, n);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

int launch_gemv_sub(const double* A, int64_t lda, int m, int k, const double* x, double* y, cudaStream_t s) {
  if (m <= 0 || k <= 0) return LU_OK;
  gemv_sub_kernel<<<ceil_div(m, 8), 256, 0, s>>>(A, lda, m, k, x, y);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

int launch_residual_f64_rows(const double* Arows, int64_t lda, int rows, int row0, int n, const double* x,
                             const double* b, double* r, ResidualAccum* acc, cudaStream_t s) {
  if (rows <= 0) return LU_OK;
  residual_f64_kernel<<<ceil_div(rows, 8), 256, 0, s>>>(Arows, lda, rows, row0, n, x, b, r, acc);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

int launch_gen_uniform(double* d, int64_t rows, int64_t cols, int64_t ld, uint64_t seed, uint64_t stream_id,
                       cudaStream_t s) {
  if (rows <= 0 || cols <= 0) return LU_OK;
  const int64_t total = rows * cols;
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, (int64_t)kNumSMsB200 * 64);
  gen_uniform_kernel<<<blocks, 256, 0, s>>>(d, rows, cols, ld, stream_key(seed, stream_id));
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

int launch_gather_perm(const double* b, const int32_t* perm, double* y, int n, cudaStream_t s) {
  if (n <= 0) return LU_OK;
  gather_perm_kernel<<<ceil_div(n, 256), 256, 0, s>>>(b, perm, y, n);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}
int launch_scatter_perm(const double* y, const int32_t* perm, double* b, int n, cudaStream_t s) {
  if (n <= 0) return LU_OK;
  scatter_perm_kernel<<<ceil_div(n, 256), 256, 0, s>>>(y, perm, b, n);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}
int launch_iota(int32_t* p, int n, cudaStream_t s) {
  if (n <= 0) return LU_OK;
  iota_kernel<<<ceil_div(n, 256), 256, 0, s>>>(p, n);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

}  // namespace lub
