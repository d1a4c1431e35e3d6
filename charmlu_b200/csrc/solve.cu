// Triangular solves.
//
// TRSM leaf: B <- L^{-1} B with L unit lower (m <= 32), restating
// LUBlk::computeU (lu.C:180-189, dtrsm left/lower/unit).  Larger m is
// handled by host-side recursion with the GEMM kernel.
//
// TRSV: forward (unit lower) and backward (upper, divide by u_ii)
// substitution of one right-hand side, restating forwardSolve /
// backwardSolve / offDiagSolve (lu.ci:387-458).  The reference pipelines
// block rows through multicasts and a row-sum reduction into the diagonal
// chare; here one CTA per 64-row block takes a ticket in launch order, reads
// its row block of the factor while earlier blocks finish, waits (bounded)
// on each earlier block's ready flag, accumulates the off-diagonal product,
// then one warp substitutes inside the diagonal block and publishes the
// block with a release flag.  A CTA only ever waits on lower tickets, which
// were handed to CTAs already running, so the pipeline cannot deadlock.
#include "common.cuh"
#include "kernels.h"

namespace lub {
namespace {

template <typename T>
__global__ void __launch_bounds__(128) trsm_llu_leaf_kernel(const T* L, int64_t ldl, T* B, int64_t ldb, int m,
                                                            int ncols) {
  __shared__ T sL[32][33];
  for (int idx = threadIdx.x; idx < 32 * 32; idx += blockDim.x) {
    const int i = idx >> 5, p = idx & 31;
    sL[i][p] = (i < m && p < i) ? L[(int64_t)i * ldl + p] : T(0);
  }
  __syncthreads();
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncols) return;
  T x[32];
#pragma unroll
  for (int i = 0; i < 32; i++) x[i] = i < m ? B[(int64_t)i * ldb + col] : T(0);
#pragma unroll
  for (int i = 1; i < 32; i++) {
#pragma unroll
    for (int p = 0; p < i; p++) x[i] = fma(-sL[i][p], x[p], x[i]);
  }
#pragma unroll
  for (int i = 0; i < 32; i++)
    if (i < m) B[(int64_t)i * ldb + col] = x[i];
}

constexpr int TB = 64;  // rows per TRSV block

template <typename T, bool UPPER>
__global__ void __launch_bounds__(256) trsv_kernel(const T* LU, int64_t lda, int n, T* x, int* flags,
                                                   unsigned* ticket, DevStatus* st, long long spin) {
  __shared__ T sD[TB][TB + 1];
  __shared__ T s_acc[TB];
  __shared__ int s_blk;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) s_blk = (int)atomicAdd(ticket, 1u);
  __syncthreads();
  const int nblk = (n + TB - 1) / TB;
  const int tk = s_blk;
  if (tk >= nblk) return;
  const int bi = UPPER ? nblk - 1 - tk : tk;
  const int r0 = bi * TB, rows = min(TB, n - r0);

  for (int idx = tid; idx < TB * TB; idx += blockDim.x) {
    const int i = idx / TB, j = idx - i * TB;
    sD[i][j] = (i < rows && j < rows) ? LU[(int64_t)(r0 + i) * lda + r0 + j] : T(0);
  }

  T acc[8];
#pragma unroll
  for (int i = 0; i < 8; i++) acc[i] = T(0);
  const int nvisit = UPPER ? (nblk - 1 - bi) : bi;
  bool ok = true;
  for (int q = 0; q < nvisit && ok; q++) {
    const int cb = UPPER ? nblk - 1 - q : q;
    const int c0 = cb * TB;
    T lv[8][2];
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int r = r0 + warp * 8 + i;
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int c = c0 + lane * 2 + e;
        lv[i][e] = (r < n && c < n) ? __ldcs(&LU[(int64_t)r * lda + c]) : T(0);
      }
    }
    if (lane == 0) {
      long long polls = 0;
      while (ld_acquire_s32(&flags[cb]) == 0) {
        if (++polls > spin) { dev_fail(st, LU_ERR_TIMEOUT, 301); ok = false; break; }
        if ((polls & 1023) == 0 && ld_acquire_s32(&st->code) != 0) { ok = false; break; }
      }
    }
    ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
    __syncwarp();
    if (!ok) break;
    const int c = c0 + lane * 2;
    const T x0 = c < n ? __ldcg(&x[c]) : T(0);
    const T x1 = c + 1 < n ? __ldcg(&x[c + 1]) : T(0);
#pragma unroll
    for (int i = 0; i < 8; i++) acc[i] = fma(lv[i][1], x1, fma(lv[i][0], x0, acc[i]));
  }
#pragma unroll
  for (int i = 0; i < 8; i++) {
    T v = acc[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) s_acc[warp * 8 + i] = v;
  }
  __syncthreads();
  if (!ok) return;
  if (warp == 0) {
    T v0 = lane < rows ? x[r0 + lane] - s_acc[lane] : T(0);
    T v1 = lane + 32 < rows ? x[r0 + lane + 32] - s_acc[lane + 32] : T(0);
    if (!UPPER) {
      for (int j = 0; j < rows; j++) {
        const T xj = __shfl_sync(0xffffffffu, j < 32 ? v0 : v1, j & 31);
        if (lane > j) v0 = fma(-sD[lane][j], xj, v0);
        if (lane + 32 > j) v1 = fma(-sD[lane + 32][j], xj, v1);
      }
    } else {
      for (int j = rows - 1; j >= 0; j--) {
        // owner finalises x_j, then broadcasts
        if (j < 32) { if (lane == j) v0 = v0 / sD[j][j]; }
        else        { if (lane == j - 32) v1 = v1 / sD[j][j]; }
        const T xj = __shfl_sync(0xffffffffu, j < 32 ? v0 : v1, j & 31);
        if (lane < j) v0 = fma(-sD[lane][j], xj, v0);
        if (lane + 32 < j) v1 = fma(-sD[lane + 32][j], xj, v1);
      }
    }
    if (lane < rows) x[r0 + lane] = v0;
    if (lane + 32 < rows) x[r0 + lane + 32] = v1;
    __threadfence();
    __syncwarp();
    if (lane == 0) st_release_s32(&flags[bi], 1);
  }
}

}  // namespace

template <typename T>
int launch_trsm_llu_leaf(const T* L, int64_t ldl, T* B, int64_t ldb, int m, int ncols, cudaStream_t s) {
  if (m <= 1 || ncols <= 0) return LU_OK;
  if (m > 32) return LU_ERR_ARG;
  trsm_llu_leaf_kernel<T><<<ceil_div(ncols, 128), 128, 0, s>>>(L, ldl, B, ldb, m, ncols);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

template <typename T>
int launch_trsv(const T* LU, int64_t lda, int n, T* x, int upper, int* flags, unsigned* ticket, DevStatus* st,
                long long spin, cudaStream_t s) {
  if (n <= 0) return LU_OK;
  const int nblk = ceil_div(n, TB);
  LUB_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * nblk, s));
  LUB_CUDA(cudaMemsetAsync(ticket, 0, sizeof(unsigned), s));
  if (upper)
    trsv_kernel<T, true><<<nblk, 256, 0, s>>>(LU, lda, n, x, flags, ticket, st, spin);
  else
    trsv_kernel<T, false><<<nblk, 256, 0, s>>>(LU, lda, n, x, flags, ticket, st, spin);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

template int launch_trsm_llu_leaf<double>(const double*, int64_t, double*, int64_t, int, int, cudaStream_t);
template int launch_trsm_llu_leaf<float>(const float*, int64_t, float*, int64_t, int, int, cudaStream_t);
template int launch_trsv<double>(const double*, int64_t, int, double*, int, int*, unsigned*, DevStatus*, long long,
                                 cudaStream_t);
template int launch_trsv<float>(const float*, int64_t, int, float*, int, int*, unsigned*, DevStatus*, long long,
                                cudaStream_t);

}  // namespace lub
