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

// TS: storage type of the factors; T: type of the vector and the arithmetic
// (FP32 factors with an FP64 vector give the GMRES-IR preconditioner solve
// in working precision at the FP32 factors' memory cost).
template <typename TS, typename T, bool UPPER>
__global__ void __launch_bounds__(256) trsv_kernel(const TS* LU, int64_t lda, int n, T* x, int* flags,
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
    sD[i][j] = (i < rows && j < rows) ? (T)LU[(int64_t)(r0 + i) * lda + r0 + j] : T(0);
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
        lv[i][e] = (r < n && c < n) ? (T)__ldcs(&LU[(int64_t)r * lda + c]) : T(0);
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

// ---------------------------------------------------------------------------
// Multi-right-hand-side triangular solve T Y = B in place on a row-major
// n x nrhs block (nrhs <= 16 per launch), T taken from row-major LU factors:
//   MODE 0  LN: T = L  (unit lower)      forward,  tiles L[bi][bk], bk < bi
//   MODE 1  UN: T = U  (upper)           backward, tiles U[bi][bk], bk > bi
//   MODE 2  UT: T = U^T (lower)          forward,  tiles U[bk][bi]^T, bk < bi
//   MODE 3  LT: T = L^T (unit upper)     backward, tiles L[bk][bi]^T, bk > bi
// Modes 2 and 3 are the transposed solves of the adjoint (A^T lambda = W).
// Same ticket/flag pipeline as trsv_kernel; every 64 x 64 tile is staged in
// shared memory with coalesced row reads, so the transposed modes read the
// factor by rows too.
// ---------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(256) trsm_pipe_kernel(const double* LU, int64_t lda, int n, double* Y, int64_t ldy,
                                                        int nrhs, int* flags, unsigned* ticket, DevStatus* st,
                                                        long long spin) {
  constexpr bool FWD = (MODE == 0 || MODE == 2);
  constexpr bool TRANS = (MODE >= 2);
  constexpr bool UNIT = (MODE == 0 || MODE == 3);
  __shared__ double tile[TB][TB + 1];
  __shared__ double yk[TB][17];
  __shared__ int s_blk, s_ok;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) s_blk = (int)atomicAdd(ticket, 1u);
  __syncthreads();
  const int nblk = (n + TB - 1) / TB;
  const int tk = s_blk;
  if (tk >= nblk) return;
  const int bi = FWD ? tk : nblk - 1 - tk;
  const int r0 = bi * TB, rows = min(TB, n - r0);
  // this thread's outputs: row r = tid / 4, rhs columns 4*(tid%4) .. +3
  const int orow = tid >> 2, oc = (tid & 3) * 4;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  const int nvisit = FWD ? bi : nblk - 1 - bi;
  bool ok = true;
  for (int q = 0; q < nvisit; q++) {
    const int bk = FWD ? q : nblk - 1 - q;
    const int c0 = bk * TB, cw = min(TB, n - c0);
    // stage the tile: NoTrans T[bi][bk] rows r0.., cols c0..; Trans: rows c0.., cols r0..
    for (int idx = tid; idx < TB * TB; idx += blockDim.x) {
      const int i = idx / TB, j = idx - i * TB;
      double v = 0.0;
      if (!TRANS) {
        if (i < rows && j < cw) v = __ldcs(&LU[(int64_t)(r0 + i) * lda + c0 + j]);
      } else {
        if (i < cw && j < rows) v = __ldcs(&LU[(int64_t)(c0 + i) * lda + r0 + j]);
      }
      tile[i][j] = v;
    }
    if (tid == 0) {
      long long polls = 0;
      s_ok = 1;
      while (ld_acquire_s32(&flags[bk]) == 0) {
        if (++polls > spin) { dev_fail(st, LU_ERR_TIMEOUT, 302); s_ok = 0; break; }
        if ((polls & 1023) == 0 && ld_acquire_s32(&st->code) != 0) { s_ok = 0; break; }
      }
    }
    __syncthreads();
    if (!s_ok) { ok = false; break; }
    for (int idx = tid; idx < TB * 16; idx += blockDim.x) {
      const int i = idx >> 4, c = idx & 15;
      yk[i][c] = (i < cw && c < nrhs) ? __ldcg(&Y[(int64_t)(c0 + i) * ldy + c]) : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int k = 0; k < TB; k++) {
      const double t = TRANS ? tile[k][orow] : tile[orow][k];
#pragma unroll
      for (int e = 0; e < 4; e++) acc[e] = fma(t, yk[k][oc + e], acc[e]);
    }
    __syncthreads();
  }
  if (!ok) return;
  // right-hand side minus the off-diagonal contributions, then the diagonal tile
  for (int e = 0; e < 4; e++) {
    const int c = oc + e;
    yk[orow][c] = (orow < rows && c < nrhs) ? Y[(int64_t)(r0 + orow) * ldy + c] - acc[e] : 0.0;
  }
  for (int idx = tid; idx < TB * TB; idx += blockDim.x) {
    const int i = idx / TB, j = idx - i * TB;
    // diagonal tile in the orientation of T: T(i, j)
    double v = 0.0;
    if (i < rows && j < rows) v = TRANS ? LU[(int64_t)(r0 + j) * lda + r0 + i] : LU[(int64_t)(r0 + i) * lda + r0 + j];
    tile[i][j] = v;
  }
  __syncthreads();
  // warp w solves rhs columns w and w + 8; lanes own rows lane and lane + 32
  for (int c = warp; c < nrhs; c += 8) {
    double v0 = yk[lane][c], v1 = yk[lane + 32][c];
    if (FWD) {
      for (int j = 0; j < rows; j++) {
        if (!UNIT) {
          if (j < 32) { if (lane == j) v0 = v0 / tile[j][j]; }
          else        { if (lane == j - 32) v1 = v1 / tile[j][j]; }
        }
        const double xj = __shfl_sync(0xffffffffu, j < 32 ? v0 : v1, j & 31);
        if (lane > j) v0 = fma(-tile[lane][j], xj, v0);
        if (lane + 32 > j) v1 = fma(-tile[lane + 32][j], xj, v1);
      }
    } else {
      for (int j = rows - 1; j >= 0; j--) {
        if (!UNIT) {
          if (j < 32) { if (lane == j) v0 = v0 / tile[j][j]; }
          else        { if (lane == j - 32) v1 = v1 / tile[j][j]; }
        }
        const double xj = __shfl_sync(0xffffffffu, j < 32 ? v0 : v1, j & 31);
        if (lane < j) v0 = fma(-tile[lane][j], xj, v0);
        if (lane + 32 < j) v1 = fma(-tile[lane + 32][j], xj, v1);
      }
    }
    if (lane < rows) Y[(int64_t)(r0 + lane) * ldy + c] = v0;
    if (lane + 32 < rows) Y[(int64_t)(r0 + lane + 32) * ldy + c] = v1;
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) st_release_s32(&flags[bi], 1);
}

// G = -Lam * X^T (n x n), Lam and X n x k row-major, k <= 16: the rank-k
// gradient of the adjoint.  Output-bound (8 n^2 bytes written).
__global__ void __launch_bounds__(256) neg_outer_kernel(const double* Lam, int64_t ldl, const double* X, int64_t ldx,
                                                        int n, int k, double* G, int64_t ldg, int accumulate) {
  __shared__ double sl[64][17], sx[64][17];
  const int i0 = blockIdx.y * 64, j0 = blockIdx.x * 64;
  for (int idx = threadIdx.x; idx < 64 * 16; idx += blockDim.x) {
    const int r = idx >> 4, c = idx & 15;
    sl[r][c] = (i0 + r < n && c < k) ? Lam[(int64_t)(i0 + r) * ldl + c] : 0.0;
    sx[r][c] = (j0 + r < n && c < k) ? X[(int64_t)(j0 + r) * ldx + c] : 0.0;
  }
  __syncthreads();
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads, 2 x 8 outputs each
  for (int ri = 0; ri < 8; ri++) {
    const int r = ty * 8 + ri;
    if (i0 + r >= n) break;
#pragma unroll
    for (int cj = 0; cj < 2; cj++) {
      const int c = tx + 32 * cj;
      if (j0 + c >= n) continue;
      double t = 0.0;
#pragma unroll
      for (int q = 0; q < 16; q++) t = fma(sl[r][q], sx[c][q], t);
      double* g = &G[(int64_t)(i0 + r) * ldg + j0 + c];
      if (accumulate) *g -= t;
      else __stcs(g, -t);
    }
  }
}

// Y[i][:] = X[perm[i]][:] (gather) or Y[perm[i]][:] = X[i][:] (scatter)
__global__ void permute_rows_kernel(const double* X, int64_t ldx, double* Y, int64_t ldy, const int32_t* perm, int n,
                                    int k, int scatter) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * k) return;
  const int i = (int)(idx / k), c = (int)(idx - (int64_t)i * k);
  if (scatter) Y[(int64_t)perm[i] * ldy + c] = X[(int64_t)i * ldx + c];
  else Y[(int64_t)i * ldy + c] = X[(int64_t)perm[i] * ldx + c];
}

}  // namespace

int launch_trsm_pipe(const double* LU, int64_t lda, int n, double* Y, int64_t ldy, int nrhs, int mode, int* flags,
                     unsigned* ticket, DevStatus* st, long long spin, cudaStream_t s) {
  if (n <= 0 || nrhs <= 0) return LU_OK;
  const int nblk = ceil_div(n, TB);
  for (int c0 = 0; c0 < nrhs; c0 += 16) {
    const int k = std::min(16, nrhs - c0);
    LUB_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * nblk, s));
    LUB_CUDA(cudaMemsetAsync(ticket, 0, sizeof(unsigned), s));
    switch (mode) {
      case 0: trsm_pipe_kernel<0><<<nblk, 256, 0, s>>>(LU, lda, n, Y + c0, ldy, k, flags, ticket, st, spin); break;
      case 1: trsm_pipe_kernel<1><<<nblk, 256, 0, s>>>(LU, lda, n, Y + c0, ldy, k, flags, ticket, st, spin); break;
      case 2: trsm_pipe_kernel<2><<<nblk, 256, 0, s>>>(LU, lda, n, Y + c0, ldy, k, flags, ticket, st, spin); break;
      case 3: trsm_pipe_kernel<3><<<nblk, 256, 0, s>>>(LU, lda, n, Y + c0, ldy, k, flags, ticket, st, spin); break;
      default: return LU_ERR_ARG;
    }
    LUB_LAUNCH_CHECK();
  }
  return LU_OK;
}

int launch_neg_outer(const double* Lam, int64_t ldl, const double* X, int64_t ldx, int n, int k, double* G,
                     int64_t ldg, cudaStream_t s) {
  if (n <= 0 || k <= 0) return LU_OK;
  dim3 grid(ceil_div(n, 64), ceil_div(n, 64));
  for (int c0 = 0; c0 < k; c0 += 16) {
    neg_outer_kernel<<<grid, 256, 0, s>>>(Lam + c0, ldl, X + c0, ldx, n, std::min(16, k - c0), G, ldg, c0 > 0);
    LUB_LAUNCH_CHECK();
  }
  return LU_OK;
}

int launch_permute_rows(const double* X, int64_t ldx, double* Y, int64_t ldy, const int32_t* perm, int n, int k,
                        int scatter, cudaStream_t s) {
  const int64_t tot = (int64_t)n * k;
  if (tot <= 0) return LU_OK;
  permute_rows_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(X, ldx, Y, ldy, perm, n, k, scatter);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

template <typename T>
int launch_trsm_llu_leaf(const T* L, int64_t ldl, T* B, int64_t ldb, int m, int ncols, cudaStream_t s) {
  if (m <= 1 || ncols <= 0) return LU_OK;
  if (m > 32) return LU_ERR_ARG;
  trsm_llu_leaf_kernel<T><<<ceil_div(ncols, 128), 128, 0, s>>>(L, ldl, B, ldb, m, ncols);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

template <typename TS, typename T>
int launch_trsv_mixed(const TS* LU, int64_t lda, int n, T* x, int upper, int* flags, unsigned* ticket, DevStatus* st,
                      long long spin, cudaStream_t s) {
  if (n <= 0) return LU_OK;
  const int nblk = ceil_div(n, TB);
  LUB_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * nblk, s));
  LUB_CUDA(cudaMemsetAsync(ticket, 0, sizeof(unsigned), s));
  if (upper)
    trsv_kernel<TS, T, true><<<nblk, 256, 0, s>>>(LU, lda, n, x, flags, ticket, st, spin);
  else
    trsv_kernel<TS, T, false><<<nblk, 256, 0, s>>>(LU, lda, n, x, flags, ticket, st, spin);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

template <typename T>
int launch_trsv(const T* LU, int64_t lda, int n, T* x, int upper, int* flags, unsigned* ticket, DevStatus* st,
                long long spin, cudaStream_t s) {
  return launch_trsv_mixed<T, T>(LU, lda, n, x, upper, flags, ticket, st, spin, s);
}
template int launch_trsv_mixed<float, double>(const float*, int64_t, int, double*, int, int*, unsigned*, DevStatus*,
                                              long long, cudaStream_t);

template int launch_trsm_llu_leaf<double>(const double*, int64_t, double*, int64_t, int, int, cudaStream_t);
template int launch_trsm_llu_leaf<float>(const float*, int64_t, float*, int64_t, int, int, cudaStream_t);
template int launch_trsv<double>(const double*, int64_t, int, double*, int, int*, unsigned*, DevStatus*, long long,
                                 cudaStream_t);
template int launch_trsv<float>(const float*, int64_t, int, float*, int, int*, unsigned*, DevStatus*, long long,
                                cudaStream_t);

}  // namespace lub
