// Kernels of multi-right-hand-side iterative refinement (lu_refine_apply):
// the FP64 residual R = B - op(A) X for up to 16 columns, its per-column
// norms, and the correction update.  No reference counterpart (the
// reference solves one right-hand side in FP64, lu.ci:387-456); the scaled
// residual per column follows calcScaledResidual (benchmark.C:385-400) with
// ||op(A)||_inf (row sums of A, or column sums for the transposed system).
//
// The residual product reads A once per iteration (8 n^2 bytes) and does 16
// FMAs per element, so it sits at the FP64 pipe / HBM balance point: the
// kernel stages 16-deep slices of A and X through shared memory with
// cp.async (two stages) and each thread holds a 4 x 4 block of outputs.
// The reduction dimension is split over S block rows of the grid; partial
// results go to P[s] and a second kernel sums them in a fixed order, so the
// result does not depend on scheduling.
#include "common.cuh"
#include "kernels.h"

namespace lub {
namespace {

constexpr int RB = 256;        // outputs (rows of R) per block
constexpr int KC = 16;         // reduction slice per stage
constexpr int MR_THREADS = 256;
constexpr int LDT = KC + 2;    // row pitch of the non-transposed A stage (144 B, 16-byte aligned)

template <bool TRANS>
__host__ __device__ constexpr int a_stage_elems() { return TRANS ? KC * RB : RB * LDT; }
template <bool TRANS>
__host__ __device__ constexpr int stage_elems() { return a_stage_elems<TRANS>() + KC * 16; }
template <bool TRANS>
constexpr size_t mr_smem() { return 2 * sizeof(double) * stage_elems<TRANS>(); }

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(smem)), "l"(gmem), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// P[s][o][c] = sum over the split's reduction range of op(A)[o][k] X[k][c];
// with NORM also Pn[s][o] = sum |op(A)[o][k]|.  X has 16 columns (ld 16),
// zero beyond nrhs.  grid = (ceil(n / RB), S).
template <bool TRANS, bool NORM>
__global__ void __launch_bounds__(MR_THREADS, 2)
skinny_residual_kernel(const double* __restrict__ A, int64_t lda, int n, const double* __restrict__ X, int split_len,
                       double* __restrict__ P, double* __restrict__ Pn) {
  extern __shared__ __align__(16) double sm[];
  const int tid = threadIdx.x;
  const int o0 = blockIdx.x * RB;
  const int kbeg = blockIdx.y * split_len;
  const int kend = min(n, kbeg + split_len);
  const int nk = kbeg < kend ? (kend - kbeg + KC - 1) / KC : 0;
  const int rg = tid >> 2, cg = tid & 3;

  auto issue = [&](int it) {
    double* As = sm + (it & 1) * stage_elems<TRANS>();
    double* Xs = As + a_stage_elems<TRANS>();
    const int k0 = kbeg + it * KC;
    for (int ch = tid; ch < KC * RB / 2; ch += MR_THREADS) {
      if (TRANS) {
        // As[k][o] = A[k0 + k][o0 + o]
        const int k = ch / (RB / 2), o = (ch - k * (RB / 2)) * 2;
        const int gk = k0 + k, go = o0 + o;
        const int bytes = (gk < kend && go < n) ? (go + 1 < n ? 16 : 8) : 0;
        cp_async16(As + k * RB + o, bytes ? A + (int64_t)gk * lda + go : A, bytes);
      } else {
        // As[o][k] = A[o0 + o][k0 + k]
        const int o = ch / (KC / 2), k = (ch - o * (KC / 2)) * 2;
        const int gk = k0 + k, go = o0 + o;
        const int bytes = (go < n && gk < kend) ? (gk + 1 < kend ? 16 : 8) : 0;
        cp_async16(As + o * LDT + k, bytes ? A + (int64_t)go * lda + gk : A, bytes);
      }
    }
    if (tid < KC * 8) {
      const int k = tid >> 3, c = (tid & 7) * 2;
      const int gk = k0 + k;
      cp_async16(Xs + k * 16 + c, gk < kend ? X + (int64_t)gk * 16 + c : X, gk < kend ? 16 : 0);
    }
    cp_async_commit();
  };

  double acc[4][4];
  double nrm[4];
#pragma unroll
  for (int j = 0; j < 4; j++) {
    nrm[j] = 0.0;
#pragma unroll
    for (int e = 0; e < 4; e++) acc[j][e] = 0.0;
  }
  if (nk > 0) issue(0);
  for (int it = 0; it < nk; it++) {
    if (it + 1 < nk) {
      issue(it + 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double* As = sm + (it & 1) * stage_elems<TRANS>();
    const double* Xs = As + a_stage_elems<TRANS>();
#pragma unroll
    for (int k = 0; k < KC; k++) {
      double a[4];
#pragma unroll
      for (int j = 0; j < 4; j++) a[j] = TRANS ? As[k * RB + rg + 64 * j] : As[(rg + 64 * j) * LDT + k];
      const double2 x01 = *reinterpret_cast<const double2*>(Xs + k * 16 + 4 * cg);
      const double2 x23 = *reinterpret_cast<const double2*>(Xs + k * 16 + 4 * cg + 2);
#pragma unroll
      for (int j = 0; j < 4; j++) {
        acc[j][0] = fma(a[j], x01.x, acc[j][0]);
        acc[j][1] = fma(a[j], x01.y, acc[j][1]);
        acc[j][2] = fma(a[j], x23.x, acc[j][2]);
        acc[j][3] = fma(a[j], x23.y, acc[j][3]);
        if (NORM) nrm[j] += fabs(a[j]);
      }
    }
    __syncthreads();
  }
  double* Ps = P + (int64_t)blockIdx.y * n * 16;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int o = o0 + rg + 64 * j;
    if (o >= n) continue;
    double* dst = Ps + (int64_t)o * 16 + 4 * cg;
    *reinterpret_cast<double2*>(dst) = make_double2(acc[j][0], acc[j][1]);
    *reinterpret_cast<double2*>(dst + 2) = make_double2(acc[j][2], acc[j][3]);
    if (NORM && cg == 0) Pn[(int64_t)blockIdx.y * n + o] = nrm[j];
  }
}

__device__ __forceinline__ void atomic_max_bits(unsigned long long* a, double v) {
  // non-negative doubles (NaN: the positive quiet NaN, above every finite
  // value) order like their bit patterns
  atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

// R[o][c] = B[o][c] - sum_s P[s][o][c] for c < nrhs (0 beyond); per-column
// maxima of |R|, |B| and |X| into acc[0..15], acc[16..31], acc[32..47] and,
// with norm, max_o sum_s Pn[s][o] into acc[48].  Each block covers 256 rows.
__global__ void __launch_bounds__(256) mr_reduce_kernel(const double* __restrict__ P, const double* __restrict__ Pn,
                                                        int S, int n, const double* __restrict__ B, int64_t ldb,
                                                        int nrhs, const double* __restrict__ X, double* __restrict__ R,
                                                        unsigned long long* acc, int norm) {
  __shared__ double s_r[16][17], s_b[16][17], s_x[16][17], s_n[16];
  const int tid = threadIdx.x, ro = tid >> 4, c = tid & 15;
  double mr = 0.0, mb = 0.0, mx = 0.0, mn = 0.0;
  const int row_end = min(n, (blockIdx.x + 1) * 256);
  for (int o = blockIdx.x * 256 + ro; o < row_end; o += 16) {
    double r = 0.0;
    if (c < nrhs) {
      double sum = 0.0;
      for (int s = 0; s < S; s++) sum += P[((int64_t)s * n + o) * 16 + c];
      const double b = B[(int64_t)o * ldb + c];
      r = b - sum;
      const double ar = fabs(r);
      mr = (ar > mr || isnan(ar)) ? ar : mr;
      mb = fmax(mb, fabs(b));
      mx = fmax(mx, fabs(X[(int64_t)o * 16 + c]));
    }
    R[(int64_t)o * 16 + c] = r;
    if (norm && c == 0) {
      double t = 0.0;
      for (int s = 0; s < S; s++) t += Pn[(int64_t)s * n + o];
      mn = fmax(mn, t);
    }
  }
  s_r[ro][c] = mr;
  s_b[ro][c] = mb;
  s_x[ro][c] = mx;
  if (c == 0) s_n[ro] = mn;
  __syncthreads();
  if (tid < 16) {
    double a = 0.0, b = 0.0, x = 0.0;
    for (int q = 0; q < 16; q++) {
      const double v = s_r[q][tid];
      a = (v > a || isnan(v)) ? v : a;
      b = fmax(b, s_b[q][tid]);
      x = fmax(x, s_x[q][tid]);
    }
    if (tid < nrhs) {
      atomic_max_bits(&acc[tid], isnan(a) ? __longlong_as_double(0x7ff8000000000000LL) : a);
      atomic_max_bits(&acc[16 + tid], b);
      atomic_max_bits(&acc[32 + tid], x);
    }
  } else if (tid == 32 && norm) {
    double m = 0.0;
    for (int q = 0; q < 16; q++) m = fmax(m, s_n[q]);
    atomic_max_bits(&acc[48], m);
  }
}

// X[dst(i)][c] += D[i][c], dst(i) = perm[i] (scatter) or i; ld 16
__global__ void mr_add_kernel(double* X, const double* D, const int32_t* perm, int n, int nrhs, int scatter) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * 16) return;
  const int i = (int)(idx >> 4), c = (int)(idx & 15);
  if (c >= nrhs) return;
  const int d = scatter ? perm[i] : i;
  X[(int64_t)d * 16 + c] += D[idx];
}

// out[i] = M[src(i)][c] * scale, src(i) = perm[i] (gather) or i; M ld 16
__global__ void col_get_kernel(const double* M, int c, const int32_t* perm, double* out, int n, double scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = M[(int64_t)(perm ? perm[i] : i) * 16 + c] * scale;
}
// dst[perm[i]] = src[i]
__global__ void vec_scatter_kernel(const double* src, const int32_t* perm, double* dst, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[perm[i]] = src[i];
}
// D[i][c] = S[i][c] for one column of two ld-16 blocks
__global__ void col_copy_kernel(const double* S, double* D, int c, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) D[(int64_t)i * 16 + c] = S[(int64_t)i * 16 + c];
}
// M[i][c] = v[i] (assign) or M[i][c] += v[i]; M ld 16
__global__ void col_put_kernel(double* M, int c, const double* v, int n, int assign) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    double* d = &M[(int64_t)i * 16 + c];
    *d = assign ? v[i] : *d + v[i];
  }
}

template <bool TRANS, bool NORM>
int launch_skinny(const double* A, int64_t lda, int n, const double* X, int S, int split_len, double* P, double* Pn,
                  cudaStream_t s) {
  static PerDeviceOnce once;
  LUB_TRY(once_per_device(once, [] {
    return cuda_status(cudaFuncSetAttribute(skinny_residual_kernel<TRANS, NORM>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mr_smem<TRANS>()));
  }));
  dim3 grid(ceil_div(n, RB), S);
  skinny_residual_kernel<TRANS, NORM><<<grid, MR_THREADS, mr_smem<TRANS>(), s>>>(A, lda, n, X, split_len, P, Pn);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

}  // namespace

int multi_residual_splits(int n, int num_sms, int* split_len) {
  const int strips = ceil_div(n, RB);
  int S = std::max(1, std::min(kMultiMaxSplits, ceil_div(4 * num_sms, strips)));
  int len = ceil_div(ceil_div(n, S), KC) * KC;
  S = ceil_div(n, len);
  *split_len = len;
  return S;
}

int launch_multi_residual(const double* A, int64_t lda, int n, int trans, const double* X, const double* B,
                          int64_t ldb, int nrhs, double* R, double* P, double* Pn, int S, int split_len, int norm,
                          unsigned long long* acc, cudaStream_t s) {
  if (n <= 0) return LU_OK;
  if (nrhs < 1 || nrhs > 16 || S < 1 || S > kMultiMaxSplits || (split_len % KC) || (lda & 1) ||
      (reinterpret_cast<uintptr_t>(A) & 15) || (reinterpret_cast<uintptr_t>(X) & 15))
    return LU_ERR_ARG;
  if (trans) {
    if (norm) LUB_TRY((launch_skinny<true, true>(A, lda, n, X, S, split_len, P, Pn, s)));
    else LUB_TRY((launch_skinny<true, false>(A, lda, n, X, S, split_len, P, Pn, s)));
  } else {
    if (norm) LUB_TRY((launch_skinny<false, true>(A, lda, n, X, S, split_len, P, Pn, s)));
    else LUB_TRY((launch_skinny<false, false>(A, lda, n, X, S, split_len, P, Pn, s)));
  }
  LUB_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * kMultiAccWords, s));
  mr_reduce_kernel<<<ceil_div(n, 256), 256, 0, s>>>(P, Pn, S, n, B, ldb, nrhs, X, R, acc, norm);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

int launch_multi_add(double* X, const double* D, const int32_t* perm, int n, int nrhs, int scatter, cudaStream_t s) {
  const int64_t tot = (int64_t)n * 16;
  if (tot <= 0) return LU_OK;
  mr_add_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(X, D, perm, n, nrhs, scatter);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

int launch_col_get(const double* M, int c, const int32_t* perm, double* out, int n, double scale, cudaStream_t s) {
  if (n <= 0) return LU_OK;
  col_get_kernel<<<ceil_div(n, 256), 256, 0, s>>>(M, c, perm, out, n, scale);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

int launch_vec_scatter(const double* src, const int32_t* perm, double* dst, int n, cudaStream_t s) {
  if (n <= 0) return LU_OK;
  vec_scatter_kernel<<<ceil_div(n, 256), 256, 0, s>>>(src, perm, dst, n);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

int launch_col_copy(const double* S, double* D, int c, int n, cudaStream_t s) {
  if (n <= 0) return LU_OK;
  col_copy_kernel<<<ceil_div(n, 256), 256, 0, s>>>(S, D, c, n);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

int launch_col_put(double* M, int c, const double* v, int n, int assign, cudaStream_t s) {
  if (n <= 0) return LU_OK;
  col_put_kernel<<<ceil_div(n, 256), 256, 0, s>>>(M, c, v, n, assign);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

}  // namespace lub
