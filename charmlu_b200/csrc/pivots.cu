// Row interchanges (laswp) for a batch of pivots.
//
// The reference turns each batch of recorded pivots into permutation cycles
// (recordPivot / announceAgglomeratedPivots, lu.C:305-352) and every block
// applies them to its rows and to b (sendPendingPivots / applySwap,
// lu.C:46-169).  Here a batch of sequential swaps (k0+i) <-> p_i, p_i >=
// k0+i, is composed on the device into a simultaneous assignment
// row[dst] <- row[src] over the affected rows, then applied to column strips
// with every source read into shared memory before any destination is
// written (one read and one write per moved row segment, all independent).
//
// Composition (parallel, O(cnt^2) comparisons in shared memory):
//   c_i   = content of position k0+i just before swap i
//         = c_{a(i)} if a(i) = last i' < i with p_{i'} = k0+i exists, else k0+i
//           (resolved by pointer jumping);
//   final(k0+i) = c_{b(i)} if b(i) = last i' < i with p_{i'} = p_i exists,
//                 else p_i;
//   final(x) for x = p_i >= k0+cnt, i the last swap touching x: c_i.
#include "common.cuh"
#include "kernels.h"

namespace lub {
namespace {

// Computes dst/src lists in shared memory; returns m (same in all threads).
__device__ int compose_batch(const int32_t* ipiv, int k0, int cnt, int* p, int* nxt, int* lb, int* dst, int* src,
                             int* s_m) {
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i = tid; i < cnt; i += nt) p[i] = ipiv[k0 + i];
  if (tid == 0) *s_m = 0;
  __syncthreads();
  for (int i = tid; i < cnt; i += nt) {
    int la = -1, lbi = -1;
    const int me = k0 + i, pi = p[i];
    for (int q = 0; q < i; q++) {
      const int pq = p[q];
      if (pq == me) la = q;
      if (pq == pi) lbi = q;
    }
    nxt[i] = la < 0 ? i : la;
    lb[i] = lbi;
  }
  __syncthreads();
  for (int span = 1; span < cnt; span <<= 1) {
    int tmp[4];
    int k = 0;
    for (int i = tid; i < cnt && k < 4; i += nt, k++) tmp[k] = nxt[nxt[i]];
    __syncthreads();
    k = 0;
    for (int i = tid; i < cnt && k < 4; i += nt, k++) nxt[i] = tmp[k];
    __syncthreads();
  }
  // nxt[i] = root; c_i = k0 + root
  for (int i = tid; i < cnt; i += nt) {
    const int me = k0 + i, pi = p[i];
    const int s = lb[i] >= 0 ? k0 + nxt[lb[i]] : pi;
    if (s != me) {
      int o = atomicAdd(s_m, 1);
      dst[o] = me;
      src[o] = s;
    }
    if (pi >= k0 + cnt) {
      bool last = true;
      for (int q = i + 1; q < cnt; q++)
        if (p[q] == pi) { last = false; break; }
      if (last) {
        int o = atomicAdd(s_m, 1);
        dst[o] = pi;
        src[o] = k0 + nxt[i];
      }
    }
  }
  __syncthreads();
  return *s_m;
}

// rows > 0: the pivots must satisfy k0 + i <= p_i < rows (and k0 + cnt <=
// rows); otherwise the list is left empty, so nothing moves, and LU_ERR_ARG
// is recorded in st.
__global__ void __launch_bounds__(1024) pivot_compose_kernel(const int32_t* ipiv, int k0, int cnt, PivotList pl,
                                                            int rows, DevStatus* st) {
  __shared__ int p[kMaxBatch], nxt[kMaxBatch], lb[kMaxBatch];
  __shared__ int dst[2 * kMaxBatch], src[2 * kMaxBatch];
  __shared__ int s_m;
  if (rows > 0) {
    int bad = k0 + cnt > rows;
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
      const int pi = ipiv[k0 + i];
      bad |= (pi < k0 + i) | (pi >= rows);
    }
    if (__syncthreads_or(bad)) {
      if (threadIdx.x == 0) {
        *pl.m = 0;
        if (st) dev_fail(st, LU_ERR_ARG, 301);
      }
      return;
    }
  }
  const int m = compose_batch(ipiv, k0, cnt, p, nxt, lb, dst, src, &s_m);
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    pl.dst[i] = dst[i];
    pl.src[i] = src[i];
  }
  if (threadIdx.x == 0) *pl.m = m;
}

// One CTA per 128-byte column strip: every moved row's segment of the strip
// is read into registers (16-byte chunks, eight per thread, all loads in
// flight together), then, after one barrier, written to its destination.
// Chunks that straddle the strip's valid column range (or rows that are not
// 16-byte aligned, vec_ok = 0) go element by element.
constexpr int kApplyThreads = 1024;
constexpr int kApplyUnroll = 8;  // chunks per thread: 1024 rows x 8 chunks per strip

template <typename T>
__device__ __forceinline__ bool col_live(int cc, int c_begin, int c_end, int skip_begin, int skip_end) {
  return cc >= c_begin && cc < c_end && (cc < skip_begin || cc >= skip_end);
}

template <typename T>
__global__ void __launch_bounds__(kApplyThreads) pivot_apply_kernel(T* A, int64_t lda, int c_begin, int c_end,
                                                                   int skip_begin, int skip_end, PivotList pl,
                                                                   double* rhs, int32_t* perm, int vec_ok) {
  constexpr int EPC = 16 / (int)sizeof(T);  // elements per chunk
  constexpr int CS = 8 * EPC;               // elements per strip
  __shared__ double vb[2 * kMaxBatch];
  __shared__ int32_t pb[2 * kMaxBatch];
  const int m = *pl.m;
  const int tid = threadIdx.x;
  const int c0 = c_begin + blockIdx.x * CS;
  const bool strip_live = c0 < c_end && !(c0 >= skip_begin && c0 + CS <= skip_end);
  if (strip_live && m > 0) {
    uint4 v[kApplyUnroll];
#pragma unroll
    for (int u = 0; u < kApplyUnroll; u++) {
      const int pr = tid + u * kApplyThreads;
      const int i = pr >> 3, col = c0 + (pr & 7) * EPC;
      if (i < m) {
        const T* src = A + (int64_t)pl.src[i] * lda + col;
        if (vec_ok && col_live<T>(col, c_begin, c_end, skip_begin, skip_end) &&
            col_live<T>(col + EPC - 1, c_begin, c_end, skip_begin, skip_end)) {
          v[u] = __ldcs(reinterpret_cast<const uint4*>(src));
        } else {
          T tmp[EPC];
#pragma unroll
          for (int e = 0; e < EPC; e++)
            tmp[e] = col_live<T>(col + e, c_begin, c_end, skip_begin, skip_end) ? src[e] : T(0);
          memcpy(&v[u], tmp, 16);
        }
      }
    }
    __syncthreads();  // every source segment of the strip is in registers
#pragma unroll
    for (int u = 0; u < kApplyUnroll; u++) {
      const int pr = tid + u * kApplyThreads;
      const int i = pr >> 3, col = c0 + (pr & 7) * EPC;
      if (i < m) {
        T* dst = A + (int64_t)pl.dst[i] * lda + col;
        if (vec_ok && col_live<T>(col, c_begin, c_end, skip_begin, skip_end) &&
            col_live<T>(col + EPC - 1, c_begin, c_end, skip_begin, skip_end)) {
          __stcs(reinterpret_cast<uint4*>(dst), v[u]);
        } else {
          T tmp[EPC];
          memcpy(tmp, &v[u], 16);
#pragma unroll
          for (int e = 0; e < EPC; e++)
            if (col_live<T>(col + e, c_begin, c_end, skip_begin, skip_end)) dst[e] = tmp[e];
        }
      }
    }
  }
  if (blockIdx.x == 0 && m > 0 && (rhs || perm)) {
    __syncthreads();
    for (int i = tid; i < m; i += blockDim.x) {
      if (rhs) vb[i] = rhs[pl.src[i]];
      if (perm) pb[i] = perm[pl.src[i]];
    }
    __syncthreads();
    for (int i = tid; i < m; i += blockDim.x) {
      if (rhs) rhs[pl.dst[i]] = vb[i];
      if (perm) perm[pl.dst[i]] = pb[i];
    }
  }
}

// ipiv -> perm in two launches: every batch of 256 pivots is composed into
// its (dst <- src) list independently (one CTA per batch), then one CTA
// applies the lists to iota in batch order.  work: per batch 1 + 2 * 512
// ints (count, dst, src).
constexpr int kPermBatch = 256;
constexpr int kPermListInts = 1 + 4 * kPermBatch;

__global__ void __launch_bounds__(1024) perm_compose_kernel(const int32_t* ipiv, int n, int32_t* work) {
  __shared__ int p[kPermBatch], nxt[kPermBatch], lb[kPermBatch];
  __shared__ int dst[2 * kPermBatch], src[2 * kPermBatch];
  __shared__ int s_m;
  const int k0 = blockIdx.x * kPermBatch;
  const int cnt = min(kPermBatch, n - k0);
  const int m = compose_batch(ipiv, k0, cnt, p, nxt, lb, dst, src, &s_m);
  int32_t* w = work + (int64_t)blockIdx.x * kPermListInts;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    w[1 + i] = dst[i];
    w[1 + 2 * kPermBatch + i] = src[i];
  }
  if (threadIdx.x == 0) w[0] = m;
}

__global__ void __launch_bounds__(1024) perm_apply_lists_kernel(int n, int nb, const int32_t* work, int32_t* perm) {
  __shared__ int vals[2 * kPermBatch];
  for (int i = threadIdx.x; i < n; i += blockDim.x) perm[i] = i;
  __syncthreads();
  for (int b = 0; b < nb; b++) {
    const int32_t* w = work + (int64_t)b * kPermListInts;
    const int m = w[0];
    for (int i = threadIdx.x; i < m; i += blockDim.x) vals[i] = perm[w[1 + 2 * kPermBatch + i]];
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += blockDim.x) perm[w[1 + i]] = vals[i];
    __syncthreads();
  }
}

// x <- P x in place for an ipiv vector (all swaps in order), using only
// shared memory: batches of 256 pivots are composed and applied as one
// gather/scatter each.
__global__ void __launch_bounds__(1024) ipiv_apply_vector_kernel(const int32_t* ipiv, int n, double* x) {
  __shared__ int p[256], nxt[256], lb[256];
  __shared__ int dst[512], src[512];
  __shared__ double vals[512];
  __shared__ int s_m;
  for (int k0 = 0; k0 < n; k0 += 256) {
    const int cnt = min(256, n - k0);
    const int m = compose_batch(ipiv, k0, cnt, p, nxt, lb, dst, src, &s_m);
    for (int i = threadIdx.x; i < m; i += blockDim.x) vals[i] = x[src[i]];
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += blockDim.x) x[dst[i]] = vals[i];
    __syncthreads();
  }
}

}  // namespace

int launch_pivot_compose(const int32_t* ipiv, int k0, int cnt, const PivotList& pl, cudaStream_t s, int rows,
                         DevStatus* st) {
  if (cnt <= 0) return LU_OK;
  if (cnt > kMaxBatch) return LU_ERR_ARG;
  pivot_compose_kernel<<<1, 1024, 0, s>>>(ipiv, k0, cnt, pl, rows, st);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

template <typename T>
int launch_pivot_apply(T* A, int64_t lda, int c_begin, int c_end, int skip_begin, int skip_end, const PivotList& pl,
                       int max_m, double* rhs, int32_t* perm, cudaStream_t s) {
  constexpr int CS = 8 * (16 / (int)sizeof(T));
  if (c_end <= c_begin && !rhs && !perm) return LU_OK;
  if (max_m > 2 * kMaxBatch || max_m > kApplyThreads * kApplyUnroll / 8) return LU_ERR_ARG;
  const int vec_ok = ((lda * (int64_t)sizeof(T)) % 16 == 0) && (reinterpret_cast<uintptr_t>(A) % 16 == 0) &&
                     (c_begin % (16 / (int)sizeof(T)) == 0);
  const int strips = std::max(1, ceil_div(std::max(c_end - c_begin, 0), CS));
  pivot_apply_kernel<T><<<strips, kApplyThreads, 0, s>>>(A, lda, c_begin, c_end, skip_begin, skip_end, pl, rhs,
                                                          perm, vec_ok);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

int ipiv_to_perm_work_ints(int n) { return ceil_div(std::max(n, 1), kPermBatch) * kPermListInts; }

int launch_ipiv_to_perm(const int32_t* ipiv, int n, int32_t* perm, int32_t* work, cudaStream_t s) {
  if (n <= 0) return LU_OK;
  if (!work) return LU_ERR_ARG;
  const int nb = ceil_div(n, kPermBatch);
  perm_compose_kernel<<<nb, 1024, 0, s>>>(ipiv, n, work);
  LUB_LAUNCH_CHECK();
  perm_apply_lists_kernel<<<1, 1024, 0, s>>>(n, nb, work, perm);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

int launch_ipiv_apply_vector(const int32_t* ipiv, int n, double* x, cudaStream_t s) {
  if (n <= 0) return LU_OK;
  ipiv_apply_vector_kernel<<<1, 1024, 0, s>>>(ipiv, n, x);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

template int launch_pivot_apply<double>(double*, int64_t, int, int, int, int, const PivotList&, int, double*,
                                        int32_t*, cudaStream_t);
template int launch_pivot_apply<float>(float*, int64_t, int, int, int, int, const PivotList&, int, double*,
                                       int32_t*, cudaStream_t);

}  // namespace lub
