// Batched factor + solve of many independent systems of uneven order in one
// persistent launch (no reference counterpart: charmlu factors one
// distributed matrix).  Each system is LU with partial pivoting followed by
// forward/backward substitution, the same algorithm as the single-matrix
// path (strict '>' pivot search with the lowest row on ties, true division,
// swaps of whole rows and of b).
//
// Scheduling: a small prep kernel orders the systems by decreasing order
// (counting sort on n) and builds the workspace offsets; the persistent
// kernel's CTAs (one per SM, 512 threads) take systems from an atomic
// queue in that order, so the big systems start first and the small ones
// fill the tail (longest-processing-time-first balance).
//
// Per system (one CTA):
//   n <= small threshold  the whole matrix and b in shared memory, unblocked
//   otherwise             blocked right-looking LU in global memory (L2):
//                         an m x nb panel factored in shared memory, its
//                         swaps applied to the other columns and to b, the
//                         U row by forward substitution, the trailing update
//                         in 64 x 128 tiles with 4 x 4 register blocks per
//                         thread, the tiles' C and L blocks double-buffered
//                         in shared memory by async copies
//   then                  blocked forward / backward substitution
// On B200 the FP64 SIMT pipe has the same peak as FP64 DMMA, and these
// per-SM problems are too small for the tensor-core tiles, so FP64 here runs
// on the FP64 SIMT pipe.
//
// LU_PREC_FP32: the FP32 copy of each matrix (workspace) is factored, then
// FP64 refinement (r = b - A x against the FP64 A, FP32 correction solve,
// FP64 update) until the system's scaled residual r_hpl < 16, at most 10
// steps.  One step is not enough at these orders: after one step r_hpl is
// ~1e4 for a uniform n = 109 system (the remaining error lies along the
// small singular directions); two steps bring it to O(1).
#include <mutex>

#include "common.cuh"
#include "kernels.h"

namespace lub {
namespace {

constexpr int BT = 512;                    // threads per CTA
constexpr int NWARP = BT / 32;
constexpr int kBatchMaxN = 2048;
constexpr size_t kBatchSmem = 200 * 1024;  // dynamic shared memory per CTA
constexpr int kBatchRefineMax = 10;        // FP64 refinement steps at most (FP32 mode)

struct Tuning {
  int n_max, nb, small;
};
__constant__ Tuning c_tuning[16];
__constant__ int c_tuning_n;

struct BatchArgs {
  int count;
  const int* n;
  const int64_t* a_off;
  const int64_t* b_off;
  double* A;
  double* b;
  int* info;
  int precision;  // LU_PREC_FP64 or LU_PREC_FP32
  unsigned char* work;
};

// Workspace header written by the prep kernel (offsets in bytes from work).
constexpr int kRefineHistBins = kBatchRefineMax + 2;  // steps 0 .. 10, then "not converged"
struct WorkHeader {
  unsigned queue;
  int bad;          // nonzero: an order outside [1, kBatchMaxN] or workspace too small
  long long s1, s2; // sum n, sum n^2
  long long order, offA32, offV, piv, A32, r64, v32, total;
  // FP32 mode: systems that reached r_hpl < 16 after s FP64 refinement
  // steps (s = 0 .. 10), and in the last bin those that did not
  int refine_hist[kRefineHistBins];
};
static_assert(sizeof(WorkHeader) <= 256, "workspace header exceeds its 256 bytes");

__device__ __forceinline__ void tuning_for(int n, int esize, int& nb, int& small) {
  nb = esize == 8 ? 16 : 32;
  small = esize == 8 ? 128 : 192;
  for (int i = 0; i < c_tuning_n; i++) {
    if (n <= c_tuning[i].n_max) {
      nb = c_tuning[i].nb;
      small = c_tuning[i].small;
      break;
    }
  }
  // shared-memory caps: small path n x (n+1); blocked path panel m x (nb+1) + nb x 128 staging
  const int small_cap = (int)(sqrtf((float)(kBatchSmem / esize)) - 1.f);
  if (small > small_cap) small = small_cap;
  // the update phase reuses the same space: a U slice and two L tiles of
  // depth up to the outer block width
  const size_t ob = esize == 8 ? 64 : 128;
  while (nb > 4) {
    const size_t panel_phase = (size_t)n * (nb + 1) + (size_t)nb * 128;
    const size_t update_phase = ob * 128 + (size_t)2 * 64 * ob;
    if ((panel_phase > update_phase ? panel_phase : update_phase) * esize <= kBatchSmem) break;
    nb >>= 1;
  }
}

template <typename T>
__device__ __forceinline__ bool better(T v1, int r1, T v2, int r2) {
  return r1 >= 0 && (r2 < 0 || v1 > v2 || (v1 == v2 && r1 < r2));
}

// block-wide argmax (value, row); lowest row on ties; -1 if no positive value.
// One barrier: every warp reduces the NWARP per-warp candidates itself.  The
// caller puts a barrier between the return and its next call (the slots are
// reused).
template <typename T>
__device__ int block_argmax(T v, int r, T* sv, int* sr) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T v2 = __shfl_xor_sync(0xffffffffu, v, o);
    int r2 = __shfl_xor_sync(0xffffffffu, r, o);
    if (better(v2, r2, v, r)) { v = v2; r = r2; }
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { sv[warp] = v; sr[warp] = r; }
  __syncthreads();
  v = lane < NWARP ? sv[lane] : T(0);
  r = lane < NWARP ? sr[lane] : -1;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T v2 = __shfl_xor_sync(0xffffffffu, v, o);
    int r2 = __shfl_xor_sync(0xffffffffu, r, o);
    if (better(v2, r2, v, r)) { v = v2; r = r2; }
  }
  return r;
}

// Unblocked LU with partial pivoting of an m x w block in shared memory
// (pitch ld), rows global row0.. ; pivots (local rows) into piv_s[w].
// Columns beyond w are not touched.  Returns the 1-based first zero pivot.
template <typename T>
__device__ int getf2_smem(T* a, int ld, int m, int w, int* piv_s, T* sv, int* sr) {
  int info = 0;
  const int tid = threadIdx.x;
  // candidate of column 0; later candidates come out of the update pass
  T bv = 0;
  int br = -1;
  for (int i = tid; i < m; i += BT) {
    const T v = fabs(a[i * ld]);
    if (v > bv) { bv = v; br = i; }
  }
  for (int j = 0; j < w && j < m; j++) {
    // its barrier also ends the previous update; the barrier after the
    // swap separates this call from the next
    int p = block_argmax(bv, br, sv, sr);
    if (p < 0) {
      p = j;
      if (info == 0) info = j + 1;
    }
    if (tid == 0) piv_s[j] = p;
    if (p != j)
      for (int c = tid; c < w; c += BT) {
        const T t = a[j * ld + c];
        a[j * ld + c] = a[p * ld + c];
        a[p * ld + c] = t;
      }
    __syncthreads();
    // one pass per row: multiplier (true division), rank-1 update of the
    // rest of the block, and the candidate of column j + 1
    const T piv = a[j * ld + j];
    const bool do_scale = piv != T(0) && !isnan(piv);
    bv = 0;
    br = -1;
    for (int i = j + 1 + tid; i < m; i += BT) {
      T* ar = a + i * ld;
      if (do_scale) {
        const T l = ar[j] / piv;
        ar[j] = l;
        for (int c = j + 1; c < w; c++) ar[c] = fma(-l, a[j * ld + c], ar[c]);
      }
      if (j + 1 < w) {
        const T v = fabs(ar[j + 1]);
        if (v > bv) { bv = v; br = i; }
      }
    }
  }
  __syncthreads();
  return info;
}

// Blocked forward (unit L) and backward (U) substitution in global memory,
// 32-row blocks: a warp-parallel GEMV over the solved part, then one warp
// substitutes inside the 32 x 32 diagonal block.
template <typename T>
__device__ void solve_global(const T* LU, int n, T* x, T* s_acc) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int I0 = 0; I0 < n; I0 += 32) {
    const int rows = min(32, n - I0);
    for (int i = warp; i < rows; i += NWARP) {
      const T* row = LU + (int64_t)(I0 + i) * n;
      T acc = 0;
      for (int j = lane; j < I0; j += 32) acc = fma(row[j], x[j], acc);
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) s_acc[i] = acc;
    }
    __syncthreads();
    if (warp == 0) {
      T v = lane < rows ? x[I0 + lane] - s_acc[lane] : T(0);
      for (int j = 0; j < rows; j++) {
        const T xj = __shfl_sync(0xffffffffu, v, j);
        if (lane > j && lane < rows) v = fma(-LU[(int64_t)(I0 + lane) * n + I0 + j], xj, v);
      }
      if (lane < rows) x[I0 + lane] = v;
    }
    __syncthreads();
  }
  const int nblk = (n + 31) / 32;
  for (int bi = nblk - 1; bi >= 0; bi--) {
    const int I0 = bi * 32, rows = min(32, n - I0), J0 = I0 + rows;
    for (int i = warp; i < rows; i += NWARP) {
      const T* row = LU + (int64_t)(I0 + i) * n;
      T acc = 0;
      for (int j = J0 + lane; j < n; j += 32) acc = fma(row[j], x[j], acc);
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) s_acc[i] = acc;
    }
    __syncthreads();
    if (warp == 0) {
      T v = lane < rows ? x[I0 + lane] - s_acc[lane] : T(0);
      for (int j = rows - 1; j >= 0; j--) {
        if (lane == j) v = v / LU[(int64_t)(I0 + j) * n + I0 + j];
        const T xj = __shfl_sync(0xffffffffu, v, j);
        if (lane < j) v = fma(-LU[(int64_t)(I0 + lane) * n + I0 + j], xj, v);
      }
      if (lane < rows) x[I0 + lane] = v;
    }
    __syncthreads();
  }
}

// Element copy global -> shared through the async copy unit; pred false
// zero-fills the destination (src-size 0: nothing is read).
template <int BYTES>
__device__ __forceinline__ void cp_async_elem(void* sdst, const void* gsrc, bool pred) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(smem_u32(sdst)), "l"(gsrc), "n"(BYTES),
               "r"(pred ? BYTES : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit_group() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Outer block width of the two-level blocking: the inner panels (nb
// columns) update only the outer block's own columns and U rows; the rest of
// the trailing matrix gets one update of depth kOuter per outer block.
template <typename T>
constexpr int outer_block() { return sizeof(T) == 8 ? 64 : 128; }

// C[r0:r1, c0:c1] -= A[r0:r1, kk0:kk0+K] * A[kk0:kk0+K, c0:c1] (K <=
// outer_block<T>(); the L and U blocks final in global memory) over TM x TN
// tiles, a 4 x 4 block of outputs per thread: rows tr*4 .. +3, columns
// tc + (TN/4) j (consecutive across the lanes of a column group: conflict-free
// shared reads of U and coalesced global accesses; a warp spans 32*4/TN row
// groups, whose L rows sit in distinct banks with the pitch K + 1).  Shapes:
// 64 x 128 for the outer block's trailing update, 256 x 32 for the narrow
// update of its own columns, 32 x 256 for its U rows.  Per column tile the U
// slice is staged once; the row tiles' L blocks stream through two shared
// buffers with the async copy unit.  Each thread's C values are loaded at
// the start of its tile and subtracted after the products are summed, so
// their latency hides behind the k loop.
// smem (reusing the panel's space):  Ut [K][TN] | Lt[2] [TM][K+1]
template <typename T, int TM, int TN>
__device__ void update_block(T* A, int n, int r0, int r1, int c0, int c1, int kk0, int K, unsigned char* smem) {
  static_assert((TM / 4) * (TN / 4) == BT, "one 4 x 4 block of outputs per thread");
  constexpr int GX = TN / 4;
  if (r0 >= r1 || c0 >= c1 || K <= 0) return;
  const int tid = threadIdx.x, tr = tid / GX, tc = tid % GX;
  const int KP = K + 1;
  T* ut = reinterpret_cast<T*>(smem);
  T* lt = ut + (size_t)K * TN;
  const int nrt = (r1 - r0 + TM - 1) / TM;
  auto issue = [&](int t, int buf) {
    const int rt = r0 + t * TM;
    T* ldst = lt + (size_t)buf * TM * KP;
    for (int idx = tid; idx < TM * K; idx += BT) {
      const int r = idx / K, p = idx - r * K;
      const bool ok = rt + r < r1;
      cp_async_elem<sizeof(T)>(ldst + r * KP + p, ok ? A + (int64_t)(rt + r) * n + kk0 + p : A, ok);
    }
    cp_async_commit_group();
  };
  for (int ct = c0; ct < c1; ct += TN) {
    // U slice (K x TN): all of a thread's loads in flight together
    for (int base = 0; base < K * TN; base += BT * 8) {
      T v[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int idx = base + tid + u * BT;
        const int p = idx / TN, c = idx % TN;
        v[u] = (idx < K * TN && ct + c < c1) ? A[(int64_t)(kk0 + p) * n + ct + c] : T(0);
      }
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int idx = base + tid + u * BT;
        if (idx < K * TN) ut[idx] = v[u];
      }
    }
    issue(0, 0);
    for (int t = 0; t < nrt; t++) {
      const int buf = t & 1;
      const int rbase = r0 + t * TM + tr * 4;
      T cv[4][4];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const int r = rbase + i, c = ct + tc + GX * j;
          cv[i][j] = (r < r1 && c < c1) ? A[(int64_t)r * n + c] : T(0);
        }
      if (t + 1 < nrt) {
        issue(t + 1, buf ^ 1);
        cp_async_wait_group<1>();
      } else {
        cp_async_wait_group<0>();
      }
      __syncthreads();  // L tile t (and, at t = 0, the U slice) in shared memory
      const T* ls = lt + (size_t)buf * TM * KP + (size_t)tr * 4 * KP;
      T acc[4][4];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = T(0);
      for (int p = 0; p < K; p++) {
        T av[4], bv[4];
#pragma unroll
        for (int i = 0; i < 4; i++) av[i] = ls[i * KP + p];
#pragma unroll
        for (int j = 0; j < 4; j++) bv[j] = ut[p * TN + tc + GX * j];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int j = 0; j < 4; j++) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
      }
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int r = rbase + i;
        if (r >= r1) break;
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const int c = ct + tc + GX * j;
          if (c < c1) A[(int64_t)r * n + c] = cv[i][j] - acc[i][j];
        }
      }
      __syncthreads();  // buffer `buf` (and the U slice after the last tile) free for reuse
    }
  }
}

// First q < np with key[q] == v, found by one warp (all lanes get it); -1 if none.
__device__ __forceinline__ int warp_find(const int* key, int np, int v) {
  const int lane = threadIdx.x & 31;
  for (int base = 0; base < np; base += 32) {
    const unsigned m = __ballot_sync(0xffffffffu, base + lane < np && key[base + lane] == v);
    if (m) return base + __ffs(m) - 1;
  }
  return -1;
}

// One warp: the interchanges (K0 + j) <-> piv[K0 + j], j = 0 .. S-1, in order,
// composed into one simultaneous assignment row mdst[q] <- row msrc[q]
// (q < the returned count, at most 2 S rows); pos / cont are scratch of 2 S.
__device__ int compose_moves(const int* piv, int K0, int S, int* pos, int* cont, int* mdst, int* msrc) {
  const int lane = threadIdx.x & 31;
  int np = 0;
  for (int j = 0; j < S; j++) {
    const int a = K0 + j, b = piv[K0 + j];
    if (a == b) continue;
    int ia = warp_find(pos, np, a);
    if (ia < 0) {
      if (lane == 0) { pos[np] = a; cont[np] = a; }
      ia = np++;
      __syncwarp();
    }
    int ib = warp_find(pos, np, b);
    if (ib < 0) {
      if (lane == 0) { pos[np] = b; cont[np] = b; }
      ib = np++;
      __syncwarp();
    }
    if (lane == 0) {
      const int t = cont[ia];
      cont[ia] = cont[ib];
      cont[ib] = t;
    }
    __syncwarp();
  }
  int mm = 0;
  for (int base = 0; base < np; base += 32) {
    const int q = base + lane;
    const bool mv = q < np && pos[q] != cont[q];
    const unsigned m = __ballot_sync(0xffffffffu, mv);
    if (mv) {
      const int o = mm + __popc(m & ((1u << lane) - 1u));
      mdst[o] = pos[q];
      msrc[o] = cont[q];
    }
    mm += __popc(m);
  }
  __syncwarp();
  return mm;
}

// Row moves A[mdst[q], ca:cb] <- A[msrc[q], ca:cb] (q < mm <= 256), every
// source read before any destination is written: 128-column chunks staged in
// shared memory (buf, mm x 128 elements), 16 loads in flight per thread.
template <typename T>
__device__ void apply_moves(T* A, int n, const int* mdst, const int* msrc, int mm, int ca, int cb, T* buf) {
  const int tid = threadIdx.x;
  const int tot = mm * 128;
  for (int c0 = ca; c0 < cb; c0 += 128) {
    const int w = min(128, cb - c0);
    for (int base = 0; base < tot; base += BT * 16) {
      T v[16];
#pragma unroll
      for (int u = 0; u < 16; u++) {
        const int idx = base + tid + u * BT;
        const int q = idx >> 7, c = idx & 127;
        v[u] = (idx < tot && c < w) ? A[(int64_t)msrc[q] * n + c0 + c] : T(0);
      }
#pragma unroll
      for (int u = 0; u < 16; u++) {
        const int idx = base + tid + u * BT;
        if (idx < tot) buf[idx] = v[u];
      }
    }
    __syncthreads();
    for (int idx = tid; idx < tot; idx += BT) {
      const int q = idx >> 7, c = idx & 127;
      if (c < w) A[(int64_t)mdst[q] * n + c0 + c] = buf[idx];
    }
    __syncthreads();
  }
}

// U rows: A[k0:k0+kw, c0:c1] <- L^{-1} A[k0:k0+kw, c0:c1], L the kw x kw
// unit-lower block at lsm (pitch ld, shared memory); one column per thread.
template <typename T>
__device__ void u_rows(T* A, int n, int k0, int kw, int c0, int c1, const T* lsm, int ld) {
  for (int c = c0 + threadIdx.x; c < c1; c += BT) {
    T u[32];
#pragma unroll
    for (int i = 0; i < 32; i++) u[i] = i < kw ? A[(int64_t)(k0 + i) * n + c] : T(0);
#pragma unroll
    for (int i = 1; i < 32; i++) {
      if (i >= kw) break;
#pragma unroll
      for (int p = 0; p < 32; p++) {
        if (p >= i) break;
        u[i] = fma(-lsm[i * ld + p], u[p], u[i]);
      }
    }
#pragma unroll
    for (int i = 0; i < 32; i++)
      if (i < kw) A[(int64_t)(k0 + i) * n + c] = u[i];
  }
}

// Factor A (n x n row-major in global, ld = n) in place, recording the
// pivots (global rows, LAPACK order) in piv; the caller permutes b.
template <typename T>
__device__ int factor_system(T* A, int n, int* piv, unsigned char* smem, T* sv, int* sr, int* piv_s) {
  const int tid = threadIdx.x;
  int nb, small;
  tuning_for(n, (int)sizeof(T), nb, small);
  if (n <= small) {
    const int ld = n + 1;
    T* a = reinterpret_cast<T*>(smem);
    for (int idx = tid; idx < n * n; idx += BT) a[(idx / n) * ld + idx % n] = A[idx];
    __syncthreads();
    const int info = getf2_smem(a, ld, n, n, piv_s, sv, sr);
    for (int j = tid; j < n; j += BT) piv[j] = piv_s[j];
    for (int idx = tid; idx < n * n; idx += BT) A[idx] = a[(idx / n) * ld + idx % n];
    __syncthreads();
    return info;
  }
  int info = 0;
  const int ld = nb + 1;
  T* panel = reinterpret_cast<T*>(smem);                  // n x (nb+1)
  __shared__ int sw_dst[64], sw_src[64], sw_m;             // composed row moves of a panel
  // an outer block's composed interchanges (at most 2 x outer_block rows)
  __shared__ int s_pos[256], s_cont[256], s_mdst[256], s_msrc[256];
  for (int k0 = 0; k0 < n; k0 += nb) {
    const int kw = min(nb, n - k0), m = n - k0;
    // panel in: eight loads in flight per thread
    for (int base = 0; base < m * kw; base += BT * 8) {
      T v[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int idx = base + tid + u * BT;
        const int i = idx / kw, c = idx - i * kw;
        v[u] = idx < m * kw ? A[(int64_t)(k0 + i) * n + k0 + c] : T(0);
      }
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int idx = base + tid + u * BT;
        const int i = idx / kw, c = idx - i * kw;
        if (idx < m * kw) panel[i * ld + c] = v[u];
      }
    }
    __syncthreads();
    const int pi = getf2_smem(panel, ld, m, kw, piv_s, sv, sr);
    if (pi && !info) info = k0 + pi;
    for (int idx = tid; idx < m * kw; idx += BT) {
      const int i = idx / kw, c = idx - i * kw;
      A[(int64_t)(k0 + i) * n + k0 + c] = panel[i * ld + c];
    }
    // Two-level blocking.  Inside an outer block of NB columns each panel
    // swaps rows, solves its U rows and updates all rows below only within
    // the outer block's columns.  The columns left and right of the outer
    // block are untouched until its last panel: then its interchanges,
    // composed into one assignment of rows, are applied to them in one pass;
    // its U rows right of it are solved (blocked forward substitution with its
    // unit-lower L11); and the rest of the trailing matrix gets one update of
    // depth NB.
    constexpr int NB = outer_block<T>();
    const int K0 = k0 - k0 % NB, Kend = min(n, K0 + NB);
    const int c1 = k0 + kw;
    // this panel's swaps (the pivot record, then one warp composes them into
    // one assignment of the affected rows: row dst <- row src, at most 2 kw
    // moves), applied to the outer block's other columns with every source
    // read before any destination is written
    for (int j = tid; j < kw; j += BT) piv[k0 + j] = k0 + piv_s[j];
    __syncthreads();
    if (tid < 32) {
      const int mm = compose_moves(piv, k0, kw, s_pos, s_cont, sw_dst, sw_src);
      if (tid == 0) sw_m = mm;
    }
    __syncthreads();
    {
      // at most NB - kw <= 120 columns: four threads per column, each a
      // quarter of the moves (<= 16)
      const int mm = sw_m, nleft = k0 - K0, ncols = nleft + (Kend - c1);
      const int q4 = tid & 3, c = tid >> 2;
      const bool live = c < ncols;
      const int col = c < nleft ? K0 + c : c1 + (c - nleft);
      T v[16];
#pragma unroll
      for (int u = 0; u < 16; u++) {
        const int q = q4 + 4 * u;
        v[u] = (live && q < mm) ? A[(int64_t)sw_src[q] * n + col] : T(0);
      }
      __syncthreads();
#pragma unroll
      for (int u = 0; u < 16; u++) {
        const int q = q4 + 4 * u;
        if (live && q < mm) A[(int64_t)sw_dst[q] * n + col] = v[u];
      }
      __syncthreads();
    }
    if (c1 < Kend) {
      u_rows<T>(A, n, k0, kw, c1, Kend, panel, ld);
      __syncthreads();
      update_block<T, 256, 32>(A, n, c1, n, c1, Kend, k0, kw, smem);
      continue;
    }
    // the outer block's last panel: its interchanges on the other columns
    if (tid < 32) {
      const int mm = compose_moves(piv, K0, Kend - K0, s_pos, s_cont, s_mdst, s_msrc);
      if (tid == 0) sw_m = mm;
    }
    __syncthreads();
    apply_moves<T>(A, n, s_mdst, s_msrc, sw_m, 0, K0, reinterpret_cast<T*>(smem));
    apply_moves<T>(A, n, s_mdst, s_msrc, sw_m, Kend, n, reinterpret_cast<T*>(smem));
    if (Kend >= n) break;
    T* dg = reinterpret_cast<T*>(smem);  // [32][33]: one diagonal block of L11
    for (int q0 = K0; q0 < Kend; q0 += nb) {
      const int qw = min(nb, Kend - q0);
      for (int idx = tid; idx < qw * qw; idx += BT) {
        const int i = idx / qw, p = idx - i * qw;
        dg[i * 33 + p] = A[(int64_t)(q0 + i) * n + q0 + p];
      }
      __syncthreads();
      u_rows<T>(A, n, q0, qw, Kend, n, dg, 33);
      __syncthreads();
      update_block<T, 32, 256>(A, n, q0 + qw, Kend, Kend, n, q0, qw, smem);
    }
    update_block<T, 64, 128>(A, n, Kend, n, Kend, n, K0, Kend - K0, smem);
  }
  return info;
}

// perm[i] = the original row that the interchanges j <-> piv[j] (j = 0 ..
// n-1, in order) bring to row i; piv is copied to shared memory (scratch, n
// ints) and one thread composes the sequence there.
__device__ void pivots_to_perm(const int* piv, int n, int* perm, int* scratch) {
  const int tid = threadIdx.x;
  for (int i = tid; i < n; i += BT) {
    perm[i] = i;
    scratch[i] = piv[i];
  }
  __syncthreads();
  if (tid == 0)
    for (int j = 0; j < n; j++) {
      const int p = scratch[j];
      if (p != j) {
        const int t = perm[j];
        perm[j] = perm[p];
        perm[p] = t;
      }
    }
  __syncthreads();
}

// x <- P x, x[i] <- x[perm[i]], through shared memory (buf: n elements)
template <typename T>
__device__ void gather_perm(T* x, int n, const int* perm, T* buf) {
  for (int i = threadIdx.x; i < n; i += BT) buf[i] = x[perm[i]];
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += BT) x[i] = buf[i];
  __syncthreads();
}

__global__ void __launch_bounds__(BT, 1) batched_kernel(BatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  WorkHeader* hdr = reinterpret_cast<WorkHeader*>(a.work);
  if (ld_acquire_s32(&hdr->bad) != 0) return;
  const int* order = reinterpret_cast<const int*>(a.work + hdr->order);
  const int64_t* offA32 = reinterpret_cast<const int64_t*>(a.work + hdr->offA32);
  const int64_t* offV = reinterpret_cast<const int64_t*>(a.work + hdr->offV);
  int* pivs = reinterpret_cast<int*>(a.work + hdr->piv);
  float* A32s = reinterpret_cast<float*>(a.work + hdr->A32);
  double* r64s = reinterpret_cast<double*>(a.work + hdr->r64);
  float* v32s = reinterpret_cast<float*>(a.work + hdr->v32);
  __shared__ double sv_d[NWARP];
  __shared__ float sv_f[NWARP];
  __shared__ int sr[NWARP];
  __shared__ int piv_s[kBatchMaxN];
  __shared__ double s_acc_d[32];
  __shared__ float s_acc_f[32];
  __shared__ int s_idx;
  __shared__ double s_red[4][NWARP];
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) s_idx = (int)atomicAdd(&hdr->queue, 1u);
    __syncthreads();
    const int q = s_idx;
    __syncthreads();
    if (q >= a.count) break;
    const int sys = order[q];
    const int n = a.n[sys];
    double* A = a.A + a.a_off[sys];
    double* b = a.b + a.b_off[sys];
    int* piv = pivs + offV[sys];
    int info = 0;
    if (a.precision == LU_PREC_FP64) {
      info = factor_system<double>(A, n, piv, smem, sv_d, sr, piv_s);
      __syncthreads();
      pivots_to_perm(piv, n, piv_s, reinterpret_cast<int*>(smem));
      gather_perm<double>(b, n, piv_s, reinterpret_cast<double*>(smem));
      solve_global<double>(A, n, b, s_acc_d);
    } else {
      float* A32 = A32s + offA32[sys];
      float* v = v32s + offV[sys];
      double* r = r64s + 2 * offV[sys];  // [r | b] per system
      for (int idx = tid; idx < n * n; idx += BT) A32[idx] = (float)A[idx];
      for (int i = tid; i < n; i += BT) {
        r[n + i] = b[i];  // keep b for the residual
        v[i] = (float)b[i];
      }
      __syncthreads();
      info = factor_system<float>(A32, n, piv, smem, sv_f, sr, piv_s);
      __syncthreads();
      // piv_s keeps the permutation for the refinement steps
      pivots_to_perm(piv, n, piv_s, reinterpret_cast<int*>(smem));
      gather_perm<float>(v, n, piv_s, reinterpret_cast<float*>(smem));
      solve_global<float>(A32, n, v, s_acc_f);
      // x = v, then FP64 refinement: r = b - A x (against the FP64 A), stop
      // when the scaled residual r_hpl < 16, else v = P r, FP32 solve, x += v
      for (int i = tid; i < n; i += BT) b[i] = (double)v[i];
      __syncthreads();
      const int warp = tid >> 5, lane = tid & 31;
      double anorm = 0.0, bmax = 0.0;
      for (int step = 0;; step++) {
        double rmax = 0.0, xmax = 0.0, an = 0.0;
        for (int i = warp; i < n; i += NWARP) {
          const double* row = A + (int64_t)i * n;
          double acc = 0.0, as = 0.0;
          for (int j = lane; j < n; j += 32) {
            acc = fma(row[j], b[j], acc);
            if (step == 0) as += fabs(row[j]);
          }
          for (int o = 16; o > 0; o >>= 1) {
            acc += __shfl_xor_sync(0xffffffffu, acc, o);
            as += __shfl_xor_sync(0xffffffffu, as, o);
          }
          if (lane == 0) {
            const double ri = r[i + n] - acc;  // r[n + i] keeps b
            r[i] = ri;
            rmax = fmax(rmax, fabs(ri));
            an = fmax(an, as);
          }
        }
        for (int i = tid; i < n; i += BT) xmax = fmax(xmax, fabs(b[i]));
        if (step == 0)
          for (int i = tid; i < n; i += BT) bmax = fmax(bmax, fabs(r[i + n]));
        // block maxima
        for (int o = 16; o > 0; o >>= 1) {
          rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
          xmax = fmax(xmax, __shfl_xor_sync(0xffffffffu, xmax, o));
          an = fmax(an, __shfl_xor_sync(0xffffffffu, an, o));
          bmax = fmax(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
        }
        if (lane == 0) { s_red[0][warp] = rmax; s_red[1][warp] = xmax; s_red[2][warp] = an; s_red[3][warp] = bmax; }
        __syncthreads();
        if (tid == 0) {
          double m0 = 0, m1 = 0, m2 = 0, m3 = 0;
          for (int w = 0; w < NWARP; w++) {
            m0 = fmax(m0, s_red[0][w]); m1 = fmax(m1, s_red[1][w]);
            m2 = fmax(m2, s_red[2][w]); m3 = fmax(m3, s_red[3][w]);
          }
          s_red[0][0] = m0; s_red[1][0] = m1; s_red[2][0] = m2; s_red[3][0] = m3;
        }
        __syncthreads();
        rmax = s_red[0][0];
        xmax = s_red[1][0];
        if (step == 0) { anorm = s_red[2][0]; bmax = s_red[3][0]; }
        __syncthreads();
        const double r_hpl = rmax / ((anorm * xmax + bmax) * (double)n * 2.220446049250313e-16);
        if (isnan(r_hpl)) {
          if (info == 0) info = LU_ERR_NONFINITE;
          if (tid == 0) atomicAdd(&hdr->refine_hist[kRefineHistBins - 1], 1);
          break;
        }
        if (r_hpl < 16.0) {
          if (tid == 0) atomicAdd(&hdr->refine_hist[step], 1);
          break;
        }
        if (step == kBatchRefineMax) {
          if (info == 0) info = LU_ERR_NOCONV;
          if (tid == 0) atomicAdd(&hdr->refine_hist[kRefineHistBins - 1], 1);
          break;
        }
        for (int i = tid; i < n; i += BT) v[i] = (float)r[piv_s[i]];
        __syncthreads();
        solve_global<float>(A32, n, v, s_acc_f);
        for (int i = tid; i < n; i += BT) b[i] += (double)v[i];
        __syncthreads();
      }
    }
    if (tid == 0) a.info[sys] = info;
    __syncthreads();
  }
}

__host__ __device__ inline long long align256(long long x) { return (x + 255) & ~255LL; }

// Order systems by decreasing n (counting sort on n), prefix offsets of the
// per-system workspace regions, and the workspace layout.  One CTA.
__global__ void __launch_bounds__(1024) batched_prep_kernel(int count, const int* n, int precision,
                                                            unsigned char* work, long long work_bytes,
                                                            int* info) {
  __shared__ int hist[kBatchMaxN + 1];
  __shared__ int s_bad;
  WorkHeader* hdr = reinterpret_cast<WorkHeader*>(work);
  const int tid = threadIdx.x;
  long long o = 256;
  const long long o_order = o;
  o = align256(o + 4LL * count);
  const long long o_offA32 = o;
  o = align256(o + 8LL * count);
  const long long o_offV = o;
  o = align256(o + 8LL * count);
  int* order = reinterpret_cast<int*>(work + o_order);
  int64_t* offA32 = reinterpret_cast<int64_t*>(work + o_offA32);
  int64_t* offV = reinterpret_cast<int64_t*>(work + o_offV);
  for (int i = tid; i <= kBatchMaxN; i += blockDim.x) hist[i] = 0;
  if (tid == 0) s_bad = 0;
  __syncthreads();
  for (int i = tid; i < count; i += blockDim.x) {
    const int v = n[i];
    if (v < 1 || v > kBatchMaxN) { atomicAdd(&s_bad, 1); continue; }
    atomicAdd(&hist[v], 1);
  }
  __syncthreads();
  if (tid == 0) {
    int acc = 0;  // descending start positions
    for (int v = kBatchMaxN; v >= 1; v--) {
      const int c = hist[v];
      hist[v] = acc;
      acc += c;
    }
    long long s2 = 0, s1 = 0;
    for (int i = 0; i < count; i++) {
      const int v = n[i];
      offA32[i] = s2;
      offV[i] = s1;
      if (v >= 1 && v <= kBatchMaxN) { s2 += (long long)v * v; s1 += v; }
    }
    hdr->queue = 0;
    for (int q = 0; q < kRefineHistBins; q++) hdr->refine_hist[q] = 0;
    hdr->s1 = s1;
    hdr->s2 = s2;
    hdr->order = o_order;
    hdr->offA32 = o_offA32;
    hdr->offV = o_offV;
    long long q = o;
    hdr->piv = q;
    q = align256(q + 4 * s1);
    hdr->A32 = q;
    if (precision == LU_PREC_FP32) q = align256(q + 4 * s2);
    hdr->r64 = q;
    if (precision == LU_PREC_FP32) q = align256(q + 16 * s1);
    hdr->v32 = q;
    if (precision == LU_PREC_FP32) q = align256(q + 4 * s1);
    hdr->total = q;
    if (q > work_bytes) s_bad = 1;
  }
  __syncthreads();
  for (int i = tid; i < count; i += blockDim.x) {
    const int v = n[i];
    if (v < 1 || v > kBatchMaxN) { info[i] = LU_ERR_ARG; continue; }
    if (s_bad) { info[i] = LU_ERR_ARG; continue; }
    const int pos = atomicAdd(&hist[v], 1);
    order[pos] = i;
  }
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    hdr->bad = s_bad;
  }
}

std::mutex g_tune_mu;

}  // namespace
}  // namespace lub

using namespace lub;

extern "C" LU_API size_t lu_batched_work_bytes(int32_t count, const int32_t* n_host, int32_t precision) {
  if (count <= 0 || !n_host) return 0;
  long long s2 = 0, s1 = 0;
  for (int i = 0; i < count; i++) {
    s2 += (long long)n_host[i] * n_host[i];
    s1 += n_host[i];
  }
  long long o = 256;
  o = align256(o + 4LL * count);
  o = align256(o + 8LL * count);
  o = align256(o + 8LL * count);
  o = align256(o + 4 * s1);
  if (precision == LU_PREC_FP32) {
    o = align256(o + 4 * s2);
    o = align256(o + 16 * s1);
    o = align256(o + 4 * s1);
  }
  return (size_t)o;
}

extern "C" LU_API int lu_batched_refine_histogram(const void* dWork, int32_t* hist, void* stream) {
  if (!dWork || !hist) return LU_ERR_ARG;
  const WorkHeader* hdr = static_cast<const WorkHeader*>(dWork);
  cudaStream_t s = (cudaStream_t)stream;
  LUB_CUDA(cudaMemcpyAsync(hist, hdr->refine_hist, sizeof(int) * kRefineHistBins, cudaMemcpyDeviceToHost, s));
  LUB_CUDA(cudaStreamSynchronize(s));
  return LU_OK;
}

extern "C" LU_API int lu_batched_set_tuning(int32_t entries, const int32_t* table) {
  if (entries < 0 || entries > 16 || (entries > 0 && !table)) return LU_ERR_ARG;
  Tuning t[16] = {};
  for (int i = 0; i < entries; i++) {
    t[i].n_max = table[3 * i];
    t[i].nb = table[3 * i + 1];
    t[i].small = table[3 * i + 2];
    if (t[i].nb < 4 || t[i].nb > 32 || (t[i].nb & (t[i].nb - 1)) || t[i].small < 0) return LU_ERR_ARG;
    if (i > 0 && t[i].n_max <= t[i - 1].n_max) return LU_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  LUB_CUDA(cudaMemcpyToSymbol(c_tuning, t, sizeof(t)));
  LUB_CUDA(cudaMemcpyToSymbol(c_tuning_n, &entries, sizeof(int)));
  return LU_OK;
}

extern "C" LU_API int lu_batched_factor_solve(int32_t count, const int32_t* n, const int64_t* a_off,
                                              const int64_t* b_off, double* dA, double* db, int32_t* info,
                                              int32_t precision, void* dWork, size_t work_bytes, void* stream) {
  if (count <= 0 || !n || !a_off || !b_off || !dA || !db || !info || !dWork) return LU_ERR_ARG;
  if (precision != LU_PREC_FP64 && precision != LU_PREC_FP32) return LU_ERR_ARG;
  if (work_bytes < 256 + 20 * (size_t)count) return LU_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  static PerDeviceOnce once;
  LUB_TRY(once_per_device(once, [] {
    return cuda_status(
        cudaFuncSetAttribute(batched_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBatchSmem));
  }));
  unsigned char* w = static_cast<unsigned char*>(dWork);
  batched_prep_kernel<<<1, 1024, 0, s>>>(count, n, precision, w, (long long)work_bytes, info);
  LUB_LAUNCH_CHECK();
  int dev = 0, sms = kNumSMsB200;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  BatchArgs a{count, n, a_off, b_off, dA, db, info, precision, w};
  batched_kernel<<<std::min(count, sms), BT, kBatchSmem, s>>>(a);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}
