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
  // the update phase reuses the same space: U12 slice, two L and two C tiles
  while (nb > 4) {
    const size_t panel_phase = (size_t)n * (nb + 1) + (size_t)nb * 128;
    const size_t update_phase = (size_t)nb * 128 + (size_t)2 * 64 * nb + (size_t)2 * 64 * 128;
    if ((panel_phase > update_phase ? panel_phase : update_phase) * esize <= kBatchSmem) break;
    nb >>= 1;
  }
}

template <typename T>
__device__ __forceinline__ bool better(T v1, int r1, T v2, int r2) {
  return r1 >= 0 && (r2 < 0 || v1 > v2 || (v1 == v2 && r1 < r2));
}

// block-wide argmax (value, row); lowest row on ties; -1 if no positive value
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
  if (warp == 0) {
    v = lane < NWARP ? sv[lane] : T(0);
    r = lane < NWARP ? sr[lane] : -1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      T v2 = __shfl_xor_sync(0xffffffffu, v, o);
      int r2 = __shfl_xor_sync(0xffffffffu, r, o);
      if (better(v2, r2, v, r)) { v = v2; r = r2; }
    }
    if (lane == 0) sr[NWARP] = r;
  }
  __syncthreads();
  const int out = sr[NWARP];
  __syncthreads();
  return out;
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
    int p = block_argmax(bv, br, sv, sr);  // its barriers also end the previous update
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

// Trailing update A[c1:n, c1:n] -= L21 * U12 (L21 = A[c1:n, k0:k0+kw], U12 =
// A[k0:k0+kw, c1:n], both final in global memory) over 64 x 128 tiles, 4 x 4
// outputs per thread: rows tr*4 .. +3 (one row group per warp: the L reads
// are broadcasts), columns tc + 32 j (consecutive across lanes: conflict-free
// shared reads and coalesced global writes).  Per column tile the U12 slice
// is staged once; the row tiles' C and L blocks stream through two shared
// buffers with the async copy unit, so the next tile's loads are in flight
// while this one is computed.  smem (reusing the panel's space):
//   Ut [nb][128] | Lt[2] [64][nb] | Ct[2] [64][128]
template <typename T>
__device__ void trailing_update(T* A, int n, int k0, int kw, int c1, int nb, unsigned char* smem) {
  const int tid = threadIdx.x, tr = tid >> 5, tc = tid & 31;
  T* ut = reinterpret_cast<T*>(smem);
  T* lt = ut + (size_t)nb * 128;
  T* ctb = lt + 2 * (size_t)64 * nb;
  const int nrt = (n - c1 + 63) / 64;
  auto issue = [&](int t, int ct, int buf) {
    const int rt = c1 + t * 64;
    T* cdst = ctb + (size_t)buf * 64 * 128;
    T* ldst = lt + (size_t)buf * 64 * nb;
    for (int idx = tid; idx < 64 * 128; idx += BT) {
      const int r = idx >> 7, c = idx & 127;
      const bool ok = rt + r < n && ct + c < n;
      cp_async_elem<sizeof(T)>(cdst + idx, ok ? A + (int64_t)(rt + r) * n + ct + c : A, ok);
    }
    for (int idx = tid; idx < 64 * nb; idx += BT) {
      const int r = idx / nb, p = idx - r * nb;
      const bool ok = rt + r < n && p < kw;
      cp_async_elem<sizeof(T)>(ldst + idx, ok ? A + (int64_t)(rt + r) * n + k0 + p : A, ok);
    }
    cp_async_commit_group();
  };
  for (int ct = c1; ct < n; ct += 128) {
    // U12 slice (kw x 128): all of a thread's loads in flight together
    for (int base = 0; base < kw * 128; base += BT * 8) {
      T v[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int idx = base + tid + u * BT;
        const int p = idx >> 7, c = idx & 127;
        v[u] = (idx < kw * 128 && ct + c < n) ? A[(int64_t)(k0 + p) * n + ct + c] : T(0);
      }
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int idx = base + tid + u * BT;
        if (idx < kw * 128) ut[idx] = v[u];
      }
    }
    issue(0, ct, 0);
    for (int t = 0; t < nrt; t++) {
      const int buf = t & 1;
      if (t + 1 < nrt) {
        issue(t + 1, ct, buf ^ 1);
        cp_async_wait_group<1>();
      } else {
        cp_async_wait_group<0>();
      }
      __syncthreads();  // tile t (and, at t = 0, the U12 slice) in shared memory
      const T* cs = ctb + (size_t)buf * 64 * 128;
      const T* ls = lt + (size_t)buf * 64 * nb;
      T acc[4][4];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = cs[(tr * 4 + i) * 128 + tc + 32 * j];
      for (int p = 0; p < kw; p++) {
        T av[4], bv[4];
#pragma unroll
        for (int i = 0; i < 4; i++) av[i] = ls[(tr * 4 + i) * nb + p];
#pragma unroll
        for (int j = 0; j < 4; j++) bv[j] = ut[p * 128 + tc + 32 * j];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int j = 0; j < 4; j++) acc[i][j] = fma(-av[i], bv[j], acc[i][j]);
      }
      const int rbase = c1 + t * 64 + tr * 4;
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int r = rbase + i;
        if (r >= n) break;
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const int c = ct + tc + 32 * j;
          if (c < n) A[(int64_t)r * n + c] = acc[i][j];
        }
      }
      __syncthreads();  // buffer `buf` (and the U12 slice after the last tile) free for reuse
    }
  }
}

// Factor A (n x n row-major in global, ld = n) in place, permuting x along
// with the rows and recording the pivots (global rows) in piv.
template <typename T>
__device__ int factor_system(T* A, int n, T* x, int* piv, unsigned char* smem, T* sv, int* sr, int* piv_s) {
  const int tid = threadIdx.x;
  int nb, small;
  tuning_for(n, (int)sizeof(T), nb, small);
  if (n <= small) {
    const int ld = n + 1;
    T* a = reinterpret_cast<T*>(smem);
    for (int idx = tid; idx < n * n; idx += BT) a[(idx / n) * ld + idx % n] = A[idx];
    __syncthreads();
    const int info = getf2_smem(a, ld, n, n, piv_s, sv, sr);
    // pivots -> x and global record (sequential swaps by one thread)
    if (tid == 0) {
      for (int j = 0; j < n; j++) {
        const int p = piv_s[j];
        piv[j] = p;
        if (p != j) { const T t = x[j]; x[j] = x[p]; x[p] = t; }
      }
    }
    for (int idx = tid; idx < n * n; idx += BT) A[idx] = a[(idx / n) * ld + idx % n];
    __syncthreads();
    return info;
  }
  int info = 0;
  const int ld = nb + 1;
  T* panel = reinterpret_cast<T*>(smem);                  // n x (nb+1)
  __shared__ int sw_dst[64], sw_src[64], sw_m;             // composed row moves of a panel
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
    // the panel's swaps, in order, composed into one assignment of the
    // affected rows (row dst <- row src, at most 2 kw moves), then applied to
    // the columns outside the panel with every source read before any
    // destination is written; x and the pivot record by thread 0 in order
    if (tid == 0) {
      int pos[64], cont[64], np = 0;
      for (int j = 0; j < kw; j++) {
        const int p = piv_s[j];
        piv[k0 + j] = k0 + p;
        if (p != j) {
          const T t = x[k0 + j];
          x[k0 + j] = x[k0 + p];
          x[k0 + p] = t;
          int ia = -1, ib = -1;
          for (int q = 0; q < np; q++) {
            if (pos[q] == j) ia = q;
            if (pos[q] == p) ib = q;
          }
          if (ia < 0) { pos[np] = j; cont[np] = j; ia = np++; }
          if (ib < 0) { pos[np] = p; cont[np] = p; ib = np++; }
          const int t2 = cont[ia];
          cont[ia] = cont[ib];
          cont[ib] = t2;
        }
      }
      int mm = 0;
      for (int q = 0; q < np; q++)
        if (pos[q] != cont[q]) { sw_dst[mm] = k0 + pos[q]; sw_src[mm] = k0 + cont[q]; mm++; }
      sw_m = mm;
    }
    __syncthreads();
    {
      const int mm = sw_m;
      // four threads per column, each a quarter of the moves (<= 16)
      const int q4 = tid & 3;
      for (int cb = 0; cb < n - kw; cb += BT / 4) {
        const int c = cb + (tid >> 2);
        const int col = c < k0 ? c : c + kw;
        const bool live = c < n - kw;
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
    }
    const int c1 = k0 + kw, nr = n - c1;
    if (nr <= 0) break;
    // U row: A[k0:k0+kw, c1:n] <- L11^{-1} A[k0:k0+kw, c1:n]  (one column per thread)
    for (int c = c1 + tid; c < n; c += BT) {
      T u[32];
#pragma unroll
      for (int i = 0; i < 32; i++) u[i] = i < kw ? A[(int64_t)(k0 + i) * n + c] : T(0);
#pragma unroll
      for (int i = 1; i < 32; i++) {
        if (i >= kw) break;
#pragma unroll
        for (int p = 0; p < 32; p++) {
          if (p >= i) break;
          u[i] = fma(-panel[i * ld + p], u[p], u[i]);
        }
      }
#pragma unroll
      for (int i = 0; i < 32; i++)
        if (i < kw) A[(int64_t)(k0 + i) * n + c] = u[i];
    }
    __syncthreads();
    trailing_update<T>(A, n, k0, kw, c1, nb, smem);
  }
  return info;
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
  __shared__ double sv_d[NWARP + 1];
  __shared__ float sv_f[NWARP + 1];
  __shared__ int sr[NWARP + 1];
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
      info = factor_system<double>(A, n, b, piv, smem, sv_d, sr, piv_s);
      __syncthreads();
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
      info = factor_system<float>(A32, n, v, piv, smem, sv_f, sr, piv_s);
      __syncthreads();
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
        if (tid == 0) {
          for (int j = 0; j < n; j++) {
            const int p = piv[j];
            if (p != j) { const double t = r[j]; r[j] = r[p]; r[p] = t; }
          }
        }
        __syncthreads();
        for (int i = tid; i < n; i += BT) v[i] = (float)r[i];
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
