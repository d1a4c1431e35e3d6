// Unblocked panel factorisation (getf2) of a tall, narrow column block.
//
// Restates the per-column loop of factorDiagBlock / factorBelowDiagBlock
// (lu.ci:186-370) and its kernels:
//   findMaxElm          lu.C:197-205   (strict '>', first row wins)
//   MaxElm_max reducer  lu.C:207-218   (ties: lowest global row here; the
//                                       reference's order is message-arrival
//                                       dependent)
//   swapLocal / pivotRowSwap            lu.C:172-177, lu.ci:302-323
//   computeMultipliersAndFindColMax     lu.C:259-288 (true division, fused
//                                       next-column update + candidate)
//   updateLsubBlock (dger, offset 2)    lu.C:230-254
//   singularity check                   lu.ci:339-341 (reported, not aborted)
//   the row swap on the rest of the panel's columns (the reference swaps
//   whole rows of the panel block, lu.ci:302-323)
//
// Design: a cooperative grid of G CTAs of NT threads, each holding a
// contiguous range of the panel's rows in shared memory for the whole launch
// (row pitch W+1 so a warp walking one column touches distinct banks).  Per
// column: each CTA publishes its candidate (|value|, row, the row's W values)
// and, if it owns row j, that row; one bounded grid barrier; then one round
// trip to L2: while one warp reads the G candidate values and reduces them
// (warp shuffles), the other threads read every candidate row and row j
// into registers, so the pivot row is at hand as soon as the winner is
// known.  Every CTA then swaps locally, scales and updates its rows, and
// computes its candidate for the next column in the same pass.  Slots are
// double-buffered by column parity, which is safe because a CTA cannot reach
// barrier j+2 before every CTA has left barrier j+1.
#include "common.cuh"
#include "kernels.h"

namespace lub {
namespace {


template <typename T>
__device__ __forceinline__ bool cand_better(T v1, int r1, T v2, int r2) {
  // (v1, r1) beats (v2, r2): valid and strictly larger, or equal and lower row
  return r1 >= 0 && (r2 < 0 || v1 > v2 || (v1 == v2 && r1 < r2));
}

template <typename T>
__device__ __forceinline__ void warp_argmax(T& v, int& r, int& w) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T v2 = __shfl_xor_sync(0xffffffffu, v, o);
    int r2 = __shfl_xor_sync(0xffffffffu, r, o);
    int w2 = __shfl_xor_sync(0xffffffffu, w, o);
    if (cand_better(v2, r2, v, r)) { v = v2; r = r2; w = w2; }
  }
}

// Candidate rows read speculatively per thread after the barrier (G * W
// values spread over the CTA); above this many per thread the pivot row is
// read after the argmax instead (a second round trip).
constexpr int kSpecPerThread = 2;

template <typename T, int W, int NT>
__global__ void __launch_bounds__(NT, 1)
getf2_leaf_kernel(T* P, int64_t lda, int M, int ncols, int R, int32_t* ipiv, int row_base, LeafScratch<T> scr,
                  unsigned* bar, DevStatus* st, int info_base, double thr, long long spin, T* prow0, int pw,
                  int lc0) {
  // rows a thread updates at once with explicit register staging (loads,
  // then arithmetic, then stores), so their shared-memory round trips and
  // divisions overlap: fewer when more threads share the rows
  constexpr int RU = NT >= 1024 ? 1 : (NT >= 512 ? 2 : 4);
  constexpr int NW = NT / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int LD = W + 1;
  T* a = reinterpret_cast<T*>(smem_raw);  // [R][LD]
  T* urow = a + (size_t)R * LD;           // [W] pivot row
  __shared__ T s_v[NW];
  __shared__ int s_r[NW];

  const int G = gridDim.x, cta = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r_lo = cta * R;
  const int r_hi = min(M, r_lo + R);
  const int nr = r_hi - r_lo;

  for (int idx = tid; idx < nr * ncols; idx += NT) {
    const int r = idx / ncols, c = idx - r * ncols;
    a[r * LD + c] = P[(int64_t)(r_lo + r) * lda + c];
  }
  __syncthreads();

  // every warp reduces the NW per-warp candidates in s_v / s_r itself, so
  // the whole CTA knows the result after one barrier
  auto cta_argmax = [&](T bv, int br, T& out_v, int& out_r) {
    int w = 0;
    warp_argmax(bv, br, w);
    if (lane == 0) { s_v[warp] = bv; s_r[warp] = br; }
    __syncthreads();
    T v = lane < NW ? s_v[lane] : T(0);
    int r = lane < NW ? s_r[lane] : -1;
    warp_argmax(v, r, w);
    out_v = v;
    out_r = r;
  };

  // candidate of column 0 (findMaxElm(0, 0), lu.ci:266)
  T cv = 0;
  int cr = -1;
  {
    T bv = 0;
    int br = -1;
    for (int r = tid; r < nr; r += NT) {
      T v = fabs(a[r * LD]);
      if (v > bv) { bv = v; br = r_lo + r; }
    }
    cta_argmax(bv, br, cv, cr);
  }

  for (int j = 0; j < ncols; j++) {
    const int slot = j & 1;
    // ---- publish the candidate, its row, and row j if owned (every row
    //      already holds all of the earlier columns' updates)
    if (tid < ncols) {
      if (cr >= 0) scr.cand_data[((size_t)slot * kMaxLeafCTAs + cta) * kMaxLeafW + tid] = a[(cr - r_lo) * LD + tid];
      if (j >= r_lo && j < r_hi) scr.rowj[slot * kMaxLeafW + tid] = a[(j - r_lo) * LD + tid];
    }
    if (tid == 0) {
      scr.cand_val[slot * kMaxLeafCTAs + cta] = cv;
      scr.cand_row[slot * kMaxLeafCTAs + cta] = cr;
    }
    // grid_barrier's CTA barrier followed by thread 0's release add makes
    // these writes visible to every CTA that passes the barrier
    if (!grid_barrier(bar, (unsigned)(j + 1) * (unsigned)G, st, spin, 201)) return;

    // ---- one round trip to L2: every warp reads the G candidate values and
    //      reduces them (each warp knows the winner without a barrier), and
    //      every candidate row and row j are read into registers meanwhile
    const bool spec = G * ncols <= kSpecPerThread * NT;
    T sv[kSpecPerThread];
    int sq[kSpecPerThread];
    T rj = T(0);
    if (spec) {
#pragma unroll
      for (int e = 0; e < kSpecPerThread; e++) {
        const int idx = tid + e * NT;
        sq[e] = -1;
        if (idx < G * ncols) {
          const int q = idx / ncols, c = idx - q * ncols;
          sq[e] = q;
          sv[e] = __ldcg(&scr.cand_data[((size_t)slot * kMaxLeafCTAs + q) * kMaxLeafW + c]);
        }
      }
    }
    if (tid < ncols) rj = __ldcg(&scr.rowj[slot * kMaxLeafW + tid]);
    int pwin = -1, win = 0;
    {
      T v = 0;
      int r = -1;
      for (int q = lane; q < G; q += 32) {
        const T v2 = __ldcg(&scr.cand_val[slot * kMaxLeafCTAs + q]);
        const int r2 = __ldcg(&scr.cand_row[slot * kMaxLeafCTAs + q]);
        if (cand_better(v2, r2, v, r)) { v = v2; r = r2; win = q; }
      }
      warp_argmax(v, r, win);
      pwin = r;
    }
    const bool zero_col = pwin < 0;
    const int p = zero_col ? j : pwin;
    if (zero_col) {
      if (tid < ncols) urow[tid] = rj;
    } else if (spec) {
#pragma unroll
      for (int e = 0; e < kSpecPerThread; e++)
        if (sq[e] == win) urow[tid + e * NT - win * ncols] = sv[e];
    } else if (tid < ncols) {
      urow[tid] = __ldcg(&scr.cand_data[((size_t)slot * kMaxLeafCTAs + win) * kMaxLeafW + tid]);
    }
    // the swap on the enclosing panel's other columns (prow0: panel's first
    // column in this leaf's top row, pw columns, the leaf at lc0): each CTA a
    // slice; the next grid barrier orders consecutive swaps
    if (p != j && pw > ncols) {
      const int others = pw - ncols;
      const int per = (others + G - 1) / G;
      const int q0 = cta * per, q1 = min(others, q0 + per);
      T* r1 = prow0 + (int64_t)j * lda;
      T* r2 = prow0 + (int64_t)p * lda;
      for (int q = q0 + tid; q < q1; q += NT) {
        const int col = q < lc0 ? q : q + ncols;
        const T t = r1[col];
        r1[col] = r2[col];
        r2[col] = t;
      }
    }
    __syncthreads();  // urow complete
    // ---- the local swap: row p takes the old row j, row j the pivot row
    if (tid < ncols) {
      if (p != j && p >= r_lo && p < r_hi) a[(p - r_lo) * LD + tid] = rj;
      if (j >= r_lo && j < r_hi) a[(j - r_lo) * LD + tid] = urow[tid];
    }
    const T piv = urow[j];
    if (cta == 0 && tid == 0) {
      ipiv[j] = row_base + p;
      if (!(fabs((double)piv) > thr)) dev_singular(st, info_base + j + 1);
    }
    __syncthreads();  // rows j and p in place

    // ---- multipliers (true division), rank-1 update of the leaf's
    //      remaining columns, and the candidate of column j+1, in one pass
    const bool do_scale = (piv != T(0)) && !isnan(piv);
    const bool has_next = j + 1 < ncols;
    T bv = 0;
    int br = -1;
    const int r_first = max(j + 1 - r_lo, 0);
    // pivot-row values are warp-wide broadcasts
    for (int rb = r_first + tid; rb < nr; rb += NT * RU) {
      T* rp[RU];
      bool live[RU];
#pragma unroll
      for (int u = 0; u < RU; u++) {
        const int r = rb + u * NT;
        live[u] = r < nr;
        rp[u] = a + (size_t)(live[u] ? r : rb) * LD;
      }
      if (do_scale) {
        T l[RU];
#pragma unroll
        for (int u = 0; u < RU; u++) l[u] = live[u] ? rp[u][j] : T(0);
#pragma unroll
        for (int u = 0; u < RU; u++) l[u] = l[u] / piv;
#pragma unroll
        for (int u = 0; u < RU; u++)
          if (live[u]) rp[u][j] = l[u];
        for (int c = j + 1; c < ncols; c++) {
          const T uc = urow[c];
          T v[RU];
#pragma unroll
          for (int u = 0; u < RU; u++) v[u] = live[u] ? rp[u][c] : T(0);
#pragma unroll
          for (int u = 0; u < RU; u++) v[u] = fma(-l[u], uc, v[u]);
#pragma unroll
          for (int u = 0; u < RU; u++)
            if (live[u]) rp[u][c] = v[u];
        }
      }
      if (has_next) {
#pragma unroll
        for (int u = 0; u < RU; u++) {
          if (live[u]) {
            const T v = fabs(rp[u][j + 1]);
            if (v > bv) { bv = v; br = r_lo + rb + u * NT; }
          }
        }
      }
    }
    cta_argmax(bv, br, cv, cr);
    // the barrier inside cta_argmax also ends every thread's update, so the
    // candidate row published next is complete
  }

  for (int idx = tid; idx < nr * ncols; idx += NT) {
    const int r = idx / ncols, c = idx - r * ncols;
    P[(int64_t)(r_lo + r) * lda + c] = a[r * LD + c];
  }
}

template <typename T, int W>
size_t leaf_smem(int R) { return (size_t)R * (W + 1) * sizeof(T) + W * sizeof(T); }

// threads per leaf CTA: 256, 512 or 1024 (LU_B200_LEAF_THREADS, read once).
// 512 measured best in the mixed N=65536 solve (panel phase 467 ms, against
// 499 ms with 256 and 523 ms with 1024 threads).
int leaf_threads() {
  static int nt = [] {
    const char* e = getenv("LU_B200_LEAF_THREADS");
    const int v = e ? atoi(e) : 512;
    return v >= 1024 ? 1024 : (v >= 512 ? 512 : 256);
  }();
  return nt;
}

template <typename T, int W>
int launch_leaf_w(T* P, int64_t lda, int M, int ncols, int32_t* ipiv, int row_base, const LeafScratch<T>& scr,
                  unsigned* bar, DevStatus* st, int info_base, double thr, long long spin, int max_ctas,
                  cudaStream_t s, T* prow0, int pw, int lc0) {
  // rows per CTA: enough CTAs to spread the panel, capped by max_ctas and by
  // shared memory (R * (W+1) * sizeof(T) <= ~216 KB)
  const int max_rows = (int)((216 * 1024 - W * sizeof(T)) / ((W + 1) * sizeof(T)));
  int G = std::min(std::max(ceil_div(M, 256), 1), std::min(max_ctas, kMaxLeafCTAs));
  int R = ceil_div(M, G);
  if (R > max_rows) {  // too few CTAs allowed for this height: take what shared memory needs
    R = max_rows;
    G = ceil_div(M, R);
    if (G > kMaxLeafCTAs) return LU_ERR_UNSUPPORTED;
  }
  G = ceil_div(M, R);
  size_t smem = leaf_smem<T, W>(R);
  void* args[] = {&P, &lda, &M, &ncols, &R, &ipiv, &row_base, const_cast<LeafScratch<T>*>(&scr), &bar, &st,
                  &info_base, &thr, &spin, &prow0, &pw, &lc0};
  const int nt = leaf_threads();
  const void* fn = nt == 1024 ? (const void*)getf2_leaf_kernel<T, W, 1024>
                              : (nt == 512 ? (const void*)getf2_leaf_kernel<T, W, 512>
                                           : (const void*)getf2_leaf_kernel<T, W, 256>);
  LUB_CUDA(cudaLaunchCooperativeKernel(fn, dim3(G), dim3(nt), args, smem, s));
  __atomic_add_fetch(&g_kernel_launches, 1, __ATOMIC_RELAXED);
  return LU_OK;
}

}  // namespace

template <typename T, int NT>
int leaf_init_nt() {
  LUB_CUDA(cudaFuncSetAttribute(getf2_leaf_kernel<T, 16, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                220 * 1024));
  LUB_CUDA(cudaFuncSetAttribute(getf2_leaf_kernel<T, 32, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                220 * 1024));
  LUB_CUDA(cudaFuncSetAttribute(getf2_leaf_kernel<T, 64, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                220 * 1024));
  return LU_OK;
}

template <typename T>
int leaf_init() {
  LUB_TRY((leaf_init_nt<T, 256>()));
  LUB_TRY((leaf_init_nt<T, 512>()));
  return leaf_init_nt<T, 1024>();
}

// ncols <= 64; the kernel instance is the narrowest of 16/32/64 that holds
// ncols, so narrow leaves keep more rows per CTA and need fewer CTAs.
template <typename T>
int launch_getf2_leaf(T* P, int64_t lda, int M, int ncols, int32_t* ipiv, int row_base, const LeafScratch<T>& scr,
                      unsigned* bar, DevStatus* st, int info_base, double thr, long long spin, int max_ctas,
                      cudaStream_t s, T* prow0, int pw, int lc0) {
  if (M <= 0 || ncols <= 0) return LU_OK;
  if (!prow0) {  // no enclosing panel: the leaf is the whole panel
    prow0 = P;
    pw = ncols;
    lc0 = 0;
  }
  if (lc0 < 0 || lc0 + ncols > pw) return LU_ERR_ARG;
  if (ncols <= 16)
    return launch_leaf_w<T, 16>(P, lda, M, ncols, ipiv, row_base, scr, bar, st, info_base, thr, spin, max_ctas, s,
                                prow0, pw, lc0);
  if (ncols <= 32)
    return launch_leaf_w<T, 32>(P, lda, M, ncols, ipiv, row_base, scr, bar, st, info_base, thr, spin, max_ctas, s,
                                prow0, pw, lc0);
  if (ncols <= 64)
    return launch_leaf_w<T, 64>(P, lda, M, ncols, ipiv, row_base, scr, bar, st, info_base, thr, spin, max_ctas, s,
                                prow0, pw, lc0);
  return LU_ERR_ARG;
}

template int leaf_init<double>();
template int leaf_init<float>();
template int launch_getf2_leaf<double>(double*, int64_t, int, int, int32_t*, int, const LeafScratch<double>&,
                                       unsigned*, DevStatus*, int, double, long long, int, cudaStream_t, double*,
                                       int, int);
template int launch_getf2_leaf<float>(float*, int64_t, int, int, int32_t*, int, const LeafScratch<float>&,
                                      unsigned*, DevStatus*, int, double, long long, int, cudaStream_t, float*, int,
                                      int);

}  // namespace lub
