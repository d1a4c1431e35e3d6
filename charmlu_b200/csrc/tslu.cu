// Panel leaf with tournament pivoting (TSLU) for the FP32 panels of the
// mixed-precision path.
//
// The partial-pivoting leaf (panel.cu) needs one grid-wide argmax per
// column: a grid barrier and L2 round trips that cost ~5 us per column
// whatever the panel height, which makes the panel chain the critical path
// of the mixed factorisation.  Tournament pivoting (the TSLU panel of
// communication-avoiding LU: Grigori, Demmel and Xiang, SIAM J. Matrix Anal.
// Appl. 32(4), 2011) chooses the w pivot rows of a w-wide leaf with no
// synchronisation between CTAs inside a column:
//   1. tslu_local_kernel:  each of G CTAs factors its own row block (in
//      shared memory) with partial pivoting restricted to that block and
//      nominates the rows it chose (at most w);
//   2. tslu_reduce_kernel: one CTA stacks the nominated rows (their
//      original values), factors the stack with partial pivoting, and so
//      picks the leaf's w pivot rows in order; the stack's top w x w block
//      is then L11\U11.  It also turns the choice into the sequential swaps
//      of ipiv and into a list of row moves, and saves the moved rows'
//      original values across the enclosing panel;
//   3. tslu_apply_kernel:  every row of the panel is moved (across the
//      enclosing panel's columns) and each row below the top w solves
//      l = a U11^{-1} in the leaf's columns.
// Each element of L is produced by the same FMA sequence as in partial
// pivoting with these pivots.  The pivots differ from partial pivoting's
// (the factorisation is of P A with a different P); the mixed path refines
// its solution in FP64 against the original A, so only stability matters,
// and tournament pivoting is as stable as partial pivoting in practice.
// The FP64 path (whose pivots must be the reference's) keeps the
// partial-pivoting leaf.
#include <cmath>

#include "common.cuh"
#include "kernels.h"

namespace lub {
namespace {

constexpr int TNT = 1024;                 // threads of the local and reduction kernels
constexpr size_t kTsluSmem = 216 * 1024;  // dynamic shared memory of those kernels

__device__ __forceinline__ bool tbetter(float v1, int r1, float v2, int r2) {
  return r1 >= 0 && (r2 < 0 || v1 > v2 || (v1 == v2 && r1 < r2));
}

// Partial-pivoting elimination of the nr x ncols block a (shared memory,
// pitch LD) over its first `steps` columns, with sidx carried along the row
// swaps.  Two CTA barriers per column: the argmax (every warp reduces the
// per-warp candidates itself), then the swap.  Returns, per column, through
// `pivot_ok` (bit j set: the pivot was usable, i.e. nonzero and not NaN).
template <int LD>
__device__ unsigned eliminate(float* a, int* sidx, int nr, int ncols, int steps, float* s_v, int* s_r) {
  constexpr int NW = TNT / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  unsigned ok_mask = 0;
  float bv = 0.f;
  int br = -1;
  for (int r = tid; r < nr; r += TNT) {
    const float v = fabsf(a[r * LD]);
    if (v > bv) { bv = v; br = r; }
  }
  for (int j = 0; j < steps; j++) {
    // ---- argmax over the block's rows >= j
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float v2 = __shfl_xor_sync(0xffffffffu, bv, o);
      const int r2 = __shfl_xor_sync(0xffffffffu, br, o);
      if (tbetter(v2, r2, bv, br)) { bv = v2; br = r2; }
    }
    if (lane == 0) { s_v[warp] = bv; s_r[warp] = br; }
    __syncthreads();
    float v = lane < NW ? s_v[lane] : 0.f;
    int r = lane < NW ? s_r[lane] : -1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float v2 = __shfl_xor_sync(0xffffffffu, v, o);
      const int r2 = __shfl_xor_sync(0xffffffffu, r, o);
      if (tbetter(v2, r2, v, r)) { v = v2; r = r2; }
    }
    const int p = r < 0 ? j : r;  // an all-zero column keeps its row
    // ---- swap rows j and p (every thread reads the pivot row after the barrier)
    if (p != j) {
      for (int c = tid; c < ncols; c += TNT) {
        const float t = a[j * LD + c];
        a[j * LD + c] = a[p * LD + c];
        a[p * LD + c] = t;
      }
      if (tid == 0) {
        const int t = sidx[j];
        sidx[j] = sidx[p];
        sidx[p] = t;
      }
    }
    __syncthreads();
    // ---- multipliers (true division), rank-1 update of the rows below,
    //      and their candidates for column j + 1
    const float piv = a[j * LD + j];
    const bool do_scale = piv != 0.f && !isnan(piv);
    if (do_scale) ok_mask |= 1u << (j & 31);
    bv = 0.f;
    br = -1;
    for (int rr = j + 1 + tid; rr < nr; rr += TNT) {
      float* ar = a + rr * LD;
      if (do_scale) {
        const float l = ar[j] / piv;
        ar[j] = l;
        for (int c = j + 1; c < ncols; c++) ar[c] = fmaf(-l, a[j * LD + c], ar[c]);
      }
      if (j + 1 < ncols) {
        const float vv = fabsf(ar[j + 1]);
        if (vv > bv) { bv = vv; br = rr; }
      }
    }
  }
  return ok_mask;
}

// 1. Candidate rows of each row block: local partial pivoting.
template <int W>
__global__ void __launch_bounds__(TNT, 1)
tslu_local_kernel(const float* __restrict__ P, int64_t lda, int M, int ncols, int R, int* cand_idx, int* cand_cnt) {
  constexpr int LD = W + 1;
  extern __shared__ __align__(16) unsigned char tslu_smem[];
  float* a = reinterpret_cast<float*>(tslu_smem);         // [R][LD]
  int* sidx = reinterpret_cast<int*>(a + (size_t)R * LD);  // [R]
  __shared__ float s_v[TNT / 32];
  __shared__ int s_r[TNT / 32];
  const int cta = blockIdx.x, tid = threadIdx.x;
  const int r_lo = cta * R;
  const int nr = min(M, r_lo + R) - r_lo;
  for (int idx = tid; idx < nr * ncols; idx += TNT) {
    const int r = idx / ncols, c = idx - r * ncols;
    a[r * LD + c] = P[(int64_t)(r_lo + r) * lda + c];
  }
  for (int r = tid; r < nr; r += TNT) sidx[r] = r;
  __syncthreads();
  const int steps = min(ncols, nr);
  eliminate<LD>(a, sidx, nr, ncols, steps, s_v, s_r);
  __syncthreads();
  if (tid < steps) cand_idx[cta * kMaxLeafW + tid] = r_lo + sidx[tid];
  if (tid == 0) cand_cnt[cta] = steps;
}

// 2. The tournament's final round: partial pivoting on the stacked
//    candidates; ipiv, L11\U11, the row moves and the moved rows' data.
template <int W>
__global__ void __launch_bounds__(TNT, 1)
tslu_reduce_kernel(const float* __restrict__ P, int64_t lda, int M, int ncols, int G, const int* __restrict__ cand_idx,
                   const int* __restrict__ cand_cnt, TsluScratch out, int32_t* ipiv, int row_base, DevStatus* st,
                   int info_base, double thr, const float* __restrict__ prow0, int pw) {
  constexpr int LD = W + 1;
  extern __shared__ __align__(16) unsigned char tslu_smem[];
  __shared__ float s_v[TNT / 32];
  __shared__ int s_r[TNT / 32];
  __shared__ int s_off[kMaxLeafCTAs + 1];
  __shared__ int s_mv_dst[2 * kMaxLeafW], s_mv_src[2 * kMaxLeafW], s_mv_cnt;
  const int tid = threadIdx.x;
  if (tid == 0) {
    int o = 0;
    for (int q = 0; q < G; q++) {
      s_off[q] = o;
      o += cand_cnt[q];
    }
    s_off[G] = o;
  }
  __syncthreads();
  const int S = s_off[G];
  float* a = reinterpret_cast<float*>(tslu_smem);         // [S][LD]
  int* sidx = reinterpret_cast<int*>(a + (size_t)S * LD);  // [S]: panel row of each stacked row
  for (int s = tid; s < S; s += TNT) {
    int q = 0;
    while (s_off[q + 1] <= s) q++;
    sidx[s] = cand_idx[q * kMaxLeafW + (s - s_off[q])];
  }
  __syncthreads();
  for (int idx = tid; idx < S * ncols; idx += TNT) {
    const int s = idx / ncols, c = idx - s * ncols;
    a[s * LD + c] = P[(int64_t)sidx[s] * lda + c];
  }
  __syncthreads();
  const unsigned ok_mask = eliminate<LD>(a, sidx, S, ncols, ncols, s_v, s_r);
  __syncthreads();
  // L11\U11 (the stack's top rows after elimination) and the usable-pivot mask
  for (int idx = tid; idx < ncols * ncols; idx += TNT) {
    const int i = idx / ncols, c = idx - i * ncols;
    out.lu11[i * kMaxLeafW + c] = a[i * LD + c];
  }
  if (tid == 0) {
    *out.ok_mask = ok_mask;
    // the chosen rows as sequential swaps (ipiv), and as moves dst <- src
    int pos[2 * kMaxLeafW], cont[2 * kMaxLeafW], np = 0;
    for (int j = 0; j < ncols; j++) {
      const int g = sidx[j];
      // where row g sits now: a touched position holding it, else its own
      int at = g;
      for (int q = 0; q < np; q++)
        if (cont[q] == g) { at = pos[q]; break; }
      ipiv[j] = row_base + at;
      const float u = a[j * LD + j];
      if (!(fabs((double)u) > thr)) dev_singular(st, info_base + j + 1);
      if (at != j) {
        int ia = -1, ib = -1;
        for (int q = 0; q < np; q++) {
          if (pos[q] == j) ia = q;
          if (pos[q] == at) ib = q;
        }
        if (ia < 0) { pos[np] = j; cont[np] = j; ia = np++; }
        if (ib < 0) { pos[np] = at; cont[np] = at; ib = np++; }
        const int t = cont[ia];
        cont[ia] = cont[ib];
        cont[ib] = t;
      }
    }
    int m = 0;
    for (int q = 0; q < np; q++)
      if (pos[q] != cont[q]) {
        s_mv_dst[m] = pos[q];
        s_mv_src[m] = cont[q];
        m++;
      }
    s_mv_cnt = m;
    *out.mv_cnt = m;
  }
  __syncthreads();
  const int m = s_mv_cnt;
  for (int k = tid; k < m; k += TNT) {
    out.mv_dst[k] = s_mv_dst[k];
    out.mv_src[k] = s_mv_src[k];
  }
  // the moved rows' original values across the enclosing panel (read
  // before the apply kernel overwrites any of them)
  for (int idx = tid; idx < m * pw; idx += TNT) {
    const int k = idx / pw, c = idx - k * pw;
    out.mv_data[(int64_t)k * out.mv_pitch + c] = prow0[(int64_t)s_mv_src[k] * lda + c];
  }
}

// 3. Rows into place across the enclosing panel, and l = a U11^{-1} in the
//    leaf's columns for every row below the top ncols.
constexpr int ANT = 128;  // threads of the apply kernel (one row each)

template <int W>
__global__ void __launch_bounds__(ANT)
tslu_apply_kernel(int64_t lda, int M, int ncols, TsluScratch in, float* prow0, int pw, int lc0) {
  __shared__ float u[W][W + 1];
  __shared__ int s_dst[2 * kMaxLeafW], s_src[2 * kMaxLeafW];
  __shared__ int s_m;
  __shared__ unsigned s_ok;
  const int tid = threadIdx.x;
  for (int idx = tid; idx < W * W; idx += ANT) {
    const int i = idx / W, c = idx - i * W;
    u[i][c] = (i < ncols && c < ncols) ? in.lu11[i * kMaxLeafW + c] : 0.f;
  }
  if (tid == 0) {
    s_m = *in.mv_cnt;
    s_ok = *in.ok_mask;
  }
  __syncthreads();
  const int m = s_m;
  for (int k = tid; k < m; k += ANT) {
    s_dst[k] = in.mv_dst[k];
    s_src[k] = in.mv_src[k];
  }
  __syncthreads();
  const unsigned okm = s_ok;
  for (int i = blockIdx.x * ANT + tid; i < M; i += gridDim.x * ANT) {
    int k = -1;
    for (int q = 0; q < m; q++)
      if (s_dst[q] == i) { k = q; break; }
    float* row = prow0 + (int64_t)i * lda;
    const float* mrow = k >= 0 ? in.mv_data + (int64_t)k * in.mv_pitch : nullptr;
    if (k >= 0) {  // the panel's other columns of a moved row
      for (int c = 0; c < lc0; c++) row[c] = mrow[c];
      for (int c = lc0 + ncols; c < pw; c++) row[c] = mrow[c];
    }
    float* leaf = row + lc0;
    if (i < ncols) {
      for (int c = 0; c < ncols; c++) leaf[c] = u[i][c];
      continue;
    }
    const float* src = k >= 0 ? mrow + lc0 : leaf;
    float l[W];
#pragma unroll
    for (int j = 0; j < W; j++) {
      if (j < ncols) {
        float t = src[j];
#pragma unroll
        for (int q = 0; q < j; q++)
          if ((okm >> q) & 1u) t = fmaf(-l[q], u[q][j], t);
        l[j] = ((okm >> j) & 1u) ? t / u[j][j] : t;
      }
    }
#pragma unroll
    for (int j = 0; j < W; j++)
      if (j < ncols) leaf[j] = l[j];
  }
}

template <int W>
int launch_tslu_w(float* P, int64_t lda, int M, int ncols, int32_t* ipiv, int row_base, const TsluScratch& scr,
                  DevStatus* st, int info_base, double thr, int max_ctas, cudaStream_t s, float* prow0, int pw,
                  int lc0) {
  constexpr int LD = W + 1;
  const int rmax = (int)(kTsluSmem / (LD * sizeof(float) + sizeof(int)));
  const int smax = rmax;  // the stack has the same shared-memory layout
  // balance the local blocks (R rows) against the stack (G * W rows)
  int G = (int)ceil(sqrt((double)M / W));
  G = std::max(1, std::min(G, std::min(max_ctas, std::min(kMaxLeafCTAs, smax / W))));
  const int R = ceil_div(M, G);
  if (R > rmax) return LU_ERR_UNSUPPORTED;
  G = ceil_div(M, R);
  if (pw > scr.mv_pitch) return LU_ERR_UNSUPPORTED;
  const size_t sm1 = (size_t)R * (LD * sizeof(float) + sizeof(int));
  tslu_local_kernel<W><<<G, TNT, sm1, s>>>(P, lda, M, ncols, R, scr.cand_idx, scr.cand_cnt);
  LUB_LAUNCH_CHECK();
  const size_t sm2 = (size_t)G * W * (LD * sizeof(float) + sizeof(int));
  tslu_reduce_kernel<W><<<1, TNT, sm2, s>>>(P, lda, M, ncols, G, scr.cand_idx, scr.cand_cnt, scr, ipiv, row_base,
                                           st, info_base, thr, prow0, pw);
  LUB_LAUNCH_CHECK();
  const int g3 = std::max(1, std::min(ceil_div(M, ANT), 8 * kNumSMsB200));
  tslu_apply_kernel<W><<<g3, ANT, 0, s>>>(lda, M, ncols, scr, prow0, pw, lc0);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

}  // namespace

int tslu_init() {
  LUB_CUDA(cudaFuncSetAttribute(tslu_local_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTsluSmem));
  LUB_CUDA(cudaFuncSetAttribute(tslu_local_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTsluSmem));
  LUB_CUDA(cudaFuncSetAttribute(tslu_reduce_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTsluSmem));
  LUB_CUDA(cudaFuncSetAttribute(tslu_reduce_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTsluSmem));
  return LU_OK;
}

// ncols <= 32.  P: the leaf's top-left element; prow0: the enclosing
// panel's first column in the leaf's top row (pw columns, the leaf at
// lc0); prow0 = null: the leaf is the panel.  LU_ERR_UNSUPPORTED: too tall
// for the shared-memory blocks or too wide a panel (the caller then uses
// the partial-pivoting leaf).
int launch_tslu_leaf(float* P, int64_t lda, int M, int ncols, int32_t* ipiv, int row_base, const TsluScratch& scr,
                     DevStatus* st, int info_base, double thr, int max_ctas, cudaStream_t s, float* prow0, int pw,
                     int lc0) {
  if (M <= 0 || ncols <= 0) return LU_OK;
  if (ncols > 32 || M < ncols) return LU_ERR_UNSUPPORTED;
  if (!prow0) {
    prow0 = P;
    pw = ncols;
    lc0 = 0;
  }
  if (lc0 < 0 || lc0 + ncols > pw) return LU_ERR_ARG;
  if (ncols <= 16)
    return launch_tslu_w<16>(P, lda, M, ncols, ipiv, row_base, scr, st, info_base, thr, max_ctas, s, prow0, pw, lc0);
  return launch_tslu_w<32>(P, lda, M, ncols, ipiv, row_base, scr, st, info_base, thr, max_ctas, s, prow0, pw, lc0);
}

}  // namespace lub

// Test hook (not part of the ABI): the tournament-pivoting leaf on an FP32
// panel P (M x ncols, row-major, pitch lda; the leaf is the whole panel),
// with scratch of its own.  ipiv (device, ncols) receives the pivots; the
// return value is LU_OK, LU_ERR_UNSUPPORTED, or the first singular column
// (1-based) once the stream has finished.
extern "C" __attribute__((visibility("default"))) int lub_test_tslu_leaf(float* P, int64_t lda, int M, int ncols,
                                                                       int32_t* ipiv, int max_ctas, void* stream) {
  using namespace lub;
  cudaStream_t s = (cudaStream_t)stream;
  LUB_TRY(tslu_init());
  TsluScratch t{};
  t.mv_pitch = ncols;
  DevStatus* st = nullptr;
  void* blk = nullptr;
  const size_t ints = kMaxLeafCTAs * kMaxLeafW + kMaxLeafCTAs + 4 * kMaxLeafW + 2;
  const size_t floats = kMaxLeafW * kMaxLeafW + (size_t)2 * kMaxLeafW * ncols;
  const size_t bytes = sizeof(DevStatus) + 4 * ints + 4 * floats + 4 + 256;
  LUB_CUDA(cudaMalloc(&blk, bytes));
  LUB_CUDA(cudaMemsetAsync(blk, 0, bytes, s));
  char* b = static_cast<char*>(blk);
  st = reinterpret_cast<DevStatus*>(b);
  int* ip = reinterpret_cast<int*>(b + sizeof(DevStatus));
  t.cand_idx = ip;
  t.cand_cnt = t.cand_idx + kMaxLeafCTAs * kMaxLeafW;
  t.mv_dst = t.cand_cnt + kMaxLeafCTAs;
  t.mv_src = t.mv_dst + 2 * kMaxLeafW;
  t.mv_cnt = t.mv_src + 2 * kMaxLeafW;
  t.ok_mask = reinterpret_cast<unsigned*>(t.mv_cnt + 1);
  t.lu11 = reinterpret_cast<float*>(t.ok_mask + 1);
  t.mv_data = t.lu11 + kMaxLeafW * kMaxLeafW;
  int rc = launch_tslu_leaf(P, lda, M, ncols, ipiv, 0, t, st, 0, 0.0, max_ctas, s, nullptr, 0, 0);
  DevStatus h{};
  cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  cudaFree(blk);
  if (rc != LU_OK) return rc;
  return h.code != 0 ? h.code : h.info;
}
