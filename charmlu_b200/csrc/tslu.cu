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
//      shared memory, rows updated in registers as float4 vectors) with
//      partial pivoting restricted to that block and nominates the rows it
//      chose (at most w);
//   2. tslu_merge_kernel:  later rounds of the tournament, a tree: each CTA
//      stacks a group of nominated sets (their rows' original values),
//      factors the stack with partial pivoting and nominates the rows it
//      chose; the final round (one CTA) so picks the leaf's w pivot rows in
//      order, and its stack's top w x w block is then L11\U11.  It also
//      turns the choice into the sequential swaps of ipiv and into a list of
//      row moves, and saves the moved rows' original values across the
//      enclosing panel;
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

constexpr int LNT = 512;                  // threads of the local kernel
constexpr int MNT = 512;                  // threads of the merge kernels
constexpr size_t kTsluSmem = 216 * 1024;  // dynamic shared memory of the local and merge kernels

__device__ __forceinline__ bool tbetter(float v1, int r1, float v2, int r2) {
  return r1 >= 0 && (r2 < 0 || v1 > v2 || (v1 == v2 && r1 < r2));
}

// Row pitch of the shared-memory blocks: W + 4 floats keeps every row
// 16-byte aligned (rows move as float4), and eight consecutive rows start in
// eight different 16-byte bank groups, so a quarter-warp's vector accesses
// to eight rows do not conflict.
template <int W>
constexpr int row_pitch() { return W + 4; }

// Partial-pivoting elimination of the nr x W block a (shared memory, pitch
// W + 4; columns past ncols hold zeros) over its first `steps` columns, with
// sidx carried along the row swaps.  Two CTA barriers per column: the argmax
// (every warp reduces the per-warp candidates itself), then the swap, which
// also copies the pivot row into s_u.  The column loop is unrolled, so step
// j touches only the columns from j on, with fixed register indices: a row
// is read from its 16-byte group holding column j onwards as float4
// vectors, updated in registers and written back the same way.  Returns bit
// j set when pivot j was usable (nonzero, not NaN).
template <int W, int TNT>
__device__ unsigned eliminate(float* a, int* sidx, int nr, int ncols, int steps, float* s_v, int* s_r, float* s_u) {
  constexpr int NW = TNT / 32, LD = row_pitch<W>();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  unsigned ok_mask = 0;
  float bv = 0.f;
  int br = -1;
  for (int r = tid; r < nr; r += TNT) {
    const float v = fabsf(a[r * LD]);
    if (v > bv) { bv = v; br = r; }
  }
#pragma unroll
  for (int j = 0; j < W; j++) {
    if (j >= steps) break;
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
    // ---- swap rows j and p; the pivot row also goes to s_u
    if (tid < W) {
      const float aj = a[j * LD + tid], ap = a[p * LD + tid];
      if (p != j) {
        a[j * LD + tid] = ap;
        a[p * LD + tid] = aj;
      }
      s_u[tid] = ap;
    }
    if (tid == 0 && p != j) {
      const int t = sidx[j];
      sidx[j] = sidx[p];
      sidx[p] = t;
    }
    __syncthreads();
    // ---- multipliers (true division), rank-1 update of the rows below,
    //      and their candidates for column j + 1
    const float piv = s_u[j];
    const bool do_scale = piv != 0.f && !isnan(piv);
    if (do_scale) ok_mask |= 1u << j;
    bv = 0.f;
    br = -1;
    constexpr int kQ = W / 4;
    const int q0 = j / 4;  // first 16-byte group holding column j (a constant once unrolled)
    const float4* up = reinterpret_cast<const float4*>(s_u);
    for (int rr = j + 1 + tid; rr < nr; rr += TNT) {
      float4* rp = reinterpret_cast<float4*>(a + rr * LD);
      float x[W];
#pragma unroll
      for (int q = 0; q < kQ; q++) {
        if (q >= q0) {
          const float4 f = rp[q];
          x[4 * q] = f.x; x[4 * q + 1] = f.y; x[4 * q + 2] = f.z; x[4 * q + 3] = f.w;
        }
      }
      if (do_scale) {
        const float l = x[j] / piv;
        x[j] = l;
#pragma unroll
        for (int q = 0; q < kQ; q++) {
          if (q >= q0) {
            const float4 uu = up[q];
            const float u4[4] = {uu.x, uu.y, uu.z, uu.w};
#pragma unroll
            for (int e = 0; e < 4; e++)
              if (4 * q + e > j) x[4 * q + e] = fmaf(-l, u4[e], x[4 * q + e]);
          }
        }
#pragma unroll
        for (int q = 0; q < kQ; q++)
          if (q >= q0) rp[q] = make_float4(x[4 * q], x[4 * q + 1], x[4 * q + 2], x[4 * q + 3]);
      }
      if (j + 1 < W && j + 1 < ncols) {
        const float cand = fabsf(x[j + 1 < W ? j + 1 : j]);
        if (cand > bv) { bv = cand; br = rr; }
      }
    }
  }
  return ok_mask;
}

// A row block of P (rows r0.., ncols columns) into shared memory at pitch
// W + 4, zeros past ncols.
template <int W, int TNT>
__device__ void load_rows(float* a, const float* __restrict__ P, int64_t lda, int nr, int ncols, const int* rows,
                          int r0) {
  constexpr int LD = row_pitch<W>();
  for (int idx = threadIdx.x; idx < nr * W; idx += TNT) {
    const int r = idx / W, c = idx - r * W;
    const int64_t g = rows ? rows[r] : r0 + r;
    a[r * LD + c] = c < ncols ? P[g * lda + c] : 0.f;
  }
}

// 1. Candidate rows of each row block: local partial pivoting.
template <int W>
__global__ void __launch_bounds__(LNT, 1)
tslu_local_kernel(const float* __restrict__ P, int64_t lda, int M, int ncols, int R, int* cand_idx, int* cand_cnt) {
  constexpr int TNT = LNT;
  constexpr int LD = row_pitch<W>();
  extern __shared__ __align__(16) unsigned char tslu_smem[];
  float* a = reinterpret_cast<float*>(tslu_smem);         // [R][LD]
  int* sidx = reinterpret_cast<int*>(a + (size_t)R * LD);  // [R]
  __shared__ float s_v[TNT / 32];
  __shared__ int s_r[TNT / 32];
  __shared__ __align__(16) float s_u[W];
  const int cta = blockIdx.x, tid = threadIdx.x;
  const int r_lo = cta * R;
  const int nr = min(M, r_lo + R) - r_lo;
  load_rows<W, TNT>(a, P, lda, nr, ncols, nullptr, r_lo);
  for (int r = tid; r < nr; r += TNT) sidx[r] = r;
  __syncthreads();
  const int steps = min(ncols, nr);
  eliminate<W, TNT>(a, sidx, nr, ncols, steps, s_v, s_r, s_u);
  __syncthreads();
  if (tid < steps) cand_idx[cta * kMaxLeafW + tid] = r_lo + sidx[tid];
  if (tid == 0) cand_cnt[cta] = steps;
}

// first index q < n with key[q] == v, found by one warp (all lanes get it)
__device__ __forceinline__ int warp_find(const int* key, int n, int v) {
  const int lane = threadIdx.x & 31;
  for (int base = 0; base < n; base += 32) {
    const unsigned m = __ballot_sync(0xffffffffu, base + lane < n && key[base + lane] == v);
    if (m) return base + __ffs(m) - 1;
  }
  return -1;
}

// 2. The tournament's later rounds.  CTA b stacks the candidate sets
//    [b * group, (b + 1) * group) of the previous round (their rows'
//    original values) and factors the stack with partial pivoting; the rows
//    it chooses form set b of this tournament round.  The final round (one CTA, FINAL)
//    instead turns its choice into ipiv, L11\U11, the row moves and the
//    moved rows' data.
template <int W, bool FINAL>
__global__ void __launch_bounds__(MNT, 1)
tslu_merge_kernel(const float* __restrict__ P, int64_t lda, int ncols, int nsets, int group,
                  const int* __restrict__ cand_idx, const int* __restrict__ cand_cnt, int* next_idx, int* next_cnt,
                  TsluScratch out, int32_t* ipiv, int row_base, DevStatus* st, int info_base, double thr,
                  const float* __restrict__ prow0, int pw) {
  constexpr int TNT = MNT, LD = row_pitch<W>();
  extern __shared__ __align__(16) unsigned char tslu_smem[];
  __shared__ float s_v[TNT / 32];
  __shared__ int s_r[TNT / 32];
  __shared__ __align__(16) float s_u[W];
  __shared__ int s_off[kMaxLeafCTAs + 1];
  __shared__ int t_pos[2 * kMaxLeafW], t_cont[2 * kMaxLeafW];
  __shared__ int s_mv_dst[2 * kMaxLeafW], s_mv_src[2 * kMaxLeafW], s_mv_cnt;
  const int tid = threadIdx.x, lane = tid & 31;
  const int q_lo = blockIdx.x * group, nq = min(nsets, q_lo + group) - q_lo;
  if (tid == 0) {
    int o = 0;
    for (int q = 0; q < nq; q++) {
      s_off[q] = o;
      o += cand_cnt[q_lo + q];
    }
    s_off[nq] = o;
  }
  __syncthreads();
  const int S = s_off[nq];
  float* a = reinterpret_cast<float*>(tslu_smem);         // [S][LD]
  int* sidx = reinterpret_cast<int*>(a + (size_t)S * LD);  // [S]: panel row of each stacked row
  for (int s = tid; s < S; s += TNT) {
    int q = 0;
    while (s_off[q + 1] <= s) q++;
    sidx[s] = cand_idx[(q_lo + q) * kMaxLeafW + (s - s_off[q])];
  }
  __syncthreads();
  load_rows<W, TNT>(a, P, lda, S, ncols, sidx, 0);
  __syncthreads();
  const int steps = min(ncols, S);
  const unsigned ok_mask = eliminate<W, TNT>(a, sidx, S, ncols, steps, s_v, s_r, s_u);
  __syncthreads();
  if (!FINAL) {
    if (tid < steps) next_idx[blockIdx.x * kMaxLeafW + tid] = sidx[tid];
    if (tid == 0) next_cnt[blockIdx.x] = steps;
    return;
  }
  // L11\U11 (the stack's top rows after elimination) and the usable-pivot mask
  for (int idx = tid; idx < ncols * ncols; idx += TNT) {
    const int i = idx / ncols, c = idx - i * ncols;
    out.lu11[i * kMaxLeafW + c] = a[i * LD + c];
  }
  if (tid < 32) {
    // the chosen rows as sequential swaps (ipiv) and as moves dst <- src:
    // a table of the touched positions and the row each now holds
    int np = 0;
    for (int j = 0; j < ncols; j++) {
      const int g = sidx[j];
      const int hit = warp_find(t_cont, np, g);
      const int at = hit >= 0 ? t_pos[hit] : g;  // where row g sits now
      if (lane == 0) {
        ipiv[j] = row_base + at;
        if (!(fabs((double)a[j * LD + j]) > thr)) dev_singular(st, info_base + j + 1);
      }
      if (at != j) {
        int ia = warp_find(t_pos, np, j);
        int ib = warp_find(t_pos, np, at);
        if (ia < 0) {
          if (lane == 0) { t_pos[np] = j; t_cont[np] = j; }
          ia = np++;
        }
        if (ib < 0) {
          if (lane == 0) { t_pos[np] = at; t_cont[np] = at; }
          ib = np++;
        }
        __syncwarp();
        if (lane == 0) {
          const int t = t_cont[ia];
          t_cont[ia] = t_cont[ib];
          t_cont[ib] = t;
        }
      }
      __syncwarp();
    }
    int m = 0;
    for (int base = 0; base < np; base += 32) {
      const int q = base + lane;
      const bool mv = q < np && t_pos[q] != t_cont[q];
      const unsigned bal = __ballot_sync(0xffffffffu, mv);
      if (mv) {
        const int k = m + __popc(bal & ((1u << lane) - 1u));
        s_mv_dst[k] = t_pos[q];
        s_mv_src[k] = t_cont[q];
      }
      m += __popc(bal);
    }
    if (lane == 0) {
      s_mv_cnt = m;
      *out.mv_cnt = m;
      *out.ok_mask = ok_mask;
    }
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
//    leaf's columns for every row below the top ncols.  Each CTA owns ANT
//    consecutive rows (one thread each) for the leaf's columns; the other
//    columns of the moved rows are copied element by element by all threads.
constexpr int ANT = 128;

template <int W>
__global__ void __launch_bounds__(ANT)
tslu_apply_kernel(int64_t lda, int M, int ncols, TsluScratch in, float* prow0, int pw, int lc0) {
  __shared__ float u[W][W + 1];
  __shared__ int s_map[ANT];
  __shared__ int s_m;
  __shared__ unsigned s_ok;
  const int tid = threadIdx.x;
  const int r0 = blockIdx.x * ANT;
  for (int idx = tid; idx < W * W; idx += ANT) {
    const int i = idx / W, c = idx - i * W;
    u[i][c] = (i < ncols && c < ncols) ? in.lu11[i * kMaxLeafW + c] : 0.f;
  }
  s_map[tid] = -1;
  if (tid == 0) {
    s_m = *in.mv_cnt;
    s_ok = *in.ok_mask;
  }
  __syncthreads();
  const int m = s_m;
  for (int q = tid; q < m; q += ANT) {
    const int d = in.mv_dst[q];
    if (d >= r0 && d < r0 + ANT) s_map[d - r0] = q;
  }
  __syncthreads();
  // the other columns of the moved rows
  const int others = pw - ncols;
  for (int64_t e = (int64_t)blockIdx.x * ANT + tid; e < (int64_t)m * others; e += (int64_t)gridDim.x * ANT) {
    const int k = (int)(e / others), cc = (int)(e - (int64_t)k * others);
    const int c = cc < lc0 ? cc : cc + ncols;
    prow0[(int64_t)in.mv_dst[k] * lda + c] = in.mv_data[(int64_t)k * in.mv_pitch + c];
  }
  const int i = r0 + tid;
  if (i >= M) return;
  const unsigned okm = s_ok;
  const int k = s_map[tid];
  float* leaf = prow0 + (int64_t)i * lda + lc0;
  if (i < ncols) {
    for (int c = 0; c < ncols; c++) leaf[c] = u[i][c];
    return;
  }
  const float* src = k >= 0 ? in.mv_data + (int64_t)k * in.mv_pitch + lc0 : leaf;
  float x[W];
#pragma unroll
  for (int j = 0; j < W; j++) x[j] = j < ncols ? src[j] : 0.f;
#pragma unroll
  for (int j = 0; j < W; j++) {
    if (j < ncols) {
      float t = x[j];
#pragma unroll
      for (int q = 0; q < j; q++)
        if ((okm >> q) & 1u) t = fmaf(-x[q], u[q][j], t);
      x[j] = ((okm >> j) & 1u) ? t / u[j][j] : t;
    }
  }
#pragma unroll
  for (int j = 0; j < W; j++)
    if (j < ncols) leaf[j] = x[j];
}

// candidate sets merged per CTA in the tournament's later rounds
// (LU_B200_TSLU_GROUP, read once)
int tslu_group() {
  static int g = [] {
    const char* e = getenv("LU_B200_TSLU_GROUP");
    const int v = e ? atoi(e) : kMaxLeafCTAs;  // default: one final round over every block's nominees
    return std::max(2, std::min(v, kMaxLeafCTAs));
  }();
  return g;
}

template <int W>
int launch_tslu_w(float* P, int64_t lda, int M, int ncols, int32_t* ipiv, int row_base, const TsluScratch& scr,
                  DevStatus* st, int info_base, double thr, int max_ctas, cudaStream_t s, float* prow0, int pw,
                  int lc0) {
  constexpr int LD = row_pitch<W>();
  const size_t row_bytes = LD * sizeof(float) + sizeof(int);
  const int rmax = (int)(kTsluSmem / row_bytes);
  const int group = std::min(tslu_group(), rmax / W);
  // row blocks of the first round: about sqrt(M / W) of them, at most
  // max_ctas (the SMs the panel may hold) and the candidate-set slots
  int G = (int)ceil(sqrt((double)M / W));
  G = std::max(1, std::min(G, std::min(max_ctas, kMaxLeafCTAs)));
  const int R = ceil_div(M, G);
  if (R > rmax) return LU_ERR_UNSUPPORTED;
  G = ceil_div(M, R);
  if (pw > scr.mv_pitch) return LU_ERR_UNSUPPORTED;
  tslu_local_kernel<W><<<G, LNT, (size_t)R * row_bytes, s>>>(P, lda, M, ncols, R, scr.cand_idx, scr.cand_cnt);
  LUB_LAUNCH_CHECK();
  int* in_idx = scr.cand_idx;
  int* in_cnt = scr.cand_cnt;
  int* out_idx = scr.cand_idx2;
  int* out_cnt = scr.cand_cnt2;
  int nsets = G;
  while (nsets > group) {
    const int nb = ceil_div(nsets, group);
    tslu_merge_kernel<W, false><<<nb, MNT, (size_t)group * W * row_bytes, s>>>(
        P, lda, ncols, nsets, group, in_idx, in_cnt, out_idx, out_cnt, scr, ipiv, row_base, st, info_base, thr,
        prow0, pw);
    LUB_LAUNCH_CHECK();
    std::swap(in_idx, out_idx);
    std::swap(in_cnt, out_cnt);
    nsets = nb;
  }
  tslu_merge_kernel<W, true><<<1, MNT, (size_t)nsets * W * row_bytes, s>>>(
      P, lda, ncols, nsets, nsets, in_idx, in_cnt, out_idx, out_cnt, scr, ipiv, row_base, st, info_base, thr, prow0,
      pw);
  LUB_LAUNCH_CHECK();
  tslu_apply_kernel<W><<<ceil_div(M, ANT), ANT, 0, s>>>(lda, M, ncols, scr, prow0, pw, lc0);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

}  // namespace

int tslu_init() {
  LUB_CUDA(cudaFuncSetAttribute(tslu_local_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTsluSmem));
  LUB_CUDA(cudaFuncSetAttribute(tslu_local_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTsluSmem));
  LUB_CUDA(cudaFuncSetAttribute(tslu_merge_kernel<16, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kTsluSmem));
  LUB_CUDA(cudaFuncSetAttribute(tslu_merge_kernel<32, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kTsluSmem));
  LUB_CUDA(cudaFuncSetAttribute(tslu_merge_kernel<16, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kTsluSmem));
  LUB_CUDA(cudaFuncSetAttribute(tslu_merge_kernel<32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kTsluSmem));
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
  const size_t ints = 2 * (kMaxLeafCTAs * kMaxLeafW + kMaxLeafCTAs) + 4 * kMaxLeafW + 2;
  const size_t floats = kMaxLeafW * kMaxLeafW + (size_t)2 * kMaxLeafW * ncols;
  const size_t bytes = sizeof(DevStatus) + 4 * ints + 4 * floats + 4 + 256;
  LUB_CUDA(cudaMalloc(&blk, bytes));
  LUB_CUDA(cudaMemsetAsync(blk, 0, bytes, s));
  char* b = static_cast<char*>(blk);
  st = reinterpret_cast<DevStatus*>(b);
  int* ip = reinterpret_cast<int*>(b + sizeof(DevStatus));
  t.cand_idx = ip;
  t.cand_cnt = t.cand_idx + kMaxLeafCTAs * kMaxLeafW;
  t.cand_idx2 = t.cand_cnt + kMaxLeafCTAs;
  t.cand_cnt2 = t.cand_idx2 + kMaxLeafCTAs * kMaxLeafW;
  t.mv_dst = t.cand_cnt2 + kMaxLeafCTAs;
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
