// Mixed-precision factorisation + FP64 iterative refinement (lu_refine_solve).
//
// No reference counterpart (charmlu is FP64 only); the factorisation keeps
// charmlu's right-looking blocked structure (lu.ci:31-370) with these
// precisions:
//   working matrix  FP32 copy of the FP64 A (A itself is never modified)
//   panel, TRSM     FP32 (leaf getf2 + recursive halves on the FP32 pipe)
//   trailing update BF16 operands, FP32 accumulation in TMEM (tcgen05),
//                   subtracted into the FP32 matrix with TMA reduce-add
//   refinement      FP64 residual r = b - A x against the untouched A, FP32
//                   correction solve with the low-precision factors, FP64
//                   update of x; classical IR first, GMRES-IR (flexible,
//                   right preconditioned by the LU factors, FP64 Arnoldi)
//                   when the classical iteration stops contracting.  A step
//                   whose ||b - A x||inf is not below the best so far is
//                   rolled back, so the reported residual never rises.
#include <cmath>
#include <cstring>
#include <vector>

#include "handle.h"

using namespace lub;

namespace {

constexpr int kGmresRestart = 120;  // default: long Krylov spaces, short restarts stall when kappa * u_f >> 1
constexpr int kIrStall = 3;         // default: GMRES cycles in a row with < 10% progress before giving up
constexpr double kGmresTol = 1e-10; // default: residual reduction that ends a GMRES cycle

int ensure_mixed(lu_handle h) {
  if (h->mixed_ready) return LU_OK;
  const int64_t n = h->cfg.n;
  const int64_t B = h->cfg.block_size;
  h->ld32 = (n + 31) & ~int64_t(31);
  // FP16x3 on the persistent update: operand rows [hi | lo], each part a
  // whole number of 64-wide k blocks; otherwise the parts are concatenated
  h->pairs = h->cfg.precision == LU_PREC_FP16X3 && h->gemm_ctas > 0;
  h->nparts = h->cfg.precision == LU_PREC_FP16X3 ? (h->pairs ? 2 : 3) : 1;
  h->ldk = h->pairs ? 2 * ((B + 63) & ~int64_t(63)) : (h->nparts * B + 63) & ~int64_t(63);
  h->gm = h->cfg.gmres_restart > 0 ? h->cfg.gmres_restart : kGmresRestart;
  LUB_TRY(h->alloc(&h->A32, (size_t)n * h->ld32));
  LUB_TRY(h->alloc(&h->Lb, (size_t)n * h->ldk));
  LUB_TRY(h->alloc(&h->Ub, (size_t)n * h->ldk));
  LUB_TRY(h->alloc(&h->ipiv32, n));
  LUB_TRY(h->alloc(&h->amax, 4));
  LUB_TRY(h->alloc(&h->dinv32, 16 * 1024));
  if (h->pairs && h->panel_tc) {  // panel GEMM operands: K <= B/2 rows of [hi | lo], N <= B/2 columns
    h->ldkP = 2 * ((B / 2 + 63) & ~int64_t(63));
    LUB_TRY(h->alloc(&h->Lp, (size_t)n * h->ldkP));
    LUB_TRY(h->alloc(&h->Up, (size_t)B * h->ldkP));
    LUB_TRY(h->alloc(&h->amaxP, 4));
  }
  if (h->tslu && !h->tslu_scr.cand_idx) {
    TsluScratch& t = h->tslu_scr;
    t.mv_pitch = (int)B;
    LUB_TRY(h->alloc(&t.cand_idx, kMaxLeafCTAs * kMaxLeafW));
    LUB_TRY(h->alloc(&t.cand_cnt, kMaxLeafCTAs));
    LUB_TRY(h->alloc(&t.cand_idx2, kMaxLeafCTAs * kMaxLeafW));
    LUB_TRY(h->alloc(&t.cand_cnt2, kMaxLeafCTAs));
    LUB_TRY(h->alloc(&t.lu11, kMaxLeafW * kMaxLeafW));
    LUB_TRY(h->alloc(&t.ok_mask, 1));
    LUB_TRY(h->alloc(&t.mv_dst, 2 * kMaxLeafW));
    LUB_TRY(h->alloc(&t.mv_src, 2 * kMaxLeafW));
    LUB_TRY(h->alloc(&t.mv_cnt, 1));
    LUB_TRY(h->alloc(&t.mv_data, (size_t)2 * kMaxLeafW * B));
  }
  LUB_TRY(h->alloc(&h->v32, n));
  LUB_TRY(h->alloc(&h->r64, n));
  LUB_TRY(h->alloc(&h->z64, n));
  LUB_TRY(h->alloc(&h->zero64, n));
  LUB_TRY(h->alloc(&h->xbest, n));
  LUB_TRY(h->alloc(&h->rbest, n));
  LUB_TRY(h->alloc(&h->racc_best, 1));
  LUB_CUDA(cudaMemset(h->zero64, 0, sizeof(double) * n));
  h->mixed_ready = true;
  return LU_OK;
}

// The flexible GMRES work space: Arnoldi basis V, preconditioned basis Z
// (about 2 * restart * n doubles; allocated on the first GMRES cycle)
int ensure_gmres(lu_handle h) {
  if (h->V) return LU_OK;
  const size_t n = (size_t)h->cfg.n;
  LUB_TRY(h->alloc(&h->V, (size_t)(h->gm + 1) * n));
  LUB_TRY(h->alloc(&h->Z, (size_t)h->gm * n));
  return h->alloc(&h->hdot, 128 * (h->gm + 2) + 2 * (h->gm + 2));
}

struct Ctx32 {
  lu_handle h;
  float* A;
  int64_t ld;
  int n;
  int32_t* ipiv;
  cudaStream_t s;
  double thr;
  PivotList pl;
  int leaf_w;
  int leaf_ctas;
};

inline int split_w32(int w) {
  int hh = w / 2;
  int w1 = hh >= 16 ? (hh & ~15) : (hh & ~3);
  return std::max(w1, 4);
}

// composed: the context's pivot list already holds this batch (cnt <= 512),
// composed by an earlier call on the same stream
int pivots_apply_f32(Ctx32& c, int k0, int cnt, int c_begin, int c_end, int skip_b, int skip_e, int32_t* perm,
                     bool composed = false) {
  Prof pf(c.h, c.s, LU_PH_LASWP);
  if (composed && cnt > 512) return LU_ERR_ARG;
  for (int off = 0; off < cnt; off += 512) {
    const int sub = std::min(512, cnt - off);
    if (!composed) LUB_TRY(launch_pivot_compose(c.ipiv, k0 + off, sub, c.pl, c.s));
    LUB_TRY(launch_pivot_apply<float>(c.A, c.ld, c_begin, c_end, skip_b, skip_e, c.pl, 2 * sub, nullptr, perm, c.s));
  }
  return LU_OK;
}

int sgemm(Ctx32& c, int rc, int cc, int ra, int ca, int rb, int cb, int M, int N, int K) {
  Prof pf(c.h, c.s, LU_PH_GEMM_IN, 2.0 * M * (double)N * K);
  return launch_gemm_f32_sub(c.A + (int64_t)ra * c.ld + ca, c.ld, c.A + (int64_t)rb * c.ld + cb, c.ld,
                             c.A + (int64_t)rc * c.ld + cc, c.ld, M, N, K, c.s);
}

int trsm32(Ctx32& c, int r0, int w, int rb, int cb, int ncols) {
  // the panels' inner solves (and, with trsm_block 2, every solve of w <= 256): one launch
  if (w > 32 && w <= 256 && (ncols <= 512 || c.h->trsm_block == 2) && c.h->trsm_block) {
    Prof pf(c.h, c.s, LU_PH_TRSM, (double)w * w * ncols);
    return launch_trsm_llu_block(c.A + (int64_t)r0 * c.ld + r0, c.ld, c.A + (int64_t)rb * c.ld + cb, c.ld, w, ncols,
                                 c.s);
  }
  // a step's U block row (every trailing column): one launch, 32 x 32
  // diagonal blocks inverted first
  if (w > 32 && w <= 512 && ncols > c.h->trsm_wide_min && c.h->trsm_wide) {
    Prof pf(c.h, c.s, LU_PH_TRSM, (double)w * w * ncols);
    return launch_trsm_wide(c.A + (int64_t)r0 * c.ld + r0, c.ld, c.A + (int64_t)rb * c.ld + cb, c.ld, w, ncols,
                            c.h->dinv32, c.s);
  }
  if (w <= 32) {
    Prof pf(c.h, c.s, LU_PH_TRSM, (double)w * w * ncols);
    return launch_trsm_llu_leaf<float>(c.A + (int64_t)r0 * c.ld + r0, c.ld, c.A + (int64_t)rb * c.ld + cb, c.ld, w,
                                       ncols, c.s);
  }
  const int w1 = split_w32(w);
  LUB_TRY(trsm32(c, r0, w1, rb, cb, ncols));
  LUB_TRY(sgemm(c, rb + w1, cb, r0 + w1, r0, rb, cb, w - w1, ncols, w1));
  return trsm32(c, r0 + w1, w - w1, rb + w1, cb, ncols);
}

// C(r0.., n0..n0+N) -= L(r0.., kc..kc+K) * U(kc..kc+K, n0..n0+N) inside the
// panel that ends at column cend, on the tcgen05 kernel: both operands split
// into scaled FP16 hi/lo parts (pairs layout, three products), as the
// trailing update does. The C tensor map ends at cend, so the 256-wide tiles
// leave the columns right of the panel (being updated beside it) untouched.
int panel_gemm_tc(Ctx32& c, int r0, int M, int kc, int K, int n0, int N, int cend) {
  lu_handle h = c.h;
  Prof pf(h, c.s, LU_PH_GEMM_IN, 2.0 * M * (double)N * K);
  const float* L = c.A + (int64_t)r0 * c.ld + kc;
  const float* U = c.A + (int64_t)kc * c.ld + n0;
  LUB_TRY(launch_panel_absmax(L, c.ld, M, K, U, c.ld, N, h->amaxP, c.s));
  LUB_TRY(launch_split_rows<__half>(L, c.ld, h->Lp, h->ldkP, M, K, 2, 0x2u, h->amaxP, 0, c.s, K));
  LUB_TRY(launch_split_transpose<__half>(U, c.ld, h->Up, h->ldkP, K, N, 2, 0x2u, h->amaxP, 1, c.s, K));
  CUtensorMap mL, mU, mC;
  LUB_TRY(encode_tmap_2d(&mL, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, h->Lp, 2 * K, M, h->ldkP * 2, 64, 128,
                         CU_TENSOR_MAP_SWIZZLE_128B));
  LUB_TRY(encode_tmap_2d(&mU, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, h->Up, 2 * K, N, h->ldkP * 2, 64, 128,
                         CU_TENSOR_MAP_SWIZZLE_128B));
  LUB_TRY(encode_tmap_2d(&mC, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, c.A, cend, c.n, c.ld * 4, 32, 128,
                         CU_TENSOR_MAP_SWIZZLE_128B));
  const int ctas = h->cfg.lookahead ? h->gemm_reserve : h->gemm_ctas;
  return launch_gemm_lowp_persistent(mL, mU, mC, 0, 0, r0, n0, M, N, K, false, h->amaxP, h->st, h->spin,
                                     std::max(1, ctas), c.s, K, nullptr, h->gemm_pair != 0);
}

// recursive FP32 panel of columns [c0, c0+w) inside the panel [p0, p0+pw);
// the leaves swap rows across the whole panel (no laswp in the recursion)
int panel32(Ctx32& c, int c0, int w, int p0, int pw) {
  const int M = c.n - c0;
  if (w <= c.leaf_w) {
    Prof pf(c.h, c.s, LU_PH_PANEL, (double)M * w * w);
    if (c.h->tslu && c.h->tslu_scr.cand_idx) {
      const int rc = launch_tslu_leaf(c.A + (int64_t)c0 * c.ld + c0, c.ld, M, w, c.ipiv + c0, c0, c.h->tslu_scr,
                                      c.h->st, c0, c.thr, c.leaf_ctas, c.s, c.A + (int64_t)c0 * c.ld + p0, pw, c0 - p0);
      if (rc != LU_ERR_UNSUPPORTED) return rc;
    }
    unsigned* bar = c.h->take_counter();
    if (!bar) return LU_ERR_NOMEM;
    return launch_getf2_leaf<float>(c.A + (int64_t)c0 * c.ld + c0, c.ld, M, w, c.ipiv + c0, c0, c.h->leaf32, bar,
                                    c.h->st, c0, c.thr, c.h->spin, c.leaf_ctas, c.s, c.A + (int64_t)c0 * c.ld + p0,
                                    pw, c0 - p0);
  }
  const int w1 = split_w32(w), w2 = w - w1;
  LUB_TRY(panel32(c, c0, w1, p0, pw));
  LUB_TRY(trsm32(c, c0, w1, c0, c0 + w1, w2));
  if (c.h->Lp && w2 >= 128 && w1 % 64 == 0 && 2 * w1 <= c.h->ldkP && w2 <= c.h->cfg.block_size &&
      (c0 + w1) % 4 == 0)
    LUB_TRY(panel_gemm_tc(c, c0 + w1, M - w1, c0, w1, c0 + w1, w2, p0 + pw));
  else
    LUB_TRY(sgemm(c, c0 + w1, c0 + w1, c0 + w1, c0, c0, c0 + w1, M - w1, w2, w1));
  return panel32(c, c0 + w1, w2, p0, pw);
}

// Low-precision operand panels of step k (L21 rows k1.., U12^T) and their
// tensor maps.  *K is the GEMM's k extent and *kpart the pairs layout's lo
// offset (0 when the parts are concatenated: K = nparts * kw).
int build_operands(lu_handle h, const Ctx32& c, int k0, int kw, int k1, int rest, bool bf16, CUtensorMap* mapL,
                   CUtensorMap* mapU, int* K, int* kpart, cudaStream_t s) {
  const float* L21 = c.A + (int64_t)k1 * c.ld + k0;
  const float* U12 = c.A + (int64_t)k0 * c.ld + k1;
  const bool pairs = !bf16 && h->pairs;
  const int kps = (kw + 63) & ~63;
  const int ke = pairs ? 2 * kps : h->nparts * kw;  // tensor-map width
  *K = pairs ? kps : ke;
  *kpart = pairs ? kps : 0;
  {
    Prof pf(h, s, LU_PH_OTHER);
    if (bf16) {
      LUB_TRY(launch_split_rows<__nv_bfloat16>(L21, c.ld, h->Lb, h->ldk, rest, kw, 1, 0u, nullptr, 0, s));
      LUB_TRY(launch_split_transpose<__nv_bfloat16>(U12, c.ld, h->Ub, h->ldk, kw, rest, 1, 0u, nullptr, 1, s));
    } else if (pairs) {
      // [Lh | Ll] and [Uh | Ul], each part kps wide (zero past kw)
      LUB_TRY(launch_panel_absmax(L21, c.ld, rest, kw, U12, c.ld, rest, h->amax, s));
      LUB_TRY(launch_split_rows<__half>(L21, c.ld, reinterpret_cast<__half*>(h->Lb), h->ldk, rest, kw, 2, 0x2u,
                                        h->amax, 0, s, kps));
      LUB_TRY(launch_split_transpose<__half>(U12, c.ld, reinterpret_cast<__half*>(h->Ub), h->ldk, kw, rest, 2, 0x2u,
                                             h->amax, 1, s, kps));
    } else {
      // L parts [hi, hi, lo] against U parts [hi, lo, hi]: Lh*Uh + Lh*Ul + Ll*Uh
      LUB_TRY(launch_panel_absmax(L21, c.ld, rest, kw, U12, c.ld, rest, h->amax, s));
      LUB_TRY(launch_split_rows<__half>(L21, c.ld, reinterpret_cast<__half*>(h->Lb), h->ldk, rest, kw, h->nparts,
                                        0x4u, h->amax, 0, s));
      LUB_TRY(launch_split_transpose<__half>(U12, c.ld, reinterpret_cast<__half*>(h->Ub), h->ldk, kw, rest,
                                             h->nparts, 0x2u, h->amax, 1, s));
    }
  }
  const CUtensorMapDataType dt = bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
  LUB_TRY(encode_tmap_2d(mapL, dt, 2, h->Lb, ke, rest, h->ldk * 2, 64, 128, CU_TENSOR_MAP_SWIZZLE_128B));
  LUB_TRY(encode_tmap_2d(mapU, dt, 2, h->Ub, ke, rest, h->ldk * 2, 64, 128, CU_TENSOR_MAP_SWIZZLE_128B));
  return LU_OK;
}

// Pairs-layout operands of step k for the update of trailing columns
// [u0, u0+ncols) only: the U12^T rows of those columns (and, with with_l,
// all of L21). amax[0], amax[1] receive max|L21| and max|U12| over those
// columns, and set the scales; a later part with its own amax pair scales
// its U rows by its own maximum (L21's maximum is the same number). The
// tensor maps cover every trailing column, as build_operands' do.
int build_operands_part(lu_handle h, const Ctx32& c, int k0, int kw, int k1, int rest, int u0, int ncols,
                        bool with_l, unsigned* amax, CUtensorMap* mapL, CUtensorMap* mapU, int* K, int* kpart,
                        cudaStream_t s) {
  const float* L21 = c.A + (int64_t)k1 * c.ld + k0;
  const float* U12 = c.A + (int64_t)k0 * c.ld + k1 + u0;
  const int kps = (kw + 63) & ~63;
  *K = kps;
  *kpart = kps;
  {
    Prof pf(h, s, LU_PH_OTHER);
    // a later part of the same step has L21's maximum already (amax pair 0)
    LUB_TRY(launch_panel_absmax(L21, c.ld, rest, kw, U12, c.ld, ncols, amax, s, with_l ? nullptr : h->amax));
    if (with_l)
      LUB_TRY(launch_split_rows<__half>(L21, c.ld, reinterpret_cast<__half*>(h->Lb), h->ldk, rest, kw, 2, 0x2u, amax,
                                        0, s, kps));
    LUB_TRY(launch_split_transpose<__half>(U12, c.ld, reinterpret_cast<__half*>(h->Ub) + (int64_t)u0 * h->ldk,
                                           h->ldk, kw, ncols, 2, 0x2u, amax, 1, s, kps));
  }
  LUB_TRY(encode_tmap_2d(mapL, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, h->Lb, 2 * kps, rest, h->ldk * 2, 64, 128,
                         CU_TENSOR_MAP_SWIZZLE_128B));
  return encode_tmap_2d(mapU, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, h->Ub, 2 * kps, rest, h->ldk * 2, 64, 128,
                        CU_TENSOR_MAP_SWIZZLE_128B);
}

// C(k1.., c0..c0+ncols) -= L21 * U12[:, u0..u0+ncols] on the tensor cores
// (reserve: SMs left free for a panel running beside it).  K and kpart as
// from build_operands; flops are counted as executed on the panel's kw
// columns (three products for the FP16 split).
// tile_ctr: a zeroed counter shared with a helper launch of the same
// product (helper_ctas > 0 makes this call that helper: it is not timed as
// a phase, since the main launch's span covers the whole product).
int lowp_gemm(lu_handle h, const CUtensorMap& mapL, const CUtensorMap& mapU, const CUtensorMap& mapC, int k1,
              int rest, int u0, int ncols, int K, int kpart, int kw, bool bf16, cudaStream_t s, int reserve = 0,
              unsigned* tile_ctr = nullptr, int helper_ctas = 0, const unsigned* amax_in = nullptr) {
  const unsigned* amax = bf16 ? nullptr : (amax_in ? amax_in : h->amax);
  // the main launch and its helper take the same kernel (one tile numbering)
  const bool pair = h->gemm_pair && kpart > 0;
  if (helper_ctas > 0)
    return launch_gemm_lowp_persistent(mapL, mapU, mapC, 0, u0, k1, k1 + u0, rest, ncols, K, bf16, amax, h->st,
                                       h->spin, helper_ctas, s, kpart, tile_ctr, pair);
  const int prods = bf16 ? 1 : (h->cfg.precision == LU_PREC_FP16X3 ? 3 : 1);
  Prof pf(h, s, LU_PH_GEMM, 2.0 * rest * (double)ncols * kw * prods);
  if (h->gemm_ctas > 0)
    return launch_gemm_lowp_persistent(mapL, mapU, mapC, 0, u0, k1, k1 + u0, rest, ncols, K, bf16, amax, h->st,
                                       h->spin, std::max(1, h->gemm_ctas - reserve), s, kpart, tile_ctr, pair);
  return launch_gemm_bf16_tc(mapL, mapU, mapC, 0, u0, k1, k1 + u0, rest, ncols, K, bf16, amax, h->st, h->spin, s);
}

// One look-ahead step with the next panel's columns first (pairs layout):
// on the main stream the interchanges, U solve, operands and update of
// panel k+1's nw columns; then panel k+1 starts on the panel stream while
// the main stream does the same for every other column (interchanges on
// the left columns and the row permutation included). The rest's U rows
// get their own scale (h->amax[2..3]); the helper launch, if any, waits
// for them. Per column the interchanges, U solve and products are the same
// operations as in the one-pass schedule.
int factor_mixed_split_step(lu_handle h, Ctx32& c, Ctx32& cp, const CUtensorMap& mapC, int k0, int kw,
                            cudaStream_t s) {
  const int n = (int)h->cfg.n, B = h->cfg.block_size;
  const int k1 = k0 + kw, rest = n - k1, nw = std::min(B, rest);
  LUB_TRY(pivots_apply_f32(c, k0, kw, k1, k1 + nw, 0, 0, nullptr));
  LUB_TRY(trsm32(c, k0, kw, k0, k1, nw));
  CUtensorMap mapL, mapU;
  int K = 0, kpart = 0;
  LUB_TRY(build_operands_part(h, c, k0, kw, k1, rest, 0, nw, true, h->amax, &mapL, &mapU, &K, &kpart, s));
  LUB_TRY(lowp_gemm(h, mapL, mapU, mapC, k1, rest, 0, nw, K, kpart, kw, false, s));  // next panel's columns
  LUB_CUDA(cudaEventRecord(h->evN, s));
  LUB_CUDA(cudaStreamWaitEvent(h->sP, h->evN, 0));
  std::vector<cudaGraphNode_t> mark;
  if (h->capturing) LUB_TRY(capture_deps(h->sP, &mark));
  LUB_TRY(panel32(cp, k1, nw, k1, nw));
  if (h->capturing) LUB_TRY(mark_branch_priority(h, h->sP, mark));
  // every other column: the left L columns, and the trailing ones past the
  // next panel (the panel's own columns are being factored beside this)
  LUB_TRY(pivots_apply_f32(c, k0, kw, 0, n, k0, k1 + nw, h->perm, kw <= 512));
  if (rest == nw) {
    LUB_CUDA(cudaEventRecord(h->evP, h->sP));
    return LU_OK;
  }
  LUB_TRY(trsm32(c, k0, kw, k0, k1 + nw, rest - nw));
  CUtensorMap mapL2, mapU2;
  LUB_TRY(build_operands_part(h, c, k0, kw, k1, rest, nw, rest - nw, false, h->amax + 2, &mapL2, &mapU2, &K, &kpart,
                              s));
  unsigned* ctr = (h->gemm_helper && h->gemm_ctas > 0 && h->gemm_reserve > 0) ? h->take_counter() : nullptr;
  if (ctr) {
    LUB_CUDA(cudaEventRecord(h->evR, s));
    LUB_CUDA(cudaStreamWaitEvent(h->sP, h->evR, 0));
    LUB_TRY(lowp_gemm(h, mapL2, mapU2, mapC, k1, rest, nw, rest - nw, K, kpart, kw, false, h->sP, 0, ctr,
                      h->gemm_reserve, h->amax + 2));
  }
  LUB_CUDA(cudaEventRecord(h->evP, h->sP));
  return lowp_gemm(h, mapL2, mapU2, mapC, k1, rest, nw, rest - nw, K, kpart, kw, false, s, h->gemm_reserve, ctr, 0,
                   h->amax + 2);
}

// LU of h->A32 in place: FP32 panels/TRSM, low-precision tcgen05 trailing
// updates; with look-ahead, panel k+1 overlaps the rest of update k.
// rest_src (look-ahead only): h->A32 holds only the first panel's columns;
// the FP64 source of the other columns (leading dimension rest_lda) is
// converted on the main stream while the first panel is factored.
int factor_mixed(lu_handle h, cudaStream_t s, const double* rest_src, int64_t rest_lda) {
  const int n = (int)h->cfg.n, B = h->cfg.block_size;
  const bool bf16 = h->cfg.precision == LU_PREC_BF16;
  const bool la = h->cfg.lookahead != 0;
  // the tournament-pivoting leaf handles widths up to 32
  const int lw = la ? h->leaf_w32_la : h->leaf_w32;
  Ctx32 c{h, h->A32, h->ld32, n, h->ipiv32, s, h->cfg.sing_threshold, h->plist,
          h->tslu ? std::min(lw, 32) : lw, la ? h->leaf_ctas_la : h->leaf_ctas};
  CUtensorMap mapC;
  LUB_TRY(encode_tmap_2d(&mapC, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, h->A32, n, n, h->ld32 * 4, 32, 128,
                         CU_TENSOR_MAP_SWIZZLE_128B));
  LUB_CUDA(cudaMemsetAsync(h->counters, 0, sizeof(unsigned) * h->n_counters, s));
  h->next_counter = 0;
  LUB_TRY(launch_iota(h->perm, n, s));
  if (!la) {
    for (int k0 = 0; k0 < n; k0 += B) {
      const int kw = std::min(B, n - k0);
      LUB_TRY(panel32(c, k0, kw, k0, kw));
      LUB_TRY(pivots_apply_f32(c, k0, kw, 0, n, k0, k0 + kw, h->perm));
      const int k1 = k0 + kw, rest = n - k1;
      if (rest <= 0) continue;
      LUB_TRY(trsm32(c, k0, kw, k0, k1, rest));
      CUtensorMap mapL, mapU;
      int K = 0, kpart = 0;
      LUB_TRY(build_operands(h, c, k0, kw, k1, rest, bf16, &mapL, &mapU, &K, &kpart, s));
      LUB_TRY(lowp_gemm(h, mapL, mapU, mapC, k1, rest, 0, rest, K, kpart, kw, bf16, s));
    }
    return LU_OK;
  }
  Ctx32 cp = c;
  cp.s = h->sP;
  cp.pl = h->plistP;
  // under capture the panel stream's kernel nodes are marked for its priority
  std::vector<cudaGraphNode_t> mark;
  LUB_CUDA(cudaEventRecord(h->evFork, s));
  LUB_CUDA(cudaStreamWaitEvent(h->sP, h->evFork, 0));
  if (h->capturing) LUB_TRY(capture_deps(h->sP, &mark));
  LUB_TRY(panel32(cp, 0, std::min(B, n), 0, std::min(B, n)));
  if (h->capturing) LUB_TRY(mark_branch_priority(h, h->sP, mark));
  LUB_CUDA(cudaEventRecord(h->evP, h->sP));
  if (rest_src && B < n) {
    Prof pf(h, s, LU_PH_OTHER);
    LUB_TRY(launch_f64_to_f32(rest_src + B, rest_lda, h->A32 + B, h->ld32, n, n - B, s));
  }
  const bool split = h->la_split && h->pairs && !bf16;
  for (int k0 = 0; k0 < n; k0 += B) {
    const int kw = std::min(B, n - k0), k1 = k0 + kw, rest = n - k1;
    LUB_CUDA(cudaStreamWaitEvent(s, h->evP, 0));
    if (split && rest > 0) {
      LUB_TRY(factor_mixed_split_step(h, c, cp, mapC, k0, kw, s));
      continue;
    }
    LUB_TRY(pivots_apply_f32(c, k0, kw, 0, n, k0, k1, h->perm));
    if (rest <= 0) continue;
    LUB_TRY(trsm32(c, k0, kw, k0, k1, rest));
    CUtensorMap mapL, mapU;
    int K = 0, kpart = 0;
    LUB_TRY(build_operands(h, c, k0, kw, k1, rest, bf16, &mapL, &mapU, &K, &kpart, s));
    const int nw = std::min(B, rest);
    LUB_TRY(lowp_gemm(h, mapL, mapU, mapC, k1, rest, 0, nw, K, kpart, kw, bf16, s));  // next panel's columns
    LUB_CUDA(cudaEventRecord(h->evN, s));
    LUB_CUDA(cudaStreamWaitEvent(h->sP, h->evN, 0));
    if (h->capturing) LUB_TRY(capture_deps(h->sP, &mark));
    LUB_TRY(panel32(cp, k1, nw, k1, nw));
    if (h->capturing) LUB_TRY(mark_branch_priority(h, h->sP, mark));
    // The rest of update k runs on the SMs the panel leaves free; once the
    // panel is done, a helper launch on its stream takes the remaining
    // tiles from the same counter, so the reserved SMs do not idle.
    unsigned* ctr =
        (rest > nw && h->gemm_helper && h->gemm_ctas > 0 && h->gemm_reserve > 0) ? h->take_counter() : nullptr;
    if (ctr)
      LUB_TRY(lowp_gemm(h, mapL, mapU, mapC, k1, rest, nw, rest - nw, K, kpart, kw, bf16, h->sP, 0, ctr,
                        h->gemm_reserve));
    LUB_CUDA(cudaEventRecord(h->evP, h->sP));
    if (rest > nw)
      LUB_TRY(lowp_gemm(h, mapL, mapU, mapC, k1, rest, nw, rest - nw, K, kpart, kw, bf16, s, h->gemm_reserve,
                        ctr));
  }
  return LU_OK;
}

int solve32(lu_handle h, float* v, cudaStream_t s) {
  const int n = (int)h->cfg.n;
  Prof pf(h, s, LU_PH_SOLVE, 2.0 * n * (double)n);
  LUB_TRY(launch_trsv<float>(h->A32, h->ld32, n, v, 0, h->trsv_flags, h->trsv_ticket, h->st, h->spin, s));
  return launch_trsv<float>(h->A32, h->ld32, n, v, 1, h->trsv_flags, h->trsv_ticket, h->st, h->spin, s);
}

// M^{-1} v in working precision: FP32 factors, FP64 vector and arithmetic
int solve_f32_factors_f64(lu_handle h, double* v, cudaStream_t s) {
  const int n = (int)h->cfg.n;
  Prof pf(h, s, LU_PH_SOLVE, 2.0 * n * (double)n);
  LUB_TRY((launch_trsv_mixed<float, double>(h->A32, h->ld32, n, v, 0, h->trsv_flags, h->trsv_ticket, h->st,
                                             h->spin, s)));
  return launch_trsv_mixed<float, double>(h->A32, h->ld32, n, v, 1, h->trsv_flags, h->trsv_ticket, h->st, h->spin,
                                           s);
}

double bits_to_double(unsigned long long v) {
  double x;
  memcpy(&x, &v, 8);
  return x;
}

// The FP64 matrix the mixed path reads (conversion, residuals, GMRES
// products): in device memory, or in host memory (host = true) and passed
// through the GPU row by row.
struct ASrc {
  const double* A;
  int64_t lda;
  bool host;
};

int ensure_staging(lu_handle h, int64_t lda) {
  const int64_t rows = std::max<int64_t>(1, (int64_t)(h->stage_bytes / sizeof(double)) / lda);
  const int64_t need = rows * lda;
  if (h->stage[0] && h->stage_elems >= need) return LU_OK;
  for (int b = 0; b < 2; b++) {
    h->release(h->stage[b]);
    h->stage[b] = nullptr;
    LUB_TRY(h->alloc(&h->stage[b], (size_t)need));
    if (!h->evReady[b]) LUB_CUDA(cudaEventCreateWithFlags(&h->evReady[b], cudaEventDisableTiming));
    if (!h->evFree[b]) LUB_CUDA(cudaEventCreateWithFlags(&h->evFree[b], cudaEventDisableTiming));
  }
  if (!h->sCopy) LUB_CUDA(cudaStreamCreateWithFlags(&h->sCopy, cudaStreamNonBlocking));
  h->stage_elems = need;
  return LU_OK;
}

// Sizes the device copy of the host matrix's leading rows: every row that
// fits in free device memory less a margin (2 GB or 1/32 of the device, for
// the refinement's later buffers), at most h->resident_cap bytes. The
// current copy counts as free, since it is replaced. Sets h->res_rows.
int ensure_resident(lu_handle h, int64_t lda, int n) {
  size_t free_b = 0, total_b = 0;
  LUB_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const size_t have = (size_t)h->res_elems * sizeof(double);
  const size_t margin = std::max<size_t>(size_t(2) << 30, total_b / 32);
  size_t budget = free_b + have > margin ? free_b + have - margin : 0;
  budget = std::min(budget, h->resident_cap);
  int64_t rows = std::min<int64_t>(n, (int64_t)(budget / (sizeof(double) * (size_t)lda)));
  h->res_rows = 0;
  if (rows <= 0) return LU_OK;
  if (h->res_elems < rows * lda) {
    h->release(h->resA);
    h->resA = nullptr;
    h->res_elems = 0;
    // a failed allocation (fragmentation) halves the request
    while (rows > 0 && h->alloc(&h->resA, (size_t)(rows * lda)) != LU_OK) rows /= 2;
    if (rows <= 0) return LU_OK;
    h->res_elems = rows * lda;
  }
  h->res_rows = (int)rows;
  return LU_OK;
}

// One pass over the rows of the host matrix. Rows below h->res_rows are
// copied into h->resA when fill is set (the conversion pass) and read there
// in place otherwise; the other rows pass in chunks through the two staging
// buffers. Copies run on h->sCopy and overlap the kernels that
// f(rows_dev, row0, rows) launches on s; rows_dev has pitch lda.
template <class F>
int stream_host_rows(lu_handle h, const double* hA, int64_t lda, int n, bool fill, cudaStream_t s, F f) {
  LUB_TRY(ensure_staging(h, lda));
  const int R = (int)std::min<int64_t>(n, h->stage_elems / lda);
  const int nres = h->res_rows;
  for (int b = 0; b < 2; b++) LUB_CUDA(cudaEventRecord(h->evFree[b], s));
  if (!fill && nres > 0) LUB_TRY(f(static_cast<const double*>(h->resA), 0, nres));
  for (int c = fill ? 0 : nres, k = 0; c < n; k++) {
    const int b = k & 1;
    const bool res = c < nres;
    const int rows = std::min(R, (res ? nres : n) - c);
    double* dst = res ? h->resA + (int64_t)c * lda : h->stage[b];
    LUB_CUDA(cudaStreamWaitEvent(h->sCopy, h->evFree[b], 0));  // earlier readers of dst on s are done
    LUB_CUDA(cudaMemcpyAsync(dst, hA + (int64_t)c * lda, sizeof(double) * (size_t)rows * lda,
                             cudaMemcpyHostToDevice, h->sCopy));
    h->host_copied += (int64_t)sizeof(double) * rows * lda;
    LUB_CUDA(cudaEventRecord(h->evReady[b], h->sCopy));
    LUB_CUDA(cudaStreamWaitEvent(s, h->evReady[b], 0));
    LUB_TRY(f(static_cast<const double*>(dst), c, rows));
    if (!res) LUB_CUDA(cudaEventRecord(h->evFree[b], s));
    c += rows;
  }
  return LU_OK;
}

// r = b - A x with the norms in h->racc (cleared first)
int residual_src(lu_handle h, const ASrc& a, const double* x, const double* b, double* r, cudaStream_t s) {
  const int n = (int)h->cfg.n;
  if (!a.host) return launch_residual_f64(a.A, a.lda, n, x, b, r, h->racc, s);
  LUB_CUDA(cudaMemsetAsync(h->racc, 0, sizeof(ResidualAccum), s));
  return stream_host_rows(h, a.A, a.lda, n, false, s, [&](const double* rows_dev, int r0, int rows) {
    return launch_residual_f64_rows(rows_dev, a.lda, rows, r0, n, x, b, r, h->racc, s);
  });
}

// r = b - A x, its norms, and r_hpl (synchronises).
int residual_hpl(lu_handle h, const ASrc& A, const double* x, const double* b, double* r, double* r_hpl,
                 double* rnorm, cudaStream_t s) {
  const int n = (int)h->cfg.n;
  {
    Prof pf(h, s, LU_PH_OTHER);
    LUB_TRY(residual_src(h, A, x, b, r, s));
  }
  LUB_CUDA(cudaMemcpyAsync(h->racc_host, h->racc, sizeof(ResidualAccum), cudaMemcpyDeviceToHost, s));
  LUB_CUDA(cudaStreamSynchronize(s));
  const ResidualAccum& a = *h->racc_host;
  const double eps = 2.220446049250313e-16;
  const double an = bits_to_double(a.anorm), xn = bits_to_double(a.xmax), bn = bits_to_double(a.bmax),
               rn = bits_to_double(a.rmax);
  *rnorm = rn;
  *r_hpl = rn / ((an * xn + bn) * (double)n * eps);
  return LU_OK;
}

int device_status(lu_handle h, cudaStream_t s) {
  DevStatus st;
  LUB_CUDA(cudaMemcpyAsync(&st, h->st, sizeof(st), cudaMemcpyDeviceToHost, s));
  LUB_CUDA(cudaStreamSynchronize(s));
  return st.code != 0 ? st.code : st.info;
}

// Flexible GMRES on the correction equation op(A) d = r, right
// preconditioned: Arnoldi on op(A) M^{-1} in FP64 with two passes of
// classical Gram-Schmidt, where M^{-1} (the FP32 factors applied in FP64
// arithmetic) maps each basis vector v_j to z_j = M^{-1} v_j, kept in Z.  The
// correction is d = Z y, with y minimising ||r - op(A) Z y||_2 over the
// Krylov space, so each cycle minimises the true residual of the correction
// equation (Saad, SIAM J. Sci. Comput. 14(2), 1993), not the preconditioned
// one.  The cycle ends after gm steps or once that residual has fallen by
// tol.  x += d.
//   init(v0):    v0 = r / rnorm  (rnorm = ||r||inf keeps the vectors O(1))
//   prec(v, z):  z = M^{-1} v
//   op(z, w):    w = op(A) z
template <class Init, class Prec, class Op>
int fgmres_cycle(lu_handle h, double* x, double rnorm, double tol, cudaStream_t s, int* iters_out, Init init,
                 Prec prec, Op op) {
  LUB_TRY(ensure_gmres(h));
  const int n = (int)h->cfg.n, m = h->gm;
  double* V = h->V;
  double* Z = h->Z;
  double* part = h->hdot;
  double* hd = h->hdot + 128 * (m + 2);  // m + 2 doubles of results
  std::vector<double> H((size_t)(m + 1) * m, 0.0), cs(m), sn(m), g(m + 1, 0.0), hcol(m + 1);
  LUB_TRY(init(V));
  LUB_TRY(launch_multi_dot(V, 1, V, n, part, hd, s));
  double beta2 = 0.0;
  LUB_CUDA(cudaMemcpyAsync(&beta2, hd, sizeof(double), cudaMemcpyDeviceToHost, s));
  LUB_CUDA(cudaStreamSynchronize(s));
  const double beta = std::sqrt(beta2);
  if (!(beta > 0.0) || !std::isfinite(beta)) return LU_ERR_NONFINITE;
  LUB_TRY(launch_scale_copy(V, V, n, hd, s));
  g[0] = beta * rnorm;
  int k = 0;
  for (int j = 0; j < m; j++) {
    double* vj = V + (size_t)j * n;
    double* zj = Z + (size_t)j * n;
    double* w = V + (size_t)(j + 1) * n;
    LUB_TRY(prec(vj, zj));
    LUB_TRY(op(zj, w));
    // two passes of classical Gram-Schmidt
    std::fill(hcol.begin(), hcol.end(), 0.0);
    for (int pass = 0; pass < 2; pass++) {
      LUB_TRY(launch_multi_dot(V, j + 1, w, n, part, hd, s));
      LUB_TRY(launch_multi_axpy(w, V, j + 1, hd, n, -1.0, s));
      std::vector<double> tmp(j + 1);
      LUB_CUDA(cudaMemcpyAsync(tmp.data(), hd, sizeof(double) * (j + 1), cudaMemcpyDeviceToHost, s));
      LUB_CUDA(cudaStreamSynchronize(s));
      for (int i = 0; i <= j; i++) hcol[i] += tmp[i];
    }
    LUB_TRY(launch_multi_dot(w, 1, w, n, part, hd, s));
    double hn2 = 0.0;
    LUB_CUDA(cudaMemcpyAsync(&hn2, hd, sizeof(double), cudaMemcpyDeviceToHost, s));
    LUB_CUDA(cudaStreamSynchronize(s));
    if (!std::isfinite(hn2)) break;  // keep the steps taken so far
    hcol[j + 1] = std::sqrt(hn2);
    if (hcol[j + 1] > 0.0) LUB_TRY(launch_scale_copy(w, w, n, hd, s));
    // Givens rotations
    for (int i = 0; i < j; i++) {
      const double t = cs[i] * hcol[i] + sn[i] * hcol[i + 1];
      hcol[i + 1] = -sn[i] * hcol[i] + cs[i] * hcol[i + 1];
      hcol[i] = t;
    }
    const double den = std::hypot(hcol[j], hcol[j + 1]);
    cs[j] = den > 0 ? hcol[j] / den : 1.0;
    sn[j] = den > 0 ? hcol[j + 1] / den : 0.0;
    hcol[j] = den;
    hcol[j + 1] = 0.0;
    g[j + 1] = -sn[j] * g[j];
    g[j] = cs[j] * g[j];
    for (int i = 0; i <= j; i++) H[(size_t)i * m + j] = hcol[i];
    k = j + 1;
    if (std::fabs(g[j + 1]) <= tol * beta * rnorm || !(hcol[j] > 0.0)) break;
  }
  // y = H(1:k,1:k)^{-1} g(1:k); d = Z y; x += d
  std::vector<double> y(k, 0.0);
  for (int i = k - 1; i >= 0; i--) {
    double t = g[i];
    for (int q = i + 1; q < k; q++) t -= H[(size_t)i * m + q] * y[q];
    const double d = H[(size_t)i * m + i];
    y[i] = d != 0.0 ? t / d : 0.0;
  }
  if (k > 0) {
    LUB_CUDA(cudaMemcpyAsync(hd, y.data(), sizeof(double) * k, cudaMemcpyHostToDevice, s));
    LUB_TRY(launch_multi_axpy(x, Z, k, hd, n, 1.0, s));
  }
  LUB_CUDA(cudaStreamSynchronize(s));
  *iters_out = k;
  return LU_OK;
}

double gmres_tol(lu_handle h) { return h->cfg.gmres_tol > 0.0 ? h->cfg.gmres_tol : kGmresTol; }
int ir_stall_limit(lu_handle h) { return h->cfg.ir_stall > 0 ? h->cfg.ir_stall : kIrStall; }

// z = M^{-1} v for the single-RHS solve: P, then the FP32 factors (FP64
// vector and arithmetic)
int prec_vec(lu_handle h, const int32_t* perm, const double* v, double* z, cudaStream_t s) {
  LUB_TRY(launch_gather_f64(v, perm, z, (int)h->cfg.n, 1.0, nullptr, s));
  return solve_f32_factors_f64(h, z, s);
}

// GMRES cycle of the single-RHS solve A x = b (residual in h->r64, its
// norms in h->racc)
int gmres_correction(lu_handle h, const ASrc& A, double* x, double rnorm, cudaStream_t s, int* iters_out) {
  const int n = (int)h->cfg.n;
  auto init = [&](double* v0) { return launch_scale_vec(h->r64, v0, n, 1.0 / rnorm, s); };
  auto prec = [&](const double* v, double* z) { return prec_vec(h, h->perm, v, z, s); };
  auto op = [&](const double* z, double* w) {
    {  // residual kernel with b = 0 gives -A z
      Prof pf(h, s, LU_PH_OTHER);
      LUB_TRY(residual_src(h, A, z, h->zero64, h->z64, s));
    }
    return launch_scale_vec(h->z64, w, n, -1.0, s);
  };
  return fgmres_cycle(h, x, rnorm, gmres_tol(h), s, iters_out, init, prec, op);
}

// FP32 working copy of A and its low-precision factorisation (h->A32,
// h->perm); the status word is cleared first
int mixed_factor(lu_handle h, const double* A, int64_t lda, cudaStream_t s) {
  const int n = (int)h->cfg.n;
  LUB_TRY(ensure_mixed(h));
  LUB_CUDA(cudaMemsetAsync(h->st, 0, sizeof(DevStatus), s));
  return run_graph(h, 1, A, h->A32, nullptr, lda, s, [&](cudaStream_t ss) {
    // with look-ahead the first panel starts once its own columns are in
    // FP32; the other columns are converted beside it
    const int b0 = h->cfg.lookahead ? std::min<int>((int)h->cfg.block_size, n) : n;
    {
      Prof pf(h, ss, LU_PH_OTHER);
      LUB_TRY(launch_f64_to_f32(A, lda, h->A32, h->ld32, n, b0, ss));
    }
    return factor_mixed(h, ss, b0 < n ? A : nullptr, lda);
  });
}

// The host matrix in FP32 into h->A32 (the device copy of its leading rows
// refreshed on the way), then the low-precision factorisation. No graph
// replay: the copies depend on the caller's host pointer.
int mixed_factor_host(lu_handle h, const ASrc& a, cudaStream_t s) {
  const int n = (int)h->cfg.n;
  LUB_TRY(ensure_mixed(h));
  LUB_CUDA(cudaMemsetAsync(h->st, 0, sizeof(DevStatus), s));
  LUB_TRY(ensure_staging(h, a.lda));
  LUB_TRY(ensure_resident(h, a.lda, n));
  {
    Prof pf(h, s, LU_PH_OTHER);
    LUB_TRY(stream_host_rows(h, a.A, a.lda, n, true, s, [&](const double* rows_dev, int r0, int rows) {
      return launch_f64_to_f32(rows_dev, a.lda, h->A32 + (int64_t)r0 * h->ld32, h->ld32, rows, n, s);
    }));
  }
  return factor_mixed(h, s, nullptr, 0);
}

int refine_solve(lu_handle h, const ASrc& A, const double* b, double* x, lu_refine_info* info, cudaStream_t s) {
  const int n = (int)h->cfg.n;
  const int64_t copied0 = h->host_copied;
  h->mixed_factored = false;
  if (A.host) {
    LUB_TRY(mixed_factor_host(h, A, s));
  } else {
    LUB_TRY(mixed_factor(h, A.A, A.lda, s));
  }
  // x0 = U^{-1} L^{-1} P b in FP32
  LUB_TRY(launch_gather_f64_to_f32(b, h->perm, h->v32, n, 1.0, s));
  LUB_TRY(solve32(h, h->v32, s));
  LUB_TRY(launch_f32_to_f64(h->v32, x, n, 1.0, s));
  const int fst = device_status(h, s);
  lu_refine_info ri;
  memset(&ri, 0, sizeof(ri));
  if (fst != LU_OK) {
    ri.status = fst;
    ri.host_bytes = h->host_copied - copied0;
    if (info) *info = ri;
    return LU_OK;  // numerical status is reported through lu_status / info
  }
  const double target = h->cfg.ir_target > 0 ? h->cfg.ir_target : 16.0;
  const int max_it = h->cfg.ir_max_iter > 0 ? h->cfg.ir_max_iter : 50;
  const int stall_limit = ir_stall_limit(h);
  bool gm = h->cfg.ir_mode == LU_IR_GMRES;
  const size_t nb = sizeof(double) * (size_t)n;
  // the iterate with the smallest ||b - A x||inf so far, its residual and
  // norms: a step that does not lower that norm is rolled back to it
  double r_hpl = INFINITY, rn = 0.0;
  LUB_TRY(residual_hpl(h, A, x, b, h->r64, &r_hpl, &rn, s));
  ri.r_hpl_initial = r_hpl;
  double best_rn = rn, best_hpl = r_hpl;
  auto save_best = [&]() -> int {
    LUB_CUDA(cudaMemcpyAsync(h->xbest, x, nb, cudaMemcpyDeviceToDevice, s));
    LUB_CUDA(cudaMemcpyAsync(h->rbest, h->r64, nb, cudaMemcpyDeviceToDevice, s));
    LUB_CUDA(cudaMemcpyAsync(h->racc_best, h->racc, sizeof(ResidualAccum), cudaMemcpyDeviceToDevice, s));
    return LU_OK;
  };
  LUB_TRY(save_best());
  int stall = 0, steps = 0;
  while (std::isfinite(r_hpl) && !(r_hpl < target) && steps < max_it) {
    steps++;
    const bool gm_step = gm;
    if (gm_step) {
      int k = 0;
      LUB_TRY(gmres_correction(h, A, x, rn, s, &k));
      ri.used_gmres = 1;
      ri.gmres_iterations += k;
    } else {
      LUB_TRY(launch_ir_prep(h->r64, h->perm, h->v32, n, h->racc, s));
      LUB_TRY(solve32(h, h->v32, s));
      LUB_TRY(launch_ir_update(x, h->v32, n, h->racc, s));
      ri.iterations++;
    }
    double new_hpl = INFINITY, new_rn = INFINITY;
    LUB_TRY(residual_hpl(h, A, x, b, h->r64, &new_hpl, &new_rn, s));
    if (std::isfinite(new_rn) && new_rn < best_rn) {  // accepted
      // classical steps that contract by less than 2x hand over to GMRES;
      // GMRES cycles that gain less than 10% count towards the stall limit
      if (!gm_step && !(new_hpl < 0.5 * best_hpl) && ri.iterations >= 2) gm = true;
      if (gm_step) stall = (new_hpl > 0.9 * best_hpl) ? stall + 1 : 0;
      best_rn = new_rn;
      best_hpl = new_hpl;
      r_hpl = new_hpl;
      rn = new_rn;
      LUB_TRY(save_best());
    } else {  // rolled back to the best iterate and its residual
      LUB_CUDA(cudaMemcpyAsync(x, h->xbest, nb, cudaMemcpyDeviceToDevice, s));
      LUB_CUDA(cudaMemcpyAsync(h->r64, h->rbest, nb, cudaMemcpyDeviceToDevice, s));
      LUB_CUDA(cudaMemcpyAsync(h->racc, h->racc_best, sizeof(ResidualAccum), cudaMemcpyDeviceToDevice, s));
      r_hpl = best_hpl;
      rn = best_rn;
      ri.rejected++;
      // a GMRES cycle from the same iterate would repeat itself: stop there
      if (gm_step) break;
      gm = true;
    }
    if (stall >= stall_limit) break;
  }
  ri.r_hpl = r_hpl;
  ri.status = (std::isfinite(r_hpl) && r_hpl < target) ? LU_OK : LU_ERR_NOCONV;
  if (ri.status != LU_OK) {
    int code = ri.status;
    LUB_CUDA(cudaMemcpyAsync(&h->st->code, &code, sizeof(int), cudaMemcpyHostToDevice, s));
  }
  ri.host_bytes = h->host_copied - copied0;
  if (info) *info = ri;
  return LU_OK;
}

// ---- multi-RHS refinement on kept factors --------------------------------

int ensure_multi(lu_handle h) {
  if (h->mr_acc) return LU_OK;
  const size_t n = (size_t)h->cfg.n;
  LUB_TRY(h->alloc(&h->mr_P, (size_t)kMultiMaxSplits * n * 16));
  LUB_TRY(h->alloc(&h->mr_Pn, (size_t)kMultiMaxSplits * n));
  LUB_TRY(h->alloc(&h->mr_R, n * 16));
  LUB_TRY(h->alloc(&h->mr_D, n * 16));
  LUB_TRY(h->alloc(&h->mr_X, n * 16));
  LUB_TRY(h->alloc(&h->mr_S, n * 16));
  LUB_TRY(h->alloc(&h->mr_T, n * 16));
  LUB_TRY(h->alloc(&h->mr_dc, n));
  LUB_TRY(h->alloc(&h->mr_Xbest, n * 16));
  LUB_TRY(h->alloc(&h->mr_Rbest, n * 16));
  LUB_TRY(h->alloc(&h->mr_acc, kMultiAccWords));
  LUB_CUDA(cudaMemset(h->mr_S, 0, sizeof(double) * n * 16));
  return LU_OK;
}

// M^{-T} v in place for a contiguous vector (FP32 factors, FP64
// arithmetic): v <- P^T L^{-T} U^{-T} v; tmp is n doubles of scratch
int prec_trans_vec(lu_handle h, double* v, double* tmp, cudaStream_t s) {
  const int n = (int)h->cfg.n;
  Prof pf(h, s, LU_PH_SOLVE, 2.0 * n * (double)n);
  LUB_CUDA(cudaMemcpyAsync(tmp, v, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  LUB_TRY(launch_trsm_pipe<float>(h->A32, h->ld32, n, tmp, 1, 1, 2, h->trsv_flags, h->trsv_ticket, h->st, h->spin,
                                  s));
  LUB_TRY(launch_trsm_pipe<float>(h->A32, h->ld32, n, tmp, 1, 1, 3, h->trsv_flags, h->trsv_ticket, h->st, h->spin,
                                  s));
  return launch_vec_scatter(tmp, h->perm32, v, n, s);
}

// One flexible GMRES cycle on column c of a refinement group: residual in
// h->mr_R[:, c] (||r||inf = rnorm), correction added to h->mr_X[:, c]
int multi_gmres_column(lu_handle h, const double* A, int64_t lda, int trans, int c, double rnorm, int S,
                       int split_len, cudaStream_t s, int* iters) {
  const int n = (int)h->cfg.n;
  auto init = [&](double* v0) { return launch_col_get(h->mr_R, c, nullptr, v0, n, 1.0 / rnorm, s); };
  auto prec = [&](const double* v, double* z) {
    if (!trans) return prec_vec(h, h->perm32, v, z, s);
    LUB_CUDA(cudaMemcpyAsync(z, v, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    return prec_trans_vec(h, z, h->z64, s);
  };
  auto op = [&](const double* z, double* w) {
    if (!trans) {
      {  // residual kernel with b = 0 gives -A z
        Prof pf(h, s, LU_PH_OTHER);
        LUB_TRY(launch_residual_f64(A, lda, n, z, h->zero64, h->z64, h->racc, s));
      }
      return launch_scale_vec(h->z64, w, n, -1.0, s);
    }
    LUB_TRY(launch_col_put(h->mr_S, 0, z, n, 1, s));
    {  // R = 0 - A^T z in column 0
      Prof pf(h, s, LU_PH_OTHER);
      LUB_TRY(launch_multi_residual(A, lda, n, 1, h->mr_S, h->zero64, 1, 1, h->mr_T, h->mr_P, h->mr_Pn, S,
                                    split_len, 0, h->mr_acc, s));
    }
    return launch_col_get(h->mr_T, 0, nullptr, w, n, -1.0, s);
  };
  LUB_CUDA(cudaMemsetAsync(h->mr_dc, 0, sizeof(double) * n, s));
  LUB_TRY(fgmres_cycle(h, h->mr_dc, rnorm, gmres_tol(h), s, iters, init, prec, op));
  return launch_col_put(h->mr_X, c, h->mr_dc, n, 0, s);
}

// x += op(A)^{-1} r through the FP32 factors (FP64 vectors and arithmetic):
//   op = A:   P^T L U d = r   ->  d = U^{-1} L^{-1} (P r)
//   op = A^T: U^T L^T P d = r ->  d = P^T L^{-T} U^{-T} r
// r (h->mr_R) is overwritten in the transposed case.
int multi_correction(lu_handle h, int trans, int k, cudaStream_t s) {
  const int n = (int)h->cfg.n;
  Prof pf(h, s, LU_PH_SOLVE, 2.0 * n * (double)n * k);
  if (!trans) {
    LUB_TRY(launch_permute_rows(h->mr_R, 16, h->mr_D, 16, h->perm32, n, k, 0, s));
    LUB_TRY(launch_trsm_pipe<float>(h->A32, h->ld32, n, h->mr_D, 16, k, 0, h->trsv_flags, h->trsv_ticket, h->st,
                                    h->spin, s));
    LUB_TRY(launch_trsm_pipe<float>(h->A32, h->ld32, n, h->mr_D, 16, k, 1, h->trsv_flags, h->trsv_ticket, h->st,
                                    h->spin, s));
    return launch_multi_add(h->mr_X, h->mr_D, h->perm32, n, k, 0, s);
  }
  LUB_TRY(launch_trsm_pipe<float>(h->A32, h->ld32, n, h->mr_R, 16, k, 2, h->trsv_flags, h->trsv_ticket, h->st,
                                  h->spin, s));
  LUB_TRY(launch_trsm_pipe<float>(h->A32, h->ld32, n, h->mr_R, 16, k, 3, h->trsv_flags, h->trsv_ticket, h->st,
                                  h->spin, s));
  return launch_multi_add(h->mr_X, h->mr_R, h->perm32, n, k, 1, s);
}

// op(A) X = B for k <= 16 columns: low-precision solve, then classical IR
// with the FP64 residual until every column's scaled residual is below the
// target; when classical steps stop contracting (or cfg.ir_mode asks for
// it) each column still above the target gets flexible GMRES-IR cycles
// instead.  Per column, a step that does not lower ||r||inf is rolled back
// to that column's best iterate (and a column whose GMRES cycle was rolled
// back gets no further cycles: it would repeat itself).  ri reports the
// worst column.
int refine_group(lu_handle h, const double* A, int64_t lda, int trans, const double* B, int64_t ldb, double* X,
                 int64_t ldx, int k, lu_refine_info* ri, cudaStream_t s) {
  const int n = (int)h->cfg.n;
  int split_len = 0;
  const int S = multi_residual_splits(n, h->num_sms, &split_len);
  LUB_CUDA(cudaMemsetAsync(h->mr_X, 0, sizeof(double) * n * 16, s));
  LUB_CUDA(cudaMemcpy2DAsync(h->mr_R, 16 * sizeof(double), B, ldb * sizeof(double), k * sizeof(double), n,
                             cudaMemcpyDeviceToDevice, s));
  LUB_TRY(multi_correction(h, trans, k, s));
  const double target = h->cfg.ir_target > 0 ? h->cfg.ir_target : 16.0;
  const int max_it = h->cfg.ir_max_iter > 0 ? h->cfg.ir_max_iter : 50;
  const int stall_limit = ir_stall_limit(h);
  const double eps = 2.220446049250313e-16;
  const size_t blk = sizeof(double) * (size_t)n * 16;
  double anorm = 0.0;
  unsigned long long acc[kMultiAccWords];
  double rc[16], rn[16], best_rn[16], best_rc[16];
  bool frozen[16] = {};
  bool gm = h->cfg.ir_mode == LU_IR_GMRES;
  int stall = 0;
  // residual of the current block and each column's scaled residual
  auto residual = [&](bool first) -> int {
    {
      Prof pf(h, s, LU_PH_OTHER, 2.0 * n * (double)n * k);
      LUB_TRY(launch_multi_residual(A, lda, n, trans, h->mr_X, B, ldb, k, h->mr_R, h->mr_P, h->mr_Pn, S, split_len,
                                    first ? 1 : 0, h->mr_acc, s));
    }
    LUB_CUDA(cudaMemcpyAsync(acc, h->mr_acc, sizeof(acc), cudaMemcpyDeviceToHost, s));
    LUB_CUDA(cudaStreamSynchronize(s));
    if (first) anorm = bits_to_double(acc[48]);
    for (int c = 0; c < k; c++) {
      rn[c] = bits_to_double(acc[c]);
      rc[c] = rn[c] / ((anorm * bits_to_double(acc[32 + c]) + bits_to_double(acc[16 + c])) * (double)n * eps);
    }
    return LU_OK;
  };
  auto worst_of = [&](const double* v) {
    double w = 0.0;
    for (int c = 0; c < k; c++) w = (v[c] > w || std::isnan(v[c])) ? v[c] : w;
    return w;
  };
  LUB_TRY(residual(true));
  LUB_CUDA(cudaMemcpyAsync(h->mr_Xbest, h->mr_X, blk, cudaMemcpyDeviceToDevice, s));
  LUB_CUDA(cudaMemcpyAsync(h->mr_Rbest, h->mr_R, blk, cudaMemcpyDeviceToDevice, s));
  for (int c = 0; c < k; c++) {
    best_rn[c] = std::isfinite(rn[c]) ? rn[c] : INFINITY;
    best_rc[c] = rc[c];
  }
  double worst = worst_of(best_rc);
  if (!(worst <= ri->r_hpl_initial)) ri->r_hpl_initial = worst;  // worst over groups (NaN sticks)
  int classical = 0;
  for (int it = 0; std::isfinite(worst) && !(worst < target) && it < max_it; it++) {
    const bool gm_step = gm;
    if (gm_step) {
      bool any = false;
      for (int c = 0; c < k; c++) {
        if (frozen[c] || !(best_rc[c] >= target) || !(best_rn[c] > 0.0)) continue;
        int iters = 0;
        LUB_TRY(multi_gmres_column(h, A, lda, trans, c, best_rn[c], S, split_len, s, &iters));
        ri->used_gmres = 1;
        ri->gmres_iterations += iters;
        any = true;
      }
      if (!any) break;
    } else {
      LUB_TRY(multi_correction(h, trans, k, s));
      ri->iterations++;
      classical++;
    }
    LUB_TRY(residual(false));
    const double prev_worst = worst;
    bool any_rejected = false;
    for (int c = 0; c < k; c++) {
      if (std::isfinite(rn[c]) && rn[c] < best_rn[c]) {  // accepted
        best_rn[c] = rn[c];
        best_rc[c] = rc[c];
        LUB_TRY(launch_col_copy(h->mr_X, h->mr_Xbest, c, n, s));
        LUB_TRY(launch_col_copy(h->mr_R, h->mr_Rbest, c, n, s));
      } else if (best_rc[c] >= target) {  // rolled back (converged columns keep their best silently)
        any_rejected = true;
        ri->rejected++;
        if (gm_step) frozen[c] = true;
      }
    }
    // every column continues from its best iterate and residual
    LUB_CUDA(cudaMemcpyAsync(h->mr_X, h->mr_Xbest, blk, cudaMemcpyDeviceToDevice, s));
    LUB_CUDA(cudaMemcpyAsync(h->mr_R, h->mr_Rbest, blk, cudaMemcpyDeviceToDevice, s));
    worst = worst_of(best_rc);
    if (!gm_step && (any_rejected || (classical >= 2 && worst > 0.5 * prev_worst))) gm = true;
    if (gm_step) stall = (worst > 0.9 * prev_worst) ? stall + 1 : 0;
    if (stall >= stall_limit) break;
  }
  if (!(worst <= ri->r_hpl)) ri->r_hpl = worst;  // worst over groups (NaN sticks)
  if (!(std::isfinite(worst) && worst < target)) ri->status = LU_ERR_NOCONV;
  LUB_CUDA(cudaMemcpy2DAsync(X, ldx * sizeof(double), h->mr_X, 16 * sizeof(double), k * sizeof(double), n,
                             cudaMemcpyDeviceToDevice, s));
  return LU_OK;
}

int refine_apply(lu_handle h, const double* A, int64_t lda, int trans, const double* B, int64_t ldb, double* X,
                 int64_t ldx, int64_t nrhs, lu_refine_info* info, cudaStream_t s) {
  lu_refine_info ri;
  memset(&ri, 0, sizeof(ri));
  ri.r_hpl = 0.0;
  const int fst = device_status(h, s);
  if (fst != LU_OK) {  // singular factors or an earlier device error
    ri.status = fst;
    if (info) *info = ri;
    return LU_OK;
  }
  LUB_TRY(ensure_multi(h));
  for (int64_t c0 = 0; c0 < nrhs; c0 += 16) {
    const int k = (int)std::min<int64_t>(16, nrhs - c0);
    LUB_TRY(refine_group(h, A, lda, trans, B + c0, ldb, X + c0, ldx, k, &ri, s));
  }
  if (ri.status == LU_OK) {
    const int st = device_status(h, s);
    if (st != LU_OK) ri.status = st;
  } else {
    int code = ri.status;
    LUB_CUDA(cudaMemcpyAsync(&h->st->code, &code, sizeof(int), cudaMemcpyHostToDevice, s));
  }
  if (info) *info = ri;
  return LU_OK;
}

int check_refine_args(lu_handle h, const double* dA, int64_t lda) {
  if (!h || !dA || lda < h->cfg.n) return LU_ERR_ARG;
  if (h->cfg.precision == LU_PREC_FP64 || h->cfg.precision == LU_PREC_FP32) return LU_ERR_UNSUPPORTED;
  if (h->cfg.block_size % 64) return LU_ERR_ARG;  // whole 64-wide k-blocks per panel
  return LU_OK;
}

}  // namespace

extern "C" int lu_refine_factor(lu_handle h, const double* dA, int64_t lda, void* stream) {
  LUB_TRY(check_refine_args(h, dA, lda));
  LUB_TRY(ensure_kernels_init());
  cudaStream_t s = (cudaStream_t)stream;
  h->mixed_factored = false;
  LUB_TRY(mixed_factor(h, dA, lda, s));
  if (!h->perm32) LUB_TRY(h->alloc(&h->perm32, h->cfg.n));
  LUB_CUDA(cudaMemcpyAsync(h->perm32, h->perm, sizeof(int32_t) * h->cfg.n, cudaMemcpyDeviceToDevice, s));
  h->mixed_factored = true;
  return LU_OK;
}

extern "C" int lu_refine_apply(lu_handle h, const double* dA, int64_t lda, int trans, const double* dB, int64_t ldb,
                               double* dX, int64_t ldx, int64_t nrhs, lu_refine_info* info, void* stream) {
  LUB_TRY(check_refine_args(h, dA, lda));
  if (!dB || !dX || nrhs < 1 || ldb < nrhs || ldx < nrhs || (trans != 0 && trans != 1)) return LU_ERR_ARG;
  if ((lda & 1) || (reinterpret_cast<uintptr_t>(dA) & 15)) return LU_ERR_ALIGN;
  if (!h->mixed_factored) return LU_ERR_ARG;  // no lu_refine_factor on this handle
  return refine_apply(h, dA, lda, trans, dB, ldb, dX, ldx, nrhs, info, (cudaStream_t)stream);
}

extern "C" int lu_refine_adjoint(lu_handle h, const double* dA, int64_t lda, const double* dX, int64_t ldx,
                                 const double* dW, int64_t ldw, int64_t nrhs, double* gradB, int64_t ldgb,
                                 double* gradA, int64_t ldga, lu_refine_info* info, void* stream) {
  LUB_TRY(check_refine_args(h, dA, lda));
  if (!dX || !dW || !gradB || nrhs < 1 || ldx < nrhs || ldw < nrhs || ldgb < nrhs) return LU_ERR_ARG;
  if (gradA && ldga < h->cfg.n) return LU_ERR_ARG;
  if ((lda & 1) || (reinterpret_cast<uintptr_t>(dA) & 15)) return LU_ERR_ALIGN;
  if (!h->mixed_factored) return LU_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  lu_refine_info ri;
  LUB_TRY(refine_apply(h, dA, lda, 1, dW, ldw, gradB, ldgb, nrhs, &ri, s));
  if (info) *info = ri;
  if (gradA && ri.status == LU_OK) {
    const int n = (int)h->cfg.n;
    Prof pf(h, s, LU_PH_OTHER, 2.0 * n * (double)n * nrhs);
    LUB_TRY(launch_neg_outer(gradB, ldgb, dX, ldx, n, (int)nrhs, gradA, ldga, s));
  }
  return LU_OK;
}

// Power iteration on E = I - M^{-1} A, M the low-precision factors of the
// last lu_refine_factor (applied in FP64 arithmetic): v_{i+1} = E v_i /
// ||E v_i||_2 from a seeded uniform start; *est receives ||E v||_2 for the
// last unit v, a lower bound on ||E||_2 that approaches E's spectral radius.
// Classical refinement contracts by about that factor per step (it
// converges when it is below 1); GMRES-IR needs only M^{-1} A well enough
// conditioned.
extern "C" int lu_refine_precond_norm(lu_handle h, const double* dA, int64_t lda, int32_t iters, double* est,
                                      void* stream) {
  LUB_TRY(check_refine_args(h, dA, lda));
  if (!est || iters < 1) return LU_ERR_ARG;
  if ((lda & 1) || (reinterpret_cast<uintptr_t>(dA) & 15)) return LU_ERR_ALIGN;
  if (!h->mixed_factored) return LU_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int n = (int)h->cfg.n;
  LUB_TRY(ensure_gmres(h));
  double* v = h->V;
  double* w = h->V + n;
  double* part = h->hdot;
  double* hd = h->hdot + 128 * (h->gm + 2);
  const double one = 1.0;
  LUB_TRY(launch_gen_uniform(v, n, 1, 1, 20240601ULL, 7, s));
  LUB_TRY(launch_multi_dot(v, 1, v, n, part, hd, s));
  LUB_TRY(launch_scale_copy(v, v, n, hd, s));
  double nrm = 0.0;
  for (int i = 0; i < iters; i++) {
    LUB_TRY(launch_residual_f64(dA, lda, n, v, h->zero64, h->z64, h->racc, s));  // z = -A v
    LUB_TRY(prec_vec(h, h->perm32, h->z64, w, s));                              // w = -M^{-1} A v
    LUB_CUDA(cudaMemcpyAsync(hd + 1, &one, sizeof(double), cudaMemcpyHostToDevice, s));
    LUB_TRY(launch_multi_axpy(w, v, 1, hd + 1, n, 1.0, s));                      // w = v - M^{-1} A v
    LUB_TRY(launch_multi_dot(w, 1, w, n, part, hd, s));
    double sq = 0.0;
    LUB_CUDA(cudaMemcpyAsync(&sq, hd, sizeof(double), cudaMemcpyDeviceToHost, s));
    LUB_CUDA(cudaStreamSynchronize(s));
    nrm = std::sqrt(sq);
    if (!(nrm > 0.0) || !std::isfinite(nrm)) break;
    LUB_TRY(launch_scale_copy(w, v, n, hd, s));
  }
  *est = nrm;
  const int st = device_status(h, s);
  return st < 0 ? st : LU_OK;
}

extern "C" int lu_refine_solve(lu_handle h, const double* dA, int64_t lda, const double* db, double* dx,
                               lu_refine_info* info, void* stream) {
  if (!h || !dA || !db || !dx || lda < h->cfg.n) return LU_ERR_ARG;
  if (h->cfg.precision == LU_PREC_FP64) return LU_ERR_UNSUPPORTED;
  if (h->cfg.block_size % 64) return LU_ERR_ARG;  // whole 64-wide BF16 k-blocks per panel
  LUB_TRY(ensure_kernels_init());
  return refine_solve(h, ASrc{dA, lda, false}, db, dx, info, (cudaStream_t)stream);
}

extern "C" int lu_refine_solve_host(lu_handle h, const double* hA, int64_t lda, const double* db, double* dx,
                                    lu_refine_info* info, void* stream) {
  if (!h || !hA || !db || !dx || lda < h->cfg.n) return LU_ERR_ARG;
  if (h->cfg.precision == LU_PREC_FP64 || h->cfg.precision == LU_PREC_FP32) return LU_ERR_UNSUPPORTED;
  if (h->cfg.block_size % 64) return LU_ERR_ARG;
  cudaPointerAttributes pa;
  if (cudaPointerGetAttributes(&pa, hA) != cudaSuccess) {
    cudaGetLastError();
    return LU_ERR_ARG;
  }
  if (pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged) return LU_ERR_ARG;  // lu_refine_solve
  LUB_TRY(ensure_kernels_init());
  return refine_solve(h, ASrc{hA, lda, true}, db, dx, info, (cudaStream_t)stream);
}
