// Host orchestration and C ABI (include/lu_b200.h).
//
// The reference drives the factorisation with Charm++ SDAG control flow per
// block chare (lu.ci:31-370) and a per-PE BlockScheduler (scheduler.C).  On
// one GPU that control collapses into a host loop over panel steps that
// enqueues kernels on a stream:
//   panel k     recursive getrf2: leaf getf2 kernels + laswp/TRSM/GEMM halves
//   laswp       the panel's pivots applied to every other column, to b and to
//               the row permutation (pivotBatch/applyTrailingPivots,
//               lu.ci:92-123, lu.C:46-169)
//   TRSM        U block row (factorAboveDiagBlock -> computeU, lu.ci:132-174)
//   GEMM        one trailing update for the whole step (updateMatrix)
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "handle.h"

namespace lub {

// ---------------------------------------------------------------------------
// tensor maps
// ---------------------------------------------------------------------------
typedef CUresult (*PFN_encodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static PFN_encodeTiled get_encode() {
  static PFN_encodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_encodeTiled>(p);
  });
  return fn;
}

int encode_tmap_2d(CUtensorMap* map, CUtensorMapDataType dtype, int elem_bytes, const void* base, uint64_t cols,
                   uint64_t rows, uint64_t row_pitch_bytes, uint32_t box_cols, uint32_t box_rows,
                   CUtensorMapSwizzle swizzle) {
  PFN_encodeTiled enc = get_encode();
  if (!enc) return LU_ERR_CUDA;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (row_pitch_bytes & 15)) return LU_ERR_ALIGN;
  cuuint64_t gdim[2] = {cols, rows};
  cuuint64_t gstride[1] = {row_pitch_bytes};
  cuuint32_t box[2] = {box_cols, box_rows};
  cuuint32_t estride[2] = {1, 1};
  (void)elem_bytes;
  CUresult r = enc(map, dtype, 2, const_cast<void*>(base), gdim, gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    fprintf(stderr, "[lu_b200] cuTensorMapEncodeTiled failed (%d)\n", (int)r);
    return LU_ERR_CUDA;
  }
  return LU_OK;
}

long long g_kernel_launches = 0;

static PerDeviceOnce g_init;
int ensure_kernels_init() {
  return once_per_device(g_init, [] {
    int s = gemm_f64_init();
    if (s == LU_OK) s = gemm_bf16_init();
    if (s == LU_OK) s = leaf_init<double>();
    if (s == LU_OK) s = leaf_init<float>();
    if (s == LU_OK) s = tslu_init();
    return s;
  });
}

}  // namespace lub

using namespace lub;

namespace {

// even split of a column block, multiple of 16 when wide enough
inline int split_w(int w) {
  int h = w / 2;
  int w1 = h >= 16 ? (h & ~15) : (h & ~1);
  return std::max(w1, 2);
}

struct Ctx64 {
  lu_handle h;
  MatF64 A;
  int32_t* ipiv;
  int n;
  cudaStream_t s;
  double thr;
  PivotList pl;
  int leaf_w;
  int leaf_ctas;
  int base = 0;  // global row/column of the matrix's first row (a panel view)
};

int pivots_apply_f64(Ctx64& c, int k0, int cnt, int c_begin, int c_end, int skip_b, int skip_e, double* rhs,
                     int32_t* perm) {
  Prof pf(c.h, c.s, LU_PH_LASWP);
  for (int off = 0; off < cnt; off += 512) {
    const int sub = std::min(512, cnt - off);
    LUB_TRY(launch_pivot_compose(c.ipiv, k0 + off, sub, c.pl, c.s));
    LUB_TRY(launch_pivot_apply<double>(c.A.p, c.A.ld, c_begin, c_end, skip_b, skip_e, c.pl, 2 * sub, rhs, perm, c.s));
  }
  return LU_OK;
}

// C(rc, cc) [M x N] -= A(ra, ca) [M x K] * B(rb, cb) [K x N]
int gemm64(Ctx64& c, const MatF64& Cm, int rc, int cc, const MatF64& Am, int ra, int ca, const MatF64& Bm, int rb,
           int cb, int M, int N, int K, int phase = LU_PH_GEMM_IN) {
  Prof pf(c.h, c.s, phase, 2.0 * M * (double)N * K);
  GemmArgs g;
  g.a_row0 = ra; g.a_col0 = ca; g.b_row0 = rb; g.b_col0 = cb;
  g.C = Cm.at(rc, cc); g.ldc = Cm.ld;
  g.M = M; g.N = N; g.K = K;
  g.st = c.h->st; g.spin = c.h->spin;
  return launch_gemm_f64_sub(Am.mapA, Bm.mapB, g, c.s);
}

// B(r0.., cb..) [w x ncols] <- L^{-1} B, L = unit lower of Lm at (r0, r0)
int trsm64(Ctx64& c, const MatF64& Lm, int r0, int w, const MatF64& Bm, int rb, int cb, int ncols) {
  if (w <= 32) {
    Prof pf(c.h, c.s, LU_PH_TRSM, (double)w * w * ncols);
    return launch_trsm_llu_leaf<double>(Lm.at(r0, r0), Lm.ld, Bm.at(rb, cb), Bm.ld, w, ncols, c.s);
  }
  const int w1 = split_w(w);
  LUB_TRY(trsm64(c, Lm, r0, w1, Bm, rb, cb, ncols));
  LUB_TRY(gemm64(c, Bm, rb + w1, cb, Lm, r0 + w1, r0, Bm, rb, cb, w - w1, ncols, w1));
  return trsm64(c, Lm, r0 + w1, w - w1, Bm, rb + w1, cb, ncols);
}

// recursive panel factorisation of columns [c0, c0+w), rows [c0, n), inside
// the panel [p0, p0+pw): the leaves apply their row swaps to all of the
// panel's columns, so the recursion needs no separate laswp
int panel64(Ctx64& c, int c0, int w, int p0, int pw) {
  const int M = c.n - c0;
  if (w <= c.leaf_w) {
    unsigned* bar = c.h->take_counter();
    if (!bar) return LU_ERR_NOMEM;
    Prof pf(c.h, c.s, LU_PH_PANEL, (double)M * w * w);
    return launch_getf2_leaf<double>(c.A.at(c0, c0), c.A.ld, M, w, c.ipiv + c0, c.base + c0, c.h->leaf64, bar,
                                     c.h->st, c.base + c0, c.thr, c.h->spin, c.leaf_ctas, c.s, c.A.at(c0, p0), pw,
                                     c0 - p0);
  }
  const int w1 = split_w(w), w2 = w - w1;
  LUB_TRY(panel64(c, c0, w1, p0, pw));
  LUB_TRY(trsm64(c, c.A, c0, w1, c.A, c0, c0 + w1, w2));
  LUB_TRY(gemm64(c, c.A, c0 + w1, c0 + w1, c.A, c0 + w1, c0, c.A, c0, c0 + w1, M - w1, w2, w1));
  return panel64(c, c0 + w1, w2, p0, pw);
}

int check_common(lu_handle h, const void* dA, int64_t lda) {
  if (!h || !dA) return LU_ERR_ARG;
  if (lda < h->cfg.n) return LU_ERR_ARG;
  if ((lda & 1) || (reinterpret_cast<uintptr_t>(dA) & 15)) return LU_ERR_ALIGN;
  return ensure_kernels_init();
}

int factor_f64_schedule(lu_handle h, double* dA, int64_t lda, int32_t* ipiv, double* rhs, cudaStream_t s);

int factor_f64(lu_handle h, double* dA, int64_t lda, int32_t* ipiv, double* rhs, cudaStream_t s) {
  LUB_TRY(check_common(h, dA, lda));
  if (!ipiv) return LU_ERR_ARG;
  return run_graph(h, 0, dA, ipiv, rhs, lda, s,
                   [&](cudaStream_t ss) { return factor_f64_schedule(h, dA, lda, ipiv, rhs, ss); });
}

int factor_f64_schedule(lu_handle h, double* dA, int64_t lda, int32_t* ipiv, double* rhs, cudaStream_t s) {
  const int n = (int)h->cfg.n, b = h->cfg.block_size;
  const bool la = h->cfg.lookahead != 0;
  Ctx64 c;
  c.h = h; c.ipiv = ipiv; c.n = n; c.s = s; c.thr = h->cfg.sing_threshold; c.pl = h->plist;
  c.leaf_w = la ? h->leaf_w64_la : h->leaf_w64;
  c.leaf_ctas = la ? h->leaf_ctas_la : h->leaf_ctas;
  LUB_TRY(c.A.init(dA, n, n, lda));
  LUB_CUDA(cudaMemsetAsync(h->st, 0, sizeof(DevStatus), s));
  LUB_CUDA(cudaMemsetAsync(h->counters, 0, sizeof(unsigned) * h->n_counters, s));
  h->next_counter = 0;
  LUB_TRY(launch_iota(h->perm, n, s));
  if (!la) {
    for (int k0 = 0; k0 < n; k0 += b) {
      const int kw = std::min(b, n - k0);
      LUB_TRY(panel64(c, k0, kw, k0, kw));
      LUB_TRY(pivots_apply_f64(c, k0, kw, 0, n, k0, k0 + kw, rhs, h->perm));
      const int rest = n - k0 - kw;
      if (rest > 0) {
        LUB_TRY(trsm64(c, c.A, k0, kw, c.A, k0, k0 + kw, rest));
        LUB_TRY(gemm64(c, c.A, k0 + kw, k0 + kw, c.A, k0 + kw, k0, c.A, k0, k0 + kw, rest, rest, kw, LU_PH_GEMM));
      }
    }
    return LU_OK;
  }
  // Look-ahead (replaces BlockScheduler's policy, scheduler.C:235-484, and the
  // eager U solve next to the diagonal, lu.ci:141-145): panel k+1 runs on the
  // high-priority panel stream as soon as the trailing update has reached its
  // columns, while the rest of trailing update k runs on the caller's stream.
  Ctx64 cp = c;
  cp.s = h->sP;
  cp.pl = h->plistP;
  // under capture the panel stream's kernel nodes are marked for its priority
  std::vector<cudaGraphNode_t> mark;
  LUB_CUDA(cudaEventRecord(h->evFork, s));
  LUB_CUDA(cudaStreamWaitEvent(h->sP, h->evFork, 0));
  if (h->capturing) LUB_TRY(capture_deps(h->sP, &mark));
  LUB_TRY(panel64(cp, 0, std::min(b, n), 0, std::min(b, n)));
  if (h->capturing) LUB_TRY(mark_branch_priority(h, h->sP, mark));
  LUB_CUDA(cudaEventRecord(h->evP, h->sP));
  for (int k0 = 0; k0 < n; k0 += b) {
    const int kw = std::min(b, n - k0), k1 = k0 + kw, rest = n - k1;
    LUB_CUDA(cudaStreamWaitEvent(s, h->evP, 0));  // panel k factored (joins the panel stream)
    LUB_TRY(pivots_apply_f64(c, k0, kw, 0, n, k0, k1, rhs, h->perm));
    if (rest <= 0) continue;
    LUB_TRY(trsm64(c, c.A, k0, kw, c.A, k0, k1, rest));
    const int nw = std::min(b, rest);
    LUB_TRY(gemm64(c, c.A, k1, k1, c.A, k1, k0, c.A, k0, k1, rest, nw, kw, LU_PH_GEMM));  // next panel's columns
    LUB_CUDA(cudaEventRecord(h->evN, s));
    LUB_CUDA(cudaStreamWaitEvent(h->sP, h->evN, 0));
    if (h->capturing) LUB_TRY(capture_deps(h->sP, &mark));
    LUB_TRY(panel64(cp, k1, nw, k1, nw));
    if (h->capturing) LUB_TRY(mark_branch_priority(h, h->sP, mark));
    LUB_CUDA(cudaEventRecord(h->evP, h->sP));
    if (rest > nw)
      LUB_TRY(gemm64(c, c.A, k1, k1 + nw, c.A, k1, k0, c.A, k0, k1 + nw, rest, rest - nw, kw, LU_PH_GEMM));
  }
  return LU_OK;
}

// x <- U^{-1} L^{-1} x (x already permuted)
int solve_permuted_f64(lu_handle h, const double* LU, int64_t lda, double* x, cudaStream_t s) {
  const int n = (int)h->cfg.n;
  Prof pf(h, s, LU_PH_SOLVE, 2.0 * n * (double)n);
  LUB_TRY(launch_trsv<double>(LU, lda, n, x, 0, h->trsv_flags, h->trsv_ticket, h->st, h->spin, s));
  LUB_TRY(launch_trsv<double>(LU, lda, n, x, 1, h->trsv_flags, h->trsv_ticket, h->st, h->spin, s));
  return LU_OK;
}

}  // namespace

extern "C" {

int lu_config_default(lu_config* cfg, int64_t n, int32_t block_size) {
  if (!cfg) return LU_ERR_ARG;
  memset(cfg, 0, sizeof(*cfg));
  cfg->n = n;
  cfg->block_size = block_size;
  cfg->pivot_batch = std::max(1, block_size / 4);
  cfg->precision = LU_PREC_FP64;
  cfg->lookahead = 0;
  cfg->use_graph = 0;
  cfg->ir_mode = LU_IR_CLASSIC;
  cfg->ir_max_iter = 50;
  cfg->sing_threshold = 0.0;
  cfg->ir_target = 16.0;
  cfg->spin_limit = 0;
  return LU_OK;
}

size_t lu_workspace_bytes(const lu_config* cfg) {
  if (!cfg) return 0;
  const size_t n = (size_t)cfg->n;
  size_t b = 0;
  b += sizeof(DevStatus);
  b += sizeof(unsigned) * (n / 2 + 1024);
  b += 2 * kMaxLeafCTAs * (sizeof(double) + sizeof(int)) + 2 * kMaxLeafCTAs * kMaxLeafW * sizeof(double) +
       2 * kMaxLeafW * sizeof(double);
  b += 2 * kMaxLeafCTAs * (sizeof(float) + sizeof(int)) + 2 * kMaxLeafCTAs * kMaxLeafW * sizeof(float) +
       2 * kMaxLeafW * sizeof(float);
  b += 2 * sizeof(int32_t) * (4 * kMaxBatch + 1);
  b += sizeof(int32_t) * 2 * n;
  b += sizeof(int) * (n / 64 + 2) + sizeof(unsigned);
  b += sizeof(double) * 2 * n;
  b += sizeof(ResidualAccum);
  return b;
}

int lu_create(const lu_config* cfg, lu_handle* out) {
  if (!cfg || !out) return LU_ERR_ARG;
  if (cfg->n <= 0 || cfg->n > (int64_t)1 << 30 || cfg->block_size < 2 || (cfg->block_size & 1)) return LU_ERR_ARG;
  if (cfg->precision < LU_PREC_FP64 || cfg->precision > LU_PREC_FP16X3) return LU_ERR_ARG;
  if (cfg->layout != LU_LAYOUT_ROW && cfg->layout != LU_LAYOUT_COL) return LU_ERR_ARG;
  if (cfg->layout == LU_LAYOUT_COL && cfg->precision != LU_PREC_FP64) return LU_ERR_UNSUPPORTED;
  if (cfg->gmres_restart < 0 || cfg->gmres_restart > 1000 || cfg->ir_stall < 0 || !(cfg->gmres_tol >= 0.0) ||
      !(cfg->gmres_tol < 1.0))
    return LU_ERR_ARG;
  LUB_TRY(ensure_kernels_init());
  lu_handle h = new lu_handle_s();
  h->cfg = *cfg;
  cudaGetDevice(&h->device);
  cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device);
  h->spin = cfg->spin_limit > 0 ? cfg->spin_limit : (1LL << 24);
  const int64_t n = cfg->n;
  int s = LU_OK;
  // one per leaf launch (leaves are >= 2 columns wide) and one per shared
  // trailing-update tile counter (panels are >= 64 columns wide)
  h->n_counters = (int)(n / 2 + n / 64 + 1024);
  if (s == LU_OK) s = h->alloc(&h->st, 1);
  if (s == LU_OK) s = h->alloc(&h->counters, h->n_counters);
  if (s == LU_OK) s = h->alloc(&h->leaf64.cand_val, 2 * kMaxLeafCTAs);
  if (s == LU_OK) s = h->alloc(&h->leaf64.cand_row, 2 * kMaxLeafCTAs);
  if (s == LU_OK) s = h->alloc(&h->leaf64.cand_data, 2 * kMaxLeafCTAs * kMaxLeafW);
  if (s == LU_OK) s = h->alloc(&h->leaf64.rowj, 2 * kMaxLeafW);
  if (s == LU_OK) s = h->alloc(&h->leaf32.cand_val, 2 * kMaxLeafCTAs);
  if (s == LU_OK) s = h->alloc(&h->leaf32.cand_row, 2 * kMaxLeafCTAs);
  if (s == LU_OK) s = h->alloc(&h->leaf32.cand_data, 2 * kMaxLeafCTAs * kMaxLeafW);
  if (s == LU_OK) s = h->alloc(&h->leaf32.rowj, 2 * kMaxLeafW);
  if (s == LU_OK) s = h->alloc(&h->plist.dst, 2 * kMaxBatch);
  if (s == LU_OK) s = h->alloc(&h->plist.src, 2 * kMaxBatch);
  if (s == LU_OK) s = h->alloc(&h->plist.m, 1);
  if (s == LU_OK) s = h->alloc(&h->plistP.dst, 2 * kMaxBatch);
  if (s == LU_OK) s = h->alloc(&h->plistP.src, 2 * kMaxBatch);
  if (s == LU_OK) s = h->alloc(&h->plistP.m, 1);
  if (s == LU_OK) {
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    h->prio_hi = hi;
    if (cudaStreamCreateWithPriority(&h->sP, cudaStreamNonBlocking, hi) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->evFork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->evP, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->evN, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->evR, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->sG, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->evG0, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->evG1, cudaEventDisableTiming) != cudaSuccess)
      s = LU_ERR_CUDA;
  }
  h->leaf_ctas = h->num_sms;
  h->gemm_ctas = h->num_sms;
  if (const char* e = getenv("LU_B200_LEAF_CTAS")) h->leaf_ctas = std::max(1, atoi(e));
  if (const char* e = getenv("LU_B200_LEAF_CTAS_LA")) h->leaf_ctas_la = std::max(1, atoi(e));
  if (const char* e = getenv("LU_B200_LEAF_W64")) h->leaf_w64 = std::min(32, std::max(2, atoi(e)));
  if (const char* e = getenv("LU_B200_LEAF_W64_LA")) h->leaf_w64_la = std::min(32, std::max(2, atoi(e)));
  if (const char* e = getenv("LU_B200_LEAF_W32")) h->leaf_w32 = std::min(64, std::max(4, atoi(e)));
  if (const char* e = getenv("LU_B200_LEAF_W32_LA")) h->leaf_w32_la = std::min(64, std::max(4, atoi(e)));
  if (const char* e = getenv("LU_B200_GEMM_CTAS")) h->gemm_ctas = std::max(0, atoi(e));
  if (const char* e = getenv("LU_B200_GEMM_RESERVE")) h->gemm_reserve = std::max(0, atoi(e));
  if (const char* e = getenv("LU_B200_GEMM_HELPER")) h->gemm_helper = atoi(e) != 0;
  if (const char* e = getenv("LU_B200_GEMM_PAIR")) h->gemm_pair = atoi(e) != 0;
  if (const char* e = getenv("LU_B200_PANEL_TC")) h->panel_tc = atoi(e) != 0;
  if (const char* e = getenv("LU_B200_LA_SPLIT")) h->la_split = atoi(e) != 0;
  if (const char* e = getenv("LU_B200_TSLU")) h->tslu = atoi(e) != 0;
  if (const char* e = getenv("LU_B200_TRSM_BLOCK")) h->trsm_block = std::max(0, std::min(2, atoi(e)));
  if (const char* e = getenv("LU_B200_TRSM_WIDE")) h->trsm_wide = atoi(e) != 0;
  if (const char* e = getenv("LU_B200_TRSM_WIDE_MIN")) h->trsm_wide_min = std::max(0, atoi(e));
  if (const char* e = getenv("LU_B200_STAGE_BYTES")) h->stage_bytes = std::max<size_t>(1 << 16, strtoull(e, nullptr, 10));
  if (const char* e = getenv("LU_B200_RESIDENT_BYTES")) h->resident_cap = strtoull(e, nullptr, 10);
  if (s == LU_OK) s = h->alloc(&h->perm, n);
  if (s == LU_OK) s = h->alloc(&h->perm_work, n);
  if (s == LU_OK) s = h->alloc(&h->perm_lists, lub::ipiv_to_perm_work_ints((int)n));
  if (s == LU_OK) s = h->alloc(&h->trsv_flags, n / 64 + 2);
  if (s == LU_OK) s = h->alloc(&h->trsv_ticket, 1);
  if (s == LU_OK) s = h->alloc(&h->vec, n);
  if (s == LU_OK) s = h->alloc(&h->vec2, n);
  if (s == LU_OK) s = h->alloc(&h->racc, 1);
  if (s == LU_OK && cudaMallocHost(&h->racc_host, sizeof(ResidualAccum)) != cudaSuccess) s = LU_ERR_NOMEM;
  if (s == LU_OK && cudaMemset(h->st, 0, sizeof(DevStatus)) != cudaSuccess) s = LU_ERR_CUDA;
  if (s != LU_OK) {
    lu_destroy(h);
    return s;
  }
  *out = h;
  return LU_OK;
}

int lu_destroy(lu_handle h) {
  if (!h) return LU_ERR_ARG;
  for (cudaEvent_t e : h->pool) cudaEventDestroy(e);
  if (h->evFork) cudaEventDestroy(h->evFork);
  if (h->evP) cudaEventDestroy(h->evP);
  if (h->evN) cudaEventDestroy(h->evN);
  if (h->evR) cudaEventDestroy(h->evR);
  if (h->sP) cudaStreamDestroy(h->sP);
  for (auto& g : h->gslot)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  if (h->evG0) cudaEventDestroy(h->evG0);
  if (h->evG1) cudaEventDestroy(h->evG1);
  if (h->sG) cudaStreamDestroy(h->sG);
  for (int b = 0; b < 2; b++) {
    if (h->evReady[b]) cudaEventDestroy(h->evReady[b]);
    if (h->evFree[b]) cudaEventDestroy(h->evFree[b]);
  }
  if (h->sCopy) cudaStreamDestroy(h->sCopy);
  for (void* p : h->allocs) cudaFree(p);
  if (h->racc_host) cudaFreeHost(h->racc_host);
  delete h;
  return LU_OK;
}

int lu_status(lu_handle h, void* stream) {
  if (!h) return LU_ERR_ARG;
  LUB_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  DevStatus st;
  LUB_CUDA(cudaMemcpy(&st, h->st, sizeof(st), cudaMemcpyDeviceToHost));
  if (st.code != 0) return st.code;
  return st.info;
}

int lu_status_clear(lu_handle h, void* stream) {
  if (!h) return LU_ERR_ARG;
  LUB_CUDA(cudaMemsetAsync(h->st, 0, sizeof(DevStatus), (cudaStream_t)stream));
  return LU_OK;
}

int lu_factor(lu_handle h, double* dA, int64_t lda, int32_t* ipiv, double* rhs, void* stream) {
  if (!h) return LU_ERR_ARG;
  if (h->cfg.precision != LU_PREC_FP64) return LU_ERR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  if (h->cfg.layout != LU_LAYOUT_COL) return factor_f64(h, dA, lda, ipiv, rhs, s);
  // every argument is checked before the first transpose, and a failure
  // after it transposes back, so an error leaves the caller's matrix as given
  LUB_TRY(check_common(h, dA, lda));
  if (!ipiv) return LU_ERR_ARG;
  const int n = (int)h->cfg.n;
  LUB_TRY(launch_transpose_inplace(dA, lda, n, s));
  const int rc = factor_f64(h, dA, lda, ipiv, rhs, s);
  const int rc2 = launch_transpose_inplace(dA, lda, n, s);
  return rc != LU_OK ? rc : rc2;
}

int lu_transpose_square(double* dA, int64_t n, int64_t lda, void* stream) {
  if (!dA || n < 0 || lda < n || n > ((int64_t)1 << 31) - 1) return LU_ERR_ARG;
  return launch_transpose_inplace(dA, lda, (int)n, (cudaStream_t)stream);
}

// n x nrhs staging block owned by the handle
static int ensure_tmpB(lu_handle h, size_t elems) {
  if (h->tmpB_elems >= elems) return LU_OK;
  if (h->tmpB) {
    cudaFree(h->tmpB);
    h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void*)h->tmpB), h->allocs.end());
    h->tmpB = nullptr;
  }
  LUB_TRY(h->alloc(&h->tmpB, elems));
  h->tmpB_elems = elems;
  return LU_OK;
}

// A^T Y = B with P A = L U  ->  U^T L^T (P Y) = B: solve U^T, then L^T on a
// copy of B, then Y = P^T (that): rows scattered through the permutation.
static int solve_trans_multi(lu_handle h, const double* dLU, int64_t lda, const double* B, int64_t ldb, int nrhs,
                             double* Y, int64_t ldy, cudaStream_t s) {
  const int n = (int)h->cfg.n;
  LUB_TRY(ensure_tmpB(h, (size_t)n * nrhs));
  LUB_CUDA(cudaMemcpy2DAsync(h->tmpB, sizeof(double) * nrhs, B, sizeof(double) * ldb, sizeof(double) * nrhs, n,
                             cudaMemcpyDeviceToDevice, s));
  Prof pf(h, s, LU_PH_SOLVE, 2.0 * n * (double)n * nrhs);
  LUB_TRY(launch_trsm_pipe(dLU, lda, n, h->tmpB, nrhs, nrhs, 2, h->trsv_flags, h->trsv_ticket, h->st, h->spin, s));
  LUB_TRY(launch_trsm_pipe(dLU, lda, n, h->tmpB, nrhs, nrhs, 3, h->trsv_flags, h->trsv_ticket, h->st, h->spin, s));
  return launch_permute_rows(h->tmpB, nrhs, Y, ldy, h->perm_work, n, nrhs, 1, s);
}

int lu_solve(lu_handle h, const double* dLU, int64_t lda, const int32_t* ipiv, double* dB, int64_t ldb,
             int64_t nrhs, int trans, void* stream) {
  LUB_TRY(check_common(h, dLU, lda));
  if (h->cfg.layout == LU_LAYOUT_COL) return LU_ERR_UNSUPPORTED;
  if (!ipiv || !dB || nrhs < 1 || ldb < nrhs || (trans != 0 && trans != 1)) return LU_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int n = (int)h->cfg.n;
  LUB_TRY(launch_ipiv_to_perm(ipiv, n, h->perm_work, h->perm_lists, s));
  if (trans == 0 && nrhs == 1) {
    LUB_TRY(launch_gather_perm(dB, h->perm_work, h->vec, n, s));
    LUB_TRY(solve_permuted_f64(h, dLU, lda, h->vec, s));
    LUB_CUDA(cudaMemcpyAsync(dB, h->vec, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    return LU_OK;
  }
  if (trans == 1) return solve_trans_multi(h, dLU, lda, dB, ldb, (int)nrhs, dB, ldb, s);
  // A X = B, several right-hand sides: gather P B, then L, then U
  LUB_TRY(ensure_tmpB(h, (size_t)n * nrhs));
  LUB_TRY(launch_permute_rows(dB, ldb, h->tmpB, nrhs, h->perm_work, n, (int)nrhs, 0, s));
  {
    Prof pf(h, s, LU_PH_SOLVE, 2.0 * n * (double)n * nrhs);
    LUB_TRY(launch_trsm_pipe(dLU, lda, n, h->tmpB, nrhs, (int)nrhs, 0, h->trsv_flags, h->trsv_ticket, h->st,
                             h->spin, s));
    LUB_TRY(launch_trsm_pipe(dLU, lda, n, h->tmpB, nrhs, (int)nrhs, 1, h->trsv_flags, h->trsv_ticket, h->st,
                             h->spin, s));
  }
  LUB_CUDA(cudaMemcpy2DAsync(dB, sizeof(double) * ldb, h->tmpB, sizeof(double) * nrhs, sizeof(double) * nrhs, n,
                             cudaMemcpyDeviceToDevice, s));
  return LU_OK;
}

int lu_factor_solve(lu_handle h, double* dA, int64_t lda, int32_t* ipiv, double* db, void* stream) {
  if (!h || !db) return LU_ERR_ARG;
  if (h->cfg.precision != LU_PREC_FP64) return LU_ERR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  const bool col = h->cfg.layout == LU_LAYOUT_COL;
  if (!col) {
    LUB_TRY(factor_f64(h, dA, lda, ipiv, db, s));
    return solve_permuted_f64(h, dA, lda, db, s);
  }
  // as lu_factor: check first, transpose back on every path after the first transpose
  LUB_TRY(check_common(h, dA, lda));
  if (!ipiv) return LU_ERR_ARG;
  LUB_TRY(launch_transpose_inplace(dA, lda, (int)h->cfg.n, s));
  int rc = factor_f64(h, dA, lda, ipiv, db, s);
  if (rc == LU_OK) rc = solve_permuted_f64(h, dA, lda, db, s);
  const int rc2 = launch_transpose_inplace(dA, lda, (int)h->cfg.n, s);
  return rc != LU_OK ? rc : rc2;
}

int lu_residual(lu_handle h, const double* dA, int64_t lda, const double* dx, const double* db,
                lu_residual_info* out, void* stream) {
  if (!h || !dA || !dx || !db || !out || lda < h->cfg.n) return LU_ERR_ARG;
  if (h->cfg.layout == LU_LAYOUT_COL) return LU_ERR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  const int n = (int)h->cfg.n;
  LUB_TRY(launch_residual_f64(dA, lda, n, dx, db, nullptr, h->racc, s));
  LUB_CUDA(cudaMemcpyAsync(h->racc_host, h->racc, sizeof(ResidualAccum), cudaMemcpyDeviceToHost, s));
  LUB_CUDA(cudaStreamSynchronize(s));
  const ResidualAccum& a = *h->racc_host;
  auto d = [](unsigned long long v) {
    double x;
    memcpy(&x, &v, 8);
    return x;
  };
  const double eps = 2.220446049250313e-16, dn = (double)n;
  out->amax = d(a.amax);
  out->anorm = d(a.anorm);
  out->bnorm = d(a.bmax);
  out->xnorm = d(a.xmax);
  out->rnorm = d(a.rmax);
  out->r_ref = out->rnorm / ((out->amax * out->xnorm + out->bnorm) * dn * eps);
  out->r_hpl = out->rnorm / ((out->anorm * out->xnorm + out->bnorm) * dn * eps);
  return LU_OK;
}

// Adjoint of X = A^{-1} B for a loss with upstream gradient W = dL/dX:
// lambda = A^{-T} W (the transposed triangular solves on the stored
// factors), grad_B = lambda, grad_A = -lambda X^T (rank-nrhs product).
int lu_adjoint(lu_handle h, const double* dLU, int64_t lda, const int32_t* ipiv, const double* dX, int64_t ldx,
               const double* dW, int64_t ldw, int64_t nrhs, double* gradB, int64_t ldgb, double* gradA,
               int64_t ldga, void* stream) {
  LUB_TRY(check_common(h, dLU, lda));
  if (h->cfg.layout == LU_LAYOUT_COL) return LU_ERR_UNSUPPORTED;
  const int64_t n = h->cfg.n;
  if (!ipiv || !dW || !gradB || nrhs < 1 || ldw < nrhs || ldgb < nrhs) return LU_ERR_ARG;
  if (gradA && (!dX || ldx < nrhs || ldga < n)) return LU_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  LUB_TRY(launch_ipiv_to_perm(ipiv, (int)n, h->perm_work, h->perm_lists, s));
  LUB_TRY(solve_trans_multi(h, dLU, lda, dW, ldw, (int)nrhs, gradB, ldgb, s));
  if (gradA) {
    Prof pf(h, s, LU_PH_OTHER, 2.0 * n * (double)n * nrhs);
    LUB_TRY(launch_neg_outer(gradB, ldgb, dX, ldx, (int)n, (int)nrhs, gradA, ldga, s));
  }
  return LU_OK;
}

int lu_generate_uniform(double* d, int64_t rows, int64_t cols, int64_t ld, uint64_t seed, uint64_t stream_id,
                        void* stream) {
  if (!d || rows < 0 || cols < 0 || ld < cols) return LU_ERR_ARG;
  return launch_gen_uniform(d, rows, cols, ld, seed, stream_id, (cudaStream_t)stream);
}

int lu_matgen_host(double* out, int64_t count, int32_t seed, int64_t skip) {
  if (!out || count < 0 || skip < 0) return LU_ERR_ARG;
  const int32_t MAXI = 0x7fffffff, A = 48271, Q = MAXI / A, R = MAXI % A;
  int32_t cur = seed;
  for (int64_t i = 0; i < skip + count; i++) {
    cur = A * (cur % Q) - R * (cur / Q);
    if (cur < 0) cur += MAXI;
    if (i >= skip) out[i - skip] = (double)cur / MAXI - 0.5;
  }
  return LU_OK;
}

int lu_profile(lu_handle h, int enable) {
  if (!h) return LU_ERR_ARG;
  h->profile = enable ? 1 : 0;
  return LU_OK;
}

int lu_phase_times(lu_handle h, double* ms, int64_t* launches, double* flops) {
  if (!h) return LU_ERR_ARG;
  double t[LU_NUM_PHASES] = {0}, f[LU_NUM_PHASES] = {0};
  int64_t c[LU_NUM_PHASES] = {0};
  for (auto& r : h->recs) {
    LUB_CUDA(cudaEventSynchronize(r.b));
    float e = 0.f;
    LUB_CUDA(cudaEventElapsedTime(&e, r.a, r.b));
    t[r.phase] += e;
    f[r.phase] += r.flops;
    c[r.phase] += 1;
  }
  for (int i = 0; i < LU_NUM_PHASES; i++) {
    if (ms) ms[i] = t[i];
    if (launches) launches[i] = c[i];
    if (flops) flops[i] = f[i];
  }
  h->recs.clear();
  h->pool_used = 0;
  return LU_OK;
}

int64_t lu_launch_count(void) { return __atomic_load_n(&g_kernel_launches, __ATOMIC_RELAXED); }

const char* lu_status_string(int status) {
  if (status > 0) return "singular pivot (info = first failing column, 1-based)";
  switch (status) {
    case LU_OK: return "ok";
    case LU_ERR_ARG: return "bad argument";
    case LU_ERR_CUDA: return "CUDA error";
    case LU_ERR_TIMEOUT: return "device-side wait timed out";
    case LU_ERR_NONFINITE: return "non-finite value";
    case LU_ERR_NOCONV: return "iterative refinement did not converge";
    case LU_ERR_ALIGN: return "alignment requirement violated";
    case LU_ERR_NOMEM: return "out of device memory";
    case LU_ERR_UNSUPPORTED: return "unsupported configuration";
    default: return "unknown status";
  }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Per-block building blocks for callers that distribute the matrix
// themselves (the block-cyclic multi-GPU driver): the same recursion and
// kernels as lu_factor / lu_solve, on caller-supplied views.
// ---------------------------------------------------------------------------
namespace {

int check_view(const void* p, int64_t ld, int64_t cols) {
  if (!p || ld <= 0 || ld < cols) return LU_ERR_ARG;
  if ((ld & 1) || (reinterpret_cast<uintptr_t>(p) & 15)) return LU_ERR_ALIGN;
  return LU_OK;
}

Ctx64 block_ctx(lu_handle h, cudaStream_t s) {
  const bool la = h->cfg.lookahead != 0;
  Ctx64 c;
  c.h = h;
  c.ipiv = nullptr;
  c.n = 0;
  c.s = s;
  c.thr = h->cfg.sing_threshold;
  c.pl = h->plist;
  c.leaf_w = la ? h->leaf_w64_la : h->leaf_w64;
  c.leaf_ctas = la ? h->leaf_ctas_la : h->leaf_ctas;
  return c;
}

}  // namespace

extern "C" {

int lu_panel_factor(lu_handle h, double* dP, int64_t ldp, int64_t m, int32_t w, int32_t* d_ipiv, int64_t base,
                    void* stream) {
  if (!h || !d_ipiv || w < 1 || m < w || m > h->cfg.n || base < 0 || base + m > ((int64_t)1 << 31) - 1)
    return LU_ERR_ARG;
  LUB_TRY(check_view(dP, ldp, w));
  LUB_TRY(ensure_kernels_init());
  cudaStream_t s = (cudaStream_t)stream;
  Ctx64 c = block_ctx(h, s);
  c.ipiv = d_ipiv;
  c.n = (int)m;
  c.base = (int)base;
  LUB_TRY(c.A.init(dP, m, w, ldp));
  // one barrier counter per leaf, from a pool cleared for this panel
  LUB_CUDA(cudaMemsetAsync(h->counters, 0, sizeof(unsigned) * h->n_counters, s));
  h->next_counter = 0;
  return panel64(c, 0, w, 0, w);
}

int lu_apply_pivots(lu_handle h, double* dA, int64_t lda, int64_t m, int32_t ncols, const int32_t* d_ipiv,
                    int64_t k0, int32_t cnt, int32_t skip_b, int32_t skip_e, double* db, void* stream) {
  if (!h || !d_ipiv || ncols < 0 || cnt < 0 || k0 < 0 || m < 1 || m > ((int64_t)1 << 31) - 1 || k0 + cnt > m)
    return LU_ERR_ARG;
  if (ncols > 0) LUB_TRY(check_view(dA, lda, ncols));
  LUB_TRY(ensure_kernels_init());
  cudaStream_t s = (cudaStream_t)stream;
  Prof pf(h, s, LU_PH_LASWP);
  for (int off = 0; off < cnt; off += 512) {
    const int sub = std::min(512, cnt - off);
    LUB_TRY(launch_pivot_compose(d_ipiv, (int)k0 + off, sub, h->plist, s, (int)m, h->st));
    LUB_TRY(launch_pivot_apply<double>(dA, lda, 0, ncols, skip_b, skip_e, h->plist, 2 * sub, db, nullptr, s));
  }
  return LU_OK;
}

int lu_trsm_lower_unit(lu_handle h, const double* dL, int64_t ldl, int32_t w, double* dB, int64_t ldb, int64_t ncols,
                       void* stream) {
  if (!h || w < 1 || ncols < 0 || ncols > ((int64_t)1 << 31) - 1) return LU_ERR_ARG;
  if (ncols == 0) return LU_OK;
  LUB_TRY(check_view(dL, ldl, w));
  LUB_TRY(check_view(dB, ldb, ncols));
  LUB_TRY(ensure_kernels_init());
  Ctx64 c = block_ctx(h, (cudaStream_t)stream);
  MatF64 Lm, Bm;
  LUB_TRY(Lm.init(const_cast<double*>(dL), w, w, ldl));
  LUB_TRY(Bm.init(dB, w, ncols, ldb));
  return trsm64(c, Lm, 0, w, Bm, 0, 0, (int)ncols);
}

int lu_gemm_update(lu_handle h, const double* dA, int64_t lda, const double* dB, int64_t ldb, double* dC, int64_t ldc,
                   int64_t M, int64_t N, int64_t K, void* stream) {
  const int64_t lim = ((int64_t)1 << 31) - 1;
  if (!h || M < 0 || N < 0 || K < 0 || M > lim || N > lim || K > lim) return LU_ERR_ARG;
  if (M == 0 || N == 0 || K == 0) return LU_OK;
  LUB_TRY(check_view(dA, lda, K));
  LUB_TRY(check_view(dB, ldb, N));
  LUB_TRY(check_view(dC, ldc, N));
  LUB_TRY(ensure_kernels_init());
  Ctx64 c = block_ctx(h, (cudaStream_t)stream);
  MatF64 Am, Bm, Cm;
  LUB_TRY(Am.init(const_cast<double*>(dA), M, K, lda));
  LUB_TRY(Bm.init(const_cast<double*>(dB), K, N, ldb));
  Cm.p = dC;
  Cm.ld = ldc;
  Cm.rows = M;
  Cm.cols = N;
  return gemm64(c, Cm, 0, 0, Am, 0, 0, Bm, 0, 0, (int)M, (int)N, (int)K, LU_PH_GEMM);
}

int lu_trsv_block(lu_handle h, const double* dT, int64_t ldt, int32_t w, int32_t upper, double* dx, void* stream) {
  if (!h || !dx || w < 1 || w > h->cfg.n) return LU_ERR_ARG;
  LUB_TRY(check_view(dT, ldt, w));
  LUB_TRY(ensure_kernels_init());
  cudaStream_t s = (cudaStream_t)stream;
  Prof pf(h, s, LU_PH_SOLVE, (double)w * w);
  return launch_trsv<double>(dT, ldt, w, dx, upper ? 1 : 0, h->trsv_flags, h->trsv_ticket, h->st, h->spin, s);
}

int lu_copy_2d(void* dst, int64_t dpitch, const void* src, int64_t spitch, int64_t width, int64_t rows,
               void* stream) {
  if (!dst || !src || width < 0 || rows < 0 || dpitch < width || spitch < width) return LU_ERR_ARG;
  if (width == 0 || rows == 0) return LU_OK;
  LUB_CUDA(cudaMemcpy2DAsync(dst, (size_t)dpitch, src, (size_t)spitch, (size_t)width, (size_t)rows,
                             cudaMemcpyDefault, (cudaStream_t)stream));
  return LU_OK;
}

int lu_gemv_update(lu_handle h, const double* dA, int64_t lda, int64_t m, int32_t k, const double* dx, double* dy,
                   void* stream) {
  if (!h || !dx || !dy || m < 0 || k < 0 || m > ((int64_t)1 << 31) - 1) return LU_ERR_ARG;
  if (m == 0 || k == 0) return LU_OK;
  LUB_TRY(check_view(dA, lda, k));
  LUB_TRY(ensure_kernels_init());
  cudaStream_t s = (cudaStream_t)stream;
  Prof pf(h, s, LU_PH_SOLVE, 2.0 * (double)m * k);
  return launch_gemv_sub(dA, lda, (int)m, k, dx, dy, s);
}

}  // extern "C"
