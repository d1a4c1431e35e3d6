// Internal launcher declarations shared by the host orchestration.
#pragma once
#include "common.cuh"

namespace lub {

// ---- C -= A * B (row-major sub-blocks addressed through tensor maps)
struct GemmArgs {
  int a_row0, a_col0;  // origin of A in mapA's matrix
  int b_row0, b_col0;  // origin of B in mapB's matrix
  double* C;           // origin of C
  int64_t ldc;
  int M, N, K;
  DevStatus* st;
  long long spin;
};
int gemm_f64_init();
int gemm_f64_smem_bytes();
int launch_gemm_f64_sub(const CUtensorMap& mapA, const CUtensorMap& mapB, const GemmArgs& a, cudaStream_t s);

// FP32 SIMT GEMM C -= A * B (panel / TRSM halves of the mixed path)
int launch_gemm_f32_sub(const float* A, int64_t lda, const float* B, int64_t ldb, float* C, int64_t ldc, int M,
                        int N, int K, cudaStream_t s);

// ---- unblocked panel leaf (cooperative, rows resident in shared memory)
template <typename T>
struct LeafScratch {
  T* cand_val;     // [2][kMaxLeafCTAs]
  int* cand_row;   // [2][kMaxLeafCTAs]
  T* cand_data;    // [2][kMaxLeafCTAs][kMaxLeafW]
  T* rowj;         // [2][kMaxLeafW]
};
constexpr int kMaxLeafCTAs = 160;
constexpr int kMaxLeafW = 64;
template <typename T>
int leaf_init();
// Factor P[0:M, 0:ncols] (row-major, P = diagonal of the first column) with
// partial pivoting; ipiv[j] = row_base + local pivot row.  Each swap is also
// applied to the enclosing panel's other columns: prow0 points at the
// panel's first column in the leaf's top row, the panel is pw wide and the
// leaf starts lc0 columns in (prow0 = null: the leaf is the panel).
template <typename T>
int launch_getf2_leaf(T* P, int64_t lda, int M, int ncols, int32_t* ipiv, int row_base, const LeafScratch<T>& scr,
                      unsigned* bar, DevStatus* st, int info_base, double thr, long long spin, int max_ctas,
                      cudaStream_t s, T* prow0 = nullptr, int pw = 0, int lc0 = 0);

// ---- tournament-pivoting leaf of the FP32 panels (tslu.cu)
struct TsluScratch {
  int* cand_idx;      // [kMaxLeafCTAs][kMaxLeafW] rows each block nominates
  int* cand_cnt;      // [kMaxLeafCTAs]
  int* cand_idx2;     // the same, for the tournament's alternate rounds
  int* cand_cnt2;
  float* lu11;        // [kMaxLeafW][kMaxLeafW] factored top block
  unsigned* ok_mask;  // [1] bit j: pivot j usable (nonzero, not NaN)
  int* mv_dst;        // [2 * kMaxLeafW] row moves dst <- src
  int* mv_src;
  int* mv_cnt;        // [1]
  float* mv_data;     // [2 * kMaxLeafW][mv_pitch] moved rows' original values
  int mv_pitch;       // >= the widest enclosing panel
};
int tslu_init();
// ncols <= 32; LU_ERR_UNSUPPORTED when the shapes exceed its blocks
int launch_tslu_leaf(float* P, int64_t lda, int M, int ncols, int32_t* ipiv, int row_base, const TsluScratch& scr,
                     DevStatus* st, int info_base, double thr, int max_ctas, cudaStream_t s, float* prow0, int pw,
                     int lc0);

// ---- pivot batches: compose sequential swaps into (dst <- src) lists
// batch: swaps (k0+i) <-> ipiv[k0+i] for i in [0, cnt), cnt <= kMaxBatch
constexpr int kMaxBatch = 1024;
struct PivotList {
  int32_t* dst;  // [2*kMaxBatch]
  int32_t* src;  // [2*kMaxBatch]
  int32_t* m;    // [1]
};
// rows > 0 checks k0 + i <= ipiv[k0 + i] < rows first: a batch that fails
// moves nothing and records LU_ERR_ARG in st
int launch_pivot_compose(const int32_t* ipiv, int k0, int cnt, const PivotList& pl, cudaStream_t s, int rows = 0,
                         DevStatus* st = nullptr);
// Apply to columns [c_begin, c_end) minus [skip_begin, skip_end); optional
// vector (rhs) and int permutation carried with the rows.
template <typename T>
int launch_pivot_apply(T* A, int64_t lda, int c_begin, int c_end, int skip_begin, int skip_end, const PivotList& pl,
                       int max_m, double* rhs, int32_t* perm, cudaStream_t s);
// x <- P x in place from an ipiv vector (single CTA, shared memory only).
int launch_ipiv_apply_vector(const int32_t* ipiv, int n, double* x, cudaStream_t s);
// Full permutation from an ipiv vector (single CTA, batched composition).
// work: ipiv_to_perm_work_ints(n) ints
int ipiv_to_perm_work_ints(int n);
int launch_ipiv_to_perm(const int32_t* ipiv, int n, int32_t* perm, int32_t* work, cudaStream_t s);

// ---- triangular solves
// B(m x ncols) <- L^{-1} B, L unit lower m x m (m <= 32), row-major
template <typename T>
int launch_trsm_llu_leaf(const T* L, int64_t ldl, T* B, int64_t ldb, int m, int ncols, cudaStream_t s);
// FP32 B(w x ncols) <- L^{-1} B, L unit lower w x w, w <= 256, one launch
int launch_trsm_llu_block(const float* L, int64_t ldl, float* B, int64_t ldb, int w, int ncols, cudaStream_t s);
// B (w x ncols) <- L^{-1} B, L unit lower, w <= 512, FP32; dinv: 16 x 1024 floats of scratch
int launch_trsm_wide(const float* L, int64_t ldl, float* B, int64_t ldb, int w, int ncols, float* dinv,
                     cudaStream_t s);
// single/multi right-hand side substitution with flags (persistent tickets)
template <typename T>
int launch_trsv(const T* LU, int64_t lda, int n, T* x, int upper, int* flags, unsigned* ticket, DevStatus* st,
                long long spin, cudaStream_t s);

// multi-RHS pipelined triangular solve (mode 0 L, 1 U, 2 U^T, 3 L^T) on a
// row-major n x nrhs FP64 block; factors stored as TS (double or float)
template <typename TS>
int launch_trsm_pipe(const TS* LU, int64_t lda, int n, double* Y, int64_t ldy, int nrhs, int mode, int* flags,
                     unsigned* ticket, DevStatus* st, long long spin, cudaStream_t s);

// ---- multi-RHS refinement (up to 16 columns, ld 16 work blocks)
constexpr int kMultiMaxSplits = 16;  // reduction splits of the residual product
constexpr int kMultiAccWords = 64;   // |R|, |B|, |X| maxima per column, ||op(A)||inf
// number of splits S and their length for order n
int multi_residual_splits(int n, int num_sms, int* split_len);
// R = B - op(A) X (op = A^T when trans), per-column maxima into acc;
// P: S * n * 16 doubles, Pn: S * n doubles of partials
int launch_multi_residual(const double* A, int64_t lda, int n, int trans, const double* X, const double* B,
                          int64_t ldb, int nrhs, double* R, double* P, double* Pn, int S, int split_len, int norm,
                          unsigned long long* acc, cudaStream_t s);
// X[dst(i)] += D[i] (dst = perm[i] with scatter, else i), ld 16
int launch_multi_add(double* X, const double* D, const int32_t* perm, int n, int nrhs, int scatter, cudaStream_t s);
// single columns of ld-16 blocks: out[i] = M[perm ? perm[i] : i][c] * scale;
// dst[perm[i]] = src[i]; M[i][c] = v[i] (assign) or += v[i]
int launch_col_get(const double* M, int c, const int32_t* perm, double* out, int n, double scale, cudaStream_t s);
int launch_vec_scatter(const double* src, const int32_t* perm, double* dst, int n, cudaStream_t s);
int launch_col_put(double* M, int c, const double* v, int n, int assign, cudaStream_t s);
// D[:, c] = S[:, c] (ld-16 blocks)
int launch_col_copy(const double* S, double* D, int c, int n, cudaStream_t s);
// G = -Lam X^T (rank k <= 16)
int launch_neg_outer(const double* Lam, int64_t ldl, const double* X, int64_t ldx, int n, int k, double* G,
                     int64_t ldg, cudaStream_t s);
// row permutation of an n x k block: gather Y[i] = X[perm[i]] or scatter Y[perm[i]] = X[i]
int launch_permute_rows(const double* X, int64_t ldx, double* Y, int64_t ldy, const int32_t* perm, int n, int k,
                        int scatter, cudaStream_t s);

// ---- residual / GEMV / generators
struct ResidualAccum {  // non-negative doubles stored as ordered bit patterns
  unsigned long long amax, anorm, bmax, xmax, rmax;
};
int launch_residual_f64(const double* A, int64_t lda, int n, const double* x, const double* b, double* r,
                        ResidualAccum* acc, cudaStream_t s);
// A <- A^T in place (n x n, row pitch lda)
int launch_transpose_inplace(double* A, int64_t lda, int n, cudaStream_t s);
// y[0:m] -= A[0:m, 0:k] x (one warp per row)
int launch_gemv_sub(const double* A, int64_t lda, int m, int k, const double* x, double* y, cudaStream_t s);
// the same for rows row0 .. row0 + rows - 1 only (Arows = their first row);
// accumulates into acc without clearing it
int launch_residual_f64_rows(const double* Arows, int64_t lda, int rows, int row0, int n, const double* x,
                             const double* b, double* r, ResidualAccum* acc, cudaStream_t s);
// factors stored as TS, vector and arithmetic in T (FP32 factors, FP64 vector)
template <typename TS, typename T>
int launch_trsv_mixed(const TS* LU, int64_t lda, int n, T* x, int upper, int* flags, unsigned* ticket, DevStatus* st,
                      long long spin, cudaStream_t s);
// y[i] = v[perm[i]] * scale (scale = 1/||r||inf from acc when acc is given)
int launch_gather_f64(const double* v, const int32_t* perm, double* y, int n, double scale, const ResidualAccum* acc,
                      cudaStream_t s);

int launch_gen_uniform(double* d, int64_t rows, int64_t cols, int64_t ld, uint64_t seed, uint64_t stream_id,
                       cudaStream_t s);
int launch_gather_perm(const double* b, const int32_t* perm, double* y, int n, cudaStream_t s);
int launch_scatter_perm(const double* y, const int32_t* perm, double* b, int n, cudaStream_t s);
int launch_iota(int32_t* p, int n, cudaStream_t s);

// ---- mixed precision
int gemm_bf16_init();
int launch_gemm_bf16_tc(const CUtensorMap& mapA, const CUtensorMap& mapB, const CUtensorMap& mapC, int a_row0,
                        int b_row0, int c_row0, int c_col0, int M, int N, int K, bool bf16, const unsigned* amax,
                        DevStatus* st, long long spin, cudaStream_t s);
// persistent variant: max_ctas CTAs walk the tiles (TMEM double-buffered);
// kpart > 0: error-compensated pairs layout [hi | lo] per operand row, the
// three products Lh*Uh + Lh*Ul + Ll*Uh from one stage, K = kpart;
// tile_ctr: a zeroed counter shared by launches that split the tiles
int launch_gemm_lowp_persistent(const CUtensorMap& mapA, const CUtensorMap& mapB, const CUtensorMap& mapC,
                                int a_row0, int b_row0, int c_row0, int c_col0, int M, int N, int K, bool bf16,
                                const unsigned* amax, DevStatus* st, long long spin, int max_ctas, cudaStream_t s,
                                int kpart = 0, unsigned* tile_ctr = nullptr, bool cta_pair = false);
// |max| of the L21 (rows x K) and U12 (K x N) FP32 panels into amax[0], amax[1];
// lmax_from: take amax[0] from there instead of reading L (the same L21)
int launch_panel_absmax(const float* L, int64_t ldl, int rows, int K, const float* U, int64_t ldu, int N,
                        unsigned* amax, cudaStream_t s, const unsigned* lmax_from = nullptr);
// low-precision operand panels: nparts K-wide copies, part p is the hi
// (bit p of lo_mask clear) or lo (set) component of src * scale, scale the
// power of two of amax[which] (or 1 when amax is null); OUT bf16 or fp16
// (part_stride > 0: part p starts at p * part_stride, zero-filled past K;
// 0: parts are K wide and contiguous)
template <typename OUT>
int launch_split_rows(const float* src, int64_t lds, OUT* dst, int64_t ldd, int rows, int K, int nparts,
                      unsigned lo_mask, const unsigned* amax, int which, cudaStream_t s, int part_stride = 0);
template <typename OUT>
int launch_split_transpose(const float* src, int64_t lds, OUT* dst, int64_t ldd, int K, int N, int nparts,
                           unsigned lo_mask, const unsigned* amax, int which, cudaStream_t s, int part_stride = 0);
int launch_f64_to_f32(const double* src, int64_t lds, float* dst, int64_t ldd, int rows, int cols, cudaStream_t s);
int launch_ir_prep(const double* r64, const int32_t* perm, float* r32, int n, const ResidualAccum* acc,
                   cudaStream_t s);
int launch_ir_update(double* x, const float* d32, int n, const ResidualAccum* acc, cudaStream_t s);
int launch_gather_f64_to_f32(const double* v, const int32_t* perm, float* y, int n, double scale, cudaStream_t s);
int launch_f32_to_f64(const float* y, double* x, int n, double scale, cudaStream_t s);
// GMRES vector kernels (FP64, basis stored as consecutive length-n vectors)
int launch_multi_dot(const double* V, int k, const double* w, int n, double* part, double* out, cudaStream_t s);
int launch_multi_axpy(double* w, const double* V, int k, const double* h, int n, double sign, cudaStream_t s);
int launch_scale_copy(const double* src, double* dst, int n, const double* inv_of, cudaStream_t s);
// y = a * x
int launch_scale_vec(const double* x, double* y, int n, double a, cudaStream_t s);

}  // namespace lub
