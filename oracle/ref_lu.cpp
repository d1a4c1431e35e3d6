// ORACLE — test infrastructure only.
//
// A CPU restatement of charmlu's dense LU hot path (factor with partial
// pivoting, block forward/backward substitution, scaled-residual check).  It
// is the parity reference for the CUDA path in charmlu_b200 and the timed CPU baseline
// ("kind": "port").  Nothing in the product library links or calls it; only
// tests/, __graft_entry__.smoke() and bench.py (cpu_baseline / --impl
// reference) load it.
//
// Parity status: charmlu itself cannot be built here (it needs the Charm++
// runtime, charmc and CrnStream, which are not vendored, and cblas.h).  Its
// own test (test_lu.pl) pins only "residual < 16"; there are no golden
// vectors.  This restatement is therefore pinned (a) against LAPACK dgetrf
// (an independent implementation of the same partial-pivoting algorithm, via
// scipy) on pivots and factors, (b) against the reference's residual < 16
// contract on test_lu.pl's parameter sets, and (c) the reference generator
// MatGen against the published minimal-standard known answer (a=48271,
// seed 1, 10000th draw = 399268537).  Pivot/L/U parity with charmlu's own
// binary is unpinned.
//
// Storage follows the reference: the N x N matrix is row-major and
// logically split into b x b blocks (lu.h:151-153 getIndex(i,j) = i*b + j,
// applied per block; here the whole matrix is one row-major array with
// leading dimension lda and block (x, y) starts at A + x*b*lda + y*b).
//
// Algorithm order per step k (lu.ci:31-42, lu.ci:256-370, lu.ci:186-251):
//   panel column by column (lu.ci:267-349):
//     argmax |a| over rows >= j, strict '>' scanning rows upward, so the
//       lowest row wins ties (lu.C:197-205, lu.C:207-218; across blocks the
//       reference's order is message-arrival dependent, the oracle fixes
//       "lowest global row");
//     swap whole rows j <-> p, including the right-hand side b
//       (lu.C:166-177, lu.ci:302, lu.ci:305-323; other columns receive the
//       swap through pivot batches, lu.C:46-163, which is the same
//       permutation);
//     singularity check |u_jj| <= 100 eps (lu.ci:339-341), reported as a
//       status here instead of CkAbort;
//     multipliers by true division and the fused next-column update
//       (lu.C:259-288), rank-1 update of the remaining panel columns
//       (lu.C:230-254, offset 2);
//   U block row: dtrsm left/lower/unit per b x b block (lu.C:180-189);
//   trailing update: dgemm C -= L*U per b x b block (lu.C:26-43).
// Every rank-1 element update is computed as fma(-l, u, a): the reference's
// hand loop and dger leave the contraction to its compiler/BLAS; the oracle
// fixes one rounding per update so the CUDA panel can be compared bit for bit
// where its arithmetic order matches.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <vector>
#include <omp.h>

// ---- BLAS: the OpenBLAS bundled with scipy (LP64, symbols prefixed) ----
extern "C" {
enum { kRowMajor = 101, kNoTrans = 111, kLeft = 141, kLower = 122, kUpper = 121, kUnit = 132, kNonUnit = 131 };
void scipy_cblas_dgemm(int order, int ta, int tb, int m, int n, int k, double alpha,
                       const double* a, int lda, const double* b, int ldb, double beta,
                       double* c, int ldc);
void scipy_cblas_dtrsm(int order, int side, int uplo, int ta, int diag, int m, int n,
                       double alpha, const double* a, int lda, double* b, int ldb);
void scipy_openblas_set_num_threads(int n);
}

namespace {

// SplitMix64 finaliser (Steele, Lea, Flood 2014), used as a counter-based
// generator: value i of stream s under seed is mix(mix(seed ^ s*K2) + i*K1).
// The CUDA generator in charmlu_b200/csrc computes the identical function.
inline uint64_t mix64(uint64_t z) {
  z ^= z >> 30; z *= 0xbf58476d1ce4e5b9ULL;
  z ^= z >> 27; z *= 0x94d049bb133111ebULL;
  z ^= z >> 31; return z;
}
inline double uniform_at(uint64_t key, uint64_t i) {
  uint64_t z = mix64(key + (i + 1) * 0x9E3779B97F4A7C15ULL);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0) - 0.5;  // [-0.5, 0.5)
}
inline uint64_t stream_key(uint64_t seed, uint64_t stream) {
  return mix64(seed ^ (stream * 0xD1B54A32D192ED03ULL));
}

struct Blas {
  int mode;  // 0 = plain loops, 1 = OpenBLAS
};

// Pivot candidate: the reference's MaxElm (maxelm.h:7-12) plus the runner-up
// magnitude for near-tie detection.  offer() keeps the first row unless a
// later one is strictly larger (lu.C:200); merge() combines candidates taken
// from consecutive row ranges in increasing row order (MaxElm_max,
// lu.C:207-218, with the arrival order fixed to row order).
struct Cand {
  double best = 0.0, second = 0.0;
  int row = -1;
  void offer(double v, int r) {
    if (v > best) { second = best; best = v; row = r; }
    else if (v > second) second = v;
  }
  void merge(const Cand& o) {
    if (o.best > best) { second = std::max(best, o.second); best = o.best; row = o.row; }
    else second = std::max(second, o.best);
  }
};

// C(m x n) -= A(m x k) * B(k x n), row-major.  (lu.C:26-43)
void gemm_sub(const Blas& bl, int m, int n, int k, const double* A, int lda,
              const double* B, int ldb, double* C, int ldc) {
  if (m <= 0 || n <= 0 || k <= 0) return;
  if (bl.mode == 1) {
    scipy_cblas_dgemm(kRowMajor, kNoTrans, kNoTrans, m, n, k, -1.0, A, lda, B, ldb, 1.0, C, ldc);
    return;
  }
  for (int i = 0; i < m; i++)
    for (int p = 0; p < k; p++) {
      double a = A[(int64_t)i * lda + p];
      for (int j = 0; j < n; j++) C[(int64_t)i * ldc + j] = std::fma(-a, B[(int64_t)p * ldb + j], C[(int64_t)i * ldc + j]);
    }
}

// B(m x n) <- L^{-1} B with L unit lower m x m, row-major.  (lu.C:180-189)
void trsm_llu(const Blas& bl, int m, int n, const double* L, int ldl, double* B, int ldb) {
  if (m <= 0 || n <= 0) return;
  if (bl.mode == 1) {
    scipy_cblas_dtrsm(kRowMajor, kLeft, kLower, kNoTrans, kUnit, m, n, 1.0, L, ldl, B, ldb);
    return;
  }
  for (int i = 1; i < m; i++)
    for (int p = 0; p < i; p++) {
      double l = L[(int64_t)i * ldl + p];
      for (int j = 0; j < n; j++) B[(int64_t)i * ldb + j] = std::fma(-l, B[(int64_t)p * ldb + j], B[(int64_t)i * ldb + j]);
    }
}

}  // namespace

extern "C" {

// Counter-based uniform[-0.5, 0.5) values count starting at index offset.
void oracle_gen_uniform(double* out, int64_t count, uint64_t seed, uint64_t stream, int64_t offset) {
  uint64_t key = stream_key(seed, stream);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < count; i++) out[i] = uniform_at(key, (uint64_t)(offset + i));
}

// The reference's b-vector generator MatGen (benchmark.C:28-74): Park-Miller
// minimal standard with multiplier 48271, Schrage's decomposition, value
// rnd/MAXINT - 0.5; skip draws first (benchmark.C:455-460).
void oracle_matgen(double* out, int64_t count, int32_t seed, int64_t skip, int32_t* ints_out) {
  const int32_t MAXI = 0x7fffffff, A = 48271, Q = MAXI / A, R = MAXI % A;
  int32_t cur = seed;
  auto next = [&]() {
    cur = A * (cur % Q) - R * (cur / Q);
    if (cur < 0) cur += MAXI;
    return cur;
  };
  for (int64_t i = 0; i < skip; i++) next();
  for (int64_t i = 0; i < count; i++) {
    int32_t v = next();
    if (ints_out) ints_out[i] = v;
    if (out) out[i] = (double)v / MAXI - 0.5;
  }
}

void oracle_set_threads(int n) {
  if (n <= 0) n = omp_get_max_threads();
  omp_set_num_threads(n);
  scipy_openblas_set_num_threads(1);
}

// Blocked right-looking LU with partial pivoting, restating lu.ci/lu.C.
//   A      : n x n row-major, leading dimension lda (in/out, LU in place)
//   rhs    : optional length-n vector, permuted with the rows (lu.h:66)
//   ipiv   : length n, 0-based global pivot row per column (lu.ci:329)
//   margin : optional length n, relative gap between the largest and the
//            second largest |candidate| of each column (near-tie flag)
//   sing_threshold : |u_jj| <= threshold counts as singular (the reference
//            uses 100*eps, lu.ci:339); pass 0 for exact-zero (LAPACK) rule
// Returns 0, or 1 + the first column whose pivot failed the threshold.
// Processing continues after a singular column (no scaling of that column),
// as LAPACK does, so the factors stay defined.
int oracle_lu_factor(int n, int b, double* A, int64_t lda, int32_t* ipiv, double* rhs,
                     double* margin, int blas_mode, double sing_threshold) {
  if (n < 0 || b <= 0 || lda < n) return -1;
  Blas bl{blas_mode};
  int info = 0;
  const int nb = (n + b - 1) / b;
  std::vector<double> rowbuf(n);
  for (int k = 0; k < nb; k++) {
    const int k0 = k * b, kw = std::min(b, n - k0), k1 = k0 + kw;
    // ---- panel: columns k0..k1-1, rows k0..n-1 (factorDiagBlock / factorBelowDiagBlock)
    // Candidate of the first column by a plain scan (findMaxElm(0,0), lu.ci:266);
    // later columns get theirs from the fused update (lu.C:274-277).
    Cand cand;
    for (int r = k0; r < n; r++) cand.offer(std::fabs(A[(int64_t)r * lda + k0]), r);
    for (int j = k0; j < k1; j++) {
      int p = cand.row;
      if (p < 0) p = j;  // all-zero (or NaN) column: no swap, as LAPACK
      ipiv[j] = p;
      if (margin) margin[j] = cand.best > 0 ? (cand.best - cand.second) / cand.best : 0.0;
      if (p != j) {
        double* rj = A + (int64_t)j * lda;
        double* rp = A + (int64_t)p * lda;
        std::swap_ranges(rj, rj + n, rp);
        if (rhs) std::swap(rhs[j], rhs[p]);
      }
      double piv = A[(int64_t)j * lda + j];
      bool singular = !(std::fabs(piv) > sing_threshold);
      if (singular && info == 0) info = j + 1;
      const double* urow = A + (int64_t)j * lda;
      const bool scale = !(piv == 0.0 || std::isnan(piv));  // nothing sensible to scale by
      const bool has_next = j + 1 < k1;
      Cand next;
      const int nth = ((int64_t)(n - j) * (k1 - j) > 65536) ? omp_get_max_threads() : 1;
      std::vector<Cand> part(nth);
#pragma omp parallel num_threads(nth)
      {
        int t = omp_get_thread_num(), T = omp_get_num_threads();
        int64_t rows = n - (j + 1), lo = j + 1 + rows * t / T, hi = j + 1 + rows * (t + 1) / T;
        Cand c;
        for (int64_t r = lo; r < hi; r++) {
          double* ar = A + r * lda;
          if (scale) {
            double l = ar[j] / piv;          // true division (lu.C:270)
            ar[j] = l;
            for (int cc = j + 1; cc < k1; cc++)  // next column (lu.C:272) + dger (lu.C:247)
              ar[cc] = std::fma(-l, urow[cc], ar[cc]);
          }
          if (has_next) c.offer(std::fabs(ar[j + 1]), (int)r);
        }
        part[t] = c;
      }
      for (int t = 0; t < nth; t++) next.merge(part[t]);  // row order: lowest row wins ties
      cand = next;
    }
    if (k1 >= n) break;
    // ---- U block row: per-block dtrsm (factorAboveDiagBlock, lu.C:180-189)
    const double* L11 = A + (int64_t)k0 * lda + k0;
    const int nrest = nb - k - 1;
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = k + 1; y < nb; y++) {
      int c0 = y * b, cw = std::min(b, n - c0);
      trsm_llu(bl, kw, cw, L11, (int)lda, A + (int64_t)k0 * lda + c0, (int)lda);
    }
    // ---- trailing update: per-block dgemm in step order (lu.C:26-43)
    const int64_t ntiles = (int64_t)nrest * nrest;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t t = 0; t < ntiles; t++) {
      int x = k + 1 + (int)(t / nrest), y = k + 1 + (int)(t % nrest);
      int r0 = x * b, rw = std::min(b, n - r0), c0 = y * b, cw = std::min(b, n - c0);
      gemm_sub(bl, rw, cw, kw, A + (int64_t)r0 * lda + k0, (int)lda,
               A + (int64_t)k0 * lda + c0, (int)lda, A + (int64_t)r0 * lda + c0, (int)lda);
    }
  }
  return info;
}

// Block forward/backward substitution on the already-permuted right-hand
// side (lu.ci:387-458): per diagonal block x, subtract the off-diagonal
// block matvecs (offDiagSolve, summed over blocks in increasing index), then
// substitute inside the block; backward divides by u_ii (lu.ci:421).
void oracle_lu_solve_permuted(int n, int b, const double* LU, int64_t lda, double* x) {
  const int nb = (n + b - 1) / b;
  std::vector<double> acc(b), part(b);
  for (int bx = 0; bx < nb; bx++) {
    int r0 = bx * b, rw = std::min(b, n - r0);
    std::fill(acc.begin(), acc.begin() + rw, 0.0);
    for (int by = 0; by < bx; by++) {
      int c0 = by * b;
      for (int i = 0; i < rw; i++) {
        double s = 0.0;
        for (int j = 0; j < b; j++) s += LU[(int64_t)(r0 + i) * lda + c0 + j] * x[c0 + j];
        acc[i] += s;
      }
    }
    for (int i = 0; i < rw; i++) x[r0 + i] -= acc[i];
    for (int i = 0; i < rw; i++)
      for (int j = 0; j < i; j++) x[r0 + i] -= LU[(int64_t)(r0 + i) * lda + r0 + j] * x[r0 + j];
  }
  for (int bx = nb - 1; bx >= 0; bx--) {
    int r0 = bx * b, rw = std::min(b, n - r0);
    std::fill(acc.begin(), acc.begin() + rw, 0.0);
    for (int by = bx + 1; by < nb; by++) {
      int c0 = by * b, cw = std::min(b, n - c0);
      for (int i = 0; i < rw; i++) {
        double s = 0.0;
        for (int j = 0; j < cw; j++) s += LU[(int64_t)(r0 + i) * lda + c0 + j] * x[c0 + j];
        acc[i] += s;
      }
    }
    for (int i = 0; i < rw; i++) x[r0 + i] -= acc[i];
    for (int i = rw - 1; i >= 0; i--) {
      for (int j = i + 1; j < rw; j++) x[r0 + i] -= LU[(int64_t)(r0 + i) * lda + r0 + j] * x[r0 + j];
      x[r0 + i] /= LU[(int64_t)(r0 + i) * lda + r0 + i];
    }
  }
}

// Residual check (benchmark.C:462-573, 385-400) on the original matrix.
// out[0] = max|a_ij| (the reference's "|A|inf"), out[1] = ||b||inf,
// out[2] = ||x||inf, out[3] = ||b - Ax||inf, out[4] = ||A||inf (max row sum),
// out[5] = r_ref = out3 / ((out0*out2 + out1) * n * eps),
// out[6] = r_hpl = out3 / ((out4*out2 + out1) * n * eps).
void oracle_residual(int n, const double* A, int64_t lda, const double* x, const double* rhs,
                     double* out) {
  double amax = 0, bmax = 0, xmax = 0, rmax = 0, anorm = 0;
#pragma omp parallel for reduction(max : amax, rmax, anorm) schedule(static)
  for (int i = 0; i < n; i++) {
    const double* ar = A + (int64_t)i * lda;
    double s = 0.0, rs = 0.0, m = 0.0;
    for (int j = 0; j < n; j++) {
      s += ar[j] * x[j];
      double v = std::fabs(ar[j]);
      rs += v;
      if (v > m) m = v;
    }
    double r = std::fabs(rhs[i] - s);
    if (m > amax) amax = m;
    if (r > rmax) rmax = r;
    if (rs > anorm) anorm = rs;
  }
  for (int i = 0; i < n; i++) {
    bmax = std::max(bmax, std::fabs(rhs[i]));
    xmax = std::max(xmax, std::fabs(x[i]));
  }
  const double eps = 2.220446049250313e-16, dn = (double)n;
  out[0] = amax; out[1] = bmax; out[2] = xmax; out[3] = rmax; out[4] = anorm;
  out[5] = rmax / ((amax * xmax + bmax) * dn * eps);
  out[6] = rmax / ((anorm * xmax + bmax) * dn * eps);
}

}  // extern "C"
