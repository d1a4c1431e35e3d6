// Triangular solves.
//
// TRSM leaf: B <- L^{-1} B with L unit lower (m <= 32), restating
// LUBlk::computeU (lu.C:180-189, dtrsm left/lower/unit).  Larger m is
// handled by host-side recursion with the GEMM kernel.
//
// TRSV: forward (unit lower) and backward (upper, divide by u_ii)
// substitution of one right-hand side, restating forwardSolve /
// backwardSolve / offDiagSolve (lu.ci:387-458).  The reference pipelines
// block rows through multicasts and a row-sum reduction into the diagonal
// chare; here one CTA per 64-row block takes a ticket in launch order and,
// before it joins the chain, reads its right-hand side and diagonal tile
// and inverts that tile.  It then accumulates the off-diagonal product as
// earlier blocks become final (a progress counter: CTAs finish in ticket
// order), applies the inverted tile (a 64 x 64 matrix-vector product, so
// the sequential part of each chain step is short) and publishes its rows.
// The reference's per-row division by u_ii happens inside the tile
// inversion; the result differs from plain substitution by rounding only.
// A CTA only ever waits on lower tickets, which were handed to CTAs already
// running, so the pipeline cannot deadlock.
#include "common.cuh"
#include "kernels.h"

namespace lub {
namespace {

template <typename T>
__global__ void __launch_bounds__(128) trsm_llu_leaf_kernel(const T* L, int64_t ldl, T* B, int64_t ldb, int m,
                                                            int ncols) {
  __shared__ T sL[32][33];
  for (int idx = threadIdx.x; idx < 32 * 32; idx += blockDim.x) {
    const int i = idx >> 5, p = idx & 31;
    sL[i][p] = (i < m && p < i) ? L[(int64_t)i * ldl + p] : T(0);
  }
  __syncthreads();
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncols) return;
  T x[32];
#pragma unroll
  for (int i = 0; i < 32; i++) x[i] = i < m ? B[(int64_t)i * ldb + col] : T(0);
#pragma unroll
  for (int i = 1; i < 32; i++) {
#pragma unroll
    for (int p = 0; p < i; p++) x[i] = fma(-sL[i][p], x[p], x[i]);
  }
#pragma unroll
  for (int i = 0; i < 32; i++)
    if (i < m) B[(int64_t)i * ldb + col] = x[i];
}

// B (w x ncols) <- L^{-1} B, L unit lower w x w (w <= kTrsmBlockMaxW), FP32,
// in one launch: each CTA keeps a slice of 4-32 columns of B in shared memory and
// walks down L in 32-row blocks, solving the block's diagonal part (one
// thread per column, in registers) and then updating the rows below it with
// the block's columns of L.  This replaces the recursion's chain of small
// launches (for w = 256: 8 leaf solves and 7 GEMMs) inside the mixed path's
// panels.
constexpr int kTrsmBlockMaxW = 256;
constexpr int kTrsmNT = 256;

// CB columns of B per CTA (4 .. 32): narrow slices spread a small solve over
// more SMs; each column's arithmetic is the same for every CB.
template <int CB>
__global__ void __launch_bounds__(kTrsmNT) trsm_llu_block_kernel(const float* __restrict__ L, int64_t ldl,
                                                                 float* __restrict__ B, int64_t ldb, int w,
                                                                 int ncols) {
  constexpr int TXN = CB / 4;          // groups of 4 columns
  constexpr int RS = kTrsmNT / TXN;    // rows updated in parallel
  __shared__ float sB[kTrsmBlockMaxW][CB + 1];
  __shared__ float sL[32][33];
  const int tid = threadIdx.x;
  const int c0 = blockIdx.x * CB;
  const int nc = min(CB, ncols - c0);
  for (int idx = tid; idx < w * CB; idx += kTrsmNT) {
    const int r = idx / CB, c = idx - r * CB;
    sB[r][c] = c < nc ? B[(int64_t)r * ldb + c0 + c] : 0.f;
  }
  for (int k0 = 0; k0 < w; k0 += 32) {
    const int kb = min(32, w - k0);
    for (int idx = tid; idx < 32 * 32; idx += kTrsmNT) {
      const int i = idx >> 5, p = idx & 31;
      sL[i][p] = (i < kb && p < i) ? L[(int64_t)(k0 + i) * ldl + k0 + p] : 0.f;
    }
    __syncthreads();
    // the diagonal block: forward substitution down each column
    if (tid < CB) {
      float x[32];
#pragma unroll
      for (int i = 0; i < 32; i++) x[i] = i < kb ? sB[k0 + i][tid] : 0.f;
#pragma unroll
      for (int i = 1; i < 32; i++) {
#pragma unroll
        for (int p = 0; p < i; p++) x[i] = fmaf(-sL[i][p], x[p], x[i]);
      }
#pragma unroll
      for (int i = 0; i < 32; i++)
        if (i < kb) sB[k0 + i][tid] = x[i];
    }
    __syncthreads();
    // the rows below: B[r, :] -= L[r, k0:k0+kb] B[k0:k0+kb, :], 4 columns per thread
    const int tx = tid % TXN, ty = tid / TXN;
    for (int r = k0 + kb + ty; r < w; r += RS) {
      const float* lr = L + (int64_t)r * ldl + k0;
      float a0 = sB[r][4 * tx], a1 = sB[r][4 * tx + 1], a2 = sB[r][4 * tx + 2], a3 = sB[r][4 * tx + 3];
      for (int p = 0; p < kb; p++) {
        const float l = __ldg(&lr[p]);
        a0 = fmaf(-l, sB[k0 + p][4 * tx], a0);
        a1 = fmaf(-l, sB[k0 + p][4 * tx + 1], a1);
        a2 = fmaf(-l, sB[k0 + p][4 * tx + 2], a2);
        a3 = fmaf(-l, sB[k0 + p][4 * tx + 3], a3);
      }
      sB[r][4 * tx] = a0;
      sB[r][4 * tx + 1] = a1;
      sB[r][4 * tx + 2] = a2;
      sB[r][4 * tx + 3] = a3;
    }
    __syncthreads();
  }
  for (int idx = tid; idx < w * CB; idx += kTrsmNT) {
    const int r = idx / CB, c = idx - r * CB;
    if (c < nc) B[(int64_t)r * ldb + c0 + c] = sB[r][c];
  }
}

// ---------------------------------------------------------------------------
// B (w x ncols) <- L^{-1} B for a wide right-hand block (the U block row of a
// mixed-path step: w = the panel width <= 512, ncols = every trailing
// column), FP32.  The inverses of L's 32 x 32 unit-lower diagonal blocks
// are formed first (tri_inv32_kernel, one CTA each), so every step of the
// block forward substitution is a product:
//   x_k = Dinv_k B_k,   B_below -= L_below,k x_k      (k = 0 .. w/32 - 1)
// Each CTA keeps a 32-column slice of B in shared memory for the whole
// solve and streams the L block columns through two shared buffers with
// the async copy unit (block k+1 in flight while block k is applied).
// Threads: 8 column groups of 4 x 64 rows; each thread updates 4 x 4 blocks
// (rows ty + 64 j, columns 4 tx ..): the x rows are read as float4
// broadcasts, the L rows at pitch 36 land in distinct banks.  This replaces
// the recursion's 16 leaf solves and 15 skinny GEMMs per step, which ran
// alone on the GPU between two panels.
// ---------------------------------------------------------------------------
constexpr int kWideMaxW = 512;
constexpr int kWideCB = 32;   // columns of B per CTA
constexpr int kWideNT = 256;
constexpr int kWideBP = 36;   // pitch of the B slice (16-byte rows, 8 rows in distinct banks)
constexpr int kWideLP = 36;   // pitch of a staged L block column (16-byte rows, 8 rows in distinct banks)
constexpr int kWideLBUF = (kWideMaxW - 32) * kWideLP;
constexpr size_t kWideSmem =
    ((size_t)kWideMaxW * kWideBP + 2 * (size_t)kWideLBUF + 2 * 1024) * sizeof(float);

// dinv[b] (32 x 32, row-major) = inverse of the unit-lower diagonal block b
// of L (w x w), rows / columns past w treated as identity
__global__ void __launch_bounds__(32) tri_inv32_kernel(const float* __restrict__ L, int64_t ldl, int w,
                                                       float* __restrict__ dinv) {
  __shared__ float sL[32][33];
  const int b = blockIdx.x, j = threadIdx.x, k0 = 32 * b, kb = min(32, w - k0);
#pragma unroll 4
  for (int i = 0; i < 32; i++) sL[i][j] = (i < kb && j < i) ? L[(int64_t)(k0 + i) * ldl + k0 + j] : 0.f;
  __syncthreads();
  // column j of the inverse: forward substitution on e_j
  float x[32];
#pragma unroll
  for (int i = 0; i < 32; i++) x[i] = i == j ? 1.f : 0.f;
#pragma unroll
  for (int i = 1; i < 32; i++) {
#pragma unroll
    for (int p = 0; p < i; p++) x[i] = fmaf(-sL[i][p], x[p], x[i]);
  }
  float* d = dinv + (size_t)b * 1024;
#pragma unroll
  for (int i = 0; i < 32; i++) d[i * 32 + j] = x[i];
}

__device__ __forceinline__ void cp_async16_zfill(void* sdst, const void* gsrc, bool pred) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(sdst)), "l"(gsrc), "r"(pred ? 16 : 0)
               : "memory");
}


// B rows r0 + ty + 64 i (i < NI, those below r0 + Rp) -= L_k rows x x_k,
// columns 8 tx .. 8 tx + 7.  Per 4 k: four x row segments (the same for the
// whole warp: broadcasts) and one float4 of L per row (8 consecutive rows of
// a quarter-warp in distinct banks) feed 32 NI FMAs per thread.  Rows past
// Rp read row Rp - 1 and are not stored.
template <int NI>
__device__ __forceinline__ void wide_update8(float* sB, const float* Ls, int r0, int Rp, int k0, int tx, int ty) {
  float c[NI][8];
  int lo[NI];
#pragma unroll
  for (int i = 0; i < NI; i++) {
    const int rr = ty + 64 * i;
    lo[i] = min(rr, Rp - 1) * kWideLP;
    if (rr < Rp) {
      const float4 a = *reinterpret_cast<const float4*>(&sB[(r0 + rr) * kWideBP + tx * 8]);
      const float4 b = *reinterpret_cast<const float4*>(&sB[(r0 + rr) * kWideBP + tx * 8 + 4]);
      c[i][0] = a.x; c[i][1] = a.y; c[i][2] = a.z; c[i][3] = a.w;
      c[i][4] = b.x; c[i][5] = b.y; c[i][6] = b.z; c[i][7] = b.w;
    } else {
#pragma unroll
      for (int q = 0; q < 8; q++) c[i][q] = 0.f;
    }
  }
#pragma unroll 2
  for (int k = 0; k < 32; k += 4) {
    float xv[4][8];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const float4 a = *reinterpret_cast<const float4*>(&sB[(k0 + k + q) * kWideBP + tx * 8]);
      const float4 b = *reinterpret_cast<const float4*>(&sB[(k0 + k + q) * kWideBP + tx * 8 + 4]);
      xv[q][0] = a.x; xv[q][1] = a.y; xv[q][2] = a.z; xv[q][3] = a.w;
      xv[q][4] = b.x; xv[q][5] = b.y; xv[q][6] = b.z; xv[q][7] = b.w;
    }
#pragma unroll
    for (int i = 0; i < NI; i++) {
      const float4 l = *reinterpret_cast<const float4*>(&Ls[lo[i] + k]);
#pragma unroll
      for (int e = 0; e < 8; e++) {
        float v = c[i][e];
        v = fmaf(-l.x, xv[0][e], v);
        v = fmaf(-l.y, xv[1][e], v);
        v = fmaf(-l.z, xv[2][e], v);
        v = fmaf(-l.w, xv[3][e], v);
        c[i][e] = v;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < NI; i++) {
    const int rr = ty + 64 * i;
    if (rr < Rp) {
      *reinterpret_cast<float4*>(&sB[(r0 + rr) * kWideBP + tx * 8]) = make_float4(c[i][0], c[i][1], c[i][2], c[i][3]);
      *reinterpret_cast<float4*>(&sB[(r0 + rr) * kWideBP + tx * 8 + 4]) =
          make_float4(c[i][4], c[i][5], c[i][6], c[i][7]);
    }
  }
}

// VEC: L, B, ldl and ldb allow 16-byte copies (else element loads)
template <bool VEC>
__global__ void __launch_bounds__(kWideNT, 1) trsm_wide_kernel(const float* __restrict__ L, int64_t ldl,
                                                              const float* __restrict__ dinv, float* __restrict__ B,
                                                              int64_t ldb, int w, int ncols) {
  extern __shared__ __align__(16) float wide_smem[];
  float* sB = wide_smem;                                  // [32 nkb][kWideBP]
  float* sL = wide_smem + (size_t)kWideMaxW * kWideBP;    // [2][w - 32][kWideLP]
  float* sD = sL + 2 * kWideLBUF;                         // [2][32][32]: Dinv of blocks k, k + 1
  const int tid = threadIdx.x;
  const int c0 = blockIdx.x * kWideCB, nc = min(kWideCB, ncols - c0);
  const int nkb = (w + 31) / 32, wp = nkb * 32;
  if (VEC && nc == kWideCB) {
    for (int idx = tid; idx < wp * 8; idx += kWideNT) {
      const int r = idx >> 3, q = idx & 7;
      cp_async16_zfill(&sB[r * kWideBP + q * 4], B + (int64_t)min(r, w - 1) * ldb + c0 + q * 4, r < w);
    }
  } else {
    for (int idx = tid; idx < wp * 32; idx += kWideNT) {
      const int r = idx >> 5, c = idx & 31;
      sB[r * kWideBP + c] = (r < w && c < nc) ? B[(int64_t)r * ldb + c0 + c] : 0.f;
    }
  }
  // Dinv_k, and the L block column k: rows 32 (k + 1) .. w, columns
  // 32 k .. 32 k + 31 (all inside L, since a block with rows below it is a
  // whole 32 columns), zero rows up to the padded height wp
  auto stage = [&](int k) {
    const int k0 = 32 * k, r0 = k0 + 32, R = w - r0, Rp = wp - r0;
    float* dd = sD + (k & 1) * 1024;
    cp_async16_zfill(&dd[tid * 4], dinv + (size_t)k * 1024 + tid * 4, true);
    float* dst = sL + (size_t)(k & 1) * kWideLBUF;
    if (VEC) {
      for (int idx = tid; idx < Rp * 8; idx += kWideNT) {
        const int r = idx >> 3, q = idx & 7;
        cp_async16_zfill(&dst[r * kWideLP + q * 4], L + (int64_t)(r0 + min(r, R - 1)) * ldl + k0 + q * 4, r < R);
      }
    } else {
      for (int idx = tid; idx < Rp * 32; idx += kWideNT) {
        const int r = idx >> 5, c = idx & 31;
        dst[r * kWideLP + c] = r < R ? L[(int64_t)(r0 + r) * ldl + k0 + c] : 0.f;
      }
    }
  };
  stage(0);
  asm volatile("cp.async.commit_group;" ::: "memory");
  const int tx = tid >> 6, ty = tid & 63;   // update: 8 columns from 8 tx, rows ty + 64 i
  const int xr = tid >> 3, xc = tid & 7;    // x: row xr, columns 4 xc ..
  for (int k = 0; k < nkb; k++) {
    const int k0 = 32 * k, r0 = k0 + 32, Rp = wp - r0;
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();  // B slice, Dinv_k and L block k in shared memory; step k-1 done with the other buffers
    if (k + 1 < nkb) stage(k + 1);
    asm volatile("cp.async.commit_group;" ::: "memory");
    // x_k = Dinv_k B_k
    {
      const float* drow = sD + (k & 1) * 1024 + xr * 32;
      float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int p = 0; p < 32; p += 4) {
        const float4 d = *reinterpret_cast<const float4*>(drow + p);
        const float4 b0 = *reinterpret_cast<const float4*>(&sB[(k0 + p) * kWideBP + xc * 4]);
        const float4 b1 = *reinterpret_cast<const float4*>(&sB[(k0 + p + 1) * kWideBP + xc * 4]);
        const float4 b2 = *reinterpret_cast<const float4*>(&sB[(k0 + p + 2) * kWideBP + xc * 4]);
        const float4 b3 = *reinterpret_cast<const float4*>(&sB[(k0 + p + 3) * kWideBP + xc * 4]);
        acc.x = fmaf(d.x, b0.x, acc.x); acc.y = fmaf(d.x, b0.y, acc.y); acc.z = fmaf(d.x, b0.z, acc.z); acc.w = fmaf(d.x, b0.w, acc.w);
        acc.x = fmaf(d.y, b1.x, acc.x); acc.y = fmaf(d.y, b1.y, acc.y); acc.z = fmaf(d.y, b1.z, acc.z); acc.w = fmaf(d.y, b1.w, acc.w);
        acc.x = fmaf(d.z, b2.x, acc.x); acc.y = fmaf(d.z, b2.y, acc.y); acc.z = fmaf(d.z, b2.z, acc.z); acc.w = fmaf(d.z, b2.w, acc.w);
        acc.x = fmaf(d.w, b3.x, acc.x); acc.y = fmaf(d.w, b3.y, acc.y); acc.z = fmaf(d.w, b3.z, acc.z); acc.w = fmaf(d.w, b3.w, acc.w);
      }
      __syncthreads();  // every read of the block's rows done
      *reinterpret_cast<float4*>(&sB[(k0 + xr) * kWideBP + xc * 4]) = acc;
      __syncthreads();
    }
    if (Rp <= 0) continue;
    // B rows below -= L_below,k x_k over the padded height (the rows past w
    // have zero L rows and stay zero)
    const float* Ls = sL + (size_t)(k & 1) * kWideLBUF;
    switch ((Rp + 63) >> 6) {
      case 8: wide_update8<8>(sB, Ls, r0, Rp, k0, tx, ty); break;
      case 7: wide_update8<7>(sB, Ls, r0, Rp, k0, tx, ty); break;
      case 6: wide_update8<6>(sB, Ls, r0, Rp, k0, tx, ty); break;
      case 5: wide_update8<5>(sB, Ls, r0, Rp, k0, tx, ty); break;
      case 4: wide_update8<4>(sB, Ls, r0, Rp, k0, tx, ty); break;
      case 3: wide_update8<3>(sB, Ls, r0, Rp, k0, tx, ty); break;
      case 2: wide_update8<2>(sB, Ls, r0, Rp, k0, tx, ty); break;
      default: wide_update8<1>(sB, Ls, r0, Rp, k0, tx, ty); break;
    }
  }
  __syncthreads();
  for (int idx = tid; idx < w * 32; idx += kWideNT) {
    const int r = idx >> 5, c = idx & 31;
    if (c < nc) B[(int64_t)r * ldb + c0 + c] = sB[r * kWideBP + c];
  }
}

constexpr int TB = 64;  // rows per TRSV block

// Inverse of the diagonal tile, computed by each pipeline CTA before it
// joins the chain (it depends on nothing else), so that the chain step
// itself is a 64 x 64 matrix-vector product instead of a 64-step
// substitution.  D: the tile as stored (element (i, j) at D[i * ldd + j]),
// unit lower (UPPER = false; the diagonal is not read) or upper; rows past
// `rows` are treated as identity.  Four threads per column (256 threads),
// rows in dependency order:
//   lower: Dinv[i][j] = -sum_{j <= k < i} D[i][k] Dinv[k][j]
//   upper: Dinv[i][j] = (delta_ij - sum_{i < k <= j} D[i][k] Dinv[k][j]) / D[i][i]
template <bool UPPER, typename TD, typename TI>
__device__ void tri_inverse_tile(const TD* D, int ldd, TI* Dinv, int ldi, int rows) {
  const int tid = threadIdx.x, j = tid >> 2, q = tid & 3;
  for (int step = 0; step < TB; step++) {
    const int i = UPPER ? TB - 1 - step : step;
    const bool live = i < rows && (UPPER ? i <= j : i > j);
    TI s = TI(0);
    if (live) {
      if (UPPER) {
        for (int k = i + 1 + q; k <= j; k += 4) s = fma((TI)D[i * ldd + k], Dinv[k * ldi + j], s);
      } else {
        for (int k = j + q; k < i; k += 4) s = fma((TI)D[i * ldd + k], Dinv[k * ldi + j], s);
      }
    }
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    TI v;
    if (!live) v = (i == j) ? TI(1) : TI(0);
    else if (UPPER) v = ((i == j ? TI(1) : TI(0)) - s) / (TI)D[i * ldd + i];
    else v = -s;
    if (q == 0) Dinv[i * ldi + j] = v;
    __syncwarp();
  }
}

// Pipeline progress: CTAs finish in ticket order (each waits for its
// predecessor), so one counter, set to ticket + 1 when a CTA has published
// its rows, tells every later CTA how many blocks are final.  A waiter far
// behind the front sleeps in proportion to its distance, which keeps the
// polls on that one word sparse.  Bounded: false after `spin` polls or when
// another CTA has recorded an error.
__device__ __forceinline__ bool wait_progress(const int* counter, int need, int* seen, DevStatus* st, long long spin,
                                              int where) {
  long long polls = 0;
  int v = ld_acquire_s32(counter);
  while (v < need) {
    if (++polls > spin) { dev_fail(st, LU_ERR_TIMEOUT, where); return false; }
    if ((polls & 255) == 0 && ld_acquire_s32(&st->code) != 0) return false;
    const int gap = need - v;
    if (gap > 2) __nanosleep(min(gap, 64) * 256);
    v = ld_acquire_s32(counter);
  }
  *seen = v;
  return true;
}

// TS: storage type of the factors; T: type of the vector and the arithmetic
// (FP32 factors with an FP64 vector give the GMRES-IR preconditioner solve
// in working precision at the FP32 factors' memory cost).
// Dynamic shared memory: inverse of the diagonal tile (T, [TB][TB + 1]),
// then the tile as stored (TS, [TB][TB + 1]).
template <typename TS, typename T>
__host__ __device__ constexpr size_t trsv_smem() {
  return (size_t)TB * (TB + 1) * (sizeof(T) + sizeof(TS));
}

template <typename TS, typename T, bool UPPER>
__global__ void __launch_bounds__(256) trsv_kernel(const TS* LU, int64_t lda, int n, T* x, int* flags,
                                                   unsigned* ticket, DevStatus* st, long long spin) {
  extern __shared__ __align__(16) unsigned char trsv_raw[];
  T* sInv = reinterpret_cast<T*>(trsv_raw);
  TS* sD = reinterpret_cast<TS*>(sInv + TB * (TB + 1));
  __shared__ T s_acc[TB];
  __shared__ T s_rhs[TB];
  __shared__ int s_blk;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) s_blk = (int)atomicAdd(ticket, 1u);
  __syncthreads();
  const int nblk = (n + TB - 1) / TB;
  const int tk = s_blk;
  if (tk >= nblk) return;
  const int bi = UPPER ? nblk - 1 - tk : tk;
  const int r0 = bi * TB, rows = min(TB, n - r0);

  // off the chain: this block's right-hand side, the diagonal tile and its
  // inverse (no other CTA writes these rows of x before this one does)
  const T own = tid < rows ? x[r0 + tid] : T(0);
#pragma unroll 4
  for (int u = 0; u < TB * TB / 256; u++) {
    const int idx = tid + u * 256;
    const int i = idx / TB, jj = idx - i * TB;
    sD[i * (TB + 1) + jj] = (i < rows && jj < rows) ? LU[(int64_t)(r0 + i) * lda + r0 + jj] : TS(0);
  }
  __syncthreads();
  tri_inverse_tile<UPPER, TS, T>(sD, TB + 1, sInv, TB + 1, rows);

  T acc[8];
#pragma unroll
  for (int i = 0; i < 8; i++) acc[i] = T(0);
  const int nvisit = UPPER ? (nblk - 1 - bi) : bi;
  bool ok = true;
  // a ring of D tiles in registers (this warp's 8 rows of tiles q ..
  // q + D - 1): D - 1 tiles' loads are in flight while tile q is applied,
  // and a tile's slice of x is loaded with it when its block is already
  // known final (otherwise after the wait)
  constexpr int D = sizeof(TS) == 4 ? 4 : 2;
  auto col0 = [&](int q) { return (UPPER ? nblk - 1 - q : q) * TB; };
  auto load_tile = [&](int q, TS (&dst)[8][2]) {
    const int c0 = col0(q);
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int r = r0 + warp * 8 + i;
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int c = c0 + lane * 2 + e;
        dst[i][e] = (r < n && c < n) ? __ldcs(&LU[(int64_t)r * lda + c]) : TS(0);
      }
    }
  };
  auto load_x = [&](int q, T (&xd)[2]) {
    const int c = col0(q) + lane * 2;
    xd[0] = c < n ? __ldcg(&x[c]) : T(0);
    xd[1] = c + 1 < n ? __ldcg(&x[c + 1]) : T(0);
  };
  TS ring[D][8][2];
  T xr[D][2];
  bool xok[D];
  int seen = 0;
#pragma unroll
  for (int d = 0; d < D - 1; d++) {
    if (d < nvisit) {
      load_tile(d, ring[d]);
      xok[d] = false;
    }
  }
  for (int q0 = 0; q0 < nvisit && ok; q0 += D) {
#pragma unroll
    for (int d = 0; d < D; d++) {
      const int q = q0 + d;
      if (q >= nvisit || !ok) break;
      const int qn = q + D - 1, dn = (d + D - 1) % D;
      if (qn < nvisit) {
        load_tile(qn, ring[dn]);
        xok[dn] = qn < seen;
        if (xok[dn]) load_x(qn, xr[dn]);
      }
      if (q + 1 > seen) {  // block q (in ticket order) not known to be final yet
        int v = 0;
        if (lane == 0) ok = wait_progress(&flags[0], q + 1, &v, st, spin, 301);
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
        seen = __shfl_sync(0xffffffffu, v, 0);
        __syncwarp();  // lane 0's acquire orders the other lanes' reads of x
        if (!ok) break;
      }
      if (!xok[d]) load_x(q, xr[d]);
#pragma unroll
      for (int i = 0; i < 8; i++) acc[i] = fma((T)ring[d][i][1], xr[d][1], fma((T)ring[d][i][0], xr[d][0], acc[i]));
    }
  }
#pragma unroll
  for (int i = 0; i < 8; i++) {
    T v = acc[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) s_acc[warp * 8 + i] = v;
  }
  if (!__syncthreads_and(ok ? 1 : 0)) return;
  if (tid < TB) s_rhs[tid] = own - s_acc[tid];
  __syncthreads();
  // x_bi = Dinv (b_bi - off-diagonal part): row tid / 4, a quarter of the columns
  {
    const int r = tid >> 2, q4 = tid & 3;
    T sum = T(0);
#pragma unroll
    for (int m = 0; m < TB / 4; m++) {
      const int cc = q4 + 4 * m;
      sum = fma(sInv[r * (TB + 1) + cc], s_rhs[cc], sum);
    }
    sum += __shfl_xor_sync(0xffffffffu, sum, 1);
    sum += __shfl_xor_sync(0xffffffffu, sum, 2);
    if (q4 == 0 && r < rows) x[r0 + r] = sum;
  }
  // CTA barrier, then thread 0's release store: the rows written above are
  // visible to every CTA that acquires the counter
  __syncthreads();
  if (tid == 0) st_release_s32(&flags[0], tk + 1);
}

// ---------------------------------------------------------------------------
// Multi-right-hand-side triangular solve T Y = B in place on a row-major
// n x nrhs FP64 block (nrhs <= 16 per launch), T taken from row-major LU
// factors stored as TS (FP64, or FP32 factors applied in FP64 arithmetic):
//   MODE 0  LN: T = L  (unit lower)      forward,  tiles L[bi][bk], bk < bi
//   MODE 1  UN: T = U  (upper)           backward, tiles U[bi][bk], bk > bi
//   MODE 2  UT: T = U^T (lower)          forward,  tiles U[bk][bi]^T, bk < bi
//   MODE 3  LT: T = L^T (unit upper)     backward, tiles L[bk][bi]^T, bk > bi
// Modes 2 and 3 are the transposed solves of the adjoint (A^T lambda = W).
// Same ticket / progress-counter pipeline as trsv_kernel, with the inverted
// diagonal tile.  Both 64 x 64 x 16 products of a step (an off-diagonal
// tile against the finished rows of Y, and the inverted diagonal tile
// against the block's right-hand side) run on the FP64 tensor pipe
// (mma.sync m16n8k4; warp w owns output rows 16 (w / 2).., columns
// 8 (w % 2)..).  The factor tiles do not depend on the pipeline, so they
// stream through a two-stage cp.async ring (tile q+1 in flight while the
// CTA waits for block q and applies tile q); only the 64 x 16 slice of Y
// waits for the counter.  Tiles are read by rows in every mode (the
// transposed modes index the staged tile transposed).  Pitches keep the
// fragment loads free of bank conflicts.
// Dynamic shared memory: the ring, then the FP64 inverse of the diagonal
// tile ([TB][kInvPitch], D^{-1} of the stored tile).
// ---------------------------------------------------------------------------
template <typename TS, bool TRANS>
__host__ __device__ constexpr int pipe_pitch() { return (sizeof(TS) == 4 && TRANS) ? 72 : 68; }
template <typename TS>
__host__ __device__ constexpr size_t pipe_ring_bytes() {
  return 2 * (size_t)TB * (pipe_pitch<TS, false>() > pipe_pitch<TS, true>() ? pipe_pitch<TS, false>()
                                                                            : pipe_pitch<TS, true>()) *
         sizeof(TS);
}
constexpr int kInvPitch = 68;
constexpr int kYkPitch = 20;
template <typename TS>
__host__ __device__ constexpr size_t pipe_smem() {
  return pipe_ring_bytes<TS>() + (size_t)TB * kInvPitch * sizeof(double);
}

__device__ __forceinline__ void dmma16x8x4(double (&c)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

template <typename TS, int MODE>
__global__ void __launch_bounds__(256, 2) trsm_pipe_kernel(const TS* LU, int64_t lda, int n, double* Y, int64_t ldy,
                                                        int nrhs, int* flags, unsigned* ticket, DevStatus* st,
                                                        long long spin) {
  constexpr bool FWD = (MODE == 0 || MODE == 2);
  constexpr bool TRANS = (MODE >= 2);
  constexpr int TP = pipe_pitch<TS, TRANS>();
  constexpr int EPC = 16 / (int)sizeof(TS);   // elements per 16-byte chunk
  constexpr int CPR = TB / EPC;               // chunks per tile row
  extern __shared__ __align__(16) unsigned char pipe_raw[];
  TS* ring = reinterpret_cast<TS*>(pipe_raw);  // [2][TB][TP]
  double* dinv = reinterpret_cast<double*>(pipe_raw + pipe_ring_bytes<TS>());  // [TB][kInvPitch]
  __shared__ __align__(16) double yk[TB][kYkPitch];
  __shared__ int s_blk, s_ok;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) s_blk = (int)atomicAdd(ticket, 1u);
  __syncthreads();
  const int nblk = (n + TB - 1) / TB;
  const int tk = s_blk;
  if (tk >= nblk) return;
  const int bi = FWD ? tk : nblk - 1 - tk;
  const int r0 = bi * TB, rows = min(TB, n - r0);
  const int nvisit = FWD ? bi : nblk - 1 - bi;
  // MMA fragment coordinates: group g, thread-in-group t; warp tile rows
  // m0 .. m0 + 15, columns n0 .. n0 + 7
  const int g = lane >> 2, t = lane & 3;
  const int m0 = (warp >> 1) * 16, n0 = (warp & 1) * 8;

  // stage a tile into ring slot `slot`: rows grow0.., cols gcol0.. (nrow x ncol valid)
  auto stage = [&](int slot, int grow0, int gcol0, int nrow, int ncol) {
    TS* buf = ring + slot * TB * TP;
    for (int ch = tid; ch < TB * CPR; ch += 256) {
      const int i = ch / CPR, j = (ch - i * CPR) * EPC;
      const int valid = i < nrow ? max(0, min(EPC, ncol - j)) : 0;
      const TS* src = valid ? LU + (int64_t)(grow0 + i) * lda + gcol0 + j : LU;
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(buf + i * TP + j)), "l"(src),
                   "r"(valid * (int)sizeof(TS))
                   : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  // off-diagonal tile q: NoTrans rows r0.., cols c0..; Trans rows c0.., cols r0..
  auto issue = [&](int q) {
    const int c0 = (FWD ? q : nblk - 1 - q) * TB, cw = min(TB, n - c0);
    if (TRANS) stage(q & 1, c0, r0, cw, rows);
    else stage(q & 1, r0, c0, rows, cw);
  };

  // off the chain: this block's right-hand side (in the accumulator layout),
  // the diagonal tile through ring slot 0 and its inverse
  double own[4];
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const int r = m0 + g + (e >> 1) * 8, c = n0 + 2 * t + (e & 1);
    own[e] = (r < rows && c < nrhs) ? Y[(int64_t)(r0 + r) * ldy + c] : 0.0;
  }
  stage(0, r0, r0, rows, rows);
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();
  // D^{-1} of the stored tile (U for modes 1 and 2, unit L for 0 and 3);
  // T^{-1} is D^{-1} or its transpose
  tri_inverse_tile<(MODE == 1 || MODE == 2), TS, double>(ring, TP, dinv, kInvPitch, rows);
  __syncthreads();  // ring slot 0 is reused below

  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  bool ok = true;
  int seen = 0;
  if (nvisit > 0) issue(0);
  for (int q = 0; q < nvisit; q++) {
    const int bk = FWD ? q : nblk - 1 - q;
    const int c0 = bk * TB, cw = min(TB, n - c0);
    if (q + 1 < nvisit) issue(q + 1);
    if (q + 1 > seen) {  // block q (in ticket order) not known to be final yet
      if (tid == 0) {
        int v = 0;
        s_ok = wait_progress(&flags[0], q + 1, &v, st, spin, 302) ? v : -1;
      }
      __syncthreads();
      seen = s_ok;
      if (seen < 0) { ok = false; break; }
    }
#pragma unroll
    for (int u = 0; u < TB * 16 / 256; u++) {
      const int idx = tid + u * 256;
      const int i = idx >> 4, c = idx & 15;
      yk[i][c] = (i < cw && c < nrhs) ? __ldcg(&Y[(int64_t)(c0 + i) * ldy + c]) : 0.0;
    }
    if (q + 1 < nvisit) asm volatile("cp.async.wait_group 1;" ::: "memory");
    else asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    const TS* tq = ring + (q & 1) * TB * TP;
    // acc += T[bi][bk] * Y[bk] on this warp's 16 x 8 tile
#pragma unroll
    for (int ks = 0; ks < TB / 4; ks++) {
      const int k = ks * 4 + t;
      const double a0 = (double)(TRANS ? tq[k * TP + m0 + g] : tq[(m0 + g) * TP + k]);
      const double a1 = (double)(TRANS ? tq[k * TP + m0 + g + 8] : tq[(m0 + g + 8) * TP + k]);
      dmma16x8x4(acc, a0, a1, yk[k][n0 + g]);
    }
    __syncthreads();  // ring slot, yk and s_ok are rewritten next
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  if (!ok) return;  // uniform: every thread read the same s_ok
  // R = B_bi - off-diagonal part (into yk), then Y_bi = T^{-1} R
#pragma unroll
  for (int e = 0; e < 4; e++) yk[m0 + g + (e >> 1) * 8][n0 + 2 * t + (e & 1)] = own[e] - acc[e];
  __syncthreads();
  double out[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int ks = 0; ks < TB / 4; ks++) {
    const int k = ks * 4 + t;
    const double a0 = TRANS ? dinv[k * kInvPitch + m0 + g] : dinv[(m0 + g) * kInvPitch + k];
    const double a1 = TRANS ? dinv[k * kInvPitch + m0 + g + 8] : dinv[(m0 + g + 8) * kInvPitch + k];
    dmma16x8x4(out, a0, a1, yk[k][n0 + g]);
  }
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const int r = m0 + g + (e >> 1) * 8, c = n0 + 2 * t + (e & 1);
    if (r < rows && c < nrhs) Y[(int64_t)(r0 + r) * ldy + c] = out[e];
  }
  // CTA barrier, then thread 0's release store: the rows written above are
  // visible to every CTA that acquires the counter
  __syncthreads();
  if (tid == 0) st_release_s32(&flags[0], tk + 1);
}

// G = -Lam * X^T (n x n), Lam and X n x k row-major, k <= 16: the rank-k
// gradient of the adjoint.  Output-bound (8 n^2 bytes written): each thread
// keeps its two columns' X rows in registers and reads Lam rows as
// warp-wide broadcasts, so shared-memory traffic stays well below the FMAs.
__global__ void __launch_bounds__(256) neg_outer_kernel(const double* Lam, int64_t ldl, const double* X, int64_t ldx,
                                                        int n, int k, double* G, int64_t ldg, int accumulate) {
  __shared__ __align__(16) double sl[64][16];
  __shared__ double sx[64][17];
  const int i0 = blockIdx.y * 64, j0 = blockIdx.x * 64;
  for (int idx = threadIdx.x; idx < 64 * 16; idx += blockDim.x) {
    const int r = idx >> 4, c = idx & 15;
    sl[r][c] = (i0 + r < n && c < k) ? Lam[(int64_t)(i0 + r) * ldl + c] : 0.0;
    sx[r][c] = (j0 + r < n && c < k) ? X[(int64_t)(j0 + r) * ldx + c] : 0.0;
  }
  __syncthreads();
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads, 8 rows x 2 columns each
  double xr0[16], xr1[16];
#pragma unroll
  for (int q = 0; q < 16; q++) {
    xr0[q] = sx[tx][q];
    xr1[q] = sx[tx + 32][q];
  }
  for (int ri = 0; ri < 8; ri++) {
    const int r = ty * 8 + ri;
    if (i0 + r >= n) break;
    double t0 = 0.0, t1 = 0.0;
#pragma unroll
    for (int q = 0; q < 16; q += 2) {
      const double2 l = *reinterpret_cast<const double2*>(&sl[r][q]);
      t0 = fma(l.x, xr0[q], t0);
      t1 = fma(l.x, xr1[q], t1);
      t0 = fma(l.y, xr0[q + 1], t0);
      t1 = fma(l.y, xr1[q + 1], t1);
    }
    double* g = &G[(int64_t)(i0 + r) * ldg + j0];
    if (j0 + tx < n) {
      if (accumulate) g[tx] -= t0;
      else __stcs(&g[tx], -t0);
    }
    if (j0 + tx + 32 < n) {
      if (accumulate) g[tx + 32] -= t1;
      else __stcs(&g[tx + 32], -t1);
    }
  }
}

// Y[i][:] = X[perm[i]][:] (gather) or Y[perm[i]][:] = X[i][:] (scatter)
__global__ void permute_rows_kernel(const double* X, int64_t ldx, double* Y, int64_t ldy, const int32_t* perm, int n,
                                    int k, int scatter) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * k) return;
  const int i = (int)(idx / k), c = (int)(idx - (int64_t)i * k);
  if (scatter) Y[(int64_t)perm[i] * ldy + c] = X[(int64_t)i * ldx + c];
  else Y[(int64_t)i * ldy + c] = X[(int64_t)perm[i] * ldx + c];
}

}  // namespace

template <typename TS, int MODE>
int pipe_attr() {
  static PerDeviceOnce once;
  return once_per_device(once, [] {
    return cuda_status(cudaFuncSetAttribute(trsm_pipe_kernel<TS, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)pipe_smem<TS>()));
  });
}

template <typename TS>
int launch_trsm_pipe(const TS* LU, int64_t lda, int n, double* Y, int64_t ldy, int nrhs, int mode, int* flags,
                     unsigned* ticket, DevStatus* st, long long spin, cudaStream_t s) {
  if (n <= 0 || nrhs <= 0) return LU_OK;
  // factor rows are staged in 16-byte chunks
  if (((lda * (int64_t)sizeof(TS)) & 15) || (reinterpret_cast<uintptr_t>(LU) & 15)) return LU_ERR_ALIGN;
  LUB_TRY((pipe_attr<TS, 0>()));
  LUB_TRY((pipe_attr<TS, 1>()));
  LUB_TRY((pipe_attr<TS, 2>()));
  LUB_TRY((pipe_attr<TS, 3>()));
  const size_t smem = pipe_smem<TS>();
  const int nblk = ceil_div(n, TB);
  for (int c0 = 0; c0 < nrhs; c0 += 16) {
    const int k = std::min(16, nrhs - c0);
    LUB_CUDA(cudaMemsetAsync(flags, 0, sizeof(int), s));  // progress counter
    LUB_CUDA(cudaMemsetAsync(ticket, 0, sizeof(unsigned), s));
    switch (mode) {
      case 0: trsm_pipe_kernel<TS, 0><<<nblk, 256, smem, s>>>(LU, lda, n, Y + c0, ldy, k, flags, ticket, st, spin); break;
      case 1: trsm_pipe_kernel<TS, 1><<<nblk, 256, smem, s>>>(LU, lda, n, Y + c0, ldy, k, flags, ticket, st, spin); break;
      case 2: trsm_pipe_kernel<TS, 2><<<nblk, 256, smem, s>>>(LU, lda, n, Y + c0, ldy, k, flags, ticket, st, spin); break;
      case 3: trsm_pipe_kernel<TS, 3><<<nblk, 256, smem, s>>>(LU, lda, n, Y + c0, ldy, k, flags, ticket, st, spin); break;
      default: return LU_ERR_ARG;
    }
    LUB_LAUNCH_CHECK();
  }
  return LU_OK;
}

int launch_neg_outer(const double* Lam, int64_t ldl, const double* X, int64_t ldx, int n, int k, double* G,
                     int64_t ldg, cudaStream_t s) {
  if (n <= 0 || k <= 0) return LU_OK;
  dim3 grid(ceil_div(n, 64), ceil_div(n, 64));
  for (int c0 = 0; c0 < k; c0 += 16) {
    neg_outer_kernel<<<grid, 256, 0, s>>>(Lam + c0, ldl, X + c0, ldx, n, std::min(16, k - c0), G, ldg, c0 > 0);
    LUB_LAUNCH_CHECK();
  }
  return LU_OK;
}

int launch_permute_rows(const double* X, int64_t ldx, double* Y, int64_t ldy, const int32_t* perm, int n, int k,
                        int scatter, cudaStream_t s) {
  const int64_t tot = (int64_t)n * k;
  if (tot <= 0) return LU_OK;
  permute_rows_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(X, ldx, Y, ldy, perm, n, k, scatter);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

template <typename T>
int launch_trsm_llu_leaf(const T* L, int64_t ldl, T* B, int64_t ldb, int m, int ncols, cudaStream_t s) {
  if (m <= 1 || ncols <= 0) return LU_OK;
  if (m > 32) return LU_ERR_ARG;
  trsm_llu_leaf_kernel<T><<<ceil_div(ncols, 128), 128, 0, s>>>(L, ldl, B, ldb, m, ncols);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

int launch_trsm_llu_block(const float* L, int64_t ldl, float* B, int64_t ldb, int w, int ncols, cudaStream_t s) {
  if (w <= 1 || ncols <= 0) return LU_OK;
  if (w > kTrsmBlockMaxW) return LU_ERR_ARG;
  // slices narrow enough for at least ~32 CTAs
  if (ncols >= 1024)
    trsm_llu_block_kernel<32><<<ceil_div(ncols, 32), kTrsmNT, 0, s>>>(L, ldl, B, ldb, w, ncols);
  else if (ncols >= 512)
    trsm_llu_block_kernel<16><<<ceil_div(ncols, 16), kTrsmNT, 0, s>>>(L, ldl, B, ldb, w, ncols);
  else if (ncols >= 256)
    trsm_llu_block_kernel<8><<<ceil_div(ncols, 8), kTrsmNT, 0, s>>>(L, ldl, B, ldb, w, ncols);
  else
    trsm_llu_block_kernel<4><<<ceil_div(ncols, 4), kTrsmNT, 0, s>>>(L, ldl, B, ldb, w, ncols);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

// dinv: device scratch of 16 x 1024 floats (the diagonal-block inverses)
int launch_trsm_wide(const float* L, int64_t ldl, float* B, int64_t ldb, int w, int ncols, float* dinv,
                     cudaStream_t s) {
  if (w <= 0 || ncols <= 0) return LU_OK;
  if (w > kWideMaxW || !dinv) return LU_ERR_ARG;
  static PerDeviceOnce once;
  LUB_TRY(once_per_device(once, [] {
    LUB_CUDA(cudaFuncSetAttribute(trsm_wide_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kWideSmem));
    LUB_CUDA(cudaFuncSetAttribute(trsm_wide_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kWideSmem));
    return LU_OK;
  }));
  const int nkb = ceil_div(w, 32);
  tri_inv32_kernel<<<nkb, 32, 0, s>>>(L, ldl, w, dinv);
  LUB_LAUNCH_CHECK();
  const bool vec = ((reinterpret_cast<uintptr_t>(L) | reinterpret_cast<uintptr_t>(B)) & 15) == 0 &&
                   (ldl & 3) == 0 && (ldb & 3) == 0;
  const unsigned grid = (unsigned)ceil_div(ncols, kWideCB);
  if (vec)
    trsm_wide_kernel<true><<<grid, kWideNT, kWideSmem, s>>>(L, ldl, dinv, B, ldb, w, ncols);
  else
    trsm_wide_kernel<false><<<grid, kWideNT, kWideSmem, s>>>(L, ldl, dinv, B, ldb, w, ncols);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

template <typename TS, typename T>
int launch_trsv_mixed(const TS* LU, int64_t lda, int n, T* x, int upper, int* flags, unsigned* ticket, DevStatus* st,
                      long long spin, cudaStream_t s) {
  if (n <= 0) return LU_OK;
  const int nblk = ceil_div(n, TB);
  constexpr size_t smem = trsv_smem<TS, T>();
  static PerDeviceOnce once;
  LUB_TRY(once_per_device(once, [] {
    int r = cuda_status(
        cudaFuncSetAttribute(trsv_kernel<TS, T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (r == LU_OK)
      r = cuda_status(
          cudaFuncSetAttribute(trsv_kernel<TS, T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return r;
  }));
  // flags[0] is the progress counter; the ticket hands out block order
  LUB_CUDA(cudaMemsetAsync(flags, 0, sizeof(int), s));
  LUB_CUDA(cudaMemsetAsync(ticket, 0, sizeof(unsigned), s));
  if (upper)
    trsv_kernel<TS, T, true><<<nblk, 256, smem, s>>>(LU, lda, n, x, flags, ticket, st, spin);
  else
    trsv_kernel<TS, T, false><<<nblk, 256, smem, s>>>(LU, lda, n, x, flags, ticket, st, spin);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

template <typename T>
int launch_trsv(const T* LU, int64_t lda, int n, T* x, int upper, int* flags, unsigned* ticket, DevStatus* st,
                long long spin, cudaStream_t s) {
  return launch_trsv_mixed<T, T>(LU, lda, n, x, upper, flags, ticket, st, spin, s);
}
template int launch_trsv_mixed<float, double>(const float*, int64_t, int, double*, int, int*, unsigned*, DevStatus*,
                                              long long, cudaStream_t);

template int launch_trsm_pipe<double>(const double*, int64_t, int, double*, int64_t, int, int, int*, unsigned*,
                                      DevStatus*, long long, cudaStream_t);
template int launch_trsm_pipe<float>(const float*, int64_t, int, double*, int64_t, int, int, int*, unsigned*,
                                     DevStatus*, long long, cudaStream_t);
template int launch_trsm_llu_leaf<double>(const double*, int64_t, double*, int64_t, int, int, cudaStream_t);
template int launch_trsm_llu_leaf<float>(const float*, int64_t, float*, int64_t, int, int, cudaStream_t);
template int launch_trsv<double>(const double*, int64_t, int, double*, int, int*, unsigned*, DevStatus*, long long,
                                 cudaStream_t);
template int launch_trsv<float>(const float*, int64_t, int, float*, int, int*, unsigned*, DevStatus*, long long,
                                cudaStream_t);

}  // namespace lub

namespace {
// Test hook kernel: one thread waits on a progress counter that nothing
// advances; the bounded wait must give up, record the timeout in the status
// word and return.
__global__ void wait_timeout_probe_kernel(const int* counter, lub::DevStatus* st, long long spin, int* out) {
  int seen = 0;
  const bool ok = lub::wait_progress(counter, 1, &seen, st, spin, 399);
  *out = ok ? 1 : 0;
}
}  // namespace

// Exercises the bounded pipeline wait on a counter that never advances
// (failure detection without a fault): returns the status code the device
// recorded (LU_ERR_TIMEOUT expected) or a CUDA error.
extern "C" __attribute__((visibility("default"))) int lub_test_wait_timeout(long long spin) {
  using namespace lub;
  int* buf = nullptr;
  if (cudaMalloc(&buf, 64) != cudaSuccess) return LU_ERR_NOMEM;
  DevStatus* st = reinterpret_cast<DevStatus*>(buf + 4);
  int* out = buf + 2;
  cudaMemset(buf, 0, 64);
  wait_timeout_probe_kernel<<<1, 1>>>(buf, st, spin, out);
  int rc = cudaDeviceSynchronize() == cudaSuccess ? LU_OK : LU_ERR_CUDA;
  DevStatus hst{};
  int hout = -1;
  if (rc == LU_OK) {
    cudaMemcpy(&hst, st, sizeof(hst), cudaMemcpyDeviceToHost);
    cudaMemcpy(&hout, out, sizeof(int), cudaMemcpyDeviceToHost);
    rc = (hout == 0 && hst.code == LU_ERR_TIMEOUT) ? LU_ERR_TIMEOUT : (hst.code ? hst.code : LU_OK);
  }
  cudaFree(buf);
  return rc;
}

// Test hook (not part of the ABI): the blocked FP32 TRSM B <- L^{-1} B.
extern "C" __attribute__((visibility("default"))) int lub_test_trsm_block(const float* L, int64_t ldl, float* B,
                                                                        int64_t ldb, int w, int ncols, void* stream) {
  return lub::launch_trsm_llu_block(L, ldl, B, ldb, w, ncols, (cudaStream_t)stream);
}

// Test hook (not part of include/lu_b200.h): the wide block forward
// substitution with its own diagonal-inverse scratch.
extern "C" __attribute__((visibility("default"))) int lub_test_trsm_wide(const float* L, int64_t ldl, float* B,
                                                                       int64_t ldb, int w, int ncols, void* stream) {
  float* dinv = nullptr;
  if (cudaMalloc(&dinv, sizeof(float) * 16 * 1024) != cudaSuccess) return LU_ERR_CUDA;
  int rc = lub::launch_trsm_wide(L, ldl, B, ldb, w, ncols, dinv, (cudaStream_t)stream);
  cudaStreamSynchronize((cudaStream_t)stream);
  cudaFree(dinv);
  return rc;
}
