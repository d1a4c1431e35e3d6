// FP64 trailing update C -= A * B on the FP64 tensor pipe (mma.sync DMMA),
// fed by TMA into a multi-stage mbarrier pipeline.
//
// Replaces LUBlk::updateMatrix (lu.C:26-43): the reference runs one
// b x b x b dgemm (alpha = -1, beta = 1, row-major) per (block, step); here
// one launch updates the whole trailing matrix of a panel step, and the same
// kernel serves the GEMM halves of the recursive panel and TRSM.
//
// tcgen05 has no FP64 kind, so FP64 runs on mma.sync.m16n8k4.f64.
// Tiling: CTA 128 x 128, K-tile 16, 4 stages; 8 warps as 2 (m) x 4 (n),
// warp tile 64 x 32 = 4 x 4 DMMA tiles.  Shared-memory layout is what TMA's
// 128-byte swizzle writes: A stage = 128 rows x 128 B; B stage = 8 column
// slabs of 16 k-rows x 16 doubles.  Bank-conflict-free fragment loads come
// from two free choices of the MMA:
//   * k order: in k-step s the lane with k-index t uses physical column
//     2t + (s&1) + 8(s>>1), so a lane's A values for s = 0,1 (and 2,3) are
//     adjacent and load as one 16-byte access, and the four lanes of a
//     group hit B rows whose (row % 8) differ in bits 1-2;
//   * m order: MMA row g maps to tile row (g>>1) | ((g&1)<<2), so the two
//     rows of a quarter-warp differ by 4 in (row % 8) and their swizzled
//     16-byte chunks fall in disjoint halves of the bank space.
// The C tile is loaded into the accumulators first (its latency overlaps
// the TMA prologue) and A enters negated, so the MMA chain computes
// C - A*B directly; the epilogue is a plain store.
#include "common.cuh"
#include "kernels.h"

namespace lub {
namespace {

constexpr int BM = 128, BN = 128, BK = 16, STAGES = 4, THREADS = 256;
constexpr int A_STAGE_BYTES = BM * BK * 8;          // 16 KB
constexpr int B_STAGE_BYTES = BK * BN * 8;          // 16 KB
constexpr int STAGE_BYTES = A_STAGE_BYTES + B_STAGE_BYTES;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /*align*/ + 128 /*barriers*/;

__device__ __forceinline__ void dmma(double (&c)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

__device__ __forceinline__ int mrow_perm(int g) { return (g >> 1) | ((g & 1) << 2); }

__global__ void __launch_bounds__(THREADS, 1)
gemm_f64_sub_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                    GemmArgs args) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm = warp >> 2, wn = warp & 3;
  int tm, tn;
  grouped_tile(blockIdx.x, (args.M + BM - 1) / BM, (args.N + BN - 1) / BN, 16, tm, tn);
  const int tile_m = tm * BM, tile_n = tn * BN;
  const int M = args.M, N = args.N, K = args.K;
  const int KT = (K + BK - 1) / BK;

  if (tid == 0) {
    prefetch_tmap(&mapA);
    prefetch_tmap(&mapB);
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], THREADS / 32);
    }
    fence_mbar_init();
  }
  __syncthreads();

  auto issue = [&](int kt, int s) {
    unsigned char* sa = smem + s * STAGE_BYTES;
    unsigned char* sb = sa + A_STAGE_BYTES;
    mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
    tma_load_2d(sa, &mapA, &full[s], args.a_col0 + kt * BK, args.a_row0 + tile_m);
#pragma unroll
    for (int j = 0; j < BN / 16; j++)
      tma_load_2d(sb + j * (BK * 16 * 8), &mapB, &full[s], args.b_col0 + tile_n + j * 16, args.b_row0 + kt * BK);
  };
  if (tid == 0) {
    for (int s = 0; s < STAGES - 1 && s < KT; s++) issue(s, s);
  }

  // ---- accumulators <- C tile (zero outside the M x N bounds)
  double acc[4][4][4];
  const double* C = args.C;
  const int64_t ldc = args.ldc;
#pragma unroll
  for (int mi = 0; mi < 4; mi++) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int r = tile_m + wm * 64 + mi * 16 + h * 8 + mrow_perm(g);
#pragma unroll
      for (int nj = 0; nj < 4; nj++) {
        const int c = tile_n + wn * 32 + nj * 8 + 2 * t;
        double v0 = 0.0, v1 = 0.0;
        if (r < M) {
          const double* p = C + (int64_t)r * ldc + c;
          if (c + 1 < N) {
            double2 v = __ldcs(reinterpret_cast<const double2*>(p));
            v0 = v.x; v1 = v.y;
          } else if (c < N) {
            v0 = __ldcs(p);
          }
        }
        acc[mi][nj][2 * h] = v0;
        acc[mi][nj][2 * h + 1] = v1;
      }
    }
  }

  // ---- main loop
  for (int kt = 0; kt < KT; kt++) {
    const int s = kt % STAGES;
    if (tid == 0 && kt + STAGES - 1 < KT) {
      // tile kt+S-1 goes to the slot consumed in the previous iteration
      // (at kt = 0 that slot, S-1, has not been used yet)
      const int sp = (kt + STAGES - 1) % STAGES;
      if (kt >= 1 && !mbar_wait(&empty[sp], ((kt - 1) / STAGES) & 1, args.st, args.spin >> 4, 101)) break;
      issue(kt + STAGES - 1, sp);
    }
    if (!mbar_wait(&full[s], (kt / STAGES) & 1, args.st, args.spin >> 4, 102)) break;
    const unsigned char* sa = smem + s * STAGE_BYTES;
    const unsigned char* sb = sa + A_STAGE_BYTES;
    const int krem = K - kt * BK;  // valid k in this tile (>= 16 except the last)

#pragma unroll
    for (int half = 0; half < 2; half++) {
      // A: two k values per row per 16-byte load
      double2 af[4][2];
#pragma unroll
      for (int mi = 0; mi < 4; mi++) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int r = wm * 64 + mi * 16 + h * 8 + mrow_perm(g);
          const int chunk = (t + 4 * half) ^ (r & 7);
          af[mi][h] = *reinterpret_cast<const double2*>(sa + r * 128 + chunk * 16);
        }
      }
      double bf[4][2];
#pragma unroll
      for (int nj = 0; nj < 4; nj++) {
        const int n = wn * 32 + nj * 8 + g;
#pragma unroll
        for (int q = 0; q < 2; q++) {
          const int k = 2 * t + q + 8 * half;
          bf[nj][q] = *reinterpret_cast<const double*>(sb + (n >> 4) * (BK * 128) + k * 128 +
                                                       ((((n & 15) >> 1) ^ (k & 7)) << 4) + ((n & 1) << 3));
        }
      }
      if (krem < BK) {
#pragma unroll
        for (int q = 0; q < 2; q++) {
          const bool ok = (2 * t + q + 8 * half) < krem;
#pragma unroll
          for (int mi = 0; mi < 4; mi++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
              if (q == 0) af[mi][h].x = ok ? af[mi][h].x : 0.0;
              else        af[mi][h].y = ok ? af[mi][h].y : 0.0;
            }
#pragma unroll
          for (int nj = 0; nj < 4; nj++) bf[nj][q] = ok ? bf[nj][q] : 0.0;
        }
      }
#pragma unroll
      for (int q = 0; q < 2; q++) {
#pragma unroll
        for (int mi = 0; mi < 4; mi++) {
          const double a0 = -(q == 0 ? af[mi][0].x : af[mi][0].y);
          const double a1 = -(q == 0 ? af[mi][1].x : af[mi][1].y);
#pragma unroll
          for (int nj = 0; nj < 4; nj++) dmma(acc[mi][nj], a0, a1, bf[nj][q]);
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }

  // ---- epilogue: plain stores of the updated tile
  double* Cw = args.C;
#pragma unroll
  for (int mi = 0; mi < 4; mi++) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int r = tile_m + wm * 64 + mi * 16 + h * 8 + mrow_perm(g);
      if (r >= M) continue;
#pragma unroll
      for (int nj = 0; nj < 4; nj++) {
        const int c = tile_n + wn * 32 + nj * 8 + 2 * t;
        double* p = Cw + (int64_t)r * ldc + c;
        if (c + 1 < N) {
          __stcs(reinterpret_cast<double2*>(p), make_double2(acc[mi][nj][2 * h], acc[mi][nj][2 * h + 1]));
        } else if (c < N) {
          __stcs(p, acc[mi][nj][2 * h]);
        }
      }
    }
  }
}

}  // namespace

int gemm_f64_smem_bytes() { return SMEM_BYTES; }

int gemm_f64_init() {
  LUB_CUDA(cudaFuncSetAttribute(gemm_f64_sub_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
  return LU_OK;
}

// mapA: box 16 cols x 128 rows over the matrix holding A; mapB: box 16 x 16
// over the matrix holding B; both FP64 with 128-byte swizzle.
int launch_gemm_f64_sub(const CUtensorMap& mapA, const CUtensorMap& mapB, const GemmArgs& a,
                        cudaStream_t stream) {
  if (a.M <= 0 || a.N <= 0 || a.K <= 0) return LU_OK;
  if ((a.a_col0 & 1) || (a.b_col0 & 1) || (a.ldc & 1) || (reinterpret_cast<uintptr_t>(a.C) & 15))
    return LU_ERR_ALIGN;
  const int64_t tiles = (int64_t)ceil_div(a.N, BN) * ceil_div(a.M, BM);
  if (tiles > INT32_MAX) return LU_ERR_UNSUPPORTED;
  gemm_f64_sub_kernel<<<(unsigned)tiles, THREADS, SMEM_BYTES, stream>>>(mapA, mapB, a);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

}  // namespace lub
