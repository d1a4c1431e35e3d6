// Mixed-precision trailing update on the 5th-generation tensor cores:
//   C (FP32, row-major) -= L (BF16, M x K, K-major) * U^T (BF16, N x K, K-major)
// with FP32 accumulation in tensor memory.
//
// This is the B200 form of LUBlk::updateMatrix (lu.C:26-43) for the
// mixed-precision path: the reference's FP64 dgemm becomes one tcgen05 GEMM
// per panel step over the whole trailing matrix, its operands rounded to
// BF16 (the FP32 working matrix keeps the accumulated result).
//
// Structure (one 128 x 256 output tile per CTA, 128 threads):
//   warp 0, one lane : TMA producer — an A box 64 x 128 and two B boxes
//                      64 x 128 per k-block of 64, 128-byte swizzle, into a
//                      3-stage ring
//   warp 1           : allocates 256 TMEM columns; one lane issues
//                      tcgen05.mma.cta_group::1.kind::f16 (M=128, N=256,
//                      K=16) four times per stage and commits each stage's
//                      completion to that stage's "empty" mbarrier, the last
//                      one to the accumulator barrier
//   all 4 warps      : epilogue — tcgen05.ld 32 lanes x 32 columns per warp,
//                      negate, stage in a 128-byte-swizzled smem box, and
//                      cp.reduce.async.bulk.tensor .add.f32 into C (the
//                      read-modify-write of C happens at L2; C never passes
//                      through the SM).
// Shared-memory descriptors: K-major, SWIZZLE_128B, 8-row groups 1024 B
// apart (SBO = 1024), version 1; the k-th 16-element slice of a 64-wide
// block starts 32 bytes further.  No TMA load uses cluster multicast.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"
#include "kernels.h"

namespace lub {
namespace {

constexpr int BM = 128, BN = 256, BK = 64, STAGES = 3, THREADS = 128;
constexpr int A_BYTES = BM * BK * 2;            // 16 KB
constexpr int B_BYTES = BN * BK * 2;            // 32 KB
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;  // 48 KB
constexpr int EPI_COLS = 32;                    // fp32 columns per epilogue box (128 B)
constexpr int EPI_BYTES = BM * EPI_COLS * 4;    // 16 KB
constexpr int TMEM_COLS = 256;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 2 * EPI_BYTES + 1024 + 256;

__device__ __forceinline__ uint64_t smem_desc_k128(uint32_t addr) {
  // start (>>4) | LBO 16 B (unused for swizzled K-major) | SBO 1024 B | version 1 | SWIZZLE_128B
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// kind::f16 instruction descriptor: D = F32, A and B both BF16 (format 1) or
// both FP16 (format 0) — never mixed — both K-major, M = 128, N = 256
__host__ __device__ constexpr uint32_t make_idesc(bool bf16) {
  return (1u << 4) | ((bf16 ? 1u : 0u) << 7) | ((bf16 ? 1u : 0u) << 10) | ((uint32_t)(BN >> 3) << 17) |
         ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tma_reduce_add_2d(const CUtensorMap* map, const void* smem_src, int x, int y) {
  asm volatile("cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.tile.bulk_group [%0, {%2, %3}], [%1];" ::"l"(map),
               "r"(smem_u32(smem_src)), "r"(x), "r"(y)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Zero the lanes of a four-column group at or beyond the launch's column
// count (left = columns remaining from the group's first column). mapB may
// reach past the launch's N (a narrow update of the next panel's columns
// inside a wider trailing matrix); those columns belong to another launch and
// must receive a zero increment from this one.
__device__ __forceinline__ float4 mask_cols(float4 f, int left) {
  if (left < 4) {
    if (left < 1) f.x = 0.f;
    if (left < 2) f.y = 0.f;
    if (left < 3) f.z = 0.f;
    f.w = 0.f;
  }
  return f;
}

// The U^T operand's tensor map has a 64 x 128 box (BN_BOX rows), so the
// CTA-pair kernel can load half a 256-row tile; a whole tile is two boxes
// back to back, which with the 128-byte swizzle (a pattern of 8 rows,
// 1024 B) is the same shared-memory image as one 256-row box.
constexpr int BN_BOX = 128;
__device__ __forceinline__ void load_b_tile(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  tma_load_2d(dst, map, bar, x, y);
  tma_load_2d(static_cast<unsigned char*>(dst) + BN_BOX * BK * 2, map, bar, x, y + BN_BOX);
}

struct Bf16GemmArgs {
  int a_row0;   // first row of the tile grid in mapA's matrix (L rows)
  int b_row0;   // first row in mapB's matrix (U^T rows = output columns)
  int c_row0, c_col0;
  int M, N, K;
  uint32_t idesc;
  const unsigned* amax;  // per-panel |L|max, |U|max bit patterns (scaled FP16 operands) or null
  DevStatus* st;
  long long spin;
  int kpart;    // pairs layout: element offset of the lo parts (K = kpart); 0 otherwise
  unsigned* tile_ctr;  // persistent kernel: shared tile counter (dynamic tiles) or null (static striding)
};

__global__ void __launch_bounds__(THREADS, 1)
gemm_bf16_tc_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                    const __grid_constant__ CUtensorMap mapC, Bf16GemmArgs args) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* epi = smem + STAGES * STAGE_BYTES;
  uint64_t* full = reinterpret_cast<uint64_t*>(epi + 2 * EPI_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* accum = empty + STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accum + 1);
  __shared__ int s_fail;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int tm, tn;
  grouped_tile(blockIdx.x, (args.M + BM - 1) / BM, (args.N + BN - 1) / BN, 16, tm, tn);
  const int tile_m = tm * BM, tile_n = tn * BN;
  const int KT = (args.K + BK - 1) / BK;
  const long long lim = args.spin >> 4;

  if (tid == 0) {
    prefetch_tmap(&mapA);
    prefetch_tmap(&mapB);
    prefetch_tmap(&mapC);
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accum, 1);
    fence_mbar_init();
    s_fail = 0;
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer
    for (int kt = 0; kt < KT; kt++) {
      const int s = kt % STAGES;
      if (kt >= STAGES && !mbar_wait(&empty[s], ((kt / STAGES) - 1) & 1, args.st, lim, 401)) {
        s_fail = 1;
        break;
      }
      unsigned char* sa = smem + s * STAGE_BYTES;
      mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
      tma_load_2d(sa, &mapA, &full[s], kt * BK, args.a_row0 + tile_m);
      load_b_tile(sa + A_BYTES, &mapB, &full[s], kt * BK, args.b_row0 + tile_n);
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer
    for (int kt = 0; kt < KT; kt++) {
      const int s = kt % STAGES;
      if (!mbar_wait(&full[s], (kt / STAGES) & 1, args.st, lim, 402)) {
        s_fail = 1;
        break;
      }
      tc_fence_after();
      const uint32_t a_addr = smem_u32(smem + s * STAGE_BYTES);
      const uint32_t b_addr = a_addr + A_BYTES;
#pragma unroll
      for (int kk = 0; kk < BK / 16; kk++) {
        umma_f16(tmem, smem_desc_k128(a_addr + kk * 32), smem_desc_k128(b_addr + kk * 32), args.idesc,
                 (kt > 0 || kk > 0) ? 1u : 0u);
      }
      umma_commit(&empty[s]);
    }
    umma_commit(accum);
  }
  __syncwarp();

  // ---- epilogue: all four warps
  // every thread must agree before the warp-collective tcgen05.ld
  const bool ok = __syncthreads_and(mbar_wait(accum, 0, args.st, lim, 403) ? 1 : 0) != 0;
  tc_fence_after();
  const int row = warp * 32 + lane;  // TMEM lane == tile row
  // operands were scaled by powers of two; undo exactly on the accumulator
  const float unscale = args.amax ? pow2_unscale(args.amax) : 1.f;
  for (int c = 0; c < BN / EPI_COLS; c++) {
    uint32_t v[32];
    if (ok) tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c * EPI_COLS), v);
    if (tid == 0) bulk_wait_read<1>();  // the box written two chunks ago has been read
    __syncthreads();
    unsigned char* box = epi + (c & 1) * EPI_BYTES;
    const int cols_left = args.N - (tile_n + c * EPI_COLS);
#pragma unroll
    for (int j = 0; j < 8; j++) {
      float4 f = make_float4(-__uint_as_float(v[4 * j]) * unscale, -__uint_as_float(v[4 * j + 1]) * unscale,
                             -__uint_as_float(v[4 * j + 2]) * unscale, -__uint_as_float(v[4 * j + 3]) * unscale);
      *reinterpret_cast<float4*>(box + row * 128 + ((j ^ (row & 7)) << 4)) = mask_cols(f, cols_left - 4 * j);
    }
    fence_proxy_async();
    __syncthreads();
    if (tid == 0 && ok && !s_fail) {
      tma_reduce_add_2d(&mapC, box, args.c_col0 + tile_n + c * EPI_COLS, args.c_row0 + tile_m);
      bulk_commit();
    }
  }
  if (tid == 0) bulk_wait_all();
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

// ---------------------------------------------------------------------------
// Persistent variant: a fixed grid (the SM count, less any SMs left free for
// a panel running beside it) walks the tiles in grouped-raster order.  TMEM
// holds two 128 x 256 FP32 accumulators, so the epilogue of tile i (warps
// 2-5, named barrier 1) overlaps the MMAs of tile i+1 (warp 1) while warp 0
// keeps the TMA ring full across tile boundaries.
//   barriers: full/empty[STAGES] (operand ring), tfull/tempty[2] (accumulator
//   handoff; tempty counts the four epilogue warps)
// ---------------------------------------------------------------------------
constexpr int P_THREADS = 192;
constexpr int P_TMEM_COLS = 512;
// Pairs layout (error-compensated FP16): one stage holds the hi and lo parts
// of an L and a U k-block (Lh, Ll, Uh, Ul) and feeds three MMAs per 16-wide
// k step (Lh*Uh, Lh*Ul, Ll*Uh), so each part is loaded once instead of the
// three [hi,hi,lo] x [hi,lo,hi] k-blocks of the plain layout (a third less
// operand traffic per MMA).  Two stages fit beside the epilogue boxes.
constexpr int PAIR_STAGES = 2;
constexpr int PAIR_STAGE_BYTES = 2 * STAGE_BYTES;  // 96 KB
constexpr int PAIR_SMEM_BYTES = PAIR_STAGES * PAIR_STAGE_BYTES + 2 * EPI_BYTES + 1024 + 256;
static_assert(PAIR_SMEM_BYTES <= 227 * 1024, "pairs layout exceeds shared memory");

__device__ __forceinline__ void epi_bar() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

template <bool PAIRS>
__global__ void __launch_bounds__(P_THREADS, 1)
gemm_lowp_persistent_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                            const __grid_constant__ CUtensorMap mapC, Bf16GemmArgs args) {
  constexpr int NST = PAIRS ? PAIR_STAGES : STAGES;
  constexpr int SB = PAIRS ? PAIR_STAGE_BYTES : STAGE_BYTES;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* epi = smem + NST * SB;
  uint64_t* full = reinterpret_cast<uint64_t*>(epi + 2 * EPI_BYTES);
  uint64_t* empty = full + NST;
  uint64_t* tfull = empty + NST;
  uint64_t* tempty = tfull + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
  __shared__ int s_epi_fail;  // sticky: the epilogue warps stop together
  // The producer picks each tile (from the shared counter, or by striding)
  // and publishes it here for the MMA warp and the epilogue: entry i & 7
  // holds this CTA's i-th tile, -1 once there are no more.  The producer runs
  // at most 2 tiles + one ring of k-blocks ahead of the epilogue, so an entry
  // is read before it is reused.
  __shared__ volatile int s_tiles[8];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntm = (args.M + BM - 1) / BM, ntn = (args.N + BN - 1) / BN;
  const int tiles = ntm * ntn;
  const int KT = (args.K + BK - 1) / BK;
  const long long lim = args.spin >> 4;

  if (tid == 0) {
    prefetch_tmap(&mapA);
    prefetch_tmap(&mapB);
    prefetch_tmap(&mapC);
    for (int s = 0; s < NST; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4);
    }
    fence_mbar_init();
    s_epi_fail = 0;
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(P_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {  // ---- TMA producer
      long long kb = 0;
      bool ok = true;
      for (int i = 0; ok; i++) {
        int t = args.tile_ctr ? (int)atomicAdd(args.tile_ctr, 1u) : (int)blockIdx.x + i * (int)gridDim.x;
        if (t >= tiles) t = -1;
        s_tiles[i & 7] = t;
        __threadfence_block();
        if (t < 0) {
          // no more tiles: complete the next stage's phase without data so the
          // MMA warp reads the end mark
          const int s = (int)(kb % NST);
          if (kb >= NST && !mbar_wait(&empty[s], (uint32_t)(((kb / NST) - 1) & 1), args.st, lim, 415)) break;
          mbar_arrive(&full[s]);
          break;
        }
        int tm, tn;
        grouped_tile(t, ntm, ntn, 16, tm, tn);
        for (int kt = 0; kt < KT; kt++, kb++) {
          const int s = (int)(kb % NST);
          if (kb >= NST && !mbar_wait(&empty[s], (uint32_t)(((kb / NST) - 1) & 1), args.st, lim, 411)) {
            ok = false;
            break;
          }
          unsigned char* sa = smem + s * SB;
          mbar_arrive_expect_tx(&full[s], SB);
          if (PAIRS) {  // [Lh | Ll | Uh | Ul]
            tma_load_2d(sa, &mapA, &full[s], kt * BK, args.a_row0 + tm * BM);
            tma_load_2d(sa + A_BYTES, &mapA, &full[s], args.kpart + kt * BK, args.a_row0 + tm * BM);
            load_b_tile(sa + 2 * A_BYTES, &mapB, &full[s], kt * BK, args.b_row0 + tn * BN);
            load_b_tile(sa + 2 * A_BYTES + B_BYTES, &mapB, &full[s], args.kpart + kt * BK, args.b_row0 + tn * BN);
          } else {
            tma_load_2d(sa, &mapA, &full[s], kt * BK, args.a_row0 + tm * BM);
            load_b_tile(sa + A_BYTES, &mapB, &full[s], kt * BK, args.b_row0 + tn * BN);
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {  // ---- MMA issuer
      long long kb = 0;
      bool ok = true;
      for (int i = 0; ok; i++) {
        const int ab = i & 1, u = i >> 1;
        if (u >= 1 && !mbar_wait(&tempty[ab], (uint32_t)((u - 1) & 1), args.st, lim, 412)) break;
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(ab * 256);
        for (int kt = 0; kt < KT; kt++, kb++) {
          const int s = (int)(kb % NST);
          if (!mbar_wait(&full[s], (uint32_t)((kb / NST) & 1), args.st, lim, 413)) {
            ok = false;
            break;
          }
          if (kt == 0 && s_tiles[i & 7] < 0) {  // end mark: pass it on to the epilogue
            mbar_arrive(&tfull[ab]);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a_addr = smem_u32(smem + s * SB);
          if (PAIRS) {
            const uint32_t al_addr = a_addr + A_BYTES;
            const uint32_t bh_addr = a_addr + 2 * A_BYTES;
            const uint32_t bl_addr = bh_addr + B_BYTES;
#pragma unroll
            for (int kk = 0; kk < BK / 16; kk++) {
              const uint64_t ah = smem_desc_k128(a_addr + kk * 32), al = smem_desc_k128(al_addr + kk * 32);
              const uint64_t bh = smem_desc_k128(bh_addr + kk * 32), bl = smem_desc_k128(bl_addr + kk * 32);
              umma_f16(d, ah, bh, args.idesc, (kt > 0 || kk > 0) ? 1u : 0u);
              umma_f16(d, ah, bl, args.idesc, 1u);
              umma_f16(d, al, bh, args.idesc, 1u);
            }
          } else {
            const uint32_t b_addr = a_addr + A_BYTES;
#pragma unroll
            for (int kk = 0; kk < BK / 16; kk++)
              umma_f16(d, smem_desc_k128(a_addr + kk * 32), smem_desc_k128(b_addr + kk * 32), args.idesc,
                       (kt > 0 || kk > 0) ? 1u : 0u);
          }
          umma_commit(&empty[s]);
        }
        if (ok) umma_commit(&tfull[ab]);
      }
    }
  } else {
    // ---- epilogue warps 2..5: a warp reads TMEM lanes 32 * (warp % 4) ..
    const int q = warp & 3;
    const int row = q * 32 + lane;
    const bool leader = (warp == 2 && lane == 0);
    // operands were scaled by powers of two; undo exactly on the accumulator
    const float unscale = args.amax ? pow2_unscale(args.amax) : 1.f;
    long long chunk = 0;
    for (int i = 0;; i++) {
      const int ab = i & 1, u = i >> 1;
      if (!mbar_wait(&tfull[ab], (uint32_t)(u & 1), args.st, lim, 414) && lane == 0) atomicOr(&s_epi_fail, 1);
      // agree across the four warps before the warp-collective loads
      epi_bar();
      const bool ok = *(volatile int*)&s_epi_fail == 0;
      const int t = s_tiles[i & 7];
      if (!ok || t < 0) break;
      int tm, tn;
      grouped_tile(t, ntm, ntn, 16, tm, tn);
      tc_fence_after();
      for (int c = 0; c < BN / EPI_COLS; c++, chunk++) {
        uint32_t v[32];
        if (ok) tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(ab * 256 + c * EPI_COLS), v);
        if (c == BN / EPI_COLS - 1) {
          // all of this accumulator has been read: hand it back to the MMA warp
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&tempty[ab]);
        }
        if (leader) bulk_wait_read<1>();  // the box written two chunks ago has been read
        epi_bar();
        unsigned char* box = epi + (int)(chunk & 1) * EPI_BYTES;
        const int cols_left = args.N - (tn * BN + c * EPI_COLS);
#pragma unroll
        for (int j = 0; j < 8; j++) {
          float4 f = make_float4(-__uint_as_float(v[4 * j]) * unscale, -__uint_as_float(v[4 * j + 1]) * unscale,
                                 -__uint_as_float(v[4 * j + 2]) * unscale, -__uint_as_float(v[4 * j + 3]) * unscale);
          *reinterpret_cast<float4*>(box + row * 128 + ((j ^ (row & 7)) << 4)) = mask_cols(f, cols_left - 4 * j);
        }
        fence_proxy_async();
        epi_bar();
        if (leader && ok) {
          tma_reduce_add_2d(&mapC, box, args.c_col0 + tn * BN + c * EPI_COLS, args.c_row0 + tm * BM);
          bulk_commit();
        }
      }
      if (!ok) break;
    }
    if (leader) bulk_wait_all();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(P_TMEM_COLS) : "memory");
  }
}

// ---------------------------------------------------------------------------
// CTA-pair variant of the persistent pairs-layout kernel.  A cluster of two
// CTAs computes 256 x 256 tiles with tcgen05.mma.cta_group::2 (M = 256): each
// CTA holds its 128 rows of L and 128 of the tile's 256 U^T rows, and the
// MMA issued by the even CTA reads the U halves of both.  Per SM that is
// 64 KB of operands per 64-deep k block instead of 96 KB, so three stages
// fit beside the epilogue boxes.
//   even CTA: warp 0 loads its halves and expects the pair's bytes on its own
//             full barrier; warp 1 issues the MMAs and commits each stage and
//             accumulator to the barriers of both CTAs (commit multicast)
//   odd CTA:  warp 0 loads its halves, completing on the even CTA's full
//             barrier (cta_group::2 form of the load); warp 1 only holds TMEM
//   both:     warps 2-5, the epilogue of the CTA's own 128 rows; the
//             accumulator goes back to the even CTA's tempty barrier (8 warps)
// With a tile counter the even CTA draws each tile and stores it, tagged
// with its sequence number, into the odd CTA's shared memory.  No TMA load
// uses cluster multicast.
// ---------------------------------------------------------------------------
constexpr int Q_STAGES = 3;
constexpr int Q_A_BYTES = BM * BK * 2;                        // 16 KB: 128 L rows
constexpr int Q_B_BYTES = BN_BOX * BK * 2;                    // 16 KB: 128 U^T rows
constexpr int Q_STAGE_BYTES = 2 * Q_A_BYTES + 2 * Q_B_BYTES;  // Lh Ll Uh Ul
constexpr int Q_SMEM_BYTES = Q_STAGES * Q_STAGE_BYTES + 2 * EPI_BYTES + 1024 + 256;
static_assert(Q_SMEM_BYTES <= 227 * 1024, "CTA-pair layout exceeds shared memory");
static_assert(BN == 2 * BN_BOX, "each CTA of a pair loads one U box per part");

// kind::f16, FP16 x FP16 -> F32, both K-major, M = 256 (a CTA pair), N = 256
__host__ __device__ constexpr uint32_t make_idesc_pair() {
  return (1u << 4) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)((2 * BM) >> 4) << 24);
}

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// address of the same shared-memory location in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t cluster_addr(const void* p, uint32_t rank) {
  uint32_t d;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(d) : "r"(smem_u32(p)), "r"(rank));
  return d;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t caddr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(caddr) : "memory");
}
__device__ __forceinline__ void st_cluster_u64(uint32_t caddr, unsigned long long v) {
  asm volatile("st.relaxed.cluster.shared::cluster.u64 [%0], %1;" ::"r"(caddr), "l"(v) : "memory");
}
// TMA load into this CTA's shared memory whose completion is counted on an
// mbarrier of either CTA of the pair (no multicast)
__device__ __forceinline__ void tma_load_2d_pair(void* smem_dst, const CUtensorMap* map, uint32_t bar_caddr, int x,
                                                 int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, "
      "%4}], [%2];" ::"r"(smem_u32(smem_dst)),
      "l"(map), "r"(bar_caddr), "r"(x), "r"(y)
      : "memory");
}
__device__ __forceinline__ void umma_f16_pair(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                              uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
// arrive on the barrier at this offset in both CTAs once the MMAs issued so
// far have completed
__device__ __forceinline__ void umma_commit_pair(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
          smem_u32(bar)),
      "h"((unsigned short)3)
      : "memory");
}

// The odd CTA's view of tile i under a tile counter: the even CTA's store
// tagged i + 1.  Bounded wait; -1 (and the status set) on timeout.
__device__ __forceinline__ int forwarded_tile(volatile unsigned long long* fwd, int i, DevStatus* st, long long lim,
                                              int where) {
  long long n = 0;
  for (;;) {
    const unsigned long long v = fwd[i & 7];
    if ((unsigned)(v >> 32) == (unsigned)(i + 1)) return (int)(unsigned)(v & 0xffffffffu);
    if (++n > lim) {
      dev_fail(st, LU_ERR_TIMEOUT, where);
      return -1;
    }
  }
}

__global__ void __launch_bounds__(P_THREADS, 1)
gemm_lowp_pair_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                      const __grid_constant__ CUtensorMap mapC, Bf16GemmArgs args) {
  constexpr int NST = Q_STAGES, SB = Q_STAGE_BYTES;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* epi = smem + NST * SB;
  uint64_t* full = reinterpret_cast<uint64_t*>(epi + 2 * EPI_BYTES);  // used in the even CTA
  uint64_t* empty = full + NST;
  uint64_t* tfull = empty + NST;
  uint64_t* tempty = tfull + 2;  // used in the even CTA
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
  __shared__ int s_epi_fail;
  __shared__ volatile int s_epi_tile;  // the epilogue's current tile (-1: stop)
  // this CTA's i-th tile at entry i & 7 (-1 once there are no more); the
  // producer runs at most 2 tiles + one ring of k blocks ahead of the
  // epilogue, so an entry is read before it is reused
  __shared__ volatile int s_tiles[8];
  // odd CTA, tile counter: the even CTA's tiles, tagged (i + 1) << 32
  __shared__ volatile unsigned long long s_fwd[8];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t rank = cluster_rank();
  const bool even = rank == 0;
  const int ntm = (args.M + 2 * BM - 1) / (2 * BM), ntn = (args.N + BN - 1) / BN;
  const int tiles = ntm * ntn;
  const int KT = (args.K + BK - 1) / BK;
  const int pair = (int)blockIdx.x >> 1, npairs = (int)gridDim.x >> 1;
  const long long lim = args.spin >> 4;
  // tile i of this pair without a counter (the same in both CTAs)
  auto strided_tile = [&](int i) {
    const long long t = (long long)pair + (long long)i * npairs;
    return t < tiles ? (int)t : -1;
  };

  if (tid == 0) {
    prefetch_tmap(&mapA);
    prefetch_tmap(&mapB);
    prefetch_tmap(&mapC);
    for (int s = 0; s < NST; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 8);
    }
    for (int i = 0; i < 8; i++) s_fwd[i] = 0ull;
    fence_mbar_init();
    s_epi_fail = 0;
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(P_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  // both CTAs' barriers are initialised before any remote arrive or load
  cluster_sync_all();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {  // ---- TMA producer (both CTAs)
      long long kb = 0;
      bool ok = true;
      for (int i = 0; ok; i++) {
        int t;
        if (!args.tile_ctr) {
          t = strided_tile(i);
        } else if (even) {
          t = (int)atomicAdd(args.tile_ctr, 1u);
          if (t >= tiles) t = -1;
          st_cluster_u64(cluster_addr((const void*)&s_fwd[i & 7], 1),
                         ((unsigned long long)(unsigned)(i + 1) << 32) | (unsigned)t);
        } else {
          t = forwarded_tile(s_fwd, i, args.st, lim, 426);
        }
        s_tiles[i & 7] = t;
        __threadfence_block();
        if (t < 0) {
          if (even) {
            // no more tiles: complete the next stage's phase without data so
            // the MMA warp reads the end mark
            const int s = (int)(kb % NST);
            if (kb >= NST && !mbar_wait(&empty[s], (uint32_t)(((kb / NST) - 1) & 1), args.st, lim, 425)) {
              ok = false;
              break;
            }
            mbar_arrive(&full[s]);
          }
          break;
        }
        int tm, tn;
        grouped_tile(t, ntm, ntn, 8, tm, tn);
        const int arow = args.a_row0 + tm * 2 * BM + (int)rank * BM;
        const int brow = args.b_row0 + tn * BN + (int)rank * BN_BOX;
        for (int kt = 0; kt < KT; kt++, kb++) {
          const int s = (int)(kb % NST);
          if (kb >= NST && !mbar_wait(&empty[s], (uint32_t)(((kb / NST) - 1) & 1), args.st, lim, 421)) {
            ok = false;
            break;
          }
          unsigned char* sa = smem + s * SB;
          if (even) mbar_arrive_expect_tx(&full[s], 2 * SB);
          const uint32_t fb = cluster_addr(&full[s], 0);
          tma_load_2d_pair(sa, &mapA, fb, kt * BK, arow);
          tma_load_2d_pair(sa + Q_A_BYTES, &mapA, fb, args.kpart + kt * BK, arow);
          tma_load_2d_pair(sa + 2 * Q_A_BYTES, &mapB, fb, kt * BK, brow);
          tma_load_2d_pair(sa + 2 * Q_A_BYTES + Q_B_BYTES, &mapB, fb, args.kpart + kt * BK, brow);
        }
      }
      // the MMA warp's stage releases reach this CTA's empty barriers from
      // the even CTA: wait for the last ones before the CTA may exit
      if (ok)
        for (long long j = std::max(0LL, kb - NST); j < kb; j++)
          if (!mbar_wait(&empty[j % NST], (uint32_t)((j / NST) & 1), args.st, lim, 427)) break;
    }
  } else if (warp == 1) {
    if (even && lane == 0) {  // ---- MMA issuer (even CTA)
      const uint32_t idesc = make_idesc_pair();
      long long kb = 0;
      bool ok = true;
      int issued = 0;  // tiles whose accumulator was committed
      for (int i = 0; ok; i++) {
        const int ab = i & 1, u = i >> 1;
        if (u >= 1 && !mbar_wait(&tempty[ab], (uint32_t)((u - 1) & 1), args.st, lim, 422)) break;
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(ab * 256);
        for (int kt = 0; kt < KT; kt++, kb++) {
          const int s = (int)(kb % NST);
          if (!mbar_wait(&full[s], (uint32_t)((kb / NST) & 1), args.st, lim, 423)) {
            ok = false;
            break;
          }
          if (kt == 0 && s_tiles[i & 7] < 0) {  // end mark: pass it on to both epilogues
            mbar_arrive(&tfull[ab]);
            mbar_arrive_cluster(cluster_addr(&tfull[ab], 1));
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a_addr = smem_u32(smem + s * SB);
          const uint32_t al_addr = a_addr + Q_A_BYTES;
          const uint32_t bh_addr = a_addr + 2 * Q_A_BYTES;
          const uint32_t bl_addr = bh_addr + Q_B_BYTES;
#pragma unroll
          for (int kk = 0; kk < BK / 16; kk++) {
            const uint64_t ah = smem_desc_k128(a_addr + kk * 32), al = smem_desc_k128(al_addr + kk * 32);
            const uint64_t bh = smem_desc_k128(bh_addr + kk * 32), bl = smem_desc_k128(bl_addr + kk * 32);
            umma_f16_pair(d, ah, bh, idesc, (kt > 0 || kk > 0) ? 1u : 0u);
            umma_f16_pair(d, ah, bl, idesc, 1u);
            umma_f16_pair(d, al, bh, idesc, 1u);
          }
          umma_commit_pair(&empty[s]);
        }
        if (ok) {
          umma_commit_pair(&tfull[ab]);
          issued = i + 1;
        }
      }
      // both epilogues' releases of the last accumulators (some of them
      // remote arrivals) land before the CTA may exit
      for (int i = std::max(0, issued - 2); i < issued; i++)
        if (!mbar_wait(&tempty[i & 1], (uint32_t)((i >> 1) & 1), args.st, lim, 428)) break;
    }
  } else {
    // ---- epilogue warps 2..5: a warp reads TMEM lanes 32 * (warp % 4) ..
    const int q = warp & 3;
    const int row = q * 32 + lane;
    const bool leader = (warp == 2 && lane == 0);
    const float unscale = args.amax ? pow2_unscale(args.amax) : 1.f;
    long long chunk = 0;
    for (int i = 0;; i++) {
      const int ab = i & 1, u = i >> 1;
      if (!mbar_wait(&tfull[ab], (uint32_t)(u & 1), args.st, lim, 424) && lane == 0) atomicOr(&s_epi_fail, 1);
      // agree across the four warps before the warp-collective loads: one
      // thread reads the tile, all take it from shared memory
      epi_bar();
      if (leader) {
        int t0 = -1;
        if (*(volatile int*)&s_epi_fail == 0)
          t0 = !args.tile_ctr ? strided_tile(i) : (even ? s_tiles[i & 7] : forwarded_tile(s_fwd, i, args.st, lim, 429));
        s_epi_tile = t0;
      }
      epi_bar();
      const int t = s_epi_tile;
      if (t < 0) break;
      int tm, tn;
      grouped_tile(t, ntm, ntn, 8, tm, tn);
      const int crow = args.c_row0 + tm * 2 * BM + (int)rank * BM;
      // the odd CTA's half of the last tile row may lie wholly below M
      const bool rows_in = tm * 2 * BM + (int)rank * BM < args.M;
      tc_fence_after();
      for (int c = 0; c < BN / EPI_COLS; c++, chunk++) {
        uint32_t v[32];
        tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(ab * 256 + c * EPI_COLS), v);
        if (c == BN / EPI_COLS - 1) {
          // all of this accumulator has been read: hand it back to the MMA warp
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive_cluster(cluster_addr(&tempty[ab], 0));
        }
        if (leader) bulk_wait_read<1>();  // the box written two chunks ago has been read
        epi_bar();
        unsigned char* box = epi + (int)(chunk & 1) * EPI_BYTES;
        const int cols_left = args.N - (tn * BN + c * EPI_COLS);
#pragma unroll
        for (int j = 0; j < 8; j++) {
          float4 f = make_float4(-__uint_as_float(v[4 * j]) * unscale, -__uint_as_float(v[4 * j + 1]) * unscale,
                                 -__uint_as_float(v[4 * j + 2]) * unscale, -__uint_as_float(v[4 * j + 3]) * unscale);
          *reinterpret_cast<float4*>(box + row * 128 + ((j ^ (row & 7)) << 4)) = mask_cols(f, cols_left - 4 * j);
        }
        fence_proxy_async();
        epi_bar();
        if (leader && rows_in) {
          tma_reduce_add_2d(&mapC, box, args.c_col0 + tn * BN + c * EPI_COLS, crow);
          bulk_commit();
        }
      }
    }
    if (leader) bulk_wait_all();
  }
  tc_fence_before();
  __syncthreads();
  __syncwarp();
  // neither CTA leaves while the other may still address its shared memory
  cluster_sync_all();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(P_TMEM_COLS) : "memory");
  }
}

}  // namespace

int gemm_bf16_init() {
  LUB_CUDA(cudaFuncSetAttribute(gemm_bf16_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
  LUB_CUDA(cudaFuncSetAttribute(gemm_lowp_persistent_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                SMEM_BYTES));
  LUB_CUDA(cudaFuncSetAttribute(gemm_lowp_persistent_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                PAIR_SMEM_BYTES));
  LUB_CUDA(cudaFuncSetAttribute(gemm_lowp_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, Q_SMEM_BYTES));
  return LU_OK;
}

// Persistent launch: grid = min(tiles, max_ctas).  kpart > 0 selects the
// pairs layout: operand rows [hi (kpart) | lo (kpart)], K = kpart, a
// multiple of the 64-wide k block.  tile_ctr (zeroed before the first of
// the launches that share it) hands out tiles dynamically, so several
// launches of the same product, on different streams, split its tiles
// between them; null: each CTA strides over the tiles.
//
// cta_pair (pairs layout only) runs the CTA-pair kernel on 256 x 256 tiles:
// clusters of two CTAs, max_ctas rounded down to an even count (at least
// one pair).  All launches sharing a tile counter must use the same kernel.
int launch_gemm_lowp_persistent(const CUtensorMap& mapA, const CUtensorMap& mapB, const CUtensorMap& mapC,
                                int a_row0, int b_row0, int c_row0, int c_col0, int M, int N, int K, bool bf16,
                                const unsigned* amax, DevStatus* st, long long spin, int max_ctas, cudaStream_t s,
                                int kpart, unsigned* tile_ctr, bool cta_pair) {
  if (M <= 0 || N <= 0 || K <= 0) return LU_OK;
  if (c_col0 & 3) return LU_ERR_ALIGN;
  if (kpart > 0 && (kpart != K || (kpart % BK) || bf16)) return LU_ERR_ARG;
  if (cta_pair && kpart <= 0) return LU_ERR_ARG;
  Bf16GemmArgs a{a_row0, b_row0, c_row0, c_col0, M, N, K, make_idesc(bf16), amax, st, spin, kpart, tile_ctr};
  if (cta_pair) {
    const int64_t ptiles = (int64_t)ceil_div(N, BN) * ceil_div(M, 2 * BM);
    if (ptiles > INT32_MAX / 2) return LU_ERR_UNSUPPORTED;
    const int pairs = (int)std::max<int64_t>(1, std::min<int64_t>(ptiles, std::max(1, max_ctas / 2)));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * pairs, 1, 1);
    cfg.blockDim = dim3(P_THREADS, 1, 1);
    cfg.dynamicSmemBytes = Q_SMEM_BYTES;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    LUB_CUDA(cudaLaunchKernelEx(&cfg, gemm_lowp_pair_kernel, mapA, mapB, mapC, a));
    LUB_LAUNCH_CHECK();
    return LU_OK;
  }
  const int64_t tiles = (int64_t)ceil_div(N, BN) * ceil_div(M, BM);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, std::max(1, max_ctas)));
  if (kpart > 0)
    gemm_lowp_persistent_kernel<true><<<grid, P_THREADS, PAIR_SMEM_BYTES, s>>>(mapA, mapB, mapC, a);
  else
    gemm_lowp_persistent_kernel<false><<<grid, P_THREADS, SMEM_BYTES, s>>>(mapA, mapB, mapC, a);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

// mapA: BF16 L (rows >= a_row0 + M, cols K), box 64 x 128, SW128
// mapB: BF16 U^T (rows >= b_row0 + N, cols K), box 64 x 128, SW128
// mapC: FP32 C matrix, box 32 x 128, SW128 (reduce-add target)
int launch_gemm_bf16_tc(const CUtensorMap& mapA, const CUtensorMap& mapB, const CUtensorMap& mapC, int a_row0,
                        int b_row0, int c_row0, int c_col0, int M, int N, int K, bool bf16, const unsigned* amax,
                        DevStatus* st, long long spin, cudaStream_t s) {
  if (M <= 0 || N <= 0 || K <= 0) return LU_OK;
  if (c_col0 & 3) return LU_ERR_ALIGN;  // TMA x coordinate * 4 bytes must be a multiple of 16
  Bf16GemmArgs a{a_row0, b_row0, c_row0, c_col0, M, N, K, make_idesc(bf16), amax, st, spin, 0, nullptr};
  const int64_t tiles = (int64_t)ceil_div(N, BN) * ceil_div(M, BM);
  if (tiles > INT32_MAX) return LU_ERR_UNSUPPORTED;
  gemm_bf16_tc_kernel<<<(unsigned)tiles, THREADS, SMEM_BYTES, s>>>(mapA, mapB, mapC, a);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

}  // namespace lub

// ---------------------------------------------------------------------------
// Test hook (not part of include/lu_b200.h): C -= lowp(A) * lowp(B) for FP32
// row-major A (M x K), B (K x N), C (M x N), through the same split/scale
// casts, tensor maps and kernel the mixed factorisation uses.  mode 0: BF16;
// 1: FP16 with power-of-two panel scaling; 2: error-compensated FP16 (hi/lo
// split, three products).  Allocates its own temporaries; used only by the
// GPU unit test of the tcgen05 kernel.
// ---------------------------------------------------------------------------
extern "C" __attribute__((visibility("default"))) int lub_test_gemm_lowp(const float* A, int64_t lda, const float* B,
                                                                         int64_t ldb, float* C, int64_t ldc, int M,
                                                                         int N, int K, int mode, void* stream) {
  using namespace lub;
  cudaStream_t s = (cudaStream_t)stream;
  // mode bits 0-7: 0 bf16, 1 scaled fp16, 2 split fp16 x3 (concatenated
  // parts), 3 split fp16 x3 in the pairs layout (persistent kernel only);
  // bits 8-15: CTA count of the persistent kernel (0: one CTA per tile);
  // bits 16-23: CTA count of a second persistent launch on another stream,
  // the two sharing a tile counter (dynamic tiles); bit 24: the CTA-pair
  // kernel (pairs layout)
  const int pctas = (mode >> 8) & 0xff, hctas = (mode >> 16) & 0xff;
  const bool cta_pair = ((mode >> 24) & 1) != 0;
  mode &= 0xff;
  if (cta_pair && mode != 3) return LU_ERR_ARG;
  if (M <= 0 || N <= 0 || K <= 0 || mode < 0 || mode > 3 || (ldc & 3) || (reinterpret_cast<uintptr_t>(C) & 15))
    return LU_ERR_ARG;
  if ((mode == 3 || hctas > 0) && pctas <= 0) return LU_ERR_ARG;
  LUB_TRY(gemm_bf16_init());
  const bool pairs = mode == 3;
  const int nparts = mode == 2 ? 3 : (pairs ? 2 : 1);
  const int kps = (K + 63) & ~63;
  const int Ke = pairs ? 2 * kps : nparts * K;  // tensor-map width
  const int Kg = pairs ? kps : Ke;               // GEMM k extent
  const int64_t ldk = (Ke + 63) & ~int64_t(63);
  __nv_bfloat16 *Lb = nullptr, *Ub = nullptr;
  LUB_CUDA(cudaMalloc(&Lb, sizeof(__nv_bfloat16) * M * ldk));
  LUB_CUDA(cudaMalloc(&Ub, sizeof(__nv_bfloat16) * N * ldk));
  DevStatus* st = nullptr;
  LUB_CUDA(cudaMalloc(&st, sizeof(DevStatus) + 32));
  unsigned* amax = reinterpret_cast<unsigned*>(st + 1);
  unsigned* ctr = amax + 4;
  LUB_CUDA(cudaMemsetAsync(st, 0, sizeof(DevStatus) + 32, s));
  int rc = LU_OK;
  const bool bf16 = mode == 0;
  if (bf16) {
    rc = launch_split_rows<__nv_bfloat16>(A, lda, Lb, ldk, M, K, 1, 0u, nullptr, 0, s);
    if (rc == LU_OK) rc = launch_split_transpose<__nv_bfloat16>(B, ldb, Ub, ldk, K, N, 1, 0u, nullptr, 1, s);
  } else {
    rc = launch_panel_absmax(A, lda, M, K, B, ldb, N, amax, s);
    const unsigned lmask = pairs ? 0x2u : 0x4u;
    if (rc == LU_OK)
      rc = launch_split_rows<__half>(A, lda, reinterpret_cast<__half*>(Lb), ldk, M, K, nparts, lmask, amax, 0, s,
                                     pairs ? kps : 0);
    if (rc == LU_OK)
      rc = launch_split_transpose<__half>(B, ldb, reinterpret_cast<__half*>(Ub), ldk, K, N, nparts, 0x2u, amax, 1,
                                          s, pairs ? kps : 0);
  }
  const CUtensorMapDataType dt = bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
  CUtensorMap mL, mU, mC;
  if (rc == LU_OK) rc = encode_tmap_2d(&mL, dt, 2, Lb, Ke, M, ldk * 2, 64, 128, CU_TENSOR_MAP_SWIZZLE_128B);
  if (rc == LU_OK) rc = encode_tmap_2d(&mU, dt, 2, Ub, Ke, N, ldk * 2, 64, 128, CU_TENSOR_MAP_SWIZZLE_128B);
  if (rc == LU_OK)
    rc = encode_tmap_2d(&mC, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, C, N, M, ldc * 4, 32, 128, CU_TENSOR_MAP_SWIZZLE_128B);
  if (rc == LU_OK && hctas > 0) {
    cudaStream_t s2 = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    LUB_CUDA(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
    LUB_CUDA(cudaEventCreateWithFlags(&e0, cudaEventDisableTiming));
    LUB_CUDA(cudaEventCreateWithFlags(&e1, cudaEventDisableTiming));
    LUB_CUDA(cudaEventRecord(e0, s));
    LUB_CUDA(cudaStreamWaitEvent(s2, e0, 0));
    rc = launch_gemm_lowp_persistent(mL, mU, mC, 0, 0, 0, 0, M, N, Kg, bf16, bf16 ? nullptr : amax, st, 1LL << 24,
                                     pctas, s, pairs ? kps : 0, ctr, cta_pair);
    if (rc == LU_OK)
      rc = launch_gemm_lowp_persistent(mL, mU, mC, 0, 0, 0, 0, M, N, Kg, bf16, bf16 ? nullptr : amax, st,
                                       1LL << 24, hctas, s2, pairs ? kps : 0, ctr, cta_pair);
    LUB_CUDA(cudaEventRecord(e1, s2));
    LUB_CUDA(cudaStreamWaitEvent(s, e1, 0));
    LUB_CUDA(cudaStreamSynchronize(s));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s2);
  } else if (rc == LU_OK && pctas > 0)
    rc = launch_gemm_lowp_persistent(mL, mU, mC, 0, 0, 0, 0, M, N, Kg, bf16, bf16 ? nullptr : amax, st, 1LL << 24,
                                     pctas, s, pairs ? kps : 0, nullptr, cta_pair);
  else if (rc == LU_OK)
    rc = launch_gemm_bf16_tc(mL, mU, mC, 0, 0, 0, 0, M, N, Ke, bf16, bf16 ? nullptr : amax, st, 1LL << 24, s);
  DevStatus hst{};
  cudaMemcpyAsync(&hst, st, sizeof(hst), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  cudaFree(Lb);
  cudaFree(Ub);
  cudaFree(st);
  if (rc != LU_OK) return rc;
  return hst.code;
}
