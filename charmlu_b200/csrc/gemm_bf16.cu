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
//   warp 0, one lane : TMA producer — A box 64 x 128 and B box 64 x 256 per
//                      k-block of 64, 128-byte swizzle, into a 3-stage ring
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
// block starts 32 bytes further.  No cluster launch and no multicast.
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
      tma_load_2d(sa + A_BYTES, &mapB, &full[s], kt * BK, args.b_row0 + tile_n);
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
            tma_load_2d(sa + 2 * A_BYTES, &mapB, &full[s], kt * BK, args.b_row0 + tn * BN);
            tma_load_2d(sa + 2 * A_BYTES + B_BYTES, &mapB, &full[s], args.kpart + kt * BK, args.b_row0 + tn * BN);
          } else {
            tma_load_2d(sa, &mapA, &full[s], kt * BK, args.a_row0 + tm * BM);
            tma_load_2d(sa + A_BYTES, &mapB, &full[s], kt * BK, args.b_row0 + tn * BN);
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

}  // namespace

int gemm_bf16_init() {
  LUB_CUDA(cudaFuncSetAttribute(gemm_bf16_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
  LUB_CUDA(cudaFuncSetAttribute(gemm_lowp_persistent_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                SMEM_BYTES));
  LUB_CUDA(cudaFuncSetAttribute(gemm_lowp_persistent_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                PAIR_SMEM_BYTES));
  return LU_OK;
}

// Persistent launch: grid = min(tiles, max_ctas).  kpart > 0 selects the
// pairs layout: operand rows [hi (kpart) | lo (kpart)], K = kpart, a
// multiple of the 64-wide k block.  tile_ctr (zeroed before the first of
// the launches that share it) hands out tiles dynamically, so several
// launches of the same product, on different streams, split its tiles
// between them; null: each CTA strides over the tiles.
int launch_gemm_lowp_persistent(const CUtensorMap& mapA, const CUtensorMap& mapB, const CUtensorMap& mapC,
                                int a_row0, int b_row0, int c_row0, int c_col0, int M, int N, int K, bool bf16,
                                const unsigned* amax, DevStatus* st, long long spin, int max_ctas, cudaStream_t s,
                                int kpart, unsigned* tile_ctr) {
  if (M <= 0 || N <= 0 || K <= 0) return LU_OK;
  if (c_col0 & 3) return LU_ERR_ALIGN;
  if (kpart > 0 && (kpart != K || (kpart % BK) || bf16)) return LU_ERR_ARG;
  Bf16GemmArgs a{a_row0, b_row0, c_row0, c_col0, M, N, K, make_idesc(bf16), amax, st, spin, kpart, tile_ctr};
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
// mapB: BF16 U^T (rows >= b_row0 + N, cols K), box 64 x 256, SW128
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
  // the two sharing a tile counter (dynamic tiles)
  const int pctas = (mode >> 8) & 0xff, hctas = (mode >> 16) & 0xff;
  mode &= 0xff;
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
  if (rc == LU_OK) rc = encode_tmap_2d(&mU, dt, 2, Ub, Ke, N, ldk * 2, 64, 256, CU_TENSOR_MAP_SWIZZLE_128B);
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
                                     pctas, s, pairs ? kps : 0, ctr);
    if (rc == LU_OK)
      rc = launch_gemm_lowp_persistent(mL, mU, mC, 0, 0, 0, 0, M, N, Kg, bf16, bf16 ? nullptr : amax, st,
                                       1LL << 24, hctas, s2, pairs ? kps : 0, ctr);
    LUB_CUDA(cudaEventRecord(e1, s2));
    LUB_CUDA(cudaStreamWaitEvent(s, e1, 0));
    LUB_CUDA(cudaStreamSynchronize(s));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s2);
  } else if (rc == LU_OK && pctas > 0)
    rc = launch_gemm_lowp_persistent(mL, mU, mC, 0, 0, 0, 0, M, N, Kg, bf16, bf16 ? nullptr : amax, st, 1LL << 24,
                                     pctas, s, pairs ? kps : 0);
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
