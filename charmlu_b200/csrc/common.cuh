// Shared device/host helpers for the charmlu_b200 kernels (sm_100a only).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <algorithm>
#include <mutex>

#include "../../include/lu_b200.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "charmlu_b200 kernels target sm_100a only"
#endif

namespace lub {

// Runs f() once per device (the one current when called) for each
// PerDeviceOnce object and caches its status: kernel attributes such as the
// dynamic shared-memory limit are per-device state, so one process that
// drives several GPUs must set them on each.
struct PerDeviceOnce {
  std::mutex mu;
  bool done[64] = {};
  int status[64] = {};
};
template <class F>
inline int once_per_device(PerDeviceOnce& o, F&& f) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return LU_ERR_CUDA;
  if (dev < 0 || dev >= 64) return LU_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(o.mu);
  if (!o.done[dev]) {
    o.status[dev] = f();
    o.done[dev] = true;
  }
  return o.status[dev];
}
inline int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return LU_OK;
  cudaGetLastError();
  return LU_ERR_CUDA;
}

constexpr int kNumSMsB200 = 148;

// ---------------------------------------------------------------------------
// Host error plumbing
// ---------------------------------------------------------------------------
#define LUB_CUDA(expr)                                                          \
  do {                                                                          \
    cudaError_t _e = (expr);                                                    \
    if (_e != cudaSuccess) {                                                    \
      fprintf(stderr, "[lu_b200] %s:%d %s -> %s\n", __FILE__, __LINE__, #expr,  \
              cudaGetErrorString(_e));                                          \
      return LU_ERR_CUDA;                                                       \
    }                                                                           \
  } while (0)

// Count of kernels this library has launched (reported by lu_launch_count).
extern long long g_kernel_launches;

#define LUB_LAUNCH_CHECK()                                                      \
  do {                                                                          \
    __atomic_add_fetch(&::lub::g_kernel_launches, 1, __ATOMIC_RELAXED);         \
    cudaError_t _e = cudaGetLastError();                                        \
    if (_e != cudaSuccess) {                                                    \
      fprintf(stderr, "[lu_b200] %s:%d launch -> %s\n", __FILE__, __LINE__,     \
              cudaGetErrorString(_e));                                          \
      return LU_ERR_CUDA;                                                       \
    }                                                                           \
  } while (0)

#define LUB_TRY(expr)                 \
  do {                                \
    int _s = (expr);                  \
    if (_s != LU_OK) return _s;       \
  } while (0)

// ---------------------------------------------------------------------------
// Device status word: first error wins.  Kernels never trap; a bounded wait
// that gives up records LU_ERR_TIMEOUT here and returns.
// ---------------------------------------------------------------------------
struct DevStatus {
  int code;        // LU_OK or LU_ERR_* (first non-zero recorded)
  int info;        // 1-based first singular column (min over reports), 0 if none
  int where;       // diagnostic tag of the first timeout
  int pad;
};

__device__ __forceinline__ void dev_fail(DevStatus* st, int code, int where) {
  if (atomicCAS(&st->code, 0, code) == 0) st->where = where;
}
__device__ __forceinline__ void dev_singular(DevStatus* st, int col1) {
  // info = min over reported columns (0 = none yet)
  int old = st->info;
  while ((old == 0 || col1 < old)) {
    int prev = atomicCAS(&st->info, old, col1);
    if (prev == old) break;
    old = prev;
  }
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_acquire_s32(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void red_release_add_u32(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_release_s32(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid-wide barrier on a dedicated counter (zeroed before the launch): the
// n-th call waits until the counter reaches n * nblocks.  Bounded: returns
// false after spin_limit polls (status set), or when another block already
// failed.
__device__ __forceinline__ bool grid_barrier(unsigned* counter, unsigned target, DevStatus* st,
                                             long long spin_limit, int where) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    red_release_add_u32(counter, 1u);
    long long polls = 0;
    while (ld_acquire_u32(counter) < target) {
      if (++polls > spin_limit) { dev_fail(st, LU_ERR_TIMEOUT, where); ok = 0; break; }
      if ((polls & 255) == 0 && ld_acquire_s32(&st->code) != 0) { ok = 0; break; }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Grouped raster over an ntm x ntn tile grid: blocks run down groups of
// `group` tile-rows before moving right, so the CTAs resident at one time
// share a few A row-panels and B column-panels in L2 instead of streaming
// the whole B operand once per tile-row.
__device__ __forceinline__ void grouped_tile(int bid, int ntm, int ntn, int group, int& tm, int& tn) {
  const int per_group = group * ntn;
  const int g = bid / per_group;
  const int first = g * group;
  const int gs = min(ntm - first, group);
  const int r = bid - g * per_group;
  tm = first + r % gs;
  tn = r / gs;
}

// ---------------------------------------------------------------------------
// Counter-based generator (SplitMix64 finaliser); identical to the oracle's.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z ^= z >> 30; z *= 0xbf58476d1ce4e5b9ULL;
  z ^= z >> 27; z *= 0x94d049bb133111ebULL;
  z ^= z >> 31; return z;
}
__host__ __device__ __forceinline__ uint64_t stream_key(uint64_t seed, uint64_t stream) {
  return mix64(seed ^ (stream * 0xD1B54A32D192ED03ULL));
}
__host__ __device__ __forceinline__ double uniform_at(uint64_t key, uint64_t i) {
  uint64_t z = mix64(key + (i + 1) * 0x9E3779B97F4A7C15ULL);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0) - 0.5;
}

// Power-of-two operand scaling for FP16 tensor-core operands: a panel whose
// largest magnitude is m is multiplied by 2^(13 - floor(log2 m)), which puts
// its largest entry in [2^13, 2^14) (FP16 max 65504) and keeps the low parts
// of a hi/lo split in the normal range.  amax holds float bit patterns.
__host__ __device__ __forceinline__ float pow2_scale_of(float m) {
  if (!(m > 0.f) || !(m < 3.0e38f)) return 1.f;
  int e;
  frexpf(m, &e);  // m = f * 2^e, f in [0.5, 1)  ->  floor(log2 m) = e - 1
  return ldexpf(1.f, 13 - (e - 1));
}
__device__ __forceinline__ float pow2_unscale(const unsigned* amax) {
  return 1.f / (pow2_scale_of(__uint_as_float(amax[0])) * pow2_scale_of(__uint_as_float(amax[1])));
}

// ---------------------------------------------------------------------------
// mbarrier + TMA (cp.async.bulk.tensor) wrappers.  No cluster multicast is
// used anywhere in this library.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait on an mbarrier phase; false on timeout (status recorded).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, DevStatus* st, long long limit,
                                          int where) {
  long long n = 0;
  while (!mbar_try_wait(bar, parity)) {
    if (++n > limit) { dev_fail(st, LU_ERR_TIMEOUT, where); return false; }
  }
  return true;
}
__device__ __forceinline__ void tma_load_2d(void* smem_dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
      ::"r"(smem_u32(smem_dst)), "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}
__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
}

// ---------------------------------------------------------------------------
// Host: cuTensorMapEncodeTiled through the runtime's driver entry point (no
// link-time dependency on libcuda).
// ---------------------------------------------------------------------------
int encode_tmap_2d(CUtensorMap* map, CUtensorMapDataType dtype, int elem_bytes, const void* base,
                   uint64_t cols, uint64_t rows, uint64_t row_pitch_bytes, uint32_t box_cols,
                   uint32_t box_rows, CUtensorMapSwizzle swizzle);

inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

}  // namespace lub
