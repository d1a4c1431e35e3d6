// lu_solve_noalloc: the solve of lu_solve (one right-hand side, trans = 0)
// for callers that cannot allocate device memory.
//
// Who needs it: callers that may not allocate device memory.  A plugin
// inside a host application that owns all device memory through its own
// allocator and hands the library a fixed budget up front; a real-time loop
// that cannot afford cudaMalloc/cudaFree, which may synchronise the whole
// device; and a caller that has no solver handle (lu_create allocates the
// handle's workspace).  This entry point allocates nothing: its only scratch
// (the substitution pipeline's ready flags, its ticket counter and a status
// word) lives in the file-scope device array below, which every GPU that
// loads this library holds until the process exits (about 8 KB).  The
// caller passes the factors, pivots, right-hand side and an optional status
// output.
//
// Set-up: the first call on each device looks up the array's device address
// with cudaGetSymbolAddress (with that device current) and caches it; make
// that first call before any stream capture.  The cached address belongs to
// the device's context at that time: after cudaDeviceReset (or any other end
// of the primary context) it is stale, so a process that resets a device
// must not call this entry point on it again.  Host code must not hand the
// array's name to a kernel: on the host it is only a stand-in, not a device
// address.
//
// Sharing: every call on a device uses the same array; each call clears the
// parts that must start at zero (flags, ticket, status) on its stream
// before use.  Calls that overlap on the GPU (different streams, no
// ordering) race on the array and give wrong results or timeouts.
#include <mutex>

#include "common.cuh"
#include "kernels.h"

namespace lub {
namespace {

constexpr int kNoAllocMaxN = 1 << 17;             // largest order accepted (131072)
constexpr int kNoAllocBlocks = kNoAllocMaxN / 64;  // 64-row substitution blocks
// ints: [0, 4) DevStatus, [4] ticket, [8, 8 + blocks + 2) ready flags
constexpr int kNoAllocInts = 8 + kNoAllocBlocks + 2;

static __device__ __align__(256) int g_noalloc_scratch[kNoAllocInts];

std::mutex g_noalloc_mu;
int* g_noalloc_ptr[64] = {nullptr};

// Device address of the scratch array on the current device (looked up
// once per device).
int noalloc_scratch(int** out) {
  int dev = 0;
  LUB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return LU_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    LUB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_ptr[dev] = static_cast<int*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return LU_OK;
}

__global__ void noalloc_status_kernel(const DevStatus* st, int32_t* out) {
  *out = st->code != 0 ? st->code : st->info;
}

}  // namespace
}  // namespace lub

// x <- A^{-1} b from lu_factor's factors (dLU, row-major, lda) and pivots;
// db (n doubles, device) is overwritten by x.  d_status (optional, device)
// receives LU_OK or LU_ERR_TIMEOUT when the stream reaches it.  Returns
// LU_ERR_ARG for n > 131072 or bad pointers, without launching anything.
extern "C" LU_API int lu_solve_noalloc(const double* dLU, int64_t lda, int64_t n, const int32_t* ipiv, double* db,
                                       int32_t* d_status, void* stream) {
  using namespace lub;
  if (!dLU || !ipiv || !db || n <= 0 || lda < n) return LU_ERR_ARG;
  if (n > kNoAllocMaxN) {
    fprintf(stderr, "[lu_b200] lu_solve_noalloc: n = %lld exceeds the fixed scratch limit %d\n", (long long)n,
            kNoAllocMaxN);
    return LU_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  int* base = nullptr;
  LUB_TRY(noalloc_scratch(&base));
  DevStatus* st = reinterpret_cast<DevStatus*>(base);
  unsigned* ticket = reinterpret_cast<unsigned*>(base + 4);
  int* flags = base + 8;
  const long long spin = 1LL << 24;
  LUB_CUDA(cudaMemsetAsync(st, 0, sizeof(DevStatus), s));
  LUB_TRY(launch_ipiv_apply_vector(ipiv, (int)n, db, s));
  // launch_trsv clears the flags and the ticket on the stream before each launch
  LUB_TRY(launch_trsv<double>(dLU, lda, (int)n, db, 0, flags, ticket, st, spin, s));
  LUB_TRY(launch_trsv<double>(dLU, lda, (int)n, db, 1, flags, ticket, st, spin, s));
  if (d_status) {
    noalloc_status_kernel<<<1, 1, 0, s>>>(st, d_status);
    LUB_LAUNCH_CHECK();
  }
  return LU_OK;
}
