// Internal: the solver handle, phase profiler and tensor-mapped matrices
// shared by the FP64 and mixed-precision orchestration.
#pragma once
#include <cuda_bf16.h>
#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace lub {

// A row-major FP64 matrix with the two tensor maps the GEMM reads it by.
struct MatF64 {
  double* p = nullptr;
  int64_t ld = 0, rows = 0, cols = 0;
  CUtensorMap mapA, mapB;  // boxes 16x128 and 16x16, 128-byte swizzle
  int init(double* ptr, int64_t r, int64_t c, int64_t ldd) {
    p = ptr; rows = r; cols = c; ld = ldd;
    LUB_TRY(encode_tmap_2d(&mapA, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, ptr, c, r, ld * 8, 16, 128,
                           CU_TENSOR_MAP_SWIZZLE_128B));
    LUB_TRY(encode_tmap_2d(&mapB, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, ptr, c, r, ld * 8, 16, 16,
                           CU_TENSOR_MAP_SWIZZLE_128B));
    return LU_OK;
  }
  double* at(int64_t r, int64_t c) const { return p + r * ld + c; }
};

int ensure_kernels_init();

}  // namespace lub

using lub::DevStatus;

struct lu_handle_s {
  lu_config cfg;
  int device = 0;
  int num_sms = 148;
  // workspace (device)
  DevStatus* st = nullptr;
  unsigned* counters = nullptr;
  int n_counters = 0;
  int next_counter = 0;
  lub::LeafScratch<double> leaf64{};
  lub::LeafScratch<float> leaf32{};
  lub::PivotList plist{};      // pivot lists of the trailing stream
  lub::PivotList plistP{};     // pivot lists of the panel stream (look-ahead)
  cudaStream_t sP = nullptr;   // high-priority panel stream (look-ahead)
  cudaEvent_t evFork = nullptr, evP = nullptr, evN = nullptr;
  // leaf tuning: recursion leaf width and CTA cap, without / with look-ahead
  int leaf_w64 = 32, leaf_w32 = 64, leaf_ctas = 148;
  int leaf_w64_la = 16, leaf_w32_la = 32, leaf_ctas_la = 64;
  int32_t* perm = nullptr;
  int32_t* perm_work = nullptr;
  int* trsv_flags = nullptr;
  unsigned* trsv_ticket = nullptr;
  double* vec = nullptr;
  double* vec2 = nullptr;
  double* tmpB = nullptr;      // n x nrhs staging block of multi-RHS solves (grown on demand)
  size_t tmpB_elems = 0;
  lub::ResidualAccum* racc = nullptr;
  lub::ResidualAccum* racc_host = nullptr;
  // mixed-precision workspace (allocated on first use)
  float* A32 = nullptr;        // FP32 working copy, n x ld32
  int64_t ld32 = 0;
  __nv_bfloat16* Lb = nullptr; // BF16 L21 panel, n x ldk (K-major)
  __nv_bfloat16* Ub = nullptr; // BF16 U12^T panel, n x ldk (K-major)
  int64_t ldk = 0;
  int32_t* ipiv32 = nullptr;   // pivots of the low-precision factorisation
  unsigned* amax = nullptr;    // per-panel |L|max, |U|max (scaled FP16 operands)
  int nparts = 1;              // 3 for the error-compensated FP16 split
  float* v32 = nullptr;        // FP32 work vector (solves)
  double* r64 = nullptr;       // FP64 residual
  double* z64 = nullptr;       // FP64 work vector (GMRES)
  double* zero64 = nullptr;    // zeros (A v products through the residual kernel)
  double* V = nullptr;         // GMRES basis, (gm+1) vectors of n
  double* hdot = nullptr;      // GMRES dot-product partials / results
  int gm = 0;                  // GMRES restart length
  bool mixed_ready = false;
  std::vector<void*> allocs;
  size_t bytes = 0;
  long long spin = 0;
  // phase profiling (events on the launching stream)
  int profile = 0;
  struct Rec {
    int phase;
    cudaEvent_t a, b;
    double flops;
  };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  size_t pool_used = 0;
  cudaEvent_t take_event() {
    if (pool_used == pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      pool.push_back(e);
    }
    return pool[pool_used++];
  }

  template <typename T>
  int alloc(T** p, size_t count) {
    void* q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(count * sizeof(T), 16)) != cudaSuccess) {
      cudaGetLastError();
      return LU_ERR_NOMEM;
    }
    allocs.push_back(q);
    bytes += count * sizeof(T);
    *p = static_cast<T*>(q);
    return LU_OK;
  }
  unsigned* take_counter() {
    if (next_counter >= n_counters) return nullptr;
    return counters + next_counter++;
  }
};


namespace lub {

// Brackets one phase with events when the handle is profiling.
struct Prof {
  lu_handle h;
  cudaStream_t s;
  int ph;
  double fl;
  cudaEvent_t a = nullptr;
  Prof(lu_handle h_, cudaStream_t s_, int ph_, double fl_ = 0.0) : h(h_), s(s_), ph(ph_), fl(fl_) {
    if (h->profile) {
      a = h->take_event();
      cudaEventRecord(a, s);
    }
  }
  ~Prof() {
    if (h->profile) {
      cudaEvent_t b = h->take_event();
      cudaEventRecord(b, s);
      h->recs.push_back({ph, a, b, fl});
    }
  }
};

}  // namespace lub
