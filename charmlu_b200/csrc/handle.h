// Internal: the solver handle, phase profiler and tensor-mapped matrices
// shared by the FP64 and mixed-precision orchestration.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <algorithm>
#include <cstring>
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
  cudaEvent_t evR = nullptr;  // split look-ahead: the rest's operands are built
  // mixed look-ahead: interchanges, U solve and operands of the next panel's
  // columns first, the rest after the panel has started (LU_B200_LA_SPLIT)
  int la_split = 1;  // mixed look-ahead: the next panel's columns first, then the rest
  // leaf tuning: recursion leaf width and CTA cap, without / with look-ahead
  int leaf_w64 = 32, leaf_w32 = 64, leaf_ctas = 148;
  int leaf_w64_la = 16, leaf_w32_la = 32, leaf_ctas_la = 48;
  // low-precision trailing update: CTAs of the persistent kernel (0: one CTA
  // per tile); under look-ahead the update beside a running panel leaves
  // gemm_reserve SMs to it
  // (B200, N = 65536, FP16x3 with look-ahead: 48 SMs reserved and a 48-CTA
  // leaf measured best)
  int gemm_ctas = 148, gemm_reserve = 48;
  int gemm_helper = 1;  // look-ahead: reserved SMs join the update once the panel is done
  int gemm_pair = 1;    // pairs layout on CTA pairs (tcgen05 cta_group::2, 256 x 256 tiles)
  // mixed path: FP32 panel leaves of width <= 32 by tournament pivoting
  // (no grid-wide synchronisation per column) when 1; partial pivoting by
  // default (LU_B200_TSLU=1 selects the tournament: about as fast, see
  // tslu.cu, and its refinement contraction varies with the row blocks)
  int tslu = 0;
  // mixed path: the panels' inner TRSMs (w <= 256) as one blocked launch
  // instead of the recursion (LU_B200_TRSM_BLOCK=0 restores the recursion)
  int trsm_block = 1;
  int trsm_wide = 1;  // mixed U block-row solves (w <= 512, > trsm_wide_min columns) in one launch with inverted diagonal blocks
  int trsm_wide_min = 512;
  lub::TsluScratch tslu_scr{};
  // FP16x3 mixed path: the recursive FP32 panel's GEMM halves of width >= 128
  // on the tcgen05 kernel, with their own split-operand buffers (the panel
  // runs beside the trailing update, which owns Lb/Ub/amax)
  int panel_tc = 0;
  __half* Lp = nullptr;
  __half* Up = nullptr;
  unsigned* amaxP = nullptr;
  int64_t ldkP = 0;
  int32_t* perm = nullptr;
  int32_t* perm_work = nullptr;
  int32_t* perm_lists = nullptr;  // composed pivot batches (ipiv -> perm)
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
  float* dinv32 = nullptr;     // inverses of the 32 x 32 diagonal blocks of a panel's L11 (wide U solve)
  int64_t ld32 = 0;
  __nv_bfloat16* Lb = nullptr; // BF16 L21 panel, n x ldk (K-major)
  __nv_bfloat16* Ub = nullptr; // BF16 U12^T panel, n x ldk (K-major)
  int64_t ldk = 0;
  int32_t* ipiv32 = nullptr;   // pivots of the low-precision factorisation
  unsigned* amax = nullptr;    // per-panel |L|max, |U|max (scaled FP16 operands)
  int nparts = 1;              // 3 for the error-compensated FP16 split (2 in the pairs layout)
  bool pairs = false;          // FP16x3 operands as [hi | lo] for the persistent update
  float* v32 = nullptr;        // FP32 work vector (solves)
  double* r64 = nullptr;       // FP64 residual
  double* z64 = nullptr;       // FP64 work vector (GMRES)
  double* zero64 = nullptr;    // zeros (A v products through the residual kernel)
  double* V = nullptr;         // GMRES Arnoldi basis, (gm+1) vectors of n (allocated on first use)
  double* Z = nullptr;         // flexible GMRES: the preconditioned basis M^{-1} v_j, gm vectors of n
  double* hdot = nullptr;      // GMRES dot-product partials / results
  int gm = 0;                  // GMRES restart length
  double* xbest = nullptr;     // refinement: the iterate with the smallest ||b - A x||inf so far
  double* rbest = nullptr;     //   and its residual
  lub::ResidualAccum* racc_best = nullptr;  //   and its norms
  bool mixed_ready = false;
  // factors kept for lu_refine_apply / lu_refine_adjoint
  bool mixed_factored = false;
  int32_t* perm32 = nullptr;   // row permutation of those factors
  // multi-RHS refinement work blocks (ld 16), allocated on first use
  double* mr_P = nullptr;      // residual partials, kMultiMaxSplits * n * 16
  double* mr_Pn = nullptr;     // row-norm partials, kMultiMaxSplits * n
  double* mr_R = nullptr;      // residual block
  double* mr_D = nullptr;      // correction block
  double* mr_X = nullptr;      // iterate
  double* mr_S = nullptr;      // GMRES: operand staging block (column 0 only)
  double* mr_T = nullptr;      // GMRES: product block
  double* mr_dc = nullptr;     // GMRES: correction of one column
  double* mr_Xbest = nullptr;  // per column: the iterate with the smallest residual so far
  double* mr_Rbest = nullptr;  //   and its residual
  unsigned long long* mr_acc = nullptr;
  // host-resident FP64 A (lu_refine_solve_host): row chunks staged through
  // two device buffers, copies on sCopy overlapping the kernels on the
  // caller's stream
  double* stage[2] = {nullptr, nullptr};
  int64_t stage_elems = 0;
  size_t stage_bytes = size_t(256) << 20;  // per buffer
  cudaStream_t sCopy = nullptr;
  cudaEvent_t evReady[2] = {nullptr, nullptr}, evFree[2] = {nullptr, nullptr};
  // leading rows of the host matrix kept in device memory (as many as free
  // memory allows, at most resident_cap bytes): the conversion pass of every
  // call copies them there, and each later pass over A (residuals, GMRES
  // products) streams only rows res_rows .. n-1
  double* resA = nullptr;
  int64_t res_elems = 0;
  int res_rows = 0;
  size_t resident_cap = ~size_t(0);
  int64_t host_copied = 0;  // bytes of host A copied to the device, running total
  std::vector<void*> allocs;
  size_t bytes = 0;
  long long spin = 0;
  // CUDA-graph replay of factorisation schedules (cfg.use_graph)
  struct GraphSlot {
    const void* k1 = nullptr;
    const void* k2 = nullptr;
    const void* k3 = nullptr;
    int64_t k4 = 0;
    cudaGraphExec_t exec = nullptr;
    long long kernels = 0;  // kernel nodes per replay (added to the launch count)
  };
  GraphSlot gslot[2];            // 0: FP64 factor, 1: mixed factor
  cudaStream_t sG = nullptr;     // capture / replay stream
  cudaEvent_t evG0 = nullptr, evG1 = nullptr;
  bool capturing = false;
  // kernel nodes the panel stream added during a capture: a captured kernel
  // node does not keep its stream's priority, so run_graph gives them the
  // panel stream's (highest) priority before instantiating the graph
  std::vector<cudaGraphNode_t> prio_nodes;
  int prio_hi = 0;
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
  void release(void* p) {
    if (!p) return;
    cudaFree(p);
    allocs.erase(std::remove(allocs.begin(), allocs.end(), p), allocs.end());
  }
  unsigned* take_counter() {
    if (next_counter >= n_counters) return nullptr;
    return counters + next_counter++;
  }
};


namespace lub {

// The capture dependencies of stream s at this point of a capture.
inline int capture_deps(cudaStream_t s, std::vector<cudaGraphNode_t>* out) {
  cudaStreamCaptureStatus cs;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  LUB_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, nullptr, &deps, &nd));
  out->assign(deps, deps + nd);
  return LU_OK;
}

// During a capture: the kernel nodes stream s appended since its capture
// dependencies were `before` (every node reachable backwards from its
// current dependencies without passing a node of `before`) join
// h->prio_nodes.
inline int mark_branch_priority(lu_handle h, cudaStream_t s, const std::vector<cudaGraphNode_t>& before) {
  std::vector<cudaGraphNode_t> todo, seen(before);
  LUB_TRY(capture_deps(s, &todo));
  while (!todo.empty()) {
    cudaGraphNode_t nd = todo.back();
    todo.pop_back();
    if (std::find(seen.begin(), seen.end(), nd) != seen.end()) continue;
    seen.push_back(nd);
    cudaGraphNodeType t;
    LUB_CUDA(cudaGraphNodeGetType(nd, &t));
    if (t == cudaGraphNodeTypeKernel) h->prio_nodes.push_back(nd);
    size_t np = 0;
    LUB_CUDA(cudaGraphNodeGetDependencies(nd, nullptr, &np));
    std::vector<cudaGraphNode_t> pred(np);
    if (np) LUB_CUDA(cudaGraphNodeGetDependencies(nd, pred.data(), &np));
    for (auto p : pred) todo.push_back(p);
  }
  return LU_OK;
}

// Brackets one phase with events when the handle is profiling.
struct Prof {
  lu_handle h;
  cudaStream_t s;
  int ph;
  double fl;
  cudaEvent_t a = nullptr;
  Prof(lu_handle h_, cudaStream_t s_, int ph_, double fl_ = 0.0) : h(h_), s(s_), ph(ph_), fl(fl_) {
    if (h->profile && !h->capturing) {
      a = h->take_event();
      cudaEventRecord(a, s);
    }
  }
  ~Prof() {
    if (a) {
      cudaEvent_t b = h->take_event();
      cudaEventRecord(b, s);
      h->recs.push_back({ph, a, b, fl});
    }
  }
};

// Run body(stream) as a CUDA graph keyed by (k1..k4): replay the cached graph
// when the keys match, otherwise capture body on the handle's capture stream
// (forked from and joined back to s by events), instantiate and launch.
// Without use_graph, body runs directly on s.
template <typename F>
int run_graph(lu_handle h, int slot, const void* k1, const void* k2, const void* k3, int64_t k4, cudaStream_t s,
              F&& body) {
  if (!h->cfg.use_graph) return body(s);
  auto& g = h->gslot[slot];
  LUB_CUDA(cudaEventRecord(h->evG0, s));
  LUB_CUDA(cudaStreamWaitEvent(h->sG, h->evG0, 0));
  if (!(g.exec && g.k1 == k1 && g.k2 == k2 && g.k3 == k3 && g.k4 == k4)) {
    if (g.exec) {
      cudaGraphExecDestroy(g.exec);
      g.exec = nullptr;
    }
    LUB_CUDA(cudaStreamBeginCapture(h->sG, cudaStreamCaptureModeThreadLocal));
    h->capturing = true;
    h->prio_nodes.clear();
    const long long before = __atomic_load_n(&g_kernel_launches, __ATOMIC_RELAXED);
    const int rc = body(h->sG);
    // captured, not launched: the replays below count them
    __atomic_store_n(&g_kernel_launches, before, __ATOMIC_RELAXED);
    h->capturing = false;
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->sG, &graph);
    if (rc != LU_OK) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    LUB_CUDA(e);
    for (auto nd : h->prio_nodes) {
      cudaKernelNodeAttrValue v;
      memset(&v, 0, sizeof(v));
      v.priority = h->prio_hi;
      if (cudaGraphKernelNodeSetAttribute(nd, cudaKernelNodeAttributePriority, &v) != cudaSuccess) {
        cudaGraphDestroy(graph);
        h->prio_nodes.clear();
        return LU_ERR_CUDA;
      }
    }
    h->prio_nodes.clear();
    size_t nn = 0;
    cudaGraphGetNodes(graph, nullptr, &nn);
    std::vector<cudaGraphNode_t> nodes(nn);
    if (nn) cudaGraphGetNodes(graph, nodes.data(), &nn);
    g.kernels = 0;
    for (auto nd : nodes) {
      cudaGraphNodeType t;
      if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) g.kernels++;
    }
    const cudaError_t ei = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    LUB_CUDA(ei);
    g.k1 = k1;
    g.k2 = k2;
    g.k3 = k3;
    g.k4 = k4;
  }
  LUB_CUDA(cudaGraphLaunch(g.exec, h->sG));
  __atomic_add_fetch(&g_kernel_launches, g.kernels, __ATOMIC_RELAXED);
  LUB_CUDA(cudaEventRecord(h->evG1, h->sG));
  LUB_CUDA(cudaStreamWaitEvent(s, h->evG1, 0));
  return LU_OK;
}

}  // namespace lub
