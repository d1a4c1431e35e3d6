// FP32 C -= A * B (row-major, any M, N, K) for the GEMM halves of the
// mixed-precision path's recursive FP32 panel and TRSM.  The mixed path keeps
// its panel and triangular solves in FP32 (only the trailing update drops to
// BF16 tensor cores), so these run on the FP32 SIMT pipe.
//
// Tiling: CTA 128 x 128, K-tile 16, 256 threads with a 16 x 4 register
// block each (outer products from shared memory): warp w owns rows
// 16 w .. 16 w + 15 and lane l columns 4 l .. 4 l + 3, so per k the A values
// are warp-wide broadcasts (four float4 loads, one wavefront each) and the B
// values one float4 per lane.  The A tile is stored k-major in shared memory.
// Tiles are double-buffered through registers; edges are zero-filled on load.
#include "common.cuh"
#include "kernels.h"

namespace lub {
namespace {

constexpr int BM = 128, BN = 128, BK = 16, THREADS = 256;

__global__ void __launch_bounds__(THREADS, 2)
gemm_f32_sub_kernel(const float* __restrict__ A, int64_t lda, const float* __restrict__ B, int64_t ldb,
                    float* __restrict__ C, int64_t ldc, int M, int N, int K) {
  __shared__ __align__(16) float As[2][BK][BM + 4];
  __shared__ __align__(16) float Bs[2][BK][BN + 4];
  const int tid = threadIdx.x;
  const int tm = blockIdx.y * BM, tn = blockIdx.x * BN;
  const int tx = tid & 31, ty = tid >> 5;  // 32 column groups x 8 row groups, 16 x 4 each

  // loader mapping: A tile 128 x 16 -> each thread 8 elements (rows ar, ar+64; k ak..ak+3)
  const int ar = tid >> 2, ak = (tid & 3) * 4;
  // B tile 16 x 128 -> each thread 8 elements (k rows bk, bk+8; cols bn..bn+3)
  const int bk = tid >> 5, bn = (tid & 31) * 4;

  float ra[2][4], rb[2][4];
  auto load = [&](int k0) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int r = tm + ar + h * 64;
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int k = k0 + ak + e;
        ra[h][e] = (r < M && k < K) ? __ldg(&A[(int64_t)r * lda + k]) : 0.f;
      }
      const int kb = k0 + bk + h * 8;
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int c = tn + bn + e;
        rb[h][e] = (kb < K && c < N) ? __ldg(&B[(int64_t)kb * ldb + c]) : 0.f;
      }
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
#pragma unroll
      for (int e = 0; e < 4; e++) As[buf][ak + e][ar + h * 64] = ra[h][e];
      *reinterpret_cast<float4*>(&Bs[buf][bk + h * 8][bn]) = make_float4(rb[h][0], rb[h][1], rb[h][2], rb[h][3]);
    }
  };

  float acc[16][4];
#pragma unroll
  for (int i = 0; i < 16; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = 0.f;

  const int KT = (K + BK - 1) / BK;
  load(0);
  store(0);
  __syncthreads();
  for (int kt = 0; kt < KT; kt++) {
    const int buf = kt & 1;
    if (kt + 1 < KT) load((kt + 1) * BK);
#pragma unroll
    for (int k = 0; k < BK; k++) {
      float av[16];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const float4 a = *reinterpret_cast<const float4*>(&As[buf][k][ty * 16 + q * 4]);
        av[4 * q] = a.x; av[4 * q + 1] = a.y; av[4 * q + 2] = a.z; av[4 * q + 3] = a.w;
      }
      const float4 b = *reinterpret_cast<const float4*>(&Bs[buf][k][tx * 4]);
      const float bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
      for (int i = 0; i < 16; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
    if (kt + 1 < KT) {
      store(buf ^ 1);
      __syncthreads();
    }
  }
  // C -= acc (rows ty*16 + i, cols tx*4 + j: a warp's row is 128 contiguous floats)
#pragma unroll
  for (int i = 0; i < 16; i++) {
    const int r = tm + ty * 16 + i;
    if (r >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int c = tn + tx * 4 + j;
      if (c < N) C[(int64_t)r * ldc + c] -= acc[i][j];
    }
  }
}

// Narrow products (N <= BN <= 64, K <= 64: the deep halves of the recursive
// panel and TRSM): the whole K x N operand B and a 64-row slice of A sit in
// shared memory, and each thread keeps a (64 / row groups) x 4 block of C.
// These launches are bound by the M x K and M x N traffic, which the 128 x
// 128 tile above would spend mostly on zero-filled columns.  Each element is
// accumulated over k in the same order and subtracted once, as above, so
// both kernels give the same bits.
constexpr int NBM = 64, NKMAX = 64, NTHREADS = 256;

template <int BN>
__global__ void __launch_bounds__(NTHREADS)
gemm_f32_narrow_kernel(const float* __restrict__ A, int64_t lda, const float* __restrict__ B, int64_t ldb,
                       float* __restrict__ C, int64_t ldc, int M, int N, int K) {
  constexpr int QN = BN / 4;           // column quads
  constexpr int RG = NTHREADS / QN;    // row groups
  constexpr int RPT = NBM / RG;        // rows per thread
  __shared__ __align__(16) float Bs[NKMAX][BN];
  __shared__ float As[NBM][NKMAX + 1];
  const int tid = threadIdx.x;
  const int tx = tid % QN, ty = tid / QN;
  const int row0 = blockIdx.x * NBM;
  for (int idx = tid; idx < K * BN; idx += NTHREADS) {
    const int k = idx / BN, c = idx - k * BN;
    Bs[k][c] = c < N ? __ldg(&B[(int64_t)k * ldb + c]) : 0.f;
  }
  for (int idx = tid; idx < NBM * K; idx += NTHREADS) {
    const int r = idx / K, k = idx - r * K;
    As[r][k] = row0 + r < M ? __ldg(&A[(int64_t)(row0 + r) * lda + k]) : 0.f;
  }
  __syncthreads();
  float acc[RPT][4];
#pragma unroll
  for (int i = 0; i < RPT; i++)
#pragma unroll
    for (int e = 0; e < 4; e++) acc[i][e] = 0.f;
  for (int k = 0; k < K; k++) {
    const float4 b = *reinterpret_cast<const float4*>(&Bs[k][tx * 4]);
#pragma unroll
    for (int i = 0; i < RPT; i++) {
      const float a = As[ty + i * RG][k];
      acc[i][0] = fmaf(a, b.x, acc[i][0]);
      acc[i][1] = fmaf(a, b.y, acc[i][1]);
      acc[i][2] = fmaf(a, b.z, acc[i][2]);
      acc[i][3] = fmaf(a, b.w, acc[i][3]);
    }
  }
#pragma unroll
  for (int i = 0; i < RPT; i++) {
    const int r = row0 + ty + i * RG;
    if (r >= M) continue;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int c = tx * 4 + e;
      if (c < N) C[(int64_t)r * ldc + c] -= acc[i][e];
    }
  }
}

}  // namespace

static int gemm_f32_dispatch(const float* A, int64_t lda, const float* B, int64_t ldb, float* C, int64_t ldc, int M,
                             int N, int K, bool allow_narrow, cudaStream_t s) {
  if (M <= 0 || N <= 0 || K <= 0) return LU_OK;
  if (allow_narrow && K <= NKMAX && N <= 64) {
    if (N <= 32)
      gemm_f32_narrow_kernel<32><<<ceil_div(M, NBM), NTHREADS, 0, s>>>(A, lda, B, ldb, C, ldc, M, N, K);
    else
      gemm_f32_narrow_kernel<64><<<ceil_div(M, NBM), NTHREADS, 0, s>>>(A, lda, B, ldb, C, ldc, M, N, K);
    LUB_LAUNCH_CHECK();
    return LU_OK;
  }
  dim3 grid(ceil_div(N, BN), ceil_div(M, BM));
  gemm_f32_sub_kernel<<<grid, THREADS, 0, s>>>(A, lda, B, ldb, C, ldc, M, N, K);
  LUB_LAUNCH_CHECK();
  return LU_OK;
}

int launch_gemm_f32_sub(const float* A, int64_t lda, const float* B, int64_t ldb, float* C, int64_t ldc, int M,
                        int N, int K, cudaStream_t s) {
  return gemm_f32_dispatch(A, lda, B, ldb, C, ldc, M, N, K, true, s);
}

}  // namespace lub

// Test hook (not part of the ABI): C -= A B through the FP32 panel GEMM,
// the narrow kernel where the shape allows it unless wide_only is set.
extern "C" __attribute__((visibility("default"))) int lub_test_gemm_f32(const float* A, int64_t lda, const float* B,
                                                                      int64_t ldb, float* C, int64_t ldc, int M,
                                                                      int N, int K, int wide_only, void* stream) {
  return lub::gemm_f32_dispatch(A, lda, B, ldb, C, ldc, M, N, K, wide_only == 0, (cudaStream_t)stream);
}
