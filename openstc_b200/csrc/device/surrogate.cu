// Chemistry surrogate: BF16 tensor-core GEMM (tcgen05) and its entry points.
#include <cuda_runtime.h>

#include <string>

#include "engine.hpp"
#include "openstc_b200.h"
#include "tc_gemm.cuh"

namespace ostc {

template <int BN>
static cudaError_t launch_gemm_bn(const uint16_t *A, int lda, const uint16_t *B, int ldb, float *D, int ldd, int M,
                                  int N, int K, int splits, int *err, cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(k_tc_gemm<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(GemmTile<BN>::smem));
  if (e != cudaSuccess) return e;
  const int per = (K + splits - 1) / splits;
  const int kps = (per + kGemmBK - 1) / kGemmBK * kGemmBK;
  const dim3 grid((M + 127) / 128, (N + BN - 1) / BN, splits);
  k_tc_gemm<BN><<<grid, 128, GemmTile<BN>::smem, st>>>(A, lda, B, ldb, D, ldd, M, N, K, kps, err);
  return cudaGetLastError();
}

// D = A * B^T on the tensor cores; with splits > 1, D holds `splits`
// consecutive partial results of M x ldd each.
cudaError_t tc_gemm(const uint16_t *A, int lda, const uint16_t *B, int ldb, float *D, int ldd, int M, int N, int K,
                    int splits, int *err, cudaStream_t st) {
  if (N <= 16) return launch_gemm_bn<16>(A, lda, B, ldb, D, ldd, M, N, K, splits, err, st);
  if (N <= 32) return launch_gemm_bn<32>(A, lda, B, ldb, D, ldd, M, N, K, splits, err, st);
  if (N <= 64) return launch_gemm_bn<64>(A, lda, B, ldb, D, ldd, M, N, K, splits, err, st);
  if (N <= 128) return launch_gemm_bn<128>(A, lda, B, ldb, D, ldd, M, N, K, splits, err, st);
  return launch_gemm_bn<256>(A, lda, B, ldb, D, ldd, M, N, K, splits, err, st);
}

}  // namespace ostc

extern "C" int ostc_tc_gemm_bf16(const void *A, int lda, const void *B, int ldb, float *D, int ldd, int M, int N,
                                 int K, int splits, int *err, void *stream) {
  if (!A || !B || !D || !err || M <= 0 || N <= 0 || K <= 0 || splits <= 0)
    return ostc::abi_error(OSTC_ERR_INPUT, "ostc_tc_gemm_bf16: null pointer or non-positive size");
  if (K % 8 || lda % 8 || ldb % 8 || lda < K || ldb < K || ldd < N)
    return ostc::abi_error(OSTC_ERR_INPUT, "ostc_tc_gemm_bf16: K, lda and ldb must be multiples of 8, lda/ldb >= K, ldd >= N");
  const cudaError_t e = ostc::tc_gemm(static_cast<const uint16_t *>(A), lda, static_cast<const uint16_t *>(B), ldb, D,
                                      ldd, M, N, K, splits, err, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return ostc::abi_error(OSTC_ERR_CUDA, std::string("ostc_tc_gemm_bf16: ") + cudaGetErrorString(e));
  return OSTC_OK;
}
