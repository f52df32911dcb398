// BF16 GEMM on the tcgen05 tensor cores with FP32 accumulation in tensor
// memory:  D[M x N] = A[M x K] * B[N x K]^T  (A, B row-major with K
// contiguous, D row-major FP32).  One CTA of 128 threads computes a 128 x BN
// tile over a K range (split-K along grid.z writes one partial D per split).
// K is consumed in 64-wide chunks (one 128-byte swizzled row per tile row)
// through two shared-memory stages: while the tensor cores work on one stage
// the threads fill the other.
#pragma once

#include "tc_mma.cuh"

namespace ostc {

constexpr int kGemmBK = 64;

template <int BN>
struct GemmTile {
  static constexpr uint32_t a_bytes = 128 * kGemmBK * 2;
  static constexpr uint32_t b_bytes = BN * kGemmBK * 2;
  static constexpr uint32_t stage = a_bytes + b_bytes;
  static constexpr uint32_t smem = 2 * stage + 64 + 1024;  // + alignment slack
  static constexpr uint32_t tcols = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
};

// Copy rows [r0, r0 + R) x columns [k0, k0 + 64) of a row-major bf16 matrix
// into a canonical K-major tile; rows >= rows_valid and columns >= k_end are
// zero.  k_end and ld are multiples of 8.
template <int R>
__device__ __forceinline__ void load_tile(uint8_t *dst, const uint16_t *src, int ld, int r0, int rows_valid,
                                          int k0, int k_end) {
  for (int q = threadIdx.x; q < R * 8; q += blockDim.x) {
    const int r = q >> 3, c = q & 7, kk = k0 + c * 8;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (r0 + r < rows_valid && kk < k_end)
      v = __ldg(reinterpret_cast<const uint4 *>(src + static_cast<size_t>(r0 + r) * ld + kk));
    *reinterpret_cast<uint4 *>(dst + tc::sw128_offset(r, c * 8)) = v;
  }
}

template <int BN>
__global__ void __launch_bounds__(128) k_tc_gemm(const uint16_t *__restrict__ A, int lda,
                                                 const uint16_t *__restrict__ B, int ldb, float *__restrict__ D,
                                                 int ldd, int M, int N, int K, int k_per_split, int *err) {
  using T = GemmTile<BN>;
  extern __shared__ __align__(128) uint8_t smem_raw[];
  // swizzled tiles need 1024-byte aligned bases
  uint8_t *smem = smem_raw + ((1024 - (tc::smem_u32(smem_raw) & 1023)) & 1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * 128, n0 = blockIdx.y * BN;
  const int ks = blockIdx.z * k_per_split, ke = min(K, ks + k_per_split);
  float *Dz = D + static_cast<size_t>(blockIdx.z) * M * ldd;
  uint8_t *stage[2] = {smem, smem + T::stage};
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + 2 * T::stage);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 2);
  if (warp == 0) tc::tmem_alloc(tslot, T::tcols);
  if (tid == 0) {
    tc::mbar_init(&bar[0], 1);
    tc::mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;
  const int nchunks = ke > ks ? (ke - ks + kGemmBK - 1) / kGemmBK : 0;
  uint32_t phase[2] = {0, 0};
  bool ok = true;
  for (int c = 0; c < nchunks; ++c) {
    const int s = c & 1;
    if (c >= 2) {
      // the MMAs of chunk c - 2 read this stage
      ok = tc::mbar_wait(&bar[s], phase[s]);
      phase[s] ^= 1;
      ok = __syncthreads_and(ok);
      if (!ok) break;
    }
    const int k0 = ks + c * kGemmBK;
    load_tile<128>(stage[s], A, lda, m0, M, k0, ke);
    load_tile<BN>(stage[s] + T::a_bytes, B, ldb, n0, N, k0, ke);
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      const uint32_t abase = tc::smem_u32(stage[s]), bbase = abase + T::a_bytes;
      const int ksteps = (min(kGemmBK, ke - k0) + 15) / 16;
      for (int q = 0; q < ksteps; ++q) {
        const uint64_t ad = tc::desc_sw128(abase + q * 32);
        const uint64_t bd = tc::desc_sw128(bbase + q * 32);
        tc::mma_bf16(tmem, ad, bd, tc::idesc_bf16(128, BN), (c > 0 || q > 0) ? 1u : 0u);
      }
      tc::commit(&bar[s]);
    }
  }
  if (ok && nchunks > 0) {
    const int s = (nchunks - 1) & 1;
    ok = tc::mbar_wait(&bar[s], phase[s]);
  }
  ok = __syncthreads_and(ok);
  tc::fence_after_sync();
  const int row = m0 + warp * 32 + lane;
  if (ok) {
    for (int c0 = 0; c0 < BN; c0 += 32) {
      float v[32];
      if (nchunks > 0) {
        tc::tmem_ld32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + c0, v);
      } else {
#pragma unroll
        for (int q = 0; q < 32; ++q) v[q] = 0.f;
      }
      if (row < M) {
#pragma unroll
        for (int q = 0; q < 32; ++q) {
          const int col = n0 + c0 + q;
          if (c0 + q < BN && col < N) Dz[static_cast<size_t>(row) * ldd + col] = v[q];
        }
      }
    }
  } else if (tid == 0) {
    atomicExch(err, 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, T::tcols);
}

}  // namespace ostc
