// Device side of the chemistry surrogate shared by the solver engine and the
// training code: the FP64 EPI increment (the label generator and the
// fallback), the decoding / element projection / trust gate of the network
// output, and the fused tcgen05 inference kernel that applies the increments
// to the conserved species of every cell.
#pragma once

#include <cuda_bf16.h>

#include "kernels_step.cuh"
#include "surrogate.hpp"
#include "tc_mma.cuh"

namespace ostc {
namespace sur {

// One FP64 EPI step at fixed density: rho dY = (I - dt J)^-1 dt omega, with
// omega and J as the solver computes them (finite_rate_chemistry and
// compute_chem_src_jacobian, src/FiniteRateChem.cu:7-194; EPI, :211-234).
template <int NS>
__device__ inline void epi_increment(double T, double rho, const double *Y, double dt, double *q1, double *q2,
                                     int stride, double *dy) {
  double omega[NS], omega_d[NS];
  chemistry<NS>(rho, T, Y, omega, omega_d, q1, q2, stride);
  double lhs[NS * NS];
  const int nr = cP.nr;
  for (int m = 0; m < NS; ++m) {
    for (int q = 0; q < NS; ++q) {
      double zz = 0;
      if (Y[q] > 1e-25) {
        for (int r = 0; r < nr; ++r) {
          const int dn = cP.sb[r * NS + m] - cP.sf[r * NS + m];
          if (dn == 0) continue;
          zz += dn * (cP.sf[r * NS + q] * q1[r * stride] - cP.sb[r * NS + q] * q2[r * stride]);
        }
        zz /= rho * Y[q];
      }
      const double J = cP.mw[m] * zz * 1e+3;
      lhs[m * NS + q] = (m == q ? 1.0 : 0.0) - dt * J;
    }
  }
  int piv[NS];
  lu_factor<NS>(lhs, piv);
  double x[NS];
  for (int k = 0; k < NS; ++k) x[k] = omega[k];
  lu_solve<NS>(lhs, piv, x);
  for (int k = 0; k < NS; ++k) dy[k] = dt * x[k] / rho;
}

// GELU in its tanh form; the hardware tanh in inference, tanhf in training.
__device__ __forceinline__ float gelu_tanh_fast(float x) {
  const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
  float t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
  return 0.5f * x * (1.f + t);
}

// Network output o (normalised, bias added) -> dY_k = (Y_k + eps) c_k
// sinh(s_k o_k); the increment is then projected onto element conservation
// (weighted least squares, weights |dY_k| + 1e-3 Y_k).  The cell is accepted
// when the inputs lie in the training box, every output is within
// gate.out_max, the raw element defect is below gate.defect_tol of the
// element totals, no increment exceeds gate.rel_max (Y_k + eps), and no mass
// fraction is driven below -1e-9: the network is trusted where the chemistry
// changes the composition little, the EPI step takes the reacting cells.
template <int NS>
__device__ inline bool decode(const SurrogateDev &p, const float *o, double T, double lp, double ldt, const double *Y,
                              double *dy) {
  const SurrogateGate &g = p.gate;
  bool ok = T >= g.t_min && T <= g.t_max && lp >= g.lp_min && lp <= g.lp_max && ldt >= g.ldt_min && ldt <= g.ldt_max;
  for (int k = 0; k < NS; ++k) {
    const double ok_k = fabs(o[k]) <= g.out_max;
    ok = ok && ok_k;
    const double oc = fmin(fmax(static_cast<double>(o[k]), -static_cast<double>(g.out_max)), static_cast<double>(g.out_max));
    dy[k] = (Y[k] + kSurYEps) * p.out_c[k] * sinh(oc * p.out_s[k]);
    if (fabs(dy[k]) > g.rel_max * (Y[k] + kSurYEps)) ok = false;
  }
  const int ne = p.n_elem;
  double r[kMaxElem], M[kMaxElem * kMaxElem], w[NS];
  for (int k = 0; k < NS; ++k) w[k] = fabs(dy[k]) + 1e-3 * Y[k] + 1e-30;
  for (int e = 0; e < ne; ++e) {
    double defect = 0, total = 0;
    for (int k = 0; k < NS; ++k) {
      defect += p.elem[e * kMaxSpec + k] * dy[k];
      total += p.elem[e * kMaxSpec + k] * Y[k];
    }
    r[e] = defect;
    if (total > 0 && fabs(defect) > g.defect_tol * total) ok = false;
    for (int f = 0; f < ne; ++f) {
      double s = 0;
      for (int k = 0; k < NS; ++k) s += p.elem[e * kMaxSpec + k] * w[k] * p.elem[f * kMaxSpec + k];
      M[e * kMaxElem + f] = s;
    }
  }
  // lambda = M^-1 r (Gauss-Jordan, partial pivoting; ne <= 8)
  for (int c = 0; c < ne; ++c) {
    int piv = c;
    for (int q = c + 1; q < ne; ++q)
      if (fabs(M[q * kMaxElem + c]) > fabs(M[piv * kMaxElem + c])) piv = q;
    if (fabs(M[piv * kMaxElem + c]) < 1e-300) continue;
    if (piv != c) {
      for (int q = 0; q < ne; ++q) {
        const double t = M[c * kMaxElem + q];
        M[c * kMaxElem + q] = M[piv * kMaxElem + q];
        M[piv * kMaxElem + q] = t;
      }
      const double t = r[c];
      r[c] = r[piv];
      r[piv] = t;
    }
    const double inv = 1.0 / M[c * kMaxElem + c];
    for (int q = 0; q < ne; ++q) {
      if (q == c) continue;
      const double f = M[q * kMaxElem + c] * inv;
      for (int z = 0; z < ne; ++z) M[q * kMaxElem + z] -= f * M[c * kMaxElem + z];
      r[q] -= f * r[c];
    }
    r[c] *= inv;
    for (int z = 0; z < ne; ++z) M[c * kMaxElem + z] *= inv;
  }
  for (int k = 0; k < NS; ++k) {
    double corr = 0;
    for (int e = 0; e < ne; ++e) corr += p.elem[e * kMaxSpec + k] * r[e];
    dy[k] -= w[k] * corr;
    if (Y[k] + dy[k] < -1e-9) ok = false;
  }
  return ok;
}

// ------------------------------------------------------------ fused kernel
constexpr int kThreads = 256;  // 8 warps: 2 per TMEM lane quarter
constexpr int kChunk = 32;     // K columns of a weight stage
constexpr uint32_t kA0Bytes = 128 * kSurInPad * 2;
constexpr uint32_t kA1Bytes = 128 * kSurHidden * 2;
constexpr uint32_t kStageBytes = kSurHidden * kChunk * 2;
constexpr uint32_t kSmem = kA0Bytes + kA1Bytes + 2 * kStageBytes + 64;

// 16-byte chunks of a packed weight block into shared memory
__device__ __forceinline__ void copy_bytes(uint8_t *dst, const uint8_t *src, uint32_t bytes) {
  for (uint32_t q = threadIdx.x * 16; q < bytes; q += kThreads * 16)
    *reinterpret_cast<uint4 *>(dst + q) = __ldg(reinterpret_cast<const uint4 *>(src + q));
}

struct Phases {
  uint32_t ph[3] = {0, 0, 0};
};

// Waits for the commit on bar[i]; false on timeout (all threads agree).
__device__ __forceinline__ bool wait_bar(uint64_t *bar, int i, Phases &P) {
  const bool ok = tc::mbar_wait(&bar[i], P.ph[i]);
  P.ph[i] ^= 1;
  return __syncthreads_and(ok) != 0;
}

// Epilogue of a hidden layer: accumulator + bias -> GELU -> bf16 rows of the
// next layer's input tile (K-major canonical, 256 columns).
__device__ __forceinline__ void hidden_epilogue(uint32_t tmem, const float *bias, uint8_t *a1) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = (warp & 3) * 32 + lane, half = warp >> 2;
  for (int c0 = half * 128; c0 < half * 128 + 128; c0 += 32) {
    float v[32];
    tc::tmem_ld32(tmem + (static_cast<uint32_t>((warp & 3) * 32) << 16) + c0, v);
#pragma unroll
    for (int q = 0; q < 32; q += 8) {
      uint32_t pk[4];
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const float x0 = gelu_tanh_fast(v[q + 2 * h] + __ldg(bias + c0 + q + 2 * h));
        const float x1 = gelu_tanh_fast(v[q + 2 * h + 1] + __ldg(bias + c0 + q + 2 * h + 1));
        const __nv_bfloat162 b2 = __floats2bfloat162_rn(x0, x1);
        pk[h] = *reinterpret_cast<const uint32_t *>(&b2);
      }
      *reinterpret_cast<uint4 *>(a1 + tc::tile_offset(row, c0 + q, kSurHidden)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
  }
}

// One 128-cell tile per CTA: features -> 4 x (256, GELU) -> 9 outputs on the
// tensor cores, then decode, project and gate, with dt = the cell's local
// time step.  mode 1 (in the step, before the source term): accepted cells
// are marked chemically quiet and get the rate rho dY / dt, the others keep
// the point-implicit chemistry.  mode 0 (a split step): accepted increments
// go into cv (rho Y_k) with the primitives recomputed, rejected cells are
// listed for the EPI fallback.  stats[0] += accepted, stats[1] += rejected.
template <class C>
__global__ void __launch_bounds__(kThreads) k_sur_infer(const DevBlock *__restrict__ blks, int b, SurrogateDev P,
                                                        int mode, int *fb_count, int *fb_list,
                                                        unsigned long long *stats, int *err) {
  constexpr int NS = C::ns;
  extern __shared__ __align__(128) uint8_t smem[];
  uint8_t *a0 = smem, *a1 = smem + kA0Bytes;
  uint8_t *stage[2] = {a1 + kA1Bytes, a1 + kA1Bytes + kStageBytes};
  uint64_t *bar = reinterpret_cast<uint64_t *>(stage[1] + kStageBytes);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 3);
  const DevBlock &B = blks[b];
  const int tid = threadIdx.x, warp = tid >> 5;
  const int64_t cells = static_cast<int64_t>(B.mx) * B.my * B.mz;
  const int64_t sz = B.G.size;

  // features of this tile's cells (one thread per row)
  if (tid < 128) {
    const int64_t c = static_cast<int64_t>(blockIdx.x) * 128 + tid;
    float f[kSurInPad];
#pragma unroll
    for (int q = 0; q < kSurInPad; ++q) f[q] = 0.f;
    if (c < cells) {
      const int i = static_cast<int>(c % B.mx), j = static_cast<int>((c / B.mx) % B.my),
                k = static_cast<int>(c / (static_cast<int64_t>(B.mx) * B.my));
      const int64_t n = B.G.at(i, j, k);
      float raw[kSurIn];
      raw[0] = static_cast<float>(B.bv[5 * sz + n]);
      raw[1] = static_cast<float>(log10(B.bv[4 * sz + n]));
      for (int s = 0; s < NS; ++s) raw[2 + s] = static_cast<float>(B.sv[s * sz + n]);
      raw[11] = static_cast<float>(log10(B.dt_local[B.Z.at(i, j, k)]));
#pragma unroll
      for (int q = 0; q < kSurIn; ++q) f[q] = (raw[q] - P.in_mu[q]) / P.in_sig[q];
    }
#pragma unroll
    for (int q = 0; q < kSurInPad; q += 8) {
      uint32_t pk[4];
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const __nv_bfloat162 b2 = __floats2bfloat162_rn(f[q + 2 * h], f[q + 2 * h + 1]);
        pk[h] = *reinterpret_cast<const uint32_t *>(&b2);
      }
      *reinterpret_cast<uint4 *>(a0 + tc::tile_offset(tid, q, kSurInPad)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
  }
  if (warp == 0) tc::tmem_alloc(tslot, 256);
  if (tid == 0) {
    for (int q = 0; q < 3; ++q) tc::mbar_init(&bar[q], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // layer 0 weights (256 x 16) into stage 0
  copy_bytes(stage[0], P.w_packed[0], kSurHidden * kSurInPad * 2);
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;
  Phases ph;
  bool ok = true;

  // ---- layer 0: [128 x 16] x [256 x 16]^T
  if (tid == 0) {
    const uint64_t ad = tc::desc_kmajor(tc::smem_u32(a0), 128, (kSurInPad / 8) * 128);
    const uint64_t bd = tc::desc_kmajor(tc::smem_u32(stage[0]), 128, (kSurInPad / 8) * 128);
    tc::mma_bf16(tmem, ad, bd, tc::idesc_bf16(128, kSurHidden), 0u);
    tc::commit(&bar[2]);
  }
  ok = wait_bar(bar, 2, ph);
  tc::fence_after_sync();
  if (ok) hidden_epilogue(tmem, P.bias[0], a1);
  tc::fence_before_sync();
  tc::fence_async_smem();
  __syncthreads();

  // ---- layers 1..3: [128 x 256] x [256 x 256]^T, K in chunks of 32
  constexpr int nchunk = kSurHidden / kChunk;
  for (int l = 1; l <= 3 && ok; ++l) {
    const uint8_t *w = P.w_packed[l];
    copy_bytes(stage[0], w, kStageBytes);
    tc::fence_async_smem();
    __syncthreads();
    for (int c = 0; c < nchunk && ok; ++c) {
      const int s = c & 1;
      if (tid == 0) {
        tc::fence_after_sync();
        for (int q = 0; q < kChunk / 16; ++q) {
          const int k0 = c * kChunk + q * 16;
          const uint64_t ad = tc::desc_kmajor(tc::smem_u32(a1) + k0 * 16, 128, (kSurHidden / 8) * 128);
          const uint64_t bd = tc::desc_kmajor(tc::smem_u32(stage[s]) + q * 256, 128, (kChunk / 8) * 128);
          tc::mma_bf16(tmem, ad, bd, tc::idesc_bf16(128, kSurHidden), (c > 0 || q > 0) ? 1u : 0u);
        }
        tc::commit(&bar[s]);
      }
      if (c + 1 < nchunk) {
        // stage s^1 was read by the MMAs of chunk c - 1
        if (c >= 1) ok = wait_bar(bar, s ^ 1, ph);
        if (!ok) break;
        copy_bytes(stage[s ^ 1], w + static_cast<size_t>(c + 1) * kStageBytes, kStageBytes);
        tc::fence_async_smem();
        __syncthreads();
      }
    }
    // the last two commits: chunks nchunk-2 (stage 0) and nchunk-1 (stage 1)
    if (ok) ok = wait_bar(bar, 0, ph);
    if (ok) ok = wait_bar(bar, 1, ph);
    tc::fence_after_sync();
    if (ok) hidden_epilogue(tmem, P.bias[l], a1);
    tc::fence_before_sync();
    tc::fence_async_smem();
    __syncthreads();
  }

  // ---- output layer: [128 x 256] x [16 x 256]^T (all 8 chunks in one stage)
  if (ok) {
    copy_bytes(stage[0], P.w_packed[4], kSurOutPad * kSurHidden * 2);
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      for (int q = 0; q < kSurHidden / 16; ++q) {
        const int k0 = q * 16;
        const uint64_t ad = tc::desc_kmajor(tc::smem_u32(a1) + k0 * 16, 128, (kSurHidden / 8) * 128);
        const uint32_t boff = (k0 / kChunk) * (kSurOutPad * kChunk * 2) + (k0 % kChunk) / 8 * 128;
        const uint64_t bd = tc::desc_kmajor(tc::smem_u32(stage[0]) + boff, 128, (kChunk / 8) * 128);
        tc::mma_bf16(tmem, ad, bd, tc::idesc_bf16(128, kSurOutPad), q > 0 ? 1u : 0u);
      }
      tc::commit(&bar[2]);
    }
    ok = wait_bar(bar, 2, ph);
    tc::fence_after_sync();
  }
  float o[32];
  if (ok && warp < 4) tc::tmem_ld32(tmem + (static_cast<uint32_t>(warp * 32) << 16), o);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 256);
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
    return;
  }
  if (tid >= 128) return;
  const int64_t c = static_cast<int64_t>(blockIdx.x) * 128 + tid;
  if (c >= cells) return;
  const int i = static_cast<int>(c % B.mx), j = static_cast<int>((c / B.mx) % B.my),
            k = static_cast<int>(c / (static_cast<int64_t>(B.mx) * B.my));
  const int64_t n = B.G.at(i, j, k);
  double Y[NS], dy[NS];
  for (int s = 0; s < NS; ++s) Y[s] = B.sv[s * sz + n];
  float out[NS];
  for (int s = 0; s < NS; ++s) out[s] = o[s] + __ldg(P.bias[4] + s);
  const double T = B.bv[5 * sz + n], rho = B.bv[n];
  const int64_t nz = B.Z.at(i, j, k);
  const double dt = B.dt_local[nz];
  const bool acc = dt > 0 && decode<NS>(P, out, T, log10(B.bv[4 * sz + n]), log10(dt), Y, dy);
  if (mode == 1) {
    B.chem_quiet[nz] = acc ? 1 : 0;
    if (acc)
      for (int s = 0; s < NS; ++s) B.chem_rate[s * B.Z.size + nz] = rho * dy[s] / dt;
    atomicAdd(&stats[acc ? 0 : 1], 1ull);
    return;
  }
  if (acc) {
    for (int s = 0; s < NS; ++s) B.cv[(5 + s) * sz + n] += rho * dy[s];
    primitives_from_q<C>(B, n);
    atomicAdd(&stats[0], 1ull);
  } else {
    fb_list[atomicAdd(fb_count, 1)] = static_cast<int>(c);
    atomicAdd(&stats[1], 1ull);
  }
}

// EPI fallback for the listed cells of block b (grid-stride over the list).
template <class C>
__global__ void __launch_bounds__(128) k_sur_fallback(const DevBlock *__restrict__ blks, int b, const int *fb_count,
                                                      const int *fb_list) {
  constexpr int NS = C::ns;
  extern __shared__ double sq[];
  const DevBlock &B = blks[b];
  const int count = *fb_count;
  const int64_t sz = B.G.size;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
    const int64_t c = fb_list[q];
    const int i = static_cast<int>(c % B.mx), j = static_cast<int>((c / B.mx) % B.my),
              k = static_cast<int>(c / (static_cast<int64_t>(B.mx) * B.my));
    const int64_t n = B.G.at(i, j, k);
    double Y[NS], dy[NS];
    for (int s = 0; s < NS; ++s) Y[s] = B.sv[s * sz + n];
    const double rho = B.bv[n];
    epi_increment<NS>(B.bv[5 * sz + n], rho, Y, B.dt_local[B.Z.at(i, j, k)], sq + threadIdx.x,
                      sq + cP.nr * blockDim.x + threadIdx.x, blockDim.x, dy);
    for (int s = 0; s < NS; ++s) B.cv[(5 + s) * sz + n] += rho * dy[s];
    primitives_from_q<C>(B, n);
  }
}

}  // namespace sur
}  // namespace ostc
