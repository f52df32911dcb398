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
// One CTA per SM handles two 128-cell tiles per pass over the weights (two
// accumulators fill the 512 TMEM columns), so every weight byte staged from
// L2 feeds two MMAs.  The weights stream through a ring of bulk copies in
// 8 KB chunks far enough ahead to cover the L2 latency.
constexpr int kTiles = 2;
constexpr int kCells = 128 * kTiles;
constexpr int kThreads = 512;  // 16 warps: 4 per TMEM lane quarter (tile x column half)
constexpr int kStages = 10;    // weight chunks in flight
constexpr int kLag = 2;        // chunk groups that may still be executing when their stage is refilled
// Every weight chunk is 8 KB: one K=16 slice [256 x 16] of a hidden layer,
// the whole first layer [256 x 16] or the whole output layer [16 x 256],
// all packed K-major canonical with 16-column tiles.
constexpr uint32_t kChunkBytes = kSurHidden * 16 * 2;
constexpr int kChunks = 1 + 3 * (kSurHidden / 16) + 1;
constexpr uint32_t kA0Bytes = 128 * kSurInPad * 2;
constexpr uint32_t kA1Bytes = 128 * kSurHidden * 2;
constexpr uint32_t kSmem = kTiles * (kA0Bytes + kA1Bytes) + kStages * kChunkBytes + (2 * kStages + 2) * 8 + 16;

// Source of weight chunk i in the stream
__device__ __forceinline__ const uint8_t *chunk_src(const SurrogateDev &P, int i) {
  if (i == 0) return P.w_packed[0];
  if (i == kChunks - 1) return P.w_packed[4];
  const int l = 1 + (i - 1) / (kSurHidden / 16), c = (i - 1) % (kSurHidden / 16);
  return P.w_packed[l] + static_cast<size_t>(c) * kChunkBytes;
}

// Asynchronous bulk copy of one chunk into shared memory; completion is
// counted in bytes on the stage's mbarrier.
__device__ __forceinline__ void load_chunk(uint8_t *dst, const uint8_t *src, uint64_t *full) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(kChunkBytes), "r"(tc::smem_u32(full))
               : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   tc::smem_u32(dst)),
               "l"(src), "r"(kChunkBytes), "r"(tc::smem_u32(full))
               : "memory");
}

// Epilogue of a hidden layer: accumulator + bias -> GELU -> bf16 rows of the
// next layer's input tile (K-major canonical, 256 columns).  Warp w reads
// TMEM lane quarter w % 4 of tile (w / 4) / 2, column half (w / 4) % 2.
__device__ __forceinline__ void hidden_epilogue(uint32_t tmem, const float *bias, uint8_t *a1) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int quarter = warp & 3, tile = (warp >> 2) >> 1, half = (warp >> 2) & 1;
  const int row = quarter * 32 + lane;
  uint8_t *a = a1 + tile * kA1Bytes;
  const uint32_t tbase = tmem + (static_cast<uint32_t>(quarter * 32) << 16) + tile * kSurHidden;
  for (int c0 = half * 128; c0 < half * 128 + 128; c0 += 32) {
    float v[32];
    tc::tmem_ld32(tbase + c0, v);
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
      *reinterpret_cast<uint4 *>(a + tc::tile_offset(row, c0 + q, kSurHidden)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
  }
}

// Two 128-cell tiles per CTA: features -> 4 x (256, GELU) -> 9 outputs on the
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
  uint8_t *a0 = smem, *a1 = smem + kTiles * kA0Bytes, *stages = a1 + kTiles * kA1Bytes;
  uint64_t *full = reinterpret_cast<uint64_t *>(stages + kStages * kChunkBytes);
  uint64_t *empty = full + kStages, *acc_bar = empty + kStages;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(acc_bar + 1);
  const DevBlock &B = blks[b];
  const int tid = threadIdx.x, warp = tid >> 5;
  const int64_t cells = static_cast<int64_t>(B.mx) * B.my * B.mz;
  const int64_t sz = B.G.size;

  // features of the CTA's cells: thread t < 256 -> tile t / 128, row t % 128
  if (tid < kCells) {
    const int64_t c = static_cast<int64_t>(blockIdx.x) * kCells + tid;
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
    uint8_t *a = a0 + (tid >> 7) * kA0Bytes;
#pragma unroll
    for (int q = 0; q < kSurInPad; q += 8) {
      uint32_t pk[4];
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const __nv_bfloat162 b2 = __floats2bfloat162_rn(f[q + 2 * h], f[q + 2 * h + 1]);
        pk[h] = *reinterpret_cast<const uint32_t *>(&b2);
      }
      *reinterpret_cast<uint4 *>(a + tc::tile_offset(tid & 127, q, kSurInPad)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
  }
  if (warp == 0) tc::tmem_alloc(tslot, 512);
  if (tid == 0) {
    for (int q = 0; q < kStages; ++q) {
      tc::mbar_init(&full[q], 1);
      tc::mbar_init(&empty[q], 1);
    }
    tc::mbar_init(acc_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int q = 0; q < kStages; ++q) load_chunk(stages + q * kChunkBytes, chunk_src(P, q), &full[q]);
  }
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;
  bool ok = true;
  int chunk = 0;         // next chunk of the stream
  int issued = kStages;  // chunks whose copy has been started
  constexpr uint32_t kSboA1 = (kSurHidden / 8) * 128, kSbo16 = (16 / 8) * 128;
  for (int layer = 0; layer < 5; ++layer) {
    // thread 0 issues this layer's MMAs (both tiles) as the weight chunks
    // land and refills the stage of the chunk kLag groups back
    if (tid == 0) {
      const int n_here = (layer == 0 || layer == 4) ? 1 : kSurHidden / 16;
      for (int q = 0; q < n_here && ok; ++q, ++chunk) {
        const int st = chunk % kStages;
        if (!tc::mbar_wait(&full[st], (chunk / kStages) & 1)) {
          ok = false;
          break;
        }
        tc::fence_after_sync();
        const uint32_t wb = tc::smem_u32(stages + st * kChunkBytes);
        for (int t = 0; t < kTiles; ++t) {
          const uint32_t acc = tmem + t * kSurHidden;
          if (layer == 0) {
            const uint64_t ad = tc::desc_kmajor(tc::smem_u32(a0 + t * kA0Bytes), 128, kSbo16);
            tc::mma_bf16(acc, ad, tc::desc_kmajor(wb, 128, kSbo16), tc::idesc_bf16(128, kSurHidden), 0u);
          } else if (layer < 4) {
            const uint64_t ad = tc::desc_kmajor(tc::smem_u32(a1 + t * kA1Bytes) + q * 16 * 16, 128, kSboA1);
            tc::mma_bf16(acc, ad, tc::desc_kmajor(wb, 128, kSbo16), tc::idesc_bf16(128, kSurHidden),
                         q > 0 ? 1u : 0u);
          } else {
            for (int kk = 0; kk < kSurHidden / 16; ++kk) {
              const uint64_t ad = tc::desc_kmajor(tc::smem_u32(a1 + t * kA1Bytes) + kk * 16 * 16, 128, kSboA1);
              const uint64_t bd = tc::desc_kmajor(wb + kk * (kSurOutPad * 16 * 2), 128, kSbo16);
              tc::mma_bf16(acc, ad, bd, tc::idesc_bf16(128, kSurOutPad), kk > 0 ? 1u : 0u);
            }
          }
        }
        tc::commit(&empty[st]);
        const int old = chunk - kLag;
        if (old >= 0 && old + kStages < kChunks) {
          const int os = old % kStages;
          if (!tc::mbar_wait(&empty[os], (old / kStages) & 1)) {
            ok = false;
            break;
          }
          load_chunk(stages + os * kChunkBytes, chunk_src(P, old + kStages), &full[os]);
          ++issued;
        }
      }
      if (ok) tc::commit(acc_bar);
    }
    ok = __syncthreads_and(ok) != 0;
    if (!ok) break;
    ok = __syncthreads_and(tc::mbar_wait(acc_bar, layer & 1)) != 0;
    tc::fence_after_sync();
    if (!ok || layer == 4) break;
    hidden_epilogue(tmem, P.bias[layer], a1);
    tc::fence_before_sync();
    tc::fence_async_smem();
    __syncthreads();
  }
  if (tid == 0) {
    // copies issued beyond the last consumed chunk (only on a timeout) land
    // before the CTA exits
    for (int c = chunk; c < issued; ++c) tc::mbar_wait(&full[c % kStages], (c / kStages) & 1);
  }
  // outputs: warps with (w / 4) % 2 == 0 read their tile's 16 output columns
  const int quarter = warp & 3, tile = (warp >> 2) >> 1, half = (warp >> 2) & 1;
  float o[32];
  if (ok && half == 0)
    tc::tmem_ld32(tmem + (static_cast<uint32_t>(quarter * 32) << 16) + tile * kSurHidden, o);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 512);
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
    return;
  }
  if (half != 0) return;
  const int64_t c = static_cast<int64_t>(blockIdx.x) * kCells + tile * 128 + quarter * 32 + (tid & 31);
  const bool valid = c < cells;
  bool acc = false;
  int64_t n = 0, nz = 0;
  double rho = 0, dt = 0, dy[NS];
  if (valid) {
    const int i = static_cast<int>(c % B.mx), j = static_cast<int>((c / B.mx) % B.my),
              k = static_cast<int>(c / (static_cast<int64_t>(B.mx) * B.my));
    n = B.G.at(i, j, k);
    nz = B.Z.at(i, j, k);
    double Y[NS];
    for (int s = 0; s < NS; ++s) Y[s] = B.sv[s * sz + n];
    float out[NS];
    for (int s = 0; s < NS; ++s) out[s] = o[s] + __ldg(P.bias[4] + s);
    rho = B.bv[n];
    dt = B.dt_local[nz];
    acc = dt > 0 && decode<NS>(P, out, B.bv[5 * sz + n], log10(B.bv[4 * sz + n]), log10(dt), Y, dy);
  }
  // one counter update per warp
  const unsigned a_mask = __ballot_sync(0xffffffffu, valid && acc), r_mask = __ballot_sync(0xffffffffu, valid && !acc);
  if ((tid & 31) == 0) {
    if (a_mask) atomicAdd(&stats[0], static_cast<unsigned long long>(__popc(a_mask)));
    if (r_mask) atomicAdd(&stats[1], static_cast<unsigned long long>(__popc(r_mask)));
  }
  if (!valid) return;
  if (mode == 1) {
    B.chem_quiet[nz] = acc ? 1 : 0;
    if (acc)
      for (int s = 0; s < NS; ++s) B.chem_rate[s * B.Z.size + nz] = rho * dy[s] / dt;
    return;
  }
  if (acc) {
    for (int s = 0; s < NS; ++s) B.cv[(5 + s) * sz + n] += rho * dy[s];
    primitives_from_q<C>(B, n);
  } else {
    fb_list[atomicAdd(fb_count, 1)] = static_cast<int>(c);
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
