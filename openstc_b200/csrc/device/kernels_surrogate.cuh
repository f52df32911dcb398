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

// FP32 copies of the mechanism tables the judge reads (one per translation
// unit, uploaded with the FP64 tables): sign(A) and ln|A| of both Arrhenius
// sets, b, Ea, Troe parameters, third-body efficiencies, W_k and NASA-7.
struct JudgeTables {
  float sA[kMaxReac], lnA[kMaxReac], b[kMaxReac], Ea[kMaxReac];
  float sA2[kMaxReac], lnA2[kMaxReac], b2[kMaxReac], Ea2[kMaxReac];
  float troe_a[kMaxReac], troe_t3[kMaxReac], troe_t1[kMaxReac], troe_t2[kMaxReac];
  float tb[kMaxReac * kMaxSpec];
  float sf[kMaxReac * kMaxSpec], sb[kMaxReac * kMaxSpec], nu[kMaxReac * kMaxSpec];  // stoichiometry, sb - sf
  float order[kMaxReac];
  float mw[kMaxSpec], mw_inv[kMaxSpec], t_low[kMaxSpec], ln_t_low[kMaxSpec], t_mid[kMaxSpec];
  float low[kMaxSpec * 7], high[kMaxSpec * 7];
};

static __constant__ JudgeTables cJ;

constexpr int kJudgeCta = 256;  // threads of a k_sur_judge block

inline JudgeTables make_judge_tables(const DevParams &p) {
  JudgeTables j{};
  auto sgn = [](double a) { return a > 0 ? 1.f : (a < 0 ? -1.f : 0.f); };
  for (int r = 0; r < kMaxReac; ++r) {
    j.sA[r] = sgn(p.A[r]);
    j.lnA[r] = static_cast<float>(p.lnA[r]);
    j.b[r] = static_cast<float>(p.b[r]);
    j.Ea[r] = static_cast<float>(p.Ea[r]);
    j.sA2[r] = sgn(p.A2[r]);
    j.lnA2[r] = static_cast<float>(p.lnA2[r]);
    j.b2[r] = static_cast<float>(p.b2[r]);
    j.Ea2[r] = static_cast<float>(p.Ea2[r]);
    j.troe_a[r] = static_cast<float>(p.troe_a[r]);
    j.troe_t3[r] = static_cast<float>(p.troe_t3[r]);
    j.troe_t1[r] = static_cast<float>(p.troe_t1[r]);
    j.troe_t2[r] = static_cast<float>(p.troe_t2[r]);
  }
  for (int q = 0; q < kMaxReac * kMaxSpec; ++q) {
    j.tb[q] = static_cast<float>(p.tb[q]);
    j.sf[q] = static_cast<float>(p.sf[q]);
    j.sb[q] = static_cast<float>(p.sb[q]);
    j.nu[q] = static_cast<float>(p.sb[q] - p.sf[q]);
  }
  for (int r = 0; r < kMaxReac; ++r) j.order[r] = static_cast<float>(p.order[r]);
  for (int k = 0; k < kMaxSpec; ++k) {
    j.mw[k] = static_cast<float>(p.mw[k]);
    j.mw_inv[k] = p.mw[k] > 0 ? static_cast<float>(1.0 / p.mw[k]) : 0.f;
    j.t_low[k] = static_cast<float>(p.t_low[k]);
    j.ln_t_low[k] = p.t_low[k] > 0 ? static_cast<float>(std::log(p.t_low[k])) : -80.f;
    j.t_mid[k] = static_cast<float>(p.t_mid[k]);
  }
  for (int q = 0; q < kMaxSpec * 7; ++q) {
    j.low[q] = static_cast<float>(p.low[q]);
    j.high[q] = static_cast<float>(p.high[q]);
  }
  return j;
}


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
    // reactions outside the species loop (each (m, q) still sums in reaction
    // order), as in k_source
    double zz[NS];
    for (int q = 0; q < NS; ++q) zz[q] = 0;
    for (int r = 0; r < nr; ++r) {
      const int dn = cP.sb[r * NS + m] - cP.sf[r * NS + m];
      if (dn == 0) continue;
      const double a1 = q1[r * stride], a2 = q2[r * stride];
      for (int q = 0; q < NS; ++q) zz[q] += dn * (cP.sf[r * NS + q] * a1 - cP.sb[r * NS + q] * a2);
    }
    for (int q = 0; q < NS; ++q) {
      const double v = Y[q] > 1e-25 ? zz[q] / (rho * Y[q]) : 0.0;
      const double J = cP.mw[m] * v * 1e+3;
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

// The judge's increment of one cell in FP32: the point-implicit step with the
// diagonal of the chemistry Jacobian (the reference's DA treatment,
// src/FiniteRateChem.cu:196-209, 400-412), dY_k = (dt omega_k / rho) /
// (1 + dt omega_d,k / (rho Y_k)), from the production and destruction rates of
// finite_rate_chemistry (src/FiniteRateChem.cu:7-171).  The full EPI step
// (I - dt J)^-1 dt omega / rho couples the species; the diagonal keeps each
// species' own stiffness, which is what bounds the increments of trace
// radicals, so it follows the EPI step closely where the explicit increment
// would not.  A cell whose network increment disagrees with it is reacting in
// a way the network did not capture.  p in Pa, dt in s.
// Arithmetic: every rate, equilibrium constant and concentration product is
// one exponential of a sum over the species with the stoichiometric
// coefficients as FP32 factors (q_f = k_f exp(sum_k nu'_k ln c_k)), exponents
// clamped to the FP32 range, so the loops over species have compile-time trip
// counts and read uniform constant-bank operands.  Concentrations below 1e-30
// count as 1e-30 (their products underflow to zero like the exact ones).  The
// exponentials, logarithms and quotients are the hardware approximations
// (__expf, __logf, __fdividef: relative errors near 1e-6, against the judge's
// 25 % tolerance), which have no slow paths for lanes to diverge on.
template <int NS>
__device__ __forceinline__ void judge_increment(float T, float p, float dt, const float *Y, float *e) {
  float inv_mw = 0;
#pragma unroll
  for (int k = 0; k < NS; ++k) inv_mw += Y[k] * cJ.mw_inv[k];
  const float rho = __fdividef(p, 8314.462618f * T * inv_mw);
  float c[NS], lc[NS], g[NS];
  const float ln_t = __logf(T), t_inv = __fdividef(1.f, T);
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    c[k] = rho * Y[k] * cJ.mw_inv[k] * 1e-3f;
    lc[k] = __logf(fmaxf(c[k], 1e-30f));
    // g_k / RT from the NASA-7 polynomials, frozen below T_low
    const float tt = fmaxf(T, cJ.t_low[k]), lt = fmaxf(ln_t, cJ.ln_t_low[k]);
    const bool lo = tt < cJ.t_mid[k];
    float a[7];
#pragma unroll
    for (int m = 0; m < 7; ++m) a[m] = lo ? cJ.low[k * 7 + m] : cJ.high[k * 7 + m];
    g[k] = a[0] * (1.f - lt) + __fdividef(a[5], tt) - a[6] -
           tt * (0.5f * a[1] + tt * (a[2] * (1.f / 6.f) + tt * (a[3] * (1.f / 12.f) + tt * (a[4] * 0.05f))));
  }
  float omega[NS], destruction[NS];
#pragma unroll
  for (int k = 0; k < NS; ++k) omega[k] = destruction[k] = 0;
  auto rate = [&](float sA, float lnA, float b, float Ea) {
    return sA * __expf(fminf(lnA + b * ln_t - Ea * t_inv, 80.f));
  };
  const float ln_temp_t = logf(101325.0f / 8314.462618f * 1e-3f) - ln_t;
  const int nr = cP.nr;
  for (int r = 0; r < nr; ++r) {
    const int type = cP.label[r];
    float kf = rate(cJ.sA[r], cJ.lnA[r], cJ.b[r], cJ.Ea[r]);
    if (type == 3) kf += rate(cJ.sA2[r], cJ.lnA2[r], cJ.b2[r], cJ.Ea2[r]);
    if (type > 3) {
      float cc = 0;
#pragma unroll
      for (int k = 0; k < NS; ++k) cc += c[k] * cJ.tb[r * NS + k];
      if (type == 4) {
        kf *= cc;
      } else {
        // reduced pressure; a high-pressure rate that underflows FP32 leaves
        // the rate at zero
        const float pr = fmaxf(__fdividef(rate(cJ.sA2[r], cJ.lnA2[r], cJ.b2[r], cJ.Ea2[r]) * cc, kf), 1e-30f);
        float F = 1.f;
        if (type > 5) {
          const float a = cJ.troe_a[r];
          float fc = (1 - a) * __expf(__fdividef(-T, cJ.troe_t3[r])) + a * __expf(__fdividef(-T, cJ.troe_t1[r]));
          if (type == 7) fc += __expf(-cJ.troe_t2[r] * t_inv);
          const float lfc = __log10f(fc), lpr = __log10f(pr);
          const float cq = -0.4f - 0.67f * lfc, nq = 0.75f - 1.27f * lfc;
          const float tmp = __fdividef(lpr + cq, nq - 0.14f * (lpr + cq));
          F = __exp10f(__fdividef(lfc, 1.f + tmp * tmp));
        }
        if (kf > 0.f) kf = kf * __fdividef(pr, 1.f + pr) * F;
      }
    }
    float s1 = 0, s2 = 0, dg = 0;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      s1 += cJ.sf[r * NS + k] * lc[k];
      s2 += cJ.sb[r * NS + k] * lc[k];
      dg += cJ.nu[r * NS + k] * g[k];
    }
    const float q1 = kf * __expf(fminf(s1, 80.f));
    const float q2 = type != 2 ? kf * __expf(fminf(fminf(dg - cJ.order[r] * ln_temp_t, 80.f) + s2, 80.f))
                               : rate(cJ.sA2[r], cJ.lnA2[r], cJ.b2[r], cJ.Ea2[r]) * __expf(fminf(s2, 80.f));
    const float q = q1 - q2;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      omega[k] += cJ.nu[r * NS + k] * q;
      destruction[k] += cJ.sf[r * NS + k] * q1 + cJ.sb[r * NS + k] * q2;
    }
  }
  const float f = __fdividef(dt, rho);
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    const float w = cJ.mw[k] * 1e3f;
    const float y = fmaxf(Y[k], 1e-30f);
    e[k] = __fdividef(f * omega[k] * w, 1.f + f * destruction[k] * w * __fdividef(1.f, y));
  }
}

// The judge's verdict on an increment dy of a cell (T, p, Y, dt): every
// species within gate.judge_rel of the diagonal point-implicit increment plus
// gate.judge_abs (Y_k + gate.y_floor); a non-finite judge increment fails.
template <int NS>
__device__ __forceinline__ bool judge_accepts(const SurrogateGate &g, float T, float p, float dt, const float *Y,
                                              const float *dy) {
  float e[NS];
  judge_increment<NS>(T, p, dt, Y, e);
  bool ok = true;
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    const float err = fabsf(dy[k] - e[k]);
    const float tol = g.judge_rel * fabsf(e[k]) + g.judge_abs * (Y[k] + g.y_floor);
    if (!(err <= tol)) ok = false;
  }
  return ok;
}

// Network output o (normalised, bias added) -> dY_k = (Y_k + eps) c_k
// sinh(s_k o_k); the increment is then projected onto element conservation
// (weighted least squares, weights |dY_k| + 1e-3 Y_k).  The cell is accepted
// when the inputs lie in the training box, every output is within
// gate.out_max, the raw element defect is below gate.defect_tol of the
// element totals, no increment exceeds gate.rel_max (Y_k + gate.y_floor)
// (species below the floor are judged by their absolute change), and no mass
// fraction is driven below -1e-9: the network is trusted where the chemistry
// changes the composition little, the EPI step takes the reacting cells.
// The judge: an accepted increment must also agree, species by species,
// with the diagonal point-implicit increment (judge_increment) within
// gate.judge_rel of it plus gate.judge_abs (Y_k + gate.y_floor); an
// increment the network under-predicts (down to none at all) for a reacting
// cell fails it.  gate.judge_rel < 0 turns the judge off.
// NE is a compile-time bound on the element count (elements past p.n_elem
// have zero rows and drop out), so every array lives in registers.  The
// network's own error is ~1e-2, so the transcendental functions of the decode
// run in FP32; the projection and the increments stay in FP64.
// JUDGE: apply the judge here (the fused inference kernel leaves it to
// k_sur_judge, which runs it at full occupancy over the accepted cells).
template <int NS, int NE, bool JUDGE = true>
__device__ __forceinline__ bool decode_ne(const SurrogateDev &p, const float *o, float T, float lp, float ldt,
                                          const double *Y, double *dy) {
  const SurrogateGate &g = p.gate;
  bool ok = T >= g.t_min && T <= g.t_max && lp >= g.lp_min && lp <= g.lp_max && ldt >= g.ldt_min && ldt <= g.ldt_max;
  float w[NS];  // any positive weights conserve the elements exactly; FP32 is enough for them
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    ok = ok && fabsf(o[k]) <= g.out_max;
    const float oc = fminf(fmaxf(o[k], -g.out_max), g.out_max);
    dy[k] = (Y[k] + kSurYEps) * static_cast<double>(p.out_c[k] * sinhf(oc * p.out_s[k]));
    if (fabs(dy[k]) > g.rel_max * (Y[k] + fmax(kSurYEps, static_cast<double>(g.y_floor)))) ok = false;
    w[k] = static_cast<float>(fabs(dy[k]) + 1e-3 * Y[k]) + 1e-30f;
  }
  // normal equations (E W E^T) lambda = E dy, E[e][k] = a_ek / W_k
  double r[NE], M[NE][NE];
#pragma unroll
  for (int e = 0; e < NE; ++e) {
    double defect = 0, total = 0;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      defect += p.elem[e * kMaxSpec + k] * dy[k];
      total += p.elem[e * kMaxSpec + k] * Y[k];
    }
    r[e] = defect;
    if (total > 0 && fabs(defect) > g.defect_tol * total) ok = false;
#pragma unroll
    for (int f = 0; f <= e; ++f) {
      double s = 0;
#pragma unroll
      for (int k = 0; k < NS; ++k) s += static_cast<double>(p.elem[e * kMaxSpec + k] * w[k]) * p.elem[f * kMaxSpec + k];
      M[e][f] = s;
      M[f][e] = s;
    }
  }
  // M is symmetric positive (semi-)definite: Gauss-Jordan without pivoting; an
  // element absent from the cell (zero row) gets lambda = 0
#pragma unroll
  for (int c = 0; c < NE; ++c) {
    const bool live = M[c][c] > 1e-300;
    const double inv = live ? 1.0 / M[c][c] : 0.0;
#pragma unroll
    for (int q = 0; q < NE; ++q) {
      if (q == c) continue;
      const double f = M[q][c] * inv;
#pragma unroll
      for (int z = 0; z < NE; ++z) M[q][z] -= f * M[c][z];
      r[q] -= f * r[c];
    }
    r[c] *= inv;
  }
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    double corr = 0;
#pragma unroll
    for (int e = 0; e < NE; ++e) corr += p.elem[e * kMaxSpec + k] * r[e];
    dy[k] -= w[k] * corr;
    if (Y[k] + dy[k] < -1e-9) ok = false;
  }
  if (JUDGE && ok && g.judge_rel >= 0.f) {
    float yf[NS], dyf[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      yf[k] = static_cast<float>(Y[k]);
      dyf[k] = static_cast<float>(dy[k]);
    }
    ok = judge_accepts<NS>(g, T, exp10f(lp), exp10f(ldt), yf, dyf);
  }
  return ok;
}

template <int NS>
__device__ __forceinline__ bool decode(const SurrogateDev &p, const float *o, float T, float lp, float ldt,
                                       const double *Y, double *dy) {
  if (p.n_elem <= 4) return decode_ne<NS, 4>(p, o, T, lp, ldt, Y, dy);
  return decode_ne<NS, kMaxElem>(p, o, T, lp, ldt, Y, dy);
}

// ------------------------------------------------------------ fused kernel
// A persistent kernel, one CTA per SM, that runs the tiles of 128 cells of a
// block through the network as a software pipeline on mbarriers, with two
// tiles in flight: tiles alternate between two slots (tile it uses slot
// it % 2), each with its own 256-column TMEM accumulator, 64 KB activation
// buffer and 4 KB feature buffer, so that one slot's epilogue runs while the
// tensor cores work on the other slot's layer.
//   * warp 17 (one lane) streams the hidden layers' weights through a ring
//     of kStages shared-memory stages of 16 KB (K = 32), in the order the
//     MMAs consume them; the first and output layers' weights (8 KB each)
//     stay resident;
//   * warp 16 issues the tcgen05 MMAs in the order (pair of tiles, layer,
//     slot): layer L of tile 2p, layer L of tile 2p + 1, layer L + 1 of
//     tile 2p, ...;
//   * warps 0-15 (TMEM lane quarter w % 4, column group w / 4) run the
//     hidden epilogues in the same order: accumulator + bias -> GELU -> bf16
//     activations of the slot;
//   * warps 18-21 (lane quarters 2, 3, 0, 1) compute the features of tile
//     it + 2 once tile it's first layer has read its slot's feature buffer,
//     and decode / gate / apply tile it's outputs.
// Within a slot every stage waits for the one before it (MMA of layer L ->
// epilogue of layer L -> MMA of layer L + 1 ... -> decode -> first layer of
// the slot's next tile), so each barrier of a slot completes its phases in
// that order and a waiter is never more than one phase behind.  Every wait
// is bounded: a wait that runs out raises the CTA's abort flag, every role
// then leaves its loop, the MMAs and copies in flight are drained, and the
// kernel reports the error.
constexpr int kCells = 128;
constexpr int kEpiWarps = 16;
constexpr int kMmaWarp = 16, kLoadWarp = 17, kIoWarp0 = 18;
constexpr int kThreads = 32 * 22;
constexpr int kStageChunks = 2;  // weight chunks per ring stage
constexpr int kStages = 4;       // ring stages
constexpr int kFusedElem = 4;  // largest element count of the fused kernel's conservation gate
constexpr int kRecheckEvery = 4;  // a cell the gate rejected is evaluated again within this many steps
// Every weight chunk is 8 KB: one K=16 slice [256 x 16] of a hidden layer,
// the whole first layer [256 x 16] or the whole output layer [16 x 256],
// all packed K-major canonical with 16-column tiles.
constexpr uint32_t kChunkBytes = kSurHidden * 16 * 2;
constexpr int kLayerStages = kSurHidden / 16 / kStageChunks;  // streamed stages per hidden layer
constexpr uint32_t kActBytes = 128 * kSurHidden * 2;
constexpr uint32_t kStageBytes = kStageChunks * kChunkBytes;
constexpr uint32_t kX0Bytes = 128 * kSurInPad * 2;
// barriers: full[S], empty[S], and per slot feat_full, x0_free, mma_done,
// epi_done, out_done, out_free; then res, drain.
constexpr int kBars = 2 * kStages + 6 * 2 + 1 + 1;
constexpr uint32_t kBiasBytes = (4 * kSurHidden + kSurOutPad) * 4;  // every layer's bias, staged once per CTA
constexpr uint32_t kSmem =
    2 * kActBytes + 2 * kX0Bytes + 2 * kChunkBytes + kStages * kStageBytes + kBiasBytes + kBars * 8 + 16;
static_assert(kSmem <= 232448, "shared memory of one CTA");

// Source of stage s (0 .. 3 kLayerStages - 1) of hidden layers 1-3: K chunks
// kStageChunks (s % kLayerStages) onwards of hidden layer 1 + s / kLayerStages,
// contiguous in its packed weights
__device__ __forceinline__ const uint8_t *stage_src(const SurrogateDev &P, int s) {
  return P.w_packed[1 + s / kLayerStages] + static_cast<size_t>(s % kLayerStages) * kStageBytes;
}

// Asynchronous bulk copies into shared memory: the stage's mbarrier is told
// the byte count once, and each chunk's copy completes its share.
__device__ __forceinline__ void expect_bytes(uint64_t *full, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(bytes), "r"(tc::smem_u32(full))
               : "memory");
}
__device__ __forceinline__ void load_bytes(uint8_t *dst, const uint8_t *src, uint32_t bytes, uint64_t *full) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   tc::smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(tc::smem_u32(full))
               : "memory");
}

__device__ __forceinline__ void bar_arrive(uint64_t *bar, uint32_t count = 1) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(bar)), "r"(count) : "memory");
}

// Bounded wait that gives up early once another role has aborted.
__device__ __forceinline__ bool wait_bar(uint64_t *bar, uint32_t parity, volatile int *abort) {
  for (uint32_t it = 0; it < (1u << 24); ++it) {
    if (tc::mbar_try(bar, parity)) return true;
    if ((it & 63) == 63 && *abort) return false;
  }
  *abort = 1;
  return false;
}

__device__ __forceinline__ uint64_t f2_pack(float lo, float hi) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2_unpack(uint64_t v, float &lo, float &hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}

// GELU (tanh form) of two pre-activations, returned as packed bf16x2 (lo =
// x0).  The polynomial runs on packed FP32 pairs; tanh runs on the half-
// precision pair unit (its argument saturates to the largest finite half,
// where tanh is 1): the result is rounded to bf16, whose step is 8x the
// error of the half-precision tanh.
__device__ __forceinline__ uint32_t gelu2_bf16(float x0, float x1) {
  const uint64_t x = f2_pack(x0, x1);
  const uint64_t c0 = f2_pack(0.7978845608028654f, 0.7978845608028654f);
  const uint64_t c1 = f2_pack(0.7978845608028654f * 0.044715f, 0.7978845608028654f * 0.044715f);
  const uint64_t half2 = f2_pack(0.5f, 0.5f);
  uint64_t x2, p, u, hx;
  asm("mul.rn.f32x2 %0, %1, %1;" : "=l"(x2) : "l"(x));
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(p) : "l"(c1), "l"(x2), "l"(c0));
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(u) : "l"(x), "l"(p));
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(hx) : "l"(x), "l"(half2));
  float u0, u1;
  f2_unpack(u, u0, u1);
  uint32_t h, t;
  asm("cvt.rn.satfinite.f16x2.f32 %0, %1, %2;" : "=r"(h) : "f"(u1), "f"(u0));
  asm("tanh.approx.f16x2 %0, %1;" : "=r"(t) : "r"(h));
  float t0, t1;
  asm("{\n .reg .f16 a, b;\n mov.b32 {a, b}, %2;\n cvt.f32.f16 %0, a;\n cvt.f32.f16 %1, b;\n}"
      : "=f"(t0), "=f"(t1)
      : "r"(t));
  uint64_t y;
  asm("fma.rn.f32x2 %0, %1, %2, %1;" : "=l"(y) : "l"(hx), "l"(f2_pack(t0, t1)));
  float y0, y1;
  f2_unpack(y, y0, y1);
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(y1), "f"(y0));
  return r;
}

// Features of cell c -> bf16 row `row` of the first layer's input (zeros
// for c past the last cell).
template <class C>
__device__ __forceinline__ void tile_features(const DevBlock &B, const SurrogateDev &P, int64_t c, int row,
                                              uint8_t *x0) {
  constexpr int NS = C::ns;
  const int64_t cells = static_cast<int64_t>(B.mx) * B.my * B.mz, sz = B.G.size;
  float f[kSurInPad];
#pragma unroll
  for (int q = 0; q < kSurInPad; ++q) f[q] = 0.f;
  if (c < cells) {
    const int i = static_cast<int>(c % B.mx), j = static_cast<int>((c / B.mx) % B.my),
              k = static_cast<int>(c / (static_cast<int64_t>(B.mx) * B.my));
    const int64_t n = B.G.at(i, j, k);
    float raw[kSurIn];
    raw[0] = static_cast<float>(B.bv[5 * sz + n]);
    raw[1] = log10f(static_cast<float>(B.bv[4 * sz + n]));
#pragma unroll
    for (int s = 0; s < NS; ++s) raw[2 + s] = static_cast<float>(B.sv[s * sz + n]);
    raw[11] = log10f(static_cast<float>(B.dt_local[B.Z.at(i, j, k)]));
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
    *reinterpret_cast<uint4 *>(x0 + tc::tile_offset(row, q, kSurInPad)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
  }
}

// Decode, gate and apply the network output o of cell c (warp-collective for
// the statistics).  MODE 1: mark quiet cells and their rate; MODE 0: apply the
// increment or list the cell for the EPI fallback.
template <class C, int MODE, int NE>
__device__ __forceinline__ void tile_apply(const DevBlock &B, const SurrogateDev &P, int64_t c, const float *o,
                                           const float *bias_out, int *fb_count, int *fb_list,
                                           unsigned long long *stats) {
  constexpr int NS = C::ns;
  const int64_t cells = static_cast<int64_t>(B.mx) * B.my * B.mz, sz = B.G.size;
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
#pragma unroll
    for (int s = 0; s < NS; ++s) Y[s] = B.sv[s * sz + n];
    float out[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) out[s] = o[s] + bias_out[s];
    rho = B.bv[n];
    dt = B.dt_local[nz];
    acc = dt > 0 && decode_ne<NS, NE, false>(P, out, static_cast<float>(B.bv[5 * sz + n]),
                                      log10f(static_cast<float>(B.bv[4 * sz + n])), log10f(static_cast<float>(dt)),
                                      Y, dy);
  }
  // one counter update per warp
  const unsigned a_mask = __ballot_sync(0xffffffffu, valid && acc), r_mask = __ballot_sync(0xffffffffu, valid && !acc);
  if ((threadIdx.x & 31) == 0) {
    if (a_mask) atomicAdd(&stats[0], static_cast<unsigned long long>(__popc(a_mask)));
    if (r_mask) atomicAdd(&stats[1], static_cast<unsigned long long>(__popc(r_mask)));
  }
  if (!valid) return;
  if constexpr (MODE == 1) {
    B.chem_quiet[nz] = acc ? 1 : 0;
    if (acc) {
      const double f = rho / dt;
#pragma unroll
      for (int s = 0; s < NS; ++s) B.chem_rate[s * B.Z.size + nz] = f * dy[s];
    }
  } else {
    if (acc) {
#pragma unroll
      for (int s = 0; s < NS; ++s) B.cv[(5 + s) * sz + n] += rho * dy[s];
      primitives_from_q<C>(B, n);
    } else {
      fb_list[atomicAdd(fb_count, 1)] = static_cast<int>(c);
    }
  }
}

// The tiles of block b: features -> 4 x (256, GELU) -> 9 outputs on the
// tensor cores, then decode, project and gate, with dt = the cell's local
// time step.  MODE 1 (in the step, before the source term): accepted cells
// are marked chemically quiet and get the rate rho dY / dt, the others keep
// the point-implicit chemistry.  MODE 0 (a split step): accepted increments
// go into cv (rho Y_k) with the primitives recomputed, rejected cells are
// listed for the EPI fallback.  stats[0] += accepted, stats[1] += rejected,
// stats[2] += cells evaluated.
// NE (3 or 4) bounds the element count of the conservation gate.  With a
// candidate list (cand, *cand_count; k_sur_candidates) only the listed cells
// are evaluated, and the CTA of block index 0 advances *phase_ctr at the end.
template <class C, int MODE, int NE>
__global__ void __launch_bounds__(kThreads, 1) k_sur_infer(const DevBlock *__restrict__ blks, int b, SurrogateDev P,
                                                           int *fb_count, int *fb_list, unsigned long long *stats,
                                                           int *err, const int *__restrict__ cand,
                                                           const int *cand_count, int *phase_ctr) {
  extern __shared__ __align__(128) uint8_t smem[];
  uint8_t *act = smem;                       // 2 x 64 KB, by slot
  uint8_t *x0 = smem + 2 * kActBytes;        // 2 x 4 KB, by slot
  uint8_t *wres = x0 + 2 * kX0Bytes;         // first and output layers' weights, 2 x 8 KB
  uint8_t *stages = wres + 2 * kChunkBytes;  // kStages x 16 KB
  float *sbias = reinterpret_cast<float *>(stages + kStages * kStageBytes);
  uint64_t *bars = reinterpret_cast<uint64_t *>(reinterpret_cast<uint8_t *>(sbias) + kBiasBytes);
  uint64_t *full = bars, *empty = full + kStages, *feat_full = empty + kStages, *x0_free = feat_full + 2,
           *mma_done = x0_free + 2, *epi_done = mma_done + 2, *out_done = epi_done + 2, *out_free = out_done + 2,
           *res_full = out_free + 2, *drain = res_full + 1;
  static_assert(kBars == 2 * kStages + 6 * 2 + 1 + 1, "one slot per barrier");
  uint32_t *tslot = reinterpret_cast<uint32_t *>(drain + 1);
  volatile int *abort = reinterpret_cast<volatile int *>(tslot + 1);
  const DevBlock &B = blks[b];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t cells = static_cast<int64_t>(B.mx) * B.my * B.mz;
  const int64_t n_items = cand ? static_cast<int64_t>(*cand_count) : cells;
  // the cell of item idx (past the end: an invalid cell)
  auto cell_of = [&](int64_t idx) -> int64_t { return cand ? (idx < n_items ? cand[idx] : cells) : idx; };
  const int64_t ntiles = (n_items + kCells - 1) / kCells;
  // this CTA's tiles: blockIdx.x, blockIdx.x + gridDim.x, ...; tile it sits in slot it % 2
  const int my_tiles =
      blockIdx.x < ntiles ? static_cast<int>((ntiles - 1 - blockIdx.x) / gridDim.x + 1) : 0;
  const int n_pairs = (my_tiles + 1) / 2;

  if (tid == 0) {
    for (int q = 0; q < kStages; ++q) {
      tc::mbar_init(&full[q], 1);
      tc::mbar_init(&empty[q], 1);
    }
    for (int q = 0; q < 2; ++q) {
      tc::mbar_init(&feat_full[q], 4);
      tc::mbar_init(&x0_free[q], 1);
      tc::mbar_init(&mma_done[q], 1);
      tc::mbar_init(&epi_done[q], kEpiWarps);
      tc::mbar_init(&out_done[q], 1);
      tc::mbar_init(&out_free[q], 4);
    }
    tc::mbar_init(res_full, 1);
    tc::mbar_init(drain, 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tc::tmem_alloc(tslot, 512);
  for (int q = tid; q < 4 * kSurHidden + kSurOutPad; q += kThreads)
    sbias[q] = q < 4 * kSurHidden ? P.bias[q / kSurHidden][q % kSurHidden] : P.bias[4][q - 4 * kSurHidden];
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;

  if (warp == kLoadWarp) {
    // ---- weights: the resident pair once, then every hidden layer's stages
    // in the order the MMAs consume them (each tile of a pair streams the
    // layer again); stage si goes to ring slot si % kStages once the MMAs of
    // stage si - kStages are done
    if (lane == 0) {
      expect_bytes(res_full, 2 * kChunkBytes);
      load_bytes(wres, P.w_packed[0], kChunkBytes, res_full);
      load_bytes(wres + kChunkBytes, P.w_packed[4], kChunkBytes, res_full);
      int si = 0;
      bool ok = true;
      for (int pr = 0; pr < n_pairs && ok; ++pr)
        for (int L = 1; L < 4 && ok; ++L)
          for (int t = 2 * pr; t < min(2 * pr + 2, my_tiles) && ok; ++t)
            for (int g = 0; g < kLayerStages; ++g, ++si) {
              const int slot = si % kStages;
              if (si >= kStages && !wait_bar(&empty[slot], ((si / kStages) - 1) & 1, abort)) {
                ok = false;
                break;
              }
              expect_bytes(&full[slot], kStageBytes);
              load_bytes(stages + slot * kStageBytes, stage_src(P, (L - 1) * kLayerStages + g), kStageBytes,
                         &full[slot]);
            }
      // the copies in flight land before the CTA moves on
      tc::mbar_wait(res_full, 0);
      for (int c = si > kStages ? si - kStages : 0; c < si; ++c)
        tc::mbar_wait(&full[c % kStages], (c / kStages) & 1);
    }
  } else if (warp == kMmaWarp) {
    // ---- tensor-core issue: the whole warp runs the loop, converged, and
    // one elected lane issues each MMA and commit.  Slot q's k-th tile: its
    // first layer waits for its features and for the decode of the slot's
    // previous tile (which read the same accumulator); layer L >= 1 waits for
    // the epilogue of layer L - 1 (epi_done phase 4 k + L - 1).
    constexpr uint32_t kSboAct = (kSurHidden / 8) * 128, kSbo16 = (16 / 8) * 128;
    constexpr uint32_t kIdHidden = tc::idesc_bf16(128, kSurHidden), kIdOut = tc::idesc_bf16(128, kSurOutPad);
    const uint32_t w0 = tc::smem_u32(wres), w4 = w0 + kChunkBytes;
    int si = 0;
    bool ok = __all_sync(0xffffffffu, wait_bar(res_full, 0, abort));
    for (int pr = 0; pr < n_pairs && ok; ++pr) {
      for (int L = 0; L < 5 && ok; ++L) {
        for (int t = 2 * pr; t < min(2 * pr + 2, my_tiles) && ok; ++t) {
          const int q = t & 1, k = t >> 1;
          const uint32_t acc = tmem + q * kSurHidden;
          const uint32_t in = tc::smem_u32(act + q * kActBytes);
          if (L == 0) {
            ok = __all_sync(0xffffffffu, wait_bar(&feat_full[q], k & 1, abort));
            if (ok && k >= 1) ok = __all_sync(0xffffffffu, wait_bar(&out_free[q], (k - 1) & 1, abort));
            if (!ok) break;
            tc::fence_after_sync();
            tc::mma_bf16_warp(acc, tc::desc_kmajor(tc::smem_u32(x0 + q * kX0Bytes), 128, kSbo16),
                              tc::desc_kmajor(w0, 128, kSbo16), kIdHidden, 0u);
            tc::commit_warp(&x0_free[q]);
            tc::commit_warp(&mma_done[q]);
            continue;
          }
          ok = __all_sync(0xffffffffu, wait_bar(&epi_done[q], (L - 1) & 1, abort));
          if (!ok) break;
          tc::fence_after_sync();
          if (L < 4) {
            for (int g = 0; g < kLayerStages && ok; ++g, ++si) {
              const int slot = si % kStages;
              ok = __all_sync(0xffffffffu, wait_bar(&full[slot], (si / kStages) & 1, abort));
              if (!ok) break;
              tc::fence_after_sync();
              const uint32_t wb = tc::smem_u32(stages + slot * kStageBytes);
#pragma unroll
              for (int c = 0; c < kStageChunks; ++c) {
                const int kc = g * kStageChunks + c;  // K chunk of 16 within the layer
                tc::mma_bf16_warp(acc, tc::desc_kmajor(in + kc * 16 * 16, 128, kSboAct),
                                  tc::desc_kmajor(wb + c * kChunkBytes, 128, kSbo16), kIdHidden,
                                  kc > 0 ? 1u : 0u);
              }
              tc::commit_warp(&empty[slot]);
            }
            if (!ok) break;
            tc::commit_warp(&mma_done[q]);
          } else {
#pragma unroll 4
            for (int kk = 0; kk < kSurHidden / 16; ++kk)
              tc::mma_bf16_warp(acc, tc::desc_kmajor(in + kk * 16 * 16, 128, kSboAct),
                                tc::desc_kmajor(w4 + kk * (kSurOutPad * 16 * 2), 128, kSbo16), kIdOut,
                                kk > 0 ? 1u : 0u);
            tc::commit_warp(&out_done[q]);
          }
        }
      }
    }
    // every MMA issued has completed before the TMEM columns are released
    tc::commit_warp(drain);
    tc::mbar_wait(drain, 0);
  } else if (warp < kEpiWarps) {
    // ---- hidden epilogues, in the MMAs' order: layer L of slot q's k-th
    // tile waits for mma_done phase 4 k + L
    const int quarter = warp & 3, cg = warp >> 2, row = quarter * 32 + lane;
    bool ok = true;
    for (int pr = 0; pr < n_pairs && ok; ++pr) {
      for (int L = 0; L < 4 && ok; ++L) {
        for (int t = 2 * pr; t < min(2 * pr + 2, my_tiles) && ok; ++t) {
          const int q = t & 1;
          ok = __all_sync(0xffffffffu, wait_bar(&mma_done[q], L & 1, abort));
          if (!ok) break;
          tc::fence_after_sync();
          const uint32_t tbase = tmem + q * kSurHidden + (static_cast<uint32_t>(quarter * 32) << 16) + cg * 32;
          const float *bias = sbias + L * kSurHidden + cg * 32;
          uint8_t *actq = act + q * kActBytes;
#pragma unroll 1
          for (int s = 0; s < 2; ++s) {
            uint32_t cur[32];
            tc::tmem_ld32_issue(tbase + s * 128, cur);
            tc::tmem_ld_wait(cur);
#pragma unroll
            for (int c = 0; c < 32; c += 8) {
              const float4 b0 = *reinterpret_cast<const float4 *>(bias + s * 128 + c);
              const float4 b1 = *reinterpret_cast<const float4 *>(bias + s * 128 + c + 4);
              const uint32_t p0 = gelu2_bf16(__uint_as_float(cur[c]) + b0.x, __uint_as_float(cur[c + 1]) + b0.y);
              const uint32_t p1 = gelu2_bf16(__uint_as_float(cur[c + 2]) + b0.z, __uint_as_float(cur[c + 3]) + b0.w);
              const uint32_t p2 = gelu2_bf16(__uint_as_float(cur[c + 4]) + b1.x, __uint_as_float(cur[c + 5]) + b1.y);
              const uint32_t p3 = gelu2_bf16(__uint_as_float(cur[c + 6]) + b1.z, __uint_as_float(cur[c + 7]) + b1.w);
              *reinterpret_cast<uint4 *>(actq + tc::tile_offset(row, s * 128 + cg * 32 + c, kSurHidden)) =
                  make_uint4(p0, p1, p2, p3);
            }
          }
          // the accumulator is read and the activations written: the slot's
          // next MMA may overwrite the one and read the other
          tc::fence_before_sync();
          tc::fence_async_smem();
          __syncwarp();
          if (lane == 0) bar_arrive(&epi_done[q]);
        }
      }
    }
  } else {
    // ---- features of tile it + 2 once tile it's first layer has read the
    // slot's feature buffer, then tile it's outputs
    const int quarter = warp & 3, row = quarter * 32 + lane;
    bool ok = true;
    for (int t = 0; t < min(2, my_tiles); ++t) {
      tile_features<C>(B, P, cell_of((blockIdx.x + static_cast<int64_t>(t) * gridDim.x) * kCells + row), row,
                       x0 + t * kX0Bytes);
      tc::fence_async_smem();
      __syncwarp();
      if (lane == 0) bar_arrive(&feat_full[t]);
    }
    for (int it = 0; it < my_tiles && ok; ++it) {
      const int q = it & 1, k = it >> 1;
      const int64_t tile = blockIdx.x + static_cast<int64_t>(it) * gridDim.x;
      if (it + 2 < my_tiles) {
        ok = __all_sync(0xffffffffu, wait_bar(&x0_free[q], k & 1, abort));
        if (!ok) break;
        tile_features<C>(B, P, cell_of((tile + 2 * static_cast<int64_t>(gridDim.x)) * kCells + row), row,
                         x0 + q * kX0Bytes);
        tc::fence_async_smem();
        __syncwarp();
        if (lane == 0) bar_arrive(&feat_full[q]);
      }
      ok = __all_sync(0xffffffffu, wait_bar(&out_done[q], k & 1, abort));
      if (!ok) break;
      tc::fence_after_sync();
      float o[kSurOutPad];
      tc::tmem_ld16(tmem + q * kSurHidden + (static_cast<uint32_t>(quarter * 32) << 16), o);
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) bar_arrive(&out_free[q]);
      tile_apply<C, MODE, NE>(B, P, cell_of(tile * kCells + row), o, sbias + 4 * kSurHidden, fb_count, fb_list,
                              stats);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 512);
  if (tid == 0 && *abort) atomicExch(err, 1);
  if (tid == 0 && blockIdx.x == 0) {
    if (phase_ctr) atomicAdd(phase_ctr, 1);
    atomicAdd(&stats[2], static_cast<unsigned long long>(n_items));
  }
}

// Cells the inference evaluates this step: those it judged quiet the step
// before, and every cell whose linear index is the step's phase modulo
// `every` (a reacting cell is looked at again within `every` steps; in
// between it keeps the point-implicit chemistry, so no decision goes stale).
// Clears chem_quiet; the cells left out count as EPI fallbacks in stats[1].
template <class C>
__global__ void __launch_bounds__(256) k_sur_candidates(const DevBlock *__restrict__ blks, int b, int every,
                                                        const int *phase_ctr, int *list, int *count,
                                                        unsigned long long *stats) {
  const DevBlock &B = blks[b];
  const int64_t cells = static_cast<int64_t>(B.mx) * B.my * B.mz;
  const int phase = *phase_ctr % every;
  const int lane = threadIdx.x & 31;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t base = static_cast<int64_t>(blockIdx.x) * blockDim.x; base < cells; base += stride) {
    const int64_t c = base + threadIdx.x;
    bool pick = false, valid = c < cells;
    if (valid) {
      const int i = static_cast<int>(c % B.mx), j = static_cast<int>((c / B.mx) % B.my),
                k = static_cast<int>(c / (static_cast<int64_t>(B.mx) * B.my));
      const int64_t nz = B.Z.at(i, j, k);
      pick = B.chem_quiet[nz] != 0 || c % every == phase;
      B.chem_quiet[nz] = 0;
    }
    // one atomic per warp for the list and one for the left-out cells
    const unsigned m = __ballot_sync(0xffffffffu, pick), skip = __ballot_sync(0xffffffffu, valid && !pick);
    int at = 0;
    if (lane == 0) {
      if (m) at = atomicAdd(count, __popc(m));
      if (skip) atomicAdd(&stats[1], static_cast<unsigned long long>(__popc(skip)));
    }
    at = __shfl_sync(0xffffffffu, at, 0);
    if (pick) list[at + __popc(m & ((1u << lane) - 1u))] = static_cast<int>(c);
  }
}

// The judge over the cells the fused inference accepted (the candidate list
// of this step): a cell whose increment (recovered from its rate rho dY / dt)
// the judge refuses goes back to the point-implicit chemistry, and the
// statistics move it from accepted to fallback.  Each warp reads 32
// candidates at a time and queues the accepted ones in shared memory, judging
// 32 queued cells at once, so every lane judges a cell (about half of the
// candidates are accepted).
template <class C>
__global__ void __launch_bounds__(kJudgeCta, 3) k_sur_judge(const DevBlock *__restrict__ blks, int b, SurrogateGate g,
                                                         const int *__restrict__ cand, const int *cand_count,
                                                         unsigned long long *stats) {
  constexpr int NS = C::ns;
  __shared__ int queue[kJudgeCta / 32][64];
  if (g.judge_rel < 0.f) return;
  const DevBlock &B = blks[b];
  const int count = *cand_count;
  const int64_t sz = B.G.size, sz0 = B.Z.size;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int *wq = queue[warp];
  int held = 0;  // queued cells of this warp (warp-uniform)
  auto judge = [&](bool active, int c) {
    if (!active) return;
    const int i = c % B.mx, j = (c / B.mx) % B.my, k = c / (B.mx * B.my);
    const int64_t n = B.G.at(i, j, k), nz = B.Z.at(i, j, k);
    const double rho = B.bv[n], dt = B.dt_local[nz];
    float Y[NS], dy[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      Y[s] = static_cast<float>(B.sv[s * sz + n]);
      dy[s] = static_cast<float>(B.chem_rate[s * sz0 + nz] * dt / rho);
    }
    if (!judge_accepts<NS>(g, static_cast<float>(B.bv[5 * sz + n]), static_cast<float>(B.bv[4 * sz + n]),
                           static_cast<float>(dt), Y, dy)) {
      B.chem_quiet[nz] = 0;
      atomicAdd(&stats[0], ~0ull);  // minus one
      atomicAdd(&stats[1], 1ull);
    }
  };
  const int warps = gridDim.x * (kJudgeCta / 32);
  for (int base = (blockIdx.x * (kJudgeCta / 32) + warp) * 32; base < count; base += warps * 32) {
    const int q = base + lane;
    int c = 0;
    bool acc = false;
    if (q < count) {
      c = cand[q];
      const int i = c % B.mx, j = (c / B.mx) % B.my, k = c / (B.mx * B.my);
      acc = B.chem_quiet[B.Z.at(i, j, k)] != 0;
    }
    const unsigned m = __ballot_sync(0xffffffffu, acc);
    if (acc) wq[held + __popc(m & ((1u << lane) - 1u))] = c;
    held += __popc(m);
    __syncwarp();
    if (held >= 32) {
      const int cell = wq[lane];
      __syncwarp();
      if (lane < held - 32) wq[lane] = wq[32 + lane];
      held -= 32;
      __syncwarp();
      judge(true, cell);
    }
  }
  __syncwarp();
  judge(lane < held, lane < held ? wq[lane] : 0);
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
