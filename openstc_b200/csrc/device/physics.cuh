// Per-point physics of the FP64 path, templated on the model configuration
// so that species loops unroll into registers.  Each function keeps the
// operation order of the reference function it restates (cited), which is
// what lets the FP64 path track the reference's CUDA build bit for bit where
// the compiler contracts the same expressions the same way.
//
// The reference compiles its thermodynamic functions in their own
// translation unit, so their outputs reach the callers already rounded.
// These functions are inlined here; their final scaling uses __dmul_rn so
// that no caller can fuse it into an FMA (cp - R/W, cp + 1.25 R/W, ...),
// which keeps the callers' arithmetic identical to the reference's.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

#include "common.cuh"

namespace ostc {

// One copy per translation unit; the engine uploads it through the TU's
// set_params() entry.
static __constant__ DevParams cP;

template <int MIX, int TURB, int NS, bool MIXED = false>
struct Cfg {
  static constexpr int mix = MIX;    // 0 air, 1 mixture, 2 finite-rate chemistry
  static constexpr int turb = TURB;  // 0 laminar, 1 k-omega SST
  static constexpr int ns = NS;
  static constexpr bool mixed = MIXED;  // FP32-bulk / FP64-critical kernels
  static constexpr int nsc = NS + (TURB ? 2 : 0);
  static constexpr int nv = 5 + nsc;
};

#define OSTC_UNROLL _Pragma("unroll")

__device__ __forceinline__ double ld(const double *p) { return __ldg(p); }

// ------------------------------------------------------------------ thermo
// NASA-7 coefficient q of species i at temperature t (two ranges).
__device__ __forceinline__ double nasa(int i, int q, bool lowrange) {
  return lowrange ? cP.low[i * 7 + q] : cP.high[i * 7 + q];
}

// compute_enthalpy, src/Thermo.cu:5-23
template <int NS>
__device__ __forceinline__ void enthalpy(double t, double *h) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  OSTC_UNROLL for (int i = 0; i < NS; ++i) {
    if (t < cP.t_low[i]) {
      const double tt = cP.t_low[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
      const double c0 = cP.low[i * 7], c1 = cP.low[i * 7 + 1], c2 = cP.low[i * 7 + 2], c3 = cP.low[i * 7 + 3],
                   c4 = cP.low[i * 7 + 4], c5 = cP.low[i * 7 + 5];
      h[i] = c0 * tt + 0.5 * c1 * tt2 + c2 * tt3 / 3 + 0.25 * c3 * tt4 + 0.2 * c4 * tt5 + c5;
      const double cp = c0 + c1 * tt + c2 * tt2 + c3 * tt3 + c4 * tt4;
      h[i] += cp * (t - tt);
    } else {
      const bool lo = t < cP.t_mid[i];
      h[i] = nasa(i, 0, lo) * t + 0.5 * nasa(i, 1, lo) * t2 + nasa(i, 2, lo) * t3 / 3 + 0.25 * nasa(i, 3, lo) * t4 +
             0.2 * nasa(i, 4, lo) * t5 + nasa(i, 5, lo);
    }
    h[i] = __dmul_rn(h[i], cP.ru_mw[i]);
  }
}

// compute_enthalpy_and_cp, src/Thermo.cu:25-45
template <int NS>
__device__ __forceinline__ void enthalpy_cp(double t, double *h, double *cp) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  OSTC_UNROLL for (int i = 0; i < NS; ++i) {
    if (t < cP.t_low[i]) {
      const double tt = cP.t_low[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
      const double c0 = cP.low[i * 7], c1 = cP.low[i * 7 + 1], c2 = cP.low[i * 7 + 2], c3 = cP.low[i * 7 + 3],
                   c4 = cP.low[i * 7 + 4], c5 = cP.low[i * 7 + 5];
      h[i] = c0 * tt + 0.5 * c1 * tt2 + c2 * tt3 / 3 + 0.25 * c3 * tt4 + 0.2 * c4 * tt5 + c5;
      cp[i] = c0 + c1 * tt + c2 * tt2 + c3 * tt3 + c4 * tt4;
      h[i] += cp[i] * (t - tt);
    } else {
      const bool lo = t < cP.t_mid[i];
      h[i] = nasa(i, 0, lo) * t + 0.5 * nasa(i, 1, lo) * t2 + nasa(i, 2, lo) * t3 / 3 + 0.25 * nasa(i, 3, lo) * t4 +
             0.2 * nasa(i, 4, lo) * t5 + nasa(i, 5, lo);
      cp[i] = nasa(i, 0, lo) + nasa(i, 1, lo) * t + nasa(i, 2, lo) * t2 + nasa(i, 3, lo) * t3 + nasa(i, 4, lo) * t4;
    }
    h[i] = __dmul_rn(h[i], cP.ru_mw[i]);
    cp[i] = __dmul_rn(cp[i], cP.ru_mw[i]);
  }
}

// compute_cp, src/Thermo.cu:47-61
template <int NS>
__device__ __forceinline__ void heat_capacity(double t, double *cp) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t;
  OSTC_UNROLL for (int i = 0; i < NS; ++i) {
    if (t < cP.t_low[i]) {
      const double tt = cP.t_low[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt;
      cp[i] = cP.low[i * 7] + cP.low[i * 7 + 1] * tt + cP.low[i * 7 + 2] * tt2 + cP.low[i * 7 + 3] * tt3 +
              cP.low[i * 7 + 4] * tt4;
    } else {
      const bool lo = t < cP.t_mid[i];
      cp[i] = nasa(i, 0, lo) + nasa(i, 1, lo) * t + nasa(i, 2, lo) * t2 + nasa(i, 3, lo) * t3 + nasa(i, 4, lo) * t4;
    }
    cp[i] = __dmul_rn(cp[i], cP.ru_mw[i]);
  }
}

// compute_gibbs_div_rt, src/Thermo.cu:63-79
template <int NS>
__device__ __forceinline__ void gibbs_rt(double t, double *g) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t_inv = 1 / t, log_t = std::log(t);
  OSTC_UNROLL for (int i = 0; i < NS; ++i) {
    if (t < cP.t_low[i]) {
      const double tt = cP.t_low[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt_inv = 1 / tt, log_tt = std::log(tt);
      const double *c = &cP.low[i * 7];
      g[i] = c[0] * (1.0 - log_tt) - 0.5 * c[1] * tt - c[2] * tt2 / 6.0 - c[3] * tt3 / 12.0 - c[4] * tt4 * 0.05 +
             c[5] * tt_inv - c[6];
    } else {
      const bool lo = t < cP.t_mid[i];
      g[i] = nasa(i, 0, lo) * (1.0 - log_t) - 0.5 * nasa(i, 1, lo) * t - nasa(i, 2, lo) * t2 / 6.0 -
             nasa(i, 3, lo) * t3 / 12.0 - nasa(i, 4, lo) * t4 * 0.05 + nasa(i, 5, lo) * t_inv - nasa(i, 6, lo);
    }
  }
}

// gibbs_rt for the FP32-bulk path: the same polynomials with ln T and 1 / T
// passed in and the constant divisors as products (within an ulp or two).
template <int NS>
__device__ __forceinline__ void gibbs_rt_fast(double t, double log_t, double t_inv, double *g) {
  constexpr double k6 = 1.0 / 6.0, k12 = 1.0 / 12.0;
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t;
  OSTC_UNROLL for (int i = 0; i < NS; ++i) {
    if (t < cP.t_low[i]) {
      const double tt = cP.t_low[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt_inv = 1 / tt, log_tt = std::log(tt);
      const double *c = &cP.low[i * 7];
      g[i] = c[0] * (1.0 - log_tt) - 0.5 * c[1] * tt - c[2] * tt2 * k6 - c[3] * tt3 * k12 - c[4] * tt4 * 0.05 +
             c[5] * tt_inv - c[6];
    } else {
      const bool lo = t < cP.t_mid[i];
      g[i] = nasa(i, 0, lo) * (1.0 - log_t) - 0.5 * nasa(i, 1, lo) * t - nasa(i, 2, lo) * t2 * k6 -
             nasa(i, 3, lo) * t3 * k12 - nasa(i, 4, lo) * t4 * 0.05 + nasa(i, 5, lo) * t_inv - nasa(i, 6, lo);
    }
  }
}

// ------------------------------------------------------------------ transport
// Sutherland, src/Transport.cu:6-9
__device__ __forceinline__ double sutherland(double t) {
  return 1.716e-5 * std::pow(t / 273, 1.5) * (273 + 111) / (t + 111);
}

// Pure-species viscosities and mole fractions, src/Transport.cu:46-52
template <int NS>
__device__ __forceinline__ void species_viscosity(double t, double mw_total, const double *Y, double *X, double *vis) {
  const double st = sqrt(t);
  OSTC_UNROLL for (int l = 0; l < NS; ++l) {
    X[l] = Y[l] * mw_total / cP.mw[l];
    const double t_dl = t * cP.lj_inv[l];
    const double ci = 1.147 * std::pow(t_dl, -0.145) + std::pow(t_dl + 0.5, -2);
    vis[l] = cP.vis_coeff[l] * st / ci;
  }
}

// Wilke's mixing rule denominator for species m, src/Transport.cu:57-66
template <int NS>
__device__ __forceinline__ double wilke_sum(const double *vis, const double *X, int m) {
  double vt = 0;
  OSTC_UNROLL for (int n = 0; n < NS; ++n) {
    double phi = 1.0;
    if (m != n) {
      const double num = 1 + sqrt(vis[m] / vis[n]) * cP.wq[m * NS + n];
      phi = num * num * cP.w8[m * NS + n];
    }
    vt += phi * X[n];
  }
  return vt;
}

// compute_viscosity (device), src/Transport.cu:86-115
template <int NS>
__device__ __forceinline__ double mixture_viscosity(double t, double mw_total, const double *Y) {
  double X[NS > 0 ? NS : 1], vis[NS > 0 ? NS : 1];
  species_viscosity<NS>(t, mw_total, Y, X, vis);
  double viscosity = 0;
  OSTC_UNROLL for (int m = 0; m < NS; ++m) viscosity += vis[m] * X[m] / wilke_sum<NS>(vis, X, m);
  return viscosity;
}

// ------------------------------------------------------------------ limiter
__device__ __forceinline__ double minmod(double a, double b) {
  // src/Limiter.cuh:13-16
  return 0.5 * ((a < 0 ? -1 : 1) + (b < 0 ? -1 : 1)) * fmin(fabs(a), fabs(b));
}

}  // namespace ostc
