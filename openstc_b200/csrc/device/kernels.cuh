// sm_100a kernels of the FP64 residual / implicit / update path.
//
// Included once per model configuration (see engine_*.cu).  All per-cell
// kernels take a Tiles work table so one launch covers every grid block.
#pragma once

#include "physics.cuh"

namespace ostc {

// SST model constants, src/SST.cuh:10-31
namespace sst {
constexpr double beta_star = 0.09, sqrt_beta_star = 0.3, kappa = 0.41;
constexpr double sigma_k1 = 0.85, sigma_omega1 = 0.5, beta_1 = 0.0750, a_1 = 0.31;
constexpr double gamma1 = beta_1 / beta_star - sigma_omega1 * kappa * kappa / sqrt_beta_star;
constexpr double sigma_k2 = 1, sigma_omega2 = 0.856, beta_2 = 0.0828;
constexpr double gamma2 = beta_2 / beta_star - sigma_omega2 * kappa * kappa / sqrt_beta_star;
constexpr double delta_sigma_k = sigma_k1 - sigma_k2, delta_sigma_omega = sigma_omega1 - sigma_omega2;
constexpr double delta_beta = beta_1 - beta_2, delta_gamma = gamma1 - gamma2;
}  // namespace sst

// ---------------------------------------------------------------- tiling
template <int TX, int TY, int TZ>
__device__ __forceinline__ bool tile_cell(const Tiles &T, int &b, int &i, int &j, int &k, const DevBlock *blks) {
  int t = tile_of(T, blockIdx.x, b);
  const int tx = t % T.ntx[b];
  t /= T.ntx[b];
  const int ty = t % T.nty[b];
  const int tz = t / T.nty[b];
  i = tx * TX + static_cast<int>(threadIdx.x) - T.halo;
  j = ty * TY + static_cast<int>(threadIdx.y) - T.halo;
  k = tz * TZ + static_cast<int>(threadIdx.z) - T.halo;
  const DevBlock &B = blks[b];
  return i < B.mx + T.halo && j < B.my + T.halo && k < B.mz + T.halo;
}

// ---------------------------------------------------------------- SST source
// SST::compute_source_and_mut, src/SST.cu:60-178 (gradients by central
// differences through the metric).  Returns the two source terms times J.
template <class C>
__device__ __forceinline__ void sst_source(const DevBlock &B, int64_t n, double &src_k, double &src_w, double &mut_out,
                                           double &jk, double &jw) {
  constexpr int NS = C::ns;
  const int64_t sz = B.G.size, sx = B.G.sx, sxy = B.G.sxy;
  const double *m = B.metric;
  const double xi_x = ld(m + n), xi_y = ld(m + sz + n), xi_z = ld(m + 2 * sz + n);
  const double eta_x = ld(m + 3 * sz + n), eta_y = ld(m + 4 * sz + n), eta_z = ld(m + 5 * sz + n);
  const double zeta_x = ld(m + 6 * sz + n), zeta_y = ld(m + 7 * sz + n), zeta_z = ld(m + 8 * sz + n);
  auto cgrad = [&](const double *a, double cx, double cy, double cz) {
    return 0.5 * (cx * (ld(a + n + 1) - ld(a + n - 1)) + cy * (ld(a + n + sx) - ld(a + n - sx)) +
                  cz * (ld(a + n + sxy) - ld(a + n - sxy)));
  };
  const double *u = B.bv + sz, *v = B.bv + 2 * sz, *w = B.bv + 3 * sz;
  const double u_x = cgrad(u, xi_x, eta_x, zeta_x), u_y = cgrad(u, xi_y, eta_y, zeta_y),
               u_z = cgrad(u, xi_z, eta_z, zeta_z);
  const double v_x = cgrad(v, xi_x, eta_x, zeta_x), v_y = cgrad(v, xi_y, eta_y, zeta_y),
               v_z = cgrad(v, xi_z, eta_z, zeta_z);
  const double w_x = cgrad(w, xi_x, eta_x, zeta_x), w_y = cgrad(w, xi_y, eta_y, zeta_y),
               w_z = cgrad(w, xi_z, eta_z, zeta_z);
  const double density = ld(B.bv + n);
  const double *tk = B.sv + NS * sz, *tw = B.sv + (NS + 1) * sz;
  const double omega = ld(tw + n);
  const double k_x = cgrad(tk, xi_x, eta_x, zeta_x), k_y = cgrad(tk, xi_y, eta_y, zeta_y),
               k_z = cgrad(tk, xi_z, eta_z, zeta_z);
  const double omega_x = cgrad(tw, xi_x, eta_x, zeta_x), omega_y = cgrad(tw, xi_y, eta_y, zeta_y),
               omega_z = cgrad(tw, xi_z, eta_z, zeta_z);
  const double inter_var = 2 * density * sst::sigma_omega2 / omega * (k_x * omega_x + k_y * omega_y + k_z * omega_z);
  const double tke = ld(tk + n);
  const double rhoK = density * tke;
  const double vorticity = sqrt((v_x - u_y) * (v_x - u_y) + (w_x - u_z) * (w_x - u_z) + (w_y - v_z) * (w_y - v_z));
  double f1 = 1, f2 = 1;
  const double dy = ld(B.wall_dist + n);
  if (dy > 1e-25) {
    const double param1 = sqrt(tke) / (0.09 * omega * dy);
    const double d2 = dy * dy;
    const double param2 = 500 * ld(B.mul + n) / (density * d2 * omega);
    const double arg2 = fmax(2 * param1, param2);
    f2 = tanh(arg2 * arg2);
    const double CDkomega = fmax(1e-20, inter_var);
    const double param3 = 4 * density * sst::sigma_omega2 * tke / (CDkomega * d2);
    const double arg1 = fmin(fmax(param1, param2), param3);
    f1 = tanh(arg1 * arg1 * arg1 * arg1);
  }
  double mut = 0;
  if (const double den = fmax(sst::a_1 * omega, vorticity * f2); den > 1e-25) mut = sst::a_1 * rhoK / den;
  mut_out = mut;
  const double beta = sst::beta_2 + sst::delta_beta * f1;
  src_k = 0;
  src_w = 0;
  if (mut > 1e-25) {
    const double divU = u_x + v_y + w_z;
    const double divU2 = divU * divU;
    const double prod_k = mut * (2 * (u_x * u_x + v_y * v_y + w_z * w_z) - 2.0 / 3 * divU2 + (u_y + v_x) * (u_y + v_x) +
                                 (u_z + w_x) * (u_z + w_x) + (v_z + w_y) * (v_z + w_y)) -
                          2.0 / 3 * rhoK * divU;
    const double diss_k = sst::beta_star * rhoK * omega;
    const double jac = ld(B.jac + n);
    src_k = 0.0 + jac * (prod_k - diss_k);
    const double gamma = sst::gamma2 + sst::delta_gamma * f1;
    const double prod_omega = gamma * density / mut * prod_k + (1 - f1) * inter_var;
    const double diss_omega = beta * density * omega * omega;
    src_w = 0.0 + jac * (prod_omega - diss_omega);
  }
  jk = -2 * sst::beta_star * omega;
  jw = -2 * beta * omega;
}

// SST::compute_mut, src/SST.cu:6-58 (initialisation only)
template <class C>
__device__ __forceinline__ double sst_mut(const DevBlock &B, int64_t n, double mul) {
  constexpr int NS = C::ns;
  const int64_t sz = B.G.size, sx = B.G.sx, sxy = B.G.sxy;
  const double *m = B.metric;
  const double xi_x = ld(m + n), xi_y = ld(m + sz + n), xi_z = ld(m + 2 * sz + n);
  const double eta_x = ld(m + 3 * sz + n), eta_y = ld(m + 4 * sz + n), eta_z = ld(m + 5 * sz + n);
  const double zeta_x = ld(m + 6 * sz + n), zeta_y = ld(m + 7 * sz + n), zeta_z = ld(m + 8 * sz + n);
  auto cgrad = [&](const double *a, double cx, double cy, double cz) {
    return 0.5 * (cx * (ld(a + n + 1) - ld(a + n - 1)) + cy * (ld(a + n + sx) - ld(a + n - sx)) +
                  cz * (ld(a + n + sxy) - ld(a + n - sxy)));
  };
  const double *u = B.bv + sz, *v = B.bv + 2 * sz, *w = B.bv + 3 * sz;
  const double u_y = cgrad(u, xi_y, eta_y, zeta_y), u_z = cgrad(u, xi_z, eta_z, zeta_z);
  const double v_x = cgrad(v, xi_x, eta_x, zeta_x), v_z = cgrad(v, xi_z, eta_z, zeta_z);
  const double w_x = cgrad(w, xi_x, eta_x, zeta_x), w_y = cgrad(w, xi_y, eta_y, zeta_y);
  const double rhoK = B.cv[(NS + 5) * sz + n];
  const double tke = B.sv[NS * sz + n];
  const double omega = B.sv[(NS + 1) * sz + n];
  const double vorticity = sqrt((v_x - u_y) * (v_x - u_y) + (w_x - u_z) * (w_x - u_z) + (w_y - v_z) * (w_y - v_z));
  const double density = B.bv[n];
  double f2 = 1;
  const double dy = B.wall_dist[n];
  if (dy > 1e-25) {
    const double param1 = 2 * sqrt(tke) / (0.09 * omega * dy);
    const double param2 = 500 * mul / (density * dy * dy * omega);
    const double arg2 = fmax(param1, param2);
    f2 = tanh(arg2 * arg2);
  }
  double mut = 0;
  if (const double den = fmax(sst::a_1 * omega, vorticity * f2); den > 1e-25) mut = sst::a_1 * rhoK / den;
  return mut;
}

// ---------------------------------------------------------------- chemistry
// A T^b exp(-Ea/T) evaluated as (A T^b) exp(-Ea/T), src/FiniteRateChem.cu:110-112.
// pow(T, 0) and exp(-0/T) are exactly 1, so those calls are skipped without
// changing a bit of the result.
__device__ __forceinline__ double arrhenius_pow(double t, double A, double b) {
  return b != 0 ? A * std::pow(t, b) : A;
}

__device__ __forceinline__ double arrhenius(double t, double A, double b, double Ea) {
  const double ab = arrhenius_pow(t, A, b);
  return Ea != 0 ? ab * std::exp(-Ea / t) : ab;
}

#ifndef OSTC_DUP_FMA
#define OSTC_DUP_FMA 1
#endif

// The same rate as one exponential, sign(A) exp(ln|A| + b ln T - Ea / T), for
// the FP32-bulk path (FP64 throughout, within a few ulps of arrhenius).
__device__ __forceinline__ double arrhenius_exp(double A, double lnA, double b, double Ea, double ln_t, double t_inv) {
  return A == 0 ? 0.0 : copysign(std::exp(lnA + b * ln_t - Ea * t_inv), A);
}

// c^e for a stoichiometric exponent: products for 1..3, pow otherwise.
__device__ __forceinline__ double ipow(double c, int e) {
  return e == 1 ? c : (e == 2 ? c * c : (e == 3 ? c * c * c : std::pow(c, e)));
}

// finite_rate_chemistry, src/FiniteRateChem.cu:7-63 with the rate helpers
// :65-171.  q1/q2 live in shared memory with stride `st` (CTA size).
// FAST (the FP32-bulk path, FP64 arithmetic within a few ulps of the
// reference form): every Arrhenius rate and every K_c as one exponential,
// integer concentration powers as products, the Troe 10^x as an exponential
// and the Gibbs polynomials without divisions; the FP64 path keeps the
// reference's form bit for bit.
template <int NS, bool FAST = false>
__device__ __forceinline__ void chemistry(double density, double t, const double *Y, double *omega, double *omega_d,
                                         double *q1, double *q2, int st) {
  const double ln_t = FAST ? std::log(t) : 0.0, t_inv = FAST ? 1.0 / t : 0.0;
  auto rate1 = [&](int r) { return FAST ? arrhenius_exp(cP.A[r], cP.lnA[r], cP.b[r], cP.Ea[r], ln_t, t_inv)
                                        : arrhenius(t, cP.A[r], cP.b[r], cP.Ea[r]); };
  auto rate2 = [&](int r) { return FAST ? arrhenius_exp(cP.A2[r], cP.lnA2[r], cP.b2[r], cP.Ea2[r], ln_t, t_inv)
                                        : arrhenius(t, cP.A2[r], cP.b2[r], cP.Ea2[r]); };
  double c[NS];
  OSTC_UNROLL for (int l = 0; l < NS; ++l) c[l] = density * Y[l] / cP.mw[l] * 1e-3;
  double g[NS];
  if constexpr (FAST)
    gibbs_rt_fast<NS>(t, ln_t, t_inv, g);
  else
    gibbs_rt<NS>(t, g);
  constexpr double temp_p = kDP_atm / kDR_u * 1e-3;
  const double temp_t = temp_p / t;
  // FAST: ln(temp_p / T), for K_c as one exponential
  const double ln_temp_t = FAST ? std::log(temp_p) - ln_t : 0.0;
  const int nr = cP.nr;
  for (int r = 0; r < nr; ++r) {
    const int type = cP.label[r];
    double kf = rate1(r);
    if (type == 3) {
      if constexpr (FAST) {
        kf += rate2(r);
      } else {
        // duplicate reaction: the reference adds the second rate in a new
        // basic block, so only its last product can fuse into the sum
#if OSTC_DUP_FMA
        const double e2 = cP.Ea2[r] != 0 ? std::exp(-cP.Ea2[r] / t) : 1.0;
        kf = __fma_rn(arrhenius_pow(t, cP.A2[r], cP.b2[r]), e2, kf);
#else
        kf = __dadd_rn(kf, arrhenius(t, cP.A2[r], cP.b2[r], cP.Ea2[r]));
#endif
      }
    }
    if (type > 3) {
      double cc = 0;
      OSTC_UNROLL for (int l = 0; l < NS; ++l) cc += c[l] * cP.tb[r * NS + l];
      if (type == 4) {
        kf *= cc;
      } else {
        const double kf_low = rate2(r);
        const double kf_high = kf;
        const double reduced_pressure = kf_low * cc / kf_high;
        double F = 1.0;
        if (type > 5) {
          double f_cent = (1 - cP.troe_a[r]) * std::exp(-t / cP.troe_t3[r]) + cP.troe_a[r] * std::exp(-t / cP.troe_t1[r]);
          if (type == 7) f_cent += std::exp(-cP.troe_t2[r] / t);
          const double logFc = std::log10(f_cent);
          const double cq = -0.4 - 0.67 * logFc;
          const double nq = 0.75 - 1.27 * logFc;
          const double logPr = std::log10(reduced_pressure);
          const double tempo = (logPr + cq) / (nq - 0.14 * (logPr + cq));
          const double pq = logFc / (1.0 + tempo * tempo);
          F = FAST ? std::exp(pq * 2.302585092994045684) : std::pow(10, pq);
        }
        kf = kf_high * reduced_pressure / (1.0 + reduced_pressure) * F;
      }
    }
    double kb;
    if (type != 2) {
      double d_gibbs = 0;
      OSTC_UNROLL for (int l = 0; l < NS; ++l) d_gibbs += g[l] * (cP.sb[r * NS + l] - cP.sf[r * NS + l]);
      if constexpr (FAST) {
        // kf / K_c with K_c = (p_atm / R T)^order exp(-dG / RT) as one exponential
        kb = kf * std::exp(d_gibbs - cP.order[r] * ln_temp_t);
      } else {
        const double kc = std::pow(temp_t, cP.order[r]) * std::exp(-d_gibbs);
        kb = kf / kc;
      }
    } else {
      kb = rate2(r);
    }
    // rate_of_progress: pow(c, 0) is exactly one, so zero exponents are skipped.
    double a1 = 1.0, a2 = 1.0;
    OSTC_UNROLL for (int j = 0; j < NS; ++j) {
      const int ef = cP.sf[r * NS + j], eb = cP.sb[r * NS + j];
      if constexpr (FAST) {  // integer powers by products
        if (ef != 0) a1 *= ipow(c[j], ef);
        if (eb != 0) a2 *= ipow(c[j], eb);
      } else {
        if (ef != 0) a1 *= std::pow(c[j], ef);
        if (eb != 0) a2 *= std::pow(c[j], eb);
      }
    }
    a1 *= kf;
    a2 *= kb;
    q1[r * st] = a1;
    q2[r * st] = a2;
  }
  // chemical_source, src/FiniteRateChem.cu:155-171
  OSTC_UNROLL for (int i = 0; i < NS; ++i) {
    double creation = 0, od = 0;
    for (int r = 0; r < nr; ++r) {
      const double a1 = q1[r * st], a2 = q2[r * st];
      const int f = cP.sf[r * NS + i], bb = cP.sb[r * NS + i];
      creation += a2 * f + a1 * bb;
      od += a1 * f + a2 * bb;
    }
    creation *= cP.mw[i] * 1e+3;
    od *= cP.mw[i] * 1e+3;
    omega_d[i] = od;
    omega[i] = creation - od;
  }
}

// ---------------------------------------------------------------- inviscid
// reconstruction + AUSM+ face flux between the points n and n+s along
// direction D, src/InviscidScheme.cuh:21-149, src/Reconstruction.cu:5-46.
// The direction d (0 xi, 1 eta, 2 zeta) and its index stride s are run-time
// values so that one copy of the face code serves all faces of a cell.
template <class C>
__device__ __forceinline__ void inviscid_face(const DevBlock &B, int64_t n, int d, int64_t s, double *fc) {
  constexpr int NV = C::nv, NS = C::ns;
  const int64_t sz = B.G.size;
  double pl[NV + 2], pr[NV + 2];
  const int rec = cP.reconstruction;
  OSTC_UNROLL for (int l = 0; l < NV; ++l) {
    const double *a = l < 5 ? B.bv + l * sz : B.sv + (l - 5) * sz;
    const double p0 = ld(a + n), p1 = ld(a + n + s);
    if (rec == 2 || rec == 3) {
      const double pm = ld(a + n - s), p2 = ld(a + n + 2 * s);
      const double d_i = p0 - pm, d_i1 = p1 - p0, d_i2 = p2 - p1;
      if (rec == 2) {
        constexpr double kappa = 1.0 / 3.0;
        const double neg_l = minmod(d_i, d_i1), pos_l = minmod(d_i1, d_i);
        const double neg_r = minmod(d_i1, d_i2), pos_r = minmod(d_i2, d_i1);
        pl[l] = p0 + 0.25 * ((1 - kappa) * neg_l + (1 + kappa) * pos_l);
        pr[l] = p1 - 0.25 * ((1 - kappa) * pos_r + (1 + kappa) * neg_r);
      } else {
        pl[l] = p0 + 0.5 * minmod(d_i, d_i1);
        pr[l] = p1 - 0.5 * minmod(d_i1, d_i2);
      }
    } else {
      pl[l] = p0;
      pr[l] = p1;
    }
  }
  if constexpr (C::mix != 0) {
    double el = 0.5 * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]);
    double er = 0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]);
    double mwl = 0, mwr = 0;
    OSTC_UNROLL for (int l = 0; l < NS; ++l) {
      mwl += pl[5 + l] / cP.mw[l];
      mwr += pr[5 + l] / cP.mw[l];
    }
    const double tl = pl[4] / (pl[0] * kDR_u * mwl);
    const double tr = pr[4] / (pr[0] * kDR_u * mwr);
    double hl[NS], hr[NS], cpl_i[NS], cpr_i[NS];
    enthalpy_cp<NS>(tl, hl, cpl_i);
    enthalpy_cp<NS>(tr, hr, cpr_i);
    double cpl = 0, cpr = 0, cvl = 0, cvr = 0;
    OSTC_UNROLL for (int l = 0; l < NS; ++l) {
      cpl += cpl_i[l] * pl[l + 5];
      cpr += cpr_i[l] * pr[l + 5];
      cvl += pl[l + 5] * (cpl_i[l] - cP.ru_mw[l]);
      cvr += pr[l + 5] * (cpr_i[l] - cP.ru_mw[l]);
      el += hl[l] * pl[l + 5];
      er += hr[l] * pr[l + 5];
    }
    pl[NV] = pl[0] * el - pl[4];
    pr[NV] = pr[0] * er - pr[4];
    pl[NV + 1] = cpl / cvl;
    pr[NV + 1] = cpr / cvr;
  } else {
    const double el = 0.5 * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]);
    const double er = 0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]);
    pl[NV] = el * pl[0] + pl[4] / (kDGammaAir - 1);
    pr[NV] = er * pr[0] + pr[4] / (kDGammaAir - 1);
  }
  const double *m = B.metric + 3 * d * sz;
  const double jl = ld(B.jac + n), jr = ld(B.jac + n + s);
  const double k1 = 0.5 * (jl * ld(m + n) + jr * ld(m + n + s));
  const double k2 = 0.5 * (jl * ld(m + sz + n) + jr * ld(m + sz + n + s));
  const double k3 = 0.5 * (jl * ld(m + 2 * sz + n) + jr * ld(m + 2 * sz + n + s));
  const double gk = sqrt(k1 * k1 + k2 * k2 + k3 * k3);
  const double ul = (k1 * pl[1] + k2 * pl[2] + k3 * pl[3]) / gk;
  const double ur = (k1 * pr[1] + k2 * pr[2] + k3 * pr[3]) / gk;
  const double p_l = pl[4], p_r = pr[4], rho_l = pl[0], rho_r = pr[0];
  double gam_l = kDGammaAir, gam_r = kDGammaAir;
  if constexpr (NS > 0) {
    gam_l = pl[NV + 1];
    gam_r = pr[NV + 1];
  }
  const double c = 0.5 * (sqrt(gam_l * p_l / rho_l) + sqrt(gam_r * p_r / rho_r));
  const double mach_l = ul / c, mach_r = ur / c;
  double mlp, mrn, plp, prn;
  constexpr double alpha = 3 / 16.0;
  if (fabs(mach_l) > 1) {
    mlp = 0.5 * (mach_l + fabs(mach_l));
    plp = mlp / mach_l;
  } else {
    const double a = (mach_l + 1) * (mach_l + 1) * 0.25;
    const double b = (mach_l * mach_l - 1) * (mach_l * mach_l - 1);
    mlp = a + 0.125 * b;
    plp = a * (2 - mach_l) + alpha * mach_l * b;
  }
  if (fabs(mach_r) > 1) {
    mrn = 0.5 * (mach_r - fabs(mach_r));
    prn = mrn / mach_r;
  } else {
    const double a = (mach_r - 1) * (mach_r - 1) * 0.25;
    const double b = (mach_r * mach_r - 1) * (mach_r * mach_r - 1);
    mrn = -a - 0.125 * b;
    prn = a * (2 + mach_r) - alpha * mach_r * b;
  }
  const double p_coeff = plp * p_l + prn * p_r;
  const double m_half = mlp + mrn;
  const double mach_pos = 0.5 * (m_half + fabs(m_half));
  const double mach_neg = 0.5 * (m_half - fabs(m_half));
  const double mass_flux_half = c * (rho_l * mach_pos + rho_r * mach_neg);
  // The reference stores each face flux (shared memory) before the cell
  // differences; rounding the bare products here keeps the compiler from
  // fusing them into those differences.
  const double coeff = __dmul_rn(mass_flux_half, gk);
  const bool up = mass_flux_half >= 0;
  fc[0] = coeff;
  fc[1] = coeff * (up ? pl[1] : pr[1]) + p_coeff * k1;
  fc[2] = coeff * (up ? pl[2] : pr[2]) + p_coeff * k2;
  fc[3] = coeff * (up ? pl[3] : pr[3]) + p_coeff * k3;
  fc[4] = up ? coeff * (pl[NV] + pl[4]) / pl[0] : coeff * (pr[NV] + pr[4]) / pr[0];
  OSTC_UNROLL for (int l = 5; l < NV; ++l) fc[l] = __dmul_rn(coeff, up ? pl[l] : pr[l]);
}

// ---------------------------------------------------------------- viscous
// compute_{fv,gv,hv}_2nd_order, src/ViscousScheme.cuh:22-613, for the face
// between n and n1 = n + e_D.
// Derivatives along xi, eta, zeta at the face between n and n1 = n + e_d:
// the face-normal one by a two-point difference, the others by the
// four-point average.
__device__ __forceinline__ void face_grad(const double *a, int64_t n, int64_t n1, int d, int64_t sx, int64_t sxy,
                                          double &dxi, double &deta, double &dzeta) {
  if (d == 0) {
    dxi = ld(a + n1) - ld(a + n);
  } else {
    dxi = 0.25 * (ld(a + n + 1) - ld(a + n - 1) + ld(a + n1 + 1) - ld(a + n1 - 1));
  }
  if (d == 1) {
    deta = ld(a + n1) - ld(a + n);
  } else {
    deta = 0.25 * (ld(a + n + sx) - ld(a + n - sx) + ld(a + n1 + sx) - ld(a + n1 - sx));
  }
  if (d == 2) {
    dzeta = ld(a + n1) - ld(a + n);
  } else {
    dzeta = 0.25 * (ld(a + n + sxy) - ld(a + n - sxy) + ld(a + n1 + sxy) - ld(a + n1 - sxy));
  }
}

template <class C>
__device__ __forceinline__ void viscous_face(const DevBlock &B, int64_t n, int d, int64_t s, double *fv) {
  constexpr int NS = C::ns;
  const int64_t sz = B.G.size, sx = B.G.sx, sxy = B.G.sxy;
  const int64_t n1 = n + s;
  const double *m = B.metric;
  const double xi_x = 0.5 * (ld(m + n) + ld(m + n1));
  const double xi_y = 0.5 * (ld(m + sz + n) + ld(m + sz + n1));
  const double xi_z = 0.5 * (ld(m + 2 * sz + n) + ld(m + 2 * sz + n1));
  const double eta_x = 0.5 * (ld(m + 3 * sz + n) + ld(m + 3 * sz + n1));
  const double eta_y = 0.5 * (ld(m + 4 * sz + n) + ld(m + 4 * sz + n1));
  const double eta_z = 0.5 * (ld(m + 5 * sz + n) + ld(m + 5 * sz + n1));
  const double zeta_x = 0.5 * (ld(m + 6 * sz + n) + ld(m + 6 * sz + n1));
  const double zeta_y = 0.5 * (ld(m + 7 * sz + n) + ld(m + 7 * sz + n1));
  const double zeta_z = 0.5 * (ld(m + 8 * sz + n) + ld(m + 8 * sz + n1));
  double u_xi, u_eta, u_zeta, v_xi, v_eta, v_zeta, w_xi, w_eta, w_zeta, t_xi, t_eta, t_zeta;
  face_grad(B.bv + sz, n, n1, d, sx, sxy, u_xi, u_eta, u_zeta);
  face_grad(B.bv + 2 * sz, n, n1, d, sx, sxy, v_xi, v_eta, v_zeta);
  face_grad(B.bv + 3 * sz, n, n1, d, sx, sxy, w_xi, w_eta, w_zeta);
  face_grad(B.bv + 5 * sz, n, n1, d, sx, sxy, t_xi, t_eta, t_zeta);
  const double u_x = u_xi * xi_x + u_eta * eta_x + u_zeta * zeta_x;
  const double u_y = u_xi * xi_y + u_eta * eta_y + u_zeta * zeta_y;
  const double u_z = u_xi * xi_z + u_eta * eta_z + u_zeta * zeta_z;
  const double v_x = v_xi * xi_x + v_eta * eta_x + v_zeta * zeta_x;
  const double v_y = v_xi * xi_y + v_eta * eta_y + v_zeta * zeta_y;
  const double v_z = v_xi * xi_z + v_eta * eta_z + v_zeta * zeta_z;
  const double w_x = w_xi * xi_x + w_eta * eta_x + w_zeta * zeta_x;
  const double w_y = w_xi * xi_y + w_eta * eta_y + w_zeta * zeta_y;
  const double w_z = w_xi * xi_z + w_eta * eta_z + w_zeta * zeta_z;
  const double mul = 0.5 * (ld(B.mul + n) + ld(B.mul + n1));
  double mut = 0;
  if constexpr (C::turb) mut = 0.5 * (ld(B.mut + n) + ld(B.mut + n1));
  const double viscosity = mul + mut;
  double tau_xx = viscosity * (4 * u_x - 2 * v_y - 2 * w_z) / 3.0;
  double tau_yy = viscosity * (4 * v_y - 2 * u_x - 2 * w_z) / 3.0;
  double tau_zz = viscosity * (4 * w_z - 2 * u_x - 2 * v_y) / 3.0;
  const double tau_xy = viscosity * (u_y + v_x);
  const double tau_xz = viscosity * (u_z + w_x);
  const double tau_yz = viscosity * (v_z + w_y);
  if constexpr (C::turb) {
    const double tt = -2.0 / 3 * 0.5 *
                      (ld(B.bv + n) * ld(B.sv + NS * sz + n) + ld(B.bv + n1) * ld(B.sv + NS * sz + n1));
    tau_xx += tt;
    tau_yy += tt;
    tau_zz += tt;
  }
  const double *mr = m + 3 * d * sz;
  const double ja = ld(B.jac + n), jb = ld(B.jac + n1);
  const double kx = 0.5 * (ld(mr + n) * ja + ld(mr + n1) * jb);
  const double ky = 0.5 * (ld(mr + sz + n) * ja + ld(mr + sz + n1) * jb);
  const double kz = 0.5 * (ld(mr + 2 * sz + n) * ja + ld(mr + 2 * sz + n1) * jb);
  fv[0] = 0;
  fv[1] = kx * tau_xx + ky * tau_xy + kz * tau_xz;
  fv[2] = kx * tau_xy + ky * tau_yy + kz * tau_yz;
  fv[3] = kx * tau_xz + ky * tau_yz + kz * tau_zz;
  const double um = 0.5 * (ld(B.bv + sz + n) + ld(B.bv + sz + n1));
  const double vm = 0.5 * (ld(B.bv + 2 * sz + n) + ld(B.bv + 2 * sz + n1));
  const double wm = 0.5 * (ld(B.bv + 3 * sz + n) + ld(B.bv + 3 * sz + n1));
  const double t_x = t_xi * xi_x + t_eta * eta_x + t_zeta * zeta_x;
  const double t_y = t_xi * xi_y + t_eta * eta_y + t_zeta * zeta_y;
  const double t_z = t_xi * xi_z + t_eta * eta_z + t_zeta * zeta_z;
  double conductivity = 0.5 * (ld(B.cond + n) + ld(B.cond + n1));
  if constexpr (C::turb) conductivity += 0.5 * (ld(B.turb_cond + n) + ld(B.turb_cond + n1));
  fv[4] = um * fv[1] + vm * fv[2] + wm * fv[3] + conductivity * (kx * t_x + ky * t_y + kz * t_z);
  if constexpr (C::mix != 0) {
    double turb_d = 0;
    if constexpr (C::turb) turb_d = mut / cP.Sct;
    double h[NS], dif[NS], yx[NS], yy[NS], yz[NS];
    const double tm = 0.5 * (ld(B.bv + 5 * sz + n) + ld(B.bv + 5 * sz + n1));
    enthalpy<NS>(tm, h);
    double rho_uc = 0, rho_vc = 0, rho_wc = 0;
    OSTC_UNROLL for (int l = 0; l < NS; ++l) {
      dif[l] = 0.5 * (ld(B.rho_d + l * sz + n) + ld(B.rho_d + l * sz + n1)) + turb_d;
      double y_xi, y_eta, y_zeta;
      face_grad(B.sv + l * sz, n, n1, d, sx, sxy, y_xi, y_eta, y_zeta);
      yx[l] = y_xi * xi_x + y_eta * eta_x + y_zeta * zeta_x;
      yy[l] = y_xi * xi_y + y_eta * eta_y + y_zeta * zeta_y;
      yz[l] = y_xi * xi_z + y_eta * eta_z + y_zeta * zeta_z;
      const double DMulH = dif[l] * h[l];
      fv[4] += kx * DMulH * yx[l];
      fv[4] += ky * DMulH * yy[l];
      fv[4] += kz * DMulH * yz[l];
      rho_uc += dif[l] * yx[l];
      rho_vc += dif[l] * yy[l];
      rho_wc += dif[l] * yz[l];
    }
    OSTC_UNROLL for (int l = 0; l < NS; ++l) {
      fv[5 + l] = dif[l] * (kx * yx[l] + ky * yy[l] + kz * yz[l]) -
                  0.5 * (ld(B.sv + l * sz + n) + ld(B.sv + l * sz + n1)) * (kx * rho_uc + ky * rho_vc + kz * rho_wc);
    }
  }
  if constexpr (C::turb) {
    const double *tk = B.sv + NS * sz, *tw = B.sv + (NS + 1) * sz;
    double k_xi, k_eta, k_zeta, o_xi, o_eta, o_zeta;
    face_grad(tk, n, n1, d, sx, sxy, k_xi, k_eta, k_zeta);
    const double k_x = k_xi * xi_x + k_eta * eta_x + k_zeta * zeta_x;
    const double k_y = k_xi * xi_y + k_eta * eta_y + k_zeta * zeta_y;
    const double k_z = k_xi * xi_z + k_eta * eta_z + k_zeta * zeta_z;
    face_grad(tw, n, n1, d, sx, sxy, o_xi, o_eta, o_zeta);
    const double omega_x = o_xi * xi_x + o_eta * eta_x + o_zeta * zeta_x;
    const double omega_y = o_xi * xi_y + o_eta * eta_y + o_zeta * zeta_y;
    const double omega_z = o_xi * xi_z + o_eta * eta_z + o_zeta * zeta_z;
    const double wall_dist = 0.5 * (ld(B.wall_dist + n) + ld(B.wall_dist + n1));
    double f1 = 1;
    if (wall_dist > 1e-25) {
      const double km = 0.5 * (ld(tk + n) + ld(tk + n1));
      const double omegam = 0.5 * (ld(tw + n) + ld(tw + n1));
      const double param1 = sqrt(km) / (0.09 * omegam * wall_dist);
      const double rhom = 0.5 * (ld(B.bv + n) + ld(B.bv + n1));
      const double d2 = wall_dist * wall_dist;
      const double param2 = 500 * mul / (rhom * d2 * omegam);
      const double CDkomega =
          fmax(1e-20, 2 * rhom * sst::sigma_omega2 / omegam * (k_x * omega_x + k_y * omega_y + k_z * omega_z));
      const double param3 = 4 * rhom * sst::sigma_omega2 * km / (CDkomega * d2);
      const double arg1 = fmin(fmax(param1, param2), param3);
      f1 = tanh(arg1 * arg1 * arg1 * arg1);
    }
    const double sigma_k = sst::sigma_k2 + sst::delta_sigma_k * f1;
    const double sigma_omega = sst::sigma_omega2 + sst::delta_sigma_omega * f1;
    // stored by the reference before use: keep the products rounded
    fv[5 + NS] = __dmul_rn(mul + mut * sigma_k, kx * k_x + ky * k_y + kz * k_z);
    fv[6 + NS] = __dmul_rn(mul + mut * sigma_omega, kx * omega_x + ky * omega_y + kz * omega_z);
  }
}

}  // namespace ostc
