/*
 * CPU oracle: serial FP64 restatement of OpenSTC's per-step residual and
 * update path.  TEST INFRASTRUCTURE ONLY (see ostc_oracle.h).  Every function
 * cites the reference file:line it restates; expressions keep the reference's
 * operation order so that CPU and GPU differ only by the last-ulp behaviour
 * of libm versus the CUDA math library.
 */
#include "ostc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define R_U 8314.462618
#define P_ATM 101325.0
#define GAMMA_AIR 1.4
#define MW_AIR 28.9647
#define MAXV (5 + ORC_MAX_SPEC + 2)

/* SST constants, src/SST.cuh:10-31 */
static const double SST_beta_star = 0.09, SST_sqrt_beta_star = 0.3, SST_kappa = 0.41;
static const double SST_sigma_k1 = 0.85, SST_sigma_omega1 = 0.5, SST_beta_1 = 0.0750, SST_a_1 = 0.31;
static const double SST_sigma_k2 = 1, SST_sigma_omega2 = 0.856, SST_beta_2 = 0.0828;
#define SST_gamma1 (SST_beta_1 / SST_beta_star - SST_sigma_omega1 * SST_kappa * SST_kappa / SST_sqrt_beta_star)
#define SST_gamma2 (SST_beta_2 / SST_beta_star - SST_sigma_omega2 * SST_kappa * SST_kappa / SST_sqrt_beta_star)
#define SST_delta_sigma_k (SST_sigma_k1 - SST_sigma_k2)
#define SST_delta_sigma_omega (SST_sigma_omega1 - SST_sigma_omega2)
#define SST_delta_beta (SST_beta_1 - SST_beta_2)
#define SST_delta_gamma (SST_gamma1 - SST_gamma2)

static inline double dmax(double a, double b) { return fmax(a, b); }
static inline double dmin(double a, double b) { return fmin(a, b); }

/* ------------------------------------------------------------------ storage */
typedef struct blk {
  int mx, my, mz, ngg;
  int64_t sx[4], sxy[4], size[4], off[4]; /* per ghost count 0..3 */
  double *f[ORC_N_FIELDS];
  int gf[ORC_N_FIELDS];     /* ghost layers of each field */
  int nc[ORC_N_FIELDS];     /* components */
} blk;

struct orc_solver {
  orc_params p;
  int nb, ngg, dim, nthreads;
  blk *b;
  orc_bc *bc;
  int nbc, cap_bc;
  orc_inner *inner;
  int ninner, cap_inner;
  int64_t n_grid_total;
};

static inline int64_t IX(const blk *B, int g, int i, int j, int k) {
  return (int64_t)k * B->sxy[g] + (int64_t)j * B->sx[g] + i + B->off[g];
}
#define A(F, l, i, j, k) (B->f[F][(int64_t)(l) * B->size[B->gf[F]] + IX(B, B->gf[F], i, j, k)])
#define AS(F, i, j, k) (B->f[F][IX(B, B->gf[F], i, j, k)])
/* metric(r,c), 1-based as in the reference */
#define MET(r, c, i, j, k) A(ORC_METRIC, ((r)-1) * 3 + ((c)-1), i, j, k)

static int sgn_d(double a) { return a < 0 ? -1 : 1; }

/* ------------------------------------------------------------------ thermo */
/* compute_enthalpy, src/Thermo.cu:5-23 */
static void th_h(const orc_params *p, double t, double *h) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  for (int i = 0; i < p->ns; ++i) {
    if (t < p->t_low[i]) {
      const double tt = p->t_low[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
      const double *c = &p->low_coeff[i * 7];
      h[i] = c[0] * tt + 0.5 * c[1] * tt2 + c[2] * tt3 / 3 + 0.25 * c[3] * tt4 + 0.2 * c[4] * tt5 + c[5];
      const double cp = c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * tt4;
      h[i] += cp * (t - tt);
    } else {
      const double *c = t < p->t_mid[i] ? &p->low_coeff[i * 7] : &p->high_coeff[i * 7];
      h[i] = c[0] * t + 0.5 * c[1] * t2 + c[2] * t3 / 3 + 0.25 * c[3] * t4 + 0.2 * c[4] * t5 + c[5];
    }
    h[i] *= R_U / p->mw[i];
  }
}

/* compute_enthalpy_and_cp, src/Thermo.cu:25-45 */
static void th_hcp(const orc_params *p, double t, double *h, double *cp) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  for (int i = 0; i < p->ns; ++i) {
    if (t < p->t_low[i]) {
      const double tt = p->t_low[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
      const double *c = &p->low_coeff[i * 7];
      h[i] = c[0] * tt + 0.5 * c[1] * tt2 + c[2] * tt3 / 3 + 0.25 * c[3] * tt4 + 0.2 * c[4] * tt5 + c[5];
      cp[i] = c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * tt4;
      h[i] += cp[i] * (t - tt);
    } else {
      const double *c = t < p->t_mid[i] ? &p->low_coeff[i * 7] : &p->high_coeff[i * 7];
      h[i] = c[0] * t + 0.5 * c[1] * t2 + c[2] * t3 / 3 + 0.25 * c[3] * t4 + 0.2 * c[4] * t5 + c[5];
      cp[i] = c[0] + c[1] * t + c[2] * t2 + c[3] * t3 + c[4] * t4;
    }
    h[i] *= R_U / p->mw[i];
    cp[i] *= R_U / p->mw[i];
  }
}

void orc_enthalpy_cp(const orc_params *p, double t, double *h, double *cp) { th_hcp(p, t, h, cp); }

/* compute_cp, src/Thermo.cu:47-61 */
static void th_cp(const orc_params *p, double t, double *cp) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t;
  for (int i = 0; i < p->ns; ++i) {
    if (t < p->t_low[i]) {
      const double tt = p->t_low[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt;
      const double *c = &p->low_coeff[i * 7];
      cp[i] = c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * tt4;
    } else {
      const double *c = t < p->t_mid[i] ? &p->low_coeff[i * 7] : &p->high_coeff[i * 7];
      cp[i] = c[0] + c[1] * t + c[2] * t2 + c[3] * t3 + c[4] * t4;
    }
    cp[i] *= R_U / p->mw[i];
  }
}

/* compute_gibbs_div_rt, src/Thermo.cu:63-79 */
static void th_gibbs(const orc_params *p, double t, double *g) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t_inv = 1 / t, log_t = log(t);
  for (int i = 0; i < p->ns; ++i) {
    if (t < p->t_low[i]) {
      const double tt = p->t_low[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt_inv = 1 / tt, log_tt = log(tt);
      const double *c = &p->low_coeff[i * 7];
      g[i] = c[0] * (1.0 - log_tt) - 0.5 * c[1] * tt - c[2] * tt2 / 6.0 - c[3] * tt3 / 12.0 - c[4] * tt4 * 0.05 +
             c[5] * tt_inv - c[6];
    } else {
      const double *c = t < p->t_mid[i] ? &p->low_coeff[i * 7] : &p->high_coeff[i * 7];
      g[i] = c[0] * (1.0 - log_t) - 0.5 * c[1] * t - c[2] * t2 / 6.0 - c[3] * t3 / 12.0 - c[4] * t4 * 0.05 +
             c[5] * t_inv - c[6];
    }
  }
}

/* Sutherland, src/Transport.cu:6-9 */
static double sutherland(double t) { return 1.716e-5 * pow(t / 273, 1.5) * (273 + 111) / (t + 111); }

/* species viscosities (shared head of compute_transport_property and
   compute_viscosity, src/Transport.cu:40-52, 86-99) */
static void species_visc(const orc_params *p, double t, double mw_total, const double *Y, double *X, double *vis) {
  for (int l = 0; l < p->ns; ++l) {
    X[l] = Y[l] * mw_total / p->mw[l];
    const double t_dl = t * p->lj_inv[l];
    const double ci = 1.147 * pow(t_dl, -0.145) + pow(t_dl + 0.5, -2);
    vis[l] = p->vis_coeff[l] * sqrt(t) / ci;
  }
}

static double wilke_phi(const orc_params *p, const double *vis, int m, int n) {
  if (m == n) return 1.0;
  const double num = 1 + sqrt(vis[m] / vis[n]) * p->w_quarter[m * p->ns + n];
  return num * num * p->w_sqrt8[m * p->ns + n];
}

/* compute_viscosity (device), src/Transport.cu:86-115 */
static double mix_viscosity(const orc_params *p, double t, double mw_total, const double *Y) {
  double X[ORC_MAX_SPEC], vis[ORC_MAX_SPEC];
  species_visc(p, t, mw_total, Y, X, vis);
  double viscosity = 0;
  for (int m = 0; m < p->ns; ++m) {
    double vt = 0;
    for (int n = 0; n < p->ns; ++n) vt += wilke_phi(p, vis, m, n) * X[n];
    viscosity += vis[m] * X[m] / vt;
  }
  return viscosity;
}

/* ------------------------------------------------------------------ chemistry */
/* arrhenius, src/FiniteRateChem.cu:110-112 */
static double arrhenius(double t, double A_, double b_, double Ea_) { return A_ * pow(t, b_) * exp(-Ea_ / t); }

/* forward_reaction_rate, src/FiniteRateChem.cu:65-108 */
static void kf_rates(const orc_params *p, double t, double *kf, const double *c) {
  for (int i = 0; i < p->nr; ++i) {
    kf[i] = arrhenius(t, p->A[i], p->b[i], p->Ea[i]);
    if (p->label[i] == 3) kf[i] += arrhenius(t, p->A2[i], p->b2[i], p->Ea2[i]);
    if (p->label[i] > 3) {
      double cc = 0;
      for (int l = 0; l < p->ns; ++l) cc += c[l] * p->third_body[i * p->ns + l];
      if (p->label[i] == 4) {
        kf[i] *= cc;
      } else {
        const double kf_low = arrhenius(t, p->A2[i], p->b2[i], p->Ea2[i]);
        const double kf_high = kf[i];
        const double pr = kf_low * cc / kf_high;
        double F = 1.0;
        if (p->label[i] > 5) {
          double f_cent = (1 - p->troe_alpha[i]) * exp(-t / p->troe_t3[i]) + p->troe_alpha[i] * exp(-t / p->troe_t1[i]);
          if (p->label[i] == 7) f_cent += exp(-p->troe_t2[i] / t);
          const double logFc = log10(f_cent);
          const double cc2 = -0.4 - 0.67 * logFc;
          const double n = 0.75 - 1.27 * logFc;
          const double logPr = log10(pr);
          const double tempo = (logPr + cc2) / (n - 0.14 * (logPr + cc2));
          const double pp = logFc / (1.0 + tempo * tempo);
          F = pow(10, pp);
        }
        kf[i] = kf_high * pr / (1.0 + pr) * F;
      }
    }
  }
}

/* backward_reaction_rate, src/FiniteRateChem.cu:114-136 */
static void kb_rates(const orc_params *p, double t, const double *kf, double *kb) {
  double g[ORC_MAX_SPEC];
  th_gibbs(p, t, g);
  const double temp_p = P_ATM / R_U * 1e-3;
  const double temp_t = temp_p / t;
  for (int i = 0; i < p->nr; ++i) {
    if (p->label[i] != 2) {
      double dg = 0;
      for (int l = 0; l < p->ns; ++l) dg += g[l] * (p->stoi_b[i * p->ns + l] - p->stoi_f[i * p->ns + l]);
      const double kc = pow(temp_t, p->order[i]) * exp(-dg);
      kb[i] = kf[i] / kc;
    } else {
      kb[i] = arrhenius(t, p->A2[i], p->b2[i], p->Ea2[i]);
    }
  }
}

/* rate_of_progress + chemical_source, src/FiniteRateChem.cu:138-171 */
static void progress_and_source(const orc_params *p, const double *kf, const double *kb, const double *c, double *q1,
                                double *q2, double *omega, double *omega_d) {
  const int ns = p->ns;
  for (int i = 0; i < p->nr; ++i) {
    q1[i] = 1.0;
    q2[i] = 1.0;
    for (int j = 0; j < ns; ++j) {
      q1[i] *= pow(c[j], p->stoi_f[i * ns + j]);
      q2[i] *= pow(c[j], p->stoi_b[i * ns + j]);
    }
    q1[i] *= kf[i];
    q2[i] *= kb[i];
  }
  for (int i = 0; i < ns; ++i) {
    double creation = 0;
    omega_d[i] = 0;
    for (int j = 0; j < p->nr; ++j) {
      creation += q2[j] * p->stoi_f[j * ns + i] + q1[j] * p->stoi_b[j * ns + i];
      omega_d[i] += q1[j] * p->stoi_f[j * ns + i] + q2[j] * p->stoi_b[j * ns + i];
    }
    creation *= p->mw[i] * 1e+3;
    omega_d[i] *= p->mw[i] * 1e+3;
    omega[i] = creation - omega_d[i];
  }
}

/* compute_chem_src_jacobian, src/FiniteRateChem.cu:173-194 */
static void epi_jacobian(const orc_params *p, double density, const double *Y, const double *q1, const double *q2,
                         double *jac) {
  const int ns = p->ns;
  for (int m = 0; m < ns; ++m) {
    for (int n = 0; n < ns; ++n) {
      double zz = 0;
      if (Y[n] > 1e-25) {
        for (int r = 0; r < p->nr; ++r)
          zz += (p->stoi_b[r * ns + m] - p->stoi_f[r * ns + m]) *
                (p->stoi_f[r * ns + n] * q1[r] - p->stoi_b[r * ns + n] * q2[r]);
        zz /= density * Y[n];
      }
      jac[m * ns + n] = p->mw[m] * zz * 1e+3;
    }
  }
}

/* concentrations and all of finite_rate_chemistry, src/FiniteRateChem.cu:7-63 */
static void chem_point(const orc_params *p, double density, double t, const double *Y, double *omega, double *q1,
                       double *q2, double *omega_d) {
  double c[ORC_MAX_SPEC], kf[ORC_MAX_REAC], kb[ORC_MAX_REAC];
  for (int l = 0; l < p->ns; ++l) c[l] = density * Y[l] / p->mw[l] * 1e-3;
  kf_rates(p, t, kf, c);
  kb_rates(p, t, kf, kb);
  progress_and_source(p, kf, kb, c, q1, q2, omega, omega_d);
}

void orc_chemical_source(const orc_params *p, double rho, double t, const double *Y, double *omega, double *jac) {
  double q1[ORC_MAX_REAC], q2[ORC_MAX_REAC], od[ORC_MAX_SPEC];
  chem_point(p, rho, t, Y, omega, q1, q2, od);
  if (jac) epi_jacobian(p, rho, Y, q1, q2, jac);
}

/* solve_chem_system: column-pivoted Doolittle LU, src/FiniteRateChem.cu:344-398 */
static void lu_solve(double *lhs, double *rhs, int dim) {
  int ipiv[ORC_MAX_SPEC];
  for (int n = 0; n < dim; ++n) {
    int ik = n;
    for (int m = n; m < dim; ++m) {
      for (int t = 0; t < n; ++t) lhs[m * dim + n] -= lhs[m * dim + t] * lhs[t * dim + n];
      if (fabs(lhs[m * dim + n]) > fabs(lhs[ik * dim + n])) ik = m;
    }
    ipiv[n] = ik;
    if (ik != n) {
      for (int t = 0; t < dim; ++t) {
        const double mid = lhs[ik * dim + t];
        lhs[ik * dim + t] = lhs[n * dim + t];
        lhs[n * dim + t] = mid;
      }
    }
    for (int q = n + 1; q < dim; ++q)
      for (int t = 0; t < n; ++t) lhs[n * dim + q] -= lhs[n * dim + t] * lhs[t * dim + q];
    for (int m = n + 1; m < dim; ++m) lhs[m * dim + n] /= lhs[n * dim + n];
  }
  for (int m = 0; m < dim; ++m) {
    const int t = ipiv[m];
    if (t != m) {
      const double mid = rhs[t];
      rhs[t] = rhs[m];
      rhs[m] = mid;
    }
  }
  for (int m = 1; m < dim; ++m)
    for (int t = 0; t < m; ++t) rhs[m] -= lhs[m * dim + t] * rhs[t];
  rhs[dim - 1] /= lhs[dim * dim - 1];
  for (int m = dim - 2; m >= 0; --m) {
    for (int t = m + 1; t < dim; ++t) rhs[m] -= lhs[m * dim + t] * rhs[t];
    rhs[m] /= lhs[m * dim + m];
  }
}

void orc_epi_increment(const orc_params *p, double rho, double t, const double *Y, double dt, double *dY) {
  /* The explicit-mode EPI chain for chemistry alone: compute_source's
     chemistry (src/FiniteRateChem.cu:7-63), EPI (:211-234) and the density
     update (src/FieldOperation.cuh:149-152) at fixed rho. */
  const int ns = p->ns;
  double omega[ORC_MAX_SPEC], jac[ORC_MAX_SPEC * ORC_MAX_SPEC], lhs[ORC_MAX_SPEC * ORC_MAX_SPEC], rhs[ORC_MAX_SPEC];
  orc_chemical_source(p, rho, t, Y, omega, jac);
  for (int m = 0; m < ns; ++m)
    for (int n = 0; n < ns; ++n) lhs[m * ns + n] = (m == n) ? 1.0 - dt * jac[m * ns + n] : -dt * jac[m * ns + n];
  for (int l = 0; l < ns; ++l) rhs[l] = omega[l];
  lu_solve(lhs, rhs, ns);
  for (int l = 0; l < ns; ++l) dY[l] = rhs[l] * dt / rho;
}

/* ------------------------------------------------------------------ SST */
/* SST::compute_mut, src/SST.cu:6-58 */
static void sst_mut(const orc_params *p, blk *B, int i, int j, int k, double mul) {
  const int ns = p->ns;
  const double xi_x = MET(1, 1, i, j, k), xi_y = MET(1, 2, i, j, k), xi_z = MET(1, 3, i, j, k);
  const double eta_x = MET(2, 1, i, j, k), eta_y = MET(2, 2, i, j, k), eta_z = MET(2, 3, i, j, k);
  const double zeta_x = MET(3, 1, i, j, k), zeta_y = MET(3, 2, i, j, k), zeta_z = MET(3, 3, i, j, k);
#define DBV(l, cx, cy, cz)                                                                                   \
  (0.5 * (cx * (A(ORC_BV, l, i + 1, j, k) - A(ORC_BV, l, i - 1, j, k)) +                                  \
          cy * (A(ORC_BV, l, i, j + 1, k) - A(ORC_BV, l, i, j - 1, k)) +                                  \
          cz * (A(ORC_BV, l, i, j, k + 1) - A(ORC_BV, l, i, j, k - 1))))
  const double u_y = DBV(1, xi_y, eta_y, zeta_y), u_z = DBV(1, xi_z, eta_z, zeta_z);
  const double v_x = DBV(2, xi_x, eta_x, zeta_x), v_z = DBV(2, xi_z, eta_z, zeta_z);
  const double w_x = DBV(3, xi_x, eta_x, zeta_x), w_y = DBV(3, xi_y, eta_y, zeta_y);
  const double rhoK = A(ORC_CV, ns + 5, i, j, k);
  const double tke = A(ORC_SV, ns, i, j, k);
  const double omega = A(ORC_SV, ns + 1, i, j, k);
  const double vorticity = sqrt((v_x - u_y) * (v_x - u_y) + (w_x - u_z) * (w_x - u_z) + (w_y - v_z) * (w_y - v_z));
  const double density = A(ORC_BV, 0, i, j, k);
  double f2 = 1;
  const double dy = AS(ORC_WALL_DIST, i, j, k);
  if (dy > 1e-25) {
    const double param1 = 2 * sqrt(tke) / (0.09 * omega * dy);
    const double param2 = 500 * mul / (density * dy * dy * omega);
    const double arg2 = dmax(param1, param2);
    f2 = tanh(arg2 * arg2);
  }
  double mut = 0;
  const double den = dmax(SST_a_1 * omega, vorticity * f2);
  if (den > 1e-25) mut = SST_a_1 * rhoK / den;
  AS(ORC_MUT, i, j, k) = mut;
}

/* SST::compute_source_and_mut, src/SST.cu:60-178 */
static void sst_source(const orc_params *p, blk *B, int i, int j, int k) {
  const int ns = p->ns;
  const double xi_x = MET(1, 1, i, j, k), xi_y = MET(1, 2, i, j, k), xi_z = MET(1, 3, i, j, k);
  const double eta_x = MET(2, 1, i, j, k), eta_y = MET(2, 2, i, j, k), eta_z = MET(2, 3, i, j, k);
  const double zeta_x = MET(3, 1, i, j, k), zeta_y = MET(3, 2, i, j, k), zeta_z = MET(3, 3, i, j, k);
  const double u_x = DBV(1, xi_x, eta_x, zeta_x), u_y = DBV(1, xi_y, eta_y, zeta_y), u_z = DBV(1, xi_z, eta_z, zeta_z);
  const double v_x = DBV(2, xi_x, eta_x, zeta_x), v_y = DBV(2, xi_y, eta_y, zeta_y), v_z = DBV(2, xi_z, eta_z, zeta_z);
  const double w_x = DBV(3, xi_x, eta_x, zeta_x), w_y = DBV(3, xi_y, eta_y, zeta_y), w_z = DBV(3, xi_z, eta_z, zeta_z);
#undef DBV
  const double density = A(ORC_BV, 0, i, j, k);
  const double omega = A(ORC_SV, ns + 1, i, j, k);
#define DSV(l, cx, cy, cz)                                                                                   \
  (0.5 * (cx * (A(ORC_SV, l, i + 1, j, k) - A(ORC_SV, l, i - 1, j, k)) +                                  \
          cy * (A(ORC_SV, l, i, j + 1, k) - A(ORC_SV, l, i, j - 1, k)) +                                  \
          cz * (A(ORC_SV, l, i, j, k + 1) - A(ORC_SV, l, i, j, k - 1))))
  const double k_x = DSV(ns, xi_x, eta_x, zeta_x), k_y = DSV(ns, xi_y, eta_y, zeta_y),
               k_z = DSV(ns, xi_z, eta_z, zeta_z);
  const double omega_x = DSV(ns + 1, xi_x, eta_x, zeta_x), omega_y = DSV(ns + 1, xi_y, eta_y, zeta_y),
               omega_z = DSV(ns + 1, xi_z, eta_z, zeta_z);
#undef DSV
  const double inter_var = 2 * density * SST_sigma_omega2 / omega * (k_x * omega_x + k_y * omega_y + k_z * omega_z);
  const double tke = A(ORC_SV, ns, i, j, k);
  const double rhoK = density * tke;
  const double vorticity = sqrt((v_x - u_y) * (v_x - u_y) + (w_x - u_z) * (w_x - u_z) + (w_y - v_z) * (w_y - v_z));
  double f1 = 1, f2 = 1;
  const double dy = AS(ORC_WALL_DIST, i, j, k);
  if (dy > 1e-25) {
    const double param1 = sqrt(tke) / (0.09 * omega * dy);
    const double d2 = dy * dy;
    const double param2 = 500 * AS(ORC_MUL, i, j, k) / (density * d2 * omega);
    const double arg2 = dmax(2 * param1, param2);
    f2 = tanh(arg2 * arg2);
    const double CDkomega = dmax(1e-20, inter_var);
    const double param3 = 4 * density * SST_sigma_omega2 * tke / (CDkomega * d2);
    const double arg1 = dmin(dmax(param1, param2), param3);
    f1 = tanh(arg1 * arg1 * arg1 * arg1);
  }
  double mut = 0;
  const double den = dmax(SST_a_1 * omega, vorticity * f2);
  if (den > 1e-25) mut = SST_a_1 * rhoK / den;
  AS(ORC_MUT, i, j, k) = mut;
  const double beta = SST_beta_2 + SST_delta_beta * f1;
  if (mut > 1e-25) {
    const double divU = u_x + v_y + w_z;
    const double divU2 = divU * divU;
    const double prod_k = mut * (2 * (u_x * u_x + v_y * v_y + w_z * w_z) - 2.0 / 3 * divU2 + (u_y + v_x) * (u_y + v_x) +
                                 (u_z + w_x) * (u_z + w_x) + (v_z + w_y) * (v_z + w_y)) -
                          2.0 / 3 * rhoK * divU;
    const double diss_k = SST_beta_star * rhoK * omega;
    const double jac = AS(ORC_JAC, i, j, k);
    A(ORC_DQ, ns + 5, i, j, k) += jac * (prod_k - diss_k);
    const double gamma = SST_gamma2 + SST_delta_gamma * f1;
    const double prod_omega = gamma * density / mut * prod_k + (1 - f1) * inter_var;
    const double diss_omega = beta * density * omega * omega;
    A(ORC_DQ, ns + 6, i, j, k) += jac * (prod_omega - diss_omega);
  }
  if (p->turb_implicit == 1) {
    A(ORC_TURB_SRC_JAC, 0, i, j, k) = -2 * SST_beta_star * omega;
    A(ORC_TURB_SRC_JAC, 1, i, j, k) = -2 * beta * omega;
  }
}

/* ------------------------------------------------------------------ source */
/* compute_source, src/SourceTerm.cuh:11-40 */
static void phase_source(orc_solver *s, blk *B) {
  const orc_params *p = &s->p;
#pragma omp parallel for collapse(2) schedule(static) num_threads(s->nthreads)
  for (int k = 0; k < B->mz; ++k)
    for (int j = 0; j < B->my; ++j)
      for (int i = 0; i < B->mx; ++i) {
        if (p->turb) {
          if (p->rans_model != 1) sst_source(p, B, i, j, k);
          if (p->mix != 0) {
            AS(ORC_TURB_COND, i, j, k) = AS(ORC_MUT, i, j, k) * AS(ORC_CP, i, j, k) / p->Prt;
          } else {
            const double cp = GAMMA_AIR * R_U / MW_AIR / (GAMMA_AIR - 1);
            AS(ORC_TURB_COND, i, j, k) = AS(ORC_MUT, i, j, k) * cp / p->Prt;
          }
        }
        if (p->mix == 2) {
          const int ns = p->ns;
          double Y[ORC_MAX_SPEC], omega[ORC_MAX_SPEC], q1[ORC_MAX_REAC], q2[ORC_MAX_REAC], od[ORC_MAX_SPEC];
          for (int l = 0; l < ns; ++l) Y[l] = A(ORC_SV, l, i, j, k);
          const double density = A(ORC_BV, 0, i, j, k), t = A(ORC_BV, 5, i, j, k);
          chem_point(p, density, t, Y, omega, q1, q2, od);
          for (int l = 0; l < ns; ++l) A(ORC_DQ, l + 5, i, j, k) += AS(ORC_JAC, i, j, k) * omega[l];
          if (p->chem_src_method == 1) {
            double J[ORC_MAX_SPEC * ORC_MAX_SPEC];
            epi_jacobian(p, density, Y, q1, q2, J);
            for (int q = 0; q < ns * ns; ++q) A(ORC_CHEM_JAC, q, i, j, k) = J[q];
          } else if (p->chem_src_method == 2) {
            /* compute_chem_src_jacobian_diagonal, src/FiniteRateChem.cu:196-209 */
            for (int l = 0; l < ns; ++l) {
              A(ORC_CHEM_JAC, l, i, j, k) = 0;
              if (Y[l] > 1e-25) A(ORC_CHEM_JAC, l, i, j, k) = -od[l] / (Y[l] * density);
            }
          }
        }
      }
}

/* ------------------------------------------------------------------ inviscid */
/* minmod, src/Limiter.cuh:13-16 */
static double minmod(double a, double b) { return 0.5 * (sgn_d(a) + sgn_d(b)) * dmin(fabs(a), fabs(b)); }

/* reconstruction + MUSCL/NND2/1st order, src/InviscidScheme.cuh:21-68, src/Reconstruction.cu:5-46 */
static void reconstruct(const orc_params *p, const double *pv, double *pl, double *pr, int is, int nv) {
  if (p->reconstruction == 2) {
    const double kappa = 1.0 / 3.0;
    for (int l = 0; l < nv; ++l) {
      const double d_i = pv[is * nv + l] - pv[(is - 1) * nv + l];
      const double d_i1 = pv[(is + 1) * nv + l] - pv[is * nv + l];
      const double d_i2 = pv[(is + 2) * nv + l] - pv[(is + 1) * nv + l];
      const double neg_l = minmod(d_i, d_i1), pos_l = minmod(d_i1, d_i);
      const double neg_r = minmod(d_i1, d_i2), pos_r = minmod(d_i2, d_i1);
      pl[l] = pv[is * nv + l] + 0.25 * ((1 - kappa) * neg_l + (1 + kappa) * pos_l);
      pr[l] = pv[(is + 1) * nv + l] - 0.25 * ((1 - kappa) * pos_r + (1 + kappa) * neg_r);
    }
  } else if (p->reconstruction == 3) {
    for (int l = 0; l < nv; ++l) {
      const double d_i = pv[is * nv + l] - pv[(is - 1) * nv + l];
      const double d_i1 = pv[(is + 1) * nv + l] - pv[is * nv + l];
      const double d_i2 = pv[(is + 2) * nv + l] - pv[(is + 1) * nv + l];
      pl[l] = pv[is * nv + l] + 0.5 * minmod(d_i, d_i1);
      pr[l] = pv[(is + 1) * nv + l] - 0.5 * minmod(d_i1, d_i2);
    }
  } else {
    for (int l = 0; l < nv; ++l) {
      pl[l] = pv[is * nv + l];
      pr[l] = pv[(is + 1) * nv + l];
    }
  }
  if (p->mix != 0) {
    double el = 0.5 * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]);
    double er = 0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]);
    const int ns = p->ns;
    double mwl = 0, mwr = 0;
    for (int l = 0; l < ns; ++l) {
      mwl += pl[5 + l] / p->mw[l];
      mwr += pr[5 + l] / p->mw[l];
    }
    const double tl = pl[4] / (pl[0] * R_U * mwl);
    const double tr = pr[4] / (pr[0] * R_U * mwr);
    double hl[ORC_MAX_SPEC], hr[ORC_MAX_SPEC], cpl_i[ORC_MAX_SPEC], cpr_i[ORC_MAX_SPEC];
    th_hcp(p, tl, hl, cpl_i);
    th_hcp(p, tr, hr, cpr_i);
    double cpl = 0, cpr = 0, cvl = 0, cvr = 0;
    for (int l = 0; l < ns; ++l) {
      cpl += cpl_i[l] * pl[l + 5];
      cpr += cpr_i[l] * pr[l + 5];
      cvl += pl[l + 5] * (cpl_i[l] - R_U / p->mw[l]);
      cvr += pr[l + 5] * (cpr_i[l] - R_U / p->mw[l]);
      el += hl[l] * pl[l + 5];
      er += hr[l] * pr[l + 5];
    }
    pl[nv] = pl[0] * el - pl[4];
    pr[nv] = pr[0] * er - pr[4];
    pl[nv + 1] = cpl / cvl;
    pr[nv + 1] = cpr / cvr;
  } else {
    const double el = 0.5 * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]);
    const double er = 0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]);
    pl[nv] = el * pl[0] + pl[4] / (GAMMA_AIR - 1);
    pr[nv] = er * pr[0] + pr[4] / (GAMMA_AIR - 1);
  }
}

/* AUSMP_compute_inviscid_flux, src/InviscidScheme.cuh:70-149; `is` is the
   shared index of the left point, metric/jac hold row (dir+1) and J. */
static void ausmp(const orc_params *p, const double *pv, const double *met, const double *jac, int is, int nv,
                  double *fc) {
  double pl[MAXV + 2], pr[MAXV + 2];
  reconstruct(p, pv, pl, pr, is, nv);
  const double *ml = &met[is * 3], *mr = &met[(is + 1) * 3];
  const double jl = jac[is], jr = jac[is + 1];
  const double k1 = 0.5 * (jl * ml[0] + jr * mr[0]);
  const double k2 = 0.5 * (jl * ml[1] + jr * mr[1]);
  const double k3 = 0.5 * (jl * ml[2] + jr * mr[2]);
  const double gk = sqrt(k1 * k1 + k2 * k2 + k3 * k3);
  const double ul = (k1 * pl[1] + k2 * pl[2] + k3 * pl[3]) / gk;
  const double ur = (k1 * pr[1] + k2 * pr[2] + k3 * pr[3]) / gk;
  const double pL = pl[4], pR = pr[4], rl = pl[0], rr = pr[0];
  double gl = GAMMA_AIR, gr = GAMMA_AIR;
  if (p->ns > 0) {
    gl = pl[nv + 1];
    gr = pr[nv + 1];
  }
  const double c = 0.5 * (sqrt(gl * pL / rl) + sqrt(gr * pR / rr));
  const double ml_ = ul / c, mr_ = ur / c;
  double mlp, mrn, plp, prn;
  const double alpha = 3 / 16.0;
  if (fabs(ml_) > 1) {
    mlp = 0.5 * (ml_ + fabs(ml_));
    plp = mlp / ml_;
  } else {
    const double a = (ml_ + 1) * (ml_ + 1) * 0.25;
    const double b = (ml_ * ml_ - 1) * (ml_ * ml_ - 1);
    mlp = a + 0.125 * b;
    plp = a * (2 - ml_) + alpha * ml_ * b;
  }
  if (fabs(mr_) > 1) {
    mrn = 0.5 * (mr_ - fabs(mr_));
    prn = mrn / mr_;
  } else {
    const double a = (mr_ - 1) * (mr_ - 1) * 0.25;
    const double b = (mr_ * mr_ - 1) * (mr_ * mr_ - 1);
    mrn = -a - 0.125 * b;
    prn = a * (2 + mr_) - alpha * mr_ * b;
  }
  const double p_coeff = plp * pL + prn * pR;
  const double m_half = mlp + mrn;
  const double mpos = 0.5 * (m_half + fabs(m_half));
  const double mneg = 0.5 * (m_half - fabs(m_half));
  const double mass = c * (rl * mpos + rr * mneg);
  const double coeff = mass * gk;
  const double *s = mass >= 0 ? pl : pr;
  fc[0] = coeff;
  fc[1] = coeff * s[1] + p_coeff * k1;
  fc[2] = coeff * s[2] + p_coeff * k2;
  fc[3] = coeff * s[3] + p_coeff * k3;
  fc[4] = coeff * (s[nv] + s[4]) / s[0];
  for (int l = 5; l < nv; ++l) fc[l] = coeff * s[l];
}

/* inviscid_flux_1d, src/SchemeSelector.cuh:70-157: faces idx = -1..m-1 of
   each grid line along `dir`, then dq -= F(i+1/2) - F(i-1/2). */
static void phase_inviscid(orc_solver *s, blk *B, int dir) {
  const orc_params *p = &s->p;
  const int nv = p->n_var, ng = B->ngg, ns_ = p->n_scalar;
  const int ext[3] = {B->mx, B->my, B->mz};
  const int n = ext[dir];
  const int oa = dir == 0 ? 1 : 0, ob = dir == 2 ? 1 : 2;
  const int na = ext[oa], nb = ext[ob];
#pragma omp parallel num_threads(s->nthreads)
  {
    const int npt = n + 2 * ng;
    double *pv = malloc(sizeof(double) * npt * nv);
    double *met = malloc(sizeof(double) * npt * 3);
    double *jc = malloc(sizeof(double) * npt);
    double *fc = malloc(sizeof(double) * (n + 1) * nv);
#pragma omp for collapse(2) schedule(static)
    for (int b = 0; b < nb; ++b)
      for (int a = 0; a < na; ++a) {
        int id[3];
        for (int q = -ng; q < n + ng; ++q) {
          id[dir] = q;
          id[oa] = a;
          id[ob] = b;
          const int i = id[0], j = id[1], k = id[2];
          const int sh = q + ng;
          for (int l = 0; l < 5; ++l) pv[sh * nv + l] = A(ORC_BV, l, i, j, k);
          for (int l = 0; l < ns_; ++l) pv[sh * nv + 5 + l] = A(ORC_SV, l, i, j, k);
          for (int c = 1; c < 4; ++c) met[sh * 3 + c - 1] = MET(dir + 1, c, i, j, k);
          jc[sh] = AS(ORC_JAC, i, j, k);
        }
        /* face f between points f-1 and f (f = 0..n); left point shared index f-1+ng */
        for (int f = 0; f <= n; ++f) ausmp(p, pv, met, jc, f - 1 + ng, nv, &fc[f * nv]);
        for (int q = 0; q < n; ++q) {
          id[dir] = q;
          id[oa] = a;
          id[ob] = b;
          const int i = id[0], j = id[1], k = id[2];
          for (int l = 0; l < nv; ++l) A(ORC_DQ, l, i, j, k) -= fc[(q + 1) * nv + l] - fc[q * nv + l];
        }
      }
    free(pv);
    free(met);
    free(jc);
    free(fc);
  }
}

/* ------------------------------------------------------------------ viscous */
/* compute_{fv,gv,hv}_2nd_order, src/ViscousScheme.cuh:22-613, written once
   for the face between (i,j,k) and (i,j,k)+e_dir.  The normal difference is
   taken across the face; the two tangential differences average the central
   differences of both face points. */
static void viscous_face(const orc_params *p, blk *B, int dir, int i, int j, int k, double *fv) {
  const int ns = p->ns;
  const int di = dir == 0, dj = dir == 1, dk = dir == 2;
  const int i1 = i + di, j1 = j + dj, k1 = k + dk;
  double mt[9];
  for (int q = 0; q < 9; ++q) mt[q] = 0.5 * (A(ORC_METRIC, q, i, j, k) + A(ORC_METRIC, q, i1, j1, k1));
  const double xi_x = mt[0], xi_y = mt[1], xi_z = mt[2], eta_x = mt[3], eta_y = mt[4], eta_z = mt[5];
  const double zeta_x = mt[6], zeta_y = mt[7], zeta_z = mt[8];
  /* derivative of component l of field F along xi, eta, zeta */
#define DXI(F, l)                                                                                              \
  (dir == 0 ? A(F, l, i + 1, j, k) - A(F, l, i, j, k)                                                         \
            : 0.25 * (A(F, l, i + 1, j, k) - A(F, l, i - 1, j, k) + A(F, l, i1 + 1, j1, k1) - A(F, l, i1 - 1, j1, k1)))
#define DETA(F, l)                                                                                             \
  (dir == 1 ? A(F, l, i, j + 1, k) - A(F, l, i, j, k)                                                         \
            : 0.25 * (A(F, l, i, j + 1, k) - A(F, l, i, j - 1, k) + A(F, l, i1, j1 + 1, k1) - A(F, l, i1, j1 - 1, k1)))
#define DZETA(F, l)                                                                                            \
  (dir == 2 ? A(F, l, i, j, k + 1) - A(F, l, i, j, k)                                                         \
            : 0.25 * (A(F, l, i, j, k + 1) - A(F, l, i, j, k - 1) + A(F, l, i1, j1, k1 + 1) - A(F, l, i1, j1, k1 - 1)))
  const double u_xi = DXI(ORC_BV, 1), u_eta = DETA(ORC_BV, 1), u_zeta = DZETA(ORC_BV, 1);
  const double v_xi = DXI(ORC_BV, 2), v_eta = DETA(ORC_BV, 2), v_zeta = DZETA(ORC_BV, 2);
  const double w_xi = DXI(ORC_BV, 3), w_eta = DETA(ORC_BV, 3), w_zeta = DZETA(ORC_BV, 3);
  const double t_xi = DXI(ORC_BV, 5), t_eta = DETA(ORC_BV, 5), t_zeta = DZETA(ORC_BV, 5);
  const double u_x = u_xi * xi_x + u_eta * eta_x + u_zeta * zeta_x;
  const double u_y = u_xi * xi_y + u_eta * eta_y + u_zeta * zeta_y;
  const double u_z = u_xi * xi_z + u_eta * eta_z + u_zeta * zeta_z;
  const double v_x = v_xi * xi_x + v_eta * eta_x + v_zeta * zeta_x;
  const double v_y = v_xi * xi_y + v_eta * eta_y + v_zeta * zeta_y;
  const double v_z = v_xi * xi_z + v_eta * eta_z + v_zeta * zeta_z;
  const double w_x = w_xi * xi_x + w_eta * eta_x + w_zeta * zeta_x;
  const double w_y = w_xi * xi_y + w_eta * eta_y + w_zeta * zeta_y;
  const double w_z = w_xi * xi_z + w_eta * eta_z + w_zeta * zeta_z;
  const double mul = 0.5 * (AS(ORC_MUL, i, j, k) + AS(ORC_MUL, i1, j1, k1));
  double mut = 0;
  if (p->turb) mut = 0.5 * (AS(ORC_MUT, i, j, k) + AS(ORC_MUT, i1, j1, k1));
  const double viscosity = mul + mut;
  double tau_xx = viscosity * (4 * u_x - 2 * v_y - 2 * w_z) / 3.0;
  double tau_yy = viscosity * (4 * v_y - 2 * u_x - 2 * w_z) / 3.0;
  double tau_zz = viscosity * (4 * w_z - 2 * u_x - 2 * v_y) / 3.0;
  const double tau_xy = viscosity * (u_y + v_x);
  const double tau_xz = viscosity * (u_z + w_x);
  const double tau_yz = viscosity * (v_z + w_y);
  if (p->turb && p->rans_model == 2) {
    const double tt = -2.0 / 3 * 0.5 *
                      (A(ORC_BV, 0, i, j, k) * A(ORC_SV, ns, i, j, k) + A(ORC_BV, 0, i1, j1, k1) * A(ORC_SV, ns, i1, j1, k1));
    tau_xx += tt;
    tau_yy += tt;
    tau_zz += tt;
  }
  const int r = dir * 3;
  const double kx = 0.5 * (A(ORC_METRIC, r, i, j, k) * AS(ORC_JAC, i, j, k) + A(ORC_METRIC, r, i1, j1, k1) * AS(ORC_JAC, i1, j1, k1));
  const double ky = 0.5 * (A(ORC_METRIC, r + 1, i, j, k) * AS(ORC_JAC, i, j, k) +
                           A(ORC_METRIC, r + 1, i1, j1, k1) * AS(ORC_JAC, i1, j1, k1));
  const double kz = 0.5 * (A(ORC_METRIC, r + 2, i, j, k) * AS(ORC_JAC, i, j, k) +
                           A(ORC_METRIC, r + 2, i1, j1, k1) * AS(ORC_JAC, i1, j1, k1));
  fv[0] = 0;
  fv[1] = kx * tau_xx + ky * tau_xy + kz * tau_xz;
  fv[2] = kx * tau_xy + ky * tau_yy + kz * tau_yz;
  fv[3] = kx * tau_xz + ky * tau_yz + kz * tau_zz;
  const double um = 0.5 * (A(ORC_BV, 1, i, j, k) + A(ORC_BV, 1, i1, j1, k1));
  const double vm = 0.5 * (A(ORC_BV, 2, i, j, k) + A(ORC_BV, 2, i1, j1, k1));
  const double wm = 0.5 * (A(ORC_BV, 3, i, j, k) + A(ORC_BV, 3, i1, j1, k1));
  const double t_x = t_xi * xi_x + t_eta * eta_x + t_zeta * zeta_x;
  const double t_y = t_xi * xi_y + t_eta * eta_y + t_zeta * zeta_y;
  const double t_z = t_xi * xi_z + t_eta * eta_z + t_zeta * zeta_z;
  double cond = 0.5 * (AS(ORC_CONDUCTIVITY, i, j, k) + AS(ORC_CONDUCTIVITY, i1, j1, k1));
  if (p->turb) cond += 0.5 * (AS(ORC_TURB_COND, i, j, k) + AS(ORC_TURB_COND, i1, j1, k1));
  fv[4] = um * fv[1] + vm * fv[2] + wm * fv[3] + cond * (kx * t_x + ky * t_y + kz * t_z);
  if (p->mix != 0) {
    double turb_d = 0;
    if (p->turb) turb_d = mut / p->Sct;
    double h[ORC_MAX_SPEC], dif[ORC_MAX_SPEC], yx[ORC_MAX_SPEC], yy[ORC_MAX_SPEC], yz[ORC_MAX_SPEC];
    const double tm = 0.5 * (A(ORC_BV, 5, i, j, k) + A(ORC_BV, 5, i1, j1, k1));
    th_h(p, tm, h);
    double rho_uc = 0, rho_vc = 0, rho_wc = 0;
    for (int l = 0; l < ns; ++l) {
      dif[l] = 0.5 * (A(ORC_RHO_D, l, i, j, k) + A(ORC_RHO_D, l, i1, j1, k1)) + turb_d;
      const double y_xi = DXI(ORC_SV, l), y_eta = DETA(ORC_SV, l), y_zeta = DZETA(ORC_SV, l);
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
    for (int l = 0; l < ns; ++l)
      fv[5 + l] = dif[l] * (kx * yx[l] + ky * yy[l] + kz * yz[l]) -
                  0.5 * (A(ORC_SV, l, i, j, k) + A(ORC_SV, l, i1, j1, k1)) * (kx * rho_uc + ky * rho_vc + kz * rho_wc);
  }
  if (p->turb && p->rans_model != 1) {
    const int it = ns;
    const double k_xi = DXI(ORC_SV, it), k_eta = DETA(ORC_SV, it), k_zeta = DZETA(ORC_SV, it);
    const double k_x = k_xi * xi_x + k_eta * eta_x + k_zeta * zeta_x;
    const double k_y = k_xi * xi_y + k_eta * eta_y + k_zeta * zeta_y;
    const double k_z = k_xi * xi_z + k_eta * eta_z + k_zeta * zeta_z;
    const double o_xi = DXI(ORC_SV, it + 1), o_eta = DETA(ORC_SV, it + 1), o_zeta = DZETA(ORC_SV, it + 1);
    const double omega_x = o_xi * xi_x + o_eta * eta_x + o_zeta * zeta_x;
    const double omega_y = o_xi * xi_y + o_eta * eta_y + o_zeta * zeta_y;
    const double omega_z = o_xi * xi_z + o_eta * eta_z + o_zeta * zeta_z;
    const double wall_dist = 0.5 * (AS(ORC_WALL_DIST, i, j, k) + AS(ORC_WALL_DIST, i1, j1, k1));
    double f1 = 1;
    if (wall_dist > 1e-25) {
      const double km = 0.5 * (A(ORC_SV, it, i, j, k) + A(ORC_SV, it, i1, j1, k1));
      const double omegam = 0.5 * (A(ORC_SV, it + 1, i, j, k) + A(ORC_SV, it + 1, i1, j1, k1));
      const double param1 = sqrt(km) / (0.09 * omegam * wall_dist);
      const double rhom = 0.5 * (A(ORC_BV, 0, i, j, k) + A(ORC_BV, 0, i1, j1, k1));
      const double d2 = wall_dist * wall_dist;
      const double param2 = 500 * mul / (rhom * d2 * omegam);
      const double CDkomega =
          dmax(1e-20, 2 * rhom * SST_sigma_omega2 / omegam * (k_x * omega_x + k_y * omega_y + k_z * omega_z));
      const double param3 = 4 * rhom * SST_sigma_omega2 * km / (CDkomega * d2);
      const double arg1 = dmin(dmax(param1, param2), param3);
      f1 = tanh(arg1 * arg1 * arg1 * arg1);
    }
    const double sigma_k = SST_sigma_k2 + SST_delta_sigma_k * f1;
    const double sigma_omega = SST_sigma_omega2 + SST_delta_sigma_omega * f1;
    fv[5 + ns] = (mul + mut * sigma_k) * (kx * k_x + ky * k_y + kz * k_z);
    fv[6 + ns] = (mul + mut * sigma_omega) * (kx * omega_x + ky * omega_y + kz * omega_z);
  }
#undef DXI
#undef DETA
#undef DZETA
}

/* viscous_flux_{fv,gv,hv}, src/SchemeSelector.cuh:194-280 */
static void phase_viscous(orc_solver *s, blk *B, int dir) {
  const orc_params *p = &s->p;
  const int nv = p->n_var;
  const int ext[3] = {B->mx, B->my, B->mz};
  const int n = ext[dir];
  const int oa = dir == 0 ? 1 : 0, ob = dir == 2 ? 1 : 2;
  const int na = ext[oa], nb = ext[ob];
#pragma omp parallel num_threads(s->nthreads)
  {
    double *fv = calloc((size_t)(n + 1) * nv, sizeof(double));
#pragma omp for collapse(2) schedule(static)
    for (int b = 0; b < nb; ++b)
      for (int a = 0; a < na; ++a) {
        int id[3];
        for (int f = 0; f <= n; ++f) {
          id[dir] = f - 1;
          id[oa] = a;
          id[ob] = b;
          if (p->viscous_order == 0) {
            for (int l = 0; l < nv; ++l) fv[f * nv + l] = 0;
          } else {
            viscous_face(p, B, dir, id[0], id[1], id[2], &fv[f * nv]);
          }
        }
        for (int q = 0; q < n; ++q) {
          id[dir] = q;
          id[oa] = a;
          id[ob] = b;
          for (int l = 0; l < nv; ++l) A(ORC_DQ, l, id[0], id[1], id[2]) += fv[(q + 1) * nv + l] - fv[q * nv + l];
        }
      }
    free(fv);
  }
}

/* ------------------------------------------------------------------ local dt */
/* local_time_step, src/TimeAdvanceFunc.cuh:21-71 */
static void phase_dt(orc_solver *s, blk *B) {
  const orc_params *p = &s->p;
  const int dim = B->mz == 1 ? 2 : 3;
#pragma omp parallel for collapse(2) schedule(static) num_threads(s->nthreads)
  for (int k = 0; k < B->mz; ++k)
    for (int j = 0; j < B->my; ++j)
      for (int i = 0; i < B->mx; ++i) {
        const double m11 = MET(1, 1, i, j, k), m12 = MET(1, 2, i, j, k), m13 = MET(1, 3, i, j, k);
        const double m21 = MET(2, 1, i, j, k), m22 = MET(2, 2, i, j, k), m23 = MET(2, 3, i, j, k);
        const double m31 = MET(3, 1, i, j, k), m32 = MET(3, 2, i, j, k), m33 = MET(3, 3, i, j, k);
        const double gxi = sqrt(m11 * m11 + m12 * m12 + m13 * m13);
        const double geta = sqrt(m21 * m21 + m22 * m22 + m23 * m23);
        const double gzeta = sqrt(m31 * m31 + m32 * m32 + m33 * m33);
        const double u = A(ORC_BV, 1, i, j, k), v = A(ORC_BV, 2, i, j, k), w = A(ORC_BV, 3, i, j, k);
        const double U = u * m11 + v * m12 + w * m13;
        const double V = u * m21 + v * m22 + w * m23;
        const double W = u * m31 + v * m32 + w * m33;
        const double a = AS(ORC_ACOUSTIC, i, j, k);
        const double s0 = fabs(U) + a * gxi, s1 = fabs(V) + a * geta;
        double s2 = 0;
        if (dim == 3) s2 = fabs(W) + a * gzeta;
        A(ORC_INV_SPEC, 0, i, j, k) = s0;
        A(ORC_INV_SPEC, 1, i, j, k) = s1;
        A(ORC_INV_SPEC, 2, i, j, k) = s2;
        const double sri = s0 + s1 + s2;
        double gamma = GAMMA_AIR;
        if (p->mix != 0) gamma = AS(ORC_GAMMA, i, j, k);
        const double c1 = dmax(gamma, 4.0 / 3.0) / A(ORC_BV, 0, i, j, k);
        double c2 = AS(ORC_MUL, i, j, k) / p->Pr;
        if (p->turb) c2 += AS(ORC_MUT, i, j, k) / p->Prt;
        double srv = gxi * gxi + geta * geta;
        if (dim == 3) srv += gzeta * gzeta;
        srv *= c1 * c2;
        AS(ORC_VISC_SPEC, i, j, k) = srv;
        AS(ORC_DT_LOCAL, i, j, k) = p->cfl / (sri + srv);
      }
}

void orc_phase_residual(orc_solver *s, int b) {
  blk *B = &s->b[b];
  memset(B->f[ORC_DQ], 0, sizeof(double) * B->size[B->gf[ORC_DQ]] * B->nc[ORC_DQ]);
  phase_source(s, B);
  phase_inviscid(s, B, 0);
  phase_inviscid(s, B, 1);
  if (B->mz > 1) phase_inviscid(s, B, 2);
  phase_viscous(s, B, 0);
  phase_viscous(s, B, 1);
  if (B->mz > 1) phase_viscous(s, B, 2);
  phase_dt(s, B);
}

/* ------------------------------------------------------------------ implicit */
static void epi_lhs(const orc_params *p, blk *B, int i, int j, int k, double diag, double dt, double *lhs) {
  const int ns = p->ns;
  for (int m = 0; m < ns; ++m)
    for (int n = 0; n < ns; ++n) {
      const double J = A(ORC_CHEM_JAC, m * ns + n, i, j, k);
      lhs[m * ns + n] = (m == n) ? diag - dt * J : -dt * J;
    }
}

/* compute_jacobian_times_dq, src/DPLURHPP.cuh:78-125 */
static void jac_times_dq(const orc_params *p, blk *B, int i, int j, int k, int dir, double pm_sr, double *out) {
  const double kx = MET(dir + 1, 1, i, j, k), ky = MET(dir + 1, 2, i, j, k), kz = MET(dir + 1, 3, i, j, k);
  const double u = A(ORC_BV, 1, i, j, k), v = A(ORC_BV, 2, i, j, k), w = A(ORC_BV, 3, i, j, k);
  const double U = kx * u + ky * v + kz * w;
  const double lmd1 = U + pm_sr;
  const double e = 0.5 * AS(ORC_VEL, i, j, k) * AS(ORC_VEL, i, j, k);
  double gamma = GAMMA_AIR, b3 = 0, b4 = 0, h = 0;
  if (p->mix != 0) {
    double hk[ORC_MAX_SPEC];
    const double t = A(ORC_BV, 5, i, j, k);
    th_h(p, t, hk);
    gamma = AS(ORC_GAMMA, i, j, k);
    for (int l = 0; l < p->ns; ++l) {
      b3 += R_U * t / p->mw[l] * A(ORC_DQ, 5 + l, i, j, k);
      b4 += hk[l] * A(ORC_DQ, 5 + l, i, j, k);
      h += A(ORC_SV, l, i, j, k) * hk[l];
    }
    b3 *= gamma;
    b4 *= gamma - 1;
    h += e;
  } else {
    h = gamma / (gamma - 1) * A(ORC_BV, 4, i, j, k) / A(ORC_BV, 0, i, j, k) + e;
  }
  const double d0 = A(ORC_DQ, 0, i, j, k), d1 = A(ORC_DQ, 1, i, j, k), d2 = A(ORC_DQ, 2, i, j, k);
  const double d3 = A(ORC_DQ, 3, i, j, k), d4 = A(ORC_DQ, 4, i, j, k);
  const double b1 = kx * d1 + ky * d2 + kz * d3 - U * d0;
  const double b2 = (gamma - 1) * (e * d0 - u * d1 - v * d2 - w * d3 + d4);
  out[0] = b1 + lmd1 * d0;
  out[1] = u * b1 + kx * b2 + lmd1 * d1 + kx * (b3 - b4);
  out[2] = v * b1 + ky * b2 + lmd1 * d2 + ky * (b3 - b4);
  out[3] = w * b1 + kz * b2 + lmd1 * d3 + kz * (b3 - b4);
  out[4] = h * b1 + U * b2 + lmd1 * d4 + U * (b3 - b4);
  for (int l = 0; l < p->n_scalar; ++l) out[5 + l] = lmd1 * A(ORC_DQ, l + 5, i, j, k) + A(ORC_SV, l, i, j, k) * b1;
}

void orc_phase_implicit(orc_solver *s, int bi) {
  blk *B = &s->b[bi];
  const orc_params *p = &s->p;
  const int ns = p->ns;
  if (p->implicit_method == 0) {
    /* src/ImplicitTreatmentHPP.cuh:14-54 */
#pragma omp parallel for collapse(2) schedule(static) num_threads(s->nthreads)
    for (int k = 0; k < B->mz; ++k)
      for (int j = 0; j < B->my; ++j)
        for (int i = 0; i < B->mx; ++i) {
          const double dt = AS(ORC_DT_LOCAL, i, j, k);
          if (p->mix == 2 && p->chem_src_method == 1) {
            double lhs[ORC_MAX_SPEC * ORC_MAX_SPEC], rhs[ORC_MAX_SPEC];
            epi_lhs(p, B, i, j, k, 1.0, dt, lhs);
            for (int l = 0; l < ns; ++l) rhs[l] = A(ORC_DQ, 5 + l, i, j, k);
            lu_solve(lhs, rhs, ns);
            for (int l = 0; l < ns; ++l) A(ORC_DQ, 5 + l, i, j, k) = rhs[l];
          } else if (p->mix == 2 && p->chem_src_method == 2) {
            for (int l = 0; l < ns; ++l) A(ORC_DQ, 5 + l, i, j, k) /= 1 - dt * A(ORC_CHEM_JAC, l, i, j, k);
          }
          if (p->turb && p->turb_implicit == 1) {
            A(ORC_DQ, ns + 5, i, j, k) /= 1 - dt * A(ORC_TURB_SRC_JAC, 0, i, j, k);
            A(ORC_DQ, ns + 6, i, j, k) /= 1 - dt * A(ORC_TURB_SRC_JAC, 1, i, j, k);
          }
        }
    return;
  }
  /* DPLUR, src/DPLURHPP.cuh:13-76 (compute_DQ_0) and :127-273 */
  const int nv = p->n_var;
#pragma omp parallel for collapse(2) schedule(static) num_threads(s->nthreads)
  for (int k = 0; k < B->mz; ++k)
    for (int j = 0; j < B->my; ++j)
      for (int i = 0; i < B->mx; ++i) {
        const double dt = AS(ORC_DT_LOCAL, i, j, k);
        const double diag =
            1 + dt * (A(ORC_INV_SPEC, 0, i, j, k) + A(ORC_INV_SPEC, 1, i, j, k) + A(ORC_INV_SPEC, 2, i, j, k));
        if (p->mix != 2) {
          for (int l = 0; l < 5 + ns; ++l) A(ORC_DQ, l, i, j, k) /= diag;
        } else {
          for (int l = 0; l < 5; ++l) A(ORC_DQ, l, i, j, k) /= diag;
          if (p->chem_src_method == 1) {
            double lhs[ORC_MAX_SPEC * ORC_MAX_SPEC], rhs[ORC_MAX_SPEC];
            epi_lhs(p, B, i, j, k, diag, dt, lhs);
            for (int l = 0; l < ns; ++l) rhs[l] = A(ORC_DQ, 5 + l, i, j, k);
            lu_solve(lhs, rhs, ns);
            for (int l = 0; l < ns; ++l) A(ORC_DQ, 5 + l, i, j, k) = rhs[l];
          } else if (p->chem_src_method == 2) {
            for (int l = 0; l < ns; ++l) A(ORC_DQ, 5 + l, i, j, k) /= diag - dt * A(ORC_CHEM_JAC, l, i, j, k);
          } else {
            for (int l = 0; l < ns; ++l) A(ORC_DQ, l + 5, i, j, k) /= diag;
          }
        }
        if (p->turb) {
          if (p->turb_implicit == 1) {
            A(ORC_DQ, ns + 5, i, j, k) /= diag - dt * A(ORC_TURB_SRC_JAC, 0, i, j, k);
            A(ORC_DQ, ns + 6, i, j, k) /= diag - dt * A(ORC_TURB_SRC_JAC, 1, i, j, k);
          } else {
            A(ORC_DQ, ns + 5, i, j, k) /= diag;
            A(ORC_DQ, ns + 6, i, j, k) /= diag;
          }
        }
      }
  const int64_t bytes = sizeof(double) * B->size[B->gf[ORC_DQ]] * nv;
  memcpy(B->f[ORC_DQ0], B->f[ORC_DQ], bytes);
  const int mx = B->mx, my = B->my, mz = B->mz;
  for (int it = 0; it < p->dplur_inner_step; ++it) {
#pragma omp parallel for collapse(2) schedule(static) num_threads(s->nthreads)
    for (int k = 0; k < mz; ++k)
      for (int j = 0; j < my; ++j)
        for (int i = 0; i < mx; ++i) {
          double cj[MAXV], tot[MAXV];
          for (int l = 0; l < MAXV; ++l) tot[l] = 0;
          if (i > 0) {
            jac_times_dq(p, B, i - 1, j, k, 0, A(ORC_INV_SPEC, 0, i - 1, j, k), cj);
            for (int l = 0; l < nv; ++l) tot[l] += 0.5 * cj[l];
          }
          if (j > 0) {
            jac_times_dq(p, B, i, j - 1, k, 1, A(ORC_INV_SPEC, 1, i, j - 1, k), cj);
            for (int l = 0; l < nv; ++l) tot[l] += 0.5 * cj[l];
          }
          if (k > 0) {
            jac_times_dq(p, B, i, j, k - 1, 2, A(ORC_INV_SPEC, 2, i, j, k - 1), cj);
            for (int l = 0; l < nv; ++l) tot[l] += 0.5 * cj[l];
          }
          if (i != mx - 1) {
            jac_times_dq(p, B, i + 1, j, k, 0, -A(ORC_INV_SPEC, 0, i + 1, j, k), cj);
            for (int l = 0; l < nv; ++l) tot[l] -= 0.5 * cj[l];
          }
          if (j != my - 1) {
            jac_times_dq(p, B, i, j + 1, k, 1, -A(ORC_INV_SPEC, 1, i, j + 1, k), cj);
            for (int l = 0; l < nv; ++l) tot[l] -= 0.5 * cj[l];
          }
          if (k != mz - 1) {
            jac_times_dq(p, B, i, j, k + 1, 2, -A(ORC_INV_SPEC, 2, i, j, k + 1), cj);
            for (int l = 0; l < nv; ++l) tot[l] -= 0.5 * cj[l];
          }
          const double dt = AS(ORC_DT_LOCAL, i, j, k);
          const double diag =
              1 + dt * (A(ORC_INV_SPEC, 0, i, j, k) + A(ORC_INV_SPEC, 1, i, j, k) + A(ORC_INV_SPEC, 2, i, j, k));
          if (p->mix != 2) {
            for (int l = 0; l < 5 + ns; ++l) A(ORC_DQK, l, i, j, k) = A(ORC_DQ0, l, i, j, k) + dt * tot[l] / diag;
          } else {
            for (int l = 0; l < 5; ++l) A(ORC_DQK, l, i, j, k) = A(ORC_DQ0, l, i, j, k) + dt * tot[l] / diag;
            if (p->chem_src_method == 1) {
              /* EPI_for_dqk, src/FiniteRateChem.cu:255-284 */
              double lhs[ORC_MAX_SPEC * ORC_MAX_SPEC], rhs[ORC_MAX_SPEC];
              epi_lhs(p, B, i, j, k, diag, dt, lhs);
              for (int l = 0; l < ns; ++l) rhs[l] = tot[5 + l] * dt;
              lu_solve(lhs, rhs, ns);
              for (int l = 0; l < ns; ++l) A(ORC_DQK, l + 5, i, j, k) = A(ORC_DQ0, l + 5, i, j, k) + rhs[l];
            } else if (p->chem_src_method == 2) {
              for (int l = 0; l < ns; ++l)
                A(ORC_DQK, 5 + l, i, j, k) =
                    A(ORC_DQ0, 5 + l, i, j, k) + dt * tot[5 + l] / (diag - dt * A(ORC_CHEM_JAC, l, i, j, k));
            } else {
              for (int l = 0; l < ns; ++l) A(ORC_DQK, 5 + l, i, j, k) = A(ORC_DQ0, 5 + l, i, j, k) + dt * tot[5 + l] / diag;
            }
          }
          if (p->turb) {
            if (p->turb_implicit == 1) {
              A(ORC_DQK, ns + 5, i, j, k) =
                  A(ORC_DQ0, ns + 5, i, j, k) + dt * tot[5 + ns] / (diag - dt * A(ORC_TURB_SRC_JAC, 0, i, j, k));
              A(ORC_DQK, ns + 6, i, j, k) =
                  A(ORC_DQ0, ns + 6, i, j, k) + dt * tot[6 + ns] / (diag - dt * A(ORC_TURB_SRC_JAC, 1, i, j, k));
            } else {
              A(ORC_DQK, ns + 5, i, j, k) = A(ORC_DQ0, ns + 5, i, j, k) + dt * tot[5 + ns] / diag;
              A(ORC_DQK, ns + 6, i, j, k) = A(ORC_DQ0, ns + 6, i, j, k) + dt * tot[6 + ns] / diag;
            }
          }
        }
    memcpy(B->f[ORC_DQ], B->f[ORC_DQK], bytes);
  }
}

/* ------------------------------------------------------------------ update */
/* compute_temperature, src/FieldOperation.cu:3-40 */
static void newton_temperature(const orc_params *p, blk *B, int i, int j, int k) {
  const int ns = p->ns;
  double mw = 0;
  for (int l = 0; l < ns; ++l) mw += A(ORC_SV, l, i, j, k) / p->mw[l];
  mw = 1 / mw;
  const double gas_const = R_U / mw;
  const double u = A(ORC_BV, 1, i, j, k), v = A(ORC_BV, 2, i, j, k), w = A(ORC_BV, 3, i, j, k);
  const double e = A(ORC_CV, 4, i, j, k) / A(ORC_CV, 0, i, j, k) - 0.5 * (u * u + v * v + w * w);
  double err = 1, t = A(ORC_BV, 5, i, j, k);
  int iter = 0;
  double hi[ORC_MAX_SPEC], cpi[ORC_MAX_SPEC];
  while (err > 1e-3 && iter++ < 1000) {
    th_hcp(p, t, hi, cpi);
    double cp_tot = 0, h = 0;
    for (int l = 0; l < ns; ++l) {
      cp_tot += cpi[l] * A(ORC_SV, l, i, j, k);
      h += hi[l] * A(ORC_SV, l, i, j, k);
    }
    const double e_t = h - gas_const * t;
    const double cv = cp_tot - gas_const;
    const double t1 = t - (e_t - e) / cv;
    err = fabs(1 - t1 / t);
    t = t1;
  }
  A(ORC_BV, 5, i, j, k) = t;
  A(ORC_BV, 4, i, j, k) = A(ORC_BV, 0, i, j, k) * t * gas_const;
}

/* primitive recovery shared by update_cv_and_bv and update_bv_1_point,
   src/FieldOperation.cuh:158-183, 185-215 */
static void primitives_from_cv(const orc_params *p, blk *B, int i, int j, int k) {
  A(ORC_BV, 0, i, j, k) = A(ORC_CV, 0, i, j, k);
  const double rinv = 1.0 / A(ORC_CV, 0, i, j, k);
  A(ORC_BV, 1, i, j, k) = A(ORC_CV, 1, i, j, k) * rinv;
  A(ORC_BV, 2, i, j, k) = A(ORC_CV, 2, i, j, k) * rinv;
  A(ORC_BV, 3, i, j, k) = A(ORC_CV, 3, i, j, k) * rinv;
  double vel = A(ORC_BV, 1, i, j, k) * A(ORC_BV, 1, i, j, k) + A(ORC_BV, 2, i, j, k) * A(ORC_BV, 2, i, j, k) +
               A(ORC_BV, 3, i, j, k) * A(ORC_BV, 3, i, j, k);
  AS(ORC_VEL, i, j, k) = vel;
  if (p->mix != 0 || p->turb)
    for (int l = 0; l < p->n_scalar; ++l) A(ORC_SV, l, i, j, k) = A(ORC_CV, 5 + l, i, j, k) * rinv;
  if (p->mix != 0) {
    newton_temperature(p, B, i, j, k);
  } else {
    A(ORC_BV, 4, i, j, k) = (GAMMA_AIR - 1) * (A(ORC_CV, 4, i, j, k) - 0.5 * A(ORC_BV, 0, i, j, k) * vel);
    A(ORC_BV, 5, i, j, k) = A(ORC_BV, 4, i, j, k) * MW_AIR * rinv / R_U;
  }
  AS(ORC_VEL, i, j, k) = sqrt(vel);
}

/* compute_total_energy, src/FieldOperation.cuh:15-35 */
static void total_energy(const orc_params *p, blk *B, int i, int j, int k) {
  double vel = A(ORC_BV, 1, i, j, k) * A(ORC_BV, 1, i, j, k) + A(ORC_BV, 2, i, j, k) * A(ORC_BV, 2, i, j, k) +
               A(ORC_BV, 3, i, j, k) * A(ORC_BV, 3, i, j, k);
  AS(ORC_VEL, i, j, k) = vel;
  A(ORC_CV, 4, i, j, k) = 0.5 * A(ORC_BV, 0, i, j, k) * vel;
  if (p->mix != 0) {
    double h[ORC_MAX_SPEC];
    th_h(p, A(ORC_BV, 5, i, j, k), h);
    for (int l = 0; l < p->ns; ++l) A(ORC_CV, 4, i, j, k) += h[l] * A(ORC_CV, 5 + l, i, j, k);
    A(ORC_CV, 4, i, j, k) -= A(ORC_BV, 4, i, j, k);
  } else {
    A(ORC_CV, 4, i, j, k) += A(ORC_BV, 4, i, j, k) / (GAMMA_AIR - 1);
  }
  AS(ORC_VEL, i, j, k) = sqrt(vel);
}

static int unphysical_flow(const double *v, const double *ll, const double *ul) {
  for (int l = 0; l < 5; ++l) {
    if (isnan(v[l])) return 1;
    if (v[l] < ll[l] || v[l] > ul[l]) return 1;
  }
  return 0;
}

/* limit_flow, src/TimeAdvanceFunc.cu:34-224 (the neighbour loop bounds i1 by
   mz, as the reference does) */
static void limit_flow_point(const orc_params *p, blk *B, int i, int j, int k) {
  const int mx = B->mx, my = B->my, mz = B->mz, ns = p->ns, nsc = p->n_scalar;
  (void)mx;
  double var[5];
  for (int l = 0; l < 5; ++l) var[l] = A(ORC_BV, l, i, j, k);
  if (unphysical_flow(var, p->ll, p->ul)) {
    double up[5 + ORC_MAX_SPEC + 2];
    memset(up, 0, sizeof(up));
    int kn = 0;
    for (int ka = -1; ka < 2; ++ka) {
      const int k1 = k + ka;
      if (k1 < 0 || k1 >= mz) continue;
      for (int ja = -1; ja < 2; ++ja) {
        const int j1 = j + ja;
        if (j1 < 0 || j1 >= my) continue;
        for (int ia = -1; ia < 2; ++ia) {
          const int i1 = i + ia;
          if (i1 < 0 || i1 >= mz) continue;
          double nv5[5];
          for (int l = 0; l < 5; ++l) nv5[l] = A(ORC_BV, l, i1, j1, k1);
          if (isnan(nv5[0]) || isnan(nv5[1]) || isnan(nv5[2]) || isnan(nv5[3]) || isnan(nv5[4]) || nv5[0] < p->ll[0] ||
              nv5[1] < p->ll[1] || nv5[2] < p->ll[2] || nv5[3] < p->ll[3] || nv5[4] < p->ll[4] || nv5[0] > p->ul[0] ||
              nv5[1] > p->ul[1] || nv5[2] > p->ul[2] || nv5[3] > p->ul[3] || nv5[4] > p->ul[4])
            continue;
          for (int l = 0; l < 5; ++l) up[l] += nv5[l];
          for (int l = 0; l < nsc; ++l) up[l + 5] += A(ORC_SV, l, i1, j1, k1);
          ++kn;
        }
      }
    }
    if (kn > 0) {
      const double kinv = 1.0 / kn;
      for (int l = 0; l < 5 + nsc; ++l) up[l] *= kinv;
    } else {
      for (int l = 0; l < 5; ++l) {
        up[l] = dmax(var[l], p->ll[l]);
        up[l] = dmin(up[l], p->ul[l]);
      }
      for (int l = 0; l < nsc; ++l) up[l + 5] = p->sv_inf[l];
    }
    for (int l = 0; l < 5; ++l) A(ORC_BV, l, i, j, k) = up[l];
    A(ORC_CV, 0, i, j, k) = up[0];
    A(ORC_CV, 1, i, j, k) = up[0] * up[1];
    A(ORC_CV, 2, i, j, k) = up[0] * up[2];
    A(ORC_CV, 3, i, j, k) = up[0] * up[3];
    A(ORC_CV, 4, i, j, k) = 0.5 * up[0] * (up[1] * up[1] + up[2] * up[2] + up[3] * up[3]);
    for (int l = 0; l < nsc; ++l) {
      A(ORC_SV, l, i, j, k) = up[5 + l];
      A(ORC_CV, 5 + l, i, j, k) = up[0] * up[5 + l];
    }
    if (ns > 0) {
      double mw = 0;
      for (int l = 0; l < ns; ++l) mw += A(ORC_SV, l, i, j, k) / p->mw[l];
      mw = 1 / mw;
      A(ORC_BV, 5, i, j, k) = up[4] * mw / (up[0] * R_U);
      double h[ORC_MAX_SPEC];
      th_h(p, A(ORC_BV, 5, i, j, k), h);
      for (int l = 0; l < ns; l++) A(ORC_CV, 4, i, j, k) += h[l] * A(ORC_CV, 5 + l, i, j, k);
      A(ORC_CV, 4, i, j, k) -= A(ORC_BV, 4, i, j, k);
    } else {
      A(ORC_BV, 5, i, j, k) = up[4] * MW_AIR / (up[0] * R_U);
      A(ORC_CV, 4, i, j, k) += up[4] / (GAMMA_AIR - 1);
    }
  }
  if (p->rans_model == 2) {
    const double t0 = A(ORC_SV, ns, i, j, k), t1 = A(ORC_SV, ns + 1, i, j, k);
    if (isnan(t0) || isnan(t1) || t0 < 0 || t1 < 0) {
      double up[2] = {0, 0};
      int kn = 0;
      for (int ka = -1; ka < 2; ++ka) {
        const int k1 = k + ka;
        if (k1 < 0 || k1 >= mz) continue;
        for (int ja = -1; ja < 2; ++ja) {
          const int j1 = j + ja;
          if (j1 < 0 || j1 >= my) continue;
          for (int ia = -1; ia < 2; ++ia) {
            const int i1 = i + ia;
            if (i1 < 0 || i1 >= mz) continue;
            const double a0 = A(ORC_SV, ns, i1, j1, k1), a1 = A(ORC_SV, ns + 1, i1, j1, k1);
            if (isnan(a0) || isnan(a1) || a0 < 0 || a1 < 0) continue;
            up[0] += a0;
            up[1] += a1;
            ++kn;
          }
        }
      }
      if (kn > 0) {
        const double kinv = 1.0 / kn;
        up[0] *= kinv;
        up[1] *= kinv;
      } else {
        up[0] = t0 < 0 ? p->sv_inf[ns] : t0;
        up[1] = t1 < 0 ? p->sv_inf[ns + 1] : t1;
      }
      A(ORC_SV, ns, i, j, k) = up[0];
      A(ORC_SV, ns + 1, i, j, k) = up[1];
      A(ORC_CV, ns + 5, i, j, k) = A(ORC_CV, 0, i, j, k) * up[0];
      A(ORC_CV, ns + 6, i, j, k) = A(ORC_CV, 0, i, j, k) * up[1];
    }
  }
}

void orc_phase_update(orc_solver *s, int bi) {
  blk *B = &s->b[bi];
  const orc_params *p = &s->p;
  /* update_cv_and_bv, src/FieldOperation.cuh:139-183 */
#pragma omp parallel for collapse(2) schedule(static) num_threads(s->nthreads)
  for (int k = 0; k < B->mz; ++k)
    for (int j = 0; j < B->my; ++j)
      for (int i = 0; i < B->mx; ++i) {
        const double dt_div_jac = AS(ORC_DT_LOCAL, i, j, k) / AS(ORC_JAC, i, j, k);
        for (int l = 0; l < p->n_var; ++l) A(ORC_CV, l, i, j, k) += A(ORC_DQ, l, i, j, k) * dt_div_jac;
        if (B->mz == 1) A(ORC_CV, 3, i, j, k) = 0;
        primitives_from_cv(p, B, i, j, k);
      }
  /* limit_flow runs over the block after the update; serial here so the
     neighbour averages use a defined order. */
  for (int k = 0; k < B->mz; ++k)
    for (int j = 0; j < B->my; ++j)
      for (int i = 0; i < B->mx; ++i) limit_flow_point(p, B, i, j, k);
}

/* ------------------------------------------------------------------ boundary */
/* apply_outflow / apply_inflow / apply_symmetry / apply_wall, src/BoundCond.cuh:45-319 */
static void apply_bc(const orc_params *p, blk *B, const orc_bc *bc) {
  const int ngg = B->ngg, ns = p->ns, nsc = p->n_scalar;
  int dir[3] = {0, 0, 0};
  dir[bc->face] = bc->direction;
  for (int i = bc->start[0]; i <= bc->end[0]; ++i)
    for (int j = bc->start[1]; j <= bc->end[1]; ++j)
      for (int k = bc->start[2]; k <= bc->end[2]; ++k) {
        if (bc->type == 6) {
          for (int g = 1; g <= ngg; ++g) {
            const int gi = i + g * dir[0], gj = j + g * dir[1], gk = k + g * dir[2];
            for (int l = 0; l < 6; ++l) A(ORC_BV, l, gi, gj, gk) = A(ORC_BV, l, i, j, k);
            for (int l = 0; l < nsc; ++l) A(ORC_SV, l, gi, gj, gk) = A(ORC_SV, l, i, j, k);
            if (p->turb) AS(ORC_MUT, gi, gj, gk) = AS(ORC_MUT, i, j, k);
          }
        } else if (bc->type == 5) {
          for (int g = 1; g <= ngg; ++g) {
            const int gi = i + g * dir[0], gj = j + g * dir[1], gk = k + g * dir[2];
            A(ORC_BV, 0, gi, gj, gk) = bc->density;
            A(ORC_BV, 1, gi, gj, gk) = bc->u;
            A(ORC_BV, 2, gi, gj, gk) = bc->v;
            A(ORC_BV, 3, gi, gj, gk) = bc->w;
            A(ORC_BV, 4, gi, gj, gk) = bc->pressure;
            A(ORC_BV, 5, gi, gj, gk) = bc->temperature;
            for (int l = 0; l < nsc; ++l) A(ORC_SV, l, gi, gj, gk) = bc->sv[l];
            if (p->turb) AS(ORC_MUT, gi, gj, gk) = bc->mut;
          }
        } else if (bc->type == 3) {
          const int ii0 = i - dir[0], ij0 = j - dir[1], ik0 = k - dir[2];
          double k_x = MET(bc->face + 1, 1, i, j, k), k_y = MET(bc->face + 1, 2, i, j, k),
                 k_z = MET(bc->face + 1, 3, i, j, k);
          const double km = sqrt(k_x * k_x + k_y * k_y + k_z * k_z);
          k_x /= km;
          k_y /= km;
          k_z /= km;
          const double u1 = A(ORC_BV, 1, ii0, ij0, ik0), v1 = A(ORC_BV, 2, ii0, ij0, ik0), w1 = A(ORC_BV, 3, ii0, ij0, ik0);
          double u_k = k_x * u1 + k_y * v1 + k_z * w1;
          const double u_t = u1 - k_x * u_k, v_t = v1 - k_y * u_k, w_t = w1 - k_z * u_k;
          A(ORC_BV, 1, i, j, k) = u_t;
          A(ORC_BV, 2, i, j, k) = v_t;
          A(ORC_BV, 3, i, j, k) = w_t;
          AS(ORC_VEL, i, j, k) = sqrt(u_t * u_t + v_t * v_t + w_t * w_t);
          A(ORC_BV, 0, i, j, k) = A(ORC_BV, 0, ii0, ij0, ik0);
          A(ORC_BV, 4, i, j, k) = A(ORC_BV, 4, ii0, ij0, ik0);
          A(ORC_BV, 5, i, j, k) = A(ORC_BV, 5, ii0, ij0, ik0);
          for (int l = 0; l < nsc; ++l) A(ORC_SV, l, i, j, k) = A(ORC_SV, l, ii0, ij0, ik0);
          A(ORC_CV, 0, i, j, k) = A(ORC_BV, 0, i, j, k);
          A(ORC_CV, 1, i, j, k) = A(ORC_BV, 0, i, j, k) * A(ORC_BV, 1, i, j, k);
          A(ORC_CV, 2, i, j, k) = A(ORC_BV, 0, i, j, k) * A(ORC_BV, 2, i, j, k);
          A(ORC_CV, 3, i, j, k) = A(ORC_BV, 0, i, j, k) * A(ORC_BV, 3, i, j, k);
          A(ORC_CV, 4, i, j, k) = A(ORC_CV, 4, ii0, ij0, ik0) -
                                  0.5 * A(ORC_BV, 0, ii0, ij0, ik0) * (u1 * u1 + v1 * v1 + w1 * w1) +
                                  0.5 * A(ORC_BV, 0, i, j, k) * (u_t * u_t + v_t * v_t + w_t * w_t);
          for (int l = 0; l < nsc; ++l) A(ORC_CV, 5 + l, i, j, k) = A(ORC_BV, 0, i, j, k) * A(ORC_SV, l, i, j, k);
          for (int g = 1; g <= ngg; ++g) {
            const int gi = i + g * dir[0], gj = j + g * dir[1], gk = k + g * dir[2];
            const int ii = i - g * dir[0], ij = j - g * dir[1], ik = k - g * dir[2];
            A(ORC_BV, 0, gi, gj, gk) = A(ORC_BV, 0, ii, ij, ik);
            const double u = A(ORC_BV, 1, ii, ij, ik), v = A(ORC_BV, 2, ii, ij, ik), w = A(ORC_BV, 3, ii, ij, ik);
            u_k = k_x * u + k_y * v + k_z * w;
            A(ORC_BV, 1, gi, gj, gk) = u - 2 * u_k * k_x;
            A(ORC_BV, 2, gi, gj, gk) = v - 2 * u_k * k_y;
            A(ORC_BV, 3, gi, gj, gk) = w - 2 * u_k * k_z;
            AS(ORC_VEL, gi, gj, gk) =
                sqrt(A(ORC_BV, 1, gi, gj, gk) * A(ORC_BV, 1, gi, gj, gk) + A(ORC_BV, 2, gi, gj, gk) * A(ORC_BV, 2, gi, gj, gk) +
                     A(ORC_BV, 3, gi, gj, gk) * A(ORC_BV, 3, gi, gj, gk));
            A(ORC_BV, 4, gi, gj, gk) = A(ORC_BV, 4, ii, ij, ik);
            A(ORC_BV, 5, gi, gj, gk) = A(ORC_BV, 5, ii, ij, ik);
            for (int l = 0; l < nsc; ++l) A(ORC_SV, l, gi, gj, gk) = A(ORC_SV, l, ii, ij, ik);
            if (p->turb) AS(ORC_MUT, gi, gj, gk) = AS(ORC_MUT, ii, ij, ik);
          }
        } else if (bc->type == 2) {
          const int ix0 = i - dir[0], iy0 = j - dir[1], iz0 = k - dir[2];
          double t_wall = bc->t_wall;
          if (!bc->isothermal) t_wall = A(ORC_BV, 5, ix0, iy0, iz0);
          const double pw = A(ORC_BV, 4, ix0, iy0, iz0);
          double mw = MW_AIR;
          if (p->mix != 0) {
            mw = 0;
            for (int l = 0; l < ns; ++l) {
              A(ORC_SV, l, i, j, k) = A(ORC_SV, l, ix0, iy0, iz0);
              mw += A(ORC_SV, l, i, j, k) / p->mw[l];
            }
            mw = 1 / mw;
          }
          const double rho_wall = pw * mw / (t_wall * R_U);
          A(ORC_BV, 0, i, j, k) = rho_wall;
          A(ORC_BV, 1, i, j, k) = 0;
          A(ORC_BV, 2, i, j, k) = 0;
          A(ORC_BV, 3, i, j, k) = 0;
          A(ORC_BV, 4, i, j, k) = pw;
          A(ORC_BV, 5, i, j, k) = t_wall;
          A(ORC_CV, 0, i, j, k) = rho_wall;
          A(ORC_CV, 1, i, j, k) = 0;
          A(ORC_CV, 2, i, j, k) = 0;
          A(ORC_CV, 3, i, j, k) = 0;
          for (int l = 0; l < ns; ++l) A(ORC_CV, l + 5, i, j, k) = A(ORC_SV, l, i, j, k) * rho_wall;
          total_energy(p, B, i, j, k);
          if (p->turb && p->rans_model == 2) {
            double mu_wall;
            if (p->mix != 0) {
              double Y[ORC_MAX_SPEC];
              for (int l = 0; l < ns; ++l) Y[l] = A(ORC_SV, l, i, j, k);
              mu_wall = mix_viscosity(p, t_wall, mw, Y);
            } else {
              mu_wall = sutherland(t_wall);
            }
            const double dy = AS(ORC_WALL_DIST, ix0, iy0, iz0);
            A(ORC_SV, ns, i, j, k) = 0;
            A(ORC_CV, ns + 5, i, j, k) = 0;
            if (dy > 1e-25) {
              A(ORC_SV, ns + 1, i, j, k) = 60 * mu_wall / (rho_wall * SST_beta_1 * dy * dy);
            } else {
              A(ORC_SV, ns + 1, i, j, k) = A(ORC_SV, ns + 1, ix0, iy0, iz0);
            }
            A(ORC_CV, ns + 6, i, j, k) = rho_wall * A(ORC_SV, ns + 1, i, j, k);
          }
          for (int g = 1; g <= ngg; ++g) {
            const int a0 = i - g * dir[0], a1 = j - g * dir[1], a2 = k - g * dir[2];
            const int g0 = i + g * dir[0], g1 = j + g * dir[1], g2 = k + g * dir[2];
            const double u_i = A(ORC_BV, 1, a0, a1, a2), v_i = A(ORC_BV, 2, a0, a1, a2), w_i = A(ORC_BV, 3, a0, a1, a2);
            const double p_i = A(ORC_BV, 4, a0, a1, a2), t_i = A(ORC_BV, 5, a0, a1, a2);
            double t_g = t_i;
            if (bc->isothermal) {
              t_g = 2 * t_wall - t_i;
              if (t_g <= 0.1 * t_wall) t_g = t_wall;
            }
            if (p->mix != 0) {
              mw = 0;
              for (int l = 0; l < ns; ++l) {
                A(ORC_SV, l, g0, g1, g2) = A(ORC_SV, l, a0, a1, a2);
                mw += A(ORC_SV, l, g0, g1, g2) / p->mw[l];
              }
              mw = 1 / mw;
            }
            const double rho_g = p_i * mw / (t_g * R_U);
            A(ORC_BV, 0, g0, g1, g2) = rho_g;
            A(ORC_BV, 1, g0, g1, g2) = -u_i;
            A(ORC_BV, 2, g0, g1, g2) = -v_i;
            A(ORC_BV, 3, g0, g1, g2) = -w_i;
            A(ORC_BV, 4, g0, g1, g2) = p_i;
            A(ORC_BV, 5, g0, g1, g2) = t_g;
            if (p->turb && p->rans_model == 2) {
              A(ORC_SV, ns, g0, g1, g2) = 0;
              A(ORC_SV, ns + 1, g0, g1, g2) = A(ORC_SV, ns + 1, i, j, k);
              AS(ORC_MUT, g0, g1, g2) = 0;
            }
          }
        }
      }
}

void orc_phase_bc(orc_solver *s, int b) {
  for (int q = 0; q < s->nbc; ++q)
    if (s->bc[q].block == b) apply_bc(&s->p, &s->b[b], &s->bc[q]);
}

/* ------------------------------------------------------------------ exchange */
/* inner_communication, src/DataCommunication.cuh:58-98 */
static void inner_exchange(orc_solver *s, const orc_inner *f) {
  const orc_params *p = &s->p;
  blk *B = &s->b[f->block];
  blk *T = &s->b[f->target_block];
  const int face_dir = f->direction > 0 ? f->start[f->face] : f->end[f->face];
  for (int n0 = 0; n0 < f->n_point[0]; ++n0)
    for (int n1 = 0; n1 < f->n_point[1]; ++n1)
      for (int n2 = 0; n2 < f->n_point[2]; ++n2) {
        const int n[3] = {n0, n1, n2};
        int idx[3], it[3], d[3];
        for (int q = 0; q < 3; ++q) {
          d[q] = f->loop_dir[q] * n[q];
          idx[q] = f->start[q] + d[q];
        }
        for (int q = 0; q < 3; ++q) it[q] = f->tstart[q] + f->tloop_dir[q] * d[f->src_tar[q]];
        if (idx[f->face] == face_dir) {
          for (int l = 0; l < p->n_var; ++l) {
            double *a = &B->f[ORC_CV][(int64_t)l * B->size[B->gf[ORC_CV]] + IX(B, B->gf[ORC_CV], idx[0], idx[1], idx[2])];
            double *t = &T->f[ORC_CV][(int64_t)l * T->size[T->gf[ORC_CV]] + IX(T, T->gf[ORC_CV], it[0], it[1], it[2])];
            const double ave = 0.5 * (*t + *a);
            *a = ave;
            *t = ave;
          }
          primitives_from_cv(p, B, idx[0], idx[1], idx[2]);
        } else {
          for (int l = 0; l < 6; ++l)
            B->f[ORC_BV][(int64_t)l * B->size[B->gf[ORC_BV]] + IX(B, B->gf[ORC_BV], idx[0], idx[1], idx[2])] =
                T->f[ORC_BV][(int64_t)l * T->size[T->gf[ORC_BV]] + IX(T, T->gf[ORC_BV], it[0], it[1], it[2])];
          for (int l = 0; l < p->n_scalar; ++l)
            B->f[ORC_SV][(int64_t)l * B->size[B->gf[ORC_SV]] + IX(B, B->gf[ORC_SV], idx[0], idx[1], idx[2])] =
                T->f[ORC_SV][(int64_t)l * T->size[T->gf[ORC_SV]] + IX(T, T->gf[ORC_SV], it[0], it[1], it[2])];
        }
      }
}

/* eliminate_k_gradient, src/FieldOperation.cu:42-62 */
static void copy_k_layers(const orc_params *p, blk *B) {
  const int g = B->ngg;
  for (int i = -g; i < B->mx + g; ++i)
    for (int j = -g; j < B->my + g; ++j)
      for (int k = 1; k <= g; ++k) {
        for (int l = 0; l < 6; ++l) {
          A(ORC_BV, l, i, j, k) = A(ORC_BV, l, i, j, 0);
          A(ORC_BV, l, i, j, -k) = A(ORC_BV, l, i, j, 0);
        }
        for (int l = 0; l < p->n_scalar; ++l) {
          A(ORC_SV, l, i, j, k) = A(ORC_SV, l, i, j, 0);
          A(ORC_SV, l, i, j, -k) = A(ORC_SV, l, i, j, 0);
        }
      }
}

/* update_physical_properties + compute_transport_property,
   src/FieldOperation.cuh:75-109, src/Transport.cu:40-84 */
static void properties(orc_solver *s, blk *B) {
  const orc_params *p = &s->p;
  const int ns = p->ns;
#pragma omp parallel for collapse(2) schedule(static) num_threads(s->nthreads)
  for (int k = -1; k < B->mz + 1; ++k)
    for (int j = -1; j < B->my + 1; ++j)
      for (int i = -1; i < B->mx + 1; ++i) {
        const double t = A(ORC_BV, 5, i, j, k);
        if (p->mix != 0) {
          double mw = 0, cp_tot = 0, cv = 0, cp[ORC_MAX_SPEC], Y[ORC_MAX_SPEC];
          th_cp(p, t, cp);
          for (int l = 0; l < ns; ++l) {
            Y[l] = A(ORC_SV, l, i, j, k);
            mw += Y[l] / p->mw[l];
            cp_tot += Y[l] * cp[l];
            cv += Y[l] * (cp[l] - R_U / p->mw[l]);
          }
          mw = 1 / mw;
          AS(ORC_CP, i, j, k) = cp_tot;
          AS(ORC_GAMMA, i, j, k) = cp_tot / cv;
          AS(ORC_ACOUSTIC, i, j, k) = sqrt(AS(ORC_GAMMA, i, j, k) * R_U * t / mw);
          double X[ORC_MAX_SPEC], vis[ORC_MAX_SPEC];
          species_visc(p, t, mw, Y, X, vis);
          double viscosity = 0, conductivity = 0;
          for (int m = 0; m < ns; ++m) {
            double vt = 0;
            for (int n = 0; n < ns; ++n) vt += wilke_phi(p, vis, m, n) * X[n];
            const double cond_temp = 1.065 * vt - 0.065 * X[m];
            viscosity += vis[m] * X[m] / vt;
            const double lambda = vis[m] * (cp[m] + 1.25 * R_U / p->mw[m]);
            conductivity += lambda * X[m] / cond_temp;
          }
          AS(ORC_MUL, i, j, k) = viscosity;
          AS(ORC_CONDUCTIVITY, i, j, k) = conductivity;
          for (int l = 0; l < ns; ++l) {
            if (fabs(X[l] - 1) < 1e-3) {
              A(ORC_RHO_D, l, i, j, k) = viscosity / p->Sc;
            } else {
              A(ORC_RHO_D, l, i, j, k) = (1 - Y[l]) * viscosity / ((1 - X[l]) * p->Sc);
            }
          }
        } else {
          const double c_temp = GAMMA_AIR * R_U / MW_AIR;
          const double cp = GAMMA_AIR * R_U / MW_AIR / (GAMMA_AIR - 1);
          AS(ORC_ACOUSTIC, i, j, k) = sqrt(c_temp * t);
          AS(ORC_MUL, i, j, k) = sutherland(t);
          AS(ORC_CONDUCTIVITY, i, j, k) = AS(ORC_MUL, i, j, k) * cp / p->Pr;
        }
        AS(ORC_MACH, i, j, k) = AS(ORC_VEL, i, j, k) / AS(ORC_ACOUSTIC, i, j, k);
      }
}

void orc_phase_exchange(orc_solver *s) {
  for (int q = 0; q < s->ninner; ++q) inner_exchange(s, &s->inner[q]);
  if (s->dim == 2)
    for (int b = 0; b < s->nb; ++b) copy_k_layers(&s->p, &s->b[b]);
  for (int b = 0; b < s->nb; ++b) properties(s, &s->b[b]);
}

/* ------------------------------------------------------------------ driver */
static void wall_distance(orc_solver *s) {
  /* Driver::acquire_wall_distance + compute_wall_distance, src/Driver.cu:123-189, 461-482 */
  int64_t n = 0, cap = 1024;
  double *pts = malloc(sizeof(double) * 3 * cap);
  for (int q = 0; q < s->nbc; ++q) {
    const orc_bc *bc = &s->bc[q];
    if (bc->type != 2) continue;
    blk *B = &s->b[bc->block];
    for (int k = bc->start[2]; k <= bc->end[2]; ++k)
      for (int j = bc->start[1]; j <= bc->end[1]; ++j)
        for (int i = bc->start[0]; i <= bc->end[0]; ++i) {
          if (n == cap) {
            cap *= 2;
            pts = realloc(pts, sizeof(double) * 3 * cap);
          }
          pts[3 * n] = AS(ORC_X, i, j, k);
          pts[3 * n + 1] = AS(ORC_Y, i, j, k);
          pts[3 * n + 2] = AS(ORC_Z, i, j, k);
          ++n;
        }
  }
  for (int b = 0; b < s->nb; ++b) {
    blk *B = &s->b[b];
    const int g = B->ngg;
#pragma omp parallel for collapse(2) schedule(static) num_threads(s->nthreads)
    for (int k = -g; k < B->mz + g; ++k)
      for (int j = -g; j < B->my + g; ++j)
        for (int i = -g; i < B->mx + g; ++i) {
          const double x = AS(ORC_X, i, j, k), y = AS(ORC_Y, i, j, k), z = AS(ORC_Z, i, j, k);
          double wd = 1e+6;
          for (int64_t l = 0; l < n; ++l) {
            const double d = (x - pts[3 * l]) * (x - pts[3 * l]) + (y - pts[3 * l + 1]) * (y - pts[3 * l + 1]) +
                             (z - pts[3 * l + 2]) * (z - pts[3 * l + 2]);
            if (wd > d) wd = d;
          }
          AS(ORC_WALL_DIST, i, j, k) = sqrt(wd);
        }
  }
  free(pts);
}

int orc_initialize(orc_solver *s) {
  const orc_params *p = &s->p;
  if (p->turb && p->rans_model == 2) wall_distance(s);
  if (s->dim == 2)
    for (int b = 0; b < s->nb; ++b) copy_k_layers(p, &s->b[b]);
  for (int b = 0; b < s->nb; ++b) orc_phase_bc(s, b);
  for (int b = 0; b < s->nb; ++b) {
    blk *B = &s->b[b];
    const int g = B->ngg;
    /* compute_cv_from_bv, src/FieldOperation.cuh:37-73 */
    for (int k = -g; k < B->mz + g; ++k)
      for (int j = -g; j < B->my + g; ++j)
        for (int i = -g; i < B->mx + g; ++i) {
          const double rho = A(ORC_BV, 0, i, j, k);
          A(ORC_CV, 0, i, j, k) = rho;
          A(ORC_CV, 1, i, j, k) = rho * A(ORC_BV, 1, i, j, k);
          A(ORC_CV, 2, i, j, k) = rho * A(ORC_BV, 2, i, j, k);
          A(ORC_CV, 3, i, j, k) = rho * A(ORC_BV, 3, i, j, k);
          for (int l = 0; l < p->n_scalar; ++l) A(ORC_CV, 5 + l, i, j, k) = rho * A(ORC_SV, l, i, j, k);
          total_energy(p, B, i, j, k);
        }
    if (p->turb && p->rans_model == 2) {
      /* initialize_mut, src/FieldOperation.cuh:111-137 */
      for (int k = -1; k < B->mz + 1; ++k)
        for (int j = -1; j < B->my + 1; ++j)
          for (int i = -1; i < B->mx + 1; ++i) {
            const double t = A(ORC_BV, 5, i, j, k);
            double mul = sutherland(t);
            if (p->mix != 0) {
              double mw = 0, Y[ORC_MAX_SPEC];
              for (int l = 0; l < p->ns; ++l) {
                Y[l] = A(ORC_SV, l, i, j, k);
                mw += Y[l] / p->mw[l];
              }
              mw = 1 / mw;
              mul = mix_viscosity(p, t, mw, Y);
            }
            sst_mut(p, B, i, j, k, mul);
          }
    }
  }
  /* data_communication then update_physical_properties; unlike the step
     loop there is no 2-D k copy here (src/Driver.cu:91-103) */
  for (int q = 0; q < s->ninner; ++q) inner_exchange(s, &s->inner[q]);
  for (int b = 0; b < s->nb; ++b) properties(s, &s->b[b]);
  return 0;
}

int orc_step(orc_solver *s, int step, double res[4]) {
  const int screen = s->p.output_screen > 0 ? s->p.output_screen : 1;
  if (step % screen == 0) {
    for (int b = 0; b < s->nb; ++b) {
      blk *B = &s->b[b];
      for (int k = 0; k < B->mz; ++k)
        for (int j = 0; j < B->my; ++j)
          for (int i = 0; i < B->mx; ++i) {
            A(ORC_BV_LAST, 0, i, j, k) = A(ORC_BV, 0, i, j, k);
            A(ORC_BV_LAST, 1, i, j, k) = AS(ORC_VEL, i, j, k);
            A(ORC_BV_LAST, 2, i, j, k) = A(ORC_BV, 4, i, j, k);
            A(ORC_BV_LAST, 3, i, j, k) = A(ORC_BV, 5, i, j, k);
          }
    }
  }
  for (int b = 0; b < s->nb; ++b) {
    orc_phase_residual(s, b);
    orc_phase_implicit(s, b);
    orc_phase_update(s, b);
    orc_phase_bc(s, b);
  }
  orc_phase_exchange(s);
  if (step % screen == 0 || step == 1) {
    /* compute_square_of_dbv + reduction, src/TimeAdvanceFunc.cu:18-32, src/Driver.cu:292-339 */
    double sum[4] = {0, 0, 0, 0};
    for (int b = 0; b < s->nb; ++b) {
      blk *B = &s->b[b];
      for (int k = 0; k < B->mz; ++k)
        for (int j = 0; j < B->my; ++j)
          for (int i = 0; i < B->mx; ++i) {
            const double cur[4] = {A(ORC_BV, 0, i, j, k), AS(ORC_VEL, i, j, k), A(ORC_BV, 4, i, j, k),
                                   A(ORC_BV, 5, i, j, k)};
            for (int l = 0; l < 4; ++l) {
              const double d = cur[l] - A(ORC_BV_LAST, l, i, j, k);
              sum[l] += d * d;
            }
          }
    }
    for (int l = 0; l < 4; ++l) res[l] = sqrt(sum[l] / (double)s->n_grid_total);
    return 1;
  }
  return 0;
}

/* ------------------------------------------------------------------ setup */
orc_solver *orc_create(const orc_params *p, int n_block, const int *dims, int ngg, int n_threads) {
  orc_solver *s = calloc(1, sizeof(orc_solver));
  s->p = *p;
  s->nb = n_block;
  s->ngg = ngg;
  s->nthreads = n_threads > 0 ? n_threads : 1;
  s->dim = dims[2] == 1 ? 2 : 3;
  s->b = calloc(n_block, sizeof(blk));
  const int dplur = p->implicit_method == 1;
  for (int b = 0; b < n_block; ++b) {
    blk *B = &s->b[b];
    B->mx = dims[3 * b];
    B->my = dims[3 * b + 1];
    B->mz = dims[3 * b + 2];
    B->ngg = ngg;
    s->n_grid_total += (int64_t)B->mx * B->my * B->mz;
    for (int g = 0; g < 4; ++g) {
      B->sx[g] = B->mx + 2 * g;
      B->sxy[g] = B->sx[g] * (B->my + 2 * g);
      B->size[g] = B->sxy[g] * (B->mz + 2 * g);
      B->off[g] = (B->sxy[g] + B->sx[g] + 1) * g;
    }
    const int ns = p->ns;
    struct {
      int f, g, nc;
    } spec[] = {
        {ORC_X, ngg, 1},       {ORC_Y, ngg, 1},        {ORC_Z, ngg, 1},        {ORC_JAC, ngg, 1},
        {ORC_METRIC, ngg, 9},  {ORC_WALL_DIST, ngg, 1}, {ORC_BV, ngg, 6},      {ORC_SV, ngg, p->n_scalar},
        {ORC_CV, ngg, p->n_var}, {ORC_VEL, ngg, 1},    {ORC_ACOUSTIC, ngg, 1}, {ORC_MACH, ngg, 1},
        {ORC_MUL, ngg, 1},     {ORC_CONDUCTIVITY, ngg, 1}, {ORC_RHO_D, ngg, ns}, {ORC_GAMMA, ngg, 1},
        {ORC_CP, ngg, 1},      {ORC_MUT, ngg, 1},      {ORC_TURB_COND, ngg, 1},
        {ORC_CHEM_JAC, 0, p->chem_src_method == 2 ? ns : ns * ns},
        {ORC_TURB_SRC_JAC, 0, 2}, {ORC_DQ, dplur, p->n_var}, {ORC_DQ0, dplur, p->n_var},
        {ORC_DQK, dplur, p->n_var}, {ORC_INV_SPEC, dplur, 3}, {ORC_VISC_SPEC, dplur, 1},
        {ORC_DT_LOCAL, 0, 1},  {ORC_BV_LAST, 0, 4}};
    for (size_t q = 0; q < sizeof(spec) / sizeof(spec[0]); ++q) {
      const int f = spec[q].f;
      B->gf[f] = spec[q].g;
      B->nc[f] = spec[q].nc;
      const int64_t cnt = B->size[spec[q].g] * (spec[q].nc > 0 ? spec[q].nc : 0);
      B->f[f] = cnt > 0 ? calloc((size_t)cnt, sizeof(double)) : NULL;
    }
  }
  return s;
}

void orc_destroy(orc_solver *s) {
  if (!s) return;
  for (int b = 0; b < s->nb; ++b)
    for (int f = 0; f < ORC_N_FIELDS; ++f) free(s->b[b].f[f]);
  free(s->b);
  free(s->bc);
  free(s->inner);
  free(s);
}

double *orc_array(orc_solver *s, int block, int field, int64_t *count) {
  if (block < 0 || block >= s->nb || field < 0 || field >= ORC_N_FIELDS) return NULL;
  blk *B = &s->b[block];
  if (count) *count = B->f[field] ? B->size[B->gf[field]] * B->nc[field] : 0;
  return B->f[field];
}

int orc_add_bc(orc_solver *s, const orc_bc *bc) {
  if (s->nbc == s->cap_bc) {
    s->cap_bc = s->cap_bc ? 2 * s->cap_bc : 16;
    s->bc = realloc(s->bc, sizeof(orc_bc) * s->cap_bc);
  }
  s->bc[s->nbc++] = *bc;
  return 0;
}

int orc_add_inner(orc_solver *s, const orc_inner *f) {
  if (s->ninner == s->cap_inner) {
    s->cap_inner = s->cap_inner ? 2 * s->cap_inner : 16;
    s->inner = realloc(s->inner, sizeof(orc_inner) * s->cap_inner);
  }
  s->inner[s->ninner++] = *f;
  return 0;
}
