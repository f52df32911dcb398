// FP32-bulk / FP64-critical kernels of the reacting-RANS step.
//
// Same discretisation and step structure as the FP64 kernels (and the
// reference), with the precision split:
//   FP32: reconstruction and limiter, mixture thermodynamics at faces, AUSM+
//         and viscous fluxes, local time step, SST source, DPLUR flux-Jacobian
//         products, transport properties (mu, lambda, rho D, cp, gamma, a);
//   FP64: the state arrays and the conservative update accumulation, the
//         temperature Newton inversion (k_update), the finite-rate chemistry
//         with its equilibrium constants exp(-dG/RT) and reverse rates, the
//         point-implicit (EPI) Jacobian and its LU solve, the residual norms.
// Device arrays stay FP64 (one state for both paths); the FP32 kernels
// convert on load and round their results back on store.
#pragma once

#include "kernels_step.cuh"

namespace ostc {

// Float copies of the tables the FP32 kernels read.
struct MixParams {
  float mw[kMaxSpec], mw_inv[kMaxSpec], ru_mw[kMaxSpec], t_low[kMaxSpec], t_mid[kMaxSpec];
  float low[kMaxSpec * 7], high[kMaxSpec * 7];
  float lj_inv[kMaxSpec], vis_coeff[kMaxSpec];
  float wq[kMaxSpec * kMaxSpec], w8[kMaxSpec * kMaxSpec];
  float cfl, Pr, Prt, Sct, Sc;
};

static __constant__ MixParams cF;

inline MixParams make_mix_params(const DevParams &p) {
  MixParams f{};
  for (int i = 0; i < kMaxSpec; ++i) {
    f.mw[i] = static_cast<float>(p.mw[i]);
    f.mw_inv[i] = p.mw[i] != 0 ? static_cast<float>(1.0 / p.mw[i]) : 0.f;
    f.ru_mw[i] = static_cast<float>(p.ru_mw[i]);
    f.t_low[i] = static_cast<float>(p.t_low[i]);
    f.t_mid[i] = static_cast<float>(p.t_mid[i]);
    f.lj_inv[i] = static_cast<float>(p.lj_inv[i]);
    f.vis_coeff[i] = static_cast<float>(p.vis_coeff[i]);
  }
  for (int i = 0; i < kMaxSpec * 7; ++i) {
    f.low[i] = static_cast<float>(p.low[i]);
    f.high[i] = static_cast<float>(p.high[i]);
  }
  for (int i = 0; i < kMaxSpec * kMaxSpec; ++i) {
    f.wq[i] = static_cast<float>(p.wq[i]);
    f.w8[i] = static_cast<float>(p.w8[i]);
  }
  f.cfl = static_cast<float>(p.cfl);
  f.Pr = static_cast<float>(p.Pr);
  f.Prt = static_cast<float>(p.Prt);
  f.Sct = static_cast<float>(p.Sct);
  f.Sc = static_cast<float>(p.Sc);
  return f;
}

namespace fp32 {

// tanh of a non-negative argument from one hardware exponential:
// 1 - 2 / (e^{2x} + 1) (relative error near 1e-6; 1 where e^{2x} overflows).
// The SST blending functions F1, F2 take it.
__device__ __forceinline__ float tanh_pos(float x) { return 1.f - __fdividef(2.f, __expf(2.f * x) + 1.f); }

constexpr float kRu = 8314.462618f;

__device__ __forceinline__ float ldf(const double *p) { return static_cast<float>(__ldg(p)); }

__device__ __forceinline__ float minmod(float a, float b) {
  return 0.5f * ((a < 0 ? -1.f : 1.f) + (b < 0 ? -1.f : 1.f)) * fminf(fabsf(a), fabsf(b));
}

// NASA-7 polynomial coefficient q of species i (two ranges)
__device__ __forceinline__ float nasa(int i, int q, bool lowrange) {
  return lowrange ? cF.low[i * 7 + q] : cF.high[i * 7 + q];
}

// Species h_k and cp_k (J/kg, J/kg/K) at t; below T_low h is extrapolated
// linearly with cp frozen, as in the FP64 path.
template <int NS, bool WANT_H, bool WANT_CP>
__device__ __forceinline__ void thermo(float t, float *h, float *cp) {
  OSTC_UNROLL for (int i = 0; i < NS; ++i) {
    const bool below = t < cF.t_low[i];
    const float tt = below ? cF.t_low[i] : t;
    const bool lo = below || tt < cF.t_mid[i];
    const float c0 = nasa(i, 0, lo), c1 = nasa(i, 1, lo), c2 = nasa(i, 2, lo), c3 = nasa(i, 3, lo),
                c4 = nasa(i, 4, lo);
    const float c = c0 + tt * (c1 + tt * (c2 + tt * (c3 + tt * c4)));
    if constexpr (WANT_H) {
      float hh = tt * (c0 + tt * (0.5f * c1 + tt * (c2 * (1.f / 3.f) + tt * (0.25f * c3 + tt * (0.2f * c4))))) +
                 nasa(i, 5, lo);
      if (below) hh += c * (t - tt);
      h[i] = hh * cF.ru_mw[i];
    }
    if constexpr (WANT_CP) cp[i] = c * cF.ru_mw[i];
  }
}

// Where the FP32 kernels read their operands (index n of layout G):
// Src64 converts the FP64 state arrays on load; Src32 reads their FP32 copy
// (DevBlock::f32, written once per step by k_pack32 and, for the geometry,
// once per run by k_pack32_static), half the bytes and no conversion.
// prim(v, n): primitive v, 0..5 the basic variables (rho, u, v, w, p, T),
// 6.. the scalars (Y_k, k, omega).
struct Src64 {
  const DevBlock &B;
  __device__ __forceinline__ float prim(int v, int64_t n) const {
    return ldf((v < 6 ? B.bv + v * B.G.size : B.sv + (v - 6) * B.G.size) + n);
  }
  __device__ __forceinline__ float metric(int q, int64_t n) const { return ldf(B.metric + q * B.G.size + n); }
  __device__ __forceinline__ float jac(int64_t n) const { return ldf(B.jac + n); }
  __device__ __forceinline__ float mul(int64_t n) const { return ldf(B.mul + n); }
  __device__ __forceinline__ float mut(int64_t n) const { return ldf(B.mut + n); }
  __device__ __forceinline__ float cond(int64_t n) const { return ldf(B.cond + n); }
  __device__ __forceinline__ float tcond(int64_t n) const { return ldf(B.turb_cond + n); }
  __device__ __forceinline__ float rho_d(int l, int64_t n) const { return ldf(B.rho_d + l * B.G.size + n); }
  __device__ __forceinline__ float wall(int64_t n) const { return ldf(B.wall_dist + n); }
  __device__ __forceinline__ float acoustic(int64_t n) const { return ldf(B.acoustic + n); }
  __device__ __forceinline__ float gamma(int64_t n) const { return ldf(B.gamma + n); }
};

// Component offsets of the FP32 copy (each component B.G.size floats).
template <class C>
struct F32 {
  static constexpr int prim = 0, mul = 6 + C::nsc, mut = mul + 1, cond = mul + 2, tcond = mul + 3, rho_d = mul + 4,
                       acoustic = rho_d + C::ns, gamma = acoustic + 1,
                       n_dynamic = gamma + 1,  // written every step
                       wall = n_dynamic, jac = wall + 1, metric = jac + 1, count = metric + 9;
};

template <class C>
struct Src32 {
  const float *f;
  int64_t sz;
  __device__ __forceinline__ float at(int c, int64_t n) const { return __ldg(f + c * sz + n); }
  __device__ __forceinline__ float prim(int v, int64_t n) const { return at(F32<C>::prim + v, n); }
  __device__ __forceinline__ float metric(int q, int64_t n) const { return at(F32<C>::metric + q, n); }
  __device__ __forceinline__ float jac(int64_t n) const { return at(F32<C>::jac, n); }
  __device__ __forceinline__ float mul(int64_t n) const { return at(F32<C>::mul, n); }
  __device__ __forceinline__ float mut(int64_t n) const { return at(F32<C>::mut, n); }
  __device__ __forceinline__ float cond(int64_t n) const { return at(F32<C>::cond, n); }
  __device__ __forceinline__ float tcond(int64_t n) const { return at(F32<C>::tcond, n); }
  __device__ __forceinline__ float rho_d(int l, int64_t n) const { return at(F32<C>::rho_d + l, n); }
  __device__ __forceinline__ float wall(int64_t n) const { return at(F32<C>::wall, n); }
  __device__ __forceinline__ float acoustic(int64_t n) const { return at(F32<C>::acoustic, n); }
  __device__ __forceinline__ float gamma(int64_t n) const { return at(F32<C>::gamma, n); }
};

// h_k and cp_k of species i at t (thermo<> for one species)
__device__ __forceinline__ void thermo_one(int i, float t, float &h, float &cp) {
  const bool below = t < cF.t_low[i];
  const float tt = below ? cF.t_low[i] : t;
  const bool lo = below || tt < cF.t_mid[i];
  const float c0 = nasa(i, 0, lo), c1 = nasa(i, 1, lo), c2 = nasa(i, 2, lo), c3 = nasa(i, 3, lo),
              c4 = nasa(i, 4, lo);
  const float c = c0 + tt * (c1 + tt * (c2 + tt * (c3 + tt * c4)));
  float hh = tt * (c0 + tt * (0.5f * c1 + tt * (c2 * (1.f / 3.f) + tt * (0.25f * c3 + tt * (0.2f * c4))))) +
             nasa(i, 5, lo);
  if (below) hh += c * (t - tt);
  h = hh * cF.ru_mw[i];
  cp = c * cF.ru_mw[i];
}

// ------------------------------------------------------------ inviscid face
// The face functions read the primitive stencil through a reader, so that one
// copy of the physics serves the kernels that load it from the FP64 arrays
// and the one that stages it in shared memory.  Primitive index v: 0..5 the
// basic variables (rho, u, v, w, p, T), 6.. the scalars (Y_k, k, omega);
// flux variable l is primitive l below 5 and l + 1 from 5 on.

// get(l, q): flux variable l at cell c + q (q = -1..2) of the face between
// cell c (linear index n) and c + 1 (n + s).
template <class C, class Src, class Get>
__device__ __forceinline__ void inviscid_face_r(const Src &S, int64_t n, int d, int64_t s, Get &&get,
                                                float *fc) {
  constexpr int NV = C::nv, NS = C::ns;
  float pl[NV + 2], pr[NV + 2];
  const int rec = cP.reconstruction;
  OSTC_UNROLL for (int l = 0; l < NV; ++l) {
    const float p0 = get(l, 0), p1 = get(l, 1);
    if (rec == 2 || rec == 3) {
      const float pm = get(l, -1), p2 = get(l, 2);
      const float d_i = p0 - pm, d_i1 = p1 - p0, d_i2 = p2 - p1;
      if (rec == 2) {
        const float neg_l = minmod(d_i, d_i1), pos_l = minmod(d_i1, d_i);
        const float neg_r = minmod(d_i1, d_i2), pos_r = minmod(d_i2, d_i1);
        pl[l] = p0 + 0.25f * ((2.f / 3.f) * neg_l + (4.f / 3.f) * pos_l);
        pr[l] = p1 - 0.25f * ((2.f / 3.f) * pos_r + (4.f / 3.f) * neg_r);
      } else {
        pl[l] = p0 + 0.5f * minmod(d_i, d_i1);
        pr[l] = p1 - 0.5f * minmod(d_i1, d_i2);
      }
    } else {
      pl[l] = p0;
      pr[l] = p1;
    }
  }
  float el = 0.5f * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]);
  float er = 0.5f * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]);
  if constexpr (C::mix != 0) {
    float mwl = 0, mwr = 0;
    OSTC_UNROLL for (int l = 0; l < NS; ++l) {
      mwl += pl[5 + l] * cF.mw_inv[l];
      mwr += pr[5 + l] * cF.mw_inv[l];
    }
    const float tl = pl[4] / (pl[0] * kRu * mwl);
    const float tr = pr[4] / (pr[0] * kRu * mwr);
    float cpl = 0, cpr = 0, cvl = 0, cvr = 0;
    OSTC_UNROLL for (int l = 0; l < NS; ++l) {
      float hl, hr, cpl_l, cpr_l;
      thermo_one(l, tl, hl, cpl_l);
      thermo_one(l, tr, hr, cpr_l);
      cpl += cpl_l * pl[l + 5];
      cpr += cpr_l * pr[l + 5];
      cvl += pl[l + 5] * (cpl_l - cF.ru_mw[l]);
      cvr += pr[l + 5] * (cpr_l - cF.ru_mw[l]);
      el += hl * pl[l + 5];
      er += hr * pr[l + 5];
    }
    pl[NV] = pl[0] * el - pl[4];
    pr[NV] = pr[0] * er - pr[4];
    pl[NV + 1] = cpl / cvl;
    pr[NV + 1] = cpr / cvr;
  } else {
    constexpr float g1 = 1.f / (1.4f - 1.f);
    pl[NV] = el * pl[0] + pl[4] * g1;
    pr[NV] = er * pr[0] + pr[4] * g1;
    pl[NV + 1] = 1.4f;
    pr[NV + 1] = 1.4f;
  }
  const int q0 = 3 * d;
  const float jl = S.jac(n), jr = S.jac(n + s);
  const float k1 = 0.5f * (jl * S.metric(q0, n) + jr * S.metric(q0, n + s));
  const float k2 = 0.5f * (jl * S.metric(q0 + 1, n) + jr * S.metric(q0 + 1, n + s));
  const float k3 = 0.5f * (jl * S.metric(q0 + 2, n) + jr * S.metric(q0 + 2, n + s));
  const float gk = sqrtf(k1 * k1 + k2 * k2 + k3 * k3);
  const float inv_gk = 1.f / gk;
  const float ul = (k1 * pl[1] + k2 * pl[2] + k3 * pl[3]) * inv_gk;
  const float ur = (k1 * pr[1] + k2 * pr[2] + k3 * pr[3]) * inv_gk;
  const float p_l = pl[4], p_r = pr[4], rho_l = pl[0], rho_r = pr[0];
  const float c = 0.5f * (sqrtf(pl[NV + 1] * p_l / rho_l) + sqrtf(pr[NV + 1] * p_r / rho_r));
  const float inv_c = 1.f / c;
  const float mach_l = ul * inv_c, mach_r = ur * inv_c;
  float mlp, mrn, plp, prn;
  constexpr float alpha = 3.f / 16.f;
  if (fabsf(mach_l) > 1) {
    mlp = 0.5f * (mach_l + fabsf(mach_l));
    plp = mlp / mach_l;
  } else {
    const float a = (mach_l + 1) * (mach_l + 1) * 0.25f;
    const float b = (mach_l * mach_l - 1) * (mach_l * mach_l - 1);
    mlp = a + 0.125f * b;
    plp = a * (2 - mach_l) + alpha * mach_l * b;
  }
  if (fabsf(mach_r) > 1) {
    mrn = 0.5f * (mach_r - fabsf(mach_r));
    prn = mrn / mach_r;
  } else {
    const float a = (mach_r - 1) * (mach_r - 1) * 0.25f;
    const float b = (mach_r * mach_r - 1) * (mach_r * mach_r - 1);
    mrn = -a - 0.125f * b;
    prn = a * (2 + mach_r) - alpha * mach_r * b;
  }
  const float p_coeff = plp * p_l + prn * p_r;
  const float m_half = mlp + mrn;
  const float mach_pos = 0.5f * (m_half + fabsf(m_half));
  const float mach_neg = 0.5f * (m_half - fabsf(m_half));
  const float mass_flux_half = c * (rho_l * mach_pos + rho_r * mach_neg);
  const float coeff = mass_flux_half * gk;
  const bool up = mass_flux_half >= 0;
  // upwind state, selected per element so that pl / pr stay in registers
  auto q = [&](int l) { return up ? pl[l] : pr[l]; };
  fc[0] = coeff;
  fc[1] = coeff * q(1) + p_coeff * k1;
  fc[2] = coeff * q(2) + p_coeff * k2;
  fc[3] = coeff * q(3) + p_coeff * k3;
  fc[4] = coeff * (q(NV) + q(4)) / q(0);
  OSTC_UNROLL for (int l = 5; l < NV; ++l) fc[l] = coeff * q(l);
}

template <class C, class Src>
__device__ __forceinline__ void inviscid_face_s(const Src &S, int64_t n, int d, int64_t s, float *fc) {
  inviscid_face_r<C>(S, n, d, s, [&](int l, int q) { return S.prim(l < 5 ? l : l + 1, n + q * s); }, fc);
}

template <class C>
__device__ __forceinline__ void inviscid_face(const DevBlock &B, int64_t n, int d, int64_t s, float *fc) {
  inviscid_face_s<C>(Src64{B}, n, d, s, fc);
}

// ------------------------------------------------------------- viscous face
// a(q): the variable at linear index q
template <class A>
__device__ __forceinline__ void face_grad(A &&a, int64_t n, int64_t n1, int d, int64_t sx, int64_t sxy, float &dxi,
                                          float &deta, float &dzeta) {
  dxi = d == 0 ? a(n1) - a(n) : 0.25f * (a(n + 1) - a(n - 1) + a(n1 + 1) - a(n1 - 1));
  deta = d == 1 ? a(n1) - a(n) : 0.25f * (a(n + sx) - a(n - sx) + a(n1 + sx) - a(n1 - sx));
  dzeta = d == 2 ? a(n1) - a(n) : 0.25f * (a(n + sxy) - a(n - sxy) + a(n1 + sxy) - a(n1 - sxy));
}

// val(v, side): primitive v at cell c (side 0) or c + 1 (side 1) of the face;
// grad(v, g_xi, g_eta, g_zeta): its computational-space gradient at the face
// (the face_grad stencil).
template <class C, class Src, class Val, class Grad>
__device__ __forceinline__ void viscous_face_r(const Src &S, int64_t n, int d, int64_t s, Val &&val,
                                               Grad &&grad, float *fv) {
  constexpr int NS = C::ns;
  const int64_t n1 = n + s;
  float mm[9];
  OSTC_UNROLL for (int q = 0; q < 9; ++q) mm[q] = 0.5f * (S.metric(q, n) + S.metric(q, n1));
  const float xi_x = mm[0], xi_y = mm[1], xi_z = mm[2], eta_x = mm[3], eta_y = mm[4], eta_z = mm[5];
  const float zeta_x = mm[6], zeta_y = mm[7], zeta_z = mm[8];
  auto cart = [&](float a_xi, float a_eta, float a_zeta, float &ax, float &ay, float &az) {
    ax = a_xi * xi_x + a_eta * eta_x + a_zeta * zeta_x;
    ay = a_xi * xi_y + a_eta * eta_y + a_zeta * zeta_y;
    az = a_xi * xi_z + a_eta * eta_z + a_zeta * zeta_z;
  };
  float g0, g1, g2;
  float u_x, u_y, u_z, v_x, v_y, v_z, w_x, w_y, w_z, t_x, t_y, t_z;
  grad(1, g0, g1, g2);
  cart(g0, g1, g2, u_x, u_y, u_z);
  grad(2, g0, g1, g2);
  cart(g0, g1, g2, v_x, v_y, v_z);
  grad(3, g0, g1, g2);
  cart(g0, g1, g2, w_x, w_y, w_z);
  grad(5, g0, g1, g2);
  cart(g0, g1, g2, t_x, t_y, t_z);
  const float mul = 0.5f * (S.mul(n) + S.mul(n1));
  float mut = 0;
  if constexpr (C::turb) mut = 0.5f * (S.mut(n) + S.mut(n1));
  const float viscosity = mul + mut;
  constexpr float third = 1.f / 3.f;
  float tau_xx = viscosity * (4 * u_x - 2 * v_y - 2 * w_z) * third;
  float tau_yy = viscosity * (4 * v_y - 2 * u_x - 2 * w_z) * third;
  float tau_zz = viscosity * (4 * w_z - 2 * u_x - 2 * v_y) * third;
  const float tau_xy = viscosity * (u_y + v_x);
  const float tau_xz = viscosity * (u_z + w_x);
  const float tau_yz = viscosity * (v_z + w_y);
  if constexpr (C::turb) {
    const float tt = -(1.f / 3.f) * (val(0, 0) * val(6 + NS, 0) + val(0, 1) * val(6 + NS, 1));
    tau_xx += tt;
    tau_yy += tt;
    tau_zz += tt;
  }
  const int q0 = 3 * d;
  const float ja = S.jac(n), jb = S.jac(n1);
  const float kx = 0.5f * (S.metric(q0, n) * ja + S.metric(q0, n1) * jb);
  const float ky = 0.5f * (S.metric(q0 + 1, n) * ja + S.metric(q0 + 1, n1) * jb);
  const float kz = 0.5f * (S.metric(q0 + 2, n) * ja + S.metric(q0 + 2, n1) * jb);
  fv[0] = 0;
  fv[1] = kx * tau_xx + ky * tau_xy + kz * tau_xz;
  fv[2] = kx * tau_xy + ky * tau_yy + kz * tau_yz;
  fv[3] = kx * tau_xz + ky * tau_yz + kz * tau_zz;
  const float um = 0.5f * (val(1, 0) + val(1, 1));
  const float vm = 0.5f * (val(2, 0) + val(2, 1));
  const float wm = 0.5f * (val(3, 0) + val(3, 1));
  float conductivity = 0.5f * (S.cond(n) + S.cond(n1));
  if constexpr (C::turb) conductivity += 0.5f * (S.tcond(n) + S.tcond(n1));
  fv[4] = um * fv[1] + vm * fv[2] + wm * fv[3] + conductivity * (kx * t_x + ky * t_y + kz * t_z);
  if constexpr (C::mix != 0) {
    float turb_d = 0;
    if constexpr (C::turb) turb_d = mut / cF.Sct;
    const float tm = 0.5f * (val(5, 0) + val(5, 1));
    float rho_uc = 0, rho_vc = 0, rho_wc = 0, hflux = 0;
    OSTC_UNROLL for (int l = 0; l < NS; ++l) {
      const float dif = 0.5f * (S.rho_d(l, n) + S.rho_d(l, n1)) + turb_d;
      float yx, yy, yz, h, cp_unused;
      grad(6 + l, g0, g1, g2);
      cart(g0, g1, g2, yx, yy, yz);
      thermo_one(l, tm, h, cp_unused);
      // the diffusive flux of species l through the face, before the correction
      fv[5 + l] = dif * (kx * yx + ky * yy + kz * yz);
      hflux += h * fv[5 + l];
      rho_uc += dif * yx;
      rho_vc += dif * yy;
      rho_wc += dif * yz;
    }
    fv[4] += hflux;
    const float corr = kx * rho_uc + ky * rho_vc + kz * rho_wc;
    OSTC_UNROLL for (int l = 0; l < NS; ++l) fv[5 + l] -= 0.5f * (val(6 + l, 0) + val(6 + l, 1)) * corr;
  }
  if constexpr (C::turb) {
    float k_x, k_y, k_z, o_x, o_y, o_z;
    grad(6 + NS, g0, g1, g2);
    cart(g0, g1, g2, k_x, k_y, k_z);
    grad(7 + NS, g0, g1, g2);
    cart(g0, g1, g2, o_x, o_y, o_z);
    const float wall_dist = 0.5f * (S.wall(n) + S.wall(n1));
    float f1 = 1;
    if (wall_dist > 1e-25f) {
      const float km = 0.5f * (val(6 + NS, 0) + val(6 + NS, 1));
      const float omegam = 0.5f * (val(7 + NS, 0) + val(7 + NS, 1));
      const float param1 = sqrtf(km) / (0.09f * omegam * wall_dist);
      const float rhom = 0.5f * (val(0, 0) + val(0, 1));
      const float d2 = wall_dist * wall_dist;
      const float param2 = 500 * mul / (rhom * d2 * omegam);
      constexpr float so2 = static_cast<float>(sst::sigma_omega2);
      const float CDkomega = fmaxf(1e-20f, 2 * rhom * so2 / omegam * (k_x * o_x + k_y * o_y + k_z * o_z));
      const float param3 = 4 * rhom * so2 * km / (CDkomega * d2);
      const float arg1 = fminf(fmaxf(param1, param2), param3);
      f1 = tanh_pos(arg1 * arg1 * arg1 * arg1);
    }
    const float sigma_k = static_cast<float>(sst::sigma_k2) + static_cast<float>(sst::delta_sigma_k) * f1;
    const float sigma_omega =
        static_cast<float>(sst::sigma_omega2) + static_cast<float>(sst::delta_sigma_omega) * f1;
    fv[5 + NS] = (mul + mut * sigma_k) * (kx * k_x + ky * k_y + kz * k_z);
    fv[6 + NS] = (mul + mut * sigma_omega) * (kx * o_x + ky * o_y + kz * o_z);
  }
}

template <class C, class Src>
__device__ __forceinline__ void viscous_face_s(const Src &S, int64_t sx, int64_t sxy, int64_t n, int d, int64_t s,
                                               float *fv) {
  const int64_t n1 = n + s;
  viscous_face_r<C>(
      S, n, d, s, [&](int v, int side) { return S.prim(v, side ? n1 : n); },
      [&](int v, float &g0, float &g1, float &g2) {
        face_grad([&](int64_t q) { return S.prim(v, q); }, n, n1, d, sx, sxy, g0, g1, g2);
      },
      fv);
}

template <class C>
__device__ __forceinline__ void viscous_face(const DevBlock &B, int64_t n, int d, int64_t s, float *fv) {
  viscous_face_s<C>(Src64{B}, B.G.sx, B.G.sxy, n, d, s, fv);
}

// ------------------------------------------------------------- SST source
template <class C>
__device__ __forceinline__ void sst_source(const DevBlock &B, int64_t n, double &src_k, double &src_w,
                                           double &mut_out, double &jk, double &jw) {
  constexpr int NS = C::ns;
  const int64_t sz = B.G.size, sx = B.G.sx, sxy = B.G.sxy;
  const double *m = B.metric;
  const float xi_x = ldf(m + n), xi_y = ldf(m + sz + n), xi_z = ldf(m + 2 * sz + n);
  const float eta_x = ldf(m + 3 * sz + n), eta_y = ldf(m + 4 * sz + n), eta_z = ldf(m + 5 * sz + n);
  const float zeta_x = ldf(m + 6 * sz + n), zeta_y = ldf(m + 7 * sz + n), zeta_z = ldf(m + 8 * sz + n);
  auto cgrad = [&](const double *a, float &gx, float &gy, float &gz) {
    const float a_xi = ldf(a + n + 1) - ldf(a + n - 1), a_eta = ldf(a + n + sx) - ldf(a + n - sx),
                a_zeta = ldf(a + n + sxy) - ldf(a + n - sxy);
    gx = 0.5f * (xi_x * a_xi + eta_x * a_eta + zeta_x * a_zeta);
    gy = 0.5f * (xi_y * a_xi + eta_y * a_eta + zeta_y * a_zeta);
    gz = 0.5f * (xi_z * a_xi + eta_z * a_eta + zeta_z * a_zeta);
  };
  float u_x, u_y, u_z, v_x, v_y, v_z, w_x, w_y, w_z, k_x, k_y, k_z, o_x, o_y, o_z;
  cgrad(B.bv + sz, u_x, u_y, u_z);
  cgrad(B.bv + 2 * sz, v_x, v_y, v_z);
  cgrad(B.bv + 3 * sz, w_x, w_y, w_z);
  const double *tk = B.sv + NS * sz, *tw = B.sv + (NS + 1) * sz;
  cgrad(tk, k_x, k_y, k_z);
  cgrad(tw, o_x, o_y, o_z);
  const float density = ldf(B.bv + n), omega = ldf(tw + n), tke = ldf(tk + n);
  constexpr float so2 = static_cast<float>(sst::sigma_omega2), a1 = static_cast<float>(sst::a_1);
  const float inter_var = 2 * density * so2 / omega * (k_x * o_x + k_y * o_y + k_z * o_z);
  const float rhoK = density * tke;
  const float vorticity =
      sqrtf((v_x - u_y) * (v_x - u_y) + (w_x - u_z) * (w_x - u_z) + (w_y - v_z) * (w_y - v_z));
  float f1 = 1, f2 = 1;
  const float dy = ldf(B.wall_dist + n);
  if (dy > 1e-25f) {
    const float param1 = sqrtf(tke) / (0.09f * omega * dy);
    const float d2 = dy * dy;
    const float param2 = 500 * ldf(B.mul + n) / (density * d2 * omega);
    const float arg2 = fmaxf(2 * param1, param2);
    f2 = tanh_pos(arg2 * arg2);
    const float CDkomega = fmaxf(1e-20f, inter_var);
    const float param3 = 4 * density * so2 * tke / (CDkomega * d2);
    const float arg1 = fminf(fmaxf(param1, param2), param3);
    f1 = tanh_pos(arg1 * arg1 * arg1 * arg1);
  }
  float mut = 0;
  if (const float den = fmaxf(a1 * omega, vorticity * f2); den > 1e-25f) mut = a1 * rhoK / den;
  mut_out = mut;
  const float beta = static_cast<float>(sst::beta_2) + static_cast<float>(sst::delta_beta) * f1;
  src_k = 0;
  src_w = 0;
  if (mut > 1e-25f) {
    const float divU = u_x + v_y + w_z;
    const float prod_k = mut * (2 * (u_x * u_x + v_y * v_y + w_z * w_z) - (2.f / 3.f) * divU * divU +
                                (u_y + v_x) * (u_y + v_x) + (u_z + w_x) * (u_z + w_x) + (v_z + w_y) * (v_z + w_y)) -
                         (2.f / 3.f) * rhoK * divU;
    const float diss_k = static_cast<float>(sst::beta_star) * rhoK * omega;
    const float jac = ldf(B.jac + n);
    src_k = jac * (prod_k - diss_k);
    const float gamma = static_cast<float>(sst::gamma2) + static_cast<float>(sst::delta_gamma) * f1;
    const float prod_omega = gamma * density / mut * prod_k + (1 - f1) * inter_var;
    const float diss_omega = beta * density * omega * omega;
    src_w = jac * (prod_omega - diss_omega);
  }
  jk = -2 * sst::beta_star * omega;
  jw = -2.0 * beta * omega;
}

}  // namespace fp32

// Finite-rate chemistry of one cell in FP64 (the FP64 path's code with each
// Arrhenius rate as one exponential):
// returns dq species = J omega and writes the EPI / DA Jacobian.  q1, q2:
// this thread's column of the CTA's shared rate arrays (stride kCta).
template <class C>
__device__ __forceinline__ void chem_cell(const DevBlock &B, int64_t n, int64_t nz, double *q1, double *q2,
                                          double *dq_spec) {
  constexpr int NS = C::ns;
  const int64_t sz = B.G.size, sz0 = B.Z.size;
  double Y[NS], omega[NS], omega_d[NS];
  OSTC_UNROLL for (int l = 0; l < NS; ++l) Y[l] = ld(B.sv + l * sz + n);
  const double density = ld(B.bv + n), t = ld(B.bv + 5 * sz + n);
  chemistry<NS, true>(density, t, Y, omega, omega_d, q1, q2, kCta);
  const double jac = ld(B.jac + n);
  OSTC_UNROLL for (int l = 0; l < NS; ++l) dq_spec[l] = jac * omega[l];
  const int method = cP.chem_src_method;
  if (method == 1) {
    // compute_chem_src_jacobian with the reaction loop outside the species
    // loop: each row m visits only the reactions that change species m once,
    // and every (m, q) entry still sums its terms in reaction order
    const int nr = cP.nr, na = cP.na;
    // 1 / (rho Y_q) once per species (0 below the floor): products, not
    // NS^2 divisions, within an ulp of the FP64 path's quotients
    double inv_rho_y[NS];
    OSTC_UNROLL for (int q = 0; q < NS; ++q) inv_rho_y[q] = Y[q] > 1e-25 ? 1.0 / (density * Y[q]) : 0.0;
    // only the leading na x na block (the other rows and columns are zero)
    OSTC_UNROLL for (int m = 0; m < NS; ++m) {
      if (m >= na) break;
      double zz[NS];
      OSTC_UNROLL for (int q = 0; q < NS; ++q) zz[q] = 0;
      for (int r = 0; r < nr; ++r) {
        const int dn = cP.sb[r * NS + m] - cP.sf[r * NS + m];
        if (dn == 0) continue;
        const double a1 = q1[r * kCta], a2 = q2[r * kCta];
        OSTC_UNROLL for (int q = 0; q < NS; ++q) zz[q] += dn * (cP.sf[r * NS + q] * a1 - cP.sb[r * NS + q] * a2);
      }
      OSTC_UNROLL for (int q = 0; q < NS; ++q) {
        if (q >= na) break;
        const double v = zz[q] * inv_rho_y[q];
        B.chem_jac[(m * na + q) * sz0 + nz] = cP.mw[m] * v * 1e+3;
      }
    }
  } else if (method == 2) {
    OSTC_UNROLL for (int l = 0; l < NS; ++l) {
      double v = 0;
      if (Y[l] > 1e-25) v = -omega_d[l] / (Y[l] * density);
      B.chem_jac[l * sz0 + nz] = v;
    }
  }
}

// dq = source terms: SST in FP32, finite-rate chemistry and its EPI Jacobian
// in FP64 (the same code as the FP64 path).  With the surrogate on
// (chem_quiet set) the chemistry of the cells it did not judge quiet runs in
// k_chem_list over a compacted list instead, with every lane of a warp busy;
// here those cells get zero species source, which k_chem_list overwrites.
template <class C>
__global__ void __launch_bounds__(kCta, 4) k_source_mx(const DevBlock *__restrict__ blks, Tiles T) {
  constexpr int NS = C::ns, NV = C::nv;
  extern __shared__ double sq[];
  int b, i, j, k;
  if (!tile_cell<kTX, kTY, kTZ>(T, b, i, j, k, blks)) return;
  const DevBlock &B = blks[b];
  const int64_t n = B.G.at(i, j, k), nd = B.D.at(i, j, k), nz = B.Z.at(i, j, k);
  const int64_t szd = B.D.size, sz0 = B.Z.size;
  double dq[NV];
  OSTC_UNROLL for (int l = 0; l < NV; ++l) dq[l] = 0;
  if constexpr (C::turb) {
    double sk, sw, mut, jk, jw;
    fp32::sst_source<C>(B, n, sk, sw, mut, jk, jw);
    B.mut[n] = mut;
    dq[NS + 5] = sk;
    dq[NS + 6] = sw;
    if (cP.turb_implicit == 1) {
      B.turb_src_jac[nz] = jk;
      B.turb_src_jac[sz0 + nz] = jw;
    }
    B.turb_cond[n] = static_cast<float>(mut) * fp32::ldf(B.cp + n) / cF.Prt;
  }
  if constexpr (C::mix == 2) {
    if (B.chem_quiet) {
      if (B.chem_quiet[nz]) {
        // judged chemically quiet by the surrogate: its rate and no Jacobian
        // (the implicit stages treat the cell's species diagonally and never
        // read its chem_jac)
        const double jac = ld(B.jac + n);
        OSTC_UNROLL for (int l = 0; l < NS; ++l) dq[l + 5] = jac * B.chem_rate[l * sz0 + nz];
      }
    } else {
      const int tid = threadIdx.x + kTX * (threadIdx.y + kTY * threadIdx.z);
      chem_cell<C>(B, n, nz, sq + tid, sq + cP.nr * kCta + tid, dq + 5);
    }
  }
  OSTC_UNROLL for (int l = 0; l < NV; ++l) B.dq[l * szd + nd] = dq[l];
}

// The cells of block b the surrogate did not judge quiet, listed (any order).
template <class C>
__global__ void __launch_bounds__(256) k_chem_compact(const DevBlock *__restrict__ blks, int b, int *list,
                                                      int *count) {
  const DevBlock &B = blks[b];
  const int64_t cells = static_cast<int64_t>(B.mx) * B.my * B.mz;
  const int lane = threadIdx.x & 31;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t base = static_cast<int64_t>(blockIdx.x) * blockDim.x; base < cells; base += stride) {
    const int64_t c = base + threadIdx.x;
    bool pick = false;
    if (c < cells) {
      const int i = static_cast<int>(c % B.mx), j = static_cast<int>((c / B.mx) % B.my),
                k = static_cast<int>(c / (static_cast<int64_t>(B.mx) * B.my));
      pick = B.chem_quiet[B.Z.at(i, j, k)] == 0;
    }
    const unsigned m = __ballot_sync(0xffffffffu, pick);
    int at = 0;
    if (lane == 0 && m) at = atomicAdd(count, __popc(m));
    at = __shfl_sync(0xffffffffu, at, 0);
    if (pick) list[at + __popc(m & ((1u << lane) - 1u))] = static_cast<int>(c);
  }
}

// Chemistry of the listed cells (k_chem_compact), one thread per entry, full
// warps; launched for the block's cell count, entries past the list return.
template <class C>
__global__ void __launch_bounds__(kCta, 4) k_chem_list(const DevBlock *__restrict__ blks, int b,
                                                       const int *__restrict__ list, const int *count) {
  constexpr int NS = C::ns;
  extern __shared__ double sq[];
  const int q = blockIdx.x * kCta + threadIdx.x;
  if (q >= *count) return;
  const DevBlock &B = blks[b];
  const int64_t c = list[q];
  const int i = static_cast<int>(c % B.mx), j = static_cast<int>((c / B.mx) % B.my),
            k = static_cast<int>(c / (static_cast<int64_t>(B.mx) * B.my));
  const int64_t n = B.G.at(i, j, k), nz = B.Z.at(i, j, k), nd = B.D.at(i, j, k), szd = B.D.size;
  double dqs[NS];
  chem_cell<C>(B, n, nz, sq + threadIdx.x, sq + cP.nr * kCta + threadIdx.x, dqs);
  OSTC_UNROLL for (int l = 0; l < NS; ++l) B.dq[(5 + l) * szd + nd] = dqs[l];
}

// Local time step of cell (i, j, k) in FP32 (local_time_step,
// src/TimeAdvanceFunc.cuh:21-71); also stores the spectral radii the DPLUR
// sweeps use.
template <class C, class Src>
__device__ __forceinline__ void local_time_step_s(const DevBlock &B, const Src &S, int i, int j, int k, int64_t n,
                                                  int64_t nd) {
  const int64_t szd = B.D.size;
  const bool three_d = B.mz > 1;
  const float m11 = S.metric(0, n), m12 = S.metric(1, n), m13 = S.metric(2, n);
  const float m21 = S.metric(3, n), m22 = S.metric(4, n), m23 = S.metric(5, n);
  const float m31 = S.metric(6, n), m32 = S.metric(7, n), m33 = S.metric(8, n);
  const float grad_xi = sqrtf(m11 * m11 + m12 * m12 + m13 * m13);
  const float grad_eta = sqrtf(m21 * m21 + m22 * m22 + m23 * m23);
  const float grad_zeta = sqrtf(m31 * m31 + m32 * m32 + m33 * m33);
  const float u = S.prim(1, n), v = S.prim(2, n), w = S.prim(3, n);
  const float a = S.acoustic(n);
  const float s0 = fabsf(u * m11 + v * m12 + w * m13) + a * grad_xi;
  const float s1 = fabsf(u * m21 + v * m22 + w * m23) + a * grad_eta;
  const float s2 = three_d ? fabsf(u * m31 + v * m32 + w * m33) + a * grad_zeta : 0.f;
  B.inv_spec[nd] = s0;
  B.inv_spec[szd + nd] = s1;
  B.inv_spec[2 * szd + nd] = s2;
  if (B.inv_spec32) {
    B.inv_spec32[nd] = s0;
    B.inv_spec32[szd + nd] = s1;
    B.inv_spec32[2 * szd + nd] = s2;
  }
  float gamma = 1.4f;
  if constexpr (C::mix != 0) gamma = S.gamma(n);
  const float coeff_1 = fmaxf(gamma, 4.f / 3.f) / S.prim(0, n);
  float coeff_2 = S.mul(n) / cF.Pr;
  if constexpr (C::turb) coeff_2 += S.mut(n) / cF.Prt;
  float srv = grad_xi * grad_xi + grad_eta * grad_eta;
  if (three_d) srv += grad_zeta * grad_zeta;
  srv *= coeff_1 * coeff_2;
  B.visc_spec[nd] = srv;
  B.dt_local[B.Z.at(i, j, k)] = cF.cfl / (s0 + s1 + s2 + srv);
}

// ----------------------------------------------------- direction passes
// The flux differences as three passes, one per direction d: every face
// along d is evaluated once, inviscid and viscous together, as
// G = F_viscous - F_inviscid, and each cell adds G(c + 1/2) - G(c - 1/2) to
// its FP64 dq.  A pass keeps one face's fluxes in registers and needs no
// shared memory or barrier, so its warps run independently and the SM keeps
// as many loads in flight as its register file allows; the price is dq read
// and written once per direction instead of once.  The x pass also stores
// the local time step.
//   x: a warp holds 32 consecutive faces of one row (i - 1/2 + lane) and
//      gives 31 cells their difference, the left face coming from the lane
//      below by a shuffle; a CTA covers 4 rows (j).
//   y, z: each thread marches kMarch cells along d, carrying the lower face
//      from one cell to the next; lanes run along i, the CTA's 4 warps over
//      the remaining index (k for y, j for z).
constexpr int kXSeg = 31;  // cells per warp of the x pass
// The variants of the passes an autotuner chooses from: resident CTAs per
// SM the register allocator is asked to allow (8 caps a thread at 64
// registers, ~400 B of spills) and the cells a thread of the y / z pass
// marches over.  Measured at 384x192x64 with a march of 8, the three passes
// take 5.7 ms at 4 CTAs per SM, 5.0 at 6, 4.8 at 7, 4.4 at 8.  Every variant
// computes the same values.
struct FluxVariant {
  int min_blocks, march;
};
constexpr int kFluxVariants = 4;
constexpr FluxVariant kFluxVariant[kFluxVariants] = {{8, 8}, {8, 16}, {6, 8}, {4, 8}};

// Tiles of pass d over every block: (x) i-segments x row groups x k,
// (y) i-groups x k-groups x j-segments, (z) i-groups x j-groups x k-segments
// of kMarch cells.
inline void dir_tile_counts(int d, int kMarch, int mx, int my, int mz, int &n0, int &n1, int &n2) {
  if (d == 0) {
    n0 = (mx + kXSeg - 1) / kXSeg;
    n1 = (my + kTY - 1) / kTY;
    n2 = mz;
  } else if (d == 1) {
    n0 = (mx + kTX - 1) / kTX;
    n1 = (mz + kTY - 1) / kTY;
    n2 = (my + kMarch - 1) / kMarch;
  } else {
    n0 = (mx + kTX - 1) / kTX;
    n1 = (my + kTY - 1) / kTY;
    n2 = (mz + kMarch - 1) / kMarch;
  }
}

__device__ __forceinline__ void dir_tile(const Tiles &T, int &b, int &t0, int &t1, int &t2) {
  int t = tile_of(T, blockIdx.x, b);
  t0 = t % T.ntx[b];
  t /= T.ntx[b];
  t1 = t % T.nty[b];
  t2 = t / T.nty[b];
}

// G = F_viscous - F_inviscid at the face between linear index nl and nl + s,
// from the FP32 copy of the operands
template <class C>
__device__ __forceinline__ void face_g(const DevBlock &B, int64_t nl, int d, int64_t s, float *g) {
  constexpr int NV = C::nv;
  const fp32::Src32<C> S{B.f32, B.G.size};
  fp32::inviscid_face_s<C>(S, nl, d, s, g);
  OSTC_UNROLL for (int l = 0; l < NV; ++l) g[l] = -g[l];
  if (cP.viscous_order != 0) {
    float t[NV];
    fp32::viscous_face_s<C>(S, B.G.sx, B.G.sxy, nl, d, s, t);
    OSTC_UNROLL for (int l = 0; l < NV; ++l) g[l] += t[l];
  }
}

// The FP32 copy of the operands of the direction passes, over every point of
// layout G: the fields that change every step (after the source stage, which
// writes mu_t and lambda_t) ...
template <class C>
__global__ void __launch_bounds__(256) k_pack32(const DevBlock *__restrict__ blks, int b) {
  using L = fp32::F32<C>;
  const DevBlock &B = blks[b];
  const int64_t sz = B.G.size;
  float *f = B.f32;
  for (int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; n < sz;
       n += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    // all loads, then all stores (a store would otherwise hold back the
    // loads after it: the compiler cannot rule out that they overlap)
    float v[L::n_dynamic];
    OSTC_UNROLL for (int q = 0; q < L::n_dynamic; ++q) v[q] = 0.f;
    OSTC_UNROLL for (int q = 0; q < 6; ++q) v[L::prim + q] = static_cast<float>(__ldg(B.bv + q * sz + n));
    OSTC_UNROLL for (int q = 0; q < C::nsc; ++q) v[L::prim + 6 + q] = static_cast<float>(__ldg(B.sv + q * sz + n));
    v[L::mul] = static_cast<float>(__ldg(B.mul + n));
    v[L::cond] = static_cast<float>(__ldg(B.cond + n));
    if constexpr (C::turb) {
      v[L::mut] = static_cast<float>(__ldg(B.mut + n));
      v[L::tcond] = static_cast<float>(__ldg(B.turb_cond + n));
    }
    OSTC_UNROLL for (int l = 0; l < C::ns; ++l) v[L::rho_d + l] = static_cast<float>(__ldg(B.rho_d + l * sz + n));
    v[L::acoustic] = static_cast<float>(__ldg(B.acoustic + n));
    if constexpr (C::mix != 0) v[L::gamma] = static_cast<float>(__ldg(B.gamma + n));
    OSTC_UNROLL for (int q = 0; q < L::n_dynamic; ++q) {
      if (q == L::mut || q == L::tcond) {
        if constexpr (!C::turb) continue;
      }
      if (q == L::gamma && C::mix == 0) continue;
      f[q * sz + n] = v[q];
    }
  }
}

// ... and the geometry, which changes only when the grid is set.
template <class C>
__global__ void __launch_bounds__(256) k_pack32_static(const DevBlock *__restrict__ blks, int b) {
  using L = fp32::F32<C>;
  const DevBlock &B = blks[b];
  const int64_t sz = B.G.size;
  float *f = B.f32;
  for (int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; n < sz;
       n += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    f[L::wall * sz + n] = B.wall_dist ? static_cast<float>(B.wall_dist[n]) : 0.f;
    f[L::jac * sz + n] = static_cast<float>(B.jac[n]);
    OSTC_UNROLL for (int q = 0; q < 9; ++q) f[(L::metric + q) * sz + n] = static_cast<float>(B.metric[q * sz + n]);
  }
}

template <class C, int MINB>
__global__ void __launch_bounds__(kCta, MINB) k_flux_x(const DevBlock *__restrict__ blks, Tiles T) {
  constexpr int NV = C::nv;
  int b, t0, t1, t2;
  dir_tile(T, b, t0, t1, t2);
  const DevBlock &B = blks[b];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = t1 * kTY + warp, k = t2;
  if (j >= B.my) return;  // the whole warp
  const int f = t0 * kXSeg - 1 + lane;  // the face between cells f and f + 1
  const bool face = f < B.mx;
  float g[NV];
  if (face) {
    face_g<C>(B, B.G.at(f, j, k), 0, 1, g);
  } else {
    OSTC_UNROLL for (int l = 0; l < NV; ++l) g[l] = 0;
  }
  const bool cell = face && lane > 0;
  const int64_t szd = B.D.size;
  const int64_t nd = cell ? B.D.at(f, j, k) : 0;
  OSTC_UNROLL for (int l = 0; l < NV; ++l) {
    const float gm = __shfl_up_sync(0xffffffffu, g[l], 1);
    if (cell) B.dq[l * szd + nd] += static_cast<double>(g[l] - gm);
  }
  if (cell) local_time_step_s<C>(B, fp32::Src32<C>{B.f32, B.G.size}, f, j, k, B.G.at(f, j, k), nd);
}

template <class C, int D, int MINB, int kMarch>
__global__ void __launch_bounds__(kCta, MINB) k_flux_march(const DevBlock *__restrict__ blks, Tiles T) {
  constexpr int NV = C::nv;
  static_assert(D == 1 || D == 2, "march passes run along y or z");
  int b, t0, t1, t2;
  dir_tile(T, b, t0, t1, t2);
  const DevBlock &B = blks[b];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = t0 * kTX + lane, o = t1 * kTY + warp;  // o: k for the y pass, j for the z pass
  if (i >= B.mx || o >= (D == 1 ? B.mz : B.my)) return;
  const int m = D == 1 ? B.my : B.mz;
  const int c0 = t2 * kMarch, c1 = min(c0 + kMarch, m);
  const int64_t s = D == 1 ? B.G.sx : B.G.sxy;
  const int64_t n0 = D == 1 ? B.G.at(i, c0, o) : B.G.at(i, o, c0);
  const int64_t sd = D == 1 ? B.D.sx : B.D.sxy;
  const int64_t nd0 = D == 1 ? B.D.at(i, c0, o) : B.D.at(i, o, c0);
  const int64_t szd = B.D.size;
  float gm[NV];
  face_g<C>(B, n0 - s, D, s, gm);  // face c0 - 1/2
#pragma unroll 1
  for (int c = c0; c < c1; ++c) {
    float g[NV];
    face_g<C>(B, n0 + (c - c0) * s, D, s, g);  // face c + 1/2
    const int64_t nd = nd0 + (c - c0) * sd;
    OSTC_UNROLL for (int l = 0; l < NV; ++l) {
      B.dq[l * szd + nd] += static_cast<double>(g[l] - gm[l]);
      gm[l] = g[l];
    }
  }
}

// EPI solve of a DPLUR sweep with the stored factors of the leading NA x NA
// block; the trailing species have the single pivot diag, so their solve is
// rhs / diag, the operation the full factors would do for them.
template <int NS, int NA>
__device__ __forceinline__ void epi_solve_block(const DevBlock &B, int64_t nz, int64_t sz0, double diag,
                                                double *rhs) {
  int piv[NA];
  OSTC_UNROLL for (int q = 0; q < NA; ++q) piv[q] = B.lu_piv[q * sz0 + nz];
  lu_solve_g<NA>(B.chem_jac + nz, sz0, piv, rhs);
  OSTC_UNROLL for (int l = NA; l < NS; ++l) rhs[l] /= diag;
}

// DPLUR sweep with FP32 flux-Jacobian products; the update of the point
// implicit blocks (EPI: stored LU factors) in FP64.  The increments are FP32
// arrays: reads dqf[in_sel] (neighbours) and dqf[0] (dq0), writes
// dqf[out_sel], or the FP64 dq when out_sel < 0 (the last sweep).
template <class C>
__global__ void __launch_bounds__(kCta, 4) k_sweep_mx(const DevBlock *__restrict__ blks, Tiles T, int in_sel,
                                                      int out_sel) {
  constexpr int NS = C::ns, NV = C::nv;
  using fp32::ldf;
  int b, i, j, k;
  if (!tile_cell<kTX, kTY, kTZ>(T, b, i, j, k, blks)) return;
  const DevBlock &B = blks[b];
  const float *dqin = B.dqf[in_sel];
  const float *dq0 = B.dqf[0];
  const int64_t sz = B.G.size, szd = B.D.size, sz0 = B.Z.size;
  const int64_t n = B.G.at(i, j, k), nd = B.D.at(i, j, k), nz = B.Z.at(i, j, k);
  const int64_t sx = B.G.sx, sxy = B.G.sxy, dsx = B.D.sx, dsxy = B.D.sxy;
  const fp32::Src32<C> f{B.f32, sz};
  float tot[NV];
  OSTC_UNROLL for (int l = 0; l < NV; ++l) tot[l] = 0;
  const float *isr = B.inv_spec32;  // FP32 values, as k_flux_x computed them
#pragma unroll 1
  for (int q = 0; q < 6; ++q) {
    const int dir = q < 3 ? q : q - 3;
    const bool plus = q >= 3;
    const int id = dir == 0 ? i : (dir == 1 ? j : k);
    const int ext = dir == 0 ? B.mx : (dir == 1 ? B.my : B.mz);
    if (plus ? id == ext - 1 : id == 0) continue;
    const int64_t gs = dir == 0 ? 1 : (dir == 1 ? sx : sxy), ds = dir == 0 ? 1 : (dir == 1 ? dsx : dsxy);
    const int64_t on = plus ? n + gs : n - gs, od = plus ? nd + ds : nd - ds;
    const float sr = __ldg(isr + dir * szd + od);
    // compute_jacobian_times_dq (src/DPLURHPP.cuh:78-125) at the neighbour,
    // its state from the step's FP32 copy (k_pack32; unchanged until the update)
    const float xi_x = f.metric(3 * dir, on), xi_y = f.metric(3 * dir + 1, on), xi_z = f.metric(3 * dir + 2, on);
    const float u = f.prim(1, on), v = f.prim(2, on), w = f.prim(3, on);
    const float U = xi_x * u + xi_y * v + xi_z * w;
    const float lmd1 = U + (plus ? -sr : sr);
    const float e = 0.5f * (u * u + v * v + w * w);
    float d[NV];
    OSTC_UNROLL for (int l = 0; l < NV; ++l) d[l] = __ldg(dqin + l * szd + od);
    float gamma = 1.4f, b3 = 0, b4 = 0, h = 0;
    if constexpr (C::mix != 0) {
      const float t = f.prim(5, on);
      gamma = f.gamma(on);
      OSTC_UNROLL for (int l = 0; l < NS; ++l) {
        const float hk = __ldg(B.h_spec32 + l * szd + od);
        b3 += fp32::kRu * t * cF.mw_inv[l] * d[5 + l];
        b4 += hk * d[5 + l];
        h += f.prim(6 + l, on) * hk;
      }
      b3 *= gamma;
      b4 *= gamma - 1;
      h += e;
    } else {
      h = gamma / (gamma - 1) * f.prim(4, on) / f.prim(0, on) + e;
    }
    const float b1 = xi_x * d[1] + xi_y * d[2] + xi_z * d[3] - U * d[0];
    const float b2 = (gamma - 1) * (e * d[0] - u * d[1] - v * d[2] - w * d[3] + d[4]);
    const float b34 = b3 - b4;
    const float sg = plus ? -0.5f : 0.5f;
    tot[0] += sg * (b1 + lmd1 * d[0]);
    tot[1] += sg * (u * b1 + xi_x * b2 + lmd1 * d[1] + xi_x * b34);
    tot[2] += sg * (v * b1 + xi_y * b2 + lmd1 * d[2] + xi_y * b34);
    tot[3] += sg * (w * b1 + xi_z * b2 + lmd1 * d[3] + xi_z * b34);
    tot[4] += sg * (h * b1 + U * b2 + lmd1 * d[4] + U * b34);
    OSTC_UNROLL for (int l = 0; l < C::nsc; ++l) tot[5 + l] += sg * (lmd1 * d[5 + l] + f.prim(6 + l, on) * b1);
  }
  const double dt = B.dt_local[nz];
  const double diag = 1 + dt * (static_cast<double>(isr[nd]) + static_cast<double>(isr[szd + nd]) +
                                static_cast<double>(isr[2 * szd + nd]));
  double out[NV];
  if constexpr (C::mix != 2) {
    OSTC_UNROLL for (int l = 0; l < 5 + NS; ++l) out[l] = static_cast<double>(dq0[l * szd + nd]) + dt * tot[l] / diag;
  } else {
    OSTC_UNROLL for (int l = 0; l < 5; ++l) out[l] = static_cast<double>(dq0[l * szd + nd]) + dt * tot[l] / diag;
    const int method = cP.chem_src_method;
    if (B.chem_quiet && B.chem_quiet[nz]) {
      // chemically quiet: the stored factors would be diag I
      OSTC_UNROLL for (int l = 0; l < NS; ++l) out[5 + l] = static_cast<double>(dq0[(5 + l) * szd + nd]) + dt * tot[5 + l] / diag;
    } else if (method == 1) {
      double rhs[NS];
      OSTC_UNROLL for (int l = 0; l < NS; ++l) rhs[l] = static_cast<double>(tot[5 + l]) * dt;
      if (cP.na == NS - 1)
        epi_solve_block<NS, NS - 1>(B, nz, sz0, diag, rhs);
      else
        epi_solve_block<NS, NS>(B, nz, sz0, diag, rhs);
      OSTC_UNROLL for (int l = 0; l < NS; ++l) out[5 + l] = static_cast<double>(dq0[(5 + l) * szd + nd]) + rhs[l];
    } else if (method == 2) {
      OSTC_UNROLL for (int l = 0; l < NS; ++l)
        out[5 + l] = static_cast<double>(dq0[(5 + l) * szd + nd]) + dt * tot[5 + l] / (diag - dt * B.chem_jac[l * sz0 + nz]);
    } else {
      OSTC_UNROLL for (int l = 0; l < NS; ++l) out[5 + l] = static_cast<double>(dq0[(5 + l) * szd + nd]) + dt * tot[5 + l] / diag;
    }
  }
  if constexpr (C::turb) {
    if (cP.turb_implicit == 1) {
      out[NS + 5] = static_cast<double>(dq0[(NS + 5) * szd + nd]) + dt * tot[5 + NS] / (diag - dt * B.turb_src_jac[nz]);
      out[NS + 6] = static_cast<double>(dq0[(NS + 6) * szd + nd]) + dt * tot[6 + NS] / (diag - dt * B.turb_src_jac[sz0 + nz]);
    } else {
      out[NS + 5] = static_cast<double>(dq0[(NS + 5) * szd + nd]) + dt * tot[5 + NS] / diag;
      out[NS + 6] = static_cast<double>(dq0[(NS + 6) * szd + nd]) + dt * tot[6 + NS] / diag;
    }
  }
  if (out_sel < 0) {
    OSTC_UNROLL for (int l = 0; l < NV; ++l) B.dq[l * szd + nd] = out[l];
  } else {
    float *dqout = B.dqf[out_sel];
    OSTC_UNROLL for (int l = 0; l < NV; ++l) dqout[l * szd + nd] = static_cast<float>(out[l]);
  }
}

// Thermodynamic and transport properties in FP32 (update_physical_properties).
template <class C>
__global__ void __launch_bounds__(kCta) k_props_mx(const DevBlock *__restrict__ blks, Tiles T) {
  constexpr int NS = C::ns;
  using fp32::ldf;
  int b, i, j, k;
  if (!tile_cell<kTX, kTY, kTZ>(T, b, i, j, k, blks)) return;
  const DevBlock &B = blks[b];
  const int64_t n = B.G.at(i, j, k), sz = B.G.size;
  const float t = ldf(B.bv + 5 * sz + n);
  if constexpr (C::mix != 0) {
    float cp[NS], Y[NS];
    const float vel = ldf(B.vel + n);  // read before the first store, which would hold it back
    fp32::thermo<NS, false, true>(t, nullptr, cp);
    float mw_inv = 0, cp_tot = 0, cv = 0;
    OSTC_UNROLL for (int l = 0; l < NS; ++l) {
      Y[l] = ldf(B.sv + l * sz + n);
      mw_inv += Y[l] * cF.mw_inv[l];
      cp_tot += Y[l] * cp[l];
      cv += Y[l] * (cp[l] - cF.ru_mw[l]);
    }
    const float gamma = __fdividef(cp_tot, cv);
    B.cp[n] = cp_tot;
    B.gamma[n] = gamma;
    const float a = sqrtf(gamma * fp32::kRu * t * mw_inv);
    B.acoustic[n] = a;
    const float mw = 1.f / mw_inv;
    float X[NS], vis[NS], rs[NS], sq[NS];  // sq = sqrt(mu_k), rs = 1 / sq
    const float st = sqrtf(t);
    OSTC_UNROLL for (int l = 0; l < NS; ++l) {
      X[l] = Y[l] * mw * cF.mw_inv[l];
      const float t_dl = t * cF.lj_inv[l];
      // the hardware-approximate power and quotients (errors of a few ulp)
      const float r = __fdividef(1.f, t_dl + 0.5f);
      const float ci = 1.147f * __powf(t_dl, -0.145f) + r * r;
      vis[l] = __fdividef(cF.vis_coeff[l] * st, ci);
      rs[l] = rsqrtf(vis[l]);
      sq[l] = vis[l] * rs[l];
    }
    float viscosity = 0, conductivity = 0;
    OSTC_UNROLL for (int m = 0; m < NS; ++m) {
      float vt = 0;
      OSTC_UNROLL for (int q = 0; q < NS; ++q) {
        float phi = 1.f;
        if (m != q) {  // Wilke's phi_mq with sqrt(mu_m / mu_q) as sqrt(mu_m) / sqrt(mu_q)
          const float num = 1 + sq[m] * rs[q] * cF.wq[m * NS + q];
          phi = num * num * cF.w8[m * NS + q];
        }
        vt += phi * X[q];
      }
      viscosity += __fdividef(vis[m] * X[m], vt);
      const float lambda = vis[m] * (cp[m] + 1.25f * cF.ru_mw[m]);
      conductivity += __fdividef(lambda * X[m], 1.065f * vt - 0.065f * X[m]);
    }
    B.mul[n] = viscosity;
    B.cond[n] = conductivity;
    OSTC_UNROLL for (int l = 0; l < NS; ++l) {
      const float dd = fabsf(X[l] - 1) < 1e-3f ? viscosity / cF.Sc : (1 - Y[l]) * viscosity / ((1 - X[l]) * cF.Sc);
      B.rho_d[l * sz + n] = dd;
    }
    B.mach[n] = vel / a;
  } else {
    const float a = sqrtf(1.4f * fp32::kRu / static_cast<float>(kDMwAir) * t);
    B.acoustic[n] = a;
    const float mul = 1.716e-5f * powf(t / 273.f, 1.5f) * (273.f + 111.f) / (t + 111.f);
    B.mul[n] = mul;
    B.cond[n] = mul * static_cast<float>(kDGammaAir * kDR_u / kDMwAir / (kDGammaAir - 1)) / cF.Pr;
    B.mach[n] = ldf(B.vel + n) / a;
  }
}

}  // namespace ostc
