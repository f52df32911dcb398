// Device-side data layout and parameters of the sm_100a engine.
//
// State arrays keep the reference's column-major layout with ghost layers
// (src/gxl_lib/Array.hpp:71-130) so that the C ABI can copy the host fields
// of the reference unchanged; the metric is stored as nine arrays instead of
// a 3x3 struct per point, and the inviscid spectral radius as three arrays.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define OSTC_HD __host__ __device__
#else
#define OSTC_HD
#endif

namespace ostc {

constexpr int kMaxSpec = 20;
constexpr int kMaxReac = 50;
constexpr int kMaxBlocks = 16;

constexpr double kDR_u = 8314.462618;
constexpr double kDP_atm = 101325.0;
constexpr double kDGammaAir = 1.4;
constexpr double kDMwAir = 28.9647;

// Physics constants and mechanism tables; lives in __constant__ memory.
struct DevParams {
  int ns, nr, n_var, n_scalar;
  int mix, turb, rans_model, turb_implicit, chem_src_method, implicit_method, dplur_inner_step;
  int reconstruction, limiter, viscous_order, dim;
  double cfl, Pr, Prt, Sct, Sc;
  double ll[7], ul[7];
  double sv_inf[kMaxSpec + 2];
  double mw[kMaxSpec], t_low[kMaxSpec], t_mid[kMaxSpec];
  double ru_mw[kMaxSpec];  // R_u / W_k (the quotient the reference divides out each time)
  double low[kMaxSpec * 7], high[kMaxSpec * 7];
  double lj_inv[kMaxSpec], vis_coeff[kMaxSpec];
  double wq[kMaxSpec * kMaxSpec], w8[kMaxSpec * kMaxSpec];
  int label[kMaxReac], order[kMaxReac];
  signed char sf[kMaxReac * kMaxSpec], sb[kMaxReac * kMaxSpec];
  double A[kMaxReac], b[kMaxReac], Ea[kMaxReac], A2[kMaxReac], b2[kMaxReac], Ea2[kMaxReac];
  double lnA[kMaxReac], lnA2[kMaxReac];  // ln |A|, ln |A2| (0 where A is 0): the FP32-bulk path's rates
  // FP32-bulk path under DPLUR + EPI: ns - 1 when the last species takes
  // part in no reaction (a third body only, e.g. N2), so that its EPI row and
  // column are zero; chem_jac / lu_piv then hold only the leading na x na
  // block (entry (m, q) at m * na + q).  ns everywhere else.
  int na;
  double tb[kMaxReac * kMaxSpec];
  double troe_a[kMaxReac], troe_t3[kMaxReac], troe_t1[kMaxReac], troe_t2[kMaxReac];
};

// Strides of a 3-D array with a given number of ghost layers.
struct Lay {
  int64_t sx = 0, sxy = 0, size = 0, off = 0;
  OSTC_HD int64_t at(int i, int j, int k) const { return k * sxy + j * sx + i + off; }
  static Lay make(int mx, int my, int mz, int g) {
    Lay l;
    l.sx = mx + 2 * g;
    l.sxy = l.sx * (my + 2 * g);
    l.size = l.sxy * (mz + 2 * g);
    l.off = (l.sxy + l.sx + 1) * g;
    return l;
  }
};

// One grid block's device arrays.  G: ngg ghost layers; D: layout of the
// dq family (one ghost layer under DPLUR, none otherwise); Z: no ghosts.
struct DevBlock {
  int mx, my, mz, ngg;
  Lay G, D, Z;
  double *x, *y, *z, *jac, *metric, *wall_dist;
  double *bv, *sv, *cv, *vel, *acoustic, *mach, *mul, *cond, *rho_d, *gamma, *cp, *mut, *turb_cond;
  double *chem_jac, *turb_src_jac;
  unsigned char *lu_piv;
  double *dq, *dq0, *dqk, *inv_spec, *visc_spec, *dt_local, *bv_last;
  // species enthalpies h_k(T) of each cell, written by k_dq0 for the DPLUR
  // sweeps (layout D, ns components; mixtures under DPLUR only)
  double *h_spec;
  // FP32-bulk path under DPLUR: the species enthalpies (k_dq0, instead of
  // h_spec) and the inviscid spectral radii (the x flux pass, beside
  // inv_spec) in FP32, the precision the sweeps use them in; layout D
  float *h_spec32, *inv_spec32;
  // chemistry surrogate (layout Z; null when off): cells the surrogate judged
  // chemically quiet take its increment rate rho dY/dt as an explicit source
  unsigned char *chem_quiet;
  double *chem_rate;
  // FP32-bulk path under DPLUR: the increments in FP32 (layout D, nv
  // components each): [0] dq0, [1] and [2] the ping-pong of the sweeps; the
  // last sweep writes the FP64 dq.  Null on the FP64 path.
  float *dqf[3];
  // FP32-bulk path: an FP32 copy (layout G) of every operand of the
  // direction-pass flux kernels, component by component (fp32::F32); null on
  // the FP64 path
  float *f32;
  // with exact inner faces: bit 2 d + (1 for the high side) is set when that
  // block face is an inner face whose neighbours the DPLUR sweeps take
  int inner_mask;
};

// Work table of a launch: CTA-tiles of every block.  The blocks are laid out
// in schedule order (slot s holds block block[s], whose tiles are CTAs
// begin[s] .. begin[s + 1] - 1); ntx / nty and cbegin (the block's first
// tile in block order, which fixes the residual's reduction order whatever
// the schedule) are indexed by block.
struct Tiles {
  int nblk = 0;
  int begin[kMaxBlocks + 1] = {};
  int block[kMaxBlocks] = {};
  int cbegin[kMaxBlocks] = {};
  int ntx[kMaxBlocks] = {}, nty[kMaxBlocks] = {};
  int halo = 0;  // cells [-halo, m+halo) in every direction
};

// The block of this CTA and the CTA's tile index within the block.
OSTC_HD inline int tile_of(const Tiles &T, int cta, int &b) {
  int s = 0;
  while (s + 1 < T.nblk && cta >= T.begin[s + 1]) ++s;
  b = T.block[s];
  return cta - T.begin[s];
}

}  // namespace ostc
