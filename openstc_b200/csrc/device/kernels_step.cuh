// Kernels of one pseudo-time step, instantiated per model configuration.
#pragma once

#include "kernels.cuh"

namespace ostc {

constexpr int kTX = 32, kTY = 4, kTZ = 1;  // per-cell tile (threads)
constexpr int kCta = kTX * kTY * kTZ;

// ---------------------------------------------------------------- source
// compute_source (src/SourceTerm.cuh:11-40) fused with the reset of dq:
// writes every dq component of an interior cell (zero + source).
template <class C>
__global__ void __launch_bounds__(kCta, 4) k_source(const DevBlock *__restrict__ blks, Tiles T) {
  constexpr int NS = C::ns, NV = C::nv;
  extern __shared__ double sq[];  // q1, q2: 2 * n_reac * kCta doubles
  int b, i, j, k;
  if (!tile_cell<kTX, kTY, kTZ>(T, b, i, j, k, blks)) return;
  const DevBlock &B = blks[b];
  const int64_t n = B.G.at(i, j, k), nd = B.D.at(i, j, k), nz = B.Z.at(i, j, k);
  const int64_t sz = B.G.size, szd = B.D.size, sz0 = B.Z.size;
  double dq[NV];
  OSTC_UNROLL for (int l = 0; l < NV; ++l) dq[l] = 0;
  if constexpr (C::turb) {
    double sk, sw, mut, jk, jw;
    sst_source<C>(B, n, sk, sw, mut, jk, jw);
    B.mut[n] = mut;
    dq[NS + 5] = sk;
    dq[NS + 6] = sw;
    if (cP.turb_implicit == 1) {
      B.turb_src_jac[nz] = jk;
      B.turb_src_jac[sz0 + nz] = jw;
    }
    if constexpr (C::mix != 0) {
      B.turb_cond[n] = mut * ld(B.cp + n) / cP.Prt;
    } else {
      constexpr double cp = kDGammaAir * kDR_u / kDMwAir / (kDGammaAir - 1);
      B.turb_cond[n] = mut * cp / cP.Prt;
    }
  }
  if constexpr (C::mix == 2) {
    if (B.chem_quiet && B.chem_quiet[nz]) {
      // judged chemically quiet by the surrogate: its rate and no Jacobian
      // (the implicit stages treat the cell's species diagonally and never
      // read its chem_jac)
      const double jac = ld(B.jac + n);
      OSTC_UNROLL for (int l = 0; l < NS; ++l) dq[l + 5] = jac * B.chem_rate[l * sz0 + nz];
    } else {
    const int tid = threadIdx.x + kTX * (threadIdx.y + kTY * threadIdx.z);
    double *q1 = sq + tid, *q2 = sq + cP.nr * kCta + tid;
    double Y[NS], omega[NS], omega_d[NS];
    OSTC_UNROLL for (int l = 0; l < NS; ++l) Y[l] = ld(B.sv + l * sz + n);
    const double density = ld(B.bv + n), t = ld(B.bv + 5 * sz + n);
    chemistry<NS>(density, t, Y, omega, omega_d, q1, q2, kCta);
    const double jac = ld(B.jac + n);
    OSTC_UNROLL for (int l = 0; l < NS; ++l) dq[l + 5] = 0.0 + jac * omega[l];
    const int method = cP.chem_src_method;
    if (method == 1) {
      // compute_chem_src_jacobian, src/FiniteRateChem.cu:173-194
      // the reaction loop sits outside the species loop: each row m visits
      // only the reactions that change species m (the others add an exact
      // zero in the reference), and every (m, q) entry still sums its terms
      // in reaction order, so the entries are the reference's bit for bit
      const int nr = cP.nr;
      OSTC_UNROLL for (int m = 0; m < NS; ++m) {
        double zz[NS];
        OSTC_UNROLL for (int q = 0; q < NS; ++q) zz[q] = 0;
        for (int r = 0; r < nr; ++r) {
          const int dn = cP.sb[r * NS + m] - cP.sf[r * NS + m];
          if (dn == 0) continue;
          const double a1 = q1[r * kCta], a2 = q2[r * kCta];
          OSTC_UNROLL for (int q = 0; q < NS; ++q) zz[q] += dn * (cP.sf[r * NS + q] * a1 - cP.sb[r * NS + q] * a2);
        }
        OSTC_UNROLL for (int q = 0; q < NS; ++q) {
          const double v = Y[q] > 1e-25 ? zz[q] / (density * Y[q]) : 0.0;
          B.chem_jac[(m * NS + q) * sz0 + nz] = cP.mw[m] * v * 1e+3;
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
  }
  OSTC_UNROLL for (int l = 0; l < NV; ++l) B.dq[l * szd + nd] = dq[l];
}

// Minimum resident CTAs per SM requested from the register allocator for the
// two heaviest kernels (a tuning knob: more CTAs means fewer registers per
// thread and possibly spills).
#ifndef OSTC_FLUX_MIN_BLOCKS
#define OSTC_FLUX_MIN_BLOCKS 4
#endif
#ifndef OSTC_SWEEP_MIN_BLOCKS
#define OSTC_SWEEP_MIN_BLOCKS 4
#endif

// local_time_step, src/TimeAdvanceFunc.cuh:21-71: the spectral radii the
// DPLUR stages use and the cell's local time step.
template <class C>
__device__ __forceinline__ void local_time_step(const DevBlock &B, int i, int j, int k, int64_t n, int64_t nd) {
  const int64_t szd = B.D.size;
  const bool three_d = B.mz > 1;
  const int64_t sz = B.G.size;
  const double *m = B.metric;
  const double m11 = ld(m + n), m12 = ld(m + sz + n), m13 = ld(m + 2 * sz + n);
  const double m21 = ld(m + 3 * sz + n), m22 = ld(m + 4 * sz + n), m23 = ld(m + 5 * sz + n);
  const double m31 = ld(m + 6 * sz + n), m32 = ld(m + 7 * sz + n), m33 = ld(m + 8 * sz + n);
  const double grad_xi = sqrt(m11 * m11 + m12 * m12 + m13 * m13);
  const double grad_eta = sqrt(m21 * m21 + m22 * m22 + m23 * m23);
  const double grad_zeta = sqrt(m31 * m31 + m32 * m32 + m33 * m33);
  const double u = ld(B.bv + sz + n), v = ld(B.bv + 2 * sz + n), w = ld(B.bv + 3 * sz + n);
  const double U = u * m11 + v * m12 + w * m13;
  const double V = u * m21 + v * m22 + w * m23;
  const double W = u * m31 + v * m32 + w * m33;
  const double a = ld(B.acoustic + n);
  const double s0 = fabs(U) + a * grad_xi, s1 = fabs(V) + a * grad_eta;
  double s2 = 0;
  if (three_d) s2 = fabs(W) + a * grad_zeta;
  B.inv_spec[nd] = s0;
  B.inv_spec[szd + nd] = s1;
  B.inv_spec[2 * szd + nd] = s2;
  const double sri = s0 + s1 + s2;
  double gamma = kDGammaAir;
  if constexpr (C::mix != 0) gamma = ld(B.gamma + n);
  const double coeff_1 = fmax(gamma, 4.0 / 3.0) / ld(B.bv + n);
  double coeff_2 = ld(B.mul + n) / cP.Pr;
  if constexpr (C::turb) coeff_2 += ld(B.mut + n) / cP.Prt;
  double srv = grad_xi * grad_xi + grad_eta * grad_eta;
  if (three_d) srv += grad_zeta * grad_zeta;
  srv *= coeff_1 * coeff_2;
  B.visc_spec[nd] = srv;
  B.dt_local[B.Z.at(i, j, k)] = cP.cfl / (sri + srv);
}

// ---------------------------------------------------------------- fluxes
// Inviscid (AUSM+/MUSCL) then viscous (central) flux differences in the
// reference's accumulation order, plus local_time_step
// (src/TimeAdvanceFunc.cuh:21-71).
template <class C>
__global__ void __launch_bounds__(kCta, OSTC_FLUX_MIN_BLOCKS) k_flux(const DevBlock *__restrict__ blks, Tiles T) {
  constexpr int NV = C::nv;
  extern __shared__ double sf[];
  int b, i, j, k;
  if (!tile_cell<kTX, kTY, kTZ>(T, b, i, j, k, blks)) return;
  const DevBlock &B = blks[b];
  const int tid = threadIdx.x + kTX * (threadIdx.y + kTY * threadIdx.z);
  double *fm = sf + tid;  // stride kCta
  const int64_t n = B.G.at(i, j, k), nd = B.D.at(i, j, k), szd = B.D.size;
  const int64_t sx = B.G.sx, sxy = B.G.sxy;
  const bool three_d = B.mz > 1;
  double dq[NV];
  OSTC_UNROLL for (int l = 0; l < NV; ++l) dq[l] = B.dq[l * szd + nd];
  // Inviscid faces, then viscous faces, each direction as minus face (staged
  // in shared memory) then plus face: dq -= f(+) - f(-) for inviscid and
  // dq += f(+) - f(-) for viscous, the reference's accumulation order.  The
  // loops are not unrolled: one copy of each face routine keeps the kernel
  // within the instruction cache.
  const int n_face = three_d ? 6 : 4;
#pragma unroll 1
  for (int f = 0; f < n_face; ++f) {
    const int d = f >> 1;
    const int64_t s = d == 0 ? 1 : (d == 1 ? sx : sxy);
    double t[NV];
    inviscid_face<C>(B, (f & 1) ? n : n - s, d, s, t);
    if ((f & 1) == 0) {
      OSTC_UNROLL for (int l = 0; l < NV; ++l) fm[l * kCta] = t[l];
    } else {
      OSTC_UNROLL for (int l = 0; l < NV; ++l) dq[l] -= t[l] - fm[l * kCta];
    }
  }
  if (cP.viscous_order != 0) {
#pragma unroll 1
    for (int f = 0; f < n_face; ++f) {
      const int d = f >> 1;
      const int64_t s = d == 0 ? 1 : (d == 1 ? sx : sxy);
      double t[NV];
      viscous_face<C>(B, (f & 1) ? n : n - s, d, s, t);
      if ((f & 1) == 0) {
        OSTC_UNROLL for (int l = 0; l < NV; ++l) fm[l * kCta] = t[l];
      } else {
        OSTC_UNROLL for (int l = 0; l < NV; ++l) dq[l] += t[l] - fm[l * kCta];
      }
    }
  }
  OSTC_UNROLL for (int l = 0; l < NV; ++l) B.dq[l * szd + nd] = dq[l];
  local_time_step<C>(B, i, j, k, n, nd);
}

// The same flux differences with every face evaluated once: a CTA owns a
// column of 32 x 4 cells (i, j) over kFluxKC planes of k and marches in k;
// the four compute warps evaluate the plus faces of their cells in x, y and
// z, the fifth warp the column's low-i and low-j faces, and the low-k face of
// a plane is the high-k face of the plane before (shared memory).  Each face
// value is the one k_flux computes for it and the per-cell sums run in the
// same order (dq -= f(+) - f(-) per direction, inviscid then viscous), so the
// result is bit-identical.
constexpr int kFluxKC = 8;                  // k planes per column
constexpr int kFluxThreads = kCta + 32;     // 4 compute warps + the minus-face warp

__device__ __forceinline__ void col_tile(const Tiles &T, int &b, int &i0, int &j0, int &k0) {
  int t = tile_of(T, blockIdx.x, b);
  const int tx = t % T.ntx[b];
  t /= T.ntx[b];
  const int ty = t % T.nty[b];
  const int tz = t / T.nty[b];
  i0 = tx * kTX;
  j0 = ty * kTY;
  k0 = tz * kFluxKC;
}

// Shared-memory plan of a column kernel (elements): x faces [NV][kTY][kTX+1]
// (face i0 - 1/2 + f), y faces [NV][kTY+1][kTX] (face j0 - 1/2 + f), the
// low-k faces carried between planes [2][NV][kCta] (inviscid, viscous) and
// the high-k faces of the current plane [NV][kCta].
template <int NV>
struct ColSmem {
  static constexpr int xs = 0, ys = xs + NV * kTY * (kTX + 1), zs = ys + NV * (kTY + 1) * kTX,
                       zp = zs + 2 * NV * kCta, size = zp + NV * kCta;
};

// The faces of plane k of a column and the task that evaluates each: for a
// compute thread 0 x-plus, 1 y-plus, 2 z-minus (first plane only), 3 z-plus;
// for the minus-face warp 0 the low-i face of row lane, 1 the low-j face of
// column lane.  Returns false when the thread has no face for the task.
template <int NV>
__device__ __forceinline__ bool col_task(const DevBlock &B, int i0, int j0, int k, bool first, bool cell, int q,
                                         int zs_off, int64_t &nl, int &d, int64_t &s, int &off, int &stride) {
  using S = ColSmem<NV>;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, tid = threadIdx.x;
  const int i = i0 + lane, j = j0 + warp;
  const int64_t sx = B.G.sx, sxy = B.G.sxy;
  stride = kCta;
  if (cell) {
    const int64_t n = B.G.at(i, j, k);
    const int task = (q >= 2 && !first) ? q + 1 : q;  // x, y, low z (first plane), high z
    if (task == 0) {
      nl = n; d = 0; s = 1; off = S::xs + warp * (kTX + 1) + lane + 1; stride = kTY * (kTX + 1);
    } else if (task == 1) {
      nl = n; d = 1; s = sx; off = S::ys + (warp + 1) * kTX + lane; stride = (kTY + 1) * kTX;
    } else if (task == 2) {
      nl = n - sxy; d = 2; s = sxy; off = zs_off + tid;
    } else {
      nl = n; d = 2; s = sxy; off = S::zp + tid;
    }
    return true;
  }
  if (q == 0) {
    d = 0; s = 1; off = S::xs + lane * (kTX + 1); stride = kTY * (kTX + 1);
    if (!(lane < kTY && j0 + lane < B.my && i0 < B.mx)) return false;
    nl = B.G.at(i0, j0 + lane, k) - 1;
    return true;
  }
  d = 1; s = sx; off = S::ys + lane; stride = (kTY + 1) * kTX;
  if (!(i < B.mx && j0 < B.my)) return false;
  nl = B.G.at(i, j0, k) - sx;
  return true;
}

template <class C, int VISC>
__device__ __forceinline__ void col_faces64(const DevBlock &B, int i0, int j0, int k, bool first, bool cell,
                                            double *sm, double *dq) {
  constexpr int NV = C::nv;
  using S = ColSmem<NV>;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, tid = threadIdx.x;
  const bool three_d = B.mz > 1;
  const int zs_off = S::zs + VISC * NV * kCta;
  const int ntask = cell ? (three_d ? (first ? 4 : 3) : 2) : (warp == kTY ? 2 : 0);
#pragma unroll 1
  for (int q = 0; q < ntask; ++q) {
    int64_t nl = 0, s = 1;
    int d = 0, off = 0, stride = kCta;
    if (!col_task<NV>(B, i0, j0, k, first, cell, q, zs_off, nl, d, s, off, stride)) continue;
    double t[NV];
    if constexpr (VISC == 0)
      inviscid_face<C>(B, nl, d, s, t);
    else
      viscous_face<C>(B, nl, d, s, t);
    OSTC_UNROLL for (int l = 0; l < NV; ++l) sm[off + l * stride] = t[l];
  }
  __syncthreads();
  if (cell) {
    const double *xs = sm + S::xs + warp * (kTX + 1) + lane, *ys = sm + S::ys + warp * kTX + lane;
    double *zs = sm + zs_off;
    OSTC_UNROLL for (int l = 0; l < NV; ++l) {
      const double px = xs[l * kTY * (kTX + 1) + 1], mx = xs[l * kTY * (kTX + 1)];
      const double py = ys[l * (kTY + 1) * kTX + kTX], my = ys[l * (kTY + 1) * kTX];
      if constexpr (VISC == 0) {
        dq[l] -= px - mx;
        dq[l] -= py - my;
      } else {
        dq[l] += px - mx;
        dq[l] += py - my;
      }
      if (three_d) {
        const double pz = sm[S::zp + l * kCta + tid], mz = zs[l * kCta + tid];
        zs[l * kCta + tid] = pz;
        if constexpr (VISC == 0)
          dq[l] -= pz - mz;
        else
          dq[l] += pz - mz;
      }
    }
  }
  __syncthreads();
}

template <class C>
__global__ void __launch_bounds__(kFluxThreads, 2) k_flux_col(const DevBlock *__restrict__ blks, Tiles T) {
  constexpr int NV = C::nv;
  extern __shared__ double sm64[];
  int b, i0, j0, k0;
  col_tile(T, b, i0, j0, k0);
  const DevBlock &B = blks[b];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = i0 + lane, j = j0 + warp;
  const bool cell = warp < kTY && i < B.mx && j < B.my;
  const int64_t szd = B.D.size;
  const int k1 = min(k0 + kFluxKC, B.mz);
  for (int k = k0; k < k1; ++k) {
    double dq[NV];
    int64_t n = 0, nd = 0;
    if (cell) {
      n = B.G.at(i, j, k);
      nd = B.D.at(i, j, k);
      OSTC_UNROLL for (int l = 0; l < NV; ++l) dq[l] = B.dq[l * szd + nd];
    }
    col_faces64<C, 0>(B, i0, j0, k, k == k0, cell, sm64, dq);
    if (cP.viscous_order != 0) col_faces64<C, 1>(B, i0, j0, k, k == k0, cell, sm64, dq);
    if (!cell) continue;
    OSTC_UNROLL for (int l = 0; l < NV; ++l) B.dq[l * szd + nd] = dq[l];
    local_time_step<C>(B, i, j, k, n, nd);
  }
}

// ---------------------------------------------------------------- implicit
// Column-pivoted Doolittle LU of the ns x ns point-implicit matrix,
// src/FiniteRateChem.cu:286-342.  Factor and permutation are stored so that
// the DPLUR sweeps reuse them: the reference re-factors the identical matrix
// in every sweep, which yields the same factor bit for bit.
// Element (r, c) of the matrix sits at lhs[((r * NS + c) * ST) * ST]: ST = 1 for a
// per-thread array, the CTA size for a per-thread slice of shared memory.
template <int NS, int ST = 1>
__device__ __forceinline__ void lu_factor(double *lhs, int *ipiv) {
  OSTC_UNROLL for (int n = 0; n < NS; ++n) {
    int ik = n;
    double amax = 0;  // |lhs[ik][n]|: entries of column n above row m are final
    OSTC_UNROLL for (int m = n; m < NS; ++m) {
      OSTC_UNROLL for (int t = 0; t < n; ++t) lhs[(m * NS + n) * ST] -= lhs[(m * NS + t) * ST] * lhs[(t * NS + n) * ST];
      const double a = fabs(lhs[(m * NS + n) * ST]);
      if (m == n) {
        amax = a;
      } else if (a > amax) {
        ik = m;
        amax = a;
      }
    }
    ipiv[n] = ik;
    if (ik != n) {
      OSTC_UNROLL for (int t = 0; t < NS; ++t) {
        // swap rows n and ik; ik is data dependent, so select row by row
        double rowk = lhs[(n * NS + t) * ST];
        double other = 0;
        OSTC_UNROLL for (int q = n + 1; q < NS; ++q)
          if (q == ik) other = lhs[(q * NS + t) * ST];
        OSTC_UNROLL for (int q = n + 1; q < NS; ++q)
          if (q == ik) lhs[(q * NS + t) * ST] = rowk;
        lhs[(n * NS + t) * ST] = other;
      }
    }
    OSTC_UNROLL for (int p = n + 1; p < NS; ++p)
      OSTC_UNROLL for (int t = 0; t < n; ++t) lhs[(n * NS + p) * ST] -= lhs[(n * NS + t) * ST] * lhs[(t * NS + p) * ST];
    OSTC_UNROLL for (int m = n + 1; m < NS; ++m) lhs[(m * NS + n) * ST] /= lhs[(n * NS + n) * ST];
  }
}

template <int NS, int ST = 1>
__device__ __forceinline__ void lu_solve(const double *lhs, const int *ipiv, double *rhs) {
  OSTC_UNROLL for (int m = 0; m < NS; ++m) {
    const int t = ipiv[m];
    if (t != m) {
      double a = rhs[m], other = 0;
      OSTC_UNROLL for (int q = m + 1; q < NS; ++q)
        if (q == t) other = rhs[q];
      OSTC_UNROLL for (int q = m + 1; q < NS; ++q)
        if (q == t) rhs[q] = a;
      rhs[m] = other;
    }
  }
  OSTC_UNROLL for (int m = 1; m < NS; ++m)
    OSTC_UNROLL for (int t = 0; t < m; ++t) rhs[m] -= lhs[(m * NS + t) * ST] * rhs[t];
  rhs[NS - 1] /= lhs[(NS * NS - 1) * ST];
  OSTC_UNROLL for (int m = NS - 2; m >= 0; --m) {
    OSTC_UNROLL for (int t = m + 1; t < NS; ++t) rhs[m] -= lhs[(m * NS + t) * ST] * rhs[t];
    rhs[m] /= lhs[(m * NS + m) * ST];
  }
}

// lu_solve with the factors read from the arrays (entry q of the cell at
// lhs[q * st]): each factor is used once, so none is held in registers or
// local memory; same operations in the same order as lu_solve.
template <int NS>
__device__ __forceinline__ void lu_solve_g(const double *__restrict__ lhs, int64_t st, const int *ipiv,
                                           double *rhs) {
  OSTC_UNROLL for (int m = 0; m < NS; ++m) {
    const int t = ipiv[m];
    if (t != m) {
      double a = rhs[m], other = 0;
      OSTC_UNROLL for (int q = m + 1; q < NS; ++q)
        if (q == t) other = rhs[q];
      OSTC_UNROLL for (int q = m + 1; q < NS; ++q)
        if (q == t) rhs[q] = a;
      rhs[m] = other;
    }
  }
  OSTC_UNROLL for (int m = 1; m < NS; ++m)
    OSTC_UNROLL for (int t = 0; t < m; ++t) rhs[m] -= __ldg(lhs + (m * NS + t) * st) * rhs[t];
  rhs[NS - 1] /= __ldg(lhs + (NS * NS - 1) * st);
  OSTC_UNROLL for (int m = NS - 2; m >= 0; --m) {
    OSTC_UNROLL for (int t = m + 1; t < NS; ++t) rhs[m] -= __ldg(lhs + (m * NS + t) * st) * rhs[t];
    rhs[m] /= __ldg(lhs + (m * NS + m) * st);
  }
}

// Explicit-mode point-implicit treatment: EPI / DA and the SST diagonal,
// src/ImplicitTreatmentHPP.cuh:14-54, src/FiniteRateChem.cu:211-234, 400-412,
// src/SST.cu:180-194.
template <class C>
__global__ void __launch_bounds__(kCta) k_point_implicit(const DevBlock *__restrict__ blks, Tiles T) {
  constexpr int NS = C::ns;
  int b, i, j, k;
  if (!tile_cell<kTX, kTY, kTZ>(T, b, i, j, k, blks)) return;
  const DevBlock &B = blks[b];
  const int64_t nd = B.D.at(i, j, k), nz = B.Z.at(i, j, k), szd = B.D.size, sz0 = B.Z.size;
  const double dt = B.dt_local[nz];
  if constexpr (C::mix == 2) {
    // a chemically quiet cell has no chemistry Jacobian: I x = dq leaves dq
    if (B.chem_quiet && B.chem_quiet[nz]) {
    } else if (cP.chem_src_method == 1) {
      double lhs[NS * NS];
      int piv[NS];
      OSTC_UNROLL for (int m = 0; m < NS; ++m)
        OSTC_UNROLL for (int q = 0; q < NS; ++q) {
          const double J = B.chem_jac[(m * NS + q) * sz0 + nz];
          lhs[m * NS + q] = (m == q) ? 1.0 - dt * J : -dt * J;
        }
      lu_factor<NS>(lhs, piv);
      double rhs[NS];
      OSTC_UNROLL for (int l = 0; l < NS; ++l) rhs[l] = B.dq[(5 + l) * szd + nd];
      lu_solve<NS>(lhs, piv, rhs);
      OSTC_UNROLL for (int l = 0; l < NS; ++l) B.dq[(5 + l) * szd + nd] = rhs[l];
    } else if (cP.chem_src_method == 2) {
      OSTC_UNROLL for (int l = 0; l < NS; ++l) B.dq[(5 + l) * szd + nd] /= 1 - dt * B.chem_jac[l * sz0 + nz];
    }
  }
  if constexpr (C::turb) {
    if (cP.turb_implicit == 1) {
      B.dq[(NS + 5) * szd + nd] /= 1 - dt * B.turb_src_jac[nz];
      B.dq[(NS + 6) * szd + nd] /= 1 - dt * B.turb_src_jac[sz0 + nz];
    }
  }
}

// compute_DQ_0, src/DPLURHPP.cuh:13-76.  Writes dq0; with EPI the factored
// matrix replaces the Jacobian in chem_jac and the pivots go to lu_piv.
template <class C>
__global__ void __launch_bounds__(kCta) k_dq0(const DevBlock *__restrict__ blks, Tiles T) {
  constexpr int NS = C::ns, NV = C::nv;
  int b, i, j, k;
  if (!tile_cell<kTX, kTY, kTZ>(T, b, i, j, k, blks)) return;
  const DevBlock &B = blks[b];
  const int64_t nd = B.D.at(i, j, k), nz = B.Z.at(i, j, k), szd = B.D.size, sz0 = B.Z.size;
  const double dt = B.dt_local[nz];
  const double diag = 1 + dt * (B.inv_spec[nd] + B.inv_spec[szd + nd] + B.inv_spec[2 * szd + nd]);
  double dq[NV];  // loaded before the first store, which would hold the loads back
  OSTC_UNROLL for (int l = 0; l < NV; ++l) dq[l] = B.dq[l * szd + nd];
  if constexpr (C::mix != 0) {
    // T is fixed during the sweeps: evaluate the species enthalpies once
    double hk[NS];
    enthalpy<NS>(B.bv[5 * B.G.size + B.G.at(i, j, k)], hk);
    if constexpr (C::mixed) {
      OSTC_UNROLL for (int l = 0; l < NS; ++l) B.h_spec32[l * szd + nd] = static_cast<float>(hk[l]);
    } else {
      OSTC_UNROLL for (int l = 0; l < NS; ++l) B.h_spec[l * szd + nd] = hk[l];
    }
  }
  if constexpr (C::mix != 2) {
    OSTC_UNROLL for (int l = 0; l < 5 + NS; ++l) dq[l] /= diag;
  } else {
    OSTC_UNROLL for (int l = 0; l < 5; ++l) dq[l] /= diag;
    const int method = cP.chem_src_method;
    if (B.chem_quiet && B.chem_quiet[nz]) {
      // no chemistry Jacobian: the factorisation of diag I is diag I, and
      // its solve divides by diag (bit for bit)
      OSTC_UNROLL for (int l = 0; l < NS; ++l) dq[5 + l] /= diag;
    } else if (method == 1 && C::mixed && cP.na == NS - 1) {
      // FP32-bulk path: the leading (NS-1) x (NS-1) block, the last species
      // with its single pivot diag (what the full factorisation gives it)
      extern __shared__ double sdq[];
      double *lhs = sdq + threadIdx.x + kTX * (threadIdx.y + kTY * threadIdx.z);
      constexpr int NA = NS > 1 ? NS - 1 : 1;
      int piv[NA];
      OSTC_UNROLL for (int m = 0; m < NA; ++m)
        OSTC_UNROLL for (int q = 0; q < NA; ++q) {
          const double J = B.chem_jac[(m * NA + q) * sz0 + nz];
          lhs[(m * NA + q) * kCta] = (m == q) ? diag - dt * J : -dt * J;
        }
      lu_factor<NA, kCta>(lhs, piv);
      lu_solve<NA, kCta>(lhs, piv, dq + 5);
      OSTC_UNROLL for (int l = NA; l < NS; ++l) dq[5 + l] /= diag;
      OSTC_UNROLL for (int q = 0; q < NA * NA; ++q) B.chem_jac[q * sz0 + nz] = lhs[q * kCta];
      OSTC_UNROLL for (int q = 0; q < NA; ++q) B.lu_piv[q * sz0 + nz] = static_cast<unsigned char>(piv[q]);
    } else if (method == 1) {
      // the matrix lives in this thread's slice of shared memory (stride kCta)
      extern __shared__ double sdq[];
      double *lhs = sdq + threadIdx.x + kTX * (threadIdx.y + kTY * threadIdx.z);
      int piv[NS];
      OSTC_UNROLL for (int m = 0; m < NS; ++m)
        OSTC_UNROLL for (int q = 0; q < NS; ++q) {
          const double J = B.chem_jac[(m * NS + q) * sz0 + nz];
          lhs[(m * NS + q) * kCta] = (m == q) ? diag - dt * J : -dt * J;
        }
      lu_factor<NS, kCta>(lhs, piv);
      lu_solve<NS, kCta>(lhs, piv, dq + 5);
      OSTC_UNROLL for (int q = 0; q < NS * NS; ++q) B.chem_jac[q * sz0 + nz] = lhs[q * kCta];
      OSTC_UNROLL for (int q = 0; q < NS; ++q) B.lu_piv[q * sz0 + nz] = static_cast<unsigned char>(piv[q]);
    } else if (method == 2) {
      OSTC_UNROLL for (int l = 0; l < NS; ++l) dq[5 + l] /= diag - dt * B.chem_jac[l * sz0 + nz];
    } else {
      OSTC_UNROLL for (int l = 0; l < NS; ++l) dq[5 + l] /= diag;
    }
  }
  if constexpr (C::turb) {
    if (cP.turb_implicit == 1) {
      dq[NS + 5] /= diag - dt * B.turb_src_jac[nz];
      dq[NS + 6] /= diag - dt * B.turb_src_jac[sz0 + nz];
    } else {
      dq[NS + 5] /= diag;
      dq[NS + 6] /= diag;
    }
  }
  if constexpr (C::mixed) {
    OSTC_UNROLL for (int l = 0; l < NV; ++l) B.dqf[0][l * szd + nd] = static_cast<float>(dq[l]);
    if (cP.dplur_inner_step == 0)
      OSTC_UNROLL for (int l = 0; l < NV; ++l) B.dq0[l * szd + nd] = dq[l];
  } else {
    OSTC_UNROLL for (int l = 0; l < NV; ++l) B.dq0[l * szd + nd] = dq[l];
  }
}

// compute_jacobian_times_dq, src/DPLURHPP.cuh:78-125, accumulated into tot
// with weight +-0.5 (sign < 0 subtracts), for the neighbour n along the
// run-time direction dir.  The species enthalpies come from h_spec (k_dq0).
template <class C>
__device__ __forceinline__ void add_jac_dq(const DevBlock &B, const double *__restrict__ dqin, int64_t n,
                                           int64_t nd, int dir, double pm_sr, bool subtract, double *tot) {
  constexpr int NS = C::ns, NV = C::nv;
  const int64_t sz = B.G.size, szd = B.D.size;
  const double *mr = B.metric + 3 * dir * sz;
  const double xi_x = ld(mr + n), xi_y = ld(mr + sz + n), xi_z = ld(mr + 2 * sz + n);
  const double u = ld(B.bv + sz + n), v = ld(B.bv + 2 * sz + n), w = ld(B.bv + 3 * sz + n);
  const double U = xi_x * u + xi_y * v + xi_z * w;
  const double lmd1 = U + pm_sr;
  const double vel = ld(B.vel + n);
  const double e = 0.5 * vel * vel;
  double gamma = kDGammaAir, b3 = 0, b4 = 0, h = 0;
  double d[NV];
  OSTC_UNROLL for (int l = 0; l < NV; ++l) d[l] = ld(dqin + l * szd + nd);
  if constexpr (C::mix != 0) {
    double hk[NS];
    const double t = ld(B.bv + 5 * sz + n);
    OSTC_UNROLL for (int l = 0; l < NS; ++l) hk[l] = ld(B.h_spec + l * szd + nd);
    gamma = ld(B.gamma + n);
    OSTC_UNROLL for (int l = 0; l < NS; ++l) {
      b3 += kDR_u * t / cP.mw[l] * d[5 + l];
      b4 += hk[l] * d[5 + l];
      h += ld(B.sv + l * sz + n) * hk[l];
    }
    b3 *= gamma;
    b4 *= gamma - 1;
    h += e;
  } else {
    h = gamma / (gamma - 1) * ld(B.bv + 4 * sz + n) / ld(B.bv + n) + e;
  }
  const double b1 = xi_x * d[1] + xi_y * d[2] + xi_z * d[3] - U * d[0];
  const double b2 = (gamma - 1) * (e * d[0] - u * d[1] - v * d[2] - w * d[3] + d[4]);
  double o[NV];
  o[0] = b1 + lmd1 * d[0];
  o[1] = u * b1 + xi_x * b2 + lmd1 * d[1] + xi_x * (b3 - b4);
  o[2] = v * b1 + xi_y * b2 + lmd1 * d[2] + xi_y * (b3 - b4);
  o[3] = w * b1 + xi_z * b2 + lmd1 * d[3] + xi_z * (b3 - b4);
  o[4] = h * b1 + U * b2 + lmd1 * d[4] + U * (b3 - b4);
  OSTC_UNROLL for (int l = 0; l < C::nsc; ++l) o[5 + l] = lmd1 * d[5 + l] + ld(B.sv + l * sz + n) * b1;
  if (subtract) {
    OSTC_UNROLL for (int l = 0; l < NV; ++l) tot[l] -= 0.5 * o[l];
  } else {
    OSTC_UNROLL for (int l = 0; l < NV; ++l) tot[l] += 0.5 * o[l];
  }
}

// DPLUR_inner_iteration, src/DPLURHPP.cuh:127-249: dqout = dq0 + dt*sum/diag
// with the neighbours' A(+-)*dqin; the point-implicit blocks reuse the LU.
template <class C>
__global__ void __launch_bounds__(kCta, OSTC_SWEEP_MIN_BLOCKS) k_sweep(const DevBlock *__restrict__ blks, Tiles T, int in_sel, int out_sel) {
  constexpr int NS = C::ns, NV = C::nv;
  int b, i, j, k;
  if (!tile_cell<kTX, kTY, kTZ>(T, b, i, j, k, blks)) return;
  const DevBlock &B = blks[b];
  const double *dqin = in_sel == 0 ? B.dq : (in_sel == 1 ? B.dq0 : B.dqk);
  double *dqout = out_sel == 0 ? B.dq : B.dqk;
  const int64_t szd = B.D.size, sz0 = B.Z.size;
  const int64_t n = B.G.at(i, j, k), nd = B.D.at(i, j, k), nz = B.Z.at(i, j, k);
  const int64_t sx = B.G.sx, sxy = B.G.sxy, dsx = B.D.sx, dsxy = B.D.sxy;
  double tot[NV];
  OSTC_UNROLL for (int l = 0; l < NV; ++l) tot[l] = 0;
  const double *isr = B.inv_spec;
  // neighbours i-1, j-1, k-1 (added with +lambda), then i+1, j+1, k+1
  // (subtracted with -lambda); neighbours outside the block are skipped
#pragma unroll 1
  for (int q = 0; q < 6; ++q) {
    const int d = q < 3 ? q : q - 3;
    const bool plus = q >= 3;
    const int id = d == 0 ? i : (d == 1 ? j : k);
    const int ext = d == 0 ? B.mx : (d == 1 ? B.my : B.mz);
    if ((plus ? id == ext - 1 : id == 0) && !(B.inner_mask >> (2 * d + (plus ? 1 : 0)) & 1)) continue;
    const int64_t gs = d == 0 ? 1 : (d == 1 ? sx : sxy), ds = d == 0 ? 1 : (d == 1 ? dsx : dsxy);
    const int64_t on = plus ? n + gs : n - gs, od = plus ? nd + ds : nd - ds;
    const double sr = isr[d * szd + od];
    add_jac_dq<C>(B, dqin, on, od, d, plus ? -sr : sr, plus, tot);
  }
  const double dt = B.dt_local[nz];
  const double diag = 1 + dt * (isr[nd] + isr[szd + nd] + isr[2 * szd + nd]);
  double out[NV];
  if constexpr (C::mix != 2) {
    OSTC_UNROLL for (int l = 0; l < 5 + NS; ++l) out[l] = B.dq0[l * szd + nd] + dt * tot[l] / diag;
  } else {
    OSTC_UNROLL for (int l = 0; l < 5; ++l) out[l] = B.dq0[l * szd + nd] + dt * tot[l] / diag;
    const int method = cP.chem_src_method;
    if (B.chem_quiet && B.chem_quiet[nz]) {
      // chemically quiet: the stored factors would be diag I
      OSTC_UNROLL for (int l = 0; l < NS; ++l) out[5 + l] = B.dq0[(5 + l) * szd + nd] + dt * tot[5 + l] / diag;
    } else if (method == 1) {
      int piv[NS];
      OSTC_UNROLL for (int q = 0; q < NS; ++q) piv[q] = B.lu_piv[q * sz0 + nz];
      double rhs[NS];
      OSTC_UNROLL for (int l = 0; l < NS; ++l) rhs[l] = tot[5 + l] * dt;
      lu_solve_g<NS>(B.chem_jac + nz, sz0, piv, rhs);
      OSTC_UNROLL for (int l = 0; l < NS; ++l) out[5 + l] = B.dq0[(5 + l) * szd + nd] + rhs[l];
    } else if (method == 2) {
      OSTC_UNROLL for (int l = 0; l < NS; ++l)
        out[5 + l] = B.dq0[(5 + l) * szd + nd] + dt * tot[5 + l] / (diag - dt * B.chem_jac[l * sz0 + nz]);
    } else {
      OSTC_UNROLL for (int l = 0; l < NS; ++l) out[5 + l] = B.dq0[(5 + l) * szd + nd] + dt * tot[5 + l] / diag;
    }
  }
  if constexpr (C::turb) {
    if (cP.turb_implicit == 1) {
      out[NS + 5] = B.dq0[(NS + 5) * szd + nd] + dt * tot[5 + NS] / (diag - dt * B.turb_src_jac[nz]);
      out[NS + 6] = B.dq0[(NS + 6) * szd + nd] + dt * tot[6 + NS] / (diag - dt * B.turb_src_jac[sz0 + nz]);
    } else {
      out[NS + 5] = B.dq0[(NS + 5) * szd + nd] + dt * tot[5 + NS] / diag;
      out[NS + 6] = B.dq0[(NS + 6) * szd + nd] + dt * tot[6 + NS] / diag;
    }
  }
  OSTC_UNROLL for (int l = 0; l < NV; ++l) dqout[l * szd + nd] = out[l];
}

// ---------------------------------------------------------------- update
// compute_temperature, src/FieldOperation.cu:3-40
template <int NS>
__device__ __forceinline__ void newton_temperature(const double *Y, double rho, double e, double &t, double &p) {
  double mw = 0;
  OSTC_UNROLL for (int l = 0; l < NS; ++l) mw += Y[l] / cP.mw[l];
  mw = 1 / mw;
  const double gas_const = kDR_u / mw;
  double err = 1;
  int iter = 0;
  while (err > 1e-3 && iter++ < 1000) {
    double hi[NS], cpi[NS];
    enthalpy_cp<NS>(t, hi, cpi);
    double cp_tot = 0, h = 0;
    OSTC_UNROLL for (int l = 0; l < NS; ++l) {
      cp_tot += cpi[l] * Y[l];
      h += hi[l] * Y[l];
    }
    const double e_t = h - gas_const * t;
    const double cv = cp_tot - gas_const;
    const double t1 = t - (e_t - e) / cv;
    err = fabs(1 - t1 / t);
    t = t1;
  }
  p = rho * t * gas_const;
}

// Primitive recovery from Q at one point (update_bv_1_point,
// src/FieldOperation.cuh:185-215), from the new Q held in registers: writes
// bv, sv and the velocity magnitude of point n and leaves rho, u, v, w, p in
// v5 and k, omega in turb2 (RANS) for the caller's checks.  Every load (the
// previous temperature, the Newton start) comes before the first store.
template <class C>
__device__ __forceinline__ void primitives_from_regs(const DevBlock &B, int64_t n, const double *q, double *v5,
                                                     double *turb2) {
  constexpr int NS = C::ns;
  const int64_t sz = B.G.size;
  const double rho = q[0];
  const double rinv = 1.0 / rho;
  const double u = q[1] * rinv, v = q[2] * rinv, w = q[3] * rinv;
  const double vel2 = u * u + v * v + w * w;
  double sv[C::nsc > 0 ? C::nsc : 1];
  if constexpr (C::mix != 0 || C::turb) {
    OSTC_UNROLL for (int l = 0; l < C::nsc; ++l) sv[l] = q[5 + l] * rinv;
  }
  double p, t;
  if constexpr (C::mix != 0) {
    const double e = q[4] / rho - 0.5 * (u * u + v * v + w * w);
    t = B.bv[5 * sz + n];
    newton_temperature<NS>(sv, rho, e, t, p);
  } else {
    p = (kDGammaAir - 1) * (q[4] - 0.5 * rho * vel2);
    t = p * kDMwAir * rinv / kDR_u;
  }
  B.bv[n] = rho;
  B.bv[sz + n] = u;
  B.bv[2 * sz + n] = v;
  B.bv[3 * sz + n] = w;
  B.bv[4 * sz + n] = p;
  B.bv[5 * sz + n] = t;
  if constexpr (C::mix != 0 || C::turb) {
    OSTC_UNROLL for (int l = 0; l < C::nsc; ++l) B.sv[l * sz + n] = sv[l];
  }
  B.vel[n] = sqrt(vel2);
  v5[0] = rho;
  v5[1] = u;
  v5[2] = v;
  v5[3] = w;
  v5[4] = p;
  if constexpr (C::turb) {
    turb2[0] = sv[NS];
    turb2[1] = sv[NS + 1];
  }
}

// The same from Q in memory (cv of point n must already hold the new Q).
template <class C>
__device__ __forceinline__ void primitives_from_q(const DevBlock &B, int64_t n) {
  double q[C::nv], v5[5], turb2[2];
  OSTC_UNROLL for (int l = 0; l < C::nv; ++l) q[l] = B.cv[l * B.G.size + n];
  primitives_from_regs<C>(B, n, q, v5, turb2);
}

__device__ __forceinline__ bool flow_unphysical(const double *v) {
  bool bad = false;
  OSTC_UNROLL for (int l = 0; l < 5; ++l) bad |= isnan(v[l]) || v[l] < cP.ll[l] || v[l] > cP.ul[l];
  return bad;
}

// update_cv_and_bv, src/FieldOperation.cuh:139-183.  Counts unphysical cells
// so that the limiter pass can skip the block when there are none.
template <class C>
__global__ void __launch_bounds__(kCta, 3) k_update(const DevBlock *__restrict__ blks, Tiles T, int dq_sel,
                                                 unsigned int *bad_count) {
  constexpr int NV = C::nv;
  int b, i, j, k;
  if (!tile_cell<kTX, kTY, kTZ>(T, b, i, j, k, blks)) return;
  const DevBlock &B = blks[b];
  const double *dq = dq_sel == 0 ? B.dq : (dq_sel == 1 ? B.dq0 : B.dqk);
  const int64_t n = B.G.at(i, j, k), nd = B.D.at(i, j, k), nz = B.Z.at(i, j, k);
  const int64_t sz = B.G.size, szd = B.D.size;
  // every load first (the arrays may alias as far as the compiler knows, so a
  // load after a store would wait for it), then the arithmetic, then the stores
  const double dt_div_jac = B.dt_local[nz] / B.jac[n];
  double q[NV], d[NV];
  OSTC_UNROLL for (int l = 0; l < NV; ++l) q[l] = B.cv[l * sz + n];
  OSTC_UNROLL for (int l = 0; l < NV; ++l) d[l] = dq[l * szd + nd];
  OSTC_UNROLL for (int l = 0; l < NV; ++l) q[l] += d[l] * dt_div_jac;
  if (B.mz == 1) q[3] = 0;
  double v[5], turb2[2];
  primitives_from_regs<C>(B, n, q, v, turb2);
  OSTC_UNROLL for (int l = 0; l < NV; ++l) B.cv[l * sz + n] = q[l];
  bool bad = flow_unphysical(v);
  if constexpr (C::turb) {
    const double tk = turb2[0], tw = turb2[1];
    bad |= isnan(tk) || isnan(tw) || tk < 0 || tw < 0;
  }
  if (bad) atomicAdd(bad_count, 1u);
}

// limit_flow, src/TimeAdvanceFunc.cu:34-224 (neighbour loop bounded by mz
// in i as in the reference).  Does nothing unless k_update counted a bad cell.
template <class C>
__global__ void __launch_bounds__(kCta) k_limit(const DevBlock *__restrict__ blks, Tiles T,
                                                const unsigned int *bad_count) {
  constexpr int NS = C::ns, NSC = C::nsc;
  if (*bad_count == 0) return;
  int b, i, j, k;
  if (!tile_cell<kTX, kTY, kTZ>(T, b, i, j, k, blks)) return;
  const DevBlock &B = blks[b];
  const int64_t sz = B.G.size;
  const int64_t n = B.G.at(i, j, k);
  const int mx = B.mx, my = B.my, mz = B.mz;
  (void)mx;
  double var[5];
  OSTC_UNROLL for (int l = 0; l < 5; ++l) var[l] = B.bv[l * sz + n];
  if (flow_unphysical(var)) {
    double up[5 + NSC];
    OSTC_UNROLL for (int l = 0; l < 5 + NSC; ++l) up[l] = 0;
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
          const int64_t q = B.G.at(i1, j1, k1);
          double nv5[5];
          OSTC_UNROLL for (int l = 0; l < 5; ++l) nv5[l] = B.bv[l * sz + q];
          if (flow_unphysical(nv5)) continue;
          OSTC_UNROLL for (int l = 0; l < 5; ++l) up[l] += nv5[l];
          OSTC_UNROLL for (int l = 0; l < NSC; ++l) up[l + 5] += B.sv[l * sz + q];
          ++kn;
        }
      }
    }
    if (kn > 0) {
      const double kinv = 1.0 / kn;
      OSTC_UNROLL for (int l = 0; l < 5 + NSC; ++l) up[l] *= kinv;
    } else {
      OSTC_UNROLL for (int l = 0; l < 5; ++l) up[l] = fmin(fmax(var[l], cP.ll[l]), cP.ul[l]);
      OSTC_UNROLL for (int l = 0; l < NSC; ++l) up[l + 5] = cP.sv_inf[l];
    }
    OSTC_UNROLL for (int l = 0; l < 5; ++l) B.bv[l * sz + n] = up[l];
    B.cv[n] = up[0];
    B.cv[sz + n] = up[0] * up[1];
    B.cv[2 * sz + n] = up[0] * up[2];
    B.cv[3 * sz + n] = up[0] * up[3];
    double e = 0.5 * up[0] * (up[1] * up[1] + up[2] * up[2] + up[3] * up[3]);
    OSTC_UNROLL for (int l = 0; l < NSC; ++l) {
      B.sv[l * sz + n] = up[5 + l];
      B.cv[(5 + l) * sz + n] = up[0] * up[5 + l];
    }
    if constexpr (NS > 0) {
      double mw = 0;
      OSTC_UNROLL for (int l = 0; l < NS; ++l) mw += up[5 + l] / cP.mw[l];
      mw = 1 / mw;
      const double t = up[4] * mw / (up[0] * kDR_u);
      B.bv[5 * sz + n] = t;
      double h[NS];
      enthalpy<NS>(t, h);
      OSTC_UNROLL for (int l = 0; l < NS; l++) e += h[l] * B.cv[(5 + l) * sz + n];
      e -= up[4];
    } else {
      B.bv[5 * sz + n] = up[4] * kDMwAir / (up[0] * kDR_u);
      e += up[4] / (kDGammaAir - 1);
    }
    B.cv[4 * sz + n] = e;
  }
  if constexpr (C::turb) {
    const double t0 = B.sv[NS * sz + n], t1 = B.sv[(NS + 1) * sz + n];
    if (isnan(t0) || isnan(t1) || t0 < 0 || t1 < 0) {
      double up0 = 0, up1 = 0;
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
            const int64_t q = B.G.at(i1, j1, k1);
            const double a0 = B.sv[NS * sz + q], a1 = B.sv[(NS + 1) * sz + q];
            if (isnan(a0) || isnan(a1) || a0 < 0 || a1 < 0) continue;
            up0 += a0;
            up1 += a1;
            ++kn;
          }
        }
      }
      if (kn > 0) {
        const double kinv = 1.0 / kn;
        up0 *= kinv;
        up1 *= kinv;
      } else {
        up0 = t0 < 0 ? cP.sv_inf[NS] : t0;
        up1 = t1 < 0 ? cP.sv_inf[NS + 1] : t1;
      }
      B.sv[NS * sz + n] = up0;
      B.sv[(NS + 1) * sz + n] = up1;
      B.cv[(NS + 5) * sz + n] = B.cv[n] * up0;
      B.cv[(NS + 6) * sz + n] = B.cv[n] * up1;
    }
  }
}

// update_physical_properties + compute_transport_property,
// src/FieldOperation.cuh:75-109, src/Transport.cu:40-84 (interior + one
// ghost layer: launched with halo 1).
template <class C>
__global__ void __launch_bounds__(kCta) k_props(const DevBlock *__restrict__ blks, Tiles T) {
  constexpr int NS = C::ns;
  int b, i, j, k;
  if (!tile_cell<kTX, kTY, kTZ>(T, b, i, j, k, blks)) return;
  const DevBlock &B = blks[b];
  const int64_t n = B.G.at(i, j, k), sz = B.G.size;
  const double t = B.bv[5 * sz + n];
  const double speed = B.vel[n];  // read before the first store, which would hold it back
  if constexpr (C::mix != 0) {
    double cp[NS], Y[NS];
    heat_capacity<NS>(t, cp);
    double mw = 0, cp_tot = 0, cv = 0;
    OSTC_UNROLL for (int l = 0; l < NS; ++l) {
      Y[l] = B.sv[l * sz + n];
      mw += Y[l] / cP.mw[l];
      cp_tot += Y[l] * cp[l];
      cv += Y[l] * (cp[l] - cP.ru_mw[l]);
    }
    mw = 1 / mw;
    const double gamma = cp_tot / cv;
    B.cp[n] = cp_tot;
    B.gamma[n] = gamma;
    const double a = sqrt(gamma * kDR_u * t / mw);
    B.acoustic[n] = a;
    double X[NS], vis[NS];
    species_viscosity<NS>(t, mw, Y, X, vis);
    double viscosity = 0, conductivity = 0;
    OSTC_UNROLL for (int m = 0; m < NS; ++m) {
      const double vt = wilke_sum<NS>(vis, X, m);
      const double cond_temp = 1.065 * vt - 0.065 * X[m];
      viscosity += vis[m] * X[m] / vt;
      const double lambda = vis[m] * (cp[m] + 1.25 * kDR_u / cP.mw[m]);
      conductivity += lambda * X[m] / cond_temp;
    }
    B.mul[n] = viscosity;
    B.cond[n] = conductivity;
    const double sc = cP.Sc;
    OSTC_UNROLL for (int l = 0; l < NS; ++l) {
      double d;
      if (fabs(X[l] - 1) < 1e-3) {
        d = viscosity / sc;
      } else {
        d = (1 - Y[l]) * viscosity / ((1 - X[l]) * sc);
      }
      B.rho_d[l * sz + n] = d;
    }
    B.mach[n] = speed / a;
  } else {
    constexpr double c_temp = kDGammaAir * kDR_u / kDMwAir;
    constexpr double cp = kDGammaAir * kDR_u / kDMwAir / (kDGammaAir - 1);
    const double a = sqrt(c_temp * t);
    B.acoustic[n] = a;
    const double mul = sutherland(t);
    B.mul[n] = mul;
    B.cond[n] = mul * cp / cP.Pr;
    B.mach[n] = speed / a;
  }
}

// ---------------------------------------------------------------- boundaries
// One boundary face (src/BoundCond.cuh:45-319).
struct DevBc {
  int block, type, face, direction;
  int start[3], end[3];
  double density, u, v, w, pressure, temperature, mut;
  double sv[kMaxSpec + 2];
  int isothermal;
  double t_wall;
};

// compute_total_energy, src/FieldOperation.cuh:15-35: rho E of a cell from
// its primitives and the species' rho Y; speed = |V|
template <class C>
__device__ __forceinline__ double total_energy_of(double rho, double u, double v, double w, double p, double t,
                                                  const double *rho_y, double &speed) {
  constexpr int NS = C::ns;
  const double vel = u * u + v * v + w * w;
  // the reference stores this product in cv before adding the enthalpies
  double e = __dmul_rn(0.5 * rho, vel);
  if constexpr (C::mix != 0) {
    double h[NS];
    enthalpy<NS>(t, h);
    OSTC_UNROLL for (int l = 0; l < NS; l++) e += h[l] * rho_y[l];
    e -= p;
  } else {
    e += p / (kDGammaAir - 1);
  }
  speed = sqrt(vel);
  return e;
}

template <class C>
__device__ __forceinline__ void total_energy(const DevBlock &B, int64_t n) {
  constexpr int NS = C::ns;
  const int64_t sz = B.G.size;
  double rho_y[NS > 0 ? NS : 1];
  if constexpr (C::mix != 0)
    OSTC_UNROLL for (int l = 0; l < NS; l++) rho_y[l] = B.cv[(5 + l) * sz + n];
  double speed;
  B.cv[4 * sz + n] = total_energy_of<C>(B.bv[n], B.bv[sz + n], B.bv[2 * sz + n], B.bv[3 * sz + n],
                                        B.bv[4 * sz + n], B.bv[5 * sz + n], rho_y, speed);
  B.vel[n] = speed;
}

// Each branch reads what it needs before its first store: the compiler cannot
// tell the arrays apart, so a load written after a store would wait for that
// store, one memory round trip per variable.  The arithmetic is the
// reference's, in its order.
template <class C>
__global__ void k_bc(const DevBlock *__restrict__ blks, const DevBc *__restrict__ bcs, int face) {
  constexpr int NS = C::ns, NSC = C::nsc;
  constexpr int NS1 = NS > 0 ? NS : 1, NSC1 = NSC > 0 ? NSC : 1;
  const DevBc &f = bcs[face];
  const int e0 = f.end[0] - f.start[0] + 1, e1 = f.end[1] - f.start[1] + 1, e2 = f.end[2] - f.start[2] + 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= e0 * e1 * e2) return;
  const int i = f.start[0] + t % e0, j = f.start[1] + (t / e0) % e1, k = f.start[2] + t / (e0 * e1);
  const DevBlock &B = blks[f.block];
  const int64_t sz = B.G.size;
  const int ngg = B.ngg;
  int dir[3] = {0, 0, 0};
  dir[f.face] = f.direction;
  const int64_t step = dir[0] + dir[1] * B.G.sx + dir[2] * B.G.sxy;  // +1 layer outward
  const int64_t n = B.G.at(i, j, k);
  double *bv = B.bv, *sv = B.sv, *cv = B.cv;
  if (f.type == 6) {  // apply_outflow
    double b[6], s[NSC1], mut_n = 0;
    OSTC_UNROLL for (int l = 0; l < 6; ++l) b[l] = bv[l * sz + n];
    OSTC_UNROLL for (int l = 0; l < NSC; ++l) s[l] = sv[l * sz + n];
    if constexpr (C::turb) mut_n = B.mut[n];
    for (int g = 1; g <= ngg; ++g) {
      const int64_t gn = n + g * step;
      OSTC_UNROLL for (int l = 0; l < 6; ++l) bv[l * sz + gn] = b[l];
      OSTC_UNROLL for (int l = 0; l < NSC; ++l) sv[l * sz + gn] = s[l];
      if constexpr (C::turb) B.mut[gn] = mut_n;
    }
  } else if (f.type == 5) {  // apply_inflow
    for (int g = 1; g <= ngg; ++g) {
      const int64_t gn = n + g * step;
      bv[gn] = f.density;
      bv[sz + gn] = f.u;
      bv[2 * sz + gn] = f.v;
      bv[3 * sz + gn] = f.w;
      bv[4 * sz + gn] = f.pressure;
      bv[5 * sz + gn] = f.temperature;
      for (int l = 0; l < NSC; ++l) sv[l * sz + gn] = f.sv[l];
      if constexpr (C::turb) B.mut[gn] = f.mut;
    }
  } else if (f.type == 3) {  // apply_symmetry
    const int64_t in = n - step;
    const double *mr = B.metric + 3 * f.face * sz;
    double k_x = mr[n], k_y = mr[sz + n], k_z = mr[2 * sz + n];
    double bi[6], si[NSC1];
    OSTC_UNROLL for (int l = 0; l < 6; ++l) bi[l] = bv[l * sz + in];
    OSTC_UNROLL for (int l = 0; l < NSC; ++l) si[l] = sv[l * sz + in];
    const double e_in = cv[4 * sz + in];
    const double k_magnitude = sqrt(k_x * k_x + k_y * k_y + k_z * k_z);
    k_x /= k_magnitude;
    k_y /= k_magnitude;
    k_z /= k_magnitude;
    const double u1 = bi[1], v1 = bi[2], w1 = bi[3];
    double u_k = k_x * u1 + k_y * v1 + k_z * w1;
    const double u_t = u1 - k_x * u_k, v_t = v1 - k_y * u_k, w_t = w1 - k_z * u_k;
    const double rho = bi[0];  // the face takes the interior density
    bv[sz + n] = u_t;
    bv[2 * sz + n] = v_t;
    bv[3 * sz + n] = w_t;
    B.vel[n] = sqrt(u_t * u_t + v_t * v_t + w_t * w_t);
    bv[n] = rho;
    bv[4 * sz + n] = bi[4];
    bv[5 * sz + n] = bi[5];
    OSTC_UNROLL for (int l = 0; l < NSC; ++l) sv[l * sz + n] = si[l];
    cv[n] = rho;
    cv[sz + n] = rho * u_t;
    cv[2 * sz + n] = rho * v_t;
    cv[3 * sz + n] = rho * w_t;
    cv[4 * sz + n] = e_in - 0.5 * rho * (u1 * u1 + v1 * v1 + w1 * w1) + 0.5 * rho * (u_t * u_t + v_t * v_t + w_t * w_t);
    OSTC_UNROLL for (int l = 0; l < NSC; ++l) cv[(5 + l) * sz + n] = rho * si[l];
    for (int g = 1; g <= ngg; ++g) {
      const int64_t gn = n + g * step, ig = n - g * step;
      double bg[6], sg[NSC1], mut_g = 0;
      OSTC_UNROLL for (int l = 0; l < 6; ++l) bg[l] = bv[l * sz + ig];
      OSTC_UNROLL for (int l = 0; l < NSC; ++l) sg[l] = sv[l * sz + ig];
      if constexpr (C::turb) mut_g = B.mut[ig];
      const double u = bg[1], v = bg[2], w = bg[3];
      u_k = k_x * u + k_y * v + k_z * w;
      const double ug = u - 2 * u_k * k_x, vg = v - 2 * u_k * k_y, wg = w - 2 * u_k * k_z;
      bv[gn] = bg[0];
      bv[sz + gn] = ug;
      bv[2 * sz + gn] = vg;
      bv[3 * sz + gn] = wg;
      B.vel[gn] = sqrt(ug * ug + vg * vg + wg * wg);
      bv[4 * sz + gn] = bg[4];
      bv[5 * sz + gn] = bg[5];
      OSTC_UNROLL for (int l = 0; l < NSC; ++l) sv[l * sz + gn] = sg[l];
      if constexpr (C::turb) B.mut[gn] = mut_g;
    }
  } else if (f.type == 2) {  // apply_wall
    const int64_t in = n - step;
    const double t_in = bv[5 * sz + in], p = bv[4 * sz + in];
    double s_in[NSC1];
    OSTC_UNROLL for (int l = 0; l < NSC; ++l) s_in[l] = sv[l * sz + in];
    double dy = 0;
    if constexpr (C::turb) dy = B.wall_dist[in];
    double t_wall = f.t_wall;
    if (!f.isothermal) t_wall = t_in;
    double mw = kDMwAir;
    if constexpr (C::mix != 0) {
      mw = 0;
      OSTC_UNROLL for (int l = 0; l < NS; ++l) mw += s_in[l] / cP.mw[l];
      mw = 1 / mw;
    }
    const double rho_wall = p * mw / (t_wall * kDR_u);
    double rho_y[NS1];
    OSTC_UNROLL for (int l = 0; l < NS; ++l) rho_y[l] = s_in[l] * rho_wall;
    double speed;
    const double e_wall = total_energy_of<C>(rho_wall, 0.0, 0.0, 0.0, p, t_wall, rho_y, speed);
    double omega = 0;
    if constexpr (C::turb) {
      double mu_wall;
      if constexpr (C::mix != 0)
        mu_wall = mixture_viscosity<NS>(t_wall, mw, s_in);
      else
        mu_wall = sutherland(t_wall);
      omega = dy > 1e-25 ? 60 * mu_wall / (rho_wall * sst::beta_1 * dy * dy) : s_in[NS + 1];
    }
    OSTC_UNROLL for (int l = 0; l < NS; ++l) sv[l * sz + n] = s_in[l];
    bv[n] = rho_wall;
    bv[sz + n] = 0;
    bv[2 * sz + n] = 0;
    bv[3 * sz + n] = 0;
    bv[4 * sz + n] = p;
    bv[5 * sz + n] = t_wall;
    cv[n] = rho_wall;
    cv[sz + n] = 0;
    cv[2 * sz + n] = 0;
    cv[3 * sz + n] = 0;
    OSTC_UNROLL for (int l = 0; l < NS; ++l) cv[(l + 5) * sz + n] = rho_y[l];
    cv[4 * sz + n] = e_wall;
    B.vel[n] = speed;
    if constexpr (C::turb) {
      sv[NS * sz + n] = 0;
      cv[(NS + 5) * sz + n] = 0;
      sv[(NS + 1) * sz + n] = omega;
      cv[(NS + 6) * sz + n] = rho_wall * omega;
    }
    for (int g = 1; g <= ngg; ++g) {
      const int64_t ig = n - g * step, gn = n + g * step;
      const double u_i = bv[sz + ig], v_i = bv[2 * sz + ig], w_i = bv[3 * sz + ig];
      const double p_i = bv[4 * sz + ig], t_i = bv[5 * sz + ig];
      double y_i[NS1];
      OSTC_UNROLL for (int l = 0; l < NS; ++l) y_i[l] = sv[l * sz + ig];
      double t_g = t_i;
      if (f.isothermal) {
        t_g = 2 * t_wall - t_i;
        if (t_g <= 0.1 * t_wall) t_g = t_wall;
      }
      if constexpr (C::mix != 0) {
        mw = 0;
        OSTC_UNROLL for (int l = 0; l < NS; ++l) mw += y_i[l] / cP.mw[l];
        mw = 1 / mw;
      }
      const double rho_g = p_i * mw / (t_g * kDR_u);
      OSTC_UNROLL for (int l = 0; l < NS; ++l) sv[l * sz + gn] = y_i[l];
      bv[gn] = rho_g;
      bv[sz + gn] = -u_i;
      bv[2 * sz + gn] = -v_i;
      bv[3 * sz + gn] = -w_i;
      bv[4 * sz + gn] = p_i;
      bv[5 * sz + gn] = t_g;
      if constexpr (C::turb) {
        sv[NS * sz + gn] = 0;
        sv[(NS + 1) * sz + gn] = omega;
        B.mut[gn] = 0;
      }
    }
  }
}

// ---------------------------------------------------------------- block faces
// inner_communication, src/DataCommunication.cuh:58-98: average Q on the
// shared face and copy the neighbour's interior into the ghost layers.
struct DevInner {
  int block, target_block, face, direction;
  int start[3], end[3], loop_dir[3], tstart[3], tloop_dir[3], src_tar[3], n_point[3];
};

// exact: the shared plane is computed identically by both blocks and is not
// re-averaged, and the ghost copy also covers the face's tangential ghost
// rows (tg = ngg), which the viscous stencils read next to the face
template <class C>
__global__ void k_inner(const DevBlock *__restrict__ blks, const DevInner *__restrict__ faces, int fi, bool exact,
                        int tg) {
  const DevInner &f = faces[fi];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  int ext[3];
  for (int q = 0; q < 3; ++q) ext[q] = f.n_point[q] + (q != f.face && f.n_point[q] > 1 ? 2 * tg : 0);
  const int np = ext[0] * ext[1] * ext[2];
  if (t >= np) return;
  int nn[3] = {t % ext[0], (t / ext[0]) % ext[1], t / (ext[0] * ext[1])};
  for (int q = 0; q < 3; ++q)
    if (ext[q] != f.n_point[q]) nn[q] -= tg;
  int idx[3], it[3], d[3];
  for (int q = 0; q < 3; ++q) {
    d[q] = f.loop_dir[q] * nn[q];
    idx[q] = f.start[q] + d[q];
  }
  for (int q = 0; q < 3; ++q) it[q] = f.tstart[q] + f.tloop_dir[q] * d[f.src_tar[q]];
  const DevBlock &B = blks[f.block];
  const DevBlock &Tb = blks[f.target_block];
  const int64_t n = B.G.at(idx[0], idx[1], idx[2]), tn = Tb.G.at(it[0], it[1], it[2]);
  const int64_t sz = B.G.size, tsz = Tb.G.size;
  const int face_dir = f.direction > 0 ? f.start[f.face] : f.end[f.face];
  if (idx[f.face] == face_dir) {
    if (exact) return;
    OSTC_UNROLL for (int l = 0; l < C::nv; ++l) {
      const double ave = 0.5 * (Tb.cv[l * tsz + tn] + B.cv[l * sz + n]);
      B.cv[l * sz + n] = ave;
      Tb.cv[l * tsz + tn] = ave;
    }
    primitives_from_q<C>(B, n);
  } else {
    for (int l = 0; l < 6; ++l) B.bv[l * sz + n] = Tb.bv[l * tsz + tn];
    OSTC_UNROLL for (int l = 0; l < C::nsc; ++l) B.sv[l * sz + n] = Tb.sv[l * tsz + tn];
  }
}

// Exact inner faces: the first ghost layer of an array that the stencils
// read across the face, copied from the neighbour's interior (the point map
// of k_inner).  set: 0 mu_t and lambda_t, 1 |V|, 2 the inviscid spectral
// radii, 3 the DPLUR increments of buffer dq_sel (0 dq, 1 dq0, 2 dqk), 4 the
// species enthalpies of the sweeps.
enum HaloSet { kHaloTurb = 0, kHaloVel = 1, kHaloSpec = 2, kHaloDq = 3, kHaloHspec = 4 };

template <class C>
__global__ void k_halo(const DevBlock *__restrict__ blks, const DevInner *__restrict__ faces, int fi, int set,
                       int dq_sel) {
  const DevInner &f = faces[fi];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int np = f.n_point[0] * f.n_point[1] * f.n_point[2];
  if (t >= np) return;
  const int nn[3] = {t % f.n_point[0], (t / f.n_point[0]) % f.n_point[1], t / (f.n_point[0] * f.n_point[1])};
  int idx[3], it[3], d[3];
  for (int q = 0; q < 3; ++q) {
    d[q] = f.loop_dir[q] * nn[q];
    idx[q] = f.start[q] + d[q];
  }
  for (int q = 0; q < 3; ++q) it[q] = f.tstart[q] + f.tloop_dir[q] * d[f.src_tar[q]];
  const int face_dir = f.direction > 0 ? f.start[f.face] : f.end[f.face];
  if (abs(idx[f.face] - face_dir) != 1) return;
  const DevBlock &B = blks[f.block];
  const DevBlock &Tb = blks[f.target_block];
  if (set == kHaloTurb || set == kHaloVel) {
    const int64_t n = B.G.at(idx[0], idx[1], idx[2]), tn = Tb.G.at(it[0], it[1], it[2]);
    if (set == kHaloVel) {
      B.vel[n] = Tb.vel[tn];
    } else if constexpr (C::turb) {
      B.mut[n] = Tb.mut[tn];
      B.turb_cond[n] = Tb.turb_cond[tn];
    }
    return;
  }
  const int64_t n = B.D.at(idx[0], idx[1], idx[2]), tn = Tb.D.at(it[0], it[1], it[2]);
  const int64_t sz = B.D.size, tsz = Tb.D.size;
  if (set == kHaloSpec) {
    for (int l = 0; l < 3; ++l) B.inv_spec[l * sz + n] = Tb.inv_spec[l * tsz + tn];
  } else if (set == kHaloDq) {
    double *dst = dq_sel == 0 ? B.dq : (dq_sel == 1 ? B.dq0 : B.dqk);
    const double *src = dq_sel == 0 ? Tb.dq : (dq_sel == 1 ? Tb.dq0 : Tb.dqk);
    OSTC_UNROLL for (int l = 0; l < C::nv; ++l) dst[l * sz + n] = src[l * tsz + tn];
  } else if (set == kHaloHspec) {
    if constexpr (C::ns > 0)
      OSTC_UNROLL for (int l = 0; l < C::ns; ++l) B.h_spec[l * sz + n] = Tb.h_spec[l * tsz + tn];
  }
}

// eliminate_k_gradient, src/FieldOperation.cu:42-62 (2-D cases)
template <class C>
__global__ void k_kcopy(const DevBlock *__restrict__ blks, int b) {
  const DevBlock &B = blks[b];
  const int g = B.ngg;
  const int ex = B.mx + 2 * g, ey = B.my + 2 * g;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ex * ey) return;
  const int i = t % ex - g, j = t / ex - g;
  const int64_t sz = B.G.size, n0 = B.G.at(i, j, 0);
  // the plane's values read once, before the stores
  double pb[6], ps[C::nsc > 0 ? C::nsc : 1];
  OSTC_UNROLL for (int l = 0; l < 6; ++l) pb[l] = B.bv[l * sz + n0];
  OSTC_UNROLL for (int l = 0; l < C::nsc; ++l) ps[l] = B.sv[l * sz + n0];
  for (int k = 1; k <= g; ++k) {
    const int64_t np = n0 + k * B.G.sxy, nm = n0 - k * B.G.sxy;
    OSTC_UNROLL for (int l = 0; l < 6; ++l) {
      B.bv[l * sz + np] = pb[l];
      B.bv[l * sz + nm] = pb[l];
    }
    OSTC_UNROLL for (int l = 0; l < C::nsc; ++l) {
      B.sv[l * sz + np] = ps[l];
      B.sv[l * sz + nm] = ps[l];
    }
  }
}

// ---------------------------------------------------------------- residual
// store_last_step, src/TimeAdvanceFunc.cu:5-16
static __global__ void __launch_bounds__(kCta) k_store_last(const DevBlock *__restrict__ blks, Tiles T) {
  int b, i, j, k;
  if (!tile_cell<kTX, kTY, kTZ>(T, b, i, j, k, blks)) return;
  const DevBlock &B = blks[b];
  const int64_t n = B.G.at(i, j, k), nz = B.Z.at(i, j, k), sz = B.G.size, sz0 = B.Z.size;
  B.bv_last[nz] = B.bv[n];
  B.bv_last[sz0 + nz] = B.vel[n];
  B.bv_last[2 * sz0 + nz] = B.bv[4 * sz + n];
  B.bv_last[3 * sz0 + nz] = B.bv[5 * sz + n];
}

// compute_square_of_dbv + per-CTA partial sums (src/TimeAdvanceFunc.cu:18-32,
// src/Driver.cu:418-459).  Partials are combined in a fixed order by
// k_res_final, so the residual is reproducible run to run.
static __global__ void __launch_bounds__(kCta) k_res_partial(const DevBlock *__restrict__ blks, Tiles T, double *partial) {
  __shared__ double red[4][kCta / 32];
  int b, i, j, k;
  double s[4] = {0, 0, 0, 0};
  if (tile_cell<kTX, kTY, kTZ>(T, b, i, j, k, blks)) {
    const DevBlock &B = blks[b];
    const int64_t n = B.G.at(i, j, k), nz = B.Z.at(i, j, k), sz = B.G.size, sz0 = B.Z.size;
    const double cur[4] = {B.bv[n], B.vel[n], B.bv[4 * sz + n], B.bv[5 * sz + n]};
    for (int l = 0; l < 4; ++l) {
      const double d = cur[l] - B.bv_last[l * sz0 + nz];
      s[l] = d * d;
    }
  }
  const int tid = threadIdx.x + kTX * (threadIdx.y + kTY * threadIdx.z);
  for (int l = 0; l < 4; ++l) {
    double v = s[l];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((tid & 31) == 0) red[l][tid >> 5] = v;
  }
  __syncthreads();
  if (tid < 4) {
    double v = 0;
    for (int w = 0; w < kCta / 32; ++w) v += red[tid][w];
    // stored in block order, so that the reduction's order and result do
    // not depend on the schedule of the blocks
    int bb = 0;
    const int slot = tile_of(T, blockIdx.x, bb) + T.cbegin[bb];
    partial[static_cast<int64_t>(slot) * 4 + tid] = v;
  }
}

static __global__ void k_res_final(const double *partial, int n_part, double *out) {
  __shared__ double red[4][32];
  const int tid = threadIdx.x;  // 128 threads: 4 variables x 32 lanes
  const int l = tid >> 5, lane = tid & 31;
  double v = 0;
  for (int q = lane; q < n_part; q += 32) v += partial[static_cast<int64_t>(q) * 4 + l];
  red[l][lane] = v;
  __syncthreads();
  if (lane == 0) {
    double s = 0;
    for (int q = 0; q < 32; ++q) s += red[l][q];
    out[l] = s;
  }
}

// ---------------------------------------------------------------- initialisation
// compute_cv_from_bv, src/FieldOperation.cuh:37-73 (launched with halo ngg)
template <class C>
__global__ void __launch_bounds__(kCta) k_cv_from_bv(const DevBlock *__restrict__ blks, Tiles T) {
  int b, i, j, k;
  if (!tile_cell<kTX, kTY, kTZ>(T, b, i, j, k, blks)) return;
  const DevBlock &B = blks[b];
  const int64_t n = B.G.at(i, j, k), sz = B.G.size;
  const double rho = B.bv[n];
  B.cv[n] = rho;
  B.cv[sz + n] = rho * B.bv[sz + n];
  B.cv[2 * sz + n] = rho * B.bv[2 * sz + n];
  B.cv[3 * sz + n] = rho * B.bv[3 * sz + n];
  OSTC_UNROLL for (int l = 0; l < C::nsc; ++l) B.cv[(5 + l) * sz + n] = rho * B.sv[l * sz + n];
  total_energy<C>(B, n);
}

// initialize_mut, src/FieldOperation.cuh:111-137 (launched with halo 1)
template <class C>
__global__ void __launch_bounds__(kCta) k_init_mut(const DevBlock *__restrict__ blks, Tiles T) {
  constexpr int NS = C::ns;
  int b, i, j, k;
  if (!tile_cell<kTX, kTY, kTZ>(T, b, i, j, k, blks)) return;
  const DevBlock &B = blks[b];
  const int64_t n = B.G.at(i, j, k), sz = B.G.size;
  const double t = B.bv[5 * sz + n];
  double mul = sutherland(t);
  if constexpr (C::mix != 0) {
    double mw = 0, Y[NS];
    OSTC_UNROLL for (int l = 0; l < NS; ++l) {
      Y[l] = B.sv[l * sz + n];
      mw += Y[l] / cP.mw[l];
    }
    mw = 1 / mw;
    mul = mixture_viscosity<NS>(t, mw, Y);
  }
  B.mut[n] = sst_mut<C>(B, n, mul);
}

// compute_wall_distance, src/Driver.cu:461-482 (brute force; halo ngg)
// Squared distance to wall point w: the one expression both searches use, so
// that they find the same minimum to the last bit.
__device__ __forceinline__ double wall_d2(double x, double y, double z, const double *w) {
  return (x - w[0]) * (x - w[0]) + (y - w[1]) * (y - w[1]) + (z - w[2]) * (z - w[2]);
}

// compute_wall_distance, src/Driver.cu:461-482: the square root of the least
// squared distance to every wall point, capped at 1e6 as in the reference.
static __global__ void __launch_bounds__(kCta) k_wall_distance(const DevBlock *__restrict__ blks, Tiles T,
                                                        const double *__restrict__ wall, int n_wall) {
  int b, i, j, k;
  if (!tile_cell<kTX, kTY, kTZ>(T, b, i, j, k, blks)) return;
  const DevBlock &B = blks[b];
  const int64_t n = B.G.at(i, j, k);
  const double x = B.x[n], y = B.y[n], z = B.z[n];
  double wd = 1e+6;
  for (int l = 0; l < n_wall; ++l) {
    const double d = wall_d2(x, y, z, wall + 3 * l);
    if (wd > d) wd = d;
  }
  B.wall_dist[n] = sqrt(wd);
}

// The wall points sorted into a uniform grid of buckets of edge h over their
// bounding box [lo, hi] (start: first point of each bucket, CSR; pts: x, y, z
// of the points in bucket order).
struct WallGrid {
  double lo[3], hi[3], h;
  int n[3];
  const int *start;
  const double *pts;
};

// The same distance by an exact search of the bucket grid: the buckets in
// shells of growing Chebyshev index distance s around the point's own bucket
// (clamped to the grid), stopping before shell s once the best squared
// distance cannot exceed the least squared distance of any point in it.  A
// bucket of shell s is s buckets away along some axis a that still has
// buckets there, so its points are at least max((s - 1) h, out_a) away along
// a and at least out_d along every other axis d, out_d being the point's
// distance outside the points' bounding box along d (for a flat wall this
// counts the height above it, so a point far from the wall stops after a few
// shells).  The minimum found is the brute force's minimum: same points where
// it matters, same expression (wall_d2).
static __global__ void __launch_bounds__(kCta) k_wall_distance_grid(const DevBlock *__restrict__ blks, Tiles T,
                                                             WallGrid G) {
  int b, i, j, k;
  if (!tile_cell<kTX, kTY, kTZ>(T, b, i, j, k, blks)) return;
  const DevBlock &B = blks[b];
  const int64_t n = B.G.at(i, j, k);
  const double p[3] = {B.x[n], B.y[n], B.z[n]};
  int c[3];
  double out2[3];
  for (int d = 0; d < 3; ++d) {
    const double f = floor((p[d] - G.lo[d]) / G.h);
    c[d] = f < 0 ? 0 : (f >= G.n[d] ? G.n[d] - 1 : static_cast<int>(f));
    const double o = p[d] < G.lo[d] ? G.lo[d] - p[d] : (p[d] > G.hi[d] ? p[d] - G.hi[d] : 0.0);
    out2[d] = o * o;
  }
  const int smax = max(G.n[0], max(G.n[1], G.n[2]));
  double wd = 1e+6;
  for (int s = 0; s <= smax; ++s) {
    if (s >= 1) {
      double bound = -1;  // least squared distance of a point in shell s (none: -1)
      for (int a = 0; a < 3; ++a) {
        if (c[a] + s >= G.n[a] && c[a] - s < 0) continue;
        const double g = (s - 1) * G.h;
        double lb = fmax(g * g, out2[a]);
        for (int d = 0; d < 3; ++d)
          if (d != a) lb += out2[d];
        bound = bound < 0 ? lb : fmin(bound, lb);
      }
      if (bound < 0 || wd <= bound * (1 - 1e-12)) break;
    }
    for (int dz = -s; dz <= s; ++dz) {
      const int z = c[2] + dz;
      if (z < 0 || z >= G.n[2]) continue;
      for (int dy = -s; dy <= s; ++dy) {
        const int y = c[1] + dy;
        if (y < 0 || y >= G.n[1]) continue;
        const bool face = abs(dz) == s || abs(dy) == s;
        for (int dx = -s; dx <= s; dx += (face ? 1 : 2 * max(s, 1))) {
          const int x = c[0] + dx;
          if (x < 0 || x >= G.n[0]) continue;
          const int bk = (z * G.n[1] + y) * G.n[0] + x;
          for (int q = G.start[bk]; q < G.start[bk + 1]; ++q) {
            const double d = wall_d2(p[0], p[1], p[2], G.pts + 3 * q);
            if (wd > d) wd = d;
          }
        }
      }
    }
  }
  B.wall_dist[n] = sqrt(wd);
}

// wall_friction_heatFlux_2d, src/PostProcess.cu:50-73: skin friction and
// wall heat flux along the j = 0 wall of a 2-D block, at the cells i of the
// k = 0 plane: cf = mu du_par/dn / q_inf, q_w = lambda dT/dn with the wall
// normal derivative one-sided over the first cell (|grad eta| spacing).
static __global__ void __launch_bounds__(128) k_wall_2d(const DevBlock *__restrict__ blks, int b, double *cf,
                                                       double *qw, double dyn_pressure) {
  const DevBlock &B = blks[b];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B.mx) return;
  const int64_t sz = B.G.size, n0 = B.G.at(i, 0, 0), n1 = B.G.at(i, 1, 0);
  const double *m = B.metric;
  const double xi_x = m[n0], xi_y = m[sz + n0];
  const double eta_x = m[3 * sz + n0], eta_y = m[4 * sz + n0];
  const double viscosity = B.mul[n0];
  const double u_parallel_wall = (xi_x * B.bv[sz + n1] + xi_y * B.bv[2 * sz + n1]) / sqrt(xi_x * xi_x + xi_y * xi_y);
  const double grad_eta = sqrt(eta_x * eta_x + eta_y * eta_y);
  const double du_normal_wall = u_parallel_wall * grad_eta;
  cf[i] = viscosity * du_normal_wall / dyn_pressure;
  const double conductivity = B.cond[n0];
  qw[i] = conductivity * (B.bv[5 * sz + n1] - B.bv[5 * sz + n0]) * grad_eta;
}

}  // namespace ostc
