/*
 * C ABI of the B200-native OpenSTC step engine (libopenstc_b200.so).
 *
 * The reference has no FFI: its boundary is the C++ class template
 * cfd::Driver<MixtureModel, TurbMethod> (src/Driver.cuh:12-46) driven by
 * main (src/main.cu:7-68).  These entry points are what a binding of that
 * boundary needs: open a case directory laid out like the reference's
 * (input_files/...), initialise, step, read and write fields, write the
 * Tecplot file.  Plain pointers and sizes only.  Every function returns 0 on
 * success or a negative ostc_status; ostc_last_error() describes the failure.
 *
 * Array layout for every field: the reference's column-major layout with
 * ghost layers (src/gxl_lib/Array.hpp:71-130),
 *   idx(i,j,k) = k*(mx+2g)*(my+2g) + j*(mx+2g) + i + ((mx+2g)*(my+2g)+(mx+2g)+1)*g,
 * components of a vector field stacked with the stride of one component.
 * g is the field's ghost count (ostc_field_layout).  The metric is nine
 * components (xi_x, xi_y, xi_z, eta_x, ..., zeta_z) and the inviscid
 * spectral radius three, both in this stacked form.
 */
#ifndef OPENSTC_B200_H
#define OPENSTC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ostc_driver ostc_driver;

typedef enum ostc_status {
  OSTC_OK = 0,
  OSTC_ERR_INPUT = -1,     /* bad argument, missing or malformed case file */
  OSTC_ERR_CUDA = -2,      /* CUDA runtime error */
  OSTC_ERR_STATE = -3,     /* call out of order (e.g. step before initialize) */
  OSTC_ERR_NAN = -4,       /* NaN residual: the reference aborts here (src/Driver.cu:372-377) */
  OSTC_ERR_INTERNAL = -5
} ostc_status;

/* Field identifiers (the DZone members of src/Field.h:13-57). */
typedef enum ostc_field_id {
  OSTC_X = 0, OSTC_Y, OSTC_Z, OSTC_JAC, OSTC_METRIC, OSTC_WALL_DIST,
  OSTC_BV, OSTC_SV, OSTC_CV, OSTC_VEL, OSTC_ACOUSTIC, OSTC_MACH, OSTC_MUL, OSTC_CONDUCTIVITY,
  OSTC_RHO_D, OSTC_GAMMA, OSTC_CP, OSTC_MUT, OSTC_TURB_COND, OSTC_CHEM_JAC, OSTC_TURB_SRC_JAC,
  OSTC_DQ, OSTC_DQ0, OSTC_DQK, OSTC_INV_SPEC, OSTC_VISC_SPEC, OSTC_DT_LOCAL, OSTC_BV_LAST,
  OSTC_N_FIELDS
} ostc_field_id;

/* Step phases for per-kernel parity checks (see ostc_driver_run_phase). */
typedef enum ostc_phase {
  OSTC_PHASE_RESIDUAL = 0, /* dq = source + inviscid + viscous; local dt (src/Driver.cu:234-243) */
  OSTC_PHASE_IMPLICIT = 1, /* point-implicit / DPLUR (src/ImplicitTreatmentHPP.cuh:10-59) */
  OSTC_PHASE_UPDATE = 2,   /* update_cv_and_bv + limit_flow (src/Driver.cu:248-251) */
  OSTC_PHASE_BC = 3,       /* boundary conditions (src/BoundCond.cuh:321-412) */
  OSTC_PHASE_EXCHANGE = 4, /* inner faces, 2-D k copy, properties (src/Driver.cu:257-272) */
  OSTC_PHASE_STORE = 5,    /* store_last_step (src/TimeAdvanceFunc.cu:5-16) */
  OSTC_PHASE_SOURCE = 6,   /* first half of RESIDUAL: dq = source terms (src/SourceTerm.cuh:12-40) */
  OSTC_PHASE_FLUX = 7,     /* second half of RESIDUAL: inviscid + viscous fluxes, local dt
                              (src/SchemeSelector.cuh:38-280, src/TimeAdvanceFunc.cuh:21-71) */
  OSTC_PHASE_CHEMISTRY = 8 /* one chemistry step on its own: the surrogate's dY where the gate
                              accepts, one EPI step elsewhere, applied to rho Y (needs
                              ostc_driver_set_surrogate; not part of the step) */
} ostc_phase;

typedef struct ostc_options {
  int device;    /* CUDA device ordinal */
  int quiet;     /* suppress the reference's screen output */
  int precision; /* 0: FP64, the reference's arithmetic; 1: FP32 fluxes, limiter, SST,
                    flux Jacobians and transport, FP64 state, update, temperature
                    inversion, chemistry, point-implicit solve and residual (finite-rate
                    SST cases only) */
  int exact_inner; /* 0: inner faces as the reference treats them
                      (src/DataCommunication.cuh:58-98: the shared plane averaged,
                      bv / sv ghosts copied from the neighbour, the DPLUR sweeps
                      treating the face as a boundary).  1 (FP64 path, 3-D, faces
                      that cover whole block faces): a multi-block grid computes what
                      the same grid as one block computes, bit for bit: every array a
                      stencil reads across the face (the ghost rows next to the face,
                      mu_t, lambda_t, |V|, the spectral radii, the species enthalpies,
                      the DPLUR increments of each sweep) is copied from the
                      neighbour, the sweeps take the neighbours across the face, and
                      the shared plane, computed identically on both sides, is not
                      re-averaged.  No counterpart in the reference. */
  int wall_distance; /* the wall distance of SST cases: 0 automatic (bucket search
                        above 2048 wall points), 1 the reference's brute force over
                        every wall point (src/Driver.cu:461-482), 2 an exact search of
                        a uniform bucket grid of the wall points (the same values) */
} ostc_options;

typedef struct ostc_info {
  int n_block, ngg, dimension;
  int n_spec, n_reac, n_var, n_scalar;
  int mix;       /* 0 air, 1 mixture, 2 finite-rate chemistry */
  int rans;      /* 1 if k-omega SST */
  int implicit_method, dplur_inner_step, chem_src_method;
  int step;      /* current step number */
  int64_t n_grid_total;
  int n_bc, n_inner;
} ostc_info;

/* Model constants and mechanism tables as the engine sees them (the
   reference's DParameter, src/DParameter.h:11-58).  Arrays are row-major:
   [species][7] for NASA-7 coefficients, [reaction][species] for
   stoichiometry and third-body efficiencies. */
#define OSTC_MAX_SPEC 20
#define OSTC_MAX_REAC 50
typedef struct ostc_params {
  int ns, nr, n_var, n_scalar;
  int mix, turb, rans_model, turb_implicit, chem_src_method, implicit_method, dplur_inner_step;
  int reconstruction, limiter, viscous_order, dim, output_screen;
  double cfl, Pr, Prt, Sct, Sc;
  double ll[7], ul[7];
  double sv_inf[OSTC_MAX_SPEC + 2];
  double mw[OSTC_MAX_SPEC], t_low[OSTC_MAX_SPEC], t_mid[OSTC_MAX_SPEC];
  double low_coeff[OSTC_MAX_SPEC * 7], high_coeff[OSTC_MAX_SPEC * 7];
  double lj_inv[OSTC_MAX_SPEC], vis_coeff[OSTC_MAX_SPEC];
  double w_quarter[OSTC_MAX_SPEC * OSTC_MAX_SPEC], w_sqrt8[OSTC_MAX_SPEC * OSTC_MAX_SPEC];
  int label[OSTC_MAX_REAC], order[OSTC_MAX_REAC];
  int stoi_f[OSTC_MAX_REAC * OSTC_MAX_SPEC], stoi_b[OSTC_MAX_REAC * OSTC_MAX_SPEC];
  double A[OSTC_MAX_REAC], b[OSTC_MAX_REAC], Ea[OSTC_MAX_REAC];
  double A2[OSTC_MAX_REAC], b2[OSTC_MAX_REAC], Ea2[OSTC_MAX_REAC];
  double third_body[OSTC_MAX_REAC * OSTC_MAX_SPEC];
  double troe_alpha[OSTC_MAX_REAC], troe_t3[OSTC_MAX_REAC], troe_t1[OSTC_MAX_REAC], troe_t2[OSTC_MAX_REAC];
} ostc_params;

/* One boundary face in application order (outflow 6, inflow 5, symmetry 3,
   wall 2), ranges after registration and wall trimming
   (src/Mesh.cpp:18-35, src/BoundCond.cu:215-229). */
typedef struct ostc_bc {
  int block, type, face, direction;
  int start[3], end[3];
  double density, u, v, w, pressure, temperature, mut;
  double sv[OSTC_MAX_SPEC + 2];
  int isothermal;
  double t_wall;
} ostc_bc;

/* One block-to-block face after registration (src/Mesh.cpp:47-177). */
typedef struct ostc_inner {
  int block, target_block, face, direction;
  int start[3], end[3], loop_dir[3], tstart[3], tloop_dir[3], src_tar[3], n_point[3];
} ostc_inner;

/* Reads <case_dir>/input_files (setup, grid, boundary, chemistry), builds the
   ghost geometry and metric and the initial field (fresh start or restart
   from output/field/flowfield.plt).  Host only; replaces src/main.cu:7-28 and
   the constructor Driver(Parameter&, Mesh&) (src/Driver.cu:14-40). */
int ostc_driver_create(const char *case_dir, const ostc_options *opt, ostc_driver **out);
void ostc_driver_destroy(ostc_driver *d);
const char *ostc_last_error(void);

int ostc_driver_info(const ostc_driver *d, ostc_info *info);
int ostc_driver_params(const ostc_driver *d, ostc_params *params);
int ostc_driver_bc(const ostc_driver *d, int index, ostc_bc *bc);
int ostc_driver_inner(const ostc_driver *d, int index, ostc_inner *face);
/* Block dimensions mx, my, mz. */
int ostc_driver_block_dims(const ostc_driver *d, int block, int dims[3]);
/* Ghost layers and component count of a field in this configuration
   (components 0 = not allocated). */
int ostc_field_layout(const ostc_driver *d, int field, int *ghost, int *components);

/* Host copies made while reading the case, before initialisation:
   OSTC_X/Y/Z, OSTC_JAC, OSTC_METRIC, OSTC_BV, OSTC_SV. */
int ostc_driver_get_host_field(const ostc_driver *d, int block, int field, double *out, int64_t count);

/* Driver::initialize_computation (src/Driver.cu:44-104) on the GPU. */
int ostc_driver_initialize(ostc_driver *d);
/* Driver::simulate (src/Driver.cu:107-120, 192-289): the steady loop with
   history.dat, residual_scale.txt, step.txt and flowfield.plt output.  The
   .plt files are written by a host thread while the next steps run (the
   first output page-locks two staging copies of the output fields); the call
   returns once every file is written. */
int ostc_driver_simulate(ostc_driver *d);
/* n iterations of the steady loop body, no file output.  *err_max receives
   the last normalised residual (or -1 if none was due). */
int ostc_driver_step(ostc_driver *d, int n_steps, double *err_max);
/* No counterpart in the reference, whose loop keeps the state on the device:
   a host-driven stepping loop.  n_steps iterations of ostc_driver_step, each
   preceded by the upload of n_fields fields (ostc_field_id) of block `block`
   from host[k] (counts[k] doubles, the ostc_driver_get_field layout) and
   followed by their download into the same buffers, so that the host holds
   each step's result and supplies the next step's input.  The copies run in
   chunks of chunk_bytes (0: 16 MiB) on two copy streams of their own: the
   upload of a chunk waits only for the download of the same chunk, so one
   step's download and the next step's upload overlap.  Page-locked host
   buffers let the copies run asynchronously.  Only whole state fields
   (bv, sv, cv and the like); the geometry goes through
   ostc_driver_set_field.  *err_max as for ostc_driver_step. */
int ostc_driver_step_io(ostc_driver *d, int n_steps, int block, const int *fields, double *const *host,
                        const int64_t *counts, int n_fields, int64_t chunk_bytes, double *err_max);
/* Normalised residuals of rho, |V|, p, T from the last residual step. */
int ostc_driver_residual(const ostc_driver *d, double res[4]);
int ostc_driver_run_phase(ostc_driver *d, int phase);
/* Device field of a block (count = values of the field, see layout). */
int ostc_driver_get_field(ostc_driver *d, int block, int field, double *out, int64_t count);
int ostc_driver_set_field(ostc_driver *d, int block, int field, const double *in, int64_t count);
/* MPIIO::print_field (src/MPIIO.hpp:420-546) to an explicit path. */
int ostc_driver_write_plt(ostc_driver *d, const char *path);
/* Kernel launches of one step of the cached CUDA graph. */
int ostc_driver_launches_per_step(const ostc_driver *d, int store_last, int residual);
/* Device time of the last step that computed a residual, in ms. */
int ostc_driver_last_step_ms(const ostc_driver *d, double *ms);
/* Runs one step eagerly with an event after every kernel and writes one line
   "name launches total_ms" per kernel into buf.  Advances the solution
   without counting a step.  Returns the number of lines. */
int ostc_driver_profile_step(ostc_driver *d, char *buf, int buflen);
/* The CUDA stream the engine launches on (cudaStream_t). */
void *ostc_driver_stream(ostc_driver *d);

/* ---- chemistry surrogate (no counterpart in the reference) ----------------
   The reference integrates the stiff chemistry with the point-implicit (EPI)
   step only.  These entry points serve the learned replacement of that step. */

/* D (FP32, row-major, leading dimension ldd) = A * B^T with A (M x K) and B
   (N x K) BF16 row-major, on the tcgen05 tensor cores with FP32 accumulation.
   All pointers are device memory; err is a device int set to 1 if a
   tensor-core wait timed out.  splits > 1 writes `splits` partial results
   (split-K) one after another, each M x ldd.  K, lda, ldb multiples of 8. */
int ostc_tc_gemm_bf16(const void *A, int lda, const void *B, int ldb, float *D, int ldd, int M, int N, int K,
                      int splits, int *err, void *stream);

/* The learned replacement of one point-implicit (EPI) chemistry step,
   (T, p, Y_k, dt) -> dY_k, where the EPI step at fixed density is
   rho dY = (I - dt J)^-1 dt omega (src/ImplicitTreatmentHPP.cuh:14-35 with
   src/FiniteRateChem.cu:7-234).  MLP 12 -> 4 x 256 (GELU) -> 9, BF16 weights
   and activations on the tensor cores with FP32 accumulation, FP32 master
   weights, Adam. */
typedef struct ostc_surrogate ostc_surrogate;

/* Held-out statistics against the FP64 EPI labels.  rel = max_k |dY_k -
   dY_EPI,k| / max_k |dY_EPI,k| per sample, over samples with max |dY_EPI| > 1e-6
   (smaller increments change nothing the solver resolves). */
typedef struct ostc_surrogate_eval {
  double mean_rel, max_rel; /* over the rel_count samples the trust gate accepts whose EPI
                               increment reaches 1e-6; both 0 when rel_count is 0 */
  double mean_abs;          /* accepted: mean |dY - dY_EPI| */
  double max_defect;        /* accepted: element defect of the applied (projected) dY, max over elements of
                               |sum_k a_ek dY_k/W_k| / sum_k a_ek Y_k/W_k */
  double mean_defect;
  double median_rel_all;    /* every sample: median and 90th percentile of rel */
  double p90_rel_all;
  double gate_pass;         /* fraction of samples the trust gate accepts */
  long long count;
  long long nonfinite;      /* samples whose (rejected) prediction was not finite */
  long long rel_count;      /* accepted samples with max |dY_EPI| > 1e-6 */
} ostc_surrogate_eval;

/* Mechanism and device from the driver (9-species finite-rate case). */
int ostc_surrogate_create(const ostc_driver *d, unsigned long long seed, ostc_surrogate **out);
void ostc_surrogate_destroy(ostc_surrogate *s);
/* Number of floats of ostc_surrogate_get_params / _gradients: per layer the
   weight (out x in, padded to 16 inputs / 16 outputs) then the bias. */
int ostc_surrogate_param_count(void);
/* n samples: field_fraction of them from the cells of block 0 of `field`
   (perturbed; NULL: none), the rest uniform in T [250, 2800] K, log10 p
   [4.5, 6], log10 dt [-9, -6] with Dirichlet(1) mass fractions; labels from
   the FP64 EPI step; sets the feature/target normalisation. */
int ostc_surrogate_generate(ostc_surrogate *s, const ostc_driver *field, long long n, unsigned long long seed,
                            double field_fraction);
/* Adam steps on random batches of samples [0, n_train); losses[steps] may be NULL. */
int ostc_surrogate_train(ostc_surrogate *s, int steps, int batch, double lr, long long n_train, float *losses);
int ostc_surrogate_evaluate(ostc_surrogate *s, long long begin, long long count, ostc_surrogate_eval *out);
/* states: n x 12 host doubles (T [K], p [Pa], Y[9], dt [s]); dy: n x 9. */
int ostc_surrogate_label(ostc_surrogate *s, const double *states, long long n, double *dy);
int ostc_surrogate_predict(ostc_surrogate *s, const double *states, long long n, double *dy, int *accepted);
/* Mean-squared loss of the normalised targets of one batch (n multiple of
   128) and its gradients (ostc_surrogate_param_count floats). */
int ostc_surrogate_gradients(ostc_surrogate *s, const double *states, const double *dy, long long n, float *grads,
                             double *loss);
int ostc_surrogate_get_params(const ostc_surrogate *s, float *flat);
int ostc_surrogate_set_params(ostc_surrogate *s, const float *flat);
/* Features x_j = (f_j - in_mu_j) / in_sig_j of f = (T, log10 p, Y[9], log10 dt);
   network output o_k maps to dY_k = (Y_k + 1e-10) * out_c_k * sinh(out_scale_k * o_k). */
int ostc_surrogate_normalisation(const ostc_surrogate *s, float *in_mu, float *in_sig, float *out_c, float *out_scale);
/* The per-cell trust gate: inputs in the training box, |network output| <=
   out_max, element defect <= defect_tol of the element totals, |dY_k| <=
   rel_max (Y_k + max(y_floor, 1e-10)); other cells take the EPI fallback.
   Takes effect for drivers at their next ostc_driver_set_surrogate. */
typedef struct ostc_surrogate_gate {
  float t_min, t_max, lp_min, lp_max, ldt_min, ldt_max, defect_tol, rel_max, out_max, y_floor;
  /* the judge: every accepted increment must agree with the diagonal
     point-implicit increment (dt omega_k / rho) / (1 + dt omega_d,k / (rho Y_k))
     of the cell's own chemistry (the DA treatment) within judge_rel of it
     plus judge_abs (Y_k + y_floor); judge_rel < 0 turns it off */
  float judge_rel, judge_abs;
} ostc_surrogate_gate;
int ostc_surrogate_get_gate(const ostc_surrogate *s, ostc_surrogate_gate *g);
int ostc_surrogate_set_gate(ostc_surrogate *s, const ostc_surrogate_gate *g);
int ostc_surrogate_save(const ostc_surrogate *s, const char *path);
int ostc_surrogate_load(ostc_surrogate *s, const char *path);
/* Chemistry of the driver's steps through the surrogate.  Before the source
   term of every step the network evaluates each cell (with the cell's local
   time step); cells the trust gate accepts are chemically quiet and take the
   network's rate rho dY/dt as an explicit source with no chemistry Jacobian,
   every other cell keeps the reference's point-implicit (EPI) chemistry inside
   the coupled DPLUR step -- the fallback.  s = NULL returns to EPI everywhere.
   The surrogate must stay alive while set; its weights are read at each step. */
int ostc_driver_set_surrogate(ostc_driver *d, ostc_surrogate *s);
/* Since the surrogate was set: cell-steps whose chemistry the trust gate
   accepted, cell-steps that took the point-implicit fallback, and cell
   evaluations of the network (a rejected cell is evaluated again within a few
   steps, in between it keeps EPI; evaluated may be NULL). */
int ostc_driver_chemistry_stats(ostc_driver *d, long long *accepted, long long *fallback, long long *evaluated);

/* The launch tuning of the step (no counterpart in the reference, which
   launches each block separately with fixed 2-D thread blocks,
   src/Driver.cu:205-216).  schedule: the order in which the blocks of a
   multi-block grid share each launch (0 block order, 1 largest block first);
   flux_variant: on the FP32-bulk path the variant of the flux passes
   (resident CTAs per SM and cells each thread marches over, 0-3); on the
   FP64 path 0 the column kernel (each face evaluated once) or 1 the per-cell
   kernel (each face evaluated by both of its cells, no barriers).  No choice
   changes a result. */
typedef struct ostc_tuning {
  int schedule, flux_variant;
  int candidates;     /* pairs timed */
  double ms;          /* device time of one pass of source, flux and implicit stages, chosen pair */
  double ms_default;  /* the same for (0, 0) */
} ostc_tuning;
/* Times every pair on the driver's own case (reps passes each, the flow state
   is not advanced), applies the fastest and records it in
   output/message/autotune.txt, which ostc_driver_initialize applies again
   when the configuration and block sizes match.  out may be NULL. */
int ostc_driver_autotune(ostc_driver *d, int reps, ostc_tuning *out);
int ostc_driver_set_tuning(ostc_driver *d, int schedule, int flux_variant);

/* No counterpart in the reference.  Recomputes, from the device state, the
   normalised residuals of rho, |V|, p, T of the last step, without allocating
   any device memory: the reduction runs in a static 8 MiB device scratch.
   Valid only right after a step that computed a residual (step 1 and every
   output_screen-th step, which store the previous state on the device; the
   same values ostc_driver_residual returns then); after any other step it
   returns OSTC_ERR_STATE.  For callers that must not allocate, such as a
   convergence monitor polling a solver whose flow state fills the device.
   Limit: grids of at most 262144 tiles of 32x4x1 cells (33,554,432 interior
   cells); larger grids get OSTC_ERR_INPUT.  The first successful call on a
   device performs set-up (the scratch's address is looked up and cached; a
   failed look-up is retried by the next call) and should come before any
   stream capture on that device.  The driver's device is made current for
   the call and the caller's device restored.  One scratch per device:
   overlapping calls on the same device race; serialise them.  Requires at
   least one step (OSTC_ERR_STATE). */
int ostc_driver_residual_noalloc(ostc_driver *d, double res[4]);

#ifdef __cplusplus
}
#endif
#endif
