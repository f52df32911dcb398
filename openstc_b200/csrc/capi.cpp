// extern "C" boundary of libopenstc_b200.so (declared in include/openstc_b200.h).
#include "../../include/openstc_b200.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>

#include "device/engine.hpp"
#include "device/surrogate.hpp"
#include "host/driver.hpp"

struct ostc_driver {
  ostc::Driver drv;
  ostc_driver(const std::string &dir, const ostc::DriverOptions &o) : drv(dir, o) {}
};

namespace {
int fail(int code, const std::string &msg) { return ostc::abi_error(code, msg); }

template <typename F>
int guarded(F &&f) {
  try {
    return f();
  } catch (const ostc::ParameterError &e) {
    const std::string m = e.what();
    return fail(m.rfind("Nan occurred", 0) == 0 ? OSTC_ERR_NAN : OSTC_ERR_INPUT, m);
  } catch (const std::exception &e) {
    const std::string m = e.what();
    return fail(m.rfind("CUDA error", 0) == 0 ? OSTC_ERR_CUDA : OSTC_ERR_INTERNAL, m);
  }
}

// Ghost layers / components of a field for a configuration; mirrors the
// engine's allocation (0 components: not allocated).
void field_layout(const ostc::DevParams &p, int ngg, int field, int &ghost, int &nc) {
  const bool dplur = p.implicit_method == 1;
  ghost = ngg;
  nc = 1;
  switch (field) {
    case OSTC_METRIC: nc = 9; break;
    case OSTC_WALL_DIST: case OSTC_MUT: case OSTC_TURB_COND: nc = p.turb ? 1 : 0; break;
    case OSTC_BV: nc = 6; break;
    case OSTC_SV: nc = p.n_scalar; break;
    case OSTC_CV: nc = p.n_var; break;
    case OSTC_RHO_D: nc = p.ns; break;
    case OSTC_CHEM_JAC:
      ghost = 0;
      nc = (p.mix == 2 && p.chem_src_method != 0) ? (p.chem_src_method == 2 ? p.ns : p.ns * p.ns) : 0;
      break;
    case OSTC_TURB_SRC_JAC: ghost = 0; nc = p.turb ? 2 : 0; break;
    case OSTC_DQ: ghost = dplur ? 1 : 0; nc = p.n_var; break;
    case OSTC_DQ0: case OSTC_DQK: ghost = dplur ? 1 : 0; nc = dplur ? p.n_var : 0; break;
    case OSTC_INV_SPEC: ghost = dplur ? 1 : 0; nc = 3; break;
    case OSTC_VISC_SPEC: ghost = dplur ? 1 : 0; break;
    case OSTC_DT_LOCAL: ghost = 0; break;
    case OSTC_BV_LAST: ghost = 0; nc = 4; break;
    default: break;
  }
}
}  // namespace

extern "C" {

const char *ostc_last_error(void) { return ostc::abi_last_error(); }

int ostc_driver_create(const char *case_dir, const ostc_options *opt, ostc_driver **out) {
  if (!case_dir || !out) return fail(OSTC_ERR_INPUT, "null argument");
  *out = nullptr;
  return guarded([&] {
    ostc::DriverOptions o;
    if (opt) {
      o.device = opt->device;
      o.quiet = opt->quiet != 0;
      o.precision = opt->precision;
      o.exact_inner = opt->exact_inner != 0;
      if (opt->wall_distance < 0 || opt->wall_distance > 2) throw std::invalid_argument("wall_distance must be 0, 1 or 2");
      o.wall_distance = opt->wall_distance;
    }
    *out = new ostc_driver(case_dir, o);
    return OSTC_OK;
  });
}

void ostc_driver_destroy(ostc_driver *d) { delete d; }

int ostc_driver_info(const ostc_driver *d, ostc_info *info) {
  if (!d || !info) return fail(OSTC_ERR_INPUT, "null argument");
  const ostc::Driver &D = d->drv;
  std::memset(info, 0, sizeof(*info));
  info->n_block = D.mesh.n_block;
  info->ngg = D.mesh.ngg;
  info->dimension = D.mesh.dimension;
  info->n_spec = D.spec.n_spec;
  info->n_reac = D.reac.n_reac;
  info->n_var = D.dev_params.n_var;
  info->n_scalar = D.dev_params.n_scalar;
  info->mix = D.mix;
  info->rans = D.rans ? 1 : 0;
  info->implicit_method = D.dev_params.implicit_method;
  info->dplur_inner_step = D.dev_params.dplur_inner_step;
  info->chem_src_method = D.dev_params.chem_src_method;
  info->step = D.step;
  info->n_grid_total = D.mesh.n_grid_total;
  info->n_bc = static_cast<int>(D.host_bcs.size());
  info->n_inner = static_cast<int>(D.host_inner.size());
  return OSTC_OK;
}

int ostc_driver_params(const ostc_driver *d, ostc_params *o) {
  if (!d || !o) return fail(OSTC_ERR_INPUT, "null argument");
  const ostc::DevParams &p = d->drv.dev_params;
  std::memset(o, 0, sizeof(*o));
  o->ns = p.ns;
  o->nr = p.nr;
  o->n_var = p.n_var;
  o->n_scalar = p.n_scalar;
  o->mix = p.mix;
  o->turb = p.turb;
  o->rans_model = p.rans_model;
  o->turb_implicit = p.turb_implicit;
  o->chem_src_method = p.chem_src_method;
  o->implicit_method = p.implicit_method;
  o->dplur_inner_step = p.dplur_inner_step;
  o->reconstruction = p.reconstruction;
  o->limiter = p.limiter;
  o->viscous_order = p.viscous_order;
  o->dim = p.dim;
  o->output_screen = d->drv.parameter.get_int("output_screen");
  o->cfl = p.cfl;
  o->Pr = p.Pr;
  o->Prt = p.Prt;
  o->Sct = p.Sct;
  o->Sc = p.Sc;
  std::memcpy(o->ll, p.ll, sizeof(p.ll));
  std::memcpy(o->ul, p.ul, sizeof(p.ul));
  std::memcpy(o->sv_inf, p.sv_inf, sizeof(p.sv_inf));
  const int ns = p.ns;
  for (int i = 0; i < ns; ++i) {
    o->mw[i] = p.mw[i];
    o->t_low[i] = p.t_low[i];
    o->t_mid[i] = p.t_mid[i];
    o->lj_inv[i] = p.lj_inv[i];
    o->vis_coeff[i] = p.vis_coeff[i];
  }
  std::memcpy(o->low_coeff, p.low, sizeof(double) * 7 * ns);
  std::memcpy(o->high_coeff, p.high, sizeof(double) * 7 * ns);
  std::memcpy(o->w_quarter, p.wq, sizeof(double) * ns * ns);
  std::memcpy(o->w_sqrt8, p.w8, sizeof(double) * ns * ns);
  for (int r = 0; r < p.nr; ++r) {
    o->label[r] = p.label[r];
    o->order[r] = p.order[r];
    o->A[r] = p.A[r];
    o->b[r] = p.b[r];
    o->Ea[r] = p.Ea[r];
    o->A2[r] = p.A2[r];
    o->b2[r] = p.b2[r];
    o->Ea2[r] = p.Ea2[r];
    o->troe_alpha[r] = p.troe_a[r];
    o->troe_t3[r] = p.troe_t3[r];
    o->troe_t1[r] = p.troe_t1[r];
    o->troe_t2[r] = p.troe_t2[r];
    for (int l = 0; l < ns; ++l) {
      o->stoi_f[r * ns + l] = p.sf[r * ns + l];
      o->stoi_b[r * ns + l] = p.sb[r * ns + l];
      o->third_body[r * ns + l] = p.tb[r * ns + l];
    }
  }
  return OSTC_OK;
}

int ostc_driver_bc(const ostc_driver *d, int index, ostc_bc *bc) {
  if (!d || !bc) return fail(OSTC_ERR_INPUT, "null argument");
  if (index < 0 || index >= static_cast<int>(d->drv.host_bcs.size())) return fail(OSTC_ERR_INPUT, "bc index");
  static_assert(sizeof(ostc_bc) == sizeof(ostc::HostBc), "ostc_bc layout");
  std::memcpy(bc, &d->drv.host_bcs[index], sizeof(ostc_bc));
  return OSTC_OK;
}

int ostc_driver_inner(const ostc_driver *d, int index, ostc_inner *f) {
  if (!d || !f) return fail(OSTC_ERR_INPUT, "null argument");
  if (index < 0 || index >= static_cast<int>(d->drv.host_inner.size())) return fail(OSTC_ERR_INPUT, "inner index");
  static_assert(sizeof(ostc_inner) == sizeof(ostc::HostInner), "ostc_inner layout");
  std::memcpy(f, &d->drv.host_inner[index], sizeof(ostc_inner));
  return OSTC_OK;
}

int ostc_driver_block_dims(const ostc_driver *d, int block, int dims[3]) {
  if (!d || !dims) return fail(OSTC_ERR_INPUT, "null argument");
  if (block < 0 || block >= d->drv.mesh.n_block) return fail(OSTC_ERR_INPUT, "block index");
  const ostc::Block &B = d->drv.mesh[block];
  dims[0] = B.mx;
  dims[1] = B.my;
  dims[2] = B.mz;
  return OSTC_OK;
}

int ostc_field_layout(const ostc_driver *d, int field, int *ghost, int *components) {
  if (!d || !ghost || !components) return fail(OSTC_ERR_INPUT, "null argument");
  if (field < 0 || field >= OSTC_N_FIELDS) return fail(OSTC_ERR_INPUT, "field id");
  field_layout(d->drv.dev_params, d->drv.mesh.ngg, field, *ghost, *components);
  return OSTC_OK;
}

int ostc_driver_get_host_field(const ostc_driver *d, int block, int field, double *out, int64_t count) {
  if (!d || !out) return fail(OSTC_ERR_INPUT, "null argument");
  return guarded([&] {
    const ostc::Driver &D = d->drv;
    if (block < 0 || block >= D.mesh.n_block) return fail(OSTC_ERR_INPUT, "block index");
    const ostc::Block &B = D.mesh[block];
    const ostc::HostField &F = D.field[block];
    const int64_t n = B.x.e.size();
    auto put = [&](const double *src, int64_t want) {
      if (count != want) return fail(OSTC_ERR_INPUT, "count mismatch: expected " + std::to_string(want));
      std::memcpy(out, src, sizeof(double) * want);
      return static_cast<int>(OSTC_OK);
    };
    switch (field) {
      case OSTC_X: return put(B.x.v.data(), n);
      case OSTC_Y: return put(B.y.v.data(), n);
      case OSTC_Z: return put(B.z.v.data(), n);
      case OSTC_JAC: return put(B.jac.v.data(), n);
      case OSTC_METRIC: {
        if (count != 9 * n) return fail(OSTC_ERR_INPUT, "count mismatch: expected " + std::to_string(9 * n));
        for (int q = 0; q < 9; ++q) std::memcpy(out + q * n, B.metric[q].v.data(), sizeof(double) * n);
        return static_cast<int>(OSTC_OK);
      }
      case OSTC_BV: return put(F.bv.data(), static_cast<int64_t>(F.bv.size()));
      case OSTC_SV: return put(F.sv.data(), static_cast<int64_t>(F.sv.size()));
      default: return fail(OSTC_ERR_INPUT, "field has no host copy");
    }
  });
}

int ostc_driver_initialize(ostc_driver *d) {
  if (!d) return fail(OSTC_ERR_INPUT, "null argument");
  return guarded([&] {
    d->drv.initialize_computation();
    return OSTC_OK;
  });
}

int ostc_driver_simulate(ostc_driver *d) {
  if (!d) return fail(OSTC_ERR_INPUT, "null argument");
  if (!d->drv.initialized()) return fail(OSTC_ERR_STATE, "initialize first");
  return guarded([&] {
    d->drv.simulate();
    return OSTC_OK;
  });
}

int ostc_driver_step(ostc_driver *d, int n_steps, double *err_max) {
  if (!d || n_steps < 0) return fail(OSTC_ERR_INPUT, "bad argument");
  if (!d->drv.initialized()) return fail(OSTC_ERR_STATE, "initialize first");
  return guarded([&] {
    const double e = d->drv.advance(n_steps);
    if (err_max) *err_max = e;
    return OSTC_OK;
  });
}

int ostc_driver_step_io(ostc_driver *d, int n_steps, int block, const int *fields, double *const *host,
                        const int64_t *counts, int n_fields, int64_t chunk_bytes, double *err_max) {
  if (!d || n_steps < 0 || n_fields < 0 || (n_fields > 0 && (!fields || !host || !counts)) || chunk_bytes < 0)
    return fail(OSTC_ERR_INPUT, "bad argument");
  if (!d->drv.initialized()) return fail(OSTC_ERR_STATE, "initialize first");
  return guarded([&] {
    ostc::Engine &E = d->drv.engine();
    if (block < 0 || block >= static_cast<int>(E.blocks().size())) return fail(OSTC_ERR_INPUT, "block index");
    std::vector<int> f(fields, fields + n_fields);
    std::vector<double *> h(host, host + n_fields);
    for (int k = 0; k < n_fields; ++k) {
      if (f[k] < 0 || f[k] >= OSTC_N_FIELDS) return fail(OSTC_ERR_INPUT, "field id");
      if (f[k] == ostc::F_X || f[k] == ostc::F_Y || f[k] == ostc::F_Z || f[k] == ostc::F_JAC ||
          f[k] == ostc::F_METRIC || f[k] == ostc::F_WALL_DIST)
        return fail(OSTC_ERR_INPUT, "the geometry is set with ostc_driver_set_field");
      if (!h[k]) return fail(OSTC_ERR_INPUT, "null host buffer");
      const int64_t n = E.field_count(block, f[k]);
      if (n == 0) return fail(OSTC_ERR_INPUT, "field not allocated in this configuration");
      if (counts[k] != n) return fail(OSTC_ERR_INPUT, "host buffer size does not match the field");
    }
    const double e = d->drv.step_io(n_steps, block, f, h, chunk_bytes > 0 ? chunk_bytes : (int64_t(16) << 20));
    if (err_max) *err_max = e;
    return static_cast<int>(OSTC_OK);
  });
}

int ostc_driver_residual(const ostc_driver *d, double res[4]) {
  if (!d || !res) return fail(OSTC_ERR_INPUT, "null argument");
  for (int l = 0; l < 4; ++l) res[l] = d->drv.res[l];
  return OSTC_OK;
}

int ostc_driver_autotune(ostc_driver *d, int reps, ostc_tuning *out) {
  if (!d || reps < 1) return fail(OSTC_ERR_INPUT, "bad argument");
  if (!d->drv.initialized()) return fail(OSTC_ERR_STATE, "initialize first");
  return guarded([&] {
    const ostc::Driver::Tuning t = d->drv.autotune(reps);
    if (out) {
      out->schedule = t.schedule;
      out->flux_variant = t.flux_variant;
      out->candidates = t.candidates;
      out->ms = t.ms;
      out->ms_default = t.ms_default;
    }
    return OSTC_OK;
  });
}

int ostc_driver_set_tuning(ostc_driver *d, int schedule, int flux_variant) {
  if (!d) return fail(OSTC_ERR_INPUT, "null argument");
  if (!d->drv.initialized()) return fail(OSTC_ERR_STATE, "initialize first");
  return guarded([&] {
    d->drv.engine().set_tuning(schedule, flux_variant);
    return OSTC_OK;
  });
}

int ostc_driver_residual_noalloc(ostc_driver *d, double res[4]) {
  if (!d || !res) return fail(OSTC_ERR_INPUT, "null argument");
  if (!d->drv.initialized()) return fail(OSTC_ERR_STATE, "initialize first");
  if (d->drv.step < 1) return fail(OSTC_ERR_STATE, "no step taken yet: the residual scale is set at step 1");
  if (!d->drv.last_step_residual)
    return fail(OSTC_ERR_STATE, "step " + std::to_string(d->drv.step) +
                                    " computed no residual (only step 1 and every output_screen-th step do): the "
                                    "device no longer holds the state before it");
  return guarded([&]() -> int {
    ostc::Engine &E = d->drv.engine();
    double raw[4] = {0, 0, 0, 0};
    const char *why = "";
    const int st = ostc::residual_sums_noalloc(E, d->drv.opt.device, raw, &why);
    if (st == 1)
      return fail(OSTC_ERR_INPUT, "ostc_driver_residual_noalloc: the grid has " + std::to_string(E.residual_tiles()) +
                                      " residual tiles (32x4x1 cells); the static scratch holds at most " +
                                      std::to_string(ostc::kNoAllocMaxTiles) + " (33554432 interior cells)");
    if (st != 0) return fail(OSTC_ERR_CUDA, std::string("CUDA error in ostc_driver_residual_noalloc: ") + why);
    // the normalisation of Driver::compute_residual, without touching its state
    const double n = static_cast<double>(d->drv.mesh.n_grid_total);
    for (int l = 0; l < 4; ++l) res[l] = std::sqrt(raw[l] / n) / d->drv.res_scale[l];
    return OSTC_OK;
  });
}

int ostc_driver_run_phase(ostc_driver *d, int phase) {
  if (!d) return fail(OSTC_ERR_INPUT, "null argument");
  if (!d->drv.initialized()) return fail(OSTC_ERR_STATE, "initialize first");
  return guarded([&] {
    d->drv.engine().phase(phase);
    return OSTC_OK;
  });
}

int ostc_driver_get_field(ostc_driver *d, int block, int field, double *out, int64_t count) {
  if (!d || !out) return fail(OSTC_ERR_INPUT, "null argument");
  if (!d->drv.initialized()) return fail(OSTC_ERR_STATE, "initialize first");
  return guarded([&] {
    d->drv.engine().get_field(block, field, out, count);
    return OSTC_OK;
  });
}

int ostc_driver_set_field(ostc_driver *d, int block, int field, const double *in, int64_t count) {
  if (!d || !in) return fail(OSTC_ERR_INPUT, "null argument");
  if (!d->drv.initialized()) return fail(OSTC_ERR_STATE, "initialize first");
  return guarded([&] {
    d->drv.engine().set_field(block, field, in, count);
    return OSTC_OK;
  });
}

int ostc_driver_write_plt(ostc_driver *d, const char *path) {
  if (!d || !path) return fail(OSTC_ERR_INPUT, "null argument");
  if (!d->drv.initialized()) return fail(OSTC_ERR_STATE, "initialize first");
  return guarded([&] {
    d->drv.write_field(path);
    return OSTC_OK;
  });
}

int ostc_driver_launches_per_step(const ostc_driver *d, int store_last, int residual) {
  if (!d) return fail(OSTC_ERR_INPUT, "null argument");
  if (!d->drv.initialized()) return fail(OSTC_ERR_STATE, "initialize first");
  return const_cast<ostc_driver *>(d)->drv.engine().launches_per_step(store_last != 0, residual != 0);
}

int ostc_driver_last_step_ms(const ostc_driver *d, double *ms) {
  if (!d || !ms) return fail(OSTC_ERR_INPUT, "null argument");
  if (!d->drv.initialized()) return fail(OSTC_ERR_STATE, "initialize first");
  *ms = const_cast<ostc_driver *>(d)->drv.engine().last_step_ms();
  return OSTC_OK;
}

int ostc_driver_profile_step(ostc_driver *d, char *buf, int buflen) {
  if (!d || !buf || buflen <= 0) return fail(OSTC_ERR_INPUT, "bad argument");
  if (!d->drv.initialized()) return fail(OSTC_ERR_STATE, "initialize first");
  return guarded([&] {
    const auto rows = d->drv.engine().profile_step();
    std::string text;
    for (const auto &[name, n, ms] : rows) {
      char line[160];
      std::snprintf(line, sizeof(line), "%s %d %.6f\n", name.c_str(), n, ms);
      text += line;
    }
    if (static_cast<int>(text.size()) + 1 > buflen) return fail(OSTC_ERR_INPUT, "buffer too small");
    std::memcpy(buf, text.c_str(), text.size() + 1);
    return static_cast<int>(rows.size());
  });
}

void *ostc_driver_stream(ostc_driver *d) {
  if (!d || !d->drv.initialized()) return nullptr;
  return d->drv.engine().stream();
}

}  // extern "C"

namespace ostc {
cudaError_t tc_gemm(const uint16_t *A, int lda, const uint16_t *B, int ldb, float *D, int ldd, int M, int N, int K,
                    int splits, int *err, cudaStream_t st);
}

struct ostc_surrogate {
  std::unique_ptr<ostc::Surrogate> s;
};

namespace {
constexpr int kSurParamCount() {
  int n = 0;
  const int dims[ostc::kSurLayers + 1] = {ostc::kSurInPad, ostc::kSurHidden, ostc::kSurHidden, ostc::kSurHidden,
                                          ostc::kSurHidden, ostc::kSurOutPad};
  for (int l = 0; l < ostc::kSurLayers; ++l) n += dims[l + 1] * dims[l] + dims[l + 1];
  return n;
}
}  // namespace

extern "C" {

int ostc_tc_gemm_bf16(const void *A, int lda, const void *B, int ldb, float *D, int ldd, int M, int N, int K,
                      int splits, int *err, void *stream) {
  if (!A || !B || !D || !err || M <= 0 || N <= 0 || K <= 0 || splits <= 0)
    return fail(OSTC_ERR_INPUT, "ostc_tc_gemm_bf16: null pointer or non-positive size");
  if (K % 8 || lda % 8 || ldb % 8 || lda < K || ldb < K || ldd < N)
    return fail(OSTC_ERR_INPUT, "ostc_tc_gemm_bf16: K, lda and ldb must be multiples of 8, lda/ldb >= K, ldd >= N");
  const cudaError_t e = ostc::tc_gemm(static_cast<const uint16_t *>(A), lda, static_cast<const uint16_t *>(B), ldb, D,
                                      ldd, M, N, K, splits, err, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return fail(OSTC_ERR_CUDA, std::string("ostc_tc_gemm_bf16: ") + cudaGetErrorString(e));
  return OSTC_OK;
}

int ostc_surrogate_create(const ostc_driver *d, unsigned long long seed, ostc_surrogate **out) {
  if (!d || !out) return fail(OSTC_ERR_INPUT, "null argument");
  return guarded([&] {
    const auto &sp = d->drv.spec;
    auto h = std::make_unique<ostc_surrogate>();
    h->s = std::make_unique<ostc::Surrogate>(d->drv.dev_params, sp.elem_comp, sp.n_elem(), d->drv.opt.device, seed);
    *out = h.release();
    return OSTC_OK;
  });
}

void ostc_surrogate_destroy(ostc_surrogate *s) { delete s; }

int ostc_surrogate_param_count(void) { return kSurParamCount(); }

int ostc_surrogate_generate(ostc_surrogate *s, const ostc_driver *field, long long n, unsigned long long seed,
                            double field_fraction) {
  if (!s) return fail(OSTC_ERR_INPUT, "null argument");
  if (field && !field->drv.initialized()) return fail(OSTC_ERR_STATE, "the field driver is not initialised");
  return guarded([&] {
    const ostc::DevBlock *blk = nullptr;
    ostc::DevBlock b0{};
    if (field) {
      b0 = const_cast<ostc_driver *>(field)->drv.engine().blocks().at(0);
      blk = &b0;
    }
    s->s->generate(n, seed, blk, field_fraction);
    return OSTC_OK;
  });
}

int ostc_surrogate_train(ostc_surrogate *s, int steps, int batch, double lr, long long n_train, float *losses) {
  if (!s || steps < 0 || batch <= 0) return fail(OSTC_ERR_INPUT, "bad argument");
  return guarded([&] {
    s->s->train(steps, batch, lr, n_train, losses);
    return OSTC_OK;
  });
}

int ostc_surrogate_evaluate(ostc_surrogate *s, long long begin, long long count, ostc_surrogate_eval *out) {
  if (!s || !out) return fail(OSTC_ERR_INPUT, "null argument");
  return guarded([&] {
    const ostc::SurrogateEval e = s->s->evaluate(begin, count);
    out->mean_rel = e.mean_rel;
    out->max_rel = e.max_rel;
    out->mean_abs = e.mean_abs;
    out->max_defect = e.max_defect;
    out->mean_defect = e.mean_defect;
    out->median_rel_all = e.median_rel_all;
    out->p90_rel_all = e.p90_rel_all;
    out->gate_pass = e.gate_pass;
    out->count = e.count;
    out->nonfinite = e.nonfinite;
    out->rel_count = e.rel_count;
    return OSTC_OK;
  });
}

int ostc_surrogate_label(ostc_surrogate *s, const double *states, long long n, double *dy) {
  if (!s || !states || !dy || n <= 0) return fail(OSTC_ERR_INPUT, "bad argument");
  return guarded([&] {
    s->s->label_host(states, n, dy);
    return OSTC_OK;
  });
}

int ostc_surrogate_predict(ostc_surrogate *s, const double *states, long long n, double *dy, int *accepted) {
  if (!s || !states || !dy || !accepted || n <= 0) return fail(OSTC_ERR_INPUT, "bad argument");
  return guarded([&] {
    s->s->predict_host(states, n, dy, accepted);
    return OSTC_OK;
  });
}

int ostc_surrogate_gradients(ostc_surrogate *s, const double *states, const double *dy, long long n, float *grads,
                             double *loss) {
  if (!s || !states || !dy || !grads || !loss || n <= 0) return fail(OSTC_ERR_INPUT, "bad argument");
  return guarded([&] {
    std::vector<std::vector<float>> g;
    *loss = s->s->grad_host(states, dy, n, g);
    size_t off = 0;
    for (const auto &v : g) {
      std::copy(v.begin(), v.end(), grads + off);
      off += v.size();
    }
    return OSTC_OK;
  });
}

int ostc_surrogate_get_params(const ostc_surrogate *s, float *flat) {
  if (!s || !flat) return fail(OSTC_ERR_INPUT, "null argument");
  return guarded([&] {
    size_t off = 0;
    for (const auto &v : s->s->params()) {
      std::copy(v.begin(), v.end(), flat + off);
      off += v.size();
    }
    return OSTC_OK;
  });
}

int ostc_surrogate_set_params(ostc_surrogate *s, const float *flat) {
  if (!s || !flat) return fail(OSTC_ERR_INPUT, "null argument");
  return guarded([&] {
    auto p = s->s->params();
    size_t off = 0;
    for (auto &v : p) {
      std::copy(flat + off, flat + off + v.size(), v.begin());
      off += v.size();
    }
    s->s->set_params(p);
    return OSTC_OK;
  });
}

int ostc_surrogate_normalisation(const ostc_surrogate *s, float *in_mu, float *in_sig, float *out_c, float *out_scale) {
  if (!s || !in_mu || !in_sig || !out_c || !out_scale) return fail(OSTC_ERR_INPUT, "null argument");
  std::copy(s->s->out_c.begin(), s->s->out_c.end(), out_c);
  std::copy(s->s->in_mu.begin(), s->s->in_mu.end(), in_mu);
  std::copy(s->s->in_sig.begin(), s->s->in_sig.end(), in_sig);
  std::copy(s->s->out_s.begin(), s->s->out_s.end(), out_scale);
  return OSTC_OK;
}

int ostc_driver_set_surrogate(ostc_driver *d, ostc_surrogate *s) {
  if (!d) return fail(OSTC_ERR_INPUT, "null argument");
  if (!d->drv.initialized()) return fail(OSTC_ERR_STATE, "initialize first");
  return guarded([&]() -> int {
    if (s) {
      if (s->s->device() != d->drv.opt.device) return fail(OSTC_ERR_INPUT, "surrogate and driver are on different devices");
      const ostc::SurrogateDev p = s->s->device_params();
      d->drv.engine().set_surrogate(&p);
    } else {
      d->drv.engine().set_surrogate(nullptr);
    }
    return OSTC_OK;
  });
}

int ostc_driver_chemistry_stats(ostc_driver *d, long long *accepted, long long *fallback, long long *evaluated) {
  if (!d || !accepted || !fallback) return fail(OSTC_ERR_INPUT, "null argument");
  if (!d->drv.initialized()) return fail(OSTC_ERR_STATE, "initialize first");
  return guarded([&] {
    unsigned long long st[3];
    d->drv.engine().surrogate_stats(st);
    *accepted = static_cast<long long>(st[0]);
    *fallback = static_cast<long long>(st[1]);
    if (evaluated) *evaluated = static_cast<long long>(st[2]);
    return OSTC_OK;
  });
}

int ostc_surrogate_get_gate(const ostc_surrogate *s, ostc_surrogate_gate *g) {
  if (!s || !g) return fail(OSTC_ERR_INPUT, "null argument");
  static_assert(sizeof(ostc_surrogate_gate) == sizeof(ostc::SurrogateGate), "gate layouts differ");
  std::memcpy(g, &s->s->gate, sizeof(*g));
  return OSTC_OK;
}

int ostc_surrogate_set_gate(ostc_surrogate *s, const ostc_surrogate_gate *g) {
  if (!s || !g) return fail(OSTC_ERR_INPUT, "null argument");
  std::memcpy(&s->s->gate, g, sizeof(*g));
  return OSTC_OK;
}

int ostc_surrogate_save(const ostc_surrogate *s, const char *path) {
  if (!s || !path) return fail(OSTC_ERR_INPUT, "null argument");
  return guarded([&] {
    s->s->save(path);
    return OSTC_OK;
  });
}

int ostc_surrogate_load(ostc_surrogate *s, const char *path) {
  if (!s || !path) return fail(OSTC_ERR_INPUT, "null argument");
  return guarded([&] {
    s->s->load(path);
    return OSTC_OK;
  });
}

}  // extern "C"

