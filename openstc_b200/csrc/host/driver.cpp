#include "driver.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <algorithm>
#include <condition_variable>
#include <deque>
#include <exception>
#include <limits>
#include <mutex>
#include <thread>

#include "plt_io.hpp"

namespace ostc {

// The .plt output of the steady loop without stalling it: at an output step
// the device-to-host copies of bv, sv, Mach and mu_t go into one of two
// page-locked staging sets on the engine stream, behind the step's kernels,
// and the loop goes on; a writer thread waits for the copies, then writes
// output/message/step.txt and output/field/flowfield.plt exactly as the
// synchronous path does.  A third output waits for the older set to be
// written.  flush() returns when everything enqueued is on disk and rethrows
// a writer error.
class PltPipeline {
 public:
  // wall_dyn_pressure > 0: also the reference's post-processing 0 (skin
  // friction and heat flux of the j = 0 wall, output/wall/friction_heatflux.dat)
  PltPipeline(Engine &E, const Mesh &mesh, const std::vector<HostField> &field, const Species &spec, bool rans,
              std::string case_dir, double wall_dyn_pressure)
      : E_(E), mesh_(mesh), spec_(spec), rans_(rans), dir_(std::move(case_dir)), wall_q_(wall_dyn_pressure) {
    for (auto &st : slots_) {
      st.field.resize(mesh.n_block);
      st.mach.resize(mesh.n_block);
      st.mut.resize(mesh.n_block);
      st.cf.resize(mesh.n_block);
      st.qw.resize(mesh.n_block);
      for (int b = 0; b < mesh.n_block; ++b) {
        HostField &F = st.field[b];
        F.e = field[b].e;
        F.n_scalar = field[b].n_scalar;
        F.bv.resize(field[b].bv.size());
        F.sv.resize(field[b].sv.size());
        st.mach[b].resize(static_cast<size_t>(F.e.size()));
        if (rans) st.mut[b].resize(static_cast<size_t>(F.e.size()));
        if (wall_q_ > 0) {
          st.cf[b].resize(static_cast<size_t>(mesh[b].mx));
          st.qw[b].resize(static_cast<size_t>(mesh[b].mx));
        }
        // page-locked, so that the copies do not stall the loop; where the
        // host refuses to lock them the copies are synchronous instead
        for (auto *v : {&F.bv, &F.sv, &st.mach[b], &st.mut[b], &st.cf[b], &st.qw[b]})
          if (!v->empty() && E_.pin_host(v->data(), sizeof(double) * v->size())) pinned_.push_back(v->data());
      }
    }
    writer_ = std::thread([this] { run(); });
  }

  ~PltPipeline() {
    {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait(lk, [this] { return queue_.empty() && !writing_; });
      stop_ = true;
    }
    cv_.notify_all();
    writer_.join();
    for (void *p : pinned_) {
      try {
        E_.unpin_host(p);
      } catch (...) {
      }
    }
  }

  void enqueue(int step) {
    const int s = next_++ & 1;
    Slot &st = slots_[s];
    {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait(lk, [&] { return !st.busy; });
      rethrow_locked();
      st.busy = true;
    }
    st.step = step;
    for (int b = 0; b < mesh_.n_block; ++b) {
      HostField &F = st.field[b];
      E_.get_field_async(b, F_BV, F.bv.data(), static_cast<int64_t>(F.bv.size()));
      if (!F.sv.empty()) E_.get_field_async(b, F_SV, F.sv.data(), static_cast<int64_t>(F.sv.size()));
      E_.get_field_async(b, F_MACH, st.mach[b].data(), static_cast<int64_t>(st.mach[b].size()));
      if (rans_) E_.get_field_async(b, F_MUT, st.mut[b].data(), static_cast<int64_t>(st.mut[b].size()));
      if (wall_q_ > 0) E_.wall_friction_heatflux_2d(b, wall_q_, st.cf[b].data(), st.qw[b].data());
    }
    E_.record_output_event(s);
    {
      std::lock_guard<std::mutex> lk(mu_);
      queue_.push_back(s);
    }
    cv_.notify_all();
  }

  void flush() {
    std::unique_lock<std::mutex> lk(mu_);
    cv_.wait(lk, [this] { return queue_.empty() && !writing_; });
    rethrow_locked();
  }

 private:
  struct Slot {
    std::vector<HostField> field;
    std::vector<std::vector<double>> mach, mut, cf, qw;
    int step = 0;
    bool busy = false;
  };

  // src/PostProcess.cu:35-42: one file, rewritten for every block in turn
  // (so a multi-block case keeps the last block's wall), x of the wall
  // point, cf, q_w, default stream formatting.
  void write_wall(const Slot &st) const {
    const std::filesystem::path dir = std::filesystem::path(dir_) / "output" / "wall";
    std::filesystem::create_directories(dir);
    for (int b = 0; b < mesh_.n_block; ++b) {
      std::ofstream f(dir / "friction_heatflux.dat");
      if (!f) throw ParameterError("cannot write " + (dir / "friction_heatflux.dat").string());
      f << "variables = \"x\", \"cf\", \"qw\"\n";
      const Block &blk = mesh_[b];
      for (int i = 0; i < blk.mx; ++i) f << blk.x(i, 0, 0) << '\t' << st.cf[b][i] << '\t' << st.qw[b][i] << '\n';
    }
  }

  void rethrow_locked() {
    if (error_) {
      std::exception_ptr e = error_;
      error_ = nullptr;
      std::rethrow_exception(e);
    }
  }

  void run() {
    for (;;) {
      int s;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [this] { return stop_ || !queue_.empty(); });
        if (queue_.empty()) return;
        s = queue_.front();
        queue_.pop_front();
        writing_ = true;
      }
      Slot &st = slots_[s];
      try {
        E_.wait_output_event(s);
        const std::filesystem::path dir = std::filesystem::path(dir_) / "output" / "message";
        std::filesystem::create_directories(dir);
        std::ofstream(dir / "step.txt") << st.step;
        std::vector<PltBlockData> blocks(mesh_.n_block);
        for (int b = 0; b < mesh_.n_block; ++b)
          blocks[b] = PltBlockData{&mesh_[b], &st.field[b], &st.mach[b], rans_ ? &st.mut[b] : nullptr};
        write_plt(dir_ + "/output/field/flowfield.plt", blocks, spec_, rans_);
        if (wall_q_ > 0) write_wall(st);
      } catch (...) {
        std::lock_guard<std::mutex> lk(mu_);
        error_ = std::current_exception();
      }
      {
        std::lock_guard<std::mutex> lk(mu_);
        st.busy = false;
        writing_ = false;
      }
      cv_.notify_all();
    }
  }

  Engine &E_;
  const Mesh &mesh_;
  const Species &spec_;
  bool rans_;
  std::string dir_;
  double wall_q_ = 0;  // dynamic pressure of the wall post-processing, 0: off
  Slot slots_[2];
  std::vector<void *> pinned_;
  int next_ = 0;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<int> queue_;
  bool writing_ = false, stop_ = false;
  std::exception_ptr error_;
  std::thread writer_;
};

Driver::~Driver() = default;

Driver::Driver(const std::string &dir, const DriverOptions &o) : case_dir(dir), opt(o), parameter(dir) {
  mesh = Mesh(parameter, opt.exact_inner);
  spec = Species(parameter);
  reac = Reaction(parameter, spec);
  const bool species = parameter.get_bool("species");
  const bool reaction = parameter.get_bool("reaction");
  int turb_method = parameter.get_int("turbulence_method");
  if (!parameter.get_bool("turbulence")) turb_method = 0;
  rans = turb_method == 1;
  mix = species ? (reaction ? 2 : 1) : 0;
  if (rans && parameter.get_int("RANS_model") != 2)
    throw ParameterError("only the k-omega SST model (RANS_model = 2) is implemented");
  // the step loops take step % output_screen and step % output_file
  for (const char *key : {"output_screen", "output_file"})
    if (parameter.get_int(key) < 1) throw ParameterError(std::string(key) + " must be a positive number of steps");

  // initialize_basic_variables, src/Initialize.cuh:37-55: the default inflow
  // is always constructed first, which defines rho_inf / v_inf / p_inf.
  Inflow default_inflow(parameter.get_string("default_init"), spec, parameter);
  field.resize(mesh.n_block);
  const int initial = parameter.get_int("initial");
  if (initial == 1) {
    const int n_scalar = parameter.get_int("n_scalar");
    for (int b = 0; b < mesh.n_block; ++b) {
      HostField &F = field[b];
      F.e = Extent{mesh[b].mx, mesh[b].my, mesh[b].mz, mesh[b].ngg};
      F.n_scalar = n_scalar;
      F.bv.assign(static_cast<size_t>(6 * F.e.size()), 0.0);
      F.sv.assign(static_cast<size_t>(n_scalar * F.e.size()), 0.0);
    }
    const std::string plt = case_dir + "/output/field/flowfield.plt";
    if (!read_plt_restart(plt, mesh, spec, parameter, field))
      throw ParameterError("restart requested but " + plt + " does not exist");
    std::ifstream st(case_dir + "/output/message/step.txt");
    int s = 0;
    if (st >> s) parameter.set("step", s);
    std::ifstream rs(case_dir + "/output/message/residual_scale.txt");
    rs >> res_scale[0] >> res_scale[1] >> res_scale[2] >> res_scale[3];
  } else {
    initialize_from_start(parameter, mesh, spec, field);
    std::ofstream history(case_dir + "/history.dat", std::ios::trunc);
    history << "step\terror_max\n";
  }
  step = parameter.get_int("step");
  bc.build(mesh, spec, parameter);
  build_dev_params();
  build_faces();
}

void Driver::build_dev_params() {
  DevParams &p = dev_params;
  std::memset(&p, 0, sizeof(p));
  const Parameter &P = parameter;
  p.ns = spec.n_spec;
  p.nr = reac.n_reac;
  if (p.nr > kMaxReac) throw ParameterError("at most 50 reactions are supported (MAX_REAC_NUMBER)");
  p.n_var = P.get_int("n_var");
  p.n_scalar = P.get_int("n_scalar");
  p.mix = mix;
  p.turb = rans ? 1 : 0;
  p.rans_model = P.get_int("RANS_model");
  p.turb_implicit = P.get_int("turb_implicit");
  p.chem_src_method = P.get_int("chemSrcMethod");
  p.implicit_method = P.get_int("implicit_method");
  p.dplur_inner_step = p.implicit_method == 1 ? P.get_int("DPLUR_inner_step") : 0;
  p.reconstruction = P.get_int("reconstruction");
  p.limiter = P.get_int("limiter");
  p.viscous_order = P.get_int("viscous_order");
  p.dim = mesh.dimension;
  p.cfl = P.get_real("cfl");
  p.Pr = P.get_real("prandtl_number");
  p.Prt = P.get_real("turbulent_prandtl_number");
  p.Sct = P.get_real("turbulent_schmidt_number");
  p.Sc = P.get_real("schmidt_number");
  if (p.limiter != 0 && p.limiter != 1) throw ParameterError("only the minmod limiter (0) is implemented");
  // DParameter::limit_flow, src/DParameter.cu:78-100
  const double rho_inf = P.get_real("rho_inf"), v_inf = P.get_real("v_inf"), p_inf = P.get_real("p_inf");
  p.ll[0] = 1e-6 * rho_inf;
  p.ul[0] = 1e+3 * rho_inf;
  for (int l = 1; l < 4; ++l) {
    p.ll[l] = -1e+3 * v_inf;
    p.ul[l] = 1e+3 * v_inf;
  }
  p.ll[4] = 1e-6 * p_inf;
  p.ul[4] = 1e+3 * p_inf;
  if (p.rans_model == 2) {
    p.ul[5] = std::numeric_limits<double>::max();
    p.ul[6] = std::numeric_limits<double>::max();
  }
  const auto &sv_inf = P.get_real_array("sv_inf");
  for (int l = 0; l < p.n_scalar && l < static_cast<int>(sv_inf.size()); ++l) p.sv_inf[l] = sv_inf[l];
  const int ns = p.ns;
  for (int i = 0; i < ns; ++i) {
    p.mw[i] = spec.mw[i];
    p.ru_mw[i] = kRu / spec.mw[i];
    p.t_low[i] = spec.t_low[i];
    p.t_mid[i] = spec.t_mid[i];
    for (int q = 0; q < 7; ++q) {
      p.low[i * 7 + q] = spec.low_coeff[i * 7 + q];
      p.high[i * 7 + q] = spec.high_coeff[i * 7 + q];
    }
    p.lj_inv[i] = spec.lj_potent_inv[i];
    p.vis_coeff[i] = spec.vis_coeff[i];
    for (int j = 0; j < ns; ++j) {
      p.wq[i * ns + j] = spec.wj_div_wi_quarter[i * ns + j];
      p.w8[i * ns + j] = spec.sqrt_wi_div_wj_8[i * ns + j];
    }
  }
  for (int r = 0; r < p.nr; ++r) {
    p.label[r] = reac.label[r];
    p.order[r] = reac.order[r];
    p.A[r] = reac.A[r];
    p.b[r] = reac.b[r];
    p.Ea[r] = reac.Ea[r];
    p.A2[r] = reac.A2[r];
    p.b2[r] = reac.b2[r];
    p.Ea2[r] = reac.Ea2[r];
    p.lnA[r] = reac.A[r] != 0 ? std::log(std::fabs(reac.A[r])) : 0.0;
    p.lnA2[r] = reac.A2[r] != 0 ? std::log(std::fabs(reac.A2[r])) : 0.0;
    p.troe_a[r] = reac.troe_alpha[r];
    p.troe_t3[r] = reac.troe_t3[r];
    p.troe_t1[r] = reac.troe_t1[r];
    p.troe_t2[r] = reac.troe_t2[r];
    for (int l = 0; l < ns; ++l) {
      p.sf[r * ns + l] = static_cast<signed char>(reac.stoi_f[r * ns + l]);
      p.sb[r * ns + l] = static_cast<signed char>(reac.stoi_b[r * ns + l]);
      p.tb[r * ns + l] = reac.third_body[r * ns + l];
    }
  }
  // FP32-bulk path: when only the last species takes part in no reaction
  // (a third body only, N2 here), its EPI row and column are zero and the
  // stored factors drop it
  p.na = ns;
  if (opt.precision == 1 && P.get_int("implicit_method") == 1 && P.get_int("chemSrcMethod") == 1) {
    int last = -1;
    for (int r = 0; r < p.nr; ++r)
      for (int l = 0; l < ns; ++l)
        if (p.sf[r * ns + l] != 0 || p.sb[r * ns + l] != 0) last = std::max(last, l);
    // the kernels store the block without the last species only
    if (last + 1 == ns - 1) p.na = ns - 1;
  }
}

void Driver::build_faces() {
  host_bcs.clear();
  for (const BcFace &f : bc.order) {
    const Boundary &b = mesh[f.block].boundary[f.face_index];
    HostBc h{};
    h.block = f.block;
    h.type = static_cast<int>(f.type);
    h.face = b.face;
    h.direction = b.direction;
    for (int q = 0; q < 3; ++q) {
      h.start[q] = b.start[q];
      h.end[q] = b.end[q];
    }
    if (f.type == BcType::inflow) {
      const Inflow &in = bc.inflow[f.cond];
      h.density = in.density;
      h.u = in.u;
      h.v = in.v;
      h.w = in.w;
      h.pressure = in.pressure;
      h.temperature = in.temperature;
      h.mut = in.mut;
      for (size_t l = 0; l < in.sv.size() && l < kMaxSpec + 2; ++l) h.sv[l] = in.sv[l];
    } else if (f.type == BcType::wall) {
      const Wall &w = bc.wall[f.cond];
      h.isothermal = w.isothermal ? 1 : 0;
      h.t_wall = w.temperature;
    }
    host_bcs.push_back(h);
  }
  host_inner.clear();
  for (int b = 0; b < mesh.n_block; ++b)
    for (const InnerFace &f : mesh[b].inner_face) {
      HostInner h{};
      h.block = b;
      h.target_block = f.target_block;
      h.face = f.face;
      h.direction = f.direction;
      for (int q = 0; q < 3; ++q) {
        h.start[q] = f.start[q];
        h.end[q] = f.end[q];
        h.loop_dir[q] = f.loop_dir[q];
        h.tstart[q] = f.tstart[q];
        h.tloop_dir[q] = f.target_loop_dir[q];
        h.src_tar[q] = f.src_tar[q];
        h.n_point[q] = f.n_point[q];
      }
      host_inner.push_back(h);
    }
  // Wall points of the trimmed wall faces (Driver::acquire_wall_distance,
  // src/Driver.cu:123-150).
  wall_points.clear();
  for (const HostBc &h : host_bcs) {
    if (h.type != static_cast<int>(BcType::wall)) continue;
    const Block &B = mesh[h.block];
    for (int k = h.start[2]; k <= h.end[2]; ++k)
      for (int j = h.start[1]; j <= h.end[1]; ++j)
        for (int i = h.start[0]; i <= h.end[0]; ++i) {
          wall_points.push_back(B.x(i, j, k));
          wall_points.push_back(B.y(i, j, k));
          wall_points.push_back(B.z(i, j, k));
        }
  }
}

Engine &Driver::engine() {
  if (!engine_) throw ParameterError("the device engine is not initialised");
  return *engine_;
}

void Driver::initialize_computation() {
  EngineSetup s;
  s.params = dev_params;
  s.ngg = mesh.ngg;
  for (const auto &b : mesh.block) s.dims.push_back({b.mx, b.my, b.mz});
  s.bcs = host_bcs;
  s.inner = host_inner;
  s.wall_points = wall_points;
  s.device = opt.device;
  s.precision = opt.precision;
  s.exact_inner = opt.exact_inner;
  s.wall_distance = opt.wall_distance;
  plt_out_.reset();  // bound to the engine it copies from
  engine_ = make_engine(s);
  for (int b = 0; b < mesh.n_block; ++b) {
    const Block &B = mesh[b];
    const int64_t n = B.x.e.size();
    engine_->set_field(b, F_X, B.x.v.data(), n);
    engine_->set_field(b, F_Y, B.y.v.data(), n);
    engine_->set_field(b, F_Z, B.z.v.data(), n);
    engine_->set_field(b, F_JAC, B.jac.v.data(), n);
    std::vector<double> met(static_cast<size_t>(9 * n));
    for (int q = 0; q < 9; ++q) std::copy(B.metric[q].v.begin(), B.metric[q].v.end(), met.begin() + q * n);
    engine_->set_field(b, F_METRIC, met.data(), 9 * n);
    engine_->set_field(b, F_BV, field[b].bv.data(), static_cast<int64_t>(field[b].bv.size()));
    if (!field[b].sv.empty())
      engine_->set_field(b, F_SV, field[b].sv.data(), static_cast<int64_t>(field[b].sv.size()));
  }
  engine_->initialize();
  // a choice the autotuner recorded for this configuration and these blocks
  std::ifstream tuned(std::filesystem::path(case_dir) / "output" / "message" / "autotune.txt");
  std::string key;
  int schedule = 0, variant = 0;
  if (tuned && std::getline(tuned, key) && key == tuning_key() && (tuned >> schedule >> variant) &&
      variant < engine_->flux_variants())
    engine_->set_tuning(schedule, variant);
  if (!opt.quiet) std::printf("The flowfield is completely initialized on GPU.\n");
}

std::string Driver::tuning_key() const {
  std::string k = "mix " + std::to_string(mix) + " rans " + std::to_string(rans ? 1 : 0) + " precision " +
                  std::to_string(opt.precision) + " exact " + std::to_string(opt.exact_inner ? 1 : 0) + " blocks";
  for (const auto &b : mesh.block) k += " " + std::to_string(b.mx) + "x" + std::to_string(b.my) + "x" + std::to_string(b.mz);
  return k;
}

Driver::Tuning Driver::autotune(int reps) {
  Engine &E = engine();
  Tuning t;
  t.ms = -1;
  for (int schedule = 0; schedule < 2; ++schedule) {
    for (int v = 0; v < E.flux_variants(); ++v) {
      E.set_tuning(schedule, v);
      const double ms = E.time_stages(reps);
      ++t.candidates;
      if (schedule == 0 && v == 0) t.ms_default = ms;
      if (t.ms < 0 || ms < t.ms) {
        t.ms = ms;
        t.schedule = schedule;
        t.flux_variant = v;
      }
    }
  }
  E.set_tuning(t.schedule, t.flux_variant);
  const std::filesystem::path dir = std::filesystem::path(case_dir) / "output" / "message";
  std::filesystem::create_directories(dir);
  std::ofstream out(dir / "autotune.txt");
  out << tuning_key() << '\n' << t.schedule << ' ' << t.flux_variant << '\n' << t.ms << ' ' << t.ms_default << '\n';
  return t;
}

double Driver::compute_residual(int step_no, const double raw[4]) {
  // Driver::compute_residual, src/Driver.cu:292-380
  for (int l = 0; l < 4; ++l) res[l] = std::sqrt(raw[l] / static_cast<double>(mesh.n_grid_total));
  if (step_no == 1) {
    for (int l = 0; l < 4; ++l) {
      res_scale[l] = res[l];
      if (res_scale[l] < 1e-20) res_scale[l] = 1e-20;
    }
    const std::filesystem::path dir = std::filesystem::path(case_dir) / "output" / "message";
    std::filesystem::create_directories(dir);
    std::ofstream out(dir / "residual_scale.txt");
    out << res_scale[0] << '\n' << res_scale[1] << '\n' << res_scale[2] << '\n' << res_scale[3] << '\n';
  }
  for (int l = 0; l < 4; ++l) res[l] /= res_scale[l];
  double err_max = res[0];
  for (int l = 1; l < 4; ++l)
    if (std::abs(res[l]) > err_max) err_max = res[l];
  if (std::isnan(err_max)) throw ParameterError("Nan occurred in step " + std::to_string(step_no) + ". Stop simulation.");
  return err_max;
}

double Driver::advance(int n) {
  Engine &E = engine();
  const int screen = parameter.get_int("output_screen");
  double err = -1;
  for (int q = 0; q < n; ++q) {
    ++step;
    const bool store = step % screen == 0;
    const bool due = store || step == 1;
    double raw[4] = {0, 0, 0, 0};
    last_step_residual = false;
    E.step(store, due, raw);
    if (due) err = compute_residual(step, raw);
    last_step_residual = due;
  }
  E.synchronize();
  return err;
}

double Driver::step_io(int n, int block, const std::vector<int> &fields, const std::vector<double *> &host,
                       int64_t chunk_bytes) {
  Engine &E = engine();
  const int screen = parameter.get_int("output_screen");
  const int nf = static_cast<int>(fields.size());
  double err = -1;
  try {
    for (int q = 0; q < n; ++q) {
      E.upload_chunked(block, fields.data(), host.data(), nf, chunk_bytes);
      ++step;
      const bool store = step % screen == 0;
      const bool due = store || step == 1;
      double raw[4] = {0, 0, 0, 0};
      last_step_residual = false;
      E.step(store, due, raw);
      if (due) err = compute_residual(step, raw);
      last_step_residual = due;
      E.download_chunked(block, fields.data(), host.data(), nf, chunk_bytes);
    }
  } catch (...) {
    // no copy may still touch the caller's buffers once the error reaches it
    try {
      E.sync_copies();
    } catch (...) {
    }
    throw;
  }
  E.sync_copies();
  E.synchronize();
  return err;
}

void Driver::simulate() {
  if (!parameter.get_bool("steady")) throw ParameterError("Not implemented: only steady simulations are supported");
  Engine &E = engine();
  if (!opt.quiet) std::printf("Steady flow simulation.\n");
  const int total = parameter.get_int("total_step") + step;
  const int screen = parameter.get_int("output_screen");
  const int out_file = parameter.get_int("output_file");
  const double criteria = parameter.get_real("convergence_criteria");
  bool converged = false;
  while (!converged) {
    ++step;
    if (step > total) break;
    const bool store = step % screen == 0;
    const bool due = store || step == 1;
    double raw[4] = {0, 0, 0, 0};
    last_step_residual = false;
    E.step(store, due, raw);
    last_step_residual = due;
    if (due) {
      const double err_max = compute_residual(step, raw);
      converged = err_max < criteria;
      std::FILE *h = std::fopen((case_dir + "/history.dat").c_str(), "a");
      if (h) {
        std::fprintf(h, "%d\t%11.4e\n", step, err_max);
        std::fclose(h);
      }
      if (!opt.quiet) {
        std::printf("\n%38s    converged to: %11.4e\n", "rho", res[0]);
        std::printf("  n=%8d,                       V     converged to: %11.4e   \n", step, res[1]);
        std::printf("  n=%8d,                       p     converged to: %11.4e   \n", step, res[2]);
        std::printf("%38s    converged to: %11.4e\n", "T ", res[3]);
      }
    }
    if (step % out_file == 0 || converged) {
      if (!plt_out_) {
        // Driver::post_process, src/Driver.cu:404-415: label 0, the 2-D wall
        double wall_q = 0;
        for (int p : parameter.get_int_array("post_process"))
          if (p == 0)
            wall_q = 0.5 * parameter.get_real("rho_inf") * parameter.get_real("v_inf") * parameter.get_real("v_inf");
        plt_out_ = std::make_unique<PltPipeline>(E, mesh, field, spec, rans, case_dir, wall_q);
      }
      plt_out_->enqueue(step);
    }
  }
  E.synchronize();
  if (plt_out_) plt_out_->flush();
}

void Driver::write_field(const std::string &path) {
  Engine &E = engine();
  std::vector<std::vector<double>> mach(mesh.n_block), mut(mesh.n_block);
  std::vector<PltBlockData> blocks(mesh.n_block);
  for (int b = 0; b < mesh.n_block; ++b) {
    HostField &F = field[b];
    E.get_field(b, F_BV, F.bv.data(), static_cast<int64_t>(F.bv.size()));
    if (!F.sv.empty()) E.get_field(b, F_SV, F.sv.data(), static_cast<int64_t>(F.sv.size()));
    mach[b].resize(static_cast<size_t>(F.e.size()));
    E.get_field(b, F_MACH, mach[b].data(), F.e.size());
    if (rans) {
      mut[b].resize(static_cast<size_t>(F.e.size()));
      E.get_field(b, F_MUT, mut[b].data(), F.e.size());
    }
    blocks[b] = PltBlockData{&mesh[b], &F, &mach[b], rans ? &mut[b] : nullptr};
  }
  write_plt(path, blocks, spec, rans);
}

}  // namespace ostc
