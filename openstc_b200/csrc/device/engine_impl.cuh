// Templated engine implementation; included by one .cu file per model
// configuration.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>

#include "engine.hpp"
#include "kernels_mixed.cuh"
#include "kernels_surrogate.cuh"

namespace ostc {

template <class C>
class EngineT final : public Engine {
 public:
  explicit EngineT(const EngineSetup &s) : setup_(s) {
    cuda_check(cudaSetDevice(s.device), "cudaSetDevice");
    cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    if (s.params.ns != C::ns) throw std::runtime_error("engine instantiated for another species count");
    if (static_cast<int>(s.dims.size()) > kMaxBlocks)
      throw std::runtime_error("at most " + std::to_string(kMaxBlocks) + " grid blocks per engine");
    upload_params();
    const bool dplur = s.params.implicit_method == 1;
    const int ngg = s.ngg;
    for (const auto &d : s.dims) {
      DevBlock B{};
      B.mx = d[0];
      B.my = d[1];
      B.mz = d[2];
      B.ngg = ngg;
      B.G = Lay::make(d[0], d[1], d[2], ngg);
      B.D = Lay::make(d[0], d[1], d[2], dplur ? 1 : 0);
      B.Z = Lay::make(d[0], d[1], d[2], 0);
      blocks_.push_back(B);
    }
    for (int b = 0; b < static_cast<int>(blocks_.size()); ++b) allocate(blocks_[b]);
    if (s.exact_inner) mark_exact_inner_faces();
    cuda_check(cudaMalloc(&d_blocks_, sizeof(DevBlock) * blocks_.size()), "cudaMalloc blocks");
    // uploads go through the engine's own (non-blocking) stream: a copy on the
    // legacy default stream from pageable memory may still be in flight when
    // a kernel on this stream starts
    cuda_check(cudaMemcpyAsync(d_blocks_, blocks_.data(), sizeof(DevBlock) * blocks_.size(), cudaMemcpyHostToDevice,
                               stream_),
               "copy blocks");
    // boundary and inner faces
    std::vector<DevBc> bcs;
    for (const auto &h : s.bcs) {
      DevBc d{};
      std::memcpy(&d, &h, sizeof(DevBc));
      bcs.push_back(d);
    }
    static_assert(sizeof(DevBc) == sizeof(HostBc), "DevBc / HostBc layouts differ");
    if (!bcs.empty()) {
      cuda_check(cudaMalloc(&d_bcs_, sizeof(DevBc) * bcs.size()), "cudaMalloc bcs");
      cuda_check(cudaMemcpyAsync(d_bcs_, bcs.data(), sizeof(DevBc) * bcs.size(), cudaMemcpyHostToDevice, stream_),
                 "copy bcs");
      cuda_check(cudaStreamSynchronize(stream_), "copy bcs");
    }
    static_assert(sizeof(DevInner) == sizeof(HostInner), "DevInner / HostInner layouts differ");
    if (!s.inner.empty()) {
      cuda_check(cudaMalloc(&d_inner_, sizeof(DevInner) * s.inner.size()), "cudaMalloc inner");
      cuda_check(cudaMemcpyAsync(d_inner_, s.inner.data(), sizeof(DevInner) * s.inner.size(), cudaMemcpyHostToDevice,
                                 stream_),
                 "copy inner");
    }
    make_all_tiles();
    cuda_check(cudaMalloc(&d_partial_, sizeof(double) * 4 * tiles0_.begin[tiles0_.nblk]), "cudaMalloc partial");
    cuda_check(cudaMalloc(&d_res_, sizeof(double) * 4), "cudaMalloc res");
    cuda_check(cudaMalloc(&d_bad_, sizeof(unsigned int)), "cudaMalloc bad");
    cuda_check(cudaMemset(d_bad_, 0, sizeof(unsigned int)), "memset bad");
    cuda_check(cudaMallocHost(&h_res_, sizeof(double) * 4), "cudaMallocHost res");
    if (!s.wall_points.empty()) {
      build_wall_grid(s.wall_points);
      cuda_check(cudaMalloc(&d_wall_, sizeof(double) * s.wall_points.size()), "cudaMalloc wall");
      cuda_check(cudaMemcpyAsync(d_wall_, s.wall_points.data(), sizeof(double) * s.wall_points.size(),
                                 cudaMemcpyHostToDevice, stream_),
                 "copy wall");
    }
    source_smem_ = C::mix == 2 ? 2 * std::max(1, s.params.nr) * kCta * sizeof(double) : 0;
    flux_smem_ = C::nv * kCta * (C::mixed ? sizeof(float) : sizeof(double));
    col_smem_ = sizeof(double) * ColSmem<C::nv>::size;
    dq0_smem_ = (C::mix == 2 && s.params.chem_src_method == 1) ? sizeof(double) * C::ns * C::ns * kCta : 0;
    if (dq0_smem_ > 48 * 1024)
      cuda_check(cudaFuncSetAttribute(k_dq0<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(dq0_smem_)),
                 "dq0 smem");
    if (col_smem_ > 48 * 1024)
      cuda_check(cudaFuncSetAttribute(k_flux_col<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(col_smem_)),
                 "column flux smem");
    if (source_smem_ > 48 * 1024) {
      if constexpr (C::mixed) {
        cuda_check(cudaFuncSetAttribute(k_source_mx<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(source_smem_)),
                   "smem attribute");
        cuda_check(cudaFuncSetAttribute(k_chem_list<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(source_smem_)),
                   "smem attribute");
      } else {
        cuda_check(cudaFuncSetAttribute(k_source<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(source_smem_)),
                   "smem attribute");
      }
    }
    cuda_check(cudaEventCreate(&ev0_), "event");
    cuda_check(cudaEventCreate(&ev1_), "event");
    for (auto &e : out_ev_) cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    // the cudaMemset / staged copies above ran on the legacy default stream,
    // which the engine's non-blocking stream does not wait for
    cuda_check(cudaDeviceSynchronize(), "engine setup");
  }

  ~EngineT() override {
    // a later engine of this configuration may be allocated at this address:
    // it must not take the parameter block on the device for its own
    if (static_owner() == this) static_owner() = nullptr;
    for (auto &g : graphs_)
      if (g) cudaGraphExecDestroy(g);
    for (void *q : sur_arrays_) cudaFree(q);
    cudaFree(d_fb_count_);
    cudaFree(d_fb_list_);
    cudaFree(d_sur_stats_);
    cudaFree(d_sur_err_);
    cudaFree(d_sur_phase_);
    for (void *p : allocations_) cudaFree(p);
    cudaFree(d_blocks_);
    cudaFree(d_bcs_);
    cudaFree(d_inner_);
    cudaFree(d_partial_);
    cudaFree(d_res_);
    cudaFree(d_bad_);
    cudaFree(d_wall_);
    cudaFreeHost(h_res_);
    cudaEventDestroy(ev0_);
    cudaEventDestroy(ev1_);
    for (auto e : out_ev_) cudaEventDestroy(e);
    cudaFree(d_wall2d_);
    for (auto e : chunk_ev_) cudaEventDestroy(e);
    if (ev_copy_) cudaEventDestroy(ev_copy_);
    if (cin_) cudaStreamDestroy(cin_);
    if (cout_) cudaStreamDestroy(cout_);
    cudaStreamDestroy(stream_);
  }

  // ---- chunked host transfers of the host-driven stepping loop
  void copy_streams() {
    if (cin_) return;
    cuda_check(cudaStreamCreateWithFlags(&cin_, cudaStreamNonBlocking), "copy stream");
    cuda_check(cudaStreamCreateWithFlags(&cout_, cudaStreamNonBlocking), "copy stream");
    cuda_check(cudaEventCreateWithFlags(&ev_copy_, cudaEventDisableTiming), "copy event");
  }

  // the event of chunk c of the k-th field of a call (created on first use)
  cudaEvent_t chunk_event(int k, int64_t c) {
    const size_t slot = static_cast<size_t>(k) * kMaxChunks + static_cast<size_t>(c);
    if (chunk_ev_.size() <= slot) chunk_ev_.resize(slot + 1, nullptr);
    if (!chunk_ev_[slot]) cuda_check(cudaEventCreateWithFlags(&chunk_ev_[slot], cudaEventDisableTiming), "chunk event");
    return chunk_ev_[slot];
  }

  static int64_t chunk_doubles(int64_t count, int64_t chunk_bytes) {
    const int64_t per = std::max<int64_t>(1, chunk_bytes / static_cast<int64_t>(sizeof(double)));
    return std::max<int64_t>(per, (count + kMaxChunks - 1) / kMaxChunks);  // at most kMaxChunks chunks
  }

  void upload_chunked(int b, const int *fields, const double *const *host, int n_fields,
                      int64_t chunk_bytes) override {
    copy_streams();
    upload_params();
    // nothing enqueued on the engine stream so far still reads these arrays
    cuda_check(cudaEventRecord(ev_copy_, stream_), "copy event");
    cuda_check(cudaStreamWaitEvent(cin_, ev_copy_, 0), "copy wait");
    for (int k = 0; k < n_fields; ++k) {
      double *dev = field_ptr(b, fields[k]);
      const int64_t count = field_count(b, fields[k]);
      const int64_t per = chunk_doubles(count, chunk_bytes);
      for (int64_t c = 0, off = 0; off < count; ++c, off += per) {
        const int64_t n = std::min(per, count - off);
        if (downloaded_) cuda_check(cudaStreamWaitEvent(cin_, chunk_event(k, c), 0), "chunk wait");
        cuda_check(cudaMemcpyAsync(dev + off, host[k] + off, sizeof(double) * n, cudaMemcpyHostToDevice, cin_),
                   "chunk upload");
      }
    }
    cuda_check(cudaEventRecord(ev_copy_, cin_), "copy event");
    cuda_check(cudaStreamWaitEvent(stream_, ev_copy_, 0), "copy wait");
  }

  void download_chunked(int b, const int *fields, double *const *host, int n_fields, int64_t chunk_bytes) override {
    copy_streams();
    cuda_check(cudaEventRecord(ev_copy_, stream_), "copy event");
    cuda_check(cudaStreamWaitEvent(cout_, ev_copy_, 0), "copy wait");
    for (int k = 0; k < n_fields; ++k) {
      const double *dev = field_ptr(b, fields[k]);
      const int64_t count = field_count(b, fields[k]);
      const int64_t per = chunk_doubles(count, chunk_bytes);
      for (int64_t c = 0, off = 0; off < count; ++c, off += per) {
        const int64_t n = std::min(per, count - off);
        cuda_check(cudaMemcpyAsync(host[k] + off, dev + off, sizeof(double) * n, cudaMemcpyDeviceToHost, cout_),
                   "chunk download");
        cuda_check(cudaEventRecord(chunk_event(k, c), cout_), "chunk event");
      }
    }
    downloaded_ = true;
  }

  void sync_copies() override {
    if (!cin_) return;
    cuda_check(cudaStreamSynchronize(cout_), "copy sync");
    cuda_check(cudaStreamSynchronize(cin_), "copy sync");
    downloaded_ = false;
  }

  void set_field(int b, int field, const double *host, int64_t count) override {
    double *p = field_ptr(b, field);
    check_count(b, field, count);
    upload_params();
    cuda_check(cudaMemcpyAsync(p, host, sizeof(double) * count, cudaMemcpyHostToDevice, stream_), "set_field");
    if (field == F_METRIC || field == F_JAC || field == F_WALL_DIST) pack_static(b);
    cuda_check(cudaStreamSynchronize(stream_), "set_field sync");
  }

  // the FP32 copy of block b's geometry (FP32-bulk path)
  void pack_static(int b) {
    if constexpr (C::mixed) {
      k_pack32_static<C><<<pack_grid(b), 256, 0, stream_>>>(d_blocks_, b);
      cuda_check(cudaGetLastError(), "pack32 static launch");
    }
  }

  unsigned pack_grid(int b) const {
    return static_cast<unsigned>(std::min<int64_t>((blocks_[b].G.size + 255) / 256, 16 * num_sms_));
  }

  void get_field(int b, int field, double *host, int64_t count) override {
    double *p = field_ptr(b, field);
    check_count(b, field, count);
    cuda_check(cudaMemcpyAsync(host, p, sizeof(double) * count, cudaMemcpyDeviceToHost, stream_), "get_field");
    cuda_check(cudaStreamSynchronize(stream_), "get_field sync");
  }

  void get_field_async(int b, int field, double *host, int64_t count) override {
    double *p = field_ptr(b, field);
    check_count(b, field, count);
    cuda_check(cudaMemcpyAsync(host, p, sizeof(double) * count, cudaMemcpyDeviceToHost, stream_), "get_field_async");
  }

  bool pin_host(void *p, size_t bytes) override {
    if (cudaHostRegister(p, bytes, cudaHostRegisterDefault) == cudaSuccess) return true;
    cudaGetLastError();  // not sticky: clear it so that no later check reports it
    return false;
  }

  void unpin_host(void *p) override { cuda_check(cudaHostUnregister(p), "cudaHostUnregister"); }

  void record_output_event(int slot) override {
    cuda_check(cudaEventRecord(out_ev_[slot & 1], stream_), "output event");
  }

  void wait_output_event(int slot) override {
    cuda_check(cudaSetDevice(setup_.device), "cudaSetDevice");
    cuda_check(cudaEventSynchronize(out_ev_[slot & 1]), "output event wait");
  }

  void wall_friction_heatflux_2d(int b, double dyn_pressure, double *cf, double *qw) override {
    const int mx = blocks_.at(b).mx;
    if (!d_wall2d_) {  // once, for the widest block
      for (const auto &B : blocks_) wall_cap_ = std::max(wall_cap_, B.mx);
      cuda_check(cudaMalloc(&d_wall2d_, sizeof(double) * 2 * wall_cap_), "cudaMalloc wall2d");
    }
    double *dcf = d_wall2d_, *dqw = d_wall2d_ + wall_cap_;
    k_wall_2d<<<(mx + 127) / 128, 128, 0, stream_>>>(d_blocks_, b, dcf, dqw, dyn_pressure);
    cuda_check(cudaGetLastError(), "wall_2d launch");
    cuda_check(cudaMemcpyAsync(cf, dcf, sizeof(double) * mx, cudaMemcpyDeviceToHost, stream_), "wall cf");
    cuda_check(cudaMemcpyAsync(qw, dqw, sizeof(double) * mx, cudaMemcpyDeviceToHost, stream_), "wall qw");
  }

  int64_t field_count(int b, int field) const override {
    const DevBlock &B = blocks_.at(b);
    int nc = 0;
    const Lay &L = layout_of(B, field, nc);
    return field_pointer(B, field) ? L.size * nc : 0;
  }

  void initialize() override {
    upload_params();
    const auto &p = setup_.params;
    if (C::turb && p.rans_model == 2)
    {
      if (wall_grid_.start)
        k_wall_distance_grid<<<grid(tilesg_), block3(), 0, stream_>>>(d_blocks_, tilesg_, wall_grid_);
      else
        k_wall_distance<<<grid(tilesg_), block3(), 0, stream_>>>(d_blocks_, tilesg_, d_wall_,
                                                                static_cast<int>(setup_.wall_points.size() / 3));
    }
    if (p.dim == 2) launch_kcopy();
    launch_bcs();
    k_cv_from_bv<C><<<grid(tilesg_), block3(), 0, stream_>>>(d_blocks_, tilesg_);
    if constexpr (C::turb) k_init_mut<C><<<grid(tiles1_), block3(), 0, stream_>>>(d_blocks_, tiles1_);
    launch_inner();
    launch_props();
    for (int b = 0; b < static_cast<int>(blocks_.size()); ++b) pack_static(b);  // after the wall distance
    cuda_check(cudaGetLastError(), "initialize launch");
    cuda_check(cudaStreamSynchronize(stream_), "initialize");
  }

  void step(bool store_last, bool residual, double res[4]) override {
    upload_params();
    const int key = (store_last ? 1 : 0) + (residual ? 2 : 0);
    if (!graphs_[key]) {
      cudaGraph_t g;
      cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
      enqueue_step(store_last, residual);
      cuda_check(cudaStreamEndCapture(stream_, &g), "end capture");
      cuda_check(cudaGraphInstantiate(&graphs_[key], g, 0), "graph instantiate");
      cudaGraphDestroy(g);
    }
    cuda_check(cudaEventRecord(ev0_, stream_), "event");
    cuda_check(cudaGraphLaunch(graphs_[key], stream_), "graph launch");
    cuda_check(cudaEventRecord(ev1_, stream_), "event");
    if (residual) {
      cuda_check(cudaStreamSynchronize(stream_), "step sync");
      for (int l = 0; l < 4; ++l) res[l] = h_res_[l];
      float ms = 0;
      cudaEventElapsedTime(&ms, ev0_, ev1_);
      last_ms_ = ms;
    }
  }

  void phase(int which) override {
    upload_params();
    switch (which) {
      case 0:
        launch_residual();
        break;
      case 1:
        launch_implicit();
        break;
      case 2:
        launch_update();
        break;
      case 3:
        launch_bcs();
        break;
      case 4:
        launch_exchange();
        break;
      case 5:
        k_store_last<<<grid(tiles0_), block3(), 0, stream_>>>(d_blocks_, tiles0_);
        break;
      case 6:
        launch_source();
        break;
      case 7:
        launch_flux();
        break;
      case 8:
        if (!sur_on_) throw std::runtime_error("no surrogate is set");
        launch_chemistry_split();
        break;
      default:
        throw std::runtime_error("unknown phase");
    }
    cuda_check(cudaGetLastError(), "phase launch");
    cuda_check(cudaStreamSynchronize(stream_), "phase");
  }

  void synchronize() override { cuda_check(cudaStreamSynchronize(stream_), "synchronize"); }

  std::vector<std::tuple<std::string, int, double>> profile_step() override {
    upload_params();
    std::vector<std::pair<const char *, cudaEvent_t>> marks;
    cudaEvent_t start;
    cuda_check(cudaEventCreate(&start), "event");
    cuda_check(cudaEventRecord(start, stream_), "event");
    marks_ = &marks;
    enqueue_step(false, false);
    marks_ = nullptr;
    cuda_check(cudaStreamSynchronize(stream_), "profile sync");
    std::map<std::string, std::pair<int, double>> agg;
    std::vector<std::string> order;
    cudaEvent_t prev = start;
    for (auto &[name, ev] : marks) {
      float ms = 0;
      cudaEventElapsedTime(&ms, prev, ev);
      if (!agg.count(name)) order.push_back(name);
      agg[name].first += 1;
      agg[name].second += ms;
      prev = ev;
    }
    for (auto &m : marks) cudaEventDestroy(m.second);
    cudaEventDestroy(start);
    std::vector<std::tuple<std::string, int, double>> out;
    for (const auto &n : order) out.emplace_back(n, agg[n].first, agg[n].second);
    return out;
  }
  void *stream() override { return stream_; }
  const std::vector<DevBlock> &blocks() const override { return blocks_; }
  double last_step_ms() const override { return last_ms_; }

  int launches_per_step(bool store_last, bool residual) const override {
    const auto &p = setup_.params;
    int n = 2;  // source, flux
    if constexpr (C::mixed) n += (p.dim == 3 ? 2 : 1) + static_cast<int>(blocks_.size());  // pack + one pass per direction
    if (p.implicit_method == 1) {
      n += 1 + p.dplur_inner_step;
    } else if ((C::mix == 2 && p.chem_src_method != 0) || (C::turb && p.turb_implicit == 1)) {
      n += 1;
    }
    n += 2;  // update, limiter
    n += static_cast<int>(setup_.bcs.size());
    n += static_cast<int>(setup_.inner.size());
    if (p.dim == 2) n += static_cast<int>(blocks_.size());
    n += 1;  // properties
    if (store_last) n += 1;
    if (residual) n += 2;
    if (sur_on_) n += (C::mixed ? 5 : 3) * static_cast<int>(blocks_.size());  // candidates, inference, judge (+ chemistry list)
    if (setup_.exact_inner) {  // the halo copies of exact inner faces
      int sets = 2;  // mu_t / lambda_t, |V|
      if (p.implicit_method == 1) sets += 2 + p.dplur_inner_step;  // spectral radii, enthalpies, each sweep's input
      n += sets * static_cast<int>(setup_.inner.size());
    }
    return n;
  }

 private:
  static const void *&static_owner() {
    static const void *owner = nullptr;
    return owner;
  }

  void upload_params() {
    // The __constant__ parameter block is per translation unit and per
    // device; re-upload when another engine of this configuration ran last.
    const void *&owner = static_owner();
    if (owner != this) {
      cuda_check(cudaMemcpyToSymbolAsync(cP, &setup_.params, sizeof(DevParams), 0, cudaMemcpyHostToDevice, stream_),
                 "upload params");
      if constexpr (C::mix == 2) {
        const sur::JudgeTables jt = sur::make_judge_tables(setup_.params);
        cuda_check(cudaMemcpyToSymbolAsync(sur::cJ, &jt, sizeof(jt), 0, cudaMemcpyHostToDevice, stream_),
                   "upload judge tables");
        cuda_check(cudaStreamSynchronize(stream_), "upload judge tables");
      }
      if constexpr (C::mixed) {
        const MixParams f = make_mix_params(setup_.params);
        cuda_check(cudaMemcpyToSymbolAsync(cF, &f, sizeof(MixParams), 0, cudaMemcpyHostToDevice, stream_),
                   "upload float params");
        cuda_check(cudaStreamSynchronize(stream_), "upload float params");
      }
      owner = this;
    }
  }

  double *&field_pointer(DevBlock &B, int f) const {
    switch (f) {
      case F_X: return B.x;
      case F_Y: return B.y;
      case F_Z: return B.z;
      case F_JAC: return B.jac;
      case F_METRIC: return B.metric;
      case F_WALL_DIST: return B.wall_dist;
      case F_BV: return B.bv;
      case F_SV: return B.sv;
      case F_CV: return B.cv;
      case F_VEL: return B.vel;
      case F_ACOUSTIC: return B.acoustic;
      case F_MACH: return B.mach;
      case F_MUL: return B.mul;
      case F_CONDUCTIVITY: return B.cond;
      case F_RHO_D: return B.rho_d;
      case F_GAMMA: return B.gamma;
      case F_CP: return B.cp;
      case F_MUT: return B.mut;
      case F_TURB_COND: return B.turb_cond;
      case F_CHEM_JAC: return B.chem_jac;
      case F_TURB_SRC_JAC: return B.turb_src_jac;
      case F_DQ: return B.dq;
      case F_DQ0: return B.dq0;
      case F_DQK: return B.dqk;
      case F_INV_SPEC: return B.inv_spec;
      case F_VISC_SPEC: return B.visc_spec;
      case F_DT_LOCAL: return B.dt_local;
      case F_BV_LAST: return B.bv_last;
      default: throw std::runtime_error("unknown field id " + std::to_string(f));
    }
  }
  double *field_pointer(const DevBlock &B, int f) const { return field_pointer(const_cast<DevBlock &>(B), f); }

  const Lay &layout_of(const DevBlock &B, int f, int &nc) const {
    const auto &p = setup_.params;
    nc = 1;
    switch (f) {
      case F_METRIC: nc = 9; return B.G;
      case F_BV: nc = 6; return B.G;
      case F_SV: nc = C::nsc; return B.G;
      case F_CV: nc = C::nv; return B.G;
      case F_RHO_D: nc = C::ns; return B.G;
      case F_CHEM_JAC: nc = p.chem_src_method == 2 ? C::ns : C::ns * C::ns; return B.Z;
      case F_TURB_SRC_JAC: nc = 2; return B.Z;
      case F_DQ: case F_DQ0: case F_DQK: nc = C::nv; return B.D;
      case F_INV_SPEC: nc = 3; return B.D;
      case F_VISC_SPEC: return B.D;
      case F_DT_LOCAL: return B.Z;
      case F_BV_LAST: nc = 4; return B.Z;
      default: return B.G;
    }
  }

  void allocate(DevBlock &B) {
    const auto &p = setup_.params;
    for (int f = 0; f < F_N_FIELDS; ++f) {
      int nc = 1;
      const Lay &L = layout_of(B, f, nc);
      bool need = nc > 0;
      if (f == F_RHO_D || f == F_GAMMA || f == F_CP) need = need && (C::ns > 0 || f != F_RHO_D);
      if (f == F_CHEM_JAC) need = C::mix == 2 && p.chem_src_method != 0;
      if (f == F_TURB_SRC_JAC || f == F_MUT || f == F_TURB_COND || f == F_WALL_DIST) need = C::turb;
      if (f == F_DQ0 || f == F_DQK) need = p.implicit_method == 1;
      double *&ptr = field_pointer(B, f);
      ptr = nullptr;
      if (!need) continue;
      const size_t bytes = sizeof(double) * static_cast<size_t>(L.size) * nc;
      void *q = nullptr;
      cuda_check(cudaMalloc(&q, bytes), "cudaMalloc field");
      cuda_check(cudaMemset(q, 0, bytes), "memset field");
      allocations_.push_back(q);
      ptr = static_cast<double *>(q);
    }
    B.h_spec = nullptr;
    B.h_spec32 = B.inv_spec32 = nullptr;
    if (C::mix != 0 && p.implicit_method == 1 && !C::mixed) {
      void *q = nullptr;
      const size_t bytes = sizeof(double) * static_cast<size_t>(B.D.size) * C::ns;
      cuda_check(cudaMalloc(&q, bytes), "cudaMalloc h_spec");
      cuda_check(cudaMemset(q, 0, bytes), "memset h_spec");
      allocations_.push_back(q);
      B.h_spec = static_cast<double *>(q);
    }
    if (C::mixed && p.implicit_method == 1) {
      auto falloc = [&](int n) {
        void *q = nullptr;
        const size_t bytes = sizeof(float) * static_cast<size_t>(B.D.size) * n;
        cuda_check(cudaMalloc(&q, bytes), "cudaMalloc fp32 spectra");
        cuda_check(cudaMemset(q, 0, bytes), "memset fp32 spectra");
        allocations_.push_back(q);
        return static_cast<float *>(q);
      };
      if (C::mix != 0) B.h_spec32 = falloc(C::ns);
      B.inv_spec32 = falloc(3);
    }
    for (auto &f : B.dqf) f = nullptr;
    if (C::mixed && p.implicit_method == 1) {
      for (auto &f : B.dqf) {
        void *q = nullptr;
        const size_t bytes = sizeof(float) * static_cast<size_t>(B.D.size) * C::nv;
        cuda_check(cudaMalloc(&q, bytes), "cudaMalloc dqf");
        cuda_check(cudaMemset(q, 0, bytes), "memset dqf");
        allocations_.push_back(q);
        f = static_cast<float *>(q);
      }
    }
    B.f32 = nullptr;
    if constexpr (C::mixed) {
      void *q = nullptr;
      const size_t bytes = sizeof(float) * static_cast<size_t>(B.G.size) * fp32::F32<C>::count;
      cuda_check(cudaMalloc(&q, bytes), "cudaMalloc f32");
      cuda_check(cudaMemset(q, 0, bytes), "memset f32");
      allocations_.push_back(q);
      B.f32 = static_cast<float *>(q);
    }
    B.lu_piv = nullptr;
    if (C::mix == 2 && p.chem_src_method == 1) {
      void *q = nullptr;
      const size_t bytes = static_cast<size_t>(B.Z.size) * C::ns;
      cuda_check(cudaMalloc(&q, bytes), "cudaMalloc piv");
      cuda_check(cudaMemset(q, 0, bytes), "memset piv");
      allocations_.push_back(q);
      B.lu_piv = static_cast<unsigned char *>(q);
    }
  }

  double *field_ptr(int b, int f) {
    if (b < 0 || b >= static_cast<int>(blocks_.size())) throw std::runtime_error("block index out of range");
    double *p = field_pointer(blocks_[b], f);
    if (!p) throw std::runtime_error("field " + std::to_string(f) + " is not allocated in this configuration");
    return p;
  }

  void check_count(int b, int f, int64_t count) const {
    if (count != field_count(b, f))
      throw std::runtime_error("field " + std::to_string(f) + " holds " + std::to_string(field_count(b, f)) +
                               " values, caller passed " + std::to_string(count));
  }

  // A tile table over every block: count(B, ntx, nty) gives block B's tiles
  // in x and y and returns its total; blocks laid out in order_ (the
  // schedule), cbegin in block order.
  template <class Count>
  Tiles build_tiles(Count &&count, int halo = 0) const {
    Tiles t{};
    t.nblk = static_cast<int>(blocks_.size());
    t.halo = halo;
    int n[kMaxBlocks] = {};
    int acc = 0;
    for (int b = 0; b < t.nblk; ++b) {
      n[b] = count(blocks_[b], t.ntx[b], t.nty[b]);
      t.cbegin[b] = acc;
      acc += n[b];
    }
    acc = 0;
    for (int s = 0; s < t.nblk; ++s) {
      const int b = order_.empty() ? s : order_[s];
      t.block[s] = b;
      t.begin[s] = acc;
      acc += n[b];
    }
    t.begin[t.nblk] = acc;
    return t;
  }

  // the tiles of direction pass d of the FP32-bulk flux (dir_tile_counts)
  Tiles make_dir_tiles(int d) const {
    const int march = kFluxVariant[flux_variant_].march;
    return build_tiles([d, march](const DevBlock &B, int &ntx, int &nty) {
      int n2 = 0;
      dir_tile_counts(d, march, B.mx, B.my, B.mz, ntx, nty, n2);
      return ntx * nty * n2;
    });
  }

  // columns of kTX x kTY cells over kFluxKC planes (the k-marching flux kernel)
  Tiles make_col_tiles() const {
    return build_tiles([](const DevBlock &B, int &ntx, int &nty) {
      ntx = (B.mx + kTX - 1) / kTX;
      nty = (B.my + kTY - 1) / kTY;
      return ntx * nty * ((B.mz + kFluxKC - 1) / kFluxKC);
    });
  }

  Tiles make_tiles(int halo) const {
    return build_tiles(
        [halo](const DevBlock &B, int &ntx, int &nty) {
          ntx = (B.mx + 2 * halo + kTX - 1) / kTX;
          nty = (B.my + 2 * halo + kTY - 1) / kTY;
          return ntx * nty * ((B.mz + 2 * halo + kTZ - 1) / kTZ);
        },
        halo);
  }

  void make_all_tiles() {
    tiles0_ = make_tiles(0);
    tiles1_ = make_tiles(1);
    tilesg_ = make_tiles(setup_.ngg);
    col_tiles_ = make_col_tiles();
    for (int d = 0; d < 3; ++d) dir_tiles_[d] = make_dir_tiles(d);
  }

  static dim3 grid(const Tiles &t) { return dim3(static_cast<unsigned>(t.begin[t.nblk])); }
  static dim3 block3() { return dim3(kTX, kTY, kTZ); }

  void launch_source() {
    if constexpr (C::mixed) {
      k_source_mx<C><<<grid(tiles0_), block3(), source_smem_, stream_>>>(d_blocks_, tiles0_);
      if constexpr (C::mix == 2) {
        if (sur_on_) {
          // the chemistry of the cells the surrogate did not take, compacted
          // (the candidate list of this step's inference is no longer needed)
          for (int b = 0; b < static_cast<int>(blocks_.size()); ++b) {
            const DevBlock &B = blocks_[b];
            const int64_t cells = static_cast<int64_t>(B.mx) * B.my * B.mz;
            cuda_check(cudaMemsetAsync(d_fb_count_, 0, sizeof(int), stream_), "memset chemistry list");
            const unsigned cgrid = static_cast<unsigned>(std::min<int64_t>((cells + 255) / 256, 8 * num_sms_));
            k_chem_compact<C><<<cgrid, 256, 0, stream_>>>(d_blocks_, b, d_fb_list_, d_fb_count_);
            const unsigned lgrid = static_cast<unsigned>((cells + kCta - 1) / kCta);
            k_chem_list<C><<<lgrid, kCta, source_smem_, stream_>>>(d_blocks_, b, d_fb_list_, d_fb_count_);
          }
        }
      }
    } else {
      k_source<C><<<grid(tiles0_), block3(), source_smem_, stream_>>>(d_blocks_, tiles0_);
    }
  }

  void launch_flux() {
    if constexpr (C::mixed) {
      for (int b = 0; b < static_cast<int>(blocks_.size()); ++b)
        k_pack32<C><<<pack_grid(b), 256, 0, stream_>>>(d_blocks_, b);
      mark("pack32");
      switch (flux_variant_) {
        case 0: launch_flux_passes<kFluxVariant[0].min_blocks, kFluxVariant[0].march>(); break;
        case 1: launch_flux_passes<kFluxVariant[1].min_blocks, kFluxVariant[1].march>(); break;
        case 2: launch_flux_passes<kFluxVariant[2].min_blocks, kFluxVariant[2].march>(); break;
        default: launch_flux_passes<kFluxVariant[3].min_blocks, kFluxVariant[3].march>(); break;
      }
    } else if (flux_variant_ == 1) {
      // the per-cell form: each face evaluated by both of its cells, no barriers
      k_flux<C><<<grid(tiles0_), block3(), flux_smem_, stream_>>>(d_blocks_, tiles0_);
    } else {
      k_flux_col<C><<<grid(col_tiles_), kFluxThreads, col_smem_, stream_>>>(d_blocks_, col_tiles_);
    }
  }

  template <int MINB, int MARCH>
  void launch_flux_passes() {
    k_flux_x<C, MINB><<<grid(dir_tiles_[0]), kCta, 0, stream_>>>(d_blocks_, dir_tiles_[0]);
    mark("flux_x");
    k_flux_march<C, 1, MINB, MARCH><<<grid(dir_tiles_[1]), kCta, 0, stream_>>>(d_blocks_, dir_tiles_[1]);
    mark("flux_y");
    if (setup_.params.dim == 3) {
      k_flux_march<C, 2, MINB, MARCH><<<grid(dir_tiles_[2]), kCta, 0, stream_>>>(d_blocks_, dir_tiles_[2]);
      mark("flux_z");
    }
  }

  void launch_props() {
    if constexpr (C::mixed)
      k_props_mx<C><<<grid(tiles1_), block3(), 0, stream_>>>(d_blocks_, tiles1_);
    else
      k_props<C><<<grid(tiles1_), block3(), 0, stream_>>>(d_blocks_, tiles1_);
  }

  // the surrogate marks chemically quiet cells before the source term
  void launch_classify() {
    if constexpr (C::mix == 2) {
      for (int b = 0; b < static_cast<int>(blocks_.size()); ++b) {
        const DevBlock &B = blocks_[b];
        const int64_t cells = static_cast<int64_t>(B.mx) * B.my * B.mz;
        // the cells to evaluate (quiet last step, plus a rotating 1/kRecheckEvery)
        cuda_check(cudaMemsetAsync(d_fb_count_, 0, sizeof(int), stream_), "memset candidates");
        const unsigned cgrid = static_cast<unsigned>(std::min<int64_t>((cells + 255) / 256, 8 * num_sms_));
        sur::k_sur_candidates<C><<<cgrid, 256, 0, stream_>>>(d_blocks_, b, sur::kRecheckEvery, d_sur_phase_,
                                                             d_fb_list_, d_fb_count_, d_sur_stats_);
        auto *fn = sur_.n_elem <= 3 ? sur::k_sur_infer<C, 1, 3> : sur::k_sur_infer<C, 1, 4>;
        const int64_t tiles = (cells + sur::kCells - 1) / sur::kCells;
        const bool last = b + 1 == static_cast<int>(blocks_.size());
        fn<<<static_cast<unsigned>(std::min<int64_t>(tiles, num_sms_)), sur::kThreads, sur::kSmem, stream_>>>(
            d_blocks_, b, sur_, d_fb_count_, d_fb_list_, d_sur_stats_, d_sur_err_, d_fb_list_, d_fb_count_,
            last ? d_sur_phase_ : nullptr);
        mark("surrogate");
        sur::k_sur_judge<C><<<static_cast<unsigned>(8 * num_sms_), sur::kJudgeCta, 0, stream_>>>(d_blocks_, b, sur_.gate,
                                                                                     d_fb_list_, d_fb_count_,
                                                                                     d_sur_stats_);
        mark("surrogate_judge");
      }
    }
  }

  void launch_residual() {
    if (sur_on_) launch_classify();
    launch_source();
    mark("source");
    launch_halo(kHaloTurb);
    launch_flux();
    if constexpr (!C::mixed) mark("flux");
    launch_halo(kHaloSpec);
  }

  // returns the dq buffer holding the final increment (0 dq, 1 dq0, 2 dqk)
  int launch_implicit() {
    const auto &p = setup_.params;
    if (p.implicit_method == 1) {
      k_dq0<C><<<grid(tiles0_), block3(), dq0_smem_, stream_>>>(d_blocks_, tiles0_);
      mark("dq0");
      if constexpr (C::mixed) {
        // FP32 increments dqf[0] (dq0) -> dqf[1] -> dqf[2] -> ..., the last
        // sweep into the FP64 dq (k_dq0 writes the FP64 dq0 when there is no sweep)
        int in = 0;
        for (int s = 0; s < p.dplur_inner_step; ++s) {
          const int out = s + 1 == p.dplur_inner_step ? -1 : (s % 2 == 0 ? 1 : 2);
          k_sweep_mx<C><<<grid(tiles0_), block3(), 0, stream_>>>(d_blocks_, tiles0_, in, out);
          mark("dplur_sweep");
          in = out;
        }
        final_dq_ = p.dplur_inner_step > 0 ? 0 : 1;
      } else {
        int in = 1;
        launch_halo(kHaloHspec);
        for (int s = 0; s < p.dplur_inner_step; ++s) {
          const int out = (s % 2 == 0) ? 2 : 0;
          launch_halo(kHaloDq, in);
          k_sweep<C><<<grid(tiles0_), block3(), 0, stream_>>>(d_blocks_, tiles0_, in, out);
          mark("dplur_sweep");
          in = out;
        }
        final_dq_ = in;
      }
    } else {
      if ((C::mix == 2 && p.chem_src_method != 0) || (C::turb && p.turb_implicit == 1))
        k_point_implicit<C><<<grid(tiles0_), block3(), 0, stream_>>>(d_blocks_, tiles0_);
        mark("point_implicit");
      final_dq_ = 0;
    }
    return final_dq_;
  }

  void set_surrogate(const SurrogateDev *p) override {
    if constexpr (C::mix != 2) {
      if (p) throw std::runtime_error("the chemistry surrogate needs a finite-rate chemistry case");
    } else {
      if (p && setup_.params.ns != kSurOut) throw std::runtime_error("the surrogate is built for 9 species");
      if (p && p->n_elem > sur::kFusedElem)
        throw std::runtime_error("the fused surrogate kernel handles mechanisms of at most 4 elements");
      sur_on_ = p != nullptr;
      if (p) sur_ = *p;
      if (sur_on_ && !d_fb_count_) {
        int64_t most = 0;
        for (const auto &B : blocks_) most = std::max<int64_t>(most, static_cast<int64_t>(B.mx) * B.my * B.mz);
        cuda_check(cudaMalloc(&d_fb_count_, sizeof(int)), "cudaMalloc fallback count");
        cuda_check(cudaMalloc(&d_fb_list_, sizeof(int) * most), "cudaMalloc fallback list");
        cuda_check(cudaMalloc(&d_sur_stats_, 3 * sizeof(unsigned long long)), "cudaMalloc surrogate stats");
        cuda_check(cudaMalloc(&d_sur_err_, sizeof(int)), "cudaMalloc surrogate err");
        cuda_check(cudaMemset(d_sur_err_, 0, sizeof(int)), "memset surrogate err");
        cuda_check(cudaMalloc(&d_sur_phase_, sizeof(int)), "cudaMalloc surrogate phase");
        cuda_check(cudaMemset(d_sur_phase_, 0, sizeof(int)), "memset surrogate phase");
        for (auto *fn : {sur::k_sur_infer<C, 0, 3>, sur::k_sur_infer<C, 1, 3>, sur::k_sur_infer<C, 0, 4>,
                         sur::k_sur_infer<C, 1, 4>})
          cuda_check(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sur::kSmem)),
                     "surrogate smem");
        // the persistent inference kernel runs one CTA per SM
        cuda_check(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, setup_.device), "SM count");
        const int fb_smem = static_cast<int>(2 * std::max(1, setup_.params.nr) * 128 * sizeof(double));
        if (fb_smem > 48 * 1024)
          cuda_check(cudaFuncSetAttribute(sur::k_sur_fallback<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, fb_smem),
                     "fallback smem");
      }
      if (sur_on_) cuda_check(cudaMemset(d_sur_stats_, 0, 3 * sizeof(unsigned long long)), "memset stats");
      for (auto &B : blocks_) {
        if (sur_on_ && !B.chem_quiet) {
          void *q = nullptr;
          cuda_check(cudaMalloc(&q, static_cast<size_t>(B.Z.size)), "cudaMalloc quiet");
          cuda_check(cudaMemset(q, 0, static_cast<size_t>(B.Z.size)), "memset quiet");
          sur_arrays_.push_back(q);
          quiet_store_.push_back(static_cast<unsigned char *>(q));
          cuda_check(cudaMalloc(&q, sizeof(double) * B.Z.size * C::ns), "cudaMalloc rate");
          sur_arrays_.push_back(q);
          rate_store_.push_back(static_cast<double *>(q));
        }
      }
      for (size_t b = 0; b < blocks_.size(); ++b) {
        blocks_[b].chem_quiet = sur_on_ ? quiet_store_.at(b) : nullptr;
        blocks_[b].chem_rate = sur_on_ ? rate_store_.at(b) : nullptr;
      }
      cuda_check(cudaMemcpyAsync(d_blocks_, blocks_.data(), sizeof(DevBlock) * blocks_.size(), cudaMemcpyHostToDevice,
                                 stream_),
                 "copy blocks");
    }
    // the step graphs and the parameter block change
    for (auto &g : graphs_)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
    static_owner() = nullptr;
    upload_params();
    // the cudaMemset calls above ran on the legacy default stream
    cuda_check(cudaDeviceSynchronize(), "surrogate setup");
  }

  void surrogate_stats(unsigned long long out[3]) override {
    out[0] = out[1] = out[2] = 0;
    if (!d_sur_stats_) return;
    int err = 0;
    cuda_check(cudaMemcpyAsync(out, d_sur_stats_, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream_),
               "stats");
    cuda_check(cudaMemcpyAsync(&err, d_sur_err_, sizeof(int), cudaMemcpyDeviceToHost, stream_), "surrogate err");
    cuda_check(cudaStreamSynchronize(stream_), "stats");
    if (err) throw std::runtime_error("CUDA error in the surrogate kernel: a tensor-core wait timed out");
  }

  // surrogate increments with the trust gate, then the EPI fallback
  void launch_chemistry_split() {
    if constexpr (C::mix == 2) {
      const int fb_smem = static_cast<int>(2 * std::max(1, setup_.params.nr) * 128 * sizeof(double));
      for (int b = 0; b < static_cast<int>(blocks_.size()); ++b) {
        const DevBlock &B = blocks_[b];
        const int64_t cells = static_cast<int64_t>(B.mx) * B.my * B.mz;
        cuda_check(cudaMemsetAsync(d_fb_count_, 0, sizeof(int), stream_), "memset fallback");
        auto *fn = sur_.n_elem <= 3 ? sur::k_sur_infer<C, 0, 3> : sur::k_sur_infer<C, 0, 4>;
        const int64_t tiles = (cells + sur::kCells - 1) / sur::kCells;
        fn<<<static_cast<unsigned>(std::min<int64_t>(tiles, num_sms_)), sur::kThreads, sur::kSmem, stream_>>>(
            d_blocks_, b, sur_, d_fb_count_, d_fb_list_, d_sur_stats_, d_sur_err_, nullptr, nullptr, nullptr);
        mark("surrogate");
        sur::k_sur_fallback<C><<<148 * 4, 128, fb_smem, stream_>>>(d_blocks_, b, d_fb_count_, d_fb_list_);
        mark("epi_fallback");
      }
    }
  }

  void launch_update() {
    cuda_check(cudaMemsetAsync(d_bad_, 0, sizeof(unsigned int), stream_), "memset bad");
    mark("memset");
    k_update<C><<<grid(tiles0_), block3(), 0, stream_>>>(d_blocks_, tiles0_, final_dq_, d_bad_);
    mark("update");
    k_limit<C><<<grid(tiles0_), block3(), 0, stream_>>>(d_blocks_, tiles0_, d_bad_);
    mark("limit_flow");
  }

  void launch_bcs() {
    for (int q = 0; q < static_cast<int>(setup_.bcs.size()); ++q) {
      const HostBc &f = setup_.bcs[q];
      const int np = (f.end[0] - f.start[0] + 1) * (f.end[1] - f.start[1] + 1) * (f.end[2] - f.start[2] + 1);
      if (np <= 0) continue;
      k_bc<C><<<(np + 127) / 128, 128, 0, stream_>>>(d_blocks_, d_bcs_, q);
      mark("boundary");
    }
  }

  void launch_inner() {
    for (int q = 0; q < static_cast<int>(setup_.inner.size()); ++q) {
      const HostInner &f = setup_.inner[q];
      if (f.n_point[0] * f.n_point[1] * f.n_point[2] <= 0) continue;
      const int tg = setup_.exact_inner ? setup_.ngg : 0;
      int np = 1;
      for (int d = 0; d < 3; ++d) np *= f.n_point[d] + (d != f.face && f.n_point[d] > 1 ? 2 * tg : 0);
      k_inner<C><<<(np + 127) / 128, 128, 0, stream_>>>(d_blocks_, d_inner_, q, setup_.exact_inner, tg);
      mark("inner_face");
    }
    launch_halo(kHaloVel);
  }

  // exact inner faces: the first ghost layer of one array set copied from the
  // neighbours (k_halo); nothing otherwise
  void launch_halo(int set, int dq_sel = 0) {
    if (!setup_.exact_inner) return;
    // the spectral radii, increments and enthalpies have their ghost layer under DPLUR only
    if (set != kHaloTurb && set != kHaloVel && setup_.params.implicit_method != 1) return;
    for (int q = 0; q < static_cast<int>(setup_.inner.size()); ++q) {
      const HostInner &f = setup_.inner[q];
      const int np = f.n_point[0] * f.n_point[1] * f.n_point[2];
      if (np <= 0) continue;
      k_halo<C><<<(np + 127) / 128, 128, 0, stream_>>>(d_blocks_, d_inner_, q, set, dq_sel);
      mark("halo");
    }
  }

  // The bucket grid of the wall points for k_wall_distance_grid: method 2, or
  // method 0 (automatic) with more than 2048 points; buckets of edge h chosen
  // for about four points per bucket over the points' bounding box.
  void build_wall_grid(const std::vector<double> &w) {
    const int64_t nw = static_cast<int64_t>(w.size() / 3);
    const int method = setup_.wall_distance;
    if (nw == 0 || method == 1 || (method == 0 && nw <= 2048)) return;
    double lo[3], hi[3];
    for (int d = 0; d < 3; ++d) lo[d] = hi[d] = w[d];
    for (int64_t q = 0; q < nw; ++q)
      for (int d = 0; d < 3; ++d) {
        lo[d] = std::min(lo[d], w[3 * q + d]);
        hi[d] = std::max(hi[d], w[3 * q + d]);
      }
    const double ext = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]});
    auto count = [&](double h, int *n) {
      int64_t c = 1;
      for (int d = 0; d < 3; ++d) {
        n[d] = std::max(1, static_cast<int>(std::ceil((hi[d] - lo[d]) / h)));
        c *= n[d];
      }
      return c;
    };
    const int64_t target = std::max<int64_t>(1, std::min<int64_t>(nw / 4, int64_t(1) << 22));
    double h = ext > 0 ? ext : 1.0, a = h * 1e-7;  // count(h) <= target <= count(a)
    int n[3];
    for (int it = 0; it < 80 && ext > 0; ++it) {
      const double m = std::sqrt(a * h);
      if (count(m, n) > target) a = m; else h = m;
    }
    count(h, n);
    const int nb = n[0] * n[1] * n[2];
    std::vector<int> bucket(static_cast<size_t>(nw)), start(static_cast<size_t>(nb) + 1, 0);
    for (int64_t q = 0; q < nw; ++q) {
      int c[3];
      for (int d = 0; d < 3; ++d)
        c[d] = std::min(n[d] - 1, std::max(0, static_cast<int>(std::floor((w[3 * q + d] - lo[d]) / h))));
      bucket[q] = (c[2] * n[1] + c[1]) * n[0] + c[0];
      ++start[bucket[q] + 1];
    }
    for (int b = 0; b < nb; ++b) start[b + 1] += start[b];
    std::vector<int> fill(start.begin(), start.end() - 1);
    std::vector<double> pts(w.size());
    for (int64_t q = 0; q < nw; ++q) {
      const int at = fill[bucket[q]]++;
      for (int d = 0; d < 3; ++d) pts[3 * static_cast<size_t>(at) + d] = w[3 * q + d];
    }
    int *d_start = nullptr;
    double *d_pts = nullptr;
    cuda_check(cudaMalloc(&d_start, sizeof(int) * start.size()), "cudaMalloc wall grid");
    cuda_check(cudaMalloc(&d_pts, sizeof(double) * pts.size()), "cudaMalloc wall grid");
    allocations_.push_back(d_start);
    allocations_.push_back(d_pts);
    cuda_check(cudaMemcpyAsync(d_start, start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice, stream_),
               "copy wall grid");
    cuda_check(cudaMemcpyAsync(d_pts, pts.data(), sizeof(double) * pts.size(), cudaMemcpyHostToDevice, stream_),
               "copy wall grid");
    cuda_check(cudaStreamSynchronize(stream_), "copy wall grid");  // the host vectors go out of scope
    for (int d = 0; d < 3; ++d) {
      wall_grid_.lo[d] = lo[d];
      wall_grid_.hi[d] = hi[d];
      wall_grid_.n[d] = n[d];
    }
    wall_grid_.h = h;
    wall_grid_.start = d_start;
    wall_grid_.pts = d_pts;
  }

  // exact inner faces: the block faces the DPLUR sweeps cross (each inner
  // face must cover its whole block face; FP64 path, 3-D grids)
  void mark_exact_inner_faces() {
    if (C::mixed) throw std::runtime_error("exact inner faces are implemented on the FP64 path only");
    if (setup_.params.dim != 3) throw std::runtime_error("exact inner faces are implemented for 3-D grids");
    for (const HostInner &f : setup_.inner) {
      DevBlock &B = blocks_.at(f.block);
      const int ext[3] = {B.mx, B.my, B.mz};
      for (int q = 0; q < 3; ++q) {
        if (q == f.face) continue;
        if (f.n_point[q] != ext[q])
          throw std::runtime_error("exact inner faces must cover whole block faces (block " + std::to_string(f.block) +
                                   ")");
      }
      B.inner_mask |= 1 << (2 * f.face + (f.direction > 0 ? 1 : 0));
    }
  }

  void launch_kcopy() {
    for (int b = 0; b < static_cast<int>(blocks_.size()); ++b) {
      const DevBlock &B = blocks_[b];
      const int np = (B.mx + 2 * B.ngg) * (B.my + 2 * B.ngg);
      k_kcopy<C><<<(np + 127) / 128, 128, 0, stream_>>>(d_blocks_, b);
      mark("k_copy");
    }
  }

  void launch_exchange() {
    launch_inner();
    if (setup_.params.dim == 2) launch_kcopy();
    launch_props();
    mark("properties");
  }

  void enqueue_step(bool store_last, bool residual) {
    if (store_last) {
      k_store_last<<<grid(tiles0_), block3(), 0, stream_>>>(d_blocks_, tiles0_);
      mark("store_last");
    }
    launch_residual();
    launch_implicit();
    launch_update();
    launch_bcs();
    launch_exchange();
    if (residual) {
      k_res_partial<<<grid(tiles0_), block3(), 0, stream_>>>(d_blocks_, tiles0_, d_partial_);
      k_res_final<<<1, 128, 0, stream_>>>(d_partial_, tiles0_.begin[tiles0_.nblk], d_res_);
      cuda_check(cudaMemcpyAsync(h_res_, d_res_, sizeof(double) * 4, cudaMemcpyDeviceToHost, stream_), "res copy");
    }
    cuda_check(cudaGetLastError(), "step launch");
  }

  int residual_tiles() const override { return tiles0_.begin[tiles0_.nblk]; }

  void set_tuning(int schedule, int flux_variant) override {
    if (schedule < 0 || schedule > 1) throw std::runtime_error("schedule must be 0 or 1");
    if (flux_variant < 0 || flux_variant >= flux_variants()) throw std::runtime_error("no such flux variant");
    synchronize();
    order_.clear();
    if (schedule == 1) {
      for (int b = 0; b < static_cast<int>(blocks_.size()); ++b) order_.push_back(b);
      auto cells = [this](int b) { return static_cast<int64_t>(blocks_[b].mx) * blocks_[b].my * blocks_[b].mz; };
      std::stable_sort(order_.begin(), order_.end(), [&](int a, int b) { return cells(a) > cells(b); });
    }
    flux_variant_ = flux_variant;
    make_all_tiles();
    for (auto &g : graphs_)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  }

  // FP64: 0 the column kernel (faces once), 1 the per-cell kernel
  int flux_variants() const override { return C::mixed ? kFluxVariants : 2; }

  double time_stages(int reps) override {
    upload_params();
    auto pass = [this] {
      launch_source();
      launch_halo(kHaloTurb);
      launch_flux();
      launch_halo(kHaloSpec);
      launch_implicit();
    };
    pass();
    cuda_check(cudaEventRecord(ev0_, stream_), "event");
    for (int r = 0; r < reps; ++r) pass();
    cuda_check(cudaEventRecord(ev1_, stream_), "event");
    cuda_check(cudaGetLastError(), "tuning launch");
    cuda_check(cudaEventSynchronize(ev1_), "tuning sync");
    float ms = 0;
    cuda_check(cudaEventElapsedTime(&ms, ev0_, ev1_), "event time");
    return ms / std::max(1, reps);
  }

  void residual_sums_to(double *partial, double *out) override {
    const int n_part = tiles0_.begin[tiles0_.nblk];
    k_res_partial<<<grid(tiles0_), block3(), 0, stream_>>>(d_blocks_, tiles0_, partial);
    k_res_final<<<1, 128, 0, stream_>>>(partial, n_part, out);
    cuda_check(cudaGetLastError(), "residual launch");
  }

  void mark(const char *name) {
    if (!marks_) return;
    cudaEvent_t e;
    cuda_check(cudaEventCreate(&e), "event");
    cuda_check(cudaEventRecord(e, stream_), "event");
    marks_->emplace_back(name, e);
  }

  std::vector<std::pair<const char *, cudaEvent_t>> *marks_ = nullptr;
  EngineSetup setup_;
  cudaStream_t stream_{};
  std::vector<DevBlock> blocks_;
  DevBlock *d_blocks_ = nullptr;
  DevBc *d_bcs_ = nullptr;
  DevInner *d_inner_ = nullptr;
  double *d_partial_ = nullptr, *d_res_ = nullptr, *h_res_ = nullptr, *d_wall_ = nullptr;
  unsigned int *d_bad_ = nullptr;
  std::vector<void *> allocations_;
  Tiles tiles0_, tiles1_, tilesg_, col_tiles_, dir_tiles_[3];
  std::vector<int> order_;  // the blocks' schedule in every tile table (empty: block order)
  int flux_variant_ = 0;    // kFluxVariant entry of the FP32-bulk flux passes
  WallGrid wall_grid_{};    // the bucket grid of the wall points (start null: brute force)
  size_t source_smem_ = 0, flux_smem_ = 0, col_smem_ = 0, dq0_smem_ = 0;
  int final_dq_ = 0;
  cudaGraphExec_t graphs_[4] = {nullptr, nullptr, nullptr, nullptr};
  bool sur_on_ = false;
  SurrogateDev sur_{};
  int num_sms_ = 148;
  int *d_fb_count_ = nullptr, *d_fb_list_ = nullptr, *d_sur_err_ = nullptr, *d_sur_phase_ = nullptr;
  unsigned long long *d_sur_stats_ = nullptr;
  std::vector<void *> sur_arrays_;
  std::vector<unsigned char *> quiet_store_;
  std::vector<double *> rate_store_;
  cudaEvent_t ev0_{}, ev1_{};
  cudaEvent_t out_ev_[2]{};  // output pipeline slots
  // chunked host transfers (upload_chunked / download_chunked)
  static constexpr int64_t kMaxChunks = 64;  // per field
  cudaStream_t cin_{}, cout_{};
  cudaEvent_t ev_copy_{};
  std::vector<cudaEvent_t> chunk_ev_;
  bool downloaded_ = false;  // chunk events recorded since the last sync_copies
  double *d_wall2d_ = nullptr;  // cf and qw of the 2-D wall post-processing
  int wall_cap_ = 0;
  double last_ms_ = 0;
};

}  // namespace ostc
