// Driver of the steady pseudo-time loop: the host side of the reference's
// cfd::Driver<mix, turb> (src/Driver.cuh:12-46, src/Driver.cu:14-415) on
// top of the sm_100a engine.
#pragma once

#include <array>
#include <memory>
#include <string>
#include <vector>

#include "../device/engine.hpp"
#include "boundary.hpp"
#include "chemdata.hpp"
#include "mesh.hpp"
#include "parameter.hpp"

namespace ostc {

class PltPipeline;

struct DriverOptions {
  int device = 0;
  bool quiet = false;
  int precision = 0;  // 0 FP64, 1 FP32-bulk / FP64-critical
  bool exact_inner = false;  // multi-block grids computed as one block (ostc_options::exact_inner)
  int wall_distance = 0;     // ostc_options::wall_distance
};

class Driver {
 public:
  // Reads the case directory and prepares the initial field (the reference's
  // main + Driver constructor, src/main.cu:7-28, src/Driver.cu:14-40).  No
  // GPU work happens here.
  Driver(const std::string &case_dir, const DriverOptions &opt);
  ~Driver();

  // Driver::initialize_computation: creates the engine, uploads the grid and
  // field and runs the initial boundary / exchange / property passes.
  void initialize_computation();
  // Driver::simulate: the steady loop with residual output and .plt output.
  void simulate();
  // Advances n loop iterations (residual cadence of the reference, no file
  // output).  Returns the last err_max or -1 when no residual was due.
  double advance(int n);
  // advance(n) with each step's fields uploaded before it and downloaded
  // after it (Engine::upload_chunked / download_chunked)
  double step_io(int n, int block, const std::vector<int> &fields, const std::vector<double *> &host,
                 int64_t chunk_bytes);

  void write_field(const std::string &path);

  // The autotuner: times every (schedule, flux variant) pair of the engine
  // (Engine::time_stages, `reps` passes each) on this case, applies the
  // fastest and records it in output/message/autotune.txt under a key of the
  // configuration and block sizes; initialize_computation applies a recorded
  // choice whose key matches.  Returns the chosen pair, its time per pass and
  // the time of the default (0, 0).
  struct Tuning {
    int schedule = 0, flux_variant = 0, candidates = 0;
    double ms = 0, ms_default = 0;
  };
  Tuning autotune(int reps);
  std::string tuning_key() const;
  bool initialized() const { return engine_ != nullptr; }
  Engine &engine();

  std::string case_dir;
  DriverOptions opt;
  Parameter parameter;
  Mesh mesh;
  Species spec;
  Reaction reac;
  BcRegistry bc;
  std::vector<HostField> field;
  DevParams dev_params{};
  std::vector<HostBc> host_bcs;
  std::vector<HostInner> host_inner;
  std::vector<double> wall_points;
  int step = 0;
  // whether step `step` computed a residual (step 1 and every
  // output_screen-th step): only then does bv_last hold that step's previous
  // state, so that the residual can be recomputed from the device
  bool last_step_residual = false;
  std::array<double, 4> res{1, 1, 1, 1}, res_scale{1, 1, 1, 1};
  bool rans = false;
  int mix = 0;

 private:
  double compute_residual(int step_no, const double raw[4]);
  void build_dev_params();
  void build_faces();
  std::unique_ptr<Engine> engine_;
  // the .plt output of simulate(), written by a host thread while the next
  // steps run; declared after engine_ so that it is finished first
  std::unique_ptr<PltPipeline> plt_out_;
};

}  // namespace ostc
