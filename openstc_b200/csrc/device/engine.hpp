// Host-side interface of the device engine: device memory for all grid
// blocks, the launch sequence of one pseudo-time step and its CUDA graph.
#pragma once

#include <array>
#include <cstdint>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "surrogate.hpp"

namespace ostc {

// Field identifiers of the C ABI (ostc_field_id in include/openstc_b200.h).
enum FieldId : int {
  F_X = 0, F_Y, F_Z, F_JAC, F_METRIC, F_WALL_DIST, F_BV, F_SV, F_CV, F_VEL, F_ACOUSTIC, F_MACH, F_MUL,
  F_CONDUCTIVITY, F_RHO_D, F_GAMMA, F_CP, F_MUT, F_TURB_COND, F_CHEM_JAC, F_TURB_SRC_JAC, F_DQ, F_DQ0, F_DQK,
  F_INV_SPEC, F_VISC_SPEC, F_DT_LOCAL, F_BV_LAST, F_N_FIELDS
};

struct HostBc {
  int block, type, face, direction;
  int start[3], end[3];
  double density, u, v, w, pressure, temperature, mut;
  double sv[kMaxSpec + 2];
  int isothermal;
  double t_wall;
};

struct HostInner {
  int block, target_block, face, direction;
  int start[3], end[3], loop_dir[3], tstart[3], tloop_dir[3], src_tar[3], n_point[3];
};

struct EngineSetup {
  DevParams params;
  int ngg = 2;
  std::vector<std::array<int, 3>> dims;
  std::vector<HostBc> bcs;        // application order
  std::vector<HostInner> inner;   // application order
  std::vector<double> wall_points;  // x,y,z triples for the wall distance
  int device = 0;
  int precision = 0;  // 0 FP64 (the reference's arithmetic), 1 FP32-bulk / FP64-critical
  bool exact_inner = false;  // inner faces computed as the interior of one block (FP64)
  int wall_distance = 0;     // 0 automatic, 1 brute force (the reference's), 2 bucket search
};

class Engine {
 public:
  virtual ~Engine() = default;
  // Copy a host array (reference layout) into a device field of block b.
  virtual void set_field(int b, int field, const double *host, int64_t count) = 0;
  virtual void get_field(int b, int field, double *host, int64_t count) = 0;
  virtual int64_t field_count(int b, int field) const = 0;
  // Driver::initialize_computation, src/Driver.cu:44-104.
  virtual void initialize() = 0;
  // One pass of the steady loop body; res receives the raw RMS sums when
  // `residual` is set.  Uses a cached CUDA graph per (store, residual).
  virtual void step(bool store_last, bool residual, double res[4]) = 0;
  // Phases for per-kernel parity tests.
  virtual void phase(int which) = 0;
  virtual void synchronize() = 0;
  virtual void *stream() = 0;
  virtual const std::vector<DevBlock> &blocks() const = 0;
  virtual int launches_per_step(bool store_last, bool residual) const = 0;
  // Runs one step eagerly (no graph) with an event after every launch and
  // returns (kernel name, launches, total ms).  Advances the solution.
  virtual std::vector<std::tuple<std::string, int, double>> profile_step() = 0;
  virtual double last_step_ms() const = 0;
  // Number of 32x4x1-cell tiles of the residual reduction (one partial sum
  // per variable per tile).
  virtual int residual_tiles() const = 0;
  // Launches on the engine stream the residual reduction of step(): the sums
  // over interior cells of (current - bv_last)^2 for rho, |V|, p and T, with
  // the per-tile partials in partial[4 * residual_tiles()] and the totals in
  // out[4] (both device memory supplied by the caller).  Same kernels and
  // summation order as the residual of step().
  virtual void residual_sums_to(double *partial, double *out) = 0;
  // Chemistry through the surrogate as a split step after the flow update
  // (nullptr: back to the coupled point-implicit chemistry).  The parameters
  // point into the Surrogate's device memory, which must outlive the use.
  virtual void set_surrogate(const SurrogateDev *p) = 0;
  // cells accepted by the trust gate and cells sent to the EPI fallback
  // since the surrogate was set
  // accepted, sent to the EPI fallback, evaluated by the network
  virtual void surrogate_stats(unsigned long long out[3]) = 0;
  // Output pipeline (.plt written while the next steps run): get_field_async
  // enqueues the device-to-host copy on the engine stream and returns at once
  // (asynchronous for host memory made page-locked by pin_host);
  // record_output_event(slot) marks everything enqueued so far, and
  // wait_output_event(slot), callable from any host thread, blocks until it
  // has run.  Two slots.
  virtual void get_field_async(int b, int field, double *host, int64_t count) = 0;
  virtual bool pin_host(void *p, size_t bytes) = 0;  // false (and no error left behind) if refused
  virtual void unpin_host(void *p) = 0;
  virtual void record_output_event(int slot) = 0;
  virtual void wait_output_event(int slot) = 0;
  // Post-processing 0 of the reference (src/PostProcess.cu:6-48): enqueues
  // the wall skin friction and heat flux of block b (j = 0 wall, mx values
  // each) and their device-to-host copies into cf / qw; the values are there
  // once the next output event (or a synchronize) has passed.
  virtual void wall_friction_heatflux_2d(int b, double dyn_pressure, double *cf, double *qw) = 0;

  // Tuning.  schedule: the order of the blocks in every launch (0 block
  // order, 1 largest block first); flux_variant: the variant of the FP32-bulk
  // flux passes (fp32 kFluxVariant; 0 on the FP64 path).  Neither changes a
  // result.  Drops the captured step graphs.
  virtual void set_tuning(int schedule, int flux_variant) = 0;
  virtual int flux_variants() const = 0;
  // Device time (ms) of one pass of the stages that leave the flow state
  // alone (source, flux, implicit increments), eagerly launched `reps`
  // times after one untimed pass; the state is not advanced.
  virtual double time_stages(int reps) = 0;

  // Host-driven stepping loop (Driver::step_io): whole fields of block b
  // copied in chunks of chunk_bytes on two copy streams of their own.
  // upload_chunked: every chunk waits for the previous download of the same
  // chunk (none before the first), then the engine stream waits for all of
  // them; download_chunked: after everything enqueued on the engine stream,
  // one event per chunk.  Field k of a call is matched with field k of the
  // previous call.  sync_copies waits for both copy streams.
  virtual void upload_chunked(int b, const int *fields, const double *const *host, int n_fields,
                              int64_t chunk_bytes) = 0;
  virtual void download_chunked(int b, const int *fields, double *const *host, int n_fields,
                                int64_t chunk_bytes) = 0;
  virtual void sync_copies() = 0;
};

// Largest grid ostc_driver_residual_noalloc accepts, in residual tiles
// (262144 tiles x 128 cells = 33,554,432 interior cells; the 512x256x224 grid
// has 229,376); its static device scratch holds 4 partial sums per tile plus
// the 4 totals (8 MiB + 32 B).
constexpr int kNoAllocMaxTiles = 262144;

// The residual of the last stored step through the static device scratch of
// residual_noalloc.cu, with no device allocation; `device` is made current
// for the launches and the caller's device restored.  raw receives the four
// sums.  Returns 0; 1 when the grid has more than kNoAllocMaxTiles tiles;
// 2 on a CUDA error (*why: the error's message, valid until the next call on
// this host thread).
int residual_sums_noalloc(Engine &engine, int device, double raw[4], const char **why);

std::unique_ptr<Engine> make_engine(const EngineSetup &setup);

// Sets the message of ostc_last_error() for this host thread; returns code.
int abi_error(int code, const std::string &msg);
const char *abi_last_error();

// Per-configuration factories (one translation unit each).
std::unique_ptr<Engine> make_engine_air_lam(const EngineSetup &);
std::unique_ptr<Engine> make_engine_air_sst(const EngineSetup &);
std::unique_ptr<Engine> make_engine_mix9_lam(const EngineSetup &);
std::unique_ptr<Engine> make_engine_mix9_sst(const EngineSetup &);
std::unique_ptr<Engine> make_engine_fr9_lam(const EngineSetup &);
std::unique_ptr<Engine> make_engine_fr9_sst(const EngineSetup &);
std::unique_ptr<Engine> make_engine_fr9_sst_mixed(const EngineSetup &);

void cuda_check(int err, const char *what);

}  // namespace ostc
