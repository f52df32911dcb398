// Residual of the last residual step without any device allocation, for
// ostc_driver_residual_noalloc (include/openstc_b200.h).
//
// Who cannot allocate: a convergence monitor that polls a running solver
// between steps.  At the largest grids the flow state fills the device (the
// 512x256x224 reacting case holds about 48 GB in FP64, and a host may reserve
// the rest for its own buffers), so a cudaMalloc there can fail; and a
// cudaMalloc/cudaFree pair per poll synchronises the whole device, which
// stalls every other stream the host is running.  This path therefore works
// in a fixed, file-scope device array reserved when the module loads.
//
// The scratch: 4 partial sums per residual tile for at most kNoAllocMaxTiles
// tiles, then the 4 totals: 4 * 262144 * 8 B + 32 B = 8 MiB + 32 B, enough for
// the 512x256x224 grid (229,376 tiles).  Nothing in it has to start at zero:
// every call writes each partial slot it later reads (k_res_partial stores, it
// does not accumulate) and k_res_final overwrites the 4 totals.  Grids with
// more tiles are rejected before any launch.
//
// One scratch serves every driver on a device.  Calls that overlap on the same
// device (two host threads, or two drivers on different streams) race on it
// and can return each other's sums: serialise them.
//
// Set-up: the first successful call on a device looks the scratch up with
// cudaGetSymbolAddress (which may load this module on that device) and caches
// the address for that device; a failed look-up is not cached, the next call
// tries again.  Make the first call on a device before any stream capture
// begins on it.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "engine.hpp"

namespace ostc {

static __device__ __align__(256) double g_noalloc_scratch[4 * kNoAllocMaxTiles + 4];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double *g_addr[kMaxDevices];  // nullptr until a look-up on that device succeeded

// Makes `device` current for the lifetime of the guard and restores the
// caller's device afterwards.
struct DeviceGuard {
  int prev = -1;
  cudaError_t status = cudaSuccess;
  explicit DeviceGuard(int device) {
    status = cudaGetDevice(&prev);
    if (status == cudaSuccess && prev != device) status = cudaSetDevice(device);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// The scratch's device address on the current device (`device`).
cudaError_t scratch_on(int device, double **addr) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_mutex);
  if (g_addr[device] == nullptr) {
    void *p = nullptr;
    const cudaError_t st = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (st != cudaSuccess) {
      cudaGetLastError();  // leave no sticky launch-side error behind; retried on the next call
      return st;
    }
    g_addr[device] = static_cast<double *>(p);
  }
  *addr = g_addr[device];
  return cudaSuccess;
}

}  // namespace

int residual_sums_noalloc(Engine &engine, int device, double raw[4], const char **why) {
  if (engine.residual_tiles() > kNoAllocMaxTiles) return 1;
  DeviceGuard on(device);
  if (on.status != cudaSuccess) {
    *why = cudaGetErrorString(on.status);
    return 2;
  }
  double *scratch = nullptr;
  cudaError_t st = scratch_on(device, &scratch);
  if (st != cudaSuccess || scratch == nullptr) {
    *why = cudaGetErrorString(st == cudaSuccess ? cudaErrorInvalidSymbol : st);
    return 2;
  }
  double *totals = scratch + 4 * static_cast<size_t>(kNoAllocMaxTiles);
  try {
    engine.residual_sums_to(scratch, totals);
  } catch (const std::exception &e) {
    static thread_local std::string msg;
    msg = e.what();
    *why = msg.c_str();
    return 2;
  }
  const cudaStream_t stream = static_cast<cudaStream_t>(engine.stream());
  st = cudaMemcpyAsync(raw, totals, 4 * sizeof(double), cudaMemcpyDeviceToHost, stream);
  if (st == cudaSuccess) st = cudaStreamSynchronize(stream);
  if (st != cudaSuccess) {
    *why = cudaGetErrorString(st);
    return 2;
  }
  return 0;
}

}  // namespace ostc
