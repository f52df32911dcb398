// Chemistry surrogate: data generation with the FP64 EPI step, training with
// the tcgen05 BF16 GEMM, fused tensor-core inference behind a trust gate,
// and the C-ABI entry points.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <algorithm>
#include <random>
#include <stdexcept>
#include <string>

#include "engine.hpp"
#include "kernels_surrogate.cuh"
#include "openstc_b200.h"
#include "surrogate.hpp"
#include "tc_gemm.cuh"

namespace ostc {

// Device-to-host copy ordered after the work on stream_ (a plain cudaMemcpy
// runs on the legacy default stream, which does not wait for this
// non-blocking stream).
#define d2h(dst, src, bytes, what)                                                              \
  do {                                                                                          \
    ck(cudaMemcpyAsync((dst), (src), (bytes), cudaMemcpyDeviceToHost, stream_), what);          \
    ck(cudaStreamSynchronize(stream_), what);                                                   \
  } while (0)

// ------------------------------------------------------------------ GEMM
template <int BN>
static cudaError_t launch_gemm_bn(const uint16_t *A, int lda, const uint16_t *B, int ldb, float *D, int ldd, int M,
                                  int N, int K, int splits, int *err, cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(k_tc_gemm<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(GemmTile<BN>::smem));
  if (e != cudaSuccess) return e;
  const int per = (K + splits - 1) / splits;
  const int kps = (per + kGemmBK - 1) / kGemmBK * kGemmBK;
  const dim3 grid((M + 127) / 128, (N + BN - 1) / BN, splits);
  k_tc_gemm<BN><<<grid, 128, GemmTile<BN>::smem, st>>>(A, lda, B, ldb, D, ldd, M, N, K, kps, err);
  return cudaGetLastError();
}

// D = A * B^T on the tensor cores; with splits > 1, D holds `splits`
// consecutive partial results of M x ldd each.
cudaError_t tc_gemm(const uint16_t *A, int lda, const uint16_t *B, int ldb, float *D, int ldd, int M, int N, int K,
                    int splits, int *err, cudaStream_t st) {
  if (N <= 16) return launch_gemm_bn<16>(A, lda, B, ldb, D, ldd, M, N, K, splits, err, st);
  if (N <= 32) return launch_gemm_bn<32>(A, lda, B, ldb, D, ldd, M, N, K, splits, err, st);
  if (N <= 64) return launch_gemm_bn<64>(A, lda, B, ldb, D, ldd, M, N, K, splits, err, st);
  if (N <= 128) return launch_gemm_bn<128>(A, lda, B, ldb, D, ldd, M, N, K, splits, err, st);
  return launch_gemm_bn<256>(A, lda, B, ldb, D, ldd, M, N, K, splits, err, st);
}

namespace {

using Chem = Cfg<2, 1, 9>;
constexpr int NS = 9;

void ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

// A temporary device array, freed when it leaves scope (an exception from a
// failed check included; cudaFree waits for the work still using it).
template <class T>
struct DevTemp {
  T *p = nullptr;
  DevTemp(size_t count, const char *what) { ck(cudaMalloc(&p, count * sizeof(T)), what); }
  ~DevTemp() { cudaFree(p); }
  DevTemp(const DevTemp &) = delete;
  DevTemp &operator=(const DevTemp &) = delete;
};

__host__ __device__ inline uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__device__ inline double u01(uint64_t &s) {
  s = mix64(s);
  return (static_cast<double>(s >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}
__device__ inline double gauss(uint64_t &s) {
  const double a = u01(s), b = u01(s);
  return sqrt(-2.0 * log(a)) * cos(6.283185307179586 * b);
}

__device__ inline uint16_t bf16(float v) { return __bfloat16_as_ushort(__float2bfloat16_rn(v)); }
__device__ inline float from_bf16(uint16_t v) { return __bfloat162float(__ushort_as_bfloat16(v)); }

// GELU in its tanh form (the inference kernel evaluates the same form with
// the hardware tanh)
__device__ inline float gelu(float x) {
  const float t = tanhf(0.7978845608028654f * (x + 0.044715f * x * x * x));
  return 0.5f * x * (1.f + t);
}
__device__ inline float gelu_grad(float x) {
  const float t = tanhf(0.7978845608028654f * (x + 0.044715f * x * x * x));
  return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * 0.7978845608028654f * (1.f + 3.f * 0.044715f * x * x);
}

// ------------------------------------------------------------------ samples
// T, p, Y[9], dt per sample: from the cells of a flow field (perturbed) or
// uniform in the training box with Dirichlet(1) mass fractions.
__global__ void k_sample(double *states, int64_t n, uint64_t seed, DevBlock F, int use_field, double field_fraction,
                         SurrogateGate g) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  uint64_t s = mix64(seed ^ mix64(static_cast<uint64_t>(i) + 1));
  double T, p, Y[NS];
  double dt = pow(10.0, g.ldt_min + (g.ldt_max - g.ldt_min) * u01(s));
  if (use_field && u01(s) < field_fraction) {
    const int64_t cells = static_cast<int64_t>(F.mx) * F.my * F.mz;
    int64_t c = static_cast<int64_t>(u01(s) * cells);
    if (c >= cells) c = cells - 1;
    const int ci = static_cast<int>(c % F.mx), cj = static_cast<int>((c / F.mx) % F.my),
              ck = static_cast<int>(c / (static_cast<int64_t>(F.mx) * F.my));
    const int64_t m = F.G.at(ci, cj, ck), sz = F.G.size;
    T = F.bv[5 * sz + m] * (1.0 + 0.02 * gauss(s));
    p = F.bv[4 * sz + m] * (1.0 + 0.02 * gauss(s));
    double sum = 0;
    for (int k = 0; k < NS; ++k) {
      Y[k] = fmax(F.sv[k * sz + m], 0.0) * exp(0.1 * gauss(s));
      sum += Y[k];
    }
    for (int k = 0; k < NS; ++k) Y[k] /= sum;
    // the cell's own local time step, perturbed within a factor of 2
    const double dtc = F.dt_local[F.Z.at(ci, cj, ck)];
    if (dtc > 0) dt = dtc * pow(10.0, 0.6 * u01(s) - 0.3);
  } else {
    T = g.t_min + (g.t_max - g.t_min) * u01(s);
    p = pow(10.0, g.lp_min + (g.lp_max - g.lp_min) * u01(s));
    double sum = 0;
    for (int k = 0; k < NS; ++k) {
      Y[k] = -log(u01(s));
      sum += Y[k];
    }
    for (int k = 0; k < NS; ++k) Y[k] /= sum;
  }
  T = fmin(fmax(T, static_cast<double>(g.t_min)), static_cast<double>(g.t_max));
  p = fmin(fmax(p, pow(10.0, static_cast<double>(g.lp_min))), pow(10.0, static_cast<double>(g.lp_max)));
  double *o = states + i * kSurIn;
  o[0] = T;
  o[1] = p;
  for (int k = 0; k < NS; ++k) o[2 + k] = Y[k];
  o[11] = dt;
}

__global__ void __launch_bounds__(128) k_label(const double *states, double *dy, int64_t n) {
  extern __shared__ double sq[];
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const double *s = states + i * kSurIn;
  double Y[NS], d[NS], mw_inv = 0;
  for (int k = 0; k < NS; ++k) {
    Y[k] = s[2 + k];
    mw_inv += Y[k] / cP.mw[k];
  }
  const double rho = s[1] / (kDR_u * s[0] * mw_inv);
  sur::epi_increment<NS>(s[0], rho, Y, s[11], sq + threadIdx.x, sq + cP.nr * blockDim.x + threadIdx.x, blockDim.x, d);
  for (int k = 0; k < NS; ++k) dy[i * NS + k] = d[k];
}

// ------------------------------------------------------------ normalisation
__device__ inline void raw_features(const double *s, float *f) {
  f[0] = static_cast<float>(s[0]);
  f[1] = static_cast<float>(log10(s[1]));
  for (int k = 0; k < NS; ++k) f[2 + k] = static_cast<float>(s[2 + k]);
  f[11] = static_cast<float>(log10(s[11]));
}

// sums of features, squared features and squared labels (double atomics)
__global__ void k_stats(const double *states, const double *dy, int64_t n, double *acc) {
  __shared__ double sh[2 * kSurIn + kSurOut];
  for (int q = threadIdx.x; q < 2 * kSurIn + kSurOut; q += blockDim.x) sh[q] = 0;
  __syncthreads();
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    float f[kSurIn];
    raw_features(states + i * kSurIn, f);
    for (int q = 0; q < kSurIn; ++q) {
      atomicAdd(&sh[q], static_cast<double>(f[q]));
      atomicAdd(&sh[kSurIn + q], static_cast<double>(f[q]) * f[q]);
    }
    for (int q = 0; q < kSurOut; ++q) atomicAdd(&sh[2 * kSurIn + q], dy[i * NS + q] * dy[i * NS + q]);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < 2 * kSurIn + kSurOut; q += blockDim.x) atomicAdd(&acc[q], sh[q]);
}

// features x = (f - mu) / sig; targets t_k = asinh(r_k / c_k) / s_k of the
// relative increments r_k = dY_k / (Y_k + eps) (the signed-log transform tames
// their heavy tail)
struct Norm {
  float mu[kSurIn], sig[kSurIn], c[kSurOut], s[kSurOut];
};

__global__ void k_features(const double *states, const double *dy, int64_t n, Norm nm, uint16_t *x, float *t) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  float f[kSurIn];
  raw_features(states + i * kSurIn, f);
  for (int q = 0; q < kSurInPad; ++q) x[i * kSurInPad + q] = q < kSurIn ? bf16((f[q] - nm.mu[q]) / nm.sig[q]) : 0;
  if (t)
    for (int q = 0; q < kSurOutPad; ++q)
      t[i * kSurOutPad + q] =
          q < kSurOut ? static_cast<float>(asinh(dy[i * NS + q] / (states[i * kSurIn + 2 + q] + kSurYEps) / nm.c[q]) / nm.s[q])
                      : 0.f;
}

// ---------------------------------------------------------------- training
__global__ void k_gather(const uint16_t *x, const float *t, int64_t n_train, uint64_t seed, int batch, uint16_t *a0,
                         uint16_t *a0t, float *tb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= batch) return;
  const int64_t src = static_cast<int64_t>(mix64(seed ^ mix64(static_cast<uint64_t>(i) + 7)) % n_train);
  for (int q = 0; q < kSurInPad; ++q) {
    const uint16_t v = x[src * kSurInPad + q];
    a0[static_cast<int64_t>(i) * kSurInPad + q] = v;
    a0t[static_cast<int64_t>(q) * batch + i] = v;
  }
  for (int q = 0; q < kSurOutPad; ++q) tb[static_cast<int64_t>(i) * kSurOutPad + q] = t[src * kSurOutPad + q];
}

// v = src (+ bias) [mode 0: linear; 1: store pre-activation, out = GELU;
// 2: v = src * GELU'(zpre)]; writes v (FP32, optional), out (bf16 rows x d)
// and its transpose (bf16 d x rows).  Tiles of 32 x 32 through shared memory.
__global__ void k_act(const float *src, int rows, int d, const float *bias, const float *zpre, int mode, float *vout,
                      uint16_t *out, uint16_t *outt) {
  __shared__ uint16_t tile[32][34];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int rr = threadIdx.y; rr < 32; rr += blockDim.y) {
    const int r = r0 + rr, c = c0 + threadIdx.x;
    uint16_t o = 0;
    if (r < rows && c < d) {
      const int64_t idx = static_cast<int64_t>(r) * d + c;
      float v = src[idx];
      float a = v;
      if (mode == 0) {
        if (bias) v += bias[c];
        a = v;
      } else if (mode == 1) {
        v += bias[c];
        a = gelu(v);
      } else {
        v *= gelu_grad(zpre[idx]);
        a = v;
      }
      if (vout) vout[idx] = v;
      o = bf16(a);
      out[idx] = o;
    }
    tile[rr][threadIdx.x] = o;
  }
  __syncthreads();
  for (int cc = threadIdx.y; cc < 32; cc += blockDim.y) {
    const int c = c0 + cc, r = r0 + threadIdx.x;
    if (c < d && r < rows) outt[static_cast<int64_t>(c) * rows + r] = tile[threadIdx.x][cc];
  }
}

// output layer: pred = z + b; loss += mean (pred - t)^2 over 9 outputs;
// dz = 2 (pred - t) / (batch * 9) (padding columns zero)
__global__ void k_out_grad(float *z, const float *b, const float *t, int batch, float *dz, double *loss) {
  __shared__ double sh[256];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double l = 0;
  if (i < batch) {
    for (int q = 0; q < kSurOutPad; ++q) {
      const int64_t idx = static_cast<int64_t>(i) * kSurOutPad + q;
      float g = 0;
      if (q < kSurOut) {
        const float pred = z[idx] + b[q];
        z[idx] = pred;
        const float e = pred - t[idx];
        l += static_cast<double>(e) * e;
        g = 2.f * e / (static_cast<float>(batch) * kSurOut);
      }
      dz[idx] = g;
    }
  }
  sh[threadIdx.x] = l;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, sh[0] / (static_cast<double>(batch) * kSurOut));
}

__global__ void k_colsum(const float *v, int rows, int d, float *out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d) return;
  const int per = (rows + gridDim.y - 1) / gridDim.y;
  const int r0 = blockIdx.y * per, r1 = min(rows, r0 + per);
  float s = 0;
  for (int r = r0; r < r1; ++r) s += v[static_cast<int64_t>(r) * d + c];
  atomicAdd(&out[c], s);
}

__global__ void k_transpose16(const uint16_t *in, int rows, int d, uint16_t *out) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= static_cast<int64_t>(rows) * d) return;
  const int r = static_cast<int>(i / d), c = static_cast<int>(i % d);
  out[static_cast<int64_t>(c) * rows + r] = in[i];
}

__global__ void k_reduce(const float *partial, int splits, int64_t count, float *out) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= count) return;
  float s = 0;
  for (int q = 0; q < splits; ++q) s += partial[q * count + i];
  out[i] = s;
}

__global__ void k_adam(float *p, const float *g, float *m, float *v, int64_t n, float lr, float b1, float b2,
                       float eps, float bc1, float bc2) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1 - b1) * gi, vi = b2 * v[i] + (1 - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

// bf16 copies of a weight [dout x din]: row-major, transposed, and in the
// tile order of the fused inference kernel (K chunks of 16 columns).
__global__ void k_pack(const float *w, int dout, int din, uint16_t *wb, uint16_t *wbt, uint8_t *wp) {
  // wp null: the training GEMMs' copies only
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= static_cast<int64_t>(dout) * din) return;
  const int r = static_cast<int>(i / din), k = static_cast<int>(i % din);
  const uint16_t v = bf16(w[i]);
  wb[i] = v;
  wbt[static_cast<int64_t>(k) * dout + r] = v;
  if (!wp) return;
  const int bk = 16;
  const int c = k / bk, kk = k % bk;
  *reinterpret_cast<uint16_t *>(wp + static_cast<size_t>(c) * dout * bk * 2 + tc::tile_offset(r, kk, bk)) = v;
}

}  // namespace

// ================================================================ Surrogate
Surrogate::Surrogate(const DevParams &chem, const std::vector<int> &elem_comp, int n_elem, int device, uint64_t seed)
    : chem_(chem), elem_comp_(elem_comp), n_elem_(n_elem), device_(device), seed_(seed) {
  if (chem.ns != NS || chem.mix != 2) throw std::runtime_error("the surrogate is built for the 9-species finite-rate mechanism");
  if (n_elem > kMaxElem) throw std::runtime_error("too many elements for the surrogate's conservation gate");
  ck(cudaSetDevice(device), "cudaSetDevice");
  ck(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
  const int dims[kSurLayers + 1] = {kSurInPad, kSurHidden, kSurHidden, kSurHidden, kSurHidden, kSurOutPad};
  std::mt19937_64 rng(seed);
  for (int l = 0; l < kSurLayers; ++l) {
    din_[l] = dims[l];
    dout_[l] = dims[l + 1];
    const size_t nw = static_cast<size_t>(dout_[l]) * din_[l];
    const int fan_in = l == 0 ? kSurIn : din_[l];
    std::normal_distribution<float> nd(0.f, std::sqrt(2.f / fan_in) * (l == kSurLayers - 1 ? 0.5f : 1.f));
    std::vector<float> w(nw, 0.f), b(dout_[l], 0.f);
    const int valid_out = l == kSurLayers - 1 ? kSurOut : dout_[l];
    for (int r = 0; r < valid_out; ++r)
      for (int k = 0; k < fan_in; ++k) w[static_cast<size_t>(r) * din_[l] + k] = nd(rng);
    auto alloc = [&](size_t bytes) {
      void *p = nullptr;
      ck(cudaMalloc(&p, bytes), "cudaMalloc surrogate");
      ck(cudaMemsetAsync(p, 0, bytes, stream_), "memset surrogate");
      allocs_.push_back(p);
      return p;
    };
    w_[l] = static_cast<float *>(alloc(nw * 4));
    b_[l] = static_cast<float *>(alloc(dout_[l] * 4));
    mw_[l] = static_cast<float *>(alloc(nw * 4));
    vw_[l] = static_cast<float *>(alloc(nw * 4));
    mb_[l] = static_cast<float *>(alloc(dout_[l] * 4));
    vb_[l] = static_cast<float *>(alloc(dout_[l] * 4));
    wb_[l] = static_cast<uint16_t *>(alloc(nw * 2));
    wbt_[l] = static_cast<uint16_t *>(alloc(nw * 2));
    wpack_[l] = static_cast<uint8_t *>(alloc(nw * 2));
    ck(cudaMemcpyAsync(w_[l], w.data(), nw * 4, cudaMemcpyHostToDevice, stream_), "upload weights");
    ck(cudaMemcpyAsync(b_[l], b.data(), dout_[l] * 4, cudaMemcpyHostToDevice, stream_), "upload bias");
    ck(cudaStreamSynchronize(stream_), "upload weights");
  }
  void *p = nullptr;
  ck(cudaMalloc(&p, sizeof(double)), "loss");
  allocs_.push_back(p);
  loss_ = static_cast<double *>(p);
  ck(cudaMalloc(&p, sizeof(int)), "err");
  ck(cudaMemsetAsync(p, 0, sizeof(int), stream_), "err");
  allocs_.push_back(p);
  err_ = static_cast<int *>(p);
  for (int q = 0; q < kSurIn; ++q) {
    in_mu[q] = 0.f;
    in_sig[q] = 1.f;
  }
  for (int q = 0; q < kSurOut; ++q) out_s[q] = out_c[q] = 1.f;
  upload_chem();
  pack();
}

Surrogate::~Surrogate() {
  cudaSetDevice(device_);
  for (void *p : allocs_) cudaFree(p);
  cudaFree(states_);
  cudaFree(labels_);
  cudaFree(x_);
  cudaFree(t_);
  cudaStreamDestroy(stream_);
}

// Stream-ordered: a copy on the legacy default stream from pageable memory
// may still be in flight when a kernel on this non-blocking stream starts.
void Surrogate::upload_chem() {
  ck(cudaMemcpyToSymbolAsync(cP, &chem_, sizeof(DevParams), 0, cudaMemcpyHostToDevice, stream_), "upload mechanism");
  const sur::JudgeTables jt = sur::make_judge_tables(chem_);
  ck(cudaMemcpyToSymbolAsync(sur::cJ, &jt, sizeof(jt), 0, cudaMemcpyHostToDevice, stream_), "upload judge tables");
  ck(cudaStreamSynchronize(stream_), "upload judge tables");
}

void Surrogate::pack() {
  for (int l = 0; l < kSurLayers; ++l) {
    const int64_t nw = static_cast<int64_t>(dout_[l]) * din_[l];
    k_pack<<<(nw + 255) / 256, 256, 0, stream_>>>(w_[l], dout_[l], din_[l], wb_[l], wbt_[l], wpack_[l]);
  }
  ck(cudaGetLastError(), "pack weights");
  packed_ = true;
}

static size_t label_smem(const DevParams &p) { return 2 * static_cast<size_t>(p.nr) * 128 * sizeof(double); }

void Surrogate::generate(int64_t n, uint64_t seed, const DevBlock *field, double field_fraction) {
  if (n <= 0) throw std::runtime_error("number of samples must be positive");
  ck(cudaSetDevice(device_), "cudaSetDevice");
  upload_chem();
  cudaFree(states_);
  cudaFree(labels_);
  cudaFree(x_);
  cudaFree(t_);
  states_ = nullptr;
  labels_ = nullptr;
  x_ = nullptr;
  t_ = nullptr;
  ck(cudaMalloc(&states_, n * kSurIn * sizeof(double)), "cudaMalloc samples");
  ck(cudaMalloc(&labels_, n * NS * sizeof(double)), "cudaMalloc labels");
  ck(cudaMalloc(&x_, n * kSurInPad * sizeof(uint16_t)), "cudaMalloc features");
  ck(cudaMalloc(&t_, n * kSurOutPad * sizeof(float)), "cudaMalloc targets");
  n_ = n;
  DevBlock F{};
  if (field) F = *field;
  k_sample<<<(n + 255) / 256, 256, 0, stream_>>>(states_, n, seed, F, field ? 1 : 0, field_fraction, gate);
  ck(cudaGetLastError(), "sample launch");
  const size_t smem = label_smem(chem_);
  ck(cudaFuncSetAttribute(k_label, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)), "smem");
  k_label<<<(n + 127) / 128, 128, smem, stream_>>>(states_, labels_, n);
  ck(cudaGetLastError(), "label launch");
  // normalisation from the data
  DevTemp<double> acc(2 * kSurIn + kSurOut, "cudaMalloc stats");
  ck(cudaMemsetAsync(acc.p, 0, (2 * kSurIn + kSurOut) * sizeof(double), stream_), "memset stats");
  k_stats<<<1184, 256, 0, stream_>>>(states_, labels_, n, acc.p);
  double h[2 * kSurIn + kSurOut];
  ck(cudaMemcpyAsync(h, acc.p, sizeof(h), cudaMemcpyDeviceToHost, stream_), "stats copy");
  ck(cudaStreamSynchronize(stream_), "generate");
  Norm nm{};
  for (int q = 0; q < kSurIn; ++q) {
    const double mu = h[q] / n, var = std::max(h[kSurIn + q] / n - mu * mu, 1e-12);
    in_mu[q] = nm.mu[q] = static_cast<float>(mu);
    in_sig[q] = nm.sig[q] = static_cast<float>(std::sqrt(var));
  }
  {
    // target transform from a sub-sample: c_k = median |r_k|, s_k = RMS of
    // asinh(r_k / c_k), r_k = dY_k / (Y_k + eps)
    const int64_t m = std::min<int64_t>(n, 1 << 18);
    std::vector<double> lab(static_cast<size_t>(m) * NS), st(static_cast<size_t>(m) * kSurIn);
    d2h(lab.data(), labels_, lab.size() * 8, "labels copy");
    d2h(st.data(), states_, st.size() * 8, "states copy");
    for (int64_t i = 0; i < m; ++i)
      for (int q = 0; q < NS; ++q) lab[i * NS + q] /= st[i * kSurIn + 2 + q] + kSurYEps;
    // the trust region in dt follows the data (field samples carry the
    // cells' own local time steps)
    double ldt_lo = 1e30, ldt_hi = -1e30;
    for (int64_t i = 0; i < m; ++i) {
      const double l = std::log10(st[i * kSurIn + 11]);
      ldt_lo = std::min(ldt_lo, l);
      ldt_hi = std::max(ldt_hi, l);
    }
    gate.ldt_min = static_cast<float>(ldt_lo - 0.1);
    gate.ldt_max = static_cast<float>(ldt_hi + 0.1);
    for (int q = 0; q < kSurOut; ++q) {
      std::vector<double> a(static_cast<size_t>(m));
      for (int64_t i = 0; i < m; ++i) a[i] = std::fabs(lab[i * NS + q]);
      std::nth_element(a.begin(), a.begin() + m / 2, a.end());
      const double c = std::max(a[m / 2], 1e-14);
      double ss = 0;
      for (int64_t i = 0; i < m; ++i) {
        const double t = std::asinh(lab[i * NS + q] / c);
        ss += t * t;
      }
      out_c[q] = nm.c[q] = static_cast<float>(c);
      out_s[q] = nm.s[q] = static_cast<float>(std::sqrt(ss / m) + 1e-6);
    }
  }
  k_features<<<(n + 255) / 256, 256, 0, stream_>>>(states_, labels_, n, nm, x_, t_);
  ck(cudaGetLastError(), "features launch");
  ck(cudaStreamSynchronize(stream_), "generate");
}

void Surrogate::ensure_batch(int batch) {
  if (batch == batch_) return;
  if (batch % 128) throw std::runtime_error("batch must be a multiple of 128");
  auto free_ = [](auto *&p) {
    cudaFree(p);
    p = nullptr;
  };
  for (int l = 0; l < kSurLayers; ++l) {
    free_(a_[l]);
    free_(at_[l]);
    free_(z_[l]);
  }
  free_(dz_);
  free_(dzt_);
  free_(dzf_);
  free_(da_);
  free_(partial_);
  free_(gw_);
  free_(gb_);
  free_(tb_);
  const size_t B = static_cast<size_t>(batch);
  for (int l = 0; l < kSurLayers; ++l) {
    ck(cudaMalloc(&a_[l], B * din_[l] * 2), "act");
    ck(cudaMalloc(&at_[l], B * din_[l] * 2), "act t");
    ck(cudaMalloc(&z_[l], B * dout_[l] * 4), "z");
  }
  ck(cudaMalloc(&dz_, B * kSurHidden * 2), "dz");
  ck(cudaMalloc(&dzt_, B * kSurHidden * 2), "dzt");
  ck(cudaMalloc(&dzf_, B * kSurHidden * 4), "dzf");
  ck(cudaMalloc(&da_, B * kSurHidden * 4), "da");
  ck(cudaMalloc(&partial_, 64ull * kSurHidden * kSurHidden * 4), "partial");
  ck(cudaMalloc(&gw_, static_cast<size_t>(kSurHidden) * kSurHidden * 4), "gw");
  ck(cudaMalloc(&gb_, kSurHidden * 4), "gb");
  ck(cudaMalloc(&tb_, B * kSurOutPad * 4), "tb");
  batch_ = batch;
}

// Forward pass of the batch in a_[0]: z_[l] = a_[l] W_l^T + b_l, a_[l+1] = GELU(z_[l]).
void Surrogate::forward(int batch) {
  for (int l = 0; l < kSurLayers; ++l) {
    ck(tc_gemm(a_[l], din_[l], wb_[l], din_[l], z_[l], dout_[l], batch, dout_[l], din_[l], 1, err_, stream_),
       "forward gemm");
    if (l < kSurLayers - 1) {
      const dim3 grid((dout_[l] + 31) / 32, (batch + 31) / 32);
      k_act<<<grid, dim3(32, 8), 0, stream_>>>(z_[l], batch, dout_[l], b_[l], nullptr, 1, z_[l], a_[l + 1], at_[l + 1]);
    }
  }
  ck(cudaGetLastError(), "forward");
}

double Surrogate::backward_and_step(int batch, double lr, int step) {
  ck(cudaMemsetAsync(loss_, 0, sizeof(double), stream_), "loss");
  const int L = kSurLayers - 1;
  k_out_grad<<<(batch + 255) / 256, 256, 0, stream_>>>(z_[L], b_[L], tb_, batch, dzf_, loss_);
  {
    const dim3 grid((kSurOutPad + 31) / 32, (batch + 31) / 32);
    k_act<<<grid, dim3(32, 8), 0, stream_>>>(dzf_, batch, kSurOutPad, nullptr, nullptr, 0, nullptr, dz_, dzt_);
  }
  ++adam_t_;
  const float b1 = 0.9f, b2 = 0.999f;
  const float bc1 = 1.f - std::pow(b1, static_cast<float>(adam_t_)), bc2 = 1.f - std::pow(b2, static_cast<float>(adam_t_));
  const int splits = std::max(1, std::min(64, batch / 1024));
  for (int l = L; l >= 0; --l) {
    const int dout = dout_[l], din = din_[l];
    // dW = dZ^T A  (K = batch, split-K)
    ck(tc_gemm(dzt_, batch, at_[l], batch, partial_, din, dout, din, batch, splits, err_, stream_), "dW gemm");
    const int64_t nw = static_cast<int64_t>(dout) * din;
    k_reduce<<<(nw + 255) / 256, 256, 0, stream_>>>(partial_, splits, nw, gw_);
    ck(cudaMemsetAsync(gb_, 0, dout * 4, stream_), "gb");
    k_colsum<<<dim3((dout + 127) / 128, 64), 128, 0, stream_>>>(dzf_, batch, dout, gb_);
    // dA = dZ W (B operand: W^T rows), then dZ of the layer below
    if (l > 0) {
      ck(tc_gemm(dz_, dout, wbt_[l], dout, da_, din, batch, din, dout, 1, err_, stream_), "dA gemm");
      const dim3 grid((din + 31) / 32, (batch + 31) / 32);
      k_act<<<grid, dim3(32, 8), 0, stream_>>>(da_, batch, din, nullptr, z_[l - 1], 2, dzf_, dz_, dzt_);
    }
    k_adam<<<(nw + 255) / 256, 256, 0, stream_>>>(w_[l], gw_, mw_[l], vw_[l], nw, static_cast<float>(lr), b1, b2,
                                                 1e-8f, bc1, bc2);
    k_adam<<<(dout + 255) / 256, 256, 0, stream_>>>(b_[l], gb_, mb_[l], vb_[l], dout, static_cast<float>(lr), b1, b2,
                                                   1e-8f, bc1, bc2);
  }
  ck(cudaGetLastError(), "backward");
  (void)step;
  return 0;  // the loss accumulates in loss_ on the device
}

double Surrogate::train(int steps, int batch, double lr, int64_t n_train, float *losses) {
  if (n_ == 0) throw std::runtime_error("generate samples before training");
  if (n_train <= 0 || n_train > n_) n_train = n_;
  ck(cudaSetDevice(device_), "cudaSetDevice");
  ensure_batch(batch);
  // each step's loss stays on the device until the end: no host
  // synchronisation between steps
  DevTemp<double> dloss_buf(static_cast<size_t>(std::max(1, steps)), "cudaMalloc losses");
  double *dloss = dloss_buf.p;
  for (int s = 0; s < steps; ++s) {
    k_gather<<<(batch + 255) / 256, 256, 0, stream_>>>(x_, t_, n_train, mix64(seed_ + 0x5151 * (adam_t_ + 1)), batch,
                                                       a_[0], at_[0], tb_);
    forward(batch);
    const double cosine = 0.5 * (1 + std::cos(3.141592653589793 * s / std::max(1, steps)));
    // schedule: cosine decay to 5 % of lr
    const double lr_s = lr * (0.05 + 0.95 * cosine);
    backward_and_step(batch, lr_s, s);
    ck(cudaMemcpyAsync(dloss + s, loss_, sizeof(double), cudaMemcpyDeviceToDevice, stream_), "loss copy");
    // new bf16 weights for the next step's GEMMs (the inference copy once, below)
    for (int l = 0; l < kSurLayers; ++l) {
      const int64_t nw = static_cast<int64_t>(dout_[l]) * din_[l];
      k_pack<<<(nw + 255) / 256, 256, 0, stream_>>>(w_[l], dout_[l], din_[l], wb_[l], wbt_[l], nullptr);
    }
  }
  pack();
  std::vector<double> hl(static_cast<size_t>(std::max(1, steps)), 0.0);
  cudaError_t st = cudaMemcpyAsync(hl.data(), dloss, sizeof(double) * hl.size(), cudaMemcpyDeviceToHost, stream_);
  if (st == cudaSuccess) st = cudaStreamSynchronize(stream_);
  ck(st, "train steps");
  if (losses)
    for (int s = 0; s < steps; ++s) losses[s] = static_cast<float>(hl[s]);
  const double last = steps > 0 ? hl[steps - 1] : 0.0;
  int err = 0;
  d2h(&err, err_, sizeof(int), "err copy");
  if (err) throw std::runtime_error("tensor-core wait timed out during training");
  return last;
}

std::vector<std::vector<float>> Surrogate::params() const {
  std::vector<std::vector<float>> out;
  for (int l = 0; l < kSurLayers; ++l) {
    std::vector<float> w(static_cast<size_t>(dout_[l]) * din_[l]), b(dout_[l]);
    d2h(w.data(), w_[l], w.size() * 4, "params");
    d2h(b.data(), b_[l], b.size() * 4, "params");
    out.push_back(std::move(w));
    out.push_back(std::move(b));
  }
  return out;
}

void Surrogate::set_params(const std::vector<std::vector<float>> &p) {
  if (p.size() != 2 * kSurLayers) throw std::runtime_error("expected weights and biases of 5 layers");
  for (int l = 0; l < kSurLayers; ++l) {
    if (p[2 * l].size() != static_cast<size_t>(dout_[l]) * din_[l] || p[2 * l + 1].size() != static_cast<size_t>(dout_[l]))
      throw std::runtime_error("parameter shape mismatch");
    ck(cudaMemcpyAsync(w_[l], p[2 * l].data(), p[2 * l].size() * 4, cudaMemcpyHostToDevice, stream_), "set params");
    ck(cudaMemcpyAsync(b_[l], p[2 * l + 1].data(), p[2 * l + 1].size() * 4, cudaMemcpyHostToDevice, stream_),
       "set params");
  }
  pack();
  ck(cudaStreamSynchronize(stream_), "set params");
}

// host states -> features on the device
void Surrogate::features(const double *states_dev, int64_t n, uint16_t *x_dev, float *t_dev, const double *dy_dev) {
  Norm nm{};
  for (int q = 0; q < kSurIn; ++q) {
    nm.mu[q] = in_mu[q];
    nm.sig[q] = in_sig[q];
  }
  for (int q = 0; q < kSurOut; ++q) {
    nm.s[q] = out_s[q];
    nm.c[q] = out_c[q];
  }
  k_features<<<(n + 255) / 256, 256, 0, stream_>>>(states_dev, dy_dev, n, nm, x_dev, t_dev);
  ck(cudaGetLastError(), "features");
}

void Surrogate::label_host(const double *states, int64_t n, double *dy) {
  ck(cudaSetDevice(device_), "cudaSetDevice");
  upload_chem();
  DevTemp<double> s_buf(n * kSurIn, "label alloc"), d_buf(n * NS, "label alloc");
  double *s = s_buf.p, *d = d_buf.p;
  ck(cudaMemcpyAsync(s, states, n * kSurIn * 8, cudaMemcpyHostToDevice, stream_), "label upload");
  const size_t smem = label_smem(chem_);
  ck(cudaFuncSetAttribute(k_label, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)), "smem");
  k_label<<<(n + 127) / 128, 128, smem, stream_>>>(s, d, n);
  ck(cudaGetLastError(), "label");
  ck(cudaMemcpyAsync(dy, d, n * NS * 8, cudaMemcpyDeviceToHost, stream_), "label download");
  ck(cudaStreamSynchronize(stream_), "label");
}

namespace {
// decode, project and gate the predictions z (batch x 16, bias added)
__global__ void k_decode(const float *z, const double *states, int64_t n, SurrogateDev gd, double *dy,
                         int *accepted) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const double *s = states + i * kSurIn;
  float o[NS];
  for (int k = 0; k < NS; ++k) o[k] = z[i * kSurOutPad + k];
  double d[NS];
  const bool ok = sur::decode<NS>(gd, o, static_cast<float>(s[0]), log10f(static_cast<float>(s[1])),
                                  log10f(static_cast<float>(s[11])), s + 2, d);
  for (int k = 0; k < NS; ++k) dy[i * NS + k] = d[k];
  accepted[i] = ok ? 1 : 0;
}
}  // namespace

void Surrogate::predict_host(const double *states, int64_t n, double *dy, int *accepted) {
  ck(cudaSetDevice(device_), "cudaSetDevice");
  const int batch = static_cast<int>((n + 127) / 128 * 128);
  ensure_batch(batch);
  DevTemp<double> s_buf(static_cast<size_t>(batch) * kSurIn, "predict alloc"), d_buf(n * NS, "predict alloc");
  DevTemp<int> acc_buf(n, "predict alloc");
  double *s = s_buf.p, *d = d_buf.p;
  int *acc = acc_buf.p;
  ck(cudaMemsetAsync(s, 0, static_cast<size_t>(batch) * kSurIn * 8, stream_), "predict memset");
  ck(cudaMemcpyAsync(s, states, n * kSurIn * 8, cudaMemcpyHostToDevice, stream_), "predict upload");
  features(s, n, a_[0], nullptr, nullptr);
  ck(cudaMemsetAsync(a_[0] + n * kSurInPad, 0, (batch - n) * kSurInPad * 2, stream_), "pad rows");
  forward(batch);
  const int L = kSurLayers - 1;
  k_act<<<dim3(1, (batch + 31) / 32), dim3(32, 8), 0, stream_>>>(z_[L], batch, kSurOutPad, b_[L], nullptr, 0, z_[L],
                                                                   dz_, dzt_);
  k_decode<<<(n + 255) / 256, 256, 0, stream_>>>(z_[L], s, n, device_params(), d, acc);
  ck(cudaGetLastError(), "predict");
  ck(cudaMemcpyAsync(dy, d, n * NS * 8, cudaMemcpyDeviceToHost, stream_), "predict download");
  ck(cudaMemcpyAsync(accepted, acc, n * sizeof(int), cudaMemcpyDeviceToHost, stream_), "predict download");
  ck(cudaStreamSynchronize(stream_), "predict");
}

double Surrogate::grad_host(const double *states, const double *dy, int64_t n, std::vector<std::vector<float>> &grads) {
  ck(cudaSetDevice(device_), "cudaSetDevice");
  if (n % 128) throw std::runtime_error("gradient batch must be a multiple of 128");
  const int batch = static_cast<int>(n);
  ensure_batch(batch);
  DevTemp<double> s_buf(n * kSurIn, "grad alloc"), d_buf(n * NS, "grad alloc");
  double *s = s_buf.p, *d = d_buf.p;
  ck(cudaMemcpyAsync(s, states, n * kSurIn * 8, cudaMemcpyHostToDevice, stream_), "grad upload");
  ck(cudaMemcpyAsync(d, dy, n * NS * 8, cudaMemcpyHostToDevice, stream_), "grad upload");
  features(s, n, a_[0], tb_, d);
  k_transpose16<<<(n * kSurInPad + 255) / 256, 256, 0, stream_>>>(a_[0], batch, kSurInPad, at_[0]);
  forward(batch);
  // the backward pass of training without the Adam update, one layer at a time
  grads.assign(2 * kSurLayers, {});
  ck(cudaMemsetAsync(loss_, 0, sizeof(double), stream_), "loss");
  const int L = kSurLayers - 1;
  k_out_grad<<<(batch + 255) / 256, 256, 0, stream_>>>(z_[L], b_[L], tb_, batch, dzf_, loss_);
  k_act<<<dim3(1, (batch + 31) / 32), dim3(32, 8), 0, stream_>>>(dzf_, batch, kSurOutPad, nullptr, nullptr, 0, nullptr,
                                                                   dz_, dzt_);
  const int splits = std::max(1, std::min(64, batch / 1024));
  for (int l = L; l >= 0; --l) {
    const int dout = dout_[l], din = din_[l];
    ck(tc_gemm(dzt_, batch, at_[l], batch, partial_, din, dout, din, batch, splits, err_, stream_), "dW gemm");
    const int64_t nw = static_cast<int64_t>(dout) * din;
    k_reduce<<<(nw + 255) / 256, 256, 0, stream_>>>(partial_, splits, nw, gw_);
    ck(cudaMemsetAsync(gb_, 0, dout * 4, stream_), "gb");
    k_colsum<<<dim3((dout + 127) / 128, 64), 128, 0, stream_>>>(dzf_, batch, dout, gb_);
    grads[2 * l].resize(nw);
    grads[2 * l + 1].resize(dout);
    ck(cudaMemcpyAsync(grads[2 * l].data(), gw_, nw * 4, cudaMemcpyDeviceToHost, stream_), "grad copy");
    ck(cudaMemcpyAsync(grads[2 * l + 1].data(), gb_, dout * 4, cudaMemcpyDeviceToHost, stream_), "grad copy");
    ck(cudaStreamSynchronize(stream_), "grad");
    if (l > 0) {
      ck(tc_gemm(dz_, dout, wbt_[l], dout, da_, din, batch, din, dout, 1, err_, stream_), "dA gemm");
      const dim3 grid((din + 31) / 32, (batch + 31) / 32);
      k_act<<<grid, dim3(32, 8), 0, stream_>>>(da_, batch, din, nullptr, z_[l - 1], 2, dzf_, dz_, dzt_);
    }
  }
  double loss = 0;
  ck(cudaMemcpyAsync(&loss, loss_, sizeof(double), cudaMemcpyDeviceToHost, stream_), "loss");
  ck(cudaStreamSynchronize(stream_), "grad");
  return loss;
}

// Relative errors are taken over samples whose EPI increment reaches 1e-6 in
// some species: below that the chemistry changes nothing the solver resolves,
// and the gate bounds the network's increment by rel_max (Y_k + y_floor).
constexpr double kRelFloor = 1e-6;

SurrogateEval Surrogate::evaluate(int64_t begin, int64_t count) {
  if (begin < 0 || count <= 0 || begin + count > n_) throw std::runtime_error("evaluation range outside the data set");
  std::vector<double> st(count * kSurIn), lab(count * NS), pred(count * NS);
  std::vector<int> acc(count);
  d2h(st.data(), states_ + begin * kSurIn, st.size() * 8, "eval copy");
  d2h(lab.data(), labels_ + begin * NS, lab.size() * 8, "eval copy");
  const int64_t chunk = 1 << 18;
  for (int64_t q = 0; q < count; q += chunk) {
    const int64_t m = std::min(chunk, count - q);
    predict_host(st.data() + q * kSurIn, m, pred.data() + q * NS, acc.data() + q);
  }
  SurrogateEval e{};
  e.count = count;
  double rel_sum = 0;
  int64_t rel_n = 0, n_acc = 0;
  std::vector<double> rel_all;
  rel_all.reserve(static_cast<size_t>(count));
  for (int64_t i = 0; i < count; ++i) {
    double nrm = 0, err = 0, abs_sum = 0;
    bool finite = true;
    for (int k = 0; k < NS; ++k) {
      const double d = pred[i * NS + k] - lab[i * NS + k];
      finite = finite && std::isfinite(d);
      nrm = std::max(nrm, std::fabs(lab[i * NS + k]));
      err = std::max(err, std::fabs(d));
      abs_sum += std::fabs(d);
    }
    if (!finite) {
      ++e.nonfinite;
      if (nrm > kRelFloor) rel_all.push_back(std::numeric_limits<double>::infinity());
      continue;
    }
    const double r = nrm > kRelFloor ? err / nrm : -1;
    if (r >= 0) rel_all.push_back(r);
    if (!acc[i]) continue;
    ++n_acc;
    e.mean_abs += abs_sum / NS;
    if (r >= 0) {
      rel_sum += r;
      ++rel_n;
      e.max_rel = std::max(e.max_rel, r);
    }
    double dmax = 0;
    for (int el = 0; el < n_elem_; ++el) {
      double defect = 0, total = 0;
      for (int k = 0; k < NS; ++k) {
        const double a = elem_comp_[k * n_elem_ + el] / chem_.mw[k];
        defect += a * pred[i * NS + k];
        total += a * st[i * kSurIn + 2 + k];
      }
      if (total > 0) dmax = std::max(dmax, std::fabs(defect) / total);
    }
    e.max_defect = std::max(e.max_defect, dmax);
    e.mean_defect += dmax;
  }
  e.gate_pass = static_cast<double>(n_acc) / static_cast<double>(count);
  e.mean_rel = rel_n ? rel_sum / rel_n : 0;
  e.rel_count = rel_n;
  if (n_acc) {
    e.mean_abs /= n_acc;
    e.mean_defect /= n_acc;
  }
  if (!rel_all.empty()) {
    auto at = [&](double q) {
      const size_t k = static_cast<size_t>(q * (rel_all.size() - 1));
      std::nth_element(rel_all.begin(), rel_all.begin() + k, rel_all.end());
      return rel_all[k];
    };
    e.median_rel_all = at(0.5);
    e.p90_rel_all = at(0.9);
  }
  return e;
}

const SurrogateDev &Surrogate::device_params() {
  for (int l = 0; l < kSurLayers; ++l) {
    dev_.w_packed[l] = wpack_[l];
    dev_.bias[l] = b_[l];
  }
  for (int q = 0; q < kSurIn; ++q) {
    dev_.in_mu[q] = in_mu[q];
    dev_.in_sig[q] = in_sig[q];
  }
  for (int q = 0; q < kSurOut; ++q) {
    dev_.out_s[q] = out_s[q];
    dev_.out_c[q] = out_c[q];
  }
  dev_.n_elem = n_elem_;
  for (int e = 0; e < kMaxElem * kMaxSpec; ++e) dev_.elem[e] = 0.f;
  for (int e = 0; e < n_elem_; ++e)
    for (int k = 0; k < NS; ++k) dev_.elem[e * kMaxSpec + k] = static_cast<float>(elem_comp_[k * n_elem_ + e] / chem_.mw[k]);
  dev_.gate = gate;
  return dev_;
}

void Surrogate::save(const std::string &path) const {
  std::ofstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot write " + path);
  const char magic[8] = {'O', 'S', 'T', 'C', 'M', 'L', 'P', '5'};
  f.write(magic, 8);
  f.write(reinterpret_cast<const char *>(in_mu.data()), sizeof(in_mu));
  f.write(reinterpret_cast<const char *>(in_sig.data()), sizeof(in_sig));
  f.write(reinterpret_cast<const char *>(out_c.data()), sizeof(out_c));
  f.write(reinterpret_cast<const char *>(out_s.data()), sizeof(out_s));
  f.write(reinterpret_cast<const char *>(&gate), sizeof(gate));
  for (const auto &p : params()) f.write(reinterpret_cast<const char *>(p.data()), p.size() * 4);
}

void Surrogate::load(const std::string &path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot open " + path);
  char magic[8];
  f.read(magic, 8);
  if (std::memcmp(magic, "OSTCMLP5", 8) != 0) throw std::runtime_error(path + " is not a surrogate file");
  f.read(reinterpret_cast<char *>(in_mu.data()), sizeof(in_mu));
  f.read(reinterpret_cast<char *>(in_sig.data()), sizeof(in_sig));
  f.read(reinterpret_cast<char *>(out_c.data()), sizeof(out_c));
  f.read(reinterpret_cast<char *>(out_s.data()), sizeof(out_s));
  f.read(reinterpret_cast<char *>(&gate), sizeof(gate));
  auto p = params();
  for (auto &v : p) f.read(reinterpret_cast<char *>(v.data()), v.size() * 4);
  if (!f) throw std::runtime_error(path + " is truncated");
  set_params(p);
}

}  // namespace ostc
