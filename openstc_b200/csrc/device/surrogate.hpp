// Learned replacement of the point-implicit (EPI) chemistry step:
//   (T, p, Y_k, dt)  ->  dY_k  =  (I - dt J)^-1 dt omega / rho,
// the increment one isolated EPI step (src/ImplicitTreatmentHPP.cuh:14-35,
// src/FiniteRateChem.cu:211-234) gives at fixed density.  A 12 -> 4x256
// (GELU) -> 9 MLP, trained on the GPU with the tcgen05 BF16 GEMM (FP32
// accumulation, FP32 master weights, Adam) on samples labelled by the FP64
// EPI step, and evaluated in the solver by a fused tensor-core kernel behind
// a per-cell trust gate with the EPI step as fallback.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "common.cuh"

namespace ostc {

constexpr int kSurIn = 12;      // T, log10 p, Y[9], log10 dt
constexpr int kSurInPad = 16;   // K of the first layer
constexpr int kSurOut = 9;      // dY_k
constexpr int kSurOutPad = 16;  // N of the last layer
constexpr int kSurHidden = 256;
constexpr int kSurLayers = 5;  // 4 hidden (GELU) + linear output
constexpr int kMaxElem = 8;
// The network predicts the relative increment r_k = dY_k / (Y_k + kSurYEps)
// through t_k = asinh(r_k / c_k) / s_k.
constexpr double kSurYEps = 1e-10;

// Trust region of the network: its training box.
struct SurrogateGate {
  float t_min = 250.f, t_max = 2800.f;
  float lp_min = 4.5f, lp_max = 6.0f;      // log10 p [Pa]
  float ldt_min = -9.0f, ldt_max = -6.0f;  // log10 dt [s]
  float defect_tol = 1e-3f;                // element-conservation defect (relative)
  float rel_max = 0.01f;                   // largest accepted |dY_k| / (Y_k + y_floor)
  float out_max = 6.f;                     // largest accepted |network output|
  float y_floor = 1e-10f;                  // mass fraction below which changes count as absolute
  // the judge: |dY_k - dY_DA,k| <= judge_rel |dY_DA,k| + judge_abs (Y_k +
  // y_floor) for every species, dY_DA the diagonal point-implicit increment
  // of the cell's own chemistry; judge_rel < 0 turns it off
  float judge_rel = 0.25f;
  float judge_abs = 1e-4f;
};

// Parameters the fused inference kernel reads (device memory).
struct SurrogateDev {
  const uint8_t *w_packed[kSurLayers];  // weights in tile order (bf16)
  const float *bias[kSurLayers];
  float in_mu[kSurIn], in_sig[kSurIn], out_c[kSurOut], out_s[kSurOut];
  float elem[kMaxElem * kMaxSpec];  // a_ek / W_k
  int n_elem;
  SurrogateGate gate;
};

// Held-out statistics against the FP64 EPI labels.  rel = max_k |dY_k -
// dY_EPI,k| / max_k |dY_EPI,k| per sample (samples with max_k |dY_EPI,k| >=
// 1e-6); the defect is that of the prediction the solver would apply (after
// the element projection), relative to the element totals.
struct SurrogateEval {
  double mean_rel, max_rel;            // the rel_count accepted samples with a resolvable increment
  double mean_abs;                     // the samples the trust gate accepts
  double max_defect, mean_defect;      // accepted samples
  double median_rel_all, p90_rel_all;  // every sample
  double gate_pass;                    // fraction accepted
  int64_t count, nonfinite;            // samples; predictions that were not finite
  int64_t rel_count;                   // accepted samples whose EPI increment reaches the floor
};

class Surrogate {
 public:
  // chem: the mechanism (DevParams of the case); elem_comp [ns][n_elem].
  Surrogate(const DevParams &chem, const std::vector<int> &elem_comp, int n_elem, int device, uint64_t seed);
  ~Surrogate();
  Surrogate(const Surrogate &) = delete;
  Surrogate &operator=(const Surrogate &) = delete;

  // Fills the data set with n samples: a fraction `field_fraction` from the
  // cells of `field` (perturbed), the rest uniform in the training box with
  // Dirichlet(1) mass fractions; labels from the FP64 EPI step.  Computes the
  // normalisation from the data.
  void generate(int64_t n, uint64_t seed, const DevBlock *field, double field_fraction);
  int64_t samples() const { return n_; }
  // Adam steps on random batches from samples [0, n_train); returns the
  // final loss, per-step losses into `losses` if non-null.
  double train(int steps, int batch, double lr, int64_t n_train, float *losses);
  // Statistics of the network against the labels on samples [begin, begin+count).
  SurrogateEval evaluate(int64_t begin, int64_t count);
  // FP64 EPI increments of host states (n x 12: T, p, Y[9], dt).
  void label_host(const double *states, int64_t n, double *dy);
  // Network increments of host states; accepted[i] = trust gate verdict.
  void predict_host(const double *states, int64_t n, double *dy, int *accepted);
  // Loss and gradients of one batch of host samples (for the gradient check).
  double grad_host(const double *states, const double *dy, int64_t n, std::vector<std::vector<float>> &grads);
  std::vector<std::vector<float>> params() const;  // W0, b0, W1, b1, ... (padded shapes)
  void set_params(const std::vector<std::vector<float>> &p);
  void save(const std::string &path) const;
  void load(const std::string &path);
  const SurrogateDev &device_params();  // packed for the fused kernel
  int device() const { return device_; }
  cudaStream_t stream() const { return stream_; }
  // the normalisation (features and targets)
  std::array<float, kSurIn> in_mu{}, in_sig{};
  std::array<float, kSurOut> out_c{}, out_s{};  // dY_k = (Y_k + eps) c_k sinh(s_k * output_k)
  SurrogateGate gate;

 private:
  void ensure_batch(int batch);
  void forward(int batch);
  double backward_and_step(int batch, double lr, int step);
  void pack();
  void upload_chem();
  void features(const double *states_dev, int64_t n, uint16_t *x_dev, float *t_dev, const double *dy_dev);
  DevParams chem_;
  std::vector<int> elem_comp_;
  int n_elem_;
  int device_;
  cudaStream_t stream_{};
  uint64_t seed_;
  int64_t n_ = 0;
  int adam_t_ = 0;
  bool packed_ = false;
  // data set
  double *states_ = nullptr;  // n x 12
  double *labels_ = nullptr;  // n x 9 (dY)
  uint16_t *x_ = nullptr;     // n x 16 bf16 features
  float *t_ = nullptr;        // n x 16 normalised targets
  // parameters (FP32 master), Adam moments, bf16 copies
  int din_[kSurLayers], dout_[kSurLayers];
  float *w_[kSurLayers] = {}, *b_[kSurLayers] = {};
  float *mw_[kSurLayers] = {}, *vw_[kSurLayers] = {}, *mb_[kSurLayers] = {}, *vb_[kSurLayers] = {};
  uint16_t *wb_[kSurLayers] = {}, *wbt_[kSurLayers] = {};
  uint8_t *wpack_[kSurLayers] = {};
  // batch work space
  int batch_ = 0;
  uint16_t *a_[kSurLayers] = {}, *at_[kSurLayers] = {};  // activations (input of layer l) and transposes
  float *z_[kSurLayers] = {};                              // pre-activations of layer l
  uint16_t *dz_ = nullptr, *dzt_ = nullptr;
  float *dzf_ = nullptr, *da_ = nullptr, *partial_ = nullptr, *gw_ = nullptr, *gb_ = nullptr;
  float *tb_ = nullptr;  // batch targets
  double *loss_ = nullptr;
  int *err_ = nullptr;
  SurrogateDev dev_{};
  std::vector<void *> allocs_;
};

// Launches the fused inference + trust gate over the interior cells of a
// block, applying accepted increments to cv (rho Y_k) and listing rejected
// cells; the EPI fallback then handles the list.  Defined in surrogate.cu.
void surrogate_apply(const SurrogateDev &p, const DevBlock *blocks_dev, const DevBlock &host_block, int block,
                     int *fallback_count, int *fallback_list, cudaStream_t st);

}  // namespace ostc
