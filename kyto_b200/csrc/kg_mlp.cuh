// The learned partitioner's network: a BF16 MLP d -> h -> h -> P (ReLU between) with f32
// master weights, trained with Adam on soft targets, and its inference. Hand-written
// kernels (kg_mlp.cu): a tiled SIMT GEMM with f32 accumulation over bf16 or f32
// operands and fused bias/ReLU/mask epilogues, a warp-per-row softmax cross-entropy,
// fixed-order column sums, Adam, and the bf16 weight refresh.
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

#include "kg_internal.cuh"

namespace kg {

struct MlpShape {
  uint32_t din = 0, hidden = 0, parts = 0;
  // Offsets (floats) of W1 (hidden x din), b1, W2 (hidden x hidden), b2, W3 (parts x
  // hidden), b3 in the packed parameter vector (each a multiple of 4).
  uint64_t w_off[3] = {0, 0, 0}, b_off[3] = {0, 0, 0};
  uint64_t total = 0;
  uint32_t in(int l) const { return l == 0 ? din : hidden; }
  uint32_t out(int l) const { return l == 2 ? parts : hidden; }
  void layout();
  // The layers run on the tensor cores (a shape their tiles take: din <= 64, hidden a
  // multiple of 64 up to 256, parts a multiple of 32 up to 256 or of 256), else on the
  // SIMT GEMM.
  bool tensor_cores() const {
    return din <= 64 && hidden % 64 == 0 && hidden <= 256 && parts % 32 == 0 &&
           (parts <= 256 || parts % 256 == 0);
  }
  // The row stride of the first layer's bf16 input (64 on the tensor cores).
  uint32_t h0_ld() const { return tensor_cores() ? 64u : din; }
};

// Activations of one batch (rows x widths), kept for the backward pass.
struct MlpBatch {
  uint32_t rows = 0;
  DeviceBuffer<__nv_bfloat16> h0, h1, h2;  // inputs of the three layers
  DeviceBuffer<float> z1, z2, z3;          // pre-activations (z3: the logits)
  DeviceBuffer<float> dz3, dz2, dz1;       // gradients
  DeviceBuffer<float> row_loss;
  void alloc(const MlpShape& sh, uint32_t rows, cudaStream_t s);
};

class Mlp {
 public:
  MlpShape sh;
  DeviceBuffer<float> params, grads, m1, m2;
  DeviceBuffer<__nv_bfloat16> wb;  // bf16 copy of the packed parameters
  DeviceBuffer<__nv_bfloat16> w1p; // W1 as bf16 rows of 64 (the tensor-core layer's operand)
  DeviceBuffer<int> tc_error;      // set if a tensor-core layer gave up waiting
  uint64_t step = 0;

  void init(uint32_t din, uint32_t hidden, uint32_t parts, uint64_t seed, cudaStream_t s);
  // Set the network to the nearest-centre classifier of K centres (device, K x ldc f64;
  // part j = centre j, K <= parts): logit j = beta (2 c_j.x - |c_j|^2), i.e.
  // -beta |x - c_j|^2 up to a per-row constant. The first 2 din hidden units carry
  // relu(x) and relu(-x) through both layers; the other units keep their random weights
  // with no say in the logits yet. Needs hidden >= 2 din.
  void init_from_centres(const double* centres, uint32_t K, uint32_t ldc, float beta,
                         cudaStream_t s);
  void set_params(const float* host_or_device, cudaStream_t s);
  // The bf16 copy from the f32 masters.
  void refresh(cudaStream_t s);
  // x: b.rows x din f32 (row stride ldx floats) -> logits in b.z3.
  void forward(const float* x, uint64_t ldx, MlpBatch& b, cudaStream_t s) const;
  // Soft-target cross-entropy of the logits in b.z3 (labels: rows x L part indices; a
  // row's target is the share of each part among its L labels) and every gradient into
  // `grads`; the per-row losses stay in b.row_loss.
  void backward(const uint32_t* labels, uint32_t L, MlpBatch& b, cudaStream_t s);
  void adam(float lr, cudaStream_t s);
  // Fails (KG_ERR_TIMEOUT) if a tensor-core layer gave up waiting since init.
  void check(cudaStream_t s) const;
};

// Each row's top `probe` parts and, for each of n_temps temperatures (device array
// temps; the logits are multiplied by each), the parts' summed softmax:
// confidence[t * conf_stride + row]. With n_mass, also each row's n_mass most probable
// parts and their probabilities at the first temperature (mass_part, mass_prob: rows x
// n_mass).
void top_parts(const float* logits, uint64_t rows, uint32_t parts, uint32_t probe,
               uint32_t* top, float* confidence, uint64_t conf_stride, cudaStream_t s,
               const float* temps, uint32_t n_temps, uint32_t n_mass = 0,
               uint16_t* mass_part = nullptr, float* mass_prob = nullptr);

}  // namespace kg
