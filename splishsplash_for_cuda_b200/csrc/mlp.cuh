// mlp.cuh — the per-particle MLP that predicts the warm starts of the two DFSPH solvers.
//
// No reference counterpart: the reference warm-starts the pressure solve with the previous step's
// accumulated corrections kappa (DFSPH_core_cuda.cu:3061-3065) and the divergence solve with
// kappa_v / 2 (:240). Here a small network predicts, per particle, a correction to the previous
// step's TOTAL applied kappa / kappa_v (warm start + corrections):
//   inputs  x = [(rho - rho0)/rho0, rho_dot * alpha, neighbours / 64, kappa_total_prev,
//                kappa_v_total_prev, 0, 0, 0] * in_scale
//   hidden  2 x 64, ReLU
//   outputs y = [d_kappa, d_kappa_v] * out_scale
// so warm start = max(base + y, -0.5) with base the previous total scaled by the dt ratio. The
// solve itself is unchanged (it iterates to the same tolerance), and the reference's plain warm
// start replaces the prediction whenever the prediction yields the larger initial residual.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/dfsph_c.h"

namespace dfsph {

constexpr int kMlpIn = 8;       // 5 features + 3 zero pads
constexpr int kMlpFeatures = 5;
constexpr int kMlpHidden = 64;
constexpr int kMlpOut = 2;
// parameter layout of the FP32 master copy (row-major [out][in])
constexpr int kW1 = 0;
constexpr int kB1 = kW1 + kMlpHidden * kMlpIn;
constexpr int kW2 = kB1 + kMlpHidden;
constexpr int kB2 = kW2 + kMlpHidden * kMlpHidden;
constexpr int kW3 = kB2 + kMlpHidden;
constexpr int kB3 = kW3 + kMlpOut * kMlpHidden;
constexpr int kMlpParams = kB3 + kMlpOut;  // 4866
constexpr int kTrainBlock = 128;           // samples per training block

struct MlpScales {
    float in_scale[kMlpIn];
    float out_scale[kMlpOut];
};

// Device buffers of the network (inference copies in BF16, master weights and Adam moments in FP32).
struct MlpDev {
    float* params;        // kMlpParams
    float* adam_m;        // kMlpParams
    float* adam_v;        // kMlpParams
    float* grad;          // kMlpParams (last reduced gradient)
    float* partials;      // blocks x (kMlpParams + 1) block partial gradients (+ loss)
    uint16_t* w1_bf16;    // [64][16]   (k padded to 16)
    uint16_t* w2_bf16;    // [64][64]
    uint16_t* w3_bf16;    // [8][64]    (outputs padded to 8)
    MlpScales* scales;    // device copy
    double* loss;         // last batch loss
};

// Inference: pred[2 i + o] = MLP(features[8 i ...] * in_scale)[o] for i < n, on the tcgen05 tensor
// cores (accumulators in tensor memory). A bounded wait that gives up raises DFSPH_ST_MMA_TIMEOUT in
// *status.
void launch_mlp_forward(const MlpDev& m, const float* features, uint32_t n, float* pred, uint32_t* status,
                        cudaStream_t s);
// FP32 master weights -> BF16 inference copies.
void launch_mlp_pack(const MlpDev& m, cudaStream_t s);
// One training step on a batch: per-block forward/backward partial gradients, then a deterministic
// reduction; with adam != 0 also an Adam update (lr, beta1, beta2, eps, step t for bias correction).
void launch_mlp_train_step(const MlpDev& m, const float* x, const float* t, uint32_t batch, int adam, float lr,
                           float beta1, float beta2, float eps, int step, cudaStream_t s);
// Deterministic initialisation (He-uniform from a counter-based hash; last layer zero).
void launch_mlp_init(const MlpDev& m, uint32_t seed, cudaStream_t s);

size_t mlp_partials_floats(uint32_t max_batch);

}  // namespace dfsph
