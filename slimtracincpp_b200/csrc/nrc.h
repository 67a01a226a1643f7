// Neural radiance cache: a 96-64-64-64-64-3 MLP (ReLU hidden units, exp
// output) evaluated and trained on the sm_100a tensor cores.  The network's
// raw output z regresses log(radiance + 0.01) (an L2 loss in log space, whose
// gradient 2 (z - log(y + 0.01)) never vanishes, unlike a relative L2 through
// the exp); the cache answers max(exp(z) - 0.01, 0).  No counterpart
// in the reference: the cache answers for the radiance leaving a surface point
// reached by a bounce ray, in place of the rest of the path.
//
// Samples are 16 floats (4 float4):
//   (p.xyz in [0,1]^3, roughness) (direction.xyz, 0) (normal.xyz, 0) (albedo.xyz, 0)
// Parameters are one flat f32 vector (row = output unit):
//   W0 [64][96]  W1..W3 [64][64]  W4 [3][64]
// The kernels read a bf16 image of the parameters laid out as the tensor-core
// operands in shared memory (umma.cuh), written by the Adam kernel.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "launch_count.h"

namespace slim {
namespace nrc {

constexpr int kInputs = 96, kHidden = 64, kOutputs = 3, kOutPad = 16, kTile = 128;
constexpr int kOctaves = 12;
constexpr int kParamsW0 = kHidden * kInputs;        // 6144
constexpr int kParamsW = kHidden * kHidden;         // 4096
constexpr int kParamsW4 = kOutputs * kHidden;       // 192
constexpr int kParams = kParamsW0 + 3 * kParamsW + kParamsW4;   // 18624
constexpr int kImgW0 = kHidden * kInputs * 2;       // 12288 bytes
constexpr int kImgW = kHidden * kHidden * 2;        // 8192
constexpr int kImgW4 = kOutPad * kHidden * 2;       // 2048
constexpr int kImgOff1 = kImgW0, kImgOff4 = kImgW0 + 3 * kImgW;
constexpr int kImgBytes = kImgW0 + 3 * kImgW + kImgW4;          // 38912
constexpr float kLogOffset = 0.01f;  // z regresses log(radiance + 0.01); answers exp(z) - 0.01
constexpr float kZMax = 15.0f;       // exp(min(z, 15))
constexpr uint32_t kErrTimeout = 4u;

struct AdamArgs {
    float lr, beta1, beta2, eps;
    uint32_t *step;          // device step counter: the training kernel counts a non-empty
                             // step, Adam reads it for the bias corrections (so a captured
                             // graph replays correctly)
    uint32_t parts;          // partial gradient rows to sum (set by the launcher)
};

// Sets the kernels' shared-memory limits (before any launch or graph capture).
cudaError_t prepare();

// Largest grid the training kernel uses (rows of the partial-gradient buffer).
int train_grid(uint32_t samples);

// radiance[i] = cache(features[i]) for i < n; n = *count when count is given.
cudaError_t launch_infer(const float4 *features, const uint32_t *count, uint32_t n, uint32_t capacity,
                         float4 *radiance, const uint8_t *weight_image, uint32_t *error_flags, cudaStream_t stream);

// One optimisation step over the (features, targets) pairs [offset, offset +
// samples), clipped to *count when `count` (a device counter) is given:
// gradients of the mean log-radiance L2 loss into grad (f32, kParams), Adam update
// of params / m / v, refreshed bf16 image, loss into *loss.  A step with no
// samples changes nothing.
cudaError_t launch_train_step(const float4 *features, const float4 *targets, uint32_t samples, const uint32_t *count,
                              uint32_t offset, float *params, float *adam_m, float *adam_v, uint8_t *weight_image,
                              float *partials, float *loss_partials, float *grad, float *loss, const AdamArgs &adam,
                              uint32_t *error_flags, cudaStream_t stream);

// bf16 image of `params` (after the host sets the weights).
cudaError_t launch_pack_weights(const float *params, uint8_t *weight_image, cudaStream_t stream);

}  // namespace nrc
}  // namespace slim
