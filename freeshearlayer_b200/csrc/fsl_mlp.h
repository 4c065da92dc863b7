// fsl_mlp.h -- parameter layout and launch interface of the learned closure.
#pragma once

#include <cuda_runtime.h>

namespace fsl {

// FP32 parameter vector: W1 [64][16] (inputs padded 8 -> 16 with zeros), b1
// [64], W2 [64][64], b2, W3 [64][64], b3, w4 [64], b4.  W are [out][in].
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + 64 * 16;
constexpr int kOffW2 = kOffB1 + 64;
constexpr int kOffB2 = kOffW2 + 64 * 64;
constexpr int kOffW3 = kOffB2 + 64;
constexpr int kOffB3 = kOffW3 + 64 * 64;
constexpr int kOffW4 = kOffB3 + 64;
constexpr int kOffB4 = kOffW4 + 64;
constexpr int kNParams = kOffB4 + 1;

// Feature normalisation and grid constants of one domain.
struct ClosureScales {
    float t_ref;       // time scale of the strain-rate feature (delta_w0 / dU)
    float delta_ratio; // filter width (dx dy dz)^(1/3) over the length scale delta_w0
    float r2dx, r2dy, r2dz;
    float DD;          // (dx dy dz)^(2/3), src/initialize.c:93
};

} // namespace fsl
