// Warp and team S3TTMc schedules (s3ttmc_warp.cu).
#pragma once

#include <memory>

#include "tensor.cuh"

namespace spb {

struct WarpPlan;
std::shared_ptr<WarpPlan> warp_plan(uint32_t N, uint32_t R);
bool warp_supported(const WarpPlan &pl);
void warp_launch(const WarpPlan &pl, const TensorState &t, const ItemSet &items, const void *dU, void *dYpacked,
                 int precision, cudaStream_t st);

}  // namespace spb
