// Register-tiled S3TTMc schedule (s3ttmc_tiled.cu).
#pragma once

#include <memory>

#include "tensor.cuh"

namespace spb {

struct TiledPlan;
// Plan for order N and rank R; unsupported shapes give a plan with
// tiled_supported() == false (the caller then uses the per-owner schedule).
std::shared_ptr<TiledPlan> tiled_plan(uint32_t N, uint32_t R);
bool tiled_supported(const TiledPlan &pl);
// Writes the packed Y (lexicographic columns) or the partial rows of split rows.
void tiled_launch(const TiledPlan &pl, const TensorState &t, const ItemSet &items, const void *dU, void *dYpacked,
                  int precision, cudaStream_t st);

}  // namespace spb
