// S3TTMc, pivot-chain schedule (s3ttmc_chain.cu).
#pragma once

#include "tensor.cuh"

namespace spb {

// Owners re-sorted for the chain schedule, built on first use.
struct ChainData {
  uint32_t L = 0;                 // leaf size (order - 1)
  DBuf<uint32_t> S;               // nown x sstride leaf ids, highest-degree first
  DBuf<double> c64;               // owner coefficients in chain order
  DBuf<float> c32;
  DBuf<uint8_t> flags;            // bit k: the owner starts a new prefix of k+1 pivots
  uint32_t chunk_owners = 0;
  uint32_t nchunks = 0, nsplit = 0, nslots = 0;
  DBuf<Chunk> chunks;             // work items of the heavy rows, heaviest first
  DBuf<SplitRow> split;
  uint32_t nlight = 0;            // rows of at most kChainLight owners, one item
  DBuf<Chunk> light;              // each, for the warp-per-row kernel, heaviest first
  std::map<uint32_t, std::unique_ptr<RowBands>> bands;  // by band count
};

// Order 4: rows with at most this many owners share few pivots; the chain
// schedule hands them to the warp-per-row kernel.  Order 5 keeps every row
// (the team kernel costs about 9x the chain's FMAs per owner).
constexpr uint64_t kChainLight = 16;
uint64_t chain_light_max(const TensorState &t);

// Whether the chain schedule covers this tensor and rank.
bool chain_supported(const TensorState &t, uint32_t R);
// The chain data of t (built on the first call).
ChainData &chain_data(TensorState &t);
// The chain work items in nb row bands (built on first use).
const RowBands &chain_bands(TensorState &t, uint32_t nb);
// One pass over chain work items: packed Y rows, partial rows for split rows.
void chain_launch(const TensorState &t, const ChainData &cd, const ItemSet &items, const void *dU, uint32_t R,
                  void *dYpacked, int precision, cudaStream_t st);

}  // namespace spb
