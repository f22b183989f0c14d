// Device-resident sparse symmetric tensor and the structures the S3TTMc
// kernels consume.
//
// Layout in HBM (all row-major, 0-based ids):
//   inds      nnz x order uint32         sorted unique tuples
//   vals      nnz double
//   own_S     nown x sstride uint32      the N-1 ids of each owner's leaf
//                                        (sub-multiset t \ t_j), padded to a
//                                        multiple of 4 ids (16-byte rows)
//   own_c64   nown double                owner coefficient f_j * v*mult(t)/N!
//   own_c32   nown float                 (FP32 copy)
//   row_ptr   dim+1 uint64               owners of row i: [row_ptr[i], row_ptr[i+1])
//   chunks    nchunks Chunk              work items: one row or a slice of a
//                                        long row; heaviest first
//   split     nsplit SplitRow            rows cut into several chunks and the
//                                        partial-sum slots that hold them
//
// Owners are the reference's (leaf, rem, value) records
// (src/compressed_dtree.cpp:67-74) re-segmented by their remaining index, so
// every Y row is produced by one reduction and no Y element needs a global
// atomic.  Repeated ids inside a tuple give identical owners
// (src/dtree.cpp:62-80 keeps them as duplicates); they are merged here with
// their multiplicity f_j folded into the coefficient.
#pragma once

#include <map>
#include <memory>

#include "common.cuh"

namespace spb {

struct Chunk {
  uint32_t row;
  uint32_t slot;  // partial-sum slot, or kDirect when the chunk owns its row
  uint64_t ob, oe;
};
static constexpr uint32_t kDirect = 0xffffffffu;
// work items with at most this many owners take one warp each in the
// warp-per-owner S3TTMc schedule (larger ones take a whole CTA)
static constexpr uint32_t kLightOwners = 48;

struct SplitRow {
  uint32_t row;
  uint32_t slot_begin, slot_end;
  uint32_t pad;
};

// The work items regrouped into nb bands of consecutive rows (band k holds
// rows [row0[k], row0[k+1]), its chunks [chunk0[k], chunk0[k+1]) heaviest
// first, and its split rows [split0[k], split0[k+1])).  The host-pointer
// S3TTMc runs the bands one after another so that the rows of one band are
// copied to the host while the next band is computed.  Slots are the ones of
// TensorState::split, so a band writes the same partial sums.
struct RowBands {
  uint32_t nb = 0;
  std::vector<uint32_t> row0, chunk0, split0;
  DBuf<Chunk> chunks;
  DBuf<SplitRow> split;
  std::vector<uint32_t> light0;  // chain schedule: the light rows of band k are
  DBuf<Chunk> light;             // light[light0[k], light0[k+1])
};

// The work items of one S3TTMc pass: all of them, or one row band.  After the
// pass Y rows [row0, row0 + rows) are complete.
struct ItemSet {
  const Chunk *chunks = nullptr;
  uint32_t nchunks = 0;
  const SplitRow *split = nullptr;
  uint32_t nsplit = 0;
  uint32_t row0 = 0, rows = 0;
  bool chain = false;      // items of the pivot-chain schedule (ChainData)
  uint32_t nslots = 0;     // partial-sum slots of the item list
  const Chunk *light = nullptr;  // chain schedule: light rows, one chunk each
  uint32_t nlight = 0;
};

// Reference CompressedDTree arrays, built on demand (tree.cu).
struct TreeLevels {
  uint32_t depth = 0;
  std::vector<uint64_t> size;                 // per level
  std::vector<DBuf<uint32_t>> level_idx;      // per level
  std::vector<DBuf<uint64_t>> level_ptr;      // per level (last: owner CSR)
  std::vector<DBuf<uint64_t>> dep_list;       // per level (l >= 1)
  uint64_t nown = 0;
  DBuf<uint64_t> own_rem;
  DBuf<double> own_val;
  DBuf<double> leaf_mult;  // distinct orderings of each leaf multiset
};

// Per-(order, R) index tables for the packed recursion (s3ttmc.cu) and the
// register-tiled schedule (s3ttmc_tiled.cu).
struct PackedTables;
struct TiledPlan;
struct WarpPlan;
struct ChainData;

// S3TTMc schedule: 0 = automatic (chain, else warp, else tiled, else rows),
// 1 = per-owner rows kernel, 2 = CTA register-tiled, 3 = warp per owner,
// 4 = pivot chain (2, 3 and 4 fail on shapes they do not support).
enum { kScheduleAuto = 0, kScheduleRows = 1, kScheduleTiled = 2, kScheduleWarp = 3, kScheduleChain = 4 };
int s3ttmc_schedule();
void set_s3ttmc_schedule(int s);

struct TensorState {
  int device = 0;
  uint32_t order = 0, dim = 0;
  uint64_t nnz = 0;
  double norm = 0.0;

  DBuf<uint32_t> inds;
  DBuf<double> vals;

  uint64_t nown = 0;
  uint32_t sstride = 0;
  DBuf<uint32_t> own_S;
  DBuf<double> own_c64;
  DBuf<float> own_c32;
  DBuf<uint64_t> row_ptr;
  std::vector<uint64_t> h_row_ptr;

  uint32_t chunk_owners = 0;  // max owners per chunk
  uint32_t nchunks = 0;
  uint32_t nheavy = 0;        // leading chunks with more than kLightOwners owners
  DBuf<Chunk> chunks;
  uint32_t nsplit = 0, nslots = 0;
  DBuf<SplitRow> split;

  DBuf<double> partials;  // nslots x m partial sums (grown on demand)
  DBuf<char> scratch;     // packed staging for unpacked output (grown on demand)
  DBuf<char> io_U, io_Y;  // device staging of the host-pointer entry point

  std::map<uint32_t, std::shared_ptr<PackedTables>> tables;  // by R
  std::map<uint32_t, std::shared_ptr<TiledPlan>> tiled;      // by R
  std::map<uint32_t, std::shared_ptr<WarpPlan>> warp;        // by R
  std::unique_ptr<TreeLevels> tree;
  std::map<uint32_t, std::unique_ptr<RowBands>> bands;  // by band count
  std::shared_ptr<ChainData> chain;  // owners in pivot-chain order (s3ttmc_chain.cu)
};

// s3ttmc.cu
// Builds what an S3TTMc of rank R will need (work-item layout, partial-row
// slots; kept with the tensor), so that a caller can do it ahead of time.
void s3ttmc_prepare(TensorState &t, uint32_t R, bool packed, int precision);
void s3ttmc_run(TensorState &t, const void *dU, uint32_t R, bool packed, void *dY,
                int precision, cudaStream_t stream);
// host U in, host Y out; the result rows are copied back band by band while
// the later bands are computed
void s3ttmc_host(TensorState &t, const void *U, uint32_t R, bool packed, void *Y, int precision);
uint32_t s3ttmc_launch_count(const TensorState &t, uint32_t R, bool packed);
void unpack_rows(const void *dpacked, uint64_t rows, uint32_t dim, uint32_t order,
                 void *dfull, int precision, cudaStream_t stream);
// tree.cu
void tree_build(TensorState &t);
// tensor.cu
// inds/vals in host memory, or in device memory when on_device is set
void tensor_build(TensorState &t, const uint32_t *inds, const double *vals, bool on_device = false);
// work items over owner ranges [row_ptr[i], row_ptr[i+1]): one per row,
// rows above co owners cut into slices with partial-sum slots (returns the
// slot count); and their heaviest-first order
uint32_t cut_rows(const std::vector<uint64_t> &row_ptr, uint32_t dim, uint64_t co, std::vector<Chunk> &ch,
                  std::vector<SplitRow> &sp);
void sort_heaviest_first(std::vector<Chunk> &ch, size_t b, size_t e, uint64_t max_owners);
// p[i] = i, i < n (permutation seeds of the radix sorts)
void device_iota(uint32_t *p, uint64_t n, cudaStream_t stream);
// the work items in nb row bands (built on first use, kept for later calls)
const RowBands &row_bands(TensorState &t, uint32_t nb);

}  // namespace spb

struct symprop_tensor {
  spb::TensorState s;
};
