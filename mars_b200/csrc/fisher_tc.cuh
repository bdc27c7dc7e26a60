// Launch interface of the tensor-core classified search (fisher_tc.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "kernels.cuh"
#include "tc.cuh"

namespace mars {
namespace ftc {

// Device arrays of one level's batch plan, filled on the device (per bucket b of 72):
// the level's ranges that read b (count, offset into the grouped range list), the first A
// tile (128 domains) and B tile (128 ranges) of b, its M-chunks and B tiles, and the
// offsets of its partial champions and work items.  Entries [72] of the *_base arrays are
// the totals.
struct FisherPlan {
    uint32_t* rcounts;      // [72]
    uint32_t* roffsets;     // [72]
    uint32_t* p_base;       // [72]
    uint32_t* chunks;       // [72]
    uint32_t* ntiles;       // [72]
    uint32_t* a_tile_base;  // [73]
    uint32_t* b_tile_base;  // [73]
    uint32_t* item_base;    // [73]
};
constexpr int kPlanWords = 72 * 5 + 73 * 3;

struct FisherTcArgs {
    const uint8_t* plane;
    int w, h;
    const int32_t* D;
    int dw, size, shift, ncol_d;
    const uint32_t* rows;
    const uint32_t* cols;
    int nranges;
    FisherIndex ix;           // the level's domain index (launch_fisher_index)
    const uint8_t* rbucket;   // [nranges] bucket each range reads (255: outside the plane)
    const uint8_t* riso;      // [nranges]
    const uint32_t* rlist;    // ranges grouped by bucket (launch_fisher_group)
    uint32_t* rrank;          // [nranges] scratch
    FisherPlan plan;
    uint8_t* aglob;           // a_bytes()
    uint8_t* bglob;           // b_bytes()
    size_t a_rows_max, b_rows_max, items_max;
    tc::SeedOut* seeds;       // [nranges]
    Partial* partials;        // partials_max()
    RangeStats rs;
    DomainStats ds;
    FitParams fp;
    CandidateOut* out;
    uint64_t* evals;
    int* err;
    unsigned long long* counter;
};

// Levels the tensor-core classified search serves (others keep fisher.cu's kernel).
bool supported(int size, int shift);
size_t a_bytes(int size, size_t npos);
size_t b_bytes(int size, size_t nranges);
size_t a_rows_max(size_t npos);
size_t b_rows_max(size_t nranges);
size_t items_max(size_t nranges);
size_t partials_max(size_t nranges);
// Each range's bucket (resolved through the index's `ref`) and canonicalising isometry.
cudaError_t launch_range_classes(const uint8_t* plane, int w, int h, int size, const uint32_t* rows,
                                 const uint32_t* cols, int nranges, const uint32_t* ref,
                                 uint8_t* rbucket, uint8_t* riso, cudaStream_t st);
// Plan, operands, seeds, the tcgen05 batch and the per-range answers (out, evals).
cudaError_t launch_search(const FisherTcArgs& a, cudaStream_t st);

}  // namespace ftc
}  // namespace mars
