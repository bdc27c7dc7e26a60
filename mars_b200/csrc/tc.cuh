// Launch interface of the tcgen05 correlation path (search_tc.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace mars {
namespace tc {

constexpr int kMaxStages = 6;  // shared-memory pipeline depth bound (see stages_for)
constexpr int kMaxPhases = 8;  // 16 / shift for shift = 2

// TMA descriptors of the phase copies of the plane (u8, row pitch a multiple of 16, no
// swizzle, zero fill out of bounds).  `all` is one 4-D view -- bytes x pixel rows x
// same-phase 128-byte column groups x phases -- whose 128 x 8 x (16/P) x P box is a whole
// 16 KB A stage in core-matrix order; when the driver rejects that view (`use_all` = 0)
// the stage is loaded as 16 boxes of 128 B x 8 rows through the per-phase 2-D maps.
// The digit path (S >= 16) reads the hi digit's phase copies through `all` and the lo
// digit's through `all_lo`, both 4-D views of the same shape (it has no 2-D fallback).
struct alignas(64) TcMaps {
    CUtensorMap all;
    CUtensorMap all_lo;
    CUtensorMap m[kMaxPhases];
    int32_t use_all;
};

struct SeedOut {
    double rms, sum;
    uint32_t idx;
    int32_t t1x4;  // the seed champion's exact correlation (fits int32 for S <= 64)
};

// One job of the all-levels launch (launch_corr_all): range tiles [tile_begin, tile_begin +
// tile_count) of a level, each against `msplit` splits of the level's domain tiles, with
// the operands and outputs launch_corr takes.  gch (2 x nranges) is all ones and tickets
// (one per range tile of the level) zero before the launch; the last split of a range tile
// writes the tile's candidates to `out`.
struct LevelJob {
    TcMaps maps;
    const uint8_t* bglob;
    LevelGeom g;
    int nranges;
    RangeStats rs;
    DomainStats ds;
    FitParams fp;
    const SeedOut* seeds;
    Partial* partials;  // msplit x nranges (or more)
    unsigned long long* gch;
    int* tickets;
    CandidateOut* out;
    int tile_begin, tile_count, msplit;
    int digits;
    // A coarse pre-pass job (merge_seeds set) runs before every other job: the last split
    // of each range tile merges its champions into merge_seeds (the fine level's seeds, fine
    // grid fine_ncol, coarse stride merge_ratio times the fine one) and sets ready[tile]
    // (zero before the launch); the fine level's jobs pass the same array as wait_ready.
    SeedOut* merge_seeds = nullptr;
    int merge_ratio = 0, fine_ncol = 0;
    int* ready = nullptr;
    const int* wait_ready = nullptr;
};
constexpr int kMaxLevelJobs = 8;

bool supported(int size, int shift);
// Levels the split-digit contracted operand serves (block sizes 16..64).
bool digits_supported(int size, int shift);
int phase_count(int shift);
int row_pitch(int w);
size_t phase_bytes(int w, int h, int shift);
// Digit phase copies of the contracted plane: 2 digits x (32 / shift) phases x (h / 2) rows
// of row_pitch(w / 2) bytes (plus slack).
int digit_phase_count(int shift);
size_t digit_plane_bytes(int w, int h, int shift);
size_t b_bytes(int size, int nranges, bool digits);
int msplit_for(const LevelGeom& g, int nranges, int num_sms, bool digits);
// Whether the all-levels kernel holds a level: block sizes 4 and 8 on the fold path, 16, 32
// and 64 on the split-digit path.
bool all_levels_supported(int size, bool digits);
int ranges_per_tile(bool digits);
// Split counts of the levels of one all-levels launch, from a per-kind cost model, so that
// the work items are of similar duration and several per SM.  The level with the cheapest
// items (they run last) also gets a tail: its last tail_tiles[i] range tiles at
// tail_msplit[i] splits, finer items to even out the end of the launch (0 tiles: none).
void all_levels_splits(const LevelGeom* g, const int* nranges, const bool* digits, int n,
                       int num_sms, int* msplit, int* tail_tiles, int* tail_msplit);

cudaError_t launch_phase_planes(const uint8_t* plane, int w, int h, int shift, uint8_t* out,
                                cudaStream_t st);
cudaError_t launch_digit_planes(const int32_t* D, int w, int h, int shift, uint8_t* out,
                                cudaStream_t st);
cudaError_t launch_build_b(int size, const uint8_t* plane, int w, int h, const uint32_t* rows,
                           const uint32_t* cols, int nranges, uint8_t* out, bool digits,
                           cudaStream_t st);
cudaError_t launch_seed(const int32_t* D, const LevelGeom& g, const uint8_t* plane, int w,
                        const uint32_t* rows, const uint32_t* cols, int nranges, RangeStats rs,
                        DomainStats ds, const FitParams& fp, SeedOut* out, cudaStream_t st);
cudaError_t launch_corr(const TcMaps& maps, const uint8_t* bglob, const LevelGeom& g, int nranges,
                        RangeStats rs, DomainStats ds, const FitParams& fp, const SeedOut* seeds,
                        Partial* partials, unsigned long long* gch, int msplit, bool digits,
                        int* err, unsigned long long* counter, cudaStream_t st);
// The persistent launch over jobs[0..njobs) (njobs <= kMaxLevelJobs); `work` is a device
// counter it zeroes first.
cudaError_t launch_corr_all(const LevelJob* jobs, int njobs, int* work, int* err,
                            unsigned long long* counter, int num_sms, cudaStream_t st);
// The ranked search (k = 2..kMaxTopK candidates per range) on the tcgen05 path, for the
// kinds the all-levels kernel holds: seeds (n x k, the best k distinct of the 72 seed
// candidates), then the correlation, whose partials are msplit x n x k sorted lists
// (launch_reduce_topk merges them).
bool topk_supported(int size, bool digits);
cudaError_t launch_seed_topk(const int32_t* D, const LevelGeom& g, const uint8_t* plane, int w,
                             const uint32_t* rows, const uint32_t* cols, int nranges,
                             RangeStats rs, DomainStats ds, const FitParams& fp, int k,
                             SeedOut* out, cudaStream_t st);
cudaError_t launch_corr_topk(const TcMaps& maps, const uint8_t* bglob, const LevelGeom& g,
                             int nranges, RangeStats rs, DomainStats ds, const FitParams& fp,
                             const SeedOut* seeds, int k, Partial* partials,
                             unsigned long long* gch, int msplit, bool digits, int* err,
                             unsigned long long* counter, cudaStream_t st);
cudaError_t launch_seed_merge(const Partial* partials, int nsplit, int nranges, int coarse_ncol,
                              int fine_ncol, int ratio, SeedOut* seeds, cudaStream_t st);
cudaError_t launch_finish(const Partial* partials, int nsplit, int nranges, const LevelGeom& g,
                          RangeStats rs, DomainStats ds, const FitParams& fp, CandidateOut* out,
                          cudaStream_t st);

}  // namespace tc
}  // namespace mars
