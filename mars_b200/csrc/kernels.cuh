// Device-side data layouts and launch entry points shared by the search and decode kernels.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "fit.cuh"
#include "price.hpp"

namespace mars {

// Per-level domain pool statistics (struct of arrays, one entry per domain position,
// row-major over the (nrow_d x ncol_d) position grid of that level).
struct DomainStats {
    int32_t* s1x4;   // sum of D over the s x s window (D = 2x2 box sum), exact
    int64_t* s2x16;  // sum of D^2, exact
    float* detf;     // Ndd = n*s2 - s1^2 (= the reference's det), rounded down; +huge if 0
    float* sdetf;    // sqrt(Ndd) rounded down; +huge if Ndd == 0
};

// Per-level range block statistics (one entry per requested block).
struct RangeStats {
    int32_t* t0;   // sum r
    int32_t* t2;   // sum r^2
    int64_t* nrr;  // n*t2 - t0^2
    double* sum0;  // f64 sum of any qalfa == 0 fit (domain independent)
    double* rms0;  // its rms
};

// One champion per (range, domain tile): the best candidate that tile saw.
struct Partial {
    double rms;
    double sum;
    uint32_t idx;  // dom_linear * 8 + isometry; UINT32_MAX when the tile saw nothing
    int32_t t1x4;
    uint16_t qalfa, qbeta;
    uint32_t pad;
};
static_assert(sizeof(Partial) == 32, "Partial layout");

struct LevelGeom {
    int size;      // range block side s (a power of two)
    int shift;     // domain stride in image pixels (even)
    int nrow_d;    // domain positions per column
    int ncol_d;    // domain positions per row
    int step_c;    // domain stride in contracted samples (shift / 2)
    int dw, dh;    // contracted plane width/height
    int w, h;      // plane width/height (range blocks outside it are reported invalid)
};

// Output record, bit-compatible with mars_candidate in include/mars_b200.h.
struct CandidateOut {
    uint32_t dom_row, dom_col, isometry, qalfa, qbeta, valid;
    double rms;
    int64_t s0, s1_x4, s2_x16, t0, t1_x4, t2;
};

// ---- launchers (search.cu) ----
cudaError_t launch_contract(const uint8_t* plane, int w, int h, int32_t* d_out,
                            cudaStream_t st);
// tmp (domain_stats_tmp_words(g) int32 words, or null): scratch of the separable form, used
// for block sizes >= 8; without it the direct kernel runs.  Same results either way.
size_t domain_stats_tmp_words(const LevelGeom& g);
cudaError_t launch_domain_stats(const int32_t* D, const LevelGeom& g, DomainStats ds,
                                cudaStream_t st, int32_t* tmp = nullptr);
cudaError_t launch_range_stats(const uint8_t* plane, int w, int h, const uint32_t* rows,
                               const uint32_t* cols, int nranges, int size, const FitParams& fp,
                               RangeStats rs, cudaStream_t st);
// The partial array is nsplit x nranges; nsplit from search_simt_splits().
cudaError_t launch_search_simt(const int32_t* D, const uint8_t* plane, int w,
                               const uint32_t* rows, const uint32_t* cols, int nranges,
                               const LevelGeom& g, RangeStats rs, DomainStats ds,
                               const FitParams& fp, Partial* partials, int nsplit,
                               unsigned long long* exact_counter, cudaStream_t st);
int search_simt_tiles(const LevelGeom& g);
int search_simt_splits(const LevelGeom& g, int nranges, int num_sms);
cudaError_t launch_reduce(const Partial* partials, int ntiles, int nranges, const LevelGeom& g,
                          RangeStats rs, DomainStats ds, CandidateOut* out, cudaStream_t st);
// Ranked search (search_top_k, encode.rs:695-788, k = 2..kMaxTopK): the CUDA-core kernel
// keeping the best k by (rms, reference index); partials are nsplit x nranges x k, the
// result nranges x k (valid = 0 past the ranked candidates).
constexpr int kMaxTopK = 8;
constexpr int kMaxTopKSplits = 64;  // domain-tile splits a ranked search may use
int search_topk_splits(const LevelGeom& g, int nranges, int num_sms);
cudaError_t launch_search_topk(const int32_t* D, const uint8_t* plane, int w,
                               const uint32_t* rows, const uint32_t* cols, int nranges,
                               const LevelGeom& g, RangeStats rs, DomainStats ds,
                               const FitParams& fp, int k, Partial* partials, int nsplit,
                               unsigned long long* counter, cudaStream_t st);
cudaError_t launch_reduce_topk(const Partial* partials, int nsplit, int nranges, int k,
                               const LevelGeom& g, RangeStats rs, DomainStats ds,
                               CandidateOut* out, cudaStream_t st);

// ---- Fisher classified search (fisher.cu) ----
// The index of one (size, shift) level: per domain position (raster order) its bucket
// (class * 24 + variance class) and canonicalising isometry; per bucket its length, offset
// into `list` (positions grouped by bucket, raster order within a bucket) and the bucket a
// class reads (itself, or the first non-empty bucket when it is empty).
struct FisherIndex {
    uint8_t* key;       // [npos]
    uint8_t* diso;      // [npos]
    uint32_t* counts;   // [72]
    uint32_t* offsets;  // [72]
    uint32_t* ref;      // [72]
    uint32_t* list;     // [npos]
    uint32_t* work;     // [fisher_group_work_words(npos)], the grouping's scratch
};
// Scratch words the grouping of n keys needs (per-chunk bucket counts and first slots).
size_t fisher_group_work_words(size_t n);
cudaError_t launch_fisher_index(const int32_t* D, int dw, int size, int shift, int nrow_d,
                                int ncol_d, FisherIndex ix, cudaStream_t st);
// Groups the n entries of `key` (bucket numbers 0..71; others are left out) by bucket:
// counts, offsets, the bucket each reads (ref) and the grouped indices in `list`, stable.
cudaError_t launch_fisher_group(const uint8_t* key, int n, uint32_t* counts, uint32_t* offsets,
                                uint32_t* ref, uint32_t* list, uint32_t* work, cudaStream_t st);
// One warp per range block; writes the winner (valid = 0 for none) and the eval count.
cudaError_t launch_fisher_search(const uint8_t* plane, int w, int h, const int32_t* D, int dw,
                                 int size, int shift, int ncol_d, const uint32_t* rows,
                                 const uint32_t* cols, int nranges, FisherIndex ix,
                                 const FitParams& fp, CandidateOut* out, uint64_t* evals,
                                 CandidateOut* part, uint32_t* part_e, cudaStream_t st);
// Warps per range block of the Fisher search at a size; part / part_e need
// nranges * fisher_warps_per_range(size) entries when that is above 1.
int fisher_warps_per_range(int size);

// ---- colour and metrics (color.cu) ----
// ycbcr (inverse = false: r, g, b -> y, cb, cr) or rgb_from_ycbcr (inverse = true: y, cb, cr
// -> r, g, b) over n pixels of three planes.
cudaError_t launch_ycbcr(const uint8_t* p0, const uint8_t* p1, const uint8_t* p2, size_t n,
                         uint8_t* q0, uint8_t* q1, uint8_t* q2, bool inverse, cudaStream_t st);
// w x h -> ceil(w/2) x ceil(h/2).
cudaError_t launch_downsample_box(const uint8_t* src, int w, int h, uint8_t* dst,
                                  cudaStream_t st);
// sw x sh -> w x h.
cudaError_t launch_upsample_nearest(const uint8_t* src, int sw, int sh, uint8_t* dst, int w,
                                    int h, cudaStream_t st);
// Sum of squared differences of two planes of n bytes into *out (zeroed first).
cudaError_t launch_sse(const uint8_t* a, const uint8_t* b, size_t n, int num_sms,
                       unsigned long long* out, cudaStream_t st);

// ---- decode (decode.cu) ----
// One leaf of the decode map in 16 bytes, dequantised on the device:
//   x: row | col << 16
//   y: size (bits 0-11) | mode (bits 12-13) | qbeta << 16
//   z: modes 0/2/3: dom_row | dom_col << 16;            mode 1: qgx
//   w: modes 0/2/3: qalfa (bits 0-16) | isometry << 24;  mode 1: qgy
struct DecodeLeaf {
    uint32_t x, y, z, w;
};
// Header constants of the dequantisation (ifs.rs:416-439).
struct DecodeConsts {
    double max_alfa;   // Header::max_alfa()
    double alfa_den;   // 2^bits_alfa
    double beta_den;   // 2^bits_beta - 1
};
// Kinds of expanded leaf.
enum : uint32_t { kLeafConst = 0, kLeafAffine = 1, kLeafDomain = 2, kLeafResidual = 3 };
// info bit 17 of a residual leaf with qalfa == 0: no domain read, d = 0.
constexpr uint32_t kLeafNoDomain = 1u << 17;
// A leaf expanded for the gather (built once per leaf list by launch_decode_expand):
//   const:    qalfa == 0 (modes 0/2): every pixel is the byte in info bits 24-31;
//   affine:   mode 1: round((a + gx*i) + gy*j), (i, j) = (y - row, x - col);
//   domain:   qalfa != 0 (modes 0/2): (0.5 + sum*a) + b, sum the 2x2 sum at
//             (dom_row + 2u, dom_col + 2v), (u, v) the inverse isometry of (i, j), a = alfa/4;
//   residual: mode 3: the domain value + res[roff + u*size + v], res the residual pool;
//             with qalfa == 0 (kLeafNoDomain) the domain is not read and sum = 0, so the
//             value is (0.5 + 0*a) + b + res as in the reference.
struct __align__(16) DecodeMap {
    double a, b, gx, gy;
    uint32_t rc;    // row | col << 16
    uint32_t info;  // size (0-11) | kind (12-13) | isometry (14-16) | no-domain (17) | const byte (24-31)
    uint32_t dom;   // dom_row | dom_col << 16
    int32_t roff;   // residual pool offset (kind residual), else -1
};
// resid_off: per leaf, the offset of its size*size residual values in the pool (or -1);
// may be null when no leaf is mode 3.
cudaError_t launch_decode_expand(const DecodeLeaf* leaves, const int32_t* resid_off, int n,
                                 DecodeConsts c, DecodeMap* maps, cudaStream_t st);
// owner: leaf index (or -1) per cell of 2^lg x 2^lg pixels, row-major, ceil(w/2^lg) wide.
// resid: the residual pool (f64), or null.
// One step of decode_until_stable (ifs.rs:321-353): a no-op once *done is set; otherwise
// the step, its max |next - prev| into *delta, then *done / *used (= iter + 1) when that
// delta is <= threshold.  done and done_w name the same flag.
cudaError_t launch_decode_step_stable(const uint8_t* src, uint8_t* dst, int w, int h, int lg,
                                      const int32_t* owner, const DecodeMap* maps,
                                      const double* resid, const int* done, int* delta,
                                      int threshold, int iter, int* done_w, int* used,
                                      cudaStream_t st);
cudaError_t launch_decode_step(const uint8_t* src, uint8_t* dst, int w, int h, int lg,
                               const int32_t* owner, const DecodeMap* maps, const double* resid,
                               cudaStream_t st);

// Source-ordered decode of large planes (decode.cu): the domain cells' jobs sorted by the
// source row of their windows (built once per leaf list), then per step a gather into a
// 16-byte-per-cell buffer and a placement in output order.  Eligible: cells of 4 x 4 pixels
// or more (lg >= 2), width % 4 == 0, no mode-3 residuals.  key / inv hold one word per 4x4
// cell, jobs and the cell buffer 16 bytes per domain cell (at most one per cell), row_count
// h words and cursor h + 1 (cursor[h]: the number of domain cells after the build).
size_t decode_sorted_cells(int w, int h);
bool decode_sorted_eligible(int w, int h, int lg, bool residuals);
cudaError_t launch_decode_sorted_build(int w, int h, int lg, const int32_t* owner,
                                       const DecodeMap* maps, const DecodeLeaf* leaves,
                                       uint32_t* key, uint32_t* row_count, uint32_t* cursor,
                                       uint4* jobs, uint32_t* inv, cudaStream_t st);
cudaError_t launch_decode_sorted_step(const uint8_t* src, uint8_t* dst, int w, int h, int lg,
                                      const int32_t* owner, const DecodeMap* maps,
                                      const uint4* jobs, uint32_t njobs, const uint32_t* inv,
                                      DecodeConsts c, uint4* cellbuf, cudaStream_t st);

// RD pricing of one node size (rdprice.cu): count nodes of size x size at (rows, cols), k
// candidates each; out[i] the node's priced winner, levels[levels_at[i]..] its mode-3 levels.
// basis: basis(size, k, i) at [k * size + i], computed on the host.  Sizes 2..64; size 64
// needs global_scratch of price_scratch_bytes() for scratch_slots warp slots.
struct PriceLaunch {
    const uint8_t* px;
    uint32_t stride, size, count;
    const uint32_t* rows;
    const uint32_t* cols;
    const void* cands;     // k per node, cand_stride bytes apart (0: packed price::Cand)
    uint32_t cand_stride;  // sizeof(mars_candidate) to read a search table in place
    uint32_t k;
    price::Setup setup;
    price::RateTable table;
    const double* basis;
    price::Priced* out;
    int8_t* levels;
    const uint64_t* levels_at;
    unsigned char* global_scratch;
    uint32_t scratch_slots;
};
size_t price_scratch_bytes(uint32_t size, uint32_t count, uint32_t* slots);
cudaError_t launch_price_nodes(const PriceLaunch& a, cudaStream_t st);

// The warm-up and RD walks over a search plan's nodes (rdprice.cu).  Nodes in plan order:
// level L holds count[L] nodes of size[L] from first[L], levels by ascending size, each in
// walk order.  child: 4 per node (TL, BL, TR, BR; -1 at min_size); roots: the unforced nodes
// below the forced splits, in walk order; levels_at: each node's offset in the pricing's
// level buffer; px/stride: the plane.
struct WalkPlan {
    uint32_t nodes, nlevels, nroots;
    uint32_t first[32], count[32], size[32];
    const uint32_t* rows;
    const uint32_t* cols;
    const int32_t* child;
    const int32_t* roots;
    const uint64_t* evals;
    const uint64_t* levels_at;
    const uint8_t* px;
    uint32_t stride;
};
// Per-call device scratch of the walks, `nodes` entries each (totals: 2).
struct WalkScratch {
    uint8_t* split;
    uint32_t* cnt;
    uint64_t* ev;  // warm-up: subtree evals; RD: subtree residual levels
    uint32_t* ofs;
    uint64_t* rofs;
    double* rd;
    double* rr;
    unsigned long long* totals;
};
// Warm-up walk with threshold t_rms: leaves (totals[0] of them, in walk order) into out;
// totals[1] = the evals of the visited nodes.
cudaError_t launch_warm_walk(const WalkPlan& w, const void* cands, uint32_t cand_stride,
                             double t_rms, uint32_t min_size, uint32_t zero_threshold,
                             uint32_t bits_beta, WalkScratch& s, mars_leaf* out, cudaStream_t st);
// RD walk over priced nodes: leaves (totals[0]) into out and their mode-3 levels (totals[1]
// values) into out_res, in walk order.  split0/split1: the split flag's bits per size class.
cudaError_t launch_rd_walk(const WalkPlan& w, const price::Priced* priced, const int8_t* levels,
                           double lambda, const double* split0, const double* split1,
                           uint32_t min_size, WalkScratch& s, mars_leaf* out, int32_t* out_res,
                           cudaStream_t st);

}  // namespace mars
