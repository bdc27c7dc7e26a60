/*
 * CPU restatement of the Mars encoder's domain-range block search, its partition walks
 * and the fixed-point decode iteration.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA path and
 * the timed CPU baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  The product library (mars_b200) never links or calls it.
 *
 * Every function restates the reference Rust (daleobrien/mars) line by line; the
 * citations in oracle.cpp give crates/<crate>/src/<file>:<line> for each one.
 * Parity is pinned by the reference's own known-answer tests and golden fixtures
 * (tests/test_oracle_golden.py).
 */
#ifndef MARS_ORACLE_H
#define MARS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* EncodeParams (mars-codec/src/encode.rs:27-52). lambda is Option<f64>: has_lambda. */
typedef struct orc_params {
    uint32_t min_size, max_size, shift, bits_alfa, bits_beta, zero_threshold;
    double max_alfa;
    double t_rms;
    int32_t has_lambda;
    int32_t pad_;
    double lambda;
} orc_params;

/* The knobs of EncodeOptions (encode.rs:78-109) this restatement supports. */
typedef struct orc_options {
    uint8_t allowed_modes[4];
    int32_t adaptive_density;
    int32_t residual_adaptive; /* ResidualQuantisation::LambdaAdaptive */
    float residual_qstep;      /* Fixed(step); 0 = ResidualQstep::LEGACY (8) */
    int32_t method;            /* 0 ExhaustiveSearch, 1 Fisher (IndexedSearchProvider) */
    uint32_t rd_candidates;    /* EncodeOptions::rd_candidates; 0 or 1 = the single winner */
} orc_options;

/* RawMoments (encode.rs:225-232). */
typedef struct orc_moments {
    int64_t s0, s1_x4, s2_x16, t0, t1_x4, t2;
} orc_moments;

/* Candidate (encode.rs:236-244) plus a validity flag standing in for Option. */
typedef struct orc_candidate {
    uint32_t dom_row, dom_col, isometry, qalfa, qbeta, valid;
    double rms;
    orc_moments m;
} orc_candidate;

/* ifs::Leaf (mars-codec/src/ifs.rs:101-117) without the mode-3 residual. */
typedef struct orc_leaf {
    uint32_t row, col, size, mode, qalfa, qbeta, isometry, dom_row, dom_col;
    int32_t qgx, qgy;
} orc_leaf;

/* ifs::Header (ifs.rs:13-22). */
typedef struct orc_header {
    uint32_t bits_alfa, bits_beta, min_size, max_size, shift, width, height, int_max_alfa;
    float residual_qstep; /* binary32 wire value; 0 = 8 */
} orc_header;

void orc_contract(const uint8_t* px, uint32_t w, uint32_t h, int32_t* out);
void orc_fit_f64(const orc_moments* m, double max_alfa, uint32_t bits_alfa, uint32_t bits_beta,
                 uint32_t* qalfa, uint32_t* qbeta, double* rms);
uint32_t orc_best_beta(int64_t range_sum, int64_t pixel_count, uint32_t bits_beta);

/* search_top_k for one range block: up to k best candidates, ascending rms. */
int orc_search(const uint8_t* px, uint32_t w, uint32_t h, const int32_t* contracted,
               uint32_t row, uint32_t col, uint32_t size, uint32_t shift, const orc_params* p,
               uint32_t k, orc_candidate* out, uint32_t* nout, uint64_t* evals);

/* search_block over the fixed grid of aligned size x size blocks (row-major). */
int orc_search_grid(const uint8_t* px, uint32_t w, uint32_t h, uint32_t size, uint32_t shift,
                    const orc_params* p, orc_candidate* out, uint64_t* evals_per_block,
                    int nthreads);

/* Same, over an explicit list of block origins (rows[i], cols[i]). */
/* Fisher::index at (size, shift) + Fisher::candidates / search_block_fitted for each block. */
int orc_fisher_search_blocks(const uint8_t* px, uint32_t w, uint32_t h, uint32_t size,
                             uint32_t shift, const orc_params* p, const uint32_t* rows,
                             const uint32_t* cols, size_t n, orc_candidate* out,
                             uint64_t* evals_per_block, int nthreads);
/* The bucket (class * 24 + variance class) and canonicalising isometry of every domain
 * position at (size, shift), raster order (classify.rs newclass / variance_class). */
int orc_fisher_classify_domains(const uint8_t* px, uint32_t w, uint32_t h, uint32_t size,
                                uint32_t shift, uint8_t* bucket, uint8_t* iso);

int orc_search_blocks(const uint8_t* px, uint32_t w, uint32_t h, uint32_t size, uint32_t shift,
                      const orc_params* p, const uint32_t* rows, const uint32_t* cols,
                      size_t n, orc_candidate* out, uint64_t* evals_per_block, int nthreads);

/* encode_image_with_search(.., ExhaustiveSearch): header, leaves, counters. */
/* residuals: the size*size levels of every mode-3 leaf, in leaf order (freed with orc_free). */
int orc_encode(const uint8_t* px, uint32_t w, uint32_t h, const orc_params* p,
               const orc_options* o, orc_header* hdr, orc_leaf** leaves, size_t* nleaves,
               int32_t** residuals, size_t* nresiduals, uint64_t* search_evals,
               uint64_t* warmup_evals, int nthreads);
void orc_free(void* ptr);

/* decode_iterative from the flat-128 seed, modes 0/1/2. */
// Attractor refinement model (f64): the leaves' dequantised (s, o), and the loss, fixed
// point x (after fwd_iters steps from 128), and adjoint gradients (adj_iters steps from 0).
int orc_refine_params(const orc_header* hdr, const orc_leaf* leaves, size_t n, double* s,
                      double* o);
int orc_refine_eval(const orc_header* hdr, const orc_leaf* leaves, size_t n,
                    const int32_t* residuals, size_t nres, const uint8_t* target, const double* s,
                    const double* o, uint32_t fwd_iters, uint32_t adj_iters, double* x_out,
                    double* loss, double* gs, double* go);
int orc_decode(const orc_header* hdr, const orc_leaf* leaves, size_t n, const int32_t* residuals,
               size_t nresiduals, uint32_t iterations, uint8_t* out);
int orc_decode_until_stable(const orc_header* hdr, const orc_leaf* leaves, size_t n,
                            const int32_t* residuals, size_t nresiduals, uint8_t threshold,
                            uint32_t max_iterations, uint8_t* out, uint32_t* used);
int orc_zoom_leaves(const orc_header* hdr, const orc_leaf* leaves, size_t n, double factor,
                    orc_header* out_hdr, orc_leaf* out);

/* metrics::ycbcr / rgb_from_ycbcr (crates/mars-core/src/metrics.rs:377-460),
 * color::downsample_box / upsample_nearest (crates/mars-codec/src/color.rs:60-101) and
 * metrics::mse (metrics.rs:29-48). */
void orc_ycbcr(const uint8_t* r, const uint8_t* g, const uint8_t* b, size_t n, uint8_t* y,
               uint8_t* cb, uint8_t* cr);
void orc_rgb_from_ycbcr(const uint8_t* y, const uint8_t* cb, const uint8_t* cr, size_t n,
                        uint8_t* r, uint8_t* g, uint8_t* b);
void orc_downsample_box(const uint8_t* src, uint32_t w, uint32_t h, uint8_t* dst);
void orc_upsample_nearest(const uint8_t* src, uint32_t sw, uint32_t sh, uint8_t* dst, uint32_t w,
                          uint32_t h);
double orc_mse(const uint8_t* a, const uint8_t* b, size_t n);

/* dct.rs forward_dct2d / inverse_dct2d and quant.rs dead-zone quantiser, for tests. */
void orc_forward_dct2d(const double* block, uint32_t size, double* out);
void orc_inverse_dct2d(const double* coeffs, uint32_t size, double* out);
int32_t orc_dead_zone_quantize(double x, double step, double dz);
double orc_dead_zone_dequantize(int32_t level, double step, double dz);

/* .ifs bitstream (ifs.rs:186-260 parse, 525-599 write). */
int orc_ifs_parse(const uint8_t* data, size_t len, orc_header* hdr, orc_leaf** leaves,
                  size_t* nleaves);
int orc_ifs_write(const orc_header* hdr, const orc_leaf* leaves, size_t n, uint8_t** out,
                  size_t* len);

/* RD rate snapshot query used by tests: bits to code a leaf's events. */
double orc_leaf_bits(const orc_header* warm_hdr, const orc_leaf* warm_leaves, size_t nwarm,
                     const orc_leaf* leaf);

#ifdef __cplusplus
}
#endif
#endif
