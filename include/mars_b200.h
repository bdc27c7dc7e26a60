/*
 * mars_b200 -- B200 (sm_100a) domain-range block search and decode for the Mars fractal
 * codec, behind a plain C ABI.
 *
 * This is the drop-in boundary a host encoder binds.  It replaces, entry point by entry
 * point, the reference's (daleobrien/mars, Rust) search-provider boundary:
 *
 *   SearchProvider factory    crates/mars-codec/src/encode.rs:1054-1076
 *     (make_search(&Contracted) -> Box<dyn SearchProvider>)   -> mars_search_table_build
 *   SearchProvider::search    encode.rs:558-560, ExhaustiveSearch encode.rs:582-596
 *                                                              -> mars_search_table_lookup
 *   SearchProvider::search_candidates  encode.rs:561-578, 598-601 (search_top_k)
 *                              -> mars_search_table_build_ranked / _lookup_ranked
 *   search_block              encode.rs:610-619 (the fixed-grid GPU differential of
 *                             crates/mars-bench/src/gpu_search.rs:124-193) -> mars_search_blocks
 *   encode_image_with_search  encode.rs:1054-1126 with build_rate_snapshot :1139-1169
 *                                                              -> mars_encode
 *   decode_iterative          crates/mars-codec/src/ifs.rs:281-309   -> mars_decode
 *   ifs::parse / ifs::write   ifs.rs:186-217, 525-552           -> mars_ifs_parse / _write
 *   mars_format::write / read crates/mars-codec/src/mars_format.rs:232-400
 *                                                              -> mars_format_write / _read
 *   mars_entropy::encode / Decoder  crates/mars-entropy/src/lib.rs:200-335
 *                                                              -> mars_entropy_encode / _decode
 *
 * Conventions: every call returns MARS_OK (0) or a negative MARS_E* status; the text of the
 * last error on the calling thread is available from mars_last_error().  There is no CPU
 * fallback: without a usable CUDA device every compute call returns MARS_ENODEV.
 * Host pointers are caller-owned; tables and leaf arrays returned by the library are freed
 * with the matching *_free call.  Lookups on a built table are thread-safe.
 */
#ifndef MARS_B200_H
#define MARS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    MARS_OK = 0,
    MARS_EINVAL = -1,    /* bad argument or geometry */
    MARS_ENODEV = -2,    /* no usable CUDA device */
    MARS_ECUDA = -3,     /* a CUDA runtime call failed */
    MARS_ENOMEM = -4,    /* host or device allocation failed */
    MARS_ENOTFOUND = -5, /* lookup of a node the table does not hold */
    MARS_ETIMEOUT = -6,  /* a bounded device wait expired */
    MARS_EFORMAT = -7,   /* malformed bitstream */
    MARS_EUNSUPPORTED = -8
};

/* EncodeParams, crates/mars-codec/src/encode.rs:27-52 (lambda: Option<f64>). */
typedef struct mars_params {
    uint32_t min_size, max_size, shift, bits_alfa, bits_beta, zero_threshold;
    double max_alfa;
    double t_rms;
    int32_t has_lambda;
    int32_t reserved;
    double lambda;
} mars_params;

/* The EncodeOptions fields supported (encode.rs:78-109): allowed_modes (modes 0-3),
 * adaptive_density, residual_quantisation (residual_adaptive != 0 is LambdaAdaptive: the
 * step from lambda, 8 without one; else Fixed(residual_qstep) with 0 meaning the default
 * step 8, ResidualQstep::LEGACY) and rd_candidates (0 or 1: the single winner; 2..8: the
 * RD walk prices modes 2/3 for the best rd_candidates domains, which needs a lambda and the
 * exhaustive method, as encmars.rs:553-566 requires). */
typedef struct mars_options {
    uint8_t allowed_modes[4];
    int32_t adaptive_density;
    int32_t residual_adaptive;
    float residual_qstep;
    int32_t method; /* MARS_METHOD_*: the search provider of the final walk */
    uint32_t rd_candidates;
} mars_options;

/* Search methods (MethodName, crates/mars-search/src/lib.rs): the exhaustive search
 * (ExhaustiveSearch, encode.rs:582-602) and Fisher's classified search
 * (IndexedSearchProvider with Fisher, lib.rs:471-552, fisher.rs). */
enum { MARS_METHOD_EXHAUSTIVE = 0, MARS_METHOD_FISHER = 1 };

/* RawMoments, encode.rs:225-232. */
typedef struct mars_moments {
    int64_t s0, s1_x4, s2_x16, t0, t1_x4, t2;
} mars_moments;

/* Candidate, encode.rs:236-244; valid = 0 stands for None (no legal domain). */
typedef struct mars_candidate {
    uint32_t dom_row, dom_col, isometry, qalfa, qbeta, valid;
    double rms;
    mars_moments moments;
} mars_candidate;

/* ifs::Leaf, crates/mars-codec/src/ifs.rs:101-117.  A mode-3 leaf's `residual` (size*size
 * quantised DCT levels) travels outside the struct: calls that take or return leaves take or
 * return a residual pool with the levels of every mode-3 leaf, concatenated in leaf order. */
typedef struct mars_leaf {
    uint32_t row, col, size, mode, qalfa, qbeta, isometry, dom_row, dom_col;
    int32_t qgx, qgy;
} mars_leaf;

/* mars_format::Header (mars_format.rs:62-67): the ifs::Header geometry (ifs.rs:13-22) and
 * the residual step, binary32; 0 stands for the default step 8 (ResidualQstep::LEGACY). */
typedef struct mars_header {
    uint32_t bits_alfa, bits_beta, min_size, max_size, shift, width, height, int_max_alfa;
    float residual_qstep;
} mars_header;

/* EncodeCounters, encode.rs:1011-1021. */
typedef struct mars_counters {
    uint64_t search_evals, warmup_evals;
} mars_counters;

typedef struct mars_ctx mars_ctx;
typedef struct mars_table mars_table;
typedef struct mars_decode_plan mars_decode_plan;
typedef struct mars_search_plan mars_search_plan;

const char* mars_last_error(void);
const char* mars_version(void);

/* One context per device; a context owns a CUDA stream and cached device buffers.
 * A context serialises its own calls: use one context per host thread for concurrency. */
int mars_ctx_create(mars_ctx** out, int device);
void mars_ctx_destroy(mars_ctx* ctx);
/* Use `stream` (a cudaStream_t) for all of this context's work; NULL restores its own. */
int mars_ctx_set_stream(mars_ctx* ctx, void* stream);
/* Kernel launches made by this context since creation (instrumentation). */
uint64_t mars_ctx_launch_count(const mars_ctx* ctx);
/* Correlation kernel selection for A/B checks: 0 = automatic (tensor cores wherever the
 * level allows, CUDA cores otherwise), 1 = CUDA cores only, 2 = automatic as well (the
 * tensor-core path never serves a level it does not support), 3 = automatic with the
 * tensor-core operand loads split into per-phase boxes and the 2x2 box folded into K at
 * every block size, 4 = automatic with the fold at every block size (no split-digit
 * contracted operand at sizes 16..64), 5 = automatic with one correlation launch per level
 * (no all-levels persistent launch in search plans and tables).  Results are identical. */
int mars_ctx_set_search_path(mars_ctx* ctx, int32_t path);

/* The provider factory (encode.rs:1076): search every quadtree node an encode of this
 * plane can request -- every aligned block of size min_size..max_size, plus the smaller
 * border blocks reached through forced splits -- at `params->shift`, and also at
 * 2*shift for the nodes adaptive density routes there when `adaptive_density` is set.
 * `plane` is a host pointer to width*height bytes, row-major. */
int mars_search_table_build(mars_ctx* ctx, const uint8_t* plane, uint32_t width, uint32_t height,
                            const mars_params* params, int32_t adaptive_density,
                            mars_table** out);
/* SearchProvider::search for one node: the winning candidate (valid = 0 when the node has
 * no legal domain) and the eval count the reference reports for it. */
int mars_search_table_lookup(const mars_table* table, uint32_t row, uint32_t col, uint32_t size,
                             uint32_t shift, mars_candidate* out, uint64_t* evals);
/* The ranked provider factory (ExhaustiveSearch::search_candidates with max = k,
 * encode.rs:598-601 over search_top_k, encode.rs:695-788): every node's best k <= 8
 * candidates by (rms, reference order), as retain_top_k keeps them.  k = 1 is
 * mars_search_table_build. */
int mars_search_table_build_ranked(mars_ctx* ctx, const uint8_t* plane, uint32_t width,
                                   uint32_t height, const mars_params* params,
                                   int32_t adaptive_density, uint32_t k, mars_table** out);
/* SearchProvider::search_candidates for one node: up to `max` ranked candidates into
 * out[0..*count) and the node's evals.  A table built with k = 1 (or by the classified
 * provider) returns its single winner, as the trait's default does (encode.rs:561-578). */
int mars_search_table_lookup_ranked(const mars_table* table, uint32_t row, uint32_t col,
                                    uint32_t size, uint32_t shift, uint32_t max,
                                    mars_candidate* out, uint32_t* count, uint64_t* evals);
/* Total evals the table's searches stand for (all nodes, all shifts, counted as the
 * reference counts them: domain positions x 8 per node). */
uint64_t mars_search_table_evals(const mars_table* table);
/* How many of those candidates survived the exact-bound filter and took the exact f64 fit
 * (instrumentation). */
uint64_t mars_search_table_exact_fits(const mars_table* table);
void mars_search_table_free(mars_table* table);

/* Search plans: the provider factory for repeated planes of one geometry.  Creation plans
 * every node an encode can request (as mars_search_table_build without adaptive density),
 * uploads the node lists, keeps the device buffers and captures the whole search -- the
 * contraction and every quadtree level's statistics, seed, correlation and finish
 * kernels -- into one CUDA graph; each run is one graph launch.
 *   mars_search_plan_run: host plane in (copied through pinned staging), table out;
 *   mars_search_plan_run_device: device plane in, asynchronous on the context's stream,
 *     results kept on the device until mars_search_plan_table fetches them.
 * Tables from a plan answer mars_search_table_lookup like any other and may outlive it. */
int mars_search_plan_create(mars_ctx* ctx, uint32_t width, uint32_t height,
                            const mars_params* params, mars_search_plan** out);
int mars_search_plan_run(mars_search_plan* plan, const uint8_t* plane, mars_table** out);
int mars_search_plan_run_device(mars_search_plan* plan, const uint8_t* d_plane);
int mars_search_plan_table(mars_search_plan* plan, mars_table** out);
uint64_t mars_search_plan_evals(const mars_search_plan* plan);
/* Kernel launches one run replays (the graph's kernel nodes). */
uint64_t mars_search_plan_launches(const mars_search_plan* plan);
/* Device time in ms of the last completed replay's all-levels correlation launch (the one
 * persistent kernel over every tensor-core level), from CUDA events recorded inside the
 * plan's graph.  MARS_EUNSUPPORTED for plans without that launch (Fisher plans, one launch
 * per level); MARS_EINVAL before a replay has completed. */
int mars_search_plan_kernel_ms(const mars_search_plan* plan, float* ms);
void mars_search_plan_free(mars_search_plan* plan);
/* mars_encode through a plan (the plan's geometry and parameters): one graph launch for
 * the search, then the walks.  Exhaustive, single-winner, no adaptive density; the
 * outputs are mars_encode's.  Thread-safe per plan: concurrent calls overlap one plane's
 * walks with another's search. */
int mars_encode_planned(mars_search_plan* plan, const uint8_t* plane,
                        const mars_options* options, mars_header* header, mars_leaf** leaves,
                        size_t* nleaves, int32_t** residuals, size_t* nresiduals,
                        mars_counters* counters);

/* IndexedSearchProvider::build (crates/mars-search/src/lib.rs:480-513) for `method`: the
 * per-size domain indexes (plus the doubled-stride ones when adaptive_density and a
 * lambda are set) and the searches of every node an encode can request, answered through
 * mars_search_table_lookup.  MARS_METHOD_EXHAUSTIVE builds what mars_search_table_build
 * builds. */
int mars_indexed_table_build(mars_ctx* ctx, const uint8_t* plane, uint32_t width,
                             uint32_t height, const mars_params* params, int32_t adaptive_density,
                             int32_t method, mars_table** out);
/* A search plan for `method` (MARS_METHOD_EXHAUSTIVE is mars_search_plan_create): the same
 * nodes as mars_indexed_table_build without adaptive density, the whole search of a plane
 * -- for Fisher the per-size domain indexes, range classification and bucketed searches --
 * captured once as a CUDA graph.  The run / run_device / table calls are the plan calls
 * above; a Fisher table's eval counts are the bucket lengths of that run's plane.  Planned
 * encodes (mars_encode_planned) take exhaustive plans only. */
int mars_indexed_plan_create(mars_ctx* ctx, uint32_t width, uint32_t height,
                             const mars_params* params, int32_t method, mars_search_plan** out);

/* search_block over an explicit list of block origins at one size and shift (host
 * buffers).  out[i] / evals[i] belong to (rows[i], cols[i]). */
int mars_search_blocks(mars_ctx* ctx, const uint8_t* plane, uint32_t width, uint32_t height,
                       uint32_t size, uint32_t shift, const mars_params* params,
                       const uint32_t* rows, const uint32_t* cols, size_t n,
                       mars_candidate* out, uint64_t* evals);

/* Device-resident form for callers that keep the plane in HBM: `d_plane` is a device
 * pointer; results stay on the device in `d_out` (n candidates).  Asynchronous on the
 * context's stream. */
int mars_search_blocks_device(mars_ctx* ctx, const uint8_t* d_plane, uint32_t width,
                              uint32_t height, uint32_t size, uint32_t shift,
                              const mars_params* params, const uint32_t* d_rows,
                              const uint32_t* d_cols, size_t n, mars_candidate* d_out);

/* The searches of mars_search_table_build (every node an encode can request, at
 * params->shift) with the plane already in device memory and the results left on the
 * device, in the node order the table uses.  *n_nodes receives the node count and
 * *total_evals the reference eval count; call with d_out = NULL to query only.
 * Asynchronous on the context's stream. */
int mars_search_nodes_device(mars_ctx* ctx, const uint8_t* d_plane, uint32_t width,
                             uint32_t height, const mars_params* params, mars_candidate* d_out,
                             size_t capacity, size_t* n_nodes, uint64_t* total_evals);

/* mars_search_blocks_device with the range blocks read from one device plane and the domain
 * pool from another of the same size (both width*height u8): the attractor re-search of
 * mars_refine_domains, whose domain plane is a decode of the code being refined.  No
 * reference counterpart (the reference searches one plane); the per-range result is
 * mars_search_blocks_device's over the domain plane's pool, the same on identical planes. */
int mars_search_blocks_cross_device(mars_ctx* ctx, const uint8_t* d_range_plane,
                                    const uint8_t* d_domain_plane, uint32_t width,
                                    uint32_t height, uint32_t size, uint32_t shift,
                                    const mars_params* params, const uint32_t* d_rows,
                                    const uint32_t* d_cols, size_t n, mars_candidate* d_out);

/* The level search of mars_search_blocks_device for callers that cannot allocate device
 * memory -- real-time pipelines that forbid allocation once they are running, plug-ins
 * whose host application owns every device allocation, hosts with a fixed device-memory
 * budget.  It has no
 * counterpart in the reference.  It needs no context (creating one allocates) and calls no
 * allocator: its scratch is one 16 MiB device array inside the library, which every GPU
 * that loads the library holds until the process exits.  A search that needs more scratch
 * (roughly: planes beyond 512 x 512 at the smallest block sizes) is rejected with
 * MARS_EINVAL.  It runs on the current device and on `stream` (a cudaStream_t; NULL is the
 * legacy default stream), with the CUDA-core correlation kernel; results are identical to
 * the other entry points.  The first call on each device looks up the array's device
 * address, so make that first call before any stream capture.  All calls share the one
 * array: calls that overlap on the GPU (other streams, other host threads) race and must
 * be serialised by the caller.  Inputs and outputs are device pointers, as in
 * mars_search_blocks_device; the call is asynchronous. */
int mars_search_blocks_noalloc(const uint8_t* d_plane, uint32_t width, uint32_t height,
                               uint32_t size, uint32_t shift, const mars_params* params,
                               const uint32_t* d_rows, const uint32_t* d_cols, size_t n,
                               mars_candidate* d_out, void* stream);

/* encode_image_with_search with this library as the provider: the threshold walk when
 * params->has_lambda == 0, else the exhaustive t_rms = 8 warm-up (served from the same
 * table) followed by the bottom-up RD walk over modes 0-3.  *leaves is freed with
 * mars_leaves_free, *residuals (the mode-3 levels) with mars_residuals_free. */
int mars_encode(mars_ctx* ctx, const uint8_t* plane, uint32_t width, uint32_t height,
                const mars_params* params, const mars_options* options, mars_header* header,
                mars_leaf** leaves, size_t* nleaves, int32_t** residuals, size_t* nresiduals,
                mars_counters* counters);
void mars_leaves_free(mars_leaf* leaves);
void mars_residuals_free(int32_t* residuals);

/* decode_iterative: `iterations` fixed-point steps from the flat-128 seed (modes 0-3).
 * `out` is a host buffer of width*height bytes. */
int mars_decode(mars_ctx* ctx, const mars_header* header, const mars_leaf* leaves, size_t n,
                const int32_t* residuals, size_t nresiduals, uint32_t iterations, uint8_t* out);

/* Repeated decodes of one leaf list (progressive display, the attractor's forward map):
 * the leaf table and the owner map are validated and uploaded once; each run writes
 * `iterations` steps from the flat-128 seed into the device buffer d_out (width*height
 * bytes), asynchronously on the context's stream. */
int mars_decode_plan_create(mars_ctx* ctx, const mars_header* header, const mars_leaf* leaves,
                            size_t n, const int32_t* residuals, size_t nresiduals,
                            mars_decode_plan** out);
int mars_decode_plan_run(mars_decode_plan* plan, uint32_t iterations, uint8_t* d_out);
void mars_decode_plan_free(mars_decode_plan* plan);

/* decode_until_stable (crates/mars-codec/src/ifs.rs:321-353): steps from the flat-128
 * seed until the largest per-pixel change of a step is <= threshold, at most
 * max_iterations (>= 1) steps; *iterations_used is the number run.  The steps are queued
 * ahead on the device (a step after convergence is a no-op), so the host waits once. */
int mars_decode_until_stable(mars_ctx* ctx, const mars_header* header, const mars_leaf* leaves,
                             size_t n, const int32_t* residuals, size_t nresiduals,
                             uint8_t threshold, uint32_t max_iterations, uint8_t* out,
                             uint32_t* iterations_used);
int mars_decode_plan_run_until_stable(mars_decode_plan* plan, uint8_t threshold,
                                      uint32_t max_iterations, uint8_t* d_out,
                                      uint32_t* iterations_used);
/* zoom_leaves (ifs.rs:356-392): the leaf list and canvas scaled by `factor` (positions,
 * sizes (at least 1) and domain origins rounded half away from zero; affine gradients
 * divided by it), so the same contractive map decodes at another resolution.  Residuals
 * are dropped at any factor but 1: a mode-3 leaf comes back as mode 2, which decodes
 * exactly as the reference's mode-3 leaf without a residual.  out_leaves holds n leaves. */
int mars_zoom_leaves(const mars_header* header, const mars_leaf* leaves, size_t n,
                     double factor, mars_header* out_header, mars_leaf* out_leaves);

/* Attractor refinement (no reference counterpart: the reference fits each leaf to the
 * collage error only).  The decode map of decode_leaf (crates/mars-codec/src/ifs.rs:406-484)
 * is read as a continuous map of the plane, x_p = s_L * d_p(x) + o_L (+ the mode-3 residual),
 * d_p the 2x2 domain mean at the inverse isometry of p, flat leaves x_p = o_L and mode-1
 * leaves fixed; its fixed point x* is differentiated against the target t by the adjoint
 * lambda = 2(x* - t) + D^T(S lambda), so dL/ds_L = sum_L lambda*d and dL/do_L = sum_L lambda
 * for L = sum (x* - t)^2.
 *
 *   mars_refine_plan_create: validates and uploads the leaf list, its residual levels and the
 *     w*h target plane, and builds the transposed-map gather lists;
 *   mars_refine_params: the leaves' dequantised (s, o), n floats each (s = 0 for leaves
 *     without a domain; o = 0 for mode 1);
 *   mars_refine_forward: iterates from the flat-128 seed until max |x' - x| < tol or
 *     max_iters; returns the loss, the iterations run and, when x_out is non-NULL, x*
 *     (w*h floats, host);
 *   mars_refine_backward: the adjoint at the last forward's x*, until the relative step
 *     |lambda' - lambda| / |lambda'| < tol or max_iters, then the per-leaf gradients;
 *   mars_refine_run: `steps` damped per-leaf Newton updates of (s, o) (initial damping `lr`,
 *     halved on every step that does not lower the loss), re-quantised to the header's grid
 *     (qalfa >= 1 kept on domain leaves), decoded exactly with `decode_iterations` steps;
 *     out_leaves gets the best-decoding of the refined list and the refined list with the
 *     leaves that decode worse put back, when it beats the input list, else the input list.
 *     Geometry, modes, isometries, domains and residual levels are unchanged. */
typedef struct mars_refine_plan mars_refine_plan;
typedef struct mars_refine_report {
    double loss_start, loss_end;     /* continuous-model loss before and after the updates */
    double psnr_plain, psnr_refined; /* exact decodes of the input and refined lists, dB */
    uint32_t steps;                  /* gradient steps taken */
    uint32_t improving_steps;        /* of which lowered the loss (the others halve the step) */
    uint32_t changed_leaves;         /* leaves of out_leaves whose qalfa/qbeta changed */
    uint32_t accepted;               /* 1 when out_leaves is the refined list */
} mars_refine_report;
int mars_refine_plan_create(mars_ctx* ctx, const mars_header* header, const mars_leaf* leaves,
                            size_t n, const int32_t* residuals, size_t nresiduals,
                            const uint8_t* target, mars_refine_plan** out);
int mars_refine_params(mars_refine_plan* plan, float* s, float* o);
int mars_refine_forward(mars_refine_plan* plan, const float* s, const float* o,
                        uint32_t max_iters, double tol, float* x_out, double* loss,
                        uint32_t* iters);
int mars_refine_backward(mars_refine_plan* plan, uint32_t max_iters, double tol, float* grad_s,
                         float* grad_o, uint32_t* iters, double* residual);
int mars_refine_run(mars_refine_plan* plan, uint32_t steps, float lr, uint32_t decode_iterations,
                    mars_leaf* out_leaves, mars_refine_report* report);
void mars_refine_plan_free(mars_refine_plan* plan);

/* Domain re-search against the attractor (local iterative improvement of the domain choices):
 * `passes` rounds, each decoding the current list exactly (`decode_iterations` steps) and
 * searching every mode-2 leaf again (mars_search_blocks_cross_device: range block from
 * `target`, domain pool from the decoded plane, stride header->shift, the fit of `params`).
 * A round's new (domain, isometry, qalfa, qbeta) replace the old where the candidate is
 * valid with qalfa >= 1; the round is kept when the exact decode's squared error falls,
 * else with only the leaves whose own pixels decode better, if that lowers it; otherwise
 * the rounds stop.  Geometry, modes and the mode-3 residuals are unchanged.  out_leaves
 * holds n leaves; report: loss_start / loss_end = the decodes' squared error, psnr_plain /
 * psnr_refined their PSNR, steps = rounds run, improving_steps = rounds kept,
 * changed_leaves = leaves that differ from the input, accepted = any round kept. */
int mars_refine_domains(mars_ctx* ctx, const mars_params* params, const mars_header* header,
                        const mars_leaf* leaves, size_t n, const int32_t* residuals,
                        size_t nresiduals, const uint8_t* target, uint32_t passes,
                        uint32_t decode_iterations, mars_leaf* out_leaves,
                        mars_refine_report* report);

/* Colour input of the codec and its metric, on device planes, asynchronous on the context's
 * stream except mars_mse_device:
 *   ycbcr / rgb_from_ycbcr (crates/mars-core/src/metrics.rs:377-460): BT.601 full range,
 *     n pixels of three planes each way;
 *   downsample_box (crates/mars-codec/src/color.rs:60-83): w x h -> ceil(w/2) x ceil(h/2);
 *   upsample_nearest (color.rs:85-101): sw x sh -> w x h;
 *   mse (metrics.rs:29-48): exact sum of squared differences / n, returned on the host. */
int mars_ycbcr_device(mars_ctx* ctx, const uint8_t* d_r, const uint8_t* d_g, const uint8_t* d_b,
                      size_t n, uint8_t* d_y, uint8_t* d_cb, uint8_t* d_cr);
int mars_rgb_from_ycbcr_device(mars_ctx* ctx, const uint8_t* d_y, const uint8_t* d_cb,
                               const uint8_t* d_cr, size_t n, uint8_t* d_r, uint8_t* d_g,
                               uint8_t* d_b);
int mars_downsample_box_device(mars_ctx* ctx, const uint8_t* d_src, uint32_t width,
                               uint32_t height, uint8_t* d_dst);
int mars_upsample_nearest_device(mars_ctx* ctx, const uint8_t* d_src, uint32_t src_width,
                                 uint32_t src_height, uint8_t* d_dst, uint32_t width,
                                 uint32_t height);
int mars_mse_device(mars_ctx* ctx, const uint8_t* d_a, const uint8_t* d_b, size_t n, double* mse);

/* .ifs bitstream.  Buffers returned here are freed with mars_bytes_free / mars_leaves_free. */
int mars_ifs_parse(const uint8_t* data, size_t len, mars_header* header, mars_leaf** leaves,
                   size_t* nleaves);
int mars_ifs_write(const mars_header* header, const mars_leaf* leaves, size_t n, uint8_t** out,
                   size_t* len);
void mars_bytes_free(uint8_t* bytes);

/* .mars v0 plane container (mars_format.rs:232-400): 24-byte header carrying the residual
 * step as binary32, then the TREE section entropy-coded with adaptive models over the rANS
 * stack coder, modes 0-3.  Format errors (bad magic, truncation, degenerate header,
 * out-of-image domain, ...) return MARS_EFORMAT on read and MARS_EINVAL on write, with the
 * reference's message text.  Read output is freed with mars_leaves_free and
 * mars_residuals_free. */
int mars_format_write(const mars_header* header, const mars_leaf* leaves, size_t n,
                      const int32_t* residuals, size_t nresiduals, uint8_t** out, size_t* len);
int mars_format_read(const uint8_t* data, size_t len, mars_header* header, mars_leaf** leaves,
                     size_t* nleaves, int32_t** residuals, size_t* nresiduals);

/* mars_entropy::Event (lib.rs:188-193): context = (field, disambiguator). */
typedef struct mars_event {
    uint8_t field;
    uint8_t pad[3];
    uint32_t disambiguator, alphabet, symbol;
} mars_event;
/* mars_entropy::encode (lib.rs:200-202); bytes freed with mars_bytes_free. */
int mars_entropy_encode(const mars_event* events, size_t n, uint8_t** out, size_t* len);
/* Decoder::next once per entry of `shape` (its symbol fields are ignored), lib.rs:303-335. */
int mars_entropy_decode(const uint8_t* data, size_t len, const mars_event* shape, size_t n,
                        uint32_t* symbols);

#ifdef __cplusplus
}
#endif
#endif /* MARS_B200_H */
