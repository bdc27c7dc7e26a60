// Host-side mirror of the reference encoder around the search boundary: the partition
// walks that call SearchProvider::search, the frozen rate snapshot that prices RD leaves,
// and the .ifs bitstream.  Restated from daleobrien/mars (crates/mars-codec) in the same
// f64 operation order (this translation unit is built with -ffp-contract=off).
#pragma once

#include <array>
#include <cstdint>
#include <functional>
#include <map>
#include <tuple>
#include <utility>
#include <vector>

#include "../../include/mars_b200.h"
#include "entropy.hpp"
#include "price.hpp"

namespace mars {
namespace codec {

// One SearchProvider::search answer (encode.rs:543-546).
struct SearchAnswer {
    mars_candidate cand;  // cand.valid == 0 <=> None
    uint64_t evals;
};

// The provider the walks call, with the node and effective stride of SearchRequest
// (encode.rs:532-540).  Must be callable from any thread.
using Provider = std::function<int(uint32_t row, uint32_t col, uint32_t size, uint32_t shift,
                                   SearchAnswer* out)>;
// SearchProvider::search_candidates (encode.rs:561-578): up to `max` candidates ascending by
// (rms, encounter order) and the node's evals.
using RankedProvider =
    std::function<int(uint32_t row, uint32_t col, uint32_t size, uint32_t shift, uint32_t max,
                      std::vector<mars_candidate>* out, uint64_t* evals)>;

struct Image {
    const uint8_t* px;
    uint32_t w, h;
};

// Every node the RD walk prices (best_mode_leaf, encode.rs:1536-1714), handed in one batch
// to a pricer that runs price::price_node elsewhere (the device) before the walk reads the
// answers.  Nodes are grouped by size, largest first (group g is [first[g], first[g+1]) of
// size sizes[g], DCT basis basis[g]); each node has k candidates (invalid ones pad a short
// list).  The pricer fills `priced` (one per node) and, when mode 3 is allowed, `levels`
// (size*size per node at levels_at[i], written for nodes whose winner is mode 3; the levels
// fit int8).
struct PriceBatch {
    Image im;
    price::Setup setup;
    const double* bits;
    size_t nbits;
    const int64_t* offset;  // price::kFields * price::kCtx entries
    uint32_t k;
    std::vector<uint32_t> sizes, first;
    std::vector<const double*> basis;
    std::vector<uint32_t> row, col;
    std::vector<price::Cand> cands;
    std::vector<uint64_t> evals;  // the provider's evals for the node
    std::vector<uint64_t> levels_at;
    uint64_t nlevels = 0;
    std::vector<price::Priced> priced;
    std::vector<int8_t> levels;
};
using Pricer = std::function<int(PriceBatch& batch)>;

uint32_t quantise_f64(double x, uint32_t max);
uint32_t best_beta(int64_t range_sum, int64_t pixel_count, uint32_t bits_beta);
mars_header build_header(uint32_t w, uint32_t h, const mars_params& p);
uint32_t virtual_size(const mars_header& h);
double block_rms(const Image& im, uint32_t row, uint32_t col, uint32_t size);
uint32_t adaptive_shift(uint32_t base, double rms);

// encode_image_with_search (encode.rs:1054-1126): returns MARS_OK or an error status.
// `residuals` receives the levels of the mode-3 leaves, size*size each, in leaf order.
// `warmup` answers the exhaustive t_rms = 8 warm-up walk of an RD encode
// (build_rate_snapshot searches exhaustively whatever the provider is); `provider` answers
// the final walk.
// `ranked` answers the final walk's search_candidates when o.rd_candidates > 1.
// `pricer`, when given, prices the RD walk's nodes in one batch; without it the walk prices
// each node on the host as it reaches it (the same price::price_node, the same doubles).
int encode(const Image& im, const mars_params& p, const mars_options& o, const Provider& provider,
           const Provider& warmup, mars_header* hdr, std::vector<mars_leaf>* leaves,
           std::vector<int32_t>* residuals, mars_counters* counters,
           const RankedProvider* ranked = nullptr, const Pricer* pricer = nullptr);

// The header an encode writes: build_header plus the residual step the options choose
// (encode.rs:1066-1071); MARS_EINVAL for a step outside the format's range.
int encode_header(uint32_t w, uint32_t h, const mars_params& p, const mars_options& o,
                  mars_header* out);
// The RD pricing's bits table from the warm-up walk's leaves (build_rate_snapshot,
// encode.rs:1139-1169, then RateModels as price::RateTable): bits and offsets.
int rate_table_from_warmup(const mars_header& hdr, const std::vector<mars_leaf>& warm,
                           uint32_t max_size, std::vector<double>* bits,
                           std::vector<int64_t>* offset);
// The constants best_mode_leaf reads for one encode (walk_rd's node lambda = lambda * 1.0).
price::Setup price_setup(const mars_header& hdr, const mars_params& p, const uint8_t allowed[4],
                         double lambda);
// The unforced quadtree nodes directly below the forced splits, in walk order.
std::vector<std::array<uint32_t, 3>> quadtree_roots(const mars_header& hdr);

// The residual step of a header as f64 (ResidualQstep::get, quant.rs:54-56); 0 in the
// struct stands for the default step 8.
double qstep_of(const mars_header& h);
// ResidualQstep::new / from_lambda (quant.rs:29-52), as binary32; false when out of range.
bool qstep_new(double step, float* out);
float qstep_from_lambda(double lambda);
// Offsets of each mode-3 leaf's levels in a residual pool of `npool` values (-1 for other
// leaves); false when the pool size does not match the leaves.
bool residual_offsets(const mars_leaf* leaves, size_t n, size_t npool, std::vector<int64_t>* offs);

// .ifs (ifs.rs:186-279 parse, 525-599 write).
int ifs_parse(const uint8_t* data, size_t len, mars_header* hdr, std::vector<mars_leaf>* leaves);
int ifs_write(const mars_header& hdr, const std::vector<mars_leaf>& leaves,
              std::vector<uint8_t>* out);

// The isometry map of isometry.rs:7-19.
void iso_map(uint32_t k, uint32_t u, uint32_t v, uint32_t size, uint32_t* i, uint32_t* j);

// .mars event vocabulary (mars_format.rs:113-133, 453-595).
using entropy::AdaptiveModel;
using entropy::ContextKey;
using entropy::Event;
constexpr uint8_t FIELD_SPLIT = 0, FIELD_MODE = 1, FIELD_QALFA = 2, FIELD_QBETA = 3,
                  FIELD_QBETA_DC = 4, FIELD_ISOMETRY = 5, FIELD_DOM_ROW = 6, FIELD_DOM_COL = 7,
                  FIELD_GX = 8, FIELD_GY = 9;
constexpr uint32_t MODE_ALPHABET = 4;
constexpr double AFFINE_GRAD_SCALE = 64.0;
constexpr int32_t AFFINE_GRAD_CLAMP = 2048;

// The domain-position predictor threaded through traversal order (mars_format.rs:386-395).
struct Predictor {
    int64_t row = 0, col = 0;
};
struct LeafRef {
    const mars_leaf* leaf;
    const int32_t* levels;  // mode 3: size*size residual levels, else null
};
using LeafMap = std::map<std::tuple<uint32_t, uint32_t, uint32_t>, LeafRef>;

uint32_t ceil_log2(uint32_t q);
uint32_t bits_coord_row(const mars_header& h);
uint32_t bits_coord_col(const mars_header& h);
uint32_t zigzag(int64_t x);
int64_t unzigzag(uint32_t z);

void emit_leaf(const mars_header& hdr, const mars_leaf& leaf, const int32_t* levels, uint32_t sc,
               Predictor& pred, std::vector<Event>& ev);
bool walk_write(const mars_header& hdr, uint32_t row, uint32_t col, uint32_t size,
                const LeafMap& by_pos, Predictor& pred, std::vector<Event>& ev);

}  // namespace codec
}  // namespace mars
