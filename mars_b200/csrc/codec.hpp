// Host-side mirror of the reference encoder around the search boundary: the partition
// walks that call SearchProvider::search, the frozen rate snapshot that prices RD leaves,
// and the .ifs bitstream.  Restated from daleobrien/mars (crates/mars-codec) in the same
// f64 operation order (this translation unit is built with -ffp-contract=off).
#pragma once

#include <cstdint>
#include <functional>
#include <map>
#include <tuple>
#include <utility>
#include <vector>

#include "../../include/mars_b200.h"

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

struct Image {
    const uint8_t* px;
    uint32_t w, h;
};

uint32_t quantise_f64(double x, uint32_t max);
uint32_t best_beta(int64_t range_sum, int64_t pixel_count, uint32_t bits_beta);
mars_header build_header(uint32_t w, uint32_t h, const mars_params& p);
uint32_t virtual_size(const mars_header& h);
double block_rms(const Image& im, uint32_t row, uint32_t col, uint32_t size);
uint32_t adaptive_shift(uint32_t base, double rms);

// encode_image_with_search (encode.rs:1054-1126): returns MARS_OK or an error status.
int encode(const Image& im, const mars_params& p, const mars_options& o, const Provider& provider,
           mars_header* hdr, std::vector<mars_leaf>* leaves, mars_counters* counters);

// .ifs (ifs.rs:186-279 parse, 525-599 write).
int ifs_parse(const uint8_t* data, size_t len, mars_header* hdr, std::vector<mars_leaf>* leaves);
int ifs_write(const mars_header& hdr, const std::vector<mars_leaf>& leaves,
              std::vector<uint8_t>* out);

// The isometry map of isometry.rs:7-19.
void iso_map(uint32_t k, uint32_t u, uint32_t v, uint32_t size, uint32_t* i, uint32_t* j);

}  // namespace codec
}  // namespace mars
