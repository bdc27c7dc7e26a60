// CPU restatement of the reference's search, walks, rate snapshot and decode.
//
// TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA library and the timed CPU
// baseline.  Nothing in the product (mars_b200/) links or calls this file.
//
// Every function below restates one reference function of daleobrien/mars (Rust), in the
// same operation order, so that the f64 results are bit-identical.  Paths are relative to
// the reference project root.  Build flags keep that order: -ffp-contract=off and no
// fast-math (gcc would otherwise fuse a*b+c into an FMA, which Rust never does).
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <tuple>
#include <utility>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ------------------------------------------------------------------ fit and quantise

// quantise_f64 (crates/mars-codec/src/encode.rs:446-448): trunc(0.5 + x) clamped to
// [0, max], then `as u32` (NaN -> 0).
inline uint32_t quantise_f64(double x, uint32_t max) {
    double y = std::trunc(0.5 + x);
    if (std::isnan(y)) return 0;
    if (y < 0.0) y = 0.0;
    if (y > (double)max) y = (double)max;
    return (uint32_t)y;
}

// fit_f64 (encode.rs:247-289).
void fit_f64(const orc_moments& m, double max_alfa, uint32_t bits_alfa, uint32_t bits_beta,
             uint32_t* qalfa_out, uint32_t* qbeta_out, double* rms_out) {
    const double s0 = (double)m.s0;
    const double s1 = (double)m.s1_x4 / 4.0;
    const double s2 = (double)m.s2_x16 / 16.0;
    const double t0 = (double)m.t0;
    const double t1 = (double)m.t1_x4 / 4.0;
    const double t2 = (double)m.t2;

    const double det = s0 * s2 - s1 * s1;
    double alfa = (det == 0.0) ? 0.0 : (s0 * t1 - s1 * t0) / det;
    if (alfa < 0.0) alfa = 0.0;

    const uint32_t max_qalfa = (1u << bits_alfa) - 1;
    const uint32_t qalfa = quantise_f64(alfa / max_alfa * (double)(1u << bits_alfa), max_qalfa);
    const double alfa2 = (double)qalfa / (double)(1u << bits_alfa) * max_alfa;

    double beta = (t0 - alfa2 * s1) / s0;
    if (alfa2 > 0.0) beta += alfa2 * 255.0;
    const uint32_t max_qbeta = (1u << bits_beta) - 1;
    const uint32_t qbeta = quantise_f64(
        beta / ((1.0 + std::fabs(alfa2)) * 255.0) * (double)max_qbeta, max_qbeta);
    double beta2 = (double)qbeta / (double)max_qbeta * ((1.0 + std::fabs(alfa2)) * 255.0);
    if (alfa2 > 0.0) beta2 -= alfa2 * 255.0;

    const double sum = t2 - 2.0 * alfa2 * t1 - 2.0 * beta2 * t0 + alfa2 * alfa2 * s2 +
                       2.0 * alfa2 * beta2 * s1 + s0 * beta2 * beta2;
    double q = sum / s0;
    // f64::max(0.0): the non-NaN operand wins.
    if (!(q >= 0.0)) q = 0.0;
    *qalfa_out = qalfa;
    *qbeta_out = qbeta;
    *rms_out = std::sqrt(q);
}

// best_beta (encode.rs:456-460).
uint32_t best_beta(int64_t range_sum, int64_t pixel_count, uint32_t bits_beta) {
    const double mean = (double)range_sum / (double)pixel_count;
    const uint32_t max_qbeta = (1u << bits_beta) - 1;
    return quantise_f64(mean / 255.0 * (double)max_qbeta, max_qbeta);
}

// isometry::map (crates/mars-codec/src/isometry.rs:7-19).
inline void iso_map(uint32_t k, uint32_t u, uint32_t v, uint32_t size, uint32_t* i, uint32_t* j) {
    switch (k) {
        case 0: *i = u; *j = v; break;
        case 1: *i = size - 1 - v; *j = u; break;
        case 2: *i = v; *j = size - 1 - u; break;
        case 3: *i = size - 1 - u; *j = size - 1 - v; break;
        case 4: *i = u; *j = size - 1 - v; break;
        case 5: *i = size - 1 - u; *j = v; break;
        case 6: *i = v; *j = u; break;
        default: *i = size - 1 - v; *j = size - 1 - u; break;
    }
}

// ------------------------------------------------------------------ the plane types

struct Image {
    const uint8_t* px;
    uint32_t w, h;
};

// Contracted::build (encode.rs:478-502): D(r, c) = sum of the 2x2 block at (2r, 2c).
struct Contracted {
    std::vector<int32_t> data;
    size_t stride = 0;
    static Contracted build(const Image& im) {
        Contracted c;
        const size_t w = im.w, h = im.h;
        c.stride = w / 2;
        const size_t rows = h / 2;
        c.data.assign(c.stride * rows, 0);
        for (size_t i = 0; i < rows; ++i) {
            const size_t r0 = 2 * i;
            for (size_t j = 0; j < c.stride; ++j) {
                const size_t c0 = 2 * j;
                c.data[i * c.stride + j] = (int32_t)im.px[r0 * w + c0] +
                                           (int32_t)im.px[r0 * w + c0 + 1] +
                                           (int32_t)im.px[(r0 + 1) * w + c0] +
                                           (int32_t)im.px[(r0 + 1) * w + c0 + 1];
            }
        }
        return c;
    }
};

// domain_sums (encode.rs:800-802 -> mars-simd/src/moments.rs:20-36, the scalar form).
inline void domain_sums(const Contracted& c, size_t dr, size_t dc, size_t size, int64_t* s1,
                        int64_t* s2) {
    int64_t a = 0, b = 0;
    for (size_t u = 0; u < size; ++u) {
        const int32_t* row = &c.data[(dr + u) * c.stride + dc];
        for (size_t v = 0; v < size; ++v) {
            const int64_t d = row[v];
            a += d;
            b += d * d;
        }
    }
    *s1 = a;
    *s2 = b;
}

// cross_term_permuted (encode.rs:849-864 -> moments.rs dot_u8_i32_window).
inline int64_t cross_term_permuted(const Contracted& c, size_t dr, size_t dc, size_t size,
                                   const uint8_t* range_k) {
    int64_t acc = 0;
    for (size_t u = 0; u < size; ++u) {
        const int32_t* row = &c.data[(dr + u) * c.stride + dc];
        const uint8_t* rr = range_k + u * size;
        for (size_t v = 0; v < size; ++v) acc += (int64_t)rr[v] * (int64_t)row[v];
    }
    return acc;
}

// permute_range (encode.rs:833-842).
void permute_range(const uint8_t* range, uint32_t k, uint32_t size, uint8_t* out) {
    for (uint32_t u = 0; u < size; ++u)
        for (uint32_t v = 0; v < size; ++v) {
            uint32_t i, j;
            iso_map(k, u, v, size, &i, &j);
            out[u * size + v] = range[i * size + j];
        }
}

// retain_top_k (encode.rs:676-685): strict `<`, so equal-rms candidates keep encounter
// order.
void retain_top_k(std::vector<orc_candidate>& top, const orc_candidate& cand, size_t k) {
    size_t pos = top.size();
    for (size_t i = 0; i < top.size(); ++i)
        if (cand.rms < top[i].rms) {
            pos = i;
            break;
        }
    if (pos < k) {
        top.insert(top.begin() + (long)pos, cand);
        if (top.size() > k) top.resize(k);
    }
}

// search_top_k (encode.rs:695-788): every domain position (dom_row outer, dom_col inner,
// step `shift`) x the 8 isometries, integer moments, fit_f64, strict-< retention.
uint64_t search_top_k(const Image& im, const Contracted& c, uint32_t row, uint32_t col,
                      uint32_t size, uint32_t shift, const orc_params& p, size_t k,
                      std::vector<orc_candidate>& top) {
    top.clear();
    const size_t su = size;
    std::vector<uint8_t> range(su * su);
    int64_t t0 = 0, t2 = 0;
    for (size_t i = 0; i < su; ++i) {
        const size_t src = (row + i) * (size_t)im.w + col;
        for (size_t j = 0; j < su; ++j) {
            const uint8_t r = im.px[src + j];
            range[i * su + j] = r;
            t0 += r;
            t2 += (int64_t)r * r;
        }
    }
    const int64_t s0 = (int64_t)size * size;
    std::vector<uint8_t> by_iso(8 * su * su);
    for (uint32_t kk = 0; kk < 8; ++kk) permute_range(range.data(), kk, size, &by_iso[kk * su * su]);

    if (im.h < 2 * size || im.w < 2 * size) return 0;
    const uint32_t max_dom_row = im.h - 2 * size, max_dom_col = im.w - 2 * size;
    uint64_t evals = 0;
    for (uint32_t dom_row = 0; dom_row <= max_dom_row; dom_row += shift) {
        for (uint32_t dom_col = 0; dom_col <= max_dom_col; dom_col += shift) {
            const size_t drh = dom_row / 2, dch = dom_col / 2;
            int64_t s1_x4, s2_x16;
            domain_sums(c, drh, dch, su, &s1_x4, &s2_x16);
            for (uint32_t kk = 0; kk < 8; ++kk) {
                const int64_t t1_x4 = cross_term_permuted(c, drh, dch, su, &by_iso[kk * su * su]);
                orc_candidate cand;
                cand.dom_row = dom_row;
                cand.dom_col = dom_col;
                cand.isometry = kk;
                cand.valid = 1;
                cand.m = orc_moments{s0, s1_x4, s2_x16, t0, t1_x4, t2};
                fit_f64(cand.m, p.max_alfa, p.bits_alfa, p.bits_beta, &cand.qalfa, &cand.qbeta,
                        &cand.rms);
                evals += 1;
                retain_top_k(top, cand, k);
            }
        }
    }
    return evals;
}

// ------------------------------------------------------------------ Fisher (classified)

// ORDERING and MAPPING (crates/mars-search/src/tables.rs:13-51), data from Mars 1's
// globals.h.
const int FISHER_ORDERING[24][6] = {
    {3, 2, 1, 0, 3, 0}, {2, 3, 1, 0, 5, 1}, {2, 1, 3, 0, 5, 2}, {3, 1, 2, 0, 7, 0},
    {1, 3, 2, 0, 1, 1}, {1, 2, 3, 0, 1, 2}, {3, 2, 0, 1, 3, 1}, {2, 3, 0, 1, 5, 0},
    {2, 1, 0, 3, 2, 2}, {3, 1, 0, 2, 7, 1}, {1, 3, 0, 2, 1, 0}, {1, 2, 0, 3, 4, 2},
    {3, 0, 2, 1, 3, 2}, {2, 0, 3, 1, 2, 0}, {2, 0, 1, 3, 2, 1}, {3, 0, 1, 2, 7, 2},
    {1, 0, 2, 3, 4, 1}, {1, 0, 3, 2, 4, 0}, {0, 3, 2, 1, 6, 2}, {0, 2, 3, 1, 6, 1},
    {0, 2, 1, 3, 6, 0}, {0, 3, 1, 2, 0, 2}, {0, 1, 3, 2, 0, 1}, {0, 1, 2, 3, 0, 0},
};
const uint8_t FISHER_MAPPING[8][8] = {
    {0, 1, 2, 3, 4, 5, 6, 7}, {2, 0, 3, 1, 7, 6, 4, 5}, {1, 3, 0, 2, 6, 7, 5, 4},
    {3, 2, 1, 0, 5, 4, 7, 6}, {4, 7, 6, 5, 0, 3, 2, 1}, {5, 6, 7, 4, 3, 0, 1, 2},
    {6, 4, 5, 7, 1, 2, 0, 3}, {7, 5, 4, 6, 2, 1, 3, 0},
};

// classify::Block (classify.rs:21-37).
struct FBlock {
    std::vector<double> data;
    size_t size;
    double at(size_t i, size_t j) const { return data[i * size + j]; }
};

// match_order (tables.rs:57-62).
size_t match_order(const int order[4]) {
    for (size_t r = 0; r < 24; ++r)
        if (FISHER_ORDERING[r][0] == order[0] && FISHER_ORDERING[r][1] == order[1] &&
            FISHER_ORDERING[r][2] == order[2] && FISHER_ORDERING[r][3] == order[3])
            return r;
    std::abort();  // order is always a permutation of 0..3
}

// bubble_sort_desc_with_order (classify.rs:62-73).
void bubble_sort_desc(double a[4], int order[4]) {
    for (int k = 0; k < 4; ++k) order[k] = k;
    for (int i = 2; i >= 0; --i)
        for (int j = 0; j <= i; ++j)
            if (a[j] < a[j + 1]) {
                std::swap(a[j], a[j + 1]);
                std::swap(order[j], order[j + 1]);
            }
}

// newclass (classify.rs:42-55, 94-101).
void newclass(const FBlock& b, uint8_t* iso, uint8_t* clas) {
    const size_t h = b.size / 2;
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    for (size_t i = 0; i < h; ++i)
        for (size_t j = 0; j < h; ++j) {
            a[0] += b.at(i, j);
            a[1] += b.at(i, j + h);
            a[2] += b.at(i + h, j);
            a[3] += b.at(i + h, j + h);
        }
    int order[4];
    bubble_sort_desc(a, order);
    const size_t r = match_order(order);
    *iso = (uint8_t)FISHER_ORDERING[r][4];
    *clas = (uint8_t)FISHER_ORDERING[r][5];
}

// variance_2 (classify.rs:77-89).
double variance_2(const FBlock& b, size_t atx, size_t aty, size_t size) {
    double sum = 0.0, sum2 = 0.0;
    for (size_t i = atx; i < atx + size; ++i)
        for (size_t j = aty; j < aty + size; ++j) {
            const double v = b.at(i, j);
            sum += v;
            sum2 += v * v;
        }
    const double n = (double)(size * size);
    return sum2 / n - (sum / n) * (sum / n);
}

// variance_class (classify.rs:106-118).
uint8_t variance_class(const FBlock& b) {
    const size_t h = b.size / 2;
    double a[4] = {variance_2(b, 0, 0, h), variance_2(b, 0, h, h), variance_2(b, h, 0, h),
                   variance_2(b, h, h, h)};
    int order[4];
    bubble_sort_desc(a, order);
    return (uint8_t)match_order(order);
}

// flips (classify.rs:139-164): out[i][j] = b[src(i, j)].
FBlock flips(const FBlock& b, uint8_t iso) {
    const size_t s = b.size;
    FBlock out{std::vector<double>(s * s), s};
    for (size_t i = 0; i < s; ++i)
        for (size_t j = 0; j < s; ++j) {
            size_t si, sj;
            switch (iso) {
                case 0: si = i; sj = j; break;
                case 1: si = j; sj = s - i - 1; break;
                case 2: si = s - j - 1; sj = i; break;
                case 3: si = s - i - 1; sj = s - j - 1; break;
                case 4: si = i; sj = s - j - 1; break;
                case 5: si = s - i - 1; sj = j; break;
                case 6: si = j; sj = i; break;
                default: si = s - j - 1; sj = s - i - 1; break;
            }
            out.data[i * s + j] = b.at(si, sj);
        }
    return out;
}

// Fisher::index for one (size, shift) (fisher.rs:30-56): [clas][var_class] buckets of
// (dom_row, dom_col, dom_iso) in raster order; empty buckets copy the first non-empty one.
struct FisherLevel {
    std::vector<std::tuple<uint32_t, uint32_t, uint8_t>> bucket[3][24];
};

FisherLevel fisher_index(const Image& im, const Contracted& c, uint32_t size, uint32_t shift) {
    FisherLevel L;
    if (im.h >= 2 * size && im.w >= 2 * size) {
        const uint32_t step = std::max<uint32_t>(shift, 1);
        for (uint32_t r = 0; r <= im.h - 2 * size; r += step)
            for (uint32_t cc = 0; cc <= im.w - 2 * size; cc += step) {
                FBlock b{std::vector<double>((size_t)size * size), size};
                for (uint32_t u = 0; u < size; ++u)
                    for (uint32_t v = 0; v < size; ++v)
                        b.data[u * size + v] = (double)c.data[(r / 2 + u) * c.stride + cc / 2 + v];
                uint8_t iso, clas;
                newclass(b, &iso, &clas);
                const uint8_t var = variance_class(flips(b, iso));
                L.bucket[clas][var].emplace_back(r, cc, iso);
            }
    }
    const std::vector<std::tuple<uint32_t, uint32_t, uint8_t>>* fb = nullptr;
    for (auto& row : L.bucket)
        for (auto& b : row)
            if (!fb && !b.empty()) fb = &b;
    if (fb) {
        const auto copy = *fb;
        for (auto& row : L.bucket)
            for (auto& b : row)
                if (b.empty()) b = copy;
    }
    return L;
}

// Fisher::candidates + search_block_fitted (fisher.rs:58-78, lib.rs:211-297): the range's
// bucket in order, isometry MAPPING[range iso][domain iso], strict `<` on rms.
uint64_t fisher_search(const Image& im, const Contracted& c, const FisherLevel& L, uint32_t row,
                       uint32_t col, uint32_t size, const orc_params& p, orc_candidate* best) {
    const size_t su = size;
    std::vector<uint8_t> range(su * su);
    int64_t t0 = 0, t2 = 0;
    FBlock rb{std::vector<double>(su * su), su};
    for (size_t i = 0; i < su; ++i)
        for (size_t j = 0; j < su; ++j) {
            const uint8_t r = im.px[(row + i) * (size_t)im.w + col + j];
            range[i * su + j] = r;
            rb.data[i * su + j] = (double)r;
            t0 += r;
            t2 += (int64_t)r * r;
        }
    std::vector<uint8_t> by_iso(8 * su * su);
    for (uint32_t k = 0; k < 8; ++k) permute_range(range.data(), k, size, &by_iso[k * su * su]);
    uint8_t isom, clas;
    newclass(rb, &isom, &clas);
    const uint8_t var = variance_class(flips(rb, isom));
    const auto& bucket = L.bucket[clas][var];
    std::memset(best, 0, sizeof *best);
    uint64_t evals = 0;
    const int64_t s0 = (int64_t)size * size;
    for (const auto& e : bucket) {
        const uint32_t dr = std::get<0>(e), dc = std::get<1>(e);
        const uint8_t iso = FISHER_MAPPING[isom][std::get<2>(e)];
        int64_t s1_x4, s2_x16;
        domain_sums(c, dr / 2, dc / 2, su, &s1_x4, &s2_x16);
        const int64_t t1_x4 = cross_term_permuted(c, dr / 2, dc / 2, su, &by_iso[iso * su * su]);
        orc_candidate cand;
        cand.dom_row = dr;
        cand.dom_col = dc;
        cand.isometry = iso;
        cand.valid = 1;
        cand.m = orc_moments{s0, s1_x4, s2_x16, t0, t1_x4, t2};
        fit_f64(cand.m, p.max_alfa, p.bits_alfa, p.bits_beta, &cand.qalfa, &cand.qbeta, &cand.rms);
        evals += 1;
        if (!best->valid || cand.rms < best->rms) *best = cand;
    }
    return evals;
}

// IndexedSearchProvider with Fisher (lib.rs:426-513): indexes per power-of-two size from
// min_size (from 2 when the borders are not min_size-aligned) to max_size, at the base
// stride and, for adaptive-density RD encodes, at the doubled stride.
struct FisherIndexes {
    std::map<std::pair<uint32_t, uint32_t>, FisherLevel> levels;  // (size, shift)
    static FisherIndexes build(const Image& im, const Contracted& c, const orc_params& p,
                               bool adaptive) {
        FisherIndexes F;
        std::vector<uint32_t> shifts{p.shift};
        if (p.has_lambda && adaptive) shifts.push_back(p.shift * 2);
        for (uint32_t sh : shifts) {
            uint32_t size = (im.w % p.min_size != 0 || im.h % p.min_size != 0)
                                ? 2
                                : std::max<uint32_t>(p.min_size, 2);
            for (; size <= p.max_size; size *= 2) F.levels[{size, sh}] = fisher_index(im, c, size, sh);
        }
        return F;
    }
};

// ------------------------------------------------------------------ rate snapshot

// AdaptiveModel (crates/mars-entropy/src/lib.rs:36-121).
constexpr uint32_t PRECISION = 24;
constexpr uint64_t PRECISION_TOTAL = 1ull << PRECISION;
constexpr uint64_t RESCALE_THRESHOLD = 1ull << 16;

struct AdaptiveModel {
    std::vector<uint32_t> counts;
    uint64_t total = 0;
    explicit AdaptiveModel(uint32_t alphabet = 2) : counts(alphabet, 1u), total(alphabet) {}
    void update(uint32_t symbol) {
        counts[symbol] += 32;
        total += 32;
        if (total >= RESCALE_THRESHOLD) {
            uint64_t t = 0;
            for (auto& c : counts) {
                c = std::max<uint32_t>(c >> 1, 1u);
                t += c;
            }
            total = t;
        }
    }
    uint32_t scaled(uint64_t c) const {
        const uint64_t free_weight = PRECISION_TOTAL - counts.size();
        return (uint32_t)(((unsigned __int128)c * free_weight) / total);
    }
    uint32_t prob(uint32_t symbol) const {
        uint64_t before = 0;
        for (uint32_t i = 0; i < symbol; ++i) before += counts[i];
        const uint64_t after = before + counts[symbol];
        const uint32_t left = scaled(before) + symbol;
        const uint32_t right = scaled(after) + symbol + 1;
        return right - left;
    }
    // bits_for (lib.rs:98-101).
    double bits_for(uint32_t symbol) const {
        return -std::log2((double)prob(symbol) / (double)PRECISION_TOTAL);
    }
};

using ContextKey = std::pair<uint8_t, uint32_t>;
struct Event {
    ContextKey ctx;
    uint32_t alphabet, symbol;
};

// Field ids (crates/mars-codec/src/mars_format.rs:113-128) and MODE_ALPHABET (:133).
constexpr uint8_t FIELD_SPLIT = 0, FIELD_MODE = 1, FIELD_QALFA = 2, FIELD_QBETA = 3,
                  FIELD_QBETA_DC = 4, FIELD_ISOMETRY = 5, FIELD_DOM_ROW = 6, FIELD_DOM_COL = 7,
                  FIELD_GX = 8, FIELD_GY = 9;
constexpr uint32_t MODE_ALPHABET = 4;
// AFFINE_GRAD_SCALE / AFFINE_GRAD_CLAMP (encode.rs:353-360).
constexpr double AFFINE_GRAD_SCALE = 64.0;
constexpr int32_t AFFINE_GRAD_CLAMP = 2048;

uint32_t ceil_log2(uint32_t q) { return q <= 1 ? 0 : 32 - (uint32_t)__builtin_clz(q - 1); }
uint32_t virtual_size(const orc_header& h) {
    return 1u << ceil_log2(std::max(h.width, h.height));
}
uint32_t bits_coord_row(const orc_header& h) { return ceil_log2(h.height / h.shift); }
uint32_t bits_coord_col(const orc_header& h) { return ceil_log2(h.width / h.shift); }
uint32_t zigzag(int64_t x) { return (uint32_t)((x << 1) ^ (x >> 63)); }
uint32_t size_class_of(uint32_t size) { return (uint32_t)__builtin_ctz(size); }

struct Predictor {
    int64_t prev_row_units = 0, prev_col_units = 0;
};

// residual::encode_events (crates/mars-codec/src/residual.rs): FIELD_RESID_NZ = 10,
// FIELD_RESID_MAG = 11, LEVEL_CLAMP = 63, 4 bands over the coefficient index.
constexpr uint8_t FIELD_RESID_NZ = 10, FIELD_RESID_MAG = 11;
constexpr int32_t LEVEL_CLAMP = 63;
constexpr uint32_t RESID_BANDS = 4;
uint32_t resid_band(size_t index, size_t n) {
    return std::min<uint32_t>((uint32_t)((index * RESID_BANDS) / n), RESID_BANDS - 1);
}
void residual_events(const int32_t* levels, size_t n, uint32_t sc, std::vector<Event>& ev) {
    for (size_t i = 0; i < n; ++i) {
        const uint32_t band = resid_band(i, n);
        const int32_t c = std::max(-LEVEL_CLAMP, std::min(LEVEL_CLAMP, levels[i]));
        ev.push_back({{FIELD_RESID_NZ, sc * RESID_BANDS + band}, 2, c != 0 ? 1u : 0u});
        if (c != 0)
            ev.push_back({{FIELD_RESID_MAG, sc * RESID_BANDS + band}, (uint32_t)(2 * LEVEL_CLAMP + 1),
                          (uint32_t)((c << 1) ^ (c >> 31))});
    }
}

// emit_leaf (mars_format.rs:515-595); `levels` is the mode-3 residual (else unused).
void emit_leaf(const orc_header& hdr, const orc_leaf& leaf, const int32_t* levels, uint32_t sc,
               Predictor& pred, std::vector<Event>& ev) {
    ev.push_back({{FIELD_MODE, sc}, MODE_ALPHABET, leaf.mode});
    if (leaf.mode == 0) {
        ev.push_back({{FIELD_QBETA_DC, sc}, 1u << hdr.bits_beta, leaf.qbeta});
    } else if (leaf.mode == 1) {
        ev.push_back({{FIELD_QBETA_DC, sc}, 1u << hdr.bits_beta, leaf.qbeta});
        const uint32_t alph = (uint32_t)(2 * (int64_t)AFFINE_GRAD_CLAMP + 1);
        ev.push_back({{FIELD_GX, sc}, alph, zigzag(leaf.qgx)});
        ev.push_back({{FIELD_GY, sc}, alph, zigzag(leaf.qgy)});
    } else {
        ev.push_back({{FIELD_QALFA, sc}, (1u << hdr.bits_alfa) - 1, leaf.qalfa - 1});
        ev.push_back({{FIELD_QBETA, sc}, 1u << hdr.bits_beta, leaf.qbeta});
        ev.push_back({{FIELD_ISOMETRY, sc}, 8, leaf.isometry});
        const int64_t row_units = leaf.dom_row / hdr.shift;
        const int64_t col_units = leaf.dom_col / hdr.shift;
        const int64_t row_range = 1ll << bits_coord_row(hdr);
        const int64_t col_range = 1ll << bits_coord_col(hdr);
        ev.push_back({{FIELD_DOM_ROW, sc}, (uint32_t)(2 * row_range),
                      zigzag(row_units - pred.prev_row_units)});
        ev.push_back({{FIELD_DOM_COL, sc}, (uint32_t)(2 * col_range),
                      zigzag(col_units - pred.prev_col_units)});
        pred.prev_row_units = row_units;
        pred.prev_col_units = col_units;
        if (leaf.mode == 3) residual_events(levels, (size_t)leaf.size * leaf.size, sc, ev);
    }
}

using LeafMap = std::map<std::tuple<uint32_t, uint32_t, uint32_t>,
                         std::pair<const orc_leaf*, const int32_t*>>;

// walk_write (mars_format.rs:460-512): canonical NW, SW, NE, SE traversal.
bool walk_write(const orc_header& hdr, uint32_t row, uint32_t col, uint32_t size,
                const LeafMap& by_pos, Predictor& pred, std::vector<Event>& ev) {
    if (row >= hdr.height || col >= hdr.width) return true;
    const uint32_t half = size / 2;
    const bool forced = size > hdr.max_size || row + size > hdr.height || col + size > hdr.width;
    const uint32_t sc = size_class_of(size);
    auto it = by_pos.find({row, col, size});
    if (it != by_pos.end()) {
        if (!forced && size > hdr.min_size) ev.push_back({{FIELD_SPLIT, sc}, 2, 0});
        emit_leaf(hdr, *it->second.first, it->second.second, sc, pred, ev);
        return true;
    }
    if (!forced) {
        if (size <= hdr.min_size) return false;
        ev.push_back({{FIELD_SPLIT, sc}, 2, 1});
    }
    return walk_write(hdr, row, col, half, by_pos, pred, ev) &&
           walk_write(hdr, row + half, col, half, by_pos, pred, ev) &&
           walk_write(hdr, row, col + half, half, by_pos, pred, ev) &&
           walk_write(hdr, row + half, col + half, half, by_pos, pred, ev);
}

// RateModels (crates/mars-codec/src/rate.rs:55-80) over build_models
// (mars-entropy/src/lib.rs:269-278).
struct RateModels {
    std::map<ContextKey, AdaptiveModel> models;
    static bool from_leaves(const orc_header& hdr, const std::vector<orc_leaf>& leaves,
                            RateModels& out) {
        LeafMap by_pos;
        for (const auto& l : leaves) by_pos[{l.row, l.col, l.size}] = {&l, nullptr};
        std::vector<Event> ev;
        Predictor pred;
        if (!walk_write(hdr, 0, 0, virtual_size(hdr), by_pos, pred, ev)) return false;
        for (const auto& e : ev) {
            auto it = out.models.find(e.ctx);
            if (it == out.models.end()) it = out.models.emplace(e.ctx, AdaptiveModel(e.alphabet)).first;
            it->second.update(e.symbol);
        }
        return true;
    }
    double bits_for(ContextKey ctx, uint32_t alphabet, uint32_t symbol) const {
        auto it = models.find(ctx);
        if (it != models.end()) return it->second.bits_for(symbol);
        return AdaptiveModel(std::max<uint32_t>(alphabet, 2)).bits_for(symbol);
    }
};

// event_bits (encode.rs:1513-1518) over leaf_events (mars_format.rs:453-458).
double leaf_bits(const RateModels& rate, const orc_header& hdr, const orc_leaf& leaf,
                 uint32_t sc, const int32_t* levels = nullptr) {
    std::vector<Event> ev;
    Predictor pred;
    emit_leaf(hdr, leaf, levels, sc, pred, ev);
    double s = -0.0;
    for (const auto& e : ev) s += rate.bits_for(e.ctx, e.alphabet, e.symbol);
    return s;
}

// ------------------------------------------------------------------ partition walks

struct Ctx {
    Image im;
    const Contracted* contracted;
    orc_header hdr;
    orc_params params;
    const RateModels* rate;
    uint8_t allowed[4];
    bool adaptive_density;
    const FisherIndexes* fisher = nullptr;  // the final walk's provider when classified
    uint32_t rd_candidates = 1;             // search_candidates' max in walk_rd
};

// SearchProvider::search of the walk (k = 1), or search_candidates with max = k
// (encode.rs:561-601): ExhaustiveSearch ranks, the Fisher provider proposes one.
uint64_t provider_search(const Ctx& ctx, uint32_t row, uint32_t col, uint32_t size,
                         uint32_t shift, std::vector<orc_candidate>& top, uint32_t k = 1) {
    if (!ctx.fisher)
        return search_top_k(ctx.im, *ctx.contracted, row, col, size, shift, ctx.params, k, top);
    top.clear();
    orc_candidate best;
    const uint64_t ev = fisher_search(ctx.im, *ctx.contracted, ctx.fisher->levels.at({size, shift}),
                                      row, col, size, ctx.params, &best);
    if (best.valid) top.push_back(best);
    return ev;
}

orc_leaf make_leaf(uint32_t row, uint32_t col, uint32_t size) {
    orc_leaf l;
    std::memset(&l, 0, sizeof l);
    l.row = row;
    l.col = col;
    l.size = size;
    return l;
}

uint32_t pixel_at(const Image& im, uint32_t row, uint32_t col) {
    return im.px[(size_t)row * im.w + col];
}

int64_t range_sum(const Image& im, uint32_t row, uint32_t col, uint32_t size) {
    int64_t s = 0;
    for (uint32_t i = 0; i < size; ++i)
        for (uint32_t j = 0; j < size; ++j) s += pixel_at(im, row + i, col + j);
    return s;
}

struct WalkResult {
    std::vector<orc_leaf> leaves;
    uint64_t evals = 0;
};

constexpr uint32_t PARALLEL_SIZE_CUTOFF = 8;  // encode.rs:1321

WalkResult walk(const Ctx& ctx, uint32_t row, uint32_t col, uint32_t size);

// split (encode.rs:1442-1468): TL, BL, TR, BR, concatenated in that order.
WalkResult split(const Ctx& ctx, uint32_t row, uint32_t col, uint32_t half) {
    WalkResult q[4];
    const uint32_t rs[4] = {row, row + half, row, row + half};
    const uint32_t cs[4] = {col, col, col + half, col + half};
    if (half >= PARALLEL_SIZE_CUTOFF) {
        for (int i = 0; i < 4; ++i) {
#pragma omp task shared(q, ctx) firstprivate(i)
            q[i] = walk(ctx, rs[i], cs[i], half);
        }
#pragma omp taskwait
    } else {
        for (int i = 0; i < 4; ++i) q[i] = walk(ctx, rs[i], cs[i], half);
    }
    WalkResult out;
    for (auto& r : q) {
        out.leaves.insert(out.leaves.end(), r.leaves.begin(), r.leaves.end());
        out.evals += r.evals;
    }
    return out;
}

// walk (encode.rs:1330-1435): the top-down threshold walk with the §8.1 zero-alfa refit.
WalkResult walk(const Ctx& ctx, uint32_t row, uint32_t col, uint32_t size) {
    const orc_header& hdr = ctx.hdr;
    if (row >= hdr.height || col >= hdr.width) return {};
    const bool forced = size > hdr.max_size || row + size > hdr.height || col + size > hdr.width;
    if (forced) return split(ctx, row, col, size / 2);
    if (size == 1) {
        orc_leaf l = make_leaf(row, col, 1);
        l.qbeta = best_beta(pixel_at(ctx.im, row, col), 1, hdr.bits_beta);
        WalkResult r;
        r.leaves.push_back(l);
        return r;
    }
    std::vector<orc_candidate> top;
    const uint64_t block_evals = provider_search(ctx, row, col, size, ctx.params.shift, top);
    const double best_rms = top.empty() ? INFINITY : top[0].rms;
    if (best_rms > ctx.params.t_rms && size > hdr.min_size) {
        WalkResult r = split(ctx, row, col, size / 2);
        r.evals += block_evals;
        return r;
    }
    orc_leaf leaf = make_leaf(row, col, size);
    if (!top.empty()) {
        const orc_candidate& c = top[0];
        leaf.mode = 2;
        leaf.qalfa = c.qalfa;
        leaf.qbeta = c.qbeta;
        leaf.isometry = c.isometry;
        leaf.dom_row = c.dom_row;
        leaf.dom_col = c.dom_col;
    }
    const uint32_t diff = leaf.qalfa;  // qalfa.abs_diff(0)
    if (diff <= ctx.params.zero_threshold) {
        leaf.qbeta = best_beta(range_sum(ctx.im, row, col, size), (int64_t)size * size,
                               hdr.bits_beta);
        leaf.qalfa = 0;
        leaf.mode = 0;
        leaf.isometry = 0;
        leaf.dom_row = 0;
        leaf.dom_col = 0;
    }
    WalkResult r;
    r.leaves.push_back(leaf);
    r.evals = block_evals;
    return r;
}

// affine_fit (encode.rs:1724-1781), mode 1.
void affine_fit(const std::vector<double>& block, uint32_t size, uint32_t bits_beta,
                uint32_t* qbeta_out, int32_t* qgx_out, int32_t* qgy_out, double* sse_out) {
    const double n = (double)size * (double)size;
    double t0 = 0.0, tu = 0.0, tv = 0.0;
    for (uint32_t u = 0; u < size; ++u)
        for (uint32_t v = 0; v < size; ++v) {
            const double p = block[u * size + v];
            t0 += p;
            tu += p * (double)u;
            tv += p * (double)v;
        }
    double su = -0.0, suu = -0.0;
    for (uint32_t u = 0; u < size; ++u) su += (double)u;
    for (uint32_t u = 0; u < size; ++u) suu += (double)u * (double)u;
    const double s0 = n;
    const double s_u = (double)size * su;
    const double s_v = s_u;
    const double s_uu = (double)size * suu;
    const double s_vv = s_uu;
    const double s_uv = su * su;
    auto det3 = [](const double m[3][3]) {
        return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
               m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
               m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    };
    const double a[3][3] = {{s0, s_u, s_v}, {s_u, s_uu, s_uv}, {s_v, s_uv, s_vv}};
    const double det_a = det3(a);
    double b0, gx, gy;
    if (std::fabs(det_a) < 1e-9) {
        b0 = t0 / s0;
        gx = 0.0;
        gy = 0.0;
    } else {
        const double a_b0[3][3] = {{t0, s_u, s_v}, {tu, s_uu, s_uv}, {tv, s_uv, s_vv}};
        const double a_gx[3][3] = {{s0, t0, s_v}, {s_u, tu, s_uv}, {s_v, tv, s_vv}};
        const double a_gy[3][3] = {{s0, s_u, t0}, {s_u, s_uu, tu}, {s_v, s_uv, tv}};
        b0 = det3(a_b0) / det_a;
        gx = det3(a_gx) / det_a;
        gy = det3(a_gy) / det_a;
    }
    const uint32_t max_qbeta = (1u << bits_beta) - 1;
    const uint32_t qbeta = quantise_f64(std::max(b0 / 255.0 * (double)max_qbeta, 0.0), max_qbeta);
    auto qgrad = [](double g) {
        double r = std::round(g * AFFINE_GRAD_SCALE);
        if (r < -(double)AFFINE_GRAD_CLAMP) r = -(double)AFFINE_GRAD_CLAMP;
        if (r > (double)AFFINE_GRAD_CLAMP) r = (double)AFFINE_GRAD_CLAMP;
        return (int32_t)r;
    };
    const int32_t qgx = qgrad(gx), qgy = qgrad(gy);
    const double b0q = (double)qbeta / (double)max_qbeta * 255.0;
    const double gxq = (double)qgx / AFFINE_GRAD_SCALE;
    const double gyq = (double)qgy / AFFINE_GRAD_SCALE;
    double sse = 0.0;
    for (uint32_t u = 0; u < size; ++u)
        for (uint32_t v = 0; v < size; ++v) {
            const double pred = b0q + gxq * (double)u + gyq * (double)v;
            const double diff = block[u * size + v] - pred;
            sse += diff * diff;
        }
    *qbeta_out = qbeta;
    *qgx_out = qgx;
    *qgy_out = qgy;
    *sse_out = sse;
}

// ------------------------------------------------------------------ mode 3 (residual)

// basis (crates/mars-codec/src/dct.rs:13-20), evaluated at every use as there.
double dct_basis(size_t n_size, size_t k, size_t n) {
    const double c_k = k == 0 ? 0.707106781186547524400844362104849039 : 1.0;
    const double pi = 3.14159265358979323846264338327950288;
    return std::sqrt(2.0 / (double)n_size) * c_k *
           std::cos(pi / (double)n_size * ((double)n + 0.5) * (double)k);
}
// dct1d / idct1d (dct.rs:22-36): Iterator::sum folds from -0.0 (Rust >= 1.83).
std::vector<double> dct1d(const std::vector<double>& x) {
    const size_t n = x.size();
    std::vector<double> out(n);
    for (size_t k = 0; k < n; ++k) {
        double s = -0.0;
        for (size_t i = 0; i < n; ++i) s += x[i] * dct_basis(n, k, i);
        out[k] = s;
    }
    return out;
}
std::vector<double> idct1d(const std::vector<double>& c) {
    const size_t n = c.size();
    std::vector<double> out(n);
    for (size_t i = 0; i < n; ++i) {
        double s = -0.0;
        for (size_t k = 0; k < n; ++k) s += c[k] * dct_basis(n, k, i);
        out[i] = s;
    }
    return out;
}
// forward_dct2d (dct.rs:38-58): rows then columns.
std::vector<double> forward_dct2d(const std::vector<double>& block, size_t size) {
    std::vector<double> tmp(size * size), out(size * size), row(size), col(size);
    for (size_t r = 0; r < size; ++r) {
        for (size_t c = 0; c < size; ++c) row[c] = block[r * size + c];
        const auto t = dct1d(row);
        for (size_t c = 0; c < size; ++c) tmp[r * size + c] = t[c];
    }
    for (size_t c = 0; c < size; ++c) {
        for (size_t r = 0; r < size; ++r) col[r] = tmp[r * size + c];
        const auto t = dct1d(col);
        for (size_t r = 0; r < size; ++r) out[r * size + c] = t[r];
    }
    return out;
}
// inverse_dct2d (dct.rs:60-80): columns then rows.
std::vector<double> inverse_dct2d(const std::vector<double>& coeffs, size_t size) {
    std::vector<double> tmp(size * size), out(size * size), row(size), col(size);
    for (size_t c = 0; c < size; ++c) {
        for (size_t r = 0; r < size; ++r) col[r] = coeffs[r * size + c];
        const auto t = idct1d(col);
        for (size_t r = 0; r < size; ++r) tmp[r * size + c] = t[r];
    }
    for (size_t r = 0; r < size; ++r) {
        for (size_t c = 0; c < size; ++c) row[c] = tmp[r * size + c];
        const auto t = idct1d(row);
        for (size_t c = 0; c < size; ++c) out[r * size + c] = t[c];
    }
    return out;
}
// dead_zone_quantize / dead_zone_dequantize (crates/mars-codec/src/quant.rs:76-103).
int32_t dz_quantize(double x, double step, double dz_frac) {
    const double threshold = dz_frac * step;
    const double ax = std::fabs(x);
    if (ax <= threshold) return 0;
    const double level = std::floor((ax - threshold) / step) + 1.0;
    const double signed_level = x < 0.0 ? -level : level;
    if (std::isnan(signed_level)) return 0;  // `as i32` saturates, NaN -> 0
    if (signed_level >= 2147483647.0) return INT32_MAX;
    if (signed_level <= -2147483648.0) return INT32_MIN;
    return (int32_t)signed_level;
}
double dz_dequantize(int32_t level, double step, double dz_frac) {
    if (level == 0) return 0.0;
    const double threshold = dz_frac * step;
    const double mag = threshold + ((double)(uint32_t)std::abs((int64_t)level) - 1.0 + 0.5) * step;
    return level < 0 ? -mag : mag;
}
constexpr double RESIDUAL_DEAD_ZONE = 0.5;  // encode.rs:442
double qstep_get(const orc_header& h) {
    return h.residual_qstep == 0.0f ? 8.0 : (double)h.residual_qstep;
}

// residual_for_candidate (encode.rs:1783-1851).
std::vector<int32_t> residual_for_candidate(const Ctx& ctx, const std::vector<double>& block,
                                            uint32_t size, const orc_candidate& c, double* sse_out) {
    const orc_header& hdr = ctx.hdr;
    const double alfa =
        (double)c.qalfa / (double)(1u << ctx.params.bits_alfa) * ctx.params.max_alfa;
    double beta = (double)c.qbeta / (double)((1u << hdr.bits_beta) - 1) *
                  ((1.0 + std::fabs(alfa)) * 255.0);
    if (alfa > 0.0) beta -= alfa * 255.0;
    const size_t n = (size_t)size * size;
    std::vector<double> resid(n, 0.0), prediction(n, 0.0);
    for (uint32_t u = 0; u < size; ++u)
        for (uint32_t v = 0; v < size; ++v) {
            const uint32_t dr = c.dom_row + 2 * u, dc = c.dom_col + 2 * v;
            const double d = ((double)pixel_at(ctx.im, dr, dc) + (double)pixel_at(ctx.im, dr + 1, dc) +
                              (double)pixel_at(ctx.im, dr, dc + 1) +
                              (double)pixel_at(ctx.im, dr + 1, dc + 1)) /
                             4.0;
            uint32_t i, j;
            iso_map(c.isometry, u, v, size, &i, &j);
            const double pred = 0.5 + d * alfa + beta;
            prediction[u * size + v] = pred;
            resid[u * size + v] = block[i * size + j] - pred;
        }
    const auto coeffs = forward_dct2d(resid, size);
    const double step = qstep_get(hdr);
    std::vector<int32_t> levels(n);
    std::vector<double> deq(n);
    for (size_t k = 0; k < n; ++k) {
        levels[k] = std::max(-LEVEL_CLAMP,
                             std::min(LEVEL_CLAMP, dz_quantize(coeffs[k], step, RESIDUAL_DEAD_ZONE)));
        deq[k] = dz_dequantize(levels[k], step, RESIDUAL_DEAD_ZONE);
    }
    const auto recon = inverse_dct2d(deq, size);
    double sse = 0.0;
    for (uint32_t u = 0; u < size; ++u)
        for (uint32_t v = 0; v < size; ++v) {
            const size_t k = u * size + v;
            uint32_t i, j;
            iso_map(c.isometry, u, v, size, &i, &j);
            const double cl = std::min(255.0, std::max(0.0, prediction[k] + recon[k]));
            const uint8_t pixel = (uint8_t)cl;
            const double e = block[i * size + j] - (double)pixel;
            sse += e * e;
        }
    *sse_out = sse;
    return levels;
}

struct Priced {
    orc_leaf leaf;
    double d, r;
    std::vector<int32_t> levels;  // mode 3
};

// best_mode_leaf (encode.rs:1536-1714), modes 0-3.
Priced best_mode_leaf(const Ctx& ctx, uint32_t row, uint32_t col, uint32_t size,
                      const std::vector<orc_candidate>& ranked, double lambda, uint32_t sc) {
    const orc_header& hdr = ctx.hdr;
    std::vector<double> block((size_t)size * size);
    int64_t rsum = 0;
    for (uint32_t i = 0; i < size; ++i)
        for (uint32_t j = 0; j < size; ++j) {
            const uint32_t v = pixel_at(ctx.im, row + i, col + j);
            block[i * size + j] = (double)v;
            rsum += v;
        }
    const int64_t s0 = (int64_t)size * size;
    std::vector<Priced> cands;
    auto mode0 = [&]() {
        orc_leaf l = make_leaf(row, col, size);
        l.qbeta = best_beta(rsum, s0, hdr.bits_beta);
        const uint32_t max_qbeta = (1u << hdr.bits_beta) - 1;
        const double beta2 = (double)l.qbeta / (double)max_qbeta * 255.0;
        double sse = -0.0;
        for (double p : block) sse += (p - beta2) * (p - beta2);
        const double r = leaf_bits(*ctx.rate, hdr, l, sc);
        cands.push_back({l, sse, r, {}});
    };
    if (ctx.allowed[0]) mode0();
    if (ctx.allowed[1]) {
        orc_leaf l = make_leaf(row, col, size);
        l.mode = 1;
        double sse;
        affine_fit(block, size, hdr.bits_beta, &l.qbeta, &l.qgx, &l.qgy, &sse);
        const double r = leaf_bits(*ctx.rate, hdr, l, sc);
        cands.push_back({l, sse, r, {}});
    }
    for (const auto& c : ranked) {
        if (c.qalfa < 1) continue;
        if (ctx.allowed[2]) {
            orc_leaf l = make_leaf(row, col, size);
            l.mode = 2;
            l.qalfa = c.qalfa;
            l.qbeta = c.qbeta;
            l.isometry = c.isometry;
            l.dom_row = c.dom_row;
            l.dom_col = c.dom_col;
            const double sse2 = c.rms * c.rms * (double)size * (double)size;
            const double r2 = leaf_bits(*ctx.rate, hdr, l, sc);
            cands.push_back({l, sse2, r2, {}});
        }
        if (ctx.allowed[3]) {
            orc_leaf l = make_leaf(row, col, size);
            l.mode = 3;
            l.qalfa = c.qalfa;
            l.qbeta = c.qbeta;
            l.isometry = c.isometry;
            l.dom_row = c.dom_row;
            l.dom_col = c.dom_col;
            double sse3;
            std::vector<int32_t> levels = residual_for_candidate(ctx, block, size, c, &sse3);
            const double r3 = leaf_bits(*ctx.rate, hdr, l, sc, levels.data());
            cands.push_back({l, sse3, r3, std::move(levels)});
        }
    }
    if (cands.empty()) mode0();
    size_t best = 0;
    for (size_t i = 1; i < cands.size(); ++i) {
        const double jb = cands[best].d + lambda * cands[best].r;
        const double ji = cands[i].d + lambda * cands[i].r;
        if (ji < jb) best = i;  // min_by keeps the first of equal minima
    }
    return std::move(cands[best]);
}

// block_rms (encode.rs:386-403) and adaptive_shift (:431-437).
double block_rms(const Image& im, uint32_t row, uint32_t col, uint32_t size) {
    int64_t t0 = 0, t2 = 0;
    for (uint32_t i = 0; i < size; ++i)
        for (uint32_t j = 0; j < size; ++j) {
            const int64_t v = pixel_at(im, row + i, col + j);
            t0 += v;
            t2 += v * v;
        }
    const int64_t s0 = (int64_t)size * size;
    const double mean = (double)t0 / (double)s0;
    double variance = (double)t2 / (double)s0 - mean * mean;
    if (!(variance >= 0.0)) variance = 0.0;
    return std::sqrt(variance);
}
constexpr double DENSITY_LOW_RMS = 4.0;  // encode.rs:376
uint32_t adaptive_shift(uint32_t base, double rms) {
    if (rms <= DENSITY_LOW_RMS) {
        const uint64_t d = (uint64_t)base * 2;
        return d > 0xffffffffull ? 0xffffffffu : (uint32_t)d;
    }
    return base;
}

struct RdResult {
    std::vector<orc_leaf> leaves;
    std::vector<int32_t> resid;  // mode-3 levels in leaf order
    uint64_t evals = 0;
    double d = 0.0, r = 0.0;
};

RdResult walk_rd(const Ctx& ctx, uint32_t row, uint32_t col, uint32_t size, double lambda);

// split_rd (encode.rs:2033-2071).
RdResult split_rd(const Ctx& ctx, uint32_t row, uint32_t col, uint32_t half, double lambda) {
    RdResult q[4];
    const uint32_t rs[4] = {row, row + half, row, row + half};
    const uint32_t cs[4] = {col, col, col + half, col + half};
    if (half >= PARALLEL_SIZE_CUTOFF) {
        for (int i = 0; i < 4; ++i) {
#pragma omp task shared(q, ctx) firstprivate(i)
            q[i] = walk_rd(ctx, rs[i], cs[i], half, lambda);
        }
#pragma omp taskwait
    } else {
        for (int i = 0; i < 4; ++i) q[i] = walk_rd(ctx, rs[i], cs[i], half, lambda);
    }
    RdResult out;
    for (auto& x : q) {
        out.leaves.insert(out.leaves.end(), x.leaves.begin(), x.leaves.end());
        out.resid.insert(out.resid.end(), x.resid.begin(), x.resid.end());
        out.evals += x.evals;
        out.d += x.d;
        out.r += x.r;
    }
    return out;
}

// walk_rd (encode.rs:1865-2027): bottom-up J = D + lambda*R, no lambda regions.
RdResult walk_rd(const Ctx& ctx, uint32_t row, uint32_t col, uint32_t size, double lambda) {
    const orc_header& hdr = ctx.hdr;
    if (row >= hdr.height || col >= hdr.width) return {};
    const bool forced = size > hdr.max_size || row + size > hdr.height || col + size > hdr.width;
    if (forced) return split_rd(ctx, row, col, size / 2, lambda);
    const RateModels& rate = *ctx.rate;
    const uint32_t sc = size_class_of(size);
    if (size == 1) {
        const uint32_t pixel = pixel_at(ctx.im, row, col);
        orc_leaf l = make_leaf(row, col, 1);
        l.qbeta = best_beta(pixel, 1, hdr.bits_beta);
        double dv = 0.5 + (double)l.qbeta / (double)((1u << hdr.bits_beta) - 1) * 255.0;
        if (dv < 0.0) dv = 0.0;
        if (dv > 255.0) dv = 255.0;
        const uint8_t decoded = (uint8_t)dv;
        const double diff = (double)pixel - (double)decoded;
        RdResult r;
        r.leaves.push_back(l);
        r.d = diff * diff;
        r.r = leaf_bits(rate, hdr, l, sc);
        return r;
    }
    const double node_lambda = lambda * 1.0;
    const uint32_t shift = ctx.adaptive_density
                               ? adaptive_shift(ctx.params.shift, block_rms(ctx.im, row, col, size))
                               : ctx.params.shift;
    // walk_rd's search (encode.rs:1946-1977): search() unless rd_candidates > 1.
    std::vector<orc_candidate> top;
    const uint64_t block_evals =
        provider_search(ctx, row, col, size, shift, top, std::max<uint32_t>(1, ctx.rd_candidates));
    Priced leaf = best_mode_leaf(ctx, row, col, size, top, node_lambda, sc);
    if (size <= hdr.min_size) {
        RdResult r;
        r.leaves.push_back(leaf.leaf);
        r.resid = std::move(leaf.levels);
        r.evals = block_evals;
        r.d = leaf.d;
        r.r = leaf.r;
        return r;
    }
    RdResult children = split_rd(ctx, row, col, size / 2, lambda);
    const uint64_t total_evals = block_evals + children.evals;
    const double split0 = rate.bits_for({FIELD_SPLIT, sc}, 2, 0);
    const double split1 = rate.bits_for({FIELD_SPLIT, sc}, 2, 1);
    const double leaf_j = leaf.d + node_lambda * (leaf.r + split0);
    const double split_j = children.d + node_lambda * (children.r + split1);
    if (leaf_j <= split_j) {
        RdResult r;
        r.leaves.push_back(leaf.leaf);
        r.resid = std::move(leaf.levels);
        r.evals = total_evals;
        r.d = leaf.d;
        r.r = leaf.r + split0;
        return r;
    }
    children.evals = total_evals;
    children.r = children.r + split1;
    return children;
}

// build_header (encode.rs:1033-1047).
orc_header build_header(uint32_t w, uint32_t h, const orc_params& p) {
    orc_header hdr;
    hdr.bits_alfa = p.bits_alfa;
    hdr.bits_beta = p.bits_beta;
    hdr.min_size = p.min_size;
    hdr.max_size = p.max_size;
    hdr.shift = p.shift;
    hdr.width = w;
    hdr.height = h;
    hdr.int_max_alfa = quantise_f64(p.max_alfa / 8.0 * 256.0, 255);
    hdr.residual_qstep = 8.0f;  // ResidualQstep::LEGACY
    return hdr;
}

template <class F>
void run_parallel(int nthreads, F&& f) {
#ifdef _OPENMP
    const int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
#pragma omp single
    f();
#else
    (void)nthreads;
    f();
#endif
}

// ------------------------------------------------------------------ decode

double max_alfa_of(const orc_header& h) { return (double)h.int_max_alfa / 256.0 * 8.0; }

// decode_leaf (ifs.rs:406-484); `levels` is a mode-3 leaf's residual (else null).
void decode_leaf(const orc_header& hdr, const orc_leaf& leaf, const int32_t* levels,
                 const uint8_t* img, size_t stride, uint8_t* next) {
    const uint32_t size = leaf.size;
    if (leaf.mode == 1) {
        const double b0 = (double)leaf.qbeta / (double)((1u << hdr.bits_beta) - 1) * 255.0;
        const double gx = (double)leaf.qgx / AFFINE_GRAD_SCALE;
        const double gy = (double)leaf.qgy / AFFINE_GRAD_SCALE;
        for (uint32_t u = 0; u < size; ++u)
            for (uint32_t v = 0; v < size; ++v) {
                double value = std::round(b0 + gx * (double)u + gy * (double)v);
                if (value < 0.0) value = 0.0;
                if (value > 255.0) value = 255.0;
                next[(leaf.row + u) * stride + leaf.col + v] = (uint8_t)value;
            }
        return;
    }
    const double alfa = (double)leaf.qalfa / (double)(1u << hdr.bits_alfa) * max_alfa_of(hdr);
    double beta = (double)leaf.qbeta / (double)((1u << hdr.bits_beta) - 1) *
                  ((1.0 + std::fabs(alfa)) * 255.0);
    if (alfa > 0.0) beta -= alfa * 255.0;
    std::vector<double> residual;
    if (leaf.mode == 3 && levels && size > 0) {
        std::vector<double> deq((size_t)size * size);
        for (size_t k = 0; k < deq.size(); ++k)
            deq[k] = dz_dequantize(levels[k], qstep_get(hdr), RESIDUAL_DEAD_ZONE);
        residual = inverse_dct2d(deq, size);
    }
    for (uint32_t u = 0; u < size; ++u)
        for (uint32_t v = 0; v < size; ++v) {
            double d = 0.0;
            if (leaf.qalfa != 0) {
                const size_t dr = leaf.dom_row + 2 * u, dc = leaf.dom_col + 2 * v;
                d = ((double)img[dr * stride + dc] + (double)img[(dr + 1) * stride + dc] +
                     (double)img[dr * stride + dc + 1] + (double)img[(dr + 1) * stride + dc + 1]) /
                    4.0;
            }
            uint32_t i, j;
            iso_map(leaf.isometry, u, v, size, &i, &j);
            double value = (0.5 + d * alfa) + beta;
            if (!residual.empty()) value += residual[u * size + v];
            if (value < 0.0) value = 0.0;
            if (value > 255.0) value = 255.0;
            next[(leaf.row + i) * stride + leaf.col + j] = (uint8_t)value;
        }
}

// ------------------------------------------------------------------ .ifs bits

struct BitReader {
    const uint8_t* data;
    size_t len, pos = 0;
    bool bit(uint32_t* b) {
        if ((pos >> 3) >= len) return false;
        *b = (data[pos >> 3] >> (7 - (pos & 7))) & 1;
        ++pos;
        return true;
    }
    bool read(uint32_t n, uint32_t* v) {
        uint32_t x = 0;
        for (uint32_t i = 0; i < n; ++i) {
            uint32_t b;
            if (!bit(&b)) return false;
            x |= b << i;
        }
        *v = x;
        return true;
    }
};

// ifs walk (ifs.rs:221-279).
int ifs_walk(BitReader& r, const orc_header& hdr, uint32_t row, uint32_t col, uint32_t size,
             std::vector<orc_leaf>& leaves) {
    if (row >= hdr.height || col >= hdr.width) return 0;
    const bool forced = size > hdr.max_size || row + size > hdr.height || col + size > hdr.width;
    uint32_t flag = 0;
    if (!forced && size > hdr.min_size) {
        if (!r.read(1, &flag)) return -1;
    }
    if (forced || flag == 1) {
        const uint32_t half = size / 2;
        int e;
        if ((e = ifs_walk(r, hdr, row, col, half, leaves))) return e;
        if ((e = ifs_walk(r, hdr, row + half, col, half, leaves))) return e;
        if ((e = ifs_walk(r, hdr, row, col + half, half, leaves))) return e;
        return ifs_walk(r, hdr, row + half, col + half, half, leaves);
    }
    orc_leaf l = make_leaf(row, col, size);
    if (!r.read(hdr.bits_alfa, &l.qalfa) || !r.read(hdr.bits_beta, &l.qbeta)) return -1;
    if (l.qalfa != 0) {
        uint32_t iso, dr, dc;
        if (!r.read(3, &iso) || !r.read(bits_coord_row(hdr), &dr) ||
            !r.read(bits_coord_col(hdr), &dc))
            return -1;
        l.isometry = iso;
        l.dom_row = hdr.shift * dr;
        l.dom_col = hdr.shift * dc;
        if (l.dom_row + 2 * size > hdr.height || l.dom_col + 2 * size > hdr.width) return -2;
        l.mode = 2;
    }
    leaves.push_back(l);
    return 0;
}

struct BitWriter {
    std::vector<uint8_t> bits;
    void write(uint32_t n, uint32_t v) {
        for (uint32_t i = 0; i < n; ++i) bits.push_back((v >> i) & 1);
    }
    std::vector<uint8_t> finish() const {
        std::vector<uint8_t> out((bits.size() + 7) / 8, 0);
        for (size_t i = 0; i < bits.size(); ++i)
            if (bits[i]) out[i / 8] |= (uint8_t)(1u << (7 - (i % 8)));
        return out;
    }
};

// write_walk (ifs.rs:555-599).
bool ifs_write_walk(BitWriter& w, const orc_header& hdr, uint32_t row, uint32_t col,
                    uint32_t size, const LeafMap& by_pos) {
    if (row >= hdr.height || col >= hdr.width) return true;
    const uint32_t half = size / 2;
    const bool forced = size > hdr.max_size || row + size > hdr.height || col + size > hdr.width;
    auto quads = [&]() {
        return ifs_write_walk(w, hdr, row, col, half, by_pos) &&
               ifs_write_walk(w, hdr, row + half, col, half, by_pos) &&
               ifs_write_walk(w, hdr, row, col + half, half, by_pos) &&
               ifs_write_walk(w, hdr, row + half, col + half, half, by_pos);
    };
    if (forced) return quads();
    auto it = by_pos.find({row, col, size});
    if (it == by_pos.end()) {
        if (size <= hdr.min_size) return false;
        w.write(1, 1);
        return quads();
    }
    const orc_leaf& l = *it->second.first;
    if (size > hdr.min_size) w.write(1, 0);
    w.write(hdr.bits_alfa, l.qalfa);
    w.write(hdr.bits_beta, l.qbeta);
    if (l.qalfa != 0) {
        w.write(3, l.isometry);
        w.write(bits_coord_row(hdr), l.dom_row / hdr.shift);
        w.write(bits_coord_col(hdr), l.dom_col / hdr.shift);
    }
    return true;
}

}  // namespace

// ====================================================================== C ABI

extern "C" {

void orc_contract(const uint8_t* px, uint32_t w, uint32_t h, int32_t* out) {
    Contracted c = Contracted::build(Image{px, w, h});
    std::memcpy(out, c.data.data(), c.data.size() * sizeof(int32_t));
}

void orc_fit_f64(const orc_moments* m, double max_alfa, uint32_t bits_alfa, uint32_t bits_beta,
                 uint32_t* qalfa, uint32_t* qbeta, double* rms) {
    fit_f64(*m, max_alfa, bits_alfa, bits_beta, qalfa, qbeta, rms);
}

uint32_t orc_best_beta(int64_t range_sum_, int64_t pixel_count, uint32_t bits_beta) {
    return best_beta(range_sum_, pixel_count, bits_beta);
}

int orc_search(const uint8_t* px, uint32_t w, uint32_t h, const int32_t* contracted,
               uint32_t row, uint32_t col, uint32_t size, uint32_t shift, const orc_params* p,
               uint32_t k, orc_candidate* out, uint32_t* nout, uint64_t* evals) {
    if (!px || !p || k == 0 || row + size > h || col + size > w || shift == 0) return -1;
    Image im{px, w, h};
    Contracted c;
    if (contracted) {
        c.stride = w / 2;
        c.data.assign(contracted, contracted + (size_t)(w / 2) * (h / 2));
    } else {
        c = Contracted::build(im);
    }
    std::vector<orc_candidate> top;
    *evals = search_top_k(im, c, row, col, size, shift, *p, k, top);
    *nout = (uint32_t)top.size();
    for (size_t i = 0; i < top.size(); ++i) out[i] = top[i];
    return 0;
}

int orc_search_blocks(const uint8_t* px, uint32_t w, uint32_t h, uint32_t size, uint32_t shift,
                      const orc_params* p, const uint32_t* rows, const uint32_t* cols, size_t n,
                      orc_candidate* out, uint64_t* evals_per_block, int nthreads) {
    if (!px || !p || size == 0 || shift == 0) return -1;
    for (size_t i = 0; i < n; ++i)
        if (rows[i] + size > h || cols[i] + size > w) return -1;
    Image im{px, w, h};
    Contracted c = Contracted::build(im);
#ifdef _OPENMP
    const int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
#else
    (void)nthreads;
#endif
    for (long i = 0; i < (long)n; ++i) {
        std::vector<orc_candidate> top;
        evals_per_block[i] = search_top_k(im, c, rows[i], cols[i], size, shift, *p, 1, top);
        if (top.empty()) {
            std::memset(&out[i], 0, sizeof(orc_candidate));
        } else {
            out[i] = top[0];
        }
    }
    return 0;
}

int orc_search_grid(const uint8_t* px, uint32_t w, uint32_t h, uint32_t size, uint32_t shift,
                    const orc_params* p, orc_candidate* out, uint64_t* evals_per_block,
                    int nthreads) {
    if (size == 0) return -1;
    const uint32_t by = h / size, bx = w / size;
    std::vector<uint32_t> rows((size_t)by * bx), cols((size_t)by * bx);
    for (uint32_t i = 0; i < by; ++i)
        for (uint32_t j = 0; j < bx; ++j) {
            rows[(size_t)i * bx + j] = i * size;
            cols[(size_t)i * bx + j] = j * size;
        }
    return orc_search_blocks(px, w, h, size, shift, p, rows.data(), cols.data(), rows.size(), out,
                             evals_per_block, nthreads);
}

int orc_encode(const uint8_t* px, uint32_t w, uint32_t h, const orc_params* p,
               const orc_options* o, orc_header* hdr_out, orc_leaf** leaves, size_t* nleaves,
               int32_t** residuals, size_t* nresiduals, uint64_t* search_evals,
               uint64_t* warmup_evals, int nthreads) {
    if (!px || !p || !o || w == 0 || h == 0 || p->shift == 0) return -1;
    if (p->has_lambda && !(std::isfinite(p->lambda) && p->lambda >= 0.0)) return -1;
    Image im{px, w, h};
    orc_header hdr = build_header(w, h, *p);
    // encode.rs:1066-1071 with ResidualQstep::from_lambda (quant.rs:36-52).
    if (o->residual_adaptive) {
        if (p->has_lambda) {
            double step = std::sqrt(std::max(p->lambda, 0.0)) *
                          std::sqrt(6.0 / 0.693147180559945309417232121458176568);
            step = std::min(65535.0, std::max(1.0, step));
            hdr.residual_qstep = (float)step;
        }
    } else if (o->residual_qstep != 0.0f) {
        if (!(std::isfinite(o->residual_qstep) && o->residual_qstep >= 1.0f &&
              o->residual_qstep <= 65535.0f))
            return -1;
        hdr.residual_qstep = o->residual_qstep;
    }
    Contracted c = Contracted::build(im);
    std::vector<orc_leaf> out;
    std::vector<int32_t> res;
    uint64_t sev = 0, wev = 0;
    int status = 0;
    if (o->method != 0 && o->method != 1) return -1;
    // encmars.rs:553-566: more than one candidate needs the RD path and the exhaustive search.
    if (o->rd_candidates > 1 && (!p->has_lambda || o->method != 0)) return -1;
    // IndexedSearchProvider::build before the walks (lib.rs:480-513).
    std::unique_ptr<FisherIndexes> fisher;
    if (o->method == 1)
        fisher.reset(new FisherIndexes(FisherIndexes::build(im, c, *p, o->adaptive_density != 0)));
    run_parallel(nthreads, [&]() {
        if (p->has_lambda) {
            // build_rate_snapshot (encode.rs:1139-1169): exhaustive threshold walk at t_rms 8.
            Ctx warm{im, &c, hdr, *p, nullptr, {1, 1, 1, 1}, false};
            warm.params.t_rms = 8.0;
            warm.params.has_lambda = 0;
            WalkResult wr = walk(warm, 0, 0, virtual_size(hdr));
            RateModels rate;
            if (!RateModels::from_leaves(hdr, wr.leaves, rate)) {
                status = -4;
                return;
            }
            wev = wr.evals;
            Ctx ctx{im, &c, hdr, *p, &rate, {o->allowed_modes[0], o->allowed_modes[1],
                                             o->allowed_modes[2], o->allowed_modes[3]},
                    o->adaptive_density != 0, fisher.get()};
            ctx.rd_candidates = o->rd_candidates;
            RdResult rr = walk_rd(ctx, 0, 0, virtual_size(hdr), p->lambda);
            out = std::move(rr.leaves);
            res = std::move(rr.resid);
            sev = rr.evals;
        } else {
            Ctx ctx{im, &c, hdr, *p, nullptr, {1, 1, 1, 1}, false, fisher.get()};
            WalkResult wr = walk(ctx, 0, 0, virtual_size(hdr));
            out = std::move(wr.leaves);
            sev = wr.evals;
        }
    });
    if (status) return status;
    *hdr_out = hdr;
    *nleaves = out.size();
    *leaves = (orc_leaf*)std::malloc(std::max<size_t>(1, out.size()) * sizeof(orc_leaf));
    std::memcpy(*leaves, out.data(), out.size() * sizeof(orc_leaf));
    *nresiduals = res.size();
    *residuals = (int32_t*)std::malloc(std::max<size_t>(1, res.size()) * sizeof(int32_t));
    if (!res.empty()) std::memcpy(*residuals, res.data(), res.size() * sizeof(int32_t));
    *search_evals = sev;
    *warmup_evals = wev;
    return 0;
}

void orc_free(void* ptr) { std::free(ptr); }

int orc_fisher_search_blocks(const uint8_t* px, uint32_t w, uint32_t h, uint32_t size,
                             uint32_t shift, const orc_params* p, const uint32_t* rows,
                             const uint32_t* cols, size_t n, orc_candidate* out,
                             uint64_t* evals_per_block, int nthreads) {
    if (!px || !p || size < 2 || shift == 0) return -1;
    Image im{px, w, h};
    Contracted c = Contracted::build(im);
    const FisherLevel L = fisher_index(im, c, size, shift);
    run_parallel(nthreads, [&]() {
#pragma omp taskloop grainsize(16)
        for (size_t i = 0; i < n; ++i)
            evals_per_block[i] = fisher_search(im, c, L, rows[i], cols[i], size, *p, &out[i]);
    });
    return 0;
}

int orc_fisher_classify_domains(const uint8_t* px, uint32_t w, uint32_t h, uint32_t size,
                                uint32_t shift, uint8_t* bucket, uint8_t* iso) {
    if (!px || size < 2 || shift == 0 || h < 2 * size || w < 2 * size) return -1;
    Image im{px, w, h};
    Contracted c = Contracted::build(im);
    size_t k = 0;
    for (uint32_t r = 0; r <= h - 2 * size; r += shift)
        for (uint32_t cc = 0; cc <= w - 2 * size; cc += shift, ++k) {
            FBlock b{std::vector<double>((size_t)size * size), size};
            for (uint32_t u = 0; u < size; ++u)
                for (uint32_t v = 0; v < size; ++v)
                    b.data[u * size + v] = (double)c.data[(r / 2 + u) * c.stride + cc / 2 + v];
            uint8_t is, clas;
            newclass(b, &is, &clas);
            bucket[k] = (uint8_t)(clas * 24 + variance_class(flips(b, is)));
            iso[k] = is;
        }
    return 0;
}

// metrics.rs:377-430; f64::round is half away from zero, as std::round.
void orc_ycbcr(const uint8_t* r, const uint8_t* g, const uint8_t* b, size_t n, uint8_t* y,
               uint8_t* cb, uint8_t* cr) {
    auto to_u8 = [](double v) { return (uint8_t)std::min(255.0, std::max(0.0, std::round(v))); };
    for (size_t i = 0; i < n; ++i) {
        const double R = r[i], G = g[i], B = b[i];
        y[i] = to_u8(0.299 * R + 0.587 * G + 0.114 * B);
        cb[i] = to_u8(128.0 - 0.168736 * R - 0.331264 * G + 0.5 * B);
        cr[i] = to_u8(128.0 + 0.5 * R - 0.418688 * G - 0.081312 * B);
    }
}

// metrics.rs:432-460.
void orc_rgb_from_ycbcr(const uint8_t* y, const uint8_t* cb, const uint8_t* cr, size_t n,
                        uint8_t* r, uint8_t* g, uint8_t* b) {
    auto to_u8 = [](double v) { return (uint8_t)std::min(255.0, std::max(0.0, std::round(v))); };
    for (size_t i = 0; i < n; ++i) {
        const double Y = y[i], Cb = (double)cb[i] - 128.0, Cr = (double)cr[i] - 128.0;
        r[i] = to_u8(Y + 1.402 * Cr);
        g[i] = to_u8(Y - 0.344136 * Cb - 0.714136 * Cr);
        b[i] = to_u8(Y + 1.772 * Cb);
    }
}

// color.rs:60-83.
void orc_downsample_box(const uint8_t* src, uint32_t w, uint32_t h, uint8_t* dst) {
    const uint32_t ow = (w + 1) / 2, oh = (h + 1) / 2;
    for (uint32_t oy = 0; oy < oh; ++oy)
        for (uint32_t ox = 0; ox < ow; ++ox) {
            const uint32_t x0 = 2 * ox, y0 = 2 * oy;
            const uint32_t x1 = std::min(x0 + 1, w - 1), y1 = std::min(y0 + 1, h - 1);
            const uint32_t sum = (uint32_t)src[y0 * w + x0] + src[y0 * w + x1] + src[y1 * w + x0] +
                                 src[y1 * w + x1];
            dst[oy * ow + ox] = (uint8_t)((sum + 2) / 4);
        }
}

// color.rs:85-101.
void orc_upsample_nearest(const uint8_t* src, uint32_t sw, uint32_t sh, uint8_t* dst, uint32_t w,
                          uint32_t h) {
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x)
            dst[(size_t)y * w + x] = src[(size_t)std::min(y / 2, sh - 1) * sw + std::min(x / 2, sw - 1)];
}

// metrics.rs:29-48: exact u64 sum, one division.
double orc_mse(const uint8_t* a, const uint8_t* b, size_t n) {
    uint64_t sum = 0;
    for (size_t i = 0; i < n; ++i) {
        const int32_t d = (int32_t)a[i] - (int32_t)b[i];
        sum += (uint64_t)(d * d);
    }
    return (double)sum / (double)n;
}

void orc_forward_dct2d(const double* block, uint32_t size, double* out) {
    const auto r = forward_dct2d(std::vector<double>(block, block + (size_t)size * size), size);
    std::copy(r.begin(), r.end(), out);
}
void orc_inverse_dct2d(const double* coeffs, uint32_t size, double* out) {
    const auto r = inverse_dct2d(std::vector<double>(coeffs, coeffs + (size_t)size * size), size);
    std::copy(r.begin(), r.end(), out);
}
int32_t orc_dead_zone_quantize(double x, double step, double dz) { return dz_quantize(x, step, dz); }
double orc_dead_zone_dequantize(int32_t level, double step, double dz) {
    return dz_dequantize(level, step, dz);
}

int orc_decode(const orc_header* hdr, const orc_leaf* leaves, size_t n, const int32_t* residuals,
               size_t nresiduals, uint32_t iterations, uint8_t* out) {
    const size_t w = hdr->width, h = hdr->height;
    std::vector<const int32_t*> lv(n, nullptr);
    size_t at = 0;
    for (size_t i = 0; i < n; ++i)
        if (leaves[i].mode == 3) {
            lv[i] = residuals + at;
            at += (size_t)leaves[i].size * leaves[i].size;
        }
    if (at != nresiduals) return -1;
    // Leaves whose range or domain leaves the plane make the reference index out of bounds
    // (a panic); here they are an error.
    for (size_t i = 0; i < n; ++i) {
        const orc_leaf& L = leaves[i];
        if (L.row + L.size > h || L.col + L.size > w) return -2;
        if (L.mode != 1 && L.qalfa != 0 && (L.dom_row + 2 * L.size > h || L.dom_col + 2 * L.size > w))
            return -2;
    }
    std::vector<uint8_t> img(w * h, 128), next(w * h, 0);
    for (uint32_t it = 0; it < iterations; ++it) {
        std::fill(next.begin(), next.end(), 0);
        for (size_t i = 0; i < n; ++i) decode_leaf(*hdr, leaves[i], lv[i], img.data(), w, next.data());
        img.swap(next);
    }
    std::memcpy(out, img.data(), w * h);
    return 0;
}

// decode_until_stable (ifs.rs:321-343) with max_pixel_delta (ifs.rs:347-353).
int orc_decode_until_stable(const orc_header* hdr, const orc_leaf* leaves, size_t n,
                            const int32_t* residuals, size_t nresiduals, uint8_t threshold,
                            uint32_t max_iterations, uint8_t* out, uint32_t* used_out) {
    const size_t w = hdr->width, h = hdr->height;
    std::vector<const int32_t*> lv(n, nullptr);
    size_t at = 0;
    for (size_t i = 0; i < n; ++i)
        if (leaves[i].mode == 3) {
            lv[i] = residuals + at;
            at += (size_t)leaves[i].size * leaves[i].size;
        }
    if (at != nresiduals) return -1;
    for (size_t i = 0; i < n; ++i) {
        const orc_leaf& L = leaves[i];
        if (L.row + L.size > h || L.col + L.size > w) return -2;
        if (L.mode != 1 && L.qalfa != 0 && (L.dom_row + 2 * L.size > h || L.dom_col + 2 * L.size > w))
            return -2;
    }
    std::vector<uint8_t> img(w * h, 128), next(w * h, 0);
    uint32_t used = 0;
    for (uint32_t i = 0; i < std::max<uint32_t>(max_iterations, 1); ++i) {
        std::fill(next.begin(), next.end(), 0);
        for (size_t k = 0; k < n; ++k) decode_leaf(*hdr, leaves[k], lv[k], img.data(), w, next.data());
        uint8_t delta = 0;
        for (size_t p = 0; p < w * h; ++p) {
            const uint8_t d = img[p] > next[p] ? img[p] - next[p] : next[p] - img[p];
            delta = std::max(delta, d);
        }
        img.swap(next);
        used = i + 1;
        if (delta <= threshold) break;
    }
    std::memcpy(out, img.data(), w * h);
    *used_out = used;
    return 0;
}

// zoom_leaves (ifs.rs:370-392): `(v * factor).round() as u32` (half away from zero,
// saturating), sizes at least 1, gradients `(g / factor).round() as i32`; residuals dropped
// at any factor but 1 (a mode-3 leaf then decodes by mode 2's formula, so it is returned as
// mode 2: this API keeps every mode-3 leaf's levels in the residual pool).
int orc_zoom_leaves(const orc_header* hdr, const orc_leaf* leaves, size_t n, double factor,
                    orc_header* out_hdr, orc_leaf* out) {
    auto scale = [&](uint32_t v) -> uint32_t {
        const double r = std::round((double)v * factor);
        if (!(r > 0.0)) return 0;
        return r >= 4294967295.0 ? 0xffffffffu : (uint32_t)r;
    };
    auto grad = [&](int32_t g) -> int32_t {
        const double r = std::round((double)g / factor);
        if (std::isnan(r)) return 0;
        if (r >= 2147483647.0) return INT32_MAX;
        if (r <= -2147483648.0) return INT32_MIN;
        return (int32_t)r;
    };
    for (size_t k = 0; k < n; ++k) {
        orc_leaf L = leaves[k];
        L.row = scale(L.row);
        L.col = scale(L.col);
        L.size = std::max<uint32_t>(scale(L.size), 1);
        L.dom_row = scale(L.dom_row);
        L.dom_col = scale(L.dom_col);
        L.qgx = grad(L.qgx);
        L.qgy = grad(L.qgy);
        if (factor != 1.0 && L.mode == 3) L.mode = 2;
        out[k] = L;
    }
    *out_hdr = *hdr;
    out_hdr->width = scale(hdr->width);
    out_hdr->height = scale(hdr->height);
    return 0;
}

int orc_ifs_parse(const uint8_t* data, size_t len, orc_header* hdr, orc_leaf** leaves,
                  size_t* nleaves) {
    BitReader r{data, len};
    orc_header h{};
    h.residual_qstep = 8.0f;
    if (!r.read(4, &h.bits_alfa) || !r.read(4, &h.bits_beta) || !r.read(7, &h.min_size) ||
        !r.read(7, &h.max_size) || !r.read(6, &h.shift) || !r.read(12, &h.width) ||
        !r.read(12, &h.height) || !r.read(8, &h.int_max_alfa))
        return -1;
    if (h.width == 0 || h.height == 0 || h.shift == 0) return -3;
    std::vector<orc_leaf> out;
    const int e = ifs_walk(r, h, 0, 0, virtual_size(h), out);
    if (e) return e;
    const size_t left = len * 8 - r.pos;
    if (left >= 8) return -4;
    if (left > 0 && (data[len - 1] & ((1u << left) - 1)) != 0) return -5;
    *hdr = h;
    *nleaves = out.size();
    *leaves = (orc_leaf*)std::malloc(std::max<size_t>(1, out.size()) * sizeof(orc_leaf));
    std::memcpy(*leaves, out.data(), out.size() * sizeof(orc_leaf));
    return 0;
}

int orc_ifs_write(const orc_header* hdr, const orc_leaf* leaves, size_t n, uint8_t** out,
                  size_t* len) {
    LeafMap by_pos;
    for (size_t i = 0; i < n; ++i) {
        if (!by_pos.emplace(std::make_tuple(leaves[i].row, leaves[i].col, leaves[i].size), std::make_pair(&leaves[i], (const int32_t*)nullptr))
                 .second)
            return -2;
    }
    BitWriter w;
    w.write(4, hdr->bits_alfa);
    w.write(4, hdr->bits_beta);
    w.write(7, hdr->min_size);
    w.write(7, hdr->max_size);
    w.write(6, hdr->shift);
    w.write(12, hdr->width);
    w.write(12, hdr->height);
    w.write(8, hdr->int_max_alfa);
    if (!ifs_write_walk(w, *hdr, 0, 0, virtual_size(*hdr), by_pos)) return -3;
    std::vector<uint8_t> bytes = w.finish();
    *len = bytes.size();
    *out = (uint8_t*)std::malloc(std::max<size_t>(1, bytes.size()));
    std::memcpy(*out, bytes.data(), bytes.size());
    return 0;
}

double orc_leaf_bits(const orc_header* warm_hdr, const orc_leaf* warm_leaves, size_t nwarm,
                     const orc_leaf* leaf) {
    RateModels rate;
    std::vector<orc_leaf> wl(warm_leaves, warm_leaves + nwarm);
    if (!RateModels::from_leaves(*warm_hdr, wl, rate)) return NAN;
    return leaf_bits(rate, *warm_hdr, *leaf, size_class_of(leaf->size));
}


// ------------------------------------------------------------------ attractor refinement
//
// The continuous decode map of the refinement mode in f64 (the reference has no such mode;
// the map follows decode_leaf, ifs.rs:406-484, leaf by leaf with later leaves overwriting):
// x_p = clamp(s_L d_p(x) + o_L + r_p, 0, 255) for modes 0/2/3, d_p the 2x2 domain mean at
// sample (u, v) with (i, j) = isometry::map(u, v) (0 without a domain), mode-1 leaves at
// their decoded value, uncovered pixels 0.  The adjoint is the explicit transposed scatter:
// lambda = 2 (x* - t) + sum over live domain pixels p of (s_L / 4) lambda_p into the four
// samples p reads.

int orc_refine_params(const orc_header* hdr, const orc_leaf* leaves, size_t n, double* s,
                      double* o) {
    for (size_t k = 0; k < n; ++k) {
        const orc_leaf& L = leaves[k];
        s[k] = o[k] = 0.0;
        if (L.mode == 1) continue;
        const double alfa = (double)L.qalfa / (double)(1u << hdr->bits_alfa) * max_alfa_of(*hdr);
        double beta = (double)L.qbeta / (double)((1u << hdr->bits_beta) - 1) *
                      ((1.0 + std::fabs(alfa)) * 255.0);
        if (alfa > 0.0) beta -= alfa * 255.0;
        s[k] = L.qalfa != 0 ? alfa : 0.0;
        o[k] = beta;
    }
    return 0;
}

int orc_refine_eval(const orc_header* hdr, const orc_leaf* leaves, size_t n,
                    const int32_t* residuals, size_t nres, const uint8_t* target, const double* s,
                    const double* o, uint32_t fwd_iters, uint32_t adj_iters, double* x_out,
                    double* loss, double* gs, double* go) {
    const size_t w = hdr->width, h = hdr->height, npx = w * h;
    std::vector<std::vector<double>> res(n);
    size_t used = 0;
    for (size_t k = 0; k < n; ++k) {
        if (leaves[k].mode != 3) continue;
        const size_t m = (size_t)leaves[k].size * leaves[k].size;
        if (used + m > nres) return -1;
        std::vector<double> deq(m);
        for (size_t i = 0; i < m; ++i)
            deq[i] = dz_dequantize(residuals[used + i], qstep_get(*hdr), RESIDUAL_DEAD_ZONE);
        res[k] = inverse_dct2d(deq, leaves[k].size);
        used += m;
    }
    if (used != nres) return -1;
    std::vector<double> x(npx, 128.0), next(npx), dmean(npx), raw(npx);
    std::vector<int64_t> owner(npx, -1);
    std::vector<size_t> src(npx);  // top-left domain pixel read by p
    auto step = [&](const std::vector<double>& cur) {
        std::fill(next.begin(), next.end(), 0.0);
        for (size_t k = 0; k < n; ++k) {
            const orc_leaf& L = leaves[k];
            const uint32_t S = L.size;
            for (uint32_t u = 0; u < S; ++u)
                for (uint32_t v = 0; v < S; ++v) {
                    uint32_t i, j;
                    double value, d = 0.0;
                    size_t q = 0;
                    if (L.mode == 1) {
                        i = u;
                        j = v;
                        const double b0 = (double)L.qbeta / (double)((1u << hdr->bits_beta) - 1) * 255.0;
                        value = std::round(b0 + (double)L.qgx / AFFINE_GRAD_SCALE * (double)u +
                                           (double)L.qgy / AFFINE_GRAD_SCALE * (double)v);
                    } else {
                        iso_map(L.isometry, u, v, S, &i, &j);
                        if (L.qalfa != 0) {
                            q = (L.dom_row + 2 * u) * w + L.dom_col + 2 * v;
                            d = (cur[q] + cur[q + 1] + cur[q + w] + cur[q + w + 1]) / 4.0;
                        }
                        value = s[k] * d + o[k];
                        if (!res[k].empty()) value += res[k][u * S + v];
                    }
                    const size_t pp = (L.row + i) * w + L.col + j;
                    owner[pp] = (int64_t)k;
                    dmean[pp] = d;
                    raw[pp] = value;
                    src[pp] = q;
                    next[pp] = std::min(std::max(value, 0.0), 255.0);
                }
        }
    };
    for (uint32_t it = 0; it < fwd_iters; ++it) {
        step(x);
        x.swap(next);
    }
    step(x);  // the linearisation at x (next = F(x) is discarded)
    double l = 0.0;
    std::vector<double> g(npx), lam(npx, 0.0), acc(npx);
    for (size_t p = 0; p < npx; ++p) {
        const double r = x[p] - (double)target[p];
        g[p] = 2.0 * r;
        l += r * r;
    }
    *loss = l;
    auto live = [&](size_t p) {
        const int64_t k = owner[p];
        return k >= 0 && leaves[k].mode != 1 && raw[p] >= 0.0 && raw[p] <= 255.0;
    };
    for (uint32_t it = 0; it < adj_iters; ++it) {
        std::fill(acc.begin(), acc.end(), 0.0);
        for (size_t p = 0; p < npx; ++p) {
            const int64_t k = owner[p];
            if (!live(p) || leaves[k].qalfa == 0) continue;
            const double c = s[k] * lam[p] / 4.0;
            const size_t q = src[p];
            acc[q] += c;
            acc[q + 1] += c;
            acc[q + w] += c;
            acc[q + w + 1] += c;
        }
        for (size_t p = 0; p < npx; ++p) lam[p] = g[p] + acc[p];
    }
    for (size_t k = 0; k < n; ++k) gs[k] = go[k] = 0.0;
    for (size_t p = 0; p < npx; ++p) {
        if (!live(p)) continue;
        const int64_t k = owner[p];
        gs[k] += leaves[k].qalfa != 0 ? lam[p] * dmean[p] : 0.0;
        go[k] += lam[p];
    }
    if (x_out) std::copy(x.begin(), x.end(), x_out);
    return 0;
}

}  // extern "C"
