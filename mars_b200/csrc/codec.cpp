// Host mirror of the reference partition walks, rate snapshot and .ifs bitstream.
// Every function cites the reference function it restates (paths relative to the
// daleobrien/mars root).  Compiled with -ffp-contract=off: Rust never fuses a*b+c.
#include "codec.hpp"
#include "residual.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>

namespace mars {
namespace codec {

// quantise_f64 (crates/mars-codec/src/encode.rs:446-448).
uint32_t quantise_f64(double x, uint32_t max) {
    double y = std::trunc(0.5 + x);
    if (std::isnan(y)) return 0;
    if (y < 0.0) y = 0.0;
    if (y > (double)max) y = (double)max;
    return (uint32_t)y;
}

// best_beta (encode.rs:456-460).
uint32_t best_beta(int64_t range_sum, int64_t pixel_count, uint32_t bits_beta) {
    const double mean = (double)range_sum / (double)pixel_count;
    const uint32_t max_qbeta = (1u << bits_beta) - 1;
    return quantise_f64(mean / 255.0 * (double)max_qbeta, max_qbeta);
}

void iso_map(uint32_t k, uint32_t u, uint32_t v, uint32_t size, uint32_t* i, uint32_t* j) {
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

// ceil_log2, virtual_size, bits_coord_* (ifs.rs:58-84); zigzag / unzigzag (mars_format.rs:183-189).
uint32_t ceil_log2(uint32_t q) { return q <= 1 ? 0 : 32 - (uint32_t)__builtin_clz(q - 1); }
uint32_t virtual_size(const mars_header& h) { return 1u << ceil_log2(std::max(h.width, h.height)); }
uint32_t bits_coord_row(const mars_header& h) { return ceil_log2(h.height / h.shift); }
uint32_t bits_coord_col(const mars_header& h) { return ceil_log2(h.width / h.shift); }
uint32_t zigzag(int64_t x) { return (uint32_t)((x << 1) ^ (x >> 63)); }
int64_t unzigzag(uint32_t z) { return (int64_t)(z >> 1) ^ -(int64_t)(z & 1); }
static uint32_t size_class_of(uint32_t size) { return (uint32_t)__builtin_ctz(size); }

// build_header (encode.rs:1033-1047).
mars_header build_header(uint32_t w, uint32_t h, const mars_params& p) {
    mars_header hdr;
    hdr.bits_alfa = p.bits_alfa;
    hdr.bits_beta = p.bits_beta;
    hdr.min_size = p.min_size;
    hdr.max_size = p.max_size;
    hdr.shift = p.shift;
    hdr.width = w;
    hdr.height = h;
    hdr.int_max_alfa = quantise_f64(p.max_alfa / 8.0 * 256.0, 255);
    hdr.residual_qstep = 8.0f;
    return hdr;
}

static uint32_t pixel_at(const Image& im, uint32_t row, uint32_t col) {
    return im.px[(size_t)row * im.w + col];
}

// block_rms (encode.rs:386-403).
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

// adaptive_shift (encode.rs:431-437) with DENSITY_LOW_RMS = 4.0 (encode.rs:376).
uint32_t adaptive_shift(uint32_t base, double rms) {
    if (rms <= 4.0) {
        const uint64_t d = (uint64_t)base * 2;
        return d > 0xffffffffull ? 0xffffffffu : (uint32_t)d;
    }
    return base;
}

// emit_leaf (mars_format.rs:515-595); mode 3 appends residual::encode_events.
void emit_leaf(const mars_header& hdr, const mars_leaf& leaf, const int32_t* levels, uint32_t sc,
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
        const int64_t ru = leaf.dom_row / hdr.shift, cu = leaf.dom_col / hdr.shift;
        ev.push_back({{FIELD_DOM_ROW, sc}, (uint32_t)(2 * (1ll << bits_coord_row(hdr))),
                      zigzag(ru - pred.row)});
        ev.push_back({{FIELD_DOM_COL, sc}, (uint32_t)(2 * (1ll << bits_coord_col(hdr))),
                      zigzag(cu - pred.col)});
        pred.row = ru;
        pred.col = cu;
        if (leaf.mode == 3)
            residual::encode_events(levels, (size_t)leaf.size * leaf.size, sc, ev);
    }
}

// walk_write (mars_format.rs:460-512).
bool walk_write(const mars_header& hdr, uint32_t row, uint32_t col, uint32_t size,
                const LeafMap& by_pos, Predictor& pred, std::vector<Event>& ev) {
    if (row >= hdr.height || col >= hdr.width) return true;
    const uint32_t half = size / 2;
    const bool forced = size > hdr.max_size || row + size > hdr.height || col + size > hdr.width;
    const uint32_t sc = size_class_of(size);
    auto it = by_pos.find({row, col, size});
    if (it != by_pos.end()) {
        if (!forced && size > hdr.min_size) ev.push_back({{FIELD_SPLIT, sc}, 2, 0});
        emit_leaf(hdr, *it->second.leaf, it->second.levels, sc, pred, ev);
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

namespace {

// ---------------------------------------------------------------- rate snapshot

// RateModels (crates/mars-codec/src/rate.rs:55-80) over build_models (lib.rs:269-278).
struct RateModels {
    std::map<ContextKey, AdaptiveModel> models;
    bool build(const mars_header& hdr, const std::vector<mars_leaf>& leaves) {
        LeafMap by_pos;
        for (const auto& l : leaves) by_pos[{l.row, l.col, l.size}] = LeafRef{&l, nullptr};
        std::vector<Event> ev;
        Predictor pred;
        if (!walk_write(hdr, 0, 0, virtual_size(hdr), by_pos, pred, ev)) return false;
        for (const auto& e : ev) {
            auto it = models.find(e.ctx);
            if (it == models.end()) it = models.emplace(e.ctx, AdaptiveModel(e.alphabet)).first;
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

// event_bits over leaf_events (encode.rs:1513-1518, mars_format.rs:453-458).
double leaf_bits(const RateModels& rate, const mars_header& hdr, const mars_leaf& leaf,
                 uint32_t sc, const int32_t* levels = nullptr) {
    std::vector<Event> ev;
    Predictor pred;
    emit_leaf(hdr, leaf, levels, sc, pred, ev);
    double s = -0.0;
    for (const auto& e : ev) s += rate.bits_for(e.ctx, e.alphabet, e.symbol);
    return s;
}

// ---------------------------------------------------------------- walks

struct Ctx {
    Image im;
    mars_header hdr;
    mars_params params;
    const Provider* provider;
    const RateModels* rate;
    uint8_t allowed[4];
    bool adaptive_density;
    int status = MARS_OK;
    const RankedProvider* ranked = nullptr;  // search_candidates, when rd_candidates > 1
    uint32_t rd_candidates = 1;
};

mars_leaf make_leaf(uint32_t row, uint32_t col, uint32_t size) {
    mars_leaf l;
    std::memset(&l, 0, sizeof l);
    l.row = row;
    l.col = col;
    l.size = size;
    return l;
}

int64_t range_sum(const Image& im, uint32_t row, uint32_t col, uint32_t size) {
    int64_t s = 0;
    for (uint32_t i = 0; i < size; ++i)
        for (uint32_t j = 0; j < size; ++j) s += pixel_at(im, row + i, col + j);
    return s;
}

struct WalkResult {
    std::vector<mars_leaf> leaves;
    uint64_t evals = 0;
};

WalkResult walk(Ctx& ctx, uint32_t row, uint32_t col, uint32_t size);

// split (encode.rs:1442-1468): TL, BL, TR, BR.
WalkResult split(Ctx& ctx, uint32_t row, uint32_t col, uint32_t half) {
    WalkResult out;
    const uint32_t rs[4] = {row, row + half, row, row + half};
    const uint32_t cs[4] = {col, col, col + half, col + half};
    for (int i = 0; i < 4; ++i) {
        WalkResult q = walk(ctx, rs[i], cs[i], half);
        out.leaves.insert(out.leaves.end(), q.leaves.begin(), q.leaves.end());
        out.evals += q.evals;
    }
    return out;
}

// walk (encode.rs:1330-1435).
WalkResult walk(Ctx& ctx, uint32_t row, uint32_t col, uint32_t size) {
    const mars_header& hdr = ctx.hdr;
    if (ctx.status || row >= hdr.height || col >= hdr.width) return {};
    const bool forced = size > hdr.max_size || row + size > hdr.height || col + size > hdr.width;
    if (forced) return split(ctx, row, col, size / 2);
    if (size == 1) {
        mars_leaf l = make_leaf(row, col, 1);
        l.qbeta = best_beta(pixel_at(ctx.im, row, col), 1, hdr.bits_beta);
        WalkResult r;
        r.leaves.push_back(l);
        return r;
    }
    SearchAnswer ans;
    const int st = (*ctx.provider)(row, col, size, ctx.params.shift, &ans);
    if (st) {
        ctx.status = st;
        return {};
    }
    const double best_rms = ans.cand.valid ? ans.cand.rms : INFINITY;
    if (best_rms > ctx.params.t_rms && size > hdr.min_size) {
        WalkResult r = split(ctx, row, col, size / 2);
        r.evals += ans.evals;
        return r;
    }
    mars_leaf leaf = make_leaf(row, col, size);
    if (ans.cand.valid) {
        leaf.mode = 2;
        leaf.qalfa = ans.cand.qalfa;
        leaf.qbeta = ans.cand.qbeta;
        leaf.isometry = ans.cand.isometry;
        leaf.dom_row = ans.cand.dom_row;
        leaf.dom_col = ans.cand.dom_col;
    }
    if (leaf.qalfa <= ctx.params.zero_threshold) {  // qalfa.abs_diff(0) <= zero_threshold
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
    r.evals = ans.evals;
    return r;
}

// affine_fit (encode.rs:1724-1781).
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
    const double s0 = n, s_u = (double)size * su, s_v = s_u, s_uu = (double)size * suu,
                 s_vv = s_uu, s_uv = su * su;
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
    const double gxq = (double)qgx / AFFINE_GRAD_SCALE, gyq = (double)qgy / AFFINE_GRAD_SCALE;
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

struct Priced {
    mars_leaf leaf;
    double d, r;
    std::vector<int32_t> levels;  // mode 3
};

// residual_for_candidate (encode.rs:1783-1851): the mode-2 prediction's error in
// domain-local (u, v) order, forward DCT, dead-zone quantised and clamped, then priced by
// the SSE of the pixels the decoder will produce.
std::vector<int32_t> residual_for_candidate(const Ctx& ctx, const std::vector<double>& block,
                                            uint32_t size, const mars_candidate& c,
                                            double* sse_out) {
    const mars_header& hdr = ctx.hdr;
    const double alfa = (double)c.qalfa / (double)(1u << ctx.params.bits_alfa) * ctx.params.max_alfa;
    double beta = (double)c.qbeta / (double)((1u << hdr.bits_beta) - 1) *
                  ((1.0 + std::fabs(alfa)) * 255.0);
    if (alfa > 0.0) beta -= alfa * 255.0;
    const size_t n = (size_t)size * size;
    std::vector<double> resid(n), prediction(n);
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
    const std::vector<double> coeffs = residual::forward_dct2d(resid, size);
    const double step = qstep_of(hdr);
    std::vector<int32_t> levels(n);
    std::vector<double> deq(n);
    for (size_t k = 0; k < n; ++k) {
        int32_t l = residual::dead_zone_quantize(coeffs[k], step, residual::kDeadZone);
        if (l < -residual::kLevelClamp) l = -residual::kLevelClamp;
        if (l > residual::kLevelClamp) l = residual::kLevelClamp;
        levels[k] = l;
        deq[k] = residual::dead_zone_dequantize(l, step, residual::kDeadZone);
    }
    const std::vector<double> recon = residual::inverse_dct2d(deq, size);
    double sse = 0.0;
    for (uint32_t u = 0; u < size; ++u)
        for (uint32_t v = 0; v < size; ++v) {
            const size_t k = u * size + v;
            uint32_t i, j;
            iso_map(c.isometry, u, v, size, &i, &j);
            double pv = prediction[k] + recon[k];
            if (pv < 0.0) pv = 0.0;
            if (pv > 255.0) pv = 255.0;
            const double diff = block[i * size + j] - (double)(uint8_t)pv;
            sse += diff * diff;
        }
    *sse_out = sse;
    return levels;
}

// best_mode_leaf (encode.rs:1536-1714), modes 0-3 over the provider's ranked list (the
// single winner unless rd_candidates > 1); candidates with qalfa < 1 are skipped.
Priced best_mode_leaf(const Ctx& ctx, uint32_t row, uint32_t col, uint32_t size,
                      const mars_candidate* ranked, size_t nranked, double lambda, uint32_t sc) {
    const mars_header& hdr = ctx.hdr;
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
        mars_leaf l = make_leaf(row, col, size);
        l.qbeta = best_beta(rsum, s0, hdr.bits_beta);
        const double beta2 = (double)l.qbeta / (double)((1u << hdr.bits_beta) - 1) * 255.0;
        double sse = -0.0;
        for (double p : block) sse += (p - beta2) * (p - beta2);
        cands.push_back({l, sse, leaf_bits(*ctx.rate, hdr, l, sc), {}});
    };
    if (ctx.allowed[0]) mode0();
    if (ctx.allowed[1]) {
        mars_leaf l = make_leaf(row, col, size);
        l.mode = 1;
        double sse;
        affine_fit(block, size, hdr.bits_beta, &l.qbeta, &l.qgx, &l.qgy, &sse);
        cands.push_back({l, sse, leaf_bits(*ctx.rate, hdr, l, sc), {}});
    }
    for (size_t ci = 0; ci < nranked; ++ci) {
        const mars_candidate& c = ranked[ci];
        if (!c.valid || c.qalfa < 1) continue;
        if (ctx.allowed[2]) {
            mars_leaf l = make_leaf(row, col, size);
            l.mode = 2;
            l.qalfa = c.qalfa;
            l.qbeta = c.qbeta;
            l.isometry = c.isometry;
            l.dom_row = c.dom_row;
            l.dom_col = c.dom_col;
            const double sse2 = c.rms * c.rms * (double)size * (double)size;
            cands.push_back({l, sse2, leaf_bits(*ctx.rate, hdr, l, sc), {}});
        }
        if (!ctx.allowed[3]) continue;
        mars_leaf l = make_leaf(row, col, size);
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
    if (cands.empty()) mode0();
    size_t best = 0;
    for (size_t i = 1; i < cands.size(); ++i) {
        const double jb = cands[best].d + lambda * cands[best].r;
        const double ji = cands[i].d + lambda * cands[i].r;
        if (ji < jb) best = i;
    }
    return std::move(cands[best]);
}

struct RdResult {
    std::vector<mars_leaf> leaves;
    std::vector<int32_t> resid;  // levels of the mode-3 leaves, in leaf order
    uint64_t evals = 0;
    double d = 0.0, r = 0.0;
};

RdResult walk_rd(Ctx& ctx, uint32_t row, uint32_t col, uint32_t size, double lambda);

// split_rd (encode.rs:2033-2071).
RdResult split_rd(Ctx& ctx, uint32_t row, uint32_t col, uint32_t half, double lambda) {
    RdResult out;
    const uint32_t rs[4] = {row, row + half, row, row + half};
    const uint32_t cs[4] = {col, col, col + half, col + half};
    for (int i = 0; i < 4; ++i) {
        RdResult q = walk_rd(ctx, rs[i], cs[i], half, lambda);
        out.leaves.insert(out.leaves.end(), q.leaves.begin(), q.leaves.end());
        out.resid.insert(out.resid.end(), q.resid.begin(), q.resid.end());
        out.evals += q.evals;
        out.d += q.d;
        out.r += q.r;
    }
    return out;
}

// walk_rd (encode.rs:1865-2027) without lambda regions.
RdResult walk_rd(Ctx& ctx, uint32_t row, uint32_t col, uint32_t size, double lambda) {
    const mars_header& hdr = ctx.hdr;
    if (ctx.status || row >= hdr.height || col >= hdr.width) return {};
    const bool forced = size > hdr.max_size || row + size > hdr.height || col + size > hdr.width;
    if (forced) return split_rd(ctx, row, col, size / 2, lambda);
    const RateModels& rate = *ctx.rate;
    const uint32_t sc = size_class_of(size);
    if (size == 1) {
        const uint32_t pixel = pixel_at(ctx.im, row, col);
        mars_leaf l = make_leaf(row, col, 1);
        l.qbeta = best_beta(pixel, 1, hdr.bits_beta);
        double dv = 0.5 + (double)l.qbeta / (double)((1u << hdr.bits_beta) - 1) * 255.0;
        if (dv < 0.0) dv = 0.0;
        if (dv > 255.0) dv = 255.0;
        const double diff = (double)pixel - (double)(uint8_t)dv;
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
    // rd_candidates == 1 keeps the single-winner search(); above 1 the ranked list widens
    // modes 2/3's competition (encode.rs:1946-1977).
    SearchAnswer ans;
    std::vector<mars_candidate> ranked;
    int st;
    if (ctx.rd_candidates > 1 && ctx.ranked) {
        st = (*ctx.ranked)(row, col, size, shift, ctx.rd_candidates, &ranked, &ans.evals);
    } else {
        st = (*ctx.provider)(row, col, size, shift, &ans);
        if (!st && ans.cand.valid) ranked.push_back(ans.cand);
    }
    if (st) {
        ctx.status = st;
        return {};
    }
    Priced leaf = best_mode_leaf(ctx, row, col, size, ranked.data(), ranked.size(), node_lambda, sc);
    if (size <= hdr.min_size) {
        RdResult r;
        r.leaves.push_back(leaf.leaf);
        r.resid = std::move(leaf.levels);
        r.evals = ans.evals;
        r.d = leaf.d;
        r.r = leaf.r;
        return r;
    }
    RdResult children = split_rd(ctx, row, col, size / 2, lambda);
    const uint64_t total = ans.evals + children.evals;
    const double split0 = rate.bits_for({FIELD_SPLIT, sc}, 2, 0);
    const double split1 = rate.bits_for({FIELD_SPLIT, sc}, 2, 1);
    const double leaf_j = leaf.d + node_lambda * (leaf.r + split0);
    const double split_j = children.d + node_lambda * (children.r + split1);
    if (leaf_j <= split_j) {
        RdResult r;
        r.leaves.push_back(leaf.leaf);
        r.resid = std::move(leaf.levels);
        r.evals = total;
        r.d = leaf.d;
        r.r = leaf.r + split0;
        return r;
    }
    children.evals = total;
    children.r = children.r + split1;
    return children;
}

// ---------------------------------------------------------------- .ifs bits

struct BitReader {
    const uint8_t* data;
    size_t len, pos = 0;
    bool read(uint32_t n, uint32_t* v) {
        uint32_t x = 0;
        for (uint32_t i = 0; i < n; ++i) {
            if ((pos >> 3) >= len) return false;
            x |= (uint32_t)((data[pos >> 3] >> (7 - (pos & 7))) & 1) << i;
            ++pos;
        }
        *v = x;
        return true;
    }
};

int ifs_walk(BitReader& r, const mars_header& hdr, uint32_t row, uint32_t col, uint32_t size,
             std::vector<mars_leaf>& leaves) {
    if (row >= hdr.height || col >= hdr.width) return MARS_OK;
    const bool forced = size > hdr.max_size || row + size > hdr.height || col + size > hdr.width;
    uint32_t flag = 0;
    if (!forced && size > hdr.min_size && !r.read(1, &flag)) return MARS_EFORMAT;
    if (forced || flag == 1) {
        const uint32_t half = size / 2;
        int e;
        if ((e = ifs_walk(r, hdr, row, col, half, leaves))) return e;
        if ((e = ifs_walk(r, hdr, row + half, col, half, leaves))) return e;
        if ((e = ifs_walk(r, hdr, row, col + half, half, leaves))) return e;
        return ifs_walk(r, hdr, row + half, col + half, half, leaves);
    }
    mars_leaf l = make_leaf(row, col, size);
    if (!r.read(hdr.bits_alfa, &l.qalfa) || !r.read(hdr.bits_beta, &l.qbeta)) return MARS_EFORMAT;
    if (l.qalfa != 0) {
        uint32_t iso, dr, dc;
        if (!r.read(3, &iso) || !r.read(bits_coord_row(hdr), &dr) ||
            !r.read(bits_coord_col(hdr), &dc))
            return MARS_EFORMAT;
        l.isometry = iso;
        l.dom_row = hdr.shift * dr;
        l.dom_col = hdr.shift * dc;
        if (l.dom_row + 2 * size > hdr.height || l.dom_col + 2 * size > hdr.width)
            return MARS_EFORMAT;
        l.mode = 2;
    }
    leaves.push_back(l);
    return MARS_OK;
}

struct BitWriter {
    std::vector<uint8_t> bits;
    void write(uint32_t n, uint32_t v) {
        for (uint32_t i = 0; i < n; ++i) bits.push_back((v >> i) & 1);
    }
};

bool ifs_write_walk(BitWriter& w, const mars_header& hdr, uint32_t row, uint32_t col,
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
    const mars_leaf& l = *it->second.leaf;
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

double qstep_of(const mars_header& h) {
    return h.residual_qstep == 0.0f ? 8.0 : (double)h.residual_qstep;
}

bool qstep_new(double step, float* out) {
    if (!(std::isfinite(step) && step >= 1.0 && step <= 65535.0)) return false;
    *out = (float)step;
    return true;
}

float qstep_from_lambda(double lambda) {
    double step = std::sqrt(std::max(lambda, 0.0)) * std::sqrt(6.0 / 0.693147180559945309417232121458176568);
    if (!(step >= 1.0)) step = 1.0;  // NaN and below-range map to MIN
    if (step > 65535.0) step = 65535.0;
    return (float)step;
}

bool residual_offsets(const mars_leaf* leaves, size_t n, size_t npool, std::vector<int64_t>* offs) {
    offs->assign(n, -1);
    size_t at = 0;
    for (size_t k = 0; k < n; ++k)
        if (leaves[k].mode == 3) {
            const size_t need = (size_t)leaves[k].size * leaves[k].size;
            if (need > npool - at) return false;
            (*offs)[k] = (int64_t)at;
            at += need;
        }
    return at == npool;
}

// ------------------------------------------------------------- host parallelism
//
// Below the forced splits every node's subtree is independent of the others (the walks read
// the plane, the provider and the frozen rate snapshot only), which is what lets the
// reference run them as Rayon tasks (encode.rs:1442-1468, 2033-2071).  Here the roots of
// those subtrees are collected in the order the sequential walk visits them, walked on a
// pool of host threads, and their results concatenated in that order, so the leaf list,
// the residual pool and the eval counts are the sequential walk's exactly.

struct Root {
    uint32_t row, col, size;
};

// The nodes the forced splits reach (split order TL, BL, TR, BR), skipping those outside.
void collect_roots(const mars_header& hdr, uint32_t row, uint32_t col, uint32_t size,
                   std::vector<Root>* out) {
    if (row >= hdr.height || col >= hdr.width) return;
    const bool forced = size > hdr.max_size || row + size > hdr.height || col + size > hdr.width;
    if (!forced) {
        out->push_back({row, col, size});
        return;
    }
    const uint32_t half = size / 2;
    collect_roots(hdr, row, col, half, out);
    collect_roots(hdr, row + half, col, half, out);
    collect_roots(hdr, row, col + half, half, out);
    collect_roots(hdr, row + half, col + half, half, out);
}

// Host threads for the walks: MARS_HOST_THREADS when set (>= 1), else every core.
unsigned host_threads() {
    if (const char* e = std::getenv("MARS_HOST_THREADS")) {
        const long v = std::strtol(e, nullptr, 10);
        if (v >= 1) return (unsigned)std::min<long>(v, 1024);
    }
    const unsigned hc = std::thread::hardware_concurrency();
    return hc ? hc : 1;
}

// Runs fn(i) for i in [0, n) on up to host_threads() threads (dynamic assignment).
template <class F>
void parallel_for(size_t n, F&& fn) {
    const unsigned nt = (unsigned)std::min<size_t>(host_threads(), n);
    if (nt <= 1) {
        for (size_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<size_t> next{0};
    auto worker = [&] {
        for (size_t i; (i = next.fetch_add(1)) < n;) fn(i);
    };
    std::vector<std::thread> pool;
    pool.reserve(nt - 1);
    for (unsigned t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
}

// walk / walk_rd over the whole plane, root subtrees in parallel; the first failing root's
// status (in walk order) is returned.
int walk_all(const Ctx& base, WalkResult* out) {
    std::vector<Root> roots;
    collect_roots(base.hdr, 0, 0, virtual_size(base.hdr), &roots);
    std::vector<WalkResult> res(roots.size());
    std::vector<int> status(roots.size(), MARS_OK);
    parallel_for(roots.size(), [&](size_t i) {
        Ctx ctx = base;
        res[i] = walk(ctx, roots[i].row, roots[i].col, roots[i].size);
        status[i] = ctx.status;
    });
    for (size_t i = 0; i < roots.size(); ++i) {
        if (status[i]) return status[i];
        out->leaves.insert(out->leaves.end(), res[i].leaves.begin(), res[i].leaves.end());
        out->evals += res[i].evals;
    }
    return MARS_OK;
}

int walk_rd_all(const Ctx& base, double lambda, RdResult* out) {
    std::vector<Root> roots;
    collect_roots(base.hdr, 0, 0, virtual_size(base.hdr), &roots);
    std::vector<RdResult> res(roots.size());
    std::vector<int> status(roots.size(), MARS_OK);
    parallel_for(roots.size(), [&](size_t i) {
        Ctx ctx = base;
        res[i] = walk_rd(ctx, roots[i].row, roots[i].col, roots[i].size, lambda);
        status[i] = ctx.status;
    });
    for (size_t i = 0; i < roots.size(); ++i) {
        if (status[i]) return status[i];
        out->leaves.insert(out->leaves.end(), res[i].leaves.begin(), res[i].leaves.end());
        out->resid.insert(out->resid.end(), res[i].resid.begin(), res[i].resid.end());
        out->evals += res[i].evals;
    }
    return MARS_OK;
}

int encode(const Image& im, const mars_params& p, const mars_options& o, const Provider& provider,
           const Provider& warmup, mars_header* hdr_out, std::vector<mars_leaf>* leaves,
           std::vector<int32_t>* residuals, mars_counters* counters,
           const RankedProvider* ranked) {
    mars_header hdr = build_header(im.w, im.h, p);
    // encode.rs:1066-1071: LambdaAdaptive -> from_lambda (8 without lambda); Fixed(step).
    if (o.residual_adaptive)
        hdr.residual_qstep = p.has_lambda ? qstep_from_lambda(p.lambda) : 8.0f;
    else if (o.residual_qstep == 0.0f)
        hdr.residual_qstep = 8.0f;
    else if (!qstep_new((double)o.residual_qstep, &hdr.residual_qstep))
        return MARS_EINVAL;
    residuals->clear();
    if (p.has_lambda) {
        // build_rate_snapshot (encode.rs:1139-1169): the t_rms = 8 threshold walk with the
        // exhaustive search, here answered by the same provider (it is exhaustive too).
        Ctx warm{im, hdr, p, &warmup, nullptr, {1, 1, 1, 1}, false};
        warm.params.t_rms = 8.0;
        warm.params.has_lambda = 0;
        WalkResult wr;
        if (int st = walk_all(warm, &wr)) return st;
        RateModels rate;
        if (!rate.build(hdr, wr.leaves)) return MARS_EINVAL;
        Ctx ctx{im, hdr, p, &provider, &rate,
                {o.allowed_modes[0], o.allowed_modes[1], o.allowed_modes[2], o.allowed_modes[3]},
                o.adaptive_density != 0};
        ctx.ranked = ranked;
        ctx.rd_candidates = std::max<uint32_t>(1, o.rd_candidates);
        RdResult rr;
        if (int st = walk_rd_all(ctx, p.lambda, &rr)) return st;
        *leaves = std::move(rr.leaves);
        *residuals = std::move(rr.resid);
        counters->search_evals = rr.evals;
        counters->warmup_evals = wr.evals;
    } else {
        Ctx ctx{im, hdr, p, &provider, nullptr, {1, 1, 1, 1}, false};
        WalkResult wr;
        if (int st = walk_all(ctx, &wr)) return st;
        *leaves = std::move(wr.leaves);
        counters->search_evals = wr.evals;
        counters->warmup_evals = 0;
    }
    *hdr_out = hdr;
    return MARS_OK;
}

int ifs_parse(const uint8_t* data, size_t len, mars_header* hdr, std::vector<mars_leaf>* leaves) {
    BitReader r{data, len};
    mars_header h{};
    h.residual_qstep = 8.0f;
    if (!r.read(4, &h.bits_alfa) || !r.read(4, &h.bits_beta) || !r.read(7, &h.min_size) ||
        !r.read(7, &h.max_size) || !r.read(6, &h.shift) || !r.read(12, &h.width) ||
        !r.read(12, &h.height) || !r.read(8, &h.int_max_alfa))
        return MARS_EFORMAT;
    if (h.width == 0 || h.height == 0 || h.shift == 0) return MARS_EFORMAT;
    leaves->clear();
    const int e = ifs_walk(r, h, 0, 0, virtual_size(h), *leaves);
    if (e) return e;
    const size_t left = len * 8 - r.pos;
    if (left >= 8) return MARS_EFORMAT;
    if (left > 0 && (data[len - 1] & ((1u << left) - 1)) != 0) return MARS_EFORMAT;
    *hdr = h;
    return MARS_OK;
}

int ifs_write(const mars_header& hdr, const std::vector<mars_leaf>& leaves,
              std::vector<uint8_t>* out) {
    LeafMap by_pos;
    for (const auto& l : leaves)
        if (!by_pos.emplace(std::make_tuple(l.row, l.col, l.size), LeafRef{&l, nullptr}).second)
            return MARS_EINVAL;
    BitWriter w;
    w.write(4, hdr.bits_alfa);
    w.write(4, hdr.bits_beta);
    w.write(7, hdr.min_size);
    w.write(7, hdr.max_size);
    w.write(6, hdr.shift);
    w.write(12, hdr.width);
    w.write(12, hdr.height);
    w.write(8, hdr.int_max_alfa);
    if (!ifs_write_walk(w, hdr, 0, 0, virtual_size(hdr), by_pos)) return MARS_EINVAL;
    out->assign((w.bits.size() + 7) / 8, 0);
    for (size_t i = 0; i < w.bits.size(); ++i)
        if (w.bits[i]) (*out)[i / 8] |= (uint8_t)(1u << (7 - (i % 8)));
    return MARS_OK;
}

}  // namespace codec
}  // namespace mars
