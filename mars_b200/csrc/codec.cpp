// Host mirror of the reference partition walks, rate snapshot and .ifs bitstream.
// Every function cites the reference function it restates (paths relative to the
// daleobrien/mars root).  Compiled with -ffp-contract=off: Rust never fuses a*b+c.
#include "codec.hpp"
#include "residual.hpp"

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <functional>
#include <mutex>
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
    const struct HostRates* table = nullptr;     // the snapshot as a bits table
    const struct PricedNodes* priced = nullptr;  // the nodes priced in one batch, if any
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

// The pricing of one node runs price::price_node (price.hpp), the code the device pricing
// kernel runs too.  HostRates holds the frozen snapshot as its bits table.
struct HostRates {
    std::vector<double> bits;
    std::vector<int64_t> offset;
    price::RateTable view() const { return {bits.data(), offset.data()}; }
};

// Every (field, context) best_mode_leaf can price for nodes up to max_size: the snapshot's
// model where it has one, else a fresh model of the field's alphabet (RateModels::bits_for).
HostRates build_rate_table(const RateModels& rate, const mars_header& hdr, uint32_t max_size) {
    HostRates t;
    t.offset.assign((size_t)price::kFields * price::kCtx, -1);
    const uint32_t sc_max = std::min<uint32_t>(size_class_of(std::max<uint32_t>(max_size, 1)),
                                               price::kSizeClasses - 1);
    auto alphabet_of = [&](uint32_t field) -> uint32_t {
        switch (field) {
            case price::F_SPLIT: return 2;
            case price::F_MODE: return MODE_ALPHABET;
            case price::F_QALFA: return (1u << hdr.bits_alfa) - 1;
            case price::F_QBETA:
            case price::F_QBETA_DC: return 1u << hdr.bits_beta;
            case price::F_ISOMETRY: return 8;
            case price::F_DOM_ROW: return (uint32_t)(2 * (1ll << bits_coord_row(hdr)));
            case price::F_DOM_COL: return (uint32_t)(2 * (1ll << bits_coord_col(hdr)));
            case price::F_GX:
            case price::F_GY: return (uint32_t)(2 * (int64_t)AFFINE_GRAD_CLAMP + 1);
            case price::F_RESID_NZ: return 2;
            default: return (uint32_t)(2 * price::kLevelClamp + 1);
        }
    };
    std::map<uint32_t, int64_t> fresh;  // alphabet -> where its fresh model's bits start
    auto add = [&](uint32_t field, uint32_t ctx) {
        int64_t& at = t.offset[(size_t)field * price::kCtx + ctx];
        auto it = rate.models.find({(uint8_t)field, ctx});
        if (it != rate.models.end()) {
            at = (int64_t)t.bits.size();
            t.bits.resize(t.bits.size() + it->second.counts.size());
            it->second.all_bits(t.bits.data() + at);
            return;
        }
        // Contexts without a model share one table per alphabet.
        const uint32_t a = std::max<uint32_t>(alphabet_of(field), 2);
        auto f = fresh.find(a);
        if (f == fresh.end()) {
            f = fresh.emplace(a, (int64_t)t.bits.size()).first;
            t.bits.resize(t.bits.size() + a);
            AdaptiveModel(a).all_bits(t.bits.data() + f->second);
        }
        at = f->second;
    };
    for (uint32_t sc = 0; sc <= sc_max; ++sc) {
        for (uint32_t field = 0; field < price::F_RESID_NZ; ++field) add(field, sc);
        for (uint32_t band = 0; band < price::kBands; ++band) {
            add(price::F_RESID_NZ, sc * price::kBands + band);
            add(price::F_RESID_MAG, sc * price::kBands + band);
        }
    }
    return t;
}

price::Setup make_setup(const mars_header& hdr, const mars_params& p, const uint8_t allowed[4],
                        double lambda) {
    price::Setup s;
    s.bits_alfa = p.bits_alfa;
    s.max_alfa = p.max_alfa;
    s.bits_beta = hdr.bits_beta;
    s.shift = hdr.shift;
    s.qstep = qstep_of(hdr);
    s.lambda = lambda;
    for (int m = 0; m < 4; ++m) s.allowed[m] = allowed[m];
    return s;
}

struct Priced {
    mars_leaf leaf;
    double d, r;
    std::vector<int32_t> levels;  // mode 3
};

// The transposed basis (bt[i * n + k] = basis(n, k, i)) the forward transform's row pass
// reads; cached per thread.
const double* basis_t(uint32_t n) {
    thread_local std::map<uint32_t, std::vector<double>> cache;
    auto it = cache.find(n);
    if (it == cache.end()) {
        const std::vector<double>& b = residual::basis(n);
        std::vector<double> t((size_t)n * n);
        for (uint32_t k = 0; k < n; ++k)
            for (uint32_t i = 0; i < n; ++i) t[(size_t)i * n + k] = b[(size_t)k * n + i];
        it = cache.emplace(n, std::move(t)).first;
    }
    return it->second.data();
}

price::Cand to_cand(const mars_candidate& c) {
    return {c.dom_row, c.dom_col, c.isometry, c.qalfa, c.qbeta, c.valid, c.rms};
}

// best_mode_leaf (encode.rs:1536-1714) on the host: price::price_node as a team of one
// lane with thread-local scratch.
Priced best_mode_leaf(const Ctx& ctx, uint32_t row, uint32_t col, uint32_t size,
                      const mars_candidate* ranked, size_t nranked, double lambda, uint32_t sc) {
    thread_local std::vector<double> dscr;
    thread_local std::vector<int32_t> iscr;
    const size_t n = (size_t)size * size;
    if (dscr.size() < 5 * n) dscr.resize(5 * n);
    if (iscr.size() < 2 * n) iscr.resize(2 * n);
    price::Scratch s{dscr.data(), dscr.data() + n, dscr.data() + 2 * n, dscr.data() + 3 * n,
                     dscr.data() + 4 * n, iscr.data(), iscr.data() + n};
    thread_local std::vector<price::Cand> cands;
    cands.resize(nranked);
    for (size_t i = 0; i < nranked; ++i) cands[i] = to_cand(ranked[i]);
    const price::Setup setup = make_setup(ctx.hdr, ctx.params, ctx.allowed, lambda);
    const price::RateTable view = ctx.table->view();
    const price::Priced p =
        price::price_node(ctx.im.px, ctx.im.w, row, col, size, cands.data(), (uint32_t)nranked,
                          setup, view, residual::basis(size).data(), basis_t(size), sc, s, {0, 1});
    Priced out{p.leaf, p.d, p.r, {}};
    if (p.has_levels) out.levels.assign(s.best_levels, s.best_levels + n);
    return out;
}

// A pricer's answers for the RD walk: node (row, col, size) -> its entry in the batch,
// through one dense grid per node size.
struct PricedNodes {
    const PriceBatch* batch = nullptr;
    std::vector<uint32_t> sizes, cols;
    std::vector<size_t> base;
    std::vector<int64_t> at;  // grid cell -> batch index, -1 when absent
    void build(const PriceBatch& b) {
        batch = &b;
        size_t total = 0;
        for (uint32_t s : b.sizes) {
            const uint32_t c = (b.im.w + s - 1) / s, r = (b.im.h + s - 1) / s;
            sizes.push_back(s);
            cols.push_back(c);
            base.push_back(total);
            total += (size_t)c * r;
        }
        at.assign(total, -1);
        for (size_t g = 0; g < b.sizes.size(); ++g)
            for (uint32_t i = b.first[g]; i < b.first[g + 1]; ++i)
                at[base[g] + (size_t)(b.row[i] / sizes[g]) * cols[g] + b.col[i] / sizes[g]] = i;
    }
    bool get(uint32_t row, uint32_t col, uint32_t size, Priced* out, uint64_t* evals) const {
        for (size_t g = 0; g < sizes.size(); ++g) {
            if (sizes[g] != size) continue;
            const int64_t i = at[base[g] + (size_t)(row / size) * cols[g] + col / size];
            if (i < 0 || batch->row[i] != row || batch->col[i] != col) return false;
            const price::Priced& p = batch->priced[i];
            *evals = batch->evals[i];
            out->leaf = p.leaf;
            out->d = p.d;
            out->r = p.r;
            out->levels.clear();
            if (p.has_levels) {
                const int8_t* l = batch->levels.data() + batch->levels_at[i];
                out->levels.assign(l, l + (size_t)size * size);
            }
            return true;
        }
        return false;
    }
};

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
    SearchAnswer ans;
    Priced leaf;
    if (ctx.priced) {
        // Priced in one batch beforehand, with the provider's answer for this node.
        if (!ctx.priced->get(row, col, size, &leaf, &ans.evals)) {
            ctx.status = MARS_ENOTFOUND;
            return {};
        }
    } else {
        const uint32_t shift =
            ctx.adaptive_density ? adaptive_shift(ctx.params.shift, block_rms(ctx.im, row, col, size))
                                 : ctx.params.shift;
        // rd_candidates == 1 keeps the single-winner search(); above 1 the ranked list widens
        // modes 2/3's competition (encode.rs:1946-1977).
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
        leaf = best_mode_leaf(ctx, row, col, size, ranked.data(), ranked.size(), node_lambda, sc);
    }
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
// A process-wide pool of host workers that parallel_for calls share (threads are started
// once, not per walk).  The calling thread works on its own call's items too, so every call
// finishes even while all workers serve other calls; a call takes at most `max_helpers`
// workers.
class HostPool {
public:
    static HostPool& get() {
        static HostPool* pool = new HostPool();  // never destroyed: workers outlive main()
        return *pool;
    }
    void run(size_t n, unsigned max_helpers, const std::function<void(size_t)>& fn) {
        Job job{&fn, n, max_helpers};
        {
            std::lock_guard<std::mutex> lk(mu_);
            jobs_.push_back(&job);
        }
        cv_.notify_all();
        work(job);
        std::unique_lock<std::mutex> lk(mu_);
        auto it = std::find(jobs_.begin(), jobs_.end(), &job);
        if (it != jobs_.end()) jobs_.erase(it);
        done_.wait(lk, [&] { return job.helpers == 0; });
    }

private:
    struct Job {
        const std::function<void(size_t)>* fn;
        size_t n;
        unsigned max_helpers;
        std::atomic<size_t> next{0};
        unsigned helpers = 0;  // guarded by mu_
    };
    static void work(Job& j) {
        for (size_t i; (i = j.next.fetch_add(1)) < j.n;) (*j.fn)(i);
    }
    HostPool() {
        const unsigned hc = std::max(1u, std::thread::hardware_concurrency());
        for (unsigned t = 1; t < hc; ++t) std::thread([this] { loop(); }).detach();
    }
    // The first queued job with items left and room for a helper; exhausted jobs leave the
    // queue (their callers wait for the helpers still on them).
    Job* eligible() {
        while (!jobs_.empty() && jobs_.front()->next.load() >= jobs_.front()->n) jobs_.pop_front();
        for (Job* j : jobs_)
            if (j->next.load() < j->n && j->helpers < j->max_helpers) return j;
        return nullptr;
    }
    void loop() {
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
            Job* j;
            cv_.wait(lk, [&] { return (j = eligible()) != nullptr; });
            ++j->helpers;
            lk.unlock();
            work(*j);
            lk.lock();
            if (--j->helpers == 0) done_.notify_all();
        }
    }
    std::mutex mu_;
    std::condition_variable cv_, done_;
    std::deque<Job*> jobs_;
};

template <class F>
void parallel_for(size_t n, F&& fn) {
    const unsigned nt = (unsigned)std::min<size_t>(host_threads(), n);
    if (nt <= 1) {
        for (size_t i = 0; i < n; ++i) fn(i);
        return;
    }
    const std::function<void(size_t)> f = [&fn](size_t i) { fn(i); };
    HostPool::get().run(n, nt - 1, f);
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

// The nodes walk_rd prices (every in-plane, unforced node of more than one pixel down to
// min_size) below one root, with the candidates walk_rd asks its provider for.
struct NodeList {
    std::vector<uint32_t> row, col, size;
    std::vector<price::Cand> cands;  // k per node
    std::vector<uint64_t> evals;
};
void collect_priced(Ctx& ctx, uint32_t row, uint32_t col, uint32_t size, uint32_t k,
                    NodeList& out) {
    const mars_header& hdr = ctx.hdr;
    if (ctx.status || row >= hdr.height || col >= hdr.width || size < 2) return;
    const bool forced = size > hdr.max_size || row + size > hdr.height || col + size > hdr.width;
    if (!forced) {
        const uint32_t shift = ctx.adaptive_density
                                   ? adaptive_shift(ctx.params.shift, block_rms(ctx.im, row, col, size))
                                   : ctx.params.shift;
        thread_local std::vector<mars_candidate> ranked;
        ranked.clear();
        uint64_t evals = 0;
        int st;
        if (ctx.rd_candidates > 1 && ctx.ranked) {
            st = (*ctx.ranked)(row, col, size, shift, ctx.rd_candidates, &ranked, &evals);
        } else {
            SearchAnswer ans;
            st = (*ctx.provider)(row, col, size, shift, &ans);
            if (!st && ans.cand.valid) ranked.push_back(ans.cand);
            evals = ans.evals;
        }
        if (st) {
            ctx.status = st;
            return;
        }
        const price::Cand none{0, 0, 0, 0, 0, 0, 0.0};
        for (uint32_t i = 0; i < k; ++i)
            out.cands.push_back(i < ranked.size() ? to_cand(ranked[i]) : none);
        out.row.push_back(row);
        out.col.push_back(col);
        out.size.push_back(size);
        out.evals.push_back(evals);
        if (size <= hdr.min_size) return;
    }
    const uint32_t half = size / 2;
    collect_priced(ctx, row, col, half, k, out);
    collect_priced(ctx, row + half, col, half, k, out);
    collect_priced(ctx, row, col + half, half, k, out);
    collect_priced(ctx, row + half, col + half, half, k, out);
}

// Fills a PriceBatch with every node of the RD walk (grouped by size, largest first; roots
// in walk order within a group) and runs the pricer on it.
int price_all(const Ctx& base, double lambda, const Pricer& pricer, PriceBatch* batch) {
    const uint32_t k = base.rd_candidates > 1 && base.ranked ? base.rd_candidates : 1;
    std::vector<Root> roots;
    collect_roots(base.hdr, 0, 0, virtual_size(base.hdr), &roots);
    std::vector<NodeList> lists(roots.size());
    std::vector<int> status(roots.size(), MARS_OK);
    parallel_for(roots.size(), [&](size_t i) {
        Ctx ctx = base;
        collect_priced(ctx, roots[i].row, roots[i].col, roots[i].size, k, lists[i]);
        status[i] = ctx.status;
    });
    for (int st : status)
        if (st) return st;
    PriceBatch& b = *batch;
    b.im = base.im;
    b.setup = make_setup(base.hdr, base.params, base.allowed, lambda * 1.0);
    b.bits = base.table->bits.data();
    b.nbits = base.table->bits.size();
    b.offset = base.table->offset.data();
    b.k = k;
    for (uint32_t size = virtual_size(base.hdr); size >= 2; size /= 2) {
        const uint32_t start = (uint32_t)b.row.size();
        for (const NodeList& l : lists)
            for (size_t i = 0; i < l.row.size(); ++i) {
                if (l.size[i] != size) continue;
                b.row.push_back(l.row[i]);
                b.col.push_back(l.col[i]);
                b.cands.insert(b.cands.end(), l.cands.begin() + i * k, l.cands.begin() + (i + 1) * k);
                b.evals.push_back(l.evals[i]);
                b.levels_at.push_back(b.nlevels);
                b.nlevels += (uint64_t)size * size;
            }
        if (b.row.size() == start) continue;
        b.sizes.push_back(size);
        b.first.push_back(start);
        b.basis.push_back(residual::basis(size).data());
    }
    b.first.push_back((uint32_t)b.row.size());
    if (b.row.empty()) return MARS_OK;
    return pricer(b);
}

int encode_header(uint32_t w, uint32_t h, const mars_params& p, const mars_options& o,
                  mars_header* out) {
    mars_header hdr = build_header(w, h, p);
    // encode.rs:1066-1071: LambdaAdaptive -> from_lambda (8 without lambda); Fixed(step).
    if (o.residual_adaptive)
        hdr.residual_qstep = p.has_lambda ? qstep_from_lambda(p.lambda) : 8.0f;
    else if (o.residual_qstep == 0.0f)
        hdr.residual_qstep = 8.0f;
    else if (!qstep_new((double)o.residual_qstep, &hdr.residual_qstep))
        return MARS_EINVAL;
    *out = hdr;
    return MARS_OK;
}

int rate_table_from_warmup(const mars_header& hdr, const std::vector<mars_leaf>& warm,
                           uint32_t max_size, std::vector<double>* bits,
                           std::vector<int64_t>* offset) {
    RateModels rate;
    if (!rate.build(hdr, warm)) return MARS_EINVAL;
    HostRates t = build_rate_table(rate, hdr, max_size);
    *bits = std::move(t.bits);
    *offset = std::move(t.offset);
    return MARS_OK;
}

price::Setup price_setup(const mars_header& hdr, const mars_params& p, const uint8_t allowed[4],
                         double lambda) {
    return make_setup(hdr, p, allowed, lambda * 1.0);
}

std::vector<std::array<uint32_t, 3>> quadtree_roots(const mars_header& hdr) {
    std::vector<Root> roots;
    collect_roots(hdr, 0, 0, virtual_size(hdr), &roots);
    std::vector<std::array<uint32_t, 3>> out;
    out.reserve(roots.size());
    for (const Root& r : roots) out.push_back({r.row, r.col, r.size});
    return out;
}

int encode(const Image& im, const mars_params& p, const mars_options& o, const Provider& provider,
           const Provider& warmup, mars_header* hdr_out, std::vector<mars_leaf>* leaves,
           std::vector<int32_t>* residuals, mars_counters* counters,
           const RankedProvider* ranked, const Pricer* pricer) {
    mars_header hdr;
    if (int st = encode_header(im.w, im.h, p, o, &hdr)) return st;
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
        const HostRates rates = build_rate_table(rate, hdr, p.max_size);
        ctx.table = &rates;
        PriceBatch batch;
        PricedNodes priced;
        if (pricer) {
            if (int st = price_all(ctx, p.lambda, *pricer, &batch)) return st;
            priced.build(batch);
            ctx.priced = &priced;
        }
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
