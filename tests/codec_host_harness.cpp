// Test harness, built by tests/test_codec_host_cpu.py (not part of the library): the
// library's host codec -- mars_b200/csrc/codec.cpp's walks, rate snapshot, node pricing
// (price.hpp run as a team of one lane) and host thread pool -- with the oracle's search as
// its provider, so whole RD encodes can be compared with the oracle on a machine without a
// GPU.  With batch_pricing set, every node is priced up front through the Pricer interface
// (price_all / PricedNodes, the path the device pricer takes), here on the host.
#include <cstring>
#include <string>
#include <vector>

#include "../mars_b200/csrc/codec.hpp"
#include "../mars_b200/csrc/residual.hpp"
#include "../oracle/oracle.h"

static_assert(sizeof(orc_candidate) == sizeof(mars_candidate), "candidate layout");
static_assert(sizeof(orc_params) == sizeof(mars_params), "params layout");
static_assert(sizeof(orc_leaf) == sizeof(mars_leaf), "leaf layout");

namespace mars {
int set_last_error(int code, const std::string&) { return code; }
}  // namespace mars

using namespace mars;

namespace {

int price_on_host(codec::PriceBatch& b) {
    const size_t nodes = b.row.size();
    b.priced.resize(nodes);
    if (b.setup.allowed[3]) b.levels.assign(b.nlevels, 0);
    for (size_t g = 0; g < b.sizes.size(); ++g) {
        const uint32_t size = b.sizes[g], n = size * size;
        std::vector<double> bt(n), d(5 * n);
        std::vector<int32_t> iv(2 * n);
        for (uint32_t k = 0; k < size; ++k)
            for (uint32_t i = 0; i < size; ++i) bt[i * size + k] = b.basis[g][k * size + i];
        price::Scratch sc{d.data(), d.data() + n, d.data() + 2 * n, d.data() + 3 * n,
                          d.data() + 4 * n, iv.data(), iv.data() + n};
        for (uint32_t i = b.first[g]; i < b.first[g + 1]; ++i) {
            const price::Priced p = price::price_node(
                b.im.px, b.im.w, b.row[i], b.col[i], size, b.cands.data() + (size_t)i * b.k, b.k,
                b.setup, {b.bits, b.offset}, b.basis[g], bt.data(), (uint32_t)__builtin_ctz(size),
                sc, {0, 1});
            b.priced[i] = p;
            if (p.has_levels)
                for (uint32_t k = 0; k < n; ++k) b.levels[b.levels_at[i] + k] = (int8_t)sc.best_levels[k];
        }
    }
    return MARS_OK;
}

}  // namespace

extern "C" int host_encode(const uint8_t* px, uint32_t w, uint32_t h, const mars_params* p,
                           const mars_options* o, int batch_pricing, mars_header* hdr,
                           mars_leaf* leaves, size_t cap_leaves, size_t* nleaves, int32_t* res,
                           size_t cap_res, size_t* nres, mars_counters* counters) {
    std::vector<int32_t> contracted((size_t)(w / 2) * (h / 2) + 1);
    orc_contract(px, w, h, contracted.data());
    const orc_params* op = reinterpret_cast<const orc_params*>(p);
    auto search = [&](uint32_t row, uint32_t col, uint32_t size, uint32_t shift, uint32_t k,
                      std::vector<mars_candidate>* out, uint64_t* evals) {
        std::vector<orc_candidate> c(k ? k : 1);
        uint32_t n = 0;
        if (orc_search(px, w, h, contracted.data(), row, col, size, shift, op, k, c.data(), &n,
                       evals))
            return MARS_EINVAL;
        out->resize(n);
        if (n) std::memcpy(out->data(), c.data(), n * sizeof(mars_candidate));
        return MARS_OK;
    };
    const codec::Provider provider = [&](uint32_t row, uint32_t col, uint32_t size,
                                         uint32_t shift, codec::SearchAnswer* a) {
        std::vector<mars_candidate> v;
        const int st = search(row, col, size, shift, 1, &v, &a->evals);
        std::memset(&a->cand, 0, sizeof a->cand);
        if (!st && !v.empty()) a->cand = v[0];
        return st;
    };
    const codec::RankedProvider ranked = [&](uint32_t row, uint32_t col, uint32_t size,
                                             uint32_t shift, uint32_t max,
                                             std::vector<mars_candidate>* v, uint64_t* evals) {
        return search(row, col, size, shift, max, v, evals);
    };
    const codec::Pricer pricer = price_on_host;
    std::vector<mars_leaf> lv;
    std::vector<int32_t> rv;
    const codec::Image im{px, w, h};
    if (int e = codec::encode(im, *p, *o, provider, provider, hdr, &lv, &rv, counters,
                              o->rd_candidates > 1 ? &ranked : nullptr,
                              batch_pricing ? &pricer : nullptr))
        return e;
    *nleaves = lv.size();
    *nres = rv.size();
    if (lv.size() > cap_leaves || rv.size() > cap_res) return MARS_ENOMEM;
    std::memcpy(leaves, lv.data(), lv.size() * sizeof(mars_leaf));
    if (!rv.empty()) std::memcpy(res, rv.data(), rv.size() * sizeof(int32_t));
    return MARS_OK;
}
