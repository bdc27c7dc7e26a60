// Adaptive order-0 models and the rANS stack coder of the .mars TREE section.
//
// AdaptiveModel restates crates/mars-entropy/src/lib.rs:36-121: Laplace-seeded counts, +32
// per coded symbol, every count halved (floor 1) once the total reaches 2^16, and a 24-bit
// fixed-point CDF derived by integer division, with one reserved slot per symbol.
//
// The coder is the stack ("last in, first out") rANS that mars-entropy drives through the
// third-party crate constriction 0.5.0 (`DefaultAnsCoder` = AnsCoder<u32, u64>; lib.rs:15-17,
// 280-291, 303-335).  constriction is not part of the reference tree; its published
// algorithm is restated here: 32-bit words, a 64-bit state, 24-bit probabilities.
//   push (left, prob):  if state >> 40 >= prob, emit the low word and shift it out;
//                       state = (state / prob) << 24 | (left + state % prob)
//   finish:             append the state's nonzero words, least significant first, so the
//                       most significant word is the top of the stack
//   start (decoder):    pop a nonzero word, then pop words below it until state >= 2^32
//   pop:                q = state mod 2^24 -> (symbol, left, prob) by the model's quantile
//                       function; state = (state >> 24) * prob + (q - left), then refill
//                       one word while state < 2^32 and words remain
// mars-entropy records a forward pass of (symbol, interval) pairs against the evolving
// models and pushes them in reverse, so the decoder pops them in forward order.
#pragma once

#include <cmath>
#include <cstdint>
#include <map>
#include <utility>
#include <vector>

namespace mars {
namespace entropy {

constexpr int kPrecision = 24;
constexpr uint64_t kPrecisionTotal = 1ull << kPrecision;

struct AdaptiveModel {
    std::vector<uint32_t> counts;
    uint64_t total = 0;
    explicit AdaptiveModel(uint32_t alphabet = 2) : counts(alphabet, 1u), total(alphabet) {}

    void update(uint32_t s) {
        counts[s] += 32;
        total += 32;
        if (total >= (1ull << 16)) {
            uint64_t t = 0;
            for (auto& c : counts) {
                c = std::max<uint32_t>(c >> 1, 1u);
                t += c;
            }
            total = t;
        }
    }
    uint32_t scaled(uint64_t c) const {
        return (uint32_t)(((unsigned __int128)c * (kPrecisionTotal - counts.size())) / total);
    }
    // (left cumulative, probability) of symbol s in 24-bit fixed point (lib.rs:84-90).
    void left_and_prob(uint32_t s, uint32_t* left, uint32_t* prob) const {
        uint64_t before = 0;
        for (uint32_t i = 0; i < s; ++i) before += counts[i];
        const uint32_t l = scaled(before) + s;
        const uint32_t r = scaled(before + counts[s]) + s + 1;
        *left = l;
        *prob = r - l;
    }
    double bits_for(uint32_t s) const {
        uint32_t left, prob;
        left_and_prob(s, &left, &prob);
        return -std::log2((double)prob / (double)kPrecisionTotal);
    }
    // bits_for of every symbol, with one running prefix: the same (left, prob) pairs and
    // the same doubles as calling bits_for symbol by symbol.
    void all_bits(double* out) const {
        uint64_t before = 0;
        for (uint32_t s = 0; s < (uint32_t)counts.size(); ++s) {
            const uint32_t l = scaled(before) + s;
            const uint32_t r = scaled(before + counts[s]) + s + 1;
            out[s] = -std::log2((double)(r - l) / (double)kPrecisionTotal);
            before += counts[s];
        }
    }
    // The symbol whose interval holds `quantile` (lib.rs:102-121).
    uint32_t symbol_for_quantile(uint32_t quantile, uint32_t* left, uint32_t* prob) const {
        uint64_t cum = 0;
        for (uint32_t i = 0; i < (uint32_t)counts.size(); ++i) {
            const uint64_t next = cum + counts[i];
            const uint32_t l = scaled(cum) + i;
            const uint32_t r = scaled(next) + i + 1;
            if (quantile < r) {
                *left = l;
                *prob = r - l;
                return i;
            }
            cum = next;
        }
        // Unreachable for quantile < 2^24: the last symbol's right end is 2^24.
        *left = 0;
        *prob = 1;
        return 0;
    }
};

using ContextKey = std::pair<uint8_t, uint32_t>;
struct Event {
    ContextKey ctx;
    uint32_t alphabet, symbol;
};

// Alphabets mars-entropy's AdaptiveModel::new accepts (lib.rs:45-57).
inline bool alphabet_ok(uint32_t a) { return a >= 2 && (uint64_t)a < kPrecisionTotal; }

struct AnsEncoder {
    std::vector<uint32_t> bulk;
    uint64_t state = 0;
    void push(uint32_t left, uint32_t prob) {
        if ((state >> (64 - kPrecision)) >= prob) {
            bulk.push_back((uint32_t)state);
            state >>= 32;
        }
        const uint64_t prefix = state / prob, rem = state % prob;
        state = (prefix << kPrecision) | (left + rem);
    }
    std::vector<uint32_t> finish() {
        if (state >> 32) {
            bulk.push_back((uint32_t)state);
            bulk.push_back((uint32_t)(state >> 32));
        } else if (state) {
            bulk.push_back((uint32_t)state);
        }
        return std::move(bulk);
    }
};

// encode (lib.rs:200-202, 240-265, 280-291): forward pass over evolving per-context models,
// pushed onto the stack in reverse; words little-endian.  Returns false when an event's
// alphabet or symbol is out of range (the reference panics there).
inline bool encode_events(const std::vector<Event>& events, std::vector<uint8_t>* out) {
    std::map<ContextKey, AdaptiveModel> models;
    std::vector<std::pair<uint32_t, uint32_t>> rec;
    rec.reserve(events.size());
    for (const Event& e : events) {
        auto it = models.find(e.ctx);
        if (it == models.end()) {
            if (!alphabet_ok(e.alphabet)) return false;
            it = models.emplace(e.ctx, AdaptiveModel(e.alphabet)).first;
        }
        if (e.symbol >= it->second.counts.size()) return false;
        uint32_t left, prob;
        it->second.left_and_prob(e.symbol, &left, &prob);
        rec.emplace_back(left, prob);
        it->second.update(e.symbol);
    }
    AnsEncoder enc;
    for (size_t i = rec.size(); i-- > 0;) enc.push(rec[i].first, rec[i].second);
    const std::vector<uint32_t> words = enc.finish();
    out->resize(words.size() * 4);
    for (size_t i = 0; i < words.size(); ++i)
        for (int b = 0; b < 4; ++b) (*out)[4 * i + b] = (uint8_t)(words[i] >> (8 * b));
    return true;
}

// Decoder (lib.rs:303-335).
class Decoder {
  public:
    // False for a payload whose last whole word is zero (AnsCoder::from_compressed refuses
    // it); a trailing partial word is ignored.
    bool init(const uint8_t* data, size_t len) {
        words_.resize(len / 4);
        for (size_t i = 0; i < words_.size(); ++i)
            words_[i] = (uint32_t)data[4 * i] | (uint32_t)data[4 * i + 1] << 8 |
                        (uint32_t)data[4 * i + 2] << 16 | (uint32_t)data[4 * i + 3] << 24;
        state_ = 0;
        if (words_.empty()) return true;
        const uint32_t first = words_.back();
        words_.pop_back();
        if (first == 0) return false;
        state_ = first;
        while (!words_.empty()) {
            state_ = state_ << 32 | words_.back();
            words_.pop_back();
            if (state_ >= (1ull << 32)) break;
        }
        return true;
    }
    // The next symbol of context ctx; false when the alphabet is not one the reference's
    // model accepts (it panics there).
    bool next(ContextKey ctx, uint32_t alphabet, uint32_t* symbol) {
        auto it = models_.find(ctx);
        if (it == models_.end()) {
            if (!alphabet_ok(alphabet)) return false;
            it = models_.emplace(ctx, AdaptiveModel(alphabet)).first;
        }
        const uint32_t quantile = (uint32_t)(state_ & (kPrecisionTotal - 1));
        uint32_t left, prob;
        const uint32_t s = it->second.symbol_for_quantile(quantile, &left, &prob);
        state_ = (state_ >> kPrecision) * prob + (quantile - left);
        if (state_ < (1ull << 32) && !words_.empty()) {
            state_ = state_ << 32 | words_.back();
            words_.pop_back();
        }
        it->second.update(s);
        *symbol = s;
        return true;
    }

  private:
    std::vector<uint32_t> words_;
    uint64_t state_ = 0;
    std::map<ContextKey, AdaptiveModel> models_;
};

}  // namespace entropy
}  // namespace mars
