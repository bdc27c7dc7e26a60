// The .mars v0 plane container (crates/mars-codec/src/mars_format.rs) and the C ABI over
// it and over the entropy coder.
//
// Layout (mars_format.rs:1-16, 232-300), little-endian: "MARS", version 0, flags 0,
// channels 1, bit depth 8, colour space 0, min_size, max_size, shift, bits_alfa, bits_beta,
// int_max_alfa (one byte each), width and height (u16), section count, the residual step
// as IEEE binary32 (24 bytes in all), then (u8 id, u32 length, payload) sections.  The one
// section written is TREE (id 1): the quadtree's events (walk_write / emit_leaf) coded
// with the adaptive-model rANS stack of entropy.hpp.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>

#include "codec.hpp"
#include "residual.hpp"

namespace mars {
int set_last_error(int code, const std::string& msg);  // api.cu
}  // namespace mars

namespace {

using namespace mars::codec;
namespace ent = mars::entropy;

constexpr size_t kHeaderLen = 24;
constexpr size_t kSectionEntryLen = 5;
constexpr uint8_t kSectionTree = 1;
constexpr uint32_t kMaxBits = 24;                  // mars_format.rs:139
constexpr uint64_t kMaxLeafPositions = 1ull << 24;  // mars_format.rs:199

int fail(int code, const std::string& msg) { return mars::set_last_error(code, msg); }

// valid_header_fields + leaf_count_within_bound (mars_format.rs:201-228).
bool header_ok(const mars_header& h) {
    if (h.width == 0 || h.height == 0 || h.shift == 0 || h.bits_alfa < 2 ||
        h.bits_alfa > kMaxBits || h.bits_beta < 1 || h.bits_beta > kMaxBits || h.min_size == 0 ||
        h.max_size < h.min_size)
        return false;
    const uint64_t q = (uint64_t)virtual_size(h) / h.min_size;
    return q * q <= kMaxLeafPositions;
}

// ResidualQstep::new (quant.rs:29-35): finite and within [1, 65535].
bool qstep_ok(float q) { return std::isfinite(q) && (double)q >= 1.0 && (double)q <= 65535.0; }

struct ReadState {
    const mars_header& hdr;
    ent::Decoder& dec;
    Predictor pred;
    std::vector<mars_leaf>& leaves;
    std::vector<int32_t>& resid;
    std::string err;
    int code = MARS_OK;
};

bool next(ReadState& st, ContextKey ctx, uint32_t alphabet, uint32_t* sym) {
    if (st.dec.next(ctx, alphabet, sym)) return true;
    st.code = MARS_EFORMAT;
    st.err = "an alphabet of " + std::to_string(alphabet) + " symbols exceeds the 24-bit models";
    return false;
}

// walk_read (mars_format.rs:597-731).
bool walk_read(ReadState& st, uint32_t row, uint32_t col, uint32_t size) {
    const mars_header& hdr = st.hdr;
    if (row >= hdr.height || col >= hdr.width) return true;
    const uint32_t half = size / 2;
    const bool forced = size > hdr.max_size || row + size > hdr.height || col + size > hdr.width;
    const uint32_t sc = (uint32_t)__builtin_ctz(size);
    bool split = forced;
    if (!forced && size > hdr.min_size) {
        uint32_t s;
        if (!next(st, {FIELD_SPLIT, sc}, 2, &s)) return false;
        split = s == 1;
    }
    if (split)
        return walk_read(st, row, col, half) && walk_read(st, row + half, col, half) &&
               walk_read(st, row, col + half, half) && walk_read(st, row + half, col + half, half);

    mars_leaf L{};
    L.row = row;
    L.col = col;
    L.size = size;
    if (!next(st, {FIELD_MODE, sc}, MODE_ALPHABET, &L.mode)) return false;
    if (L.mode == 0 || L.mode == 1) {
        if (!next(st, {FIELD_QBETA_DC, sc}, 1u << hdr.bits_beta, &L.qbeta)) return false;
        if (L.mode == 1) {
            const uint32_t alph = (uint32_t)(2 * (int64_t)AFFINE_GRAD_CLAMP + 1);
            uint32_t zx, zy;
            if (!next(st, {FIELD_GX, sc}, alph, &zx) || !next(st, {FIELD_GY, sc}, alph, &zy))
                return false;
            L.qgx = (int32_t)unzigzag(zx);
            L.qgy = (int32_t)unzigzag(zy);
        }
        st.leaves.push_back(L);
        return true;
    }
    uint32_t qa, dz_r, dz_c;
    if (!next(st, {FIELD_QALFA, sc}, (1u << hdr.bits_alfa) - 1, &qa) ||
        !next(st, {FIELD_QBETA, sc}, 1u << hdr.bits_beta, &L.qbeta) ||
        !next(st, {FIELD_ISOMETRY, sc}, 8, &L.isometry))
        return false;
    L.qalfa = qa + 1;
    const uint32_t row_alph = (uint32_t)(2 * (1ll << bits_coord_row(hdr)));
    const uint32_t col_alph = (uint32_t)(2 * (1ll << bits_coord_col(hdr)));
    if (!next(st, {FIELD_DOM_ROW, sc}, row_alph, &dz_r) ||
        !next(st, {FIELD_DOM_COL, sc}, col_alph, &dz_c))
        return false;
    const int64_t ru = st.pred.row + unzigzag(dz_r), cu = st.pred.col + unzigzag(dz_c);
    st.pred.row = ru;
    st.pred.col = cu;
    const auto out_of_bounds = [&] {
        st.code = MARS_EFORMAT;
        st.err = "leaf at (" + std::to_string(row) + "," + std::to_string(col) + "," +
                 std::to_string(size) + ") references a domain that runs past the image";
        return false;
    };
    if (ru < 0 || cu < 0 || ru > 0xffffffffll || cu > 0xffffffffll) return out_of_bounds();
    // u32 arithmetic as in the reference (a wrapped product fails the bound below or not,
    // exactly as there).
    L.dom_row = hdr.shift * (uint32_t)ru;
    L.dom_col = hdr.shift * (uint32_t)cu;
    if (L.dom_row + 2 * size > hdr.height || L.dom_col + 2 * size > hdr.width)
        return out_of_bounds();
    if (L.mode == 3 &&
        !mars::residual::decode_values(st.dec, sc, (size_t)size * size, &st.resid)) {
        st.code = MARS_EFORMAT;
        st.err = "residual alphabet out of range";
        return false;
    }
    st.leaves.push_back(L);
    return true;
}

int format_write(const mars_header& hdr, const mars_leaf* leaves, size_t n, const int32_t* resid,
                 size_t nresid, std::vector<uint8_t>* out) {
    const float qstep = hdr.residual_qstep == 0.0f ? 8.0f : hdr.residual_qstep;
    if (!header_ok(hdr))
        return fail(MARS_EINVAL,
                    "degenerate header: width, height and shift must be nonzero, bits_alfa "
                    "2..24, bits_beta 1..24, 0 < min_size <= max_size, at most 2^24 leaf positions");
    if (hdr.width > 65535 || hdr.height > 65535)
        return fail(MARS_EINVAL, "width/height do not fit in the format's 16-bit fields");
    if (hdr.min_size > 255 || hdr.max_size > 255 || hdr.shift > 255)
        return fail(MARS_EINVAL, "min_size/max_size/shift do not fit in the format's 8-bit fields");
    if (!qstep_ok(qstep)) return fail(MARS_EINVAL, "residual qstep must be finite and in [1, 65535]");
    std::vector<int64_t> offs;
    if (!residual_offsets(leaves, n, nresid, &offs) || (nresid && !resid))
        return fail(MARS_EINVAL, "the residual pool does not hold size*size levels per mode-3 leaf");
    LeafMap by_pos;
    for (size_t k = 0; k < n; ++k) {
        const mars_leaf& l = leaves[k];
        if (l.mode > 3) return fail(MARS_EINVAL, "leaf mode must be 0..3");
        const int32_t* lv = offs[k] >= 0 ? resid + offs[k] : nullptr;
        if (!by_pos.emplace(std::make_tuple(l.row, l.col, l.size), LeafRef{&l, lv}).second)
            return fail(MARS_EINVAL, "two leaves claim the same position (" + std::to_string(l.row) +
                                         "," + std::to_string(l.col) + "," +
                                         std::to_string(l.size) + ")");
    }
    std::vector<Event> events;
    Predictor pred;
    if (!walk_write(hdr, 0, 0, virtual_size(hdr), by_pos, pred, events))
        return fail(MARS_EINVAL, "the leaves do not tile the quadtree (a leaf is missing)");
    std::vector<uint8_t> tree;
    if (!ent::encode_events(events, &tree))
        return fail(MARS_EINVAL, "a leaf field is outside its alphabet");
    if (tree.size() > 0xffffffffull) return fail(MARS_EINVAL, "tree section exceeds 4 GiB");
    out->clear();
    out->reserve(kHeaderLen + kSectionEntryLen + tree.size());
    const uint8_t head[14] = {'M', 'A', 'R', 'S', 0, 0, 1, 8, 0, (uint8_t)hdr.min_size,
                              (uint8_t)hdr.max_size, (uint8_t)hdr.shift, (uint8_t)hdr.bits_alfa,
                              (uint8_t)hdr.bits_beta};
    out->insert(out->end(), head, head + 14);
    out->push_back((uint8_t)hdr.int_max_alfa);
    out->push_back((uint8_t)hdr.width);
    out->push_back((uint8_t)(hdr.width >> 8));
    out->push_back((uint8_t)hdr.height);
    out->push_back((uint8_t)(hdr.height >> 8));
    out->push_back(1);  // section count
    uint32_t qbits;
    std::memcpy(&qbits, &qstep, 4);
    for (int b = 0; b < 4; ++b) out->push_back((uint8_t)(qbits >> (8 * b)));
    out->push_back(kSectionTree);
    const uint32_t tl = (uint32_t)tree.size();
    for (int b = 0; b < 4; ++b) out->push_back((uint8_t)(tl >> (8 * b)));
    out->insert(out->end(), tree.begin(), tree.end());
    return MARS_OK;
}

int format_read(const uint8_t* d, size_t len, mars_header* hdr, std::vector<mars_leaf>* leaves,
                std::vector<int32_t>* resid) {
    if (len < kHeaderLen) return fail(MARS_EFORMAT, "header truncated");
    if (std::memcmp(d, "MARS", 4) != 0) return fail(MARS_EFORMAT, "not a .mars file: bad magic");
    if (d[4] != 0) return fail(MARS_EFORMAT, "unsupported .mars version " + std::to_string(d[4]));
    const uint32_t qbits = (uint32_t)d[20] | (uint32_t)d[21] << 8 | (uint32_t)d[22] << 16 |
                           (uint32_t)d[23] << 24;
    float q;
    std::memcpy(&q, &qbits, 4);
    if (!qstep_ok(q)) return fail(MARS_EFORMAT, "residual qstep must be finite and in [1, 65535]");
    mars_header h{};
    h.min_size = d[9];
    h.max_size = d[10];
    h.shift = d[11];
    h.bits_alfa = d[12];
    h.bits_beta = d[13];
    h.int_max_alfa = d[14];
    h.width = (uint32_t)d[15] | (uint32_t)d[16] << 8;
    h.height = (uint32_t)d[17] | (uint32_t)d[18] << 8;
    const uint32_t sections = d[19];
    if (!header_ok(h)) return fail(MARS_EFORMAT, "degenerate header");
    size_t off = kHeaderLen;
    const uint8_t* tree = nullptr;
    size_t tree_len = 0;
    for (uint32_t k = 0; k < sections; ++k) {
        if (off + kSectionEntryLen > len) return fail(MARS_EFORMAT, "header truncated");
        const uint8_t id = d[off];
        const size_t sl = (size_t)d[off + 1] | (size_t)d[off + 2] << 8 | (size_t)d[off + 3] << 16 |
                          (size_t)d[off + 4] << 24;
        off += kSectionEntryLen;
        if (sl > len - off)
            return fail(MARS_EFORMAT, "section table claims " + std::to_string(sl) +
                                          " bytes but only " + std::to_string(len - off) +
                                          " remain");
        if (id == kSectionTree) {
            tree = d + off;
            tree_len = sl;
        }
        off += sl;
    }
    if (!tree) return fail(MARS_EFORMAT, "the TREE section is missing");
    mars::entropy::Decoder dec;
    if (!dec.init(tree, tree_len))
        return fail(MARS_EFORMAT, "compressed tree payload ends in an all-zero word");
    leaves->clear();
    resid->clear();
    ReadState st{h, dec, Predictor{}, *leaves, *resid, std::string(), MARS_OK};
    if (!walk_read(st, 0, 0, virtual_size(h))) return fail(st.code, st.err);
    h.residual_qstep = q;
    *hdr = h;
    return MARS_OK;
}

template <class T>
int copy_out(const std::vector<T>& v, T** out, size_t* n) {
    *n = v.size();
    *out = (T*)std::malloc(std::max<size_t>(1, v.size()) * sizeof(T));
    if (!*out) return fail(MARS_ENOMEM, "allocation failed");
    if (!v.empty()) std::memcpy(*out, v.data(), v.size() * sizeof(T));
    return MARS_OK;
}

}  // namespace

extern "C" {

int mars_format_write(const mars_header* header, const mars_leaf* leaves, size_t n,
                      const int32_t* residuals, size_t nresiduals, uint8_t** out, size_t* len) {
    if (!header || (n && !leaves) || !out || !len) return fail(MARS_EINVAL, "NULL argument");
    std::vector<uint8_t> bytes;
    if (int e = format_write(*header, leaves, n, residuals, nresiduals, &bytes)) return e;
    return copy_out(bytes, out, len);
}

int mars_format_read(const uint8_t* data, size_t len, mars_header* header, mars_leaf** leaves,
                     size_t* nleaves, int32_t** residuals, size_t* nresiduals) {
    if ((len && !data) || !header || !leaves || !nleaves || !residuals || !nresiduals)
        return fail(MARS_EINVAL, "NULL argument");
    std::vector<mars_leaf> out;
    std::vector<int32_t> res;
    if (int e = format_read(data, len, header, &out, &res)) return e;
    if (int e = copy_out(out, leaves, nleaves)) return e;
    if (int e = copy_out(res, residuals, nresiduals)) {
        std::free(*leaves);
        *leaves = nullptr;
        return e;
    }
    return MARS_OK;
}

int mars_entropy_encode(const mars_event* events, size_t n, uint8_t** out, size_t* len) {
    if ((n && !events) || !out || !len) return fail(MARS_EINVAL, "NULL argument");
    std::vector<Event> ev(n);
    for (size_t i = 0; i < n; ++i)
        ev[i] = Event{{events[i].field, events[i].disambiguator}, events[i].alphabet,
                      events[i].symbol};
    std::vector<uint8_t> bytes;
    if (!ent::encode_events(ev, &bytes))
        return fail(MARS_EINVAL, "an event's alphabet or symbol is out of range");
    return copy_out(bytes, out, len);
}

int mars_entropy_decode(const uint8_t* data, size_t len, const mars_event* shape, size_t n,
                        uint32_t* symbols) {
    if ((len && !data) || (n && (!shape || !symbols))) return fail(MARS_EINVAL, "NULL argument");
    ent::Decoder dec;
    if (!dec.init(data, len)) return fail(MARS_EFORMAT, "payload ends in an all-zero word");
    for (size_t i = 0; i < n; ++i)
        if (!dec.next({shape[i].field, shape[i].disambiguator}, shape[i].alphabet, &symbols[i]))
            return fail(MARS_EINVAL, "an alphabet is out of range");
    return MARS_OK;
}

}  // extern "C"
