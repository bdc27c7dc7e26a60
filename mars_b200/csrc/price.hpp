// RD pricing of one quadtree node (best_mode_leaf, crates/mars-codec/src/encode.rs:1536-1714)
// as __host__ __device__ code: the host walk and the device pricing kernel (rdprice.cu)
// run this one implementation, so their doubles agree bit for bit.  Everything is f64 in
// the reference's operation order; translation units that compile it for the device use
// --fmad=false (and the host ones -ffp-contract=off), so no a*b+c is fused.
//
// Pieces: best_beta (encode.rs:456-460), affine_fit (encode.rs:1724-1781),
// residual_for_candidate (encode.rs:1783-1851) with the DCT of dct.rs and the dead-zone
// quantiser of quant.rs:76-103, and the leaf's event bits (event_bits over leaf_events,
// encode.rs:1513-1518, mars_format.rs:453-595) read from a table of the frozen rate
// snapshot (RateModels, rate.rs:55-80) built once per encode on the host.
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>

#include "../../include/mars_b200.h"

#ifdef __CUDACC__
#define MARS_HD __host__ __device__
#else
#define MARS_HD
#endif

namespace mars {
namespace price {

// Event fields (mars_format.rs:113-133; residual events residual.rs) and contexts.
constexpr uint32_t F_SPLIT = 0, F_MODE = 1, F_QALFA = 2, F_QBETA = 3, F_QBETA_DC = 4,
                   F_ISOMETRY = 5, F_DOM_ROW = 6, F_DOM_COL = 7, F_GX = 8, F_GY = 9,
                   F_RESID_NZ = 10, F_RESID_MAG = 11;
constexpr uint32_t kFields = 12;
constexpr uint32_t kSizeClasses = 16;
constexpr uint32_t kBands = 4;
constexpr uint32_t kCtx = kSizeClasses * kBands;  // residual contexts are sc * 4 + band
constexpr double kGradScale = 64.0;                // AFFINE_GRAD_SCALE
constexpr int32_t kGradClamp = 2048;               // AFFINE_GRAD_CLAMP
constexpr int32_t kLevelClamp = 63;                // LEVEL_CLAMP
constexpr double kDeadZone = 0.5;                  // RESIDUAL_DEAD_ZONE

// bits[offset[field * kCtx + ctx] + symbol] = the snapshot's -log2 P(symbol) in that context
// (a fresh model's where the snapshot has none); offset -1 for contexts never asked for.
struct RateTable {
    const double* bits;
    const int64_t* offset;
};

// The fields of a search candidate (mars_candidate, Candidate of encode.rs:236-244) the
// pricing reads; the same leading layout as mars_candidate, without the moments.
struct Cand {
    uint32_t dom_row, dom_col, isometry, qalfa, qbeta, valid;
    double rms;
};
static_assert(offsetof(Cand, valid) == offsetof(mars_candidate, valid) &&
                  offsetof(Cand, rms) == offsetof(mars_candidate, rms) &&
                  alignof(mars_candidate) >= alignof(Cand),
              "a mars_candidate begins with a Cand");

// The constants one encode's pricing reads.
struct Setup {
    uint32_t bits_alfa;   // EncodeParams::bits_alfa
    double max_alfa;      // EncodeParams::max_alfa (the fit's, not the header's rounded one)
    uint32_t bits_beta;   // header
    uint32_t shift;       // header (domain coordinates are coded in units of it)
    double qstep;         // residual step (ResidualQstep::get)
    double lambda;
    uint8_t allowed[4];
};

MARS_HD inline double rbits(const RateTable& t, uint32_t field, uint32_t ctx, uint32_t sym) {
    return t.bits[t.offset[field * kCtx + ctx] + sym];
}

MARS_HD inline double dmax(double a, double b) { return a < b ? b : a; }  // std::max

// quantise_f64 (encode.rs:446-448).
MARS_HD inline uint32_t quantise(double x, uint32_t max) {
    double y = trunc(0.5 + x);
    if (y != y) return 0;  // NaN
    if (y < 0.0) y = 0.0;
    if (y > (double)max) y = (double)max;
    return (uint32_t)y;
}

// best_beta (encode.rs:456-460).
MARS_HD inline uint32_t best_beta(int64_t range_sum, int64_t count, uint32_t bits_beta) {
    const double mean = (double)range_sum / (double)count;
    const uint32_t max_qbeta = (1u << bits_beta) - 1;
    return quantise(mean / 255.0 * (double)max_qbeta, max_qbeta);
}

// isometry::map (isometry.rs:7-19).
MARS_HD inline void iso_map(uint32_t k, uint32_t u, uint32_t v, uint32_t size, uint32_t* i,
                            uint32_t* j) {
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

MARS_HD inline uint32_t zigzag(int64_t x) { return (uint32_t)((x << 1) ^ (x >> 63)); }

// dead_zone_quantize / dead_zone_dequantize (quant.rs:76-103), `as i32` saturating.
MARS_HD inline int32_t dz_quantize(double x, double step) {
    const double threshold = kDeadZone * step;
    const double ax = fabs(x);
    if (ax <= threshold) return 0;
    const double level = floor((ax - threshold) / step) + 1.0;
    const double s = x < 0.0 ? -level : level;
    if (!(s == s)) return 0;
    if (s >= 2147483647.0) return 2147483647;
    if (s <= -2147483648.0) return (-2147483647 - 1);
    return (int32_t)s;
}
MARS_HD inline double dz_dequantize(int32_t level, double step) {
    if (level == 0) return 0.0;
    const double threshold = kDeadZone * step;
    const uint32_t mag_level = level < 0 ? (uint32_t)(-(int64_t)level) : (uint32_t)level;
    const double mag = threshold + ((double)mag_level - 1.0 + 0.5) * step;
    return level < 0 ? -mag : mag;
}

MARS_HD inline uint32_t band_of(uint32_t index, uint32_t n) {
    const uint32_t b = (uint32_t)(((uint64_t)index * kBands) / n);
    return b < kBands - 1 ? b : kBands - 1;
}

// The lanes that price one node together: a warp on the device (lane 0..31), one thread
// on the host (lane 0 of 1).  Parallel loops stride by `lanes`; each output is still one
// lane's left-to-right sum, so the doubles do not depend on the lane count.  Serial sums are
// evaluated by every lane alike (no lane waits for another's result).
struct Team {
    uint32_t lane, lanes;
    MARS_HD void sync() const {
#ifdef __CUDA_ARCH__
        __syncwarp();
#endif
    }
};

// s += term(k) for k = 0..n-1, left to right: the terms of a group of eight are formed
// (loads, products) before the group's additions, so the dependent chain is additions only.
// The same values are added in the same order as a plain loop.
template <class F>
MARS_HD inline double chain(double s, uint32_t n, F term) {
    uint32_t k = 0;
    for (; k + 8 <= n; k += 8) {
        double x[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = term(k + j);
#pragma unroll
        for (int j = 0; j < 8; ++j) s += x[j];
    }
    for (; k < n; ++k) s += term(k);
    return s;
}

// Independent serial sums run side by side: sum j (j < nc <= 32) is
// init[j] + x_j[0] (+ y_j[0]) + x_j[1] (+ y_j[1]) + ..., n terms of x (and, when `pairs`,
// n terms of y read at y_j[k * ys_j]), left to right.  On the device lane j evaluates sum
// j -- the lanes run one instruction stream over different arrays -- and every lane
// receives all nc results; the host evaluates them one after another.  Each sum's order and
// values are those of a plain loop.
MARS_HD inline double one_sum(const double* x, const double* y, uint32_t ys, double init,
                              uint32_t n, bool pairs) {
    if (!pairs) return chain(init, n, [&](uint32_t k) { return x[k]; });
    return chain(init, 2 * n,
                 [&](uint32_t k) { return (k & 1) ? y[(size_t)(k >> 1) * ys] : x[k >> 1]; });
}
MARS_HD inline void team_sums(const double* const* x, const double* const* y, const uint32_t* ys,
                              const double* init, uint32_t nc, uint32_t n, bool pairs,
                              double* out, const Team& T) {
#ifdef __CUDA_ARCH__
    if (T.lanes > 1) {
        const uint32_t j = T.lane < nc ? T.lane : 0;
        const double v = one_sum(x[j], pairs ? y[j] : nullptr, pairs ? ys[j] : 0, init[j], n, pairs);
        for (uint32_t c = 0; c < nc; ++c) out[c] = __shfl_sync(0xffffffffu, v, c);
        return;
    }
#endif
    for (uint32_t j = 0; j < nc; ++j)
        out[j] = one_sum(x[j], pairs ? y[j] : nullptr, pairs ? ys[j] : 0, init[j], n, pairs);
}

// One pass of the 2-D transforms of dct.rs:22-80: for every output idx < n*n (the team's
// share, four interleaved per lane), out[idx] = the left-to-right sum from -0.0 over
// i < n of a[abase(idx) + i * sa] * b[bbase(idx) + i * sb].  A base is (idx / n) * n
// ("row"), idx % n ("col") or idx / n ("div").
enum Base : uint32_t { ROW, COL, DIV };
MARS_HD inline uint32_t base_of(Base m, uint32_t idx, uint32_t n) {
    return m == ROW ? (idx / n) * n : m == COL ? idx % n : idx / n;
}
MARS_HD inline void dct_pass(const double* a, Base am, uint32_t sa, const double* b, Base bm,
                             uint32_t sb, double* out, uint32_t n, const Team& T) {
    const uint32_t nn = n * n;
    for (uint32_t first = T.lane; first < nn; first += 4 * T.lanes) {
        uint32_t ia[4], ib[4];
        double acc[4];
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            uint32_t idx = first + g * T.lanes;
            if (idx >= nn) idx = nn - 1;  // computed, not stored
            ia[g] = base_of(am, idx, n);
            ib[g] = base_of(bm, idx, n);
            acc[g] = -0.0;
        }
        for (uint32_t i = 0; i < n; ++i) {
            double x[4];
#pragma unroll
            for (int g = 0; g < 4; ++g) x[g] = a[ia[g] + i * sa] * b[ib[g] + i * sb];
#pragma unroll
            for (int g = 0; g < 4; ++g) acc[g] += x[g];
        }
#pragma unroll
        for (int g = 0; g < 4; ++g)
            if (first + g * T.lanes < nn) out[first + g * T.lanes] = acc[g];
    }
    T.sync();
}

// b[k * n + i] = basis(n, k, i); bt its transpose (bt[i * n + k]), which only changes which
// lane reads which address.  Forward (dct.rs:38-58): rows (tmp[r][k] = sum_i in[r][i] *
// basis(k, i)), then columns (out[k][c] = sum_i tmp[i][c] * basis(k, i)).
MARS_HD inline void forward_dct2d(const double* in, uint32_t n, const double* b, const double* bt,
                                  double* tmp, double* out, const Team& T) {
    dct_pass(in, ROW, 1, bt, COL, n, tmp, n, T);
    dct_pass(tmp, COL, n, b, ROW, 1, out, n, T);
}
// Inverse (dct.rs:60-80): columns (tmp[i][c] = sum_k in[k][c] * basis(k, i)), then rows
// (out[r][i] = sum_k tmp[r][k] * basis(k, i)).
MARS_HD inline void inverse_dct2d(const double* in, uint32_t n, const double* b, double* tmp,
                                  double* out, const Team& T) {
    dct_pass(in, COL, n, b, DIV, n, tmp, n, T);
    dct_pass(tmp, ROW, 1, b, COL, n, out, n, T);
}

MARS_HD inline mars_leaf make_leaf(uint32_t row, uint32_t col, uint32_t size) {
    mars_leaf l;
    l.row = row;
    l.col = col;
    l.size = size;
    l.mode = l.qalfa = l.qbeta = l.isometry = l.dom_row = l.dom_col = 0;
    l.qgx = l.qgy = 0;
    return l;
}

// The residual's event bits per coefficient (residual.rs): nzb[i] the nonzero flag's, magb[i]
// the magnitude's (+0.0 for a zero level, which adds nothing to a positive total), looked up
// by the team in parallel.
MARS_HD inline void residual_event_bits(const RateTable& t, uint32_t sc, const int32_t* levels,
                                        uint32_t n, double* nzb, double* magb, const Team& T) {
    for (uint32_t i = T.lane; i < n; i += T.lanes) {
        const uint32_t band = band_of(i, n);
        int32_t l = levels[i];
        if (l < -kLevelClamp) l = -kLevelClamp;
        if (l > kLevelClamp) l = kLevelClamp;
        nzb[i] = rbits(t, F_RESID_NZ, sc * kBands + band, l != 0 ? 1u : 0u);
        magb[i] = l != 0 ? rbits(t, F_RESID_MAG, sc * kBands + band,
                                 ((uint32_t)l << 1) ^ (uint32_t)(l >> 31))
                         : 0.0;
    }
    T.sync();
}

// The leaf's event bits with a fresh domain predictor (emit_leaf, mars_format.rs:515-595;
// the residual's events for mode 3, residual.rs), summed left to right from -0.0.  Mode 3
// reads its events' bits from residual_event_bits; without them (nzb null) the result is
// the sum up to the first residual event, which the residual's events then continue.
MARS_HD inline double leaf_bits(const RateTable& t, const Setup& s, const mars_leaf& leaf,
                                uint32_t sc, const double* nzb = nullptr,
                                const double* magb = nullptr) {
    double r = -0.0;
    r += rbits(t, F_MODE, sc, leaf.mode);
    if (leaf.mode == 0) {
        r += rbits(t, F_QBETA_DC, sc, leaf.qbeta);
    } else if (leaf.mode == 1) {
        r += rbits(t, F_QBETA_DC, sc, leaf.qbeta);
        r += rbits(t, F_GX, sc, zigzag(leaf.qgx));
        r += rbits(t, F_GY, sc, zigzag(leaf.qgy));
    } else {
        r += rbits(t, F_QALFA, sc, leaf.qalfa - 1);
        r += rbits(t, F_QBETA, sc, leaf.qbeta);
        r += rbits(t, F_ISOMETRY, sc, leaf.isometry);
        r += rbits(t, F_DOM_ROW, sc, zigzag((int64_t)(leaf.dom_row / s.shift)));
        r += rbits(t, F_DOM_COL, sc, zigzag((int64_t)(leaf.dom_col / s.shift)));
        if (leaf.mode == 3 && nzb) {
            // r > 0 here (every event costs bits), so adding a zero level's +0.0 is exact.
            const uint32_t n = leaf.size * leaf.size;
            r = chain(r, 2 * n, [&](uint32_t k) { return (k & 1) ? magb[k >> 1] : nzb[k >> 1]; });
        }
    }
    return r;
}

// affine_fit (encode.rs:1724-1781) from the block's sums t0 = sum p, tu = sum p*u,
// tv = sum p*v (each from 0.0, raster order): the quantised plane and its coefficients.
struct Affine {
    uint32_t qbeta;
    int32_t qgx, qgy;
    double b0q, gxq, gyq;
};
MARS_HD inline Affine affine_from_sums(double t0, double tu, double tv, uint32_t size,
                                       uint32_t bits_beta) {
    const double n = (double)size * (double)size;
    double su = -0.0, suu = -0.0;
    for (uint32_t u = 0; u < size; ++u) su += (double)u;
    for (uint32_t u = 0; u < size; ++u) suu += (double)u * (double)u;
    const double s0 = n, s_u = (double)size * su, s_v = s_u, s_uu = (double)size * suu,
                 s_vv = s_uu, s_uv = su * su;
    struct M3 {
        double m[3][3];
    };
    auto det3 = [](const M3& a) {
        const double(&m)[3][3] = a.m;
        return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
               m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
               m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    };
    const M3 a{{{s0, s_u, s_v}, {s_u, s_uu, s_uv}, {s_v, s_uv, s_vv}}};
    const double det_a = det3(a);
    double b0, gx, gy;
    if (fabs(det_a) < 1e-9) {
        b0 = t0 / s0;
        gx = 0.0;
        gy = 0.0;
    } else {
        const M3 a_b0{{{t0, s_u, s_v}, {tu, s_uu, s_uv}, {tv, s_uv, s_vv}}};
        const M3 a_gx{{{s0, t0, s_v}, {s_u, tu, s_uv}, {s_v, tv, s_vv}}};
        const M3 a_gy{{{s0, s_u, t0}, {s_u, s_uu, tu}, {s_v, s_uv, tv}}};
        b0 = det3(a_b0) / det_a;
        gx = det3(a_gx) / det_a;
        gy = det3(a_gy) / det_a;
    }
    const uint32_t max_qbeta = (1u << bits_beta) - 1;
    Affine f;
    f.qbeta = quantise(dmax(b0 / 255.0 * (double)max_qbeta, 0.0), max_qbeta);
    auto qgrad = [](double g) {
        double r = round(g * kGradScale);
        if (r < -(double)kGradClamp) r = -(double)kGradClamp;
        if (r > (double)kGradClamp) r = (double)kGradClamp;
        return (int32_t)r;
    };
    f.qgx = qgrad(gx);
    f.qgy = qgrad(gy);
    f.b0q = (double)f.qbeta / (double)max_qbeta * 255.0;
    f.gxq = (double)f.qgx / kGradScale;
    f.gyq = (double)f.qgy / kGradScale;
    return f;
}
// The squared error of pixel k against the quantised plane (affine_fit's SSE term).
MARS_HD inline double affine_term(const Affine& f, double p, uint32_t k, uint32_t size) {
    const double pred = f.b0q + f.gxq * (double)(k / size) + f.gyq * (double)(k % size);
    const double diff = p - pred;
    return diff * diff;
}

// Scratch of one node's pricing: five double and two int32 arrays of size*size each.
struct Scratch {
    double *block, *pred, *resid, *tmp, *coef;
    int32_t *levels, *best_levels;
};

// The sum of the team's int64 partials (integer addition: the grouping does not matter).
MARS_HD inline int64_t team_sum(int64_t v, const Team& T) {
#ifdef __CUDA_ARCH__
    if (T.lanes > 1)
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
#else
    (void)T;
#endif
    return v;
}

// residual_for_candidate (encode.rs:1783-1851): levels into sc.levels and, in sc.pred, the
// squared error of every pixel of the clamped, truncated reconstruction (their sum, from 0.0
// in raster order, is the candidate's SSE).
MARS_HD inline void residual_for_candidate(const uint8_t* px, uint32_t stride, uint32_t size,
                                             const Cand& c, const Setup& s, const double* b,
                                             const double* bt, Scratch& sc, const Team& T) {
    const double alfa = (double)c.qalfa / (double)(1u << s.bits_alfa) * s.max_alfa;
    double beta = (double)c.qbeta / (double)((1u << s.bits_beta) - 1) * ((1.0 + fabs(alfa)) * 255.0);
    if (alfa > 0.0) beta -= alfa * 255.0;
    const uint32_t n = size * size;
    T.sync();  // the previous candidate's reads of pred / coef are done
    for (uint32_t k = T.lane; k < n; k += T.lanes) {
        const uint32_t u = k / size, v = k % size;
        const uint32_t dr = c.dom_row + 2 * u, dc = c.dom_col + 2 * v;
        const double d = ((double)px[(size_t)dr * stride + dc] + (double)px[(size_t)(dr + 1) * stride + dc] +
                          (double)px[(size_t)dr * stride + dc + 1] +
                          (double)px[(size_t)(dr + 1) * stride + dc + 1]) /
                         4.0;
        uint32_t i, j;
        iso_map(c.isometry, u, v, size, &i, &j);
        const double pred = 0.5 + d * alfa + beta;
        sc.pred[k] = pred;
        sc.resid[k] = sc.block[i * size + j] - pred;
    }
    T.sync();
    forward_dct2d(sc.resid, size, b, bt, sc.tmp, sc.coef, T);
    for (uint32_t k = T.lane; k < n; k += T.lanes) {
        int32_t l = dz_quantize(sc.coef[k], s.qstep);
        if (l < -kLevelClamp) l = -kLevelClamp;
        if (l > kLevelClamp) l = kLevelClamp;
        sc.levels[k] = l;
        sc.resid[k] = dz_dequantize(l, s.qstep);  // the dequantised coefficients
    }
    T.sync();
    inverse_dct2d(sc.resid, size, b, sc.tmp, sc.coef, T);  // coef <- the reconstruction
    // The decoded pixels' squared errors replace the prediction, element by element.
    for (uint32_t k = T.lane; k < n; k += T.lanes) {
        uint32_t i, j;
        iso_map(c.isometry, k / size, k % size, size, &i, &j);
        double pv = sc.pred[k] + sc.coef[k];
        if (pv < 0.0) pv = 0.0;
        if (pv > 255.0) pv = 255.0;
        const double diff = sc.block[i * size + j] - (double)(uint8_t)pv;
        sc.pred[k] = diff * diff;
    }
    T.sync();
}

// The priced winner of one node.
struct Priced {
    mars_leaf leaf;
    double d, r;
    uint32_t has_levels;  // mode 3: the levels are in sc.best_levels
    uint32_t pad;
};

// best_mode_leaf (encode.rs:1536-1714) for the node's block over the ranked candidates
// (the single winner unless rd_candidates > 1; invalid or qalfa < 1 ones are skipped);
// candidates are compared in the reference's order by J = d + lambda * r, first minimum.
// Every lane returns the same Priced; sc.best_levels is complete when it returns.  The
// candidates sit `cand_bytes` apart (a mars_candidate array, whose leading fields are a Cand,
// is read in place).
MARS_HD inline Priced price_node(const uint8_t* px, uint32_t stride, uint32_t row, uint32_t col,
                                 uint32_t size, const Cand* ranked, uint32_t nranked,
                                 const Setup& s, const RateTable& t, const double* b,
                                 const double* bt, uint32_t sc_class, Scratch& sc, const Team& T,
                                 uint32_t cand_bytes = sizeof(Cand)) {
    const uint32_t n = size * size;
    int64_t part = 0;
    for (uint32_t k = T.lane; k < n; k += T.lanes) {
        const uint32_t v = px[(size_t)(row + k / size) * stride + col + k % size];
        sc.block[k] = (double)v;
        part += v;
    }
    const int64_t rsum = team_sum(part, T);
    T.sync();
    const int64_t s0 = (int64_t)size * size;
    // Mode 0's SSE and mode 1's moments t0, tu, tv: four independent sums side by side.
    const uint32_t qbeta0 = best_beta(rsum, s0, s.bits_beta);
    const double beta2 = (double)qbeta0 / (double)((1u << s.bits_beta) - 1) * 255.0;
    for (uint32_t k = T.lane; k < n; k += T.lanes) {
        const double p = sc.block[k];
        sc.pred[k] = (p - beta2) * (p - beta2);
        sc.resid[k] = p * (double)(k / size);
        sc.tmp[k] = p * (double)(k % size);
    }
    T.sync();
    double sums[4];
    {
        const double* xs[4] = {sc.pred, sc.block, sc.resid, sc.tmp};
        const double init[4] = {-0.0, 0.0, 0.0, 0.0};
        team_sums(xs, nullptr, nullptr, init, 4, n, false, sums, T);
    }
    T.sync();
    Affine aff{};
    double sse1 = 0.0;
    if (s.allowed[1]) {
        aff = affine_from_sums(sums[1], sums[2], sums[3], size, s.bits_beta);
        for (uint32_t k = T.lane; k < n; k += T.lanes) sc.pred[k] = affine_term(aff, sc.block[k], k, size);
        T.sync();
        const double* xs[1] = {sc.pred};
        const double init[1] = {0.0};
        team_sums(xs, nullptr, nullptr, init, 1, n, false, &sse1, T);
        T.sync();
    }
    Priced best;
    best.leaf = make_leaf(row, col, size);
    best.d = best.r = 0.0;
    best.has_levels = 0;
    best.pad = 0;
    bool have = false;
    auto offer = [&](const mars_leaf& l, double d, double r, bool levels) {
        if (!have || d + s.lambda * r < best.d + s.lambda * best.r) {
            best.leaf = l;
            best.d = d;
            best.r = r;
            best.has_levels = levels ? 1u : 0u;
            if (levels)
                for (uint32_t k = T.lane; k < n; k += T.lanes) sc.best_levels[k] = sc.levels[k];
            have = true;
        }
    };
    auto mode0 = [&]() {
        mars_leaf l = make_leaf(row, col, size);
        l.qbeta = qbeta0;
        offer(l, sums[0], leaf_bits(t, s, l, sc_class), false);
    };
    if (s.allowed[0]) mode0();
    if (s.allowed[1]) {
        mars_leaf l = make_leaf(row, col, size);
        l.mode = 1;
        l.qbeta = aff.qbeta;
        l.qgx = aff.qgx;
        l.qgy = aff.qgy;
        offer(l, sse1, leaf_bits(t, s, l, sc_class), false);
    }
    const double zero = 0.0;
    for (uint32_t ci = 0; ci < nranked; ++ci) {
        const Cand& c = *reinterpret_cast<const Cand*>(
            reinterpret_cast<const unsigned char*>(ranked) + (size_t)ci * cand_bytes);
        if (!c.valid || c.qalfa < 1) continue;
        mars_leaf l = make_leaf(row, col, size);
        l.qalfa = c.qalfa;
        l.qbeta = c.qbeta;
        l.isometry = c.isometry;
        l.dom_row = c.dom_row;
        l.dom_col = c.dom_col;
        if (s.allowed[2]) {
            l.mode = 2;
            const double sse2 = c.rms * c.rms * (double)size * (double)size;
            offer(l, sse2, leaf_bits(t, s, l, sc_class), false);
        }
        if (s.allowed[3]) {
            l.mode = 3;
            residual_for_candidate(px, stride, size, c, s, b, bt, sc, T);
            // resid and tmp are free once the reconstruction's squared errors are in pred.
            residual_event_bits(t, sc_class, sc.levels, n, sc.tmp, sc.resid, T);
            // The SSE (each term paired with +0.0: the sum is >= 0, so nothing changes) and
            // the bits (the leaf's events up to the residual, then every coefficient's nonzero
            // flag and magnitude) side by side.
            double v[2];
            const double* xs[2] = {sc.pred, sc.tmp};
            const double* ys[2] = {&zero, sc.resid};
            const uint32_t ystride[2] = {0, 1};
            const double init[2] = {0.0, leaf_bits(t, s, l, sc_class)};
            team_sums(xs, ys, ystride, init, 2, n, true, v, T);
            offer(l, v[0], v[1], true);
        }
    }
    if (!have) mode0();
    T.sync();
    return best;
}

}  // namespace price
}  // namespace mars
