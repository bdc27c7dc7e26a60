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

// The 2-D transforms of dct.rs:22-80 with every 1-D output a left-to-right sum seeded with
// -0.0; b[k * n + i] = basis(n, k, i) and bt its transpose (bt[i * n + k]), which only
// changes which lane reads which address.  Forward (dct.rs:38-58): rows, then columns.
MARS_HD inline void forward_dct2d(const double* in, uint32_t n, const double* b, const double* bt,
                                  double* tmp, double* out, const Team& T) {
    for (uint32_t idx = T.lane; idx < n * n; idx += T.lanes) {
        const uint32_t r = idx / n, k = idx % n;
        double s = -0.0;
        for (uint32_t i = 0; i < n; ++i) s += in[r * n + i] * bt[i * n + k];
        tmp[r * n + k] = s;
    }
    T.sync();
    for (uint32_t idx = T.lane; idx < n * n; idx += T.lanes) {
        const uint32_t k = idx / n, c = idx % n;
        double s = -0.0;
        for (uint32_t i = 0; i < n; ++i) s += tmp[i * n + c] * b[k * n + i];
        out[k * n + c] = s;
    }
    T.sync();
}
// Inverse (dct.rs:60-80): columns, then rows.
MARS_HD inline void inverse_dct2d(const double* in, uint32_t n, const double* b, double* tmp,
                                  double* out, const Team& T) {
    for (uint32_t idx = T.lane; idx < n * n; idx += T.lanes) {
        const uint32_t i = idx / n, c = idx % n;
        double s = -0.0;
        for (uint32_t k = 0; k < n; ++k) s += in[k * n + c] * b[k * n + i];
        tmp[i * n + c] = s;
    }
    T.sync();
    for (uint32_t idx = T.lane; idx < n * n; idx += T.lanes) {
        const uint32_t r = idx / n, i = idx % n;
        double s = -0.0;
        for (uint32_t k = 0; k < n; ++k) s += tmp[r * n + k] * b[k * n + i];
        out[r * n + i] = s;
    }
    T.sync();
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

// The leaf's event bits with a fresh domain predictor (emit_leaf, mars_format.rs:515-595;
// the residual's events for mode 3, residual.rs), summed left to right from -0.0.
MARS_HD inline double leaf_bits(const RateTable& t, const Setup& s, const mars_leaf& leaf,
                                uint32_t sc, const int32_t* levels) {
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
        if (leaf.mode == 3) {
            const uint32_t n = leaf.size * leaf.size;
            for (uint32_t i = 0; i < n; ++i) {
                const uint32_t band = band_of(i, n);
                int32_t l = levels[i];
                if (l < -kLevelClamp) l = -kLevelClamp;
                if (l > kLevelClamp) l = kLevelClamp;
                r += rbits(t, F_RESID_NZ, sc * kBands + band, l != 0 ? 1u : 0u);
                if (l != 0)
                    r += rbits(t, F_RESID_MAG, sc * kBands + band,
                               ((uint32_t)l << 1) ^ (uint32_t)(l >> 31));
            }
        }
    }
    return r;
}

// affine_fit (encode.rs:1724-1781) on the block's doubles in range raster order.
MARS_HD inline void affine_fit(const double* block, uint32_t size, uint32_t bits_beta,
                               uint32_t* qbeta_out, int32_t* qgx_out, int32_t* qgy_out,
                               double* sse_out) {
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
    const uint32_t qbeta = quantise(dmax(b0 / 255.0 * (double)max_qbeta, 0.0), max_qbeta);
    auto qgrad = [](double g) {
        double r = round(g * kGradScale);
        if (r < -(double)kGradClamp) r = -(double)kGradClamp;
        if (r > (double)kGradClamp) r = (double)kGradClamp;
        return (int32_t)r;
    };
    const int32_t qgx = qgrad(gx), qgy = qgrad(gy);
    const double b0q = (double)qbeta / (double)max_qbeta * 255.0;
    const double gxq = (double)qgx / kGradScale, gyq = (double)qgy / kGradScale;
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

// residual_for_candidate (encode.rs:1783-1851): levels into sc.levels, returns the SSE of
// the clamped, truncated reconstruction.
MARS_HD inline double residual_for_candidate(const uint8_t* px, uint32_t stride, uint32_t size,
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
    double sse = 0.0;
    for (uint32_t u = 0; u < size; ++u)
        for (uint32_t v = 0; v < size; ++v) {
            const uint32_t k = u * size + v;
            uint32_t i, j;
            iso_map(c.isometry, u, v, size, &i, &j);
            double pv = sc.pred[k] + sc.coef[k];
            if (pv < 0.0) pv = 0.0;
            if (pv > 255.0) pv = 255.0;
            const double diff = sc.block[i * size + j] - (double)(uint8_t)pv;
            sse += diff * diff;
        }
    return sse;
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
// Every lane returns the same Priced; sc.best_levels is complete when it returns.
MARS_HD inline Priced price_node(const uint8_t* px, uint32_t stride, uint32_t row, uint32_t col,
                                 uint32_t size, const Cand* ranked, uint32_t nranked,
                                 const Setup& s, const RateTable& t, const double* b,
                                 const double* bt, uint32_t sc_class, Scratch& sc, const Team& T) {
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
        l.qbeta = best_beta(rsum, s0, s.bits_beta);
        const double beta2 = (double)l.qbeta / (double)((1u << s.bits_beta) - 1) * 255.0;
        double sse = -0.0;
        for (uint32_t k = 0; k < n; ++k) sse += (sc.block[k] - beta2) * (sc.block[k] - beta2);
        offer(l, sse, leaf_bits(t, s, l, sc_class, nullptr), false);
    };
    if (s.allowed[0]) mode0();
    if (s.allowed[1]) {
        mars_leaf l = make_leaf(row, col, size);
        l.mode = 1;
        double sse;
        affine_fit(sc.block, size, s.bits_beta, &l.qbeta, &l.qgx, &l.qgy, &sse);
        offer(l, sse, leaf_bits(t, s, l, sc_class, nullptr), false);
    }
    for (uint32_t ci = 0; ci < nranked; ++ci) {
        const Cand& c = ranked[ci];
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
            offer(l, sse2, leaf_bits(t, s, l, sc_class, nullptr), false);
        }
        if (s.allowed[3]) {
            l.mode = 3;
            const double sse3 = residual_for_candidate(px, stride, size, c, s, b, bt, sc, T);
            offer(l, sse3, leaf_bits(t, s, l, sc_class, sc.levels), true);
        }
    }
    if (!have) mode0();
    T.sync();
    return best;
}

}  // namespace price
}  // namespace mars
