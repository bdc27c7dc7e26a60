// Mode 3's residual: the orthonormal 2-D DCT-II (crates/mars-codec/src/dct.rs), the
// dead-zone quantiser (quant.rs:66-103) and the residual event vocabulary (residual.rs).
//
// The DCT is evaluated exactly as the reference does: basis(n, k, i) =
// sqrt(2/n) * c_k * cos(pi/n * (i + 0.5) * k) with c_0 = 1/sqrt(2), every 1-D transform a
// left-to-right sum of x[i] * basis seeded with -0.0 (Rust's f64 Sum), rows then columns
// forward, columns then rows inverse.  The basis values are cached per n; each is the same
// expression the reference evaluates at every use, so the cached doubles are identical.
// Host code only: the cosine is the C library's, as the reference's is.
#pragma once

#include <cmath>
#include <cstdint>
#include <map>
#include <mutex>
#include <vector>

#include "entropy.hpp"

namespace mars {
namespace residual {

constexpr double kDeadZone = 0.5;      // RESIDUAL_DEAD_ZONE, encode.rs:442
constexpr int32_t kLevelClamp = 63;    // LEVEL_CLAMP, residual.rs
constexpr uint32_t kBands = 4;         // BANDS, residual.rs
constexpr uint8_t FIELD_RESID_NZ = 10, FIELD_RESID_MAG = 11;

// basis(n, k, i) at [k * n + i] (dct.rs:13-20).  Each table is built once; the map's
// nodes never move, so a reference handed out stays valid while other threads insert.
inline const std::vector<double>& basis(uint32_t n) {
    static std::mutex mu;
    static std::map<uint32_t, std::vector<double>> cache;
    thread_local std::map<uint32_t, const std::vector<double>*> local;  // lock-free hits
    auto hit = local.find(n);
    if (hit != local.end()) return *hit->second;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(n);
    if (it != cache.end()) {
        local.emplace(n, &it->second);
        return it->second;
    }
    std::vector<double> b((size_t)n * n);
    const double pi = 3.14159265358979323846264338327950288;
    const double frac_1_sqrt_2 = 0.707106781186547524400844362104849039;
    for (uint32_t k = 0; k < n; ++k)
        for (uint32_t i = 0; i < n; ++i) {
            const double ck = k == 0 ? frac_1_sqrt_2 : 1.0;
            b[(size_t)k * n + i] =
                std::sqrt(2.0 / (double)n) * ck * std::cos(pi / (double)n * ((double)i + 0.5) * (double)k);
        }
    const std::vector<double>& ref = cache.emplace(n, std::move(b)).first->second;
    local.emplace(n, &ref);
    return ref;
}

// dct1d / idct1d over a strided vector (dct.rs:22-36).
inline void dct1d(const double* x, size_t stride, uint32_t n, const std::vector<double>& b,
                  double* out, size_t ostride) {
    for (uint32_t k = 0; k < n; ++k) {
        double s = -0.0;
        for (uint32_t i = 0; i < n; ++i) s += x[i * stride] * b[(size_t)k * n + i];
        out[k * ostride] = s;
    }
}
inline void idct1d(const double* c, size_t stride, uint32_t n, const std::vector<double>& b,
                   double* out, size_t ostride) {
    for (uint32_t i = 0; i < n; ++i) {
        double s = -0.0;
        for (uint32_t k = 0; k < n; ++k) s += c[k * stride] * b[(size_t)k * n + i];
        out[i * ostride] = s;
    }
}

// forward_dct2d (dct.rs:38-58): rows, then columns.
inline std::vector<double> forward_dct2d(const std::vector<double>& block, uint32_t n) {
    const auto& b = basis(n);
    std::vector<double> tmp((size_t)n * n), out((size_t)n * n);
    for (uint32_t r = 0; r < n; ++r) dct1d(&block[(size_t)r * n], 1, n, b, &tmp[(size_t)r * n], 1);
    for (uint32_t c = 0; c < n; ++c) dct1d(&tmp[c], n, n, b, &out[c], n);
    return out;
}

// inverse_dct2d (dct.rs:60-80): columns, then rows.
inline std::vector<double> inverse_dct2d(const std::vector<double>& coeffs, uint32_t n) {
    const auto& b = basis(n);
    std::vector<double> tmp((size_t)n * n), out((size_t)n * n);
    for (uint32_t c = 0; c < n; ++c) idct1d(&coeffs[c], n, n, b, &tmp[c], n);
    for (uint32_t r = 0; r < n; ++r) idct1d(&tmp[(size_t)r * n], 1, n, b, &out[(size_t)r * n], 1);
    return out;
}

// dead_zone_quantize / dead_zone_dequantize (quant.rs:76-103).
inline int32_t dead_zone_quantize(double x, double step, double dz) {
    const double threshold = dz * step;
    const double ax = std::fabs(x);
    if (ax <= threshold) return 0;
    const double level = std::floor((ax - threshold) / step) + 1.0;
    const double s = x < 0.0 ? -level : level;
    // `as i32` saturates.
    if (!(s == s)) return 0;
    if (s >= 2147483647.0) return 2147483647;
    if (s <= -2147483648.0) return (-2147483647 - 1);
    return (int32_t)s;
}
inline double dead_zone_dequantize(int32_t level, double step, double dz) {
    if (level == 0) return 0.0;
    const double threshold = dz * step;
    const uint32_t mag_level = level < 0 ? (uint32_t)(-(int64_t)level) : (uint32_t)level;
    const double mag = threshold + ((double)mag_level - 1.0 + 0.5) * step;
    return level < 0 ? -mag : mag;
}

// The reconstructed residual a decoder adds, in domain-local (u, v) order
// (ifs.rs:441-456).
inline std::vector<double> values(const int32_t* levels, uint32_t size, double step) {
    std::vector<double> deq((size_t)size * size);
    for (size_t k = 0; k < deq.size(); ++k) deq[k] = dead_zone_dequantize(levels[k], step, kDeadZone);
    return inverse_dct2d(deq, size);
}

inline uint32_t band_of(size_t index, size_t n) {
    const uint32_t b = (uint32_t)((index * kBands) / n);
    return b < kBands - 1 ? b : kBands - 1;
}

// encode_events (residual.rs): per coefficient a nonzero flag, then the zigzag level.
inline void encode_events(const int32_t* levels, size_t n, uint32_t size_class,
                          std::vector<entropy::Event>& ev) {
    for (size_t i = 0; i < n; ++i) {
        const uint32_t band = band_of(i, n);
        int32_t l = levels[i];
        if (l < -kLevelClamp) l = -kLevelClamp;
        if (l > kLevelClamp) l = kLevelClamp;
        ev.push_back({{FIELD_RESID_NZ, size_class * kBands + band}, 2, (uint32_t)(l != 0)});
        if (l != 0)
            ev.push_back({{FIELD_RESID_MAG, size_class * kBands + band},
                          (uint32_t)(2 * kLevelClamp + 1),
                          (uint32_t)(((uint32_t)l << 1) ^ (uint32_t)(l >> 31))});
    }
}

// decode_values (residual.rs): false when the entropy decoder refuses an alphabet.
inline bool decode_values(entropy::Decoder& dec, uint32_t size_class, size_t n,
                          std::vector<int32_t>* out) {
    for (size_t i = 0; i < n; ++i) {
        const uint32_t band = band_of(i, n);
        uint32_t nz, sym;
        if (!dec.next({FIELD_RESID_NZ, size_class * kBands + band}, 2, &nz)) return false;
        if (nz == 1) {
            if (!dec.next({FIELD_RESID_MAG, size_class * kBands + band},
                          (uint32_t)(2 * kLevelClamp + 1), &sym))
                return false;
            out->push_back((int32_t)(sym >> 1) ^ -(int32_t)(sym & 1));
        } else {
            out->push_back(0);
        }
    }
    return true;
}

}  // namespace residual
}  // namespace mars
