// Exact affine fit and the rigorous pruning bound shared by every search kernel.
//
// fit_exact() restates fit_f64 (crates/mars-codec/src/encode.rs:247-289) with explicit
// round-to-nearest intrinsics so nvcc can never contract a*b+c into an FMA: the result is
// bit-identical to the reference's f64 arithmetic.
//
// The pruning bound: for a range block R (n = s*s pixels) and a domain D,
//   Nrr = n*t2 - t0^2,  Ndd = det = n*s2 - s1^2,  Nrd = n*t1 - s1*t0,
// and for any contrast a >= 0 the least-squares brightness gives
//   SSE(a) = (Nrr - 2*a*Nrd + a^2*Ndd) / n.
// The quantised fit's sum is SSE(alfa2, beta2) >= min over beta of SSE(alfa2, .), so
//   * every candidate has SSE >= LB_any = (Nrr - max(0,Nrd)^2/Ndd) / n, and
//   * a candidate with qalfa >= 1 has alfa2 >= a_min = max_alfa / 2^bits_alfa, so
//     SSE >= LB_1 = min over a >= a_min of SSE(a);
//   * a candidate with qalfa == 0 has exactly the domain-independent f64 sum `sum0`.
// A candidate x cannot beat the current champion c (rms_c, idx_c) when
//   LB_any(x) > T, or  [LB_1(x) > T and (rms0 > rms_c or (rms0 == rms_c and
//   idx_x > idx_c))],   with T = sum_c + eta,
// eta covering the f64 rounding of both sums (|f64 sum - exact SSE| <= 2.2e-9 * n *
// (1 + max_alfa)^2, eta = 1e-6 * n * (1 + max_alfa)^2).  Rewritten as a threshold on the
// exact integer t1_x4 = 4 * sum(r * D/4):
//   prune  <=>  t1_x4 < (s1_x4 * t0 + 4 * tau) / n,
//   tau = min(g2, max(g1, a_min*Ndd))     when the qalfa == 0 class cannot win,
//   tau = g1 (only if W > 0)               otherwise,
//   g1 = sqrt(W * Ndd), g2 = W / (2 a_min) + a_min * Ndd / 2, W = Nrr - n * T.
// Every float step rounds toward -inf, so the computed threshold never exceeds the true
// one: the filter can only keep extra candidates, never drop the winner.  A flat domain
// (Ndd == 0) always has qalfa == 0 (sum == sum0); giving it Ndd = +huge makes the same
// formula prune it exactly when that is valid.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mars {

struct FitParams {
    double max_alfa;
    uint32_t bits_alfa, bits_beta;
    float a_min;       // smallest nonzero alfa2, max_alfa / 2^bits_alfa, rounded down
    float a_half;      // a_min / 2 (exact)
    float two_a;       // 2 * a_min (exact)
    double eta_per_n;  // 1e-6 * (1 + max_alfa)^2
};

struct FitResult {
    uint32_t qalfa, qbeta;
    double sum, rms;
};

__device__ __forceinline__ uint32_t quantise_exact(double x, uint32_t max) {
    double y = trunc(__dadd_rn(0.5, x));
    if (isnan(y)) return 0u;
    if (y < 0.0) y = 0.0;
    if (y > (double)max) y = (double)max;
    return (uint32_t)y;
}

// fit_f64 with the reference's operation order (encode.rs:247-289).
__device__ __forceinline__ FitResult fit_exact(int64_t s0i, int64_t s1_x4, int64_t s2_x16,
                                               int64_t t0i, int64_t t1_x4, int64_t t2i,
                                               const FitParams& fp) {
    const double s0 = (double)s0i;
    const double s1 = __dmul_rn((double)s1_x4, 0.25);     // == / 4.0 (exact scaling)
    const double s2 = __dmul_rn((double)s2_x16, 0.0625);  // == / 16.0
    const double t0 = (double)t0i;
    const double t1 = __dmul_rn((double)t1_x4, 0.25);
    const double t2 = (double)t2i;

    const double det = __dsub_rn(__dmul_rn(s0, s2), __dmul_rn(s1, s1));
    double alfa = 0.0;
    if (det != 0.0) alfa = __ddiv_rn(__dsub_rn(__dmul_rn(s0, t1), __dmul_rn(s1, t0)), det);
    if (alfa < 0.0) alfa = 0.0;

    const double qscale = (double)(1u << fp.bits_alfa);
    const uint32_t max_qalfa = (1u << fp.bits_alfa) - 1u;
    FitResult r;
    r.qalfa = quantise_exact(__dmul_rn(__ddiv_rn(alfa, fp.max_alfa), qscale), max_qalfa);
    const double alfa2 = __dmul_rn(__ddiv_rn((double)r.qalfa, qscale), fp.max_alfa);

    double beta = __ddiv_rn(__dsub_rn(t0, __dmul_rn(alfa2, s1)), s0);
    if (alfa2 > 0.0) beta = __dadd_rn(beta, __dmul_rn(alfa2, 255.0));
    const uint32_t max_qbeta = (1u << fp.bits_beta) - 1u;
    const double span = __dmul_rn(__dadd_rn(1.0, fabs(alfa2)), 255.0);
    r.qbeta = quantise_exact(__dmul_rn(__ddiv_rn(beta, span), (double)max_qbeta), max_qbeta);
    double beta2 = __dmul_rn(__ddiv_rn((double)r.qbeta, (double)max_qbeta), span);
    if (alfa2 > 0.0) beta2 = __dsub_rn(beta2, __dmul_rn(alfa2, 255.0));

    // t2 - 2*alfa2*t1 - 2*beta2*t0 + alfa2*alfa2*s2 + 2*alfa2*beta2*s1 + s0*beta2*beta2,
    // evaluated left to right with each product left-associated, as Rust does.
    double x = __dsub_rn(t2, __dmul_rn(__dmul_rn(2.0, alfa2), t1));
    x = __dsub_rn(x, __dmul_rn(__dmul_rn(2.0, beta2), t0));
    x = __dadd_rn(x, __dmul_rn(__dmul_rn(alfa2, alfa2), s2));
    x = __dadd_rn(x, __dmul_rn(__dmul_rn(__dmul_rn(2.0, alfa2), beta2), s1));
    x = __dadd_rn(x, __dmul_rn(__dmul_rn(s0, beta2), beta2));
    r.sum = x;
    double q = __ddiv_rn(x, s0);
    if (!(q >= 0.0)) q = 0.0;
    r.rms = __dsqrt_rn(q);
    return r;
}

// Per-range pruning state derived from the current champion c.
//   mode 2: rms0 > rms_c      -- every qalfa == 0 candidate is strictly worse: Z-form.
//   mode 1: rms0 == rms_c     -- a qalfa == 0 candidate ties; it loses only when it comes
//                                later in reference order, i.e. at a domain > tie_dom.
//   mode 0: rms0 < rms_c      -- only the LB_any form is valid (and only when W > 0).
struct Threshold {
    float w2a;         // W / (2 a_min), rounded down
    float sqrt_w;      // sqrt(max(W, 0)), rounded down
    int32_t mode;
    int32_t wpos;      // W > 0
    uint32_t tie_dom;  // champion's domain index (mode 1)
};

__device__ __forceinline__ Threshold make_threshold(double champ_sum, double champ_rms,
                                                    uint32_t champ_dom, double rms0, int64_t nrr,
                                                    int32_t n, const FitParams& fp) {
    Threshold t;
    const double eta = fp.eta_per_n * (double)n;
    // Two etas: one is the rounding allowance above, the other absorbs the rounding of W.
    const double w = (double)nrr - (double)n * (champ_sum + 2.0 * eta);
    const float wf = __double2float_rd(w);
    t.w2a = __fdiv_rd(wf, fp.two_a);
    t.wpos = wf > 0.0f;
    t.sqrt_w = t.wpos ? __fsqrt_rd(wf) : 0.0f;
    t.mode = rms0 > champ_rms ? 2 : (rms0 == champ_rms ? 1 : 0);
    t.tie_dom = champ_dom;
    return t;
}

// The t1_x4 threshold for one (range, domain) pair: candidates with t1_x4 < result are
// pruned.  s1f = s1_x4 and t0f = t0 are exact in float; detf/sdetf are Ndd and sqrt(Ndd)
// rounded down (or +huge for a flat domain); inv_n = 1/n exactly (n is a power of four).
__device__ __forceinline__ int32_t prune_below(const Threshold& t, uint32_t dom, float s1f,
                                               float t0f, float detf, float sdetf, float inv_n,
                                               const FitParams& fp) {
    const float g1 = __fmul_rd(t.sqrt_w, sdetf);
    float tau;
    if (t.mode == 2 || (t.mode == 1 && dom > t.tie_dom)) {
        const float ad = __fmul_rd(fp.a_min, detf);
        const float g2 = __fadd_rd(t.w2a, __fmul_rd(fp.a_half, detf));
        tau = fminf(g2, fmaxf(g1, ad));
    } else if (t.wpos) {
        tau = g1;
    } else {
        return INT32_MIN;
    }
    const float num = __fadd_rd(__fmul_rd(s1f, t0f), __fmul_rd(4.0f, tau));
    return __float2int_rd(__fmul_rd(num, inv_n));
}

}  // namespace mars
