// Attractor refinement: the decode map's fixed point as a differentiable function of the
// leaves' contrast s and offset o.  The reference has no counterpart (its encoder fits each
// leaf to the collage error only); the map refined here is decode_leaf
// (crates/mars-codec/src/ifs.rs:406-484) iterated by decode_iterative (ifs.rs:281-309).
//
// Model.  Reading the decoder's 0.5 + truncation as rounding, a pixel p of leaf L is
//   x_p = clamp(s_L * d_p(x) + o_L (+ r_p), 0, 255),   d_p(x) = mean of the 2x2 domain
// sample at the inverse isometry of p, r_p the mode-3 residual; flat leaves have no d term
// and mode-1 leaves keep their decoded affine value.  The plane solves x* = F(x*; s, o).
// For L = sum_p (x*_p - t_p)^2 against the target t, implicit differentiation gives
//   lambda = g + D^T (S G lambda),  g = 2 (x* - t),
//   dL/ds_L = sum_{p in L} G_p lambda_p d_p(x*),   dL/do_L = sum_{p in L} G_p lambda_p,
// with G_p = 1 where the clamp is inactive and D^T (S G lambda) the transposed, s-weighted,
// 2x2-spread, inverse-isometry scatter-add of the decode map.  The scatter is evaluated as a
// gather: lists built once per leaf list name, for every source pixel q, the output pixels
// whose domain sample covers q, so every adjoint step is deterministic and free of atomics.
// The iterate carried beside lambda is mu_p = G_p s_{L(p)} lambda_p, so one gathered load
// serves each list entry.
//
// Iterates and parameters are f32; reductions (loss, convergence norms, per-leaf gradient
// and curvature sums) are f64 in a fixed order, so results do not depend on scheduling.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "codec.hpp"
#include "context.hpp"
#include "residual.hpp"

namespace {

enum : uint32_t { kRConst = 0, kRAffine = 1, kRDomain = 2 };

struct RefineLeaf {
    uint32_t rc;    // row | col << 16
    uint32_t info;  // size (bits 0-11) | kind (12-13) | isometry (14-16)
    uint32_t dom;   // dom_row | dom_col << 16
    int32_t roff;   // offset of the mode-3 residual in the f32 pool, or -1
    double b0, gx, gy;  // mode-1 leaves
};

constexpr int kBlock = 256;
constexpr int kGradStats = 5;  // per leaf: sum G*lam*d, sum G*lam, sum G*d^2, sum G*d, sum G

// (u, v) = the domain sample that isometry::map (isometry.rs:7-19) sends to (i, j).
__host__ __device__ __forceinline__ void inverse_iso(int k, int S, int i, int j, int* u, int* v) {
    switch (k) {
        case 0: *u = i; *v = j; break;
        case 1: *u = j; *v = S - 1 - i; break;
        case 2: *u = S - 1 - j; *v = i; break;
        case 3: *u = S - 1 - i; *v = S - 1 - j; break;
        case 4: *u = i; *v = S - 1 - j; break;
        case 5: *u = S - 1 - i; *v = j; break;
        case 6: *u = j; *v = i; break;
        default: *u = S - 1 - j; *v = S - 1 - i; break;
    }
}

// Block-wide reduction of one double into part[blockIdx.x] (fixed order).
template <bool use_max>
__device__ __forceinline__ void block_reduce(double v, double* part) {
    __shared__ double sh[kBlock / 32];
    for (int o = 16; o > 0; o >>= 1) {
        const double t = __shfl_xor_sync(0xffffffffu, v, o);
        v = use_max ? fmax(v, t) : v + t;
    }
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = sh[0];
        for (int k = 1; k < kBlock / 32; ++k) a = use_max ? fmax(a, sh[k]) : a + sh[k];
        part[blockIdx.x] = a;
    }
    __syncthreads();
}

// The unclamped model value of pixel (y, xx), its domain mean (0 without a domain), leaf
// and kind (affine for pixels no leaf covers: fixed at 0).
struct PixelModel {
    float v, d;
    int32_t leaf;
    uint32_t kind;
};

__device__ __forceinline__ PixelModel model_at(const float* __restrict__ x, int w, int y, int xx,
                                               int lg, int mw, const int32_t* __restrict__ owner,
                                               const RefineLeaf* __restrict__ leaves,
                                               const float* __restrict__ s,
                                               const float* __restrict__ o,
                                               const float* __restrict__ resid) {
    PixelModel m{0.0f, 0.0f, owner[(size_t)(y >> lg) * mw + (xx >> lg)], kRAffine};
    if (m.leaf < 0) return m;
    const RefineLeaf L = leaves[m.leaf];
    m.kind = (L.info >> 12) & 3u;
    const int i = y - (int)(L.rc & 0xFFFFu), j = xx - (int)(L.rc >> 16);
    if (m.kind == kRAffine) {
        // The decoder's own value (ifs.rs:416-431); these leaves are not refined.
        const double a = round(__dadd_rn(__dadd_rn(L.b0, __dmul_rn(L.gx, (double)i)),
                                         __dmul_rn(L.gy, (double)j)));
        m.v = (float)fmin(fmax(a, 0.0), 255.0);
        return m;
    }
    const int S = (int)(L.info & 0xFFFu);
    int u, vv;
    inverse_iso((int)((L.info >> 14) & 7u), S, i, j, &u, &vv);
    float v = o[m.leaf];
    if (m.kind == kRDomain) {
        const size_t q = ((size_t)(L.dom & 0xFFFFu) + 2 * u) * w + (L.dom >> 16) + 2 * vv;
        m.d = 0.25f * ((x[q] + x[q + 1]) + (x[q + w] + x[q + w + 1]));
        v = fmaf(s[m.leaf], m.d, v);
    }
    // The mode-3 residual, zero-alpha leaves included (ifs.rs:459-479).
    if (L.roff >= 0) v += resid[L.roff + u * S + vv];
    m.v = v;
    return m;
}

// One step x -> xn = F(x); per-block max |xn - x|.
__global__ void __launch_bounds__(kBlock) refine_forward_kernel(
    const float* __restrict__ x, float* __restrict__ xn, int w, int h, int lg, int mw,
    const int32_t* __restrict__ owner, const RefineLeaf* __restrict__ leaves,
    const float* __restrict__ s, const float* __restrict__ o, const float* __restrict__ resid,
    double* __restrict__ part) {
    const size_t n = (size_t)w * h;
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    double change = 0.0;
    if (p < n) {
        const PixelModel m =
            model_at(x, w, (int)(p / w), (int)(p % w), lg, mw, owner, leaves, s, o, resid);
        const float v = fminf(fmaxf(m.v, 0.0f), 255.0f);
        xn[p] = v;
        change = fabs((double)v - (double)x[p]);
    }
    block_reduce<true>(change, part);
}

// The linearisation at x*: d_p, the clamp gate G_p, G_p s_L (domain pixels), g = 2 (x - t);
// per-block sums of (x - t)^2.
__global__ void __launch_bounds__(kBlock) refine_linearise_kernel(
    const float* __restrict__ x, const float* __restrict__ t, int w, int h, int lg, int mw,
    const int32_t* __restrict__ owner, const RefineLeaf* __restrict__ leaves,
    const float* __restrict__ s, const float* __restrict__ o, const float* __restrict__ resid,
    float* __restrict__ dm, float* __restrict__ gate, float* __restrict__ spl,
    float* __restrict__ g, double* __restrict__ part) {
    const size_t n = (size_t)w * h;
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (p < n) {
        const PixelModel m =
            model_at(x, w, (int)(p / w), (int)(p % w), lg, mw, owner, leaves, s, o, resid);
        const bool live = m.kind != kRAffine && m.v >= 0.0f && m.v <= 255.0f;
        dm[p] = m.d;
        gate[p] = live ? 1.0f : 0.0f;
        spl[p] = (live && m.kind == kRDomain) ? s[m.leaf] : 0.0f;
        const float r = x[p] - t[p];
        g[p] = 2.0f * r;
        e = (double)r * (double)r;
    }
    block_reduce<false>(e, part);
}

// mu = spl * lam (the adjoint's warm start after the linearisation changed).
__global__ void refine_mu_kernel(const float* __restrict__ lam, const float* __restrict__ spl,
                                 size_t n, float* __restrict__ mu) {
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) mu[p] = spl[p] * lam[p];
}

// One adjoint step: lamn_q = g_q + 1/4 sum_{e in list(q)} mu[pix_e], mun_q = spl_q lamn_q;
// per-block sums of (lamn - lam)^2 and lamn^2.
__global__ void __launch_bounds__(kBlock) refine_adjoint_kernel(
    const float* __restrict__ lam, const float* __restrict__ mu, float* __restrict__ lamn,
    float* __restrict__ mun, const float* __restrict__ g, const float* __restrict__ spl,
    size_t n, const uint32_t* __restrict__ csr_off, const uint32_t* __restrict__ csr_pix,
    double* __restrict__ part_diff, double* __restrict__ part_norm) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    double dd = 0.0, nn = 0.0;
    if (q < n) {
        float acc = 0.0f;
        const uint32_t e1 = csr_off[q + 1];
        for (uint32_t e = csr_off[q]; e < e1; ++e) acc += mu[csr_pix[e]];
        const float v = fmaf(0.25f, acc, g[q]);
        lamn[q] = v;
        mun[q] = spl[q] * v;
        const double dv = (double)v - (double)lam[q];
        dd = dv * dv;
        nn = (double)v * (double)v;
    }
    block_reduce<false>(dd, part_diff);
    block_reduce<false>(nn, part_norm);
}

// One block: the fixed-order sum (or max) of `n` partials into out[0].
template <bool use_max>
__global__ void __launch_bounds__(kBlock) reduce_parts_kernel(const double* __restrict__ part,
                                                              int n, double* __restrict__ out) {
    __shared__ double sh[kBlock];
    double a = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) a = use_max ? fmax(a, part[k]) : a + part[k];
    sh[threadIdx.x] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = sh[0];
        for (int k = 1; k < kBlock; ++k) r = use_max ? fmax(r, sh[k]) : r + sh[k];
        out[0] = r;
    }
}

// One warp per leaf: the kGradStats sums over the pixels the leaf owns (a later leaf may
// overwrite part of an earlier one), stored leaf-major.
__global__ void refine_grad_kernel(const float* __restrict__ lam, const float* __restrict__ dm,
                                   const float* __restrict__ gate, int w, int lg, int mw,
                                   const int32_t* __restrict__ owner,
                                   const RefineLeaf* __restrict__ leaves, int nleaves,
                                   double* __restrict__ stats) {
    const int li = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (li >= nleaves) return;
    const RefineLeaf L = leaves[li];
    const int S = (int)(L.info & 0xFFFu), r0 = (int)(L.rc & 0xFFFFu), c0 = (int)(L.rc >> 16);
    double acc[kGradStats] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int k = lane; k < S * S; k += 32) {
        const int y = r0 + k / S, x = c0 + k % S;
        if (owner[(size_t)(y >> lg) * mw + (x >> lg)] != li) continue;
        const size_t p = (size_t)y * w + x;
        const double G = gate[p], l = lam[p], d = dm[p];
        acc[0] += G * l * d;
        acc[1] += G * l;
        acc[2] += G * d * d;
        acc[3] += G * d;
        acc[4] += G;
    }
#pragma unroll
    for (int c = 0; c < kGradStats; ++c)
        for (int o = 16; o > 0; o >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
    if (lane == 0)
#pragma unroll
        for (int c = 0; c < kGradStats; ++c) stats[(size_t)li * kGradStats + c] = acc[c];
}

int fail(int code, const std::string& msg) { return mars::set_last_error(code, msg); }

#define RF_CUDA(call)                                                                     \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(MARS_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

}  // namespace

struct mars_refine_plan {
    mars_ctx* ctx = nullptr;
    mars_header hdr{};
    uint32_t w = 0, h = 0;
    int lg = 0, mw = 0;
    size_t nleaves = 0;
    std::vector<mars_leaf> leaves;
    std::vector<int32_t> levels;  // the mode-3 residual levels (kept by refinement)
    std::vector<uint8_t> target;
    std::vector<uint8_t> kind;    // per leaf: kRConst / kRAffine / kRDomain
    std::vector<int32_t> owner_host;  // the owner map (cells of 2^lg pixels)
    std::vector<float> s0, o0;    // the dequantised starting parameters
    int nblocks = 0;
    bool have_forward = false;
    // device
    int32_t* owner = nullptr;
    RefineLeaf* dleaves = nullptr;
    float* resid = nullptr;
    uint32_t* csr_off = nullptr;
    uint32_t* csr_pix = nullptr;
    float* t = nullptr;
    float *x = nullptr, *xn = nullptr;
    float *dm = nullptr, *gate = nullptr, *spl = nullptr, *g = nullptr;
    float *lam = nullptr, *lamn = nullptr, *mu = nullptr, *mun = nullptr;
    float *s = nullptr, *o = nullptr;
    double* stats = nullptr;
    double *part = nullptr, *part2 = nullptr, *red = nullptr;
};

namespace {

void free_plan(mars_refine_plan* p) {
    for (void* q : {(void*)p->owner, (void*)p->dleaves, (void*)p->resid, (void*)p->csr_off,
                    (void*)p->csr_pix, (void*)p->t, (void*)p->x, (void*)p->xn, (void*)p->dm,
                    (void*)p->gate, (void*)p->spl, (void*)p->g, (void*)p->lam, (void*)p->lamn,
                    (void*)p->mu, (void*)p->mun, (void*)p->s, (void*)p->o, (void*)p->stats,
                    (void*)p->part, (void*)p->part2, (void*)p->red})
        cudaFree(q);
    delete p;
}

template <class T>
cudaError_t upload(T** d, const std::vector<T>& v) {
    cudaError_t e = cudaMalloc(d, std::max<size_t>(1, v.size()) * sizeof(T));
    if (e == cudaSuccess && !v.empty())
        e = cudaMemcpy(*d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    return e;
}

double max_alfa_of(const mars_header& hdr) { return (double)hdr.int_max_alfa / 256.0 * 8.0; }

// decode_leaf's dequantisation of modes 0/2/3 (ifs.rs:434-439), in f64.
void dequantise(const mars_header& hdr, const mars_leaf& L, double* alfa, double* beta) {
    *alfa = (double)L.qalfa / (double)(1u << hdr.bits_alfa) * max_alfa_of(hdr);
    *beta = (double)L.qbeta / (double)((1u << hdr.bits_beta) - 1) * ((1.0 + std::fabs(*alfa)) * 255.0);
    if (*alfa > 0.0) *beta -= *alfa * 255.0;
}

// Iterates F until max |x' - x| < tol or max_iters, from the flat-128 seed (warm = false)
// or from the current x; reduces every `chunk` steps.
int run_forward(mars_refine_plan* p, uint32_t max_iters, double tol, bool warm, uint32_t* iters) {
    const cudaStream_t st = p->ctx->stream;
    const size_t n = (size_t)p->w * p->h;
    if (!warm) {
        std::vector<float> seed(n, 128.0f);
        RF_CUDA(cudaMemcpyAsync(p->x, seed.data(), n * 4, cudaMemcpyHostToDevice, st));
        if (int e = mars::ctx_sync(p->ctx)) return e;
    }
    uint32_t it = 0;
    double change = 0.0;
    const uint32_t chunk = 8;
    while (it < max_iters) {
        const uint32_t m = std::min(chunk, max_iters - it);
        for (uint32_t k = 0; k < m; ++k) {
            refine_forward_kernel<<<p->nblocks, kBlock, 0, st>>>(
                p->x, p->xn, (int)p->w, (int)p->h, p->lg, p->mw, p->owner, p->dleaves, p->s, p->o,
                p->resid, p->part);
            std::swap(p->x, p->xn);
        }
        reduce_parts_kernel<true><<<1, kBlock, 0, st>>>(p->part, p->nblocks, p->red);
        p->ctx->launches += m + 1;
        RF_CUDA(cudaGetLastError());
        RF_CUDA(cudaMemcpyAsync(&change, p->red, 8, cudaMemcpyDeviceToHost, st));
        if (int e = mars::ctx_sync(p->ctx)) return e;
        it += m;
        if (change < tol) break;
    }
    *iters = it;
    return MARS_OK;
}

// The linearisation at the current x and the loss there.
int run_linearise(mars_refine_plan* p, double* loss) {
    const cudaStream_t st = p->ctx->stream;
    refine_linearise_kernel<<<p->nblocks, kBlock, 0, st>>>(
        p->x, p->t, (int)p->w, (int)p->h, p->lg, p->mw, p->owner, p->dleaves, p->s, p->o,
        p->resid, p->dm, p->gate, p->spl, p->g, p->part);
    reduce_parts_kernel<false><<<1, kBlock, 0, st>>>(p->part, p->nblocks, p->red);
    p->ctx->launches += 2;
    RF_CUDA(cudaGetLastError());
    RF_CUDA(cudaMemcpyAsync(loss, p->red, 8, cudaMemcpyDeviceToHost, st));
    return mars::ctx_sync(p->ctx);
}

// The adjoint at the last linearisation, from lambda = 0 (warm = false) or from the current
// lambda, until the relative step < tol or max_iters; then the per-leaf statistics.
int run_backward(mars_refine_plan* p, uint32_t max_iters, double tol, bool warm, uint32_t* iters,
                 double* residual) {
    const cudaStream_t st = p->ctx->stream;
    const size_t n = (size_t)p->w * p->h;
    if (warm) {
        refine_mu_kernel<<<p->nblocks, kBlock, 0, st>>>(p->lam, p->spl, n, p->mu);
        p->ctx->launches += 1;
    } else {
        RF_CUDA(cudaMemsetAsync(p->lam, 0, n * 4, st));
        RF_CUDA(cudaMemsetAsync(p->mu, 0, n * 4, st));
    }
    uint32_t it = 0;
    double rel = 0.0;
    double sums[2] = {0.0, 0.0};
    const uint32_t chunk = 8;
    while (it < max_iters) {
        const uint32_t m = std::min(chunk, max_iters - it);
        for (uint32_t k = 0; k < m; ++k) {
            refine_adjoint_kernel<<<p->nblocks, kBlock, 0, st>>>(
                p->lam, p->mu, p->lamn, p->mun, p->g, p->spl, n, p->csr_off, p->csr_pix, p->part,
                p->part2);
            std::swap(p->lam, p->lamn);
            std::swap(p->mu, p->mun);
        }
        reduce_parts_kernel<false><<<1, kBlock, 0, st>>>(p->part, p->nblocks, p->red);
        reduce_parts_kernel<false><<<1, kBlock, 0, st>>>(p->part2, p->nblocks, p->red + 1);
        p->ctx->launches += m + 2;
        RF_CUDA(cudaGetLastError());
        RF_CUDA(cudaMemcpyAsync(sums, p->red, 16, cudaMemcpyDeviceToHost, st));
        if (int e = mars::ctx_sync(p->ctx)) return e;
        it += m;
        rel = sums[1] > 0.0 ? std::sqrt(sums[0] / sums[1]) : 0.0;
        if (rel < tol) break;
    }
    *iters = it;
    *residual = rel;
    if (p->nleaves) {
        const int warps = 4;
        refine_grad_kernel<<<(unsigned)((p->nleaves + warps - 1) / warps), 32 * warps, 0, st>>>(
            p->lam, p->dm, p->gate, (int)p->w, p->lg, p->mw, p->owner, p->dleaves, (int)p->nleaves,
            p->stats);
        p->ctx->launches += 1;
        RF_CUDA(cudaGetLastError());
    }
    return MARS_OK;
}

int upload_params(mars_refine_plan* p, const float* s, const float* o) {
    const cudaStream_t st = p->ctx->stream;
    if (!p->nleaves) return MARS_OK;
    std::vector<float> sv(s, s + p->nleaves), ov(o, o + p->nleaves);
    // Parameters a leaf does not have stay at zero.
    for (size_t k = 0; k < p->nleaves; ++k) {
        if (p->kind[k] != kRDomain) sv[k] = 0.0f;
        if (p->kind[k] == kRAffine) ov[k] = 0.0f;
    }
    RF_CUDA(cudaMemcpyAsync(p->s, sv.data(), p->nleaves * 4, cudaMemcpyHostToDevice, st));
    RF_CUDA(cudaMemcpyAsync(p->o, ov.data(), p->nleaves * 4, cudaMemcpyHostToDevice, st));
    return mars::ctx_sync(p->ctx);
}

int download_stats(mars_refine_plan* p, std::vector<double>* stats) {
    stats->resize(p->nleaves * kGradStats);
    if (!p->nleaves) return MARS_OK;
    RF_CUDA(cudaMemcpyAsync(stats->data(), p->stats, stats->size() * 8, cudaMemcpyDeviceToHost,
                            p->ctx->stream));
    return mars::ctx_sync(p->ctx);
}

double psnr_of(const std::vector<uint8_t>& a, const std::vector<uint8_t>& b) {
    uint64_t sum = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        const int d = (int)a[i] - (int)b[i];
        sum += (uint64_t)(d * d);
    }
    const double mse = (double)sum / (double)a.size();
    return mse > 0.0 ? 10.0 * std::log10(255.0 * 255.0 / mse) : INFINITY;
}

}  // namespace

extern "C" {

int mars_refine_plan_create(mars_ctx* ctx, const mars_header* hdr, const mars_leaf* leaves,
                            size_t n, const int32_t* residuals, size_t nresiduals,
                            const uint8_t* target, mars_refine_plan** out) {
    if (!ctx || !hdr || !target || !out || (n && !leaves)) return fail(MARS_EINVAL, "NULL argument");
    const uint32_t w = hdr->width, h = hdr->height;
    if (w == 0 || h == 0 || w > 65535 || h > 65535)
        return fail(MARS_EINVAL, "plane dimensions must be in 1..65535");
    if (hdr->bits_alfa < 1 || hdr->bits_alfa > 16 || hdr->bits_beta < 1 || hdr->bits_beta > 16)
        return fail(MARS_EINVAL, "header bit widths must be in 1..16");
    if (n > 0x7fffffffull) return fail(MARS_EINVAL, "too many leaves");
    std::vector<int64_t> offs;
    if (!mars::codec::residual_offsets(leaves, n, nresiduals, &offs) || (nresiduals && !residuals))
        return fail(MARS_EINVAL, "the residual pool does not hold size*size levels per mode-3 leaf");
    const size_t npx = (size_t)w * h;
    if (npx * 4 > 0xffffffffull) return fail(MARS_EUNSUPPORTED, "plane too large for the gather lists");
    const uint32_t qalfa_max = 1u << hdr->bits_alfa, qbeta_max = (1u << hdr->bits_beta) - 1;

    std::unique_ptr<mars_refine_plan> p(new (std::nothrow) mars_refine_plan);
    if (!p) return fail(MARS_ENOMEM, "plan allocation failed");
    p->ctx = ctx;
    p->hdr = *hdr;
    p->w = w;
    p->h = h;
    p->nleaves = n;
    p->leaves.assign(leaves, leaves + n);
    p->levels.assign(residuals, residuals + nresiduals);
    p->target.assign(target, target + npx);
    p->kind.resize(n);
    p->s0.assign(n, 0.0f);
    p->o0.assign(n, 0.0f);

    // Leaves, the owner map (the largest power-of-two cell dividing every leaf), residuals.
    uint32_t align_bits = 1u << 15;
    std::vector<RefineLeaf> rl(n);
    std::vector<float> rvals;
    const double step = mars::codec::qstep_of(*hdr);
    for (size_t k = 0; k < n; ++k) {
        const mars_leaf& L = leaves[k];
        const std::string at = "leaf " + std::to_string(k);
        if (L.size == 0 || L.size > 4095 || L.row + L.size > h || L.col + L.size > w ||
            L.isometry > 7 || L.mode > 3)
            return fail(MARS_EINVAL, at + " is invalid for this plane");
        if (L.qbeta > qbeta_max || (L.mode != 1 && L.qalfa > qalfa_max))
            return fail(MARS_EINVAL, at + " has coefficients wider than the header's bits");
        const bool domain = L.mode != 1 && L.qalfa != 0;
        if (domain && (L.dom_row + 2 * L.size > h || L.dom_col + 2 * L.size > w))
            return fail(MARS_EINVAL, at + " domain runs past the plane");
        align_bits |= L.row | L.col | L.size;
        RefineLeaf& r = rl[k];
        r.rc = L.row | (L.col << 16);
        r.dom = L.dom_row | (L.dom_col << 16);
        r.roff = -1;
        r.b0 = r.gx = r.gy = 0.0;
        uint32_t kind;
        if (L.mode == 1) {
            kind = kRAffine;
            r.b0 = (double)L.qbeta / (double)qbeta_max * 255.0;
            r.gx = (double)L.qgx / 64.0;
            r.gy = (double)L.qgy / 64.0;
        } else {
            double alfa, beta;
            dequantise(*hdr, L, &alfa, &beta);
            kind = domain ? kRDomain : kRConst;
            p->s0[k] = domain ? (float)alfa : 0.0f;
            p->o0[k] = (float)beta;
            if (L.mode == 3 && offs[k] >= 0) {
                r.roff = (int32_t)rvals.size();
                for (double v : mars::residual::values(residuals + offs[k], L.size, step))
                    rvals.push_back((float)v);
            }
        }
        p->kind[k] = (uint8_t)kind;
        r.info = L.size | (kind << 12) | (L.isometry << 14);
    }
    p->lg = __builtin_ctz(align_bits);
    const uint32_t cell = 1u << p->lg;
    p->mw = (int)((w + cell - 1) >> p->lg);
    const uint32_t mh = (h + cell - 1) >> p->lg;
    std::vector<int32_t> owner((size_t)p->mw * mh, -1);
    for (size_t k = 0; k < n; ++k) {
        const mars_leaf& L = leaves[k];
        const uint32_t c = L.size >> p->lg;
        for (uint32_t i = 0; i < c; ++i)
            std::fill_n(owner.begin() + (long)((size_t)((L.row >> p->lg) + i) * p->mw + (L.col >> p->lg)),
                        c, (int32_t)k);
    }
    // The gather lists of the transposed domain operator: for every source pixel q, the
    // output pixels whose 2x2 domain sample covers q, in output-pixel order.
    std::vector<uint32_t> off(npx + 1, 0);
    auto for_each_entry = [&](auto&& f) {
        for (uint32_t y = 0; y < h; ++y)
            for (uint32_t x = 0; x < w; ++x) {
                const int32_t li = owner[(size_t)(y >> p->lg) * p->mw + (x >> p->lg)];
                if (li < 0 || p->kind[li] != kRDomain) continue;
                const mars_leaf& L = leaves[li];
                int u, v;
                inverse_iso((int)L.isometry, (int)L.size, (int)(y - L.row), (int)(x - L.col), &u, &v);
                const size_t q = ((size_t)L.dom_row + 2 * u) * w + L.dom_col + 2 * v;
                const uint32_t pp = (uint32_t)((size_t)y * w + x);
                f(q, pp);
                f(q + 1, pp);
                f(q + w, pp);
                f(q + w + 1, pp);
            }
    };
    for_each_entry([&](size_t q, uint32_t) { off[q + 1] += 1; });
    p->owner_host = owner;
    for (size_t q = 0; q < npx; ++q) off[q + 1] += off[q];
    std::vector<uint32_t> pix(off[npx]), fillp(off.begin(), off.end() - 1);
    for_each_entry([&](size_t q, uint32_t pp) { pix[fillp[q]++] = pp; });
    std::vector<float> tf(p->target.begin(), p->target.end());

    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaError_t e = cudaSetDevice(ctx->device);
    p->nblocks = (int)((npx + kBlock - 1) / kBlock);
    if (e == cudaSuccess) e = upload(&p->owner, owner);
    if (e == cudaSuccess) e = upload(&p->dleaves, rl);
    if (e == cudaSuccess) e = upload(&p->resid, rvals);
    if (e == cudaSuccess) e = upload(&p->csr_off, off);
    if (e == cudaSuccess) e = upload(&p->csr_pix, pix);
    if (e == cudaSuccess) e = upload(&p->t, tf);
    for (float** b : {&p->x, &p->xn, &p->dm, &p->gate, &p->spl, &p->g, &p->lam, &p->lamn, &p->mu,
                      &p->mun})
        if (e == cudaSuccess) e = cudaMalloc(b, npx * 4);
    for (float** b : {&p->s, &p->o})
        if (e == cudaSuccess) e = cudaMalloc(b, std::max<size_t>(1, n) * 4);
    if (e == cudaSuccess) e = cudaMalloc(&p->stats, std::max<size_t>(1, n) * kGradStats * 8);
    if (e == cudaSuccess) e = cudaMalloc(&p->part, (size_t)p->nblocks * 8);
    if (e == cudaSuccess) e = cudaMalloc(&p->part2, (size_t)p->nblocks * 8);
    if (e == cudaSuccess) e = cudaMalloc(&p->red, 16);
    if (e != cudaSuccess) {
        free_plan(p.release());
        return fail(MARS_ECUDA, std::string("refine plan: ") + cudaGetErrorString(e));
    }
    *out = p.release();
    return MARS_OK;
}

int mars_refine_params(mars_refine_plan* p, float* s, float* o) {
    if (!p || (p->nleaves && (!s || !o))) return fail(MARS_EINVAL, "NULL argument");
    std::copy(p->s0.begin(), p->s0.end(), s);
    std::copy(p->o0.begin(), p->o0.end(), o);
    return MARS_OK;
}

int mars_refine_forward(mars_refine_plan* p, const float* s, const float* o, uint32_t max_iters,
                        double tol, float* x_out, double* loss, uint32_t* iters) {
    if (!p || !loss || !iters || (p->nleaves && (!s || !o))) return fail(MARS_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(p->ctx->mu);
    RF_CUDA(cudaSetDevice(p->ctx->device));
    p->have_forward = false;
    if (int e = upload_params(p, s, o)) return e;
    if (int e = run_forward(p, max_iters, tol, false, iters)) return e;
    if (int e = run_linearise(p, loss)) return e;
    if (x_out) {
        RF_CUDA(cudaMemcpyAsync(x_out, p->x, (size_t)p->w * p->h * 4, cudaMemcpyDeviceToHost,
                                p->ctx->stream));
        if (int e = mars::ctx_sync(p->ctx)) return e;
    }
    p->have_forward = true;
    return MARS_OK;
}

int mars_refine_backward(mars_refine_plan* p, uint32_t max_iters, double tol, float* grad_s,
                         float* grad_o, uint32_t* iters, double* residual) {
    if (!p || !iters || !residual || (p->nleaves && (!grad_s || !grad_o)))
        return fail(MARS_EINVAL, "NULL argument");
    if (!p->have_forward) return fail(MARS_EINVAL, "mars_refine_forward must run first");
    std::lock_guard<std::mutex> lock(p->ctx->mu);
    RF_CUDA(cudaSetDevice(p->ctx->device));
    if (int e = run_backward(p, max_iters, tol, false, iters, residual)) return e;
    std::vector<double> st;
    if (int e = download_stats(p, &st)) return e;
    for (size_t k = 0; k < p->nleaves; ++k) {
        grad_s[k] = p->kind[k] == kRDomain ? (float)st[k * kGradStats + 0] : 0.0f;
        grad_o[k] = p->kind[k] == kRAffine ? 0.0f : (float)st[k * kGradStats + 1];
    }
    return MARS_OK;
}

int mars_refine_run(mars_refine_plan* p, uint32_t steps, float lr, uint32_t decode_iterations,
                    mars_leaf* out_leaves, mars_refine_report* report) {
    if (!p || !report || (p->nleaves && !out_leaves)) return fail(MARS_EINVAL, "NULL argument");
    if (!(lr > 0.0f) || !(lr <= 1.0f)) return fail(MARS_EINVAL, "lr must be in (0, 1]");
    const size_t n = p->nleaves;
    const mars_header& hdr = p->hdr;
    const double max_alfa = max_alfa_of(hdr);
    const double alfa_unit = max_alfa / (double)(1u << hdr.bits_alfa);
    const uint32_t max_qalfa = (1u << hdr.bits_alfa) - 1, max_qbeta = (1u << hdr.bits_beta) - 1;
    const double s_lo = alfa_unit, s_hi = (double)max_qalfa * alfa_unit;
    const uint32_t kIters = 1000;  // cap on forward and adjoint sweeps per solve
    const int kTries = 8;          // step halvings per gradient step
    const double kMaxDs = 0.25, kMaxShift = 16.0;  // per-leaf trust region of a step
    const int kPasses = 6;         // discrete descent passes on the format grid
    // Progressive re-quantisation: the fractions of the live leaves fixed to the grid in
    // turn (those whose rounding the model prices cheapest first), each followed by
    // kRefixSteps continuous steps of the leaves still free, which absorb the fixed
    // leaves' rounding through the attractor's coupling.
    const double kFixFractions[] = {0.5, 0.75, 0.9};
    const uint32_t kRefixSteps = 3;
    std::memset(report, 0, sizeof *report);

    // decode_leaf's dequantisation (ifs.rs:434-439) of a grid point.
    auto alfa_of = [&](uint32_t qa) { return (double)qa / (double)(1u << hdr.bits_alfa) * max_alfa; };
    auto beta_of = [&](uint32_t qa, uint32_t qb) {
        const double a = alfa_of(qa);
        double b = (double)qb / (double)max_qbeta * ((1.0 + a) * 255.0);
        if (a > 0.0) b -= a * 255.0;
        return b;
    };
    // The grid offset index nearest below / above offset `ot` at contrast index qa.
    auto qbeta_real = [&](uint32_t qa, double ot) {
        const double a = alfa_of(qa);
        return (ot + a * 255.0) / ((1.0 + a) * 255.0) * (double)max_qbeta;
    };
    auto clamp_qb = [&](double q) { return (uint32_t)std::min(std::max(q, 0.0), (double)max_qbeta); };

    std::vector<mars_leaf> grid(p->leaves);  // the current grid point of every leaf
    {
        std::lock_guard<std::mutex> lock(p->ctx->mu);
        RF_CUDA(cudaSetDevice(p->ctx->device));
        p->have_forward = false;
        uint32_t fi = 0, bi = 0;
        double res = 0.0;
        // Loss of (s, o), warm-started from the last solve unless `cold`.
        auto evaluate = [&](const std::vector<float>& sv, const std::vector<float>& ov, bool cold,
                            double* loss) -> int {
            if (int e = upload_params(p, sv.data(), ov.data())) return e;
            if (int e = run_forward(p, kIters, 1e-3, !cold, &fi)) return e;
            return run_linearise(p, loss);
        };
        std::vector<double> st;  // gradient and curvature sums at the last accepted point
        auto gradients = [&](bool cold) -> int {
            if (int e = run_backward(p, kIters, 1e-4, !cold, &bi, &res)) return e;
            return download_stats(p, &st);
        };

        // 1. Continuous steps from the plain search's dequantised parameters.
        std::vector<float> s = p->s0, o = p->o0, ts(n), to(n);
        std::vector<char> fixed(n, 0);  // leaves already put on the grid (phase 1b)
        double loss = 0.0;
        if (int e = evaluate(s, o, true, &loss)) return e;
        if (int e = gradients(true)) return e;
        report->loss_start = loss;
        double step = lr;
        // `count` damped Newton steps of the free leaves; false when a step found no descent.
        auto newton_steps = [&](uint32_t count, uint32_t* taken, int* err) -> bool {
            for (uint32_t it = 0; it < count; ++it) {
                ++*taken;
                bool moved = false;
                for (int tr = 0; tr < kTries && !moved; ++tr, step *= 0.5) {
                    // Per leaf, the damped Newton step of the 2x2 model H = 2 [[sum d^2,
                    // sum d], [sum d, n]] (the curvature without the feedback through the
                    // domains) on the exact gradient.  When s hits its bounds, o takes the
                    // model's optimum for the clamped s, so near-flat domains cannot trade a
                    // clamped s for a runaway o.
                    for (size_t k = 0; k < n; ++k) {
                        ts[k] = s[k];
                        to[k] = o[k];
                        const double* c = &st[k * kGradStats];
                        const double gs = c[0], go = c[1], A = c[2], B = c[3], C = c[4];
                        if (fixed[k] || p->kind[k] == kRAffine || C <= 0.0) continue;
                        double ds = 0.0;
                        if (p->kind[k] == kRDomain) {
                            const double det = A * C - B * B;
                            if (det > 1e-9 * A * C) {
                                double sn = (double)s[k] - step * (C * gs - B * go) / (2.0 * det);
                                sn = std::min(std::max(sn, s_lo), s_hi);
                                ds = sn - (double)s[k];
                            }
                        }
                        // A trust region per leaf: |ds| <= kMaxDs and the leaf's mean value
                        // moves by at most kMaxShift grey levels, so one ill-conditioned leaf
                        // cannot spoil the step of all the others.
                        ds = std::min(std::max(ds, -kMaxDs), kMaxDs);
                        const double sn = (double)s[k] + ds;
                        double dov = -step * go / (2.0 * C) - B / C * ds;
                        const double shift = ds * B / C + dov;
                        dov -= shift - std::min(std::max(shift, -kMaxShift), kMaxShift);
                        const double on = (double)o[k] + dov;
                        // The offsets the header's beta grid can express for this contrast.
                        const double a = p->kind[k] == kRDomain ? sn : 0.0;
                        ts[k] = (float)sn;
                        to[k] = (float)std::min(std::max(on, -a * 255.0), 255.0);
                    }
                    double tl = 0.0;
                    if ((*err = evaluate(ts, to, false, &tl))) return false;
                    if (tl < loss) {
                        loss = tl;
                        s.swap(ts);
                        o.swap(to);
                        moved = true;
                        report->improving_steps += 1;
                    }
                }
                if (!moved) return false;  // no descent along this direction at any damping
                step = std::min((double)lr, step * 4.0);  // undo the last halving, then grow
                // The accepted trial was the last solve: the linearisation is at (s, o).
                if ((*err = gradients(false))) return false;
            }
            return true;
        };
        {
            int err = 0;
            uint32_t taken = 0;
            newton_steps(steps, &taken, &err);
            if (err) return err;
            report->steps = taken;
        }
        report->loss_end = loss;

        // The grid point of leaf k nearest its continuous (s, o) under the quadratic model of
        // the last statistics: qalfa rounded down and up, each with the offset moved to the
        // model's optimum for that alfa, qbeta rounded down and up; domain leaves keep
        // qalfa >= 1.  Returns the model cost of the move (or -1 for a leaf left as it is).
        auto nearest_grid = [&](size_t k, mars_leaf* L) -> double {
            const double* c = &st[k * kGradStats];
            const double A = c[2], B = c[3], C = c[4];
            if (p->kind[k] == kRAffine || C <= 0.0) return -1.0;  // no live pixel
            const bool domain = p->kind[k] == kRDomain;
            const double qs = domain ? (double)s[k] / alfa_unit : 0.0;
            const uint32_t qa_lo = domain ? (uint32_t)std::max(1.0, std::min((double)max_qalfa, std::floor(qs))) : 0;
            const uint32_t qa_hi = domain ? (uint32_t)std::max(1.0, std::min((double)max_qalfa, std::ceil(qs))) : 0;
            double best = INFINITY;
            for (uint32_t qa = qa_lo; qa <= qa_hi; ++qa) {
                const double dsv = domain ? alfa_of(qa) - (double)s[k] : 0.0;
                const double qbf = qbeta_real(qa, (double)o[k] - B / C * dsv);
                for (double qbr : {std::floor(qbf), std::ceil(qbf)}) {
                    const uint32_t qb = clamp_qb(qbr);
                    const double dov = beta_of(qa, qb) - (double)o[k];
                    const double cost = A * dsv * dsv + 2.0 * B * dsv * dov + C * dov * dov;
                    if (cost < best) {
                        best = cost;
                        if (domain) L->qalfa = qa;
                        L->qbeta = qb;
                    }
                }
            }
            return best;
        };

        // 1b. Progressive re-quantisation: fix the cheapest-to-round leaves to their grid
        // points, let the free ones absorb the change, and fix more.
        {
            size_t live = 0;
            for (size_t k = 0; k < n; ++k) live += nearest_grid(k, &grid[k]) >= 0.0 ? 1u : 0u;
            std::vector<std::pair<double, size_t>> order;
            for (double frac : kFixFractions) {
                order.clear();
                size_t nfixed = 0;
                for (size_t k = 0; k < n; ++k) {
                    if (fixed[k]) {
                        ++nfixed;
                        continue;
                    }
                    mars_leaf L = grid[k];
                    const double cost = nearest_grid(k, &L);
                    if (cost >= 0.0) order.push_back({cost, k});
                }
                const size_t want = (size_t)(frac * (double)live);
                if (want <= nfixed || order.empty()) continue;
                std::sort(order.begin(), order.end());
                const size_t add = std::min(order.size(), want - nfixed);
                for (size_t i = 0; i < add; ++i) {
                    const size_t k = order[i].second;
                    nearest_grid(k, &grid[k]);
                    fixed[k] = 1;
                    s[k] = p->kind[k] == kRDomain ? (float)alfa_of(grid[k].qalfa) : 0.0f;
                    o[k] = (float)beta_of(p->kind[k] == kRDomain ? grid[k].qalfa : 0, grid[k].qbeta);
                }
                if (int e = evaluate(s, o, false, &loss)) return e;
                if (int e = gradients(false)) return e;
                int err = 0;
                uint32_t taken = 0;
                step = lr;
                newton_steps(kRefixSteps, &taken, &err);
                if (err) return err;
            }
        }

        // 2. Re-quantisation of the leaves still free, aware of the (s, o) coupling (the
        // model-cheapest grid point around each continuous optimum).
        for (size_t k = 0; k < n; ++k)
            if (!fixed[k]) nearest_grid(k, &grid[k]);

        // 3. Discrete descent on the grid: at the current grid point, the exact gradient and
        // the 2x2 model rank each leaf's neighbouring grid points (qalfa +-1 with the model's
        // best qbeta around it); the predicted improvements are applied together, then to
        // the best half, quarter, ... until the loss falls.
        auto params_of = [&](const std::vector<mars_leaf>& ls, std::vector<float>* sv,
                             std::vector<float>* ov) {
            for (size_t k = 0; k < n; ++k) {
                (*sv)[k] = p->kind[k] == kRDomain ? (float)alfa_of(ls[k].qalfa) : 0.0f;
                (*ov)[k] = p->kind[k] == kRAffine ? 0.0f
                         : (float)beta_of(p->kind[k] == kRDomain ? ls[k].qalfa : 0, ls[k].qbeta);
            }
        };
        std::vector<float> gsv(n), gov(n);
        params_of(grid, &gsv, &gov);
        double gloss = 0.0;
        if (int e = evaluate(gsv, gov, false, &gloss)) return e;
        if (int e = gradients(false)) return e;
        std::vector<std::pair<double, size_t>> gains;
        std::vector<mars_leaf> cand(n), trial;
        for (int pass = 0; pass < kPasses; ++pass) {
            gains.clear();
            for (size_t k = 0; k < n; ++k) {
                cand[k] = grid[k];
                if (p->kind[k] == kRAffine) continue;
                const double* c = &st[k * kGradStats];
                const double gs = c[0], go = c[1], A = c[2], B = c[3], C = c[4];
                if (C <= 0.0) continue;
                const bool domain = p->kind[k] == kRDomain;
                const double s_now = gsv[k], o_now = gov[k];
                const uint32_t qa0 = grid[k].qalfa;
                double best = 0.0;
                for (int da = domain ? -1 : 0; da <= (domain ? 1 : 0); ++da) {
                    const int64_t qa = (int64_t)qa0 + da;
                    if (domain && (qa < 1 || qa > (int64_t)max_qalfa)) continue;
                    const double dsv = domain ? alfa_of((uint32_t)qa) - s_now : 0.0;
                    // The model's best offset for this contrast, then the grid around it.
                    const double ot = o_now - (go + 2.0 * B * dsv) / (2.0 * C);
                    const double qbf = qbeta_real(domain ? (uint32_t)qa : 0, ot);
                    for (double qbr : {std::floor(qbf), std::ceil(qbf)}) {
                        const uint32_t qb = clamp_qb(qbr);
                        const double dov = beta_of(domain ? (uint32_t)qa : 0, qb) - o_now;
                        const double dl = gs * dsv + go * dov + A * dsv * dsv +
                                          2.0 * B * dsv * dov + C * dov * dov;
                        if (dl < best - 1e-9) {
                            best = dl;
                            if (domain) cand[k].qalfa = (uint32_t)qa;
                            cand[k].qbeta = qb;
                        }
                    }
                }
                if (best < 0.0) gains.push_back({best, k});
            }
            if (gains.empty()) break;
            std::sort(gains.begin(), gains.end());
            bool moved = false;
            for (size_t take = gains.size(); take > 0 && !moved; take /= 2) {
                trial = grid;
                for (size_t i = 0; i < take; ++i) trial[gains[i].second] = cand[gains[i].second];
                std::vector<float> tsv(n), tov(n);
                params_of(trial, &tsv, &tov);
                double tl = 0.0;
                if (int e = evaluate(tsv, tov, false, &tl)) return e;
                if (tl < gloss) {
                    gloss = tl;
                    grid.swap(trial);
                    gsv.swap(tsv);
                    gov.swap(tov);
                    moved = true;
                }
                if (take == 1) break;
            }
            if (!moved) break;
            if (int e = gradients(false)) return e;  // the accepted trial was the last solve
        }
    }

    // 4. Exact decodes: the input list, the refined list, and the refined list with every
    // leaf whose own pixels decode worse than in the input list put back; the best of the
    // three is returned, so the plain search result is the fallback.
    const size_t npx = (size_t)p->w * p->h;
    std::vector<uint8_t> plain(npx), ref(npx), mix_img(npx);
    auto decode = [&](const std::vector<mars_leaf>& ls, std::vector<uint8_t>* img) {
        return mars_decode(p->ctx, &hdr, ls.data(), n, p->levels.data(), p->levels.size(),
                           decode_iterations, img->data());
    };
    if (int e = decode(p->leaves, &plain)) return e;
    if (int e = decode(grid, &ref)) return e;
    std::vector<double> sse_plain(n, 0.0), sse_ref(n, 0.0);
    for (uint32_t y = 0; y < p->h; ++y)
        for (uint32_t x = 0; x < p->w; ++x) {
            const int32_t li = p->owner_host[(size_t)(y >> p->lg) * p->mw + (x >> p->lg)];
            if (li < 0) continue;
            const size_t q = (size_t)y * p->w + x;
            const double t = p->target[q];
            sse_plain[li] += ((double)plain[q] - t) * ((double)plain[q] - t);
            sse_ref[li] += ((double)ref[q] - t) * ((double)ref[q] - t);
        }
    std::vector<mars_leaf> mixed(grid);
    for (size_t k = 0; k < n; ++k)
        if (sse_ref[k] > sse_plain[k]) mixed[k] = p->leaves[k];
    if (int e = decode(mixed, &mix_img)) return e;
    const double pp = psnr_of(plain, p->target), pr = psnr_of(ref, p->target),
                 pm = psnr_of(mix_img, p->target);
    const std::vector<mars_leaf>& pick = pm > pr ? mixed : grid;
    const double pbest = std::max(pm, pr);
    report->psnr_plain = pp;
    report->accepted = pbest > pp ? 1u : 0u;
    report->psnr_refined = report->accepted ? pbest : pp;
    const std::vector<mars_leaf>& keep = report->accepted ? pick : p->leaves;
    uint32_t changed = 0;
    for (size_t k = 0; k < n; ++k)
        changed += (keep[k].qalfa != p->leaves[k].qalfa || keep[k].qbeta != p->leaves[k].qbeta) ? 1u : 0u;
    report->changed_leaves = changed;
    std::copy(keep.begin(), keep.end(), out_leaves);
    return MARS_OK;
}

void mars_refine_plan_free(mars_refine_plan* p) {
    if (!p) return;
    cudaSetDevice(p->ctx->device);
    cudaStreamSynchronize(p->ctx->stream);
    free_plan(p);
}

}  // extern "C"
