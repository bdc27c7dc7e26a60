// Exhaustive domain-range block search for one quadtree level (one block size s and one
// domain stride), sm_100a.
//
// Data flow per level (all device-resident, one stream):
//   contract      : D(r, c) = 2x2 box sum of the plane          (Contracted::build,
//                   crates/mars-codec/src/encode.rs:478-502)
//   domain_stats  : per domain position, exact s1_x4 = sum D, s2_x16 = sum D^2 and the
//                   rounded-down Ndd / sqrt(Ndd) the pruning bound needs
//                   (domain_sums, encode.rs:800-802)
//   range_stats   : per range block t0, t2, Nrr and the domain-independent qalfa == 0 fit
//   search        : per (range block, domain tile) the 8 isometry correlations
//                   t1_x4 = sum range[map(k,u,v)] * D[u][v] (cross_term_permuted,
//                   encode.rs:849-864), the exact-bound filter of fit.cuh, and the exact f64
//                   fit of every survivor; keeps the tile champion under the reference's
//                   strict-< / encounter-order rule (retain_top_k, encode.rs:676-685)
//   reduce        : per range block, the champion over tiles by (rms, reference index).
#include <algorithm>
#include <cfloat>
#include <climits>

#include "kernels.cuh"

namespace mars {
namespace {

constexpr float kHugeDet = 1.0e30f;
constexpr float kHugeSqrtDet = 1.0e15f;
constexpr int kTileRowsMax = 16;  // domain positions per tile, vertically
constexpr int kTileColsMax = 32;  // and horizontally
constexpr size_t kSmemBudget = 200 * 1024;

// isometry::map (crates/mars-codec/src/isometry.rs:7-19) as a flat range index i*S + j.
__host__ __device__ constexpr int iso_src(int k, int u, int v, int S) {
    return k == 0   ? u * S + v
           : k == 1 ? (S - 1 - v) * S + u
           : k == 2 ? v * S + (S - 1 - u)
           : k == 3 ? (S - 1 - u) * S + (S - 1 - v)
           : k == 4 ? u * S + (S - 1 - v)
           : k == 5 ? (S - 1 - u) * S + v
           : k == 6 ? v * S + u
                    : (S - 1 - v) * S + (S - 1 - u);
}

__global__ void contract_kernel(const uint8_t* __restrict__ plane, int w, int dw, int dh,
                                int32_t* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;
    if (c >= dw || r >= dh) return;
    const uint8_t* p0 = plane + (size_t)(2 * r) * w + 2 * c;
    const uint8_t* p1 = p0 + w;
    out[(size_t)r * dw + c] = (int32_t)p0[0] + (int32_t)p0[1] + (int32_t)p1[0] + (int32_t)p1[1];
}

__device__ __forceinline__ void store_domain_stats(DomainStats& ds, int idx, int64_t n,
                                                   int64_t s1, int64_t s2) {
    const int64_t det16 = n * s2 - s1 * s1;  // 16 * Ndd, exact
    ds.s1x4[idx] = (int32_t)s1;
    ds.s2x16[idx] = s2;
    if (det16 == 0) {
        ds.detf[idx] = kHugeDet;
        ds.sdetf[idx] = kHugeSqrtDet;
    } else {
        const float df = __double2float_rd((double)det16 * 0.0625);
        ds.detf[idx] = df;
        ds.sdetf[idx] = __fsqrt_rd(df);
    }
}

__global__ void domain_stats_kernel(const int32_t* __restrict__ D, LevelGeom g, DomainStats ds) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const int ndom = g.nrow_d * g.ncol_d;
    if (idx >= ndom) return;
    const int a = idx / g.ncol_d, b = idx % g.ncol_d;
    const int32_t* base = D + (size_t)(a * g.step_c) * g.dw + b * g.step_c;
    int64_t s1 = 0, s2 = 0;
    for (int u = 0; u < g.size; ++u) {
        const int32_t* row = base + (size_t)u * g.dw;
        for (int v = 0; v < g.size; ++v) {
            const int64_t d = row[v];
            s1 += d;
            s2 += d * d;
        }
    }
    store_domain_stats(ds, idx, (int64_t)g.size * g.size, s1, s2);
}

// Separable form of the domain statistics for block sizes >= 8: per (domain row, contracted
// column) the sums of D and D^2 over the window's S rows, then per domain the S column sums
// of its window -- S + S loads a domain instead of S^2 (at S = 32 on a 512 x 512 plane
// 40 us of loads become a few).  Integer sums: the results are the direct kernel's.  The
// column sums fit int32: S * 1020^2 < 2^31 for S <= 64.
__global__ void domain_vsum_kernel(const int32_t* __restrict__ D, LevelGeom g,
                                   int32_t* __restrict__ v1, int32_t* __restrict__ v2) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int a = blockIdx.y;
    if (x >= g.dw) return;
    const int32_t* col = D + (size_t)(a * g.step_c) * g.dw + x;
    int32_t s1 = 0, s2 = 0;
    for (int u = 0; u < g.size; ++u) {
        const int32_t d = col[(size_t)u * g.dw];
        s1 += d;
        s2 += d * d;
    }
    v1[(size_t)a * g.dw + x] = s1;
    v2[(size_t)a * g.dw + x] = s2;
}

__global__ void domain_hsum_kernel(const int32_t* __restrict__ v1, const int32_t* __restrict__ v2,
                                   LevelGeom g, DomainStats ds) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const int ndom = g.nrow_d * g.ncol_d;
    if (idx >= ndom) return;
    const int a = idx / g.ncol_d, b = idx % g.ncol_d;
    const int32_t* r1 = v1 + (size_t)a * g.dw + b * g.step_c;
    const int32_t* r2 = v2 + (size_t)a * g.dw + b * g.step_c;
    int64_t s1 = 0, s2 = 0;
    for (int v = 0; v < g.size; ++v) {
        s1 += r1[v];
        s2 += r2[v];
    }
    store_domain_stats(ds, idx, (int64_t)g.size * g.size, s1, s2);
}

__device__ __forceinline__ void store_range_stats(RangeStats& rs, int r, int64_t n, int32_t t0,
                                                  int32_t t2, const FitParams& fp) {
    rs.t0[r] = t0;
    rs.t2[r] = t2;
    rs.nrr[r] = n * (int64_t)t2 - (int64_t)t0 * t0;
    // Any candidate whose fit quantises to qalfa == 0 has exactly this f64 sum: with
    // alfa2 == 0 every domain term of fit_f64 is an exact zero.
    const FitResult f0 = fit_exact(n, 0, 0, t0, 0, t2, fp);
    rs.sum0[r] = f0.sum;
    rs.rms0[r] = f0.rms;
}

__device__ __forceinline__ bool range_outside(const uint32_t* rows, const uint32_t* cols, int r,
                                              int size, int w, int h, RangeStats& rs) {
    if (rows[r] + (uint32_t)size > (uint32_t)h || cols[r] + (uint32_t)size > (uint32_t)w) {
        // A block outside the plane is never read; the search skips it (result invalid).
        rs.t0[r] = 0;
        rs.t2[r] = 0;
        rs.nrr[r] = 0;
        rs.sum0[r] = 0.0;
        rs.rms0[r] = 0.0;
        return true;
    }
    return false;
}

__global__ void range_stats_kernel(const uint8_t* __restrict__ plane, int w, int h,
                                   const uint32_t* __restrict__ rows,
                                   const uint32_t* __restrict__ cols, int nranges, int size,
                                   FitParams fp, RangeStats rs) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nranges) return;
    if (range_outside(rows, cols, r, size, w, h, rs)) return;
    const uint8_t* base = plane + (size_t)rows[r] * w + cols[r];
    int32_t t0 = 0, t2 = 0;
    for (int i = 0; i < size; ++i)
        for (int j = 0; j < size; ++j) {
            const int32_t p = base[(size_t)i * w + j];
            t0 += p;
            t2 += p * p;
        }
    store_range_stats(rs, r, (int64_t)size * size, t0, t2, fp);
}

// Warp-per-range form for block sizes >= 16, where a thread per range leaves the GPU nearly
// idle (256 ranges of 32 x 32 in a 512 x 512 plane: 36 -> 7 us).  The sums are integers, so
// splitting them over lanes changes nothing.  (The domain statistics keep a thread per
// domain: neighbouring domains' windows overlap, so a warp's loads already coalesce.)
__global__ void range_stats_warp_kernel(const uint8_t* __restrict__ plane, int w, int h,
                                        const uint32_t* __restrict__ rows,
                                        const uint32_t* __restrict__ cols, int nranges,
                                        int size, FitParams fp, RangeStats rs) {
    const int r = (int)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= nranges) return;  // the whole warp
    if (rows[r] + (uint32_t)size > (uint32_t)h || cols[r] + (uint32_t)size > (uint32_t)w) {
        if (lane == 0) range_outside(rows, cols, r, size, w, h, rs);
        return;
    }
    const uint8_t* base = plane + (size_t)rows[r] * w + cols[r];
    const int n = size * size, lg = __ffs(size) - 1;
    int32_t t0 = 0, t2 = 0;
    for (int k = lane; k < n; k += 32) {
        const int32_t p = base[(size_t)(k >> lg) * w + (k & (size - 1))];
        t0 += p;
        t2 += p * p;
    }
    for (int o = 16; o; o >>= 1) {
        t0 += __shfl_xor_sync(0xffffffffu, t0, o);
        t2 += __shfl_xor_sync(0xffffffffu, t2, o);
    }
    if (lane == 0) store_range_stats(rs, r, n, t0, t2, fp);
}

// One CTA = RPB range blocks (one per thread) x a strided subset of the domain tiles
// (tile = blockIdx.y, blockIdx.y + gridDim.y, ...).  Per tile the contracted strip and the
// domain statistics are staged in shared memory; every thread correlates its range block
// with each domain of the tile under all 8 isometries, applies the exact-bound filter and
// runs the exact f64 fit on survivors only.
// KMAX = 1 keeps the single champion (search_with_shift); KMAX > 1 keeps the best k <= KMAX
// candidates by (rms, reference index) -- search_top_k's retain_top_k list -- and prunes
// against the k-th once the list is full.  Partials hold k entries per (split, range).
template <int S, int RPB, int KMAX>
__global__ void __launch_bounds__(RPB) search_simt_kernel(
    const int32_t* __restrict__ D, LevelGeom g, const uint8_t* __restrict__ plane, int w,
    const uint32_t* __restrict__ rows, const uint32_t* __restrict__ cols, int nranges,
    RangeStats rs, DomainStats ds, FitParams fp, Partial* __restrict__ partials, int tiles_c,
    int ntiles, int tile_rows, int tile_cols, unsigned long long* __restrict__ exact_counter,
    int k) {
    constexpr int N = S * S;
    constexpr bool kRegs = S <= 8;
    extern __shared__ __align__(16) unsigned char smem[];

    const int step = g.step_c;
    const int strip_ld = (tile_cols - 1) * step + S;
    const int strip_rows_max = (tile_rows - 1) * step + S;
    int32_t* Ds = reinterpret_cast<int32_t*>(smem);
    float* s1s = reinterpret_cast<float*>(Ds + strip_rows_max * strip_ld);
    float* dets = s1s + tile_rows * tile_cols;
    float* sdets = dets + tile_rows * tile_cols;
    uint8_t* Rs = reinterpret_cast<uint8_t*>(sdets + tile_rows * tile_cols);

    const int tid = threadIdx.x;
    const int r = blockIdx.x * RPB + tid;
    const bool active = r < nranges && rows[r] + (uint32_t)S <= (uint32_t)g.h &&
                        cols[r] + (uint32_t)S <= (uint32_t)g.w;
    const bool in_grid = r < nranges;

    int rr[kRegs ? N : 1];
    {
        const uint8_t* base = active ? plane + (size_t)rows[r] * w + cols[r] : nullptr;
        if constexpr (kRegs) {
#pragma unroll
            for (int p = 0; p < N; ++p) rr[p] = active ? base[(size_t)(p / S) * w + (p % S)] : 0;
        } else {
            for (int p = 0; p < N; ++p)
                Rs[p * RPB + tid] = active ? base[(size_t)(p / S) * w + (p % S)] : 0;
        }
    }

    int32_t t0 = 0, t2 = 0;
    int64_t nrr = 0;
    double rms0 = 0.0;
    if (active) {
        t0 = rs.t0[r];
        t2 = rs.t2[r];
        nrr = rs.nrr[r];
        rms0 = rs.rms0[r];
    }
    const float t0f = (float)t0;
    const float inv_n = 1.0f / (float)N;  // exact: N is a power of four
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    double ch_rms[KMAX], ch_sum[KMAX];
    uint32_t ch_idx[KMAX];
    int32_t ch_t1[KMAX];
    uint32_t ch_qa[KMAX], ch_qb[KMAX];
#pragma unroll
    for (int j = 0; j < KMAX; ++j) {
        ch_rms[j] = inf;
        ch_sum[j] = inf;
        ch_idx[j] = UINT32_MAX;
        ch_t1[j] = 0;
        ch_qa[j] = ch_qb[j] = 0;
    }
    const int kk = KMAX == 1 ? 1 : k;  // entries kept; the list is full once ch_idx[kk-1] is set
    // Until the list is full nothing can be pruned: the infinite cut-off below does that.
    Threshold th = make_threshold(inf, inf, UINT32_MAX, rms0, nrr, N, fp);
    unsigned long long exact = 0;

    for (int tile = blockIdx.y; tile < ntiles; tile += gridDim.y) {
        const int a0 = (tile / tiles_c) * tile_rows, b0 = (tile % tiles_c) * tile_cols;
        const int na = min(tile_rows, g.nrow_d - a0), nb = min(tile_cols, g.ncol_d - b0);
        const int strip_h = (na - 1) * step + S, strip_w = (nb - 1) * step + S;
        __syncthreads();
        for (int i = tid; i < strip_h * strip_w; i += RPB) {
            const int y = i / strip_w, x = i % strip_w;
            Ds[y * strip_ld + x] = D[(size_t)(a0 * step + y) * g.dw + b0 * step + x];
        }
        for (int i = tid; i < na * nb; i += RPB) {
            const int da = i / nb, db = i % nb;
            const int dom = (a0 + da) * g.ncol_d + (b0 + db);
            s1s[da * tile_cols + db] = (float)ds.s1x4[dom];
            dets[da * tile_cols + db] = ds.detf[dom];
            sdets[da * tile_cols + db] = ds.sdetf[dom];
        }
        __syncthreads();
        if (!active) continue;

        for (int da = 0; da < na; ++da) {
            for (int db = 0; db < nb; ++db) {
                const int32_t* Dw = Ds + (da * step) * strip_ld + db * step;
                int acc[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) acc[k] = 0;
                if constexpr (kRegs) {
#pragma unroll
                    for (int u = 0; u < S; ++u)
#pragma unroll
                        for (int v = 0; v < S; ++v) {
                            const int d = Dw[u * strip_ld + v];
#pragma unroll
                            for (int k = 0; k < 8; ++k) acc[k] += rr[iso_src(k, u, v, S)] * d;
                        }
                } else {
                    for (int u = 0; u < S; ++u) {
#pragma unroll 4
                        for (int v = 0; v < S; ++v) {
                            const int d = Dw[u * strip_ld + v];
#pragma unroll
                            for (int k = 0; k < 8; ++k)
                                acc[k] += (int)Rs[iso_src(k, u, v, S) * RPB + tid] * d;
                        }
                    }
                }
                const int li = da * tile_cols + db;
                const uint32_t dom = (uint32_t)((a0 + da) * g.ncol_d + (b0 + db));
                const int32_t lim = prune_below(th, dom, s1s[li], t0f, dets[li], sdets[li], inv_n, fp);
                int mx = acc[0];
#pragma unroll
                for (int k = 1; k < 8; ++k) mx = max(mx, acc[k]);
                if (mx < lim) continue;
                const int32_t s1 = ds.s1x4[dom];
                const int64_t s2 = ds.s2x16[dom];
#pragma unroll 1
                for (int k = 0; k < 8; ++k) {
                    if (acc[k] < lim) continue;
                    ++exact;
                    const FitResult f = fit_exact(N, s1, s2, t0, acc[k], t2, fp);
                    const uint32_t idx = dom * 8u + (uint32_t)k;
                    if constexpr (KMAX == 1) {
                        if (f.rms < ch_rms[0] || (f.rms == ch_rms[0] && idx < ch_idx[0])) {
                            ch_rms[0] = f.rms;
                            ch_sum[0] = f.sum;
                            ch_idx[0] = idx;
                            ch_t1[0] = acc[k];
                            ch_qa[0] = f.qalfa;
                            ch_qb[0] = f.qbeta;
                            th = make_threshold(f.sum, f.rms, dom, rms0, nrr, N, fp);
                        }
                    } else {
                        // Sorted insertion by (rms, index); an empty slot holds (inf, MAX).
                        const int last = kk - 1;
                        if (f.rms < ch_rms[last] || (f.rms == ch_rms[last] && idx < ch_idx[last])) {
                            int pos = last;
                            while (pos > 0 && (f.rms < ch_rms[pos - 1] ||
                                               (f.rms == ch_rms[pos - 1] && idx < ch_idx[pos - 1]))) {
                                ch_rms[pos] = ch_rms[pos - 1];
                                ch_sum[pos] = ch_sum[pos - 1];
                                ch_idx[pos] = ch_idx[pos - 1];
                                ch_t1[pos] = ch_t1[pos - 1];
                                ch_qa[pos] = ch_qa[pos - 1];
                                ch_qb[pos] = ch_qb[pos - 1];
                                --pos;
                            }
                            ch_rms[pos] = f.rms;
                            ch_sum[pos] = f.sum;
                            ch_idx[pos] = idx;
                            ch_t1[pos] = acc[k];
                            ch_qa[pos] = f.qalfa;
                            ch_qb[pos] = f.qbeta;
                            if (ch_idx[last] != UINT32_MAX)
                                th = make_threshold(ch_sum[last], ch_rms[last], ch_idx[last] >> 3,
                                                    rms0, nrr, N, fp);
                        }
                    }
                }
            }
        }
    }
    if (!in_grid) return;
#pragma unroll
    for (int j = 0; j < KMAX; ++j) {
        if (j >= kk) break;
        Partial p;
        p.rms = ch_rms[j];
        p.sum = ch_sum[j];
        p.idx = ch_idx[j];
        p.t1x4 = ch_t1[j];
        p.qalfa = (uint16_t)ch_qa[j];
        p.qbeta = (uint16_t)ch_qb[j];
        p.pad = 0;
        partials[((size_t)blockIdx.y * nranges + r) * kk + j] = p;
    }
    if (exact_counter && exact) atomicAdd(exact_counter, exact);
}

__global__ void reduce_kernel(const Partial* __restrict__ partials, int ntiles, int nranges,
                              LevelGeom g, RangeStats rs, DomainStats ds,
                              CandidateOut* __restrict__ out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nranges) return;
    Partial best = partials[r];
    for (int t = 1; t < ntiles; ++t) {
        const Partial p = partials[(size_t)t * nranges + r];
        if (p.rms < best.rms || (p.rms == best.rms && p.idx < best.idx)) best = p;
    }
    CandidateOut c;
    const int64_t n = (int64_t)g.size * g.size;
    if (best.idx == UINT32_MAX) {
        c = CandidateOut{0, 0, 0, 0, 0, 0, 0.0, 0, 0, 0, 0, 0, 0};
    } else {
        const uint32_t dom = best.idx >> 3;
        c.dom_row = (dom / g.ncol_d) * g.shift;
        c.dom_col = (dom % g.ncol_d) * g.shift;
        c.isometry = best.idx & 7u;
        c.qalfa = best.qalfa;
        c.qbeta = best.qbeta;
        c.valid = 1;
        c.rms = best.rms;
        c.s0 = n;
        c.s1_x4 = ds.s1x4[dom];
        c.s2_x16 = ds.s2x16[dom];
        c.t0 = rs.t0[r];
        c.t1_x4 = best.t1x4;
        c.t2 = rs.t2[r];
    }
    out[r] = c;
}

// The best k of each range over the splits' sorted k-lists, by (rms, reference index);
// out holds k candidates per range (valid = 0 past the ranked ones).
__global__ void reduce_topk_kernel(const Partial* __restrict__ partials, int nsplit, int nranges,
                                   int k, LevelGeom g, RangeStats rs, DomainStats ds,
                                   CandidateOut* __restrict__ out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nranges) return;
    const int64_t n = (int64_t)g.size * g.size;
    // Each split's list is sorted, so one cursor per split walks them in merge order.  A
    // candidate in several splits' lists (the tensor-core kernel's splits all start from the
    // same seeds) comes out of the merge once: its copies are adjacent in merge order.
    uint8_t cursor[kMaxTopKSplits];
    for (int t = 0; t < nsplit; ++t) cursor[t] = 0;
    uint32_t last = UINT32_MAX;
    for (int j = 0; j < k;) {
        int bt = -1;
        Partial best;
        best.rms = __longlong_as_double(0x7ff0000000000000ll);
        best.idx = UINT32_MAX;
        for (int t = 0; t < nsplit; ++t) {
            if (cursor[t] >= k) continue;
            const Partial p = partials[((size_t)t * nranges + r) * k + cursor[t]];
            if (p.idx == UINT32_MAX) continue;
            if (bt < 0 || p.rms < best.rms || (p.rms == best.rms && p.idx < best.idx)) {
                best = p;
                bt = t;
            }
        }
        if (bt >= 0 && best.idx == last) {
            ++cursor[bt];
            continue;
        }
        CandidateOut c;
        if (bt < 0) {
            c = CandidateOut{0, 0, 0, 0, 0, 0, 0.0, 0, 0, 0, 0, 0, 0};
        } else {
            ++cursor[bt];
            last = best.idx;
            const uint32_t dom = best.idx >> 3;
            c.dom_row = (dom / g.ncol_d) * g.shift;
            c.dom_col = (dom % g.ncol_d) * g.shift;
            c.isometry = best.idx & 7u;
            c.qalfa = best.qalfa;
            c.qbeta = best.qbeta;
            c.valid = 1;
            c.rms = best.rms;
            c.s0 = n;
            c.s1_x4 = ds.s1x4[dom];
            c.s2_x16 = ds.s2x16[dom];
            c.t0 = rs.t0[r];
            c.t1_x4 = best.t1x4;
            c.t2 = rs.t2[r];
        }
        out[(size_t)r * k + j] = c;
        ++j;
    }
}

int rpb_for(int size) { return size <= 16 ? 64 : (size == 32 ? 32 : 16); }

// Domain tile of the CUDA-core kernel: as large as 16 x 32 positions while the staged
// strip, the per-domain statistics and the range pixels stay within the budget.
void simt_tile(int S, int step, int rpb, int* tr, int* tcn) {
    int r = kTileRowsMax, c = kTileColsMax;
    for (;;) {
        const size_t strip = (size_t)((c - 1) * step + S) * ((r - 1) * step + S) * 4;
        const size_t smem = strip + 3 * (size_t)r * c * 4 + (S > 8 ? (size_t)S * S * rpb : 0);
        if (smem <= kSmemBudget || (r == 1 && c == 1)) break;
        if (c >= r && c > 1) c /= 2; else r /= 2;
    }
    *tr = r;
    *tcn = c;
}

template <int S, int RPB, int KMAX>
cudaError_t launch_simt_t(const int32_t* D, const uint8_t* plane, int w, const uint32_t* rows,
                          const uint32_t* cols, int nranges, const LevelGeom& g, RangeStats rs,
                          DomainStats ds, const FitParams& fp, Partial* partials, int nsplit,
                          unsigned long long* counter, cudaStream_t st, int k) {
    int tr, tcn;
    simt_tile(S, g.step_c, RPB, &tr, &tcn);
    const int tiles_c = (g.ncol_d + tcn - 1) / tcn;
    const int ntiles = ((g.nrow_d + tr - 1) / tr) * tiles_c;
    const int strip_ld = (tcn - 1) * g.step_c + S;
    const int strip_rows = (tr - 1) * g.step_c + S;
    size_t smem = (size_t)strip_ld * strip_rows * 4 + 3 * (size_t)tr * tcn * 4;
    if (S > 8) smem += (size_t)S * S * RPB;
    auto kern = search_simt_kernel<S, RPB, KMAX>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid((nranges + RPB - 1) / RPB, nsplit);
    kern<<<grid, RPB, smem, st>>>(D, g, plane, w, rows, cols, nranges, rs, ds, fp, partials,
                                  tiles_c, ntiles, tr, tcn, counter, k);
    return cudaGetLastError();
}

template <int KMAX>
cudaError_t launch_simt_k(const int32_t* D, const uint8_t* plane, int w, const uint32_t* rows,
                          const uint32_t* cols, int nranges, const LevelGeom& g, RangeStats rs,
                          DomainStats ds, const FitParams& fp, Partial* partials, int nsplit,
                          unsigned long long* counter, cudaStream_t st, int k) {
    switch (g.size) {
        case 2: return launch_simt_t<2, 64, KMAX>(D, plane, w, rows, cols, nranges, g, rs, ds, fp, partials, nsplit, counter, st, k);
        case 4: return launch_simt_t<4, 64, KMAX>(D, plane, w, rows, cols, nranges, g, rs, ds, fp, partials, nsplit, counter, st, k);
        case 8: return launch_simt_t<8, 64, KMAX>(D, plane, w, rows, cols, nranges, g, rs, ds, fp, partials, nsplit, counter, st, k);
        case 16: return launch_simt_t<16, 64, KMAX>(D, plane, w, rows, cols, nranges, g, rs, ds, fp, partials, nsplit, counter, st, k);
        case 32: return launch_simt_t<32, 32, KMAX>(D, plane, w, rows, cols, nranges, g, rs, ds, fp, partials, nsplit, counter, st, k);
        case 64: return launch_simt_t<64, 16, KMAX>(D, plane, w, rows, cols, nranges, g, rs, ds, fp, partials, nsplit, counter, st, k);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t launch_contract(const uint8_t* plane, int w, int h, int32_t* d_out, cudaStream_t st) {
    const int dw = w / 2, dh = h / 2;
    if (dw == 0 || dh == 0) return cudaSuccess;
    dim3 grid((dw + 127) / 128, dh);
    contract_kernel<<<grid, 128, 0, st>>>(plane, w, dw, dh, d_out);
    return cudaGetLastError();
}

size_t domain_stats_tmp_words(const LevelGeom& g) {
    if (g.size < 8 || g.nrow_d <= 0 || g.ncol_d <= 0) return 0;
    return 2 * (size_t)g.nrow_d * (size_t)g.dw;
}

cudaError_t launch_domain_stats(const int32_t* D, const LevelGeom& g, DomainStats ds,
                                cudaStream_t st, int32_t* tmp) {
    const int ndom = g.nrow_d * g.ncol_d;
    if (ndom == 0) return cudaSuccess;
    if (tmp && domain_stats_tmp_words(g) > 0) {
        int32_t* v1 = tmp;
        int32_t* v2 = tmp + (size_t)g.nrow_d * g.dw;
        dim3 grid((g.dw + 255) / 256, g.nrow_d);
        domain_vsum_kernel<<<grid, 256, 0, st>>>(D, g, v1, v2);
        domain_hsum_kernel<<<(ndom + 255) / 256, 256, 0, st>>>(v1, v2, g, ds);
    } else {
        domain_stats_kernel<<<(ndom + 255) / 256, 256, 0, st>>>(D, g, ds);
    }
    return cudaGetLastError();
}

cudaError_t launch_range_stats(const uint8_t* plane, int w, int h, const uint32_t* rows,
                               const uint32_t* cols, int nranges, int size, const FitParams& fp,
                               RangeStats rs, cudaStream_t st) {
    if (nranges == 0) return cudaSuccess;
    if (size >= 16)
        range_stats_warp_kernel<<<(unsigned)(((size_t)nranges * 32 + 255) / 256), 256, 0, st>>>(
            plane, w, h, rows, cols, nranges, size, fp, rs);
    else
        range_stats_kernel<<<(nranges + 127) / 128, 128, 0, st>>>(plane, w, h, rows, cols,
                                                                   nranges, size, fp, rs);
    return cudaGetLastError();
}

int search_simt_tiles(const LevelGeom& g) {
    int tr, tcn;
    simt_tile(g.size, g.step_c, rpb_for(g.size), &tr, &tcn);
    return ((g.nrow_d + tr - 1) / tr) * ((g.ncol_d + tcn - 1) / tcn);
}

int search_simt_splits(const LevelGeom& g, int nranges, int num_sms) {
    const int groups = (nranges + rpb_for(g.size) - 1) / rpb_for(g.size);
    const int want = (num_sms * 16 + groups - 1) / groups;
    return std::max(1, std::min(want, search_simt_tiles(g)));
}

cudaError_t launch_search_simt(const int32_t* D, const uint8_t* plane, int w,
                               const uint32_t* rows, const uint32_t* cols, int nranges,
                               const LevelGeom& g, RangeStats rs, DomainStats ds,
                               const FitParams& fp, Partial* partials, int nsplit,
                               unsigned long long* counter, cudaStream_t st) {
    if (nranges == 0 || g.nrow_d <= 0 || g.ncol_d <= 0) return cudaSuccess;
    return launch_simt_k<1>(D, plane, w, rows, cols, nranges, g, rs, ds, fp, partials, nsplit,
                            counter, st, 1);
}

int search_topk_splits(const LevelGeom& g, int nranges, int num_sms) {
    return std::min(search_simt_splits(g, nranges, num_sms), kMaxTopKSplits);
}

cudaError_t launch_search_topk(const int32_t* D, const uint8_t* plane, int w,
                               const uint32_t* rows, const uint32_t* cols, int nranges,
                               const LevelGeom& g, RangeStats rs, DomainStats ds,
                               const FitParams& fp, int k, Partial* partials, int nsplit,
                               unsigned long long* counter, cudaStream_t st) {
    if (k < 1 || k > kMaxTopK || nsplit > kMaxTopKSplits) return cudaErrorInvalidValue;
    if (nranges == 0 || g.nrow_d <= 0 || g.ncol_d <= 0) return cudaSuccess;
    return launch_simt_k<kMaxTopK>(D, plane, w, rows, cols, nranges, g, rs, ds, fp, partials,
                                   nsplit, counter, st, k);
}

cudaError_t launch_reduce_topk(const Partial* partials, int nsplit, int nranges, int k,
                               const LevelGeom& g, RangeStats rs, DomainStats ds,
                               CandidateOut* out, cudaStream_t st) {
    if (nranges == 0) return cudaSuccess;
    if (k < 1 || k > kMaxTopK || nsplit > kMaxTopKSplits) return cudaErrorInvalidValue;
    reduce_topk_kernel<<<(nranges + 127) / 128, 128, 0, st>>>(partials, nsplit, nranges, k, g,
                                                               rs, ds, out);
    return cudaGetLastError();
}

cudaError_t launch_reduce(const Partial* partials, int ntiles, int nranges, const LevelGeom& g,
                          RangeStats rs, DomainStats ds, CandidateOut* out, cudaStream_t st) {
    if (nranges == 0) return cudaSuccess;
    reduce_kernel<<<(nranges + 127) / 128, 128, 0, st>>>(partials, ntiles, nranges, g, rs, ds, out);
    return cudaGetLastError();
}

}  // namespace mars
