// Fisher classified search (crates/mars-search/src/{fisher,classify,tables}.rs and the
// shared fit loop search_block_fitted, lib.rs:211-297), on the device.
//
// Indexing (Fisher::index, fisher.rs:30-56): every domain position of a level is classified
// from its s x s window of the contracted plane D.  newclass (classify.rs:94-101) sorts the
// four quadrant sums with the reference's 3-pass descending bubble sort, carrying the index
// permutation, and reads (isometry, class) off the ORDERING row that permutation matches;
// variance_class (classify.rs:106-118) does the same with the quadrant variances
// sum2/n - (sum/n)^2 of the block after `flips` by that isometry.  All quadrant sums and
// sums of squares are exact integers (D <= 1020, pixels <= 255), so the f64 sums the
// reference accumulates are those integers whatever their order: the sums are taken here in
// integer arithmetic, the flip becomes a permutation of the four quadrants, and only the
// variance formula is evaluated in f64, with the reference's operations.  Positions are
// then grouped into the 3 x 24 buckets in raster order (stable), and an empty bucket reads
// the first non-empty one in (class, variance class) order.
//
// Search (Fisher::candidates + search_block_fitted): one warp per range block.  The range
// is classified the same way (on its pixels), its bucket's candidates are fitted lane by
// lane with the exact integer moments and fit_f64, each under the isometry
// MAPPING[range isometry][domain isometry], and the winner is the first minimum rms in
// bucket order (strict `<`); evals = the bucket's length, duplicates included.
#include <cuda_runtime.h>

#include "fisher_common.cuh"
#include "fit.cuh"
#include "kernels.cuh"

namespace mars {
namespace {

__global__ void fisher_classify_domains_kernel(const int32_t* __restrict__ D, int dw, int size,
                                               int shift, int nrow_d, int ncol_d,
                                               uint8_t* __restrict__ key,
                                               uint8_t* __restrict__ diso) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nrow_d * ncol_d) return;
    const int r0 = (p / ncol_d) * shift / 2, c0 = (p % ncol_d) * shift / 2;
    const int h = size / 2;
    int64_t q[4] = {0, 0, 0, 0}, q2[4] = {0, 0, 0, 0};
    for (int u = 0; u < size; ++u) {
        const int32_t* row = D + (size_t)(r0 + u) * dw + c0;
        for (int v = 0; v < size; ++v) {
            const int64_t d = row[v];
            const int k = (u >= h ? 2 : 0) + (v >= h ? 1 : 0);
            q[k] += d;
            q2[k] += d * d;
        }
    }
    int iso, bucket;
    fisher_classify(q, q2, h, &iso, &bucket);
    key[p] = (uint8_t)bucket;
    diso[p] = (uint8_t)iso;
}

// Bucket sizes: block b counts the positions of bucket b.
// Grouping by bucket, a stable counting sort in three kernels.  Keys are bucket numbers
// 0..71; other values are left out.  The keys are cut into chunks of kGroupChunk, each chunk
// taken by one block of 8 warps, each warp a run of kGroupWarpKeys consecutive keys.
constexpr int kGroupChunk = 4096;
constexpr int kGroupWarps = 8;
constexpr int kGroupWarpKeys = kGroupChunk / kGroupWarps;

// Per chunk, the count of each bucket (hist[chunk * 72 + bucket]).  Equal keys of a warp step
// are added once by their lowest lane.
__global__ void __launch_bounds__(32 * kGroupWarps)
    fisher_hist_kernel(const uint8_t* __restrict__ key, int n, uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[72];
    const int lane = threadIdx.x & 31;
    for (int b = threadIdx.x; b < 72; b += blockDim.x) h[b] = 0;
    __syncthreads();
    const int base = blockIdx.x * kGroupChunk;
    for (int i = threadIdx.x; i < kGroupChunk; i += blockDim.x) {
        const int p = base + i;
        const unsigned k = p < n ? key[p] : 255u;
        const unsigned peers = __match_any_sync(0xffffffffu, k);
        if (k < 72 && lane == __ffs(peers) - 1) atomicAdd(&h[k], (uint32_t)__popc(peers));
    }
    __syncthreads();
    for (int b = threadIdx.x; b < 72; b += blockDim.x) hist[(size_t)blockIdx.x * 72 + b] = h[b];
}

// Bucket totals and offsets, the bucket each class reads (itself, or the first non-empty
// one when it is empty), and every chunk's first slot in each bucket (cbase).
__global__ void fisher_scan_kernel(const uint32_t* __restrict__ hist, int nchunks,
                                   uint32_t* __restrict__ counts, uint32_t* __restrict__ offsets,
                                   uint32_t* __restrict__ ref, uint32_t* __restrict__ cbase) {
    __shared__ uint32_t tot[72], offs[72];
    const int b = threadIdx.x;
    if (b < 72) {
        uint32_t t = 0;
        for (int c = 0; c < nchunks; ++c) t += hist[(size_t)c * 72 + b];
        tot[b] = t;
        counts[b] = t;
    }
    __syncthreads();
    if (b == 0) {
        uint32_t off = 0;
        int first = -1;
        for (int bb = 0; bb < 72; ++bb) {
            offs[bb] = off;
            offsets[bb] = off;
            off += tot[bb];
            if (first < 0 && tot[bb] > 0) first = bb;
        }
        for (int bb = 0; bb < 72; ++bb) ref[bb] = tot[bb] > 0 ? bb : (first < 0 ? bb : first);
    }
    __syncthreads();
    if (b < 72) {
        uint32_t run = offs[b];
        for (int c = 0; c < nchunks; ++c) {
            cbase[(size_t)c * 72 + b] = run;
            run += hist[(size_t)c * 72 + b];
        }
    }
}

// Stable scatter: each warp counts its run per bucket, the block turns the counts into
// per-warp first slots, then each warp writes its run's positions in order (the rank among
// equal keys of a step from __match_any_sync).  The result is raster order within a bucket.
__global__ void __launch_bounds__(32 * kGroupWarps)
    fisher_scatter_kernel(const uint8_t* __restrict__ key, int n,
                          const uint32_t* __restrict__ cbase, uint32_t* __restrict__ list) {
    __shared__ uint32_t wh[kGroupWarps][72];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < kGroupWarps * 72; i += blockDim.x) (&wh[0][0])[i] = 0;
    __syncthreads();
    const int w0 = blockIdx.x * kGroupChunk + warp * kGroupWarpKeys;
    for (int s = 0; s < kGroupWarpKeys; s += 32) {
        const int p = w0 + s + lane;
        const unsigned k = p < n ? key[p] : 255u;
        const unsigned peers = __match_any_sync(0xffffffffu, k);
        if (k < 72 && lane == __ffs(peers) - 1) wh[warp][k] += (uint32_t)__popc(peers);
        __syncwarp();
    }
    __syncthreads();
    if (threadIdx.x < 72) {
        const int bk = threadIdx.x;
        uint32_t run = cbase[(size_t)blockIdx.x * 72 + bk];
        for (int w = 0; w < kGroupWarps; ++w) {
            const uint32_t c = wh[w][bk];
            wh[w][bk] = run;
            run += c;
        }
    }
    __syncthreads();
    for (int s = 0; s < kGroupWarpKeys; s += 32) {
        const int p = w0 + s + lane;
        const unsigned k = p < n ? key[p] : 255u;
        const unsigned peers = __match_any_sync(0xffffffffu, k);
        if (k < 72) list[wh[warp][k] + (uint32_t)__popc(peers & ((1u << lane) - 1))] = (uint32_t)p;
        __syncwarp();
        if (k < 72 && lane == __ffs(peers) - 1) wh[warp][k] += (uint32_t)__popc(peers);
        __syncwarp();
    }
}

cudaError_t launch_group(const uint8_t* key, int n, uint32_t* counts, uint32_t* offsets,
                         uint32_t* ref, uint32_t* list, uint32_t* work, cudaStream_t st) {
    const int nchunks = n > 0 ? (n + kGroupChunk - 1) / kGroupChunk : 1;
    uint32_t* hist = work;
    uint32_t* cbase = work + (size_t)nchunks * 72;
    fisher_hist_kernel<<<nchunks, 32 * kGroupWarps, 0, st>>>(key, n, hist);
    fisher_scan_kernel<<<1, 96, 0, st>>>(hist, nchunks, counts, offsets, ref, cbase);
    if (n > 0) fisher_scatter_kernel<<<nchunks, 32 * kGroupWarps, 0, st>>>(key, n, cbase, list);
    return cudaGetLastError();
}

// `wpr` warps per range block (1, or 2 / 4 for the large sizes, whose levels have few
// ranges): warp `sub` of a range takes the bucket candidates e = 32 sub + lane,
// 32 sub + lane + 32 wpr, ...; with wpr > 1 each warp leaves its first minimum in `part`
// and fisher_merge_kernel picks the range's (rms, bucket index) minimum.  Shared memory per
// range: the 8 permuted copies of the range (permute_range, encode.rs:833-842:
// range_k[u*s + v] = range[map(k, u, v)]), built by the range's wpr warps together (wpr
// divides kFisherWarps, so they share a CTA; named barrier 1 + warp / wpr).
constexpr int kFisherWarps = 4;
constexpr uint32_t kNoCandidate = 0xffffffffu;

__global__ void __launch_bounds__(32 * kFisherWarps) fisher_search_kernel(
    const uint8_t* __restrict__ plane, int w, int h, const int32_t* __restrict__ D, int dw,
    int size, int shift, int ncol_d, const uint32_t* __restrict__ rows,
    const uint32_t* __restrict__ cols, int nranges, const uint32_t* __restrict__ counts,
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ ref,
    const uint32_t* __restrict__ list, const uint8_t* __restrict__ diso, FitParams fp, int wpr,
    CandidateOut* __restrict__ out, uint64_t* __restrict__ evals_out,
    CandidateOut* __restrict__ part, uint32_t* __restrict__ part_e) {
    extern __shared__ uint8_t smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gw = blockIdx.x * kFisherWarps + warp;
    const int ri = gw / wpr, sub = gw % wpr;
    if (ri >= nranges) return;
    // Where this warp's answer goes: the range's output, or its slot among the partials.
    CandidateOut* const dst = wpr == 1 ? out + ri : part + (size_t)ri * wpr + sub;
    const int n = size * size, hq = size / 2;
    uint8_t* perm = smem + (size_t)(warp / wpr) * 8 * n;
    const uint32_t row = rows[ri], col = cols[ri];
    CandidateOut res;
    res.dom_row = res.dom_col = res.isometry = res.qalfa = res.qbeta = res.valid = 0;
    res.rms = 0.0;
    res.s0 = res.s1_x4 = res.s2_x16 = res.t0 = res.t1_x4 = res.t2 = 0;
    if (row + size > (uint32_t)h || col + size > (uint32_t)w) {
        // Blocks outside the plane are reported as no candidate and no evals.
        if (lane == 0) {
            *dst = res;
            if (wpr > 1) part_e[(size_t)ri * wpr + sub] = kNoCandidate;
            if (sub == 0) evals_out[ri] = 0;
        }
        return;
    }
    // Range pixels -> quadrant sums and sums of squares, then the 8 permuted copies.
    int64_t q[4] = {0, 0, 0, 0}, q2[4] = {0, 0, 0, 0}, t0 = 0, t2 = 0;
    for (int k = lane; k < n; k += 32) {
        const int i = k / size, j = k % size;
        const int64_t p = plane[(size_t)(row + i) * w + col + j];
        const int qk = (i >= hq ? 2 : 0) + (j >= hq ? 1 : 0);
        q[qk] += p;
        q2[qk] += p * p;
        t0 += p;
        t2 += p * p;
    }
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            q[k] += __shfl_xor_sync(0xffffffffu, q[k], o);
            q2[k] += __shfl_xor_sync(0xffffffffu, q2[k], o);
        }
        t0 += __shfl_xor_sync(0xffffffffu, t0, o);
        t2 += __shfl_xor_sync(0xffffffffu, t2, o);
    }
    for (int e = 32 * sub + lane; e < 8 * n; e += 32 * wpr) {
        const int k = e / n, uv = e % n, u = uv / size, v = uv % size;
        int i, j;
        switch (k) {  // isometry::map (isometry.rs:7-19)
            case 0: i = u; j = v; break;
            case 1: i = size - 1 - v; j = u; break;
            case 2: i = v; j = size - 1 - u; break;
            case 3: i = size - 1 - u; j = size - 1 - v; break;
            case 4: i = u; j = size - 1 - v; break;
            case 5: i = size - 1 - u; j = v; break;
            case 6: i = v; j = u; break;
            default: i = size - 1 - v; j = size - 1 - u; break;
        }
        perm[e] = plane[(size_t)(row + i) * w + col + j];
    }
    // The range's warps returned above together or not at all (same ri), so the group
    // barrier sees all 32 * wpr threads.
    if (wpr > 1)
        asm volatile("bar.sync %0, %1;" ::"r"(1 + warp / wpr), "r"(32 * wpr) : "memory");
    else
        __syncwarp();
    int isom, key;
    fisher_classify(q, q2, hq, &isom, &key);
    const uint32_t b = ref[key];
    const uint32_t len = counts[b], off = offsets[b];

    double best_rms = 0.0;
    uint32_t best_e = 0xffffffffu;
    FitResult best_fit{};
    int64_t best_s1 = 0, best_s2 = 0, best_t1 = 0;
    for (uint32_t e = 32u * sub + lane; e < len; e += 32u * wpr) {
        const uint32_t p = list[off + e];
        const int iso = fisher_mapping(isom, diso[p]);
        const int dr = (int)((p / ncol_d) * shift / 2), dc = (int)((p % ncol_d) * shift / 2);
        const uint8_t* rp = perm + iso * n;
        int64_t s1 = 0, s2 = 0, t1 = 0;
        for (int u = 0; u < size; ++u) {
            const int32_t* drow = D + (size_t)(dr + u) * dw + dc;
            for (int v = 0; v < size; ++v) {
                const int64_t d = drow[v];
                s1 += d;
                s2 += d * d;
                t1 += d * rp[u * size + v];
            }
        }
        const FitResult f = fit_exact(n, s1, s2, t0, t1, t2, fp);
        if (best_e == 0xffffffffu || f.rms < best_rms) {
            best_rms = f.rms;
            best_e = e;
            best_fit = f;
            best_s1 = s1;
            best_s2 = s2;
            best_t1 = t1;
        }
    }
    // First minimum in bucket order: lexicographic (rms, index) over the lanes.
    double r = best_e == 0xffffffffu ? __longlong_as_double(0x7ff0000000000000ll) : best_rms;
    uint32_t ie = best_e;
    for (int o = 16; o > 0; o >>= 1) {
        const double r2 = __shfl_xor_sync(0xffffffffu, r, o);
        const uint32_t e2 = __shfl_xor_sync(0xffffffffu, ie, o);
        if (r2 < r || (r2 == r && e2 < ie)) {
            r = r2;
            ie = e2;
        }
    }
    if (ie != 0xffffffffu && ie == best_e) {
        const uint32_t p = list[off + ie];
        res.dom_row = (p / ncol_d) * shift;
        res.dom_col = (p % ncol_d) * shift;
        res.isometry = fisher_mapping(isom, diso[p]);
        res.qalfa = best_fit.qalfa;
        res.qbeta = best_fit.qbeta;
        res.valid = 1;
        res.rms = best_fit.rms;
        res.s0 = n;
        res.s1_x4 = best_s1;
        res.s2_x16 = best_s2;
        res.t0 = t0;
        res.t1_x4 = best_t1;
        res.t2 = t2;
        *dst = res;
        if (wpr > 1) part_e[(size_t)ri * wpr + sub] = ie;
    } else if (ie == 0xffffffffu && lane == 0) {
        *dst = res;
        if (wpr > 1) part_e[(size_t)ri * wpr + sub] = kNoCandidate;
    }
    if (sub == 0 && lane == 0) evals_out[ri] = len;
}

// The range's answer from its warps' first minima: the smallest rms, then the smallest
// bucket index (the first minimum in bucket order).
__global__ void fisher_merge_kernel(const CandidateOut* __restrict__ part,
                                    const uint32_t* __restrict__ part_e, int wpr, int nranges,
                                    CandidateOut* __restrict__ out) {
    const int ri = blockIdx.x * blockDim.x + threadIdx.x;
    if (ri >= nranges) return;
    int best = -1;
    for (int s = 0; s < wpr; ++s) {
        const uint32_t e = part_e[(size_t)ri * wpr + s];
        if (e == kNoCandidate) continue;
        if (best < 0) {
            best = s;
            continue;
        }
        const double r = part[(size_t)ri * wpr + s].rms, rb = part[(size_t)ri * wpr + best].rms;
        if (r < rb || (r == rb && e < part_e[(size_t)ri * wpr + best])) best = s;
    }
    out[ri] = part[(size_t)ri * wpr + (best < 0 ? 0 : best)];
}

}  // namespace

cudaError_t launch_fisher_index(const int32_t* D, int dw, int size, int shift, int nrow_d,
                                int ncol_d, FisherIndex ix, cudaStream_t st) {
    const int npos = nrow_d * ncol_d;
    if (npos > 0)
        fisher_classify_domains_kernel<<<(npos + 255) / 256, 256, 0, st>>>(
            D, dw, size, shift, nrow_d, ncol_d, ix.key, ix.diso);
    return launch_group(ix.key, npos, ix.counts, ix.offsets, ix.ref, ix.list, ix.work, st);
}

size_t fisher_group_work_words(size_t n) {
    const size_t nchunks = n > 0 ? (n + kGroupChunk - 1) / kGroupChunk : 1;
    return 2 * nchunks * 72;
}

cudaError_t launch_fisher_group(const uint8_t* key, int n, uint32_t* counts, uint32_t* offsets,
                                uint32_t* ref, uint32_t* list, uint32_t* work, cudaStream_t st) {
    return launch_group(key, n, counts, offsets, ref, list, work, st);
}

cudaError_t launch_fisher_search(const uint8_t* plane, int w, int h, const int32_t* D, int dw,
                                 int size, int shift, int ncol_d, const uint32_t* rows,
                                 const uint32_t* cols, int nranges, FisherIndex ix,
                                 const FitParams& fp, CandidateOut* out, uint64_t* evals,
                                 CandidateOut* part, uint32_t* part_e, cudaStream_t st) {
    if (nranges <= 0) return cudaSuccess;
    const int wpr = fisher_warps_per_range(size);
    const size_t smem = (size_t)(kFisherWarps / wpr) * 8 * size * size;
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(
            fisher_search_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const long long warps = (long long)nranges * wpr;
    fisher_search_kernel<<<(unsigned)((warps + kFisherWarps - 1) / kFisherWarps),
                           32 * kFisherWarps, smem, st>>>(
        plane, w, h, D, dw, size, shift, ncol_d, rows, cols, nranges, ix.counts, ix.offsets,
        ix.ref, ix.list, ix.diso, fp, wpr, out, evals, part, part_e);
    if (wpr > 1)
        fisher_merge_kernel<<<(nranges + 127) / 128, 128, 0, st>>>(part, part_e, wpr, nranges,
                                                                   out);
    return cudaGetLastError();
}

int fisher_warps_per_range(int size) { return size >= 16 ? 4 : (size == 8 ? 2 : 1); }

}  // namespace mars
