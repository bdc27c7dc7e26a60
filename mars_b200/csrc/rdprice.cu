// RD pricing of every quadtree node on the device: best_mode_leaf
// (crates/mars-codec/src/encode.rs:1536-1714) for all the nodes walk_rd can visit, one warp
// per node, before the host walk compares leaf and split costs.
//
// The warp runs price::price_node (price.hpp), the code the host walk runs as a team of one
// lane: each DCT output, SSE and bit total is one lane's left-to-right f64 sum in the
// reference's order, and this translation unit is compiled with --fmad=false so no product
// is fused into a sum.  The DCT basis and the rate snapshot's bits come from the host (its
// cosine and log2), so device and host produce the same doubles and the same winners.
//
// Layout: the nodes of one size are one launch; a block holds warps_per_block<N>() warps,
// each with its node's scratch (five f64 and two int32 arrays of N*N) in shared memory, and
// the basis and its transpose staged once per block.  N = 64 does not fit: its warps use
// global scratch slots and stride over the level's nodes.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"
#include "price.hpp"

namespace mars {
namespace {

constexpr uint32_t kScratchBytesPerPixel = 5 * sizeof(double) + 2 * sizeof(int32_t);

template <int N>
__host__ __device__ constexpr uint32_t warps_per_block() {
    return N >= 32 ? 4 : N >= 16 ? 8 : 16;
}
template <int N>
__host__ __device__ constexpr bool shared_scratch() {
    return N <= 32;
}

__device__ price::Scratch carve(unsigned char* p, uint32_t n) {
    double* d = reinterpret_cast<double*>(p);
    int32_t* i = reinterpret_cast<int32_t*>(d + 5 * n);
    return {d, d + n, d + 2 * n, d + 3 * n, d + 4 * n, i, i + n};
}

template <int N>
__global__ void __launch_bounds__(32 * warps_per_block<N>())
    price_nodes_kernel(const uint8_t* __restrict__ px, uint32_t stride, uint32_t count,
                       const uint32_t* __restrict__ rows, const uint32_t* __restrict__ cols,
                       const unsigned char* __restrict__ cands, uint32_t cand_stride,
                       uint32_t k, price::Setup setup,
                       price::RateTable table, const double* __restrict__ basis,
                       price::Priced* __restrict__ out, int8_t* __restrict__ levels,
                       const uint64_t* __restrict__ levels_at, unsigned char* global_scratch) {
    constexpr uint32_t n = (uint32_t)N * N;
    constexpr uint32_t W = warps_per_block<N>();
    extern __shared__ __align__(16) unsigned char smem[];
    double* b = reinterpret_cast<double*>(smem);
    double* bt = b + n;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        b[i] = basis[i];
        bt[(i % N) * N + i / N] = basis[i];
    }
    __syncthreads();
    const uint32_t warp = threadIdx.x / 32;
    const price::Team T{threadIdx.x % 32, 32};
    unsigned char* mine;
    if constexpr (shared_scratch<N>())
        mine = smem + 2 * n * sizeof(double) + (size_t)warp * n * kScratchBytesPerPixel;
    else
        mine = global_scratch + ((size_t)blockIdx.x * W + warp) * n * kScratchBytesPerPixel;
    price::Scratch sc = carve(mine, n);
    constexpr uint32_t sc_class = N == 2 ? 1 : N == 4 ? 2 : N == 8 ? 3 : N == 16 ? 4 : N == 32 ? 5 : 6;
    for (uint32_t node = blockIdx.x * W + warp; node < count; node += gridDim.x * W) {
        const price::Cand* nc =
            reinterpret_cast<const price::Cand*>(cands + (size_t)node * k * cand_stride);
        const price::Priced p = price::price_node(px, stride, rows[node], cols[node], N, nc, k,
                                                  setup, table, b, bt, sc_class, sc, T,
                                                  cand_stride);
        if (T.lane == 0) out[node] = p;
        if (p.has_levels) {
            int8_t* dst = levels + levels_at[node];
            for (uint32_t i = T.lane; i < n; i += 32) dst[i] = (int8_t)sc.best_levels[i];
        }
        __syncwarp();
    }
}

template <int N>
cudaError_t launch_size(const PriceLaunch& a, cudaStream_t st) {
    constexpr uint32_t n = (uint32_t)N * N;
    constexpr uint32_t W = warps_per_block<N>();
    size_t smem = 2 * n * sizeof(double);
    uint32_t blocks = (a.count + W - 1) / W;
    if constexpr (shared_scratch<N>()) {
        smem += (size_t)W * n * kScratchBytesPerPixel;
    } else {
        if (blocks > a.scratch_slots / W) blocks = a.scratch_slots / W;
        if (blocks == 0 || !a.global_scratch) return cudaErrorInvalidValue;
    }
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(
            price_nodes_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    price_nodes_kernel<N><<<blocks, 32 * W, smem, st>>>(
        a.px, a.stride, a.count, a.rows, a.cols,
        reinterpret_cast<const unsigned char*>(a.cands),
        a.cand_stride ? a.cand_stride : (uint32_t)sizeof(price::Cand), a.k, a.setup, a.table, a.basis,
        a.out, a.levels, a.levels_at, a.global_scratch);
    return cudaGetLastError();
}

}  // namespace

size_t price_scratch_bytes(uint32_t size, uint32_t count, uint32_t* slots) {
    if (size <= 32) {
        *slots = 0;
        return 0;
    }
    const uint32_t W = warps_per_block<64>();
    uint32_t s = 148 * 2 * W;
    if (s > ((count + W - 1) / W) * W) s = ((count + W - 1) / W) * W;
    *slots = s;
    return (size_t)s * size * size * kScratchBytesPerPixel;
}

cudaError_t launch_price_nodes(const PriceLaunch& a, cudaStream_t st) {
    if (a.count == 0) return cudaSuccess;
    switch (a.size) {
        case 2: return launch_size<2>(a, st);
        case 4: return launch_size<4>(a, st);
        case 8: return launch_size<8>(a, st);
        case 16: return launch_size<16>(a, st);
        case 32: return launch_size<32>(a, st);
        case 64: return launch_size<64>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

// ---------------------------------------------------------------- the walks on the device
//
// The warm-up walk (walk, encode.rs:1330-1435, t_rms = 8 for build_rate_snapshot) and the RD
// walk's decisions (walk_rd / split_rd, encode.rs:1865-2027) over a search plan's nodes, so
// the host touches only the leaves that come out.  Nodes are in the plan's order (one level
// per size, each in walk order); child[4 i + q] names node i's children TL, BL, TR, BR, -1
// below min_size.  Bottom-up passes (smallest size first) decide and count; a scan over the
// roots and top-down passes (largest first) give every emitted leaf its place in walk order.

namespace {

constexpr uint32_t kNone = 0xffffffffu;

__global__ void warm_bottom_kernel(uint32_t first, uint32_t count, uint32_t size,
                                   uint32_t min_size, double t_rms,
                                   const unsigned char* __restrict__ cands, uint32_t cand_stride,
                                   const int32_t* __restrict__ child,
                                   const uint64_t* __restrict__ evals, uint8_t* __restrict__ split,
                                   uint32_t* __restrict__ cnt, uint64_t* __restrict__ ev) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const uint32_t i = first + t;
    const price::Cand& c = *reinterpret_cast<const price::Cand*>(cands + (size_t)i * cand_stride);
    const double best_rms = c.valid ? c.rms : INFINITY;
    const bool sp = best_rms > t_rms && size > min_size;
    uint32_t n = 1;
    uint64_t e = evals[i];
    if (sp) {
        n = 0;
        for (int q = 0; q < 4; ++q) {
            const int32_t ch = child[4 * (size_t)i + q];
            n += cnt[ch];
            e += ev[ch];
        }
    }
    split[i] = sp ? 1 : 0;
    cnt[i] = n;
    ev[i] = e;
}

// split_rd sums the children's d and r in order from 0.0; leaf_j <= split_j keeps the leaf.
__global__ void rd_bottom_kernel(uint32_t first, uint32_t count, uint32_t size, uint32_t min_size,
                                 double lambda, double split0, double split1,
                                 const price::Priced* __restrict__ priced,
                                 const int32_t* __restrict__ child, uint8_t* __restrict__ split,
                                 double* __restrict__ rd, double* __restrict__ rr,
                                 uint32_t* __restrict__ cnt, uint64_t* __restrict__ res) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const uint32_t i = first + t;
    const price::Priced& p = priced[i];
    const uint64_t own = p.has_levels ? (uint64_t)size * size : 0;
    if (size <= min_size) {
        split[i] = 0;
        rd[i] = p.d;
        rr[i] = p.r;
        cnt[i] = 1;
        res[i] = own;
        return;
    }
    double cd = 0.0, cr = 0.0;
    uint32_t n = 0;
    uint64_t m = 0;
    for (int q = 0; q < 4; ++q) {
        const int32_t ch = child[4 * (size_t)i + q];
        cd += rd[ch];
        cr += rr[ch];
        n += cnt[ch];
        m += res[ch];
    }
    const double leaf_j = p.d + lambda * (p.r + split0);
    const double split_j = cd + lambda * (cr + split1);
    if (leaf_j <= split_j) {
        split[i] = 0;
        rd[i] = p.d;
        rr[i] = p.r + split0;
        cnt[i] = 1;
        res[i] = own;
    } else {
        split[i] = 1;
        rd[i] = cd;
        rr[i] = cr + split1;
        cnt[i] = n;
        res[i] = m;
    }
}

// Exclusive scan over the roots in walk order: ofs_a from cnt, ofs_b (if given) from b;
// totals[0] = sum of cnt, totals[1] = sum of b.  One block.
__global__ void __launch_bounds__(1024)
    roots_scan_kernel(const int32_t* __restrict__ roots, uint32_t nroots,
                      const uint32_t* __restrict__ cnt, const uint64_t* __restrict__ b,
                      uint32_t* __restrict__ ofs_a, uint64_t* __restrict__ ofs_b,
                      unsigned long long* __restrict__ totals) {
    __shared__ unsigned long long sa[1024], sb[1024];
    const uint32_t per = (nroots + blockDim.x - 1) / blockDim.x;
    const uint32_t lo = threadIdx.x * per, hi = min(nroots, lo + per);
    unsigned long long ta = 0, tb = 0;
    for (uint32_t j = lo; j < hi; ++j) {
        ta += cnt[roots[j]];
        tb += b[roots[j]];
    }
    sa[threadIdx.x] = ta;
    sb[threadIdx.x] = tb;
    __syncthreads();
    for (uint32_t o = 1; o < blockDim.x; o <<= 1) {  // inclusive Hillis-Steele scan
        const unsigned long long xa = threadIdx.x >= o ? sa[threadIdx.x - o] : 0ull;
        const unsigned long long xb = threadIdx.x >= o ? sb[threadIdx.x - o] : 0ull;
        __syncthreads();
        sa[threadIdx.x] += xa;
        sb[threadIdx.x] += xb;
        __syncthreads();
    }
    unsigned long long a = sa[threadIdx.x] - ta, bb = sb[threadIdx.x] - tb;
    for (uint32_t j = lo; j < hi; ++j) {
        const int32_t r = roots[j];
        ofs_a[r] = (uint32_t)a;
        if (ofs_b) ofs_b[r] = bb;
        a += cnt[r];
        bb += b[r];
    }
    if (threadIdx.x == blockDim.x - 1) {
        totals[0] = sa[threadIdx.x];
        totals[1] = sb[threadIdx.x];
    }
}

// The warm-up leaf of an emitted node (walk's leaf branch).
__global__ void warm_topdown_kernel(uint32_t first, uint32_t count, uint32_t size,
                                    const WalkPlan w, const unsigned char* __restrict__ cands,
                                    uint32_t cand_stride, const uint8_t* __restrict__ split,
                                    const uint32_t* __restrict__ cnt, uint32_t* __restrict__ ofs,
                                    uint32_t zero_threshold, uint32_t bits_beta,
                                    mars_leaf* __restrict__ out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const uint32_t i = first + t;
    const uint32_t o = ofs[i];
    if (o == kNone) return;
    if (split[i]) {
        uint32_t acc = o;
        for (int q = 0; q < 4; ++q) {
            const int32_t ch = w.child[4 * (size_t)i + q];
            ofs[ch] = acc;
            acc += cnt[ch];
        }
        return;
    }
    const price::Cand& c = *reinterpret_cast<const price::Cand*>(cands + (size_t)i * cand_stride);
    const uint32_t row = w.rows[i], col = w.cols[i];
    mars_leaf l = price::make_leaf(row, col, size);
    if (c.valid) {
        l.mode = 2;
        l.qalfa = c.qalfa;
        l.qbeta = c.qbeta;
        l.isometry = c.isometry;
        l.dom_row = c.dom_row;
        l.dom_col = c.dom_col;
    }
    if (l.qalfa <= zero_threshold) {
        int64_t sum = 0;
        for (uint32_t r = 0; r < size; ++r)
            for (uint32_t q = 0; q < size; ++q) sum += w.px[(size_t)(row + r) * w.stride + col + q];
        l = price::make_leaf(row, col, size);
        l.qbeta = price::best_beta(sum, (int64_t)size * size, bits_beta);
    }
    out[o] = l;
}

// The RD walk's leaf of an emitted node and its mode-3 levels (as int32).
__global__ void rd_topdown_kernel(uint32_t first, uint32_t count, uint32_t size,
                                  const WalkPlan w, const price::Priced* __restrict__ priced,
                                  const int8_t* __restrict__ levels,
                                  const uint8_t* __restrict__ split,
                                  const uint32_t* __restrict__ cnt,
                                  const uint64_t* __restrict__ res, uint32_t* __restrict__ ofs,
                                  uint64_t* __restrict__ rofs, mars_leaf* __restrict__ out,
                                  int32_t* __restrict__ out_res) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const uint32_t i = first + t;
    const uint32_t o = ofs[i];
    if (o == kNone) return;
    if (split[i]) {
        uint32_t acc = o;
        uint64_t racc = rofs[i];
        for (int q = 0; q < 4; ++q) {
            const int32_t ch = w.child[4 * (size_t)i + q];
            ofs[ch] = acc;
            rofs[ch] = racc;
            acc += cnt[ch];
            racc += res[ch];
        }
        return;
    }
    const price::Priced& p = priced[i];
    out[o] = p.leaf;
    if (p.has_levels) {
        const int8_t* src = levels + w.levels_at[i];
        int32_t* dst = out_res + rofs[i];
        for (uint32_t k = 0; k < size * size; ++k) dst[k] = src[k];
    }
}

uint32_t blocks_for(uint32_t n) { return (n + 255) / 256; }

}  // namespace

cudaError_t launch_warm_walk(const WalkPlan& w, const void* cands, uint32_t cand_stride,
                             double t_rms, uint32_t min_size, uint32_t zero_threshold,
                             uint32_t bits_beta, WalkScratch& s, mars_leaf* out,
                             cudaStream_t st) {
    const unsigned char* cb = reinterpret_cast<const unsigned char*>(cands);
    for (uint32_t L = 0; L < w.nlevels; ++L)  // smallest size first
        if (w.count[L])
            warm_bottom_kernel<<<blocks_for(w.count[L]), 256, 0, st>>>(
                w.first[L], w.count[L], w.size[L], min_size, t_rms, cb, cand_stride, w.child,
                w.evals, s.split, s.cnt, s.ev);
    cudaError_t e = cudaMemsetAsync(s.ofs, 0xff, (size_t)w.nodes * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    roots_scan_kernel<<<1, 1024, 0, st>>>(w.roots, w.nroots, s.cnt, s.ev, s.ofs, nullptr, s.totals);
    for (uint32_t L = w.nlevels; L-- > 0;)
        if (w.count[L])
            warm_topdown_kernel<<<blocks_for(w.count[L]), 256, 0, st>>>(
                w.first[L], w.count[L], w.size[L], w, cb, cand_stride, s.split, s.cnt, s.ofs,
                zero_threshold, bits_beta, out);
    return cudaGetLastError();
}

cudaError_t launch_rd_walk(const WalkPlan& w, const price::Priced* priced, const int8_t* levels,
                           double lambda, const double* split0, const double* split1,
                           uint32_t min_size, WalkScratch& s, mars_leaf* out, int32_t* out_res,
                           cudaStream_t st) {
    for (uint32_t L = 0; L < w.nlevels; ++L) {
        if (!w.count[L]) continue;
        const uint32_t sc = (uint32_t)__builtin_ctz(w.size[L]);
        rd_bottom_kernel<<<blocks_for(w.count[L]), 256, 0, st>>>(
            w.first[L], w.count[L], w.size[L], min_size, lambda, split0[sc], split1[sc], priced,
            w.child, s.split, s.rd, s.rr, s.cnt, s.ev);
    }
    cudaError_t e = cudaMemsetAsync(s.ofs, 0xff, (size_t)w.nodes * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    roots_scan_kernel<<<1, 1024, 0, st>>>(w.roots, w.nroots, s.cnt, s.ev, s.ofs, s.rofs, s.totals);
    for (uint32_t L = w.nlevels; L-- > 0;)
        if (w.count[L])
            rd_topdown_kernel<<<blocks_for(w.count[L]), 256, 0, st>>>(
                w.first[L], w.count[L], w.size[L], w, priced, levels, s.split, s.cnt, s.ev,
                s.ofs, s.rofs, out, out_res);
    return cudaGetLastError();
}

}  // namespace mars
