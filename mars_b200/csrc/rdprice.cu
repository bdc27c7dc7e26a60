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
                       const price::Cand* __restrict__ cands, uint32_t k, price::Setup setup,
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
        const price::Priced p = price::price_node(px, stride, rows[node], cols[node], N,
                                                  cands + (size_t)node * k, k, setup, table, b,
                                                  bt, sc_class, sc, T);
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
        a.px, a.stride, a.count, a.rows, a.cols, a.cands, a.k, a.setup, a.table, a.basis,
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

}  // namespace mars
