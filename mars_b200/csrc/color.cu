// Colour input of the codec and the error metric, on the device.
//
//   ycbcr / rgb_from_ycbcr (crates/mars-core/src/metrics.rs:377-460): BT.601 full range in
//     f64, the reference's operations in its order, rounded half away from zero (CUDA's
//     round() is f64::round), clamped to 0..255 and truncated;
//   downsample_box / upsample_nearest (crates/mars-codec/src/color.rs:60-101): 2x2 box mean
//     (sum + 2) / 4 with the last row/column replicated at odd sides, and its nearest-
//     neighbour inverse;
//   mse (metrics.rs:29-48): the exact integer sum of squared differences (u64), divided by
//     the pixel count on the host.
// All are elementwise or small-stencil byte work, so each is bound by HBM; pixels are
// processed four to a thread where the planes are word-aligned.
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.cuh"

namespace mars {
namespace {

__device__ __forceinline__ uint32_t round_u8(double x) {
    double r = round(x);
    if (r < 0.0) r = 0.0;
    if (r > 255.0) r = 255.0;
    return (uint32_t)r;
}

__device__ __forceinline__ void ycc_pixel(uint32_t r8, uint32_t g8, uint32_t b8, uint32_t* y,
                                          uint32_t* cb, uint32_t* cr) {
    const double r = (double)r8, g = (double)g8, b = (double)b8;
    *y = round_u8(__dadd_rn(__dadd_rn(__dmul_rn(0.299, r), __dmul_rn(0.587, g)),
                            __dmul_rn(0.114, b)));
    *cb = round_u8(__dadd_rn(__dsub_rn(__dsub_rn(128.0, __dmul_rn(0.168736, r)),
                                       __dmul_rn(0.331264, g)),
                             __dmul_rn(0.5, b)));
    *cr = round_u8(__dsub_rn(__dsub_rn(__dadd_rn(128.0, __dmul_rn(0.5, r)),
                                       __dmul_rn(0.418688, g)),
                             __dmul_rn(0.081312, b)));
}

__device__ __forceinline__ void rgb_pixel(uint32_t y8, uint32_t cb8, uint32_t cr8, uint32_t* r,
                                          uint32_t* g, uint32_t* b) {
    const double y = (double)y8, cb = (double)cb8 - 128.0, cr = (double)cr8 - 128.0;
    *r = round_u8(__dadd_rn(y, __dmul_rn(1.402, cr)));
    *g = round_u8(__dsub_rn(__dsub_rn(y, __dmul_rn(0.344136, cb)), __dmul_rn(0.714136, cr)));
    *b = round_u8(__dadd_rn(y, __dmul_rn(1.772, cb)));
}

// Three input planes -> three output planes, pixel by pixel; `inverse` picks the direction.
template <bool inverse>
__global__ void convert_kernel(const uint8_t* __restrict__ p0, const uint8_t* __restrict__ p1,
                               const uint8_t* __restrict__ p2, size_t n,
                               uint8_t* __restrict__ q0, uint8_t* __restrict__ q1,
                               uint8_t* __restrict__ q2, bool words) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t i = 4 * t;
    if (i >= n) return;
    if (words && i + 4 <= n) {
        const uint32_t a = *reinterpret_cast<const uint32_t*>(p0 + i);
        const uint32_t b = *reinterpret_cast<const uint32_t*>(p1 + i);
        const uint32_t c = *reinterpret_cast<const uint32_t*>(p2 + i);
        uint32_t o0 = 0, o1 = 0, o2 = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            uint32_t x, y, z;
            const uint32_t s = 8 * k;
            if (inverse) rgb_pixel((a >> s) & 255u, (b >> s) & 255u, (c >> s) & 255u, &x, &y, &z);
            else ycc_pixel((a >> s) & 255u, (b >> s) & 255u, (c >> s) & 255u, &x, &y, &z);
            o0 |= x << s;
            o1 |= y << s;
            o2 |= z << s;
        }
        *reinterpret_cast<uint32_t*>(q0 + i) = o0;
        *reinterpret_cast<uint32_t*>(q1 + i) = o1;
        *reinterpret_cast<uint32_t*>(q2 + i) = o2;
        return;
    }
    for (size_t k = i; k < n && k < i + 4; ++k) {
        uint32_t x, y, z;
        if (inverse) rgb_pixel(p0[k], p1[k], p2[k], &x, &y, &z);
        else ycc_pixel(p0[k], p1[k], p2[k], &x, &y, &z);
        q0[k] = (uint8_t)x;
        q1[k] = (uint8_t)y;
        q2[k] = (uint8_t)z;
    }
}

__global__ void downsample_box_kernel(const uint8_t* __restrict__ src, int w, int h,
                                      uint8_t* __restrict__ dst, int ow, int oh) {
    const int ox = blockIdx.x * blockDim.x + threadIdx.x, oy = blockIdx.y;
    if (ox >= ow || oy >= oh) return;
    const int x0 = 2 * ox, y0 = 2 * oy;
    const int x1 = min(x0 + 1, w - 1), y1 = min(y0 + 1, h - 1);
    const uint32_t sum = (uint32_t)src[(size_t)y0 * w + x0] + src[(size_t)y0 * w + x1] +
                         src[(size_t)y1 * w + x0] + src[(size_t)y1 * w + x1];
    dst[(size_t)oy * ow + ox] = (uint8_t)((sum + 2) / 4);
}

__global__ void upsample_nearest_kernel(const uint8_t* __restrict__ src, int sw, int sh,
                                        uint8_t* __restrict__ dst, int w, int h) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= w || y >= h) return;
    const int sy = min(y / 2, sh - 1), sx = min(x / 2, sw - 1);
    dst[(size_t)y * w + x] = src[(size_t)sy * sw + sx];
}

// Sum of squared differences: per-thread partial sums over 16-byte chunks, a warp and block
// reduction, one 64-bit atomic per block (exact: integers throughout).
__global__ void sse_kernel(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b,
                           size_t n, bool vec, unsigned long long* __restrict__ out) {
    __shared__ unsigned long long part[32];
    unsigned long long acc = 0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (vec) {
        const size_t nv = n / 16;
        for (size_t v = tid; v < nv; v += stride) {
            const uint4 x = reinterpret_cast<const uint4*>(a)[v];
            const uint4 y = reinterpret_cast<const uint4*>(b)[v];
            const uint32_t xs[4] = {x.x, x.y, x.z, x.w}, ys[4] = {y.x, y.y, y.z, y.w};
            uint32_t s = 0;  // 16 squares of at most 65025: fits 32 bits
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int d = (int)((xs[k] >> (8 * j)) & 255u) - (int)((ys[k] >> (8 * j)) & 255u);
                    s += (uint32_t)(d * d);
                }
            acc += s;
        }
        for (size_t i = nv * 16 + tid; i < n; i += stride) {
            const int d = (int)a[i] - (int)b[i];
            acc += (unsigned long long)(d * d);
        }
    } else {
        for (size_t i = tid; i < n; i += stride) {
            const int d = (int)a[i] - (int)b[i];
            acc += (unsigned long long)(d * d);
        }
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) part[warp] = acc;
    __syncthreads();
    if (warp == 0) {
        acc = lane < (int)(blockDim.x >> 5) ? part[lane] : 0ull;
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) atomicAdd(out, acc);
    }
}

}  // namespace

cudaError_t launch_ycbcr(const uint8_t* r, const uint8_t* g, const uint8_t* b, size_t n,
                         uint8_t* y, uint8_t* cb, uint8_t* cr, bool inverse, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const bool words = ((reinterpret_cast<uintptr_t>(r) | reinterpret_cast<uintptr_t>(g) |
                         reinterpret_cast<uintptr_t>(b) | reinterpret_cast<uintptr_t>(y) |
                         reinterpret_cast<uintptr_t>(cb) | reinterpret_cast<uintptr_t>(cr)) &
                        3) == 0;
    const size_t threads = (n + 3) / 4;
    const unsigned blocks = (unsigned)((threads + 255) / 256);
    if (inverse) convert_kernel<true><<<blocks, 256, 0, st>>>(r, g, b, n, y, cb, cr, words);
    else convert_kernel<false><<<blocks, 256, 0, st>>>(r, g, b, n, y, cb, cr, words);
    return cudaGetLastError();
}

cudaError_t launch_downsample_box(const uint8_t* src, int w, int h, uint8_t* dst,
                                  cudaStream_t st) {
    const int ow = (w + 1) / 2, oh = (h + 1) / 2;
    if (ow == 0 || oh == 0) return cudaSuccess;
    downsample_box_kernel<<<dim3((ow + 255) / 256, oh), 256, 0, st>>>(src, w, h, dst, ow, oh);
    return cudaGetLastError();
}

cudaError_t launch_upsample_nearest(const uint8_t* src, int sw, int sh, uint8_t* dst, int w,
                                    int h, cudaStream_t st) {
    if (w == 0 || h == 0) return cudaSuccess;
    upsample_nearest_kernel<<<dim3((w + 255) / 256, h), 256, 0, st>>>(src, sw, sh, dst, w, h);
    return cudaGetLastError();
}

cudaError_t launch_sse(const uint8_t* a, const uint8_t* b, size_t n, int num_sms,
                       unsigned long long* out, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess || n == 0) return e;
    const bool vec = ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 15) == 0;
    const size_t want = (n / 16 + 255) / 256;
    const unsigned blocks = (unsigned)std::max<size_t>(1, std::min<size_t>(want, (size_t)num_sms * 8));
    sse_kernel<<<blocks, 256, 0, st>>>(a, b, n, vec, out);
    return cudaGetLastError();
}

}  // namespace mars
