// Fixed-point decode iteration as a gather: one thread per output pixel.
//
// decode_step / decode_leaf (crates/mars-codec/src/ifs.rs:299-309, 406-484) scatter each
// leaf's (u, v) domain samples to range positions (i, j) = map(iso, u, v).  Every output
// pixel belongs to exactly one leaf, so the same map is computed here as a gather: the
// thread for pixel (y, x) finds its leaf through a per-pixel leaf index, inverts the
// isometry to get (u, v), reads the 2x2 domain block of the previous iterate and applies
// the leaf's affine map with the reference's f64 association, (0.5 + d*alfa) + beta.
// Pixels no leaf covers are written 0, as the reference's zero-filled `next` buffer is.
#include "kernels.cuh"

namespace mars {
namespace {

// Inverse of isometry::map (isometry.rs:7-19): the (u, v) whose image is (i, j).
__device__ __forceinline__ void iso_inverse(uint32_t k, int i, int j, int S, int* u, int* v) {
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

__global__ void decode_step_kernel(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst,
                                   int w, int h, const int32_t* __restrict__ leaf_of_pixel,
                                   const DecodeLeaf* __restrict__ leaves) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= w || y >= h) return;
    const size_t o = (size_t)y * w + x;
    const int32_t li = leaf_of_pixel[o];
    if (li < 0) {
        dst[o] = 0;
        return;
    }
    const DecodeLeaf L = leaves[li];
    const int i = y - (int)L.row, j = x - (int)L.col;
    double value;
    if (L.mode == 1) {
        // Mode 1: round(b0 + gx*u + gy*v) with (u, v) = (i, j) (ifs.rs:416-431).
        // f64::round: half away from zero, as CUDA's round().
        value = round(__dadd_rn(__dadd_rn(L.alfa, __dmul_rn(L.gx, (double)i)),
                                __dmul_rn(L.gy, (double)j)));
    } else {
        double d = 0.0;
        if (L.qalfa != 0) {
            int u, v;
            iso_inverse(L.iso, i, j, (int)L.size, &u, &v);
            const size_t dr = L.dom_row + 2 * u, dc = L.dom_col + 2 * v;
            const double p00 = src[dr * w + dc], p10 = src[(dr + 1) * w + dc];
            const double p01 = src[dr * w + dc + 1], p11 = src[(dr + 1) * w + dc + 1];
            d = __dmul_rn(__dadd_rn(__dadd_rn(__dadd_rn(p00, p10), p01), p11), 0.25);
        }
        value = __dadd_rn(__dadd_rn(0.5, __dmul_rn(d, L.alfa)), L.beta);
    }
    if (!(value >= 0.0)) value = 0.0;
    if (value > 255.0) value = 255.0;
    dst[o] = (uint8_t)value;
}

}  // namespace

cudaError_t launch_decode_step(const uint8_t* src, uint8_t* dst, int w, int h,
                               const int32_t* leaf_of_pixel, const DecodeLeaf* leaves,
                               cudaStream_t st) {
    dim3 grid((w + 255) / 256, h);
    decode_step_kernel<<<grid, 256, 0, st>>>(src, dst, w, h, leaf_of_pixel, leaves);
    return cudaGetLastError();
}

}  // namespace mars
