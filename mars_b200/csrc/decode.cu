// Fixed-point decode iteration as a gather: each thread produces output pixels.
//
// decode_step / decode_leaf (crates/mars-codec/src/ifs.rs:299-309, 406-484) scatter each
// leaf's (u, v) domain samples to range positions (i, j) = map(iso, u, v).  Every output
// pixel belongs to exactly one leaf, so the same map is computed here as a gather: the
// thread for pixel (y, x) finds its leaf through an owner map kept at the granularity of
// the smallest leaf (cell = 2^lg x 2^lg pixels: one 4-byte entry per 16 pixels for the
// usual 4x4 minimum), inverts the isometry to get (u, v), reads the 2x2 domain block of the
// previous iterate and applies the leaf's affine map with the reference's f64 association,
// (0.5 + d*alfa) + beta.  Leaves are 16 bytes and carry the quantised coefficients; alfa and
// beta are dequantised here with the reference's operations in its order, so the doubles
// are the ones decode_leaf computes.  Pixels no leaf covers are written 0, as the
// reference's zero-filled `next` buffer is.  When cells are at least 4 pixels wide, a thread
// produces 4 consecutive pixels of one leaf and stores them as one word.
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

// A leaf unpacked and dequantised (ifs.rs:416-439).
struct LeafMap {
    double alfa, beta, gx, gy;  // mode 1: alfa holds b0
    int row, col, size, mode, iso, dom_row, dom_col;
    bool domain;                // qalfa != 0: the leaf reads a domain block
};

__device__ __forceinline__ LeafMap unpack(const DecodeLeaf p, const DecodeConsts& c) {
    LeafMap L;
    L.row = (int)(p.x & 0xFFFFu);
    L.col = (int)(p.x >> 16);
    L.size = (int)(p.y & 0xFFFu);
    L.mode = (int)((p.y >> 12) & 3u);
    const double qbeta = (double)(p.y >> 16);
    L.gx = L.gy = 0.0;
    L.iso = 0;
    L.dom_row = L.dom_col = 0;
    L.domain = false;
    if (L.mode == 1) {
        L.alfa = __dmul_rn(__ddiv_rn(qbeta, c.beta_den), 255.0);
        L.beta = 0.0;
        L.gx = __ddiv_rn((double)(int32_t)p.z, 64.0);
        L.gy = __ddiv_rn((double)(int32_t)p.w, 64.0);
    } else {
        const uint32_t qalfa = p.w & 0x1FFFFu;
        L.iso = (int)(p.w >> 24);
        L.dom_row = (int)(p.z & 0xFFFFu);
        L.dom_col = (int)(p.z >> 16);
        L.domain = qalfa != 0;
        L.alfa = __dmul_rn(__ddiv_rn((double)qalfa, c.alfa_den), c.max_alfa);
        L.beta = __dmul_rn(__ddiv_rn(qbeta, c.beta_den),
                           __dmul_rn(__dadd_rn(1.0, fabs(L.alfa)), 255.0));
        if (L.alfa > 0.0) L.beta = __dsub_rn(L.beta, __dmul_rn(L.alfa, 255.0));
    }
    return L;
}

__device__ __forceinline__ uint8_t leaf_pixel(const uint8_t* __restrict__ src, int w,
                                              const LeafMap& L, int y, int x) {
    const int i = y - L.row, j = x - L.col;
    double value;
    if (L.mode == 1) {
        // Mode 1: round(b0 + gx*u + gy*v) with (u, v) = (i, j) (ifs.rs:416-431);
        // f64::round and CUDA's round() both round half away from zero.
        value = round(__dadd_rn(__dadd_rn(L.alfa, __dmul_rn(L.gx, (double)i)),
                                __dmul_rn(L.gy, (double)j)));
    } else {
        double d = 0.0;
        if (L.domain) {
            int u, v;
            iso_inverse(L.iso, i, j, L.size, &u, &v);
            const size_t dr = L.dom_row + 2 * u, dc = L.dom_col + 2 * v;
            const double p00 = src[dr * w + dc], p10 = src[(dr + 1) * w + dc];
            const double p01 = src[dr * w + dc + 1], p11 = src[(dr + 1) * w + dc + 1];
            d = __dmul_rn(__dadd_rn(__dadd_rn(__dadd_rn(p00, p10), p01), p11), 0.25);
        }
        value = __dadd_rn(__dadd_rn(0.5, __dmul_rn(d, L.alfa)), L.beta);
    }
    if (!(value >= 0.0)) value = 0.0;
    if (value > 255.0) value = 255.0;
    return (uint8_t)value;
}

// One pixel per thread (any owner-map granularity).
__global__ void decode_step_kernel(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst,
                                   int w, int h, int lg, int mw,
                                   const int32_t* __restrict__ owner,
                                   const DecodeLeaf* __restrict__ leaves, DecodeConsts c) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= w || y >= h) return;
    const int32_t li = owner[(size_t)(y >> lg) * mw + (x >> lg)];
    uint8_t out = 0;
    if (li >= 0) {
        const LeafMap L = unpack(leaves[li], c);
        out = leaf_pixel(src, w, L, y, x);
    }
    dst[(size_t)y * w + x] = out;
}

// Four consecutive pixels of one owner cell per thread (granularity >= 4, w % 4 == 0).
__global__ void decode_step4_kernel(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst,
                                    int w, int h, int lg, int mw,
                                    const int32_t* __restrict__ owner,
                                    const DecodeLeaf* __restrict__ leaves, DecodeConsts c) {
    const int x = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int y = blockIdx.y;
    if (x >= w || y >= h) return;
    const int32_t li = owner[(size_t)(y >> lg) * mw + (x >> lg)];
    uint32_t packed = 0;
    if (li >= 0) {
        const LeafMap L = unpack(leaves[li], c);
#pragma unroll
        for (int q = 0; q < 4; ++q) packed |= (uint32_t)leaf_pixel(src, w, L, y, x + q) << (8 * q);
    }
    *reinterpret_cast<uint32_t*>(dst + (size_t)y * w + x) = packed;
}

}  // namespace

cudaError_t launch_decode_step(const uint8_t* src, uint8_t* dst, int w, int h, int lg,
                               const int32_t* owner, const DecodeLeaf* leaves, DecodeConsts c,
                               cudaStream_t st) {
    const int mw = (w + (1 << lg) - 1) >> lg;
    if (lg >= 2 && (w % 4) == 0) {
        dim3 grid((w / 4 + 127) / 128, h);
        decode_step4_kernel<<<grid, 128, 0, st>>>(src, dst, w, h, lg, mw, owner, leaves, c);
    } else {
        dim3 grid((w + 255) / 256, h);
        decode_step_kernel<<<grid, 256, 0, st>>>(src, dst, w, h, lg, mw, owner, leaves, c);
    }
    return cudaGetLastError();
}

}  // namespace mars
