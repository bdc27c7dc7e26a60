// Fixed-point decode iteration as a gather.
//
// decode_step / decode_leaf (crates/mars-codec/src/ifs.rs:299-309, 406-484) scatter each
// leaf's (u, v) domain samples to range positions (i, j) = map(iso, u, v).  Every output
// pixel belongs to exactly one leaf, so the same map is computed here as a gather: the
// owner map (one leaf index per 2^lg x 2^lg cell, lg the largest power of two dividing
// every leaf's row, column and size) names the leaf of each pixel, and the inverse
// isometry names its domain sample.  Values use the reference's f64 association,
// (0.5 + d*alfa) + beta (+ the mode-3 residual); pixels no leaf covers are written 0, as
// the reference's zero-filled `next` buffer is.
//
// The 16-byte packed leaves are expanded once per leaf list (decode_expand_kernel): alfa
// and beta are dequantised with the reference's operations in its order, so the doubles
// are the ones decode_leaf computes.
//
// decode_cell_kernel (lg >= 2, width % 4 == 0): one thread per 4x4 output cell.  A cell lies
// in one leaf, and the inverse isometry maps it onto a 4x4 set of domain samples, i.e. one
// 8x8 byte window of the previous iterate: the thread reads it as eight 8-byte rows, forms
// the sixteen 2x2 sums with byte-pair SIMD adds in 16-bit lanes, evaluates the sixteen
// values in sample order, moves them to output order with byte permutes (row reversal,
// byte reversal, 4x4 transpose) and stores four 4-byte rows.  decode_pixel_kernel covers
// any other geometry.
#include "kernels.cuh"

namespace mars {
namespace {

struct Unpacked {
    double alfa, beta, gx, gy;  // mode 1: alfa holds b0
    int row, col, size, mode, iso, dom_row, dom_col;
    bool domain;                // qalfa != 0 and mode != 1: the leaf reads a domain block
};

// ifs.rs:416-439.
__device__ __forceinline__ Unpacked unpack(const DecodeLeaf p, const DecodeConsts& c) {
    Unpacked L;
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

__device__ __forceinline__ uint32_t clamp_u8(double value) {
    if (!(value >= 0.0)) value = 0.0;
    if (value > 255.0) value = 255.0;
    return (uint32_t)value;
}

// clamp(0, 255) then truncation: truncating first and clamping the integer gives the same
// byte (a NaN converts to 0 either way).
__device__ __forceinline__ uint32_t to_u8(double value) {
    return (uint32_t)min(max(__double2int_rz(value), 0), 255);
}

// (u, v) = (cu + ai*i + aj*j, cv + bi*i + bj*j): the inverse of isometry::map
// (isometry.rs:7-19) as an affine map of the range position (i, j), with S1 = size - 1.
// Three bits describe it: tr (u follows j and v follows i: isometries 1, 2, 6, 7), uneg (u
// counts down from S1: 2, 3, 5, 7) and vneg (v counts down: 1, 3, 4, 7).
struct IsoInv {
    int cu, ai, aj, cv, bi, bj;
};
__device__ __forceinline__ IsoInv iso_inverse(int k, int S1) {
    const bool tr = (0xC6u >> k) & 1u, uneg = (0xACu >> k) & 1u, vneg = (0x9Au >> k) & 1u;
    const int su = uneg ? -1 : 1, sv = vneg ? -1 : 1;
    return {uneg ? S1 : 0, tr ? 0 : su, tr ? su : 0, vneg ? S1 : 0, tr ? sv : 0, tr ? 0 : sv};
}

// A 4x4 byte tile in four row words (byte q of word p = element (p, q)): transposed.
__device__ __forceinline__ void transpose4x4(uint32_t& r0, uint32_t& r1, uint32_t& r2,
                                             uint32_t& r3) {
    // 2x2 blocks of bytes first, then bytes within each block.
    const uint32_t a0 = __byte_perm(r0, r2, 0x5410), a1 = __byte_perm(r1, r3, 0x5410);
    const uint32_t a2 = __byte_perm(r0, r2, 0x7632), a3 = __byte_perm(r1, r3, 0x7632);
    r0 = __byte_perm(a0, a1, 0x6240);
    r1 = __byte_perm(a0, a1, 0x7351);
    r2 = __byte_perm(a2, a3, 0x6240);
    r3 = __byte_perm(a2, a3, 0x7351);
}

__global__ void decode_expand_kernel(const DecodeLeaf* __restrict__ leaves,
                                     const int32_t* __restrict__ resid_off, int n,
                                     DecodeConsts c, DecodeMap* __restrict__ maps) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const Unpacked L = unpack(leaves[k], c);
    DecodeMap m;
    // Domain kinds keep alfa / 4: (sum / 4) * alfa == sum * (alfa / 4) exactly, both
    // scalings by 1/4 being exact.
    m.a = L.mode == 1 ? L.alfa : __dmul_rn(L.alfa, 0.25);
    m.b = L.beta;
    m.gx = L.gx;
    m.gy = L.gy;
    m.rc = (uint32_t)L.row | ((uint32_t)L.col << 16);
    m.dom = (uint32_t)L.dom_row | ((uint32_t)L.dom_col << 16);
    m.roff = -1;
    uint32_t kind, cbyte = 0, flags = 0;
    if (L.mode == 1) {
        kind = kLeafAffine;
    } else if (L.mode == 3 && resid_off && resid_off[k] >= 0) {
        // A zero-alpha residual leaf still adds its residual (ifs.rs:459-479).
        kind = kLeafResidual;
        m.roff = resid_off[k];
        if (!L.domain) flags = kLeafNoDomain;
    } else if (!L.domain) {
        // d = 0: (0.5 + 0*alfa) + beta, the same for every pixel of the leaf.
        kind = kLeafConst;
        cbyte = clamp_u8(__dadd_rn(__dadd_rn(0.5, __dmul_rn(0.0, L.alfa)), L.beta));
    } else {
        kind = kLeafDomain;
    }
    m.info = (uint32_t)L.size | (kind << 12) | ((uint32_t)L.iso << 14) | flags | (cbyte << 24);
    maps[k] = m;
}

__device__ __forceinline__ double domain_value(int sum, const DecodeMap& m) {
    // The four samples are small integers, so their f64 sum in the reference's order is
    // the integer sum exactly, and d * alfa = (sum / 4) * alfa = sum * (alfa / 4).
    return __dadd_rn(__dadd_rn(0.5, __dmul_rn((double)sum, m.a)), m.b);
}

// Mode 1: round(b0 + gx*u + gy*v) with (u, v) = (i, j) (ifs.rs:416-431); f64::round and
// CUDA's round() both round half away from zero.
__device__ __forceinline__ uint32_t affine_pixel(const DecodeMap& m, int i, int j) {
    return clamp_u8(round(__dadd_rn(__dadd_rn(m.a, __dmul_rn(m.gx, (double)i)),
                                    __dmul_rn(m.gy, (double)j))));
}

// Max-delta bookkeeping of the convergence-tested decode (decode_until_stable,
// ifs.rs:321-353): a step that starts after convergence writes nothing, and every step
// folds max |next - prev| of its pixels into its slot.
struct StableState {
    const int* done;  // set once an earlier step's delta met the threshold
    int* delta;       // this step's max |next - prev|
};

__device__ __forceinline__ void fold_delta(uint32_t d, int* slot) {
    for (int o = 16; o > 0; o >>= 1) d = max(d, __shfl_xor_sync(0xffffffffu, d, o));
    if ((threadIdx.x & 31) == 0 && d) atomicMax(slot, (int)d);
}

// One pixel per thread (any owner-map granularity or width).
template <bool kStable>
__global__ void decode_pixel_kernel(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst,
                                    int w, int h, int lg, int mw,
                                    const int32_t* __restrict__ owner,
                                    const DecodeMap* __restrict__ maps,
                                    const double* __restrict__ resid, StableState ss) {
    if (kStable && *ss.done) return;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (kStable && (x >= w || y >= h)) {
        fold_delta(0u, ss.delta);
        return;
    }
    if (x >= w || y >= h) return;
    const int32_t li = owner[(size_t)(y >> lg) * mw + (x >> lg)];
    uint32_t out = 0;
    if (li >= 0) {
        const DecodeMap m = maps[li];
        const uint32_t kind = (m.info >> 12) & 3u;
        const int i = y - (int)(m.rc & 0xFFFFu), j = x - (int)(m.rc >> 16);
        if (kind == kLeafConst) {
            out = m.info >> 24;
        } else if (kind == kLeafAffine) {
            out = affine_pixel(m, i, j);
        } else {
            const int S = (int)(m.info & 0xFFFu);
            const IsoInv t = iso_inverse((int)((m.info >> 14) & 7u), S - 1);
            const int u = t.cu + t.ai * i + t.aj * j, v = t.cv + t.bi * i + t.bj * j;
            int sum = 0;
            if (!(m.info & kLeafNoDomain)) {
                const size_t p = ((size_t)(m.dom & 0xFFFFu) + 2 * u) * w + (m.dom >> 16) + 2 * v;
                sum = (int)src[p] + (int)src[p + w] + (int)src[p + 1] + (int)src[p + w + 1];
            }
            double value = domain_value(sum, m);
            if (kind == kLeafResidual) value = __dadd_rn(value, resid[m.roff + u * S + v]);
            out = to_u8(value);
        }
    }
    dst[(size_t)y * w + x] = (uint8_t)out;
    if (kStable) {
        const uint32_t prev = src[(size_t)y * w + x];
        fold_delta(out > prev ? out - prev : prev - out, ss.delta);
    }
}

// Eight bytes of the plane from byte offset `off` (off + 8 <= total), through aligned
// 8-byte loads where they stay inside the plane.
__device__ __forceinline__ uint64_t load8(const uint8_t* __restrict__ src, size_t off,
                                          size_t total) {
    const size_t a = off & ~(size_t)7;
    const unsigned s = (unsigned)(off & 7);
    const uint64_t* p = reinterpret_cast<const uint64_t*>(src + a);
    if (s == 0) return __ldg(p);
    if (a + 16 <= total) return (__ldg(p) >> (8 * s)) | (__ldg(p + 1) << (64 - 8 * s));
    uint64_t v = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) v |= (uint64_t)__ldg(src + off + k) << (8 * k);
    return v;
}

// Byte-pair sums of a 4-byte word in two 16-bit lanes: [b0 + b1, b2 + b3].
__device__ __forceinline__ uint32_t pair_sums(uint32_t x) {
    return (x & 0x00FF00FFu) + ((x >> 8) & 0x00FF00FFu);
}

template <bool kStable>
__global__ void __launch_bounds__(128) decode_cell_kernel(
    const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, int w, int h, int lg, int mw,
    const int32_t* __restrict__ owner, const DecodeMap* __restrict__ maps,
    const double* __restrict__ resid, StableState ss) {
    if (kStable && *ss.done) return;
    const int x0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int y0 = 4 * blockIdx.y;
    if (kStable && (x0 >= w || y0 >= h)) {
        fold_delta(0u, ss.delta);
        return;
    }
    if (x0 >= w || y0 >= h) return;
    const int32_t li = owner[(size_t)(y0 >> lg) * mw + (x0 >> lg)];
    uint64_t lo = 0, hi = 0;  // output rows 0-1 and 2-3, byte 4*a + b = pixel (y0 + a, x0 + b)
    if (li >= 0) {
        const DecodeMap m = maps[li];
        const uint32_t kind = (m.info >> 12) & 3u;
        const int i0 = y0 - (int)(m.rc & 0xFFFFu), j0 = x0 - (int)(m.rc >> 16);
        if (kind == kLeafConst) {
            lo = hi = 0x0101010101010101ull * (uint64_t)(m.info >> 24);
        } else if (kind == kLeafAffine) {
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const uint64_t v = affine_pixel(m, i0 + a, j0 + b);
                    if (a < 2) lo |= v << (8 * (4 * a + b));
                    else hi |= v << (8 * (4 * (a - 2) + b));
                }
        } else {
            const int S = (int)(m.info & 0xFFFu);
            const int k = (int)((m.info >> 14) & 7u);
            const IsoInv t = iso_inverse(k, S - 1);
            const int u00 = t.cu + t.ai * i0 + t.aj * j0, v00 = t.cv + t.bi * i0 + t.bj * j0;
            const int umin = u00 - 3 * ((t.ai < 0) | (t.aj < 0));
            const int vmin = v00 - 3 * ((t.bi < 0) | (t.bj < 0));
            const size_t total = (size_t)w * h;
            size_t off = ((size_t)(m.dom & 0xFFFFu) + 2 * umin) * w + (m.dom >> 16) + 2 * vmin;
            // 2x2 sums of sample (umin + p, vmin + q) in 16-bit lanes; zero without a domain.
            uint32_t sums[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
            if (!(m.info & kLeafNoDomain)) {
#pragma unroll
                for (int r = 0; r < 8; ++r, off += w) {
                    const uint64_t row = load8(src, off, total);
                    const uint32_t s0 = pair_sums((uint32_t)row);
                    const uint32_t s1 = pair_sums((uint32_t)(row >> 32));
                    sums[r >> 1][0] += s0;
                    sums[r >> 1][1] += s1;
                }
            }
            // Values in sample order: byte q of word p is sample (umin + p, vmin + q).
            uint32_t rw[4] = {0, 0, 0, 0};
#pragma unroll
            for (int p = 0; p < 4; ++p)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int sum = (int)((sums[p][q >> 1] >> (16 * (q & 1))) & 0xFFFFu);
                    double value = domain_value(sum, m);
                    if (kind == kLeafResidual)
                        value = __dadd_rn(value, __ldg(resid + m.roff + (umin + p) * S + vmin + q));
                    rw[p] |= to_u8(value) << (8 * q);
                }
            // Sample (p, q) is output pixel (a, b) with a = p (or 3 - p when u counts down)
            // and b = q (or 3 - q when v counts down), transposed for isometries 1, 2, 6, 7.
            const bool tr = (0xC6u >> k) & 1u, uneg = (0xACu >> k) & 1u, vneg = (0x9Au >> k) & 1u;
            if (vneg) {
#pragma unroll
                for (int p = 0; p < 4; ++p) rw[p] = __byte_perm(rw[p], 0, 0x0123);
            }
            if (uneg) {
                const uint32_t t0 = rw[0], t1 = rw[1];
                rw[0] = rw[3];
                rw[1] = rw[2];
                rw[2] = t1;
                rw[3] = t0;
            }
            if (tr) transpose4x4(rw[0], rw[1], rw[2], rw[3]);
            lo = (uint64_t)rw[0] | ((uint64_t)rw[1] << 32);
            hi = (uint64_t)rw[2] | ((uint64_t)rw[3] << 32);
        }
    }
    uint8_t* out = dst + (size_t)y0 * w + x0;
    const uint32_t rows_out[4] = {(uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi,
                                  (uint32_t)(hi >> 32)};
    *reinterpret_cast<uint32_t*>(out) = rows_out[0];
    if (y0 + 1 < h) *reinterpret_cast<uint32_t*>(out + w) = rows_out[1];
    if (y0 + 2 < h) *reinterpret_cast<uint32_t*>(out + 2 * (size_t)w) = rows_out[2];
    if (y0 + 3 < h) *reinterpret_cast<uint32_t*>(out + 3 * (size_t)w) = rows_out[3];
    if (kStable) {
        uint32_t m = 0;  // per-byte max |next - prev| over the cell's rows in the plane
        const uint8_t* prev = src + (size_t)y0 * w + x0;
#pragma unroll
        for (int a = 0; a < 4; ++a)
            if (y0 + a < h)
                m = __vmaxu4(m, __vabsdiffu4(rows_out[a],
                                             *reinterpret_cast<const uint32_t*>(prev + (size_t)a * w)));
        m = max(max(m & 255u, (m >> 8) & 255u), max((m >> 16) & 255u, m >> 24));
        fold_delta(m, ss.delta);
    }
}

// After step `iter`: the first step whose delta met the threshold ends the decode.
__global__ void decode_converged_kernel(const int* __restrict__ delta, int threshold, int iter,
                                    int* __restrict__ done, int* __restrict__ used) {
    if (!*done && *delta <= threshold) {
        *done = 1;
        *used = iter + 1;
    }
}

// ---- source-ordered decode of planes larger than L2 (decode_sorted_*) ----
//
// Gathering cell by cell in output order reads each cell's 8x8 domain window from a random
// place of the previous iterate; once the plane no longer fits in L2, every 8-byte row read
// costs whole DRAM sectors.  The source-ordered form splits a step in two:
//   gather : the domain cells in the order of their windows' source rows (a list built once
//            per leaf list), each computing its 16 output bytes into a cell buffer; the
//            windows of cells running together lie in a narrow band of source rows, which
//            L2 keeps, so the plane is read about once;
//   place  : every output cell in output order, copying its 16 bytes from the cell buffer
//            (domain cells) or computing them (constant and affine cells), four coalesced
//            4-byte row stores.
// The values are the cell kernel's, operation for operation.  Maps with mode-3 residuals keep
// the cell kernel.

// The window of a domain cell: the byte offset of its top-left sample pixel and the source
// row it starts at.
__device__ __forceinline__ void cell_window(const DecodeMap& m, int x0, int y0, int w,
                                            size_t* off, int* row) {
    const int S = (int)(m.info & 0xFFFu);
    const int k = (int)((m.info >> 14) & 7u);
    const IsoInv t = iso_inverse(k, S - 1);
    const int i0 = y0 - (int)(m.rc & 0xFFFFu), j0 = x0 - (int)(m.rc >> 16);
    const int u00 = t.cu + t.ai * i0 + t.aj * j0, v00 = t.cv + t.bi * i0 + t.bj * j0;
    const int umin = u00 - 3 * ((t.ai < 0) | (t.aj < 0));
    const int vmin = v00 - 3 * ((t.bi < 0) | (t.bj < 0));
    *row = (int)(m.dom & 0xFFFFu) + 2 * umin;
    *off = (size_t)(*row) * w + (m.dom >> 16) + 2 * vmin;
}

__device__ __forceinline__ bool is_domain_cell(const DecodeMap& m) {
    return ((m.info >> 12) & 3u) == kLeafDomain;
}

// Pass 1 of the list build: per 4x4 cell its window's source row (or ~0 for a cell without
// a domain window) and the rows' cell counts.
__global__ void sorted_key_kernel(int w, int h, int lg, int mw, const int32_t* __restrict__ owner,
                                  const DecodeMap* __restrict__ maps, uint32_t* __restrict__ key,
                                  uint32_t* __restrict__ row_count) {
    const int cw = w / 4, chh = (h + 3) / 4;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long long)cw * chh) return;
    const int x0 = 4 * (int)(c % cw), y0 = 4 * (int)(c / cw);
    const int32_t li = owner[(size_t)(y0 >> lg) * mw + (x0 >> lg)];
    uint32_t k = 0xFFFFFFFFu;
    if (li >= 0) {
        const DecodeMap m = maps[li];
        if (is_domain_cell(m)) {
            size_t off;
            int row;
            cell_window(m, x0, y0, w, &off, &row);
            k = (uint32_t)row;
            atomicAdd(&row_count[row], 1u);
        }
    }
    key[c] = k;
}

// Exclusive scan of the row counts (one block): the first list slot of each source row, and
// in cursor[h] the total.
__global__ void sorted_scan_kernel(const uint32_t* __restrict__ row_count, int h,
                                   uint32_t* __restrict__ cursor) {
    __shared__ uint32_t carry;
    __shared__ uint32_t warp_tot[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int base = 0; base < h; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const uint32_t v = i < h ? row_count[i] : 0u;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_tot[warp] = x;
        __syncthreads();
        uint32_t before = carry;
        for (int k = 0; k < warp; ++k) before += warp_tot[k];
        if (i < h) cursor[i] = before + x - v;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t all = 0;
            for (int k = 0; k < nw; ++k) all += warp_tot[k];
            carry += all;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) cursor[h] = carry;  // the number of domain cells
}

// Pass 2: each domain cell takes the next slot of its source row and writes its job
// (window offset, qalfa | isometry << 24, beta) there and the slot into inv.
__global__ void sorted_scatter_kernel(int w, int h, int lg, int mw,
                                      const int32_t* __restrict__ owner,
                                      const DecodeMap* __restrict__ maps,
                                      const DecodeLeaf* __restrict__ leaves,
                                      const uint32_t* __restrict__ key, uint32_t* __restrict__ cursor,
                                      uint4* __restrict__ jobs, uint32_t* __restrict__ inv) {
    const int cw = w / 4, chh = (h + 3) / 4;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long long)cw * chh) return;
    const uint32_t row = key[c];
    if (row == 0xFFFFFFFFu) return;
    const int x0 = 4 * (int)(c % cw), y0 = 4 * (int)(c / cw);
    const int32_t li = owner[(size_t)(y0 >> lg) * mw + (x0 >> lg)];
    const DecodeMap m = maps[li];
    size_t off;
    int r;
    cell_window(m, x0, y0, w, &off, &r);
    const uint32_t pos = atomicAdd(&cursor[row], 1u);
    const uint32_t qalfa = leaves[li].w & 0x1FFFFu;
    const uint32_t k = (m.info >> 14) & 7u;
    jobs[pos] = make_uint4((uint32_t)off, qalfa | (k << 24),
                           (uint32_t)__double2loint(m.b), (uint32_t)__double2hiint(m.b));
    inv[c] = pos;
}

// Gather pass: job -> the cell's 16 output bytes (row-major 4x4) in the cell buffer.
__global__ void __launch_bounds__(128) sorted_gather_kernel(
    const uint8_t* __restrict__ src, size_t total, int w, const uint4* __restrict__ jobs,
    uint32_t n, DecodeConsts cst, uint4* __restrict__ cellbuf) {
    const uint32_t pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const uint4 jb = jobs[pos];
    size_t off = jb.x;
    const int k = (int)(jb.y >> 24);
    DecodeMap m;
    // decode_expand's a = alfa / 4, alfa = (qalfa / 2^bits_alfa) * max_alfa (ifs.rs:434-439).
    m.a = __dmul_rn(__dmul_rn(__ddiv_rn((double)(jb.y & 0x1FFFFu), cst.alfa_den), cst.max_alfa), 0.25);
    m.b = __hiloint2double((int)jb.w, (int)jb.z);
    uint32_t sums[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
#pragma unroll
    for (int r = 0; r < 8; ++r, off += w) {
        const uint64_t row = load8(src, off, total);
        sums[r >> 1][0] += pair_sums((uint32_t)row);
        sums[r >> 1][1] += pair_sums((uint32_t)(row >> 32));
    }
    uint32_t rw[4] = {0, 0, 0, 0};
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int sum = (int)((sums[p][q >> 1] >> (16 * (q & 1))) & 0xFFFFu);
            rw[p] |= to_u8(domain_value(sum, m)) << (8 * q);
        }
    const bool tr = (0xC6u >> k) & 1u, uneg = (0xACu >> k) & 1u, vneg = (0x9Au >> k) & 1u;
    if (vneg) {
#pragma unroll
        for (int p = 0; p < 4; ++p) rw[p] = __byte_perm(rw[p], 0, 0x0123);
    }
    if (uneg) {
        const uint32_t t0 = rw[0], t1 = rw[1];
        rw[0] = rw[3];
        rw[1] = rw[2];
        rw[2] = t1;
        rw[3] = t0;
    }
    if (tr) transpose4x4(rw[0], rw[1], rw[2], rw[3]);
    cellbuf[pos] = make_uint4(rw[0], rw[1], rw[2], rw[3]);
}

// Place pass: every 4x4 output cell in output order.
__global__ void __launch_bounds__(128) sorted_place_kernel(
    uint8_t* __restrict__ dst, int w, int h, int lg, int mw, const int32_t* __restrict__ owner,
    const DecodeMap* __restrict__ maps, const uint32_t* __restrict__ inv,
    const uint4* __restrict__ cellbuf) {
    const int x0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int y0 = 4 * blockIdx.y;
    if (x0 >= w || y0 >= h) return;
    const int32_t li = owner[(size_t)(y0 >> lg) * mw + (x0 >> lg)];
    uint32_t rw[4] = {0, 0, 0, 0};
    if (li >= 0) {
        const DecodeMap m = maps[li];
        const uint32_t kind = (m.info >> 12) & 3u;
        if (kind == kLeafDomain) {
            const uint4 v = cellbuf[inv[(size_t)(y0 / 4) * (w / 4) + x0 / 4]];
            rw[0] = v.x;
            rw[1] = v.y;
            rw[2] = v.z;
            rw[3] = v.w;
        } else if (kind == kLeafConst) {
            rw[0] = rw[1] = rw[2] = rw[3] = 0x01010101u * (m.info >> 24);
        } else {
            const int i0 = y0 - (int)(m.rc & 0xFFFFu), j0 = x0 - (int)(m.rc >> 16);
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) rw[a] |= affine_pixel(m, i0 + a, j0 + b) << (8 * b);
        }
    }
    uint8_t* out = dst + (size_t)y0 * w + x0;
#pragma unroll
    for (int a = 0; a < 4; ++a)
        if (y0 + a < h) *reinterpret_cast<uint32_t*>(out + (size_t)a * w) = rw[a];
}

}  // namespace

cudaError_t launch_decode_expand(const DecodeLeaf* leaves, const int32_t* resid_off, int n,
                                 DecodeConsts c, DecodeMap* maps, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    decode_expand_kernel<<<(n + 255) / 256, 256, 0, st>>>(leaves, resid_off, n, c, maps);
    return cudaGetLastError();
}

cudaError_t launch_decode_step(const uint8_t* src, uint8_t* dst, int w, int h, int lg,
                               const int32_t* owner, const DecodeMap* maps, const double* resid,
                               cudaStream_t st) {
    const int mw = (w + (1 << lg) - 1) >> lg;
    const bool aligned =
        ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 7) == 0;
    const StableState none{nullptr, nullptr};
    if (lg >= 2 && (w % 4) == 0 && aligned) {
        dim3 grid((w / 4 + 127) / 128, (h + 3) / 4);
        decode_cell_kernel<false><<<grid, 128, 0, st>>>(src, dst, w, h, lg, mw, owner, maps, resid,
                                                        none);
    } else {
        dim3 grid((w + 255) / 256, h);
        decode_pixel_kernel<false><<<grid, 256, 0, st>>>(src, dst, w, h, lg, mw, owner, maps,
                                                         resid, none);
    }
    return cudaGetLastError();
}

cudaError_t launch_decode_step_stable(const uint8_t* src, uint8_t* dst, int w, int h, int lg,
                                      const int32_t* owner, const DecodeMap* maps,
                                      const double* resid, const int* done, int* delta,
                                      int threshold, int iter, int* done_w, int* used,
                                      cudaStream_t st) {
    const int mw = (w + (1 << lg) - 1) >> lg;
    const bool aligned =
        ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 7) == 0;
    const StableState ss{done, delta};
    if (lg >= 2 && (w % 4) == 0 && aligned) {
        dim3 grid((w / 4 + 127) / 128, (h + 3) / 4);
        decode_cell_kernel<true><<<grid, 128, 0, st>>>(src, dst, w, h, lg, mw, owner, maps, resid,
                                                       ss);
    } else {
        dim3 grid((w + 255) / 256, h);
        decode_pixel_kernel<true><<<grid, 256, 0, st>>>(src, dst, w, h, lg, mw, owner, maps,
                                                        resid, ss);
    }
    decode_converged_kernel<<<1, 1, 0, st>>>(delta, threshold, iter, done_w, used);
    return cudaGetLastError();
}


size_t decode_sorted_cells(int w, int h) { return (size_t)(w / 4) * ((h + 3) / 4); }

bool decode_sorted_eligible(int w, int h, int lg, bool residuals) {
    return lg >= 2 && (w % 4) == 0 && !residuals && w > 0 && h > 0;
}

cudaError_t launch_decode_sorted_build(int w, int h, int lg, const int32_t* owner,
                                       const DecodeMap* maps, const DecodeLeaf* leaves,
                                       uint32_t* key, uint32_t* row_count, uint32_t* cursor,
                                       uint4* jobs, uint32_t* inv, cudaStream_t st) {
    const int mw = (w + (1 << lg) - 1) >> lg;
    const size_t cells = decode_sorted_cells(w, h);
    cudaError_t e = cudaMemsetAsync(row_count, 0, (size_t)h * 4, st);
    if (e != cudaSuccess) return e;
    const unsigned blocks = (unsigned)((cells + 255) / 256);
    sorted_key_kernel<<<blocks, 256, 0, st>>>(w, h, lg, mw, owner, maps, key, row_count);
    sorted_scan_kernel<<<1, 1024, 0, st>>>(row_count, h, cursor);
    sorted_scatter_kernel<<<blocks, 256, 0, st>>>(w, h, lg, mw, owner, maps, leaves, key, cursor,
                                                   jobs, inv);
    return cudaGetLastError();
}

cudaError_t launch_decode_sorted_step(const uint8_t* src, uint8_t* dst, int w, int h, int lg,
                                      const int32_t* owner, const DecodeMap* maps,
                                      const uint4* jobs, uint32_t njobs, const uint32_t* inv,
                                      DecodeConsts c, uint4* cellbuf, cudaStream_t st) {
    const int mw = (w + (1 << lg) - 1) >> lg;
    if (njobs)
        sorted_gather_kernel<<<(njobs + 127) / 128, 128, 0, st>>>(src, (size_t)w * h, w, jobs,
                                                                 njobs, c, cellbuf);
    dim3 grid((w / 4 + 127) / 128, (h + 3) / 4);
    sorted_place_kernel<<<grid, 128, 0, st>>>(dst, w, h, lg, mw, owner, maps, inv, cellbuf);
    return cudaGetLastError();
}

}  // namespace mars
