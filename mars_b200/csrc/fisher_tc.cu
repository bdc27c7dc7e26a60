// Fisher's classified search on tcgen05 tensor cores, as a class-bucketed batch.
//
// The classified search (crates/mars-search/src/fisher.rs:30-78 over search_block_fitted,
// lib.rs:211-297) compares a range block only with the domains of one bucket (its class x
// variance class, or the first non-empty bucket when that one is empty), each pair under
// one isometry, MAPPING[range isometry][domain isometry] (tables.rs:42-51).  Flipping each
// range by its own isometry and each domain by its own (`flips`, classify.rs:139-164) turns
// every pair's cross term  sum R[map_iso(u, v)] * D[u, v]  into  sum R_c[u, v] * D_c[u, v]
// of the two canonical blocks (the identity holds for all 64 isometry pairs; checked in
// tests/test_fisher_ref_pin.py), so the pairs of one bucket are one plain matrix product.
//
// Per level (block size S in {4, 8, 16}):
//   fisher_range_kernel  : each range's bucket (as the device index classifies, resolved
//                          through `ref`) and isometry, from exact quadrant sums;
//   count / fill         : ranges grouped by bucket (fisher.cu's kernels over that key);
//   fisher_plan_kernel   : per bucket the A tiles (its domains, 128 a tile), the B tiles
//                          (its ranges, 128 a tile), the M-chunks and the work items;
//   build_a / build_b    : the canonical operands in the shared-memory core-matrix order,
//                          A = the contracted plane D (0..1020) split into two u8 digits
//                          (D = 128 hi + lo), B = canonical range pixels - 128 (s8),
//                          K = S^2 samples (S = 4 padded to 32);
//   fisher_seed_kernel   : each range's exact best of the first 32 candidates of its bucket;
//   fisher_tc_kernel     : per work item (bucket, M-chunk, B tile) the tcgen05 GEMM of
//                          digits x ranges with the exact-bound epilogue of search_tc.cu
//                          (one threshold per candidate: a column is one range), survivors
//                          fitted exactly, the champion by (rms, bucket index);
//   fisher_finish_kernel : per range the champion over its bucket's M-chunks, re-fitted
//                          for qalfa / qbeta, with domain, isometry and moments.
// Results equal the CUDA-core Fisher kernel's (fisher.cu) bit for bit; evals are the bucket
// lengths.  Every mbarrier wait is bounded, as in search_tc.cu.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "fisher_common.cuh"
#include "fisher_tc.cuh"
#include "kernels.cuh"
#include "tc_ptx.cuh"

namespace mars {
namespace ftc {
namespace {

using namespace mars::tc;

constexpr int kNt = 128;                    // ranges (accumulator columns) per tile, per digit
constexpr int kCols = 4 * kNt / kEpiWarps;  // 64 columns per epilogue warp
constexpr int kChunks = kCols / 32;         // 2
constexpr int kQueueCap = 2048;
constexpr int kWarpCap = kQueueCap / kEpiWarps;
constexpr int kWarpFlush = 48;
constexpr int kStagesMax = 4;
constexpr int kMaxChunkItems = 8;  // a bucket with few B tiles is split into up to 8 M-chunks
constexpr uint32_t kNone = 0xffffffffu;

// K layout: the S^2 canonical samples in flat order u*S + v, 16 to a K-group, padded to an
// even number of K-groups (one MMA reads 32 bytes of K).  A stage holds up to 8 K-groups.
__host__ __device__ constexpr int kgroups(int S) { return S * S / 16 < 2 ? 2 : S * S / 16; }
__host__ __device__ constexpr int stage_kg(int S) { return kgroups(S) < 8 ? kgroups(S) : 8; }
__host__ __device__ constexpr int kstages(int S) { return kgroups(S) / stage_kg(S); }
// Bytes of one stage: A = 2 digits x 16 row groups x stage_kg x 128 B; B = 16 row groups.
__host__ __device__ constexpr int a_stage_bytes(int S) { return 2 * 16 * stage_kg(S) * 128; }
__host__ __device__ constexpr int b_stage_bytes(int S) { return 16 * stage_kg(S) * 128; }
__host__ __device__ constexpr int pipe_stages(int S) { return S == 16 ? 3 : 4; }

// flips (classify.rs:139-164; Mars 1 coding_func.c:1200-1247): the canonical block's (i, j)
// reads the original block at the returned flat index.
__device__ __forceinline__ int flip_src(int iso, int i, int j, int s) {
    switch (iso) {
        case 0: return i * s + j;
        case 1: return j * s + (s - i - 1);
        case 2: return (s - j - 1) * s + i;
        case 3: return (s - i - 1) * s + (s - j - 1);
        case 4: return i * s + (s - j - 1);
        case 5: return (s - i - 1) * s + j;
        case 6: return j * s + i;
        default: return (s - j - 1) * s + (s - i - 1);
    }
}

struct Champ {
    double rms, sum, rms0;
    int64_t nrr;
    uint32_t idx;  // bucket index of the champion (kNone: none yet)
    int32_t t0, t2, valid;
    int32_t t1x4;
};

// Pruning record per range (column); the same forms as search_tc.cu's ThrRec: short form
// t1' < s1_x4 * c + fma(sqrt_w, sqrt(Ndd), neg), the full Z-form when `full`.
struct __align__(16) ThrRec {
    float sqrt_w, w2a, neg, c;
    int32_t tie, full, pad1, pad2;
};

struct __align__(8) QEntry {
    int32_t t1;     // t1' = t1_x4 - 128 * s1_x4 (canonical operands)
    uint32_t e;     // bucket index of the domain
    uint32_t code;  // tile tag << 16 | lane << 8 | column
    uint32_t pad;
    double rms, sum;
};

struct Smem {
    uint64_t full[kStagesMax];
    uint64_t empty[kStagesMax];
    uint64_t tfull[2];
    uint64_t tempty[2];
    uint64_t bres;
    uint32_t tmem_base;
    int abort_flag;
    int wcount[kEpiWarps];
    uint32_t full_bits[kNt / 32];
    unsigned long long key_rms[kNt];
    uint32_t key_idx[kNt];
    double key_sum[kNt];
    int32_t key_t1[kNt];
    ThrRec thr[kNt];
    Champ ch[kNt];
    uint32_t evaluated[kM * kNt / 32];
    QEntry queue[kQueueCap];
};

template <int S>
constexpr size_t smem_bytes() {
    return 1024 + (size_t)pipe_stages(S) * a_stage_bytes(S) +
           (size_t)kstages(S) * b_stage_bytes(S) + sizeof(Smem);
}
static_assert(smem_bytes<4>() <= 232448 && smem_bytes<8>() <= 232448 && smem_bytes<16>() <= 232448,
              "shared memory per CTA (227 KB)");
static_assert(pipe_stages(16) <= kStagesMax && pipe_stages(8) <= kStagesMax, "stages");

__device__ __forceinline__ void publish(Smem& sm, int c, const FitParams& fp, int n) {
    const Champ& C = sm.ch[c];
    ThrRec t;
    const uint32_t bit = 1u << (c & 31);
    if (!C.valid) {
        // Padding column: nothing survives (short form +inf).
        t = ThrRec{INFINITY, INFINITY, 0.0f, 3.0e38f, -1, 0, 0, 0};
        sm.thr[c] = t;
        atomicAnd(&sm.full_bits[c >> 5], ~bit);
        return;
    }
    if (C.idx == kNone) {
        // No champion yet: keep everything (short form -inf).
        t = ThrRec{0.0f, 0.0f, -INFINITY, 0.0f, INT32_MAX, 0, 0, 0};
        sm.thr[c] = t;
        atomicAnd(&sm.full_bits[c >> 5], ~bit);
        return;
    }
    const Threshold th = make_threshold(C.sum, C.rms, C.idx, C.rms0, C.nrr, n, fp);
    const float four_inv_n = 4.0f / (float)n;
    t.sqrt_w = th.sqrt_w * four_inv_n;
    t.w2a = th.w2a * four_inv_n;
    t.neg = th.wpos ? 0.0f : -INFINITY;
    t.c = (float)C.t0 / (float)n - 128.0f;
    t.tie = th.mode == 2 ? -1 : (th.mode == 1 ? (int32_t)th.tie_dom : INT32_MAX);
    t.full = th.mode != 0 && !th.wpos;
    t.pad1 = t.pad2 = 0;
    sm.thr[c] = t;
    if (t.full)
        atomicOr(&sm.full_bits[c >> 5], bit);
    else
        atomicAnd(&sm.full_bits[c >> 5], ~bit);
}

__device__ __forceinline__ bool live(const Smem& sm, int qi) {
    return (qi % kWarpCap) < sm.wcount[qi / kWarpCap];
}

// Exact fits of the queued survivors and the champion updates (all epilogue threads, after
// a barrier: every warp's count is final).
template <int N>
__device__ __noinline__ void drain(Smem& sm, bool mark, uint32_t tag, int et, const uint32_t* list,
                                   uint32_t off, const DomainStats& ds, const FitParams& fp,
                                   unsigned long long& exact) {
    for (int qi = et; qi < kQueueCap; qi += kEpiThreads) {
        if (!live(sm, qi)) continue;
        QEntry& q = sm.queue[qi];
        const int c = (int)(q.code & 255u);
        const Champ& C = sm.ch[c];
        const uint32_t p = list[off + q.e];
        const int32_t s1 = ds.s1x4[p];
        const FitResult f =
            fit_exact(N, s1, ds.s2x16[p], C.t0, (int64_t)q.t1 + 128ll * s1, C.t2, fp);
        q.rms = f.rms;
        q.sum = f.sum;
        ++exact;
        atomicMin(&sm.key_rms[c], (unsigned long long)__double_as_longlong(f.rms));
    }
    epi_barrier();
    for (int qi = et; qi < kQueueCap; qi += kEpiThreads) {
        if (!live(sm, qi)) continue;
        const QEntry& q = sm.queue[qi];
        const int c = (int)(q.code & 255u);
        if ((unsigned long long)__double_as_longlong(q.rms) == sm.key_rms[c])
            atomicMin(&sm.key_idx[c], q.e);
    }
    epi_barrier();
    for (int qi = et; qi < kQueueCap; qi += kEpiThreads) {
        if (!live(sm, qi)) continue;
        const QEntry& q = sm.queue[qi];
        const int c = (int)(q.code & 255u);
        if ((unsigned long long)__double_as_longlong(q.rms) == sm.key_rms[c] &&
            q.e == sm.key_idx[c]) {
            sm.key_sum[c] = q.sum;
            sm.key_t1[c] = q.t1 + 128 * ds.s1x4[list[off + q.e]];
        }
        if (mark && (q.code >> 16) == tag) {
            const int qm = (int)(q.code >> 8) & 127;
            atomicOr(&sm.evaluated[(qm * kNt + c) >> 5], 1u << (c & 31));
        }
    }
    epi_barrier();
    for (int c = et; c < kNt; c += kEpiThreads) {
        if (sm.key_rms[c] == ~0ull) continue;
        Champ& C = sm.ch[c];
        const double r2 = __longlong_as_double((long long)sm.key_rms[c]);
        const uint32_t i2 = sm.key_idx[c];
        if (C.valid && (C.idx == kNone || r2 < C.rms || (r2 == C.rms && i2 < C.idx))) {
            C.rms = r2;
            C.idx = i2;
            C.sum = sm.key_sum[c];
            C.t1x4 = sm.key_t1[c];
            publish(sm, c, fp, N);
        }
        sm.key_rms[c] = ~0ull;
        sm.key_idx[c] = kNone;
    }
    epi_barrier();
    if (et < kEpiWarps) sm.wcount[et] = 0;
    epi_barrier();
}

// Work item -> (bucket, M-chunk, B tile) through the per-bucket item offsets.
__device__ __forceinline__ void locate(const FisherPlan& pl, int item, int* b, int* mc, int* nt) {
    int bb = 0;
    while (bb < 71 && pl.item_base[bb + 1] <= (uint32_t)item) ++bb;
    const int rest = item - (int)pl.item_base[bb];
    const int ntb = (int)pl.ntiles[bb];
    *b = bb;
    *mc = rest / ntb;
    *nt = rest % ntb;
}

template <int S>
__global__ void __launch_bounds__(kThreads, 1)
    fisher_tc_kernel(const uint8_t* __restrict__ aglob, const uint8_t* __restrict__ bglob,
                     FisherPlan pl, const uint32_t* __restrict__ counts,
                     const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ list,
                     const uint32_t* __restrict__ rlist, RangeStats rs, DomainStats ds,
                     FitParams fp, const tc::SeedOut* __restrict__ seeds,
                     Partial* __restrict__ partials, int* __restrict__ err,
                     unsigned long long* __restrict__ exact_counter) {
    constexpr int N = S * S;
    constexpr int KST = kstages(S);
    constexpr int SKG = stage_kg(S);
    constexpr int kStages = pipe_stages(S);
    constexpr int ASB = a_stage_bytes(S);
    constexpr int BSB = b_stage_bytes(S);
    constexpr uint32_t kSbo = SKG * 128;  // bytes between 8-row groups

    const int item = blockIdx.x;
    if ((uint32_t)item >= pl.item_base[72]) return;
    int b, mc, nt;
    locate(pl, item, &b, &mc, &nt);
    const uint32_t dcount = counts[b], doff = offsets[b];
    const uint32_t rcount = pl.rcounts[b], roff = pl.roffsets[b];
    const int dtiles = (int)((dcount + kM - 1) / kM);
    const int nchunks = (int)pl.chunks[b];
    const int per = (dtiles + nchunks - 1) / nchunks;
    const int m_begin = mc * per, m_end = min(dtiles, m_begin + per);

    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char* stA = base;
    unsigned char* stB = stA + kStages * ASB;  // resident: KST stages
    Smem& sm = *reinterpret_cast<Smem*>(stB + KST * BSB);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint8_t* atiles = aglob + ((size_t)pl.a_tile_base[b] + m_begin) * KST * ASB;
    const uint8_t* btile = bglob + ((size_t)pl.b_tile_base[b] + nt) * KST * BSB;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&sm.full[s], 1);
            mbar_init(&sm.empty[s], 1);
        }
        for (int q = 0; q < 2; ++q) {
            mbar_init(&sm.tfull[q], 1);
            mbar_init(&sm.tempty[q], kEpiThreads);
        }
        mbar_init(&sm.bres, 1);
        sm.abort_flag = 0;
        for (int w = 0; w < kEpiWarps; ++w) sm.wcount[w] = 0;
        for (int w = 0; w < kNt / 32; ++w) sm.full_bits[w] = 0u;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = threadIdx.x; i < kM * kNt / 32; i += kThreads) sm.evaluated[i] = 0u;
    for (int c = threadIdx.x; c < kNt; c += kThreads) {
        Champ& C = sm.ch[c];
        const uint32_t k = (uint32_t)nt * kNt + (uint32_t)c;
        C.valid = k < rcount;
        if (C.valid) {
            const uint32_t r = rlist[roff + k];
            C.t0 = rs.t0[r];
            C.t2 = rs.t2[r];
            C.nrr = rs.nrr[r];
            C.rms0 = rs.rms0[r];
            const tc::SeedOut sd = seeds[r];
            C.rms = sd.rms;
            C.sum = sd.sum;
            C.idx = sd.idx;
            C.t1x4 = sd.t1x4;
        } else {
            C.rms = INFINITY;
            C.sum = 0.0;
            C.idx = kNone;
            C.t1x4 = 0;
        }
        sm.key_rms[c] = ~0ull;
        sm.key_idx[c] = kNone;
    }
    __syncthreads();
    for (int c = threadIdx.x; c < kNt; c += kThreads) publish(sm, c, fp, N);
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&sm.tmem_base)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tmem_fence_before();
    __syncthreads();
    tmem_fence_after();
    const uint32_t tmem = sm.tmem_base;
    volatile int* abort_flag = &sm.abort_flag;

    if (warp == 0) {
        // ---------------------------------------------------------------- loads
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            int issued = 0;
            mbar_expect_tx(&sm.bres, KST * BSB);
            for (int t = 0; t < KST; ++t)
                bulk_load(stB + t * BSB, btile + (size_t)t * BSB, BSB, &sm.bres);
            for (int mt = m_begin; mt < m_end && !*abort_flag; ++mt) {
                for (int t = 0; t < KST; ++t) {
                    if (issued >= kStages && !mbar_wait(&sm.empty[s], ph ^ 1, abort_flag, err, 1)) break;
                    mbar_expect_tx(&sm.full[s], ASB);
                    bulk_load(stA + s * ASB, atiles + ((size_t)(mt - m_begin) * KST + t) * ASB, ASB,
                              &sm.full[s]);
                    ++issued;
                    if (++s == kStages) {
                        s = 0;
                        ph ^= 1;
                    }
                }
            }
            // Wait (bounded) for the copies still in flight before leaving.
            {
                int s2 = s;
                uint32_t ph2 = ph;
                for (int i = 0; i < kStages && i < issued && *abort_flag; ++i) {
                    if (--s2 < 0) {
                        s2 = kStages - 1;
                        ph2 ^= 1;
                    }
                    const long long t0 = clock64();
                    while (!mbar_try_wait(&sm.full[s2], ph2) && clock64() - t0 < kWaitCycles) {
                    }
                }
                const long long t0 = clock64();
                while (!mbar_try_wait(&sm.bres, 0) && clock64() - t0 < kWaitCycles) {
                }
            }
        }
    } else if (warp == 1) {
        // ---------------------------------------------------------------- MMA
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            bool ok = mbar_wait(&sm.bres, 0, abort_flag, err, 2);
            int i = 0;
            for (int mt = m_begin; ok && mt < m_end; ++mt, ++i) {
                const int q = i & 1;
                const uint32_t qph = (uint32_t)((i >> 1) & 1);
                if (i >= 2 && !mbar_wait(&sm.tempty[q], qph ^ 1, abort_flag, err, 4)) break;
                tmem_fence_after();
                const uint32_t dcol = tmem + (uint32_t)(q * 2 * kNt);
                for (int t = 0; t < KST; ++t) {
                    if (!mbar_wait(&sm.full[s], ph, abort_flag, err, 8)) {
                        ok = false;
                        break;
                    }
                    tmem_fence_after();
                    const uint32_t a_addr = smem_u32(stA + s * ASB);
                    const uint32_t b_addr = smem_u32(stB + t * BSB);
#pragma unroll
                    for (int kk = 0; kk < SKG / 2; ++kk) {
                        const uint64_t bd = smem_desc(b_addr + kk * 256, kSbo);
                        const uint32_t acc = (t > 0 || kk > 0) ? 1u : 0u;
                        mma_i8<kNt>(dcol, smem_desc(a_addr + kk * 256, kSbo), bd, acc);
                        mma_i8<kNt>(dcol + kNt, smem_desc(a_addr + ASB / 2 + kk * 256, kSbo), bd,
                                    acc);
                    }
                    mma_commit(&sm.empty[s]);
                    if (++s == kStages) {
                        s = 0;
                        ph ^= 1;
                    }
                }
                if (!ok) break;
                mma_commit(&sm.tfull[q]);
            }
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------------------- epilogue
        const int et = threadIdx.x - 64;
        const int ew = et >> 5;
        const int e4 = warp & 3;
        const int part = (warp - 2) >> 2;
        const int m = e4 * 32 + lane;
        const float four_inv_n = 4.0f / (float)N;
        unsigned long long exact = 0;
        int i = 0;
        for (int mt = m_begin; mt < m_end; ++mt, ++i) {
            const int q = i & 1;
            const uint32_t qph = (uint32_t)((i >> 1) & 1);
            // This lane's domain: bucket index e (lanes past the bucket's end are skipped).
            const uint32_t e = (uint32_t)mt * kM + (uint32_t)m;
            float s1f = 0.f, detf = 1.f, sdetf = 1.f;
            int32_t edom = -1;
            if (e < dcount) {
                const uint32_t p = list[doff + e];
                s1f = (float)ds.s1x4[p];
                detf = ds.detf[p];
                sdetf = ds.sdetf[p];
                edom = (int32_t)e;
            }
            const float ad = __fmul_rd(fp.a_min, detf) * four_inv_n;
            const float ahd = __fmul_rd(fp.a_half, detf) * four_inv_n;
            const uint32_t tcol = tmem + ((uint32_t)(e4 * 32) << 16) +
                                  (uint32_t)(q * 2 * kNt + part * kCols);
            const uint32_t tag = (uint32_t)(mt & 0xFFFF);
            bool rescan = false;

            // The threshold of this lane's domain against column c (one range); `full` is
            // the column's bit of full_bits (the same for every lane of the warp).
            auto threshold = [&](int c, bool full) -> int32_t {
                const float4 ra = reinterpret_cast<const float4*>(sm.thr)[2 * c];
                float tau;
                if (full) {
                    const int tie = sm.thr[c].tie;
                    const float g1 = __fmul_rd(ra.x, sdetf);
                    const float tz = fminf(__fadd_rd(ra.y, ahd), fmaxf(g1, ad));
                    tau = edom > tie ? tz : __fadd_rd(g1, ra.z);
                } else {
                    tau = __fmaf_rd(ra.x, sdetf, ra.z);
                }
                return edom < 0 ? INT32_MAX : __float2int_rd(__fmaf_rd(s1f, ra.w, tau));
            };
            auto test_chunk = [&](const int32_t (&v)[32], int ch) {
                const int col0 = part * kCols + ch * 32;
                const uint32_t fw = sm.full_bits[col0 >> 5];
                uint32_t mask = 0u;
                if (fw == 0u) {
#pragma unroll
                    for (int c = 0; c < 32; ++c)
                        mask |= (v[c] >= threshold(col0 + c, false) ? 1u : 0u) << c;
                } else {
#pragma unroll
                    for (int c = 0; c < 32; ++c)
                        mask |= (v[c] >= threshold(col0 + c, (fw >> c) & 1u) ? 1u : 0u) << c;
                }
                if (rescan && mask) mask &= ~sm.evaluated[(m * kNt + col0) >> 5];
                if (mask) {
                    int slot = atomicAdd(&sm.wcount[ew], __popc(mask));
                    while (mask) {
                        const int c = __ffs(mask) - 1;
                        mask &= mask - 1;
                        int32_t val = v[0];
#pragma unroll
                        for (int k2 = 1; k2 < 32; ++k2) val = c == k2 ? v[k2] : val;
                        if (slot < kWarpCap)
                            sm.queue[ew * kWarpCap + slot] = QEntry{
                                val, e, (uint32_t)(tag << 16 | m << 8 | (col0 + c)), 0u, 0.0, 0.0};
                        ++slot;
                    }
                }
            };
            // Warp-uniform, so the aligned TMEM loads run with every lane.
            bool got = __all_sync(0xffffffffu, mbar_wait(&sm.tfull[q], qph, abort_flag, err, 16));
            bool first = true;
            for (;;) {
                if (got) {
                    if (first) tmem_fence_after();
                    int32_t va[32], vb[32];
                    __syncwarp();
#pragma unroll
                    for (int ch = 0; ch < kChunks; ++ch) {
                        tmem_ld32(tcol + 32u * ch, va);
                        tmem_ld32(tcol + (uint32_t)kNt + 32u * ch, vb);
                        tmem_wait(va);
                        tmem_wait(vb);
#pragma unroll
                        for (int c = 0; c < 32; ++c) va[c] = va[c] * 128 + vb[c];
                        test_chunk(va, ch);
                        __syncwarp();
                    }
                }
                first = false;
                __syncwarp();
                const bool last = mt + 1 == m_end;
                if (epi_barrier_and(got && !last && sm.wcount[ew] < kWarpFlush)) break;
                if (!epi_barrier_and(got)) {
                    got = false;
                    break;
                }
                bool over = false;
#pragma unroll
                for (int w2 = 0; w2 < kEpiWarps; ++w2) over |= sm.wcount[w2] > kWarpCap;
                drain<N>(sm, over, tag, et, list, doff, ds, fp, exact);
                if (over) {
                    rescan = true;
                    continue;
                }
                break;
            }
            if (!got) break;
            if (rescan) {
                for (int w2 = et; w2 < kM * kNt / 32; w2 += kEpiThreads) sm.evaluated[w2] = 0u;
                epi_barrier();
            }
            tmem_fence_before();
            mbar_arrive(&sm.tempty[q]);
        }
        if (exact_counter && exact) atomicAdd(exact_counter, exact);
    }

    tmem_fence_before();
    __syncthreads();
    if (warp == 1) {
        tmem_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
    }
    for (int c = threadIdx.x; c < kNt; c += kThreads) {
        const Champ& C = sm.ch[c];
        const uint32_t k = (uint32_t)nt * kNt + (uint32_t)c;
        if (k >= rcount) continue;
        Partial p;
        p.rms = C.rms;
        p.sum = C.sum;
        p.idx = C.idx;
        p.t1x4 = C.t1x4;
        p.qalfa = 0;
        p.qbeta = 0;
        p.pad = 0;
        partials[(size_t)pl.p_base[b] + (size_t)mc * rcount + k] = p;
    }
}

// Each range's bucket (through `ref`) and isometry from exact quadrant sums (the same
// classification fisher.cu's search kernel runs); 255 for a block outside the plane.
__global__ void fisher_range_kernel(const uint8_t* __restrict__ plane, int w, int h, int size,
                                    const uint32_t* __restrict__ rows,
                                    const uint32_t* __restrict__ cols, int nranges,
                                    const uint32_t* __restrict__ ref,
                                    uint8_t* __restrict__ rbucket, uint8_t* __restrict__ riso) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nranges) return;
    if (rows[r] + (uint32_t)size > (uint32_t)h || cols[r] + (uint32_t)size > (uint32_t)w) {
        rbucket[r] = 255;
        riso[r] = 0;
        return;
    }
    const int hq = size / 2;
    int64_t qs[4] = {0, 0, 0, 0}, q2[4] = {0, 0, 0, 0};
    const uint8_t* base = plane + (size_t)rows[r] * w + cols[r];
    for (int i = 0; i < size; ++i)
        for (int j = 0; j < size; ++j) {
            const int64_t p = base[(size_t)i * w + j];
            const int k = (i >= hq ? 2 : 0) + (j >= hq ? 1 : 0);
            qs[k] += p;
            q2[k] += p * p;
        }
    int iso, key;
    fisher_classify(qs, q2, hq, &iso, &key);
    rbucket[r] = (uint8_t)ref[key];
    riso[r] = (uint8_t)iso;
}

// Per bucket: A tiles, B tiles, M-chunks, partial and work-item offsets (one thread).
__global__ void fisher_plan_kernel(const uint32_t* __restrict__ counts, FisherPlan pl) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    uint32_t a = 0, bt = 0, items = 0, pb = 0;
    for (int b = 0; b < 72; ++b) {
        const uint32_t rc = pl.rcounts[b];
        const uint32_t dt = rc ? (counts[b] + kM - 1) / kM : 0;
        const uint32_t nt = (rc + kNt - 1) / kNt;
        uint32_t ch = 0;
        if (rc && dt) {
            const uint32_t want = nt >= kMaxChunkItems ? 1 : (kMaxChunkItems + nt - 1) / nt;
            ch = want < dt ? want : dt;
        }
        pl.a_tile_base[b] = a;
        pl.b_tile_base[b] = bt;
        pl.p_base[b] = pb;
        pl.item_base[b] = items;
        pl.chunks[b] = ch ? ch : 1;
        pl.ntiles[b] = nt ? nt : 1;
        a += dt;
        bt += dt ? nt : 0;
        pb += ch * rc;
        items += ch * nt;
    }
    pl.item_base[72] = items;
    pl.a_tile_base[72] = a;
    pl.b_tile_base[72] = bt;
}

// A operand: for each needed bucket, its domains in bucket order, canonical (flipped by the
// domain's isometry), as the two digits of D, in core-matrix order.  One thread per (row,
// K-group); rows past a bucket's end are not written (their lanes are skipped).
template <int S>
__global__ void fisher_build_a_kernel(const int32_t* __restrict__ D, int dw, int shift,
                                      int ncol_d, const uint32_t* __restrict__ counts,
                                      const uint32_t* __restrict__ offsets,
                                      const uint32_t* __restrict__ list,
                                      const uint8_t* __restrict__ diso, FisherPlan pl,
                                      uint8_t* __restrict__ out) {
    constexpr int KG = kgroups(S), SKG = stage_kg(S), KST = kstages(S), ASB = a_stage_bytes(S);
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long rows_total = (long long)pl.a_tile_base[72] * kM;
    if (tid >= rows_total * KG) return;
    const int kg = (int)(tid % KG);
    const long long row = tid / KG;
    const uint32_t tile = (uint32_t)(row / kM);
    const int r = (int)(row % kM);
    int b = 0;
    while (b < 71 && pl.a_tile_base[b + 1] <= tile) ++b;
    const uint32_t e = (tile - pl.a_tile_base[b]) * kM + (uint32_t)r;
    if (e >= counts[b]) return;
    const uint32_t p = list[offsets[b] + e];
    const int dr = (int)(p / (uint32_t)ncol_d) * (shift / 2);
    const int dc = (int)(p % (uint32_t)ncol_d) * (shift / 2);
    const int iso = diso[p];
    uint8_t hi[16], lo[16];
#pragma unroll
    for (int x = 0; x < 16; ++x) {
        const int f = kg * 16 + x;  // flat canonical sample u * S + v
        int32_t d = 0;
        if (f < S * S) {
            const int src = flip_src(iso, f / S, f % S, S);
            d = D[(size_t)(dr + src / S) * dw + dc + src % S];
        }
        hi[x] = (uint8_t)(d >> 7);
        lo[x] = (uint8_t)(d & 127);
    }
    const int st = kg / SKG, kgl = kg % SKG;
    unsigned char* dst = out + ((size_t)tile * KST + st) * ASB + (size_t)(r >> 3) * SKG * 128 +
                         (size_t)kgl * 128 + (size_t)(r & 7) * 16;
    uint4 h4, l4;
    h4.x = hi[0] | hi[1] << 8 | hi[2] << 16 | (uint32_t)hi[3] << 24;
    h4.y = hi[4] | hi[5] << 8 | hi[6] << 16 | (uint32_t)hi[7] << 24;
    h4.z = hi[8] | hi[9] << 8 | hi[10] << 16 | (uint32_t)hi[11] << 24;
    h4.w = hi[12] | hi[13] << 8 | hi[14] << 16 | (uint32_t)hi[15] << 24;
    l4.x = lo[0] | lo[1] << 8 | lo[2] << 16 | (uint32_t)lo[3] << 24;
    l4.y = lo[4] | lo[5] << 8 | lo[6] << 16 | (uint32_t)lo[7] << 24;
    l4.z = lo[8] | lo[9] << 8 | lo[10] << 16 | (uint32_t)lo[11] << 24;
    l4.w = lo[12] | lo[13] << 8 | lo[14] << 16 | (uint32_t)lo[15] << 24;
    *reinterpret_cast<uint4*>(dst) = h4;
    *reinterpret_cast<uint4*>(dst + ASB / 2) = l4;
}

// B operand: for each bucket, its ranges (in grouped order), canonical (flipped by the
// range's isometry), pixel - 128 as s8, in core-matrix order.  Rows past a bucket's ranges
// are zero.
template <int S>
__global__ void fisher_build_b_kernel(const uint8_t* __restrict__ plane, int w,
                                      const uint32_t* __restrict__ rows,
                                      const uint32_t* __restrict__ cols,
                                      const uint32_t* __restrict__ rlist,
                                      const uint8_t* __restrict__ riso, FisherPlan pl,
                                      uint8_t* __restrict__ out) {
    constexpr int KG = kgroups(S), SKG = stage_kg(S), KST = kstages(S), BSB = b_stage_bytes(S);
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long rows_total = (long long)pl.b_tile_base[72] * kNt;
    if (tid >= rows_total * KG) return;
    const int kg = (int)(tid % KG);
    const long long row = tid / KG;
    const uint32_t tile = (uint32_t)(row / kNt);
    const int n = (int)(row % kNt);
    int b = 0;
    while (b < 71 && pl.b_tile_base[b + 1] <= tile) ++b;
    const uint32_t k = (tile - pl.b_tile_base[b]) * kNt + (uint32_t)n;
    uint8_t bytes[16];
#pragma unroll
    for (int x = 0; x < 16; ++x) bytes[x] = 0;
    if (k < pl.rcounts[b]) {
        const uint32_t ri = rlist[pl.roffsets[b] + k];
        const int iso = riso[ri];
        const uint8_t* base = plane + (size_t)rows[ri] * w + cols[ri];
#pragma unroll
        for (int x = 0; x < 16; ++x) {
            const int f = kg * 16 + x;
            if (f < S * S) {
                const int src = flip_src(iso, f / S, f % S, S);
                bytes[x] = (uint8_t)(int8_t)((int)base[(size_t)(src / S) * w + src % S] - 128);
            }
        }
    }
    const int st = kg / SKG, kgl = kg % SKG;
    unsigned char* dst = out + ((size_t)tile * KST + st) * BSB + (size_t)(n >> 3) * SKG * 128 +
                         (size_t)kgl * 128 + (size_t)(n & 7) * 16;
    uint4 pk;
    pk.x = bytes[0] | bytes[1] << 8 | bytes[2] << 16 | (uint32_t)bytes[3] << 24;
    pk.y = bytes[4] | bytes[5] << 8 | bytes[6] << 16 | (uint32_t)bytes[7] << 24;
    pk.z = bytes[8] | bytes[9] << 8 | bytes[10] << 16 | (uint32_t)bytes[11] << 24;
    pk.w = bytes[12] | bytes[13] << 8 | bytes[14] << 16 | (uint32_t)bytes[15] << 24;
    *reinterpret_cast<uint4*>(dst) = pk;
}

// Exact canonical cross term t1_x4 = sum D_c * R_c of a range with a bucket entry; each
// lane sums its share of the samples (the warp reduces).
template <int S>
__device__ __forceinline__ int32_t canon_t1(const int32_t* D, int dw, int dr, int dc, int diso,
                                            const uint8_t* rb, int w, int riso, int lane) {
    int32_t t1 = 0;
    for (int f = lane; f < S * S; f += 32) {
        const int sd = flip_src(diso, f / S, f % S, S);
        const int sr = flip_src(riso, f / S, f % S, S);
        t1 += D[(size_t)(dr + sd / S) * dw + dc + sd % S] * (int32_t)rb[(size_t)(sr / S) * w + sr % S];
    }
    return t1;
}

// Seed champion of each range: the exact best of the first 32 entries of its bucket, first
// minimum by (rms, bucket index).  One warp per range: the range's canonical samples are
// staged once in shared memory, then lane e correlates entry e whole.  The domain's flip
// (flip_src) is affine in the canonical (i, j), so each lane walks its domain with two
// strides chosen once, and the warp reduces once.
template <int S>
__global__ void __launch_bounds__(256) fisher_seed_kernel(
    const uint8_t* __restrict__ plane, int w, const int32_t* __restrict__ D, int dw, int shift,
    int ncol_d, const uint32_t* __restrict__ rows, const uint32_t* __restrict__ cols,
    int nranges, const uint8_t* __restrict__ rbucket, const uint8_t* __restrict__ riso,
    const uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets,
    const uint32_t* __restrict__ list, const uint8_t* __restrict__ diso, RangeStats rs,
    DomainStats ds, FitParams fp, tc::SeedOut* __restrict__ out) {
    __shared__ uint8_t canon[8][S * S];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gw = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (gw >= nranges) return;
    const int b = rbucket[gw];
    if (b == 255 || counts[b] == 0) {
        if (lane == 0) out[gw] = tc::SeedOut{INFINITY, 0.0, kNone, 0};
        return;
    }
    const uint8_t* rb = plane + (size_t)rows[gw] * w + cols[gw];
    const int ri = riso[gw];
    for (int f = lane; f < S * S; f += 32) {
        const int sr = flip_src(ri, f / S, f % S, S);
        canon[warp][f] = rb[(size_t)(sr / S) * w + sr % S];
    }
    __syncwarp();
    const uint32_t n = counts[b] < 32u ? counts[b] : 32u;
    double best = INFINITY, best_sum = 0.0;
    uint32_t best_e = kNone;
    int32_t best_t1 = 0;
    if ((uint32_t)lane < n) {
        const uint32_t e = (uint32_t)lane;
        const uint32_t p = list[offsets[b] + e];
        const int dr = (int)(p / (uint32_t)ncol_d) * (shift / 2);
        const int dc = (int)(p % (uint32_t)ncol_d) * (shift / 2);
        // flip_src(iso, i, j) = (row, col) of the domain sample, affine in (i, j): the
        // sample's offset in D is o0 + i * oi + j * oj.
        int r0, c0, ri_i, ri_j, ci_i, ci_j;  // row = r0 + i ri_i + j ri_j, col likewise
        switch (diso[p]) {
            case 0: r0 = 0; ri_i = 1; ri_j = 0; c0 = 0; ci_i = 0; ci_j = 1; break;
            case 1: r0 = 0; ri_i = 0; ri_j = 1; c0 = S - 1; ci_i = -1; ci_j = 0; break;
            case 2: r0 = S - 1; ri_i = 0; ri_j = -1; c0 = 0; ci_i = 1; ci_j = 0; break;
            case 3: r0 = S - 1; ri_i = -1; ri_j = 0; c0 = S - 1; ci_i = 0; ci_j = -1; break;
            case 4: r0 = 0; ri_i = 1; ri_j = 0; c0 = S - 1; ci_i = 0; ci_j = -1; break;
            case 5: r0 = S - 1; ri_i = -1; ri_j = 0; c0 = 0; ci_i = 0; ci_j = 1; break;
            case 6: r0 = 0; ri_i = 0; ri_j = 1; c0 = 0; ci_i = 1; ci_j = 0; break;
            default: r0 = S - 1; ri_i = 0; ri_j = -1; c0 = S - 1; ci_i = -1; ci_j = 0; break;
        }
        const int32_t* d0 = D + (size_t)(dr + r0) * dw + dc + c0;
        const long long oi = (long long)ri_i * dw + ci_i, oj = (long long)ri_j * dw + ci_j;
        const uint8_t* rc = canon[warp];
        int32_t t1 = 0;
        for (int i = 0; i < S; ++i) {
            const int32_t* di = d0 + i * oi;
#pragma unroll
            for (int j = 0; j < S; ++j) t1 += di[j * oj] * (int32_t)rc[i * S + j];
        }
        const FitResult f = fit_exact(S * S, ds.s1x4[p], ds.s2x16[p], rs.t0[gw], t1, rs.t2[gw], fp);
        best = f.rms;
        best_sum = f.sum;
        best_e = e;
        best_t1 = t1;
    }
    double r = best;
    uint32_t ie = best_e;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double r2 = __shfl_xor_sync(0xffffffffu, r, o);
        const uint32_t e2 = __shfl_xor_sync(0xffffffffu, ie, o);
        if (r2 < r || (r2 == r && e2 < ie)) {
            r = r2;
            ie = e2;
        }
    }
    if (ie == best_e && ie != kNone) out[gw] = tc::SeedOut{best, best_sum, best_e, best_t1};
}

// Rank of each range within its bucket's group (rlist holds the ranges grouped by bucket).
__global__ void fisher_rank_kernel(const uint32_t* __restrict__ rlist, FisherPlan pl,
                                   uint32_t* __restrict__ rrank) {
    const int b = blockIdx.x;
    for (uint32_t k = threadIdx.x; k < pl.rcounts[b]; k += blockDim.x)
        rrank[rlist[pl.roffsets[b] + k]] = k;
}

// Each range's answer: the champion over its bucket's M-chunks by (rms, bucket index), then
// the candidate record (domain, isometry MAPPING[range iso][domain iso], exact fit).
__global__ void fisher_finish_kernel(const Partial* __restrict__ partials, FisherPlan pl,
                                     const uint8_t* __restrict__ rbucket,
                                     const uint8_t* __restrict__ riso,
                                     const uint32_t* __restrict__ rrank,
                                     const uint32_t* __restrict__ counts,
                                     const uint32_t* __restrict__ offsets,
                                     const uint32_t* __restrict__ list,
                                     const uint8_t* __restrict__ diso, int size, int shift,
                                     int ncol_d, int nranges, RangeStats rs, DomainStats ds,
                                     FitParams fp, CandidateOut* __restrict__ out,
                                     uint64_t* __restrict__ evals) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nranges) return;
    const int b = rbucket[r];
    CandidateOut c{0, 0, 0, 0, 0, 0, 0.0, 0, 0, 0, 0, 0, 0};
    if (b == 255 || counts[b] == 0) {
        out[r] = c;
        evals[r] = b == 255 ? 0 : counts[b];
        return;
    }
    const uint32_t k = rrank[r], rc = pl.rcounts[b];
    Partial best = partials[(size_t)pl.p_base[b] + k];
    for (uint32_t mc = 1; mc < pl.chunks[b]; ++mc) {
        const Partial q = partials[(size_t)pl.p_base[b] + (size_t)mc * rc + k];
        if (q.idx != kNone &&
            (best.idx == kNone || q.rms < best.rms || (q.rms == best.rms && q.idx < best.idx)))
            best = q;
    }
    evals[r] = counts[b];
    if (best.idx == kNone) {
        out[r] = c;
        return;
    }
    const uint32_t p = list[offsets[b] + best.idx];
    const int64_t n = (int64_t)size * size;
    const FitResult f = fit_exact(n, ds.s1x4[p], ds.s2x16[p], rs.t0[r], best.t1x4, rs.t2[r], fp);
    c.dom_row = (p / (uint32_t)ncol_d) * (uint32_t)shift;
    c.dom_col = (p % (uint32_t)ncol_d) * (uint32_t)shift;
    c.isometry = (uint32_t)fisher_mapping(riso[r], diso[p]);
    c.qalfa = f.qalfa;
    c.qbeta = f.qbeta;
    c.valid = 1;
    c.rms = f.rms;
    c.s0 = n;
    c.s1_x4 = ds.s1x4[p];
    c.s2_x16 = ds.s2x16[p];
    c.t0 = rs.t0[r];
    c.t1_x4 = best.t1x4;
    c.t2 = rs.t2[r];
    out[r] = c;
}

template <int S>
cudaError_t launch_level(const FisherTcArgs& a, cudaStream_t st) {
    constexpr int KG = kgroups(S);
    fisher_plan_kernel<<<1, 32, 0, st>>>(a.ix.counts, a.plan);
    fisher_rank_kernel<<<72, 128, 0, st>>>(a.rlist, a.plan, a.rrank);
    const long long ta = (long long)a.a_rows_max * KG;
    if (ta > 0)
        fisher_build_a_kernel<S><<<(unsigned)((ta + 255) / 256), 256, 0, st>>>(
            a.D, a.dw, a.shift, a.ncol_d, a.ix.counts, a.ix.offsets, a.ix.list, a.ix.diso, a.plan,
            a.aglob);
    const long long tb = (long long)a.b_rows_max * KG;
    if (tb > 0)
        fisher_build_b_kernel<S><<<(unsigned)((tb + 255) / 256), 256, 0, st>>>(
            a.plane, a.w, a.rows, a.cols, a.rlist, a.riso, a.plan, a.bglob);
    fisher_seed_kernel<S><<<(unsigned)((a.nranges * 32LL + 255) / 256), 256, 0, st>>>(
        a.plane, a.w, a.D, a.dw, a.shift, a.ncol_d, a.rows, a.cols, a.nranges, a.rbucket, a.riso,
        a.ix.counts, a.ix.offsets, a.ix.list, a.ix.diso, a.rs, a.ds, a.fp, a.seeds);
    const size_t smem = smem_bytes<S>();
    cudaError_t e = cudaFuncSetAttribute(fisher_tc_kernel<S>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (a.items_max > 0)
        fisher_tc_kernel<S><<<(unsigned)a.items_max, kThreads, smem, st>>>(
            a.aglob, a.bglob, a.plan, a.ix.counts, a.ix.offsets, a.ix.list, a.rlist, a.rs, a.ds,
            a.fp, a.seeds, a.partials, a.err, a.counter);
    fisher_finish_kernel<<<(a.nranges + 127) / 128, 128, 0, st>>>(
        a.partials, a.plan, a.rbucket, a.riso, a.rrank, a.ix.counts, a.ix.offsets, a.ix.list,
        a.ix.diso, a.size, a.shift, a.ncol_d, a.nranges, a.rs, a.ds, a.fp, a.out, a.evals);
    return cudaGetLastError();
}

}  // namespace

bool supported(int size, int shift) {
    return (size == 4 || size == 8 || size == 16) && shift >= 2 && (shift & 1) == 0;
}

// Operand bytes of one 128-row tile (all K stages) at a supported size.
size_t tile_bytes(int size, bool a) {
    const int s = size == 16 ? 16 : (size == 8 ? 8 : 4);
    return (size_t)kstages(s) * (size_t)(a ? a_stage_bytes(s) : b_stage_bytes(s));
}
size_t a_bytes(int size, size_t npos) { return (npos / kM + 73) * tile_bytes(size, true); }
size_t b_bytes(int size, size_t nranges) { return (nranges / kNt + 73) * tile_bytes(size, false); }
size_t a_rows_max(size_t npos) { return (npos / kM + 73) * kM; }
size_t b_rows_max(size_t nranges) { return (nranges / kNt + 73) * kNt; }
size_t items_max(size_t nranges) { return nranges / kNt + 73 + 72 * 15; }
size_t partials_max(size_t nranges) { return kMaxChunkItems * nranges + 72; }

cudaError_t launch_range_classes(const uint8_t* plane, int w, int h, int size,
                                 const uint32_t* rows, const uint32_t* cols, int nranges,
                                 const uint32_t* ref, uint8_t* rbucket, uint8_t* riso,
                                 cudaStream_t st) {
    if (nranges <= 0) return cudaSuccess;
    fisher_range_kernel<<<(nranges + 127) / 128, 128, 0, st>>>(plane, w, h, size, rows, cols,
                                                               nranges, ref, rbucket, riso);
    return cudaGetLastError();
}

cudaError_t launch_search(const FisherTcArgs& a, cudaStream_t st) {
    if (a.nranges <= 0) return cudaSuccess;
    switch (a.size) {
        case 4: return launch_level<4>(a, st);
        case 8: return launch_level<8>(a, st);
        case 16: return launch_level<16>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ftc
}  // namespace mars
