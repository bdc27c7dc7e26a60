// Tensor-core (tcgen05, sm_100a) domain-range correlation with the fused exact-bound
// epilogue.
//
// For one quadtree level (block size S, domain stride `shift` in {2, 4, 8, 16}) the
// correlations t1'(domain, range, isometry) = sum_{y,x} P[dom_row+y][dom_col+x] *
// (r[map_k(y/2, x/2)] - 128) over the 2S x 2S pixel block of a domain are one exact int8
// GEMM with INT32 accumulation:
//   A (M = 128 lanes)  = 128 consecutive domain positions of one domain row, K-major:
//                        each domain's pixels, grouped in 16-byte K-groups (pixel row y,
//                        16-pixel column group j); u8.
//   B (N = 256)        = 32 range blocks x 8 isometries: the range pixel r[map_k(u, v)]
//                        minus 128, upsampled 2x2 onto the same K positions; s8.  Zero on
//                        K positions past 2S (S = 4 pads each pixel row to 16 bytes).
//   D (TMEM, 128 x 256 int32) = t1' = t1_x4 - 128 * s1_x4, exact (|t1'| < 2^31).
// The pixel sum over the 2x2 box that the reference folds into D = 4d
// (Contracted::build, crates/mars-codec/src/encode.rs:478-502) is folded into K instead,
// so every operand is a plain u8 pixel or an s8 range sample and nothing rounds.
//
// A is fed by TMA from `shift`-phase copies of the plane: copy p holds the plane shifted
// left by shift*p pixels, so the P = 16/shift domains of one 16-byte column group start on
// 16-byte boundaries and 8 consecutive same-phase domains' K-group is one contiguous
// 128-byte row segment -- exactly one 8 x 16 B core matrix of the SWIZZLE_NONE K-major
// canonical layout.  A 128 B x 8-row TMA box therefore lands as 8 core matrices along K
// (LBO = 128 B), and the 16 boxes of a stage are 16 row groups (SBO = 1024 B).  B is
// pre-built in global memory in the same core-matrix order and copied with 1-D bulk
// copies.
//
// Warp roles (320 threads): warp 0 issues the loads, warp 1 owns TMEM and issues the MMAs
// (one elected lane), warps 2-9 are the epilogue (TMEM lane quadrant = warp % 4, two warps
// per quadrant splitting the 256 columns, 16 ranges each).  (Sixteen epilogue warps of 8
// ranges each measured slower: the per-tile barriers, not the issue slots, set the pace.)  The accumulator is double-buffered in TMEM
// (2 x 256 columns).  The epilogue runs the pruning test of fit.cuh once per (domain
// lane, range) -- shared by the 8 isometry columns -- and queues survivors in shared
// memory; batches of survivors get the exact f64 fit and update the ranges' champions
// and thresholds.
// Every mbarrier wait is bounded (clock64 deadline): on expiry the kernel records an
// error, stops issuing work, waits (bounded) for its own loads, frees TMEM and returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"
#include "tc.cuh"

namespace mars {
namespace tc {
namespace {

constexpr int kEpiWarps = 8;                    // 2 per TMEM lane quadrant
constexpr int kThreads = 64 + 32 * kEpiWarps;   // 10 warps: load, MMA, 8 epilogue
constexpr int kEpiThreads = 32 * kEpiWarps;
constexpr int kColsPerWarp = 4 * 256 / kEpiWarps;  // accumulator columns per epilogue warp
constexpr int kRangesPerWarp = kColsPerWarp / 8;
constexpr int kChunks = kColsPerWarp / 32;         // 32-column TMEM loads per pass
constexpr int kM = 128;
constexpr int kN = 256;
constexpr int kRangesPerTile = kN / 8;         // 32
constexpr int kStageA = 16 * 1024;             // 16 row groups x 8 K-groups x 128 B
constexpr int kStageB = 32 * 1024;             // 32 row groups x 8 K-groups x 128 B
constexpr int kQueueCap = 2048;                // survivors the queue can hold
// Each epilogue warp owns kWarpCap consecutive queue entries and its own count, so no warp
// reads a count another warp may still be adding to; the queue is drained when any warp's
// region holds kWarpFlush entries.
constexpr int kWarpCap = kQueueCap / kEpiWarps;  // 256
constexpr int kWarpFlush = 48;
constexpr long long kWaitCycles = 4000000000ll;  // ~2 s at 1.965 GHz

// Pipeline depth: as many A stages as fit beside the resident B tile (S <= 8), otherwise
// three stages of A + B.
__host__ __device__ constexpr int stages_for(int S) { return S == 4 ? 6 : (S == 8 ? 4 : 3); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// One bounded poll of an mbarrier phase.  The suspend-time hint lets the hardware park
// the waiting thread until the phase completes (or ~20 us pass) instead of spinning, so
// waiting warps leave the issue slots to the epilogue warps sharing their scheduler.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(20000u)
        : "memory");
    return ok != 0;
}

// Bounded wait: false when the deadline passed or another warp already gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                          int* err_global, int code) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (*abort_flag) return false;
        if (clock64() - t0 > kWaitCycles) {
            *abort_flag = 1;
            atomicOr(err_global, code);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(0), "r"(0), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(dst)),
        "l"((uint64_t)src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// SWIZZLE_NONE K-major shared-memory matrix descriptor: core matrices of 8 rows x 16 B,
// LBO = 128 B between K-adjacent core matrices, SBO = 1024 B between 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)(128u >> 4) << 16;
    d |= (uint64_t)(1024u >> 4) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100
    return d;                // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor, kind::i8: D = s32, A = u8, B = s8, both K-major, M = 128, N = 256.
constexpr uint32_t kIdesc = (2u << 4) | (0u << 7) | (1u << 10) | ((uint32_t)(kN >> 3) << 17) |
                            ((uint32_t)(kM >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// TMEM -> registers, 32 columns of this warp's 32 lanes.  The load completes
// asynchronously: tmem_wait() names the destination registers as read-write operands so
// no consumer can be scheduled ahead of it.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, int32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
          "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
          "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
          "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
          "=r"(v[31])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait(int32_t (&v)[32]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]),
                   "+r"(v[6]), "+r"(v[7]), "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]),
                   "+r"(v[12]), "+r"(v[13]), "+r"(v[14]), "+r"(v[15]), "+r"(v[16]), "+r"(v[17]),
                   "+r"(v[18]), "+r"(v[19]), "+r"(v[20]), "+r"(v[21]), "+r"(v[22]), "+r"(v[23]),
                   "+r"(v[24]), "+r"(v[25]), "+r"(v[26]), "+r"(v[27]), "+r"(v[28]), "+r"(v[29]),
                   "+r"(v[30]), "+r"(v[31])
                 :
                 : "memory");
}

__device__ __forceinline__ void epi_barrier() {
    asm volatile("bar.sync 1, %0;" ::"n"(kEpiThreads) : "memory");
}

// Named barrier over the epilogue warps that also ANDs a predicate across them, so the
// warps always agree on whether to go on.
__device__ __forceinline__ bool epi_barrier_and(bool pred) {
    uint32_t out;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, 1, %2, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(out)
        : "r"((uint32_t)pred), "n"(kEpiThreads)
        : "memory");
    return out != 0;
}

// Champion of one range block (reference order: smaller rms, then smaller index).
struct Champ {
    double rms, sum, rms0;
    int64_t nrr;
    uint32_t idx;
    int32_t t0, t2, valid;
    int32_t t1x4;  // the champion's exact correlation, handed to the finish kernel
};

// The per-range pruning record the epilogue reads for every (domain lane, range) pair,
// branch-free form of prune_below (fit.cuh):
//   g1 = sqrt_w * sqrt(Ndd);  tau_z = min(w2a + a_half*Ndd, max(g1, a_min*Ndd));
//   tau = (dom > tie) ? tau_z : g1 + neg;   prune  <=>  t1' < s1_x4 * c + 4 tau / n.
// tie = -1 puts every domain in the Z-form, INT32_MAX none; neg = 0 or -inf (W <= 0).
// Since tau_z >= g1 whenever W > 0 (W/(2a) + a*Ndd/2 >= sqrt(W*Ndd) by the AM-GM
// inequality, and max(g1, .) >= g1), the short form  t1' < s1_x4 * c + (g1 + neg) * 4/n
// is a valid threshold for every range with W > 0, whatever its tie mode; it is also the
// exact threshold outside the Z-form.  It differs from the full one only when
// a_min^2 * Ndd > W, which the best candidates of a range almost never meet, so it prunes
// the same candidates at a third of the instructions.  `full` marks the ranges that need
// the full form: a Z-form range with W <= 0, for which the short form prunes nothing.
struct __align__(16) ThrRec {
    float sqrt_w, w2a, neg, c;  // sqrt_w, w2a, neg pre-scaled by 4 / n (exact: n = 4^k)
    int32_t tie, full, pad1, pad2;
};

// A survivor waiting for its exact fit.  Survivors of several tiles are batched: the
// queue is drained when a warp's region holds kWarpFlush entries, when a tile overflows a
// region, and at the end.
struct __align__(8) QEntry {
    int32_t t1;     // t1' = t1_x4 - 128 * s1_x4
    uint32_t dom;   // domain position index (row-major)
    uint32_t code;  // tile tag << 16 | lane << 8 | tile column (range * 8 + iso)
    uint32_t pad;
    double rms, sum;
};

struct Smem {
    uint64_t full[kMaxStages];
    uint64_t empty[kMaxStages];
    uint64_t tfull[2];
    uint64_t tempty[2];
    uint64_t bres;
    uint32_t tmem_base;
    int abort_flag;
    int wcount[kEpiWarps];  // entries each epilogue warp queued (may exceed kWarpCap)
    uint32_t full_bits;     // bit r: range r of the tile needs the full threshold form
    unsigned long long key_rms[kRangesPerTile];  // per-pass winner: f64 bits (rms >= 0)
    uint32_t key_idx[kRangesPerTile];
    double key_sum[kRangesPerTile];
    int32_t key_t1[kRangesPerTile];
    ThrRec thr[kRangesPerTile];
    Champ ch[kRangesPerTile];
    uint32_t evaluated[kM * kN / 32];           // candidates already fitted in this tile
    QEntry queue[kQueueCap];
};

__device__ __forceinline__ int domain_of_lane(int m, int P, int tile_q0) {
    const int g = m >> 3, r8 = m & 7;
    const int per_phase = 16 / P;
    const int p = g / per_phase, h = g % per_phase;
    return P * (tile_q0 + 8 * h + r8) + p;
}

__device__ __forceinline__ void publish_threshold(Smem& sm, int rl, const FitParams& fp, int n) {
    const Champ& C = sm.ch[rl];
    ThrRec t;
    if (!C.valid) {
        // An invalid range never survives: in the Z-form (tie = -1) with sqrt_w = w2a =
        // +inf, tau = +inf for every domain, flat all-zero ones (s1 = 0) included; in the
        // short form g1 = +inf (sqrt(Ndd) > 0 always: +huge for a flat domain).
        t = ThrRec{INFINITY, INFINITY, 0.0f, 3.0e38f, -1, 0, 0, 0};
        sm.thr[rl] = t;
        atomicAnd(&sm.full_bits, ~(1u << rl));
        return;
    }
    const Threshold th = make_threshold(C.sum, C.rms, C.idx >> 3, C.rms0, C.nrr, n, fp);
    // Scaling by 4 / n (a power of two) is exact, so folding it in keeps every bound
    // rounded toward -inf.
    const float four_inv_n = 4.0f / (float)n;
    t.sqrt_w = th.sqrt_w * four_inv_n;
    t.w2a = th.w2a * four_inv_n;
    t.neg = th.wpos ? 0.0f : -INFINITY;
    t.c = (float)C.t0 / (float)n - 128.0f;  // exact: t0 < 2^24, n a power of four
    t.tie = th.mode == 2 ? -1 : (th.mode == 1 ? (int32_t)th.tie_dom : INT32_MAX);
    t.full = th.mode != 0 && !th.wpos;
    t.pad1 = t.pad2 = 0;
    sm.thr[rl] = t;
    if (t.full)
        atomicOr(&sm.full_bits, 1u << rl);
    else
        atomicAnd(&sm.full_bits, ~(1u << rl));
}

// Exact fits of every queued survivor, then the per-range winners of the batch (atomic
// min on the f64 bit pattern of rms >= 0, then on the reference index) and the champion /
// threshold update.  All epilogue threads call this together, after a barrier, so every
// warp's count is final.  Entry qi is live when it lies inside its warp's filled part.
__device__ __forceinline__ bool queued_entry(const Smem& sm, int qi) {
    return (qi % kWarpCap) < sm.wcount[qi / kWarpCap];
}

template <int N>
__device__ __noinline__ void drain_queue(Smem& sm, bool mark, uint32_t tag, int et,
                                         const DomainStats& ds, const FitParams& fp,
                                         unsigned long long& exact) {
    for (int qi = et; qi < kQueueCap; qi += kEpiThreads) {
        if (!queued_entry(sm, qi)) continue;
        QEntry& q = sm.queue[qi];
        const int rl = (int)(q.code & 255u) >> 3;
        const Champ& C = sm.ch[rl];
        const int32_t s1 = ds.s1x4[q.dom];
        const int64_t t1x4 = (int64_t)q.t1 + 128ll * s1;
        const FitResult f = fit_exact(N, s1, ds.s2x16[q.dom], C.t0, t1x4, C.t2, fp);
        q.rms = f.rms;
        q.sum = f.sum;
        ++exact;
        atomicMin(&sm.key_rms[rl], (unsigned long long)__double_as_longlong(f.rms));
    }
    epi_barrier();
    for (int qi = et; qi < kQueueCap; qi += kEpiThreads) {
        if (!queued_entry(sm, qi)) continue;
        const QEntry& q = sm.queue[qi];
        const int col = (int)(q.code & 255u), rl = col >> 3;
        if ((unsigned long long)__double_as_longlong(q.rms) == sm.key_rms[rl])
            atomicMin(&sm.key_idx[rl], q.dom * 8u + (uint32_t)(col & 7));
    }
    epi_barrier();
    for (int qi = et; qi < kQueueCap; qi += kEpiThreads) {
        if (!queued_entry(sm, qi)) continue;
        const QEntry& q = sm.queue[qi];
        const int col = (int)(q.code & 255u), rl = col >> 3;
        if ((unsigned long long)__double_as_longlong(q.rms) == sm.key_rms[rl] &&
            q.dom * 8u + (uint32_t)(col & 7) == sm.key_idx[rl]) {
            sm.key_sum[rl] = q.sum;
            sm.key_t1[rl] = q.t1 + 128 * ds.s1x4[q.dom];  // t1_x4, exact in int32 (S <= 64)
        }
        if (mark && (q.code >> 16) == tag) {
            // A region overflowed in this tile: remember what was fitted so the next pass
            // over the same accumulator only queues candidates not yet seen.
            const int qm = (int)(q.code >> 8) & 127;
            atomicOr(&sm.evaluated[(qm * kN + col) >> 5], 1u << (col & 31));
        }
    }
    epi_barrier();
    if (et < kRangesPerTile && sm.key_rms[et] != ~0ull) {
        Champ& C = sm.ch[et];
        const double r2 = __longlong_as_double((long long)sm.key_rms[et]);
        const uint32_t i2 = sm.key_idx[et];
        if (C.valid && (r2 < C.rms || (r2 == C.rms && i2 < C.idx))) {
            C.rms = r2;
            C.idx = i2;
            C.sum = sm.key_sum[et];
            C.t1x4 = sm.key_t1[et];
            publish_threshold(sm, et, fp, N);
        }
        sm.key_rms[et] = ~0ull;
        sm.key_idx[et] = UINT32_MAX;
    }
    epi_barrier();
    if (et < kEpiWarps) sm.wcount[et] = 0;
    epi_barrier();
}

template <int S>
__global__ void __launch_bounds__(kThreads, 1)
    corr_tc_kernel(const __grid_constant__ TcMaps maps, const uint8_t* __restrict__ bglob,
                   LevelGeom g, int nranges, RangeStats rs, DomainStats ds, FitParams fp,
                   const SeedOut* __restrict__ seeds, int m_tiles, int m_per_cta,
                   Partial* __restrict__ partials, int* __restrict__ err,
                   unsigned long long* __restrict__ exact_counter) {
    constexpr int N = S * S;
    constexpr int J = S >= 8 ? S / 8 : 1;  // 16-byte column groups per pixel row
    constexpr int ROWS = 2 * S;            // pixel rows of a domain block
    constexpr int KST = J * ROWS / 8;      // 128-byte K stages per tile
    constexpr bool kBRes = KST <= 2;       // B tile stays resident in shared memory
    constexpr int kStages = stages_for(S);
    constexpr uint32_t kTxStage = kBRes ? kStageA : kStageA + kStageB;

    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char* stA = base;                                  // kStages x 16 KB
    unsigned char* stB = stA + kStages * kStageA;               // kStages x 32 KB or resident
    unsigned char* after_b = stB + (kBRes ? KST * kStageB : kStages * kStageB);
    Smem& sm = *reinterpret_cast<Smem*>(after_b);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntile = blockIdx.x;
    const int m_begin = blockIdx.y * m_per_cta;
    const int m_end = min(m_tiles, m_begin + m_per_cta);
    const int P = 16 / g.shift;
    const int tiles_per_row = (g.ncol_d + kM - 1) / kM;
    const uint8_t* btile = bglob + (size_t)ntile * KST * kStageB;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&sm.full[s], 1);
            mbar_init(&sm.empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&sm.tfull[b], 1);
            mbar_init(&sm.tempty[b], kEpiThreads);
        }
        mbar_init(&sm.bres, 1);
        sm.abort_flag = 0;
        for (int w = 0; w < kEpiWarps; ++w) sm.wcount[w] = 0;
        sm.full_bits = 0u;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = threadIdx.x; i < kM * kN / 32; i += kThreads) sm.evaluated[i] = 0u;
    if (threadIdx.x < kRangesPerTile) {
        Champ& C = sm.ch[threadIdx.x];
        const int r = ntile * kRangesPerTile + threadIdx.x;
        C.valid = r < nranges && seeds[r].idx != UINT32_MAX;
        if (C.valid) {
            C.t0 = rs.t0[r];
            C.t2 = rs.t2[r];
            C.nrr = rs.nrr[r];
            C.rms0 = rs.rms0[r];
            const SeedOut sd = seeds[r];
            C.rms = sd.rms;
            C.sum = sd.sum;
            C.idx = sd.idx;
            C.t1x4 = sd.t1x4;
        } else {
            // Padding of the last N tile, or a block outside the plane: no candidate.
            C.rms = INFINITY;
            C.sum = 0.0;
            C.idx = UINT32_MAX;
            C.t1x4 = 0;
        }
        sm.key_rms[threadIdx.x] = ~0ull;
        sm.key_idx[threadIdx.x] = UINT32_MAX;
    }
    __syncthreads();  // full_bits and the champions are set before the records
    if (threadIdx.x < kRangesPerTile) publish_threshold(sm, threadIdx.x, fp, N);
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
            if (kBRes) {
                mbar_expect_tx(&sm.bres, KST * kStageB);
                for (int t = 0; t < KST; ++t)
                    bulk_load(stB + t * kStageB, btile + (size_t)t * kStageB, kStageB, &sm.bres);
            }
            for (int mt = m_begin; mt < m_end && !*abort_flag; ++mt) {
                const int a = mt / tiles_per_row;
                const int q0 = (mt % tiles_per_row) * (kM / P);
                const int dom_row = a * g.shift;
                for (int t = 0; t < KST; ++t) {
                    if (issued >= kStages && !mbar_wait(&sm.empty[s], ph ^ 1, abort_flag, err, 1)) break;
                    mbar_expect_tx(&sm.full[s], kTxStage);
                    const int kg0 = t * 8;
                    const int j = kg0 / ROWS, y0 = kg0 % ROWS;
                    unsigned char* dstA = stA + s * kStageA;
                    if (maps.use_all) {
                        tma_load_4d(dstA, &maps.all, 16 * (q0 + j), dom_row + y0, &sm.full[s]);
                    } else {
                        const int per_phase = 16 / P;
#pragma unroll 1
                        for (int gg = 0; gg < 16; ++gg) {
                            const int p = gg / per_phase, h = gg % per_phase;
                            tma_load_2d(dstA + gg * 1024, &maps.m[p], 16 * (q0 + 8 * h + j),
                                        dom_row + y0, &sm.full[s]);
                        }
                    }
                    if (!kBRes)
                        bulk_load(stB + s * kStageB, btile + (size_t)t * kStageB, kStageB, &sm.full[s]);
                    ++issued;
                    if (++s == kStages) {
                        s = 0;
                        ph ^= 1;
                    }
                }
            }
            // Drain: wait (bounded) for the loads still in flight before leaving.
            if (*abort_flag) {
                int s2 = s;
                uint32_t ph2 = ph;
                for (int i = 0; i < kStages && i < issued; ++i) {
                    if (--s2 < 0) {
                        s2 = kStages - 1;
                        ph2 ^= 1;
                    }
                    const long long t0 = clock64();
                    while (!mbar_try_wait(&sm.full[s2], ph2) && clock64() - t0 < kWaitCycles) {
                    }
                }
            }
        }
    } else if (warp == 1) {
        // ---------------------------------------------------------------- MMA
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            bool ok = true;
            if (kBRes) ok = mbar_wait(&sm.bres, 0, abort_flag, err, 2);
            int i = 0;
            for (int mt = m_begin; ok && mt < m_end; ++mt, ++i) {
                const int b = i & 1;
                const uint32_t bph = (uint32_t)((i >> 1) & 1);
                if (i >= 2 && !mbar_wait(&sm.tempty[b], bph ^ 1, abort_flag, err, 4)) break;
                tmem_fence_after();
                const uint32_t dcol = tmem + (uint32_t)(b * kN);
                for (int t = 0; t < KST; ++t) {
                    if (!mbar_wait(&sm.full[s], ph, abort_flag, err, 8)) {
                        ok = false;
                        break;
                    }
                    tmem_fence_after();
                    const uint32_t a_addr = smem_u32(stA + s * kStageA);
                    const uint32_t b_addr = smem_u32(kBRes ? stB + t * kStageB : stB + s * kStageB);
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk)
                        mma_i8(dcol, smem_desc(a_addr + kk * 256), smem_desc(b_addr + kk * 256),
                               (t > 0 || kk > 0) ? 1u : 0u);
                    mma_commit(&sm.empty[s]);
                    if (++s == kStages) {
                        s = 0;
                        ph ^= 1;
                    }
                }
                if (!ok) break;
                mma_commit(&sm.tfull[b]);
            }
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------------------- epilogue
        // Warps 2..: TMEM lane quadrant = warp % 4; column part (kRangesPerWarp ranges from
        // part * kRangesPerWarp) = which of the quadrant's warps.
        const int et = threadIdx.x - 64;         // 0..kEpiThreads-1
        const int ew = et >> 5;                  // epilogue warp 0..kEpiWarps-1
        const int e = warp & 3;
        const int part = (warp - 2) >> 2;
        const int m = e * 32 + lane;             // this thread's domain lane
        const float four_inv_n = 4.0f / (float)N;
        unsigned long long exact = 0;

        // This lane's domain statistics, prefetched one tile ahead.  The lane's column
        // offset within a tile is fixed (domain_of_lane is P * (q0 + 8h + r8) + p), and
        // the tile's domain row and column step forward with mt, so no division runs per
        // tile.
        const int lane_col = domain_of_lane(m, P, 0);
        const int tile_cols = kM;  // domain columns a tile spans: (kM / P) groups of P
        int nx_a = m_begin / tiles_per_row, nx_t = m_begin % tiles_per_row;
        auto load_dom = [&](int mt, float& s1f, float& detf, float& sdetf, int& dom) {
            if (mt >= m_end) return;
            const int c = nx_t * tile_cols + lane_col;
            if (c < g.ncol_d) {
                dom = nx_a * g.ncol_d + c;
                s1f = (float)ds.s1x4[dom];
                detf = ds.detf[dom];
                sdetf = ds.sdetf[dom];
            } else {
                dom = -1;
            }
            if (++nx_t == tiles_per_row) {
                nx_t = 0;
                ++nx_a;
            }
        };
        float n_s1 = 0.f, n_det = 0.f, n_sdet = 0.f;
        int n_dom = -1;
        load_dom(m_begin, n_s1, n_det, n_sdet, n_dom);

        int i = 0;
        for (int mt = m_begin; mt < m_end; ++mt, ++i) {
            const int b = i & 1;
            const uint32_t bph = (uint32_t)((i >> 1) & 1);
            const float s1f = n_s1, detf = n_det, sdetf = n_sdet;
            const int dom = n_dom;
            load_dom(mt + 1, n_s1, n_det, n_sdet, n_dom);
            // a_min * Ndd and a_min/2 * Ndd, pre-scaled by 4 / n like the range records.
            const float ad = __fmul_rd(fp.a_min, detf) * four_inv_n;
            const float ahd = __fmul_rd(fp.a_half, detf) * four_inv_n;
            const uint32_t tcol =
                tmem + ((uint32_t)(e * 32) << 16) + (uint32_t)(b * kN + part * kColsPerWarp);
            bool rescan = false;

            // Max of 8 accumulator columns with three-input integer max instructions.
            auto max8 = [](const int32_t (&v)[32], int o) {
                return __vimax3_s32(__vimax3_s32(v[o], v[o + 1], v[o + 2]),
                                    __vimax3_s32(v[o + 3], v[o + 4], v[o + 5]),
                                    max(v[o + 6], v[o + 7]));
            };
            const uint32_t tag = (uint32_t)(mt & 0xFFFF);
            // Thresholds of this lane's domain against its ranges (fit.cuh, branch-free
            // form).  They do not depend on the accumulator; each stage below runs over all
            // of them so the independent chains overlap.
            int32_t thr[kRangesPerWarp];
            auto all_thresholds = [&]() {
                const float4* rec = reinterpret_cast<const float4*>(sm.thr);
                const uint32_t fullw = (sm.full_bits >> (part * kRangesPerWarp)) &
                                       ((1u << kRangesPerWarp) - 1u);
                if (fullw == 0u) {
                    // Short form for every range: s1 * c + (g1 + neg), each step rounded
                    // toward -inf (the inner fma is exactly fmul_rd(sqrt_w, sqrt(Ndd))
                    // plus 0 or -inf).
#pragma unroll
                    for (int r = 0; r < kRangesPerWarp; ++r) {
                        const float4 ra = rec[2 * (part * kRangesPerWarp + r)];
                        const float g = __fmaf_rd(ra.x, sdetf, ra.z);
                        thr[r] = dom < 0 ? INT32_MAX : __float2int_rd(__fmaf_rd(s1f, ra.w, g));
                    }
                    return;
                }
                float4 ra[kRangesPerWarp];
                int4 rb[kRangesPerWarp];
#pragma unroll
                for (int r = 0; r < kRangesPerWarp; ++r) {
                    ra[r] = rec[2 * (part * kRangesPerWarp + r)];
                    rb[r] = reinterpret_cast<const int4*>(rec)[2 * (part * kRangesPerWarp + r) + 1];
                }
                // s1 * c + tau with one rounding toward -inf (fma): still never above the
                // exact threshold.
                float tau[kRangesPerWarp];
#pragma unroll
                for (int r = 0; r < kRangesPerWarp; ++r) {
                    const float g1 = __fmul_rd(ra[r].x, sdetf);
                    const float tz = fminf(__fadd_rd(ra[r].y, ahd), fmaxf(g1, ad));
                    tau[r] = dom > rb[r].x ? tz : __fadd_rd(g1, ra[r].z);
                }
#pragma unroll
                for (int r = 0; r < kRangesPerWarp; ++r)
                    thr[r] = dom < 0 ? INT32_MAX : __float2int_rd(__fmaf_rd(s1f, ra[r].w, tau[r]));
            };
            auto test_chunk = [&](const int32_t (&v)[32], int ch) {
                const int32_t t0 = thr[ch * 4], t1 = thr[ch * 4 + 1];
                const int32_t t2 = thr[ch * 4 + 2], t3 = thr[ch * 4 + 3];
                const bool any = (max8(v, 0) >= t0) | (max8(v, 8) >= t1) | (max8(v, 16) >= t2) |
                                 (max8(v, 24) >= t3);
                if (any) {
                    // Rare: bit c of `mask` = column c of this chunk survives (and was not
                    // fitted by an earlier pass over this accumulator).
                    uint32_t mask = 0u;
#pragma unroll
                    for (int c = 0; c < 32; ++c) {
                        const int32_t tc = c < 8 ? t0 : (c < 16 ? t1 : (c < 24 ? t2 : t3));
                        mask |= (v[c] >= tc ? 1u : 0u) << c;
                    }
                    const int col0 = part * kColsPerWarp + ch * 32;
                    if (rescan) mask &= ~sm.evaluated[(m * kN + col0) >> 5];
                    int slot = atomicAdd(&sm.wcount[ew], __popc(mask));
                    while (mask) {
                        const int c = __ffs(mask) - 1;
                        mask &= mask - 1;
                        int32_t val = v[0];
#pragma unroll
                        for (int q = 1; q < 32; ++q) val = c == q ? v[q] : val;
                        if (slot < kWarpCap)
                            sm.queue[ew * kWarpCap + slot] =
                                QEntry{val, (uint32_t)dom, (uint32_t)(tag << 16 | m << 8 | (col0 + c)),
                                       0u, 0.0, 0.0};
                        ++slot;
                    }
                }
            };
            all_thresholds();  // overlaps the MMAs of this tile
            // Every warp waits for the accumulator on its own and scans it; one barrier per
            // pass makes the warps agree to go on (a warp whose bounded wait gave up scans
            // nothing and votes to stop) and tells them whether a drain is due.  The result
            // of the wait is made warp-uniform, so the scan's aligned TMEM loads run with
            // every lane.
            bool got = __all_sync(0xffffffffu, mbar_wait(&sm.tfull[b], bph, abort_flag, err, 16));
            bool first = true;
            for (;;) {
                if (got) {
                    if (first) tmem_fence_after();
                    // ---- scan: this thread's accumulator columns in 32-column chunks, each
                    // chunk's load overlapped with the previous chunk's test
                    static_assert(kChunks % 2 == 0, "chunks are scanned in pairs");
                    int32_t va[32], vb[32];
                    __syncwarp();
                    tmem_ld32(tcol, va);
                    tmem_wait(va);
#pragma unroll
                    for (int ch = 0; ch < kChunks; ch += 2) {
                        tmem_ld32(tcol + 32u * (ch + 1), vb);
                        test_chunk(va, ch);
                        __syncwarp();
                        tmem_wait(vb);
                        if (ch + 2 < kChunks) tmem_ld32(tcol + 32u * (ch + 2), va);
                        test_chunk(vb, ch + 1);
                        __syncwarp();
                        if (ch + 2 < kChunks) tmem_wait(va);
                    }
                }
                first = false;
                // Common case: every warp got its accumulator and no region needs draining.
                // This warp's count is final here (its lanes' atomics are done).
                __syncwarp();
                const bool last = mt + 1 == m_end;
                if (epi_barrier_and(got && !last && sm.wcount[ew] < kWarpFlush)) break;
                // Rare: some warp gave up waiting (stop), or a drain is due.
                if (!epi_barrier_and(got)) {
                    got = false;
                    break;
                }
                bool over = false;
#pragma unroll
                for (int w2 = 0; w2 < kEpiWarps; ++w2) over |= sm.wcount[w2] > kWarpCap;
                drain_queue<N>(sm, over, tag, et, ds, fp, exact);
                if (over) {
                    rescan = true;
                    all_thresholds();
                    continue;  // pass again over the same accumulator
                }
                break;
            }
            if (!got) break;
            if (rescan) {
                for (int w2 = et; w2 < kM * kN / 32; w2 += kEpiThreads) sm.evaluated[w2] = 0u;
                epi_barrier();
            }
            // The accumulator has been read completely: hand it back to the MMA warp.
            tmem_fence_before();
            mbar_arrive(&sm.tempty[b]);
        }
        if (exact_counter && exact) atomicAdd(exact_counter, exact);
    }

    tmem_fence_before();
    __syncthreads();
    if (warp == 1) {
        tmem_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
    }
    if (threadIdx.x < kRangesPerTile) {
        const Champ& C = sm.ch[threadIdx.x];
        const int r = ntile * kRangesPerTile + threadIdx.x;
        if (r < nranges) {
            Partial p;
            p.rms = C.rms;
            p.sum = C.sum;
            p.idx = C.idx;
            p.t1x4 = C.t1x4;
            p.qalfa = 0;
            p.qbeta = 0;
            p.pad = 0;
            partials[(size_t)blockIdx.y * nranges + r] = p;
        }
    }
}

// B operand of one level: rows n = range * 8 + isometry; for each 256-row N tile and each
// 128-byte K stage, 32 row groups x 8 K-groups x (8 rows x 16 B).
template <int S>
__global__ void build_b_kernel(const uint8_t* __restrict__ plane, int w, int h,
                               const uint32_t* rows, const uint32_t* cols, int nranges,
                               int ntiles, uint8_t* __restrict__ out) {
    constexpr int J = S >= 8 ? S / 8 : 1;
    constexpr int ROWS = 2 * S;
    constexpr int KG = J * ROWS;
    constexpr int KST = KG / 8;
    // one thread per (n, kg): writes one 16-byte K-group of one B row
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)ntiles * kN * KG;
    if (tid >= total) return;
    const int kg = (int)(tid % KG);
    const long long nglob = tid / KG;
    const int nt = (int)(nglob / kN), n = (int)(nglob % kN);
    const int r = nt * kRangesPerTile + n / 8, k = n % 8;
    const int j = kg / ROWS, y = kg % ROWS;
    const int t = kg / 8, kgl = kg % 8;
    const bool inside = r < nranges && rows[r] + (uint32_t)S <= (uint32_t)h &&
                        cols[r] + (uint32_t)S <= (uint32_t)w;
    uint8_t bytes[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        const int x = 16 * j + e;
        int8_t val = 0;
        if (inside && x < 2 * S) {
            const int u = y >> 1, vv = x >> 1;
            int i, jj;
            switch (k) {
                case 0: i = u; jj = vv; break;
                case 1: i = S - 1 - vv; jj = u; break;
                case 2: i = vv; jj = S - 1 - u; break;
                case 3: i = S - 1 - u; jj = S - 1 - vv; break;
                case 4: i = u; jj = S - 1 - vv; break;
                case 5: i = S - 1 - u; jj = vv; break;
                case 6: i = vv; jj = u; break;
                default: i = S - 1 - vv; jj = S - 1 - u; break;
            }
            val = (int8_t)((int)plane[(size_t)(rows[r] + i) * w + cols[r] + jj] - 128);
        }
        bytes[e] = (uint8_t)val;
    }
    const size_t off = (((size_t)nt * KST + t) * 32 + (n >> 3)) * 1024 + (size_t)kgl * 128 +
                       (size_t)(n & 7) * 16;
    uint4 pk;
    pk.x = bytes[0] | bytes[1] << 8 | bytes[2] << 16 | (uint32_t)bytes[3] << 24;
    pk.y = bytes[4] | bytes[5] << 8 | bytes[6] << 16 | (uint32_t)bytes[7] << 24;
    pk.z = bytes[8] | bytes[9] << 8 | bytes[10] << 16 | (uint32_t)bytes[11] << 24;
    pk.w = bytes[12] | bytes[13] << 8 | bytes[14] << 16 | (uint32_t)bytes[15] << 24;
    *reinterpret_cast<uint4*>(out + off) = pk;
}

// Phase copies of the plane: copy p (of P = 16 / shift) is the plane shifted left by
// shift * p pixels, zero past the right edge; row pitch wp (a multiple of 16).
__global__ void phase_planes_kernel(const uint8_t* __restrict__ plane, int w, int h, int wp,
                                    int shift, int P, uint8_t* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int p = blockIdx.z;
    if (x >= wp || y >= h || p >= P) return;
    const int sx = x + shift * p;
    out[((size_t)p * h + y) * wp + x] = sx < w ? plane[(size_t)y * w + sx] : 0;
}

// isometry::map (crates/mars-codec/src/isometry.rs:7-19) as a flat range index i*S + j.
__device__ __forceinline__ int iso_src_rt(int k, int u, int v, int S) {
    switch (k) {
        case 0: return u * S + v;
        case 1: return (S - 1 - v) * S + u;
        case 2: return v * S + (S - 1 - u);
        case 3: return (S - 1 - u) * S + (S - 1 - v);
        case 4: return u * S + (S - 1 - v);
        case 5: return (S - 1 - u) * S + v;
        case 6: return v * S + u;
        default: return (S - 1 - v) * S + (S - 1 - u);
    }
}

// Seed champion of each range: the exact best of the 8 isometries at the 3 x 3 domain
// positions around the range's own position (any real candidate is a valid champion; a
// good one makes the filter tight from the first tile).  One warp per range: the 32 lanes
// share each candidate's correlation (S*S terms), then each lane fits the candidates it
// owns.
// One CTA of 9 warps per range block: warp nb correlates the block with domain nb of the
// 3 x 3 positions around the co-located one (clamped to the pool) under all 8 isometries,
// each D sample loaded once for the 8 permuted range pixels (staged in shared memory);
// lanes 0-7 fit their isometry exactly and the CTA keeps the best of the 72 by (rms,
// reference index).  Exact int32 sums: |r * D| * N < 255 * 1020 * 4096 < 2^31.
template <int S>
__global__ void __launch_bounds__(288) seed_kernel(
    const int32_t* __restrict__ D, LevelGeom g, const uint8_t* __restrict__ plane, int w,
    const uint32_t* rows, const uint32_t* cols, int nranges, RangeStats rs, DomainStats ds,
    FitParams fp, SeedOut* __restrict__ out) {
    constexpr int N = S * S;
    __shared__ uint8_t rsm[N];
    __shared__ double c_rms[72], c_sum[72];
    __shared__ uint32_t c_idx[72];
    __shared__ int32_t c_t1[72];
    const int r = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (r >= nranges) return;
    if (rows[r] + (uint32_t)S > (uint32_t)g.h || cols[r] + (uint32_t)S > (uint32_t)g.w) {
        if (threadIdx.x == 0) out[r] = SeedOut{INFINITY, 0.0, UINT32_MAX, 0};
        return;
    }
    const uint8_t* rb = plane + (size_t)rows[r] * w + cols[r];
    for (int t = threadIdx.x; t < N; t += blockDim.x) rsm[t] = rb[(size_t)(t / S) * w + (t % S)];
    __syncthreads();
    const int ac = min(max(((int)rows[r] - S / 2 + g.shift / 2) / g.shift, 0), g.nrow_d - 1);
    const int bc = min(max(((int)cols[r] - S / 2 + g.shift / 2) / g.shift, 0), g.ncol_d - 1);
    const int nb = warp;
    const int a = min(max(ac + nb / 3 - 1, 0), g.nrow_d - 1);
    const int bb = min(max(bc + nb % 3 - 1, 0), g.ncol_d - 1);
    const int32_t* db = D + (size_t)(a * g.step_c) * g.dw + bb * g.step_c;
    int32_t acc[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[k] = 0;
    for (int t = lane; t < N; t += 32) {
        const int u = t / S, v = t % S;
        const int32_t d = db[(size_t)u * g.dw + v];
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] += (int32_t)rsm[iso_src_rt(k, u, v, S)] * d;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], off);
    if (lane < 8) {
        int32_t t1 = acc[0];
#pragma unroll
        for (int k = 1; k < 8; ++k) t1 = lane == k ? acc[k] : t1;
        const uint32_t dom = (uint32_t)(a * g.ncol_d + bb);
        const FitResult f = fit_exact(N, ds.s1x4[dom], ds.s2x16[dom], rs.t0[r], t1, rs.t2[r], fp);
        c_rms[nb * 8 + lane] = f.rms;
        c_sum[nb * 8 + lane] = f.sum;
        c_idx[nb * 8 + lane] = dom * 8u + (uint32_t)lane;
        c_t1[nb * 8 + lane] = t1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int b = 0;
        for (int c = 1; c < 72; ++c)
            if (c_rms[c] < c_rms[b] || (c_rms[c] == c_rms[b] && c_idx[c] < c_idx[b])) b = c;
        out[r] = SeedOut{c_rms[b], c_sum[b], c_idx[b], c_t1[b]};
    }
}

// Final champion over the M-splits; its exact correlation travels with it, so only the
// (cheap) exact fit is redone here to fill in qalfa / qbeta.
__global__ void finish_kernel(const Partial* __restrict__ partials, int nsplit, int nranges,
                              LevelGeom g, RangeStats rs, DomainStats ds, FitParams fp,
                              CandidateOut* __restrict__ out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nranges) return;
    Partial best = partials[r];
    for (int t = 1; t < nsplit; ++t) {
        const Partial p = partials[(size_t)t * nranges + r];
        if (p.rms < best.rms || (p.rms == best.rms && p.idx < best.idx)) best = p;
    }
    if (best.idx == UINT32_MAX) {
        out[r] = CandidateOut{0, 0, 0, 0, 0, 0, 0.0, 0, 0, 0, 0, 0, 0};
        return;
    }
    const uint32_t dom = best.idx >> 3, k = best.idx & 7u;
    const int a = (int)(dom / (uint32_t)g.ncol_d), bb = (int)(dom % (uint32_t)g.ncol_d);
    const int64_t n = (int64_t)g.size * g.size;
    const int64_t t1 = best.t1x4;
    const FitResult f = fit_exact(n, ds.s1x4[dom], ds.s2x16[dom], rs.t0[r], t1, rs.t2[r], fp);
    CandidateOut c;
    c.dom_row = (uint32_t)a * (uint32_t)g.shift;
    c.dom_col = (uint32_t)bb * (uint32_t)g.shift;
    c.isometry = k;
    c.qalfa = f.qalfa;
    c.qbeta = f.qbeta;
    c.valid = 1;
    c.rms = f.rms;
    c.s0 = n;
    c.s1_x4 = ds.s1x4[dom];
    c.s2_x16 = ds.s2x16[dom];
    c.t0 = rs.t0[r];
    c.t1_x4 = t1;
    c.t2 = rs.t2[r];
    out[r] = c;
}

template <int S>
size_t smem_bytes() {
    constexpr int J = S >= 8 ? S / 8 : 1;
    constexpr int KST = J * 2 * S / 8;
    constexpr bool kBRes = KST <= 2;
    constexpr int kStages = stages_for(S);
    static_assert(kStages <= kMaxStages, "pipeline depth");
    return 1024 + (size_t)kStages * kStageA + (kBRes ? (size_t)KST * kStageB : (size_t)kStages * kStageB) +
           sizeof(Smem);
}

template <int S>
cudaError_t launch_t(const TcMaps& maps, const uint8_t* bglob, const LevelGeom& g, int nranges,
                     RangeStats rs, DomainStats ds, const FitParams& fp, const SeedOut* seeds,
                     Partial* partials, int msplit, int* err, unsigned long long* counter,
                     cudaStream_t st) {
    const int tiles_per_row = (g.ncol_d + kM - 1) / kM;
    const int m_tiles = g.nrow_d * tiles_per_row;
    const int m_per_cta = (m_tiles + msplit - 1) / msplit;
    const int ntiles = (nranges + kRangesPerTile - 1) / kRangesPerTile;
    const size_t smem = smem_bytes<S>();
    auto kern = corr_tc_kernel<S>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid(ntiles, msplit);
    kern<<<grid, kThreads, smem, st>>>(maps, bglob, g, nranges, rs, ds, fp, seeds, m_tiles,
                                      m_per_cta, partials, err, counter);
    return cudaGetLastError();
}

template <int S>
cudaError_t build_b_t(const uint8_t* plane, int w, int h, const uint32_t* rows,
                      const uint32_t* cols, int nranges, uint8_t* out, cudaStream_t st) {
    constexpr int J = S >= 8 ? S / 8 : 1;
    constexpr int KG = J * 2 * S;
    const int ntiles = (nranges + kRangesPerTile - 1) / kRangesPerTile;
    const long long total = (long long)ntiles * kN * KG;
    build_b_kernel<S><<<(unsigned)((total + 255) / 256), 256, 0, st>>>(plane, w, h, rows, cols,
                                                                       nranges, ntiles, out);
    return cudaGetLastError();
}

}  // namespace

bool supported(int size, int shift) {
    return (size == 4 || size == 8 || size == 16 || size == 32 || size == 64) &&
           (shift == 2 || shift == 4 || shift == 8 || shift == 16);
}

size_t b_bytes(int size, int nranges) {
    const int J = size >= 8 ? size / 8 : 1;
    const int KG = J * 2 * size;
    const size_t ntiles = (size_t)(nranges + kRangesPerTile - 1) / kRangesPerTile;
    return ntiles * (size_t)kN * (size_t)KG * 16;
}

int phase_count(int shift) { return 16 / shift; }
int row_pitch(int w) { return ((w + 15) / 16) * 16 + 16; }
// The 4-D view reads up to (16/P - 1) * 128 bytes past a row's end (columns no valid
// domain uses); the allocation carries that much slack after the last phase copy.
size_t phase_bytes(int w, int h, int shift) {
    return (size_t)phase_count(shift) * h * row_pitch(w) + 2048;
}

cudaError_t launch_phase_planes(const uint8_t* plane, int w, int h, int shift, uint8_t* out,
                                cudaStream_t st) {
    const int P = phase_count(shift), wp = row_pitch(w);
    dim3 grid((wp + 255) / 256, h, P);
    phase_planes_kernel<<<grid, 256, 0, st>>>(plane, w, h, wp, shift, P, out);
    return cudaGetLastError();
}

cudaError_t launch_build_b(int size, const uint8_t* plane, int w, int h, const uint32_t* rows,
                           const uint32_t* cols, int nranges, uint8_t* out, cudaStream_t st) {
    switch (size) {
        case 4: return build_b_t<4>(plane, w, h, rows, cols, nranges, out, st);
        case 8: return build_b_t<8>(plane, w, h, rows, cols, nranges, out, st);
        case 16: return build_b_t<16>(plane, w, h, rows, cols, nranges, out, st);
        case 32: return build_b_t<32>(plane, w, h, rows, cols, nranges, out, st);
        case 64: return build_b_t<64>(plane, w, h, rows, cols, nranges, out, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_seed(const int32_t* D, const LevelGeom& g, const uint8_t* plane, int w,
                        const uint32_t* rows, const uint32_t* cols, int nranges, RangeStats rs,
                        DomainStats ds, const FitParams& fp, SeedOut* out, cudaStream_t st) {
    if (nranges == 0) return cudaSuccess;
    const unsigned blocks = (unsigned)nranges;
    switch (g.size) {
        case 4: seed_kernel<4><<<blocks, 288, 0, st>>>(D, g, plane, w, rows, cols, nranges, rs, ds, fp, out); break;
        case 8: seed_kernel<8><<<blocks, 288, 0, st>>>(D, g, plane, w, rows, cols, nranges, rs, ds, fp, out); break;
        case 16: seed_kernel<16><<<blocks, 288, 0, st>>>(D, g, plane, w, rows, cols, nranges, rs, ds, fp, out); break;
        case 32: seed_kernel<32><<<blocks, 288, 0, st>>>(D, g, plane, w, rows, cols, nranges, rs, ds, fp, out); break;
        case 64: seed_kernel<64><<<blocks, 288, 0, st>>>(D, g, plane, w, rows, cols, nranges, rs, ds, fp, out); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// M-split of a level: the grid is (N tiles) x msplit CTAs, one CTA per SM at a time, each
// CTA sweeping ceil(m_tiles / msplit) domain tiles after a fixed set-up (B load, range
// records, pipeline fill) worth about kSetupTiles tiles.  Pick the split with the fewest
// tile-times over all waves.
int msplit_for(const LevelGeom& g, int nranges, int num_sms) {
    constexpr long long kSetupTiles = 4;
    const int tiles_per_row = (g.ncol_d + kM - 1) / kM;
    const int m_tiles = g.nrow_d * tiles_per_row;
    const int ntiles = (nranges + kRangesPerTile - 1) / kRangesPerTile;
    int best = 1;
    long long best_cost = -1;
    for (int ms = 1; ms <= m_tiles; ++ms) {
        const long long waves = ((long long)ntiles * ms + num_sms - 1) / num_sms;
        const long long per_cta = (m_tiles + ms - 1) / ms + kSetupTiles;
        const long long cost = waves * per_cta;
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = ms;
        }
    }
    return best;
}

cudaError_t launch_corr(const TcMaps& maps, const uint8_t* bglob, const LevelGeom& g, int nranges,
                        RangeStats rs, DomainStats ds, const FitParams& fp, const SeedOut* seeds,
                        Partial* partials, int msplit, int* err, unsigned long long* counter,
                        cudaStream_t st) {
    switch (g.size) {
        case 4: return launch_t<4>(maps, bglob, g, nranges, rs, ds, fp, seeds, partials, msplit, err, counter, st);
        case 8: return launch_t<8>(maps, bglob, g, nranges, rs, ds, fp, seeds, partials, msplit, err, counter, st);
        case 16: return launch_t<16>(maps, bglob, g, nranges, rs, ds, fp, seeds, partials, msplit, err, counter, st);
        case 32: return launch_t<32>(maps, bglob, g, nranges, rs, ds, fp, seeds, partials, msplit, err, counter, st);
        case 64: return launch_t<64>(maps, bglob, g, nranges, rs, ds, fp, seeds, partials, msplit, err, counter, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_finish(const Partial* partials, int nsplit, int nranges, const LevelGeom& g,
                          RangeStats rs, DomainStats ds, const FitParams& fp, CandidateOut* out,
                          cudaStream_t st) {
    finish_kernel<<<(nranges + 127) / 128, 128, 0, st>>>(partials, nsplit, nranges, g, rs, ds, fp,
                                                         out);
    return cudaGetLastError();
}

}  // namespace tc
}  // namespace mars
