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
//
// One body (process_item) serves three kernels: corr_tc_kernel<S, DIG, false>, one level
// per launch (CTA = range tile x domain-tile split); corr_tc_kernel<S, DIG, true>, the
// ranked search keeping each range's best k; and corr_tc_all_kernel, every tensor-core
// level of a plane in one persistent launch over (level, range tile, split) work items.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>

#include "kernels.cuh"
#include "tc.cuh"
#include "tc_ptx.cuh"

namespace mars {
namespace tc {
namespace {

constexpr int kN = 256;                        // accumulator columns of a TMEM buffer
constexpr int kRangesPerTile = kN / 8;         // 32: the most ranges a tile holds
constexpr int kStageA = 16 * 1024;             // 16 row groups x 8 K-groups x 128 B
constexpr int kGroups = 2;                     // independent epilogue groups of 4 warps
constexpr int kGroupThreads = kEpiThreads / kGroups;
constexpr int kQueueCap = 1024;                // survivors a group's queue can hold
constexpr int kFlush = 128;                    // drain a group's queue once it holds this many

// Pipeline depth of the fold path: as many A stages as fit beside the resident B tile
// (S <= 8), otherwise three stages of A + B.
__host__ __device__ constexpr int stages_for(int S) { return S == 4 ? 6 : (S == 8 ? 4 : 3); }

// Tile shape of a level.
//   Fold path (DIG = false): A is u8 pixels of the 2S x 2S domain block (K = 4 S^2, the
//     2x2 box sum folded into K); N = 256 columns = 32 ranges x 8 isometries.
//   Digit path (DIG = true, S >= 16): A is the contracted plane D = 4d of the reference
//     (Contracted::build, encode.rs:478-502; 0..1020) split into two u8 digits,
//     D = 128 hi + lo (hi 0..7, lo 0..127), K = S^2 per digit, half the fold's MACs; N = 128
//     columns per digit = 16 ranges x 8 isometries, the two digits' accumulators side by
//     side in a 256-column TMEM buffer (hi at +0, lo at +128), t1' = 128 hi + lo exactly.
//   Either way a TMEM buffer is 256 columns and two of them double-buffer the 512.
template <int S, bool DIG>
struct Cfg {
    static constexpr int kNt = DIG ? 128 : 256;         // accumulator columns per digit
    static constexpr int kRt = kNt / 8;                 // ranges per tile
    static constexpr int kCols = 4 * kNt / kEpiWarps;   // columns per epilogue warp and digit
    static constexpr int kRw = kCols / 8;               // ranges per epilogue warp
    static constexpr int kCh = kCols / 32;              // 32-column chunks per warp and digit
    static constexpr int kStageBt = kNt * 128;          // B bytes per 128-byte K stage
    static constexpr int kDigits = DIG ? 2 : 1;
    static constexpr int ROWS = DIG ? S : 2 * S;        // rows of a domain's K window
    static constexpr int J = DIG ? S / 16 : (S >= 8 ? S / 8 : 1);  // 16-byte groups a row
    static constexpr int KST = J * ROWS / 8;            // 128-byte K stages per tile
    static constexpr bool kBRes = KST * kStageBt <= 64 * 1024;  // B stays resident
    static constexpr int kStages = DIG ? 3 : stages_for(S);
    static constexpr uint32_t kTx = kDigits * kStageA + (kBRes ? 0 : kStageBt);
    static_assert(!DIG || S >= 16, "the digit path needs whole 16-byte digit rows");
};

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
//   tau = (dom > tie) ? tau_z : g1;   prune  <=>  t1' < s1_x4 * c + 4 tau / n.
// tie = -1 puts every domain in the Z-form, INT32_MAX none.  W <= 0 is sqrt_w = -inf:
// g1 = -inf (sqrt(Ndd) > 0), nothing pruned in the plain form, and tau_z unchanged
// (max(-inf, a_min Ndd) = max(0, a_min Ndd)).
struct __align__(16) ThrRec {
    float sqrt_w, w2a, c;  // sqrt_w, w2a pre-scaled by 4 / n (exact: n = 4^k)
    int32_t tie;
};

// A survivor waiting for its exact fit.  Survivors of several tiles are batched: the
// queue is drained when it holds kFlush entries, when a tile overflows it, and at the end.
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
    int qcount[kGroups];
    int item;  // the all-levels launch: this CTA's current work item
    int last;  // this CTA finished the last split of its range tile
    unsigned long long key_rms[kRangesPerTile];  // per-pass winner: f64 bits (rms >= 0)
    uint32_t key_idx[kRangesPerTile];
    double key_sum[kRangesPerTile];
    int32_t key_t1[kRangesPerTile];
    ThrRec thr[kRangesPerTile];
    Champ ch[kRangesPerTile];
    uint32_t evaluated[kM * kN / 32];           // candidates already fitted in this tile
    QEntry queue[kGroups][kQueueCap];
};

// Barriers of one epilogue group (its 4 warps, one per TMEM lane quadrant): named barrier
// 1 + group over kGroupThreads threads.
__device__ __forceinline__ void group_barrier(int grp) {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "n"(kGroupThreads) : "memory");
}
__device__ __forceinline__ bool group_barrier_and(int grp, bool pred) {
    uint32_t out;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(out)
        : "r"((uint32_t)pred), "r"(1 + grp), "n"(kGroupThreads)
        : "memory");
    return out != 0;
}

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
        // +inf, tau = +inf for every domain, flat all-zero ones (s1 = 0) included.
        sm.thr[rl] = ThrRec{INFINITY, INFINITY, 3.0e38f, -1};
        return;
    }
    const Threshold th = make_threshold(C.sum, C.rms, C.idx >> 3, C.rms0, C.nrr, n, fp);
    // Scaling by 4 / n (a power of two) is exact, so folding it in keeps every bound
    // rounded toward -inf.
    const float four_inv_n = 4.0f / (float)n;
    t.sqrt_w = th.wpos ? th.sqrt_w * four_inv_n : -INFINITY;
    t.w2a = th.w2a * four_inv_n;
    t.c = (float)C.t0 / (float)n - 128.0f;  // exact: t0 < 2^24, n a power of four
    t.tie = th.mode == 2 ? -1 : (th.mode == 1 ? (int32_t)th.tie_dom : INT32_MAX);
    sm.thr[rl] = t;
}

// 128-bit compare-and-swap on a global record (two 64-bit halves); returns the old value.
// With cmp = val = 0 it is an atomic read.
__device__ __forceinline__ void cas128(unsigned long long* addr, unsigned long long clo,
                                       unsigned long long chi, unsigned long long vlo,
                                       unsigned long long vhi, unsigned long long& olo,
                                       unsigned long long& ohi) {
    asm volatile(
        "{\n\t.reg .b128 c, v, o;\n\t"
        "mov.b128 c, {%2, %3};\n\t"
        "mov.b128 v, {%4, %5};\n\t"
        "atom.global.cas.b128 o, [%6], c, v;\n\t"
        "mov.b128 {%0, %1}, o;\n\t}"
        : "=l"(olo), "=l"(ohi)
        : "l"(clo), "l"(chi), "l"(vlo), "l"(vhi), "l"(addr)
        : "memory");
}

// Exact fits of every queued survivor, then the per-range winners of the batch (atomic
// min on the f64 bit pattern of rms >= 0, then on the reference index) and the champion /
// threshold update.  All epilogue threads call this together.
template <int N, int NT, int RG>
__device__ __noinline__ void drain_queue(Smem& sm, int grp, int n, bool mark, uint32_t tag,
                                         int gt, const DomainStats& ds, const FitParams& fp,
                                         unsigned long long& exact, unsigned long long* gch,
                                         int rbase) {
    QEntry* const queue = sm.queue[grp];
    for (int qi = gt; qi < n; qi += kGroupThreads) {
        QEntry& q = queue[qi];
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
    group_barrier(grp);
    for (int qi = gt; qi < n; qi += kGroupThreads) {
        const QEntry& q = queue[qi];
        const int col = (int)(q.code & 255u), rl = col >> 3;
        if ((unsigned long long)__double_as_longlong(q.rms) == sm.key_rms[rl])
            atomicMin(&sm.key_idx[rl], q.dom * 8u + (uint32_t)(col & 7));
    }
    group_barrier(grp);
    for (int qi = gt; qi < n; qi += kGroupThreads) {
        const QEntry& q = queue[qi];
        const int col = (int)(q.code & 255u), rl = col >> 3;
        if ((unsigned long long)__double_as_longlong(q.rms) == sm.key_rms[rl] &&
            q.dom * 8u + (uint32_t)(col & 7) == sm.key_idx[rl]) {
            sm.key_sum[rl] = q.sum;
            sm.key_t1[rl] = q.t1 + 128 * ds.s1x4[q.dom];  // t1_x4, exact in int32 (S <= 64)
        }
        if (mark && (q.code >> 16) == tag) {
            // The tile overflowed the queue: remember what was fitted so the next pass
            // over the same accumulator only queues candidates not yet seen.
            const int qm = (int)(q.code >> 8) & 127;
            atomicOr(&sm.evaluated[(qm * NT + col) >> 5], 1u << (col & 31));
        }
    }
    group_barrier(grp);
    // The group's ranges: RG of them from grp * RG.
    const int rl = grp * RG + gt;
    if (gt < RG && sm.key_rms[rl] != ~0ull) {
        Champ& C = sm.ch[rl];
        const double r2 = __longlong_as_double((long long)sm.key_rms[rl]);
        const uint32_t i2 = sm.key_idx[rl];
        if (C.valid && (r2 < C.rms || (r2 == C.rms && i2 < C.idx))) {
            C.rms = r2;
            C.idx = i2;
            C.sum = sm.key_sum[rl];
            C.t1x4 = sm.key_t1[rl];
            publish_threshold(sm, rl, fp, N);
        }
        sm.key_rms[rl] = ~0ull;
        sm.key_idx[rl] = UINT32_MAX;
    }
    // The M-splits of a range share their champions through one global record per range
    // (rms bits, reference index, t1_x4): publish ours when better, adopt the record when
    // it is better.  An adopted champion is a real candidate of another split; its fit sum
    // is recomputed exactly from its domain statistics.
    if (gt < RG && gch && sm.ch[rl].valid) {
        Champ& C = sm.ch[rl];
        unsigned long long* rec = gch + 2 * (size_t)(rbase + rl);
        unsigned long long clo, chi;
        cas128(rec, 0ull, 0ull, 0ull, 0ull, clo, chi);
        for (int tries = 0; tries < 64; ++tries) {
            const unsigned long long mlo = (unsigned long long)__double_as_longlong(C.rms);
            const uint32_t gidx = (uint32_t)chi;
            if (mlo < clo || (mlo == clo && C.idx < gidx)) {
                const unsigned long long vhi = (unsigned long long)C.idx |
                                               (unsigned long long)(uint32_t)C.t1x4 << 32;
                unsigned long long olo, ohi;
                cas128(rec, clo, chi, mlo, vhi, olo, ohi);
                if (olo == clo && ohi == chi) break;
                clo = olo;
                chi = ohi;
            } else {
                if (clo < mlo || (clo == mlo && gidx < C.idx)) {
                    const uint32_t dom = gidx >> 3;
                    C.rms = __longlong_as_double((long long)clo);
                    C.idx = gidx;
                    C.t1x4 = (int32_t)(uint32_t)(chi >> 32);
                    C.sum = fit_exact(N, ds.s1x4[dom], ds.s2x16[dom], C.t0, (int64_t)C.t1x4,
                                      C.t2, fp).sum;
                    publish_threshold(sm, rl, fp, N);
                }
                break;
            }
        }
    }
    if (gt == 0) sm.qcount[grp] = 0;
    group_barrier(grp);
}

// Final champion of range r over its M-splits' partials; its exact correlation travels with
// it, so only the (cheap) exact fit is redone to fill in qalfa / qbeta.  The partials are
// read around L1 (ld.global.cg): in the all-levels launch other CTAs wrote them.
__device__ __forceinline__ void finish_range(const Partial* partials, int nsplit, int nranges,
                                             int r, const LevelGeom& g, const RangeStats& rs,
                                             const DomainStats& ds, const FitParams& fp,
                                             CandidateOut* out) {
    double best_rms = 0.0;
    uint32_t best_idx = UINT32_MAX;
    int32_t best_t1 = 0;
    for (int t = 0; t < nsplit; ++t) {
        const Partial* p = partials + (size_t)t * nranges + r;
        const double rms = __ldcg(reinterpret_cast<const double*>(p));
        const uint2 it = __ldcg(reinterpret_cast<const uint2*>(p) + 2);  // idx, t1x4
        if (t == 0 || rms < best_rms || (rms == best_rms && it.x < best_idx)) {
            best_rms = rms;
            best_idx = it.x;
            best_t1 = (int32_t)it.y;
        }
    }
    if (best_idx == UINT32_MAX) {
        out[r] = CandidateOut{0, 0, 0, 0, 0, 0, 0.0, 0, 0, 0, 0, 0, 0};
        return;
    }
    const uint32_t dom = best_idx >> 3, k = best_idx & 7u;
    const int a = (int)(dom / (uint32_t)g.ncol_d), bb = (int)(dom % (uint32_t)g.ncol_d);
    const int64_t n = (int64_t)g.size * g.size;
    const int64_t t1 = best_t1;
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

// The ranked search's lists (search_top_k, encode.rs:695-788): per range of the tile its
// best k <= kMaxTopK candidates by (rms, reference index), in shared memory after the
// stages (the ranked kernel only).
struct TopkLists {
    double rms[kRangesPerTile][kMaxTopK];
    double sum[kRangesPerTile][kMaxTopK];
    uint32_t idx[kRangesPerTile][kMaxTopK];
    int32_t t1[kRangesPerTile][kMaxTopK];
    uint32_t q[kRangesPerTile][kMaxTopK];  // qalfa | qbeta << 16
    int cnt[kRangesPerTile];
};

// Insert a fitted candidate into range rl's list (capacity k), keeping it sorted by (rms,
// index) -- retain_top_k's strict-< insertion in encounter order gives the same set.  A
// candidate already listed (a seed the sweep meets again) is skipped.  True when the list
// changed.
__device__ __forceinline__ bool topk_insert(TopkLists& L, int rl, int k, double rms, double sum,
                                            uint32_t idx, int32_t t1, uint32_t q) {
    const int c = L.cnt[rl];
    if (c == k && !(rms < L.rms[rl][k - 1] || (rms == L.rms[rl][k - 1] && idx < L.idx[rl][k - 1])))
        return false;
    for (int j = 0; j < c; ++j)
        if (L.idx[rl][j] == idx) return false;
    int pos = c < k ? c : k - 1;
    while (pos > 0 && (rms < L.rms[rl][pos - 1] ||
                       (rms == L.rms[rl][pos - 1] && idx < L.idx[rl][pos - 1]))) {
        L.rms[rl][pos] = L.rms[rl][pos - 1];
        L.sum[rl][pos] = L.sum[rl][pos - 1];
        L.idx[rl][pos] = L.idx[rl][pos - 1];
        L.t1[rl][pos] = L.t1[rl][pos - 1];
        L.q[rl][pos] = L.q[rl][pos - 1];
        --pos;
    }
    L.rms[rl][pos] = rms;
    L.sum[rl][pos] = sum;
    L.idx[rl][pos] = idx;
    L.t1[rl][pos] = t1;
    L.q[rl][pos] = q;
    if (c < k) L.cnt[rl] = c + 1;
    return true;
}

// The pruning record of a ranked range: against its k-th entry once the list is full (the
// same bound as the single winner's, fit.cuh); before that every candidate passes (sqrt_w
// = w2a = -inf: tau = -inf for every domain).  With a shared record (rec, the range's
// 128-bit record of the best k-th entry any split holds) the bound is the better of the two:
// a candidate that k others of one split beat is not among the k best at all.  The list
// keeps this split's own candidates either way.
__device__ __forceinline__ void topk_publish(Smem& sm, const TopkLists& L, int rl, int k,
                                             const FitParams& fp, int n,
                                             unsigned long long* rec = nullptr,
                                             const DomainStats* ds = nullptr) {
    Champ& C = sm.ch[rl];
    if (!C.valid) {
        publish_threshold(sm, rl, fp, n);
        return;
    }
    bool have = L.cnt[rl] == k;
    if (have) {
        C.rms = L.rms[rl][k - 1];
        C.sum = L.sum[rl][k - 1];
        C.idx = L.idx[rl][k - 1];
        C.t1x4 = L.t1[rl][k - 1];
    }
    if (rec) {
        unsigned long long clo, chi;
        cas128(rec, 0ull, 0ull, 0ull, 0ull, clo, chi);
        for (int tries = 0; tries < 64; ++tries) {
            const uint32_t gidx = (uint32_t)chi;
            const unsigned long long mlo =
                have ? (unsigned long long)__double_as_longlong(C.rms) : ~0ull;
            if (have && (mlo < clo || (mlo == clo && C.idx < gidx))) {
                // Publish this split's k-th entry.
                const unsigned long long vhi = (unsigned long long)C.idx |
                                               (unsigned long long)(uint32_t)C.t1x4 << 32;
                unsigned long long olo, ohi;
                cas128(rec, clo, chi, mlo, vhi, olo, ohi);
                if (olo == clo && ohi == chi) break;
                clo = olo;
                chi = ohi;
            } else {
                if (clo != ~0ull && (!have || clo < mlo || (clo == mlo && gidx < C.idx))) {
                    // Another split's k-th entry is the tighter bound.
                    const uint32_t dom = gidx >> 3;
                    C.rms = __longlong_as_double((long long)clo);
                    C.idx = gidx;
                    C.t1x4 = (int32_t)(uint32_t)(chi >> 32);
                    C.sum = fit_exact(n, ds->s1x4[dom], ds->s2x16[dom], C.t0, (int64_t)C.t1x4,
                                      C.t2, fp).sum;
                    have = true;
                }
                break;
            }
        }
    }
    if (!have) {
        sm.thr[rl] = ThrRec{-INFINITY, -INFINITY, 0.0f, INT32_MAX};
        return;
    }
    publish_threshold(sm, rl, fp, n);
}

// drain_queue for the ranked search: exact fits of the queued survivors, then one thread per
// range inserts its range's entries into the range's list and republishes the threshold.
template <int N, int NT, int RG>
__device__ __noinline__ void drain_queue_topk(Smem& sm, TopkLists& L, int k, int grp, int n,
                                              bool mark, uint32_t tag, int gt,
                                              const DomainStats& ds, const FitParams& fp,
                                              unsigned long long& exact, unsigned long long* gch,
                                              int rbase) {
    QEntry* const queue = sm.queue[grp];
    for (int qi = gt; qi < n; qi += kGroupThreads) {
        QEntry& q = queue[qi];
        const int col = (int)(q.code & 255u), rl = col >> 3;
        const Champ& C = sm.ch[rl];
        const int32_t s1 = ds.s1x4[q.dom];
        const int64_t t1x4 = (int64_t)q.t1 + 128ll * s1;
        const FitResult f = fit_exact(N, s1, ds.s2x16[q.dom], C.t0, t1x4, C.t2, fp);
        q.rms = f.rms;
        q.sum = f.sum;
        q.pad = f.qalfa | (f.qbeta << 16);
        ++exact;
        if (mark && (q.code >> 16) == tag) {
            const int qm = (int)(q.code >> 8) & 127;
            atomicOr(&sm.evaluated[(qm * NT + col) >> 5], 1u << (col & 31));
        }
    }
    group_barrier(grp);
    const int rl = grp * RG + gt;
    if (gt < RG && sm.ch[rl].valid) {
        bool changed = false;
        for (int qi = 0; qi < n; ++qi) {
            const QEntry& q = queue[qi];
            const int col = (int)(q.code & 255u);
            if ((col >> 3) != rl) continue;
            changed |= topk_insert(L, rl, k, q.rms, q.sum, q.dom * 8u + (uint32_t)(col & 7),
                                   q.t1 + 128 * ds.s1x4[q.dom], q.pad);
        }
        // With shared records the bound is refreshed after every drain: another split may
        // have tightened it.
        if (changed || gch)
            topk_publish(sm, L, rl, k, fp, N, gch ? gch + 2 * (size_t)(rbase + rl) : nullptr,
                         &ds);
    }
    if (gt == 0) sm.qcount[grp] = 0;
    group_barrier(grp);
}

// A seed read around L1: in the all-levels launch another CTA may have just merged it.
__device__ __forceinline__ SeedOut load_seed(const SeedOut* p) {
    const uint2 it = __ldcg(reinterpret_cast<const uint2*>(p) + 2);
    return SeedOut{__ldcg(reinterpret_cast<const double*>(p)),
                   __ldcg(reinterpret_cast<const double*>(p) + 1), it.x, (int32_t)it.y};
}

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_gpu(int* p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// The coarse pre-pass's champion of range r (the best of its M-splits over every
// `ratio`-th domain position of each axis) as a seed on the full grid: its domain index is
// mapped to the fine grid, and it replaces the seed when it is better by (rms, index).
// Any real candidate is a valid seed; a better one prunes more from the first tile.
__device__ __forceinline__ void seed_merge_range(const Partial* partials, int nsplit, int nranges,
                                                 int r, int coarse_ncol, int fine_ncol,
                                                 int ratio, SeedOut* seeds) {
    const SeedOut s = load_seed(seeds + r);
    if (s.idx == UINT32_MAX) return;  // no range block here
    // The pre-pass started from this seed, whose index is on the fine grid.  A split's
    // champion only ever changes to a strictly better (rms, index) pair, so a partial equal
    // to the seed's pair is the seed itself; every other one is a coarse-grid candidate.
    bool have = false;
    double best_rms = 0.0, best_sum = 0.0;
    uint32_t best_idx = UINT32_MAX;
    int32_t best_t1 = 0;
    for (int t = 0; t < nsplit; ++t) {
        const Partial* p = partials + (size_t)t * nranges + r;
        const double rms = __ldcg(reinterpret_cast<const double*>(p));
        const double sum = __ldcg(reinterpret_cast<const double*>(p) + 1);
        const uint2 it = __ldcg(reinterpret_cast<const uint2*>(p) + 2);
        if (it.x == UINT32_MAX || (rms == s.rms && it.x == s.idx)) continue;
        if (!have || rms < best_rms || (rms == best_rms && it.x < best_idx)) {
            best_rms = rms;
            best_sum = sum;
            best_idx = it.x;
            best_t1 = (int32_t)it.y;
        }
        have = true;
    }
    if (!have) return;
    const uint32_t dom1 = best_idx >> 3;
    const uint32_t a1 = dom1 / (uint32_t)coarse_ncol, b1 = dom1 % (uint32_t)coarse_ncol;
    const uint32_t idx =
        ((a1 * (uint32_t)ratio) * (uint32_t)fine_ncol + b1 * (uint32_t)ratio) * 8u + (best_idx & 7u);
    if (best_rms < s.rms || (best_rms == s.rms && idx < s.idx))
        seeds[r] = SeedOut{best_rms, best_sum, idx, best_t1};
}

// What one work item reads and writes: a level's B operand, statistics, seeds, its split
// of the domain tiles and the outputs of its range tile.
struct ItemArgs {
    const uint8_t* bglob;
    LevelGeom g;
    int nranges;
    RangeStats rs;
    DomainStats ds;
    FitParams fp;
    const SeedOut* seeds;
    int m_tiles, m_per_cta, msplit;
    Partial* partials;        // msplit x nranges
    unsigned long long* gch;  // 2 x nranges shared champion records, or null
    int* tickets;             // per range tile: splits done (all-levels launch), or null
    CandidateOut* out;        // the level's candidates when tickets is set
    int k;                    // candidates kept per range (> 1: the ranked kernel)
    // The all-levels launch's coarse pre-pass job: the last split of a range tile merges
    // the tile's champions into merge_seeds (the fine level's seeds) and sets ready[tile];
    // the fine level's items wait for wait_ready[tile] before reading their seeds.
    SeedOut* merge_seeds;
    int merge_ratio, fine_ncol;
    int* ready;
    const int* wait_ready;
};

// Per-thread pipeline state of the roles (each role thread keeps its own copy).  It carries
// over from one work item to the next, so the mbarriers are initialised once per CTA:
// bit s of stage_par is the parity of this role's uses of shared-memory stage s so far
// (fills for the load thread, consumptions for the MMA thread), bit s of stage_used says
// the load thread filled stage s before; `tiles` counts the accumulator tiles handed over
// (TMEM buffer tiles & 1, phase (tiles >> 1) & 1); `bres` counts resident-B loads.
struct PipeState {
    uint32_t stage_par = 0, stage_used = 0, tiles = 0, bres = 0;
};

// Shared-memory layout of both correlation kernels: the Smem record first (mbarriers at
// fixed addresses for every level), then the A stages and the B stages / resident B tile,
// 1024-byte aligned.
constexpr size_t kSmemHead = (sizeof(Smem) + 1023) / 1024 * 1024;

__device__ __forceinline__ Smem& smem_record(unsigned char* raw) {
    return *reinterpret_cast<Smem*>(((uintptr_t)raw + 1023) & ~(uintptr_t)1023);
}

// CTA set-up shared by both kernels: mbarriers, the epilogue's queues and bitmap, TMEM
// (all 512 columns, held until cta_teardown).
__device__ __forceinline__ uint32_t cta_setup(Smem& sm) {
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kMaxStages; ++s) {
            mbar_init(&sm.full[s], 1);
            mbar_init(&sm.empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&sm.tfull[b], 1);
            mbar_init(&sm.tempty[b], kEpiThreads);
        }
        mbar_init(&sm.bres, 1);
        sm.abort_flag = 0;
        for (int q = 0; q < kGroups; ++q) sm.qcount[q] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = threadIdx.x; i < kM * kN / 32; i += kThreads) sm.evaluated[i] = 0u;
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&sm.tmem_base)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tmem_fence_before();
    __syncthreads();
    tmem_fence_after();
    return sm.tmem_base;
}

__device__ __forceinline__ void cta_teardown(Smem& sm, uint32_t tmem, unsigned long long exact,
                                             unsigned long long* exact_counter) {
    if (exact_counter && exact) atomicAdd(exact_counter, exact);
    tmem_fence_before();
    __syncthreads();
    if ((threadIdx.x >> 5) == 1) {
        tmem_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
    }
}

// One work item: range tile `ntile` of a level against domain tiles [split * m_per_cta,
// ...) -- the champions seeded, the loads / MMAs / exact-bound epilogue over those domain
// tiles, the tile's partial champions written.  With tickets set, the last split of the
// range tile to finish also writes the tile's final candidates, or, for a coarse pre-pass
// job, merges them into the fine level's seeds and sets the tile's ready flag; with
// wait_ready set the item first waits for that flag.  TOPK: the ranked search, a k-list
// per range in *tk.  Every thread of the CTA calls this together; it begins and ends with a
// CTA barrier.
template <int S, bool DIG, bool TOPK = false>
__device__ __forceinline__ void process_item(const TcMaps& maps, const ItemArgs& a, int ntile,
                                             int split, Smem& sm, unsigned char* stages,
                                             uint32_t tmem, PipeState& ps, int* err,
                                             unsigned long long& exact,
                                             TopkLists* tk = nullptr) {
    using C_ = Cfg<S, DIG>;
    constexpr int N = S * S;
    constexpr int NT = C_::kNt;
    constexpr int RT = C_::kRt;
    constexpr int ROWS = C_::ROWS;
    constexpr int KST = C_::KST;
    constexpr bool kBRes = C_::kBRes;
    constexpr int kStages = C_::kStages;
    constexpr int kStageB = C_::kStageBt;
    constexpr int kStageAll = C_::kDigits * kStageA;  // A bytes of one stage (both digits)
    constexpr int kColsPerWarp = C_::kCols;
    constexpr int kRangesPerWarp = C_::kRw;
    constexpr int kChunks = C_::kCh;

    unsigned char* stA = stages;                     // kStages x (1 or 2) x 16 KB
    unsigned char* stB = stA + kStages * kStageAll;  // kStages B stages or resident

    const LevelGeom& g = a.g;
    const DomainStats& ds = a.ds;
    const FitParams& fp = a.fp;
    const int nranges = a.nranges;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m_begin = split * a.m_per_cta;
    const int m_end = min(a.m_tiles, m_begin + a.m_per_cta);
    // Phase copies: domains lie shift pixels (fold) or shift / 2 contracted samples
    // (digits) apart; P same-phase copies put each group of 16 / P domains' starts on
    // 16-byte boundaries.
    const int P = DIG ? 32 / g.shift : 16 / g.shift;
    const int tiles_per_row = (g.ncol_d + kM - 1) / kM;
    const uint8_t* btile = a.bglob + (size_t)ntile * KST * kStageB;

    if (a.wait_ready) {
        // The coarse pre-pass items of this range tile were claimed before any item of this
        // level, by CTAs that are running them: the wait ends (bounded all the same).
        if (threadIdx.x == 0) {
            const long long t0 = clock64();
            while (ld_acquire_gpu(a.wait_ready + ntile) == 0) {
                if (clock64() - t0 > kWaitCycles) {
                    sm.abort_flag = 1;
                    atomicOr(err, 32);
                    break;
                }
                __nanosleep(256);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x < RT) {
        Champ& C = sm.ch[threadIdx.x];
        const int r = ntile * RT + threadIdx.x;
        const int ks = TOPK ? a.k : 1;  // seeds per range
        C.valid = r < nranges && load_seed(a.seeds + (size_t)r * ks).idx != UINT32_MAX;
        if (C.valid) {
            C.t0 = a.rs.t0[r];
            C.t2 = a.rs.t2[r];
            C.nrr = a.rs.nrr[r];
            C.rms0 = a.rs.rms0[r];
            const SeedOut sd = load_seed(a.seeds + (size_t)r * ks);
            C.rms = sd.rms;
            C.sum = sd.sum;
            C.idx = sd.idx;
            C.t1x4 = sd.t1x4;
            if (TOPK) {
                // The ranked list starts from the range's k seeds (distinct candidates);
                // their quantised coefficients come from the same exact fit.
                tk->cnt[threadIdx.x] = 0;
                for (int j = 0; j < a.k; ++j) {
                    const SeedOut sj = a.seeds[(size_t)r * ks + j];
                    if (sj.idx == UINT32_MAX) continue;
                    const uint32_t dom = sj.idx >> 3;
                    const FitResult f = fit_exact(N, a.ds.s1x4[dom], a.ds.s2x16[dom], C.t0,
                                                  (int64_t)sj.t1x4, C.t2, fp);
                    topk_insert(*tk, threadIdx.x, a.k, f.rms, f.sum, sj.idx, sj.t1x4,
                                f.qalfa | (f.qbeta << 16));
                }
            } else if (a.gch) {
                // Start from the range's shared champion when the splits that ran before
                // this one found a better one than the seed (an atomic 128-bit read).
                unsigned long long clo, chi;
                cas128(a.gch + 2 * (size_t)r, 0ull, 0ull, 0ull, 0ull, clo, chi);
                const uint32_t gidx = (uint32_t)chi;
                const unsigned long long mlo = (unsigned long long)__double_as_longlong(C.rms);
                if (clo < mlo || (clo == mlo && gidx < C.idx)) {
                    const uint32_t dom = gidx >> 3;
                    C.rms = __longlong_as_double((long long)clo);
                    C.idx = gidx;
                    C.t1x4 = (int32_t)(uint32_t)(chi >> 32);
                    C.sum = fit_exact(N, a.ds.s1x4[dom], a.ds.s2x16[dom], C.t0, (int64_t)C.t1x4,
                                      C.t2, fp).sum;
                }
            }
        } else {
            // Padding of the last N tile, or a block outside the plane: no candidate.
            C.rms = INFINITY;
            C.sum = 0.0;
            C.idx = UINT32_MAX;
            C.t1x4 = 0;
        }
        sm.key_rms[threadIdx.x] = ~0ull;
        sm.key_idx[threadIdx.x] = UINT32_MAX;
        if (TOPK) {
            if (!C.valid) tk->cnt[threadIdx.x] = 0;
            topk_publish(sm, *tk, threadIdx.x, a.k, fp, N,
                         (a.gch && C.valid) ? a.gch + 2 * (size_t)r : nullptr, &a.ds);
        } else {
            publish_threshold(sm, threadIdx.x, fp, N);
        }
    }
    __syncthreads();
    volatile int* abort_flag = &sm.abort_flag;

    if (warp == 0) {
        // ---------------------------------------------------------------- loads
        if (lane == 0) {
            int s = 0;
            if (kBRes) {
                mbar_expect_tx(&sm.bres, KST * kStageB);
                for (int t = 0; t < KST; ++t)
                    bulk_load(stB + t * kStageB, btile + (size_t)t * kStageB, kStageB, &sm.bres);
            }
            for (int mt = m_begin; mt < m_end && !*abort_flag; ++mt) {
                const int ar = mt / tiles_per_row;
                const int q0 = (mt % tiles_per_row) * (kM / P);
                // First row of the domain row's window: a pixel row (fold) or a
                // contracted-plane row (digits).
                const int dom_row = DIG ? ar * (g.shift / 2) : ar * g.shift;
                for (int t = 0; t < KST; ++t) {
                    const uint32_t bit = 1u << s;
                    // A stage filled before is refilled once the MMAs of its last fill
                    // have completed.
                    if ((ps.stage_used & bit) &&
                        !mbar_wait(&sm.empty[s], (ps.stage_par & bit) ? 0u : 1u, abort_flag, err, 1))
                        break;
                    mbar_expect_tx(&sm.full[s], C_::kTx);
                    const int kg0 = t * 8;
                    const int j = kg0 / ROWS, y0 = kg0 % ROWS;
                    unsigned char* dstA = stA + s * kStageAll;
                    if (DIG) {
                        tma_load_4d(dstA, &maps.all, 16 * (q0 + j), dom_row + y0, &sm.full[s]);
                        tma_load_4d(dstA + kStageA, &maps.all_lo, 16 * (q0 + j), dom_row + y0,
                                    &sm.full[s]);
                    } else if (maps.use_all) {
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
                    ps.stage_used |= bit;
                    ps.stage_par ^= bit;
                    if (++s == kStages) s = 0;
                }
            }
            // Drain: wait (bounded) for the loads still in flight before leaving -- each
            // stage's last fill, and the resident B tile.
            if (*abort_flag) {
                for (int s2 = 0; s2 < kMaxStages; ++s2) {
                    const uint32_t bit = 1u << s2;
                    if (!(ps.stage_used & bit)) continue;
                    const uint32_t par = (ps.stage_par & bit) ? 0u : 1u;  // the last fill's
                    const long long t0 = clock64();
                    while (!mbar_try_wait(&sm.full[s2], par) && clock64() - t0 < kWaitCycles) {
                    }
                }
                if (kBRes) {
                    const long long t0 = clock64();
                    while (!mbar_try_wait(&sm.bres, ps.bres & 1u) && clock64() - t0 < kWaitCycles) {
                    }
                }
            }
            if (kBRes) ++ps.bres;
        }
    } else if (warp == 1) {
        // ---------------------------------------------------------------- MMA
        if (lane == 0) {
            int s = 0;
            bool ok = true;
            if (kBRes) {
                ok = mbar_wait(&sm.bres, ps.bres & 1u, abort_flag, err, 2);
                ++ps.bres;
            }
            for (int mt = m_begin; ok && mt < m_end; ++mt) {
                const uint32_t i = ps.tiles++;
                const int b = (int)(i & 1u);
                const uint32_t bph = (i >> 1) & 1u;
                if (i >= 2 && !mbar_wait(&sm.tempty[b], bph ^ 1, abort_flag, err, 4)) break;
                tmem_fence_after();
                const uint32_t dcol = tmem + (uint32_t)(b * kN);
                for (int t = 0; t < KST; ++t) {
                    const uint32_t bit = 1u << s;
                    if (!mbar_wait(&sm.full[s], (ps.stage_par & bit) ? 1u : 0u, abort_flag, err, 8)) {
                        ok = false;
                        break;
                    }
                    ps.stage_par ^= bit;
                    tmem_fence_after();
                    const uint32_t a_addr = smem_u32(stA + s * kStageAll);
                    const uint32_t b_addr = smem_u32(kBRes ? stB + t * kStageB : stB + s * kStageB);
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) {
                        const uint64_t bd = smem_desc(b_addr + kk * 256);
                        const uint32_t acc = (t > 0 || kk > 0) ? 1u : 0u;
                        mma_i8<NT>(dcol, smem_desc(a_addr + kk * 256), bd, acc);
                        if (DIG)  // low digit into the buffer's second half
                            mma_i8<NT>(dcol + NT, smem_desc(a_addr + kStageA + kk * 256), bd, acc);
                    }
                    mma_commit(&sm.empty[s]);
                    if (++s == kStages) s = 0;
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
        const int e = warp & 3;
        const int part = (warp - 2) >> 2;        // = the epilogue group
        const int gt = threadIdx.x - 64 - part * kGroupThreads;  // 0..kGroupThreads-1
        const int m = e * 32 + lane;             // this thread's domain lane
        const float four_inv_n = 4.0f / (float)N;

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

        for (int mt = m_begin; mt < m_end; ++mt) {
            const uint32_t i = ps.tiles++;
            const int b = (int)(i & 1u);
            const uint32_t bph = (i >> 1) & 1u;
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
            // form).  They do not depend on the accumulator: the 4 of 32-column chunk ch are
            // computed while that chunk's accumulator load and the previous chunk's test are
            // in flight, so the independent chains interleave (all 16 up front, before the
            // scan, measured 10 % slower at s = 4 with the 32-byte record).
            int32_t thr[kRangesPerWarp];
            auto chunk_thresholds = [&](int ch) {
                const float4* rec = reinterpret_cast<const float4*>(sm.thr);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int r = 4 * ch + q;
                    const float4 ra = rec[part * kRangesPerWarp + r];
                    const int tie = __float_as_int(ra.w);
                    // s1 * c + tau with one rounding toward -inf (fma): still never above
                    // the exact threshold.
                    const float g1 = __fmul_rd(ra.x, sdetf);
                    const float tz = fminf(__fadd_rd(ra.y, ahd), fmaxf(g1, ad));
                    const float tau = dom > tie ? tz : g1;
                    thr[r] = __float2int_rd(__fmaf_rd(s1f, ra.z, tau));
                }
            };
            // Whether any column of chunk ch can survive.  A lane past the domain row's end
            // (dom < 0) never passes; its thresholds, from stale or zero statistics, are
            // never read.
            auto chunk_pass = [&](const int32_t (&v)[32], int ch) {
                return (dom >= 0) & ((max8(v, 0) >= thr[ch * 4]) | (max8(v, 8) >= thr[ch * 4 + 1]) |
                                     (max8(v, 16) >= thr[ch * 4 + 2]) |
                                     (max8(v, 24) >= thr[ch * 4 + 3]));
            };
            auto chunk_rare = [&](const int32_t (&v)[32], int ch) {
                const int32_t t0 = thr[ch * 4], t1 = thr[ch * 4 + 1];
                const int32_t t2 = thr[ch * 4 + 2], t3 = thr[ch * 4 + 3];
                {
                    // Rare: bit c of `mask` = column c of this chunk survives (and was not
                    // fitted by an earlier pass over this accumulator).
                    uint32_t mask = 0u;
#pragma unroll
                    for (int c = 0; c < 32; ++c) {
                        const int32_t tc = c < 8 ? t0 : (c < 16 ? t1 : (c < 24 ? t2 : t3));
                        mask |= (v[c] >= tc ? 1u : 0u) << c;
                    }
                    const int col0 = part * kColsPerWarp + ch * 32;
                    if (rescan) mask &= ~sm.evaluated[(m * NT + col0) >> 5];
                    int slot = atomicAdd(&sm.qcount[part], __popc(mask));
                    while (mask) {
                        const int c = __ffs(mask) - 1;
                        mask &= mask - 1;
                        int32_t val = v[0];
#pragma unroll
                        for (int q = 1; q < 32; ++q) val = c == q ? v[q] : val;
                        if (slot < kQueueCap)
                            sm.queue[part][slot] = QEntry{val, (uint32_t)dom,
                                                    (uint32_t)(tag << 16 | m << 8 | (col0 + c)), 0u, 0.0, 0.0};
                        ++slot;
                    }
                }
            };
            auto test_chunk = [&](const int32_t (&v)[32], int ch) {
                if (chunk_pass(v, ch)) chunk_rare(v, ch);
            };
            const bool got = mbar_wait(&sm.tfull[b], bph, abort_flag, err, 16);
            if (!group_barrier_and(part, got)) break;
            tmem_fence_after();
            for (;;) {
                // ---- scan: this thread's accumulator columns in 32-column chunks, each
                // chunk's load overlapped with the previous chunk's test
                static_assert(kChunks % 2 == 0, "chunks are scanned in pairs");
                int32_t va[32], vb[32];
                __syncwarp();
                if (DIG) {
                    // t1' = 128 hi + lo per column, both digits' accumulators loaded together
                    // (exact: |t1'| < 2^31).
#pragma unroll
                    for (int ch = 0; ch < kChunks; ++ch) {
                        tmem_ld32(tcol + 32u * ch, va);
                        tmem_ld32(tcol + (uint32_t)NT + 32u * ch, vb);
                        chunk_thresholds(ch);
                        tmem_wait(va);
                        tmem_wait(vb);
#pragma unroll
                        for (int c = 0; c < 32; ++c) va[c] = va[c] * 128 + vb[c];
                        test_chunk(va, ch);
                        __syncwarp();
                    }
                } else {
#pragma unroll
                    for (int ch = 0; ch < kChunks; ch += 2) {
                        // Two chunks per round: both loads in flight while their 8
                        // thresholds are computed, one branch for the pair.
                        tmem_ld32(tcol + 32u * ch, va);
                        tmem_ld32(tcol + 32u * (ch + 1), vb);
                        chunk_thresholds(ch);
                        chunk_thresholds(ch + 1);
                        tmem_wait(va);
                        tmem_wait(vb);
                        const bool pa = chunk_pass(va, ch), pb = chunk_pass(vb, ch + 1);
                        if (pa | pb) {
                            if (pa) chunk_rare(va, ch);
                            if (pb) chunk_rare(vb, ch + 1);
                        }
                        __syncwarp();
                    }
                }

                group_barrier(part);
                const int queued = sm.qcount[part];
                const bool last = mt + 1 == m_end;
                if (queued > kQueueCap) {
                    if (TOPK)
                        drain_queue_topk<N, NT, kRangesPerWarp>(sm, *tk, a.k, part, kQueueCap,
                                                                true, tag, gt, ds, fp, exact,
                                                                a.gch, ntile * RT);
                    else
                        drain_queue<N, NT, kRangesPerWarp>(sm, part, kQueueCap, true, tag, gt,
                                                           ds, fp, exact, a.gch, ntile * RT);
                    rescan = true;
                    continue;  // pass again over the same accumulator (fresh thresholds)
                }
                if (queued >= kFlush || (last && queued > 0)) {
                    if (TOPK)
                        drain_queue_topk<N, NT, kRangesPerWarp>(sm, *tk, a.k, part, queued,
                                                                false, tag, gt, ds, fp, exact,
                                                                a.gch, ntile * RT);
                    else
                        drain_queue<N, NT, kRangesPerWarp>(sm, part, queued, false, tag, gt,
                                                           ds, fp, exact, a.gch, ntile * RT);
                }
                break;
            }
            if (rescan) {
                // This group's words of the bitmask: NT / 64 of each lane's NT / 32.
                constexpr int kWg = NT / 64;
                for (int w2 = gt; w2 < kM * kWg; w2 += kGroupThreads)
                    sm.evaluated[(w2 / kWg) * (NT / 32) + part * kWg + w2 % kWg] = 0u;
                group_barrier(part);
            }
            // The accumulator has been read completely: hand it back to the MMA warp.
            tmem_fence_before();
            mbar_arrive(&sm.tempty[b]);
        }
    }

    // ---------------------------------------------------------------- item end
    tmem_fence_before();
    __syncthreads();
    tmem_fence_after();
    if (TOPK && threadIdx.x < RT) {
        // The range's sorted list as this split's k partials (idx UINT32_MAX past its end).
        const int r = ntile * RT + threadIdx.x;
        if (r < nranges) {
            const int c = sm.ch[threadIdx.x].valid ? tk->cnt[threadIdx.x] : 0;
            for (int j = 0; j < a.k; ++j) {
                Partial p;
                if (j < c) {
                    p.rms = tk->rms[threadIdx.x][j];
                    p.sum = tk->sum[threadIdx.x][j];
                    p.idx = tk->idx[threadIdx.x][j];
                    p.t1x4 = tk->t1[threadIdx.x][j];
                    p.qalfa = (uint16_t)(tk->q[threadIdx.x][j] & 0xFFFFu);
                    p.qbeta = (uint16_t)(tk->q[threadIdx.x][j] >> 16);
                } else {
                    p.rms = INFINITY;
                    p.sum = 0.0;
                    p.idx = UINT32_MAX;
                    p.t1x4 = 0;
                    p.qalfa = 0;
                    p.qbeta = 0;
                }
                p.pad = 0;
                a.partials[((size_t)split * nranges + r) * a.k + j] = p;
            }
        }
    } else if (threadIdx.x < RT) {
        const Champ& C = sm.ch[threadIdx.x];
        const int r = ntile * RT + threadIdx.x;
        if (r < nranges) {
            Partial p;
            p.rms = C.rms;
            p.sum = C.sum;
            p.idx = C.idx;
            p.t1x4 = C.t1x4;
            p.qalfa = 0;
            p.qbeta = 0;
            p.pad = 0;
            a.partials[(size_t)split * nranges + r] = p;
        }
    }
    if (a.tickets) {
        // The last of the range tile's splits to get here finishes its ranges (the
        // threadfence-reduction pattern: partials, fence, ticket; the last CTA fences
        // again and reads every split's partials around L1).
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) sm.last = atomicAdd(&a.tickets[ntile], 1) == a.msplit - 1;
        __syncthreads();
        if (sm.last) {
            __threadfence();
            const int r = ntile * RT + threadIdx.x;
            if (a.merge_seeds) {
                if (threadIdx.x < RT && r < nranges)
                    seed_merge_range(a.partials, a.msplit, nranges, r, g.ncol_d, a.fine_ncol,
                                     a.merge_ratio, a.merge_seeds);
                __threadfence();
                __syncthreads();
                if (threadIdx.x == 0) st_release_gpu(a.ready + ntile, 1);
            } else if (threadIdx.x < RT && r < nranges) {
                finish_range(a.partials, a.msplit, nranges, r, g, a.rs, ds, fp, a.out);
            }
        }
    }
}

// Shared-memory bytes of a level's pipeline stages (A, and B stages or the resident B tile).
template <int S, bool DIG>
__host__ __device__ constexpr size_t stage_bytes() {
    using C_ = Cfg<S, DIG>;
    return (size_t)C_::kStages * C_::kDigits * kStageA +
           (C_::kBRes ? (size_t)C_::KST * C_::kStageBt : (size_t)C_::kStages * C_::kStageBt);
}

// The correlation of one level: CTA (x, y) = range tile x against domain-tile split y.
// TOPK: the ranked search (a.k candidates per range; its lists after the stages).
template <int S, bool DIG, bool TOPK>
__global__ void __launch_bounds__(kThreads, 1)
    corr_tc_kernel(const __grid_constant__ TcMaps maps, const __grid_constant__ ItemArgs a,
                   int* __restrict__ err,
                   unsigned long long* __restrict__ exact_counter) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    Smem& sm = smem_record(smem_raw);
    unsigned char* stages = reinterpret_cast<unsigned char*>(&sm) + kSmemHead;
    TopkLists* tk = TOPK ? reinterpret_cast<TopkLists*>(stages + stage_bytes<S, DIG>()) : nullptr;
    const uint32_t tmem = cta_setup(sm);
    PipeState ps;
    unsigned long long exact = 0;
    process_item<S, DIG, TOPK>(maps, a, blockIdx.x, blockIdx.y, sm, stages, tmem, ps, err, exact,
                               tk);
    cta_teardown(sm, tmem, exact, exact_counter);
}

// All tensor-core levels of a plane in one persistent launch: one CTA per SM takes work
// items -- (level job, range tile, domain-tile split) -- from a global counter until none
// are left.  TMEM, the mbarriers and the epilogue's queues are set up once per CTA; the
// pipelines' phases carry over from item to item (PipeState).  Jobs are ordered by item
// cost, largest first, so the cheap items fill the end.  Each range tile's last split
// writes the tile's final candidates (no finish launch).
struct AllLevels {
    TcMaps maps[kMaxLevelJobs];
    ItemArgs args[kMaxLevelJobs];
    int kind[kMaxLevelJobs];  // 0: S=4 fold, 1: S=8 fold, 2/3/4: S=16/32/64 digits
    int tile_begin[kMaxLevelJobs];
    int tile_count[kMaxLevelJobs];
    int item_begin[kMaxLevelJobs + 1];
    int njobs;
};

static_assert(sizeof(AllLevels) <= 32000, "kernel parameter space");

__global__ void __launch_bounds__(kThreads, 1)
    corr_tc_all_kernel(const __grid_constant__ AllLevels L, int* __restrict__ work,
                       int* __restrict__ err, unsigned long long* __restrict__ exact_counter) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    Smem& sm = smem_record(smem_raw);
    unsigned char* stages = reinterpret_cast<unsigned char*>(&sm) + kSmemHead;
    const uint32_t tmem = cta_setup(sm);
    PipeState ps;
    unsigned long long exact = 0;
    const int nitems = L.item_begin[L.njobs];
    volatile int* abort_flag = &sm.abort_flag;
    if (threadIdx.x == 0) sm.item = (int)blockIdx.x;
    __syncthreads();
    for (;;) {
        const int item = sm.item;
        if (item >= nitems || *abort_flag) break;
        int j = 0;
        while (j + 1 < L.njobs && item >= L.item_begin[j + 1]) ++j;
        // Parameter-space references: nothing of the job is copied.
        const TcMaps& maps = L.maps[j];
        const ItemArgs& a = L.args[j];
        // Split-major within a job: a range tile's later splits start after its earlier
        // ones have finished and begin from their champions (the shared records).
        const int local = item - L.item_begin[j];
        const int ntile = L.tile_begin[j] + local % L.tile_count[j];
        const int split = local / L.tile_count[j];
        switch (L.kind[j]) {
            case 0:
                process_item<4, false>(maps, a, ntile, split, sm, stages, tmem, ps, err, exact);
                break;
            case 1:
                process_item<8, false>(maps, a, ntile, split, sm, stages, tmem, ps, err, exact);
                break;
            case 2:
                process_item<16, true>(maps, a, ntile, split, sm, stages, tmem, ps, err, exact);
                break;
            case 3:
                process_item<32, true>(maps, a, ntile, split, sm, stages, tmem, ps, err, exact);
                break;
            default:
                process_item<64, true>(maps, a, ntile, split, sm, stages, tmem, ps, err, exact);
                break;
        }
        if (threadIdx.x == 0) sm.item = (int)gridDim.x + atomicAdd(work, 1);
        __syncthreads();
    }
    cta_teardown(sm, tmem, exact, exact_counter);
}

// B operand of one level: rows n = range * 8 + isometry; for each N tile (NT rows) and each
// 128-byte K stage, NT / 8 row groups x 8 K-groups x (8 rows x 16 B).  Fold path: the range
// sample r[map_k(u, v)] - 128 upsampled 2x2 onto the domain's 2S x 2S pixel positions;
// digit path: the S x S samples themselves (the positions of the contracted window).
template <int S, bool DIG>
__global__ void build_b_kernel(const uint8_t* __restrict__ plane, int w, int h,
                               const uint32_t* rows, const uint32_t* cols, int nranges,
                               int ntiles, uint8_t* __restrict__ out) {
    using C_ = Cfg<S, DIG>;
    constexpr int NT = C_::kNt;
    constexpr int ROWS = C_::ROWS;
    constexpr int KG = C_::J * ROWS;
    constexpr int KST = KG / 8;
    constexpr int XMAX = DIG ? S : 2 * S;  // K positions per row that carry a sample
    // one thread per (n, kg): writes one 16-byte K-group of one B row
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)ntiles * NT * KG;
    if (tid >= total) return;
    const int kg = (int)(tid % KG);
    const long long nglob = tid / KG;
    const int nt = (int)(nglob / NT), n = (int)(nglob % NT);
    const int r = nt * C_::kRt + n / 8, k = n % 8;
    const int j = kg / ROWS, y = kg % ROWS;
    const int t = kg / 8, kgl = kg % 8;
    const bool inside = r < nranges && rows[r] + (uint32_t)S <= (uint32_t)h &&
                        cols[r] + (uint32_t)S <= (uint32_t)w;
    uint8_t bytes[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        const int x = 16 * j + e;
        int8_t val = 0;
        if (inside && x < XMAX) {
            const int u = DIG ? y : y >> 1, vv = DIG ? x : x >> 1;
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
    const size_t off = (((size_t)nt * KST + t) * (NT / 8) + (n >> 3)) * 1024 + (size_t)kgl * 128 +
                       (size_t)(n & 7) * 16;
    uint4 pk;
    pk.x = bytes[0] | bytes[1] << 8 | bytes[2] << 16 | (uint32_t)bytes[3] << 24;
    pk.y = bytes[4] | bytes[5] << 8 | bytes[6] << 16 | (uint32_t)bytes[7] << 24;
    pk.z = bytes[8] | bytes[9] << 8 | bytes[10] << 16 | (uint32_t)bytes[11] << 24;
    pk.w = bytes[12] | bytes[13] << 8 | bytes[14] << 16 | (uint32_t)bytes[15] << 24;
    *reinterpret_cast<uint4*>(out + off) = pk;
}

// Digit phase copies of the contracted plane D (dw x dh, i32, 0..1020): plane
// z = digit * P + p (digit 0 = hi = D >> 7, 1 = lo = D & 127) is that digit shifted left by
// STEP * p samples, zero past the right edge; row pitch wp (a multiple of 16).  One thread
// per 16 output columns of a row: it loads the 32 - STEP samples every phase of those
// columns reads once and writes 16 bytes to each of the 2 P planes.
template <int STEP>
__global__ void digit_planes_kernel(const int32_t* __restrict__ D, int dw, int dh, int wp,
                                    uint8_t* __restrict__ out) {
    constexpr int P = 16 / STEP, SPAN = 16 + STEP * (P - 1);
    const int x = 16 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int y = blockIdx.y;
    if (x >= wp || y >= dh) return;
    const int32_t* row = D + (size_t)y * dw;
    uint8_t hi[SPAN], lo[SPAN];
#pragma unroll
    for (int i = 0; i < SPAN; ++i) {
        const int v = x + i < dw ? __ldg(row + x + i) : 0;
        hi[i] = (uint8_t)(v >> 7);
        lo[i] = (uint8_t)(v & 127);
    }
#pragma unroll
    for (int p = 0; p < P; ++p) {
        uint32_t wh[4], wl[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int b = STEP * p + 4 * k;
            wh[k] = hi[b] | hi[b + 1] << 8 | hi[b + 2] << 16 | (uint32_t)hi[b + 3] << 24;
            wl[k] = lo[b] | lo[b + 1] << 8 | lo[b + 2] << 16 | (uint32_t)lo[b + 3] << 24;
        }
        *reinterpret_cast<uint4*>(out + ((size_t)p * dh + y) * wp + x) =
            make_uint4(wh[0], wh[1], wh[2], wh[3]);
        *reinterpret_cast<uint4*>(out + ((size_t)(P + p) * dh + y) * wp + x) =
            make_uint4(wl[0], wl[1], wl[2], wl[3]);
    }
}

// Phase copies of the plane: copy p (of P = 16 / SHIFT) is the plane shifted left by
// SHIFT * p pixels, zero past the right edge; row pitch wp (a multiple of 16).  One thread
// per 16 output columns of a row: the 32 - SHIFT source bytes all phases read, loaded once,
// and one 16-byte store per phase.
template <int SHIFT>
__global__ void phase_planes_kernel(const uint8_t* __restrict__ plane, int w, int h, int wp,
                                    uint8_t* __restrict__ out) {
    constexpr int P = 16 / SHIFT, SPAN = 16 + SHIFT * (P - 1);
    const int x = 16 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int y = blockIdx.y;
    if (x >= wp || y >= h) return;
    const uint8_t* row = plane + (size_t)y * w;
    uint8_t v[SPAN];
#pragma unroll
    for (int i = 0; i < SPAN; ++i) v[i] = x + i < w ? __ldg(row + x + i) : (uint8_t)0;
#pragma unroll
    for (int p = 0; p < P; ++p) {
        uint32_t wd[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int b = SHIFT * p + 4 * k;
            wd[k] = v[b] | v[b + 1] << 8 | v[b + 2] << 16 | (uint32_t)v[b + 3] << 24;
        }
        *reinterpret_cast<uint4*>(out + ((size_t)p * h + y) * wp + x) =
            make_uint4(wd[0], wd[1], wd[2], wd[3]);
    }
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
    if (warp == 0) {
        // The best of the 72 by (rms, reference index): each lane takes candidates lane,
        // lane + 32, lane + 64, then a shuffle reduction.
        int b = lane;
        for (int c = lane + 32; c < 72; c += 32)
            if (c_rms[c] < c_rms[b] || (c_rms[c] == c_rms[b] && c_idx[c] < c_idx[b])) b = c;
        double br = c_rms[b];
        uint32_t bi = c_idx[b];
        for (int o = 16; o > 0; o >>= 1) {
            const double r2 = __shfl_xor_sync(0xffffffffu, br, o);
            const uint32_t i2 = __shfl_xor_sync(0xffffffffu, bi, o);
            const int b2 = __shfl_xor_sync(0xffffffffu, b, o);
            if (r2 < br || (r2 == br && i2 < bi)) {
                br = r2;
                bi = i2;
                b = b2;
            }
        }
        if (lane == 0) out[r] = SeedOut{c_rms[b], c_sum[b], c_idx[b], c_t1[b]};
    }
}

// Seeds of the ranked search: the same 72 candidates as seed_kernel (3 x 3 domains around
// the co-located one x 8 isometries, exact int32 correlations, exact fits), of which the
// best k distinct ones by (rms, reference index) start the range's list.  The patch is
// clamped to the pool, so a domain can appear twice; "distinct" drops the repeats.  At least
// one domain x 8 isometries is always there, so k <= 8 candidates exist.
template <int S>
__global__ void __launch_bounds__(288) seed_topk_kernel(
    const int32_t* __restrict__ D, LevelGeom g, const uint8_t* __restrict__ plane, int w,
    const uint32_t* rows, const uint32_t* cols, int nranges, RangeStats rs, DomainStats ds,
    FitParams fp, int k, SeedOut* __restrict__ out) {
    constexpr int N = S * S;
    __shared__ uint8_t rsm[N];
    __shared__ double c_rms[72], c_sum[72];
    __shared__ uint32_t c_idx[72];
    __shared__ int32_t c_t1[72];
    const int r = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (r >= nranges) return;
    if (rows[r] + (uint32_t)S > (uint32_t)g.h || cols[r] + (uint32_t)S > (uint32_t)g.w) {
        if (threadIdx.x < k) out[(size_t)r * k + threadIdx.x] = SeedOut{INFINITY, 0.0, UINT32_MAX, 0};
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
    for (int q = 0; q < 8; ++q) acc[q] = 0;
    for (int t = lane; t < N; t += 32) {
        const int u = t / S, v = t % S;
        const int32_t d = db[(size_t)u * g.dw + v];
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[q] += (int32_t)rsm[iso_src_rt(q, u, v, S)] * d;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], off);
    if (lane < 8) {
        int32_t t1 = acc[0];
#pragma unroll
        for (int q = 1; q < 8; ++q) t1 = lane == q ? acc[q] : t1;
        const uint32_t dom = (uint32_t)(a * g.ncol_d + bb);
        const FitResult f = fit_exact(N, ds.s1x4[dom], ds.s2x16[dom], rs.t0[r], t1, rs.t2[r], fp);
        c_rms[nb * 8 + lane] = f.rms;
        c_sum[nb * 8 + lane] = f.sum;
        c_idx[nb * 8 + lane] = dom * 8u + (uint32_t)lane;
        c_t1[nb * 8 + lane] = t1;
    }
    __syncthreads();
    if (warp == 0) {
        // k rounds of a warp arg-min over the candidates strictly after the previous pick
        // in (rms, index) order.
        double pr = 0.0;
        uint32_t pi = 0;
        for (int j = 0; j < k; ++j) {
            int b = -1;
            for (int c = lane; c < 72; c += 32) {
                if (j > 0 && !(c_rms[c] > pr || (c_rms[c] == pr && c_idx[c] > pi))) continue;
                if (b < 0 || c_rms[c] < c_rms[b] || (c_rms[c] == c_rms[b] && c_idx[c] < c_idx[b]))
                    b = c;
            }
            double br = b < 0 ? INFINITY : c_rms[b];
            uint32_t bi = b < 0 ? UINT32_MAX : c_idx[b];
            for (int o = 16; o > 0; o >>= 1) {
                const double r2 = __shfl_xor_sync(0xffffffffu, br, o);
                const uint32_t i2 = __shfl_xor_sync(0xffffffffu, bi, o);
                const int b2 = __shfl_xor_sync(0xffffffffu, b, o);
                if (r2 < br || (r2 == br && i2 < bi)) {
                    br = r2;
                    bi = i2;
                    b = b2;
                }
            }
            if (lane == 0)
                out[(size_t)r * k + j] = b < 0 ? SeedOut{INFINITY, 0.0, UINT32_MAX, 0}
                                               : SeedOut{c_rms[b], c_sum[b], c_idx[b], c_t1[b]};
            pr = br;
            pi = bi;
        }
    }
}

constexpr int kSeedSide = 3;                       // seed domains: a 3 x 3 patch
constexpr int kSeedCands = 8 * kSeedSide * kSeedSide;  // x 8 isometries

// seed_kernel for the small blocks (S = 4, 8): the same 72 candidates, one warp per range
// block (8 per CTA).  Lane l correlates candidates l, l + 32, l + 64 whole (S^2 terms) from the
// range staged in shared memory; isometry::map is affine in (u, v), so a candidate walks the
// staged range with a base and two strides and lanes of different isometries do not
// diverge.  One (rms, reference index) reduction picks the winner.
template <int S>
__global__ void __launch_bounds__(256) seed_small_kernel(
    const int32_t* __restrict__ D, LevelGeom g, const uint8_t* __restrict__ plane, int w,
    const uint32_t* rows, const uint32_t* cols, int nranges, RangeStats rs, DomainStats ds,
    FitParams fp, SeedOut* __restrict__ out) {
    constexpr int N = S * S;
    __shared__ uint8_t rsm[8][N];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = blockIdx.x * 8 + warp;
    if (r >= nranges) return;
    if (rows[r] + (uint32_t)S > (uint32_t)g.h || cols[r] + (uint32_t)S > (uint32_t)g.w) {
        if (lane == 0) out[r] = SeedOut{INFINITY, 0.0, UINT32_MAX, 0};
        return;
    }
    const uint8_t* rb = plane + (size_t)rows[r] * w + cols[r];
    for (int t = lane; t < N; t += 32) rsm[warp][t] = rb[(size_t)(t / S) * w + (t % S)];
    __syncwarp();
    const int ac = min(max(((int)rows[r] - S / 2 + g.shift / 2) / g.shift, 0), g.nrow_d - 1);
    const int bc = min(max(((int)cols[r] - S / 2 + g.shift / 2) / g.shift, 0), g.ncol_d - 1);
    double best = INFINITY, best_sum = 0.0;
    uint32_t best_idx = UINT32_MAX;
    int32_t best_t1 = 0;
    for (int c = lane; c < kSeedCands; c += 32) {
        const int nb = c >> 3, k = c & 7;
        const int a = min(max(ac + nb / kSeedSide - kSeedSide / 2, 0), g.nrow_d - 1);
        const int bb = min(max(bc + nb % kSeedSide - kSeedSide / 2, 0), g.ncol_d - 1);
        const int32_t* db = D + (size_t)(a * g.step_c) * g.dw + bb * g.step_c;
        // iso_src_rt(k, u, v, S) = base + u * du + v * dv
        int base, du, dv;
        switch (k) {
            case 0: base = 0; du = S; dv = 1; break;
            case 1: base = (S - 1) * S; du = 1; dv = -S; break;
            case 2: base = S - 1; du = -1; dv = S; break;
            case 3: base = (S - 1) * S + S - 1; du = -S; dv = -1; break;
            case 4: base = S - 1; du = S; dv = -1; break;
            case 5: base = (S - 1) * S; du = -S; dv = 1; break;
            case 6: base = 0; du = 1; dv = S; break;
            default: base = (S - 1) * S + S - 1; du = -1; dv = -S; break;
        }
        const uint8_t* rr = rsm[warp];
        int32_t t1 = 0;
#pragma unroll
        for (int u = 0; u < S; ++u)
#pragma unroll
            for (int v = 0; v < S; ++v)
                t1 += (int32_t)rr[base + u * du + v * dv] * db[(size_t)u * g.dw + v];
        const uint32_t dom = (uint32_t)(a * g.ncol_d + bb);
        const FitResult f = fit_exact(N, ds.s1x4[dom], ds.s2x16[dom], rs.t0[r], t1, rs.t2[r], fp);
        const uint32_t idx = dom * 8u + (uint32_t)k;
        if (f.rms < best || (f.rms == best && idx < best_idx)) {
            best = f.rms;
            best_sum = f.sum;
            best_idx = idx;
            best_t1 = t1;
        }
    }
    double br = best;
    uint32_t bi = best_idx;
    int bl = lane;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double r2 = __shfl_xor_sync(0xffffffffu, br, o);
        const uint32_t i2 = __shfl_xor_sync(0xffffffffu, bi, o);
        const int l2 = __shfl_xor_sync(0xffffffffu, bl, o);
        if (r2 < br || (r2 == br && i2 < bi)) {
            br = r2;
            bi = i2;
            bl = l2;
        }
    }
    if (lane == bl) out[r] = SeedOut{best, best_sum, best_idx, best_t1};
}

// The coarse pre-pass's seeds merged into the full grid's (seed_merge_range), one thread
// per range.
__global__ void seed_merge_kernel(const Partial* __restrict__ partials, int nsplit, int nranges,
                                  int coarse_ncol, int fine_ncol, int ratio,
                                  SeedOut* __restrict__ seeds) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nranges)
        seed_merge_range(partials, nsplit, nranges, r, coarse_ncol, fine_ncol, ratio, seeds);
}

// Final champion over the M-splits of each range (finish_range).
__global__ void finish_kernel(const Partial* __restrict__ partials, int nsplit, int nranges,
                              LevelGeom g, RangeStats rs, DomainStats ds, FitParams fp,
                              CandidateOut* __restrict__ out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nranges) finish_range(partials, nsplit, nranges, r, g, rs, ds, fp, out);
}

template <int S, bool DIG>
constexpr size_t smem_bytes() {
    using C_ = Cfg<S, DIG>;
    static_assert(C_::kStages <= kMaxStages, "pipeline depth");
    return 1024 + kSmemHead + stage_bytes<S, DIG>();
}
static_assert(smem_bytes<32, true>() + sizeof(TopkLists) <= 232448 &&
                  smem_bytes<64, true>() + sizeof(TopkLists) <= 232448 &&
                  smem_bytes<4, false>() + sizeof(TopkLists) <= 232448,
              "shared memory per CTA of the ranked kernel (227 KB)");
static_assert(smem_bytes<4, false>() <= 232448 && smem_bytes<8, false>() <= 232448 &&
                  smem_bytes<16, false>() <= 232448 && smem_bytes<32, false>() <= 232448 &&
                  smem_bytes<16, true>() <= 232448 && smem_bytes<32, true>() <= 232448 &&
                  smem_bytes<64, true>() <= 232448,
              "shared memory per CTA (227 KB)");

template <int S, bool DIG, bool TOPK = false>
cudaError_t launch_t(const TcMaps& maps, const uint8_t* bglob, const LevelGeom& g, int nranges,
                     RangeStats rs, DomainStats ds, const FitParams& fp, const SeedOut* seeds,
                     Partial* partials, unsigned long long* gch, int msplit, int* err,
                     unsigned long long* counter, cudaStream_t st, int k = 1) {
    const int tiles_per_row = (g.ncol_d + kM - 1) / kM;
    const int m_tiles = g.nrow_d * tiles_per_row;
    const int m_per_cta = (m_tiles + msplit - 1) / msplit;
    const int ntiles = (nranges + Cfg<S, DIG>::kRt - 1) / Cfg<S, DIG>::kRt;
    const size_t smem = smem_bytes<S, DIG>() + (TOPK ? sizeof(TopkLists) : 0);
    auto kern = corr_tc_kernel<S, DIG, TOPK>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid(ntiles, msplit);
    const ItemArgs a{bglob, g,        nranges,  rs,       ds,      fp,     seeds,
                     m_tiles, m_per_cta, msplit, partials, gch, nullptr, nullptr, k,
                     nullptr, 0, 0, nullptr, nullptr};
    kern<<<grid, kThreads, smem, st>>>(maps, a, err, counter);
    return cudaGetLastError();
}

template <int S, bool DIG>
cudaError_t build_b_t(const uint8_t* plane, int w, int h, const uint32_t* rows,
                      const uint32_t* cols, int nranges, uint8_t* out, cudaStream_t st) {
    using C_ = Cfg<S, DIG>;
    constexpr int KG = C_::J * C_::ROWS;
    const int ntiles = (nranges + C_::kRt - 1) / C_::kRt;
    const long long total = (long long)ntiles * C_::kNt * KG;
    build_b_kernel<S, DIG><<<(unsigned)((total + 255) / 256), 256, 0, st>>>(
        plane, w, h, rows, cols, nranges, ntiles, out);
    return cudaGetLastError();
}

}  // namespace

bool supported(int size, int shift) {
    return (size == 4 || size == 8 || size == 16 || size == 32 || size == 64) &&
           (shift == 2 || shift == 4 || shift == 8 || shift == 16);
}

bool digits_supported(int size, int shift) {
    return (size == 16 || size == 32 || size == 64) &&
           (shift == 2 || shift == 4 || shift == 8 || shift == 16);
}

int ranges_per_tile(bool digits) { return digits ? 16 : 32; }

size_t b_bytes(int size, int nranges, bool digits) {
    // K-groups of 16 bytes per B row: fold J * 2S with J = max(1, S / 8); digits S * S / 16.
    const int KG = digits ? size * size / 16 : (size >= 8 ? size / 8 : 1) * 2 * size;
    const int rt = ranges_per_tile(digits);
    const size_t ntiles = (size_t)(nranges + rt - 1) / rt;
    return ntiles * (size_t)(rt * 8) * (size_t)KG * 16;
}

int phase_count(int shift) { return 16 / shift; }
int row_pitch(int w) { return ((w + 15) / 16) * 16 + 16; }
// The 4-D view reads up to (16/P - 1) * 128 bytes past a row's end (columns no valid
// domain uses); the allocation carries that much slack after the last phase copy.
size_t phase_bytes(int w, int h, int shift) {
    return (size_t)phase_count(shift) * h * row_pitch(w) + 2048;
}
int digit_phase_count(int shift) { return 32 / shift; }
size_t digit_plane_bytes(int w, int h, int shift) {
    return 2 * (size_t)digit_phase_count(shift) * (h / 2) * row_pitch(w / 2) + 2048;
}

cudaError_t launch_digit_planes(const int32_t* D, int w, int h, int shift, uint8_t* out,
                                cudaStream_t st) {
    const int dw = w / 2, dh = h / 2, wp = row_pitch(dw);
    if (dh == 0) return cudaSuccess;
    dim3 grid((wp / 16 + 127) / 128, dh);
    switch (shift) {
        case 2: digit_planes_kernel<1><<<grid, 128, 0, st>>>(D, dw, dh, wp, out); break;
        case 4: digit_planes_kernel<2><<<grid, 128, 0, st>>>(D, dw, dh, wp, out); break;
        case 8: digit_planes_kernel<4><<<grid, 128, 0, st>>>(D, dw, dh, wp, out); break;
        case 16: digit_planes_kernel<8><<<grid, 128, 0, st>>>(D, dw, dh, wp, out); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_phase_planes(const uint8_t* plane, int w, int h, int shift, uint8_t* out,
                                cudaStream_t st) {
    const int wp = row_pitch(w);
    dim3 grid((wp / 16 + 127) / 128, h);
    switch (shift) {
        case 2: phase_planes_kernel<2><<<grid, 128, 0, st>>>(plane, w, h, wp, out); break;
        case 4: phase_planes_kernel<4><<<grid, 128, 0, st>>>(plane, w, h, wp, out); break;
        case 8: phase_planes_kernel<8><<<grid, 128, 0, st>>>(plane, w, h, wp, out); break;
        case 16: phase_planes_kernel<16><<<grid, 128, 0, st>>>(plane, w, h, wp, out); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_build_b(int size, const uint8_t* plane, int w, int h, const uint32_t* rows,
                           const uint32_t* cols, int nranges, uint8_t* out, bool digits,
                           cudaStream_t st) {
    if (digits) {
        switch (size) {
            case 16: return build_b_t<16, true>(plane, w, h, rows, cols, nranges, out, st);
            case 32: return build_b_t<32, true>(plane, w, h, rows, cols, nranges, out, st);
            case 64: return build_b_t<64, true>(plane, w, h, rows, cols, nranges, out, st);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (size) {
        case 4: return build_b_t<4, false>(plane, w, h, rows, cols, nranges, out, st);
        case 8: return build_b_t<8, false>(plane, w, h, rows, cols, nranges, out, st);
        case 16: return build_b_t<16, false>(plane, w, h, rows, cols, nranges, out, st);
        case 32: return build_b_t<32, false>(plane, w, h, rows, cols, nranges, out, st);
        case 64: return build_b_t<64, false>(plane, w, h, rows, cols, nranges, out, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_seed(const int32_t* D, const LevelGeom& g, const uint8_t* plane, int w,
                        const uint32_t* rows, const uint32_t* cols, int nranges, RangeStats rs,
                        DomainStats ds, const FitParams& fp, SeedOut* out, cudaStream_t st) {
    if (nranges == 0) return cudaSuccess;
    const unsigned blocks = (unsigned)nranges;
    switch (g.size) {
        case 4: seed_small_kernel<4><<<(blocks + 7) / 8, 256, 0, st>>>(D, g, plane, w, rows, cols, nranges, rs, ds, fp, out); break;
        case 8: seed_small_kernel<8><<<(blocks + 7) / 8, 256, 0, st>>>(D, g, plane, w, rows, cols, nranges, rs, ds, fp, out); break;
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
int msplit_for(const LevelGeom& g, int nranges, int num_sms, bool digits) {
    constexpr long long kSetupTiles = 4;
    const int tiles_per_row = (g.ncol_d + kM - 1) / kM;
    const int m_tiles = g.nrow_d * tiles_per_row;
    const int rt = ranges_per_tile(digits);
    const int ntiles = (nranges + rt - 1) / rt;
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
                        Partial* partials, unsigned long long* gch, int msplit, bool digits,
                        int* err, unsigned long long* counter, cudaStream_t st) {
#define MARS_CORR(S_, D_) \
    launch_t<S_, D_>(maps, bglob, g, nranges, rs, ds, fp, seeds, partials, gch, msplit, err, \
                     counter, st)
    if (digits) {
        switch (g.size) {
            case 16: return MARS_CORR(16, true);
            case 32: return MARS_CORR(32, true);
            case 64: return MARS_CORR(64, true);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (g.size) {
        case 4: return MARS_CORR(4, false);
        case 8: return MARS_CORR(8, false);
        case 16: return MARS_CORR(16, false);
        case 32: return MARS_CORR(32, false);
        case 64: return MARS_CORR(64, false);
        default: return cudaErrorInvalidValue;
    }
#undef MARS_CORR
}

bool all_levels_supported(int size, bool digits) {
    return digits ? (size == 16 || size == 32 || size == 64) : (size == 4 || size == 8);
}

namespace {
int all_levels_kind(int size, bool digits) {
    if (!digits) return size == 4 ? 0 : 1;
    return size == 16 ? 2 : (size == 32 ? 3 : 4);
}

// Device time of one domain tile of one range tile, by kind (per-level CUDA-event times of a
// 512 x 512 plane on one B200 / tiles: S = 4 fold 1.48 us, S = 8 fold 1.93, S = 16 digits
// 2.09, S = 32 digits 8.0; S = 64 digits four times S = 32, K being four times larger).
double all_levels_tile_us(int size, bool digits) {
    if (!digits) return size == 4 ? 1.48 : 1.93;
    return size == 16 ? 2.09 : (size == 32 ? 8.0 : 32.0);
}
constexpr double kItemSetupTiles = 4.0;  // B load, champions, pipeline fill: ~4 tiles
constexpr int kItemsPerSm = 8;           // work items per SM the splits aim at
// Longest item the splits allow.  On large planes the levels' phase planes exceed L2; short
// split-major items keep the CTAs running together inside one band of domain rows (one
// split), which L2 then holds for all of them.
constexpr double kMaxItemUs = 1500.0;
}  // namespace

void all_levels_splits(const LevelGeom* g, const int* nranges, const bool* digits, int n,
                       int num_sms, int* msplit, int* tail_tiles, int* tail_msplit) {
    double total = 0.0;
    for (int i = 0; i < n; ++i) {
        const int tiles_per_row = (g[i].ncol_d + kM - 1) / kM;
        const double m_tiles = (double)g[i].nrow_d * tiles_per_row;
        const int rt = ranges_per_tile(digits[i]);
        const double ntiles = (double)((nranges[i] + rt - 1) / rt);
        total += ntiles * m_tiles * all_levels_tile_us(g[i].size, digits[i]);
    }
    const double target = std::min(kMaxItemUs, total / ((double)num_sms * kItemsPerSm));
    int last = -1;
    double last_cost = 0.0;
    for (int i = 0; i < n; ++i) {
        const int tiles_per_row = (g[i].ncol_d + kM - 1) / kM;
        const int m_tiles = g[i].nrow_d * tiles_per_row;
        const double tile_us = all_levels_tile_us(g[i].size, digits[i]);
        const int ms = (int)((m_tiles * tile_us + target - 1e-9) / target);
        msplit[i] = std::max(1, std::min(ms, m_tiles));
        tail_tiles[i] = 0;
        tail_msplit[i] = msplit[i];
        const double cost = ((m_tiles + msplit[i] - 1) / msplit[i] + kItemSetupTiles) * tile_us;
        if (last < 0 || cost < last_cost) {
            last = i;
            last_cost = cost;
        }
    }
    if (last < 0) return;
    // The tail: items a quarter as long, about two per SM.
    const int tiles_per_row = (g[last].ncol_d + kM - 1) / kM;
    const int m_tiles = g[last].nrow_d * tiles_per_row;
    const int rt = ranges_per_tile(digits[last]);
    const int ntiles = (nranges[last] + rt - 1) / rt;
    const int fine = std::min(m_tiles, 4 * msplit[last]);
    if (fine > msplit[last] && ntiles >= 2) {
        tail_msplit[last] = fine;
        tail_tiles[last] = std::min(ntiles / 2, (2 * num_sms + fine - 1) / fine);
    }
}

cudaError_t launch_corr_all(const LevelJob* jobs, int njobs, int* work, int* err,
                            unsigned long long* counter, int num_sms, cudaStream_t st) {
    if (njobs <= 0) return cudaSuccess;
    if (njobs > kMaxLevelJobs) return cudaErrorInvalidValue;
    // Largest items first.
    int order[kMaxLevelJobs];
    double cost[kMaxLevelJobs];
    for (int i = 0; i < njobs; ++i) {
        const LevelJob& J = jobs[i];
        if (!all_levels_supported(J.g.size, J.digits != 0) || J.msplit < 1) return cudaErrorInvalidValue;
        const int tiles_per_row = (J.g.ncol_d + kM - 1) / kM;
        const int m_tiles = J.g.nrow_d * tiles_per_row;
        const int m_per = (m_tiles + J.msplit - 1) / J.msplit;
        cost[i] = (m_per + kItemSetupTiles) * all_levels_tile_us(J.g.size, J.digits != 0);
        if (J.merge_seeds) cost[i] = 1e30;  // coarse pre-pass jobs first: others wait on them
        order[i] = i;
    }
    std::sort(order, order + njobs, [&](int x, int y) { return cost[x] > cost[y]; });
    std::unique_ptr<AllLevels> hold(new AllLevels());  // the kernel parameter, ~10 KB
    AllLevels& L = *hold;
    L.njobs = njobs;
    L.item_begin[0] = 0;
    for (int k = 0; k < njobs; ++k) {
        const LevelJob& J = jobs[order[k]];
        const int tiles_per_row = (J.g.ncol_d + kM - 1) / kM;
        const int m_tiles = J.g.nrow_d * tiles_per_row;
        L.maps[k] = J.maps;
        L.args[k] = ItemArgs{J.bglob,  J.g,      J.nranges,
                             J.rs,     J.ds,     J.fp,
                             J.seeds,  m_tiles,  (m_tiles + J.msplit - 1) / J.msplit,
                             J.msplit, J.partials, J.gch,
                             J.tickets, J.out, 1,
                             J.merge_seeds, J.merge_ratio, J.fine_ncol,
                             J.ready, J.wait_ready};
        L.kind[k] = all_levels_kind(J.g.size, J.digits != 0);
        L.tile_begin[k] = J.tile_begin;
        L.tile_count[k] = J.tile_count;
        L.item_begin[k + 1] = L.item_begin[k] + J.tile_count * J.msplit;
    }
    const int nitems = L.item_begin[njobs];
    if (nitems == 0) return cudaSuccess;
    size_t smem = 0;
    for (int k = 0; k < njobs; ++k) {
        constexpr size_t sz[5] = {smem_bytes<4, false>(), smem_bytes<8, false>(),
                                  smem_bytes<16, true>(), smem_bytes<32, true>(),
                                  smem_bytes<64, true>()};
        smem = std::max(smem, sz[L.kind[k]]);
    }
    cudaError_t e = cudaFuncSetAttribute(corr_tc_all_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(work, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    const int grid = std::min(nitems, num_sms);
    corr_tc_all_kernel<<<grid, kThreads, smem, st>>>(L, work, err, counter);
    return cudaGetLastError();
}

bool topk_supported(int size, bool digits) { return all_levels_supported(size, digits); }

cudaError_t launch_corr_topk(const TcMaps& maps, const uint8_t* bglob, const LevelGeom& g,
                             int nranges, RangeStats rs, DomainStats ds, const FitParams& fp,
                             const SeedOut* seeds, int k, Partial* partials,
                             unsigned long long* gch, int msplit, bool digits, int* err,
                             unsigned long long* counter, cudaStream_t st) {
    if (k < 2 || k > kMaxTopK) return cudaErrorInvalidValue;
#define MARS_CORR_TOPK(S_, D_)                                                               \
    launch_t<S_, D_, true>(maps, bglob, g, nranges, rs, ds, fp, seeds, partials, gch, msplit, \
                           err, counter, st, k)
    if (digits) {
        switch (g.size) {
            case 16: return MARS_CORR_TOPK(16, true);
            case 32: return MARS_CORR_TOPK(32, true);
            case 64: return MARS_CORR_TOPK(64, true);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (g.size) {
        case 4: return MARS_CORR_TOPK(4, false);
        case 8: return MARS_CORR_TOPK(8, false);
        default: return cudaErrorInvalidValue;
    }
#undef MARS_CORR_TOPK
}

cudaError_t launch_seed_topk(const int32_t* D, const LevelGeom& g, const uint8_t* plane, int w,
                             const uint32_t* rows, const uint32_t* cols, int nranges,
                             RangeStats rs, DomainStats ds, const FitParams& fp, int k,
                             SeedOut* out, cudaStream_t st) {
    if (nranges == 0) return cudaSuccess;
    if (k < 1 || k > kMaxTopK) return cudaErrorInvalidValue;
#define MARS_SEED_TOPK(S_)                                                                   \
    seed_topk_kernel<S_><<<nranges, 288, 0, st>>>(D, g, plane, w, rows, cols, nranges, rs, ds, \
                                                  fp, k, out)
    switch (g.size) {
        case 4: MARS_SEED_TOPK(4); break;
        case 8: MARS_SEED_TOPK(8); break;
        case 16: MARS_SEED_TOPK(16); break;
        case 32: MARS_SEED_TOPK(32); break;
        case 64: MARS_SEED_TOPK(64); break;
        default: return cudaErrorInvalidValue;
    }
#undef MARS_SEED_TOPK
    return cudaGetLastError();
}

cudaError_t launch_seed_merge(const Partial* partials, int nsplit, int nranges, int coarse_ncol,
                              int fine_ncol, int ratio, SeedOut* seeds, cudaStream_t st) {
    if (nranges == 0) return cudaSuccess;
    seed_merge_kernel<<<(nranges + 127) / 128, 128, 0, st>>>(partials, nsplit, nranges,
                                                             coarse_ncol, fine_ncol, ratio, seeds);
    return cudaGetLastError();
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
