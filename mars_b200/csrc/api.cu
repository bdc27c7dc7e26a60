// The C ABI of include/mars_b200.h: contexts, the per-plane search table (the provider
// factory of crates/mars-codec/src/encode.rs:1054-1076), fixed-grid block search, the
// encode driver and the decode iteration.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/mars_b200.h"
#include "codec.hpp"
#include "context.hpp"
#include "fisher_tc.cuh"
#include "residual.hpp"
#include "kernels.cuh"
#include "tc.cuh"

#include <cudaTypedefs.h>

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define MARS_CUDA(call)                                                                   \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(MARS_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

bool is_pow2(uint32_t x) { return x && !(x & (x - 1)); }

}  // namespace

namespace mars {
// The message mars_last_error() reports, for entry points defined in other files.
int set_last_error(int code, const std::string& msg) { return fail(code, msg); }

int check_fit_params(const mars_params& p) {
    if (p.bits_alfa < 1 || p.bits_alfa > 16 || p.bits_beta < 1 || p.bits_beta > 16)
        return set_last_error(MARS_EINVAL, "bits_alfa/bits_beta must be in 1..16");
    if (!(p.max_alfa > 0.0) || !std::isfinite(p.max_alfa))
        return set_last_error(MARS_EINVAL, "max_alfa must be finite and positive");
    return MARS_OK;
}

FitParams make_fit_params(const mars_params& p) {
    FitParams fp;
    fp.max_alfa = p.max_alfa;
    fp.bits_alfa = p.bits_alfa;
    fp.bits_beta = p.bits_beta;
    const double a = p.max_alfa / (double)(1u << p.bits_alfa);  // exact (power-of-two scale)
    float af = (float)a;
    if ((double)af > a) af = std::nextafter(af, 0.0f);
    fp.a_min = af;
    fp.two_a = 2.0f * af;
    fp.a_half = 0.5f * af;
    fp.eta_per_n = 1e-6 * (1.0 + p.max_alfa) * (1.0 + p.max_alfa);
    return fp;
}

LevelGeom level_geom(uint32_t w, uint32_t h, uint32_t size, uint32_t shift) {
    LevelGeom g;
    g.size = (int)size;
    g.shift = (int)shift;
    g.step_c = (int)(shift / 2);
    g.dw = (int)(w / 2);
    g.dh = (int)(h / 2);
    g.w = (int)w;
    g.h = (int)h;
    g.nrow_d = h >= 2 * size ? (int)((h - 2 * size) / shift + 1) : 0;
    g.ncol_d = w >= 2 * size ? (int)((w - 2 * size) / shift + 1) : 0;
    return g;
}
}  // namespace mars

namespace mars {
// The node index of a search table: (row, col, size, shift) -> position in the node table.
// Every node of one (size, shift) job sits on the size-aligned grid, so a job's nodes are a
// dense grid of ceil(w/size) x ceil(h/size) cells; a job with few nodes in a large grid (the
// border blocks below min_size) keeps a sorted list instead, so memory stays bounded by the
// node count.  A node added twice keeps the last position.
class NodeIndex {
  public:
    void add_job(uint32_t size, uint32_t shift, uint32_t w, uint32_t h, const uint32_t* rows,
                 const uint32_t* cols, size_t n, uint32_t first) {
        Level* L = level(size, shift);
        if (!L) {
            levels_.push_back(Level{size, shift, (w + size - 1) / size, (h + size - 1) / size, {}, {}});
            L = &levels_.back();
            const uint64_t cells = (uint64_t)L->gw * L->gh;
            if ((uint64_t)n * 8 >= cells) L->dense.assign((size_t)cells, UINT32_MAX);
        }
        for (size_t i = 0; i < n; ++i) {
            const uint32_t r = rows[i], c = cols[i], at = first + (uint32_t)i;
            if (!L->dense.empty() && r % size == 0 && c % size == 0 && r / size < L->gh &&
                c / size < L->gw)
                L->dense[(size_t)(r / size) * L->gw + c / size] = at;
            else
                L->sparse.push_back({key(r, c), at});
        }
        // Stable: for a repeated node the later entry stays last and wins below.
        std::stable_sort(L->sparse.begin(), L->sparse.end(),
                         [](const auto& x, const auto& y) { return x.first < y.first; });
    }
    // The node's position, or -1 when the table does not hold it.
    int64_t find(uint32_t row, uint32_t col, uint32_t size, uint32_t shift) const {
        for (const Level& L : levels_) {
            if (L.size != size || L.shift != shift) continue;
            if (!L.dense.empty() && row % size == 0 && col % size == 0 && row / size < L.gh &&
                col / size < L.gw) {
                const uint32_t v = L.dense[(size_t)(row / size) * L.gw + col / size];
                if (v != UINT32_MAX) return v;
            }
            const uint64_t k = key(row, col);
            auto it = std::upper_bound(L.sparse.begin(), L.sparse.end(), k,
                                       [](uint64_t x, const auto& e) { return x < e.first; });
            if (it != L.sparse.begin() && (it - 1)->first == k) return (it - 1)->second;
            return -1;
        }
        return -1;
    }

  private:
    struct Level {
        uint32_t size, shift, gw, gh;
        std::vector<uint32_t> dense;
        std::vector<std::pair<uint64_t, uint32_t>> sparse;
    };
    static uint64_t key(uint32_t r, uint32_t c) { return (uint64_t)r << 32 | c; }
    Level* level(uint32_t size, uint32_t shift) {
        for (Level& L : levels_)
            if (L.size == size && L.shift == shift) return &L;
        return nullptr;
    }
    std::vector<Level> levels_;
};
}  // namespace mars

struct mars_table {
    uint32_t width = 0, height = 0;
    uint32_t k = 1;  // ranked candidates per node (cands holds the first of each)
    mars::NodeIndex index;
    // A search plan's tables share the plan's node index instead of owning one.
    std::shared_ptr<const mars::NodeIndex> shared_index;
    const mars::NodeIndex& nodes() const { return shared_index ? *shared_index : index; }
    std::vector<mars_candidate> cands;
    std::vector<mars_candidate> ranked;  // k per node, when k > 1
    std::vector<uint64_t> evals;
    uint64_t total_evals = 0;
    uint64_t exact_fits = 0;
};

namespace {

static_assert(sizeof(mars_candidate) == sizeof(mars::CandidateOut), "candidate layout");

// Device waits are bounded: poll an event until it completes or the deadline passes.  The
// work waited for is the context's stream's, or `stream`'s when one is given.
int sync_bounded(mars_ctx* ctx, cudaStream_t stream = nullptr) {
    static const double limit_s = [] {
        const char* e = std::getenv("MARS_SYNC_TIMEOUT_S");
        return e ? std::atof(e) : 300.0;
    }();
    // On the context's stream (its callers hold ctx->mu) the kernel error word travels back
    // with the work, ahead of the event; other streams read it after the wait.
    const bool err_async = !stream && ctx->h_err;
    if (err_async)
        MARS_CUDA(cudaMemcpyAsync(ctx->h_err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost,
                                  ctx->stream));
    cudaEvent_t ev;
    MARS_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    MARS_CUDA(cudaEventRecord(ev, stream ? stream : ctx->stream));
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        const cudaError_t q = cudaEventQuery(ev);
        if (q == cudaSuccess) break;
        if (q != cudaErrorNotReady) {
            cudaEventDestroy(ev);
            return fail(MARS_ECUDA, std::string("device error: ") + cudaGetErrorString(q));
        }
        const double el =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > limit_s) {
            cudaEventDestroy(ev);
            return fail(MARS_ETIMEOUT, "device work did not finish within MARS_SYNC_TIMEOUT_S");
        }
        // The first milliseconds poll without sleeping (a short sleep overshoots by tens of
        // microseconds, a search step's whole host overhead), then every 20 us, then 500 us.
        if (el < 0.005)
            std::this_thread::yield();
        else
            std::this_thread::sleep_for(std::chrono::microseconds(el < 0.05 ? 20 : 500));
    }
    cudaEventDestroy(ev);
    int kerr = 0;
    if (err_async)
        kerr = *reinterpret_cast<volatile int*>(ctx->h_err);
    else
        MARS_CUDA(cudaMemcpy(&kerr, ctx->d_err, sizeof kerr, cudaMemcpyDeviceToHost));
    if (kerr) {
        cudaMemset(ctx->d_err, 0, sizeof(int));
        return fail(MARS_ETIMEOUT, "a bounded wait inside the search kernel expired (code " +
                                       std::to_string(kerr) + ")");
    }
    return MARS_OK;
}

int check_params(const mars_params* p) {
    if (!p) return fail(MARS_EINVAL, "params is NULL");
    if (int e = mars::check_fit_params(*p)) return e;
    if (p->shift == 0 || (p->shift & 1))
        return fail(MARS_EUNSUPPORTED, "the domain stride must be even (the reference CLI "
                                       "enforces an even shift in 2..=254)");
    if (!is_pow2(p->min_size) || !is_pow2(p->max_size) || p->min_size > p->max_size)
        return fail(MARS_EINVAL, "min_size/max_size must be powers of two, min <= max");
    if (p->max_size > 64)
        return fail(MARS_EUNSUPPORTED, "block sizes above 64 are not supported on the GPU path");
    if (p->has_lambda && !(std::isfinite(p->lambda) && p->lambda >= 0.0))
        return fail(MARS_EINVAL, "lambda must be finite and nonnegative");
    return MARS_OK;
}

using mars::level_geom;
using mars::make_fit_params;


// Grow-nothing scratch: every buffer is taken from the stream-ordered pool and returned
// to it at the end of the call (the pool keeps the memory cached between calls).
struct Scratch {
    cudaStream_t st;
    std::vector<void*> ptrs;
    explicit Scratch(cudaStream_t s) : st(s) {}
    template <class T>
    cudaError_t get(T** p, size_t count) {
        void* v = nullptr;
        const cudaError_t e = cudaMallocAsync(&v, std::max<size_t>(count, 1) * sizeof(T), st);
        if (e == cudaSuccess) ptrs.push_back(v);
        *p = (T*)v;
        return e;
    }
    ~Scratch() {
        for (void* v : ptrs) cudaFreeAsync(v, st);
    }
};

// Which correlation kernel serves a level: the tcgen05 path wherever it applies (block
// sizes 4..64, domain stride 2, 4, 8 or 16), the CUDA-core path otherwise.
// mars_ctx_set_search_path (or the MARS_SEARCH_PATH environment variable, simt / tc)
// pins the CUDA-core path for A/B checks.
bool use_tc(const mars_ctx* ctx, uint32_t size, uint32_t shift) {
    static const int env = [] {
        const char* e = std::getenv("MARS_SEARCH_PATH");
        if (!e) return 0;
        if (std::string(e) == "simt") return 1;
        if (std::string(e) == "tc") return 2;
        return 0;
    }();
    const int forced = ctx->search_path ? ctx->search_path : env;
    if (forced == 1) return false;
    return mars::tc::supported((int)size, (int)shift);
}

int make_maps(mars_ctx* ctx, const uint8_t* d_phases, uint32_t w, uint32_t h, uint32_t shift,
              mars::tc::TcMaps* maps) {
    if (!ctx->encode_tiled) return fail(MARS_ECUDA, "cuTensorMapEncodeTiled is unavailable");
    std::memset(maps, 0, sizeof(*maps));
    const int P = mars::tc::phase_count((int)shift);
    const uint64_t wp = (uint64_t)mars::tc::row_pitch((int)w);
    for (int p = 0; p < P; ++p) {
        const cuuint64_t dims[2] = {wp, h};
        const cuuint64_t strides[1] = {wp};
        const cuuint32_t box[2] = {128, 8};
        const cuuint32_t estr[2] = {1, 1};
        void* addr = (void*)(d_phases + (size_t)p * h * wp);
        const CUresult r = ctx->encode_tiled(&maps->m[p], CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, addr,
                                             dims, strides, box, estr,
                                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                             CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS)
            return fail(MARS_ECUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    }
    // One box for the whole stage: (bytes, pixel rows, same-phase 128-byte groups, phases).
    const uint32_t per_phase = 16u / (uint32_t)P;
    const cuuint64_t dims4[4] = {wp, h, per_phase, (cuuint64_t)P};
    const cuuint64_t strides4[3] = {wp, 128, (cuuint64_t)h * wp};
    const cuuint32_t box4[4] = {128, 8, per_phase, (cuuint32_t)P};
    const cuuint32_t estr4[4] = {1, 1, 1, 1};
    const CUresult r4 = ctx->encode_tiled(&maps->all, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4,
                                          (void*)d_phases, dims4, strides4, box4, estr4,
                                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    maps->use_all = (r4 == CUDA_SUCCESS && !ctx->tma_16_boxes) ? 1 : 0;
    return MARS_OK;
}

// The two 4-D views of the split-digit path over the digit phase copies (hi digit's P
// phase planes, then lo's), the same box shape as the pixel view.  False when the driver
// rejects them; the level then takes the fold path.
bool make_digit_maps(mars_ctx* ctx, const uint8_t* d_digits, uint32_t w, uint32_t h,
                     uint32_t shift, mars::tc::TcMaps* maps) {
    if (!ctx->encode_tiled) return false;
    std::memset(maps, 0, sizeof(*maps));
    const uint32_t P = (uint32_t)mars::tc::digit_phase_count((int)shift);
    const uint64_t dh = h / 2;
    const uint64_t wp = (uint64_t)mars::tc::row_pitch((int)(w / 2));
    const uint32_t per_phase = 16u / P;
    const cuuint64_t dims4[4] = {wp, dh, per_phase, (cuuint64_t)P};
    const cuuint64_t strides4[3] = {wp, 128, dh * wp};
    const cuuint32_t box4[4] = {128, 8, per_phase, P};
    const cuuint32_t estr4[4] = {1, 1, 1, 1};
    for (int digit = 0; digit < 2; ++digit) {
        void* addr = (void*)(d_digits + (size_t)digit * P * dh * wp);
        const CUresult r = ctx->encode_tiled(digit ? &maps->all_lo : &maps->all,
                                             CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, addr, dims4,
                                             strides4, box4, estr4, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                             CU_TENSOR_MAP_SWIZZLE_NONE,
                                             CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return false;
    }
    maps->use_all = 1;
    return true;
}

// A tensor-core level set up for its correlation: buffers taken from a Scratch, tensor
// maps, split count, and the coarse pre-pass of block size 8.
struct TcLevel {
    mars::LevelGeom g{};
    size_t n = 0;
    bool digits = false;
    int msplit = 1;
    mars::RangeStats rs{};
    mars::DomainStats ds{};
    uint8_t* d_phases = nullptr;
    uint8_t* d_b = nullptr;
    mars::tc::SeedOut* d_seed = nullptr;
    mars::tc::TcMaps maps{};
    mars::Partial* partials = nullptr;
    unsigned long long* gch = nullptr;
    int* tickets = nullptr;  // all-levels launch only
    int32_t* dtmp = nullptr;  // the separable domain statistics' scratch (all-levels launch)
    int* coarse_tickets = nullptr;  // all-levels launch: the in-kernel coarse pre-pass
    int* ready = nullptr;
    int tail_tiles = 0, tail_msplit = 0;  // all-levels launch: the finer-split tail
    bool coarse = false;
    mars::LevelGeom g1{};
    mars::DomainStats ds1{};
    uint8_t* d_ph1 = nullptr;
    mars::tc::TcMaps maps1{};
    int ms1 = 1;
    mars::Partial* part1 = nullptr;
};

// The separable domain statistics take scratch up to this many words (256 MiB); larger
// levels use the direct kernel.
constexpr size_t kDomainTmpWords = 64ull << 20;

// Whether a level takes the split-digit operand (block sizes 16..64 unless pinned off).
bool tc_digits(const mars_ctx* ctx, const mars::LevelGeom& g) {
    return mars::tc::digits_supported(g.size, g.shift) && !ctx->tma_16_boxes && !ctx->fold_only;
}

// Coarse pre-pass at block size 8: the same search over every 4th domain position of each
// axis, whose champions seed the full sweep (tighter thresholds from the first tile: exact
// fits of the 512x512 level 1.09 M -> 0.23 M, 0.98 -> 0.86 ms).  At size 4 its cost
// outweighs the survivors it saves, and at 16..64 it is neutral or slower.
constexpr int kCoarseRatio = 4;
constexpr size_t kCoarseAllLevels = 65536;

// Buffers and tensor maps of a level (g, rs and ds already set).  msplit 0 picks the
// per-level launch's split count; tickets adds the all-levels launch's per-tile counters;
// coarse_ok allows the coarse pre-pass.  The all-levels launch keeps it for large levels
// only (kCoarseAllLevels ranges and up): the pre-pass sits on the path before the one
// launch, where at 512 x 512 it costs 0.16 ms, more than the 0.12 ms of correlation it
// saves; on large planes it is a small part of the step and cuts the level's exact fits.
// A level whose digit views the driver rejects takes the fold path (L.digits false).
int tc_level_setup(mars_ctx* ctx, Scratch& sc, uint32_t w, uint32_t h, size_t n, int msplit,
                   bool tickets, bool coarse_ok, TcLevel& L) {
    const mars::LevelGeom& g = L.g;
    L.n = n;
    L.digits = tc_digits(ctx, g);
    if (L.digits) {
        MARS_CUDA(sc.get(&L.d_phases, mars::tc::digit_plane_bytes((int)w, (int)h, g.shift)));
        L.digits = make_digit_maps(ctx, L.d_phases, w, h, (uint32_t)g.shift, &L.maps);
    }
    if (!L.digits) {
        MARS_CUDA(sc.get(&L.d_phases, mars::tc::phase_bytes((int)w, (int)h, g.shift)));
        if (int e = make_maps(ctx, L.d_phases, w, h, (uint32_t)g.shift, &L.maps)) return e;
    }
    MARS_CUDA(sc.get(&L.d_b, mars::tc::b_bytes(g.size, (int)n, L.digits)));
    MARS_CUDA(sc.get(&L.d_seed, n));
    L.msplit = msplit > 0 ? msplit : mars::tc::msplit_for(g, (int)n, ctx->num_sms, L.digits);
    MARS_CUDA(sc.get(&L.partials, (size_t)L.msplit * n));
    // The M-splits' shared champion records (rms bits, index, t1_x4).
    MARS_CUDA(sc.get(&L.gch, 2 * n));
    if (tickets) {
        const int rt = mars::tc::ranges_per_tile(L.digits);
        MARS_CUDA(sc.get(&L.tickets, (n + rt - 1) / rt));
    }
    L.coarse = false;
    if (coarse_ok && !L.digits && g.size == 8 && g.shift * kCoarseRatio <= 16 && n >= 256) {
        L.g1 = level_geom(w, h, (uint32_t)g.size, (uint32_t)(g.shift * kCoarseRatio));
        if (L.g1.nrow_d > 0 && L.g1.ncol_d > 0) {
            L.coarse = true;
            const size_t ndom1 = (size_t)L.g1.nrow_d * L.g1.ncol_d;
            MARS_CUDA(sc.get(&L.ds1.s1x4, ndom1));
            MARS_CUDA(sc.get(&L.ds1.s2x16, ndom1));
            MARS_CUDA(sc.get(&L.ds1.detf, ndom1));
            MARS_CUDA(sc.get(&L.ds1.sdetf, ndom1));
            MARS_CUDA(sc.get(&L.d_ph1, mars::tc::phase_bytes((int)w, (int)h, L.g1.shift)));
            if (int e = make_maps(ctx, L.d_ph1, w, h, (uint32_t)L.g1.shift, &L.maps1)) return e;
            L.ms1 = mars::tc::msplit_for(L.g1, (int)n, ctx->num_sms, false);
            MARS_CUDA(sc.get(&L.part1, (size_t)L.ms1 * n));
        }
    }
    return MARS_OK;
}

// Everything of a level before its correlation, on stream st: phase (or digit phase)
// copies, the B operand, seed champions, the coarse pre-pass (its statistics and planes
// only when the all-levels launch runs it: L.ready set), the shared champion records and
// tickets.
// st_planes (all-levels launch only): a second stream for the phase planes and the B
// operand, which do not depend on the statistics the seeds need.
int tc_level_prep(mars_ctx* ctx, const TcLevel& L, const uint8_t* d_plane, const int32_t* d_D,
                  const uint8_t* d_dplane, uint32_t w, uint32_t h, const mars::FitParams& fp,
                  const uint32_t* d_rows, const uint32_t* d_cols, cudaStream_t st,
                  cudaStream_t st_planes = nullptr) {
    const mars::LevelGeom& g = L.g;
    const int n = (int)L.n;
    const cudaStream_t sp = st_planes ? st_planes : st;
    if (L.digits)
        MARS_CUDA(mars::tc::launch_digit_planes(d_D, (int)w, (int)h, g.shift, L.d_phases, sp));
    else
        MARS_CUDA(mars::tc::launch_phase_planes(d_dplane, (int)w, (int)h, g.shift, L.d_phases, sp));
    MARS_CUDA(mars::tc::launch_build_b(g.size, d_plane, (int)w, (int)h, d_rows, d_cols, n, L.d_b,
                                       L.digits, sp));
    MARS_CUDA(mars::tc::launch_seed(d_D, g, d_plane, (int)w, d_rows, d_cols, n, L.rs, L.ds, fp,
                                    L.d_seed, st));
    ctx->launches += 3;
    if (L.coarse) {
        MARS_CUDA(mars::launch_domain_stats(d_D, L.g1, L.ds1, st));
        MARS_CUDA(mars::tc::launch_phase_planes(d_dplane, (int)w, (int)h, L.g1.shift, L.d_ph1, sp));
        ctx->launches += 2;
        if (L.ready) {
            const int rt = mars::tc::ranges_per_tile(false);
            const size_t nt = (L.n + rt - 1) / rt;
            MARS_CUDA(cudaMemsetAsync(L.ready, 0, nt * sizeof(int), st));
            MARS_CUDA(cudaMemsetAsync(L.coarse_tickets, 0, nt * sizeof(int), st));
        } else {
            MARS_CUDA(mars::tc::launch_corr(L.maps1, L.d_b, L.g1, n, L.rs, L.ds1, fp, L.d_seed,
                                            L.part1, nullptr, L.ms1, false, ctx->d_err,
                                            ctx->d_counter, st));
            MARS_CUDA(mars::tc::launch_seed_merge(L.part1, L.ms1, n, L.g1.ncol_d, g.ncol_d,
                                                  kCoarseRatio, L.d_seed, st));
            ctx->launches += 2;
        }
    }
    MARS_CUDA(cudaMemsetAsync(L.gch, 0xFF, 2 * L.n * sizeof(unsigned long long), st));
    if (L.tickets) {
        const int rt = mars::tc::ranges_per_tile(L.digits);
        MARS_CUDA(cudaMemsetAsync(L.tickets, 0, (L.n + rt - 1) / rt * sizeof(int), st));
    }
    return MARS_OK;
}

// The tcgen05 path for one level: set-up, the correlation + exact-bound kernel, and the
// final champion per block.
int run_level_tc(mars_ctx* ctx, Scratch& sc, const uint8_t* d_plane, const int32_t* d_D,
                 uint32_t w, uint32_t h, const mars::LevelGeom& g, const mars::FitParams& fp,
                 const uint32_t* d_rows, const uint32_t* d_cols, size_t n, mars::RangeStats rs,
                 mars::DomainStats ds, mars::CandidateOut* d_out, const uint8_t* d_dplane) {
    const cudaStream_t st = ctx->stream;
    TcLevel L;
    L.g = g;
    L.rs = rs;
    L.ds = ds;
    if (int e = tc_level_setup(ctx, sc, w, h, n, 0, false, true, L)) return e;
    if (int e = tc_level_prep(ctx, L, d_plane, d_D, d_dplane, w, h, fp, d_rows, d_cols, st))
        return e;
    MARS_CUDA(mars::tc::launch_corr(L.maps, L.d_b, g, (int)n, rs, ds, fp, L.d_seed, L.partials,
                                    L.gch, L.msplit, L.digits, ctx->d_err, ctx->d_counter, st));
    MARS_CUDA(mars::tc::launch_finish(L.partials, L.msplit, (int)n, g, rs, ds, fp, d_out, st));
    ctx->launches += 2;
    return MARS_OK;
}

// The ranked search (k = 2..kMaxTopK) of one level on the tcgen05 path: phase (or digit)
// planes, the B operand, k seeds per range, the correlation keeping each range's best k,
// and the merge of the splits' lists (reduce_topk).
int run_level_tc_topk(mars_ctx* ctx, Scratch& sc, const uint8_t* d_plane, const int32_t* d_D,
                      uint32_t w, uint32_t h, const mars::LevelGeom& g, const mars::FitParams& fp,
                      const uint32_t* d_rows, const uint32_t* d_cols, size_t n,
                      mars::RangeStats rs, mars::DomainStats ds, mars::CandidateOut* d_out,
                      uint32_t k, const uint8_t* d_dplane) {
    const cudaStream_t st = ctx->stream;
    uint8_t* d_phases = nullptr;
    mars::tc::TcMaps maps{};
    bool digits = tc_digits(ctx, g);
    if (digits) {
        MARS_CUDA(sc.get(&d_phases, mars::tc::digit_plane_bytes((int)w, (int)h, g.shift)));
        digits = make_digit_maps(ctx, d_phases, w, h, (uint32_t)g.shift, &maps);
    }
    if (!digits) {
        MARS_CUDA(sc.get(&d_phases, mars::tc::phase_bytes((int)w, (int)h, g.shift)));
        if (int e = make_maps(ctx, d_phases, w, h, (uint32_t)g.shift, &maps)) return e;
    }
    if (!mars::tc::topk_supported(g.size, digits))
        return fail(MARS_EUNSUPPORTED, "no ranked tensor-core kernel for this level");
    uint8_t* d_b = nullptr;
    mars::tc::SeedOut* d_seed = nullptr;
    mars::Partial* partials = nullptr;
    const int msplit = std::min(mars::tc::msplit_for(g, (int)n, ctx->num_sms, digits),
                                mars::kMaxTopKSplits);
    MARS_CUDA(sc.get(&d_b, mars::tc::b_bytes(g.size, (int)n, digits)));
    MARS_CUDA(sc.get(&d_seed, n * k));
    MARS_CUDA(sc.get(&partials, (size_t)msplit * n * k));
    if (digits)
        MARS_CUDA(mars::tc::launch_digit_planes(d_D, (int)w, (int)h, g.shift, d_phases, st));
    else
        MARS_CUDA(mars::tc::launch_phase_planes(d_dplane, (int)w, (int)h, g.shift, d_phases, st));
    MARS_CUDA(mars::tc::launch_build_b(g.size, d_plane, (int)w, (int)h, d_rows, d_cols, (int)n,
                                       d_b, digits, st));
    MARS_CUDA(mars::tc::launch_seed_topk(d_D, g, d_plane, (int)w, d_rows, d_cols, (int)n, rs, ds,
                                         fp, (int)k, d_seed, st));
    // The splits share each range's best k-th entry (rms bits, index, t1_x4) as a bound.
    unsigned long long* gch = nullptr;
    MARS_CUDA(sc.get(&gch, 2 * n));
    MARS_CUDA(cudaMemsetAsync(gch, 0xFF, 2 * n * sizeof(unsigned long long), st));
    MARS_CUDA(mars::tc::launch_corr_topk(maps, d_b, g, (int)n, rs, ds, fp, d_seed, (int)k,
                                         partials, gch, msplit, digits, ctx->d_err,
                                         ctx->d_counter, st));
    MARS_CUDA(mars::launch_reduce_topk(partials, msplit, (int)n, (int)k, g, rs, ds, d_out, st));
    ctx->launches += 5;
    return MARS_OK;
}

// Search every block of one (size, shift) level.  rows/cols/out are device pointers.
// k > 1: the ranked search (n x k results); k == 1: the single winner.
// One level of the search: ranges are read from d_plane; domains from d_D (the contracted
// domain plane) and, on the tensor-core path, from the pixel plane d_dplane (d_plane when
// null).  The two planes differ only for the attractor re-search of mars_refine_domains.
int run_level(mars_ctx* ctx, Scratch& sc, const uint8_t* d_plane, const int32_t* d_D,
              uint32_t w, uint32_t h, uint32_t size, uint32_t shift, const mars::FitParams& fp,
              const uint32_t* d_rows, const uint32_t* d_cols, size_t n,
              mars::CandidateOut* d_out, uint32_t k = 1, const uint8_t* d_dplane = nullptr) {
    if (n == 0) return MARS_OK;
    const cudaStream_t st = ctx->stream;
    const mars::LevelGeom g = level_geom(w, h, size, shift);
    if (g.nrow_d <= 0 || g.ncol_d <= 0) {
        // No legal domain: every candidate is None (encode.rs:734-739).
        MARS_CUDA(cudaMemsetAsync(d_out, 0, n * k * sizeof(mars::CandidateOut), st));
        return MARS_OK;
    }
    const size_t ndom = (size_t)g.nrow_d * g.ncol_d;
    mars::RangeStats rs;
    mars::DomainStats ds;
    MARS_CUDA(sc.get(&rs.t0, n));
    MARS_CUDA(sc.get(&rs.t2, n));
    MARS_CUDA(sc.get(&rs.nrr, n));
    MARS_CUDA(sc.get(&rs.sum0, n));
    MARS_CUDA(sc.get(&rs.rms0, n));
    MARS_CUDA(sc.get(&ds.s1x4, ndom));
    MARS_CUDA(sc.get(&ds.s2x16, ndom));
    MARS_CUDA(sc.get(&ds.detf, ndom));
    MARS_CUDA(sc.get(&ds.sdetf, ndom));
    MARS_CUDA(mars::launch_range_stats(d_plane, (int)w, (int)h, d_rows, d_cols, (int)n,
                                       (int)size, fp, rs, st));
    int32_t* dtmp = nullptr;
    const size_t dwords = mars::domain_stats_tmp_words(g);
    if (dwords > 0 && dwords <= kDomainTmpWords) MARS_CUDA(sc.get(&dtmp, dwords));
    MARS_CUDA(mars::launch_domain_stats(d_D, g, ds, st, dtmp));
    ctx->launches += 2;
    if (k > 1 && use_tc(ctx, size, shift) && mars::tc::topk_supported(g.size, tc_digits(ctx, g)))
        return run_level_tc_topk(ctx, sc, d_plane, d_D, w, h, g, fp, d_rows, d_cols, n, rs, ds,
                                 d_out, k, d_dplane ? d_dplane : d_plane);
    if (k > 1) {
        const int nsplit = mars::search_topk_splits(g, (int)n, ctx->num_sms);
        mars::Partial* partials;
        MARS_CUDA(sc.get(&partials, (size_t)nsplit * n * k));
        MARS_CUDA(mars::launch_search_topk(d_D, d_plane, (int)w, d_rows, d_cols, (int)n, g, rs,
                                           ds, fp, (int)k, partials, nsplit, ctx->d_counter, st));
        MARS_CUDA(mars::launch_reduce_topk(partials, nsplit, (int)n, (int)k, g, rs, ds, d_out, st));
        ctx->launches += 2;
        return MARS_OK;
    }
    if (use_tc(ctx, size, shift))
        return run_level_tc(ctx, sc, d_plane, d_D, w, h, g, fp, d_rows, d_cols, n, rs, ds, d_out,
                            d_dplane ? d_dplane : d_plane);
    const int nsplit = mars::search_simt_splits(g, (int)n, ctx->num_sms);
    mars::Partial* partials;
    MARS_CUDA(sc.get(&partials, (size_t)nsplit * n));
    MARS_CUDA(mars::launch_search_simt(d_D, d_plane, (int)w, d_rows, d_cols, (int)n, g, rs, ds,
                                       fp, partials, nsplit, ctx->d_counter, st));
    MARS_CUDA(mars::launch_reduce(partials, nsplit, (int)n, g, rs, ds, d_out, st));
    ctx->launches += 2;
    return MARS_OK;
}

// Quadtree nodes an encode can request a search for (walk / walk_rd, encode.rs:1330-1468,
// 1865-2071): every non-forced node of size >= 2, and the children of non-forced nodes
// above min_size; forced nodes split unconditionally.
void enumerate_nodes(uint32_t w, uint32_t h, uint32_t min_size, uint32_t max_size,
                     uint32_t row, uint32_t col, uint32_t size,
                     std::vector<std::vector<std::pair<uint32_t, uint32_t>>>& by_log2) {
    if (row >= h || col >= w || size == 0) return;
    const bool forced = size > max_size || row + size > h || col + size > w;
    const uint32_t half = size / 2;
    if (!forced) {
        if (size >= 2) by_log2[__builtin_ctz(size)].push_back({row, col});
        if (size <= min_size) return;
    }
    if (half == 0) return;
    enumerate_nodes(w, h, min_size, max_size, row, col, half, by_log2);
    enumerate_nodes(w, h, min_size, max_size, row + half, col, half, by_log2);
    enumerate_nodes(w, h, min_size, max_size, row, col + half, half, by_log2);
    enumerate_nodes(w, h, min_size, max_size, row + half, col + half, half, by_log2);
}

struct Job {
    uint32_t size, shift;
    std::vector<uint32_t> rows, cols;
};

std::vector<Job> plan_jobs(const uint8_t* plane, uint32_t w, uint32_t h, const mars_params& p,
                           bool adaptive) {
    mars_header hdr = mars::codec::build_header(w, h, p);
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> by_log2(32);
    enumerate_nodes(w, h, p.min_size, p.max_size, 0, 0, mars::codec::virtual_size(hdr), by_log2);
    std::vector<Job> jobs;
    for (uint32_t lg = 1; lg < 32; ++lg) {
        if (by_log2[lg].empty()) continue;
        Job base{1u << lg, p.shift, {}, {}};
        Job dense{1u << lg, std::min<uint32_t>(p.shift * 2, 0xffffu), {}, {}};
        for (const auto& rc : by_log2[lg]) {
            base.rows.push_back(rc.first);
            base.cols.push_back(rc.second);
            if (adaptive) {
                const mars::codec::Image im{plane, w, h};
                const double rms = mars::codec::block_rms(im, rc.first, rc.second, 1u << lg);
                if (mars::codec::adaptive_shift(p.shift, rms) != p.shift) {
                    dense.rows.push_back(rc.first);
                    dense.cols.push_back(rc.second);
                }
            }
        }
        jobs.push_back(std::move(base));
        if (!dense.rows.empty()) jobs.push_back(std::move(dense));
    }
    return jobs;
}

uint64_t level_evals(uint32_t w, uint32_t h, uint32_t size, uint32_t shift) {
    const mars::LevelGeom g = level_geom(w, h, size, shift);
    if (g.nrow_d <= 0 || g.ncol_d <= 0) return 0;
    return (uint64_t)g.nrow_d * (uint64_t)g.ncol_d * 8ull;
}

// Runs all jobs on the device plane; results land in d_out (concatenated in job order).
// The jobs' node origins as one list: all rows, then all columns, in job order.
std::vector<uint32_t> job_origins(const std::vector<Job>& jobs, size_t* total_out) {
    size_t total = 0;
    for (const Job& j : jobs) total += j.rows.size();
    std::vector<uint32_t> rc(2 * total);
    size_t off = 0;
    for (const Job& j : jobs) {
        std::copy(j.rows.begin(), j.rows.end(), rc.begin() + (long)off);
        std::copy(j.cols.begin(), j.cols.end(), rc.begin() + (long)(total + off));
        off += j.rows.size();
    }
    *total_out = total;
    return rc;
}

// `d_rc_in`: the job origins already on the device (job_origins layout), else uploaded here.
int run_jobs(mars_ctx* ctx, Scratch& sc, const uint8_t* d_plane, uint32_t w, uint32_t h,
             const mars::FitParams& fp, const std::vector<Job>& jobs, mars::CandidateOut* d_out,
             uint32_t k = 1, const uint32_t* d_rc_in = nullptr) {
    const cudaStream_t st = ctx->stream;
    int32_t* d_D = nullptr;
    MARS_CUDA(sc.get(&d_D, std::max<size_t>(1, (size_t)(w / 2) * (h / 2))));
    MARS_CUDA(mars::launch_contract(d_plane, (int)w, (int)h, d_D, st));
    ctx->launches += 1;
    size_t total = 0;
    const uint32_t* d_rc = d_rc_in;
    if (!d_rc) {
        const std::vector<uint32_t> rc = job_origins(jobs, &total);
        uint32_t* d = nullptr;
        MARS_CUDA(sc.get(&d, rc.size()));
        // A pageable source: the call returns once the bytes are staged, so `rc` may go.
        MARS_CUDA(cudaMemcpyAsync(d, rc.data(), rc.size() * 4, cudaMemcpyHostToDevice, st));
        d_rc = d;
    } else {
        for (const Job& j : jobs) total += j.rows.size();
    }
    size_t off = 0;
    for (const Job& j : jobs) {
        const int e = run_level(ctx, sc, d_plane, d_D, w, h, j.size, j.shift, fp, d_rc + off,
                                d_rc + total + off, j.rows.size(), d_out + off * k, k);
        if (e) return e;
        off += j.rows.size();
    }
    return MARS_OK;
}

// Whether the exhaustive single-candidate search of `jobs` runs its tensor-core levels as
// one all-levels persistent launch: not pinned off (mars_ctx_set_search_path 5 or the
// MARS_LEVEL_LAUNCH=per_level environment variable), every tensor-core level a kind the
// kernel holds, at most kMaxLevelJobs of them.
bool all_levels_eligible(const mars_ctx* ctx, uint32_t w, uint32_t h, const std::vector<Job>& jobs) {
    static const bool env_per_level = [] {
        const char* e = std::getenv("MARS_LEVEL_LAUNCH");
        return e && std::string(e) == "per_level";
    }();
    if (ctx->per_level || env_per_level) return false;
    int levels = 0;
    for (const Job& j : jobs) {
        if (j.rows.empty() || !use_tc(ctx, j.size, j.shift)) continue;
        const mars::LevelGeom g = level_geom(w, h, j.size, j.shift);
        if (g.nrow_d <= 0 || g.ncol_d <= 0) continue;
        if (!mars::tc::all_levels_supported(g.size, tc_digits(ctx, g))) return false;
        ++levels;
    }
    // A level may add a tail job, and the block-size-8 level a coarse pre-pass job.
    return levels > 0 && levels + 2 <= mars::tc::kMaxLevelJobs;
}

// run_jobs for the exhaustive single-candidate search with the correlation of every
// tensor-core level in one persistent launch (launch_corr_all, which also writes the
// levels' final candidates).  Every buffer is taken on the context's stream before the
// fork; each level's statistics, operands and seeds (and every other level, whole) then
// run on one of the branch streams; the persistent launch follows the join.  The caller
// holds ctx->mu and has checked all_levels_eligible.
int run_jobs_all_levels(mars_ctx* ctx, Scratch& sc, const uint8_t* d_plane, uint32_t w,
                        uint32_t h, const mars::FitParams& fp, const std::vector<Job>& jobs,
                        mars::CandidateOut* d_out, const uint32_t* d_rc_in,
                        cudaEvent_t* timing = nullptr) {
    const cudaStream_t main = ctx->stream;
    if (!ctx->fork_ev) {
        MARS_CUDA(cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming));
        for (int b = 0; b < mars_ctx::kBranches; ++b) {
            MARS_CUDA(cudaStreamCreateWithFlags(&ctx->branch[b], cudaStreamNonBlocking));
            MARS_CUDA(cudaEventCreateWithFlags(&ctx->join_ev[b], cudaEventDisableTiming));
        }
    }
    int32_t* d_D = nullptr;
    MARS_CUDA(sc.get(&d_D, std::max<size_t>(1, (size_t)(w / 2) * (h / 2))));
    MARS_CUDA(mars::launch_contract(d_plane, (int)w, (int)h, d_D, main));
    ctx->launches += 1;
    size_t total = 0;
    const uint32_t* d_rc = d_rc_in;
    if (!d_rc) {
        const std::vector<uint32_t> rc = job_origins(jobs, &total);
        uint32_t* d = nullptr;
        MARS_CUDA(sc.get(&d, rc.size()));
        MARS_CUDA(cudaMemcpyAsync(d, rc.data(), rc.size() * 4, cudaMemcpyHostToDevice, main));
        d_rc = d;
    } else {
        for (const Job& j : jobs) total += j.rows.size();
    }
    // Which jobs are all-levels levels, and their split counts (chosen together).
    std::vector<int> level_of(jobs.size(), -1);
    std::vector<TcLevel> lv;
    std::vector<size_t> lv_off;
    {
        size_t off = 0;
        for (size_t i = 0; i < jobs.size(); ++i) {
            const Job& j = jobs[i];
            const mars::LevelGeom g = level_geom(w, h, j.size, j.shift);
            if (!j.rows.empty() && use_tc(ctx, j.size, j.shift) && g.nrow_d > 0 && g.ncol_d > 0) {
                level_of[i] = (int)lv.size();
                TcLevel L;
                L.g = g;
                L.n = j.rows.size();
                L.digits = tc_digits(ctx, g);
                lv.push_back(L);
                lv_off.push_back(off);
            }
            off += j.rows.size();
        }
    }
    const int nl = (int)lv.size();
    std::vector<mars::LevelGeom> gs(nl);
    std::vector<int> ns(nl), ms(nl), tail_t(nl), tail_ms(nl);
    std::unique_ptr<bool[]> dg(new bool[std::max(1, nl)]);
    for (int l = 0; l < nl; ++l) {
        gs[l] = lv[l].g;
        ns[l] = (int)lv[l].n;
        dg[l] = lv[l].digits;
    }
    mars::tc::all_levels_splits(gs.data(), ns.data(), dg.get(), nl, ctx->num_sms, ms.data(),
                                tail_t.data(), tail_ms.data());
    for (int l = 0; l < nl; ++l) {
        TcLevel& L = lv[l];
        const size_t n = L.n;
        const size_t ndom = (size_t)L.g.nrow_d * L.g.ncol_d;
        MARS_CUDA(sc.get(&L.rs.t0, n));
        MARS_CUDA(sc.get(&L.rs.t2, n));
        MARS_CUDA(sc.get(&L.rs.nrr, n));
        MARS_CUDA(sc.get(&L.rs.sum0, n));
        MARS_CUDA(sc.get(&L.rs.rms0, n));
        MARS_CUDA(sc.get(&L.ds.s1x4, ndom));
        MARS_CUDA(sc.get(&L.ds.s2x16, ndom));
        MARS_CUDA(sc.get(&L.ds.detf, ndom));
        MARS_CUDA(sc.get(&L.ds.sdetf, ndom));
        const size_t dwords = mars::domain_stats_tmp_words(L.g);
        if (dwords > 0 && dwords <= kDomainTmpWords) MARS_CUDA(sc.get(&L.dtmp, dwords));
        const bool wanted = L.digits;
        if (int e = tc_level_setup(ctx, sc, w, h, n, std::max(ms[l], tail_ms[l]), true,
                                   n >= kCoarseAllLevels, L))
            return e;
        if (L.digits != wanted)  // the driver rejected the digit views: no fold kernel here
            return fail(MARS_ECUDA, "the split-digit tensor maps were rejected");
        L.msplit = ms[l];
        L.tail_tiles = tail_t[l];
        L.tail_msplit = tail_ms[l];
        if (L.coarse) {
            // The coarse pre-pass runs inside the launch, ahead of this level's items.
            const int rt = mars::tc::ranges_per_tile(false);
            MARS_CUDA(sc.get(&L.ready, (n + rt - 1) / rt));
            MARS_CUDA(sc.get(&L.coarse_tickets, (n + rt - 1) / rt));
        }
    }
    int* d_work = nullptr;
    MARS_CUDA(sc.get(&d_work, 1));
    // Every branch is forked: a level's statistics and seeds run on branch b, its planes and
    // B operand on branch b + kBranches / 2.
    MARS_CUDA(cudaEventRecord(ctx->fork_ev, main));
    const int nb = mars_ctx::kBranches;
    constexpr int kHalf = mars_ctx::kBranches / 2;
    for (int b = 0; b < nb; ++b) MARS_CUDA(cudaStreamWaitEvent(ctx->branch[b], ctx->fork_ev, 0));
    int err = MARS_OK;
    size_t off = 0;
    for (size_t i = 0; i < jobs.size() && !err; ++i) {
        const Job& j = jobs[i];
        const int b = (int)(i % kHalf);
        const cudaStream_t bs = ctx->branch[b];
        const uint32_t* rows = d_rc + off;
        const uint32_t* cols = d_rc + total + off;
        const int l = level_of[i];
        if (l >= 0) {
            TcLevel& L = lv[l];
            const mars::LevelGeom& g = L.g;
            if (cudaError_t ce = mars::launch_range_stats(d_plane, (int)w, (int)h, rows, cols,
                                                          (int)L.n, g.size, fp, L.rs, bs)) {
                err = fail(MARS_ECUDA, cudaGetErrorString(ce));
            } else if (cudaError_t ce2 = mars::launch_domain_stats(d_D, g, L.ds, bs, L.dtmp)) {
                err = fail(MARS_ECUDA, cudaGetErrorString(ce2));
            } else {
                ctx->launches += 2;
                err = tc_level_prep(ctx, L, d_plane, d_D, d_plane, w, h, fp, rows, cols, bs,
                                    ctx->branch[b + kHalf]);
            }
        } else {
            ctx->stream = bs;
            {
                Scratch sb(bs);
                err = run_level(ctx, sb, d_plane, d_D, w, h, j.size, j.shift, fp, rows, cols,
                                j.rows.size(), d_out + off, 1);
            }
            ctx->stream = main;
        }
        off += j.rows.size();
    }
    // Join every branch that was forked, also after an error (a capture must end joined).
    for (int b = 0; b < nb; ++b) {
        MARS_CUDA(cudaEventRecord(ctx->join_ev[b], ctx->branch[b]));
        MARS_CUDA(cudaStreamWaitEvent(main, ctx->join_ev[b], 0));
    }
    if (err) return err;
    std::vector<mars::tc::LevelJob> lj;
    for (int l = 0; l < nl; ++l) {
        const TcLevel& L = lv[l];
        mars::tc::LevelJob J;
        J.maps = L.maps;
        J.bglob = L.d_b;
        J.g = L.g;
        J.nranges = (int)L.n;
        J.rs = L.rs;
        J.ds = L.ds;
        J.fp = fp;
        J.seeds = L.d_seed;
        J.partials = L.partials;
        J.gch = L.gch;
        J.tickets = L.tickets;
        J.out = d_out + lv_off[l];
        const int rt = mars::tc::ranges_per_tile(L.digits);
        const int ntiles = (int)((L.n + rt - 1) / rt);
        J.digits = L.digits ? 1 : 0;
        J.tile_begin = 0;
        J.tile_count = ntiles - L.tail_tiles;
        J.msplit = L.msplit;
        if (L.coarse) {
            // The pre-pass job: the same B operand and ranges, the coarse grid's planes and
            // statistics; its last split of each tile merges the tile's seeds.
            mars::tc::LevelJob C = J;
            C.maps = L.maps1;
            C.g = L.g1;
            C.ds = L.ds1;
            C.partials = L.part1;
            C.gch = nullptr;
            C.tickets = L.coarse_tickets;
            C.out = nullptr;
            C.tile_begin = 0;
            C.tile_count = ntiles;
            C.msplit = L.ms1;
            C.merge_seeds = L.d_seed;
            C.merge_ratio = kCoarseRatio;
            C.fine_ncol = L.g.ncol_d;
            C.ready = L.ready;
            lj.push_back(C);
            J.wait_ready = L.ready;
        }
        lj.push_back(J);
        if (L.tail_tiles > 0) {
            J.tile_begin = ntiles - L.tail_tiles;
            J.tile_count = L.tail_tiles;
            J.msplit = L.tail_msplit;
            lj.push_back(J);
        }
    }
    // Optional timing events around the launch: event-record nodes inside a capture (the
    // external flag is for captures only), plain records otherwise.
    unsigned rec_flags = cudaEventRecordDefault;
    if (timing) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        MARS_CUDA(cudaStreamIsCapturing(main, &cs));
        if (cs == cudaStreamCaptureStatusActive) rec_flags = cudaEventRecordExternal;
        MARS_CUDA(cudaEventRecordWithFlags(timing[0], main, rec_flags));
    }
    MARS_CUDA(mars::tc::launch_corr_all(lj.data(), (int)lj.size(), d_work, ctx->d_err,
                                        ctx->d_counter, ctx->num_sms, main));
    if (timing) MARS_CUDA(cudaEventRecordWithFlags(timing[1], main, rec_flags));
    ctx->launches += 1;
    return MARS_OK;
}

// Whether the classified search of a level runs as the tensor-core bucketed batch
// (fisher_tc.cu): block sizes 4, 8, 16 at an even stride, unless the CUDA-core path is
// pinned (mars_ctx_set_search_path 1 or MARS_SEARCH_PATH=simt).
bool use_fisher_tc(const mars_ctx* ctx, uint32_t size, uint32_t shift) {
    if (!use_tc(ctx, 4, 2)) return false;  // the CUDA-core path is pinned
    return mars::ftc::supported((int)size, (int)shift);
}

// One level of the classified search on tensor cores: statistics, each range's bucket,
// the ranges grouped by bucket, then the batch (fisher_tc.cu).
int run_fisher_tc(mars_ctx* ctx, Scratch& sc, const uint8_t* d_plane, const int32_t* d_D,
                  uint32_t w, uint32_t h, const mars::LevelGeom& g, const mars::FitParams& fp,
                  const uint32_t* d_rows, const uint32_t* d_cols, int n,
                  const mars::FisherIndex& ix, mars::CandidateOut* d_out, uint64_t* d_evals) {
    const cudaStream_t st = ctx->stream;
    const size_t npos = (size_t)g.nrow_d * g.ncol_d;
    mars::RangeStats rs;
    mars::DomainStats ds;
    MARS_CUDA(sc.get(&rs.t0, n));
    MARS_CUDA(sc.get(&rs.t2, n));
    MARS_CUDA(sc.get(&rs.nrr, n));
    MARS_CUDA(sc.get(&rs.sum0, n));
    MARS_CUDA(sc.get(&rs.rms0, n));
    MARS_CUDA(sc.get(&ds.s1x4, npos));
    MARS_CUDA(sc.get(&ds.s2x16, npos));
    MARS_CUDA(sc.get(&ds.detf, npos));
    MARS_CUDA(sc.get(&ds.sdetf, npos));
    MARS_CUDA(mars::launch_range_stats(d_plane, (int)w, (int)h, d_rows, d_cols, n, g.size, fp, rs,
                                       st));
    MARS_CUDA(mars::launch_domain_stats(d_D, g, ds, st));
    mars::ftc::FisherTcArgs a{};
    uint8_t *rbucket = nullptr, *riso = nullptr;
    uint32_t *rlist = nullptr, *plan = nullptr, *ref_scratch = nullptr;
    MARS_CUDA(sc.get(&rbucket, n));
    MARS_CUDA(sc.get(&riso, n));
    MARS_CUDA(sc.get(&rlist, n));
    MARS_CUDA(sc.get(&a.rrank, n));
    MARS_CUDA(sc.get(&plan, mars::ftc::kPlanWords));
    MARS_CUDA(sc.get(&ref_scratch, 72));
    uint32_t* group_work = nullptr;
    MARS_CUDA(sc.get(&group_work, mars::fisher_group_work_words((size_t)n)));
    a.plan.rcounts = plan;
    a.plan.roffsets = plan + 72;
    a.plan.p_base = plan + 144;
    a.plan.chunks = plan + 216;
    a.plan.ntiles = plan + 288;
    a.plan.a_tile_base = plan + 360;
    a.plan.b_tile_base = plan + 433;
    a.plan.item_base = plan + 506;
    MARS_CUDA(mars::ftc::launch_range_classes(d_plane, (int)w, (int)h, g.size, d_rows, d_cols, n,
                                              ix.ref, rbucket, riso, st));
    MARS_CUDA(mars::launch_fisher_group(rbucket, n, a.plan.rcounts, a.plan.roffsets, ref_scratch,
                                        rlist, group_work, st));
    a.a_rows_max = mars::ftc::a_rows_max(npos);
    a.b_rows_max = mars::ftc::b_rows_max((size_t)n);
    a.items_max = mars::ftc::items_max((size_t)n);
    MARS_CUDA(sc.get(&a.aglob, mars::ftc::a_bytes(g.size, npos)));
    MARS_CUDA(sc.get(&a.bglob, mars::ftc::b_bytes(g.size, (size_t)n)));
    MARS_CUDA(sc.get(&a.seeds, n));
    MARS_CUDA(sc.get(&a.partials, mars::ftc::partials_max((size_t)n)));
    a.plane = d_plane;
    a.w = (int)w;
    a.h = (int)h;
    a.D = d_D;
    a.dw = g.dw;
    a.size = g.size;
    a.shift = g.shift;
    a.ncol_d = g.ncol_d;
    a.rows = d_rows;
    a.cols = d_cols;
    a.nranges = n;
    a.ix = ix;
    a.rbucket = rbucket;
    a.riso = riso;
    a.rlist = rlist;
    a.rs = rs;
    a.ds = ds;
    a.fp = fp;
    a.out = d_out;
    a.evals = d_evals;
    a.err = ctx->d_err;
    a.counter = ctx->d_counter;
    MARS_CUDA(mars::ftc::launch_search(a, st));
    ctx->launches += 13;
    return MARS_OK;
}

// Fisher's classified search for every job: per (size, shift) the domain index
// (Fisher::index) and the searches of the job's nodes (Fisher::candidates +
// search_block_fitted); per-node eval counts come back from the device.
// `d_rc_in`: the job origins already on the device (job_origins layout), else uploaded here.
int run_jobs_fisher(mars_ctx* ctx, Scratch& sc, const uint8_t* d_plane, uint32_t w, uint32_t h,
                    const mars::FitParams& fp, const std::vector<Job>& jobs,
                    mars::CandidateOut* d_out, uint64_t* d_evals,
                    const uint32_t* d_rc_in = nullptr) {
    const cudaStream_t st = ctx->stream;
    int32_t* d_D = nullptr;
    const int dw = (int)(w / 2);
    MARS_CUDA(sc.get(&d_D, std::max<size_t>(1, (size_t)(w / 2) * (h / 2))));
    MARS_CUDA(mars::launch_contract(d_plane, (int)w, (int)h, d_D, st));
    ctx->launches += 1;
    size_t total = 0, max_pos = 0;
    for (const Job& j : jobs) {
        total += j.rows.size();
        const mars::LevelGeom g = level_geom(w, h, j.size, j.shift);
        if (g.nrow_d > 0 && g.ncol_d > 0) max_pos = std::max(max_pos, (size_t)g.nrow_d * g.ncol_d);
    }
    const uint32_t* d_rc = d_rc_in;
    size_t off = 0;
    if (!d_rc) {
        std::vector<uint32_t> rc(2 * total);
        for (const Job& j : jobs) {
            std::copy(j.rows.begin(), j.rows.end(), rc.begin() + (long)off);
            std::copy(j.cols.begin(), j.cols.end(), rc.begin() + (long)(total + off));
            off += j.rows.size();
        }
        uint32_t* d = nullptr;
        MARS_CUDA(sc.get(&d, std::max<size_t>(1, rc.size())));
        // A pageable source: the call returns once the bytes are staged, so `rc` may go.
        MARS_CUDA(cudaMemcpyAsync(d, rc.data(), rc.size() * 4, cudaMemcpyHostToDevice, st));
        d_rc = d;
    }
    mars::FisherIndex ix;
    MARS_CUDA(sc.get(&ix.key, std::max<size_t>(1, max_pos)));
    MARS_CUDA(sc.get(&ix.diso, std::max<size_t>(1, max_pos)));
    MARS_CUDA(sc.get(&ix.list, std::max<size_t>(1, max_pos)));
    MARS_CUDA(sc.get(&ix.counts, 72));
    MARS_CUDA(sc.get(&ix.offsets, 72));
    MARS_CUDA(sc.get(&ix.ref, 72));
    MARS_CUDA(sc.get(&ix.work, mars::fisher_group_work_words(max_pos)));
    size_t max_part = 1;
    for (const Job& j : jobs)
        max_part = std::max(max_part, j.rows.size() * (size_t)mars::fisher_warps_per_range((int)j.size));
    mars::CandidateOut* part = nullptr;
    uint32_t* part_e = nullptr;
    MARS_CUDA(sc.get(&part, max_part));
    MARS_CUDA(sc.get(&part_e, max_part));
    off = 0;
    for (const Job& j : jobs) {
        const mars::LevelGeom g = level_geom(w, h, j.size, j.shift);
        const int nrow = std::max(g.nrow_d, 0), ncol = std::max(g.ncol_d, 0);
        const int n = (int)j.rows.size();
        MARS_CUDA(mars::launch_fisher_index(d_D, dw, (int)j.size, (int)j.shift, nrow, ncol, ix, st));
        ctx->launches += nrow * ncol > 0 ? 4 : 2;
        if (use_fisher_tc(ctx, j.size, j.shift) && nrow * ncol > 0 && n > 0) {
            if (int e = run_fisher_tc(ctx, sc, d_plane, d_D, w, h, g, fp, d_rc + off,
                                      d_rc + total + off, n, ix, d_out + off, d_evals + off))
                return e;
        } else {
            MARS_CUDA(mars::launch_fisher_search(d_plane, (int)w, (int)h, d_D, dw, (int)j.size,
                                                 (int)j.shift, std::max(ncol, 1), d_rc + off,
                                                 d_rc + total + off, n, ix, fp, d_out + off,
                                                 d_evals + off, part, part_e, st));
            ctx->launches += 1 + (mars::fisher_warps_per_range((int)j.size) > 1);
        }
        off += j.rows.size();
    }
    return MARS_OK;
}

int run_jobs_branched(mars_ctx* ctx, Scratch& sc, const uint8_t* d_plane, uint32_t w, uint32_t h,
                      const mars::FitParams& fp, const std::vector<Job>& jobs,
                      mars::CandidateOut* d_out, const uint32_t* d_rc, uint32_t k);

int build_table(mars_ctx* ctx, const uint8_t* plane, const uint8_t* d_plane_in, uint32_t w,
                uint32_t h, const mars_params* params, bool adaptive, mars_table** out,
                int method = MARS_METHOD_EXHAUSTIVE, uint32_t k = 1) {
    if (!ctx || !out) return fail(MARS_EINVAL, "NULL argument");
    if (int e = check_params(params)) return e;
    if (k < 1 || k > (uint32_t)mars::kMaxTopK)
        return fail(MARS_EUNSUPPORTED, "ranked searches keep 1.." + std::to_string(mars::kMaxTopK) +
                                           " candidates per node");
    if (k > 1 && method != MARS_METHOD_EXHAUSTIVE)
        return fail(MARS_EINVAL, "a ranked search needs the exhaustive method; other methods "
                                 "propose one candidate");
    if (method != MARS_METHOD_EXHAUSTIVE && method != MARS_METHOD_FISHER)
        return fail(MARS_EUNSUPPORTED, "unknown search method " + std::to_string(method));
    if (method == MARS_METHOD_FISHER && params->max_size > 64)
        return fail(MARS_EUNSUPPORTED, "the classified search supports block sizes up to 64");
    if (w == 0 || h == 0 || w > 65535 || h > 65535)
        return fail(MARS_EINVAL, "plane dimensions must be in 1..65535");
    std::lock_guard<std::mutex> lock(ctx->mu);
    MARS_CUDA(cudaSetDevice(ctx->device));
    const mars::FitParams fp = make_fit_params(*params);
    std::vector<uint8_t> host_plane;
    if (!plane && adaptive) {
        host_plane.resize((size_t)w * h);
        MARS_CUDA(cudaMemcpy(host_plane.data(), d_plane_in, host_plane.size(),
                             cudaMemcpyDeviceToHost));
        plane = host_plane.data();
    }
    const std::vector<Job> jobs = plan_jobs(plane, w, h, *params, adaptive);
    size_t total = 0;
    for (const Job& j : jobs) total += j.rows.size();
    if (total > 0xffffffffull) return fail(MARS_EINVAL, "too many quadtree nodes");
    auto* t = new (std::nothrow) mars_table;
    if (!t) return fail(MARS_ENOMEM, "table allocation failed");
    std::unique_ptr<mars_table> guard(t);
    t->width = w;
    t->height = h;
    t->k = k;
    t->cands.resize(total);
    t->evals.resize(total);
    if (k > 1) t->ranked.resize(total * k);
    {
        Scratch sc(ctx->stream);
        const uint8_t* d_plane = d_plane_in;
        if (!d_plane) {
            uint8_t* dp = nullptr;
            MARS_CUDA(sc.get(&dp, (size_t)w * h));
            MARS_CUDA(cudaMemcpyAsync(dp, plane, (size_t)w * h, cudaMemcpyHostToDevice,
                                      ctx->stream));
            d_plane = dp;
        }
        mars::CandidateOut* d_out = nullptr;
        MARS_CUDA(sc.get(&d_out, total * k));
        MARS_CUDA(cudaMemsetAsync(ctx->d_counter, 0, sizeof(unsigned long long), ctx->stream));
        if (method == MARS_METHOD_FISHER) {
            uint64_t* d_evals = nullptr;
            MARS_CUDA(sc.get(&d_evals, total));
            if (int e = run_jobs_fisher(ctx, sc, d_plane, w, h, fp, jobs, d_out, d_evals)) return e;
            MARS_CUDA(cudaMemcpyAsync(t->evals.data(), d_evals, total * sizeof(uint64_t),
                                      cudaMemcpyDeviceToHost, ctx->stream));
        } else if (k == 1 && all_levels_eligible(ctx, w, h, jobs)) {
            if (int e = run_jobs_all_levels(ctx, sc, d_plane, w, h, fp, jobs, d_out, nullptr))
                return e;
        } else if (k > 1) {
            // The ranked search: the levels as parallel branches (run_jobs_branched).
            size_t tot = 0;
            const std::vector<uint32_t> rc = job_origins(jobs, &tot);
            uint32_t* d_rc = nullptr;
            MARS_CUDA(sc.get(&d_rc, rc.size()));
            MARS_CUDA(cudaMemcpyAsync(d_rc, rc.data(), rc.size() * 4, cudaMemcpyHostToDevice,
                                      ctx->stream));
            if (int e = run_jobs_branched(ctx, sc, d_plane, w, h, fp, jobs, d_out, d_rc, k))
                return e;
        } else {
            if (int e = run_jobs(ctx, sc, d_plane, w, h, fp, jobs, d_out, k)) return e;
        }
        MARS_CUDA(cudaMemcpyAsync(k > 1 ? t->ranked.data() : t->cands.data(), d_out,
                                  total * k * sizeof(mars_candidate), cudaMemcpyDeviceToHost,
                                  ctx->stream));
        unsigned long long exact = 0;
        MARS_CUDA(cudaMemcpyAsync(&exact, ctx->d_counter, sizeof exact, cudaMemcpyDeviceToHost,
                                  ctx->stream));
        if (int e = sync_bounded(ctx)) return e;
        t->exact_fits = exact;
        if (k > 1)
            for (size_t i = 0; i < total; ++i) t->cands[i] = t->ranked[i * k];
    }
    size_t off = 0;
    for (const Job& j : jobs) {
        const uint64_t ev = level_evals(w, h, j.size, j.shift);
        t->index.add_job(j.size, j.shift, w, h, j.rows.data(), j.cols.data(), j.rows.size(),
                         (uint32_t)off);
        for (size_t i = 0; i < j.rows.size(); ++i) {
            if (method == MARS_METHOD_EXHAUSTIVE) t->evals[off + i] = ev;
            t->total_evals += t->evals[off + i];
        }
        off += j.rows.size();
    }
    *out = guard.release();
    return MARS_OK;
}

}  // namespace

extern "C" {

const char* mars_last_error(void) { return g_err.c_str(); }
const char* mars_version(void) { return "mars_b200 0.1 (sm_100a)"; }

int mars_ctx_create(mars_ctx** out, int device) {
    if (!out) return fail(MARS_EINVAL, "out is NULL");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
        return fail(MARS_ENODEV, "no CUDA device is available");
    if (device < 0 || device >= n) return fail(MARS_EINVAL, "device index out of range");
    cudaDeviceProp prop;
    MARS_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10)
        return fail(MARS_ENODEV, "mars_b200 is built for sm_100a (B200); this device is sm_" +
                                     std::to_string(prop.major) + std::to_string(prop.minor));
    auto* c = new (std::nothrow) mars_ctx;
    if (!c) return fail(MARS_ENOMEM, "context allocation failed");
    c->device = device;
    c->num_sms = prop.multiProcessorCount;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_counter, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&c->d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(c->d_err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&c->h_err, sizeof(int));
    if (e == cudaSuccess) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            c->encode_tiled = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    if (e == cudaSuccess) {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t thr = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
    }
    if (e != cudaSuccess) {
        if (c->own_stream) cudaStreamDestroy(c->own_stream);
        if (c->h_err) cudaFreeHost(c->h_err);
        delete c;
        return fail(MARS_ECUDA, std::string("context setup: ") + cudaGetErrorString(e));
    }
    c->stream = c->own_stream;
    *out = c;
    return MARS_OK;
}

void mars_ctx_destroy(mars_ctx* ctx) {
    if (!ctx) return;
    for (auto& kp : ctx->plan_cache) mars_search_plan_free(kp.second);
    ctx->plan_cache.clear();
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->d_counter) cudaFree(ctx->d_counter);
    if (ctx->d_err) cudaFree(ctx->d_err);
    if (ctx->h_err) cudaFreeHost(ctx->h_err);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    for (int b = 0; b < mars_ctx::kBranches; ++b) {
        if (ctx->branch[b]) cudaStreamDestroy(ctx->branch[b]);
        if (ctx->join_ev[b]) cudaEventDestroy(ctx->join_ev[b]);
    }
    if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
    delete ctx;
}

int mars_ctx_set_stream(mars_ctx* ctx, void* stream) {
    if (!ctx) return fail(MARS_EINVAL, "ctx is NULL");
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return MARS_OK;
}

uint64_t mars_ctx_launch_count(const mars_ctx* ctx) { return ctx ? ctx->launches.load() : 0; }

int mars_ctx_set_search_path(mars_ctx* ctx, int32_t path) {
    if (!ctx || path < 0 || path > 5) return fail(MARS_EINVAL, "path must be 0 .. 5");
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->search_path = path >= 3 ? 0 : path;
    ctx->tma_16_boxes = path == 3;
    ctx->fold_only = path == 4;
    ctx->per_level = path == 5;
    return MARS_OK;
}

int mars_search_table_build(mars_ctx* ctx, const uint8_t* plane, uint32_t width, uint32_t height,
                            const mars_params* params, int32_t adaptive_density,
                            mars_table** out) {
    if (!plane) return fail(MARS_EINVAL, "plane is NULL");
    return build_table(ctx, plane, nullptr, width, height, params, adaptive_density != 0, out);
}

int mars_indexed_table_build(mars_ctx* ctx, const uint8_t* plane, uint32_t width,
                             uint32_t height, const mars_params* params, int32_t adaptive_density,
                             int32_t method, mars_table** out) {
    if (!plane) return fail(MARS_EINVAL, "plane is NULL");
    return build_table(ctx, plane, nullptr, width, height, params, adaptive_density != 0, out,
                       method);
}

int mars_search_table_lookup(const mars_table* t, uint32_t row, uint32_t col, uint32_t size,
                             uint32_t shift, mars_candidate* out, uint64_t* evals) {
    if (!t || !out) return fail(MARS_EINVAL, "NULL argument");
    const int64_t at = t->nodes().find(row, col, size, shift);
    if (at < 0)
        return fail(MARS_ENOTFOUND, "node (" + std::to_string(row) + "," + std::to_string(col) +
                                        "," + std::to_string(size) + ") at shift " +
                                        std::to_string(shift) + " is not in the table");
    *out = t->cands[(size_t)at];
    if (evals) *evals = t->evals[(size_t)at];
    return MARS_OK;
}

int mars_search_table_build_ranked(mars_ctx* ctx, const uint8_t* plane, uint32_t width,
                                   uint32_t height, const mars_params* params,
                                   int32_t adaptive_density, uint32_t k, mars_table** out) {
    if (!plane) return fail(MARS_EINVAL, "plane is NULL");
    return build_table(ctx, plane, nullptr, width, height, params, adaptive_density != 0, out,
                       MARS_METHOD_EXHAUSTIVE, k);
}

int mars_search_table_lookup_ranked(const mars_table* t, uint32_t row, uint32_t col,
                                    uint32_t size, uint32_t shift, uint32_t max,
                                    mars_candidate* out, uint32_t* count, uint64_t* evals) {
    if (!t || !count || (max && !out)) return fail(MARS_EINVAL, "NULL argument");
    const int64_t at = t->nodes().find(row, col, size, shift);
    if (at < 0)
        return fail(MARS_ENOTFOUND, "node (" + std::to_string(row) + "," + std::to_string(col) +
                                        "," + std::to_string(size) + ") at shift " +
                                        std::to_string(shift) + " is not in the table");
    const size_t i = (size_t)at;
    const mars_candidate* src = t->k > 1 ? &t->ranked[i * t->k] : &t->cands[i];
    uint32_t n = 0;
    const uint32_t lim = std::min<uint32_t>(std::max<uint32_t>(max, 1), t->k);
    for (uint32_t j = 0; j < lim && n < max; ++j)
        if (src[j].valid) out[n++] = src[j];
    *count = n;
    if (evals) *evals = t->evals[i];
    return MARS_OK;
}

uint64_t mars_search_table_evals(const mars_table* t) { return t ? t->total_evals : 0; }
uint64_t mars_search_table_exact_fits(const mars_table* t) { return t ? t->exact_fits : 0; }

void mars_search_table_free(mars_table* t) { delete t; }

int mars_search_blocks(mars_ctx* ctx, const uint8_t* plane, uint32_t width, uint32_t height,
                       uint32_t size, uint32_t shift, const mars_params* params,
                       const uint32_t* rows, const uint32_t* cols, size_t n,
                       mars_candidate* out, uint64_t* evals) {
    if (!ctx || !plane || (n && (!rows || !cols || !out))) return fail(MARS_EINVAL, "NULL argument");
    if (int e = check_params(params)) return e;
    if (!is_pow2(size) || size < 2 || size > 64)
        return fail(size > 64 ? MARS_EUNSUPPORTED : MARS_EINVAL, "size must be a power of two in 2..64");
    if (shift == 0 || (shift & 1)) return fail(MARS_EUNSUPPORTED, "shift must be even");
    for (size_t i = 0; i < n; ++i)
        if (rows[i] + size > height || cols[i] + size > width)
            return fail(MARS_EINVAL, "block " + std::to_string(i) + " runs past the plane");
    std::lock_guard<std::mutex> lock(ctx->mu);
    MARS_CUDA(cudaSetDevice(ctx->device));
    const mars::FitParams fp = make_fit_params(*params);
    Job job{size, shift, std::vector<uint32_t>(rows, rows + n), std::vector<uint32_t>(cols, cols + n)};
    {
        Scratch sc(ctx->stream);
        uint8_t* dp = nullptr;
        mars::CandidateOut* d_out = nullptr;
        MARS_CUDA(sc.get(&dp, (size_t)width * height));
        MARS_CUDA(sc.get(&d_out, n));
        MARS_CUDA(cudaMemcpyAsync(dp, plane, (size_t)width * height, cudaMemcpyHostToDevice,
                                  ctx->stream));
        if (int e = run_jobs(ctx, sc, dp, width, height, fp, {job}, d_out)) return e;
        MARS_CUDA(cudaMemcpyAsync(out, d_out, n * sizeof(mars_candidate), cudaMemcpyDeviceToHost,
                                  ctx->stream));
        if (int e = sync_bounded(ctx)) return e;
    }
    const uint64_t ev = level_evals(width, height, size, shift);
    if (evals)
        for (size_t i = 0; i < n; ++i) evals[i] = ev;
    return MARS_OK;
}

int mars_search_blocks_device(mars_ctx* ctx, const uint8_t* d_plane, uint32_t width,
                              uint32_t height, uint32_t size, uint32_t shift,
                              const mars_params* params, const uint32_t* d_rows,
                              const uint32_t* d_cols, size_t n, mars_candidate* d_out) {
    if (!ctx || !d_plane || (n && (!d_rows || !d_cols || !d_out)))
        return fail(MARS_EINVAL, "NULL argument");
    if (int e = check_params(params)) return e;
    if (!is_pow2(size) || size < 2 || size > 64)
        return fail(size > 64 ? MARS_EUNSUPPORTED : MARS_EINVAL, "size must be a power of two in 2..64");
    if (shift == 0 || (shift & 1)) return fail(MARS_EUNSUPPORTED, "shift must be even");
    std::lock_guard<std::mutex> lock(ctx->mu);
    MARS_CUDA(cudaSetDevice(ctx->device));
    const mars::FitParams fp = make_fit_params(*params);
    Scratch sc(ctx->stream);
    int32_t* d_D = nullptr;
    MARS_CUDA(sc.get(&d_D, (size_t)(width / 2) * (height / 2)));
    MARS_CUDA(mars::launch_contract(d_plane, (int)width, (int)height, d_D, ctx->stream));
    ctx->launches += 1;
    return run_level(ctx, sc, d_plane, d_D, width, height, size, shift, fp, d_rows, d_cols, n,
                     (mars::CandidateOut*)d_out);
}

int mars_search_blocks_cross_device(mars_ctx* ctx, const uint8_t* d_range_plane,
                                    const uint8_t* d_domain_plane, uint32_t width,
                                    uint32_t height, uint32_t size, uint32_t shift,
                                    const mars_params* params, const uint32_t* d_rows,
                                    const uint32_t* d_cols, size_t n, mars_candidate* d_out) {
    if (!ctx || !d_range_plane || !d_domain_plane || (n && (!d_rows || !d_cols || !d_out)))
        return fail(MARS_EINVAL, "NULL argument");
    if (int e = check_params(params)) return e;
    if (!is_pow2(size) || size < 2 || size > 64)
        return fail(size > 64 ? MARS_EUNSUPPORTED : MARS_EINVAL, "size must be a power of two in 2..64");
    if (shift == 0 || (shift & 1)) return fail(MARS_EUNSUPPORTED, "shift must be even");
    std::lock_guard<std::mutex> lock(ctx->mu);
    MARS_CUDA(cudaSetDevice(ctx->device));
    const mars::FitParams fp = make_fit_params(*params);
    Scratch sc(ctx->stream);
    int32_t* d_D = nullptr;
    MARS_CUDA(sc.get(&d_D, (size_t)(width / 2) * (height / 2)));
    MARS_CUDA(mars::launch_contract(d_domain_plane, (int)width, (int)height, d_D, ctx->stream));
    ctx->launches += 1;
    return run_level(ctx, sc, d_range_plane, d_D, width, height, size, shift, fp, d_rows, d_cols,
                     n, (mars::CandidateOut*)d_out, 1, d_domain_plane);
}

int mars_search_nodes_device(mars_ctx* ctx, const uint8_t* d_plane, uint32_t width,
                             uint32_t height, const mars_params* params, mars_candidate* d_out,
                             size_t capacity, size_t* n_nodes, uint64_t* total_evals) {
    if (!ctx || !d_plane || !n_nodes) return fail(MARS_EINVAL, "NULL argument");
    if (int e = check_params(params)) return e;
    if (width == 0 || height == 0 || width > 65535 || height > 65535)
        return fail(MARS_EINVAL, "plane dimensions must be in 1..65535");
    const std::vector<Job> jobs = plan_jobs(nullptr, width, height, *params, false);
    size_t total = 0;
    uint64_t ev = 0;
    for (const Job& j : jobs) {
        total += j.rows.size();
        ev += level_evals(width, height, j.size, j.shift) * j.rows.size();
    }
    *n_nodes = total;
    if (total_evals) *total_evals = ev;
    if (!d_out) return MARS_OK;
    if (capacity < total) return fail(MARS_EINVAL, "d_out holds fewer entries than nodes");
    std::lock_guard<std::mutex> lock(ctx->mu);
    MARS_CUDA(cudaSetDevice(ctx->device));
    Scratch sc(ctx->stream);
    return run_jobs(ctx, sc, d_plane, width, height, make_fit_params(*params), jobs,
                    (mars::CandidateOut*)d_out);
}

}  // extern "C"

namespace {

// The RD walk's node pricing on the device (rdprice.cu): the batch's plane, rate table,
// bases, nodes and candidates up, one launch per node size, the winners and levels down.
// Where it runs: on the device when the residual mode is allowed (a forward and an inverse
// DCT per node and candidate) or candidates are ranked; otherwise the host walk's per-node
// fits (O(size^2) each) cost less than the batch's round trip.  MARS_PRICING=host or
// =device pins either (the same price_node code, the same doubles).
bool price_on_device_for(const mars_options& o) {
    static const int pinned = [] {
        const char* e = std::getenv("MARS_PRICING");
        if (!e) return 0;
        if (std::string(e) == "host") return 1;
        if (std::string(e) == "device") return 2;
        return 0;
    }();
    if (pinned) return pinned == 2;
    return o.allowed_modes[3] != 0 || o.rd_candidates > 1;
}

// A stream of its own for one call, so concurrent encodes on a context do not wait behind
// each other's searches; destroyed (after its queued work) when the call returns.
struct OwnStream {
    cudaStream_t st = nullptr;
    ~OwnStream() {
        if (st) cudaStreamDestroy(st);
    }
};

int price_on_device(mars_ctx* ctx, mars::codec::PriceBatch& b) {
    MARS_CUDA(cudaSetDevice(ctx->device));
    OwnStream own;
    MARS_CUDA(cudaStreamCreateWithFlags(&own.st, cudaStreamNonBlocking));
    const cudaStream_t st = own.st;
    Scratch sc(st);
    const size_t nodes = b.row.size();
    const bool residual = b.setup.allowed[3] != 0;
    size_t nbasis = 0;
    for (uint32_t s : b.sizes) nbasis += (size_t)s * s;
    uint8_t* d_px;
    double *d_bits, *d_basis;
    int64_t* d_off;
    uint32_t *d_rows, *d_cols;
    mars::price::Cand* d_cands;
    uint64_t* d_lat;
    mars::price::Priced* d_out;
    int8_t* d_lev;
    const size_t noff = (size_t)mars::price::kFields * mars::price::kCtx;
    MARS_CUDA(sc.get(&d_px, (size_t)b.im.w * b.im.h));
    MARS_CUDA(sc.get(&d_bits, b.nbits));
    MARS_CUDA(sc.get(&d_off, noff));
    MARS_CUDA(sc.get(&d_basis, nbasis));
    MARS_CUDA(sc.get(&d_rows, nodes));
    MARS_CUDA(sc.get(&d_cols, nodes));
    MARS_CUDA(sc.get(&d_cands, b.cands.size()));
    MARS_CUDA(sc.get(&d_lat, nodes));
    MARS_CUDA(sc.get(&d_out, nodes));
    MARS_CUDA(sc.get(&d_lev, residual ? b.nlevels : 1));
    MARS_CUDA(cudaMemcpyAsync(d_px, b.im.px, (size_t)b.im.w * b.im.h, cudaMemcpyHostToDevice, st));
    MARS_CUDA(cudaMemcpyAsync(d_bits, b.bits, b.nbits * sizeof(double), cudaMemcpyHostToDevice, st));
    MARS_CUDA(cudaMemcpyAsync(d_off, b.offset, noff * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    MARS_CUDA(cudaMemcpyAsync(d_rows, b.row.data(), nodes * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    MARS_CUDA(cudaMemcpyAsync(d_cols, b.col.data(), nodes * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    MARS_CUDA(cudaMemcpyAsync(d_cands, b.cands.data(), b.cands.size() * sizeof(mars::price::Cand),
                              cudaMemcpyHostToDevice, st));
    if (residual)
        MARS_CUDA(cudaMemcpyAsync(d_lat, b.levels_at.data(), nodes * sizeof(uint64_t),
                                  cudaMemcpyHostToDevice, st));
    size_t at = 0;
    for (size_t g = 0; g < b.sizes.size(); ++g) {
        const size_t n = (size_t)b.sizes[g] * b.sizes[g];
        MARS_CUDA(cudaMemcpyAsync(d_basis + at, b.basis[g], n * sizeof(double),
                                  cudaMemcpyHostToDevice, st));
        at += n;
    }
    at = 0;
    for (size_t g = 0; g < b.sizes.size(); ++g) {
        const uint32_t size = b.sizes[g], first = b.first[g], count = b.first[g + 1] - first;
        mars::PriceLaunch a{};
        a.px = d_px;
        a.stride = b.im.w;
        a.size = size;
        a.count = count;
        a.rows = d_rows + first;
        a.cols = d_cols + first;
        a.cands = d_cands + (size_t)first * b.k;
        a.k = b.k;
        a.setup = b.setup;
        a.table = {d_bits, d_off};
        a.basis = d_basis + at;
        a.out = d_out + first;
        a.levels = d_lev;
        a.levels_at = d_lat + first;
        const size_t gbytes = mars::price_scratch_bytes(size, count, &a.scratch_slots);
        if (gbytes) MARS_CUDA(sc.get(&a.global_scratch, gbytes));
        MARS_CUDA(mars::launch_price_nodes(a, st));
        ctx->launches += 1;
        at += (size_t)size * size;
    }
    b.priced.resize(nodes);
    MARS_CUDA(cudaMemcpyAsync(b.priced.data(), d_out, nodes * sizeof(mars::price::Priced),
                              cudaMemcpyDeviceToHost, st));
    if (residual) {
        b.levels.resize(b.nlevels);
        MARS_CUDA(cudaMemcpyAsync(b.levels.data(), d_lev, b.nlevels, cudaMemcpyDeviceToHost, st));
    }
    return sync_bounded(ctx, st);
}

// The walks of encode_image_with_search over filled tables (`table` for the final walk,
// `warm` for the RD warm-up), and the C-ABI outputs.
int encode_on_tables(mars_ctx* ctx, const uint8_t* plane, uint32_t width, uint32_t height,
                     const mars_params* params, const mars_options* options, mars_table* table,
                     mars_table* warm, uint32_t rd_k, mars_header* header, mars_leaf** leaves,
                     size_t* nleaves, int32_t** residuals, size_t* nresiduals,
                     mars_counters* counters) {
    auto lookup = [](mars_table* t) {
        return [t](uint32_t row, uint32_t col, uint32_t size, uint32_t shift,
                   mars::codec::SearchAnswer* ans) {
            return mars_search_table_lookup(t, row, col, size, shift, &ans->cand, &ans->evals);
        };
    };
    const mars::codec::Provider provider = lookup(table);
    const mars::codec::Provider warmup = lookup(warm);
    const mars::codec::RankedProvider ranked = [table](uint32_t row, uint32_t col, uint32_t size,
                                                       uint32_t shift, uint32_t max,
                                                       std::vector<mars_candidate>* v,
                                                       uint64_t* evals) {
        v->resize(std::max<uint32_t>(max, 1));
        uint32_t n = 0;
        const int e = mars_search_table_lookup_ranked(table, row, col, size, shift, max, v->data(),
                                                      &n, evals);
        v->resize(e ? 0 : n);
        return e;
    };
    std::vector<mars_leaf> out;
    std::vector<int32_t> res;
    const mars::codec::Image im{plane, width, height};
    const mars::codec::Pricer pricer = [ctx](mars::codec::PriceBatch& b) {
        return price_on_device(ctx, b);
    };
    if (int e = mars::codec::encode(im, *params, *options, provider, warmup, header, &out, &res,
                                    counters, rd_k > 1 ? &ranked : nullptr,
                                    price_on_device_for(*options) ? &pricer : nullptr))
        return e;
    *nleaves = out.size();
    *leaves = (mars_leaf*)std::malloc(std::max<size_t>(1, out.size()) * sizeof(mars_leaf));
    if (!*leaves) return fail(MARS_ENOMEM, "leaf array allocation failed");
    std::memcpy(*leaves, out.data(), out.size() * sizeof(mars_leaf));
    *nresiduals = res.size();
    *residuals = (int32_t*)std::malloc(std::max<size_t>(1, res.size()) * sizeof(int32_t));
    if (!*residuals) {
        std::free(*leaves);
        *leaves = nullptr;
        return fail(MARS_ENOMEM, "residual array allocation failed");
    }
    if (!res.empty()) std::memcpy(*residuals, res.data(), res.size() * sizeof(int32_t));
    return MARS_OK;
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {

// The plan mars_encode uses for a plane geometry it has encoded before: one search plan
// per (width, height, params), made on the second encode of that geometry (the first takes
// the one-shot path), for planes up to kPlanCachePixels and at most kPlanCacheSize
// geometries per context.  Null when the geometry should take the one-shot path.
// MARS_PLAN_CACHE=0 turns the cache off.
constexpr uint64_t kPlanCachePixels = 2048ull * 2048ull;
constexpr size_t kPlanCacheSize = 8, kPlansSeen = 64;

mars_search_plan* cached_encode_plan(mars_ctx* ctx, uint32_t w, uint32_t h,
                                     const mars_params* p,
                                     int32_t method = MARS_METHOD_EXHAUSTIVE) {
    static const bool off = [] {
        const char* e = std::getenv("MARS_PLAN_CACHE");
        return e && std::string(e) == "0";
    }();
    if (off || (uint64_t)w * h > kPlanCachePixels) return nullptr;
    std::string key(reinterpret_cast<const char*>(&w), sizeof w);
    key.append(reinterpret_cast<const char*>(&h), sizeof h);
    key.append(reinterpret_cast<const char*>(p), sizeof *p);
    key.append(reinterpret_cast<const char*>(&method), sizeof method);
    std::lock_guard<std::mutex> lock(ctx->plan_cache_mu);
    for (auto& kp : ctx->plan_cache)
        if (kp.first == key) return kp.second;
    auto seen = std::find(ctx->plans_seen.begin(), ctx->plans_seen.end(), key);
    if (seen == ctx->plans_seen.end() || ctx->plan_cache.size() >= kPlanCacheSize) {
        if (seen == ctx->plans_seen.end()) {
            if (ctx->plans_seen.size() >= kPlansSeen) ctx->plans_seen.erase(ctx->plans_seen.begin());
            ctx->plans_seen.push_back(key);
        }
        return nullptr;
    }
    mars_search_plan* plan = nullptr;
    if (mars_indexed_plan_create(ctx, w, h, p, method, &plan) != MARS_OK) {
        cudaGetLastError();  // the one-shot path serves this call: leave no stale error
        return nullptr;
    }
    ctx->plan_cache.emplace_back(key, plan);
    return plan;
}

}  // namespace

extern "C" {

int mars_encode(mars_ctx* ctx, const uint8_t* plane, uint32_t width, uint32_t height,
                const mars_params* params, const mars_options* options, mars_header* header,
                mars_leaf** leaves, size_t* nleaves, int32_t** residuals, size_t* nresiduals,
                mars_counters* counters) {
    if (!ctx || !plane || !options || !header || !leaves || !nleaves || !residuals ||
        !nresiduals || !counters)
        return fail(MARS_EINVAL, "NULL argument");
    if (int e = check_params(params)) return e;
    if (!options->residual_adaptive && options->residual_qstep != 0.0f &&
        !(std::isfinite(options->residual_qstep) && options->residual_qstep >= 1.0f &&
          options->residual_qstep <= 65535.0f))
        return fail(MARS_EINVAL, "residual qstep must be finite and in [1, 65535]");
    const uint32_t rd_k = std::max<uint32_t>(1, options->rd_candidates);
    if (rd_k > 1 && !params->has_lambda)
        return fail(MARS_EINVAL, "rd_candidates > 1 requires the RD path (a lambda)");
    if (rd_k > 1 && options->method != MARS_METHOD_EXHAUSTIVE)
        return fail(MARS_EINVAL, "rd_candidates > 1 requires the exhaustive search; other "
                                 "methods propose one candidate");
    const bool adaptive = params->has_lambda && options->adaptive_density;
    // A geometry met before: its search plan (one graph launch, both walks on the device).
    if (options->method == MARS_METHOD_EXHAUSTIVE && rd_k == 1 && !adaptive)
        if (mars_search_plan* plan = cached_encode_plan(ctx, width, height, params))
            return mars_encode_planned(plan, plane, options, header, leaves, nleaves, residuals,
                                       nresiduals, counters);
    // A Fisher encode of a geometry met before: the final walk's table from the context's
    // Fisher plan, the warm-up walk's exhaustive table from its exhaustive plan.
    if (options->method == MARS_METHOD_FISHER && rd_k == 1 && !adaptive) {
        mars_params wp = *params;
        wp.has_lambda = 0;
        // Both keys are looked up on every call, so both plans are made on the second encode.
        mars_search_plan* fplan = cached_encode_plan(ctx, width, height, params, MARS_METHOD_FISHER);
        mars_search_plan* wplan =
            params->has_lambda ? cached_encode_plan(ctx, width, height, &wp) : nullptr;
        if (fplan && (!params->has_lambda || wplan)) {
            mars_table* ft = nullptr;
            mars_table* wt = nullptr;
            if (int e = mars_search_plan_run(fplan, plane, &ft)) return e;
            std::unique_ptr<mars_table, void (*)(mars_table*)> fguard(ft, mars_search_table_free);
            if (wplan)
                if (int e = mars_search_plan_run(wplan, plane, &wt)) return e;
            std::unique_ptr<mars_table, void (*)(mars_table*)> wguard(wt, mars_search_table_free);
            return encode_on_tables(ctx, plane, width, height, params, options, ft, wt ? wt : ft,
                                    rd_k, header, leaves, nleaves, residuals, nresiduals,
                                    counters);
        }
    }
    // The final walk's provider (the options' method) and, for an RD encode, the
    // exhaustive table the warm-up walk reads (the warm-up is exhaustive for every method).
    mars_table* table = nullptr;
    mars_table* warm = nullptr;
    if (int e = build_table(ctx, plane, nullptr, width, height, params, adaptive, &table,
                            options->method, rd_k))
        return e;
    std::unique_ptr<mars_table, void (*)(mars_table*)> guard(table, mars_search_table_free);
    if (params->has_lambda && options->method != MARS_METHOD_EXHAUSTIVE) {
        mars_params wp = *params;
        wp.has_lambda = 0;
        if (int e = build_table(ctx, plane, nullptr, width, height, &wp, false, &warm)) return e;
    }
    std::unique_ptr<mars_table, void (*)(mars_table*)> wguard(warm, mars_search_table_free);
    return encode_on_tables(ctx, plane, width, height, params, options, table, warm ? warm : table,
                            rd_k, header, leaves, nleaves, residuals, nresiduals, counters);
}

// ---------------------------------------------------------------- search plans
//
// A plan fixes one plane geometry and parameter set: the node lists are uploaded once, the
// device buffers stay allocated, and the whole search -- contraction and every quadtree
// level, each level's statistics, seed, correlation and finish kernels -- is captured once
// into a CUDA graph (the levels' scratch as graph memory nodes, so their addresses and the
// tensor maps built on them hold for every replay).  A run is one graph launch.

}  // extern "C"

struct mars_search_plan {
    mars_ctx* ctx = nullptr;
    uint32_t w = 0, h = 0;
    mars_params params{};
    int method = MARS_METHOD_EXHAUSTIVE;
    // Fisher plans: the eval counts are the bucket lengths, found on the device each run.
    uint64_t* d_evals = nullptr;
    uint64_t* h_evals = nullptr;  // pinned
    std::vector<Job> jobs;
    size_t total = 0;
    uint32_t* d_rc = nullptr;
    uint8_t* d_plane = nullptr;
    mars::CandidateOut* d_out = nullptr;
    uint8_t* h_plane = nullptr;        // pinned staging of the input plane
    mars_candidate* h_out = nullptr;   // pinned staging of the node table
    unsigned long long* h_exact = nullptr;
    cudaGraph_t g_host = nullptr, g_dev = nullptr;
    cudaGraphExec_t x_host = nullptr, x_dev = nullptr;
    uint64_t launches_per_run = 0;
    std::vector<uint64_t> evals;
    uint64_t total_evals = 0;
    std::shared_ptr<const mars::NodeIndex> index;
    // The walks on the device (built on the first encode that uses them).
    std::mutex walk_mu;
    int walk_state = 0;  // 0 not built, 1 built, -1 this plan's tree needs the host walk
    mars::WalkPlan walk{};
    uint32_t *d_wrows = nullptr, *d_wcols = nullptr;
    int32_t *d_child = nullptr, *d_roots = nullptr;
    uint64_t *d_wevals = nullptr, *d_levels_at = nullptr;
    double* d_basis = nullptr;
    std::vector<size_t> basis_at;  // per level, into d_basis
    uint64_t nlevels_total = 0;    // sum of size^2 over the nodes
    // CUDA events recorded inside the graph around the all-levels correlation launch.
    cudaEvent_t ev_corr[2] = {nullptr, nullptr};
    bool corr_timed = false;
};

namespace {

void plan_release(mars_search_plan* p) {
    if (!p) return;
    if (p->x_host) cudaGraphExecDestroy(p->x_host);
    if (p->x_dev) cudaGraphExecDestroy(p->x_dev);
    if (p->g_host) cudaGraphDestroy(p->g_host);
    if (p->g_dev) cudaGraphDestroy(p->g_dev);
    cudaFree(p->d_rc);
    cudaFree(p->d_plane);
    cudaFree(p->d_out);
    cudaFreeHost(p->h_plane);
    cudaFreeHost(p->h_out);
    cudaFreeHost(p->h_exact);
    cudaFree(p->d_evals);
    cudaFreeHost(p->h_evals);
    cudaFree(p->d_wrows);
    cudaFree(p->d_wcols);
    cudaFree(p->d_child);
    cudaFree(p->d_roots);
    cudaFree(p->d_wevals);
    cudaFree(p->d_levels_at);
    cudaFree(p->d_basis);
    if (p->ev_corr[0]) cudaEventDestroy(p->ev_corr[0]);
    if (p->ev_corr[1]) cudaEventDestroy(p->ev_corr[1]);
    delete p;
}

// The plan's device work on the context's stream: with_copies adds the pinned input
// upload and the table / counter downloads around it.
// run_jobs with the levels as parallel branches: the contraction on the context's stream,
// then each level on one of the context's branch streams (its own scratch, allocated and
// freed on that branch), joined back before the results are read.  Inside a capture the
// branches become parallel paths of the graph, so one level's set-up kernels and tail
// overlap another level's correlation.  The caller holds ctx->mu.
int run_jobs_branched(mars_ctx* ctx, Scratch& sc, const uint8_t* d_plane, uint32_t w, uint32_t h,
                      const mars::FitParams& fp, const std::vector<Job>& jobs,
                      mars::CandidateOut* d_out, const uint32_t* d_rc, uint32_t k) {
    const cudaStream_t main = ctx->stream;
    if (!ctx->fork_ev) {
        MARS_CUDA(cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming));
        for (int b = 0; b < mars_ctx::kBranches; ++b) {
            MARS_CUDA(cudaStreamCreateWithFlags(&ctx->branch[b], cudaStreamNonBlocking));
            MARS_CUDA(cudaEventCreateWithFlags(&ctx->join_ev[b], cudaEventDisableTiming));
        }
    }
    int32_t* d_D = nullptr;
    MARS_CUDA(sc.get(&d_D, std::max<size_t>(1, (size_t)(w / 2) * (h / 2))));
    MARS_CUDA(mars::launch_contract(d_plane, (int)w, (int)h, d_D, main));
    ctx->launches += 1;
    size_t total = 0;
    for (const Job& j : jobs) total += j.rows.size();
    MARS_CUDA(cudaEventRecord(ctx->fork_ev, main));
    const int nb = (int)std::min<size_t>(jobs.size(), mars_ctx::kBranches);
    for (int b = 0; b < nb; ++b) MARS_CUDA(cudaStreamWaitEvent(ctx->branch[b], ctx->fork_ev, 0));
    size_t off = 0;
    int err = MARS_OK;
    for (size_t i = 0; i < jobs.size() && !err; ++i) {
        const Job& j = jobs[i];
        const int b = (int)(i % mars_ctx::kBranches);
        ctx->stream = ctx->branch[b];
        {
            Scratch sb(ctx->branch[b]);
            err = run_level(ctx, sb, d_plane, d_D, w, h, j.size, j.shift, fp, d_rc + off,
                            d_rc + total + off, j.rows.size(), d_out + off * k, k);
        }
        ctx->stream = main;
        off += j.rows.size();
    }
    // Join every branch that was forked, also after an error (a capture must end joined).
    for (int b = 0; b < nb; ++b) {
        MARS_CUDA(cudaEventRecord(ctx->join_ev[b], ctx->branch[b]));
        MARS_CUDA(cudaStreamWaitEvent(main, ctx->join_ev[b], 0));
    }
    return err;
}

int plan_enqueue(mars_search_plan* p, bool with_copies) {
    mars_ctx* ctx = p->ctx;
    const cudaStream_t st = ctx->stream;
    Scratch sc(st);
    if (with_copies)
        MARS_CUDA(cudaMemcpyAsync(p->d_plane, p->h_plane, (size_t)p->w * p->h,
                                  cudaMemcpyHostToDevice, st));
    MARS_CUDA(cudaMemsetAsync(ctx->d_counter, 0, sizeof(unsigned long long), st));
    const mars::FitParams fp = make_fit_params(p->params);
    if (p->method == MARS_METHOD_FISHER) {
        if (int e = run_jobs_fisher(ctx, sc, p->d_plane, p->w, p->h, fp, p->jobs, p->d_out,
                                    p->d_evals, p->d_rc))
            return e;
    } else if (all_levels_eligible(ctx, p->w, p->h, p->jobs)) {
        if (!p->ev_corr[0]) {
            MARS_CUDA(cudaEventCreate(&p->ev_corr[0]));
            MARS_CUDA(cudaEventCreate(&p->ev_corr[1]));
        }
        if (int e = run_jobs_all_levels(ctx, sc, p->d_plane, p->w, p->h, fp, p->jobs, p->d_out,
                                        p->d_rc, p->ev_corr))
            return e;
        p->corr_timed = true;
    } else if (int e = run_jobs_branched(ctx, sc, p->d_plane, p->w, p->h, fp, p->jobs, p->d_out,
                                         p->d_rc, 1)) {
        return e;
    }
    if (with_copies) {
        MARS_CUDA(cudaMemcpyAsync(p->h_out, p->d_out, p->total * sizeof(mars_candidate),
                                  cudaMemcpyDeviceToHost, st));
        if (p->method == MARS_METHOD_FISHER)
            MARS_CUDA(cudaMemcpyAsync(p->h_evals, p->d_evals, p->total * sizeof(uint64_t),
                                      cudaMemcpyDeviceToHost, st));
        MARS_CUDA(cudaMemcpyAsync(p->h_exact, ctx->d_counter, sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, st));
    }
    return MARS_OK;
}

int plan_capture(mars_search_plan* p, bool with_copies, cudaGraph_t* g, cudaGraphExec_t* x) {
    const cudaStream_t st = p->ctx->stream;
    MARS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const uint64_t l0 = p->ctx->launches.load();
    const int err = plan_enqueue(p, with_copies);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (err || ce != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return err ? err : fail(MARS_ECUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    }
    p->launches_per_run = p->ctx->launches.load() - l0;
    p->ctx->launches -= p->launches_per_run;  // captured, not launched
    const cudaError_t ie = cudaGraphInstantiate(x, graph, 0);
    if (ie != cudaSuccess) {
        cudaGraphDestroy(graph);
        return fail(MARS_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
    }
    *g = graph;
    return MARS_OK;
}

}  // namespace

extern "C" {

int mars_search_plan_create(mars_ctx* ctx, uint32_t width, uint32_t height,
                            const mars_params* params, mars_search_plan** out) {
    return mars_indexed_plan_create(ctx, width, height, params, MARS_METHOD_EXHAUSTIVE, out);
}

int mars_indexed_plan_create(mars_ctx* ctx, uint32_t width, uint32_t height,
                             const mars_params* params, int32_t method, mars_search_plan** out) {
    if (!ctx || !params || !out) return fail(MARS_EINVAL, "NULL argument");
    if (int e = check_params(params)) return e;
    if (method != MARS_METHOD_EXHAUSTIVE && method != MARS_METHOD_FISHER)
        return fail(MARS_EUNSUPPORTED, "unknown search method " + std::to_string(method));
    if (method == MARS_METHOD_FISHER && params->max_size > 64)
        return fail(MARS_EUNSUPPORTED, "the classified search supports block sizes up to 64");
    if (width == 0 || height == 0 || width > 65535 || height > 65535)
        return fail(MARS_EINVAL, "plane dimensions must be in 1..65535");
    std::unique_ptr<mars_search_plan, void (*)(mars_search_plan*)> p(new (std::nothrow)
                                                                         mars_search_plan,
                                                                     plan_release);
    if (!p) return fail(MARS_ENOMEM, "plan allocation failed");
    p->ctx = ctx;
    p->w = width;
    p->h = height;
    p->params = *params;
    p->method = method;
    p->jobs = plan_jobs(nullptr, width, height, *params, false);
    const std::vector<uint32_t> rc = job_origins(p->jobs, &p->total);
    if (p->total > 0xffffffffull) return fail(MARS_EINVAL, "too many quadtree nodes");
    auto index = std::make_shared<mars::NodeIndex>();
    p->evals.resize(p->total);
    size_t off = 0;
    for (const Job& j : p->jobs) {
        const uint64_t ev = level_evals(width, height, j.size, j.shift);
        index->add_job(j.size, j.shift, width, height, j.rows.data(), j.cols.data(), j.rows.size(),
                       (uint32_t)off);
        if (method == MARS_METHOD_EXHAUSTIVE)
            for (size_t i = 0; i < j.rows.size(); ++i) {
                p->evals[off + i] = ev;
                p->total_evals += ev;
            }
        off += j.rows.size();
    }
    p->index = index;
    std::lock_guard<std::mutex> lock(ctx->mu);
    MARS_CUDA(cudaSetDevice(ctx->device));
    MARS_CUDA(cudaMalloc(&p->d_rc, std::max<size_t>(1, rc.size()) * 4));
    MARS_CUDA(cudaMalloc(&p->d_plane, (size_t)width * height));
    MARS_CUDA(cudaMalloc(&p->d_out, std::max<size_t>(1, p->total) * sizeof(mars::CandidateOut)));
    MARS_CUDA(cudaMallocHost(&p->h_plane, (size_t)width * height));
    MARS_CUDA(cudaMallocHost(&p->h_out, std::max<size_t>(1, p->total) * sizeof(mars_candidate)));
    MARS_CUDA(cudaMallocHost(&p->h_exact, sizeof(unsigned long long)));
    if (method == MARS_METHOD_FISHER) {
        MARS_CUDA(cudaMalloc(&p->d_evals, std::max<size_t>(1, p->total) * sizeof(uint64_t)));
        MARS_CUDA(cudaMallocHost(&p->h_evals, std::max<size_t>(1, p->total) * sizeof(uint64_t)));
    }
    if (!rc.empty())
        MARS_CUDA(cudaMemcpyAsync(p->d_rc, rc.data(), rc.size() * 4, cudaMemcpyHostToDevice,
                                  ctx->stream));
    MARS_CUDA(cudaMemsetAsync(p->d_plane, 0, (size_t)width * height, ctx->stream));
    // One ordinary run first: it sets every kernel's attributes outside the capture and
    // checks the plan end to end.
    if (int e = plan_enqueue(p.get(), false)) return e;
    if (int e = sync_bounded(ctx)) return e;
    if (int e = plan_capture(p.get(), true, &p->g_host, &p->x_host)) return e;
    if (int e = plan_capture(p.get(), false, &p->g_dev, &p->x_dev)) return e;
    *out = p.release();
    return MARS_OK;
}

int mars_search_plan_run(mars_search_plan* p, const uint8_t* plane, mars_table** out) {
    if (!p || !plane || !out) return fail(MARS_EINVAL, "NULL argument");
    mars_ctx* ctx = p->ctx;
    std::unique_ptr<mars_table> t(new (std::nothrow) mars_table);
    if (!t) return fail(MARS_ENOMEM, "table allocation failed");
    std::lock_guard<std::mutex> lock(ctx->mu);
    MARS_CUDA(cudaSetDevice(ctx->device));
    std::memcpy(p->h_plane, plane, (size_t)p->w * p->h);
    MARS_CUDA(cudaGraphLaunch(p->x_host, ctx->stream));
    ctx->launches += p->launches_per_run;
    if (int e = sync_bounded(ctx)) return e;
    t->width = p->w;
    t->height = p->h;
    t->cands.assign(p->h_out, p->h_out + p->total);
    if (p->method == MARS_METHOD_FISHER) {
        p->evals.assign(p->h_evals, p->h_evals + p->total);
        p->total_evals = 0;
        for (uint64_t e : p->evals) p->total_evals += e;
    }
    t->evals = p->evals;
    t->total_evals = p->total_evals;
    t->exact_fits = *p->h_exact;
    t->shared_index = p->index;
    *out = t.release();
    return MARS_OK;
}

int mars_search_plan_run_device(mars_search_plan* p, const uint8_t* d_plane) {
    if (!p || !d_plane) return fail(MARS_EINVAL, "NULL argument");
    mars_ctx* ctx = p->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    MARS_CUDA(cudaSetDevice(ctx->device));
    if (d_plane != p->d_plane)
        MARS_CUDA(cudaMemcpyAsync(p->d_plane, d_plane, (size_t)p->w * p->h,
                                  cudaMemcpyDeviceToDevice, ctx->stream));
    MARS_CUDA(cudaGraphLaunch(p->x_dev, ctx->stream));
    ctx->launches += p->launches_per_run;
    return MARS_OK;
}

int mars_search_plan_table(mars_search_plan* p, mars_table** out) {
    if (!p || !out) return fail(MARS_EINVAL, "NULL argument");
    mars_ctx* ctx = p->ctx;
    std::unique_ptr<mars_table> t(new (std::nothrow) mars_table);
    if (!t) return fail(MARS_ENOMEM, "table allocation failed");
    std::lock_guard<std::mutex> lock(ctx->mu);
    MARS_CUDA(cudaSetDevice(ctx->device));
    MARS_CUDA(cudaMemcpyAsync(p->h_out, p->d_out, p->total * sizeof(mars_candidate),
                              cudaMemcpyDeviceToHost, ctx->stream));
    if (p->method == MARS_METHOD_FISHER)
        MARS_CUDA(cudaMemcpyAsync(p->h_evals, p->d_evals, p->total * sizeof(uint64_t),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    if (int e = sync_bounded(ctx)) return e;
    t->width = p->w;
    t->height = p->h;
    t->cands.assign(p->h_out, p->h_out + p->total);
    if (p->method == MARS_METHOD_FISHER) {
        p->evals.assign(p->h_evals, p->h_evals + p->total);
        p->total_evals = 0;
        for (uint64_t e : p->evals) p->total_evals += e;
    }
    t->evals = p->evals;
    t->total_evals = p->total_evals;
    t->shared_index = p->index;
    *out = t.release();
    return MARS_OK;
}

uint64_t mars_search_plan_evals(const mars_search_plan* p) { return p ? p->total_evals : 0; }
uint64_t mars_search_plan_launches(const mars_search_plan* p) { return p ? p->launches_per_run : 0; }

int mars_search_plan_kernel_ms(const mars_search_plan* p, float* ms) {
    if (!p || !ms) return fail(MARS_EINVAL, "NULL argument");
    if (!p->corr_timed)
        return fail(MARS_EUNSUPPORTED, "this plan has no all-levels correlation launch");
    MARS_CUDA(cudaSetDevice(p->ctx->device));
    if (cudaEventQuery(p->ev_corr[1]) != cudaSuccess)
        return fail(MARS_EINVAL, "no completed replay to time");
    MARS_CUDA(cudaEventElapsedTime(ms, p->ev_corr[0], p->ev_corr[1]));
    return MARS_OK;
}

void mars_search_plan_free(mars_search_plan* p) {
    if (!p) return;
    cudaSetDevice(p->ctx->device);
    cudaStreamSynchronize(p->ctx->stream);
    plan_release(p);
}

}  // extern "C"

namespace {

// The static tables of the walks on the device for one plan: its nodes with their children
// (TL, BL, TR, BR), the roots, evals, level offsets and DCT bases.  Returns false (and
// marks the plan) when the tree has nodes the plan does not search (pixel leaves at
// min_size 1 or at the edges of thin planes): those encodes keep the host walk.
int plan_walk_setup(mars_search_plan* p, bool* usable) {
    std::lock_guard<std::mutex> lock(p->walk_mu);
    if (p->walk_state) {
        *usable = p->walk_state > 0;
        return MARS_OK;
    }
    *usable = false;
    p->walk_state = -1;
    const mars_params& prm = p->params;
    if (prm.min_size < 2 || p->jobs.size() > 32 || p->total == 0) return MARS_OK;
    const mars_header hdr = mars::codec::build_header(p->w, p->h, prm);
    const auto& index = *p->index;
    mars::WalkPlan w{};
    std::vector<uint32_t> rows, cols;
    std::vector<uint64_t> levels_at;
    std::vector<double> basis;
    uint64_t lev = 0;
    for (const Job& j : p->jobs) {
        if (j.shift != prm.shift) return MARS_OK;
        w.first[w.nlevels] = (uint32_t)rows.size();
        w.count[w.nlevels] = (uint32_t)j.rows.size();
        w.size[w.nlevels] = j.size;
        ++w.nlevels;
        p->basis_at.push_back(basis.size());
        const std::vector<double>& b = mars::residual::basis(j.size);
        basis.insert(basis.end(), b.begin(), b.end());
        for (size_t i = 0; i < j.rows.size(); ++i) {
            rows.push_back(j.rows[i]);
            cols.push_back(j.cols[i]);
            levels_at.push_back(lev);
            lev += (uint64_t)j.size * j.size;
        }
    }
    for (uint32_t L = 1; L < w.nlevels; ++L)
        if (w.size[L] <= w.size[L - 1]) return MARS_OK;  // one level per size, ascending
    auto find = [&](uint32_t r, uint32_t c, uint32_t size) -> int64_t {
        return index.find(r, c, size, prm.shift);
    };
    std::vector<int32_t> child(4 * rows.size(), -1);
    for (uint32_t L = 0; L < w.nlevels; ++L) {
        const uint32_t size = w.size[L], half = size / 2;
        if (size <= prm.min_size) continue;
        for (uint32_t i = w.first[L]; i < w.first[L] + w.count[L]; ++i) {
            const uint32_t rs[4] = {rows[i], rows[i] + half, rows[i], rows[i] + half};
            const uint32_t cs[4] = {cols[i], cols[i], cols[i] + half, cols[i] + half};
            for (int q = 0; q < 4; ++q) {
                const int64_t c = find(rs[q], cs[q], half);
                if (c < 0) return MARS_OK;
                child[4 * (size_t)i + q] = (int32_t)c;
            }
        }
    }
    std::vector<int32_t> roots;
    for (const auto& r : mars::codec::quadtree_roots(hdr)) {
        const int64_t c = r[2] >= 2 ? find(r[0], r[1], r[2]) : -1;
        if (c < 0) return MARS_OK;
        roots.push_back((int32_t)c);
    }
    mars_ctx* ctx = p->ctx;
    MARS_CUDA(cudaSetDevice(ctx->device));
    auto up = [&](auto** dst, const auto& v) -> cudaError_t {
        using T = typename std::decay_t<decltype(v)>::value_type;
        cudaError_t e = cudaMalloc((void**)dst, std::max<size_t>(1, v.size()) * sizeof(T));
        if (e == cudaSuccess && !v.empty())
            e = cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
        return e;
    };
    MARS_CUDA(up(&p->d_wrows, rows));
    MARS_CUDA(up(&p->d_wcols, cols));
    MARS_CUDA(up(&p->d_child, child));
    MARS_CUDA(up(&p->d_roots, roots));
    MARS_CUDA(up(&p->d_wevals, p->evals));
    MARS_CUDA(up(&p->d_levels_at, levels_at));
    MARS_CUDA(up(&p->d_basis, basis));
    w.nodes = (uint32_t)rows.size();
    w.nroots = (uint32_t)roots.size();
    w.rows = p->d_wrows;
    w.cols = p->d_wcols;
    w.child = p->d_child;
    w.roots = p->d_roots;
    w.evals = p->d_wevals;
    w.levels_at = p->d_levels_at;
    w.stride = p->w;
    p->walk = w;
    p->nlevels_total = lev;
    p->walk_state = 1;
    *usable = true;
    return MARS_OK;
}

// MARS_PLAN_WALK=host keeps planned encodes on the host walk over a downloaded table.
bool plan_walk_on_host() {
    static const bool on = [] {
        const char* e = std::getenv("MARS_PLAN_WALK");
        return e && std::string(e) == "host";
    }();
    return on;
}

template <class T>
int copy_out_array(const std::vector<T>& v, T** out, size_t* n) {
    *n = v.size();
    *out = (T*)std::malloc(std::max<size_t>(1, v.size()) * sizeof(T));
    if (!*out) return fail(MARS_ENOMEM, "output allocation failed");
    if (!v.empty()) std::memcpy(*out, v.data(), v.size() * sizeof(T));
    return MARS_OK;
}

// A planned encode with both walks on the device: the plan's search, then the warm-up walk
// over its candidates, the rate snapshot on the host from the warm-up leaves, the pricing of
// every node and the RD walk's decisions -- the host receives only leaves.
int plan_encode_device(mars_search_plan* plan, const uint8_t* plane, const mars_options* o,
                       mars_header* header, mars_leaf** leaves, size_t* nleaves,
                       int32_t** residuals, size_t* nresiduals, mars_counters* counters) {
    mars_ctx* ctx = plan->ctx;
    const mars_params& prm = plan->params;
    mars_header hdr;
    if (mars::codec::encode_header(plan->w, plan->h, prm, *o, &hdr))
        return fail(MARS_EINVAL, "residual qstep out of range");
    const mars::WalkPlan& w = plan->walk;
    const size_t nodes = w.nodes;
    MARS_CUDA(cudaSetDevice(ctx->device));
    OwnStream own;
    MARS_CUDA(cudaStreamCreateWithFlags(&own.st, cudaStreamNonBlocking));
    const cudaStream_t st = own.st;
    Scratch sc(st);
    unsigned char* d_cands;
    uint8_t* d_px;
    mars::WalkScratch ws{};
    mars_leaf *d_warm, *d_leaves;
    MARS_CUDA(sc.get(&d_cands, nodes * sizeof(mars_candidate)));
    MARS_CUDA(sc.get(&d_px, (size_t)plan->w * plan->h));
    MARS_CUDA(sc.get(&ws.split, nodes));
    MARS_CUDA(sc.get(&ws.cnt, nodes));
    MARS_CUDA(sc.get(&ws.ev, nodes));
    MARS_CUDA(sc.get(&ws.ofs, nodes));
    MARS_CUDA(sc.get(&ws.rofs, nodes));
    MARS_CUDA(sc.get(&ws.rd, nodes));
    MARS_CUDA(sc.get(&ws.rr, nodes));
    MARS_CUDA(sc.get(&ws.totals, 2));
    MARS_CUDA(sc.get(&d_warm, nodes));
    MARS_CUDA(sc.get(&d_leaves, nodes));
    cudaEvent_t ev_alloc, ev_search;
    MARS_CUDA(cudaEventCreateWithFlags(&ev_alloc, cudaEventDisableTiming));
    MARS_CUDA(cudaEventCreateWithFlags(&ev_search, cudaEventDisableTiming));
    struct Events {
        cudaEvent_t a, b;
        ~Events() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } evs{ev_alloc, ev_search};
    MARS_CUDA(cudaEventRecord(ev_alloc, st));
    {
        // The search on the plan's buffers, then this call's copies of its candidates and
        // plane, in the context's stream order (the next run of the plan queues behind them).
        std::lock_guard<std::mutex> lock(ctx->mu);
        MARS_CUDA(cudaStreamWaitEvent(ctx->stream, ev_alloc, 0));
        MARS_CUDA(cudaMemcpyAsync(plan->d_plane, plane, (size_t)plan->w * plan->h,
                                  cudaMemcpyHostToDevice, ctx->stream));
        MARS_CUDA(cudaGraphLaunch(plan->x_dev, ctx->stream));
        ctx->launches += plan->launches_per_run;
        MARS_CUDA(cudaMemcpyAsync(d_cands, plan->d_out, nodes * sizeof(mars_candidate),
                                  cudaMemcpyDeviceToDevice, ctx->stream));
        MARS_CUDA(cudaMemcpyAsync(d_px, plan->d_plane, (size_t)plan->w * plan->h,
                                  cudaMemcpyDeviceToDevice, ctx->stream));
        MARS_CUDA(cudaEventRecord(ev_search, ctx->stream));
    }
    MARS_CUDA(cudaStreamWaitEvent(st, ev_search, 0));
    mars::WalkPlan wp = w;
    wp.px = d_px;
    // The warm-up walk (t_rms = 8 for the rate snapshot; the plain walk itself without RD).
    const double t_rms = prm.has_lambda ? 8.0 : prm.t_rms;
    MARS_CUDA(mars::launch_warm_walk(wp, d_cands, sizeof(mars_candidate), t_rms, prm.min_size,
                                     prm.zero_threshold, hdr.bits_beta, ws, d_warm, st));
    ctx->launches += 2 * w.nlevels + 1;
    unsigned long long tot[2];
    MARS_CUDA(cudaMemcpyAsync(tot, ws.totals, sizeof tot, cudaMemcpyDeviceToHost, st));
    if (int e = sync_bounded(ctx, st)) return e;
    std::vector<mars_leaf> warm(tot[0]);
    MARS_CUDA(cudaMemcpyAsync(warm.data(), d_warm, warm.size() * sizeof(mars_leaf),
                              cudaMemcpyDeviceToHost, st));
    if (int e = sync_bounded(ctx, st)) return e;
    const uint64_t warm_evals = tot[1];
    *header = hdr;
    if (!prm.has_lambda) {
        counters->search_evals = warm_evals;
        counters->warmup_evals = 0;
        if (int e = copy_out_array(warm, leaves, nleaves)) return e;
        return copy_out_array(std::vector<int32_t>(), residuals, nresiduals);
    }
    // The rate snapshot from the warm-up leaves, then every node priced and the RD walk.
    std::vector<double> bits;
    std::vector<int64_t> off;
    if (mars::codec::rate_table_from_warmup(hdr, warm, prm.max_size, &bits, &off))
        return fail(MARS_EINVAL, "rate snapshot of the warm-up leaves failed");
    double split0[32] = {0}, split1[32] = {0};
    for (uint32_t L = 0; L < w.nlevels; ++L) {
        const uint32_t c = (uint32_t)__builtin_ctz(w.size[L]);
        const int64_t at = off[(size_t)mars::price::F_SPLIT * mars::price::kCtx + c];
        if (at < 0) return fail(MARS_EINVAL, "rate table misses a split context");
        split0[c] = bits[at];
        split1[c] = bits[at + 1];
    }
    const uint8_t allowed[4] = {o->allowed_modes[0], o->allowed_modes[1], o->allowed_modes[2],
                                o->allowed_modes[3]};
    const mars::price::Setup setup = mars::codec::price_setup(hdr, prm, allowed, prm.lambda);
    double* d_bits;
    int64_t* d_off;
    mars::price::Priced* d_priced;
    int8_t* d_lev;
    int32_t* d_res;
    const bool residual = allowed[3] != 0;
    MARS_CUDA(sc.get(&d_bits, bits.size()));
    MARS_CUDA(sc.get(&d_off, off.size()));
    MARS_CUDA(sc.get(&d_priced, nodes));
    MARS_CUDA(sc.get(&d_lev, residual ? plan->nlevels_total : 1));
    MARS_CUDA(sc.get(&d_res, residual ? plan->nlevels_total : 1));
    MARS_CUDA(cudaMemcpyAsync(d_bits, bits.data(), bits.size() * sizeof(double),
                              cudaMemcpyHostToDevice, st));
    MARS_CUDA(cudaMemcpyAsync(d_off, off.data(), off.size() * sizeof(int64_t),
                              cudaMemcpyHostToDevice, st));
    for (uint32_t L = w.nlevels; L-- > 0;) {  // largest nodes first
        mars::PriceLaunch a{};
        a.px = d_px;
        a.stride = plan->w;
        a.size = w.size[L];
        a.count = w.count[L];
        a.rows = plan->d_wrows + w.first[L];
        a.cols = plan->d_wcols + w.first[L];
        a.cands = d_cands + (size_t)w.first[L] * sizeof(mars_candidate);
        a.cand_stride = sizeof(mars_candidate);
        a.k = 1;
        a.setup = setup;
        a.table = {d_bits, d_off};
        a.basis = plan->d_basis + plan->basis_at[L];
        a.out = d_priced + w.first[L];
        a.levels = d_lev;
        a.levels_at = plan->d_levels_at + w.first[L];
        const size_t gbytes = mars::price_scratch_bytes(a.size, a.count, &a.scratch_slots);
        if (gbytes) MARS_CUDA(sc.get(&a.global_scratch, gbytes));
        MARS_CUDA(mars::launch_price_nodes(a, st));
        ctx->launches += 1;
    }
    MARS_CUDA(mars::launch_rd_walk(wp, d_priced, d_lev, prm.lambda * 1.0, split0, split1,
                                   prm.min_size, ws, d_leaves, d_res, st));
    ctx->launches += 2 * w.nlevels + 1;
    MARS_CUDA(cudaMemcpyAsync(tot, ws.totals, sizeof tot, cudaMemcpyDeviceToHost, st));
    if (int e = sync_bounded(ctx, st)) return e;
    std::vector<mars_leaf> out(tot[0]);
    std::vector<int32_t> res(tot[1]);
    MARS_CUDA(cudaMemcpyAsync(out.data(), d_leaves, out.size() * sizeof(mars_leaf),
                              cudaMemcpyDeviceToHost, st));
    if (!res.empty())
        MARS_CUDA(cudaMemcpyAsync(res.data(), d_res, res.size() * sizeof(int32_t),
                                  cudaMemcpyDeviceToHost, st));
    if (int e = sync_bounded(ctx, st)) return e;
    counters->search_evals = plan->total_evals;
    counters->warmup_evals = warm_evals;
    if (int e = copy_out_array(out, leaves, nleaves)) return e;
    if (int e = copy_out_array(res, residuals, nresiduals)) {
        std::free(*leaves);
        *leaves = nullptr;
        return e;
    }
    return MARS_OK;
}

}  // namespace

extern "C" {

int mars_encode_planned(mars_search_plan* plan, const uint8_t* plane,
                        const mars_options* options, mars_header* header, mars_leaf** leaves,
                        size_t* nleaves, int32_t** residuals, size_t* nresiduals,
                        mars_counters* counters) {
    if (!plan || !plane || !options || !header || !leaves || !nleaves || !residuals ||
        !nresiduals || !counters)
        return fail(MARS_EINVAL, "NULL argument");
    if (plan->method != MARS_METHOD_EXHAUSTIVE || options->method != MARS_METHOD_EXHAUSTIVE ||
        std::max<uint32_t>(1, options->rd_candidates) > 1 ||
        (plan->params.has_lambda && options->adaptive_density))
        return fail(MARS_EUNSUPPORTED, "a search plan serves exhaustive single-winner encodes "
                                       "without adaptive density");
    if (!options->residual_adaptive && options->residual_qstep != 0.0f &&
        !(std::isfinite(options->residual_qstep) && options->residual_qstep >= 1.0f &&
          options->residual_qstep <= 65535.0f))
        return fail(MARS_EINVAL, "residual qstep must be finite and in [1, 65535]");
    bool device_walk = false;
    if (!plan_walk_on_host())
        if (int e = plan_walk_setup(plan, &device_walk)) return e;
    if (device_walk)
        return plan_encode_device(plan, plane, options, header, leaves, nleaves, residuals,
                                  nresiduals, counters);
    mars_table* table = nullptr;
    if (int e = mars_search_plan_run(plan, plane, &table)) return e;
    std::unique_ptr<mars_table, void (*)(mars_table*)> guard(table, mars_search_table_free);
    return encode_on_tables(plan->ctx, plane, plan->w, plan->h, &plan->params, options, table, table, 1,
                            header, leaves, nleaves, residuals, nresiduals, counters);
}


void mars_leaves_free(mars_leaf* leaves) { std::free(leaves); }
void mars_residuals_free(int32_t* residuals) { std::free(residuals); }
void mars_bytes_free(uint8_t* bytes) { std::free(bytes); }

}  // extern "C"

namespace {

// Leaf table and owner map of one leaf list, validated on the host so that every read and
// write the gather kernel makes stays inside the plane.  Leaves are packed into 16 bytes
// (the layout is documented beside DecodeLeaf), which bounds plane sides to 65535, leaf
// sizes to 4095 and qalfa to 2^bits_alfa, qbeta to 2^bits_beta - 1 -- the ranges every
// .ifs stream and every encoder output lie in.  The owner map's cell is the largest power
// of two dividing every leaf's row, column and size (4 for the usual quadtree with
// min_size 4), capped at 32; later leaves overwrite earlier ones, as in the reference.
// Mode-3 residuals are rebuilt here on the host exactly as decode_leaf does
// (ifs.rs:441-456) -- the inverse DCT uses the C library's cosine, as the reference's
// does -- in domain-local (u, v) order, and their offsets are returned per leaf.
int prepare_decode(const mars_header* hdr, const mars_leaf* leaves, size_t n,
                   const int32_t* residuals, size_t nresiduals, std::vector<mars::DecodeLeaf>* dl,
                   std::vector<int32_t>* owner, int* lg_out, mars::DecodeConsts* consts,
                   std::vector<int32_t>* resid_off, std::vector<double>* resid_values) {
    const uint32_t w = hdr->width, h = hdr->height;
    if (w == 0 || h == 0) return fail(MARS_EINVAL, "empty plane");
    if (w > 65535 || h > 65535) return fail(MARS_EINVAL, "plane sides must be at most 65535");
    if (hdr->bits_alfa > 16 || hdr->bits_beta < 1 || hdr->bits_beta > 16)
        return fail(MARS_EINVAL, "header bit widths out of range");
    dl->assign(n, mars::DecodeLeaf{});
    uint32_t align_bits = 32u;
    const uint32_t qalfa_max = 1u << hdr->bits_alfa, qbeta_max = (1u << hdr->bits_beta) - 1;
    for (size_t k = 0; k < n; ++k) {
        const mars_leaf& L = leaves[k];
        if (L.size == 0 || L.row + L.size > h || L.col + L.size > w || L.isometry > 7)
            return fail(MARS_EINVAL, "leaf " + std::to_string(k) + " lies outside the plane");
        if (L.size > 4095)
            return fail(MARS_EUNSUPPORTED, "leaf " + std::to_string(k) + " is wider than 4095");
        if (L.mode > 3) return fail(MARS_EINVAL, "leaf " + std::to_string(k) + " has mode > 3");
        if (L.qbeta > qbeta_max || (L.mode != 1 && L.qalfa > qalfa_max))
            return fail(MARS_EINVAL, "leaf " + std::to_string(k) +
                                         " has coefficients wider than the header's bits");
        if (L.mode != 1 && L.qalfa != 0 &&
            (L.dom_row + 2 * L.size > h || L.dom_col + 2 * L.size > w))
            return fail(MARS_EINVAL, "leaf " + std::to_string(k) + " domain runs past the plane");
        align_bits |= L.row | L.col | L.size;
        mars::DecodeLeaf& d = (*dl)[k];
        d.x = L.row | (L.col << 16);
        d.y = L.size | (L.mode << 12) | (L.qbeta << 16);
        if (L.mode == 1) {
            d.z = (uint32_t)L.qgx;
            d.w = (uint32_t)L.qgy;
        } else {
            d.z = L.dom_row | (L.dom_col << 16);
            d.w = L.qalfa | (L.isometry << 24);
        }
    }
    consts->max_alfa = (double)hdr->int_max_alfa / 256.0 * 8.0;
    consts->alfa_den = (double)qalfa_max;
    consts->beta_den = (double)qbeta_max;
    std::vector<int64_t> offs;
    if (!mars::codec::residual_offsets(leaves, n, nresiduals, &offs) || (nresiduals && !residuals))
        return fail(MARS_EINVAL, "the residual pool does not hold size*size levels per mode-3 leaf");
    resid_off->clear();
    resid_values->clear();
    if (nresiduals) {
        if (nresiduals > 0x7fffffffull) return fail(MARS_EINVAL, "residual pool too large");
        resid_off->assign(n, -1);
        const double step = mars::codec::qstep_of(*hdr);
        for (size_t k = 0; k < n; ++k) {
            if (offs[k] < 0) continue;
            (*resid_off)[k] = (int32_t)resid_values->size();
            const std::vector<double> v =
                mars::residual::values(residuals + offs[k], leaves[k].size, step);
            resid_values->insert(resid_values->end(), v.begin(), v.end());
        }
    }
    const int lg = __builtin_ctz(align_bits);
    const uint32_t cell = 1u << lg;
    const uint32_t mw = (w + cell - 1) >> lg, mh = (h + cell - 1) >> lg;
    owner->assign((size_t)mw * mh, -1);
    for (size_t k = 0; k < n; ++k) {
        const mars_leaf& L = leaves[k];
        for (uint32_t i = 0; i < (L.size >> lg); ++i)
            std::fill_n(owner->begin() + (long)((size_t)((L.row >> lg) + i) * mw + (L.col >> lg)),
                        L.size >> lg, (int32_t)k);
    }
    *lg_out = lg;
    return MARS_OK;
}

}  // namespace

struct mars_decode_plan {
    mars_ctx* ctx = nullptr;
    uint32_t w = 0, h = 0;
    int lg = 0;
    size_t nleaves = 0;
    int32_t* d_owner = nullptr;
    mars::DecodeMap* d_maps = nullptr;
    double* d_rvals = nullptr;  // mode-3 residual values, or null
    uint8_t* d_tmp = nullptr;   // ping-pong partner of the caller's output buffer
    // Source-ordered steps (planes larger than L2; decode.cu): the domain cells' jobs in
    // source-row order, each 4x4 cell's job slot, and the per-cell output buffer.
    mars::DecodeConsts consts{};
    uint4* d_jobs = nullptr;
    uint32_t* d_inv = nullptr;
    uint4* d_cellbuf = nullptr;
    uint32_t njobs = 0;
};

namespace {
// Whether a decode plan of a w x h plane takes the source-ordered steps: by default when
// the two ping-pong planes exceed 96 MB (they no longer stay in L2 between steps);
// MARS_DECODE_SORTED=1 / 0 forces it on (where eligible) / off.
bool want_sorted_decode(uint32_t w, uint32_t h) {
    const char* e = std::getenv("MARS_DECODE_SORTED");
    if (e && *e) return std::string(e) != "0";
    return 2ull * w * h > (96ull << 20);
}
}  // namespace

extern "C" {

int mars_decode(mars_ctx* ctx, const mars_header* hdr, const mars_leaf* leaves, size_t n,
                const int32_t* residuals, size_t nresiduals, uint32_t iterations, uint8_t* out) {
    if (!ctx || !hdr || !out || (n && !leaves)) return fail(MARS_EINVAL, "NULL argument");
    std::vector<mars::DecodeLeaf> dl;
    std::vector<int32_t> owner, roff;
    std::vector<double> rvals;
    int lg = 0;
    mars::DecodeConsts consts;
    if (int e = prepare_decode(hdr, leaves, n, residuals, nresiduals, &dl, &owner, &lg, &consts,
                               &roff, &rvals))
        return e;
    const uint32_t w = hdr->width, h = hdr->height;
    std::lock_guard<std::mutex> lock(ctx->mu);
    MARS_CUDA(cudaSetDevice(ctx->device));
    Scratch sc(ctx->stream);
    uint8_t *a = nullptr, *b = nullptr;
    int32_t* d_owner = nullptr;
    mars::DecodeLeaf* d_leaves = nullptr;
    mars::DecodeMap* d_maps = nullptr;
    int32_t* d_roff = nullptr;
    double* d_rvals = nullptr;
    const size_t px = (size_t)w * h;
    MARS_CUDA(sc.get(&a, px));
    MARS_CUDA(sc.get(&b, px));
    MARS_CUDA(sc.get(&d_owner, owner.size()));
    MARS_CUDA(sc.get(&d_leaves, n));
    MARS_CUDA(sc.get(&d_maps, n));
    MARS_CUDA(cudaMemcpyAsync(d_owner, owner.data(), owner.size() * 4, cudaMemcpyHostToDevice,
                              ctx->stream));
    if (!rvals.empty()) {
        MARS_CUDA(sc.get(&d_roff, n));
        MARS_CUDA(sc.get(&d_rvals, rvals.size()));
        MARS_CUDA(cudaMemcpyAsync(d_roff, roff.data(), n * 4, cudaMemcpyHostToDevice, ctx->stream));
        MARS_CUDA(cudaMemcpyAsync(d_rvals, rvals.data(), rvals.size() * 8, cudaMemcpyHostToDevice,
                                  ctx->stream));
    }
    if (n) {
        MARS_CUDA(cudaMemcpyAsync(d_leaves, dl.data(), n * sizeof(mars::DecodeLeaf),
                                  cudaMemcpyHostToDevice, ctx->stream));
        MARS_CUDA(mars::launch_decode_expand(d_leaves, d_roff, (int)n, consts, d_maps,
                                             ctx->stream));
        ctx->launches += 1;
    }
    MARS_CUDA(cudaMemsetAsync(a, 128, px, ctx->stream));
    for (uint32_t it = 0; it < iterations; ++it) {
        MARS_CUDA(mars::launch_decode_step(a, b, (int)w, (int)h, lg, d_owner, d_maps, d_rvals,
                                           ctx->stream));
        ctx->launches += 1;
        std::swap(a, b);
    }
    MARS_CUDA(cudaMemcpyAsync(out, a, px, cudaMemcpyDeviceToHost, ctx->stream));
    return sync_bounded(ctx);
}

int mars_decode_plan_create(mars_ctx* ctx, const mars_header* hdr, const mars_leaf* leaves,
                            size_t n, const int32_t* residuals, size_t nresiduals,
                            mars_decode_plan** out) {
    if (!ctx || !hdr || !out || (n && !leaves)) return fail(MARS_EINVAL, "NULL argument");
    std::vector<mars::DecodeLeaf> dl;
    std::vector<int32_t> owner, roff;
    std::vector<double> rvals;
    int lg = 0;
    mars::DecodeConsts consts;
    if (int e = prepare_decode(hdr, leaves, n, residuals, nresiduals, &dl, &owner, &lg, &consts,
                               &roff, &rvals))
        return e;
    std::lock_guard<std::mutex> lock(ctx->mu);
    MARS_CUDA(cudaSetDevice(ctx->device));
    auto* p = new (std::nothrow) mars_decode_plan;
    if (!p) return fail(MARS_ENOMEM, "plan allocation failed");
    p->ctx = ctx;
    p->w = hdr->width;
    p->h = hdr->height;
    p->lg = lg;
    p->nleaves = n;
    mars::DecodeLeaf* d_leaves = nullptr;
    int32_t* d_roff = nullptr;
    cudaError_t e = cudaMalloc(&p->d_owner, std::max<size_t>(1, owner.size()) * 4);
    if (e == cudaSuccess) e = cudaMalloc(&d_leaves, std::max<size_t>(1, n) * sizeof(mars::DecodeLeaf));
    if (e == cudaSuccess) e = cudaMalloc(&p->d_maps, std::max<size_t>(1, n) * sizeof(mars::DecodeMap));
    if (e == cudaSuccess) e = cudaMalloc(&p->d_tmp, (size_t)p->w * p->h);
    if (e == cudaSuccess && !rvals.empty()) {
        e = cudaMalloc(&d_roff, n * 4);
        if (e == cudaSuccess) e = cudaMalloc(&p->d_rvals, rvals.size() * 8);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_roff, roff.data(), n * 4, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(p->d_rvals, rvals.data(), rvals.size() * 8, cudaMemcpyHostToDevice,
                                ctx->stream);
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p->d_owner, owner.data(), owner.size() * 4, cudaMemcpyHostToDevice,
                            ctx->stream);
    if (e == cudaSuccess && n)
        e = cudaMemcpyAsync(d_leaves, dl.data(), n * sizeof(mars::DecodeLeaf),
                            cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && n) {
        e = mars::launch_decode_expand(d_leaves, d_roff, (int)n, consts, p->d_maps, ctx->stream);
        ctx->launches += 1;
    }
    p->consts = consts;
    uint32_t *d_key = nullptr, *d_rows = nullptr, *d_cursor = nullptr;
    if (e == cudaSuccess && n && want_sorted_decode(p->w, p->h) &&
        mars::decode_sorted_eligible((int)p->w, (int)p->h, lg, !rvals.empty())) {
        const size_t cells = mars::decode_sorted_cells((int)p->w, (int)p->h);
        e = cudaMalloc(&d_key, cells * 4);
        if (e == cudaSuccess) e = cudaMalloc(&d_rows, (size_t)p->h * 4);
        if (e == cudaSuccess) e = cudaMalloc(&d_cursor, ((size_t)p->h + 1) * 4);
        if (e == cudaSuccess) e = cudaMalloc(&p->d_jobs, cells * sizeof(uint4));
        if (e == cudaSuccess) e = cudaMalloc(&p->d_inv, cells * 4);
        if (e == cudaSuccess) e = cudaMalloc(&p->d_cellbuf, cells * sizeof(uint4));
        if (e == cudaSuccess)
            e = mars::launch_decode_sorted_build((int)p->w, (int)p->h, lg, p->d_owner, p->d_maps,
                                                 d_leaves, d_key, d_rows, d_cursor, p->d_jobs,
                                                 p->d_inv, ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&p->njobs, d_cursor + p->h, 4, cudaMemcpyDeviceToHost, ctx->stream);
        ctx->launches += 3;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d_leaves);
    cudaFree(d_roff);
    cudaFree(d_key);
    cudaFree(d_rows);
    cudaFree(d_cursor);
    if (e != cudaSuccess) {
        cudaFree(p->d_owner);
        cudaFree(p->d_maps);
        cudaFree(p->d_rvals);
        cudaFree(p->d_tmp);
        cudaFree(p->d_jobs);
        cudaFree(p->d_inv);
        cudaFree(p->d_cellbuf);
        delete p;
        return fail(MARS_ECUDA, std::string("decode plan: ") + cudaGetErrorString(e));
    }
    *out = p;
    return MARS_OK;
}

int mars_decode_plan_run(mars_decode_plan* p, uint32_t iterations, uint8_t* d_out) {
    if (!p || !d_out) return fail(MARS_EINVAL, "NULL argument");
    mars_ctx* ctx = p->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    MARS_CUDA(cudaSetDevice(ctx->device));
    // Ping-pong so that the last iteration lands in d_out.
    uint8_t* a = (iterations & 1) ? p->d_tmp : d_out;
    uint8_t* b = (iterations & 1) ? d_out : p->d_tmp;
    MARS_CUDA(cudaMemsetAsync(a, 128, (size_t)p->w * p->h, ctx->stream));
    for (uint32_t it = 0; it < iterations; ++it) {
        if (p->d_jobs) {
            MARS_CUDA(mars::launch_decode_sorted_step(a, b, (int)p->w, (int)p->h, p->lg, p->d_owner,
                                                      p->d_maps, p->d_jobs, p->njobs, p->d_inv,
                                                      p->consts, p->d_cellbuf, ctx->stream));
            ctx->launches += 2;
        } else {
            MARS_CUDA(mars::launch_decode_step(a, b, (int)p->w, (int)p->h, p->lg, p->d_owner,
                                               p->d_maps, p->d_rvals, ctx->stream));
            ctx->launches += 1;
        }
        std::swap(a, b);
    }
    return MARS_OK;
}

int mars_decode_plan_run_until_stable(mars_decode_plan* p, uint8_t threshold,
                                      uint32_t max_iterations, uint8_t* d_out,
                                      uint32_t* iterations_used) {
    if (!p || !d_out || !iterations_used) return fail(MARS_EINVAL, "NULL argument");
    const uint32_t iters = std::max<uint32_t>(1, max_iterations);
    if (iters > (1u << 20)) return fail(MARS_EINVAL, "max_iterations is above 2^20");
    mars_ctx* ctx = p->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    MARS_CUDA(cudaSetDevice(ctx->device));
    const size_t px = (size_t)p->w * p->h;
    Scratch sc(ctx->stream);
    int* d_state = nullptr;  // [0] done, [1] used, [2 + i] step i's max delta
    MARS_CUDA(sc.get(&d_state, 2 + (size_t)iters));
    MARS_CUDA(cudaMemsetAsync(d_state, 0, (2 + (size_t)iters) * sizeof(int), ctx->stream));
    // Step i reads buf[i % 2] and writes buf[(i + 1) % 2]; the decode that stopped after
    // `used` steps ends in buf[used % 2].
    uint8_t* buf[2] = {d_out, p->d_tmp};
    MARS_CUDA(cudaMemsetAsync(buf[0], 128, px, ctx->stream));
    for (uint32_t it = 0; it < iters; ++it) {
        MARS_CUDA(mars::launch_decode_step_stable(buf[it & 1], buf[(it + 1) & 1], (int)p->w,
                                                  (int)p->h, p->lg, p->d_owner, p->d_maps,
                                                  p->d_rvals, d_state, d_state + 2 + it,
                                                  (int)threshold, (int)it, d_state, d_state + 1,
                                                  ctx->stream));
        ctx->launches += 2;
    }
    int state[2] = {0, 0};
    MARS_CUDA(cudaMemcpyAsync(state, d_state, sizeof state, cudaMemcpyDeviceToHost, ctx->stream));
    if (int e = sync_bounded(ctx)) return e;
    const uint32_t used = state[0] ? (uint32_t)state[1] : iters;
    if (used & 1)
        MARS_CUDA(cudaMemcpyAsync(d_out, p->d_tmp, px, cudaMemcpyDeviceToDevice, ctx->stream));
    *iterations_used = used;
    return MARS_OK;
}

int mars_decode_until_stable(mars_ctx* ctx, const mars_header* hdr, const mars_leaf* leaves,
                             size_t n, const int32_t* residuals, size_t nresiduals,
                             uint8_t threshold, uint32_t max_iterations, uint8_t* out,
                             uint32_t* iterations_used) {
    if (!ctx || !hdr || !out || !iterations_used) return fail(MARS_EINVAL, "NULL argument");
    mars_decode_plan* plan = nullptr;
    if (int e = mars_decode_plan_create(ctx, hdr, leaves, n, residuals, nresiduals, &plan))
        return e;
    std::unique_ptr<mars_decode_plan, void (*)(mars_decode_plan*)> guard(plan,
                                                                         mars_decode_plan_free);
    uint8_t* d_out = nullptr;
    {
        std::lock_guard<std::mutex> lock(ctx->mu);
        MARS_CUDA(cudaSetDevice(ctx->device));
        MARS_CUDA(cudaMalloc(&d_out, std::max<size_t>(1, (size_t)hdr->width * hdr->height)));
    }
    std::unique_ptr<uint8_t, cudaError_t (*)(void*)> dguard(d_out, cudaFree);
    if (int e = mars_decode_plan_run_until_stable(plan, threshold, max_iterations, d_out,
                                                  iterations_used))
        return e;
    std::lock_guard<std::mutex> lock(ctx->mu);
    MARS_CUDA(cudaMemcpyAsync(out, d_out, (size_t)hdr->width * hdr->height,
                              cudaMemcpyDeviceToHost, ctx->stream));
    return sync_bounded(ctx);
}

// `(x * factor).round() as u32`: f64::round (half away from zero), then Rust's saturating
// cast (NaN and negatives to 0).
static uint32_t zoom_scale(uint32_t v, double factor) {
    const double r = std::round((double)v * factor);
    if (!(r > 0.0)) return 0;
    if (r >= 4294967295.0) return 0xffffffffu;
    return (uint32_t)r;
}
static int32_t zoom_grad(int32_t g, double factor) {
    const double r = std::round((double)g / factor);
    if (std::isnan(r)) return 0;
    if (r >= 2147483647.0) return INT32_MAX;
    if (r <= -2147483648.0) return INT32_MIN;
    return (int32_t)r;
}

int mars_zoom_leaves(const mars_header* hdr, const mars_leaf* leaves, size_t n, double factor,
                     mars_header* out_hdr, mars_leaf* out_leaves) {
    if (!hdr || !out_hdr || (n && (!leaves || !out_leaves)))
        return fail(MARS_EINVAL, "NULL argument");
    if (!std::isfinite(factor) || factor <= 0.0)
        return fail(MARS_EINVAL, "the zoom factor must be finite and positive");
    for (size_t k = 0; k < n; ++k) {
        mars_leaf L = leaves[k];
        L.row = zoom_scale(L.row, factor);
        L.col = zoom_scale(L.col, factor);
        L.size = std::max<uint32_t>(zoom_scale(L.size, factor), 1);
        L.dom_row = zoom_scale(L.dom_row, factor);
        L.dom_col = zoom_scale(L.dom_col, factor);
        L.qgx = zoom_grad(L.qgx, factor);
        L.qgy = zoom_grad(L.qgy, factor);
        // The residual is dropped at any factor but 1; a mode-3 leaf without one decodes by
        // mode 2's formula (ifs.rs:441-456), and in this ABI every mode-3 leaf carries its
        // levels in the residual pool, so the zoomed leaf comes back as mode 2.
        if (factor != 1.0 && L.mode == 3) L.mode = 2;
        out_leaves[k] = L;
    }
    *out_hdr = *hdr;
    out_hdr->width = zoom_scale(hdr->width, factor);
    out_hdr->height = zoom_scale(hdr->height, factor);
    return MARS_OK;
}

void mars_decode_plan_free(mars_decode_plan* p) {
    if (!p) return;
    cudaSetDevice(p->ctx->device);
    cudaStreamSynchronize(p->ctx->stream);
    cudaFree(p->d_owner);
    cudaFree(p->d_maps);
    cudaFree(p->d_rvals);
    cudaFree(p->d_tmp);
    cudaFree(p->d_jobs);
    cudaFree(p->d_inv);
    cudaFree(p->d_cellbuf);
    delete p;
}

int mars_ycbcr_device(mars_ctx* ctx, const uint8_t* d_r, const uint8_t* d_g, const uint8_t* d_b,
                      size_t n, uint8_t* d_y, uint8_t* d_cb, uint8_t* d_cr) {
    if (!ctx || (n && (!d_r || !d_g || !d_b || !d_y || !d_cb || !d_cr)))
        return fail(MARS_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    MARS_CUDA(cudaSetDevice(ctx->device));
    MARS_CUDA(mars::launch_ycbcr(d_r, d_g, d_b, n, d_y, d_cb, d_cr, false, ctx->stream));
    ctx->launches += n ? 1 : 0;
    return MARS_OK;
}

int mars_rgb_from_ycbcr_device(mars_ctx* ctx, const uint8_t* d_y, const uint8_t* d_cb,
                               const uint8_t* d_cr, size_t n, uint8_t* d_r, uint8_t* d_g,
                               uint8_t* d_b) {
    if (!ctx || (n && (!d_r || !d_g || !d_b || !d_y || !d_cb || !d_cr)))
        return fail(MARS_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    MARS_CUDA(cudaSetDevice(ctx->device));
    MARS_CUDA(mars::launch_ycbcr(d_y, d_cb, d_cr, n, d_r, d_g, d_b, true, ctx->stream));
    ctx->launches += n ? 1 : 0;
    return MARS_OK;
}

int mars_downsample_box_device(mars_ctx* ctx, const uint8_t* d_src, uint32_t width,
                               uint32_t height, uint8_t* d_dst) {
    if (!ctx || !d_src || !d_dst) return fail(MARS_EINVAL, "NULL argument");
    if (width == 0 || height == 0 || width > 65535 || height > 65535)
        return fail(MARS_EINVAL, "plane dimensions must be in 1..65535");
    std::lock_guard<std::mutex> lock(ctx->mu);
    MARS_CUDA(cudaSetDevice(ctx->device));
    MARS_CUDA(mars::launch_downsample_box(d_src, (int)width, (int)height, d_dst, ctx->stream));
    ctx->launches += 1;
    return MARS_OK;
}

int mars_upsample_nearest_device(mars_ctx* ctx, const uint8_t* d_src, uint32_t src_width,
                                 uint32_t src_height, uint8_t* d_dst, uint32_t width,
                                 uint32_t height) {
    if (!ctx || !d_src || !d_dst) return fail(MARS_EINVAL, "NULL argument");
    if (src_width == 0 || src_height == 0 || width > 65535 || height > 65535)
        return fail(MARS_EINVAL, "plane dimensions out of range");
    std::lock_guard<std::mutex> lock(ctx->mu);
    MARS_CUDA(cudaSetDevice(ctx->device));
    MARS_CUDA(mars::launch_upsample_nearest(d_src, (int)src_width, (int)src_height, d_dst,
                                            (int)width, (int)height, ctx->stream));
    ctx->launches += 1;
    return MARS_OK;
}

int mars_mse_device(mars_ctx* ctx, const uint8_t* d_a, const uint8_t* d_b, size_t n, double* mse) {
    if (!ctx || !mse || (n && (!d_a || !d_b))) return fail(MARS_EINVAL, "NULL argument");
    if (n == 0) return fail(MARS_EINVAL, "MSE of an empty plane is undefined");
    std::lock_guard<std::mutex> lock(ctx->mu);
    MARS_CUDA(cudaSetDevice(ctx->device));
    MARS_CUDA(mars::launch_sse(d_a, d_b, n, ctx->num_sms, ctx->d_counter, ctx->stream));
    ctx->launches += 1;
    unsigned long long sum = 0;
    MARS_CUDA(cudaMemcpyAsync(&sum, ctx->d_counter, sizeof sum, cudaMemcpyDeviceToHost,
                              ctx->stream));
    if (int e = sync_bounded(ctx)) return e;
    // Exact numerator, one rounding in the division, as the reference.
    *mse = (double)sum / (double)n;
    return MARS_OK;
}

int mars_ifs_parse(const uint8_t* data, size_t len, mars_header* header, mars_leaf** leaves,
                   size_t* nleaves) {
    if (!data || !header || !leaves || !nleaves) return fail(MARS_EINVAL, "NULL argument");
    std::vector<mars_leaf> out;
    if (int e = mars::codec::ifs_parse(data, len, header, &out))
        return fail(e, "malformed .ifs bitstream");
    *nleaves = out.size();
    *leaves = (mars_leaf*)std::malloc(std::max<size_t>(1, out.size()) * sizeof(mars_leaf));
    if (!*leaves) return fail(MARS_ENOMEM, "leaf array allocation failed");
    std::memcpy(*leaves, out.data(), out.size() * sizeof(mars_leaf));
    return MARS_OK;
}

int mars_ifs_write(const mars_header* header, const mars_leaf* leaves, size_t n, uint8_t** out,
                   size_t* len) {
    if (!header || (n && !leaves) || !out || !len) return fail(MARS_EINVAL, "NULL argument");
    std::vector<mars_leaf> v(leaves, leaves + n);
    std::vector<uint8_t> bytes;
    if (int e = mars::codec::ifs_write(*header, v, &bytes))
        return fail(e, "leaves do not tile the quadtree");
    *len = bytes.size();
    *out = (uint8_t*)std::malloc(std::max<size_t>(1, bytes.size()));
    if (!*out) return fail(MARS_ENOMEM, "byte buffer allocation failed");
    std::memcpy(*out, bytes.data(), bytes.size());
    return MARS_OK;
}

}  // extern "C"

namespace mars {
int ctx_sync(mars_ctx* ctx) { return sync_bounded(ctx); }
}  // namespace mars

extern "C" {

// Local iterative improvement of the domain choices (the decoder-side re-search of
// Hamzaoui, Hartenstein and Saupe's local iterative improvement of fractal codes): each pass
// decodes the current list, searches every mode-2 leaf again with its range block taken
// from the target and the domain pool from the decoded plane, and keeps the pass when the
// exact decode improves (else the leaves whose own pixels improved, if that improves it).
int mars_refine_domains(mars_ctx* ctx, const mars_params* params, const mars_header* hdr,
                        const mars_leaf* leaves, size_t n, const int32_t* residuals,
                        size_t nresiduals, const uint8_t* target, uint32_t passes,
                        uint32_t decode_iterations, mars_leaf* out_leaves,
                        mars_refine_report* report) {
    if (!ctx || !params || !hdr || !target || !report || (n && (!leaves || !out_leaves)))
        return fail(MARS_EINVAL, "NULL argument");
    if (int e = check_params(params)) return e;
    const uint32_t w = hdr->width, h = hdr->height;
    if (w == 0 || h == 0 || w > 65535 || h > 65535)
        return fail(MARS_EINVAL, "plane dimensions must be in 1..65535");
    if (hdr->shift == 0 || (hdr->shift & 1)) return fail(MARS_EUNSUPPORTED, "shift must be even");
    for (size_t k = 0; k < n; ++k) {
        const mars_leaf& L = leaves[k];
        if (L.size == 0 || L.row + L.size > h || L.col + L.size > w)
            return fail(MARS_EINVAL, "leaf " + std::to_string(k) + " is outside the plane");
    }
    std::memset(report, 0, sizeof *report);
    const size_t npx = (size_t)w * h;
    std::vector<mars_leaf> cur(leaves, leaves + n), trial;
    std::vector<uint8_t> x(npx), y(npx);
    auto decode = [&](const std::vector<mars_leaf>& ls, std::vector<uint8_t>* img) {
        return mars_decode(ctx, hdr, ls.data(), n, residuals, nresiduals, decode_iterations,
                           img->data());
    };
    auto sse_of = [&](const std::vector<uint8_t>& img) {
        double acc = 0.0;
        for (size_t q = 0; q < npx; ++q) {
            const double d = (double)img[q] - (double)target[q];
            acc += d * d;
        }
        return acc;
    };
    auto psnr_of = [&](double sse) {
        return sse > 0.0 ? 10.0 * std::log10(255.0 * 255.0 * (double)npx / sse) : INFINITY;
    };
    if (int e = decode(cur, &x)) return e;
    double sse = sse_of(x);
    report->loss_start = sse;
    report->psnr_plain = psnr_of(sse);

    // The mode-2 leaves by size, the order their candidates come back in.
    std::vector<size_t> order;
    std::vector<std::pair<uint32_t, size_t>> levels;  // (size, count)
    for (uint32_t size = 64; size >= 2; size /= 2) {
        const size_t before = order.size();
        for (size_t k = 0; k < n; ++k) {
            const mars_leaf& L = cur[k];
            if (L.mode == 2 && L.size == size && 2 * size <= w && 2 * size <= h) order.push_back(k);
        }
        if (order.size() > before) levels.push_back({size, order.size() - before});
    }
    std::vector<int32_t> owner(npx, -1);
    for (size_t k = 0; k < n; ++k)
        for (uint32_t r = 0; r < cur[k].size; ++r)
            std::fill_n(owner.begin() + (long)((size_t)(cur[k].row + r) * w + cur[k].col),
                        cur[k].size, (int32_t)k);
    std::vector<uint32_t> rc(2 * order.size());
    for (size_t i = 0; i < order.size(); ++i) {
        rc[i] = cur[order[i]].row;
        rc[order.size() + i] = cur[order[i]].col;
    }
    std::vector<mars::CandidateOut> cand(order.size());
    const mars::FitParams fp = make_fit_params(*params);

    for (uint32_t pass = 0; pass < passes && !order.empty(); ++pass) {
        report->steps += 1;
        {
            std::lock_guard<std::mutex> lock(ctx->mu);
            MARS_CUDA(cudaSetDevice(ctx->device));
            const cudaStream_t st = ctx->stream;
            Scratch sc(st);
            uint8_t *d_t = nullptr, *d_x = nullptr;
            int32_t* d_D = nullptr;
            uint32_t* d_rc = nullptr;
            mars::CandidateOut* d_out = nullptr;
            MARS_CUDA(sc.get(&d_t, npx));
            MARS_CUDA(sc.get(&d_x, npx));
            MARS_CUDA(sc.get(&d_D, std::max<size_t>(1, (size_t)(w / 2) * (h / 2))));
            MARS_CUDA(sc.get(&d_rc, rc.size()));
            MARS_CUDA(sc.get(&d_out, cand.size()));
            MARS_CUDA(cudaMemcpyAsync(d_t, target, npx, cudaMemcpyHostToDevice, st));
            MARS_CUDA(cudaMemcpyAsync(d_x, x.data(), npx, cudaMemcpyHostToDevice, st));
            MARS_CUDA(cudaMemcpyAsync(d_rc, rc.data(), rc.size() * 4, cudaMemcpyHostToDevice, st));
            MARS_CUDA(mars::launch_contract(d_x, (int)w, (int)h, d_D, st));
            ctx->launches += 1;
            size_t off = 0;
            for (const auto& lv : levels) {
                const int e = run_level(ctx, sc, d_t, d_D, w, h, lv.first, hdr->shift, fp,
                                        d_rc + off, d_rc + order.size() + off, lv.second,
                                        d_out + off, 1, d_x);
                if (e) return e;
                off += lv.second;
            }
            MARS_CUDA(cudaMemcpyAsync(cand.data(), d_out, cand.size() * sizeof(mars::CandidateOut),
                                      cudaMemcpyDeviceToHost, st));
            if (int e = sync_bounded(ctx)) return e;
        }
        trial = cur;
        size_t changed = 0;
        for (size_t i = 0; i < order.size(); ++i) {
            const mars::CandidateOut& c = cand[i];
            mars_leaf& L = trial[order[i]];
            if (!c.valid || c.qalfa < 1) continue;
            if (c.dom_row == L.dom_row && c.dom_col == L.dom_col && c.isometry == L.isometry &&
                c.qalfa == L.qalfa && c.qbeta == L.qbeta)
                continue;
            L.dom_row = c.dom_row;
            L.dom_col = c.dom_col;
            L.isometry = c.isometry;
            L.qalfa = c.qalfa;
            L.qbeta = c.qbeta;
            ++changed;
        }
        if (!changed) break;
        if (int e = decode(trial, &y)) return e;
        double sse_y = sse_of(y);
        if (!(sse_y < sse)) {
            // Keep the re-searched leaves whose own pixels decode better.
            std::vector<double> before(n, 0.0), after(n, 0.0);
            for (size_t q = 0; q < npx; ++q) {
                if (owner[q] < 0) continue;
                const double t = target[q];
                before[owner[q]] += ((double)x[q] - t) * ((double)x[q] - t);
                after[owner[q]] += ((double)y[q] - t) * ((double)y[q] - t);
            }
            for (size_t k = 0; k < n; ++k)
                if (after[k] >= before[k]) trial[k] = cur[k];
            if (int e = decode(trial, &y)) return e;
            sse_y = sse_of(y);
            if (!(sse_y < sse)) break;
        }
        cur.swap(trial);
        x.swap(y);
        sse = sse_y;
        report->improving_steps += 1;
    }
    report->loss_end = sse;
    report->psnr_refined = psnr_of(sse);
    report->accepted = report->improving_steps > 0 ? 1u : 0u;
    uint32_t changed = 0;
    for (size_t k = 0; k < n; ++k)
        changed += std::memcmp(&cur[k], &leaves[k], sizeof(mars_leaf)) != 0 ? 1u : 0u;
    report->changed_leaves = changed;
    std::copy(cur.begin(), cur.end(), out_leaves);
    return MARS_OK;
}

}  // extern "C"
