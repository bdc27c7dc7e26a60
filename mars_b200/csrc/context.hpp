// The library context (mars_ctx) and the host helpers shared by the files that implement
// the C ABI.  Internal: not part of include/mars_b200.h.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <atomic>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/mars_b200.h"
#include "kernels.cuh"

struct mars_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::atomic<uint64_t> launches{0};
    std::mutex mu;
    unsigned long long* d_counter = nullptr;  // survivors that took the exact f64 fit
    int* d_err = nullptr;                     // kernel-side error bits (bounded waits)
    int* h_err = nullptr;                     // pinned copy of d_err, read by sync_bounded
    int search_path = 0;                      // 0 auto, 1 CUDA cores only, 2 tensor cores
    bool tma_16_boxes = false;                // load A stages as 16 2-D boxes (A/B checks)
    bool fold_only = false;                   // no split-digit operand at sizes 16..64 (A/B)
    bool per_level = false;                   // one correlation launch per level (A/B)
    PFN_cuTensorMapEncodeTiled_v12000 encode_tiled = nullptr;
    // Streams and events a search plan's capture forks its levels onto (created on first use;
    // the levels of a plane run as parallel branches of the plan's graph).
    static constexpr int kBranches = 8;
    cudaStream_t branch[kBranches] = {};
    cudaEvent_t fork_ev = nullptr;
    cudaEvent_t join_ev[kBranches] = {};
    // Search plans mars_encode keeps for plane geometries it has met before (api.cu).
    std::mutex plan_cache_mu;
    std::vector<std::pair<std::string, mars_search_plan*>> plan_cache;
    std::vector<std::string> plans_seen;
};

namespace mars {
// Records the message mars_last_error() reports and returns `code`.
int set_last_error(int code, const std::string& msg);
// Waits for the context's stream with the library's deadline (MARS_SYNC_TIMEOUT_S) and
// turns kernel-reported errors into a status.  The caller holds ctx->mu.
int ctx_sync(mars_ctx* ctx);
// The bits_alfa / bits_beta / max_alfa checks every search entry point makes (MARS_EINVAL
// with a message on failure).
int check_fit_params(const mars_params& p);
// The device-side fit constants of a parameter set (fit.cuh).
FitParams make_fit_params(const mars_params& p);
// The domain pool geometry of one (size, shift) level of a w x h plane.
LevelGeom level_geom(uint32_t w, uint32_t h, uint32_t size, uint32_t shift);
}  // namespace mars
