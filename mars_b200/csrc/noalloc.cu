// An allocation-free form of the level search, for callers that cannot allocate device
// memory: real-time pipelines that forbid allocation once they are running, plug-ins whose
// host application owns every device allocation, hosts with a fixed device-memory budget.
// The scratch the search needs lives in one file-scope device array instead of the
// stream-ordered pool the other entry points use.  Each call rewrites every part of the
// array it reads (contracted plane, statistics, partial champions), so nothing carried
// over from the previous call needs clearing; calls that overlap on the GPU race.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/mars_b200.h"
#include "context.hpp"
#include "kernels.cuh"

namespace {

// 16 MiB of scratch, held by every GPU that loads the library until the process exits.
constexpr size_t kScratchBytes = 16u << 20;
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};

}  // namespace

namespace {

int fail(int code, const std::string& msg) { return mars::set_last_error(code, msg); }

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Once per device, with that device current: the device address of g_scratch.  The host
// name of the array is only a host-side stand-in and must never be handed to a kernel.
int scratch_address(int device, unsigned char** out) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess)
            return fail(MARS_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_addr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_addr[device]);
    return MARS_OK;
}

}  // namespace

extern "C" int mars_search_blocks_noalloc(const uint8_t* d_plane, uint32_t width, uint32_t height,
                                          uint32_t size, uint32_t shift, const mars_params* params,
                                          const uint32_t* d_rows, const uint32_t* d_cols, size_t n,
                                          mars_candidate* d_out, void* stream) {
    if (!d_plane || !params || (n && (!d_rows || !d_cols || !d_out)))
        return fail(MARS_EINVAL, "NULL argument");
    if (size < 2 || size > 64 || (size & (size - 1)))
        return fail(MARS_EINVAL, "size must be a power of two in 2..64");
    if (shift == 0 || (shift & 1)) return fail(MARS_EUNSUPPORTED, "shift must be even");
    if (int e = mars::check_fit_params(*params)) return e;
    if (width == 0 || height == 0 || width > 65535 || height > 65535)
        return fail(MARS_EINVAL, "plane dimensions must be in 1..65535");
    if (n == 0) return MARS_OK;

    int device = 0, num_sms = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices)
        return fail(MARS_ENODEV, "no current CUDA device");
    if (cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return fail(MARS_ENODEV, "cannot query the current device");

    const mars::LevelGeom g = mars::level_geom(width, height, size, shift);
    const cudaStream_t st = (cudaStream_t)stream;
    if (g.nrow_d <= 0 || g.ncol_d <= 0) {
        const cudaError_t e = cudaMemsetAsync(d_out, 0, n * sizeof(mars_candidate), st);
        return e == cudaSuccess ? MARS_OK : fail(MARS_ECUDA, cudaGetErrorString(e));
    }

    // Carve the scratch: contracted plane, range and domain statistics, partial champions.
    const size_t ndom = (size_t)g.nrow_d * g.ncol_d;
    const int nsplit = mars::search_simt_splits(g, (int)n, num_sms);
    size_t off[12], need = 0;
    const size_t sizes[12] = {(size_t)g.dw * g.dh * 4, n * 4, n * 4, n * 8, n * 8, n * 8,
                              ndom * 4, ndom * 8, ndom * 4, ndom * 4,
                              (size_t)nsplit * n * sizeof(mars::Partial), 0};
    for (int i = 0; i < 11; ++i) {
        off[i] = need;
        need += align256(sizes[i]);
    }
    if (need > kScratchBytes)
        return fail(MARS_EINVAL, "this search needs " + std::to_string(need) +
                                     " bytes of scratch; the allocation-free entry point holds " +
                                     std::to_string(kScratchBytes));
    unsigned char* base = nullptr;
    if (int e = scratch_address(device, &base)) return e;

    int32_t* d_D = reinterpret_cast<int32_t*>(base + off[0]);
    mars::RangeStats rs;
    rs.t0 = reinterpret_cast<int32_t*>(base + off[1]);
    rs.t2 = reinterpret_cast<int32_t*>(base + off[2]);
    rs.nrr = reinterpret_cast<int64_t*>(base + off[3]);
    rs.sum0 = reinterpret_cast<double*>(base + off[4]);
    rs.rms0 = reinterpret_cast<double*>(base + off[5]);
    mars::DomainStats ds;
    ds.s1x4 = reinterpret_cast<int32_t*>(base + off[6]);
    ds.s2x16 = reinterpret_cast<int64_t*>(base + off[7]);
    ds.detf = reinterpret_cast<float*>(base + off[8]);
    ds.sdetf = reinterpret_cast<float*>(base + off[9]);
    mars::Partial* partials = reinterpret_cast<mars::Partial*>(base + off[10]);

    const mars::FitParams fp = mars::make_fit_params(*params);

    cudaError_t e = mars::launch_contract(d_plane, (int)width, (int)height, d_D, st);
    if (e == cudaSuccess)
        e = mars::launch_range_stats(d_plane, (int)width, (int)height, d_rows, d_cols, (int)n,
                                     (int)size, fp, rs, st);
    if (e == cudaSuccess) e = mars::launch_domain_stats(d_D, g, ds, st);
    if (e == cudaSuccess)
        e = mars::launch_search_simt(d_D, d_plane, (int)width, d_rows, d_cols, (int)n, g, rs, ds,
                                     fp, partials, nsplit, nullptr, st);
    if (e == cudaSuccess)
        e = mars::launch_reduce(partials, nsplit, (int)n, g, rs, ds,
                                reinterpret_cast<mars::CandidateOut*>(d_out), st);
    return e == cudaSuccess ? MARS_OK : fail(MARS_ECUDA, cudaGetErrorString(e));
}
