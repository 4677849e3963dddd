// mpm_noalloc.cu — mpm_compact_noalloc: the COMPACT pass of mpm_compact with
// its per-block scratch in a fixed device array of this library, so a call
// allocates nothing (no cudaMalloc / cudaMallocAsync / cudaFree, no library
// allocator).
//
// Scratch: g_compact_scratch holds one survivor count per block of
// kCompactTile (2048) particles for up to MPM_COMPACT_NOALLOC_MAX_N particles
// (8,193 words = 32,772 bytes per device).  The count pass writes every word it uses
// before the scan and write passes read it, so nothing has to start at zero
// and no clearing is needed between calls.
//
// Setup: the array's device address is looked up (cudaGetSymbolAddress with
// the device current, under a mutex) on the first call on each device, and
// again on the first call after that device's context was re-created (for
// example after cudaDeviceReset, when the module may be loaded at another
// address): the address is cached per device together with the unique id of
// the context it was looked up in (cuCtxGetId, reached through
// cudaGetDriverEntryPoint so the library needs no link to libcuda).  That
// first call may also load the library's module onto the device, so make it
// before capturing a stream.
//
// Concurrency: all calls on one device share the one array.  Calls enqueued
// in order on a single stream are safe; calls that may overlap (different
// streams, or threads racing on streams without ordering) race on the
// scratch and give wrong results.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/mpm_b200.h"
#include "mpm_edit.h"

namespace mpm {

void set_error(const std::string& msg);

namespace {

constexpr uint64_t kNoAllocWords = (uint64_t(MPM_COMPACT_NOALLOC_MAX_N) + kCompactTile - 1) / kCompactTile + 1;
static_assert(kNoAllocWords * 4 <= 64 * 1024, "no-alloc compaction scratch is meant to stay small");

static __device__ __align__(256) uint32_t g_compact_scratch[kNoAllocWords];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint32_t* g_scratch_ptr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};   // context id the address belongs to

// Driver entry points for the current context's unique id (never reused
// within a process, unlike a context handle).
typedef int (*CtxGetCurrentFn)(void**);
typedef int (*CtxGetIdFn)(void*, unsigned long long*);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;
bool g_ctx_fns_looked_up = false;

// Unique id of the calling thread's current context; false when it cannot be
// read (then the caller looks the address up on every call).
bool current_context_id(unsigned long long& id) {
    if (!g_ctx_fns_looked_up) {
        g_ctx_fns_looked_up = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f);
    }
    if (!g_ctx_get_current || !g_ctx_get_id) return false;
    void* ctx = nullptr;
    if (g_ctx_get_current(&ctx) != 0 || !ctx) return false;
    return g_ctx_get_id(ctx, &id) == 0;
}

}  // namespace
}  // namespace mpm

using namespace mpm;

extern "C" mpm_status mpm_compact_noalloc(const mpm_ray_params* del, uint32_t n, const float* pos_in,
                                          const float* vel_in, const float* mass_in, float* pos_out,
                                          float* vel_out, float* mass_out, uint32_t* count_dev, void* stream) {
    if (!del || !count_dev || (n && (!pos_in || !vel_in || !mass_in || !pos_out || !vel_out || !mass_out))) {
        set_error("mpm_compact_noalloc: NULL argument");
        return MPM_ERR_INVALID_ARG;
    }
    if (n > MPM_COMPACT_NOALLOC_MAX_N) {
        char msg[160];
        std::snprintf(msg, sizeof msg,
                      "mpm_compact_noalloc: n = %u exceeds the fixed scratch limit of %u particles "
                      "(MPM_COMPACT_NOALLOC_MAX_N); use mpm_compact",
                      n, (unsigned)MPM_COMPACT_NOALLOC_MAX_N);
        set_error(msg);
        return MPM_ERR_CAPACITY;
    }
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error(std::string("mpm_compact_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
        return MPM_ERR_DEVICE;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("mpm_compact_noalloc: device ordinal beyond the supported 64");
        return MPM_ERR_UNSUPPORTED;
    }
    uint32_t* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        // cudaGetDevice above made the device's primary context current
        unsigned long long ctx_id = 0;
        const bool have_id = current_context_id(ctx_id);
        if (!g_scratch_ptr[dev] || !have_id || g_scratch_ctx[dev] != ctx_id) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_compact_scratch);   // device `dev` is current
            if (e != cudaSuccess || !p) {
                g_scratch_ptr[dev] = nullptr;
                set_error(std::string("mpm_compact_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
                return MPM_ERR_DEVICE;
            }
            g_scratch_ptr[dev] = static_cast<uint32_t*>(p);
            g_scratch_ctx[dev] = have_id ? ctx_id : 0ull;
        }
        scratch = g_scratch_ptr[dev];
    }
    e = launch_compact(*del, n, (const float4*)pos_in, (const float4*)vel_in, mass_in, (float4*)pos_out,
                       (float4*)vel_out, mass_out, scratch, count_dev, (cudaStream_t)stream);
    if (e != cudaSuccess) {
        set_error(std::string("mpm_compact_noalloc: launch: ") + cudaGetErrorString(e));
        return MPM_ERR_DEVICE;
    }
    return MPM_OK;
}
