// mpm_noalloc.cu — mpm_compact_noalloc: the COMPACT pass of mpm_compact with
// its per-block scratch in a fixed device array of this library, so a call
// allocates nothing (no cudaMalloc / cudaMallocAsync / cudaFree, no library
// allocator).
//
// Scratch: g_compact_scratch holds one survivor count per block of
// kCompactTile (2048) particles for up to MPM_COMPACT_NOALLOC_MAX_N particles
// (8193 words, 32 KB per device).  The count pass writes every word it uses
// before the scan and write passes read it, so nothing has to start at zero
// and no clearing is needed between calls.
//
// Setup: the array's device address is looked up once per device
// (cudaGetSymbolAddress with that device current, under a mutex) on the first
// call on that device; that call may also load the library's module onto the
// device.  Make the first call on each device before capturing a stream.
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
        if (!g_scratch_ptr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_compact_scratch);   // device `dev` is current
            if (e != cudaSuccess || !p) {
                set_error(std::string("mpm_compact_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
                return MPM_ERR_DEVICE;
            }
            g_scratch_ptr[dev] = static_cast<uint32_t*>(p);
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
