// mpm_alloc.cu — accounting device allocator behind every long-lived device
// buffer of the library, and the process-wide cap on it
// (mpm_set_device_memory_limit / mpm_device_memory_in_use).
#include "mpm_alloc.h"

#include <mutex>
#include <unordered_map>

#include "../../include/mpm_b200.h"

namespace mpm {
namespace {
std::mutex g_mu;
std::unordered_map<const void*, size_t> g_sizes;
uint64_t g_in_use = 0;
uint64_t g_limit = 0;   // 0: no cap
}  // namespace

cudaError_t dmalloc(void** p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        if (g_limit && g_in_use + bytes > g_limit) return cudaErrorMemoryAllocation;
        g_in_use += bytes;   // reserved before the call so concurrent callers see it
    }
    const cudaError_t e = cudaMalloc(p, bytes);
    std::lock_guard<std::mutex> lock(g_mu);
    if (e != cudaSuccess) {
        g_in_use -= bytes;
        *p = nullptr;
        return e;
    }
    g_sizes[*p] = bytes;
    return cudaSuccess;
}

void dfree(const void* p) {
    if (!p) return;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        auto it = g_sizes.find(p);
        if (it != g_sizes.end()) {
            g_in_use -= it->second;
            g_sizes.erase(it);
        }
    }
    cudaFree(const_cast<void*>(p));
}

uint64_t device_bytes_in_use() {
    std::lock_guard<std::mutex> lock(g_mu);
    return g_in_use;
}

}  // namespace mpm

extern "C" {

mpm_status mpm_set_device_memory_limit(uint64_t bytes) {
    std::lock_guard<std::mutex> lock(mpm::g_mu);
    mpm::g_limit = bytes;
    return MPM_OK;
}

mpm_status mpm_device_memory_in_use(uint64_t* bytes) {
    if (!bytes) return MPM_ERR_INVALID_ARG;
    *bytes = mpm::device_bytes_in_use();
    return MPM_OK;
}

}  // extern "C"
