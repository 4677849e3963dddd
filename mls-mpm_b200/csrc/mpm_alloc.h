// mpm_alloc.h — every device allocation the library holds goes through here,
// so a process-wide cap (mpm_set_device_memory_limit) can refuse one the way
// an exhausted device would: the caller sees cudaErrorMemoryAllocation and
// returns MPM_ERR_OOM with its object left as it was.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace mpm {

// cudaMalloc with accounting; bytes == 0 allocates 16.  Refused with
// cudaErrorMemoryAllocation (nothing allocated) when the cap would be passed.
cudaError_t dmalloc(void** p, size_t bytes);
template <class T> inline cudaError_t dmalloc(T** p, size_t bytes) {
    void* q = nullptr;
    const cudaError_t e = dmalloc(&q, bytes);
    *p = static_cast<T*>(q);
    return e;
}
// cudaFree of a pointer from dmalloc (null is ignored).
void dfree(const void* p);
// Bytes currently held through dmalloc.
uint64_t device_bytes_in_use();

}  // namespace mpm
