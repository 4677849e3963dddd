// mpm_edit.cu — COMPACT (deleteNear) and RAYCAST (raycastFluid) passes.
//
// The reference compacts with one atomic counter (shaders.js:542), so its
// survivor order depends on thread scheduling.  Here the survivors keep their
// index order (a deterministic order the reference can also produce): one pass
// counts survivors per block of kCompactTile particles, one block scans the
// counts, and a third pass writes each survivor at its block offset plus its
// rank inside the block (warp ballots).  All three passes stream the inputs
// with coalesced 16-byte loads; the work is HBM-bound (68 B per particle).
#include <cuda_runtime.h>

#include "mpm_device.cuh"
#include "mpm_edit.h"

namespace mpm {
namespace {

// shaders.js:80-84
__device__ __forceinline__ float ray_perp_dist(f3 pos, f3 origin, f3 dir) {
    const f3 to_p = sub(pos, origin);
    const float d = dot3(to_p, dir);
    const f3 perp = mk(to_p.x - d * dir.x, to_p.y - d * dir.y, to_p.z - d * dir.z);
    return len3(perp);
}

// shaders.js:536-540: a particle survives unless it lies inside the cylinder.
__device__ __forceinline__ bool survives(const float4 q, const mpm_ray_params& del) {
    return !(ray_perp_dist(mk(q.x, q.y, q.z), mk(del.ox, del.oy, del.oz), mk(del.dx, del.dy, del.dz)) < del.radius);
}

__global__ void __launch_bounds__(kCompactThreads) k_compact_count(mpm_ray_params del, uint32_t n,
                                                                   const float4* __restrict__ pos,
                                                                   uint32_t* __restrict__ counts) {
    const uint64_t base = (uint64_t)blockIdx.x * kCompactTile;
    uint32_t total = 0;
#pragma unroll
    for (uint32_t r = 0; r < kCompactRounds; ++r) {
        const uint64_t p = base + r * kCompactThreads + threadIdx.x;
        const bool keep = p < n && survives(pos[p], del);
        total += (uint32_t)__syncthreads_count(keep);
    }
    if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

// One block: exclusive scan of the per-block counts in place; the total goes
// to *count_dev.
__global__ void __launch_bounds__(1024) k_compact_scan(uint32_t nblocks, uint32_t* __restrict__ counts,
                                                       uint32_t* __restrict__ count_dev) {
    __shared__ uint32_t ws[33];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t carry = 0;
    for (uint32_t b0 = 0; b0 < nblocks; b0 += 1024) {
        const uint32_t b = b0 + threadIdx.x;
        const uint32_t x = b < nblocks ? counts[b] : 0u;
        uint32_t sc = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, sc, o);
            if (lane >= o) sc += y;
        }
        if (lane == 31) ws[wid] = sc;
        __syncthreads();
        if (wid == 0) {
            const uint32_t w = ws[lane];
            uint32_t ww = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, ww, o);
                if (lane >= o) ww += y;
            }
            ws[lane] = ww - w;
            if (lane == 31) ws[32] = ww;
        }
        __syncthreads();
        if (b < nblocks) counts[b] = carry + ws[wid] + sc - x;
        carry += ws[32];
        __syncthreads();
    }
    if (threadIdx.x == 0) *count_dev = carry;
}

__global__ void __launch_bounds__(kCompactThreads) k_compact_write(mpm_ray_params del, uint32_t n,
                                                                   const float4* __restrict__ pos_in,
                                                                   const float4* __restrict__ vel_in,
                                                                   const float* __restrict__ mass_in,
                                                                   float4* __restrict__ pos_out,
                                                                   float4* __restrict__ vel_out,
                                                                   float* __restrict__ mass_out,
                                                                   const uint32_t* __restrict__ offsets) {
    __shared__ uint32_t wsum[kCompactThreads / 32];
    const uint64_t base = (uint64_t)blockIdx.x * kCompactTile;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t off = offsets[blockIdx.x];
#pragma unroll 1
    for (uint32_t r = 0; r < kCompactRounds; ++r) {
        const uint64_t p = base + r * kCompactThreads + threadIdx.x;
        float4 q = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        bool keep = false;
        if (p < n) {
            q = pos_in[p];
            keep = survives(q, del);
        }
        const uint32_t bal = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) wsum[wid] = __popc(bal);
        __syncthreads();
        uint32_t before = 0, round_total = 0;
#pragma unroll
        for (int w = 0; w < (int)(kCompactThreads / 32); ++w) {
            const uint32_t c = wsum[w];
            if (w < wid) before += c;
            round_total += c;
        }
        if (keep) {
            const uint32_t idx = off + before + __popc(bal & ((1u << lane) - 1u));
            pos_out[idx] = q;
            vel_out[idx] = vel_in[p];
            mass_out[idx] = mass_in[p];
        }
        off += round_total;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) k_raycast(mpm_ray_params ray, uint32_t n, const float4* __restrict__ pos,
                                                 uint32_t* __restrict__ hit) {
    const f3 origin = mk(ray.ox, ray.oy, ray.oz), dir = mk(ray.dx, ray.dy, ray.dz);
    uint32_t best = 0xFFFFFFFFu;
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (uint64_t)gridDim.x * blockDim.x) {
        const float4 q = pos[p];
        const f3 pp = mk(q.x, q.y, q.z);
        const float t = dot3(sub(pp, origin), dir);            // shaders.js:570
        if (t <= 0.0f) continue;                                 // shaders.js:571
        if (ray_perp_dist(pp, origin, dir) >= ray.radius) continue;   // shaders.js:572
        const uint32_t bits = __float_as_uint(t);
        best = bits < best ? bits : best;                        // atomicMin on the bits (shaders.js:574)
    }
    best = __reduce_min_sync(0xffffffffu, best);
    if ((threadIdx.x & 31) == 0 && best != 0xFFFFFFFFu) atomicMin(hit, best);
}

}  // namespace

cudaError_t launch_compact(const mpm_ray_params& del, uint32_t n, const float4* pos_in, const float4* vel_in,
                           const float* mass_in, float4* pos_out, float4* vel_out, float* mass_out,
                           uint32_t* scratch, uint32_t* count_dev, cudaStream_t stream) {
    if (n == 0) return cudaMemsetAsync(count_dev, 0, 4, stream);
    const uint32_t nblocks = (uint32_t)((n + (uint64_t)kCompactTile - 1) / kCompactTile);
    k_compact_count<<<nblocks, kCompactThreads, 0, stream>>>(del, n, pos_in, scratch);
    k_compact_scan<<<1, 1024, 0, stream>>>(nblocks, scratch, count_dev);
    k_compact_write<<<nblocks, kCompactThreads, 0, stream>>>(del, n, pos_in, vel_in, mass_in, pos_out, vel_out,
                                                             mass_out, scratch);
    return cudaGetLastError();
}

cudaError_t launch_raycast(const mpm_ray_params& ray, uint32_t n, const float4* pos_in, uint32_t* hit_dev,
                           cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(hit_dev, 0xFF, 4, stream);   // fluid-gpu.js:601 sentinel
    if (e != cudaSuccess || n == 0) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t want = (n + 255u) / 256u;
    const uint32_t blocks = (uint32_t)(want < (uint64_t)sms * 8 ? want : (uint64_t)sms * 8);
    k_raycast<<<blocks, 256, 0, stream>>>(ray, n, pos_in, hit_dev);
    return cudaGetLastError();
}

}  // namespace mpm
