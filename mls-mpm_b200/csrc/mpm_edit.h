// mpm_edit.h — launchers of the particle-editing passes: COMPACT (deleteNear)
// and RAYCAST (raycastFluid).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/mpm_types.h"

namespace mpm {

// Particles per block of the compaction passes (256 threads x 8 rounds).
constexpr uint32_t kCompactThreads = 256;
constexpr uint32_t kCompactRounds = 8;
constexpr uint32_t kCompactTile = kCompactThreads * kCompactRounds;

// Scratch words the compaction needs for n particles: one survivor count per
// block of kCompactTile particles.  Every word is written by the count pass
// before any pass reads it, so the scratch needs no clearing between calls.
inline uint64_t compact_scratch_words(uint64_t n) { return (n + kCompactTile - 1) / kCompactTile + 1; }

// Stable stream compaction (shaders.js:521-546 with the ascending survivor
// order): particles of pos_in/vel_in/mass_in at perpendicular distance >=
// del.radius from the line (origin, dir) go to the front of the outputs in
// index order; *count_dev receives the survivor count.  `scratch` holds
// compact_scratch_words(n) words.  Inputs and outputs must not overlap.
cudaError_t launch_compact(const mpm_ray_params& del, uint32_t n, const float4* pos_in, const float4* vel_in,
                           const float* mass_in, float4* pos_out, float4* vel_out, float* mass_out,
                           uint32_t* scratch, uint32_t* count_dev, cudaStream_t stream);

// RAYCAST (shaders.js:563-576): *hit_dev = min over hit particles of the f32
// bit pattern of t (0xFFFFFFFF when none).  Sets *hit_dev itself.
cudaError_t launch_raycast(const mpm_ray_params& ray, uint32_t n, const float4* pos_in, uint32_t* hit_dev,
                           cudaStream_t stream);

}  // namespace mpm
