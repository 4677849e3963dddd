// mpm_kernels.h — launchers of the per-pass kernels.
#pragma once

#include <cuda_runtime.h>

#include "mpm_scene.h"

namespace mpm {

// One substep of the plain engine (one kernel per reference pass).
cudaError_t launch_substep_plain(Scene& s);

// APPLY_HAND over the scene's hand box (both engines).
cudaError_t launch_apply_hand(Scene& s);

// Rebuilds the diffuse alive mask from the pool (after the pool was uploaded).
cudaError_t launch_alive_mask_build(Scene& s);

// DiffuseGPU.step after G2P; eval = run the spawn-decision pass here.
// P_dev / W_dev (binned engine): the scene's uniforms in device memory, read
// by ADVECT instead of the host copies, so the launches can be captured in a
// CUDA graph and replayed with uniforms uploaded later.  stream: where to
// enqueue (null: the scene's stream).
cudaError_t launch_diffuse(Scene& s, bool eval, const mpm_params* P_dev = nullptr,
                           const mpm_wall_params* W_dev = nullptr, cudaStream_t stream = nullptr);

}  // namespace mpm
