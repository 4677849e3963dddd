// mpm_kernels.h — launchers of the per-pass kernels.
#pragma once

#include <cuda_runtime.h>

#include "mpm_scene.h"

namespace mpm {

// One substep of the plain engine (one kernel per reference pass).
cudaError_t launch_substep_plain(Scene& s);

// APPLY_HAND over the scene's hand box (both engines).
cudaError_t launch_apply_hand(Scene& s);

// DiffuseGPU.step after G2P; eval = run the spawn-decision pass here.
cudaError_t launch_diffuse(Scene& s, bool eval);

}  // namespace mpm
