// mpm_kernels.h — launch entry points of the substep kernels.
#pragma once

#include <cuda_runtime.h>

#include "mpm_scene.h"

namespace mpm {

// Enqueue one substep (fluid passes + diffuse when enabled) on s.stream.
cudaError_t launch_substep(Scene& s);

}  // namespace mpm
