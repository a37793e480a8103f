// Internal host-side helpers shared by the C-ABI entry points.
#pragma once

#include <cuda_runtime.h>

#include "glide_b200.h"

namespace glide {

// Records a printf-style message as the calling thread's last error and
// returns `code`.
glide_status set_error(glide_status code, const char* fmt, ...);

// Checks the launch that was just issued (no synchronisation).
glide_status check_launch(const char* what);

// Maps a CUDA error code to GLIDE_ERR_CUDA with its text.
glide_status cuda_error(cudaError_t err, const char* what);

}  // namespace glide
