// Library-level C-ABI entry points: version and thread-local error text.
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "glide_internal.h"

namespace glide {

static thread_local char g_last_error[512] = "";

glide_status set_error(glide_status code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return code;
}

glide_status cuda_error(cudaError_t err, const char* what) {
    return set_error(GLIDE_ERR_CUDA, "%s: CUDA error %d (%s)", what, (int)err, cudaGetErrorString(err));
}

glide_status check_launch(const char* what) {
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return cuda_error(err, what);
    return GLIDE_OK;
}

}  // namespace glide

extern "C" int32_t glide_version(void) { return 200; /* 0.2.0 */ }

extern "C" glide_status glide_last_error(char* buf, size_t len) {
    if (!buf || len == 0) return GLIDE_ERR_INVALID_ARG;
    std::strncpy(buf, glide::g_last_error, len - 1);
    buf[len - 1] = '\0';
    return GLIDE_OK;
}

extern "C" glide_status glide_abi_struct_sizes(size_t* out, int32_t n) {
    if (!out || n < 0) return GLIDE_ERR_INVALID_ARG;
    const size_t sizes[9] = {sizeof(glide_grid),        sizeof(glide_window_desc), sizeof(glide_step_sched),
                             sizeof(glide_footprint_grid), sizeof(glide_step_args), sizeof(glide_convect_args),
                             sizeof(glide_ou_args),     sizeof(glide_regrid_args), sizeof(glide_compact_args)};
    for (int i = 0; i < n && i < 9; ++i) out[i] = sizes[i];
    return GLIDE_OK;
}
