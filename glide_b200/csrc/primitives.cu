// Engine primitives: the per-substep particle updates of the fused step kernel
// as separate launches (exact-OU velocity update, vertical and horizontal
// displacement, smooth-wall reflection, one RK2 stage). They mirror the
// reference's GPUEngine methods (src/lpdm/gpu_engine.py:308-507) and run the
// same device functions as glide_step's substep loop (common.cuh), so that
// engine-level tests (OU statistics, Taylor dispersion, the diffusion limit)
// exercise the fused path's arithmetic.
#include "common.cuh"
#include "glide_internal.h"

namespace glide {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ float pick(const float* arr, float scalar, int64_t i) { return arr ? arr[i] : scalar; }

__global__ void ou_update_kernel(const glide_ou_args a) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const float dt = pick(a.dt, a.dt_scalar, i);
    const float decay = ou_decay(dt, pick(a.t_l, a.t_l_scalar, i));
    const float amp = ou_amplitude(pick(a.sigma2, a.sigma2_scalar, i), decay);
    float eta;
    if (a.noise) {
        eta = a.noise[i];
    } else {
        StepNormals rng((uint64_t)i, a.counter, (uint32_t)a.seed, (uint32_t)(a.seed >> 32));
        eta = rng.next();
    }
    a.w[i] = ou_step(a.w[i], decay, pick(a.drift, a.drift_scalar, i) * dt, amp, eta);
}

__global__ void displace_vertical_kernel(int64_t n, float* z, int64_t stride, const float* w, const float* dt,
                                         float dt_scalar, float dir) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    z[i * stride] = displace_z(z[i * stride], w[i], pick(dt, dt_scalar, i), dir);
}

__global__ void displace_horizontal_kernel(int64_t n, float* lon, float* lat, int64_t stride, const float* u,
                                           const float* v, const float* dt, float dt_scalar, float dir) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float la = lat[i * stride], d = pick(dt, dt_scalar, i);
    lon[i * stride] = displace_lon(lon[i * stride], u[i], d, dir, m_per_deg_lon(la));
    lat[i * stride] = displace_lat(la, v[i], d, dir);
}

__global__ void reflect_kernel(int64_t n, float* z, int64_t stride, float* w, float z_surface) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float zz = z[i * stride], ww = w[i];
    reflect_surface(zz, ww, z_surface);
    z[i * stride] = zz;
    w[i] = ww;
}

// out = x - h v on the three position columns (the RK2 stages of hanna.py:866-896)
__global__ void rk2_stage_kernel(int64_t n, const float* x, int64_t x_stride, const float* v, int64_t v_stride, float h,
                                 float* out, int64_t out_stride) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int c = 0; c < 3; ++c) out[i * out_stride + c] = x[i * x_stride + c] - h * v[i * v_stride + c];
}

unsigned blocks_for(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

glide_status check_n(int64_t n, const char* what) {
    if (n < 0 || (n + kThreads - 1) / kThreads > 0x7fffffff) return set_error(GLIDE_ERR_INVALID_ARG, "%s: n out of range", what);
    return GLIDE_OK;
}

}  // namespace
}  // namespace glide

using namespace glide;

extern "C" glide_status glide_ou_update(const glide_ou_args* a, void* stream) {
    if (!a) return set_error(GLIDE_ERR_INVALID_ARG, "glide_ou_update: args is NULL");
    if (glide_status st = check_n(a->n, "glide_ou_update")) return st;
    if (a->n == 0) return GLIDE_OK;
    if (!a->w) return set_error(GLIDE_ERR_INVALID_ARG, "glide_ou_update: w is NULL");
    if (!a->t_l && !(a->t_l_scalar > 0.0f))
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_ou_update: t_lagrangian must be > 0");
    if (!a->dt && !(a->dt_scalar > 0.0f)) return set_error(GLIDE_ERR_INVALID_ARG, "glide_ou_update: dt must be > 0");
    if (!a->sigma2 && !(a->sigma2_scalar >= 0.0f))
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_ou_update: sigma_w2 must be >= 0");
    ou_update_kernel<<<blocks_for(a->n), kThreads, 0, (cudaStream_t)stream>>>(*a);
    return check_launch("glide_ou_update");
}

extern "C" glide_status glide_displace_vertical(int64_t n, float* z, int64_t z_stride, const float* w, const float* dt,
                                                float dt_scalar, int32_t backward, void* stream) {
    if (glide_status st = check_n(n, "glide_displace_vertical")) return st;
    if (n == 0) return GLIDE_OK;
    if (!z || !w || z_stride < 1) return set_error(GLIDE_ERR_INVALID_ARG, "glide_displace_vertical: bad pointer or stride");
    if (!dt && !(dt_scalar > 0.0f)) return set_error(GLIDE_ERR_INVALID_ARG, "glide_displace_vertical: dt must be > 0");
    displace_vertical_kernel<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(n, z, z_stride, w, dt, dt_scalar,
                                                                                   backward ? -1.0f : 1.0f);
    return check_launch("glide_displace_vertical");
}

extern "C" glide_status glide_displace_horizontal(int64_t n, float* lon, float* lat, int64_t stride, const float* u,
                                                  const float* v, const float* dt, float dt_scalar, int32_t backward,
                                                  void* stream) {
    if (glide_status st = check_n(n, "glide_displace_horizontal")) return st;
    if (n == 0) return GLIDE_OK;
    if (!lon || !lat || !u || !v || stride < 1)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_displace_horizontal: bad pointer or stride");
    if (!dt && !(dt_scalar > 0.0f)) return set_error(GLIDE_ERR_INVALID_ARG, "glide_displace_horizontal: dt must be > 0");
    displace_horizontal_kernel<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(n, lon, lat, stride, u, v, dt,
                                                                                     dt_scalar, backward ? -1.0f : 1.0f);
    return check_launch("glide_displace_horizontal");
}

extern "C" glide_status glide_reflect_surface(int64_t n, float* z, int64_t z_stride, float* w, float z_surface,
                                              void* stream) {
    if (glide_status st = check_n(n, "glide_reflect_surface")) return st;
    if (n == 0) return GLIDE_OK;
    if (!z || !w || z_stride < 1) return set_error(GLIDE_ERR_INVALID_ARG, "glide_reflect_surface: bad pointer or stride");
    reflect_kernel<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(n, z, z_stride, w, z_surface);
    return check_launch("glide_reflect_surface");
}

extern "C" glide_status glide_rk2_stage(int64_t n, const float* x, int64_t x_stride, const float* v, int64_t v_stride,
                                        float h, float* out, int64_t out_stride, void* stream) {
    if (glide_status st = check_n(n, "glide_rk2_stage")) return st;
    if (n == 0) return GLIDE_OK;
    if (!x || !v || !out || x_stride < 3 || v_stride < 3 || out_stride < 3)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_rk2_stage: bad pointer or stride");
    rk2_stage_kernel<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(n, x, x_stride, v, v_stride, h, out,
                                                                           out_stride);
    return check_launch("glide_rk2_stage");
}
