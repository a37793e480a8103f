// Pressure-level -> terrain-following (AGL) vertical regrid of one met hour, on
// the device: the met reader's per-hour resampling (MetReader._resample_hour_to_agl,
// src/lpdm/met_reader.py:641-693, with lpdm/vertical_grid.py:166-318), which the
// reference runs on the host prefetch thread.
//
//   level_mean_kernel  bbox means of the first and last stored level: levels stored
//                      top-of-atmosphere first are read surface-first (flipped)
//   weights_kernel     per (target level, column), FP64: lower bracket by binary
//                      search (searchsorted, left) in the surface-first column,
//                      clamped to the first above-ground level and to Zp - 2;
//                      fraction (t - h_lo) / max(h_hi - h_lo, 1e-6) in [0, 1]
//   apply_kernel       per (channel, target level, column): the two bracketing
//                      levels in the stored order, torch.lerp (FMA form) with the
//                      fraction rounded to float32
//   slope_kernel       w -= taper(z) (u dh/dx + v dh/dy) in FP64 (a float32 slope's
//                      product in float32, as numpy promotes), rounded to float32
//   pressure_kernel    per target level: the regridded FP64 pressure's bbox mean
#include <cmath>

#include "common.cuh"
#include "glide_internal.h"

namespace glide {
namespace {

constexpr int kMaxAgl = GLIDE_REGRID_MAX_LEVELS;

struct RegridDev {
    int nc, zp, za;
    int64_t plane;
    const float* h;         // [zp][plane]
    const float* f;         // [nc][zp][plane]
    float* out;             // [nc][za][plane]
    const double* p;        // [zp][plane] or null
    double* p_level;        // [za]
    int ui, vi, wi;
    const double* dhdx; const double* dhdy;  // [plane]
    int slope_f32;                           // bit 0 / 1: the dhdx / dhdy product in float32
    int32_t* lower;         // [za][plane]
    double* frac;           // [za][plane]
    double* means;          // [2]
    double agl[kMaxAgl];
    double taper[kMaxAgl];
};

__device__ __forceinline__ bool flipped_of(const RegridDev& d) { return d.means[0] > d.means[1]; }

__global__ void level_mean_kernel(const __grid_constant__ RegridDev d) {
    __shared__ double s_sum[256];
    __shared__ double s_cnt[256];
    const int lev = blockIdx.x == 0 ? 0 : d.zp - 1;
    double s = 0.0, c = 0.0;
    for (int64_t k = threadIdx.x; k < d.plane; k += blockDim.x) {
        const float v = d.h[(int64_t)lev * d.plane + k];
        if (v == v) {
            s += (double)v;
            c += 1.0;
        }
    }
    s_sum[threadIdx.x] = s;
    s_cnt[threadIdx.x] = c;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off) {
            s_sum[threadIdx.x] += s_sum[threadIdx.x + off];
            s_cnt[threadIdx.x] += s_cnt[threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) d.means[blockIdx.x] = s_cnt[0] > 0.0 ? s_sum[0] / s_cnt[0] : NAN;
}

__global__ void weights_kernel(const __grid_constant__ RegridDev d) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)d.za * d.plane) return;
    const int a = (int)(t / d.plane);
    const int64_t col = t - (int64_t)a * d.plane;
    const bool flipped = flipped_of(d);
    const int zp = d.zp;
    auto row = [&](int k) -> double { return (double)d.h[(int64_t)(flipped ? zp - 1 - k : k) * d.plane + col]; };
    const double target = d.agl[a];
    int lo = 0, hi = zp;  // first index with row(i) >= target
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (row(mid) < target) lo = mid + 1; else hi = mid;
    }
    int k0 = 0;  // sub-surface (negative AGL) levels of the column
    for (int k = 0; k < zp; ++k) k0 += row(k) < 0.0 ? 1 : 0;
    const int lower = min(max(max(lo - 1, 0), k0), zp - 2);
    const double h_lo = row(lower), h_hi = row(lower + 1);
    const double span = h_hi - h_lo;
    double fr = (target - h_lo) / (span < 1e-6 ? 1e-6 : span);
    fr = fr < 0.0 ? 0.0 : (fr > 1.0 ? 1.0 : fr);
    d.lower[t] = lower;
    d.frac[t] = fr;
}

__global__ void apply_kernel(const __grid_constant__ RegridDev d) {
    const int64_t n = (int64_t)d.nc * d.za * d.plane;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int64_t per_c = (int64_t)d.za * d.plane;
    const int c = (int)(t / per_c);
    const int64_t r = t - (int64_t)c * per_c;  // (a, col)
    const int64_t col = r % d.plane;
    const int lower = d.lower[r];
    const bool flipped = flipped_of(d);
    const int lo = flipped ? (d.zp - 1) - lower : lower;
    const int hi = flipped ? lo - 1 : lo + 1;
    const float* fc = d.f + (int64_t)c * d.zp * d.plane;
    d.out[t] = torch_lerp(fc[(int64_t)lo * d.plane + col], fc[(int64_t)hi * d.plane + col], (float)d.frac[r]);
}

__global__ void slope_kernel(const __grid_constant__ RegridDev d) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)d.za * d.plane) return;
    const int a = (int)(t / d.plane);
    const int64_t col = t - (int64_t)a * d.plane;
    const int64_t per_c = (int64_t)d.za * d.plane;
    const double u = (double)d.out[(int64_t)d.ui * per_c + t];
    const double v = (double)d.out[(int64_t)d.vi * per_c + t];
    float* w = d.out + (int64_t)d.wi * per_c + t;
    // numpy's promotion: a float32 slope times the float32 channel is a float32 product
    const double px = (d.slope_f32 & 1) ? (double)((float)u * (float)d.dhdx[col]) : u * d.dhdx[col];
    const double py = (d.slope_f32 & 2) ? (double)((float)v * (float)d.dhdy[col]) : v * d.dhdy[col];
    const double slope = px + py;
    *w = (float)((double)*w - d.taper[a] * slope);
}

__device__ __forceinline__ double lerp64(double s, double e, double w) {
    const double diff = e - s;
    return (fabs(w) < 0.5) ? fma(w, diff, s) : fma(w - 1.0, diff, e);
}

__global__ void pressure_kernel(const __grid_constant__ RegridDev d) {
    __shared__ double s_sum[256];
    const int a = blockIdx.x;
    const bool flipped = flipped_of(d);
    double s = 0.0;
    for (int64_t col = threadIdx.x; col < d.plane; col += blockDim.x) {
        const int64_t r = (int64_t)a * d.plane + col;
        const int lower = d.lower[r];
        const int lo = flipped ? (d.zp - 1) - lower : lower;
        const int hi = flipped ? lo - 1 : lo + 1;
        s += lerp64(d.p[(int64_t)lo * d.plane + col], d.p[(int64_t)hi * d.plane + col], d.frac[r]);
    }
    s_sum[threadIdx.x] = s;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off) s_sum[threadIdx.x] += s_sum[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) d.p_level[a] = s_sum[0] / (double)d.plane;
}

size_t scratch_of(int za, int64_t plane) {
    return (size_t)za * (size_t)plane * (sizeof(int32_t) + sizeof(double)) + 4 * sizeof(double);
}

}  // namespace
}  // namespace glide

using namespace glide;

extern "C" glide_status glide_agl_regrid_scratch_bytes(int32_t za, int32_t ny, int32_t nx, size_t* bytes) {
    if (!bytes || za < 1 || ny < 1 || nx < 1)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_agl_regrid_scratch_bytes: bad sizes or NULL");
    *bytes = scratch_of(za, (int64_t)ny * nx);
    return GLIDE_OK;
}

extern "C" glide_status glide_agl_regrid(const glide_regrid_args* a, void* stream) {
    if (!a) return set_error(GLIDE_ERR_INVALID_ARG, "glide_agl_regrid: args is NULL");
    if (a->n_channels < 1 || a->zp < 2 || a->za < 1 || a->za > kMaxAgl || a->ny < 1 || a->nx < 1)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_agl_regrid: bad sizes (channels %d, zp %d, za %d <= %d)",
                         a->n_channels, a->zp, a->za, kMaxAgl);
    if (!a->height_agl_p || !a->fields_p || !a->fields_agl || !a->agl_levels || !a->scratch)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_agl_regrid: NULL pointer");
    for (int k = 1; k < a->za; ++k)
        if (!(a->agl_levels[k] > a->agl_levels[k - 1]))
            return set_error(GLIDE_ERR_INVALID_ARG, "glide_agl_regrid: agl_levels must be strictly ascending");
    const bool slope = a->w_channel >= 0;
    if (slope && (a->u_channel < 0 || a->v_channel < 0 || a->u_channel >= a->n_channels ||
                  a->v_channel >= a->n_channels || a->w_channel >= a->n_channels || !a->dhdx || !a->dhdy))
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_agl_regrid: slope correction needs u, v, w channels and slopes");
    if (a->pressure_p_hpa && !a->pressure_level_hpa)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_agl_regrid: pressure_level_hpa is NULL");
    if ((uintptr_t)a->scratch & 7u) return set_error(GLIDE_ERR_INVALID_ARG, "glide_agl_regrid: scratch misaligned");
    const int64_t plane = (int64_t)a->ny * a->nx;
    if (a->scratch_bytes < scratch_of(a->za, plane))
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_agl_regrid: scratch is %zu bytes, %zu needed", a->scratch_bytes,
                         scratch_of(a->za, plane));
    RegridDev d;
    d.nc = a->n_channels; d.zp = a->zp; d.za = a->za; d.plane = plane;
    d.h = a->height_agl_p; d.f = a->fields_p; d.out = a->fields_agl;
    d.p = a->pressure_p_hpa; d.p_level = a->pressure_level_hpa;
    d.ui = a->u_channel; d.vi = a->v_channel; d.wi = a->w_channel;
    d.dhdx = a->dhdx; d.dhdy = a->dhdy; d.slope_f32 = a->slope_f32;
    char* s = static_cast<char*>(a->scratch);
    d.frac = reinterpret_cast<double*>(s);
    d.means = d.frac + (size_t)a->za * plane;
    d.lower = reinterpret_cast<int32_t*>(d.means + 4);
    const double z_top = fmax(a->z_top_m, 1.0);
    for (int k = 0; k < kMaxAgl; ++k) {
        d.agl[k] = k < a->za ? a->agl_levels[k] : 0.0;
        const double tp = 1.0 - d.agl[k] / z_top;  // slope_correct_w's taper (vertical_grid.py:313)
        d.taper[k] = tp < 0.0 ? 0.0 : (tp > 1.0 ? 1.0 : tp);
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t n2 = (int64_t)a->za * plane, n3 = (int64_t)a->n_channels * n2;
    level_mean_kernel<<<2, 256, 0, st>>>(d);
    weights_kernel<<<(unsigned)((n2 + 255) / 256), 256, 0, st>>>(d);
    apply_kernel<<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(d);
    if (slope) slope_kernel<<<(unsigned)((n2 + 255) / 256), 256, 0, st>>>(d);
    if (a->pressure_p_hpa) pressure_kernel<<<(unsigned)a->za, 256, 0, st>>>(d);
    return check_launch("glide_agl_regrid");
}
