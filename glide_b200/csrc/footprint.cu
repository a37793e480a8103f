// Stand-alone footprint scatter-add: FootprintGridder.accumulate
// (src/lpdm/footprint_gridder.py:117-197) for the per-step plug-in path, with
// the same warp-aggregated atomics as the fused step kernel.
#include "common.cuh"
#include "glide_internal.h"

namespace glide {

struct FpDev {
    int64_t n;
    const float* lon; const float* lat; const float* z; int64_t ps;
    const uint8_t* active; const float* w; int64_t ws;
    const int32_t* t_idx; const int32_t* rid;
    float dt;
    float lon0, lon_span, lat0, lat_span;
    int R, T, Z, Y, X;
    const float* edges;
    void* fp;
};

// V = float: the float32 gridder (w_eff = weight * dt in float32); V = double: the
// float64 gridder (weight * dt formed and summed in FP64)
template <typename V>
__global__ void footprint_kernel(const FpDev d) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = false;
    int64_t flat = -1;
    V w_eff = 0;
    if (i < d.n && (!d.active || d.active[i])) {
        const float lon = d.lon[i * d.ps], lat = d.lat[i * d.ps], z = d.z[i * d.ps];
        const float xf = floorf(((lon - d.lon0) / d.lon_span) * (float)d.X);
        const float yf = floorf(((lat - d.lat0) / d.lat_span) * (float)d.Y);
        int zb = -1;
        for (int e = 0; e <= d.Z; ++e) zb += (__ldg(d.edges + e) < z) ? 1 : 0;
        const int tb = d.t_idx[i];
        const int r = d.rid ? d.rid[i] : 0;
        valid = (r >= 0) && (r < d.R) && (xf >= 0.0f) && (xf < (float)d.X) && (yf >= 0.0f) && (yf < (float)d.Y) &&
                (zb >= 0) && (zb < d.Z) && (tb >= 0) && (tb < d.T);
        if (valid) {
            flat = ((((int64_t)r * d.T + tb) * d.Z + zb) * d.Y + (int64_t)yf) * d.X + (int64_t)xf;
            w_eff = (V)d.w[i * d.ws] * (V)d.dt;
        }
    }
    const unsigned vmask = __ballot_sync(0xffffffffu, valid);
    if (valid) {
        const unsigned peers = __match_any_sync(vmask, (unsigned long long)flat);
        V sum = 0;
        unsigned m = peers;
        while (m) {
            const int src = __ffs(m) - 1;
            m &= m - 1;
            sum += __shfl_sync(peers, w_eff, src);
        }
        if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(static_cast<V*>(d.fp) + flat, sum);
    }
}

}  // namespace glide

using namespace glide;

extern "C" glide_status glide_footprint_accumulate(int64_t n, const float* lon, const float* lat, const float* z,
                                                   int64_t pos_stride, const uint8_t* active, const float* weights,
                                                   int64_t weight_stride, const int32_t* t_idx,
                                                   const int32_t* release_idx, float dt_seconds,
                                                   const glide_footprint_grid* g, void* footprint, void* stream) {
    if (n < 0) return set_error(GLIDE_ERR_INVALID_ARG, "glide_footprint_accumulate: n < 0");
    if (n == 0) return GLIDE_OK;
    if (!lon || !lat || !z || !weights || !t_idx || !g || !footprint || !g->z_edges)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_footprint_accumulate: NULL pointer");
    if (g->n_releases < 1 || g->n_time_bins < 1 || g->n_z < 1 || g->n_y < 1 || g->n_x < 1)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_footprint_accumulate: empty grid");
    if (g->ring != 0)
        return set_error(GLIDE_ERR_UNSUPPORTED, "glide_footprint_accumulate: ring layout is only for glide_step");
    if (pos_stride < 1 || weight_stride < 1)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_footprint_accumulate: stride < 1");
    if (g->value_f64 && ((uintptr_t)footprint & 7u))
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_footprint_accumulate: float64 footprint not 8-byte aligned");
    FpDev d;
    d.n = n; d.lon = lon; d.lat = lat; d.z = z; d.ps = pos_stride;
    d.active = active; d.w = weights; d.ws = weight_stride; d.t_idx = t_idx; d.rid = release_idx;
    d.dt = dt_seconds;
    d.lon0 = (float)g->lon_min; d.lon_span = (float)fmax(1e-6, g->lon_max - g->lon_min);
    d.lat0 = (float)g->lat_min; d.lat_span = (float)fmax(1e-6, g->lat_max - g->lat_min);
    d.R = g->n_releases; d.T = g->n_time_bins; d.Z = g->n_z; d.Y = g->n_y; d.X = g->n_x;
    d.edges = g->z_edges; d.fp = footprint;
    const int threads = 256;
    const unsigned blocks = (unsigned)((n + threads - 1) / threads);
    if (g->value_f64) footprint_kernel<double><<<blocks, threads, 0, (cudaStream_t)stream>>>(d);
    else footprint_kernel<float><<<blocks, threads, 0, (cudaStream_t)stream>>>(d);
    return check_launch("glide_footprint_accumulate");
}
