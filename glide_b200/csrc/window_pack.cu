// Per-window met packing: raw float32 snapshot fields -> the three bricks the
// step kernel gathers from.
//
//   wind    [nz][ny][nx][8]  u0 v0 w0 u1 v1 w1 0 0       (both snapshots in one record)
//   surf    [ny][nx][16]     blh sp ustar shf t_lowest 0 0 0 | same for the end snapshot
//   support [nz][ny][nx][8]  ft_sigma_w ft_T_Lw rho drho/dz meander_su meander_sv 0 0
//
// The support channels are the reference's per-window cached stacks, built
// at the window midpoint (HannaScheme._cached_window_field,
// src/lpdm/turbulence/hanna.py:1598-1633): the free-troposphere Richardson
// closure (_free_trop_fields :1694-1745 with the free functions :340-402),
// the density stack (_density_fields :1747-1784) and the meander sigmas
// (_meander_sigma_fields :1786-1830). Vertical gradients follow
// _vertical_gradient (:1855-1869).
#include <algorithm>

#include "common.cuh"
#include "glide_internal.h"

namespace glide {

template <typename T> struct PackScales {
    static constexpr float sp_store = 1.0f;
    static constexpr float drho_store = 1.0f;
};
template <> struct PackScales<__half> {  // keep sp (~1e5 Pa) and drho/dz (~1e-4) inside fp16's range
    static constexpr float sp_store = 0.01f;
    static constexpr float drho_store = 1e4f;
};

template <typename T>
__device__ __forceinline__ void store8(T* dst, const float v[8]) {
#pragma unroll
    for (int k = 0; k < 8; ++k) dst[k] = from_f<T>(v[k]);
}
template <>
__device__ __forceinline__ void store8<float>(float* dst, const float v[8]) {
    reinterpret_cast<float4*>(dst)[0] = make_float4(v[0], v[1], v[2], v[3]);
    reinterpret_cast<float4*>(dst)[1] = make_float4(v[4], v[5], v[6], v[7]);
}

struct PackDev {
    int nz, ny, nx;
    const float* u[2]; const float* v[2]; const float* w[2]; const float* t[2];
    const float* t_low[2]; const float* blh[2]; const float* sp[2]; const float* ustar[2]; const float* shf[2];
    const float* h3; const float* hlev; const float* p_hpa;
    float meander_coeff; int radius; int build_meander;
    void* wind; void* surf; void* support;
    double* wind_sum;
};

// Sums of u, v, w of both snapshots over every cell (the grid means of the per-step
// wind diagnostic, main.py:892-938): a grid-stride loop, warp and block reductions in
// FP64, one atomic per block and channel.
constexpr int kSumThreads = 256;
__global__ void __launch_bounds__(kSumThreads) wind_sum_kernel(const PackDev d) {
    __shared__ double s_part[kSumThreads / 32][6];
    const int64_t ncell = (int64_t)d.nz * d.ny * d.nx;
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (int64_t)gridDim.x * blockDim.x) {
        acc[0] += __ldg(d.u[0] + c);
        acc[1] += __ldg(d.v[0] + c);
        acc[2] += __ldg(d.w[0] + c);
        acc[3] += __ldg(d.u[1] + c);
        acc[4] += __ldg(d.v[1] + c);
        acc[5] += __ldg(d.w[1] + c);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        double v = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) s_part[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double v = 0.0;
        for (int w = 0; w < kSumThreads / 32; ++w) v += s_part[w][threadIdx.x];
        atomicAdd(d.wind_sum + threadIdx.x, v);
    }
}

template <typename T>
__global__ void pack_surf_kernel(const PackDev d) {
    const int64_t ncol = (int64_t)d.ny * d.nx;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncol; c += (int64_t)gridDim.x * blockDim.x) {
        T* dst = static_cast<T*>(d.surf) + c * 16;
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const float v[8] = {d.blh[s][c], d.sp[s][c] * PackScales<T>::sp_store, d.ustar[s][c], d.shf[s][c],
                                d.t_low[s][c], 0.0f, 0.0f, 0.0f};
            store8<T>(dst + 8 * s, v);
        }
    }
}

__device__ __forceinline__ float height_at(const PackDev& d, int k, int64_t col) {
    return d.h3 ? d.h3[(int64_t)k * d.ny * d.nx + col] : __ldg(d.hlev + k);
}

__device__ __forceinline__ float mid_at(const float* const f[2], int64_t idx) {
    return 0.5f * (f[0][idx] + f[1][idx]);  // _window_mid (hanna.py:1682-1692)
}

__device__ __forceinline__ float safe_den(float den) { return fabsf(den) < 1e-6f ? 1e-6f : den; }

constexpr int kTileX = 32, kTileY = 8;   // cells of one level per block
constexpr int kMaxTileRadius = 8;          // meander stencils up to this radius read a shared tile

// One thread per cell of a 32 x 8 tile of one level (blockIdx.z): the cell's wind
// record (both snapshots) and support record. The per-level pressures and theta
// factors are computed once per block; the meander stencil reads the level's
// mid-window u / v from a shared tile with a halo of the stencil radius, summed in
// the same row-major order as a direct loop, so the result does not depend on it.
template <typename T>
__global__ void __launch_bounds__(kTileX * kTileY) pack_cells_kernel(const PackDev d) {
    extern __shared__ float s_mid[];  // [2][th][tw]: mid-window u, then v
    __shared__ float s_lev[6];        // p (Pa) of k, ka, kb; (1e5 / p)^kappa of the same
    const int k = blockIdx.z;
    const int x = blockIdx.x * kTileX + threadIdx.x;
    const int y = blockIdx.y * kTileY + threadIdx.y;
    const int tid = threadIdx.y * kTileX + threadIdx.x;
    const int64_t plane = (int64_t)d.ny * d.nx;
    // one-sided at the ends, centred inside (hanna.py:1855-1869)
    const int ka = (k == 0) ? 1 : ((k == d.nz - 1) ? d.nz - 1 : k + 1);
    const int kb = (k == 0) ? 0 : ((k == d.nz - 1) ? d.nz - 2 : k - 1);
    const float kappa = (float)(287.05 / 1005.0);
    if (tid < 3) {
        const int kk = tid == 0 ? k : (tid == 1 ? ka : kb);
        const float pp = __ldg(d.p_hpa + kk) * 100.0f;
        s_lev[tid] = pp;
        s_lev[3 + tid] = powf(100000.0f / pp, kappa);
    }
    const int r = d.radius;
    const bool tiled = d.build_meander && r <= kMaxTileRadius;
    const int tw = kTileX + 2 * r, th = kTileY + 2 * r;
    const int x0 = blockIdx.x * kTileX - r, y0 = blockIdx.y * kTileY - r;
    if (tiled) {
        for (int q = tid; q < tw * th; q += kTileX * kTileY) {
            const int ty = q / tw, tx = q - ty * tw;
            const int gy = y0 + ty, gx = x0 + tx;
            float um = 0.0f, vm = 0.0f;
            if (gy >= 0 && gy < d.ny && gx >= 0 && gx < d.nx) {
                const int64_t idx = (int64_t)k * plane + (int64_t)gy * d.nx + gx;
                um = mid_at(d.u, idx);
                vm = mid_at(d.v, idx);
            }
            s_mid[q] = um;
            s_mid[tw * th + q] = vm;
        }
    }
    __syncthreads();
    if (x >= d.nx || y >= d.ny) return;
    const int64_t col = (int64_t)y * d.nx + x;
    const int64_t c = (int64_t)k * plane + col;
    {
        const float v[8] = {d.u[0][c], d.v[0][c], d.w[0][c], d.u[1][c], d.v[1][c], d.w[1][c], 0.0f, 0.0f};
        store8<T>(static_cast<T*>(d.wind) + c * 8, v);
    }
    const int64_t ia = (int64_t)ka * plane + col, ib = (int64_t)kb * plane + col;
    const float dh = safe_den(height_at(d, ka, col) - height_at(d, kb, col));
    const float pk = s_lev[0], pa = s_lev[1], pb = s_lev[2];
    const float tk = mid_at(d.t, c), ta = mid_at(d.t, ia), tb = mid_at(d.t, ib);
    // free troposphere: theta, N^2, shear, Ri, K_z, (sigma_w, T_Lw) (hanna.py:340-402, 1722-1742)
    const float th_k = tk * s_lev[3];
    const float th_a = ta * s_lev[4];
    const float th_b = tb * s_lev[5];
    const float n2 = (GRAVITY / fmaxf(th_k, 1.0f)) * ((th_a - th_b) / dh);
    const float du = (mid_at(d.u, ia) - mid_at(d.u, ib)) / dh;
    const float dv = (mid_at(d.v, ia) - mid_at(d.v, ib)) / dh;
    const float shear_sq = du * du + dv * dv;
    const float shear_mag = sqrtf(fmaxf(shear_sq, 1e-8f));
    const float ri = n2 / fmaxf(shear_sq, 1e-8f);
    const float zc = fmaxf(height_at(d, k, col), Z_MIN);
    const float ml = (KARMAN * zc) / (1.0f + (KARMAN * zc) / 100.0f);
    float fs = fmaxf(1.0f - ri / 0.25f, 0.0f);
    fs = fs * fs;
    const float fu = sqrtf(fmaxf(1.0f - 16.0f * ri, 0.0f));
    const float kz = fminf(fmaxf(((ml * ml) * shear_mag) * (ri < 0.0f ? fu : fs), 0.1f), 50.0f);
    const float tl = (n2 > 1e-6f) ? fminf(fmaxf(0.5f / sqrtf(fmaxf(n2, 1e-6f)), 1.0f), 1000.0f) : 100.0f;
    const float sw = sqrtf(fmaxf(kz / tl, SIGMA_MIN * SIGMA_MIN));
    // density and its vertical gradient (hanna.py:1778-1782)
    const float rho_k = pk / (R_DRY * fmaxf(tk, 1.0f));
    const float rho_a = pa / (R_DRY * fmaxf(ta, 1.0f));
    const float rho_b = pb / (R_DRY * fmaxf(tb, 1.0f));
    const float drho = (rho_a - rho_b) / dh;
    // meander: coefficient x local (2r+1)^2 std of the mid-window wind (hanna.py:1813-1830)
    float msu = 0.0f, msv = 0.0f;
    if (d.build_meander) {
        float su = 0.f, su2 = 0.f, sv = 0.f, sv2 = 0.f;
        int cnt = 0;
        for (int yy = max(y - r, 0); yy < min(y + r + 1, d.ny); ++yy) {
            for (int xx = max(x - r, 0); xx < min(x + r + 1, d.nx); ++xx) {
                float um, vm;
                if (tiled) {
                    const int q = (yy - y0) * tw + (xx - x0);
                    um = s_mid[q];
                    vm = s_mid[tw * th + q];
                } else {
                    const int64_t q = (int64_t)k * plane + (int64_t)yy * d.nx + xx;
                    um = mid_at(d.u, q);
                    vm = mid_at(d.v, q);
                }
                su += um; su2 += um * um;
                sv += vm; sv2 += vm * vm;
                ++cnt;
            }
        }
        const float fc = (float)cnt;
        const float mu = su / fc, mv = sv / fc;
        msu = d.meander_coeff * sqrtf(fmaxf(su2 / fc - mu * mu, 0.0f));
        msv = d.meander_coeff * sqrtf(fmaxf(sv2 / fc - mv * mv, 0.0f));
    }
    const float out[8] = {sw, tl, rho_k, drho * PackScales<T>::drho_store, msu, msv, 0.0f, 0.0f};
    store8<T>(static_cast<T*>(d.support) + c * 8, out);
}

static int elem_size(int32_t dt) {
    switch (dt) {
        case GLIDE_MET_F32: return 4;
        case GLIDE_MET_BF16: return 2;
        case GLIDE_MET_F16: return 2;
        default: return 0;
    }
}

template <typename T>
static glide_status launch_pack(const PackDev& d, cudaStream_t s) {
    const int threads = 256;
    const int64_t ncol = (int64_t)d.ny * d.nx;
    const unsigned b2 = (unsigned)std::min<int64_t>((ncol + threads - 1) / threads, 148 * 64);
    pack_surf_kernel<T><<<b2, threads, 0, s>>>(d);
    const dim3 grid((unsigned)((d.nx + kTileX - 1) / kTileX), (unsigned)((d.ny + kTileY - 1) / kTileY), (unsigned)d.nz);
    const bool tiled = d.build_meander && d.radius <= kMaxTileRadius;
    const size_t smem = tiled ? sizeof(float) * 2 * (size_t)(kTileX + 2 * d.radius) * (kTileY + 2 * d.radius) : 0;
    pack_cells_kernel<T><<<grid, dim3(kTileX, kTileY), smem, s>>>(d);
    if (d.wind_sum) wind_sum_kernel<<<148 * 2, kSumThreads, 0, s>>>(d);
    return check_launch("glide_window_pack");
}

}  // namespace glide

using namespace glide;

extern "C" glide_status glide_window_packed_bytes(int32_t nz, int32_t ny, int32_t nx, int32_t met_dtype,
                                                  size_t* wind_bytes, size_t* surf_bytes, size_t* support_bytes) {
    const int es = elem_size(met_dtype);
    if (es == 0) return set_error(GLIDE_ERR_UNSUPPORTED, "glide_window_packed_bytes: unknown met_dtype %d", met_dtype);
    if (nz < 2 || ny < 2 || nx < 2) return set_error(GLIDE_ERR_INVALID_ARG, "glide_window_packed_bytes: grid < 2");
    const size_t ncell = (size_t)nz * ny * nx;
    if (wind_bytes) *wind_bytes = ncell * 8 * es;
    if (surf_bytes) *surf_bytes = (size_t)ny * nx * 16 * es;
    if (support_bytes) *support_bytes = ncell * 8 * es;
    return GLIDE_OK;
}

extern "C" glide_status glide_window_pack(const glide_window_desc* w, void* stream) {
    if (!w) return set_error(GLIDE_ERR_INVALID_ARG, "glide_window_pack: desc is NULL");
    const glide_grid& g = w->grid;
    if (g.nz < 2 || g.ny < 2 || g.nx < 2) return set_error(GLIDE_ERR_INVALID_ARG, "glide_window_pack: grid < 2");
    for (int s = 0; s < 2; ++s) {
        if (!w->u[s] || !w->v[s] || !w->w[s] || !w->t[s] || !w->t_lowest[s] || !w->blh[s] || !w->sp[s] ||
            !w->ustar[s] || !w->shf[s])
            return set_error(GLIDE_ERR_INVALID_ARG, "glide_window_pack: a field pointer of snapshot %d is NULL", s);
    }
    if (!w->height3d && !w->height_level)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_window_pack: no height (height3d or height_level)");
    if (!w->pressure_hpa) return set_error(GLIDE_ERR_INVALID_ARG, "glide_window_pack: pressure_hpa is NULL");
    if (!w->wind_packed || !w->surf_packed || !w->support_packed)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_window_pack: an output brick is NULL");
    if (((uintptr_t)w->wind_packed | (uintptr_t)w->surf_packed | (uintptr_t)w->support_packed) & 15u)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_window_pack: output bricks must be 16-byte aligned");
    if ((uintptr_t)w->wind_sum & 7u)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_window_pack: wind_sum must be 8-byte aligned");
    if (w->build_meander && w->meander_radius < 1)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_window_pack: meander_radius must be >= 1");
    if (g.nz > 65535 || (g.ny + kTileY - 1) / kTileY > 65535)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_window_pack: grid %d x %d x %d too large", g.nz, g.ny, g.nx);
    PackDev d;
    d.nz = g.nz; d.ny = g.ny; d.nx = g.nx;
    for (int s = 0; s < 2; ++s) {
        d.u[s] = w->u[s]; d.v[s] = w->v[s]; d.w[s] = w->w[s]; d.t[s] = w->t[s]; d.t_low[s] = w->t_lowest[s];
        d.blh[s] = w->blh[s]; d.sp[s] = w->sp[s]; d.ustar[s] = w->ustar[s]; d.shf[s] = w->shf[s];
    }
    d.h3 = w->height3d; d.hlev = w->height_level; d.p_hpa = w->pressure_hpa;
    d.meander_coeff = w->meander_coefficient; d.radius = w->meander_radius; d.build_meander = w->build_meander;
    d.wind = w->wind_packed; d.surf = w->surf_packed; d.support = w->support_packed;
    d.wind_sum = w->wind_sum;
    cudaStream_t s = (cudaStream_t)stream;
    switch (w->met_dtype) {
        case GLIDE_MET_F32: return launch_pack<float>(d, s);
        case GLIDE_MET_BF16: return launch_pack<__nv_bfloat16>(d, s);
        case GLIDE_MET_F16: return launch_pack<__half>(d, s);
        default: return set_error(GLIDE_ERR_UNSUPPORTED, "glide_window_pack: unknown met_dtype %d", w->met_dtype);
    }
}
