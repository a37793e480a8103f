// Shared device helpers of the glide_b200 kernels.
//
// The whole library is compiled with -fmad=false so that a*b+c is rounded
// twice, as in torch's scalar CPU kernels that the reference runs; where
// torch's vectorised CPU kernels use a fused multiply-add (2-D bilinear
// grid_sample accumulation, torch.lerp) the code calls __fmaf_rn explicitly.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "glide_b200.h"

namespace glide {

// Physical constants (src/lpdm/turbulence/hanna.py:46-106).
constexpr float KARMAN = 0.4f;
constexpr double GRAVITY_D = 9.80665;
constexpr float GRAVITY = 9.80665f;
constexpr float R_DRY = 287.05f;
constexpr float C_P = 1005.0f;
constexpr double OMEGA_D = 7.2921e-5;
constexpr float SIGMA_MIN = 1e-3f;
constexpr float T_L_MIN = 1.0f;
constexpr float USTAR_MIN = 1e-3f;
constexpr float BLH_MIN = 50.0f;
constexpr float Z_MIN = 1.0f;
constexpr float M_PER_DEG_LAT = 110540.0f;
constexpr float M_PER_DEG_LON = 111320.0f;
// float32(pi / 180), the scalar torch.deg2rad multiplies by
constexpr float DEG2RAD = 0.017453292519943295f;

// ---------------------------------------------------------------------------
// packed met element types
// ---------------------------------------------------------------------------

template <typename T> struct MetType;
template <> struct MetType<float> { static constexpr int code = GLIDE_MET_F32; };
template <> struct MetType<__nv_bfloat16> { static constexpr int code = GLIDE_MET_BF16; };
template <> struct MetType<__half> { static constexpr int code = GLIDE_MET_F16; };

__device__ __forceinline__ float to_f(float x) { return x; }
__device__ __forceinline__ float to_f(__nv_bfloat16 x) { return __bfloat162float(x); }
__device__ __forceinline__ float to_f(__half x) { return __half2float(x); }

template <typename T> __device__ __forceinline__ T from_f(float x);
template <> __device__ __forceinline__ float from_f<float>(float x) { return x; }
template <> __device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float x) { return __float2bfloat16_rn(x); }
template <> __device__ __forceinline__ __half from_f<__half>(float x) { return __float2half_rn(x); }

// Eight consecutive packed values through the read-only path: two 128-bit
// loads for float32, one for 16-bit types. p must be 16-byte aligned.
__device__ __forceinline__ void load8(const float* p, float out[8]) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(p));
    const float4 b = __ldg(reinterpret_cast<const float4*>(p) + 1);
    out[0] = a.x; out[1] = a.y; out[2] = a.z; out[3] = a.w;
    out[4] = b.x; out[5] = b.y; out[6] = b.z; out[7] = b.w;
}
__device__ __forceinline__ void load8(const __nv_bfloat16* p, float out[8]) {
    const uint4 r = __ldg(reinterpret_cast<const uint4*>(p));
    const uint32_t w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        out[2 * i] = __uint_as_float(w[i] << 16);
        out[2 * i + 1] = __uint_as_float(w[i] & 0xffff0000u);
    }
}
__device__ __forceinline__ void load8(const __half* p, float out[8]) {
    const uint4 r = __ldg(reinterpret_cast<const uint4*>(p));
    const uint32_t w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const __half2 h = *reinterpret_cast<const __half2*>(&w[i]);
        const float2 f = __half22float2(h);
        out[2 * i] = f.x;
        out[2 * i + 1] = f.y;
    }
}

// ---------------------------------------------------------------------------
// Philox-4x32-10 counter-based generator (Salmon, Moraes, Dror & Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC11): ten rounds of the
// published multiply/xor round with the published multipliers and Weyl key
// increments.
// ---------------------------------------------------------------------------

struct U4 { uint32_t x, y, z, w; };

__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
    constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    constexpr uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
        const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += W0;
        k1 += W1;
    }
    return c;
}

// uniform in (0, 1): 24 random bits, centred in their bin
__device__ __forceinline__ float u01(uint32_t x) { return ((x >> 8) + 0.5f) * (1.0f / 16777216.0f); }

// two standard normals by the Box-Muller transform (hardware approximations of
// log and sin/cos: relative errors ~1e-6, far below what a Gaussian sample needs)
__device__ __forceinline__ float2 box_muller(uint32_t a, uint32_t b) {
    const float r = __fsqrt_rn(-2.0f * __logf(u01(a)));
    float s, c;
    __sincosf(6.2831853071795865f * u01(b) - 3.1415926535897932f, &s, &c);
    return make_float2(r * c, r * s);
}

// Philox streams used by the kernels (fourth counter word).
enum : uint32_t { STREAM_SUBSTEP = 0x10000u, STREAM_MEANDER = 0x20000u, STREAM_CONVECTION = 0x30000u,
                  STREAM_STEP = 0x40000u };

// Normal deviates of one particle-step: one Philox-4x32-10 block keyed by
// (particle, step) seeds a SplitMix64 sequence (Steele, Lea & Flood, "Fast
// splittable pseudorandom number generators", OOPSLA 2014: Weyl increment and
// the published two-multiply finaliser), whose 64-bit outputs feed Box-Muller
// pairs; the second deviate of a pair is kept for the next draw.
struct StepNormals {
    uint64_t s;
    float spare;
    bool has_spare;

    __device__ __forceinline__ StepNormals(uint64_t particle, uint32_t step, uint32_t k0, uint32_t k1) {
        const U4 r = philox4x32_10(U4{(uint32_t)particle, (uint32_t)(particle >> 32), step, STREAM_STEP}, k0, k1);
        s = ((uint64_t)r.y << 32 | r.x) ^ (((uint64_t)r.w << 32 | r.z) * 0x9E3779B97F4A7C15ull);
        has_spare = false;
        spare = 0.0f;
    }
    __device__ __forceinline__ uint64_t next64() {
        s += 0x9E3779B97F4A7C15ull;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    __device__ __forceinline__ float next() {
        if (has_spare) {
            has_spare = false;
            return spare;
        }
        const uint64_t z = next64();
        const float2 g = box_muller((uint32_t)z, (uint32_t)(z >> 32));
        spare = g.y;
        has_spare = true;
        return g.x;
    }
};

// ---------------------------------------------------------------------------
// Grid normalisation (src/lpdm/gpu_engine.py:210-299) and torch grid_sample
// index arithmetic (align_corners=True, zero padding).
// ---------------------------------------------------------------------------

struct GridDev {
    int nz, ny, nx;
    int ascending;
    float lon0, lon_span;  // float32(lon_first), float32(lon_last - lon_first)
    float lat0, lat_span;
    float zmax_idx;        // float32(nz - 1)
    const float* level;    // ascending [nz]
    const int32_t* lut;    // optional: lut[b] = searchsorted(level, b / lut_inv_dz)
    int lut_n;
    float lut_inv_dz;
};

__host__ inline GridDev make_grid_dev(const glide_grid& g) {
    GridDev d;
    d.nz = g.nz; d.ny = g.ny; d.nx = g.nx;
    d.ascending = g.ascending;
    d.lon0 = (float)g.lon_first;
    d.lon_span = (float)(g.lon_last - g.lon_first);
    d.lat0 = (float)g.lat_first;
    d.lat_span = (float)(g.lat_last - g.lat_first);
    d.zmax_idx = (float)(g.nz - 1);
    d.level = g.level_sorted;
    d.lut = g.level_lut;
    d.lut_n = g.lut_n;
    d.lut_inv_dz = g.lut_inv_dz;
    return d;
}

__device__ __forceinline__ float clamp11(float v) { return fminf(fmaxf(v, -1.0f), 1.0f); }

// normalised x or y: 2 ((v - v0) / span) - 1, clamped (gpu_engine.py:242-250, 298)
__device__ __forceinline__ float norm_h(float v, float v0, float span) {
    return clamp11(2.0f * ((v - v0) / span) - 1.0f);
}

// normalised z through the piecewise-linear level lookup (gpu_engine.py:263-293)
__device__ __forceinline__ float norm_z(float z, const GridDev& g) {
    const int n = g.nz;
    int lo;
    if (g.lut) {
        // searchsorted is monotone in z, so the table entry of the bucket below z's
        // (z * inv_dz may round up across a bucket edge) is a lower bound of the
        // answer; scan forward to the leftmost level >= z (NaN: 0, as below)
        const float fb = z * g.lut_inv_dz;
        const int b = (fb >= 1.0f) ? min((int)fb, g.lut_n) - 1 : 0;
        lo = __ldg(g.lut + b);
        while (lo < n && __ldg(g.level + lo) < z) ++lo;
    } else {
        lo = 0;
        int hi = n;
        while (lo < hi) {  // searchsorted(level, z), left insertion
            const int mid = (lo + hi) >> 1;
            if (__ldg(g.level + mid) < z) lo = mid + 1; else hi = mid;
        }
    }
    const int iu = min(max(lo, 1), n - 1);
    const int il = iu - 1;
    const float L_lo = __ldg(g.level + il);
    const float L_hi = __ldg(g.level + iu);
    const float frac = (z - L_lo) / fmaxf(L_hi - L_lo, 1e-6f);
    float fi = (float)il + fminf(fmaxf(frac, 0.0f), 1.0f);
    if (!g.ascending) fi = g.zmax_idx - fi;
    return clamp11(2.0f * fi / g.zmax_idx - 1.0f);
}

// grid_sample unnormalise, align_corners=True: ((c + 1) / 2) (size - 1)
__device__ __forceinline__ float unnorm(float c, float size_m1) { return ((c + 1.0f) / 2.0f) * size_m1; }

// Trilinear corner set of torch's 3-D CPU grid_sample: base indices (clamped
// so every gather stays in bounds; an out-of-grid corner only occurs at the
// exact upper edge, where its weight is exactly 0) and the eight weights in
// torch's order tnw, tne, tsw, tse, bnw, bne, bsw, bse.
struct Tri {
    int x0, y0, z0, x1, y1, z1;
    float w[8];
};

__device__ __forceinline__ void tri_weights(float ix, float iy, float iz, int nx, int ny, int nz, Tri& t) {
    const float fx0 = floorf(ix), fy0 = floorf(iy), fz0 = floorf(iz);
    const float fx1 = fx0 + 1.0f, fy1 = fy0 + 1.0f, fz1 = fz0 + 1.0f;
    t.w[0] = (fx1 - ix) * (fy1 - iy) * (fz1 - iz);
    t.w[1] = (ix - fx0) * (fy1 - iy) * (fz1 - iz);
    t.w[2] = (fx1 - ix) * (iy - fy0) * (fz1 - iz);
    t.w[3] = (ix - fx0) * (iy - fy0) * (fz1 - iz);
    t.w[4] = (fx1 - ix) * (fy1 - iy) * (iz - fz0);
    t.w[5] = (ix - fx0) * (fy1 - iy) * (iz - fz0);
    t.w[6] = (fx1 - ix) * (iy - fy0) * (iz - fz0);
    t.w[7] = (ix - fx0) * (iy - fy0) * (iz - fz0);
    const int xi = (int)fx0, yi = (int)fy0, zi = (int)fz0;
    t.x0 = min(max(xi, 0), nx - 1); t.x1 = min(max(xi + 1, 0), nx - 1);
    t.y0 = min(max(yi, 0), ny - 1); t.y1 = min(max(yi + 1, 0), ny - 1);
    t.z0 = min(max(zi, 0), nz - 1); t.z1 = min(max(zi + 1, 0), nz - 1);
}

// z-only part of the weights for a second query in the same (x, y) column
__device__ __forceinline__ void tri_weights_z(float ix, float iy, float iz, Tri& t) {
    const float fx0 = floorf(ix), fy0 = floorf(iy), fz0 = floorf(iz);
    const float fx1 = fx0 + 1.0f, fy1 = fy0 + 1.0f, fz1 = fz0 + 1.0f;
    t.w[0] = (fx1 - ix) * (fy1 - iy) * (fz1 - iz);
    t.w[1] = (ix - fx0) * (fy1 - iy) * (fz1 - iz);
    t.w[2] = (fx1 - ix) * (iy - fy0) * (fz1 - iz);
    t.w[3] = (ix - fx0) * (iy - fy0) * (fz1 - iz);
    t.w[4] = (fx1 - ix) * (fy1 - iy) * (iz - fz0);
    t.w[5] = (ix - fx0) * (fy1 - iy) * (iz - fz0);
    t.w[6] = (fx1 - ix) * (iy - fy0) * (iz - fz0);
    t.w[7] = (ix - fx0) * (iy - fy0) * (iz - fz0);
}

__device__ __forceinline__ int64_t cell_index(int z, int y, int x, int ny, int nx) {
    return ((int64_t)z * ny + y) * nx + x;
}

// torch.lerp(s, e, w) for a scalar weight (FMA form of the CPU kernel)
__device__ __forceinline__ float torch_lerp(float s, float e, float w) {
    const float d = e - s;
    return (fabsf(w) < 0.5f) ? __fmaf_rn(w, d, s) : __fmaf_rn(w - 1.0f, d, e);
}

// ---------------------------------------------------------------------------
// Particle-update arithmetic shared by the fused step kernel and the engine
// primitives (src/lpdm/gpu_engine.py:26-42, 345-507), in the reference's
// operation order.
// ---------------------------------------------------------------------------

// exact Ornstein-Uhlenbeck step: decay a = exp(-dt / T_L), noise amplitude
// sqrt(max(sigma^2 (1 - a^2), 0)), update a w + drift dt + amplitude eta
__device__ __forceinline__ float ou_decay(float dt, float tl) { return expf(-dt / tl); }
__device__ __forceinline__ float ou_amplitude(float sigma2, float a) { return sqrtf(fmaxf(sigma2 * (1.0f - a * a), 0.0f)); }
__device__ __forceinline__ float ou_step(float prev, float a, float drift_dt, float amp, float eta) {
    return (a * prev + drift_dt) + amp * eta;
}

// x / c for a constant c, given r = RN(1 / c): q = RN(x r) and one correction step
// q + RN(x - q c) r, both with fused multiply-adds (the division-by-a-known-divisor
// scheme of P. Markstein, "IA-64 and Elementary Functions", 2000). For the divisor
// used here (110540 m per degree of latitude) the result equals the IEEE quotient for
// every float32 with |x| in [2^-120, 2^120] (checked over all 2^32 inputs by the
// engine-primitive tests); zeros, tiny and huge values, infinities and NaN take the
// IEEE division.
__device__ __forceinline__ float div_known(float x, float c, float r) {
    const float ax = fabsf(x);
    if (ax >= 0x1p-120f && ax <= 0x1p120f) {
        const float q = __fmul_rn(x, r);
        return __fmaf_rn(__fmaf_rn(-q, c, x), r, q);
    }
    return x / c;
}
constexpr float INV_M_PER_DEG_LAT = (float)(1.0 / 110540.0);

// metres per degree of longitude at a latitude (cos clamped at 0.05)
__device__ __forceinline__ float m_per_deg_lon(float lat) { return M_PER_DEG_LON * fmaxf(fabsf(cosf(lat * DEG2RAD)), 0.05f); }

// displacement by a velocity over dt in the given direction (-1 backward, +1 forward)
__device__ __forceinline__ float displace_z(float z, float w, float dt, float dir) { return z + (dir * w) * dt; }
__device__ __forceinline__ float displace_lon(float lon, float u, float dt, float dir, float m_lon) {
    return lon + ((dir * u) * dt) / m_lon;
}
__device__ __forceinline__ float displace_lat(float lat, float v, float dt, float dir) {
    return lat + div_known((dir * v) * dt, M_PER_DEG_LAT, INV_M_PER_DEG_LAT);
}

// smooth-wall reflection at z_surface: (z, w) -> (2 z_surface - z, -w) below it
__device__ __forceinline__ void reflect_surface(float& z, float& w, float z_surface) {
    if (z < z_surface) {
        z = 2.0f * z_surface - z;
        w = -w;
    }
}

}  // namespace glide
