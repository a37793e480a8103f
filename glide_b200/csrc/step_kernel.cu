// Fused particle-step kernel: n_steps outer steps of GLIDE's static step body
// per launch, one thread per particle, particle state held in registers
// across steps.
//
// Per step (reference: src/lpdm/turbulence/hanna.py:898-1068 and the runtime
// body src/lpdm/main.py:1396-1477):
//   active mask -> RK2 midpoint advection through trilinear wind (two
//   snapshots lerped by alpha) -> bilinear surface fields (lerped) -> Obukhov
//   length / w* -> Hanna column turbulence at z_eval and z_eval +- 1 m (free
//   troposphere override from the support bricks) -> well-mixed + density
//   drift -> per-particle exact-OU substeps (clip, displacement, reflection)
//   -> meander OU -> [at the window's first step, when fused] convective
//   redistribution against the prebuilt column -> [post] time-ago bin, footprint
//   residence time (cached per particle, one atomic per change of cell), escape
//   kill.
//
// Threads map to particles through an optional permutation (the work-class
// order) and write each particle's work class for the next order. The same body
// runs as one batch per launch (step_kernel) or as several independent batches
// in one grouped launch (step_kernel_batched).
//
// Met is read from the packed per-window bricks (window_pack.cu): the wind
// brick holds u, v, w of both snapshots in one 32-byte (float32) or 16-byte
// (bf16/fp16) cell record, the support brick the six per-window support
// channels, so every trilinear corner is one or two 128-bit loads.
#include <cmath>
#include <cstdio>

#include "common.cuh"
#include "convect.cuh"
#include "glide_internal.h"

namespace glide {

template <typename T> struct Scales {
    static constexpr float sp = 1.0f;    // stored sp  = sp  / sp
    static constexpr float drho = 1.0f;  // stored drho = drho * drho_store
};
template <> struct Scales<__half> {
    static constexpr float sp = 100.0f;
    static constexpr float drho = 1e-4f;
};

struct StepDev {
    int64_t n;
    float* lon; float* lat; float* z; float* weight; int64_t ps;
    float* up; float* vp; float* wp; float* um; float* vm;
    const float* rel_off; const float* win_end_off; const int32_t* release_idx;
    uint8_t* alive; const uint8_t* active_mask;
    float sim_length;
    const void* wind; const void* surf; const void* support;
    GridDev g;
    float substep_c; int max_substeps; float z_ubl;
    int floors; int sl_override; int meander; float meander_T;
    const glide_step_sched* sched; glide_step_sched sched0;
    int n_steps, phys_begin, post_begin;
    const float* noise_sub; const float* noise_mea; uint32_t seed_lo, seed_hi;
    void* fp; int fp64;
    float fp_lon0, fp_lon_span, fp_lat0, fp_lat_span;
    int fp_R, fp_T, fp_Z, fp_Y, fp_X, fp_ring;
    const float* fp_edges;
    float dom_lon0, dom_lon1, dom_lat0, dom_lat1, dom_alt;
    int32_t* esc; int32_t* act;
    uint32_t* status;
    const int32_t* order; uint8_t* work_key;
    const double* conv_column; int conv_step, conv_nz; const float* conv_uniforms; int32_t* conv_moved;
    long long* diag;
};

// Dynamic shared memory of one block: when the launch sums the position diagnostic,
// [3] fixed-point position sums of the block's idle warps (constant over the launch)
// and [n_steps][3] fixed-point position sums of the others; then [2][n_steps] int32
// escaped / active counts.
__host__ __device__ inline size_t step_smem_bytes(int n_steps, bool diag) {
    return (diag ? sizeof(long long) * 3 * (size_t)(n_steps + 1) : 0) + sizeof(int32_t) * 2 * (size_t)n_steps;
}

// Sum over the 32 lanes of a converged warp of v quantised to 1 / scale (v * scale,
// scale a power of two, rounded to the nearest integer; |v * scale| < 2^31), exactly:
// the quantised values' high and low bits summed by two integer warp reductions.
// Integer sums do not depend on the order of the additions, so the diagnostic is the
// same from run to run and for any launch shape or particle order.
__device__ __forceinline__ long long warp_sum_fixed(float v, float scale) {
    const int q = __float2int_rn(v * scale);
    const int hi = __reduce_add_sync(0xffffffffu, q >> 12);  // floor(q / 4096): |hi| < 2^19, sum < 2^24
    const unsigned lo = __reduce_add_sync(0xffffffffu, (unsigned)(q & 0xfff));
    return ((long long)hi << 12) + (long long)lo;
}

// The three position sums of a warp (lanes without a particle add zero).
__device__ __forceinline__ void warp_position_sums(bool have, float lon, float lat, float z, long long* dst) {
    const long long sx = warp_sum_fixed(have ? lon : 0.0f, (float)GLIDE_DIAG_DEG_SCALE);
    const long long sy = warp_sum_fixed(have ? lat : 0.0f, (float)GLIDE_DIAG_DEG_SCALE);
    const long long sz = warp_sum_fixed(have ? z : 0.0f, (float)GLIDE_DIAG_M_SCALE);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(reinterpret_cast<unsigned long long*>(dst), (unsigned long long)sx);
        atomicAdd(reinterpret_cast<unsigned long long*>(dst + 1), (unsigned long long)sy);
        atomicAdd(reinterpret_cast<unsigned long long*>(dst + 2), (unsigned long long)sz);
    }
}

// Smallest and largest cursor offset of the launch's steps, in every lane of the warp.
__device__ __forceinline__ void launch_cursor_range(const StepDev& p, int lane, float& lo, float& hi) {
    if (!p.sched) {
        lo = hi = p.sched0.cursor_off;
        return;
    }
    float mn = INFINITY, mx = -INFINITY;
    for (int j = lane; j < p.n_steps; j += 32) {
        const float c = p.sched[j].cursor_off;
        mn = fminf(mn, c);
        mx = fmaxf(mx, c);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    lo = mn;
    hi = mx;
}

// One footprint cell's residence time accumulated in a register, added to the
// footprint (float32 or float64 values) with one atomic.
__device__ __forceinline__ void footprint_flush(const StepDev& p, int64_t cell, double acc) {
    if (p.fp64) atomicAdd(static_cast<double*>(p.fp) + cell, acc);
    else atomicAdd(static_cast<float*>(p.fp) + cell, (float)acc);
}

// ---------------------------------------------------------------------------
// Hanna column turbulence (hanna.py:192-337, 1500-1596)
// ---------------------------------------------------------------------------

struct Surface {
    float blh, ustar, w_star, hL, L, f_abs;
};

struct Sig6 {
    float su, sv, sw, tlu, tlv, tlw;
    int branch;  // which closure branch produced them: 0 stable, 1 neutral, 2-4 unstable (T_Lw forms)
};

// sigma_w of the three regimes (no surface-layer override)
__device__ __forceinline__ float sigma_w_bl(float z, const Surface& s) {
    const float blh = s.blh, us = s.ustar;
    if (s.hL > 1.0f) {
        const float zoh = fminf(fmaxf(z / blh, 0.0f), 1.0f);
        return (1.3f * us) * fmaxf(1.0f - zoh, 0.0f);
    }
    if (s.hL < -1.0f) {
        const float zoh = fminf(fmaxf(z / blh, 0.0f), 1.0f);
        const float sw2 = (((1.2f * (s.w_star * s.w_star)) * fmaxf(1.0f - 0.9f * zoh, 0.0f))
                           * powf(zoh, 2.0f / 3.0f)) + ((1.8f - 1.4f * zoh) * (us * us));
        return sqrtf(fmaxf(sw2, SIGMA_MIN * SIGMA_MIN));
    }
    return (1.3f * us) * expf(((-2.0f * s.f_abs) * z) / us);
}

// the other five outputs of the regimes given sw = sigma_w_bl(z, s)
__device__ __forceinline__ Sig6 in_bl(float z, const Surface& s, float sw) {
    Sig6 o;
    const float blh = s.blh, us = s.ustar;
    o.sw = sw;
    if (s.hL > 1.0f) {  // stable (hanna.py:192-222)
        o.branch = 0;
        const float zoh = fminf(fmaxf(z / blh, 0.0f), 1.0f);
        const float om = fmaxf(1.0f - zoh, 0.0f);
        o.su = (2.0f * us) * om;
        o.sv = o.sw;
        const float zf = fmaxf(zoh, 1e-6f);
        const float sq = sqrtf(zf);
        o.tlu = ((0.15f * blh) / fmaxf(o.su, SIGMA_MIN)) * sq;
        o.tlv = ((0.07f * blh) / fmaxf(o.sv, SIGMA_MIN)) * sq;
        o.tlw = ((0.10f * blh) / fmaxf(o.sw, SIGMA_MIN)) * powf(zf, 0.8f);
    } else if (s.hL < -1.0f) {  // unstable (hanna.py:255-298)
        const float zoh = fminf(fmaxf(z / blh, 0.0f), 1.0f);
        const float hl = fminf(fmaxf(s.hL, -1000.0f), 0.0f);
        o.su = powf(fmaxf(12.0f - 0.5f * hl, 1e-3f), 1.0f / 3.0f) * us;
        o.sv = o.su;
        o.tlu = (0.15f * blh) / fmaxf(o.su, SIGMA_MIN);
        o.tlv = o.tlu;
        const float azl = fmaxf(zoh * (-hl), 0.0f);
        const float swc = fmaxf(o.sw, SIGMA_MIN);
        if (azl < 1.0f) {
            o.branch = 2;
            o.tlw = (0.1f * z) / (swc * fmaxf(0.55f - 0.38f * azl, 1e-2f));
        } else if (zoh < 0.1f) {
            o.branch = 3;
            o.tlw = (0.59f * z) / swc;
        } else {
            o.branch = 4;
            o.tlw = ((0.15f * blh) / swc) * (1.0f - expf(-5.0f * zoh));
        }
    } else {  // neutral (hanna.py:225-252)
        o.branch = 1;
        const float fa = s.f_abs;
        o.su = (2.0f * us) * expf(((-3.0f * fa) * z) / us);
        o.sv = o.sw;
        const float den = 1.0f + (((15.0f * fa) * z) / us);
        o.tlw = ((0.5f * z) / fmaxf(o.sw, SIGMA_MIN)) / fmaxf(den, 1.0f);
        o.tlu = o.tlw;
        o.tlv = o.tlw;
    }
    return o;
}

// surface_layer_sigma_w (hanna.py:405-426)
__device__ __forceinline__ float sl_sigma_w(float z, float us, float L) {
    const bool finite = fabsf(L) > 1e-6f;
    const float Ls = finite ? L : 1.0f;
    const float zl = finite ? fminf(fmaxf(z / Ls, -50.0f), 50.0f) : 0.0f;
    return (zl < 0.0f) ? (1.3f * us) * powf(fmaxf(1.0f - 3.0f * zl, 1e-6f), 1.0f / 3.0f) : 1.3f * us;
}

// sigma_w alone of bl_profile (the z_eval +- 1 m probes of the well-mixed drift
// need nothing else; floors only touch the timescales)
__device__ __forceinline__ float bl_sigma_w(float z, const Surface& s, int sl_override) {
    if (sl_override && z < 0.1f * s.blh) return sl_sigma_w(z, s.ustar, s.L);
    return sigma_w_bl(z, s);
}

// BL profile + optional surface-layer override + FLEXPART floors, before the
// free-troposphere override (hanna.py:1529-1565)
__device__ __forceinline__ Sig6 bl_profile(float z, const Surface& s, int sl_override, int floors, float sw_z) {
    Sig6 o = in_bl(z, s, sw_z);
    if (sl_override) {
        const float z_sl = 0.1f * s.blh;
        if (z < z_sl) {
            const float zc = fmaxf(z, z_sl);
            const Sig6 c = in_bl(zc, s, sigma_w_bl(zc, s));
            o.su = c.su;
            o.sv = c.sv;
            o.sw = sl_sigma_w(z, s.ustar, s.L);
            const float zt = fmaxf(z, Z_MIN);
            o.tlu = (KARMAN * zt) / fmaxf(o.su, SIGMA_MIN);
            o.tlv = (KARMAN * zt) / fmaxf(o.sv, SIGMA_MIN);
            o.tlw = (KARMAN * zt) / fmaxf(o.sw, SIGMA_MIN);
        }
    }
    if (floors) {
        o.tlu = fmaxf(o.tlu, 10.0f);
        o.tlv = fmaxf(o.tlv, 10.0f);
        o.tlw = fmaxf(o.tlw, 30.0f);
    }
    return o;
}

// ---------------------------------------------------------------------------
// met sampling
// ---------------------------------------------------------------------------

// trilinear sample of the six leading channels of an 8-channel brick at
// (lon, lat, z) (torch grid_sample, align_corners=True, zero padding; the
// normalisation of gpu_engine.py:210-299); also returns the grid x / y indices
template <typename T>
__device__ __forceinline__ void sample6(const T* brick, const GridDev& g, float lon, float lat, float z, float acc[6],
                                        float& ix, float& iy) {
    ix = unnorm(norm_h(lon, g.lon0, g.lon_span), (float)(g.nx - 1));
    iy = unnorm(norm_h(lat, g.lat0, g.lat_span), (float)(g.ny - 1));
    Tri t;
    tri_weights(ix, iy, unnorm(norm_z(z, g), g.zmax_idx), g.nx, g.ny, g.nz, t);
#pragma unroll
    for (int k = 0; k < 6; ++k) acc[k] = 0.f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int zz = (c & 4) ? t.z1 : t.z0;
        const int yy = (c & 2) ? t.y1 : t.y0;
        const int xx = (c & 1) ? t.x1 : t.x0;
        float v[8];
        load8(brick + cell_index(zz, yy, xx, g.ny, g.nx) * 8, v);
#pragma unroll
        for (int k = 0; k < 6; ++k) acc[k] = acc[k] + v[k] * t.w[c];
    }
}

template <typename T>
__device__ __forceinline__ void surface_at(const StepDev& p, float lon, float lat, float alpha, float out[5]) {
    // _bilinear_at (hanna.py:1070-1085) of the lerped fields (hanna.py:805-813)
    const GridDev& g = p.g;
    const float xn = clamp11((2.0f * (lon - g.lon0)) / g.lon_span - 1.0f);
    const float yn = clamp11((2.0f * (lat - g.lat0)) / g.lat_span - 1.0f);
    const float ix = unnorm(xn, (float)(g.nx - 1));
    const float iy = unnorm(yn, (float)(g.ny - 1));
    const float fx = floorf(ix), fy = floorf(iy);
    const float w = ix - fx, e = 1.0f - w, nn = iy - fy, s = 1.0f - nn;
    const float wts[4] = {s * e, s * w, nn * e, nn * w};  // nw, ne, sw, se
    const int xi = (int)fx, yi = (int)fy;
    const int x0 = min(max(xi, 0), g.nx - 1), x1 = min(max(xi + 1, 0), g.nx - 1);
    const int y0 = min(max(yi, 0), g.ny - 1), y1 = min(max(yi + 1, 0), g.ny - 1);
    const T* sb = static_cast<const T*>(p.surf);
    float lerped[4][5];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int yy = (c & 2) ? y1 : y0;
        const int xx = (c & 1) ? x1 : x0;
        const T* rec = sb + ((int64_t)yy * g.nx + xx) * 16;
        float a[8], b[8];
        load8(rec, a);
        load8(rec + 8, b);
#pragma unroll
        for (int f = 0; f < 5; ++f) lerped[c][f] = torch_lerp(a[f], b[f], alpha);
    }
#pragma unroll
    for (int f = 0; f < 5; ++f) {
        out[f] = __fmaf_rn(lerped[3][f], wts[3],
                           __fmaf_rn(lerped[2][f], wts[2], __fmaf_rn(lerped[1][f], wts[1], lerped[0][f] * wts[0])));
    }
    out[1] *= Scales<T>::sp;
}

// ---------------------------------------------------------------------------
// the kernel
// ---------------------------------------------------------------------------

__device__ __forceinline__ float noise_or_philox(const StepDev& p, const float* base, int64_t idx, float philox) {
    return base ? __ldg(base + idx) : philox;
}

// Launch shapes (threads per block, resident blocks per SM the register budget
// is compiled for). Variant 0, 128 x 6 (<= 80 registers, 24 warps per SM), is
// the measured default; the others exist for the autotuner: the best shape
// depends on the particle count (wave quantisation of a batch across 148 SMs) and
// on the trade between resident warps and spills (128 x 7 and 896 x 1 cap the
// kernel at 72 registers, 28 warps per SM, with a few spilled values).
struct LaunchShape { int threads, min_blocks; };
constexpr LaunchShape kShapes[] = {{128, 6}, {64, 12}, {256, 3}, {128, 5}, {128, 8}, {768, 1}, {128, 7}, {896, 1}};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);
// variant kNumShapes: the general kernel at shape 0 whatever the arguments
constexpr int kNumVariants = kNumShapes + 1;

// GENERAL = false compiles out the paths the production configuration never
// takes (surface-layer override, injected noise, caller-supplied active mask):
// the kernel is smaller, which matters because it is bound by instruction
// issue and instruction-cache misses. Arguments that need one of those paths
// run the GENERAL = true instantiation; both compute identical results.
// The whole launch body for one batch; `block` is the block's index within the batch.
template <typename T, bool GENERAL>
__device__ __forceinline__ void step_body(const StepDev& p, int64_t block) {
    extern __shared__ long long s_dyn[];
    long long* const s_static = s_dyn;     // [3] when p.diag
    long long* const s_diag = s_dyn + 3;   // [n_steps][3] when p.diag
    int32_t* const s_counts = reinterpret_cast<int32_t*>(s_dyn + (p.diag ? 3 * (p.n_steps + 1) : 0));  // [2][n_steps]
    const int64_t th = block * blockDim.x + threadIdx.x;
    bool have = th < p.n;
    bool bad_order = false;
    int64_t i = th;  // the particle this thread steps
    if (have && p.order) {
        const int64_t o = p.order[th];
        if (o >= 0 && o < p.n) i = o;
        else { have = false; bad_order = true; }
    }
    const int lane = threadIdx.x & 31;
    for (int k = threadIdx.x; k < 2 * p.n_steps; k += blockDim.x) s_counts[k] = 0;
    if (p.diag)
        for (int k = threadIdx.x; k < 3 * (p.n_steps + 1); k += blockDim.x) s_dyn[k] = 0;
    __syncthreads();

    float lon = 0.f, lat = 0.f, z = 0.f, wgt = 0.f, up = 0.f, vp = 0.f, wp = 0.f, um = 0.f, vm = 0.f;
    float rel = 0.f, wend = 0.f;
    int rid = 0;
    bool alive = false;
    if (have) {
        lon = p.lon[i * p.ps];
        lat = p.lat[i * p.ps];
        z = p.z[i * p.ps];
        wgt = p.weight[i * p.ps];
        up = p.up[i];
        vp = p.vp[i];
        wp = p.wp[i];
        if (p.meander) { um = p.um[i]; vm = p.vm[i]; }
        rel = p.rel_off ? p.rel_off[i] : 0.f;
        wend = p.win_end_off ? p.win_end_off[i] : 0.f;
        rid = p.release_idx ? p.release_idx[i] : 0;
        alive = p.alive ? (p.alive[i] != 0) : true;
    }
    const float L_sim = p.sim_length;
    const int ms = p.max_substeps;
    bool nonfinite = false;
    // footprint cache: a particle stays in one output cell for many steps, so its
    // residence time accumulates in a register (FP64) and goes to global memory (one
    // atomic) only when the cell (or time bin) changes, and at the end of the launch
    int64_t fp_cell = -1;
    double fp_acc = 0.0;
    int last_k = 1;         // work class of the last physics step (work key)
    bool last_active = false;

    // A warp whose particles are all inactive at every step of the launch (absent,
    // escaped, past the simulation length at the launch's latest cursor, or not yet
    // released at its earliest) has nothing to step: it skips the step loop, adds its
    // unchanged positions to the diagnostic once for all steps, and writes its keys.
    bool idle_warp = false;
    if (!(GENERAL && p.active_mask)) {
        float c_lo, c_hi;
        launch_cursor_range(p, lane, c_lo, c_hi);
        const bool idle = !have || !alive || ((rel - L_sim) > c_hi) || !(rel >= c_lo);
        idle_warp = __all_sync(0xffffffffu, idle);
    }
    if (idle_warp) {
        if (p.diag) warp_position_sums(have, lon, lat, z, s_static);
        if (have && p.work_key) {
            const glide_step_sched sl = p.sched ? p.sched[p.n_steps - 1] : p.sched0;
            p.work_key[i] = (uint8_t)((alive && !(rel >= sl.cursor_off)) ? GLIDE_WORK_PENDING : GLIDE_WORK_DONE);
        }
    } else {
        for (int j = 0; j < p.n_steps; ++j) {
            const glide_step_sched sc = p.sched ? p.sched[j] : p.sched0;
            bool active;
            if (GENERAL && p.active_mask) active = have && p.active_mask[i] != 0;
            else active = have && alive && (rel >= sc.cursor_off) && ((rel - L_sim) <= sc.cursor_off);
            last_active = active;

            if (j >= p.phys_begin && active) {
                const float delta = sc.delta, alpha = sc.alpha;
                // --- RK2 midpoint advection, backward (hanna.py:855-896), then the support
                // brick at z_eval. One sampling loop serves all three trilinear samples (one
                // copy of the level search and gather in the code): stage 0 the wind at the
                // start point, stage 1 at the midpoint (hanna.py:866-889, two snapshots lerped
                // by alpha), stage 2 the support brick (FT sigma_w / T_Lw, rho, drho/dz,
                // meander sigmas) at the advected position and z_eval = max(z, z_ubl).
                const GridDev& g = p.g;
                const float z_ubl = p.z_ubl;
                float acc[6];
                float ix, iy;
                {
                    const float hd = 0.5f * delta;
                    float qx = lon, qy = lat, qz = z;
#pragma unroll 1
                    for (int stage = 0; stage < 3; ++stage) {
                        sample6<T>(static_cast<const T*>(stage < 2 ? p.wind : p.support), g, qx, qy, qz, acc, ix, iy);
                        if (stage < 2) {
                            const float om = 1.0f - alpha;
                            const float u = acc[0] * om + acc[3] * alpha;
                            const float vv = acc[1] * om + acc[4] * alpha;
                            const float w = acc[2] * om + acc[5] * alpha;
                            const float vx = u / m_per_deg_lon(qy);
                            const float vy = div_known(vv, M_PER_DEG_LAT, INV_M_PER_DEG_LAT);
                            if (stage == 0) {
                                qx = lon - hd * vx;
                                qy = lat - hd * vy;
                                qz = z - hd * w;
                            } else {
                                lon = lon - delta * vx;
                                lat = lat - delta * vy;
                                z = z - delta * w;
                                qx = lon;
                                qy = lat;
                                qz = fmaxf(z, z_ubl);
                            }
                        }
                    }
                }
                const float z_eval = fmaxf(z, z_ubl);
                const float ft_sw = acc[0], ft_tl = acc[1];
                const float rho_p = acc[2];
                const float drho_p = acc[3] * Scales<T>::drho;
                const float m_su = acc[4], m_sv = acc[5];

                // --- surface fields and stability (hanna.py:950-966, 142-189)
                float sf[5];
                surface_at<T>(p, lon, lat, alpha, sf);
                Surface S;
                S.blh = fmaxf(sf[0], BLH_MIN);
                const float sp_ = sf[1];
                S.ustar = fmaxf(sf[2], USTAR_MIN);
                const float shf = sf[3], ts = sf[4];
                {
                    const float rho = sp_ / (R_DRY * ts);
                    const float denom = (float)(0.4 * GRAVITY_D) * shf;
                    const float num = -(S.ustar * S.ustar * S.ustar) * ts * rho * C_P;
                    S.L = (fabsf(denom) > 1e-10f) ? num / denom : INFINITY;
                    S.hL = S.blh / S.L;
                    const float cube = ((GRAVITY * S.blh) * shf) / ((ts * rho) * C_P);
                    S.w_star = (cube > 0.0f) ? powf(fmaxf(cube, 0.0f), 1.0f / 3.0f) : 0.0f;
                    const float f_cor = (float)(2.0 * OMEGA_D) * sinf(lat * DEG2RAD);
                    S.f_abs = fmaxf(fabsf(f_cor), 1e-5f);
                }

                // --- sigma_w: the BL profile's at z_eval (column turbulence) and the closure's
                // at z_eval +- 1 m for the well-mixed drift (hanna.py:984-991; above the BL the
                // free-troposphere value from the support brick's channel 0). One rolled loop
                // keeps one copy of the regime code.
                const int sl = GENERAL ? p.sl_override : 0;
                const float z_hi = z_eval + 1.0f;
                const float z_lo = fmaxf(z_eval - 1.0f, z_ubl);
                float sw_col = 0.f, sw_hi = 0.f, sw_lo = 0.f;
#pragma unroll 1
                for (int q = 0; q < 3; ++q) {
                    const float zq = q == 0 ? z_eval : (q == 1 ? z_hi : z_lo);
                    float s = bl_sigma_w(zq, S, q == 0 ? 0 : sl);
                    if (q > 0 && zq > S.blh) {
                        const float izq = unnorm(norm_z(zq, g), g.zmax_idx);
                        Tri tq;
                        tri_weights(ix, iy, izq, g.nx, g.ny, g.nz, tq);
                        const T* sup = static_cast<const T*>(p.support);
                        float a = 0.f;
#pragma unroll
                        for (int c = 0; c < 8; ++c) {
                            const int zz = (c & 4) ? tq.z1 : tq.z0;
                            const int yy = (c & 2) ? tq.y1 : tq.y0;
                            const int xx = (c & 1) ? tq.x1 : tq.x0;
                            a = a + to_f(sup[cell_index(zz, yy, xx, g.ny, g.nx) * 8]) * tq.w[c];
                        }
                        s = a;
                    }
                    if (q == 0) sw_col = s;
                    else if (q == 1) sw_hi = fmaxf(s, SIGMA_MIN);
                    else sw_lo = fmaxf(s, SIGMA_MIN);
                }

                // --- column turbulence at z_eval (hanna.py:976-982)
                Sig6 col = bl_profile(z_eval, S, sl, p.floors, sw_col);
                if (z_eval > S.blh) {
                    col.su = ft_sw; col.sv = ft_sw; col.sw = ft_sw;
                    col.tlu = ft_tl; col.tlv = ft_tl; col.tlw = ft_tl;
                }
                const float su = fmaxf(col.su, SIGMA_MIN), sv = fmaxf(col.sv, SIGMA_MIN), sw = fmaxf(col.sw, SIGMA_MIN);
                const float tlu = fmaxf(col.tlu, T_L_MIN), tlv = fmaxf(col.tlv, T_L_MIN), tlw = fmaxf(col.tlw, T_L_MIN);

                const float dsig2 = (sw_hi * sw_hi - sw_lo * sw_lo) / fmaxf(z_hi - z_lo, 1.0f);
                const float sw_sq = fmaxf(sw * sw, SIGMA_MIN * SIGMA_MIN);

                // --- density drift (hanna.py:993-1006)
                const float rho_c = fmaxf(rho_p, 1e-3f);
                const float drift_fwd = (sw_sq * drho_p) / rho_c;
                const float half_bwd = -0.5f * dsig2;
                const float dens_bwd = -drift_fwd;

                // --- substep count (hanna.py:1162-1186)
                const float kq = ceilf(delta / (p.substep_c * fmaxf(tlw, 1e-3f)));
                int k = (kq >= (float)ms) ? ms : ((kq >= 1.0f) ? (int)kq : 1);
                if (!(kq == kq)) k = 1;  // NaN
                const float sub_dt = delta / (float)k;
                // work class of this step (glide_step_args.work_key): the stability regime, the
                // height band of z_eval within (or above) the BL and the substep count. Height
                // bands rather than the closure's branches: a particle's branch and its BL/FT
                // side follow its height relative to the BL top, which drifts within a window,
                // so warps built from neighbouring bands stay converged longer
                {
                    const float hr = z_eval / S.blh;
                    const int band = hr < 0.25f ? 0 : (hr < 0.5f ? 1 : (hr < 0.8f ? 2 : (hr <= 1.0f ? 3 : 4)));
                    const int regime = S.hL > 1.0f ? 0 : (S.hL < -1.0f ? 2 : 1);
                    last_k = 1 + (min(k, 3) - 1) + 3 * (band + 5 * regime);
                }

                // --- exact-OU substeps (hanna.py:1224-1368, gpu_engine.py:26-42, 400-507)
                const float su2 = su * su, sv2 = sv * sv, sw2 = sw * sw;
                const float umax = 4.0f * su, vmax = 4.0f * sv, wmax = 4.0f * sw;
                const float au = ou_decay(sub_dt, tlu), av = ou_decay(sub_dt, tlv), aw = ou_decay(sub_dt, tlw);
                const float ru = ou_amplitude(su2, au), rv = ou_amplitude(sv2, av), rw = ou_amplitude(sw2, aw);
                const int64_t nn = p.n;
                StepNormals rng((uint64_t)i, (uint32_t)sc.step_index, p.seed_lo, p.seed_hi);
                for (int it = 0; it < k; ++it) {
                    float eu, ev, ew;
                    if (GENERAL && p.noise_sub) {
                        const float* b = p.noise_sub + ((int64_t)(j * ms + it) * 3) * nn + i;
                        eu = __ldg(b);
                        ev = __ldg(b + nn);
                        ew = __ldg(b + 2 * nn);
                    } else {
                        eu = rng.next();
                        ev = rng.next();
                        ew = rng.next();
                    }
                    const float factor = 1.0f + (wp * wp) / sw_sq;
                    const float drift_w = factor * half_bwd + dens_bwd;
                    float un = ou_step(up, au, 0.0f * sub_dt, ru, eu);
                    float vn = ou_step(vp, av, 0.0f * sub_dt, rv, ev);
                    float wn = ou_step(wp, aw, drift_w * sub_dt, rw, ew);
                    wn = fminf(fmaxf(wn, -wmax), wmax);
                    un = fminf(fmaxf(un, -umax), umax);
                    vn = fminf(fmaxf(vn, -vmax), vmax);
                    z = displace_z(z, wn, sub_dt, -1.0f);
                    lon = displace_lon(lon, un, sub_dt, -1.0f, m_per_deg_lon(lat));
                    lat = displace_lat(lat, vn, sub_dt, -1.0f);
                    reflect_surface(z, wn, 0.0f);
                    up = un; vp = vn; wp = wn;
                }

                // --- meander (hanna.py:1028-1054)
                if (p.meander) {
                    float e0, e1;
                    if (GENERAL && p.noise_mea) {
                        const float* b = p.noise_mea + ((int64_t)j * 2) * nn + i;
                        e0 = __ldg(b);
                        e1 = __ldg(b + nn);
                    } else {
                        e0 = rng.next();
                        e1 = rng.next();
                    }
                    const float am = ou_decay(delta, p.meander_T);
                    const float umn = ou_step(um, am, 0.0f * delta, ou_amplitude(m_su * m_su, am), e0);
                    const float vmn = ou_step(vm, am, 0.0f * delta, ou_amplitude(m_sv * m_sv, am), e1);
                    lon = displace_lon(lon, umn, delta, -1.0f, m_per_deg_lon(lat));
                    lat = displace_lat(lat, vmn, delta, -1.0f);
                    um = umn; vm = vmn;
                }
                nonfinite |= !(isfinite(lon) && isfinite(lat) && isfinite(z) && isfinite(up) && isfinite(vp) &&
                               isfinite(wp));
            }

            // --- the window's convection, fused: after the physics of its first step, before
            // that step's footprint and escape kill (main.py:1446-1458, emanuel.py:772-805)
            if (p.conv_column && j == p.conv_step) {
                bool moved = false;
                if (active) {
                    double u1, u2;
                    if (GENERAL && p.conv_uniforms) {
                        u1 = (double)p.conv_uniforms[i];
                        u2 = (double)p.conv_uniforms[p.n + i];
                    } else {
                        convection_uniforms(i, (uint32_t)sc.step_index, p.seed_lo, p.seed_hi, u1, u2);
                    }
                    moved = convect_particle(p.conv_column, p.conv_nz, z, u1, u2);
                }
                const int n_mv = __popc(__ballot_sync(0xffffffffu, moved));
                if (p.conv_moved && lane == 0 && n_mv) atomicAdd(p.conv_moved, n_mv);
            }

            if (j >= p.post_begin) {
                // --- time-ago bin (main.py:1459-1465) and footprint (footprint_gridder.py:154-197)
                bool valid = false;
                int64_t flat = -1;
                if (active && p.fp) {
                    const float el = fmaxf(wend - sc.cursor_off, 0.0f);
                    int tb = (int)floorf(el / 3600.0f);
                    if (p.fp_T == 1) tb = min(tb, 0);
                    const float xf = floorf(((lon - p.fp_lon0) / p.fp_lon_span) * (float)p.fp_X);
                    const float yf = floorf(((lat - p.fp_lat0) / p.fp_lat_span) * (float)p.fp_Y);
                    int zb = 0;
#pragma unroll 1
                    for (int e = 0; e <= p.fp_Z; ++e) zb += (__ldg(p.fp_edges + e) < z) ? 1 : 0;
                    zb -= 1;
                    valid = (rid >= 0) && (rid < p.fp_R) && (xf >= 0.0f) && (xf < (float)p.fp_X) && (yf >= 0.0f) &&
                            (yf < (float)p.fp_Y) && (zb >= 0) && (zb < p.fp_Z) && (tb >= 0) && (tb < p.fp_T);
                    if (valid) {
                        const int slot = p.fp_ring > 0 ? tb % p.fp_ring : tb;
                        const int n_slot = p.fp_ring > 0 ? p.fp_ring : p.fp_T;
                        flat = ((((int64_t)rid * n_slot + slot) * p.fp_Z + zb) * p.fp_Y + (int64_t)yf) * p.fp_X +
                               (int64_t)xf;
                    }
                }
                // weight * dt: a float32 product (the float32 gridder's w_eff) or an FP64 one
                const double w_dt = p.fp64 ? (double)wgt * (double)sc.delta : (double)(wgt * sc.delta);
                if (valid && flat == fp_cell) {
                    fp_acc += w_dt;
                } else {
                    if (fp_cell >= 0) footprint_flush(p, fp_cell, fp_acc);
                    fp_cell = valid ? flat : -1;
                    fp_acc = valid ? w_dt : 0.0;
                }
                // --- escape kill (main.py:690-711, 1475-1477)
                bool escaped = false;
                if (active) {
                    const bool within = (lon >= p.dom_lon0) && (lon <= p.dom_lon1) && (lat >= p.dom_lat0) &&
                                        (lat <= p.dom_lat1) && (z <= p.dom_alt);
                    escaped = !within;
                    if (escaped) alive = false;
                }
                const int n_esc = __popc(__ballot_sync(0xffffffffu, escaped));
                const int n_act = __popc(__ballot_sync(0xffffffffu, active));
                if (lane == 0) {
                    if (n_esc) atomicAdd(&s_counts[j], n_esc);
                    if (n_act) atomicAdd(&s_counts[p.n_steps + j], n_act);
                }
                // --- mean-position diagnostic (main.py:1565-1566): sums over every particle
                if (p.diag) warp_position_sums(have, lon, lat, z, s_diag + 3 * j);
            }
        }

        if (fp_cell >= 0) footprint_flush(p, fp_cell, fp_acc);
        if (have) {
            p.lon[i * p.ps] = lon;
            p.lat[i * p.ps] = lat;
            p.z[i * p.ps] = z;
            p.up[i] = up;
            p.vp[i] = vp;
            p.wp[i] = wp;
            if (p.meander) { p.um[i] = um; p.vm[i] = vm; }
            if (p.alive) p.alive[i] = alive ? 1 : 0;
            if (nonfinite && p.status) atomicOr(p.status, (uint32_t)GLIDE_STATUS_NONFINITE_STATE);
            if (p.work_key) {
                int key = GLIDE_WORK_DONE;
                if (alive) {
                    const glide_step_sched sl = p.sched ? p.sched[p.n_steps - 1] : p.sched0;
                    if (!(GENERAL && p.active_mask) && !(rel >= sl.cursor_off)) key = GLIDE_WORK_PENDING;
                    else if (last_active) key = last_k;
                }
                p.work_key[i] = (uint8_t)key;
            }
        }
    }
    if (bad_order && p.status) atomicOr(p.status, (uint32_t)GLIDE_STATUS_BAD_ORDER);
    __syncthreads();
    for (int k = threadIdx.x; k < p.n_steps; k += blockDim.x) {
        if (p.esc && s_counts[k]) atomicAdd(p.esc + k, s_counts[k]);
        if (p.act && s_counts[p.n_steps + k]) atomicAdd(p.act + k, s_counts[p.n_steps + k]);
    }
    if (p.diag)
        for (int k = threadIdx.x + p.post_begin * 3; k < 3 * p.n_steps; k += blockDim.x)
            atomicAdd(reinterpret_cast<unsigned long long*>(p.diag + k),
                      (unsigned long long)(s_diag[k] + s_static[k % 3]));
}

template <typename T, int THREADS, int MIN_BLOCKS, bool GENERAL>
__global__ void __launch_bounds__(THREADS, MIN_BLOCKS) step_kernel(const StepDev p) {
    step_body<T, GENERAL>(p, blockIdx.x);
}

// Several independent batches (own particles, schedule, met window, footprint) in
// one launch: batch k owns blocks [block_start[k], block_start[k + 1]).
struct StepBatch {
    StepDev d[GLIDE_STEP_BATCH_MAX];
    uint32_t block_start[GLIDE_STEP_BATCH_MAX + 1];
    int count;
};

template <typename T, bool GENERAL>
__global__ void __launch_bounds__(128, 6) step_kernel_batched(const __grid_constant__ StepBatch b) {
    int lo = 0, hi = b.count - 1;  // the last batch starting at or before this block (skips empty ones)
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (b.block_start[mid] <= blockIdx.x) lo = mid; else hi = mid - 1;
    }
    step_body<T, GENERAL>(b.d[lo], (int64_t)(blockIdx.x - b.block_start[lo]));
}

template <typename T, int V, bool GENERAL>
static void launch_shape(const StepDev& d, cudaStream_t stream, size_t smem) {
    constexpr int threads = kShapes[V].threads;
    const int64_t blocks = (d.n + threads - 1) / threads;
    step_kernel<T, threads, kShapes[V].min_blocks, GENERAL><<<(unsigned)blocks, threads, smem, stream>>>(d);
}

template <typename T>
static glide_status launch_step(const StepDev& d, cudaStream_t stream, int variant) {
    const size_t smem = step_smem_bytes(d.n_steps, d.diag != nullptr);
    if (smem > 48 * 1024)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: n_steps %d too large%s", d.n_steps,
                         d.diag ? " with diag_pos_fixed (at most 1535)" : "");
    switch (variant) {
        case 0: launch_shape<T, 0, false>(d, stream, smem); break;
        case 1: launch_shape<T, 1, false>(d, stream, smem); break;
        case 2: launch_shape<T, 2, false>(d, stream, smem); break;
        case 3: launch_shape<T, 3, false>(d, stream, smem); break;
        case 4: launch_shape<T, 4, false>(d, stream, smem); break;
        case 5: launch_shape<T, 5, false>(d, stream, smem); break;
        case 6: launch_shape<T, 6, false>(d, stream, smem); break;
        case 7: launch_shape<T, 7, false>(d, stream, smem); break;
        case kNumShapes: launch_shape<T, 0, true>(d, stream, smem); break;
        default: return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: launch_variant %d out of range", variant);
    }
    return check_launch("glide_step");
}

}  // namespace glide

using namespace glide;

// Argument checks of one launch (GLIDE_OK when it can run; n == 0 passes).
static glide_status validate_step(const glide_step_args* a) {
    if (!a) return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: args is NULL");
    if (a->n < 0) return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: n < 0");
    if (a->n_steps < 1) return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: n_steps < 1");
    if (!a->sched && a->n_steps != 1)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: sched is NULL but n_steps = %d", a->n_steps);
    if (a->n == 0) return GLIDE_OK;  // nothing else is read
    if (!a->lon || !a->lat || !a->z || !a->weight || !a->u_prime || !a->v_prime || !a->w_prime)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: a particle state pointer is NULL");
    if (!a->active_mask && !a->rel_off)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: rel_off is NULL and no active_mask is given");
    if (a->meander_enabled && (!a->u_meander || !a->v_meander || !a->support_packed))
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: meander enabled but meander state is NULL");
    if (!a->wind_packed || !a->surf_packed || !a->support_packed || !a->grid.level_sorted)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: packed met pointer is NULL");
    if (a->grid.nz < 2 || a->grid.ny < 2 || a->grid.nx < 2)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: grid must be at least 2x2x2");
    if (a->max_substeps < 1) return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: max_substeps < 1");
    if (a->phys_begin < 0 || a->post_begin < 0)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: phys_begin / post_begin < 0");
    if (a->diag_pos_fixed && ((uintptr_t)a->diag_pos_fixed & 7u))
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: diag_pos_fixed must be 8-byte aligned");
    if (a->footprint && a->fp.value_f64 && ((uintptr_t)a->footprint & 7u))
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: a float64 footprint must be 8-byte aligned");
    if (a->launch_variant < 0 || a->launch_variant >= kNumVariants)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: launch_variant %d out of range", a->launch_variant);
    if (a->pos_stride < 1) return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: pos_stride < 1");
    if (a->conv_column && (a->conv_nz < 2 || a->conv_step < 0 || a->conv_step >= a->n_steps))
        return set_error(GLIDE_ERR_INVALID_ARG,
                         "glide_step: fused convection needs conv_nz >= 2 and 0 <= conv_step < n_steps");
    if (a->conv_column && ((uintptr_t)a->conv_column & 7u))
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: conv_column must be 8-byte aligned");
    if (a->footprint && (!a->fp.z_edges || a->fp.n_z < 1 || a->fp.n_x < 1 || a->fp.n_y < 1 ||
                         a->fp.n_time_bins < 1 || a->fp.n_releases < 1 || a->fp.ring < 0))
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: invalid footprint grid");
    if (a->post_begin < a->n_steps && !a->active_mask && a->footprint && !a->win_end_off)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: footprint needs win_end_off");
    if (a->grid.lon_last == a->grid.lon_first || a->grid.lat_last == a->grid.lat_first)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: met grid has zero span");
    if (((uintptr_t)a->wind_packed | (uintptr_t)a->surf_packed | (uintptr_t)a->support_packed) & 15u)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_step: packed met must be 16-byte aligned");

    return GLIDE_OK;
}

static StepDev make_step_dev(const glide_step_args* a) {
    StepDev d;
    d.n = a->n;
    d.lon = a->lon; d.lat = a->lat; d.z = a->z; d.weight = a->weight; d.ps = a->pos_stride;
    d.up = a->u_prime; d.vp = a->v_prime; d.wp = a->w_prime; d.um = a->u_meander; d.vm = a->v_meander;
    d.rel_off = a->rel_off; d.win_end_off = a->win_end_off; d.release_idx = a->release_idx;
    d.alive = a->alive; d.active_mask = a->active_mask;
    d.sim_length = a->sim_length_s;
    d.wind = a->wind_packed; d.surf = a->surf_packed; d.support = a->support_packed;
    d.g = make_grid_dev(a->grid);
    d.substep_c = a->substep_c; d.max_substeps = a->max_substeps; d.z_ubl = a->z_ubl_m;
    d.floors = a->flexpart_tl_floors; d.sl_override = a->surface_layer_override;
    d.meander = a->meander_enabled; d.meander_T = a->meander_timescale_s;
    d.sched = a->sched; d.sched0 = a->sched0;
    d.n_steps = a->n_steps; d.phys_begin = a->phys_begin; d.post_begin = a->post_begin;
    d.noise_sub = a->noise_substep; d.noise_mea = a->noise_meander;
    d.seed_lo = (uint32_t)a->seed; d.seed_hi = (uint32_t)(a->seed >> 32);
    d.fp = a->footprint;
    d.fp64 = a->fp.value_f64 != 0;
    d.fp_lon0 = (float)a->fp.lon_min;
    d.fp_lon_span = (float)fmax(1e-6, a->fp.lon_max - a->fp.lon_min);
    d.fp_lat0 = (float)a->fp.lat_min;
    d.fp_lat_span = (float)fmax(1e-6, a->fp.lat_max - a->fp.lat_min);
    d.fp_R = a->fp.n_releases; d.fp_T = a->fp.n_time_bins; d.fp_Z = a->fp.n_z; d.fp_Y = a->fp.n_y;
    d.fp_X = a->fp.n_x; d.fp_edges = a->fp.z_edges;
    d.fp_ring = a->fp.ring;
    d.dom_lon0 = (float)a->dom_lon_min; d.dom_lon1 = (float)a->dom_lon_max;
    d.dom_lat0 = (float)a->dom_lat_min; d.dom_lat1 = (float)a->dom_lat_max;
    d.dom_alt = (float)a->dom_alt_max;
    d.esc = a->escaped_per_step; d.act = a->active_per_step;
    d.status = a->status;
    d.order = a->order; d.work_key = a->work_key;
    d.conv_column = static_cast<const double*>(a->conv_column); d.conv_step = a->conv_step; d.conv_nz = a->conv_nz;
    d.conv_uniforms = a->conv_uniforms; d.conv_moved = a->conv_moved;
    d.diag = reinterpret_cast<long long*>(a->diag_pos_fixed);
    return d;
}

static bool needs_general(const StepDev& d) {
    return d.sl_override || d.noise_sub || d.noise_mea || d.active_mask || d.conv_uniforms;
}

extern "C" glide_status glide_step(const glide_step_args* a, void* stream) {
    if (glide_status st = validate_step(a)) return st;
    if (a->n == 0) return GLIDE_OK;
    const StepDev d = make_step_dev(a);
    cudaStream_t s = (cudaStream_t)stream;
    const int variant = needs_general(d) ? kNumShapes : a->launch_variant;
    switch (a->met_dtype) {
        case GLIDE_MET_F32: return launch_step<float>(d, s, variant);
        case GLIDE_MET_BF16: return launch_step<__nv_bfloat16>(d, s, variant);
        case GLIDE_MET_F16: return launch_step<__half>(d, s, variant);
        default: return set_error(GLIDE_ERR_UNSUPPORTED, "glide_step: unknown met_dtype %d", a->met_dtype);
    }
}

template <typename T>
static glide_status launch_batched(const StepBatch& b, bool general, size_t smem, uint32_t blocks, cudaStream_t s) {
    if (general) step_kernel_batched<T, true><<<blocks, 128, smem, s>>>(b);
    else step_kernel_batched<T, false><<<blocks, 128, smem, s>>>(b);
    return check_launch("glide_step_batched");
}

extern "C" glide_status glide_step_batched(const glide_step_args* args, int32_t count, void* stream) {
    if (!args || count < 0 || count > GLIDE_STEP_BATCH_MAX)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_step_batched: args NULL or count %d not in [0, %d]",
                         count, GLIDE_STEP_BATCH_MAX);
    StepBatch b;
    b.count = 0;
    bool general = false;
    int32_t dtype = -1;
    int max_steps = 1;
    bool diag = false;
    uint64_t blocks = 0;
    for (int k = 0; k < count; ++k) {
        const glide_step_args* a = args + k;
        if (glide_status st = validate_step(a)) return st;
        if (a->n == 0) continue;
        if (dtype >= 0 && a->met_dtype != dtype)
            return set_error(GLIDE_ERR_INVALID_ARG, "glide_step_batched: batches mix met dtypes");
        dtype = a->met_dtype;
        const StepDev d = make_step_dev(a);
        general = general || needs_general(d);
        max_steps = max(max_steps, d.n_steps);
        diag = diag || d.diag != nullptr;
        b.d[b.count] = d;
        b.block_start[b.count] = (uint32_t)blocks;
        blocks += (uint64_t)((d.n + 127) / 128);
        ++b.count;
    }
    if (b.count == 0) return GLIDE_OK;
    if (blocks > 0x7fffffffull) return set_error(GLIDE_ERR_INVALID_ARG, "glide_step_batched: too many particles");
    b.block_start[b.count] = (uint32_t)blocks;
    // every block lays out shared memory for the longest batch (and the diagnostic sums
    // when any batch asks for them); a block uses the part its own batch needs
    const size_t smem = step_smem_bytes(max_steps, diag);
    if (smem > 48 * 1024)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_step_batched: n_steps %d too large", max_steps);
    cudaStream_t s = (cudaStream_t)stream;
    switch (dtype) {
        case GLIDE_MET_F32: return launch_batched<float>(b, general, smem, (uint32_t)blocks, s);
        case GLIDE_MET_BF16: return launch_batched<__nv_bfloat16>(b, general, smem, (uint32_t)blocks, s);
        case GLIDE_MET_F16: return launch_batched<__half>(b, general, smem, (uint32_t)blocks, s);
        default: return set_error(GLIDE_ERR_UNSUPPORTED, "glide_step_batched: unknown met_dtype %d", dtype);
    }
}

extern "C" glide_status glide_step_launch_variants(int32_t* count) {
    if (!count) return set_error(GLIDE_ERR_INVALID_ARG, "glide_step_launch_variants: count is NULL");
    *count = kNumVariants;
    return GLIDE_OK;
}

extern "C" glide_status glide_step_launch_variant_info(int32_t v, int32_t* threads, int32_t* min_blocks) {
    if (v < 0 || v >= kNumVariants)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_step_launch_variant_info: variant %d out of range", v);
    const LaunchShape sh = kShapes[v < kNumShapes ? v : 0];
    if (threads) *threads = sh.threads;
    if (min_blocks) *min_blocks = sh.min_blocks;
    return GLIDE_OK;
}
