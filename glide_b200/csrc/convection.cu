// Reduced Emanuel convection for one met window, entirely on the device and
// without host synchronisation (the reference's maybe_convect has several,
// src/lpdm/convection/emanuel.py:352-397, 635-660, 774, 792).
//
//   1. column_reduce_kernel  bbox-mean t, q (time-lerped at alpha) and height
//                            per level, accumulated in FP64 (emanuel.py:593-609)
//   2. column_build_kernel   one block, FP64: parcel lift (Bolton LCL, theta_e
//                            bisection), CAPE/LNB, trigger, cloud-base mass
//                            flux, non-divergent mass-flux matrix with CFL cap,
//                            diagonal closure and the backward (transposed
//                            column) transition CDF (emanuel.py:124-506, 720-770)
//   3. redistribute_kernel   per particle: nearest host level, destination by
//                            CDF inversion, uniform height inside the
//                            destination layer (emanuel.py:772-805)
//
// Scratch layout (doubles): header[8] | t[nz] | q[nz] | h[nz] | h_asc[nz] | cum[nz][nz]
//   header: fires, i_lcl, i_lnb, cape, dtv, m_b, ascending, -
#include <mutex>

#include "common.cuh"
#include "convect.cuh"
#include "glide_internal.h"

namespace glide {

namespace conv {
constexpr double G = 9.80665, RD = 287.05, RV = 461.5, EPS = RD / RV, CP = 1005.0, LV = 2.5e6;
constexpr double P0 = 100000.0, KAPPA = RD / CP, P_MIN = 1.0, T_MIN = 150.0, W_MAX = 5.0, CFL = 0.9;
constexpr double INTERVAL_S = 3600.0;

__device__ inline double e_sat(double t) {  // Bolton (1980) Eq. 10
    const double tc = t - 273.15;
    return 611.2 * exp(17.67 * tc / (tc + 243.5));
}
__device__ inline double q_to_e(double q, double p) { return q * p / (EPS + (1.0 - EPS) * q); }
__device__ inline double e_to_q(double e, double p) { return EPS * e / (fmax(p, P_MIN) - (1.0 - EPS) * e); }
__device__ inline double tv(double t, double q) { return t * (1.0 + (1.0 / EPS - 1.0) * q); }
__device__ inline double t_lcl_bolton(double t, double q, double p) {  // Bolton (1980) Eq. 22
    const double e_hpa = fmax(q_to_e(q, p), 1.0) / 100.0;
    return 2840.0 / fmax(3.5 * log(t) - log(e_hpa) - 4.805, 1e-3) + 55.0;
}
__device__ inline double theta(double t, double p) { return t * pow(P0 / fmax(p, P_MIN), KAPPA); }
__device__ inline double theta_e(double t, double q, double p) {
    return theta(t, p) * exp(LV * q / (CP * fmax(t_lcl_bolton(t, q, p), T_MIN)));
}
}  // namespace conv

// Lanes per level of the parcel lift's parallel bisection (a power of two dividing 32;
// eight lanes resolve three bisection steps per round, ten rounds the thirty steps).
constexpr int kLiftLanes = 8;
constexpr int kBuildThreads = 512;

struct ConvDev {
    int64_t n;
    float* z; int64_t zs;
    const float* rel_off; const uint8_t* alive; const uint8_t* active_mask;
    float sim_length;
    glide_step_sched sched;
    int nz, ny, nx;
    const float* t[2]; const float* q[2];
    const float* h3; const float* hlev; const float* p_hpa;
    double alpha;
    double closure_c, trigger_dtv, min_cape, min_depth;
    const float* uniforms; uint32_t seed_lo, seed_hi;
    double* scratch;
    int32_t* n_moved;
};

__global__ void column_reduce_kernel(const ConvDev d) {
    const int k = blockIdx.x;
    const int64_t plane = (int64_t)d.ny * d.nx;
    const double a = d.alpha, om = 1.0 - d.alpha;
    double st = 0.0, sq = 0.0, sh = 0.0;
    for (int64_t c = threadIdx.x; c < plane; c += blockDim.x) {
        const int64_t idx = (int64_t)k * plane + c;
        st += (double)d.t[0][idx] * om + (double)d.t[1][idx] * a;
        sq += (double)d.q[0][idx] * om + (double)d.q[1][idx] * a;
        if (d.h3) sh += (double)d.h3[idx];
    }
    __shared__ double red[3][32];
    for (int o = 16; o > 0; o >>= 1) {
        st += __shfl_down_sync(0xffffffffu, st, o);
        sq += __shfl_down_sync(0xffffffffu, sq, o);
        sh += __shfl_down_sync(0xffffffffu, sh, o);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { red[0][warp] = st; red[1][warp] = sq; red[2][warp] = sh; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a0 = 0, a1 = 0, a2 = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { a0 += red[0][w]; a1 += red[1][w]; a2 += red[2][w]; }
        double* S = d.scratch;
        S[8 + k] = a0 / (double)plane;
        S[8 + d.nz + k] = fmax(a1 / (double)plane, 0.0);
        S[8 + 2 * d.nz + k] = d.h3 ? a2 / (double)plane : (double)__ldg(d.hlev + k);
    }
}

// Dynamic shared memory of the column build: ten per-level arrays, and the nz x nz
// matrix too when the whole fits the default 48 KB (nz <= 73); a larger matrix is
// built in the scratch buffer itself.
__host__ inline bool column_matrix_in_smem(int nz) {
    return sizeof(double) * (10 * (size_t)nz + (size_t)nz * nz) <= 48 * 1024;
}
__host__ inline size_t column_build_smem(int nz) {
    return sizeof(double) * (10 * (size_t)nz + (column_matrix_in_smem(nz) ? (size_t)nz * nz : 0));
}

// One block of kBuildThreads threads; shared arrays sized by the launch (dynamic smem). The
// matrix is built in shared memory when the launch provides room for it (the
// per-row passes then read shared instead of global memory) and copied to the
// scratch buffer at the end.
__global__ void __launch_bounds__(kBuildThreads) column_build_kernel(const ConvDev d, int matrix_in_smem) {
    const int n = d.nz;
    extern __shared__ double sm[];
    double* T = sm;            // ascending-ordered columns
    double* Q = T + n;
    double* P = Q + n;
    double* H = P + n;
    double* LP = H + n;        // log of the (floored) pressure
    double* TVE = LP + n;      // tv env
    double* TVP = TVE + n;     // tv parcel
    double* M = TVP + n;       // layer mass
    double* E = M + n;         // entrainment
    double* D = E + n;         // detrainment
    __shared__ double s_plcl, s_te, s_thsfc, s_scale;
    __shared__ int s_fires, s_ilcl, s_ilnb;
    double* S = d.scratch;
    double* const cum_out = S + 8 + 4 * n;
    double* const cum = matrix_in_smem ? D + n : cum_out;
    const int tid = threadIdx.x;
    const bool asc = S[8 + 2 * n + (n - 1)] > S[8 + 2 * n];
    for (int k = tid; k < n; k += blockDim.x) {
        const int src = asc ? k : n - 1 - k;
        T[k] = S[8 + src];
        Q[k] = S[8 + n + src];
        H[k] = S[8 + 2 * n + src];
        P[k] = (double)__ldg(d.p_hpa + src) * 100.0;
    }
    __syncthreads();
    if (tid == 0) {  // surface parcel (emanuel.py:316-334)
        const double t0 = T[0], q0 = Q[0], p0 = P[0];
        const double tl = conv::t_lcl_bolton(t0, q0, p0);
        s_plcl = p0 * pow(tl / fmax(t0, conv::T_MIN), conv::CP / conv::RD);
        s_te = conv::theta_e(t0, q0, p0);
        s_thsfc = conv::theta(t0, p0);
    }
    __syncthreads();
    // parcel lift per level (emanuel.py:343-359). A moist level's temperature solves
    // theta_e(T, q_sat(T, p), p) = theta_e of the surface parcel by a fixed 30-step
    // bisection in [180, 350] K (the temperature returned is the final bracket's
    // midpoint), run here as ten rounds of an eight-way
    // split: the eight lanes of a level evaluate the seven interior points of its
    // bracket at once (exactly the midpoints the bisection can visit in its next
    // three steps: dyadic points of [180, 350] K, exact in FP64), then every lane
    // replays the bisection's three steps on those results, so the bracket, and the
    // temperature, are the serial bisection's bit for bit in a tenth of its latency.
    for (int base = 0; base < n; base += (int)blockDim.x / kLiftLanes) {  // block-uniform trip count
        const int k = base + tid / kLiftLanes, sub = tid % kLiftLanes;
        const bool valid = k < n;
        const double pk = valid ? P[k] : P[0];
        double lo = 180.0, hi = 350.0;
        for (int round = 0; round < 10; ++round) {
            const double w = hi - lo;
            bool above = false;
            if (sub > 0) {
                const double x = lo + w * (double)sub / (double)kLiftLanes;
                above = conv::theta_e(x, conv::e_to_q(conv::e_sat(x), pk), pk) > s_te;
            }
            const unsigned bits = __ballot_sync(0xffffffffu, above) >> ((tid & 31) & ~(kLiftLanes - 1));
            int i_lo = 0, i_hi = kLiftLanes;
            for (int step = 0; step < 3; ++step) {
                const int mid = (i_lo + i_hi) >> 1;
                if ((bits >> mid) & 1u) i_hi = mid; else i_lo = mid;
            }
            const double nlo = lo + w * (double)i_lo / (double)kLiftLanes;
            hi = lo + w * (double)i_hi / (double)kLiftLanes;
            lo = nlo;
        }
        if (valid && sub == 0) {
            const bool below = P[k] >= s_plcl;
            const double dry = s_thsfc * pow(P[k] / conv::P0, conv::KAPPA);
            const double tp = below ? dry : 0.5 * (lo + hi);
            LP[k] = log(fmax(P[k], conv::P_MIN));
            TVE[k] = conv::tv(T[k], Q[k]);
            const double qp = below ? Q[0] : conv::e_to_q(conv::e_sat(tp), P[k]);
            TVP[k] = conv::tv(tp, qp);
        }
    }
    __syncthreads();
    if (tid == 0) {
        int i_lcl = -1;
        for (int k = 0; k < n; ++k) if (!(P[k] >= s_plcl)) { i_lcl = k; break; }
        const double dtv = (i_lcl >= 0 && i_lcl + 1 < n) ? TVP[i_lcl + 1] - TVE[i_lcl + 1] : -1.0;
        int i_lnb = -1;
        double cape = 0.0;
        if (i_lcl >= 0) {  // emanuel.py:370-397
            for (int k = 1; k < n; ++k) {
                const double buoy = (TVP[k] - TVE[k]) / fmax(TVE[k], conv::T_MIN);
                const double dz = conv::RD * 0.5 * (T[k - 1] + T[k]) * (LP[k - 1] - LP[k]) / conv::G;
                if (k >= i_lcl) cape += conv::G * fmax(buoy, 0.0) * dz;
            }
            i_lnb = n - 1;
            for (int k = i_lcl + 1; k < n; ++k) {
                if ((TVP[k] - TVE[k]) / fmax(TVE[k], conv::T_MIN) <= 0.0) { i_lnb = k; break; }
            }
        }
        // trigger (emanuel.py:626-638)
        bool fires = i_lcl >= 0 && i_lnb > i_lcl && cape >= d.min_cape && dtv >= d.trigger_dtv;
        if (fires && (H[i_lnb] - H[i_lcl]) < d.min_depth) fires = false;
        double m_b = 0.0;
        if (fires) {  // closure (emanuel.py:646-650)
            const double rho_lcl = P[i_lcl] / (conv::RD * fmax(T[i_lcl], conv::T_MIN));
            m_b = d.closure_c * rho_lcl * fmin(sqrt(2.0 * fmax(cape, 0.0)), conv::W_MAX);
        }
        S[0] = fires ? 1.0 : 0.0; S[1] = i_lcl; S[2] = i_lnb; S[3] = cape; S[4] = dtv; S[5] = m_b;
        S[6] = asc ? 1.0 : 0.0;
        s_fires = fires; s_ilcl = i_lcl; s_ilnb = i_lnb;
        s_scale = m_b * conv::INTERVAL_S;
    }
    __syncthreads();
    for (int k = tid; k < n; k += blockDim.x) S[8 + 3 * n + k] = H[k];
    if (!s_fires) return;
    const int i_lcl = s_ilcl, i_lnb = s_ilnb;
    const double mb = s_scale;
    for (int k = tid; k < n; k += blockDim.x) {  // layer masses (emanuel.py:263-279)
        double dp;
        if (k == 0) dp = fabs(P[0] - P[1]) * 0.5;
        else if (k == n - 1) dp = fabs(P[n - 2] - P[n - 1]) * 0.5;
        else dp = 0.5 * fabs(P[k - 1] - P[k + 1]);
        M[k] = dp / conv::G;
    }
    __syncthreads();
    if (tid == 0) {  // entrainment / detrainment profiles (emanuel.py:475-486, 402-426)
        double bl = 0.0;
        for (int k = 0; k < i_lcl; ++k) bl += M[k];
        bl = fmax(bl, 1e-12);
        const int depth = i_lnb - i_lcl;
        double wt = 0.0;
        for (int k = 0; k < n; ++k) {
            E[k] = (k < i_lcl) ? mb * M[k] / bl : 0.0;
            const double w = (k >= i_lcl && k <= i_lnb && depth > 0) ? 1.0 - (double)(k - i_lcl) / depth : 0.0;
            D[k] = w;
            wt += w;
        }
        wt = fmax(wt, 1e-12);
        for (int k = 0; k < n; ++k) D[k] = mb * D[k] / wt;
    }
    __syncthreads();
    // fmass = outer(e, d)/m_b + subdiagonal subsidence phi (emanuel.py:488-495), built in cum[]
    for (int idx = tid; idx < n * n; idx += blockDim.x) {
        const int r = idx / n, c = idx - r * n;
        cum[idx] = E[r] * D[c] / mb;
    }
    __syncthreads();
    if (tid == 0) {  // the subdiagonal is a running sum: one thread, in level order
        double ce = 0.0, cd = 0.0;
        for (int k = 0; k < n - 1; ++k) {
            ce += E[k];
            cd += D[k];
            cum[(k + 1) * n + k] += fmax(ce - cd, 0.0);
        }
    }
    __syncthreads();
    // CFL cap (emanuel.py:497-504): each row's outflow over its mass, one thread per row
    // (the row summed in column order), then the largest of them
    for (int r = tid; r < n; r += blockDim.x) {
        double rs = 0.0;
        for (int c = 0; c < n; ++c) rs += cum[r * n + c];
        TVP[r] = rs / fmax(M[r], 1e-12);
    }
    __syncthreads();
    if (tid == 0) {
        double mx = -1.0;
        for (int r = 0; r < n; ++r) mx = fmax(mx, TVP[r]);
        s_scale = (mx > conv::CFL) ? conv::CFL / mx : 1.0;
    }
    __syncthreads();
    for (int idx = tid; idx < n * n; idx += blockDim.x) cum[idx] *= s_scale;
    __syncthreads();
    // diagonal closure with the clamped layer mass, transpose, normalise (emanuel.py:752-759, 771-772)
    for (int k = tid; k < n; k += blockDim.x) {
        double rs = 0.0;
        for (int c = 0; c < n; ++c) rs += cum[k * n + c];
        cum[k * n + k] += fmax(fmax(M[k], 1e-6) - rs, 0.0);  // stay mass (diagonal); row k is this thread's
    }
    __syncthreads();
    // backward transition: row i = column i of fmassfrac / m_i (emanuel.py:757-759); each
    // off-diagonal pair swapped by the thread that owns its upper element
    for (int idx = tid; idx < n * n; idx += blockDim.x) {
        const int r = idx / n, c = idx - r * n;
        if (c > r) {
            const double a = cum[r * n + c];
            cum[r * n + c] = cum[c * n + r];
            cum[c * n + r] = a;
        }
    }
    __syncthreads();
    for (int r = tid; r < n; r += blockDim.x) {
        const double mr = fmax(fmax(M[r], 1e-6), 1e-12);
        double tot = 0.0;
        for (int c = 0; c < n; ++c) {
            const double pr = fmax(cum[r * n + c] / mr, 0.0);
            cum[r * n + c] = pr;
            tot += pr;
        }
        tot = fmax(tot, 1e-12);
        double run = 0.0;
        for (int c = 0; c < n; ++c) {
            run += cum[r * n + c] / tot;
            cum[r * n + c] = run;
        }
    }
    if (matrix_in_smem) {
        __syncthreads();
        for (int idx = tid; idx < n * n; idx += blockDim.x) cum_out[idx] = cum[idx];
    }
}

__global__ void redistribute_kernel(const ConvDev d) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int moved = 0;
    if (i < d.n && d.scratch[0] != 0.0) {
        bool active;
        if (d.active_mask) active = d.active_mask[i] != 0;
        else {
            const float rel = d.rel_off[i];
            active = (!d.alive || d.alive[i]) && rel >= d.sched.cursor_off && (rel - d.sim_length) <= d.sched.cursor_off;
        }
        if (active) {
            double u1, u2;
            if (d.uniforms) {
                u1 = (double)d.uniforms[i];
                u2 = (double)d.uniforms[d.n + i];
            } else {
                convection_uniforms(i, (uint32_t)d.sched.step_index, d.seed_lo, d.seed_hi, u1, u2);
            }
            float z = d.z[i * d.zs];
            if (convect_particle(d.scratch, d.nz, z, u1, u2)) {
                d.z[i * d.zs] = z;
                moved = 1;
            }
        }
    }
    if (d.n_moved) {
        const int cnt = __popc(__ballot_sync(0xffffffffu, moved != 0));
        if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(d.n_moved, cnt);
    }
}

}  // namespace glide

using namespace glide;

extern "C" glide_status glide_convect_scratch_bytes(int32_t nz, size_t* bytes) {
    if (nz < 2 || !bytes) return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect_scratch_bytes: nz < 2 or NULL");
    *bytes = sizeof(double) * (8 + 4 * (size_t)nz + (size_t)nz * nz);
    return GLIDE_OK;
}

extern "C" glide_status glide_convect(const glide_convect_args* a, void* stream) {
    if (!a) return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect: args is NULL");
    if (a->nz < 2 || a->nz > 512 || a->ny < 1 || a->nx < 1)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect: grid out of range (2 <= nz <= 512)");
    if (a->n < 0) return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect: n < 0");
    if (!a->t[0] || !a->t[1] || !a->q[0] || !a->q[1] || !a->pressure_hpa || !a->scratch ||
        (!a->height3d && !a->height_level))
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect: NULL input");
    if (a->n > 0 && (!a->z || (!a->active_mask && !a->rel_off)))
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect: NULL particle input");
    if (a->z_stride < 1) return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect: z_stride < 1");
    if (((uintptr_t)a->scratch) & 7u) return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect: scratch misaligned");
    ConvDev d;
    d.n = a->n; d.z = a->z; d.zs = a->z_stride;
    d.rel_off = a->rel_off; d.alive = a->alive; d.active_mask = a->active_mask;
    d.sim_length = a->sim_length_s; d.sched = a->sched;
    d.nz = a->nz; d.ny = a->ny; d.nx = a->nx;
    d.t[0] = a->t[0]; d.t[1] = a->t[1]; d.q[0] = a->q[0]; d.q[1] = a->q[1];
    d.h3 = a->height3d; d.hlev = a->height_level; d.p_hpa = a->pressure_hpa;
    d.alpha = (double)a->alpha;
    d.closure_c = a->closure_c; d.trigger_dtv = a->trigger_dtv_k; d.min_cape = a->min_cape_j_kg;
    d.min_depth = a->min_cloud_depth_m;
    d.uniforms = a->uniforms; d.seed_lo = (uint32_t)a->seed; d.seed_hi = (uint32_t)(a->seed >> 32);
    d.scratch = static_cast<double*>(a->scratch);
    d.n_moved = a->n_moved;
    cudaStream_t s = (cudaStream_t)stream;
    column_reduce_kernel<<<a->nz, 512, 0, s>>>(d);
    column_build_kernel<<<1, kBuildThreads, column_build_smem(a->nz), s>>>(d, column_matrix_in_smem(a->nz) ? 1 : 0);
    if (a->n > 0) redistribute_kernel<<<(unsigned)((a->n + 255) / 256), 256, 0, s>>>(d);
    return check_launch("glide_convect");
}

extern "C" glide_status glide_convect_redistribute(const glide_convect_args* a, void* stream) {
    if (!a) return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect_redistribute: args is NULL");
    if (a->nz < 2 || a->nz > 512) return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect_redistribute: nz out of range");
    if (a->n < 0) return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect_redistribute: n < 0");
    if (!a->scratch) return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect_redistribute: scratch is NULL");
    if (a->n > 0 && (!a->z || (!a->active_mask && !a->rel_off)))
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect_redistribute: NULL particle input");
    if (a->z_stride < 1) return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect_redistribute: z_stride < 1");
    if (((uintptr_t)a->scratch) & 7u)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect_redistribute: scratch misaligned");
    if (a->n == 0) return GLIDE_OK;
    ConvDev d = {};
    d.n = a->n; d.z = a->z; d.zs = a->z_stride;
    d.rel_off = a->rel_off; d.alive = a->alive; d.active_mask = a->active_mask;
    d.sim_length = a->sim_length_s; d.sched = a->sched;
    d.nz = a->nz;
    d.uniforms = a->uniforms; d.seed_lo = (uint32_t)a->seed; d.seed_hi = (uint32_t)(a->seed >> 32);
    d.scratch = static_cast<double*>(a->scratch);
    d.n_moved = a->n_moved;
    redistribute_kernel<<<(unsigned)((a->n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(d);
    return check_launch("glide_convect_redistribute");
}

extern "C" glide_status glide_convect_column_info(const void* scratch, int32_t nz, void* stream, int32_t* fires,
                                                  int32_t* i_lcl, int32_t* i_lnb, double* cape, double* dtv,
                                                  double* m_b) {
    (void)nz;
    if (!scratch) return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect_column_info: scratch is NULL");
    double h[8];
    cudaError_t e = cudaMemcpyAsync(h, scratch, sizeof(h), cudaMemcpyDeviceToHost, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_error(e, "glide_convect_column_info");
    e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_error(e, "glide_convect_column_info");
    if (fires) *fires = (int32_t)h[0];
    if (i_lcl) *i_lcl = (int32_t)h[1];
    if (i_lnb) *i_lnb = (int32_t)h[2];
    if (cape) *cape = h[3];
    if (dtv) *dtv = h[4];
    if (m_b) *m_b = h[5];
    return GLIDE_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant: the scratch is a file-scope device array instead of
// a caller buffer. Host code cannot use the array's name as a device address;
// each device's address is looked up once (cudaGetSymbolAddress, with that
// device current) and passed to the kernels.
// ---------------------------------------------------------------------------

namespace glide {

constexpr int NOALLOC_MAX_NZ = GLIDE_CONVECT_NOALLOC_MAX_NZ;
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) double g_convect_scratch[8 + 4 * NOALLOC_MAX_NZ + NOALLOC_MAX_NZ * NOALLOC_MAX_NZ];

static std::mutex g_scratch_mu;
static double* g_scratch_addr[NOALLOC_MAX_DEVICES] = {};

// The device address of g_convect_scratch on the current device. Looked up with
// cudaGetSymbolAddress on every call made outside stream capture (so the address
// follows the module if the device's context was reset and the library's module
// loaded again); a call on a capturing stream uses the address the last
// uncaptured call on that device found.
static glide_status noalloc_scratch(cudaStream_t stream, double** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "glide_convect_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
        return set_error(GLIDE_ERR_UNSUPPORTED, "glide_convect_noalloc: device ordinal %d out of range", dev);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(stream, &cs);
    if (e != cudaSuccess) return cuda_error(e, "glide_convect_noalloc: cudaStreamIsCapturing");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (cs == cudaStreamCaptureStatusNone || !g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_convect_scratch);
        if (e != cudaSuccess) return cuda_error(e, "glide_convect_noalloc: cudaGetSymbolAddress");
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return GLIDE_OK;
}

}  // namespace glide

extern "C" glide_status glide_convect_noalloc(const glide_convect_args* a, void* stream) {
    if (!a) return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect_noalloc: args is NULL");
    if (a->nz > NOALLOC_MAX_NZ)
        return set_error(GLIDE_ERR_INVALID_ARG,
                         "glide_convect_noalloc: nz = %d exceeds the %d levels of its static scratch "
                         "(use glide_convect with a caller scratch buffer)", a->nz, NOALLOC_MAX_NZ);
    if (a->nz < 2 || a->ny < 1 || a->nx < 1)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect_noalloc: grid out of range (2 <= nz)");
    if (a->n < 0) return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect_noalloc: n < 0");
    if (!a->t[0] || !a->t[1] || !a->q[0] || !a->q[1] || !a->pressure_hpa || (!a->height3d && !a->height_level))
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect_noalloc: NULL input");
    if (a->n > 0 && (!a->z || (!a->active_mask && !a->rel_off)))
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect_noalloc: NULL particle input");
    if (a->z_stride < 1) return set_error(GLIDE_ERR_INVALID_ARG, "glide_convect_noalloc: z_stride < 1");
    double* scratch = nullptr;
    const glide_status st = noalloc_scratch((cudaStream_t)stream, &scratch);
    if (st != GLIDE_OK) return st;
    ConvDev d;
    d.n = a->n; d.z = a->z; d.zs = a->z_stride;
    d.rel_off = a->rel_off; d.alive = a->alive; d.active_mask = a->active_mask;
    d.sim_length = a->sim_length_s; d.sched = a->sched;
    d.nz = a->nz; d.ny = a->ny; d.nx = a->nx;
    d.t[0] = a->t[0]; d.t[1] = a->t[1]; d.q[0] = a->q[0]; d.q[1] = a->q[1];
    d.h3 = a->height3d; d.hlev = a->height_level; d.p_hpa = a->pressure_hpa;
    d.alpha = (double)a->alpha;
    d.closure_c = a->closure_c; d.trigger_dtv = a->trigger_dtv_k; d.min_cape = a->min_cape_j_kg;
    d.min_depth = a->min_cloud_depth_m;
    d.uniforms = a->uniforms; d.seed_lo = (uint32_t)a->seed; d.seed_hi = (uint32_t)(a->seed >> 32);
    d.scratch = scratch;
    d.n_moved = a->n_moved;
    cudaStream_t s = (cudaStream_t)stream;
    column_reduce_kernel<<<a->nz, 512, 0, s>>>(d);
    column_build_kernel<<<1, kBuildThreads, column_build_smem(a->nz), s>>>(d, column_matrix_in_smem(a->nz) ? 1 : 0);
    if (a->n > 0) redistribute_kernel<<<(unsigned)((a->n + 255) / 256), 256, 0, s>>>(d);
    return check_launch("glide_convect_noalloc");
}
