// Per-particle backward convective redistribution against a prebuilt column
// (EmanuelReducedConvection._redistribute_particles, src/lpdm/convection/emanuel.py:772-805),
// shared by glide_convect_redistribute's kernel and the step kernel's fused
// per-window convection.
//
// Column layout (doubles, written by column_build_kernel):
//   header[8] | t[nz] | q[nz] | h[nz] | h_asc[nz] | cum[nz][nz]
//   header: fires, i_lcl, i_lnb, cape, dtv, m_b, ascending, -
#pragma once

#include "common.cuh"

namespace glide {

// the two uniforms of particle i at a step, when not injected: one Philox block
__device__ inline void convection_uniforms(int64_t i, uint32_t step_index, uint32_t seed_lo, uint32_t seed_hi,
                                           double& u1, double& u2) {
    const U4 r = philox4x32_10(U4{(uint32_t)i, (uint32_t)((uint64_t)i >> 32), step_index, STREAM_CONVECTION}, seed_lo,
                               seed_hi);
    u1 = (double)u01(r.x);
    u2 = (double)u01(r.y);
}

// nearest host level of z, destination level by inverting the host row of the
// backward transition CDF with u1, new height uniform (u2) in the destination
// layer; returns true when the particle moved (only when the column fires)
__device__ inline bool convect_particle(const double* column, int nz, float& z, double u1, double u2) {
    if (column[0] == 0.0) return false;
    const double* h = column + 8 + 3 * nz;
    const double* cum = column + 8 + 4 * nz;
    const double zd = (double)z;
    int lo = 0, hi = nz;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (h[mid] < zd) lo = mid + 1; else hi = mid;
    }
    const int iu = min(max(lo, 1), nz - 1), il = iu - 1;
    const int host = ((zd - h[il]) < (h[iu] - zd)) ? il : iu;
    const double* row = cum + (int64_t)host * nz;
    int dest = 0;
    for (int c = 0; c < nz; ++c) dest += (row[c] < u1) ? 1 : 0;
    dest = min(dest, nz - 1);
    if (dest == host) return false;
    const double zl = h[max(dest - 1, 0)], zh = h[dest];
    z = (float)(zl + u2 * (zh - zl));
    return true;
}

}  // namespace glide
