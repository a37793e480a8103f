// Particle ordering by work class: a stable counting sort of particle indices by
// the work key the step kernel writes (glide_step_args.work_key), descending.
//
// The step kernel runs one particle per thread, and a particle's path through a
// step (substep count, stability regime, closure branch, boundary layer or free
// troposphere) follows its height relative to the boundary-layer top: a warp runs
// every path one of its lanes takes. Grouping particles of one class (substeps x
// height band x regime) into the same warps, and escaped particles into warps that
// exit at once, removes that idle-lane time; ordering classes descending puts
// pending particles first. The sort is stable within a class so that neighbouring
// particles (same release, nearby met cells) stay neighbours.
//
//   tile_hist     per 1024-particle tile, counts per class -> hist[class][tile]
//   scan_offsets  one block: exclusive scan of hist in class-major order
//   tile_scatter  per tile, stable in-tile ranks (warp match + per-warp counts)
//                 -> order[offset[class][tile] + rank] = particle
#include "glide_internal.h"

namespace glide {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kItems = 4;
constexpr int kTile = kThreads * kItems;
constexpr int kClasses = GLIDE_WORK_CLASSES;

// descending key -> ascending bucket
__device__ __forceinline__ int bucket_of(uint8_t key) { return (kClasses - 1) - min((int)key, kClasses - 1); }

__global__ void __launch_bounds__(kThreads) tile_hist(const uint8_t* __restrict__ key, int64_t n,
                                                      int32_t* __restrict__ hist, int n_tiles) {
    __shared__ int32_t h[kClasses];
    if (threadIdx.x < kClasses) h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t t0 = (int64_t)blockIdx.x * kTile;
#pragma unroll
    for (int r = 0; r < kItems; ++r) {
        const int64_t i = t0 + (int64_t)r * kThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[bucket_of(key[i])], 1);
    }
    __syncthreads();
    if (threadIdx.x < kClasses) hist[(int64_t)threadIdx.x * n_tiles + blockIdx.x] = h[threadIdx.x];
}

// exclusive scan of m int32 in place, one block of 1024 threads (m is at most
// 16 x ceil(INT32_MAX / 1024), so every partial sum fits in int32)
__global__ void __launch_bounds__(1024) scan_offsets(int32_t* __restrict__ h, int64_t m) {
    __shared__ int32_t s[1024];
    const int64_t per = (m + 1023) / 1024;
    const int64_t b = (int64_t)threadIdx.x * per;
    const int64_t e = b + per < m ? b + per : m;
    int32_t sum = 0;
    for (int64_t k = b; k < e; ++k) sum += h[k];
    s[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int32_t v = threadIdx.x >= (unsigned)off ? s[threadIdx.x - off] : 0;
        __syncthreads();
        s[threadIdx.x] += v;
        __syncthreads();
    }
    int32_t run = s[threadIdx.x] - sum;
    for (int64_t k = b; k < e; ++k) {
        const int32_t v = h[k];
        h[k] = run;
        run += v;
    }
}

__global__ void __launch_bounds__(kThreads) tile_scatter(const uint8_t* __restrict__ key, int64_t n,
                                                         const int32_t* __restrict__ offsets, int n_tiles,
                                                         int32_t* __restrict__ order) {
    __shared__ int32_t warp_base[kWarps][kClasses];
    __shared__ int32_t base[kClasses];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (tid < kClasses) base[tid] = offsets[(int64_t)tid * n_tiles + blockIdx.x];
    const int64_t t0 = (int64_t)blockIdx.x * kTile;
    for (int r = 0; r < kItems; ++r) {
        for (int k = tid; k < kWarps * kClasses; k += kThreads) (&warp_base[0][0])[k] = 0;
        __syncthreads();
        // items of round r in index order: tid-major within the round, rounds in sequence
        const int64_t i = t0 + (int64_t)r * kThreads + tid;
        const int b = i < n ? bucket_of(key[i]) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, b);
        const int rank = __popc(peers & ((1u << lane) - 1u));
        if (b >= 0 && rank == 0) warp_base[w][b] = __popc(peers);
        __syncthreads();
        if (tid < kClasses) {  // per class: counts of the warps -> their starting slots
            int32_t run = base[tid];
            for (int ww = 0; ww < kWarps; ++ww) {
                const int32_t c = warp_base[ww][tid];
                warp_base[ww][tid] = run;
                run += c;
            }
            base[tid] = run;
        }
        __syncthreads();
        if (b >= 0) {
            const int64_t slot = (int64_t)warp_base[w][b] + rank;
            if (slot >= 0 && slot < n) order[slot] = (int32_t)i;
        }
        __syncthreads();
    }
}

int64_t tiles_of(int64_t n) { return (n + kTile - 1) / kTile; }

}  // namespace
}  // namespace glide

using namespace glide;

extern "C" glide_status glide_reorder_scratch_bytes(int64_t n, size_t* bytes) {
    if (!bytes) return set_error(GLIDE_ERR_INVALID_ARG, "glide_reorder_scratch_bytes: bytes is NULL");
    if (n < 0 || n > INT32_MAX) return set_error(GLIDE_ERR_INVALID_ARG, "glide_reorder_scratch_bytes: n out of range");
    *bytes = sizeof(int32_t) * (size_t)kClasses * (size_t)(n > 0 ? tiles_of(n) : 1);
    return GLIDE_OK;
}

extern "C" glide_status glide_reorder_by_key(int64_t n, const uint8_t* work_key, int32_t* order, void* scratch,
                                             size_t scratch_bytes, void* stream) {
    if (n < 0 || n > INT32_MAX) return set_error(GLIDE_ERR_INVALID_ARG, "glide_reorder_by_key: n out of range");
    if (n == 0) return GLIDE_OK;
    if (!work_key || !order || !scratch) return set_error(GLIDE_ERR_INVALID_ARG, "glide_reorder_by_key: NULL pointer");
    const int64_t tiles = tiles_of(n);
    const size_t need = sizeof(int32_t) * (size_t)kClasses * (size_t)tiles;
    if (scratch_bytes < need)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_reorder_by_key: scratch is %zu bytes, %zu needed", scratch_bytes,
                         need);
    if ((uintptr_t)scratch & 3u) return set_error(GLIDE_ERR_INVALID_ARG, "glide_reorder_by_key: scratch misaligned");
    cudaStream_t s = (cudaStream_t)stream;
    int32_t* hist = static_cast<int32_t*>(scratch);
    tile_hist<<<(unsigned)tiles, kThreads, 0, s>>>(work_key, n, hist, (int)tiles);
    scan_offsets<<<1, 1024, 0, s>>>(hist, (int64_t)kClasses * tiles);
    tile_scatter<<<(unsigned)tiles, kThreads, 0, s>>>(work_key, n, hist, (int)tiles, order);
    return check_launch("glide_reorder_by_key");
}
