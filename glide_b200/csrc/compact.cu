// Sparse form of completed footprint slices: (cell, value) lists of the cells whose
// float32 (or float64) bit pattern is not zero, slices in the caller's order, cells
// ascending.
//
// A slice (one release's time_ago bin, Zb x Y x X float32) of a backward plume is
// mostly zero: the plume of one release covers a few thousand of the 1.1e5 cells of
// the EUROPE grid in an hour. The reference copies the dense footprint to the host
// for OutputWriter.write_footprint_region (src/lpdm/output_writer.py:215-243); here
// the slices are compacted on the device, so only the non-zero cells cross PCIe.
//
//   compact_count  per 2048-cell tile of each slice: non-zero count -> count[tile]
//   compact_scan   one block: exclusive scan of the counts (int64) -> offset[tile],
//                  offset[m] = total, and each slice's first entry -> slice_offset
//   compact_write  per tile, in cell order (warp ballot + per-warp counts): the
//                  cells and values at offset[tile] + rank, and optionally the
//                  compacted cells set to zero (the ring slot is free again)
//
// The tiles are HBM/L2 streams of 4-byte words, read twice (count, write); the
// kernels are short beside the step launch that filled the slices.
#include "glide_internal.h"

namespace glide {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;

// W: the value word, uint32_t (float32 footprints) or unsigned long long (float64)
template <typename W>
__global__ void __launch_bounds__(kThreads)
    compact_count(const W* __restrict__ rows, int64_t n_rows, int64_t cells,
                  const int64_t* __restrict__ row_index, int64_t tiles, int32_t* __restrict__ count,
                  uint32_t* status) {
    __shared__ int32_t warp_n[kWarps];
    const int64_t blk = blockIdx.x;
    const int64_t s = blk / tiles, t = blk - s * tiles;
    const int64_t row = row_index[s];
    int32_t c = 0;
    if (row >= 0 && row < n_rows) {
        const W* src = rows + row * cells;
        const int64_t t0 = t * kTile;
#pragma unroll
        for (int r = 0; r < kItems; ++r) {
            const int64_t i = t0 + (int64_t)r * kThreads + threadIdx.x;
            if (i < cells) c += src[i] != W(0) ? 1 : 0;
        }
    } else if (t == 0 && threadIdx.x == 0 && status) {
        atomicOr(status, (uint32_t)GLIDE_STATUS_BAD_ROW);
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0) warp_n[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int32_t sum = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) sum += warp_n[w];
        count[blk] = sum;
    }
}

// exclusive scan of m tile counts into int64 offsets, one block of 1024 threads
// (each thread a contiguous run of ceil(m / 1024) tiles)
__global__ void __launch_bounds__(1024)
    compact_scan(const int32_t* __restrict__ count, int64_t m, int64_t tiles, int32_t k,
                 int64_t* __restrict__ offset, int64_t* __restrict__ slice_offset) {
    __shared__ int64_t s[1024];
    const int64_t per = (m + 1023) / 1024;
    const int64_t b = (int64_t)threadIdx.x * per;
    const int64_t e = b + per < m ? b + per : m;
    int64_t sum = 0;
    for (int64_t i = b; i < e; ++i) sum += count[i];
    s[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int64_t v = threadIdx.x >= (unsigned)off ? s[threadIdx.x - off] : 0;
        __syncthreads();
        s[threadIdx.x] += v;
        __syncthreads();
    }
    int64_t run = s[threadIdx.x] - sum;
    for (int64_t i = b; i < e; ++i) {
        offset[i] = run;
        run += count[i];
    }
    if (threadIdx.x == 1023) offset[m] = s[1023];
    __syncthreads();  // the block's offset writes are visible to all its threads
    for (int64_t j = threadIdx.x; j <= k; j += 1024) slice_offset[j] = offset[j * tiles];
}

template <typename W>
__global__ void __launch_bounds__(kThreads)
    compact_write(W* __restrict__ rows, int64_t n_rows, int64_t cells, const int64_t* __restrict__ row_index,
                  int64_t tiles, const int64_t* __restrict__ offset, int64_t m, int64_t capacity, int clear,
                  int32_t* __restrict__ out_cell, W* __restrict__ out_value, uint32_t* status) {
    __shared__ int32_t warp_n[kWarps];
    // both conditions below are the same for every thread of the block: it returns as a whole
    const int64_t total = offset[m];
    if (total > capacity) {
        if (blockIdx.x == 0 && threadIdx.x == 0 && status) atomicOr(status, (uint32_t)GLIDE_STATUS_COMPACT_OVERFLOW);
        return;
    }
    const int64_t blk = blockIdx.x;
    const int64_t s = blk / tiles, t = blk - s * tiles;
    const int64_t row = row_index[s];
    if (row < 0 || row >= n_rows) return;  // counted as an empty slice
    W* src = rows + row * cells;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t t0 = t * kTile;
    int64_t base = offset[blk];
    for (int r = 0; r < kItems; ++r) {
        // the items of round r are cells t0 + r * kThreads + [0, kThreads): in cell order
        // across the warps of the block, so rounds in sequence keep the tile in cell order
        const int64_t i = t0 + (int64_t)r * kThreads + threadIdx.x;
        const W bits = i < cells ? src[i] : W(0);
        const unsigned ball = __ballot_sync(0xffffffffu, bits != W(0));
        if (lane == 0) warp_n[w] = __popc(ball);
        __syncthreads();
        int32_t before = 0, all = 0;
#pragma unroll
        for (int ww = 0; ww < kWarps; ++ww) {
            const int32_t c = warp_n[ww];
            before += ww < w ? c : 0;
            all += c;
        }
        if (bits != W(0)) {
            const int64_t o = base + before + __popc(ball & ((1u << lane) - 1u));
            if (o < capacity) {
                out_cell[o] = (int32_t)i;
                out_value[o] = bits;
            }
            if (clear) src[i] = W(0);
        }
        base += all;
        __syncthreads();  // warp_n is rewritten by the next round
    }
}

int64_t tiles_of(int64_t cells) { return (cells + kTile - 1) / kTile; }

bool aligned(const void* p, uintptr_t a) { return ((uintptr_t)p & (a - 1)) == 0; }

template <typename W>
void launch_compact(const glide_compact_args* a, W* rows, int64_t tiles, int64_t m, int64_t* offset, int32_t* count,
                    cudaStream_t s) {
    if (m > 0)
        compact_count<W><<<(unsigned)m, kThreads, 0, s>>>(rows, a->n_rows, a->cells, a->row_index, tiles, count,
                                                           a->status);
    compact_scan<<<1, 1024, 0, s>>>(count, m, tiles, a->k, offset, a->slice_offset);
    if (m > 0)
        compact_write<W><<<(unsigned)m, kThreads, 0, s>>>(rows, a->n_rows, a->cells, a->row_index, tiles, offset, m,
                                                           a->capacity, a->clear != 0, a->out_cell,
                                                           static_cast<W*>(a->out_value), a->status);
}

}  // namespace
}  // namespace glide

using namespace glide;

extern "C" glide_status glide_footprint_compact_scratch_bytes(int32_t k, int64_t cells, size_t* bytes) {
    if (!bytes) return set_error(GLIDE_ERR_INVALID_ARG, "glide_footprint_compact_scratch_bytes: bytes is NULL");
    if (k < 0) return set_error(GLIDE_ERR_INVALID_ARG, "glide_footprint_compact: k = %d is negative", (int)k);
    if (cells < 1 || cells > INT32_MAX)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_footprint_compact: cells = %lld outside [1, INT32_MAX]",
                         (long long)cells);
    const int64_t m = (int64_t)k * tiles_of(cells);
    if (m > INT32_MAX)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_footprint_compact: %lld tiles of 2048 cells (at most INT32_MAX)",
                         (long long)m);
    *bytes = sizeof(int64_t) * (size_t)(m + 1) + sizeof(int32_t) * (size_t)m;
    return GLIDE_OK;
}

extern "C" glide_status glide_footprint_compact(const glide_compact_args* a, void* stream) {
    if (!a) return set_error(GLIDE_ERR_INVALID_ARG, "glide_footprint_compact: args is NULL");
    size_t need = 0;
    const glide_status st = glide_footprint_compact_scratch_bytes(a->k, a->cells, &need);
    if (st != GLIDE_OK) return st;
    if (a->n_rows < 0 || a->n_rows > INT64_MAX / a->cells)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_footprint_compact: n_rows = %lld out of range",
                         (long long)a->n_rows);
    if (a->capacity < 0) return set_error(GLIDE_ERR_INVALID_ARG, "glide_footprint_compact: capacity is negative");
    if (!a->slice_offset || !a->scratch) return set_error(GLIDE_ERR_INVALID_ARG, "glide_footprint_compact: NULL pointer");
    if (a->k > 0 && (!a->rows || !a->row_index))
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_footprint_compact: NULL rows or row_index");
    if (a->capacity > 0 && (!a->out_cell || !a->out_value))
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_footprint_compact: NULL output with capacity > 0");
    if (a->scratch_bytes < need)
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_footprint_compact: scratch is %zu bytes, %zu needed",
                         a->scratch_bytes, need);
    const uintptr_t word = a->value_f64 ? 8 : 4;
    if (!aligned(a->scratch, 8) || !aligned(a->slice_offset, 8) || !aligned(a->row_index, 8) ||
        !aligned(a->rows, word) || !aligned(a->out_cell, 4) || !aligned(a->out_value, word) || !aligned(a->status, 4))
        return set_error(GLIDE_ERR_INVALID_ARG, "glide_footprint_compact: misaligned pointer");
    const int64_t tiles = tiles_of(a->cells);
    const int64_t m = (int64_t)a->k * tiles;
    cudaStream_t s = (cudaStream_t)stream;
    int64_t* offset = static_cast<int64_t*>(a->scratch);
    int32_t* count = reinterpret_cast<int32_t*>(offset + m + 1);
    if (a->value_f64) launch_compact(a, static_cast<unsigned long long*>(a->rows), tiles, m, offset, count, s);
    else launch_compact(a, static_cast<uint32_t*>(a->rows), tiles, m, offset, count, s);
    return check_launch("glide_footprint_compact");
}
