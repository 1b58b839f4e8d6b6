// Device-side generator of the chunk-mix workload: the application side of
// Pyrit's generator hook (PyrWorldInfo.generate, include/pyrit.h:818-834) for
// synthetic benchmarks. Produces exactly the voxel lists of wl_mix_chunk (same
// integer math from workloads.h, same scan order z, y, x per chunk), packed chunk
// after chunk. Three kernels: column heights, per-row counts, row fill; the caller
// scans the row counts in between.
#include <cuda_runtime.h>

#include <cstdint>

#include "workloads.h"

namespace {

struct Chunk {
    uint32_t log2;
    uint32_t index;
    uint64_t col_base;   // first column of the chunk in the height buffer
    uint64_t row_base;   // first row (z, y) of the chunk
    uint32_t ncaves;
    int32_t caves[20][4];
};

__device__ __forceinline__ uint32_t find_chunk(const uint64_t* bases, uint32_t n, uint64_t v) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (bases[mid] <= v) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void k_heights(const Chunk* chunks, const uint64_t* col_bases, uint32_t count, uint64_t total_cols,
                          uint32_t seed, int32_t* heights) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < total_cols; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t c = find_chunk(col_bases, count, i);
        const Chunk& ch = chunks[c];
        const uint64_t local = i - ch.col_base;
        const uint32_t e = 1u << ch.log2;
        const int64_t x = int64_t(local % e), z = int64_t(local / e);
        const int64_t tx = ch.index % 32, tz = ch.index / 32;
        const int64_t u = (tx << 17) + (x << (17 - ch.log2)), v = (tz << 17) + (z << (17 - ch.log2));
        heights[i] = int32_t((wl_height_q16(u, v, seed) * int64_t(e)) >> 22);
    }
}

__device__ __forceinline__ uint32_t cell_value(const Chunk& ch, const int32_t* h, uint32_t x, uint32_t y, uint32_t z) {
    const uint32_t e = 1u << ch.log2;
    const int32_t hh = h[ch.col_base + uint64_t(z) * e + x];
    if (int32_t(y) >= hh) return 0;
    for (uint32_t k = 0; k < ch.ncaves; ++k) {
        const int32_t dx = int32_t(x) - ch.caves[k][0], dy = int32_t(y) - ch.caves[k][1], dz = int32_t(z) - ch.caves[k][2];
        if (dx * dx + dy * dy + dz * dz < ch.caves[k][3] * ch.caves[k][3]) return 0;
    }
    return wl_layer_material(int32_t(y), hh);
}

__global__ void k_row_counts(const Chunk* chunks, const uint64_t* row_bases, uint32_t count, uint64_t total_rows,
                             const int32_t* heights, uint32_t* row_counts) {
    for (uint64_t r = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; r < total_rows; r += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t c = find_chunk(row_bases, count, r);
        const Chunk& ch = chunks[c];
        const uint32_t e = 1u << ch.log2;
        const uint64_t local = r - ch.row_base;
        const uint32_t y = uint32_t(local % e), z = uint32_t(local / e);
        uint32_t n = 0;
        for (uint32_t x = 0; x < e; ++x) n += cell_value(ch, heights, x, y, z) != 0;
        row_counts[r] = n;
    }
}

__global__ void k_row_fill(const Chunk* chunks, const uint64_t* row_bases, uint32_t count, uint64_t total_rows,
                           const int32_t* heights, const uint64_t* row_offsets, uint4* out) {
    for (uint64_t r = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; r < total_rows; r += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t c = find_chunk(row_bases, count, r);
        const Chunk& ch = chunks[c];
        const uint32_t e = 1u << ch.log2;
        const uint64_t local = r - ch.row_base;
        const uint32_t y = uint32_t(local % e), z = uint32_t(local / e);
        uint64_t o = r == 0 ? 0 : row_offsets[r - 1];
        for (uint32_t x = 0; x < e; ++x) {
            const uint32_t a = cell_value(ch, heights, x, y, z);
            if (a) out[o++] = make_uint4(x, y, z, a);
        }
    }
}

}  // namespace

extern "C" {

// Host part: chunk descriptors (caves drawn exactly as wl_mix_chunk draws them).
// out_chunks must hold count descriptors of wlg_chunk_desc_bytes() bytes each.
uint64_t wlg_chunk_desc_bytes() { return sizeof(Chunk); }

void wlg_describe(uint32_t count, const uint32_t* log2s, uint32_t first_index, uint32_t seed, void* out_chunks,
                  uint64_t* col_bases, uint64_t* row_bases, uint64_t* total_cols, uint64_t* total_rows) {
    Chunk* ch = static_cast<Chunk*>(out_chunks);
    uint64_t cols = 0, rows = 0;
    for (uint32_t c = 0; c < count; ++c) {
        const uint32_t l = log2s[c], e = 1u << l, index = first_index + c;
        ch[c].log2 = l;
        ch[c].index = index;
        ch[c].col_base = cols;
        ch[c].row_base = rows;
        col_bases[c] = cols;
        row_bases[c] = rows;
        cols += uint64_t(e) * e;
        rows += uint64_t(e) * e;
        const uint32_t nc = uint32_t(wl_hash4(index, seed, 0xCA7Eu, 0) % 21);
        ch[c].ncaves = nc;
        for (uint32_t k = 0; k < nc; ++k) {
            const uint64_t a = wl_hash4(index, seed, 0xCA7Eu, k + 1);
            ch[c].caves[k][0] = int32_t(a % e);
            ch[c].caves[k][1] = int32_t((a >> 16) % e);
            ch[c].caves[k][2] = int32_t((a >> 32) % e);
            ch[c].caves[k][3] = 3 + int32_t((a >> 48) % 10);
        }
    }
    *total_cols = cols;
    *total_rows = rows;
}

// Device part; all pointers are device memory, the work is enqueued on `stream`.
int wlg_heights(const void* chunks, const uint64_t* col_bases, uint32_t count, uint64_t total_cols, uint32_t seed,
                int32_t* heights, void* stream) {
    k_heights<<<1184, 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const Chunk*>(chunks), col_bases, count,
                                                                    total_cols, seed, heights);
    return int(cudaGetLastError());
}

int wlg_row_counts(const void* chunks, const uint64_t* row_bases, uint32_t count, uint64_t total_rows,
                   const int32_t* heights, uint32_t* row_counts, void* stream) {
    k_row_counts<<<4736, 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const Chunk*>(chunks), row_bases,
                                                                       count, total_rows, heights, row_counts);
    return int(cudaGetLastError());
}

int wlg_row_fill(const void* chunks, const uint64_t* row_bases, uint32_t count, uint64_t total_rows,
                 const int32_t* heights, const uint64_t* row_offsets, void* out, void* stream) {
    k_row_fill<<<4736, 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const Chunk*>(chunks), row_bases, count,
                                                                     total_rows, heights, row_offsets,
                                                                     static_cast<uint4*>(out));
    return int(cudaGetLastError());
}

}  // extern "C"
