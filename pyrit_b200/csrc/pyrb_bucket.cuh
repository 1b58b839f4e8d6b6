// Sparse builds without a sort: brick buckets (sm_100a).
//
// The cell grid (pyrb_grid.cuh) orders the voxels of dense chunks without sorting,
// but it moves 8 bytes per cell, and sparse volumes have many cells per entry (the
// worst case, Bernoulli(0.15), has 6.6). Brick buckets keep the grid's idea for the
// 64 cells of a brick and replace the rest of the grid by a one-pass counting sort on
// the brick number, whose counters (4 bytes per brick position: 64 MB for a 1024^3
// volume) stay in the L2:
//
//   k_bkt_count       every entry adds 1 to the counter of its brick position
//   k_bkt_scan_*      the counters become the start of every brick's bucket (tile
//                     sums, one block scanning them, every tile scanned)
//   k_bkt_scatter     every entry takes the next slot of its bucket (an atomic add on
//                     the brick's cursor) and leaves (entry index + 1) << 32 | value
//                     there and its cell in the brick (key & 63); the cursor ends at
//                     the bucket's end
//   k_grid_count<1>,  the grid path's compaction, with each tile's 64 bricks rebuilt
//   k_grid_write<1>   as a 32 KB cell grid in shared memory from their buckets (the
//                     same atomic max: the largest entry index of a cell wins, the
//                     last entry in input order, as a stable sort keeps it)
//
// The order of the entries inside a bucket does not matter: the index they carry
// decides. Bytes per entry: 16 (input) twice, 9 written and read twice, against
// 16 + (kb + 4) (2 passes + 1) for an encode and a 4-pass sort.
#pragma once

#include "pyrb_grid.cuh"

namespace pyrb {

constexpr uint32_t kBucketScanTile = 8192;  // counters per tile of the counter scan

__device__ __forceinline__ void red_add_u32(uint32_t* p, uint32_t v) {
    asm volatile("red.relaxed.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__global__ void __launch_bounds__(kBlock) k_bkt_count(BuildDesc d) {
    grid_dep_wait();
    const uint32_t tile = blockIdx.x;
    if (tile >= d.seg_tile[d.seg_count]) return;
    const TileSpan sp = tile_span(d, tile);
    uint32_t* counts = d.bcount + (__ldg(d.grid_off + sp.seg) >> 6);
    for_tile_entries(d, sp, [&](uint32_t, uint32_t key, uint32_t) { red_add_u32(counts + (key >> 6), 1u); });
}

// Counter sums of tiles of kBucketScanTile counters.
__global__ void __launch_bounds__(kBlock) k_bkt_scan_tiles(BuildDesc d) {
    grid_dep_wait();
    __shared__ uint32_t s_w[kWarps];
    const uint64_t nb = d.grid_cells >> 6;
    const uint64_t t0 = uint64_t(blockIdx.x) * kBucketScanTile;
    uint32_t sum = 0;
#pragma unroll 8
    for (uint32_t k = threadIdx.x; k < kBucketScanTile; k += kBlock)
        sum += t0 + k < nb ? __ldcg(d.bcount + t0 + k) : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t t = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) t += s_w[w];
        d.bsum[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(kGridScanThreads) k_bkt_scan_top(BuildDesc d) {
    grid_dep_wait();
    block_scan_inplace(d.bsum, d.bucket_scan_tiles);
}

// Every tile of counters -> the start of each brick's bucket (exclusive scan, in place).
// Warp w scans its 1024 counters as 32 rows of 32 (carry from row to row), the warps'
// totals by a block scan.
__global__ void __launch_bounds__(kBlock) k_bkt_scan_apply(BuildDesc d) {
    grid_dep_wait();
    __shared__ uint32_t s_scan[2 * kWarps + 2];
    constexpr int kRows = kBucketScanTile / kBlock;  // 32 rows of 32 counters per warp
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t nb = d.grid_cells >> 6;
    const uint64_t w0 = uint64_t(blockIdx.x) * kBucketScanTile + uint64_t(warp) * 32 * kRows;
    uint32_t v[kRows];
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
        const uint64_t i = w0 + r * 32 + lane;
        v[r] = i < nb ? __ldcg(d.bcount + i) : 0u;
    }
    uint32_t run = 0;  // the warp's counters before this row
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
        uint32_t x = v[r];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, x, o);
            if (lane >= unsigned(o)) x += y;
        }
        const uint32_t row_total = __shfl_sync(kFull, x, 31);
        v[r] = run + x - v[r];
        run += row_total;
    }
    uint32_t total;
    uint32_t wexcl = block_excl_scan(lane == 0 ? run : 0u, s_scan, &total);
    wexcl = __shfl_sync(kFull, wexcl, 0);
    const uint32_t base = uint32_t(d.bsum[blockIdx.x]) + wexcl;
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
        const uint64_t i = w0 + r * 32 + lane;
        if (i < nb) d.bcount[i] = base + v[r];
    }
}

__global__ void __launch_bounds__(kBlock) k_bkt_scatter(BuildDesc d) {
    grid_dep_wait();
    const uint32_t tile = blockIdx.x;
    if (tile >= d.seg_tile[d.seg_count]) return;
    const TileSpan sp = tile_span(d, tile);
    uint32_t* cursor = d.bcount + (__ldg(d.grid_off + sp.seg) >> 6);
    for_tile_entries(d, sp, [&](uint32_t e, uint32_t key, uint32_t val) {
        const uint32_t slot = atomicAdd(cursor + (key >> 6), 1u);
        if (slot < d.n_total) {
            d.brec[slot] = (uint64_t(e + 1) << 32) | val;
            d.bloc[slot] = uint8_t(key & 63);
        } else {
            atomicOr(d.counters + kCtrError, kErrBound);
        }
    });
}

}  // namespace pyrb
