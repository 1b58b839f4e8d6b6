// Dense builds without a sort: a cell grid in HBM (sm_100a).
//
// The reference orders a build's entries with a radix sort and keeps the last entry
// of every key (src/device/gbuild.zig:277-388: stable LSD passes, then uniqueFlags /
// keep / uniqueScatter), and groups the kept keys into bricks (brickHeads /
// brickBuild, :394-428). When the chunks are dense -- a few cells per entry, as in
// generated terrain -- the same result comes from a grid with one 64-bit cell per
// voxel position, laid out in key order (the local key IS the cell's index):
//
//   k_grid_scatter  every entry e at position k does an atomic max of
//                   (e + 1) << 32 | attribute into cell k. The cell keeps the entry
//                   with the largest index: the last one in input order, which is the
//                   entry a stable sort puts last among equal keys. Entries out of
//                   range are dropped, as their invalid key is.
//   k_grid_compact  one streaming pass over the cells in key order, 64 bricks of 64
//                   cells per tile: a cell is a voxel if some entry reached it and its
//                   winner's attribute is not 0 (attribute 0 deletes). Ballots give each
//                   brick's 64-bit mask directly; voxel and brick positions come from
//                   one decoupled look-back over the tiles (both counts packed in one
//                   status word). Output: the sorted unique keys and attributes, the
//                   brick records and the per-chunk first voxel, exactly what the sort
//                   path's k_unique writes.
//
// Bytes: 8 per cell for the zeroing, the atomics' line traffic and the read, against
// 2 (kb + 4) per entry and pass of a sort: the grid wins while a chunk has at most a
// few cells per entry (the host picks the path, see plan_build).
#pragma once

#include "pyrb_kernels.cuh"

namespace pyrb {

constexpr int kGridWarpBricks = 8;                          // bricks per warp and tile
constexpr int kGridTileBricks = kWarps * kGridWarpBricks;   // 64 bricks = 4096 cells per tile

__device__ __forceinline__ void red_max_u64(uint64_t* p, uint64_t v) {
    asm volatile("red.relaxed.gpu.global.max.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Entries -> cells. Tiles follow the per-segment tiling of the sort path (tile_span),
// so the entry index (the order that decides) and the chunk are those of the sort.
__global__ void __launch_bounds__(kBlock) k_grid_scatter(BuildDesc d) {
    grid_dep_wait();
    const uint32_t tile = blockIdx.x;
    if (tile >= d.seg_tile[d.seg_count]) return;
    const TileSpan sp = tile_span(d, tile);
    const uint32_t seg_begin = __ldg(d.seg_entry + sp.seg);
    uint64_t* cells = d.grid + __ldg(d.grid_off + sp.seg);
    const uint32_t inv = 1u << d.lb;
#pragma unroll 4
    for (uint32_t idx = threadIdx.x; idx < sp.count; idx += kBlock) {
        const uint32_t e = sp.start + idx;
        uint32_t key = 0, val = 0;
        load_raw(d, sp.seg, e - seg_begin, key, val);
        if (!(key & inv)) red_max_u64(cells + key, (uint64_t(e + 1) << 32) | val);
    }
}

// Chunk holding cell `cell` (grid_off non-decreasing, grid_off[0] = 0 <= cell).
__device__ __forceinline__ uint32_t grid_chunk(const BuildDesc& d, uint64_t cell) {
    uint32_t lo = 0, hi = d.seg_count;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(d.grid_off + mid) <= cell) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(kBlock) k_grid_compact(BuildDesc d) {
    grid_dep_wait();
    __shared__ uint32_t s_tile;
    __shared__ uint64_t s_scan[2 * kWarps + 2];
    __shared__ uint64_t s_base;
    __shared__ uint32_t s_rcount[kMaxLeafRegions];
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile = dyn_tile(d.counters, 8, &s_tile);
    if (tile >= d.grid_tiles) return;
    const bool regions = d.leaf_regions > 1;
    if (threadIdx.x < kMaxLeafRegions) s_rcount[threadIdx.x] = 0;
    const uint64_t nbricks = d.grid_cells >> 6;
    const uint64_t wb0 = uint64_t(tile) * kGridTileBricks + uint64_t(warp) * kGridWarpBricks;

    // all loads first (16 per lane in flight), cells lane and 32 + lane of each brick;
    // the grid is read once, so the loads stream past L1
    uint64_t c0[kGridWarpBricks], c1[kGridWarpBricks];
#pragma unroll
    for (int k = 0; k < kGridWarpBricks; ++k) {
        const uint64_t b = wb0 + k;
        const uint64_t* cell = d.grid + (b << 6);
        c0[k] = b < nbricks ? __ldcs(reinterpret_cast<const unsigned long long*>(cell + lane)) : 0ull;
        c1[k] = b < nbricks ? __ldcs(reinterpret_cast<const unsigned long long*>(cell + 32 + lane)) : 0ull;
    }
    // a voxel: some entry reached the cell and its winner's attribute is not 0
    unsigned m0[kGridWarpBricks], m1[kGridWarpBricks];
    uint32_t wvox = 0, wbricks = 0;
#pragma unroll
    for (int k = 0; k < kGridWarpBricks; ++k) {
        m0[k] = __ballot_sync(kFull, (c0[k] >> 32) != 0 && uint32_t(c0[k]) != 0);
        m1[k] = __ballot_sync(kFull, (c1[k] >> 32) != 0 && uint32_t(c1[k]) != 0);
        const uint32_t n = __popc(m0[k]) + __popc(m1[k]);
        wvox += n;
        wbricks += n ? 1u : 0u;
    }
    // tile scan of (voxels | bricks << 31) over the warps, then the look-back
    uint64_t total;
    const uint64_t wexcl = block_excl_scan64(lane == 0 ? (uint64_t(wvox) | (uint64_t(wbricks) << 31)) : 0, s_scan, &total);
    const uint64_t wofs = __shfl_sync(kFull, wexcl, 0);
    if (warp == 0) {
        if (lane == 0 && tile != 0) st_relaxed(d.uniq_status + tile, kFlagAgg | total);
        const uint64_t ex = lookback_warp(d.uniq_status, tile, 0, total, d.counters + kCtrError);
        if (lane == 0) s_base = ex;
    }
    __syncthreads();
    const uint64_t base = s_base;
    uint64_t vpos = (base & 0x7FFFFFFFull) + (wofs & 0x7FFFFFFFull);
    uint64_t bpos = (base >> 31) + (wofs >> 31);
    const unsigned lt = lanemask_lt();
    uint32_t seg = 0;
    uint64_t seg_lo = 0, seg_hi = 0;
    if (wb0 < nbricks) {
        seg = grid_chunk(d, wb0 << 6);
        seg_lo = __ldg(d.grid_off + seg);
        seg_hi = __ldg(d.grid_off + seg + 1);
    }
#pragma unroll
    for (int k = 0; k < kGridWarpBricks; ++k) {
        const unsigned lo = m0[k], hi = m1[k];
        if (!(lo | hi)) continue;                       // warp-uniform
        const uint64_t cell = (wb0 + k) << 6;
        while (cell >= seg_hi) {                         // bricks never straddle chunks
            ++seg;
            seg_lo = seg_hi;
            seg_hi = __ldg(d.grid_off + seg + 1);
        }
        const uint64_t key0 = (uint64_t(seg) << d.lb) | (cell - seg_lo);  // key of the brick's first cell
        const uint32_t n0 = __popc(lo);
        if ((lo >> lane) & 1) {
            const uint64_t p = vpos + __popc(lo & lt);
            if (p < d.n_total) {
                d.ukey[p] = key0 + lane;
                d.uval[p] = uint32_t(c0[k]);
            } else {
                atomicOr(d.counters + kCtrError, kErrBound);
            }
        }
        if ((hi >> lane) & 1) {
            const uint64_t p = vpos + n0 + __popc(hi & lt);
            if (p < d.n_total) {
                d.ukey[p] = key0 + 32 + lane;
                d.uval[p] = uint32_t(c1[k]);
            } else {
                atomicOr(d.counters + kCtrError, kErrBound);
            }
        }
        if (lane == 0) {
            const uint64_t mask = uint64_t(lo) | (uint64_t(hi) << 32);
            if (bpos < d.brick_bound) {
                d.bkey[bpos] = key0 >> 6;
                d.bmask[bpos] = mask;
                d.bfirst[bpos] = uint32_t(vpos);
                if (regions) atomicAdd(&s_rcount[leaf_region(d, mask)], 1u);
                if (d.chunked) atomicMin(d.chunk_first + seg, uint32_t(vpos));
            } else {
                atomicOr(d.counters + kCtrError, kErrBound);
            }
        }
        vpos += n0 + __popc(hi);
        ++bpos;
    }
    if (regions) {
        __syncthreads();
        if (threadIdx.x < d.leaf_regions && s_rcount[threadIdx.x])
            atomicAdd(d.region_count + threadIdx.x, s_rcount[threadIdx.x]);
    }
    if (tile == d.grid_tiles - 1 && threadIdx.x == 0) {
        const uint64_t t = base + total;
        d.counters[kCtrUnique] = uint32_t(t & 0x7FFFFFFFull);
        d.counters[kCtrBricks] = uint32_t(t >> 31);
    }
}

}  // namespace pyrb
