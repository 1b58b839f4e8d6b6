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
//   k_grid_count    the compaction, in three passes without waits between tiles:
//   k_grid_scan     a cell is a voxel if its attribute word is not 0 (a cell no entry
//   k_grid_write    reached is all zero; attribute 0 deletes). Tiles of 64 bricks of 64
//                   cells: ballots give each brick's 64-bit mask directly. The count pass
//                   writes every tile's voxels and non-empty bricks, one block scans
//                   them, and the write pass reads the cells again and writes at the
//                   final positions: the sorted unique keys and attributes, the brick
//                   records and the per-chunk first voxel, exactly what the sort path's
//                   k_unique writes. (A single pass with a decoupled look-back measured
//                   barrier-bound: every block waited for its tile's look-back.)
//
// Bytes: 8 per cell for the zeroing, the atomics' line traffic and each of the two
// reads, against 2 (kb + 4) per entry and pass of a sort: the grid wins while a chunk
// has at most a few cells per entry (the host picks the path, see plan_build).
#pragma once

#include "pyrb_kernels.cuh"

namespace pyrb {

constexpr int kGridWarpBricks = 8;                          // bricks per warp and tile
constexpr uint32_t kGridSuper = 64;                         // tiles per group sum (small grids)
constexpr int kGridTileBricks = kWarps * kGridWarpBricks;   // 64 bricks = 4096 cells per tile

__device__ __forceinline__ void red_max_u64(uint64_t* p, uint64_t v) {
    asm volatile("red.relaxed.gpu.global.max.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Every entry of a tile with a valid key, in the per-segment tiling of the sort path
// (tile_span), so the entry index (the order that decides) and the chunk are those of
// the sort: f(entry index, local key, value). PyrVoxel segments (every mode but old
// keys and downsampling) take the fast loop: the chunk's voxel and edit lists are
// resolved once per tile, and each thread keeps kScatterBatch 16-byte loads in flight
// before it encodes them.
constexpr int kScatterBatch = 4;
template <typename F>
__device__ __forceinline__ void for_tile_entries(const BuildDesc& d, const TileSpan& sp, F&& f) {
    const uint32_t seg_begin = __ldg(d.seg_entry + sp.seg);
    const uint32_t inv = 1u << d.lb;
    // the segment's entries: src[0, nv) then esrc[0, ...)
    const uint4* src = nullptr;
    const uint4* esrc = nullptr;
    uint32_t nv = 0, log2c = d.log2;
    bool fast = true;
    switch (d.mode) {
        case kModePlain:
            fast = d.n_old == 0;
            src = d.voxels;
            nv = d.n_new;
            break;
        case kModeChunks:
            src = d.voxels + uint64_t(sp.seg) * d.capacity;
            nv = d.capacity;  // offsets[] never exceed it
            break;
        case kModeChunksEdits:
            src = d.voxels + uint64_t(sp.seg) * d.capacity;
            nv = min(__ldg(d.gen_counts + sp.seg), d.capacity);
            esrc = d.edits + __ldg(d.edit_offsets + sp.seg);
            break;
        case kModeBatch: {
            const uint32_t vo = __ldg(d.voxel_offsets + sp.seg);
            src = d.voxels + (d.voxel_starts ? __ldg(d.voxel_starts + sp.seg) : uint64_t(vo));
            nv = __ldg(d.voxel_offsets + sp.seg + 1) - vo;
            esrc = d.edit_offsets2 ? d.edits + __ldg(d.edit_offsets2 + sp.seg) : nullptr;
            log2c = __ldg(d.chunk_log2 + sp.seg);
            break;
        }
        default:
            fast = false;
            break;
    }
    const uint32_t j0 = sp.start - seg_begin;
    if (!fast) {
#pragma unroll 4
        for (uint32_t idx = threadIdx.x; idx < sp.count; idx += kBlock) {
            const uint32_t e = sp.start + idx;
            uint32_t key = 0, val = 0;
            load_raw(d, sp.seg, e - seg_begin, key, val);
            if (!(key & inv)) f(e, key, val);
        }
        return;
    }
    for (uint32_t base = 0; base < sp.count; base += kScatterBatch * kBlock) {
        uint4 v[kScatterBatch];
#pragma unroll
        for (int k = 0; k < kScatterBatch; ++k) {
            const uint32_t idx = base + k * kBlock + threadIdx.x;
            const uint32_t j = j0 + idx;
            // past the voxel list: the edits, if the segment has any (else the entry is
            // dropped, as load_raw drops a chunk entry past its capacity)
            v[k] = make_uint4(0xFFFFFFFFu, 0, 0, 0);
            if (idx < sp.count) {
                if (j < nv) v[k] = __ldcs(src + j);
                else if (esrc) v[k] = __ldcs(esrc + (j - nv));
            }
        }
#pragma unroll
        for (int k = 0; k < kScatterBatch; ++k) {
            const uint32_t idx = base + k * kBlock + threadIdx.x;
            uint32_t key, val;
            encode_voxel(v[k], log2c, d.lb, key, val);
            if (idx < sp.count && !(key & inv)) f(sp.start + idx, key, val);
        }
    }
}

// Entries -> cells: an atomic max of (entry index + 1) << 32 | value.
__global__ void __launch_bounds__(kBlock) k_grid_scatter(BuildDesc d) {
    grid_dep_wait();
    const uint32_t tile = blockIdx.x;
    if (tile >= d.seg_tile[d.seg_count]) return;
    const TileSpan sp = tile_span(d, tile);
    uint64_t* cells = d.grid + __ldg(d.grid_off + sp.seg);
    for_tile_entries(d, sp, [&](uint32_t e, uint32_t key, uint32_t val) {
        red_max_u64(cells + key, (uint64_t(e + 1) << 32) | val);
    });
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

// The attribute words of a warp's kGridWarpBricks bricks: cells lane and 32 + lane of
// each (a voxel is a cell whose attribute is not 0: a cell no entry reached is all
// zero, and attribute 0 deletes). Only the low half of every 64-bit cell is loaded.
__device__ __forceinline__ void grid_load_attrs(const BuildDesc& d, uint64_t wb0, uint64_t nbricks, uint32_t* a0,
                                                uint32_t* a1) {
    const unsigned lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < kGridWarpBricks; ++k) {
        const uint64_t b = wb0 + k;
        const uint32_t* cell = reinterpret_cast<const uint32_t*>(d.grid + (b << 6));
        a0[k] = b < nbricks ? __ldcg(cell + 2 * lane) : 0u;
        a1[k] = b < nbricks ? __ldcg(cell + 2 * (32 + lane)) : 0u;
    }
}

// The attribute words of a warp's bricks from the brick buckets (sparse builds): the
// warp rebuilds its bricks' 64 cells each in shared memory (the same atomic max of
// (entry index + 1) << 32 | value as the global grid) and reads them back.
__device__ __forceinline__ void bucket_load_attrs(const BuildDesc& d, uint64_t wb0, uint64_t nbricks, uint64_t* cells,
                                                  uint32_t* a0, uint32_t* a1) {
    const unsigned lane = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < kGridWarpBricks * 64 / 32; ++i) cells[i * 32 + lane] = 0;
    // bucket boundaries: lane k < 9 holds the start of brick k (lane 8: the end of brick 7)
    uint32_t c = 0;
    if (lane <= uint32_t(kGridWarpBricks)) {
        const uint64_t b = min(wb0 + lane, nbricks);
        c = b == 0 ? 0u : __ldcg(d.bcount + b - 1);
    }
    uint32_t bound[kGridWarpBricks + 1];
#pragma unroll
    for (int k = 0; k <= kGridWarpBricks; ++k) bound[k] = __shfl_sync(kFull, c, k);
    __syncwarp();
    for (uint32_t j = bound[0] + lane; j < bound[kGridWarpBricks]; j += 32) {
        uint32_t k = 0;
#pragma unroll
        for (int q = 1; q < kGridWarpBricks; ++q) k += j >= bound[q] ? 1u : 0u;
        atomicMax(reinterpret_cast<unsigned long long*>(cells + k * 64 + __ldcs(d.bloc + j)),
                  (unsigned long long)__ldcs(d.brec + j));
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < kGridWarpBricks; ++k) {
        a0[k] = uint32_t(cells[k * 64 + lane]);
        a1[k] = uint32_t(cells[k * 64 + 32 + lane]);
    }
}

// Pass 2: exclusive scan of the tile counts in place (one block, chunks of 16 per
// thread); the totals are the build's voxel and brick counts.
constexpr int kGridScanThreads = 1024, kGridScanPer = 16;
// Exclusive scan of a[0, T) in place by one block of NT threads; returns the total
// (valid in every thread). The values may come from other blocks: read from L2.
template <int NT = kGridScanThreads, int PER = kGridScanPer>
__device__ __forceinline__ uint64_t block_scan_inplace(uint64_t* a, uint32_t T) {
    __shared__ uint64_t s_w[NT / 32];
    __shared__ uint64_t s_carry;
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = NT / 32;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < T; base += NT * PER) {
        const uint32_t i0 = base + threadIdx.x * PER;
        uint64_t v[PER], sum = 0;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            v[j] = i0 + j < T ? __ldcg(a + i0 + j) : 0;
            sum += v[j];
        }
        uint64_t x = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(kFull, x, o);
            if (lane >= unsigned(o)) x += y;
        }
        if (lane == 31) s_w[warp] = x;
        __syncthreads();
        if (warp == 0) {
            const uint64_t w = lane < unsigned(NW) ? s_w[lane] : 0;
            uint64_t sw = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint64_t y = __shfl_up_sync(kFull, sw, o);
                if (lane >= unsigned(o)) sw += y;
            }
            if (lane < unsigned(NW)) s_w[lane] = sw - w;  // exclusive warp offsets
        }
        __syncthreads();
        uint64_t run = s_carry + s_w[warp] + x - sum;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            if (i0 + j < T) a[i0 + j] = run;
            run += v[j];
        }
        __syncthreads();
        if (threadIdx.x == NT - 1) s_carry = run;
        __syncthreads();
    }
    return s_carry;
}

// Pass 1 of the compaction: voxels and non-empty bricks of every tile, packed
// (voxels | bricks << 32) into grid_count[tile]. No dependency between tiles. On grids
// of at most kGridFoldTiles tiles there is no pass 2: every tile's first voxel and
// brick come from the sums of the kGridSuper-tile groups before it and the counts of
// the tiles before it in its group, which the write pass adds up itself.
// kBucket: the cells come from the brick buckets (sparse builds), else from the grid.
template <bool kBucket>
__global__ void __launch_bounds__(kBlock, 8) k_grid_count(BuildDesc d) {
    grid_dep_wait();
    __shared__ uint64_t s_sum[kWarps];
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile = blockIdx.x;
    const uint64_t nbricks = d.grid_cells >> 6;
    const uint64_t wb0 = uint64_t(tile) * kGridTileBricks + uint64_t(warp) * kGridWarpBricks;
    uint32_t a0[kGridWarpBricks], a1[kGridWarpBricks];
    if constexpr (kBucket) {
        __shared__ uint64_t s_cells[kGridTileBricks * 64];
        bucket_load_attrs(d, wb0, nbricks, s_cells + warp * kGridWarpBricks * 64, a0, a1);
    } else {
        grid_load_attrs(d, wb0, nbricks, a0, a1);
    }
    uint32_t vox = 0, bricks = 0;
#pragma unroll
    for (int k = 0; k < kGridWarpBricks; ++k) {
        const uint32_t n = __popc(__ballot_sync(kFull, a0[k] != 0)) + __popc(__ballot_sync(kFull, a1[k] != 0));
        vox += n;
        bricks += n ? 1u : 0u;
    }
    if (lane == 0) s_sum[warp] = uint64_t(vox) | (uint64_t(bricks) << 32);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t t = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) t += s_sum[w];
        d.grid_count[tile] = t;
        // small grids: the sum of every kGridSuper tiles as well (the write pass adds
        // those before its own and the counts in its own group: no scan)
        if (d.grid_fold) atomicAdd(reinterpret_cast<unsigned long long*>(d.grid_super + tile / kGridSuper),
                                   (unsigned long long)t);
    }
}

// Pass 2 on its own (larger grids): one block of kGridScanThreads.
__global__ void __launch_bounds__(kGridScanThreads) k_grid_scan(BuildDesc d) {
    grid_dep_wait();
    const uint64_t total = block_scan_inplace(d.grid_count, d.grid_tiles);
    if (threadIdx.x == 0) {
        d.counters[kCtrUnique] = uint32_t(total);
        d.counters[kCtrBricks] = uint32_t(total >> 32);
    }
}

// Pass 3: every tile again, now with its first voxel and brick from the scan: sorted
// unique keys and attributes, brick records, first voxel of every chunk.
// 5 tiles per SM (48 registers): the tiles write as soon as their loads arrive, so
// more of them in flight keep more loads outstanding. (One pass with a decoupled
// look-back instead of count, scan and write measured slower on large grids, 9.8
// against 8.6 ms on the 1024-chunk mix, and no faster at 2^24 cells.)
template <bool kBucket>
__global__ void __launch_bounds__(kBlock, 5) k_grid_write(BuildDesc d) {
    grid_dep_wait();
    __shared__ uint64_t s_sum[kWarps];
    __shared__ uint64_t s_prefix;
    __shared__ uint32_t s_rcount[kMaxLeafRegions];
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile = blockIdx.x;
    const bool regions = d.leaf_regions > 1;
    if (threadIdx.x < kMaxLeafRegions) s_rcount[threadIdx.x] = 0;
    const uint64_t nbricks = d.grid_cells >> 6;
    const uint64_t wb0 = uint64_t(tile) * kGridTileBricks + uint64_t(warp) * kGridWarpBricks;
    uint32_t a0[kGridWarpBricks], a1[kGridWarpBricks];
    if constexpr (kBucket) {
        __shared__ uint64_t s_cells[kGridTileBricks * 64];
        bucket_load_attrs(d, wb0, nbricks, s_cells + warp * kGridWarpBricks * 64, a0, a1);
    } else {
        grid_load_attrs(d, wb0, nbricks, a0, a1);
    }
    // small grids: warp 0 loads the group sums and counts before this tile now, while
    // the cells are in flight (added up below)
    uint64_t pre = 0;
    if (d.grid_fold && warp == 0) {
        const uint32_t g = tile / kGridSuper, t0 = g * kGridSuper;
        for (uint32_t i = lane; i < g; i += 32) pre += __ldcg(d.grid_super + i);
        for (uint32_t i = t0 + lane; i < tile; i += 32) pre += __ldcg(d.grid_count + i);
    }
    uint32_t vox = 0, bricks = 0;
#pragma unroll
    for (int k = 0; k < kGridWarpBricks; ++k) {
        const uint32_t n = __popc(__ballot_sync(kFull, a0[k] != 0)) + __popc(__ballot_sync(kFull, a1[k] != 0));
        vox += n;
        bricks += n ? 1u : 0u;
    }
    if (lane == 0) s_sum[warp] = uint64_t(vox) | (uint64_t(bricks) << 32);
    __syncthreads();
    uint64_t wofs;  // the tile's first voxel | first brick << 32
    if (d.grid_fold) {
        if (warp == 0) {
            uint64_t x = pre;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
            if (lane == 0) {
                s_prefix = x;
                if (tile == d.grid_tiles - 1) {  // the build's voxel and brick counts
                    uint64_t t = x;
#pragma unroll
                    for (int w = 0; w < kWarps; ++w) t += s_sum[w];
                    d.counters[kCtrUnique] = uint32_t(t);
                    d.counters[kCtrBricks] = uint32_t(t >> 32);
                }
            }
        }
        __syncthreads();
        wofs = s_prefix;
    } else {
        wofs = d.grid_count[tile];
    }
#pragma unroll
    for (int w = 0; w < kWarps; ++w)
        if (w < int(warp)) wofs += s_sum[w];
    uint32_t vpos = uint32_t(wofs), bpos = uint32_t(wofs >> 32);
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
        if (wb0 + k >= nbricks) break;                   // warp-uniform
        const uint64_t cell = (wb0 + k) << 6;
        while (cell >= seg_hi) {                         // bricks never straddle chunks
            ++seg;
            seg_lo = seg_hi;
            seg_hi = __ldg(d.grid_off + seg + 1);
        }
        // the voxels before a chunk's first cell (k_grid_chunks turns them into its first voxel)
        if (d.chunked && cell == seg_lo && lane == 0) d.chunk_vstart[seg] = vpos;
        const unsigned lo = __ballot_sync(kFull, a0[k] != 0), hi = __ballot_sync(kFull, a1[k] != 0);
        if (!(lo | hi)) continue;                       // warp-uniform
        const uint64_t key0 = (uint64_t(seg) << d.lb) | (cell - seg_lo);  // key of the brick's first cell
        const uint32_t n0 = __popc(lo);
        if ((lo >> lane) & 1) {
            const uint32_t p = vpos + __popc(lo & lt);
            if (p < d.n_total) {
                d.ukey[p] = key0 + lane;
                d.uval[p] = a0[k];
            } else {
                atomicOr(d.counters + kCtrError, kErrBound);
            }
        }
        if ((hi >> lane) & 1) {
            const uint32_t p = vpos + n0 + __popc(hi & lt);
            if (p < d.n_total) {
                d.ukey[p] = key0 + 32 + lane;
                d.uval[p] = a1[k];
            } else {
                atomicOr(d.counters + kCtrError, kErrBound);
            }
        }
        if (lane == 0) {
            const uint64_t mask = uint64_t(lo) | (uint64_t(hi) << 32);
            if (bpos < d.brick_bound) {
                d.bkey[bpos] = key0 >> 6;
                d.bmask[bpos] = mask;
                d.bfirst[bpos] = vpos;
                if (regions) atomicAdd(&s_rcount[leaf_region(d, mask)], 1u);
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
}

// First voxel of every chunk of a chunk build (chunkFirst, gbuild.zig:237-242): the
// voxels before its first cell, or 0xFFFFFFFF for a chunk without voxels.
__global__ void __launch_bounds__(kBlock) k_grid_chunks(BuildDesc d) {
    grid_dep_wait();
    const uint32_t total = d.counters[kCtrUnique];
    for (uint32_t c = blockIdx.x * kBlock + threadIdx.x; c < d.seg_count; c += gridDim.x * kBlock) {
        const uint32_t v = d.chunk_vstart[c], next = c + 1 < d.seg_count ? d.chunk_vstart[c + 1] : total;
        d.chunk_first[c] = next > v ? v : 0xFFFFFFFFu;
    }
}

}  // namespace pyrb
