// Kernels of the DAG build (sm_100a). One build = plan -> encode/histogram ->
// onesweep radix passes -> unique -> bricks (+ leaf insert) -> leaf owners ->
// per level {node build (+ insert), node owners} -> prims -> finalize.
//
// Every kernel that assigns output positions uses a decoupled look-back over
// dynamically numbered tiles: a tile only ever waits for tiles with smaller
// numbers, which were taken by blocks that are already running, so the waits
// always end; each wait is additionally bounded (kSpinLimit) and reports
// kErrSpin instead of hanging.
#pragma once

#include "pyrb_device.cuh"

namespace pyrb {

// Programmatic dependent launch: kernels are launched so that they may start while
// the previous kernel of the stream drains; this wait (first statement of every
// kernel) returns once that kernel has completed and its memory is visible.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Largest s in [0, n) with arr[s] <= v (arr non-decreasing, arr[0] <= v).
__device__ __forceinline__ uint32_t upper_index(const uint32_t* arr, uint32_t n, uint32_t v) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(arr + mid) <= v) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ uint32_t dyn_tile(uint32_t* counters, uint32_t ctr, uint32_t* s_slot) {
    if (threadIdx.x == 0) *s_slot = atomicAdd(counters + kCtrTiles + ctr, 1u);
    __syncthreads();
    uint32_t t = *s_slot;
    __syncthreads();
    return t;
}

// The tile id and one counter word in one round trip: the load is issued before the
// atomic's result is waited for.
__device__ __forceinline__ uint32_t dyn_tile_and(uint32_t* counters, uint32_t ctr, uint32_t idx, uint32_t idx2,
                                                 uint32_t* s_slot, uint32_t* val, uint32_t* val2) {
    if (threadIdx.x == 0) {
        const uint32_t v = counters[idx], v2 = counters[idx2];
        s_slot[0] = atomicAdd(counters + kCtrTiles + ctr, 1u);
        s_slot[1] = v;
        s_slot[2] = v2;
    }
    __syncthreads();
    const uint32_t t = s_slot[0];
    *val = s_slot[1];
    *val2 = s_slot[2];
    __syncthreads();
    return t;
}

// 6 tiles per SM for the small levels; large tiles keep their parent's references in
// registers and take 5 (51 registers, no spills)
// ---------------------------------------------------------------------------
// Segment plan: first entry and first sort tile of every segment.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_plan(BuildDesc d) {
    grid_dep_wait();
    __shared__ uint32_t s_scan[2][1024];
    __shared__ uint32_t s_carry[2];
    __shared__ uint64_t s_cells[1024];
    __shared__ uint64_t s_cell_carry;
    const uint32_t K = d.seg_count;
    if (K == 1 && d.mode != kModeChunksEdits) {
        // one segment (a single volume): no scans
        if (threadIdx.x == 0) {
            uint32_t size = d.n_total;
            if (d.mode == kModeChunks) size = __ldg(d.offsets + 1) - __ldg(d.offsets);
            if (d.mode == kModeBatch) {
                size = __ldg(d.voxel_offsets + 1) - __ldg(d.voxel_offsets);
                if (d.edit_offsets2) size += __ldg(d.edit_offsets2 + 1) - __ldg(d.edit_offsets2);
            }
            d.seg_entry[0] = 0;
            d.seg_entry[1] = size;
            d.seg_tile[0] = 0;
            d.seg_tile[1] = (size + d.tile_keys - 1) / d.tile_keys;
            if (d.use_grid | d.use_bucket) {
                const uint32_t l = d.mode == kModeBatch ? __ldg(d.chunk_log2) : d.log2;
                d.grid_off[0] = 0;
                d.grid_off[1] = uint64_t(1) << (3 * l);
            }
        }
        return;
    }
    if (threadIdx.x == 0) { s_carry[0] = 0; s_carry[1] = 0; s_cell_carry = 0; }
    __syncthreads();
    for (uint32_t base = 0; base < K; base += 1024) {
        uint32_t c = base + threadIdx.x;
        uint32_t size = 0;
        if (c < K) {
            switch (d.mode) {
                case kModeChunks: size = __ldg(d.offsets + c + 1) - __ldg(d.offsets + c); break;
                case kModeChunksEdits: {
                    // a count above the capacity is reported, never cut off silently: the
                    // host gets PYRB_ERROR_CAPACITY with the largest count and keeps no
                    // result (reads stay inside the chunk's capacity meanwhile)
                    const uint32_t g = __ldg(d.gen_counts + c);
                    if (g > d.capacity) {
                        atomicMax(d.counters + kCtrNeed, g);
                        atomicOr(d.counters + kCtrError, kErrCapacity);
                    }
                    size = min(g, d.capacity) + (__ldg(d.edit_offsets + c + 1) - __ldg(d.edit_offsets + c));
                    break;
                }
                case kModeBatch:
                    size = __ldg(d.voxel_offsets + c + 1) - __ldg(d.voxel_offsets + c);
                    if (d.edit_offsets2) size += __ldg(d.edit_offsets2 + c + 1) - __ldg(d.edit_offsets2 + c);
                    break;
                default: size = d.n_total; break;
            }
        }
        uint32_t tiles = (size + d.tile_keys - 1) / d.tile_keys;
        s_scan[0][threadIdx.x] = size;
        s_scan[1][threadIdx.x] = tiles;
        __syncthreads();
        // inclusive Hillis-Steele scan of both arrays
        for (uint32_t o = 1; o < 1024; o <<= 1) {
            uint32_t a = threadIdx.x >= o ? s_scan[0][threadIdx.x - o] : 0;
            uint32_t b = threadIdx.x >= o ? s_scan[1][threadIdx.x - o] : 0;
            __syncthreads();
            s_scan[0][threadIdx.x] += a;
            s_scan[1][threadIdx.x] += b;
            __syncthreads();
        }
        if (c < K) {
            d.seg_entry[c] = s_carry[0] + s_scan[0][threadIdx.x] - size;
            d.seg_tile[c] = s_carry[1] + s_scan[1][threadIdx.x] - tiles;
        }
        if (d.use_grid | d.use_bucket) {
            // first cell of every chunk in the cell grid (chunk after chunk)
            const uint32_t l = c < K ? (d.mode == kModeBatch ? __ldg(d.chunk_log2 + c) : d.log2) : 0;
            const uint64_t cells = c < K ? uint64_t(1) << (3 * l) : 0;
            s_cells[threadIdx.x] = cells;
            __syncthreads();
            for (uint32_t o = 1; o < 1024; o <<= 1) {
                const uint64_t a = threadIdx.x >= o ? s_cells[threadIdx.x - o] : 0;
                __syncthreads();
                s_cells[threadIdx.x] += a;
                __syncthreads();
            }
            if (c < K) d.grid_off[c] = s_cell_carry + s_cells[threadIdx.x] - cells;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_carry[0] += s_scan[0][1023];
            s_carry[1] += s_scan[1][1023];
            if (d.use_grid | d.use_bucket) s_cell_carry += s_cells[1023];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        d.seg_entry[K] = s_carry[0];
        d.seg_tile[K] = s_carry[1];
        if (d.use_grid | d.use_bucket) d.grid_off[K] = s_cell_carry;
    }
}

// ---------------------------------------------------------------------------
// Encode: raw entry -> (key, value). Out-of-range voxels get the invalid bit
// (bit lb), which sorts them behind every valid key of their segment; the
// unique stage drops them (same rule as gbuild.encode / packChunks).
// ---------------------------------------------------------------------------
template <typename KeyT>
__device__ __forceinline__ void encode_voxel(uint4 v, uint32_t log2, uint32_t lb, KeyT& key, uint32_t& val) {
    const int32_t n = int32_t(1u << log2);
    int32_t x = int32_t(v.x), y = int32_t(v.y), z = int32_t(v.z);
    if (x < 0 || y < 0 || z < 0 || x >= n || y >= n || z >= n) {
        key = KeyT(1) << lb;
        val = 0;
    } else {
        key = KeyT(voxel_key(uint32_t(x), uint32_t(y), uint32_t(z)));
        val = v.w;
    }
}

template <typename KeyT>
__device__ __forceinline__ void load_raw(const BuildDesc& d, uint32_t seg, uint32_t j, KeyT& key, uint32_t& val) {
    switch (d.mode) {
        case kModePlain:
            if (j < d.n_old) {
                key = KeyT(__ldg(d.old_keys + j));
                val = __ldg(d.old_vals + j);
            } else {
                encode_voxel(__ldg(d.voxels + (j - d.n_old)), d.log2, d.lb, key, val);
            }
            break;
        case kModeChunks:
            if (j < d.capacity) encode_voxel(__ldg(d.voxels + uint64_t(seg) * d.capacity + j), d.log2, d.lb, key, val);
            else { key = KeyT(1) << d.lb; val = 0; }
            break;
        case kModeChunksEdits: {
            uint32_t g = min(__ldg(d.gen_counts + seg), d.capacity);
            uint4 v = j < g ? __ldg(d.voxels + uint64_t(seg) * d.capacity + j)
                            : __ldg(d.edits + __ldg(d.edit_offsets + seg) + (j - g));
            encode_voxel(v, d.log2, d.lb, key, val);
            break;
        }
        case kModeBatch: {
            const uint32_t vo = __ldg(d.voxel_offsets + seg), vn = __ldg(d.voxel_offsets + seg + 1) - vo;
            const uint64_t vb = d.voxel_starts ? __ldg(d.voxel_starts + seg) : uint64_t(vo);
            const uint4 v = j < vn ? __ldg(d.voxels + vb + j) : __ldg(d.edits + __ldg(d.edit_offsets2 + seg) + (j - vn));
            encode_voxel(v, __ldg(d.chunk_log2 + seg), d.lb, key, val);
            break;
        }
        default: {  // downsample (gbuild.zig:262-274): coarse key of the source voxel
            uint64_t k = __ldg(d.src_keys + j);
            uint64_t brick = k >> 6;
            uint32_t bit = uint32_t(k & 63), sh = d.shift;
            uint32_t x = ((compact3(brick) << 2) | (bit & 3)) >> sh;
            uint32_t y = ((compact3(brick >> 1) << 2) | ((bit >> 2) & 3)) >> sh;
            uint32_t z = ((compact3(brick >> 2) << 2) | (bit >> 4)) >> sh;
            key = KeyT(voxel_key(x, y, z));
            val = __ldg(d.src_vals + j);
            break;
        }
    }
}

// Tile -> (segment, first entry, entry count) of the per-segment sort tiling.
struct TileSpan { uint32_t seg, start, count, first_tile; };
__device__ __forceinline__ TileSpan tile_span(const BuildDesc& d, uint32_t tile) {
    TileSpan t;
    t.seg = upper_index(d.seg_tile, d.seg_count + 1, tile);
    // empty segments share tile numbers with the next one: move to the segment owning the tile
    while (t.seg + 1 < d.seg_count && __ldg(d.seg_tile + t.seg + 1) <= tile) ++t.seg;
    t.first_tile = __ldg(d.seg_tile + t.seg);
    uint32_t seg_begin = __ldg(d.seg_entry + t.seg), seg_end = __ldg(d.seg_entry + t.seg + 1);
    t.start = seg_begin + (tile - t.first_tile) * d.tile_keys;
    t.count = min(d.tile_keys, seg_end - t.start);
    return t;
}

// ---------------------------------------------------------------------------
// Encode + histogram of every pass ("onesweep" upfront histogram).
// ---------------------------------------------------------------------------
template <int RB, int IT, typename KeyT>
__global__ void __launch_bounds__(kBlock) k_encode_hist(BuildDesc d) {
    grid_dep_wait();
    constexpr int RADIX = 1 << RB;
    extern __shared__ uint32_t smem[];
    uint32_t* hist = smem;  // [passes][RADIX]
    const uint32_t tile = blockIdx.x;
    if (tile >= d.seg_tile[d.seg_count]) return;
    const TileSpan sp = tile_span(d, tile);
    for (uint32_t i = threadIdx.x; i < d.passes * RADIX; i += kBlock) hist[i] = 0;
    __syncthreads();
    const uint32_t seg_begin = __ldg(d.seg_entry + sp.seg);
    // one shared-memory increment per entry and pass (counting runs of equal digits per
    // lane first measured 1.7x slower: a lane's entries are kBlock apart, so its runs are
    // short, and the run bookkeeping costs registers and branches)
#pragma unroll 4
    for (int j = 0; j < IT; ++j) {
        uint32_t idx = j * kBlock + threadIdx.x;
        if (idx < sp.count) {
            KeyT key = 0;
            uint32_t val = 0;
            uint32_t e = sp.start + idx;
            load_raw(d, sp.seg, e - seg_begin, key, val);
            static_cast<KeyT*>(d.kbuf[0])[e] = key;
            d.vbuf[0][e] = val;
#pragma unroll
            for (int p = 0; p < kMaxPasses; ++p) {
                if (uint32_t(p) >= d.passes) break;
                const uint32_t dig = uint32_t(key >> d.pass_shift[p]) & ((1u << d.pass_bits[p]) - 1);
                atomicAdd(hist + p * RADIX + dig, 1u);
            }
        }
    }
    __syncthreads();
    uint32_t* gh = d.hist + uint64_t(sp.seg) * d.passes * RADIX;
    for (uint32_t i = threadIdx.x; i < d.passes * RADIX; i += kBlock) {
        uint32_t v = hist[i];
        if (v) atomicAdd(gh + i, v);
    }
}

// Exclusive scan of RADIX digit counts in smem (in -> out) by NT threads, DPT
// consecutive digits per thread.
template <int RADIX, int NT = kBlock>
__device__ __forceinline__ void scan_digits(const uint32_t* in, uint32_t* out, uint32_t* scratch) {
    constexpr int DPT = (RADIX + NT - 1) / NT;
    uint32_t local[DPT];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < DPT; ++k) {
        uint32_t dg = threadIdx.x * DPT + k;
        local[k] = dg < uint32_t(RADIX) ? in[dg] : 0;
        sum += local[k];
    }
    uint32_t total;
    uint32_t run = block_excl_scan<NT / 32>(sum, scratch, &total);
#pragma unroll
    for (int k = 0; k < DPT; ++k) {
        uint32_t dg = threadIdx.x * DPT + k;
        if (dg < uint32_t(RADIX)) out[dg] = run;
        run += local[k];
    }
}

// ---------------------------------------------------------------------------
// Onesweep radix sort passes.
// ---------------------------------------------------------------------------
// Digit bases: the histogram of every (segment, pass) becomes its exclusive prefix
// in place, once, so that the tiles of the sort passes read their segment's digit
// starts instead of each scanning the histogram again.
template <int RB>
__global__ void __launch_bounds__(kBlock) k_digit_base(BuildDesc d) {
    grid_dep_wait();
    constexpr int RADIX = 1 << RB;
    __shared__ uint32_t s_in[RADIX], s_out[RADIX], s_scratch[2 * kWarps + 4];
    uint32_t* h = d.hist + uint64_t(blockIdx.x) * RADIX;  // blockIdx.x = seg * passes + pass
    for (uint32_t i = threadIdx.x; i < uint32_t(RADIX); i += kBlock) s_in[i] = h[i];
    __syncthreads();
    scan_digits<RADIX>(s_in, s_out, s_scratch);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < uint32_t(RADIX); i += kBlock) h[i] = s_out[i];
}

template <int RB, int IT, typename KeyT, int NT = kBlock>
constexpr size_t sort_smem_bytes() {
    constexpr int RADIX = 1 << RB, TILE = NT * IT, NW = NT / 32;
    constexpr int KW = int(sizeof(KeyT) / 4);  // words per key
    constexpr int U = (NW * RADIX > (KW + 1) * TILE) ? NW * RADIX : (KW + 1) * TILE;
    return size_t(U + 3 * RADIX + 2 * NW + 8 + TILE) * 4;
}

// Asynchronous 4-byte global -> shared copies (cp.async): no register holds the value
// while it is in flight.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// One LSD pass of the onesweep radix sort over a tile of NT * IT entries (NT threads):
//  1. keys are loaded warp-striped (a warp owns 32 * IT consecutive entries) and
//     ranked in input order with match_any against per-warp digit counters;
//  2. the tile's digit counts are published at once as aggregates for the
//     decoupled look-back of later tiles, and their exclusive scan gives the
//     tile-local position of every key, so the keys go to shared memory in digit
//     order while their registers free up;
//  3. the values are loaded only now (fewer live registers during ranking, so more
//     tiles per SM) and their loads overlap the look-back of this tile's digits;
//  4. each digit's run is written contiguously from shared memory at the segment's
//     digit base (k_digit_base) + the look-back prefix.
#ifndef PYRB_SORT_WINDOW
#define PYRB_SORT_WINDOW 2
#endif
constexpr int kSortWindow = PYRB_SORT_WINDOW;  // predecessors per look-back round
#ifndef PYRB_MATCH_MAX_GROUPS
#define PYRB_MATCH_MAX_GROUPS 16
#endif
constexpr int kMatchMaxGroups = PYRB_MATCH_MAX_GROUPS;  // distinct digits per warp above which ballots are cheaper

// 4 resident 256-thread tiles (or 2 of 512 threads) per SM: caps the pass at 64
// registers (the 16-key tiles spill a few words, cheaper than the lost occupancy)
#ifndef PYRB_SORT_MIN_BLOCKS
#define PYRB_SORT_MIN_BLOCKS 4
#endif
template <int RB, int IT, typename KeyT, int NT = kBlock>
__global__ void __launch_bounds__(NT, PYRB_SORT_MIN_BLOCKS * kBlock / NT) k_sort_pass(BuildDesc d, uint32_t pass, uint32_t src) {
    grid_dep_wait();
    constexpr int RADIX = 1 << RB, TILE = NT * IT, NW = NT / 32;
    constexpr int KW = int(sizeof(KeyT) / 4);
    constexpr int U = (NW * RADIX > (KW + 1) * TILE) ? NW * RADIX : (KW + 1) * TILE;
    extern __shared__ uint32_t smem[];
    uint32_t* whist = smem;               // [NW][RADIX], later staging keys|vals
    uint32_t* tcnt = smem + U;            // tile count per digit
    uint32_t* texcl = tcnt + RADIX;       // tile-exclusive digit offsets
    uint32_t* gofs = texcl + RADIX;       // global write offset per digit
    uint32_t* scratch = gofs + RADIX;     // 2*NW + 1 words
    uint32_t* s_tile = scratch + 2 * NW + 4;
    uint32_t* vland = s_tile + 4;         // [TILE] values in tile order, copied asynchronously

    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile = dyn_tile(d.counters, kTileSort0 + pass, s_tile);
    if (tile >= d.seg_tile[d.seg_count]) return;
    const TileSpan sp = tile_span(d, tile);
    const uint32_t shift = d.pass_shift[pass], dmask = (1u << d.pass_bits[pass]) - 1;
    const KeyT* kin = static_cast<const KeyT*>(d.kbuf[src]);
    const uint32_t* vin = d.vbuf[src];
    KeyT* kout = static_cast<KeyT*>(d.kbuf[src ^ 1]);
    uint32_t* vout = d.vbuf[src ^ 1];
    const uint32_t* gbase = d.hist + (uint64_t(sp.seg) * d.passes + pass) * RADIX;

    for (uint32_t i = threadIdx.x; i < uint32_t(NW * RADIX); i += NT) whist[i] = 0;
    KeyT keys[IT];
    uint32_t rank[IT];
#pragma unroll
    for (int j = 0; j < IT; ++j) {
        uint32_t idx = warp * 32 * IT + j * 32 + lane;
        keys[j] = idx < sp.count ? kin[sp.start + idx] : KeyT(0);
    }
    // the values travel to shared memory while the keys are ranked (each thread copies
    // and later reads the same entries, so its own wait suffices)
#pragma unroll
    for (int j = 0; j < IT; ++j) {
        uint32_t idx = warp * 32 * IT + j * 32 + lane;
        if (idx < sp.count) cp_async4(vland + idx, vin + sp.start + idx);
    }
    cp_async_commit();
    __syncthreads();
    const unsigned lt = lanemask_lt();
    uint32_t* wh = whist + warp * RADIX;
    // Peer masks first (independent of each other), then the counter chain. match_any
    // costs grow with the number of distinct digits in the warp; once a warp sees
    // more than kMatchMaxGroups of them, it switches to RB ballots (one per digit bit),
    // whose cost is fixed. Both give the same masks.
    unsigned pm[IT];
    bool by_bits = false;  // warp-uniform
#pragma unroll
    for (int j = 0; j < IT; ++j) {
        const uint32_t idx = warp * 32 * IT + j * 32 + lane;
        const bool valid = idx < sp.count;
        const uint32_t dig = valid ? uint32_t(keys[j] >> shift) & dmask : 0xFFFFFFFFu;
        if (!by_bits) {
            pm[j] = __match_any_sync(kFull, dig);
            const unsigned heads = __ballot_sync(kFull, lane == unsigned(__ffs(pm[j]) - 1));
            by_bits = __popc(heads) > kMatchMaxGroups;
        } else {
            unsigned peers = __ballot_sync(kFull, valid);
#pragma unroll
            for (int b = 0; b < RB; ++b) {
                const unsigned bb = __ballot_sync(kFull, (dig >> b) & 1u);
                peers &= ((dig >> b) & 1u) ? bb : ~bb;
            }
            pm[j] = peers;
        }
    }
#pragma unroll
    for (int j = 0; j < IT; ++j) {
        uint32_t idx = warp * 32 * IT + j * 32 + lane;
        bool valid = idx < sp.count;
        uint32_t dig = valid ? uint32_t(keys[j] >> shift) & dmask : 0xFFFFFFFFu;
        const unsigned peers = pm[j];
        uint32_t cnt = valid ? wh[dig] : 0;
        rank[j] = cnt + __popc(peers & lt);
        __syncwarp();
        if (valid && lane == unsigned(__ffs(peers) - 1)) wh[dig] = cnt + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // cross-warp exclusive offsets per digit, tile totals, published at once
    uint64_t* status = d.sort_status + uint64_t(pass) * d.sort_tiles * RADIX;
    for (uint32_t dg = threadIdx.x; dg < uint32_t(RADIX); dg += NT) {
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            uint32_t c = whist[w * RADIX + dg];
            whist[w * RADIX + dg] = run;
            run += c;
        }
        tcnt[dg] = run;
        if (tile != sp.first_tile) st_relaxed(status + uint64_t(tile) * RADIX + dg, kFlagAgg | run);
    }
    __syncthreads();
    scan_digits<RADIX, NT>(tcnt, texcl, scratch);
    __syncthreads();
    // tile-local ranks; then keys to shared memory in digit order
#pragma unroll
    for (int j = 0; j < IT; ++j) {
        uint32_t idx = warp * 32 * IT + j * 32 + lane;
        if (idx < sp.count) {
            uint32_t dig = uint32_t(keys[j] >> shift) & dmask;
            rank[j] += texcl[dig] + wh[dig];
        }
    }
    __syncthreads();
    KeyT* sk = reinterpret_cast<KeyT*>(whist);
    uint32_t* sv = whist + KW * TILE;
    cp_async_wait_all();
#pragma unroll
    for (int j = 0; j < IT; ++j) {
        uint32_t idx = warp * 32 * IT + j * 32 + lane;
        if (idx < sp.count) {
            sk[rank[j]] = keys[j];
            sv[rank[j]] = vland[idx];
        }
    }
    // look-back per digit (the tile's entries are staged: few live registers)
    const uint32_t seg_begin = __ldg(d.seg_entry + sp.seg);
    for (uint32_t dg = threadIdx.x; dg < uint32_t(RADIX); dg += NT) {
        uint64_t excl = lookback_window<kSortWindow>(status + dg, RADIX, tile, sp.first_tile, tcnt[dg],
                                                     d.counters + kCtrError);
        gofs[dg] = seg_begin + __ldg(gbase + dg) + uint32_t(excl) - texcl[dg];
    }
    __syncthreads();
    const uint32_t seg_end = __ldg(d.seg_entry + sp.seg + 1);
    bool oob = false;
    for (uint32_t i = threadIdx.x; i < sp.count; i += NT) {
        KeyT k = sk[i];
        uint32_t pos = gofs[uint32_t(k >> shift) & dmask] + i;
        if (pos >= seg_begin && pos < seg_end) {
            kout[pos] = k;
            vout[pos] = sv[i];
        } else {
            oob = true;
        }
    }
    if (oob) atomicOr(d.counters + kCtrError, kErrBound);
}

// ---------------------------------------------------------------------------
// Unique voxels and bricks, one pass over the entries ordered by brick.
// The sort orders the entries by brick (key >> 6 with the invalid bit left out) and,
// being stable, by entry index inside a brick; the 6 cell bits stay unsorted, which
// saves a sort pass. Unique: the last entry of each key decides; it is kept if it is
// valid and its attribute is non-zero (gbuild.zig:366-388). Bricks (brickHeads/
// brickBuild, :394-428): the kept voxels of a brick give its 64-bit mask, and the
// voxels are written in cell order at the brick's first voxel + the rank of their cell
// in the mask, so the unique keys come out sorted as the reference's do. Positions by
// look-backs over the tiles in global (segment-major) order; keys get the segment
// (chunk) number above bit lb, like packChunks; chunkFirst (:237-242).
// A brick's run of entries belongs to the tile holding its first entry. The tile
// stages its entries in shared memory and finds the runs that start in it; one warp
// reads past the tile's end while its last run goes on, keeping per cell the last
// entry seen there. Each run is then taken by one thread, from its last entry back:
// the first sighting of a cell is its last entry, the cell's winner.
// ---------------------------------------------------------------------------

// Table region of a mask's home slot (see BuildDesc::leaf_regions).
__device__ __forceinline__ uint32_t leaf_region(const BuildDesc& d, uint64_t mask) {
    return (uint32_t(mix64(mask)) & (d.leaf_cap - 1)) >> d.leaf_region_shift;
}

template <int IT, typename KeyT>
constexpr size_t unique_smem_bytes() {
    return size_t(kBlock) * IT * (sizeof(KeyT) + 2 + 2);  // keys, run starts, destinations
}

// Unique tiles of kBlock * kUniqIT entries (4096; a larger sort tile is taken in parts):
// 2048-entry tiles at 5, 6 or 7 per SM measured 8-14 % slower, the fixed cost of a
// tile (scans, look-backs) being paid twice as often.
constexpr int kUniqIT = 16;
template <int IT, typename KeyT>
// 5 tiles per SM (48 registers): the tile mostly waits for its predecessors' counts,
// so more tiles in flight per SM measured 17 % faster than 4 at 64 registers
__global__ void __launch_bounds__(kBlock, 5) k_unique(BuildDesc d, uint32_t fin) {
    grid_dep_wait();
    constexpr int TILE = kBlock * IT;
    constexpr unsigned RA = kWarps - 1;  // reads past the tile's end, takes its last run, looks back
    constexpr uint16_t kNoDst = 0xFFFF;
    extern __shared__ __align__(16) unsigned char usmem[];
    KeyT* s_key = reinterpret_cast<KeyT*>(usmem);                  // [TILE] the tile's keys (+ zero flag)
    uint16_t* s_head = reinterpret_cast<uint16_t*>(s_key + TILE);  // [TILE] first entry of each run
    uint16_t* s_dst = s_head + TILE;                               // [TILE] a kept winner's place in the tile's voxels
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_scan[2 * kWarps];  // warp sums of the two scans
    __shared__ uint64_t s_ubase, s_bbase;
    __shared__ uint32_t s_tpos[64], s_tval[64];     // past the end: last entry (+1) and attribute per cell
    __shared__ uint32_t s_rcount[kMaxLeafRegions];  // the tile's bricks per leaf-table region
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // a sort tile larger than TILE entries is taken in parts, each a unique tile
    const uint32_t parts = d.tile_keys / TILE;
    const uint32_t tile = dyn_tile(d.counters, kTileUnique, &s_tile);
    const uint32_t ntiles = d.seg_tile[d.seg_count] * parts;
    if (tile >= ntiles) return;
    TileSpan sp = tile_span(d, tile / parts);
    {
        const uint32_t skip = (tile % parts) * TILE;
        sp.start += skip;
        sp.count = sp.count > skip ? min(sp.count - skip, uint32_t(TILE)) : 0u;
    }
    const uint32_t seg_begin = __ldg(d.seg_entry + sp.seg), seg_end = __ldg(d.seg_entry + sp.seg + 1);
    const uint32_t e_end = sp.start + sp.count;
    const KeyT* keys = static_cast<const KeyT*>(d.kbuf[fin]);
    const uint32_t* vals = d.vbuf[fin];
    const KeyT inv = KeyT(1) << d.lb;
    const KeyT zero = KeyT(1) << (d.lb + 1);  // staged keys: the entry's attribute is 0 (a free bit)
    const KeyT bbits = (KeyT(1) << (d.lb - 6)) - 1;
    const KeyT NONE = ~KeyT(0);  // never a brick: bricks have at most lb - 6 bits
    auto brick = [&](KeyT k) -> KeyT { return (k >> 6) & bbits; };
    const uint32_t wbase = warp * 32 * IT;
    const bool regions = d.leaf_regions > 1;
    if (threadIdx.x < kMaxLeafRegions) s_rcount[threadIdx.x] = 0;

    // the read-ahead warp's first loads go out with the tile's: the 32 entries after
    // the tile (a tile short of TILE entries ends its segment)
    KeyT ra_k = NONE, klast = NONE;
    uint32_t ra_v = 0;
    if (warp == RA) {
        s_tpos[lane] = 0;
        s_tpos[lane + 32] = 0;
        if (sp.count > 0 && e_end + lane < seg_end) {
            ra_k = keys[e_end + lane];
            ra_v = vals[e_end + lane];
        }
    }
    // no destination yet for any entry (IT 16-bit words per thread, 16 bytes a store)
    static_assert(IT % 8 == 0 || IT < 8, "whole 16-byte stores, or the scalar loop");
    if constexpr (IT % 8 == 0) {
#pragma unroll
        for (int q = 0; q < IT / 8; ++q)
            reinterpret_cast<uint4*>(s_dst + threadIdx.x * IT)[q] = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
    } else {
#pragma unroll
        for (int q = 0; q < IT; ++q) s_dst[threadIdx.x * IT + q] = kNoDst;
    }
    uint32_t v[IT];  // the attributes stay in registers until the voxels are written
    unsigned hb[IT];  // runs that start in the tile: an entry whose brick differs from the one before it
    uint32_t wheads = 0;
    {
        KeyT k[IT];
        // the entry before the warp's first (lane 0): the tile's lead or the previous warp's last
        KeyT kprev = NONE;
        if (lane == 0 && wbase < sp.count && (wbase > 0 || sp.start > seg_begin)) kprev = brick(keys[sp.start + wbase - 1]);
#pragma unroll
        for (int j = 0; j < IT; ++j) {
            const uint32_t idx = wbase + j * 32 + lane;
            const bool in = idx < sp.count;
            k[j] = in ? keys[sp.start + idx] : KeyT(0);
            v[j] = in ? vals[sp.start + idx] : 0u;
        }
#pragma unroll
        for (int j = 0; j < IT; ++j) {
            const uint32_t idx = wbase + j * 32 + lane;
            const bool in = idx < sp.count;
            const KeyT up = __shfl_up_sync(kFull, k[j], 1);
            const KeyT row_prev = __shfl_sync(kFull, j > 0 ? k[j > 0 ? j - 1 : 0] : k[0], 31);
            const KeyT pb = lane > 0 ? brick(up) : j > 0 ? brick(row_prev) : kprev;
            hb[j] = __ballot_sync(kFull, in && brick(k[j]) != pb);
            wheads += __popc(hb[j]);
            if (in) s_key[idx] = k[j] | (v[j] == 0 ? zero : KeyT(0));
        }
        // the tile's last entry (only a full tile can have entries after it: its last
        // entry is the read-ahead warp's lane 31's)
        klast = __shfl_sync(kFull, k[IT - 1], 31);
    }
    uint32_t R;
    {
        uint32_t hexcl = block_excl_scan1(lane == 0 ? wheads : 0u, s_scan, &R);
        hexcl = __shfl_sync(kFull, hexcl, 0);
#pragma unroll
        for (int j = 0; j < IT; ++j) {
            if ((hb[j] >> lane) & 1) s_head[hexcl + __popc(hb[j] & lanemask_lt())] = uint16_t(wbase + j * 32 + lane);
            hexcl += __popc(hb[j]);
        }
    }
    __syncthreads();
    // The tile's last run (it started here when R > 0) may go on past the tile's end:
    // the read-ahead warp keeps per cell the last entry there, while the other warps
    // walk the other runs; its lane 0 then walks the last run.
    uint64_t tcells = 0, tkeep = 0;
    if (warp == RA) {
        if (R > 0 && e_end < seg_end) {
            {  // the cleared s_tpos is visible: block barriers since
                const KeyT rb = brick(klast);
                uint32_t base = e_end;
                KeyT kk = ra_k;
                uint32_t vv = ra_v;
                while (true) {
                    const uint32_t e = base + lane;
                    const bool in_run = e < seg_end && brick(kk) == rb;
                    const bool use = in_run && !(kk & inv);
                    const uint32_t p = e - e_end + 1, c = uint32_t(kk) & 63;
                    if (use) atomicMax(s_tpos + c, p);
                    __syncwarp();
                    if (use && s_tpos[c] == p) s_tval[c] = vv;  // the cell's last entry so far
                    __syncwarp();
                    if (!__all_sync(kFull, in_run)) break;
                    base += 32;
                    const uint32_t e2 = base + lane;
                    kk = e2 < seg_end ? keys[e2] : NONE;
                    vv = e2 < seg_end ? vals[e2] : 0u;
                }
            }
        }
        const uint32_t pa = s_tpos[lane], pb = s_tpos[lane + 32];
        const unsigned ca = __ballot_sync(kFull, pa != 0), cb = __ballot_sync(kFull, pb != 0);
        const unsigned ka = __ballot_sync(kFull, pa != 0 && s_tval[lane] != 0);
        const unsigned kb = __ballot_sync(kFull, pb != 0 && s_tval[lane + 32] != 0);
        tcells = uint64_t(cb) << 32 | ca;
        tkeep = uint64_t(kb) << 32 | ka;
    }
    // kept cells of each run: thread t of the first kRunThreads takes runs [t q, t q + q)
    // of all but the last, the read-ahead warp's lane 0 the last one (it starts from the
    // cells seen past the tile's end); the read-ahead warp then looks back
    constexpr uint32_t kRunThreads = kBlock - 32;
    const uint32_t Rw = R > 0 ? R - 1 : 0;
    const uint32_t q = (Rw + kRunThreads - 1) / kRunThreads;
    uint32_t r_lo = R, r_hi = R;
    if (threadIdx.x < kRunThreads) {
        r_lo = min(threadIdx.x * q, Rw);
        r_hi = min(r_lo + q, Rw);
    } else if (threadIdx.x == kRunThreads && R > 0) {
        r_lo = R - 1;
    }
    auto run_end = [&](uint32_t r) -> uint32_t { return r + 1 < R ? uint32_t(s_head[r + 1]) : sp.count; };
    // a run from its last entry back, 4 entries a step (their loads in flight together);
    // visit(i, first_sighting_bit, k) for each entry
    auto walk = [&](uint32_t lo, uint32_t hi, uint64_t seen, auto&& visit) {
        for (uint32_t i = hi; i > lo; i = i > lo + 4 ? i - 4 : lo) {
            KeyT kq[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) kq[u] = i > lo + u ? s_key[i - 1 - u] : inv;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint64_t bit = (kq[u] & inv) ? 0ull : 1ull << (uint32_t(kq[u]) & 63);
                const uint64_t nb = bit & ~seen;
                seen |= bit;
                visit(i - 1 - u, nb, kq[u]);
            }
        }
    };
    auto run_mask = [&](uint32_t r, uint32_t lo, uint32_t hi) -> uint64_t {
        uint64_t km = r + 1 == R ? tkeep : 0;
        walk(lo, hi, r + 1 == R ? tcells : 0, [&](uint32_t, uint64_t nb, KeyT k) { km |= (k & zero) ? 0ull : nb; });
        return km;
    };
    uint64_t m0 = 0, m1 = 0;  // the masks of the thread's first two runs, kept for the second walk
    uint32_t packed = 0;      // kept voxels << 16 | bricks
    for (uint32_t r = r_lo; r < r_hi; ++r) {
        const uint64_t km = run_mask(r, s_head[r], run_end(r));
        if (r == r_lo) m0 = km;
        else if (r == r_lo + 1) m1 = km;
        packed += (uint32_t(__popcll(km)) << 16) + (km != 0 ? 1u : 0u);
    }
    uint32_t ptotal;
    const uint32_t pexcl = block_excl_scan1(packed, s_scan + kWarps, &ptotal);
    const uint32_t total = ptotal >> 16, btotal = ptotal & 0xFFFFu;
    // positions are global over all segments: the read-ahead warp publishes the tile's
    // voxel and brick counts as one status word (voxels << 31 | bricks: both stay below
    // 2^31), places the last run's winners and looks back to tile 0 for both offsets at
    // once, while the others place the winners of their runs
    const uint64_t agg = uint64_t(total) << 31 | btotal;
    if (warp == RA && lane == 0 && tile != 0) st_relaxed(d.uniq_status + tile, kFlagAgg | agg);
    // each kept cell's winner goes to the rank of its cell in the brick's mask
    {
        uint32_t uo = pexcl >> 16;
        for (uint32_t r = r_lo; r < r_hi; ++r) {
            const uint32_t lo = s_head[r], hi = run_end(r);
            const uint64_t km = r == r_lo ? m0 : r == r_lo + 1 ? m1 : run_mask(r, lo, hi);
            if (km == 0) continue;
            walk(lo, hi, r + 1 == R ? tcells : 0, [&](uint32_t i, uint64_t nb, KeyT) {
                if (nb & km) s_dst[i] = uint16_t(uo + __popcll(km & (nb - 1)));
            });
            uo += uint32_t(__popcll(km));
        }
    }
    if (warp == RA) {
        const uint64_t ex = lookback_warp(d.uniq_status, tile, 0, agg, d.counters + kCtrError);
        if (lane == 0) {
            s_ubase = ex >> 31;
            s_bbase = ex & 0x7FFFFFFFull;
        }
    }
    __syncthreads();
    const uint64_t ubase = s_ubase, bbase = s_bbase;
    const uint64_t segbits = uint64_t(sp.seg) << d.lb;
    auto put = [&](uint64_t pos, uint64_t key, uint32_t val) {
        if (pos < d.n_total) {
            d.ukey[pos] = key;
            d.uval[pos] = val;
        } else {
            atomicOr(d.counters + kCtrError, kErrBound);
        }
    };
    // the voxels, in the tile's entry order (a row's winners land close together)
#pragma unroll
    for (int j = 0; j < IT; ++j) {
        const uint32_t idx = wbase + j * 32 + lane;
        if (idx < sp.count) {
            const uint32_t dst = s_dst[idx];
            if (dst != kNoDst) put(ubase + dst, segbits | uint64_t(s_key[idx]), v[j]);
        }
    }
    // the bricks, and the last run's winners found past the tile's end
    {
        uint32_t uo = pexcl >> 16, bo = pexcl & 0xFFFFu;
        for (uint32_t r = r_lo; r < r_hi; ++r) {
            const uint32_t lo = s_head[r];
            const uint64_t km = r == r_lo ? m0 : r == r_lo + 1 ? m1 : run_mask(r, lo, run_end(r));
            if (km == 0) continue;
            const uint64_t bk = uint64_t(brick(s_key[lo]));
            const uint64_t first = ubase + uo, g = bbase + bo;
            if (g < d.brick_bound) {
                d.bkey[g] = (segbits >> 6) | bk;
                d.bmask[g] = km;
                d.bfirst[g] = uint32_t(first);
                if (regions) atomicAdd(&s_rcount[leaf_region(d, km)], 1u);
            } else {
                atomicOr(d.counters + kCtrError, kErrBound);
            }
            if (r + 1 == R) {
                for (uint64_t t = tkeep; t; t &= t - 1) {
                    const uint32_t c = uint32_t(__ffsll(t) - 1);
                    put(first + __popcll(km & ((1ull << c) - 1)), segbits | bk << 6 | c, s_tval[c]);
                }
            }
            uo += uint32_t(__popcll(km));
            ++bo;
        }
    }
    if (regions) {
        __syncthreads();
        if (threadIdx.x < d.leaf_regions && s_rcount[threadIdx.x])
            atomicAdd(d.region_count + threadIdx.x, s_rcount[threadIdx.x]);
    }
    if (d.chunked && threadIdx.x == 0 && total > 0) atomicMin(d.chunk_first + sp.seg, uint32_t(ubase));
    if (tile == ntiles - 1 && threadIdx.x == 0) {
        d.counters[kCtrUnique] = uint32_t(ubase + total);
        d.counters[kCtrBricks] = uint32_t(bbase + btotal);
    }
}

// ---------------------------------------------------------------------------
// Dedup tables. Leaf table slot: {mask lo, mask hi, ~owner, -};
// node table slot: {key + 1, 0, ~owner, node offset}. ~owner with
// atomicMax makes the minimum index the owner on zero-initialised tables.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void claim_owner(uint4* slot, uint32_t idx) {
    uint32_t* op = &slot->z;
    uint32_t inv = ~idx;
    if (ld_relaxed32(op) < inv) atomicMax(op, inv);
}

// Linear probing wraps inside the slot's region of smask + 1 slots (the whole table
// unless the table is filled region by region).
__device__ __forceinline__ uint32_t probe_next(uint32_t h, uint32_t smask) { return (h & ~smask) | ((h + 1) & smask); }

// 16-byte compare-and-swap: installs {lo, hi} if the slot holds {clo, chi}; returns the
// slot's value before (an atomic snapshot of all 16 bytes).
__device__ __forceinline__ void cas128(void* p, uint64_t clo, uint64_t chi, uint64_t lo, uint64_t hi, uint64_t& olo,
                                       uint64_t& ohi) {
    asm volatile(
        "{\n\t.reg .b128 d, b, c;\n\tmov.b128 b, {%2, %3};\n\tmov.b128 c, {%4, %5};\n\t"
        "atom.relaxed.gpu.global.cas.b128 d, [%6], b, c;\n\tmov.b128 {%0, %1}, d;\n\t}"
        : "=l"(olo), "=l"(ohi)
        : "l"(clo), "l"(chi), "l"(lo), "l"(hi), "l"(p)
        : "memory");
}

// Leaf owners without a second look at the table. A brick becomes the owner of its
// mask's slot when it installs itself (the 16-byte claim of an empty slot writes mask
// and ~index at once; a later brick with a smaller index raises ~owner with a returning
// atomicMax); whoever replaces an owner learns which one from the atomic's result and
// marks it displaced. The minimum index is the only brick that installed itself and was
// never displaced: binst holds the installed marks, bdisp the displaced ones, and the
// owner pass reads just those two streams. A brick that is not the owner finds its
// mask's slot again by probing (leaf_find), as the insert did.
constexpr uint32_t kInstalled = 0x80000000u;
constexpr uint32_t kSlotMask = 0x7FFFFFFFu;

// A brick whose mask is in slot s (its ~owner last seen as z): tries to become the
// owner. Returns kInstalled if it did.
__device__ __forceinline__ uint32_t leaf_claim(const BuildDesc& d, uint4* slot, uint32_t idx, uint32_t z) {
    const uint32_t inv = ~idx;
    if (z >= inv) return 0;  // ~owner only grows: an owner at or below idx exists already
    const uint32_t old = atomicMax(&slot->z, inv);
    if (old >= inv) return 0;
    if (old != 0) d.bdisp[~old] = 1;  // the owner replaced
    return kInstalled;
}

// Insert of mask m (brick idx) from slot h on, probe0 probes already taken; returns the
// slot | kInstalled when the brick became its owner.
__device__ __forceinline__ uint32_t leaf_insert_at(const BuildDesc& d, uint4* table, uint32_t smask, uint64_t mask,
                                                   uint32_t idx, uint32_t h, uint32_t probe0) {
    for (uint32_t probe = probe0; probe <= smask; ++probe) {
        uint4* slot = table + h;
        uint64_t cur = ld_relaxed(reinterpret_cast<const uint64_t*>(slot));
        uint32_t z = 0;
        if (cur == 0) {
            uint64_t ohi;
            cas128(slot, 0, 0, mask, uint64_t(~idx), cur, ohi);
            if (cur == 0 && ohi == 0) return h | kInstalled;
            z = uint32_t(ohi);
        } else {
            z = ld_relaxed32(&slot->z);
        }
        if (cur == mask) return h | leaf_claim(d, slot, idx, z);
        h = probe_next(h, smask);
    }
    atomicOr(d.counters + kCtrError, kErrTable);
    return 0;
}

// The first probe of N inserts, their loads and claims in flight together (each thread
// takes N bricks per round: the inserts are latency-bound on random table slots).
// out[k]: slot | kInstalled.
template <int N>
__device__ __forceinline__ void leaf_insert_n(const BuildDesc& d, uint4* table, uint32_t cap, uint32_t smask,
                                              const bool (&w)[N], const uint64_t (&m)[N], const uint32_t (&idx)[N],
                                              uint32_t (&out)[N]) {
    uint32_t h[N], z[N];
    uint64_t r[N];
    bool f[N];
#pragma unroll
    for (int k = 0; k < N; ++k) {
        h[k] = uint32_t(mix64(m[k])) & (cap - 1);
        // the slot's first 16 bytes as one load: mask and (possibly older) ~owner
        const uint4 c = w[k] ? __ldcg(table + h[k]) : make_uint4(0, 0, 0, 0);
        r[k] = uint64_t(c.y) << 32 | c.x;
        z[k] = c.z;
        f[k] = false;
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
        if (w[k] && r[k] == 0) {
            uint64_t hi;
            cas128(table + h[k], 0, 0, m[k], uint64_t(~idx[k]), r[k], hi);
            f[k] = r[k] == 0 && hi == 0;
            z[k] = uint32_t(hi);
        }
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
        if (!w[k]) continue;
        if (f[k]) out[k] = h[k] | kInstalled;
        else if (r[k] == m[k]) out[k] = h[k] | leaf_claim(d, table + h[k], idx[k], z[k]);
        else out[k] = leaf_insert_at(d, table, smask, m[k], idx[k], probe_next(h[k], smask), 1);
    }
}

// The slot holding `mask` (it was inserted): the same probe sequence as the insert,
// each probe one 16-byte load that also returns the slot's ~owner.
__device__ __forceinline__ uint4 leaf_find(const BuildDesc& d, uint64_t mask) {
    const uint32_t smask = d.leaf_regions > 1 ? d.leaf_cap / d.leaf_regions - 1 : d.leaf_cap - 1;
    uint32_t h = uint32_t(mix64(mask)) & (d.leaf_cap - 1);
    for (uint32_t probe = 0; probe <= smask; ++probe) {
        const uint4 v = __ldcg(d.leaf_table + h);
        if ((uint64_t(v.y) << 32 | v.x) == mask) return v;
        h = probe_next(h, smask);
    }
    atomicOr(d.counters + kCtrError, kErrTable);
    return make_uint4(0, 0, 0, 0);
}

// Brick-indexed kernels (leaf owners) take tiles of kBrickTile bricks.
constexpr int kBrickIT = 8;
constexpr int kBrickTile = kBlock * kBrickIT;

// Per-region starts of tiles (clearing tiles, then insert tiles) and of the region's
// bricks in the grouped list, for every region at once by warp 0 (one round trip).
__device__ __forceinline__ void region_bases(const BuildDesc& d, uint32_t nz, uint32_t per_tile, uint32_t* tbase,
                                             uint32_t* ibase) {
    static_assert(kMaxLeafRegions == 64, "two regions per lane");
    const unsigned lane = threadIdx.x & 31;
    const uint32_t R = d.leaf_regions;
    const uint32_t ra = lane, rb = lane + 32;
    const uint32_t ca = ra < R ? __ldcg(d.region_count + ra) : 0, cb = rb < R ? __ldcg(d.region_count + rb) : 0;
    const uint32_t ta = ra < R ? nz + (ca + per_tile - 1) / per_tile : 0;
    const uint32_t tb = rb < R ? nz + (cb + per_tile - 1) / per_tile : 0;
    uint32_t xa = ta, xb = tb, ya = ca, yb = cb;  // inclusive scans
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t p0 = __shfl_up_sync(kFull, xa, o), p1 = __shfl_up_sync(kFull, xb, o);
        const uint32_t p2 = __shfl_up_sync(kFull, ya, o), p3 = __shfl_up_sync(kFull, yb, o);
        if (lane >= unsigned(o)) { xa += p0; xb += p1; ya += p2; yb += p3; }
    }
    xb += __shfl_sync(kFull, xa, 31);
    yb += __shfl_sync(kFull, ya, 31);
    if (ra < R) { tbase[ra] = xa - ta; ibase[ra] = ya - ca; }
    if (rb < R) { tbase[rb] = xb - tb; ibase[rb] = yb - cb; }
    const uint32_t tt = __shfl_sync(kFull, xb, 31), tbs = __shfl_sync(kFull, yb, 31);
    if (lane == 0) { tbase[R] = tt; ibase[R] = tbs; }
}

// Bricks grouped by the leaf-table region of their mask (BuildDesc::leaf_regions):
// per tile, ranks within each region by shared-memory counters, one global cursor
// reservation per region; the order inside a region does not matter (the owner is
// the minimum brick index whatever the insert order).
__global__ void __launch_bounds__(kBlock) k_leaf_part(BuildDesc d) {
    grid_dep_wait();
    __shared__ uint32_t s_base[kMaxLeafRegions + 1], s_cnt[kMaxLeafRegions], s_res[kMaxLeafRegions];
    __shared__ uint32_t s_tb[kMaxLeafRegions + 1];
    const uint32_t B = min(d.counters[kCtrBricks], d.brick_bound);
    const uint32_t R = d.leaf_regions;
    if (threadIdx.x < 32) region_bases(d, 0, 1, s_tb, s_base);  // s_base: each region's first brick
    for (uint32_t t0 = blockIdx.x * kBrickTile; t0 < B; t0 += gridDim.x * kBrickTile) {
        if (threadIdx.x < R) s_cnt[threadIdx.x] = 0;
        __syncthreads();
        uint64_t m[kBrickIT];
        uint32_t reg[kBrickIT], rk[kBrickIT];
#pragma unroll
        for (int j = 0; j < kBrickIT; ++j) {
            const uint32_t b = t0 + j * kBlock + threadIdx.x;
            m[j] = b < B ? d.bmask[b] : 0;
        }
#pragma unroll
        for (int j = 0; j < kBrickIT; ++j) {
            const uint32_t b = t0 + j * kBlock + threadIdx.x;
            reg[j] = leaf_region(d, m[j]);
            rk[j] = b < B ? atomicAdd(&s_cnt[reg[j]], 1u) : 0u;
        }
        __syncthreads();
        if (threadIdx.x < R && s_cnt[threadIdx.x]) s_res[threadIdx.x] = atomicAdd(d.region_cursor + threadIdx.x, s_cnt[threadIdx.x]);
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kBrickIT; ++j) {
            const uint32_t b = t0 + j * kBlock + threadIdx.x;
            if (b < B) {
                const uint32_t p = s_base[reg[j]] + s_res[reg[j]] + rk[j];
                if (p < B) {
                    d.pmask[p] = m[j];
                    d.pidx[p] = b;
                } else {
                    atomicOr(d.counters + kCtrError, kErrBound);
                }
            }
        }
        __syncthreads();  // s_cnt and s_res are reused by the next tile
    }
}

// Leaf dedup insert in brick order, two bricks per thread per round. Equal masks of a
// warp row are collapsed with match_any first: only the lowest brick of each group
// touches the table.
__global__ void __launch_bounds__(kBlock) k_leaf_insert(BuildDesc d) {
    grid_dep_wait();
    constexpr int N = 2;
    const uint32_t B = min(d.counters[kCtrBricks], d.brick_bound);
    const unsigned lane = threadIdx.x & 31;
    const uint32_t stride = gridDim.x * kBlock;
    for (uint32_t base = blockIdx.x * kBlock; base < B; base += N * stride) {
        bool v[N], w[N];
        uint64_t m[N];
        uint32_t b[N], s[N], l[N];
#pragma unroll
        for (int k = 0; k < N; ++k) {
            b[k] = base + threadIdx.x + k * stride;
            v[k] = b[k] < B;
            m[k] = v[k] ? d.bmask[b[k]] : 0;  // masks are never 0
        }
#pragma unroll
        for (int k = 0; k < N; ++k) {
            l[k] = __ffs(__match_any_sync(kFull, m[k])) - 1;
            w[k] = v[k] && lane == l[k];
            s[k] = 0;
        }
        leaf_insert_n<N>(d, d.leaf_table, d.leaf_cap, d.leaf_cap - 1, w, m, b, s);
#pragma unroll
        for (int k = 0; k < N; ++k) {
            s[k] = __shfl_sync(kFull, s[k], l[k]);
            // the other bricks of a group: the lowest lane holds the lowest brick here (brick
            // order), but they claim all the same, so that the rule stays the same everywhere
            if (v[k] && lane != l[k]) {
                uint4* sl = d.leaf_table + (s[k] & kSlotMask);
                s[k] = (s[k] & kSlotMask) | leaf_claim(d, sl, b[k], ld_relaxed32(&sl->z));
            }
            if (v[k] && (s[k] & kInstalled)) d.binst[b[k]] = 1;
        }
    }
}

// Leaf dedup insert region by region (BuildDesc::leaf_regions > 1), over the bricks
// grouped by region (k_leaf_part). The tiles of a region, taken in order, first clear
// the region's slots (the table is not cleared before the build), then insert its
// bricks once every clearing tile of the region has finished: the region's slots are
// written while they sit in L2 and the inserts find them there. Probing wraps inside
// the region. A tile waits only for tiles with smaller numbers, which are running or
// done; the wait is bounded.
#ifndef PYRB_ZERO_SLOTS
#define PYRB_ZERO_SLOTS 2048
#endif
constexpr uint32_t kZeroSlots = PYRB_ZERO_SLOTS;  // slots a clearing tile clears (32 KB)
// Bricks per thread of an insert tile: one (tiles of 256 bricks) measured fastest at
// 1024^3 (leaf inserts 0.67 ms against 0.70 with two and 0.87 with four in flight per
// thread: smaller tiles keep more of them resident and waiting less)
#ifndef PYRB_INS_PER_THREAD
#define PYRB_INS_PER_THREAD 1
#endif
constexpr int kInsPerThread = PYRB_INS_PER_THREAD;
constexpr uint32_t kInsTile = kInsPerThread * kBlock;  // bricks an insert tile takes

__global__ void __launch_bounds__(kBlock) k_leaf_insert_regions(BuildDesc d) {
    grid_dep_wait();
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_tbase[kMaxLeafRegions + 1], s_ibase[kMaxLeafRegions + 1];
    const uint32_t R = d.leaf_regions, S = d.leaf_cap / R, smask = S - 1;
    const uint32_t nz = (S + kZeroSlots - 1) / kZeroSlots;
    if (threadIdx.x < 32) region_bases(d, nz, kInsTile, s_tbase, s_ibase);
    const uint32_t tile = dyn_tile(d.counters, kTileLeafInsert, &s_tile);  // its barrier publishes s_tbase
    if (tile >= s_tbase[R]) return;
    uint32_t r = 0;
    while (s_tbase[r + 1] <= tile) ++r;
    const uint32_t k = tile - s_tbase[r];
    uint4* region = d.leaf_table + size_t(r) * S;
    if (k < nz) {
        const uint32_t end = min(S, (k + 1) * kZeroSlots);
        for (uint32_t i = k * kZeroSlots + threadIdx.x; i < end; i += kBlock) region[i] = make_uint4(0u, 0u, 0u, 0u);
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(d.region_zeroed + r, 1u);
        }
        return;
    }
    if (threadIdx.x == 0) {
        uint32_t spins = 0;
        while (ld_acquire32(d.region_zeroed + r) < nz) {
            if (++spins > kSpinLimit) { atomicOr(d.counters + kCtrError, kErrSpin); break; }
            if (spins > 8) __nanosleep(128);
        }
    }
    __syncthreads();
    const uint32_t B = min(d.counters[kCtrBricks], d.brick_bound);
    const unsigned lane = threadIdx.x & 31;
    constexpr int N = kInsPerThread;
    const uint32_t iend = s_ibase[r + 1];
    uint32_t ii[N], b[N], s[N], l[N];
    bool v[N], w[N];
    uint64_t m[N];
#pragma unroll
    for (int q = 0; q < N; ++q) {
        ii[q] = s_ibase[r] + (k - nz) * kInsTile + q * kBlock + threadIdx.x;
        b[q] = ii[q] < iend ? d.pidx[ii[q]] : 0u;
        m[q] = ii[q] < iend ? d.pmask[ii[q]] : 0;
    }
#pragma unroll
    for (int q = 0; q < N; ++q) {
        v[q] = ii[q] < iend && b[q] < B;  // b >= B: never, unless counts disagree
        if (ii[q] < iend && !v[q]) atomicOr(d.counters + kCtrError, kErrBound);
        if (!v[q]) m[q] = 0;              // masks are never 0
        l[q] = __ffs(__match_any_sync(kFull, m[q])) - 1;
        w[q] = v[q] && lane == l[q];
        s[q] = 0;
    }
    leaf_insert_n<N>(d, d.leaf_table, d.leaf_cap, smask, w, m, b, s);
#pragma unroll
    for (int q = 0; q < N; ++q) {
        s[q] = __shfl_sync(kFull, s[q], l[q]);
        // the lowest lane of a group need not hold its lowest brick: the others claim too
        if (v[q] && lane != l[q]) {
            uint4* sl = d.leaf_table + (s[q] & kSlotMask);
            s[q] = (s[q] & kSlotMask) | leaf_claim(d, sl, b[q], ld_relaxed32(&sl->z));
        }
        // one byte per brick that became an owner: scattered, but the array stays in L2
        if (v[q] && (s[q] & kInstalled)) d.binst[b[q]] = 1;
    }
}

// ---------------------------------------------------------------------------
// Leaf owners: bricks whose mask they own get leaf positions in brick order
// (= first occurrence in Morton order); the table slot records the leaf index.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_leaf_own(BuildDesc d) {
    grid_dep_wait();
    __shared__ uint32_t s_tile[3];
    __shared__ uint32_t s_scan[2 * kWarps + 2];
    __shared__ uint64_t s_base;
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t bcount, unused;
    const uint32_t tile = dyn_tile_and(d.counters, kTileLeafOwn, kCtrBricks, kCtrBricks, s_tile, &bcount, &unused);
    const uint32_t B = min(bcount, d.brick_bound);
    const uint32_t ntiles = (B + kBrickTile - 1) / kBrickTile;
    if (tile >= ntiles) return;
    const uint32_t wstart = tile * kBrickTile + warp * 32 * kBrickIT;
    unsigned ob[kBrickIT];
    uint8_t inst[kBrickIT], disp[kBrickIT];
    uint32_t wc = 0;
    // owners: installed and never displaced (two coalesced streams, no table reads)
#pragma unroll
    for (int j = 0; j < kBrickIT; ++j) {
        uint32_t b = wstart + j * 32 + lane;
        inst[j] = b < B ? __ldcg(d.binst + b) : uint8_t(0);
        disp[j] = b < B ? __ldcg(d.bdisp + b) : uint8_t(1);
    }
#pragma unroll
    for (int j = 0; j < kBrickIT; ++j) {
        uint32_t b = wstart + j * 32 + lane;
        const bool own = b < B && inst[j] && !disp[j];
        ob[j] = __ballot_sync(kFull, own);
        wc += __popc(ob[j]);
    }
    uint32_t total;
    uint32_t wexcl = block_excl_scan(lane == 0 ? wc : 0, s_scan, &total);
    wexcl = __shfl_sync(kFull, wexcl, 0);
    if (warp == 0) {
        if (lane == 0 && tile != 0) st_relaxed(d.leafown_status + tile, kFlagAgg | total);
        uint64_t ex = lookback_warp(d.leafown_status, tile, 0, total, d.counters + kCtrError);
        if (lane == 0) s_base = ex;
    }
    __syncthreads();
    uint32_t run = uint32_t(s_base) + wexcl;
#pragma unroll
    for (int j = 0; j < kBrickIT; ++j) {
        uint32_t b = wstart + j * 32 + lane;
        uint32_t ref = kNoRef;
        if ((ob[j] >> lane) & 1) {
            uint32_t pos = run + __popc(ob[j] & lanemask_lt());
            if (pos < d.brick_bound) d.leaves[pos] = d.bmask[b];
            else atomicOr(d.counters + kCtrError, kErrBound);
            ref = pos;
        }
        if (b < B) d.bref[b] = ref;
        run += __popc(ob[j]);
    }
    if (tile == ntiles - 1 && threadIdx.x == 0) d.counters[kCtrLeaves] = uint32_t(s_base + total);
}

// ---------------------------------------------------------------------------
// Node level lv: children grouped by key >> 3 into parents (<= 8 children each),
// words [mask, saturating count, refs...] (gbuild.zig:484-520), inserted into
// the level's table (equal words -> same slot, owner = minimum parent index).
// ---------------------------------------------------------------------------
// Node words are [mask, count, ref_0 .. ref_{n-1}]; the hash only places table
// slots (equality is decided by comparing all words).
__device__ __forceinline__ uint64_t node_hash(uint32_t mask, uint32_t count, const uint32_t (&refs)[8], uint32_t n) {
    uint64_t h = mix64(mix64(uint64_t(n + 2) ^ mask) ^ count);
#pragma unroll
    for (uint32_t k = 0; k < 8; ++k)
        if (k < n) h = mix64(h ^ refs[k]);
    return h;
}

// Insert parent `par` into the level table. Its words are at key_words[key * stride]
// (stored before this call: the CAS releases them); colliding residents are compared
// by their words at key_words[(resident key) * stride]. h is the home slot, refs the
// parent's child references. Returns the slot; the minimum parent index owns it.
__device__ __forceinline__ uint32_t node_insert(uint4* table, uint32_t cap, const uint32_t* key_words, uint32_t key,
                                                uint32_t par, uint32_t h, uint32_t mask, uint32_t count,
                                                const uint32_t (&refs)[8], uint32_t n, uint32_t* err) {
    for (uint32_t probe = 0; probe < cap; ++probe) {
        uint32_t* kp = &table[h].x;
        uint32_t cur = ld_acquire32(kp);
        if (cur == 0) {
            // release: our words (stored before this call) are visible with the key
            cur = cas_acq_rel32(kp, 0u, key + 1);
            if (cur == 0) {
                atomicMax(&table[h].z, ~par);  // first of its words: claim without waiting
                return h;
            }
        }
        // acquired above: the resident's words are visible
        const uint32_t* ow = key_words + uint64_t(cur - 1) * kNodeStride;
        uint32_t o[kNodeStride];
#pragma unroll
        for (int k = 0; k < int(kNodeStride); k += 2) {
            uint2 v = __ldcg(reinterpret_cast<const uint2*>(ow + k));
            o[k] = v.x;
            o[k + 1] = v.y;
        }
        bool same = o[0] == mask && o[1] == count;
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (uint32_t(k) < n) same = same && o[2 + k] == refs[k];
        if (same) {
            claim_owner(table + h, par);
            return h;
        }
        h = (h + 1) & (cap - 1);
    }
    atomicOr(err, kErrTable);
    return 0;
}

__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// Leaf index of brick b: its own (it owns its mask) or its mask's owner's, found
// through the table's owner word (only bricks that repeat a mask take this gather).
__device__ __forceinline__ uint32_t brick_ref(const BuildDesc& d, uint32_t b) {
    const uint32_t r = __ldcg(d.bref + b);
    return r != kNoRef ? r : __ldcg(d.bref + ~leaf_find(d, __ldcg(d.bmask + b)).z);
}

// Per-child shared arrays of the node build are padded by one slot every 8 children:
// a thread walks its parent's children, so the lanes of a warp read children ~8 apart
// (one parent each), which without padding hit the same banks (16-way for 8-byte
// words).
__device__ __forceinline__ uint32_t cpad(uint32_t i) { return i + (i >> 3); }

// Assembles the parent whose first child is staged at i: mask, saturating count,
// number of children, their references, box (when needed; at level 2 from the brick
// masks).
struct NodeParent {
    uint32_t mask, count, n;
    uint32_t lo[3], hi[3];
    uint32_t refs[8];
};
__device__ __forceinline__ NodeParent node_assemble(const LevelDesc& L, const uint64_t* skey, const uint64_t* slo,
                                                    const uint64_t* shi, const uint32_t* scnt, const uint32_t* sref,
                                                    uint32_t i, uint32_t tn) {
    NodeParent q;
    q.mask = 0; q.count = 0; q.n = 0;
    q.lo[0] = q.lo[1] = q.lo[2] = 0xFFFFFFFFu;
    q.hi[0] = q.hi[1] = q.hi[2] = 0;
    const uint64_t pkey = skey[cpad(i)] >> 3;
    const uint32_t child_size = 1u << L.lv;
    bool in = true;
#pragma unroll
    for (uint32_t k = 0; k < 8; ++k) {
        const uint32_t j = i + k;
        uint64_t ck = 0;
        in = in && j < tn;
        if (in) {
            ck = skey[cpad(j)];
            in = (ck >> 3) == pkey;
        }
        q.refs[k] = 0;
        if (!in) continue;
        const uint32_t idx = uint32_t(ck & 7);
        q.mask |= 1u << idx;
        q.count = sat_add(q.count, scnt[cpad(j)]);
        q.refs[k] = sref[cpad(j)];
        if (L.need_box) {
            const uint32_t ox = (idx & 1) * child_size, oy = ((idx >> 1) & 1) * child_size,
                           oz = (idx >> 2) * child_size;
            uint64_t clo = slo[cpad(j)], chi = shi[cpad(j)];
            if (L.lv == 2) brick_box(clo, clo, chi);
            q.lo[0] = min(q.lo[0], cell_x(clo) + ox); q.hi[0] = max(q.hi[0], cell_x(chi) + ox);
            q.lo[1] = min(q.lo[1], cell_y(clo) + oy); q.hi[1] = max(q.hi[1], cell_y(chi) + oy);
            q.lo[2] = min(q.lo[2], cell_z(clo) + oz); q.hi[2] = max(q.hi[2], cell_z(chi) + oz);
        }
        q.n = k + 1;
    }
    return q;
}

// Records of parent `par` (key, count, first voxel, box, table slot and, when asked
// for, its words).
__device__ __forceinline__ void node_store(const LevelDesc& L, uint32_t par, const NodeParent& q, uint64_t pkey,
                                           uint32_t first, uint32_t slot, bool words) {
    if (words) {
        uint32_t* pw = L.pwords + uint64_t(par) * kNodeStride;
        pw[0] = q.mask;
        pw[1] = q.count;
#pragma unroll
        for (uint32_t k = 0; k < 8; ++k)
            if (k < q.n) pw[2 + k] = q.refs[k];
    }
    L.pkey[par] = pkey;
    L.pcnt[par] = q.count;
    L.pfirst[par] = first;
    if (L.need_box) {
        L.plo[par] = pack_cell(q.lo[0], q.lo[1], q.lo[2]);
        L.phi[par] = pack_cell(q.hi[0], q.hi[1], q.hi[2]);
    }
    L.pslot[par] = slot;
}

// Tile of the node build: kBlock * NB children staged in shared memory (plus a halo
// of up to 7 children of the tile's last parent), heads found with warp ballots,
// positions by a look-back scan, then every thread builds parents from shared memory
// and inserts them into the level's table.
// Parents per thread of the node-owner kernel and children per thread of the node
// build: large levels take 8 and 4 (tiles of 2048 parents / 1024 children), levels
// small enough to leave most SMs idle with those take 1 (tiles of 256), so that their
// tiles spread over the whole GPU (plan_build picks per level).
// Small levels (NB == 1) are latency-bound: a global round trip costs about a
// microsecond, an acquire-release atomic several. There every load of a staging step
// is in flight together, and each parent (at most one per thread) is assembled before
// the look-back: its words go to L.cwords at its first child's index (the table key of
// these levels), so that the release of the insert after the look-back finds them long
// performed, and its home slot is prefetched into the L2.
constexpr int kNodeIT = 8;
constexpr int kNodeTile = kBlock * kNodeIT;     // tile of the node-owner kernel (large levels)
constexpr int kNBIT = 4;
constexpr int kNodeBuildTile = kBlock * kNBIT;  // children per node-build tile (large levels)
constexpr int kNodeHalo = 8;
// Level 2 stages the children's brick masks (its parents' boxes come from them) rather
// than their boxes: 28 instead of 36 bytes per child, 6 tiles per SM instead of 5.
constexpr size_t node_build_smem_bytes(bool bricks, int nb = kNBIT) {
    return size_t(kBlock * nb + kNodeHalo + (kBlock * nb + kNodeHalo) / 8 + 1) *
               (bricks ? 8 + 8 + 4 + 4 + 4 : 8 + 8 + 8 + 4 + 4 + 4) +
           size_t(kBlock * nb) * 4 + 64;
}

template <int NB>
__device__ __forceinline__ void node_build_tile(const BuildDesc& d, const LevelDesc& L, const uint32_t tile,
                                                const uint32_t children) {
    extern __shared__ uint64_t smem64[];
    constexpr int kTile = kBlock * NB;
    constexpr int N = kTile + kNodeHalo;
    constexpr int NP = N + N / 8 + 1;                // padded (cpad) per-child arrays
    uint64_t* skey = smem64;
    uint64_t* slo = skey + NP;                       // level 2: the brick masks
    uint64_t* shi = L.lv == 2 ? slo : slo + NP;
    uint32_t* sref = reinterpret_cast<uint32_t*>(shi + NP);
    uint32_t* scnt = sref + NP;
    uint32_t* sfirst = scnt + NP;
    uint32_t* shead = sfirst + NP;
    __shared__ uint32_t s_scan[2 * kWarps + 2];
    __shared__ uint64_t s_base;
    __shared__ uint64_t s_prev;
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t C = min(children, L.lv == 2 ? d.brick_bound : L.child_bound);
    const uint32_t ntiles = (C + kTile - 1) / kTile;
    if (tile >= ntiles) return;
    const uint32_t t0 = tile * kTile;
    const uint32_t own_n = min(uint32_t(kTile), C - t0);
    const uint32_t tn = min(uint32_t(N), C - t0);
    constexpr int SPT = (N + kBlock - 1) / kBlock;
    if constexpr (NB == 1) {
        // stage the children, every load of a step in flight together: the records,
        // then (level 2) the owners of repeated masks and their leaf indices, or the
        // children's node offsets from the level below's table
        uint64_t key[SPT], lo[SPT], hi[SPT];
        uint32_t first[SPT], cnt[SPT], ref[SPT], slot[SPT];
#pragma unroll
        for (int r = 0; r < SPT; ++r) {
            const uint32_t i = threadIdx.x + r * kBlock;
            const bool v = i < tn;
            const uint32_t c = t0 + i;
            key[r] = v ? L.ckey[c] : 0;
            first[r] = v ? L.cfirst[c] : 0;
            lo[r] = 0;
            hi[r] = 0;
            if (L.lv == 2) {
                lo[r] = v ? L.cmask[c] : 0;
                ref[r] = v ? __ldcg(d.bref + c) : 0;
                slot[r] = 0;
                cnt[r] = __popcll(lo[r]);
            } else {
                cnt[r] = v ? L.ccnt[c] : 0;
                slot[r] = v ? L.cslot[c] : 0;
                ref[r] = 0;
                if (L.need_box && v) { lo[r] = L.clo[c]; hi[r] = L.chi[c]; }
            }
        }
        if (L.lv == 2) {
            // a brick that repeats a mask: its mask's slot (found by probing) names the owner
            uint32_t own[SPT];
#pragma unroll
            for (int r = 0; r < SPT; ++r)
                own[r] = threadIdx.x + r * kBlock < tn && ref[r] == kNoRef ? ~leaf_find(d, lo[r]).z : 0;
#pragma unroll
            for (int r = 0; r < SPT; ++r)
                if (threadIdx.x + r * kBlock < tn && ref[r] == kNoRef) ref[r] = __ldcg(d.bref + own[r]);
        } else {
#pragma unroll
            for (int r = 0; r < SPT; ++r)
                if (threadIdx.x + r * kBlock < tn) ref[r] = __ldcg(&L.ctable[slot[r]].w);
        }
#pragma unroll
        for (int r = 0; r < SPT; ++r) {
            const uint32_t i = threadIdx.x + r * kBlock;
            if (i < tn) {
                const uint32_t pi = cpad(i);
                skey[pi] = key[r];
                sfirst[pi] = first[r];
                sref[pi] = ref[r];
                scnt[pi] = cnt[r];
                if (L.need_box) {
                    slo[pi] = lo[r];
                    if (L.lv != 2) shi[pi] = hi[r];
                }
            }
        }
    } else {
        // stage the children: coalesced loads; references of bricks from the dense
        // leaf-reference array, of nodes by one gather per child from the level's table
        // (every slot index loaded before the gathers, so that they are all in flight)
        if (L.lv == 2) {
            for (uint32_t i = threadIdx.x; i < tn; i += kBlock) sref[cpad(i)] = brick_ref(d, t0 + i);
        } else {
            uint32_t cs[SPT];
#pragma unroll
            for (int r = 0; r < SPT; ++r) {
                const uint32_t i = threadIdx.x + r * kBlock;
                cs[r] = i < tn ? L.cslot[t0 + i] : 0u;
            }
#pragma unroll
            for (int r = 0; r < SPT; ++r) {
                const uint32_t i = threadIdx.x + r * kBlock;
                if (i < tn) sref[cpad(i)] = __ldcg(&L.ctable[cs[r]].w);
            }
        }
        for (uint32_t i = threadIdx.x; i < tn; i += kBlock) {
            const uint32_t c = t0 + i, pi = cpad(i);
            skey[pi] = L.ckey[c];
            sfirst[pi] = L.cfirst[c];
            if (L.lv == 2) {
                const uint64_t m = L.cmask[c];
                scnt[pi] = __popcll(m);
                if (L.need_box) slo[pi] = m;
            } else {
                scnt[pi] = L.ccnt[c];
                if (L.need_box) { slo[pi] = L.clo[c]; shi[pi] = L.chi[c]; }
            }
        }
    }
    if (threadIdx.x == 0) s_prev = t0 > 0 ? L.ckey[t0 - 1] : ~0ull;
    __syncthreads();
    // heads of this tile's own children (warp chunks of 32 * NB)
    unsigned hb[NB];
    uint32_t wc = 0;
#pragma unroll
    for (int j = 0; j < NB; ++j) {
        const uint32_t i = warp * 32 * NB + j * 32 + lane;
        bool head = false;
        if (i < own_n) {
            const uint64_t pk = i == 0 ? s_prev : skey[cpad(i - 1)];
            head = (t0 + i == 0) || (skey[cpad(i)] >> 3) != (pk >> 3);
        }
        hb[j] = __ballot_sync(kFull, head);
        wc += __popc(hb[j]);
    }
    uint32_t total;
    uint32_t wexcl = block_excl_scan(lane == 0 ? wc : 0, s_scan, &total);
    wexcl = __shfl_sync(kFull, wexcl, 0);
    if (threadIdx.x == 0 && tile != 0) st_relaxed(L.build_status + tile, kFlagAgg | total);
    uint32_t run = wexcl;
#pragma unroll
    for (int j = 0; j < NB; ++j) {
        const uint32_t i = warp * 32 * NB + j * 32 + lane;
        if ((hb[j] >> lane) & 1) shead[run + __popc(hb[j] & lanemask_lt())] = i;
        run += __popc(hb[j]);
    }
    __syncthreads();
    if constexpr (NB == 1) {
        // the tile's parents, one per thread: assembled, words published at the first
        // child's index, home slot prefetched, all before the look-back
        const bool mine = threadIdx.x < total;
        NodeParent q;
        uint32_t i = 0, h = 0;
        if (mine) {
            i = shead[threadIdx.x];
            q = node_assemble(L, skey, slo, shi, scnt, sref, i, tn);
            uint32_t* cw = L.cwords + uint64_t(t0 + i) * kNodeStride;
            cw[0] = q.mask;
            cw[1] = q.count;
#pragma unroll
            for (uint32_t k = 0; k < 8; ++k)
                if (k < q.n) cw[2 + k] = q.refs[k];
            h = uint32_t(node_hash(q.mask, q.count, q.refs, q.n)) & (L.pcap - 1);
            prefetch_l2(&L.ptable[h]);
        }
        if (warp == 0) {
            uint64_t ex = lookback_warp(L.build_status, tile, 0, total, d.counters + kCtrError);
            if (lane == 0) s_base = ex;
        }
        __syncthreads();
        if (tile == ntiles - 1 && threadIdx.x == 0) d.counters[kCtrParents + L.lv] = uint32_t(s_base + total);
        if (mine) {
            const uint32_t par = uint32_t(s_base) + threadIdx.x;
            if (par >= L.parent_bound) {
                atomicOr(d.counters + kCtrError, kErrBound);
            } else {
                // the insert first: its release then covers only the words stored above
                const uint32_t slot = node_insert(L.ptable, L.pcap, L.cwords, t0 + i, par, h, q.mask, q.count,
                                                  q.refs, q.n, d.counters + kCtrError);
                node_store(L, par, q, skey[cpad(i)] >> 3, sfirst[cpad(i)], slot, true);
            }
        }
    } else {
        if (warp == 0) {
            uint64_t ex = lookback_warp(L.build_status, tile, 0, total, d.counters + kCtrError);
            if (lane == 0) s_base = ex;
        }
        __syncthreads();
        if (tile == ntiles - 1 && threadIdx.x == 0) d.counters[kCtrParents + L.lv] = uint32_t(s_base + total);
        const uint32_t base = uint32_t(s_base);
        for (uint32_t hh = threadIdx.x; hh < total; hh += kBlock) {
            const uint32_t i = shead[hh];
            const uint32_t par = base + hh;
            const NodeParent q = node_assemble(L, skey, slo, shi, scnt, sref, i, tn);
            if (par >= L.parent_bound) {
                atomicOr(d.counters + kCtrError, kErrBound);
                continue;
            }
            // words first (the insert's release publishes them with the key)
            uint32_t* pw = L.pwords + uint64_t(par) * kNodeStride;
            pw[0] = q.mask;
            pw[1] = q.count;
#pragma unroll
            for (uint32_t k = 0; k < 8; ++k)
                if (k < q.n) pw[2 + k] = q.refs[k];
            const uint32_t h = uint32_t(node_hash(q.mask, q.count, q.refs, q.n)) & (L.pcap - 1);
            const uint32_t slot = node_insert(L.ptable, L.pcap, L.pwords, par, par, h, q.mask, q.count, q.refs,
                                              q.n, d.counters + kCtrError);
            node_store(L, par, q, skey[cpad(i)] >> 3, sfirst[cpad(i)], slot, false);
        }
    }
}

template <int NB>
__global__ void __launch_bounds__(kBlock, NB == 1 ? 6 : 5) k_node_build(BuildDesc d, LevelDesc L) {
    grid_dep_wait();
    __shared__ uint32_t s_tile[3];
    uint32_t children, unused;
    const uint32_t ci = L.lv == 2 ? kCtrBricks : kCtrParents + L.lv - 1;
    const uint32_t tile = dyn_tile_and(d.counters, L.tile_ctr_build, ci, ci, s_tile, &children, &unused);
    node_build_tile<NB>(d, L, tile, children);
}

// Owners of level lv get word offsets (scan of their lengths) and write their words.
// One tile of the node owners (k_node_own takes one per block). With one parent per
// thread (small levels) the parent's words are loaded with its slot, before the
// owner test, so that the tile takes two dependent round trips before its look-back.
template <int NIT>
__device__ __forceinline__ void node_own_tile(const BuildDesc& d, const LevelDesc& L, const uint32_t tile,
                                              const uint32_t parents, const uint32_t cursor) {
    __shared__ uint64_t s_scan[2 * kWarps + 2];
    __shared__ uint64_t s_base;
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t P = min(parents, L.parent_bound);
    constexpr uint32_t kTile = kBlock * NIT;
    const uint32_t ntiles = (P + kTile - 1) / kTile;
    if (tile >= ntiles) return;
    const uint32_t wstart = tile * kTile + warp * 32 * NIT;
    uint32_t len[NIT], slot[NIT];
    uint32_t w1[NIT == 1 ? kNodeStride : 1];  // NIT == 1: the parent's words
    uint64_t wsum = 0;  // words | count << 31
    if constexpr (NIT == 1) {
        const uint32_t i = wstart + lane;
        const bool v = i < P;
        slot[0] = v ? L.pslot[i] : 0;
        const uint2* src = reinterpret_cast<const uint2*>(L.pwords + uint64_t(v ? i : 0) * kNodeStride);
#pragma unroll
        for (int k = 0; k < int(kNodeStride) / 2; ++k) {
            const uint2 x = v ? __ldcg(src + k) : make_uint2(0, 0);
            w1[2 * k] = x.x;
            w1[2 * k + 1] = x.y;
        }
        len[0] = v && ~ld_relaxed32(&L.ptable[slot[0]].z) == i ? 2 + __popc(w1[0] & 0xFF) : 0;
        uint64_t x = len[0] | (uint64_t(len[0] ? 1 : 0) << 31);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
        wsum = x;
    } else {
        // slots and masks of all the thread's parents in flight, then their owner words
        uint32_t mw[NIT];
#pragma unroll
        for (int j = 0; j < NIT; ++j) {
            const uint32_t i = wstart + j * 32 + lane;
            slot[j] = i < P ? __ldcg(L.pslot + i) : 0u;
            mw[j] = i < P ? __ldcg(L.pwords + uint64_t(i) * kNodeStride) : 0u;
        }
#pragma unroll
        for (int j = 0; j < NIT; ++j) {
            const uint32_t i = wstart + j * 32 + lane;
            len[j] = i < P && ~ld_relaxed32(&L.ptable[slot[j]].z) == i ? 2 + __popc(mw[j] & 0xFF) : 0u;
            uint64_t v = len[j] | (uint64_t(len[j] ? 1 : 0) << 31);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
            wsum += v;
        }
    }
    uint64_t total;
    uint64_t wexcl = block_excl_scan64(lane == 0 ? wsum : 0, s_scan, &total);
    wexcl = __shfl_sync(kFull, wexcl, 0);
    if (warp == 0) {
        if (lane == 0 && tile != 0) st_relaxed(L.own_status + tile, kFlagAgg | total);
        uint64_t ex = lookback_warp(L.own_status, tile, 0, total, d.counters + kCtrError);
        if (lane == 0) s_base = ex;
    }
    __syncthreads();
    uint32_t run = uint32_t(s_base & 0x7FFFFFFFu) + uint32_t(wexcl & 0x7FFFFFFFu);
#pragma unroll
    for (int j = 0; j < NIT; ++j) {
        uint32_t i = wstart + j * 32 + lane;
        uint32_t x = len[j];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(kFull, x, o);
            if (lane >= unsigned(o)) x += y;
        }
        uint32_t off = run + x - len[j];
        if (len[j]) {
            uint32_t dst = cursor + off;
            uint32_t w[kNodeStride];
            if constexpr (NIT == 1) {
#pragma unroll
                for (int k = 0; k < int(kNodeStride); ++k) w[k] = w1[k];
            } else {
                const uint2* src = reinterpret_cast<const uint2*>(L.pwords + uint64_t(i) * kNodeStride);
#pragma unroll
                for (int k = 0; k < int(kNodeStride) / 2; ++k) {
                    uint2 v = __ldcg(src + k);  // written by the build kernel just before: bypass L1
                    w[2 * k] = v.x;
                    w[2 * k + 1] = v.y;
                }
            }
            if (uint64_t(dst) + len[j] <= d.node_bound) {
#pragma unroll
                for (int k = 0; k < int(kNodeStride); ++k)
                    if (uint32_t(k) < len[j]) d.nodes[dst + k] = w[k];
            } else {
                atomicOr(d.counters + kCtrError, kErrBound);
            }
            L.ptable[slot[j]].w = dst;
        }
        run += __shfl_sync(kFull, x, 31);
    }
    if (tile == ntiles - 1 && threadIdx.x == 0) {
        uint64_t t = s_base + total;
        d.counters[kCtrCursor + L.lv + 1] = cursor + uint32_t(t & 0x7FFFFFFFu);
        d.counters[kCtrUniqueLv + L.lv] = uint32_t(t >> 31);
    }
}

template <int NIT>
__global__ void __launch_bounds__(kBlock) k_node_own(BuildDesc d, LevelDesc L) {
    grid_dep_wait();
    __shared__ uint32_t s_tile[3];
    uint32_t parents, cursor;
    const uint32_t tile = dyn_tile_and(d.counters, L.tile_ctr_own, kCtrParents + L.lv, kCtrCursor + L.lv, s_tile,
                                       &parents, &cursor);
    node_own_tile<NIT>(d, L, tile, parents, cursor);
}

// Empty levels still have to pass the cursor on.
__global__ void k_level_cursor(BuildDesc d, uint32_t lv) {
    grid_dep_wait();
    if (threadIdx.x == 0 && d.counters[kCtrParents + lv] == 0) d.counters[kCtrCursor + lv + 1] = d.counters[kCtrCursor + lv];
}

// ---------------------------------------------------------------------------
// RT prims of the parents of level rt_log2 - 1 (gbuild.zig:574-605): node
// offset, attribute rank relative to the chunk, cell, AABB base + lo - 1/256 and
// base + hi + 1/256 in f32 (adds in the reference's order, no FMA possible).
// ---------------------------------------------------------------------------
// Prims of threads t0, t0 + stride, ... (k_prims: every thread of its grid).
__device__ __forceinline__ void prims_range(const BuildDesc& d, const LevelDesc& L, uint32_t t0, uint32_t stride) {
    const uint32_t P = min(d.counters[kCtrParents + L.lv], L.parent_bound);
    const uint32_t local_shift = 3 * (d.log2 - d.rt_log2);
    const uint32_t size = 1u << d.rt_log2;
    for (uint32_t i = t0; i < P; i += stride) {
        if (i >= d.prim_bound) { atomicOr(d.counters + kCtrError, kErrBound); break; }
        uint64_t full = L.pkey[i];
        uint64_t key = full & ((1ull << local_shift) - 1);
        uint32_t chunk = uint32_t(full >> local_shift);
        uint32_t cx = compact3(key), cy = compact3(key >> 1), cz = compact3(key >> 2);
        uint32_t first = d.chunked ? d.chunk_first[chunk] : 0;
        uint32_t node = __ldcg(&L.ptable[L.pslot[i]].w);
        uint4 rec;
        rec.x = node;
        rec.y = L.pfirst[i] - first;
        uint64_t pc = pack_cell(cx, cy, cz);
        rec.z = uint32_t(pc);
        rec.w = uint32_t(pc >> 32);
        reinterpret_cast<uint4*>(d.prims)[i] = rec;
        uint64_t lo = L.plo[i], hi = L.phi[i];
        const float eps = 1.0f / 256.0f;
        float* box = d.aabbs + uint64_t(i) * 6;
        box[0] = __fsub_rn(__fadd_rn(float(cx * size), float(cell_x(lo))), eps);
        box[1] = __fsub_rn(__fadd_rn(float(cy * size), float(cell_y(lo))), eps);
        box[2] = __fsub_rn(__fadd_rn(float(cz * size), float(cell_z(lo))), eps);
        box[3] = __fadd_rn(__fadd_rn(float(cx * size), float(cell_x(hi))), eps);
        box[4] = __fadd_rn(__fadd_rn(float(cy * size), float(cell_y(hi))), eps);
        box[5] = __fadd_rn(__fadd_rn(float(cz * size), float(cell_z(hi))), eps);
        if (d.chunked && (i == 0 || (L.pkey[i - 1] >> local_shift) != chunk)) d.prim_start[chunk] = i;
    }
    if (t0 == 0) d.counters[kCtrPrims] = P;
}

__global__ void __launch_bounds__(kBlock) k_prims(BuildDesc d, LevelDesc L) {
    grid_dep_wait();
    prims_range(d, L, blockIdx.x * kBlock + threadIdx.x, gridDim.x * kBlock);
}

// ---------------------------------------------------------------------------
// Upper levels in one CTA. Each level: stage the children in shared memory, find
// heads (block scan), build the parents' words into global memory (their hashes into
// shared memory), dedup them in a shared-memory table (owner = minimum parent index),
// give the owners word offsets (block scan of their lengths), write their words, and
// turn every parent's slot into its node offset, which the next level uses as the
// child reference. Prims (level rt_log2 - 1), roots and the final counts are written
// here as well. Same output as k_node_build/k_node_own/k_prims/k_finalize per level.
// A global round trip costs about a microsecond here and a level has only a few
// thousand parents, so the kernel is latency-bound: every load of a step is issued
// before the first is used (loops unrolled over the thread's fixed share), children
// and their boxes are staged in shared memory, and words are read back from global
// memory only to compare two parents with equal hashes and to copy the owners out.
// ---------------------------------------------------------------------------
constexpr uint32_t kTailPer = kTailMaxChildren / kTailThreads;  // children (and parents) per thread
constexpr uint32_t kTailScanWords = 72;
constexpr size_t tail_smem_bytes() {
    return size_t(kTailMaxChildren) * (8 + 8 + 8 + 4 + 4 + 4 + 2 + 1) + size_t(kTailSlots) * (4 + 4) +
           kTailScanWords * 4;
}

__device__ __forceinline__ uint32_t tail_scan(uint32_t v, uint32_t* sm, uint32_t* total) {
    // exclusive scan over kTailThreads threads (32 warps)
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= unsigned(o)) x += y;
    }
    if (lane == 31) sm[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = sm[lane], s = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(kFull, s, o);
            if (lane >= unsigned(o)) s += y;
        }
        sm[32 + lane] = s - w;
        if (lane == 31) sm[64] = s;
    }
    __syncthreads();
    uint32_t r = sm[32 + warp] + x - v;
    *total = sm[64];
    __syncthreads();
    return r;
}

// The kNodeStride words of parent q, written earlier in this kernel (L2, not L1).
__device__ __forceinline__ void tail_words(const uint32_t* words, uint32_t q, uint32_t (&w)[kNodeStride]) {
    const uint2* src = reinterpret_cast<const uint2*>(words + uint64_t(q) * kNodeStride);
#pragma unroll
    for (int k = 0; k < int(kNodeStride) / 2; ++k) {
        const uint2 v = __ldcg(src + k);
        w[2 * k] = v.x;
        w[2 * k + 1] = v.y;
    }
}

__global__ void __launch_bounds__(kTailThreads) k_tail(BuildDesc d, TailDesc T) {
    grid_dep_wait();
    extern __shared__ uint64_t tsm64[];
    uint64_t* skey = tsm64;                                            // children keys
    uint64_t* slo = skey + kTailMaxChildren;                           // children boxes (level 2: masks)
    uint64_t* shi = slo + kTailMaxChildren;
    uint32_t* sref = reinterpret_cast<uint32_t*>(shi + kTailMaxChildren);
    uint32_t* scnt = sref + kTailMaxChildren;
    uint32_t* pval = scnt + kTailMaxChildren;                          // parent: hash, then (owners) node offset
    uint32_t* tkey = pval + kTailMaxChildren;                          // table: parent index + 1
    uint32_t* towner = tkey + kTailSlots;                              // table: minimum parent index
    uint32_t* scan = towner + kTailSlots;
    uint16_t* pslot = reinterpret_cast<uint16_t*>(scan + kTailScanWords);  // parent -> slot
    uint8_t* plen = reinterpret_cast<uint8_t*>(pslot + kTailMaxChildren);  // parent -> words
    static_assert(kTailSlots <= 65536 && kNodeStride < 256, "slot and length fit their arrays");
    __shared__ uint32_t s_cursor, s_children;
    const uint32_t tid = threadIdx.x;
    const uint32_t lv0 = T.lv0;
    if (tid == 0) {
        s_cursor = d.counters[kCtrCursor + lv0];
        s_children = lv0 == 2 ? min(d.counters[kCtrBricks], d.brick_bound)
                              : min(d.counters[kCtrParents + lv0 - 1], T.parent_bound[lv0 - 1]);
    }
    for (uint32_t i = tid; i < kTailSlots; i += kTailThreads) { tkey[i] = 0; towner[i] = 0xFFFFFFFFu; }
    __syncthreads();
    const uint32_t local_shift = 3 * (d.log2 - d.rt_log2);
    for (uint32_t lv = lv0; lv < d.log2; ++lv) {
        const uint32_t C = min(s_children, kTailMaxChildren);
        const RecordSet& ps = T.set[(lv - 2) & 1];
        const RecordSet& cs = T.set[(lv - 3) & 1];
        const bool box = lv + 1 <= d.rt_log2;
        const uint32_t child_size = 1u << lv;
        // 1. stage children (coalesced: child tid + k * kTailThreads)
        if (lv == 2) {
            uint64_t key[kTailPer], mask[kTailPer];
            uint32_t ref[kTailPer], own[kTailPer];
#pragma unroll
            for (uint32_t k = 0; k < kTailPer; ++k) {
                const uint32_t i = tid + k * kTailThreads;
                const bool v = i < C;
                key[k] = v ? d.bkey[i] : 0;
                mask[k] = v ? d.bmask[i] : 0;
                ref[k] = v ? __ldcg(d.bref + i) : 0;
            }
            // a brick that repeats a mask takes the leaf index of the mask's owner
#pragma unroll
            for (uint32_t k = 0; k < kTailPer; ++k)
                own[k] = ref[k] == kNoRef ? ~leaf_find(d, mask[k]).z : 0;
#pragma unroll
            for (uint32_t k = 0; k < kTailPer; ++k)
                if (ref[k] == kNoRef) ref[k] = __ldcg(d.bref + own[k]);
#pragma unroll
            for (uint32_t k = 0; k < kTailPer; ++k) {
                const uint32_t i = tid + k * kTailThreads;
                if (i < C) {
                    skey[i] = key[k];
                    slo[i] = mask[k];
                    sref[i] = ref[k];
                    scnt[i] = __popcll(mask[k]);
                }
            }
        } else {
            uint64_t key[kTailPer], lo[kTailPer], hi[kTailPer];
            uint32_t ref[kTailPer], cnt[kTailPer];
#pragma unroll
            for (uint32_t k = 0; k < kTailPer; ++k) {
                const uint32_t i = tid + k * kTailThreads;
                const bool v = i < C;
                key[k] = v ? __ldcg(cs.key + i) : 0;
                ref[k] = v ? __ldcg(cs.slot + i) : 0;
                cnt[k] = v ? __ldcg(cs.cnt + i) : 0;
                lo[k] = v && box ? __ldcg(cs.lo + i) : 0;
                hi[k] = v && box ? __ldcg(cs.hi + i) : 0;
            }
            if (lv == lv0) {
                // references from the last kernel-built level's table (slot -> node offset)
#pragma unroll
                for (uint32_t k = 0; k < kTailPer; ++k)
                    if (tid + k * kTailThreads < C) ref[k] = __ldcg(&T.ctable0[ref[k]].w);
            }
#pragma unroll
            for (uint32_t k = 0; k < kTailPer; ++k) {
                const uint32_t i = tid + k * kTailThreads;
                if (i < C) {
                    skey[i] = key[k];
                    sref[i] = ref[k];
                    scnt[i] = cnt[k];
                    slo[i] = lo[k];
                    shi[i] = hi[k];
                }
            }
        }
        __syncthreads();
        // 2. heads (kTailPer consecutive children per thread) and parent indices
        uint32_t hmask = 0, hc = 0;
#pragma unroll
        for (uint32_t k = 0; k < kTailPer; ++k) {
            const uint32_t i = tid * kTailPer + k;
            if (i < C && (i == 0 || (skey[i] >> 3) != (skey[i - 1] >> 3))) { hmask |= 1u << k; ++hc; }
        }
        uint32_t P;
        uint32_t pbase = tail_scan(hc, scan, &P);
        // 3. build parents: records and words into global memory, hashes into pval
        uint32_t fst[kTailPer];
#pragma unroll
        for (uint32_t k = 0; k < kTailPer; ++k) {
            const uint32_t i = tid * kTailPer + k;
            fst[k] = (hmask >> k) & 1 ? (lv == 2 ? d.bfirst[i] : __ldcg(cs.first + i)) : 0;
        }
        uint32_t par = pbase;
#pragma unroll
        for (uint32_t k = 0; k < kTailPer; ++k) {
            if (!((hmask >> k) & 1)) continue;
            const uint32_t i = tid * kTailPer + k;
            const uint64_t pkey = skey[i] >> 3;
            uint32_t mask = 0, count = 0, n = 0;
            uint32_t lo[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, hi[3] = {0, 0, 0};
            uint32_t* pw = ps.words + uint64_t(par) * kNodeStride;
            uint64_t hr = 0;  // hash of the references, in order
            for (uint32_t j = i; j < C && n < 8; ++j) {
                const uint64_t ck = skey[j];
                if ((ck >> 3) != pkey) break;
                const uint32_t idx = uint32_t(ck & 7);
                mask |= 1u << idx;
                count = sat_add(count, scnt[j]);
                const uint32_t r = sref[j];
                pw[2 + n] = r;
                hr = mix64(hr ^ r);
                if (box) {
                    uint64_t clo = slo[j], chi = shi[j];
                    if (lv == 2) brick_box(slo[j], clo, chi);
                    const uint32_t ox = (idx & 1) * child_size, oy = ((idx >> 1) & 1) * child_size,
                                   oz = (idx >> 2) * child_size;
                    lo[0] = min(lo[0], cell_x(clo) + ox); hi[0] = max(hi[0], cell_x(chi) + ox);
                    lo[1] = min(lo[1], cell_y(clo) + oy); hi[1] = max(hi[1], cell_y(chi) + oy);
                    lo[2] = min(lo[2], cell_z(clo) + oz); hi[2] = max(hi[2], cell_z(chi) + oz);
                }
                ++n;
            }
            pw[0] = mask;
            pw[1] = count;
            ps.key[par] = pkey;
            ps.cnt[par] = count;
            ps.first[par] = fst[k];
            if (box) {
                ps.lo[par] = pack_cell(lo[0], lo[1], lo[2]);
                ps.hi[par] = pack_cell(hi[0], hi[1], hi[2]);
            }
            pval[par] = uint32_t(mix64(mix64(hr ^ (uint64_t(n) << 32 | mask)) ^ count));
            plen[par] = uint8_t(2 + n);
            ++par;
        }
        __syncthreads();  // all words written (visible to the block)
        // 4. dedup in the shared-memory table (owner = minimum parent index); words are
        //    compared only for equal lengths in one probe sequence
        for (uint32_t q = tid; q < P; q += kTailThreads) {
            const uint32_t len = plen[q];
            uint32_t h = pval[q] & (kTailSlots - 1);
            uint32_t w[kNodeStride];
            bool have = false;
            uint32_t probes = 0;
            for (; probes < kTailSlots; ++probes, h = (h + 1) & (kTailSlots - 1)) {
                const uint32_t cur = atomicCAS(tkey + h, 0u, q + 1);
                if (cur == 0) break;
                const uint32_t o = cur - 1;
                if (plen[o] != len || pval[o] != pval[q]) continue;
                if (!have) { tail_words(ps.words, q, w); have = true; }
                uint32_t ow[kNodeStride];
                tail_words(ps.words, o, ow);
                bool same = true;
#pragma unroll
                for (uint32_t k = 0; k < kNodeStride; ++k) same = same && (k >= len || ow[k] == w[k]);
                if (same) break;
            }
            if (probes == kTailSlots) atomicOr(d.counters + kCtrError, kErrTable);
            pslot[q] = uint16_t(h);
            atomicMin(towner + h, q);
        }
        __syncthreads();
        // 5. owners: word offsets in parent order (pval = offset), then words out, one
        //    parent per thread
        uint32_t wl = 0, owners = 0;
#pragma unroll
        for (uint32_t k = 0; k < kTailPer; ++k) {
            const uint32_t q = tid * kTailPer + k;
            if (q < P && towner[pslot[q]] == q) { wl += plen[q]; ++owners; }
        }
        uint32_t words;
        uint32_t off = tail_scan(wl, scan, &words) + s_cursor;
#pragma unroll
        for (uint32_t k = 0; k < kTailPer; ++k) {
            const uint32_t q = tid * kTailPer + k;
            if (q < P && towner[pslot[q]] == q) {
                pval[q] = off;
                off += plen[q];
            }
        }
        uint32_t utotal;
        tail_scan(owners, scan, &utotal);  // includes a barrier: pval of every owner set
        for (uint32_t q = tid; q < P; q += kTailThreads) {
            if (towner[pslot[q]] != q) continue;
            uint32_t w[kNodeStride];
            tail_words(ps.words, q, w);
            const uint32_t dst = pval[q], len = plen[q];
            if (uint64_t(dst) + len <= d.node_bound) {
#pragma unroll
                for (uint32_t m = 0; m < kNodeStride; ++m)
                    if (m < len) d.nodes[dst + m] = w[m];
            } else {
                atomicOr(d.counters + kCtrError, kErrBound);
            }
        }
        // 6. references for the next level, prims, roots
        const bool prims = lv + 1 == d.rt_log2;
        for (uint32_t q = tid; q < P; q += kTailThreads) {
            const uint32_t node = pval[towner[pslot[q]]];
            ps.slot[q] = node;
            if (prims && q < d.prim_bound) {
                const uint64_t full = __ldcg(ps.key + q), plo = __ldcg(ps.lo + q), phi = __ldcg(ps.hi + q);
                const uint32_t pfirst = __ldcg(ps.first + q);
                const uint64_t prev = q > 0 ? __ldcg(ps.key + q - 1) : 0;
                const uint64_t key = full & ((1ull << local_shift) - 1);
                const uint32_t chunk = uint32_t(full >> local_shift);
                const uint32_t first = d.chunked ? d.chunk_first[chunk] : 0;
                const uint32_t cx = compact3(key), cy = compact3(key >> 1), cz = compact3(key >> 2);
                const uint32_t size = 1u << d.rt_log2;
                uint4 rec;
                rec.x = node;
                rec.y = pfirst - first;
                const uint64_t pc = pack_cell(cx, cy, cz);
                rec.z = uint32_t(pc);
                rec.w = uint32_t(pc >> 32);
                reinterpret_cast<uint4*>(d.prims)[q] = rec;
                const float eps = 1.0f / 256.0f;
                float* b = d.aabbs + uint64_t(q) * 6;
                b[0] = __fsub_rn(__fadd_rn(float(cx * size), float(cell_x(plo))), eps);
                b[1] = __fsub_rn(__fadd_rn(float(cy * size), float(cell_y(plo))), eps);
                b[2] = __fsub_rn(__fadd_rn(float(cz * size), float(cell_z(plo))), eps);
                b[3] = __fadd_rn(__fadd_rn(float(cx * size), float(cell_x(phi))), eps);
                b[4] = __fadd_rn(__fadd_rn(float(cy * size), float(cell_y(phi))), eps);
                b[5] = __fadd_rn(__fadd_rn(float(cz * size), float(cell_z(phi))), eps);
                if (d.chunked && (q == 0 || (prev >> local_shift) != chunk)) d.prim_start[chunk] = q;
            }
            if (lv + 1 == d.log2 && d.chunked) {
                const uint32_t chunk = uint32_t(__ldcg(ps.key + q));
                if (chunk < d.seg_count) d.roots[chunk] = node;
            }
        }
        __syncthreads();  // every thread is done with the table
        // clear the table for the next level
        for (uint32_t i = tid; i < kTailSlots; i += kTailThreads) { tkey[i] = 0; towner[i] = 0xFFFFFFFFu; }
        if (tid == 0) {
            d.counters[kCtrParents + lv] = P;
            d.counters[kCtrUniqueLv + lv] = utotal;
            s_cursor += words;
            d.counters[kCtrCursor + lv + 1] = s_cursor;
            s_children = P;
            if (lv + 1 == d.rt_log2) d.counters[kCtrPrims] = P;
        }
        __syncthreads();
    }
    if (tid == 0) {
        // final counts and the empty geometry (gbuild.zig:607-624)
        const uint32_t top_set = (d.log2 - 1 - 2) & 1;
        uint32_t cursor = s_cursor;
        uint32_t root = s_children > 0 ? __ldcg(T.set[top_set].slot) : 0;
        if (d.counters[kCtrUnique] == 0) {
            if (cursor + 2 <= d.node_bound) {
                d.nodes[cursor] = 0;
                d.nodes[cursor + 1] = 0;
            }
            root = cursor;
            cursor += 2;
            d.counters[kCtrPrims] = 0;
        }
        d.counters[kCtrRoot] = root;
        d.counters[kCtrWords] = cursor;
    }
}

// Mixed batch: chunk c of edge 2^log2[c] < 2^top_log2 sits in the low corner of its
// cell, so above its own top level it hangs below single-child nodes (child index
// 0). Its root is found by descending from the cell's top node.
__global__ void k_batch_roots(BuildDesc d, uint32_t max_log2) {
    grid_dep_wait();
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < d.seg_count; c += gridDim.x * blockDim.x) {
        uint32_t node = d.roots[c];
        if (node == 0xFFFFFFFFu) continue;
        const uint32_t l = __ldg(d.chunk_log2 + c);
        for (uint32_t lv = max_log2; lv > l; --lv) node = d.nodes[node + 2];
        d.roots[c] = node;
    }
}

// Root(s), node word count and the empty geometry (gbuild.zig:607-624).
__device__ __forceinline__ void finalize_top(const BuildDesc& d, const LevelDesc& top) {
    const uint32_t P = min(d.counters[kCtrParents + top.lv], top.parent_bound);
    if (d.chunked) {
        for (uint32_t i = threadIdx.x; i < P; i += kBlock) {
            uint32_t chunk = uint32_t(top.pkey[i]);
            if (chunk < d.seg_count) d.roots[chunk] = __ldcg(&top.ptable[top.pslot[i]].w);
        }
    }
    if (threadIdx.x == 0) {
        uint32_t cursor = d.counters[kCtrCursor + top.lv + 1];
        uint32_t root = P > 0 ? __ldcg(&top.ptable[top.pslot[0]].w) : 0;
        if (d.counters[kCtrUnique] == 0) {
            if (cursor + 2 <= d.node_bound) {
                d.nodes[cursor] = 0;
                d.nodes[cursor + 1] = 0;
            }
            root = cursor;
            cursor += 2;
            d.counters[kCtrPrims] = 0;
        }
        d.counters[kCtrRoot] = root;
        d.counters[kCtrWords] = cursor;
    }
}

__global__ void __launch_bounds__(kBlock) k_finalize(BuildDesc d, LevelDesc top) {
    grid_dep_wait();
    finalize_top(d, top);
}

// Diagnostics: one bounded wait that nothing ends. Tile 1 looks back at tile 0,
// whose status is never published; the wait gives up after kSpinLimit polls and sets
// kErrSpin, exactly as a wait inside a build would (which 0: the per-digit look-back
// of the sort passes, 1: the warp look-back of the compaction kernels). status:
// 2 zeroed words; launched with one warp.
__global__ void __launch_bounds__(32) k_selftest_wait(uint64_t* status, uint32_t* counters, uint32_t which) {
    if (which == 0) {
        if (threadIdx.x == 0) lookback_window<kSortWindow>(status, 1, 1, 0, 1, counters + kCtrError);
    } else {
        lookback_warp(status, 1, 0, 1, counters + kCtrError);
    }
}

// ---------------------------------------------------------------------------
// Chunk attribute palettes (src/device/palette.zig): up to 16 distinct attribute
// values per chunk and a 4-bit index per voxel instead of 32 bits.
//
// The reference runs one CTA per chunk and inserts values into a 64-slot shared
// table in whatever order its threads arrive; the palette is the table's slot order.
// Here chunks are cut into tiles of kPalTile voxels over the whole GPU: each tile
// collects its distinct values with the first voxel index of each (warp match_any,
// then a shared table), merges them into the chunk's global table (value, first
// index by atomicMin), and one thread per chunk then inserts the values in order of
// first occurrence into the reference's 64-slot table (same hash, linear probing)
// to lay out the palette: the order the reference produces when its inserts arrive
// in voxel order, which is every order when no two values share a home slot.
// ---------------------------------------------------------------------------
constexpr uint32_t kPalSlots = 64, kPalMax = 16, kPalEmpty = 0xFFFFFFFFu, kPalOverflow = 0xFFFFFFFFu;
constexpr uint32_t kPalTile = 4096;

struct PaletteDesc {
    const uint32_t* attrs;
    const uint32_t* first;      // [count + 1]
    const uint32_t* tile_of;    // [count + 1] first tile of each chunk
    uint32_t count;
    uint32_t* gval;             // [count][kPalSlots] values, kPalEmpty = free
    uint32_t* gfirst;           // [count][kPalSlots] first voxel index (atomicMin)
    uint32_t* gflag;            // [count] 1 = more than kPalSlots values seen
    uint32_t* palettes;         // [count][kPalMax]
    uint32_t* counts;           // [count]
    const uint32_t* dst;        // [count] word offset in pool
    uint32_t* pool;
    uint32_t* err;
};

__device__ __forceinline__ uint32_t pal_hash(uint32_t v) {  // palette.zig:34-38
    uint32_t h = v * 0x9E3779B1u;
    return h ^ (h >> 15);
}

// Insert (v, idx) into a kPalSlots table (shared or global); returns false when full.
__device__ __forceinline__ bool pal_insert(uint32_t* vals, uint32_t* firsts, uint32_t v, uint32_t idx) {
    uint32_t s = pal_hash(v) & (kPalSlots - 1);
    for (uint32_t probes = 0; probes < kPalSlots; ++probes) {
        uint32_t cur = atomicAdd(vals + s, 0u);
        if (cur == kPalEmpty) {
            cur = atomicCAS(vals + s, kPalEmpty, v);
            if (cur == kPalEmpty) cur = v;
        }
        if (cur == v) {
            atomicMin(firsts + s, idx);
            return true;
        }
        s = (s + 1) & (kPalSlots - 1);
    }
    return false;
}

__device__ __forceinline__ uint32_t pal_chunk_of(const PaletteDesc& p, uint32_t tile) {
    return upper_index(p.tile_of, p.count + 1, tile);
}

__global__ void __launch_bounds__(kBlock) k_pal_collect(PaletteDesc p) {
    grid_dep_wait();
    __shared__ uint32_t s_val[kPalSlots], s_first[kPalSlots];
    __shared__ uint32_t s_full;
    const uint32_t tile = blockIdx.x;
    if (tile >= p.tile_of[p.count]) return;
    const uint32_t c = pal_chunk_of(p, tile);
    const uint32_t lo = p.first[c] + (tile - p.tile_of[c]) * kPalTile;
    const uint32_t hi = min(p.first[c + 1], lo + kPalTile);
    if (threadIdx.x < kPalSlots) {
        s_val[threadIdx.x] = kPalEmpty;
        s_first[threadIdx.x] = 0xFFFFFFFFu;
    }
    if (threadIdx.x == 0) s_full = 0;
    __syncthreads();
    const unsigned lane = threadIdx.x & 31;
    for (uint32_t base = lo; base < hi; base += kBlock) {
        const uint32_t i = base + threadIdx.x;
        const bool in = i < hi;
        const uint32_t v = in ? __ldg(p.attrs + i) : 0u;
        // one insert per distinct value of the warp, by its lowest lane (smallest index)
        const unsigned peers = __match_any_sync(kFull, in ? v : kPalEmpty);
        // (0xFFFFFFFF is the table's empty marker and never enters a palette, as in the reference)
        if (in && v != kPalEmpty && lane == unsigned(__ffs(peers) - 1)) {
            if (!pal_insert(s_val, s_first, v, i)) s_full = 1;
        }
    }
    __syncthreads();
    if (s_full) {
        if (threadIdx.x == 0) atomicOr(p.gflag + c, 1u);
        return;
    }
    if (threadIdx.x < kPalSlots && s_val[threadIdx.x] != kPalEmpty) {
        if (!pal_insert(p.gval + uint64_t(c) * kPalSlots, p.gfirst + uint64_t(c) * kPalSlots, s_val[threadIdx.x],
                        s_first[threadIdx.x]))
            atomicOr(p.gflag + c, 1u);
    }
}

__global__ void __launch_bounds__(kBlock) k_pal_layout(PaletteDesc p) {
    grid_dep_wait();
    const uint32_t c = blockIdx.x * kBlock + threadIdx.x;
    if (c >= p.count) return;
    const uint32_t* gv = p.gval + uint64_t(c) * kPalSlots;
    const uint32_t* gf = p.gfirst + uint64_t(c) * kPalSlots;
    uint32_t v[kPalMax + 1], f[kPalMax + 1], n = 0;
    bool over = p.gflag[c] != 0;
    for (uint32_t s = 0; s < kPalSlots && !over; ++s) {
        if (gv[s] == kPalEmpty) continue;
        if (n == kPalMax) { over = true; break; }
        // insertion by first occurrence
        uint32_t k = n++;
        while (k > 0 && f[k - 1] > gf[s]) { v[k] = v[k - 1]; f[k] = f[k - 1]; --k; }
        v[k] = gv[s];
        f[k] = gf[s];
    }
    if (over) {
        p.counts[c] = kPalOverflow;
        return;
    }
    // the reference's table with the values inserted in that order
    uint32_t keys[kPalSlots];
    for (uint32_t s = 0; s < kPalSlots; ++s) keys[s] = kPalEmpty;
    for (uint32_t k = 0; k < n; ++k) {
        uint32_t s = pal_hash(v[k]) & (kPalSlots - 1);
        while (keys[s] != kPalEmpty) s = (s + 1) & (kPalSlots - 1);
        keys[s] = v[k];
    }
    uint32_t* pal = p.palettes + uint64_t(c) * kPalMax;
    uint32_t m = 0, p0 = 0;
    for (uint32_t s = 0; s < kPalSlots; ++s) {
        if (keys[s] == kPalEmpty) continue;
        if (m == 0) p0 = keys[s];
        pal[m++] = keys[s];
    }
    for (; m < kPalMax; ++m) pal[m] = n > 0 ? p0 : 0u;
    p.counts[c] = n;
}

// palette.zig pack: per tile of a chunk, one thread per output word (8 voxels).
__global__ void __launch_bounds__(kBlock) k_pal_pack(PaletteDesc p) {
    grid_dep_wait();
    __shared__ uint32_t s_pal[kPalMax];
    const uint32_t tile = blockIdx.x;
    if (tile >= p.tile_of[p.count]) return;
    const uint32_t c = pal_chunk_of(p, tile);
    const uint32_t lo = p.first[c], n = p.first[c + 1] - lo;
    const uint32_t t0 = (tile - p.tile_of[c]) * kPalTile;  // first voxel of the tile within the chunk
    const uint32_t t1 = min(n, t0 + kPalTile);
    uint32_t* out = p.pool + p.dst[c];
    if (p.counts[c] == kPalOverflow) {
        for (uint32_t i = t0 + threadIdx.x; i < t1; i += kBlock) out[i] = __ldg(p.attrs + lo + i);
        return;
    }
    if (threadIdx.x < kPalMax) {
        s_pal[threadIdx.x] = p.palettes[uint64_t(c) * kPalMax + threadIdx.x];
        if (t0 == 0) out[threadIdx.x] = s_pal[threadIdx.x];
    }
    __syncthreads();
    for (uint32_t w = t0 / 8 + threadIdx.x; w < (t1 + 7) / 8; w += kBlock) {
        uint32_t word = 0;
#pragma unroll
        for (uint32_t j = 0; j < 8; ++j) {
            const uint32_t i = w * 8 + j;
            if (i >= n) break;
            const uint32_t v = __ldg(p.attrs + lo + i);
            uint32_t idx = 0;
#pragma unroll
            for (int q = kPalMax - 1; q >= 0; --q)
                if (s_pal[q] == v) idx = uint32_t(q);  // the first equal entry
            word |= idx << (j * 4);
        }
        out[kPalMax + w] = word;
    }
}

}  // namespace pyrb
