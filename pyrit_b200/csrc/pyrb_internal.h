// Internal layout shared by the host orchestration and the kernels.
#pragma once

#include <cstdint>

namespace pyrb {

// Error bits in counters[kCtrError] (device-side, read back by the host).
constexpr uint32_t kErrSpin = 1u;       // a look-back or wait gave up after its poll limit
constexpr uint32_t kErrTable = 2u;      // a dedup table had no free slot
constexpr uint32_t kErrBound = 4u;      // a count exceeded its allocated upper bound
constexpr uint32_t kErrCapacity = 8u;   // a generator count exceeded the chunk capacity (world path)

// Counter block (u32) read back at the end of a build.
constexpr int kCtrUnique = 0;      // voxel_count
constexpr int kCtrBricks = 1;      // non-empty bricks
constexpr int kCtrLeaves = 2;      // leaf_count
constexpr int kCtrWords = 3;       // node_words
constexpr int kCtrRoot = 4;
constexpr int kCtrPrims = 5;
constexpr int kCtrError = 6;
constexpr int kCtrNeed = 7;        // largest generator count above the chunk capacity (world path)
constexpr int kCtrCursor = 8;      // + lv: first node word of level lv (lv = 2..25)
constexpr int kCtrParents = 36;    // + lv: P_lv
constexpr int kCtrUniqueLv = 64;   // + lv: U_lv
constexpr int kCtrTiles = 96;      // dynamic tile counters, one per launch:
constexpr int kCtrCount = 160;
// ... disjoint ranges, so that no kernel of a build finds a counter another one advanced
constexpr uint32_t kTileUnique = 0, kTileLeafOwn = 1, kTileLeafInsert = 2;
constexpr uint32_t kTileLevel0 = 4;   // level lv: build 4 + 2 (lv - 2), owners 5 + 2 (lv - 2)
constexpr uint32_t kTileSort0 = 44;   // sort pass p: 44 + p (8 passes at most: 64-bit keys take 8-bit digits)
static_assert(kTileLevel0 + 2 * (20 - 2) + 1 < kTileSort0, "level counters below the sort's");
static_assert(kTileSort0 + 16 <= kCtrCount - kCtrTiles, "sort counters fit");
constexpr uint32_t kMaxLeafRegions = 64;
#ifndef PYRB_LEAF_REGION_LOG
#define PYRB_LEAF_REGION_LOG 22
#endif
// 2^22 slots: 64 MB regions, half of L2 (at 1024^3, 8 regions: 0.89 ms to group and
// insert; 16 MB, 32 MB and 128 MB regions measured 1.05, 0.95 and 0.98 ms)
constexpr uint32_t kLeafRegionSlots = 1u << PYRB_LEAF_REGION_LOG;

constexpr int kMaxLevels = 24;
constexpr int kMaxPasses = 8;

// Input modes of the first (encode) stage.
enum Mode : uint32_t {
    kModePlain = 0,        // [old sorted keys | PyrVoxel edits], one segment
    kModeChunks = 1,       // segments of `capacity` PyrVoxels, filled per offsets[]
    kModeChunksEdits = 2,  // generated voxels per counts[] followed by overlay edits per edit_offsets[]
    kModeDownsample = 3,   // coarse keys of sorted source keys
    kModeBatch = 4,        // packed per-chunk voxel lists (+ edits) of mixed edges 2^log2[c]
};

// Everything a build's kernels need, passed by value (kernel parameter space).
struct BuildDesc {
    uint32_t mode;
    uint32_t log2;          // edge of the (uniform) chunk / geometry
    uint32_t rt_log2;
    uint32_t lb;            // local key bits: 3 * log2
    uint32_t seg_count;     // K segments (1 for plain builds)
    uint32_t capacity;
    uint32_t shift;         // downsample
    uint32_t n_old;
    uint32_t n_new;
    uint32_t n_total;       // raw entries of the encode stage
    uint32_t top;           // top level = log2 - 1
    uint32_t chunked;       // chunk batch: per-chunk roots, first voxels, first prims

    // inputs
    const uint64_t* old_keys;
    const uint32_t* old_vals;
    const uint4* voxels;          // PyrVoxel entries (edits / chunk voxels / generated voxels)
    const uint32_t* offsets;      // kModeChunks: u32[K+1]
    const uint32_t* gen_counts;   // kModeChunksEdits: u32[K]
    const uint4* edits;           // kModeChunksEdits
    const uint32_t* edit_offsets; // kModeChunksEdits: u32[K+1]
    const uint64_t* src_keys;     // kModeDownsample
    const uint32_t* src_vals;
    const uint32_t* chunk_log2;   // kModeBatch: u32[K] edge of every chunk
    const uint32_t* voxel_offsets;  // kModeBatch: u32[K+1] into voxels
    const uint32_t* edit_offsets2;  // kModeBatch: u32[K+1] into edits (NULL = no edits)
    const uint64_t* voxel_starts;   // kModeBatch: u64[K] start of chunk c in voxels (NULL = voxel_offsets[c])

    // segment tiling of the sort / unique stages
    uint32_t* seg_entry;     // u32[K+1]: first raw entry of each segment
    uint32_t* seg_tile;      // u32[K+1]: first sort tile of each segment
    uint32_t tile_keys;
    uint32_t sort_tiles;     // upper bound of sort tiles (grid)

    // sort
    uint32_t passes;
    uint32_t radix;          // 1 << widest digit
    uint32_t pass_shift[kMaxPasses];
    uint32_t pass_bits[kMaxPasses];
    uint32_t* hist;          // [K][passes][radix]
    uint64_t* sort_status;   // [passes][sort_tiles][radix]
    void* kbuf[2];           // sort keys: u32 when 3 * log2 + 1 <= 32 bits, else u64
    uint32_t* vbuf[2];

    // unique voxels (outputs)
    uint64_t* uniq_status;   // [brick_tiles]: voxels << 31 | bricks of each unique tile
    uint64_t* ukey;
    uint32_t* uval;
    uint32_t* chunk_first;   // [K], 0xFFFFFFFF initialised

    // bricks + leaves
    uint32_t brick_bound;
    uint32_t brick_tiles;    // unique tiles (a sort tile of more than 4096 entries is taken in parts)
    uint64_t* bkey;
    uint64_t* bmask;
    uint32_t* bfirst;
    uint32_t* bref;          // [B] leaf index of an owner brick, kNoRef for the others
    uint8_t* binst;          // [B] 1: the brick made itself its mask's owner (zeroed)
    uint8_t* bdisp;          // [B] 1: ... and was replaced by a smaller brick index (zeroed)
    uint4* leaf_table;       // {mask lo, mask hi, ~owner, leaf index}
    uint32_t leaf_cap;
    // Tables larger than L2 are filled region by region: leaf_regions > 1 groups the
    // bricks by the table region (leaf_cap / leaf_regions slots) of their mask's home
    // slot first, so the inserts in flight at any time touch a slice that stays in L2.
    uint32_t leaf_regions;
    uint32_t leaf_region_shift;  // log2(leaf_cap / leaf_regions)
    uint32_t* region_count;      // [leaf_regions] bricks per region (zero-initialised)
    uint32_t* region_cursor;     // [leaf_regions] (zero-initialised)
    uint32_t* region_zeroed;     // [leaf_regions] clearing tiles finished (zero-initialised)
    uint64_t* pmask;             // [B] masks grouped by region (in the dead sort buffers)
    uint32_t* pidx;              // [B] their brick indices
    uint32_t leafown_tiles;
    uint64_t* leafown_status;
    uint64_t* leaves;        // output

    uint32_t* counters;      // u32[kCtrCount]

    // outputs
    uint32_t* nodes;
    uint32_t node_bound;     // words
    uint8_t* prims;
    float* aabbs;
    uint32_t prim_bound;
    uint32_t* roots;         // [K] (chunk builds), 0xFFFFFFFF initialised
    uint32_t* prim_start;    // [K]

    // Cell grid of a dense build (use_grid): one 64-bit cell per voxel position of
    // every chunk in key (Morton) order, chunk after chunk; an entry at a position
    // leaves (input index + 1) << 32 | attribute there by an atomic max, so the cell
    // ends up holding the last entry of its position. Replaces the sort and the
    // unique pass: a streaming compaction of the cells gives the sorted unique voxels.
    uint32_t use_grid;
    uint32_t grid_tiles;     // compaction tiles of kGridTileBricks bricks
    uint64_t grid_cells;     // cells of all chunks (a multiple of 64)
    uint64_t* grid;          // [grid_cells], zeroed before the build
    uint64_t* grid_off;      // [K + 1] first cell of every chunk (k_plan)
    uint64_t* grid_count;    // [grid_tiles] voxels | bricks << 32 per tile, then their exclusive scan
    uint32_t grid_fold;      // no scan pass (grid_tiles <= kGridFoldTiles): group sums, added up by the write pass
    uint64_t* grid_super;    // grid_fold: [grid_tiles / 64 + 1] voxels | bricks << 32 of every 64 tiles (zeroed)
    uint32_t* chunk_vstart;  // [K] voxels before the first cell of every chunk (chunk builds)

    // Brick buckets of a sparse build (use_bucket): the entries of every brick position
    // gathered together (a counting pass, a scan, a scatter), each tile of 64 bricks
    // then rebuilt as a cell grid in shared memory for the grid path's compaction.
    uint32_t use_bucket;
    uint32_t bucket_scan_tiles;  // tiles of kBucketScanTile counters
    uint32_t* bcount;        // [bricks] entries per brick position, then the end of its bucket
    uint64_t* brec;          // [n_total] (input index + 1) << 32 | value, bucket by bucket
    uint8_t* bloc;           // [n_total] the entry's cell in its brick (key & 63)
    uint64_t* bsum;          // [bucket_scan_tiles] counter sums, then their exclusive scan
};

// One node level: children (bricks at level 2) -> parents of edge 2^(lv+1).
struct LevelDesc {
    uint32_t lv;
    uint32_t child_bound;
    uint32_t parent_bound;
    uint32_t build_tiles;
    uint32_t own_tiles;
    uint32_t need_box;       // parents need a bounding box (lv + 1 <= rt_log2)
    uint32_t pcap;           // table capacity (power of two)
    uint32_t tile_ctr_build; // counter index of the dynamic tile ids
    uint32_t tile_ctr_own;
    uint32_t build_nb;       // children per thread of the build kernel (4, or 1 for small levels)
    uint32_t own_it;         // parents per thread of the owner kernel (8, or 1 for small levels)
    // children
    const uint64_t* ckey;    // lv == 2: brick keys (voxel key >> 6)
    const uint32_t* ccnt;    // lv >  2
    const uint32_t* cfirst;
    const uint32_t* cslot;
    const uint64_t* cmask;   // lv == 2
    const uint64_t* clo;     // lv >  2
    const uint64_t* chi;
    const uint4* ctable;     // .w = reference of the child (leaf index / node offset)
    // parents
    uint64_t* pkey;
    uint32_t* pcnt;
    uint32_t* pfirst;
    uint32_t* pslot;
    uint64_t* plo;
    uint64_t* phi;
    uint32_t* pwords;        // [parent_bound][10]
    uint32_t* cwords;        // build_nb == 1: [child_bound][10], words at the first child's index
                             // (the table key of these levels: the first child's index + 1)
    uint4* ptable;           // {key + 1, -, ~owner, node offset}; key: parent index, or first child index
    uint64_t* build_status;
    uint64_t* own_status;
};

constexpr uint32_t kNodeStride = 10;
constexpr uint32_t kNoRef = 0xFFFFFFFFu;

// The upper levels, once a level has at most kTailMaxChildren children, are built by
// one CTA (k_tail) that keeps each level's dedup table in shared memory.
constexpr uint32_t kTailThreads = 1024;
constexpr uint32_t kTailMaxChildren = 4096;
constexpr uint32_t kTailSlots = 8192;

// One record set of parents (levels alternate between two sets).
struct RecordSet {
    uint64_t* key;
    uint32_t* cnt;
    uint32_t* first;
    uint32_t* slot;    // k_tail: node word offset of the parent (its reference)
    uint64_t* lo;
    uint64_t* hi;
    uint32_t* words;   // [bound][kNodeStride]
};

struct TailDesc {
    uint32_t lv0;                    // first level built by the tail (children <= kTailMaxChildren)
    uint32_t parent_bound[kMaxLevels + 2];
    RecordSet set[2];                // parents of level lv live in set[(lv - 2) & 1]
    const uint4* ctable0;            // references of lv0's children: leaf table (lv0 == 2) or level lv0-1 table
};



}  // namespace pyrb
