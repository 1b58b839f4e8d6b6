// Host orchestration of the DAG build and the C ABI of include/pyrit_b200.h.
//
// A build is one stream-ordered sequence of kernels (no host round trip until the
// final read of the counters): every buffer is sized from upper bounds that the
// host can compute from the input sizes, the real counts stay on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "pyrit_b200.h"
#include "pyrb_internal.h"
#include "pyrb_kernels.cuh"
#include "pyrb_grid.cuh"
#include "pyrb_bucket.cuh"
#include "pyrb_pathedit.cuh"

using namespace pyrb;

namespace {

// ---------------------------------------------------------------------------
// diagnostics (thread-local like the reference's diag.zig)
// ---------------------------------------------------------------------------
thread_local char g_msg[512] = "";
thread_local pyrb_stats g_stats = {};

pyrb_result fail(pyrb_result r, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
    va_end(ap);
    return r;
}

#define CU(call)                                                                                   \
    do {                                                                                           \
        cudaError_t err_ = (call);                                                                 \
        if (err_ != cudaSuccess) return fail(PYRB_ERROR_CUDA, "%s: %s", #call, cudaGetErrorString(err_)); \
    } while (0)

// Every kernel is launched with programmatic stream serialisation: its blocks may be
// dispatched while the previous kernel of the stream drains, and each kernel's first
// statement (grid_dep_wait) holds them until that kernel is complete. This hides the
// launch gap between the ~16 dependent kernels of a build.
template <typename... KArgs, typename... Args>
cudaError_t launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// ---------------------------------------------------------------------------
// tuning
// ---------------------------------------------------------------------------
std::atomic<uint32_t> g_radix_bits{0};  // 0 with g_tile_keys 0: chosen per build (auto_tuning)
std::atomic<uint32_t> g_tile_keys{0};
std::atomic<uint32_t> g_load_pct{50};
// Sort or cell grid for the voxels of a build (pyrb_tuning.path)
constexpr uint32_t kPathAuto = 0, kPathSort = 1, kPathGrid = 2, kPathBucket = 3;
std::atomic<uint32_t> g_path{kPathAuto};
// The grid path is taken automatically while the chunks hold at most this many cells
// per entry (dense volumes: 256^3 noise at 30 % solid has 3.3, terrain chunks 2), and
// at most kGridMaxCells cells in all (8 B each).
constexpr uint64_t kGridCellsPerEntry = 4;
// A node level takes tiles of one item per thread below this many large tiles (2 per SM)
constexpr uint32_t kSmallLevelTiles = 296;
constexpr uint64_t kGridMaxCells = uint64_t(1) << 33;
// Up to this many compaction tiles the write pass adds up its own prefix (at most 256
// group sums and 63 tile counts); larger grids take the 1024-thread scan kernel
constexpr uint32_t kGridFoldTiles = 16384;
// The brick buckets (pyrb_tuning.path = 3) need their brick counters (4 B per brick
// position) well inside the L2: up to 2^24 bricks (64 MB, a 1024^3 volume). They are
// not chosen automatically: on the 1024^3 Bernoulli(0.15) worst case they measured
// 11.35 ms per build against 8.73 ms for the sort (their scatter's returning atomics
// and the mostly empty 64-cell bricks of the compaction cost more than the sort
// passes they replace).
constexpr uint64_t kBucketMaxBricks = uint64_t(1) << 24;

// ---------------------------------------------------------------------------
// memory: caller callbacks, else a library-owned stream-ordered pool per device
// ---------------------------------------------------------------------------
std::mutex g_pool_mu;
cudaMemPool_t g_pools[64] = {};

cudaMemPool_t device_pool(int dev) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (dev < 0 || dev >= 64) return nullptr;
    if (!g_pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
        uint64_t thr = ~0ull;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &thr);
        g_pools[dev] = p;
    }
    return g_pools[dev];
}

struct Mem {
    const pyrb_exec* e;
    cudaStream_t st;
    cudaMemPool_t pool = nullptr;

    uint64_t get(uint64_t bytes) {
        bytes = std::max<uint64_t>(bytes, 16);
        if (e && e->alloc) return e->alloc(e->ctx, bytes);
        if (!pool) {
            int dev = 0;
            cudaGetDevice(&dev);
            pool = device_pool(dev);
            if (!pool) return 0;
        }
        void* p = nullptr;
        if (cudaMallocFromPoolAsync(&p, bytes, pool, st) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        return reinterpret_cast<uint64_t>(p);
    }
    void put(uint64_t p) {
        if (!p) return;
        if (e && e->free) e->free(e->ctx, p);
        else cudaFreeAsync(reinterpret_cast<void*>(p), st);
    }
};

uint64_t align_up(uint64_t v, uint64_t a) { return (v + a - 1) / a * a; }
uint32_t next_pow2(uint64_t v, uint32_t minimum) {
    uint64_t c = minimum;
    while (c < v) c <<= 1;
    return uint32_t(c);
}

// Bump layout of one scratch block.
struct Layout {
    uint64_t size = 0;
    uint64_t take(uint64_t bytes) {
        uint64_t off = align_up(size, 256);
        size = off + std::max<uint64_t>(bytes, 16);
        return off;
    }
};

// ---------------------------------------------------------------------------
// job description
// ---------------------------------------------------------------------------
struct Job {
    uint32_t mode = kModePlain;
    uint32_t log2 = 0, rt_req = 0, K = 1;
    uint64_t old_keys = 0, old_vals = 0;
    uint32_t n_old = 0;
    uint64_t voxels = 0;
    uint32_t n_new = 0;
    uint32_t capacity = 0;
    uint64_t offsets = 0;
    uint32_t total = 0;
    uint64_t gen_counts = 0, edits = 0, edit_offsets = 0;
    uint32_t edit_total = 0;
    uint64_t src_keys = 0, src_vals = 0;
    uint32_t shift = 0;
    // kModeBatch
    const uint32_t* chunk_log2_host = nullptr;
    uint64_t chunk_log2 = 0, voxel_offsets = 0, edit_offsets2 = 0, voxel_starts = 0;
    uint32_t voxel_total = 0;
    uint32_t* roots = nullptr;
    uint32_t* first_voxel = nullptr;
    uint32_t* first_prim = nullptr;
};

// Optional per-stage CUDA events (pyrb_profile_enable): one event after every
// launch of a build; durations are read after the stream has synchronised.
thread_local bool g_prof_on = false;
thread_local std::vector<cudaEvent_t> g_prof_events;
thread_local std::vector<std::pair<const char*, uint32_t>> g_prof_names;

// PYRB_SYNC_CHECK=1 synchronises after every launch and names the first stage
// that reports an error (like the reference's PYR_CREATE_DEBUG, src/context.zig:741-745).
bool sync_check_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("PYRB_SYNC_CHECK");
        return v && v[0] == '1';
    }();
    return on;
}
thread_local char g_failed_stage[64] = "";

struct Prof {
    cudaStream_t st;
    size_t n = 0;
    explicit Prof(cudaStream_t s) : st(s) {
        g_failed_stage[0] = 0;
        if (!g_prof_on) return;
        g_prof_names.clear();
        record();
    }
    void record() {
        if (g_prof_events.size() <= n) {
            cudaEvent_t ev;
            cudaEventCreate(&ev);
            g_prof_events.push_back(ev);
        }
        cudaEventRecord(g_prof_events[n], st);
        ++n;
    }
    void mark(const char* name, uint32_t arg = 0) {
        if (sync_check_enabled() && !g_failed_stage[0]) {
            cudaError_t err = cudaStreamSynchronize(st);
            if (err == cudaSuccess) err = cudaGetLastError();
            if (err != cudaSuccess) {
                snprintf(g_failed_stage, sizeof(g_failed_stage), "%s:%u", name, arg);
                fprintf(stderr, "pyrb: stage %s failed: %s\n", g_failed_stage, cudaGetErrorString(err));
            }
        }
        if (!g_prof_on) return;
        record();
        g_prof_names.emplace_back(name, arg);
    }
};

uint32_t leaf_insert_grid(const BuildDesc& d) {
    return std::max(std::min((d.brick_bound + kBlock - 1) / kBlock, 148u * 8u), 1u);
}

// First level built by the single-CTA tail kernel (children bound <= kTailMaxChildren
// from there on); log2 means no tail (the top level is too wide, e.g. many chunks).
uint32_t tail_level(uint32_t log2, uint32_t B, const uint32_t* P) {
    for (uint32_t lv = 2; lv < log2; ++lv) {
        const uint32_t child = lv == 2 ? B : P[lv - 1];
        if (child <= kTailMaxChildren) return lv;
    }
    return log2;
}

// Node levels, prims and the final counts. Levels below lv0 run as multi-CTA
// kernels; the rest (and the finalisation) in k_tail.
uint32_t launch_levels(const BuildDesc& d, const std::vector<LevelDesc>& levels, uint32_t lv0, const TailDesc& T,
                       cudaStream_t st, Prof& prof) {
    uint32_t launches = 0;
    for (const LevelDesc& L : levels) {
        if (L.lv >= lv0) break;
        if (L.build_nb == 1)
            launch(k_node_build<1>, L.build_tiles, kBlock, node_build_smem_bytes(L.lv == 2, 1), st, d, L);
        else
            launch(k_node_build<kNBIT>, L.build_tiles, kBlock, node_build_smem_bytes(L.lv == 2), st, d, L);
        prof.mark("node_build", L.lv);
        if (L.own_it == 1)
            launch(k_node_own<1>, L.own_tiles, kBlock, 0, st, d, L);
        else
            launch(k_node_own<kNodeIT>, L.own_tiles, kBlock, 0, st, d, L);
        prof.mark("node_own", L.lv);
        launches += 2;
        if (L.lv + 1 == d.rt_log2) {
            launch(k_prims, std::max((L.parent_bound + kBlock - 1) / kBlock, 1u), kBlock, 0, st, d, L);
            prof.mark("prims", L.lv);
            ++launches;
        }
    }
    if (lv0 < d.log2) {
        static std::once_flag once;
        std::call_once(once, [] {
            cudaFuncSetAttribute(k_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tail_smem_bytes()));
        });
        launch(k_tail, 1, kTailThreads, tail_smem_bytes(), st, d, T);
        prof.mark("tail", lv0);
    } else {
        launch(k_finalize, 1, kBlock, 0, st, d, levels.back());
        prof.mark("finalize");
    }
    return launches + 1;
}

TailDesc make_tail(uint32_t lv0, const uint32_t* P, const std::vector<LevelDesc>& levels, const uint4* leaf_table) {
    TailDesc T;
    std::memset(&T, 0, sizeof(T));
    T.lv0 = lv0;
    for (int i = 0; i < kMaxLevels + 2; ++i) T.parent_bound[i] = P[i];
    for (const LevelDesc& L : levels) {
        const int ps = (L.lv - 2) & 1;
        T.set[ps] = RecordSet{L.pkey, L.pcnt, L.pfirst, L.pslot, L.plo, L.phi, L.pwords};
        if (L.lv + 1 == lv0) T.ctable0 = L.ptable;
    }
    if (lv0 == 2) T.ctable0 = leaf_table;
    return T;
}

thread_local uint32_t g_capacity_need = 0;

// Result of a build whose counter block reports an error. A generator count above
// the chunk capacity alone is PYRB_ERROR_CAPACITY with the capacity that would have
// held every chunk (nothing is cut off: the build's outputs are discarded); any
// other error bit is a device-side failure.
pyrb_result device_error(const uint32_t* ctr) {
    const uint32_t bits = ctr[kCtrError];
    if (bits == kErrCapacity) {
        g_capacity_need = ctr[kCtrNeed];
        return fail(PYRB_ERROR_CAPACITY,
                    "a chunk holds %u generated voxels, more than the capacity; grow the capacity to at least %u "
                    "and generate again (nothing was cut off, no result was kept)",
                    ctr[kCtrNeed], ctr[kCtrNeed]);
    }
    return fail(PYRB_ERROR_CUDA, "device-side build error 0x%x (%s%s%s%s)", bits,
                (bits & kErrSpin) ? "look-back wait limit " : "", (bits & kErrTable) ? "dedup table full " : "",
                (bits & kErrBound) ? "upper bound exceeded " : "", (bits & kErrCapacity) ? "chunk over capacity" : "");
}

void fill_counts(const uint32_t* ctr, pyrb_built* out) {
    out->node_words = ctr[kCtrWords];
    out->root = ctr[kCtrRoot];
    out->leaf_count = ctr[kCtrLeaves];
    out->voxel_count = ctr[kCtrUnique];
    out->prim_count = ctr[kCtrPrims];
}

// meta: log2, rt, passes, radix bits, launches, scratch bytes (2 words), output bytes (2 words)
void fill_stats(const uint32_t* ctr, const uint32_t* meta) {
    pyrb_stats s = {};
    s.brick_count = ctr[kCtrBricks];
    for (uint32_t lv = 2; lv < meta[0] && lv < 24; ++lv) {
        s.level_parents[lv] = ctr[kCtrParents + lv];
        s.level_unique[lv] = ctr[kCtrUniqueLv + lv];
    }
    s.sort_passes = meta[2];
    s.radix_bits = meta[3];
    s.kernel_launches = meta[4];
    std::memcpy(&s.scratch_bytes, meta + 5, 8);
    std::memcpy(&s.output_bytes, meta + 7, 8);
    g_stats = s;
}

// Sort tiles of IT * kBlock entries. Tiles of 8192 entries (IT = 32) are sorted by
// 512-thread blocks of 16 entries per thread and de-duplicated in two 4096-entry parts.
template <int RB, int IT, typename KeyT = uint32_t>
cudaError_t launch_sort(const BuildDesc& d, cudaStream_t st, Prof& prof) {
    constexpr int NT = IT > 16 ? 2 * kBlock : kBlock, SIT = IT * kBlock / NT;
    constexpr int UIT = SIT < kUniqIT ? SIT : kUniqIT;
    constexpr uint32_t parts = uint32_t(IT / UIT);  // unique tiles per sort tile
    const size_t hist_smem = size_t(d.passes) * (1u << RB) * 4;
    const size_t sort_smem = sort_smem_bytes<RB, SIT, KeyT, NT>();
    static std::once_flag once;
    std::call_once(once, [&] {
        cudaFuncSetAttribute(k_encode_hist<RB, IT, KeyT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
        cudaFuncSetAttribute(k_sort_pass<RB, SIT, KeyT, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sort_smem));
        cudaFuncSetAttribute(k_sort_pass<RB, SIT, KeyT, NT>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        cudaFuncSetAttribute(k_unique<UIT, KeyT>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    });
    launch(k_encode_hist<RB, IT, KeyT>, d.sort_tiles, kBlock, hist_smem, st, d);
    prof.mark("encode_hist");
    launch(k_digit_base<RB>, d.seg_count * d.passes, kBlock, 0, st, d);
    prof.mark("digit_base");
    for (uint32_t p = 0; p < d.passes; ++p) {
        launch(k_sort_pass<RB, SIT, KeyT, NT>, d.sort_tiles, NT, sort_smem, st, d, p, p & 1);
        prof.mark("sort_pass", p);
    }
    launch(k_unique<UIT, KeyT>, d.sort_tiles * parts, kBlock, unique_smem_bytes<UIT, KeyT>(), st, d, d.passes & 1);
    prof.mark("unique_brick");
    return cudaGetLastError();
}

// 64-bit sort keys (edges above 2^10): one digit width and tile, 8 bits x 2048 keys.
cudaError_t launch_sort_any(uint32_t rb, uint32_t it, const BuildDesc& d, cudaStream_t st, Prof& prof) {
    if (3 * d.log2 + 1 > 32) return launch_sort<8, 8, uint64_t>(d, st, prof);
    if (rb == 9 && it == 16) return launch_sort<9, 16>(d, st, prof);
    if (rb == 9 && it == 8) return launch_sort<9, 8>(d, st, prof);
    if (rb == 9 && it == 4) return launch_sort<9, 4>(d, st, prof);
    if (rb == 10 && it == 16) return launch_sort<10, 16>(d, st, prof);
    if (rb == 10 && it == 8) return launch_sort<10, 8>(d, st, prof);
    if (rb == 10 && it == 4) return launch_sort<10, 4>(d, st, prof);
    if (rb == 8 && it == 32) return launch_sort<8, 32>(d, st, prof);
    if (rb == 9 && it == 32) return launch_sort<9, 32>(d, st, prof);
    if (rb == 8 && it == 16) return launch_sort<8, 16>(d, st, prof);
    if (rb == 8 && it == 8) return launch_sort<8, 8>(d, st, prof);
    if (rb == 8 && it == 4) return launch_sort<8, 4>(d, st, prof);
    if (rb == 4 && it == 16) return launch_sort<4, 16>(d, st, prof);
    if (rb == 4 && it == 8) return launch_sort<4, 8>(d, st, prof);
    if (rb == 4 && it == 4) return launch_sort<4, 4>(d, st, prof);
    if (rb == 11 && it == 16) return launch_sort<11, 16>(d, st, prof);
    if (rb == 11 && it == 8) return launch_sort<11, 8>(d, st, prof);
    if (rb == 11 && it == 4) return launch_sort<11, 4>(d, st, prof);
    return cudaErrorInvalidValue;
}

// The default digit width and tile: 9-bit digits on 8192-entry tiles where they take
// one pass less than 8-bit digits (9 and 18 brick bits: edges 2^5 and 2^8), else 8-bit
// digits on 4096-entry tiles. Measured on 25-bit keys (value noise, 5.1 M entries): 3
// passes of 9 bits on 8192 entries 0.49-0.50 ms per build, 4 passes of 8 bits 0.52;
// 9 bits on 4096 entries no faster than 8 bits.
void auto_tuning(uint32_t sort_bits, uint32_t* rb, uint32_t* tile_keys) {
    const bool nine = (sort_bits + 8) / 9 < (sort_bits + 7) / 8;
    *rb = nine ? 9u : 8u;
    *tile_keys = nine ? 8192u : 4096u;
}

// Everything a build needs that the host can work out before any GPU work: the
// digit plan, the upper bounds of every count, the scratch layout and the output
// sizes. Used by the builds themselves, by the fixed-array build and by
// pyrb_build_memory (how much device memory a build would take).
struct Plan {
    BuildDesc d;
    uint32_t K = 1, rb = 8, it = 16, lf = 50, passes = 1, min_log2 = 3, rt = 3, n = 0, nmax = 1, B = 1;
    bool chunked = false, key64 = false, grid = false, bucket = false;
    uint32_t P[kMaxLevels + 2] = {};
    uint32_t cap[kMaxLevels + 2] = {}, btiles[kMaxLevels + 2] = {}, otiles[kMaxLevels + 2] = {};
    uint32_t bnb[kMaxLevels + 2] = {}, oit[kMaxLevels + 2] = {};
    uint64_t o_counters = 0, o_hist = 0, o_sort_status = 0, o_uniq_status = 0,
             o_leafown_status = 0, o_leaf_table = 0, o_regions = 0;
    uint64_t o_table[kMaxLevels + 2] = {}, o_bstat[kMaxLevels + 2] = {}, o_ostat[kMaxLevels + 2] = {};
    uint64_t o_chunk_first = 0, o_roots = 0, o_prim_start = 0, o_seg_entry = 0, o_seg_tile = 0;
    uint64_t o_k0 = 0, o_v0 = 0, o_k1 = 0, o_v1 = 0, o_bkey = 0, o_bmask = 0, o_bfirst = 0, o_bref = 0;
    uint64_t o_grid = 0, o_grid_off = 0, o_grid_count = 0, o_chunk_vstart = 0, o_grid_super = 0;
    uint64_t o_bcount = 0, o_brec = 0, o_bloc = 0, o_bsum = 0;
    uint64_t o_set[2][7] = {};
    uint64_t o_cwords = 0, o_binst = 0, o_bdisp = 0;
    uint64_t zero_bytes = 0, ff_bytes = 0, scratch_bytes = 0;
    // output buffers (bytes): nodes, leaves, keys, attrs, prims, aabbs
    uint64_t out_size[6] = {};
    uint64_t out_bytes() const {
        uint64_t s = 0;
        for (uint64_t v : out_size) s += v;
        return s;
    }
};

// Digit width, tile and load factor of a build: the fixed tuning given, else the
// library's current tuning (64-bit keys: 8-bit digits on 2048-key tiles).
struct Tune {
    uint32_t rb, tile_keys, lf, path;
};

pyrb_result plan_build(const Job& job, const Tune* fixed, Plan& p) {
    const uint32_t log2 = job.log2;
    if (log2 < 3 || log2 > 20) return fail(PYRB_ERROR_INVALID_ARGUMENT, "log2_size must lie in [3, 20] (got %u)", log2);
    const uint32_t lb = 3 * log2;
    p.key64 = lb + 1 > 32;
    const uint32_t K = p.K = job.K;
    p.chunked = job.mode == kModeChunks || job.mode == kModeChunksEdits || job.mode == kModeBatch;
    // chunks per edge (kModeBatch mixes edges; every other mode has K chunks of edge 2^log2)
    uint64_t per_log2[24] = {};
    uint32_t min_log2 = log2;
    if (job.mode == kModeBatch) {
        for (uint32_t c = 0; c < K; ++c) {
            const uint32_t l = job.chunk_log2_host[c];
            if (l < 3 || l > log2) return fail(PYRB_ERROR_INVALID_ARGUMENT, "chunk %u: log2 %u outside [3, %u]", c, l, log2);
            ++per_log2[l];
            min_log2 = std::min(min_log2, l);
        }
    } else {
        per_log2[log2] = K;
    }
    p.min_log2 = min_log2;
    if (p.chunked) {
        uint32_t bits = 0;
        while ((uint64_t(1) << bits) < K) ++bits;
        if (lb + bits + 1 > 64) return fail(PYRB_ERROR_INVALID_ARGUMENT, "too many chunks for this chunk size");
    }
    const uint32_t rt = p.rt = std::min(std::max(job.rt_req, 3u), min_log2);

    // raw entries (upper bound for the chunk modes)
    uint64_t n64 = 0;
    switch (job.mode) {
        case kModePlain: n64 = uint64_t(job.n_old) + job.n_new; break;
        case kModeChunks: n64 = job.total; break;
        case kModeChunksEdits: n64 = uint64_t(K) * job.capacity + job.edit_total; break;
        case kModeBatch: n64 = uint64_t(job.voxel_total) + job.edit_total; break;
        default: n64 = job.n_new; break;
    }
    if (n64 >= (uint64_t(1) << 31)) return fail(PYRB_ERROR_INVALID_ARGUMENT, "too many entries for one build (%llu)", (unsigned long long)n64);
    const uint32_t n = p.n = uint32_t(n64);
    const uint32_t nmax = p.nmax = std::max(n, 1u);

    // tuning (64-bit keys use 8-bit digits and 2048-key tiles)
    uint32_t rb, tile_keys, lf, path;
    if (fixed) {
        rb = fixed->rb;
        tile_keys = fixed->tile_keys;
        lf = fixed->lf;
        path = fixed->path;
    } else {
        rb = p.key64 ? 8u : g_radix_bits.load();
        tile_keys = p.key64 ? 2048u : g_tile_keys.load();
        if (rb == 0) auto_tuning(lb - 6, &rb, &tile_keys);
        lf = g_load_pct.load();
        path = g_path.load();
    }
    // cells of all chunks; the grid path needs 32-bit keys (edges up to 2^10)
    uint64_t grid_cells = 0;
    for (uint32_t l = 3; l <= log2 && !p.key64; ++l) grid_cells += per_log2[l] << (3 * l);
    if (!p.key64 && grid_cells <= kGridMaxCells)
        p.grid = path == kPathGrid || (path == kPathAuto && grid_cells <= kGridCellsPerEntry * nmax);
    if (!p.key64 && !p.grid && (grid_cells >> 6) <= kBucketMaxBricks)
        p.bucket = path == kPathBucket;
    if (p.grid || p.bucket) tile_keys = 4096;  // the scatter's tiles over the entries
    p.rb = (p.grid || p.bucket) ? 0 : rb;
    p.it = tile_keys / kBlock;
    p.lf = lf;

    BuildDesc& d = p.d;
    std::memset(&d, 0, sizeof(d));
    d.mode = job.mode;
    d.log2 = log2;
    d.rt_log2 = rt;
    d.lb = lb;
    d.seg_count = K;
    d.capacity = job.capacity;
    d.shift = job.shift;
    d.n_old = job.n_old;
    d.n_new = job.n_new;
    d.n_total = n;
    d.top = log2 - 1;
    d.chunked = p.chunked ? 1u : 0u;

    // digit plan over the brick bits 6 .. lb - 1 (k_unique resolves the cell bits and
    // the invalid bit); none for the grid
    const uint32_t sort_bits = lb - 6;
    const uint32_t passes = p.passes = (p.grid || p.bucket) ? 0 : (sort_bits + rb - 1) / rb;
    d.passes = passes;
    d.radix = passes ? 1u << rb : 0;
    if (passes) {
        uint32_t base = sort_bits / passes, extra = sort_bits % passes, sh = 6;
        for (uint32_t q = 0; q < passes; ++q) {
            uint32_t b = base + (q < extra ? 1 : 0);
            d.pass_shift[q] = sh;
            d.pass_bits[q] = b;
            sh += b;
        }
    }
    d.tile_keys = tile_keys;
    d.sort_tiles = (K == 1 ? (n + tile_keys - 1) / tile_keys : (n + tile_keys - 1) / tile_keys + K);
    d.sort_tiles = std::max(d.sort_tiles, 1u);

    // per-level upper bounds
    auto cells = [&](uint32_t edge_log2) -> uint64_t {  // cells of edge 2^edge_log2 in all chunks
        uint64_t total = 0;
        for (uint32_t l = 3; l <= log2; ++l) {
            if (!per_log2[l]) continue;
            const uint32_t e3 = l > edge_log2 ? 3 * (l - edge_log2) : 0;  // a smaller chunk: one cell
            if (e3 >= 40) return ~0ull >> 1;
            total += (uint64_t(1) << e3) * per_log2[l];
        }
        return total;
    };
    const uint32_t B = p.B = uint32_t(std::max<uint64_t>(std::min<uint64_t>(nmax, cells(2)), 1));
    uint32_t* P = p.P;
    uint64_t words = 2;
    for (uint32_t lv = 2; lv < log2; ++lv) {
        uint64_t prev = lv == 2 ? B : P[lv - 1];
        P[lv] = uint32_t(std::max<uint64_t>(std::min<uint64_t>(prev, cells(lv + 1)), 1));
        words += uint64_t(P[lv]) * kNodeStride;
    }
    if (words >= (uint64_t(1) << 32)) return fail(PYRB_ERROR_INVALID_ARGUMENT, "node buffer bound exceeds 2^32 words");
    d.brick_bound = B;
    d.brick_tiles = d.sort_tiles * std::max(1u, tile_keys / uint32_t(kBlock * kUniqIT));  // the unique tiles
    d.leafown_tiles = std::max((B + kBrickTile - 1) / kBrickTile, 1u);
    if ((uint64_t(B) * 100 + lf - 1) / lf > (uint64_t(1) << 31))
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "brick bound exceeds the leaf table's 2^31 slots");
    d.leaf_cap = next_pow2((uint64_t(B) * 100 + lf - 1) / lf, 1024);
    // region by region only for a single volume: chunk batches (terrain-like chunks)
    // repeat their masks so much that their inserts stay in a small, cached set of
    // slots, and there the build's memset clears the table faster than the insert
    // kernel does (1024-chunk mix: 46.8 ms without regions, 47.3 with)
    d.leaf_regions = 1;
    while (K == 1 && d.leaf_regions < kMaxLeafRegions && d.leaf_cap / d.leaf_regions > kLeafRegionSlots)
        d.leaf_regions <<= 1;
    d.leaf_region_shift = 0;
    while ((d.leaf_cap >> d.leaf_region_shift) > d.leaf_regions) ++d.leaf_region_shift;
    d.node_bound = uint32_t(words);
    d.prim_bound = P[rt - 1];
    if (p.grid || p.bucket) {
        d.use_grid = p.grid ? 1u : 0u;
        d.use_bucket = p.bucket ? 1u : 0u;
        d.grid_cells = grid_cells;
        d.grid_tiles = uint32_t(std::max<uint64_t>((grid_cells + 64 * kGridTileBricks - 1) / (64 * kGridTileBricks), 1));
        d.grid_fold = d.grid_tiles <= kGridFoldTiles ? 1u : 0u;
        d.bucket_scan_tiles = uint32_t(std::max<uint64_t>(((grid_cells >> 6) + kBucketScanTile - 1) / kBucketScanTile, 1));
    }

    // ---- scratch layout
    Layout zl;  // zero-initialised region
    p.o_counters = zl.take(kCtrCount * 4);
    if (p.bucket) p.o_bcount = zl.take((grid_cells >> 6) * 4);
    if (!p.grid && !p.bucket) {
        p.o_hist = zl.take(uint64_t(K) * passes * d.radix * 4);
        p.o_sort_status = zl.take(uint64_t(passes) * d.sort_tiles * d.radix * 8);
        p.o_uniq_status = zl.take(uint64_t(d.brick_tiles) * 8);
    }
    p.o_leafown_status = zl.take(uint64_t(d.leafown_tiles) * 8);
    p.o_binst = zl.take(uint64_t(B));
    p.o_bdisp = zl.take(uint64_t(B));
    // a table filled region by region is cleared by its insert kernel, not by the memset
    p.o_leaf_table = d.leaf_regions > 1 ? 0 : zl.take(uint64_t(d.leaf_cap) * 16);
    p.o_regions = zl.take(3 * kMaxLeafRegions * 4);
    for (uint32_t lv = 2; lv < log2; ++lv) {
        p.cap[lv] = next_pow2((uint64_t(P[lv]) * 100 + lf - 1) / lf, 1024);
        uint32_t child = lv == 2 ? B : P[lv - 1];
        // levels too small for two waves of large tiles take tiles of one item per thread
        p.bnb[lv] = child >= kSmallLevelTiles * kNodeBuildTile ? kNBIT : 1;
        p.oit[lv] = P[lv] >= kSmallLevelTiles * kNodeTile ? kNodeIT : 1;
        p.btiles[lv] = std::max((child + kBlock * p.bnb[lv] - 1) / (kBlock * p.bnb[lv]), 1u);
        p.otiles[lv] = std::max((P[lv] + kBlock * p.oit[lv] - 1) / (kBlock * p.oit[lv]), 1u);
        p.o_table[lv] = zl.take(uint64_t(p.cap[lv]) * 16);
        p.o_bstat[lv] = zl.take(uint64_t(p.btiles[lv]) * 8);
        p.o_ostat[lv] = zl.take(uint64_t(p.otiles[lv]) * 8);
    }
    if (p.grid) p.o_grid = zl.take(grid_cells * 8);
    if (d.grid_fold) p.o_grid_super = zl.take((uint64_t(d.grid_tiles) / 64 + 1) * 8);
    p.zero_bytes = align_up(zl.size, 256);
    Layout fl;  // 0xFF region follows
    fl.size = p.zero_bytes;
    p.o_chunk_first = fl.take(uint64_t(K) * 4);
    p.o_roots = fl.take(uint64_t(K) * 4);
    p.o_prim_start = fl.take(uint64_t(K) * 4);
    p.ff_bytes = align_up(fl.size, 256) - p.zero_bytes;
    Layout ol;
    ol.size = p.zero_bytes + p.ff_bytes;
    if (d.leaf_regions > 1) p.o_leaf_table = ol.take(uint64_t(d.leaf_cap) * 16);
    p.o_seg_entry = ol.take(uint64_t(K + 1) * 4);
    p.o_seg_tile = ol.take(uint64_t(K + 1) * 4);
    const uint64_t kbytes = p.key64 ? 8 : 4;
    if (p.bucket) {
        p.o_brec = ol.take(uint64_t(nmax) * 8);
        p.o_bloc = ol.take(uint64_t(nmax));
        p.o_bsum = ol.take(uint64_t(d.bucket_scan_tiles) * 8);
    }
    if (!p.grid && !p.bucket) {
        p.o_k0 = ol.take(uint64_t(nmax) * kbytes);
        p.o_v0 = ol.take(uint64_t(nmax) * 4);
        p.o_k1 = ol.take(uint64_t(nmax) * kbytes);
        p.o_v1 = ol.take(uint64_t(nmax) * 4);
    } else {
        p.o_grid_off = ol.take(uint64_t(K + 1) * 8);
        p.o_grid_count = ol.take(uint64_t(d.grid_tiles) * 8);
        p.o_chunk_vstart = ol.take(uint64_t(K) * 4);
    }
    p.o_bkey = ol.take(uint64_t(B) * 8);
    p.o_bmask = ol.take(uint64_t(B) * 8);
    p.o_bfirst = ol.take(uint64_t(B) * 4);
    p.o_bref = ol.take(uint64_t(B) * 4);
    // parent record sets: A for even offsets from level 2, B for odd
    const uint32_t setn[2] = {P[2], log2 > 3 ? P[3] : 1u};
    for (int s = 0; s < 2; ++s) {
        const uint64_t m = std::max(setn[s], 1u);
        p.o_set[s][0] = ol.take(m * 8);                 // key
        p.o_set[s][1] = ol.take(m * 4);                 // cnt
        p.o_set[s][2] = ol.take(m * 4);                 // first
        p.o_set[s][3] = ol.take(m * 4);                 // slot
        p.o_set[s][4] = ol.take(m * 8);                 // lo
        p.o_set[s][5] = ol.take(m * 8);                 // hi
        p.o_set[s][6] = ol.take(m * kNodeStride * 4);   // words
    }
    // words of the small levels' parents at their first child's index (one buffer,
    // levels run one after another)
    uint64_t cw = 0;
    for (uint32_t lv = 2; lv < log2; ++lv)
        if (p.bnb[lv] == 1) cw = std::max<uint64_t>(cw, lv == 2 ? B : P[lv - 1]);
    p.o_cwords = ol.take(std::max<uint64_t>(cw, 1) * kNodeStride * 4);
    p.scratch_bytes = align_up(ol.size, 256);
    const uint64_t prims = std::max(d.prim_bound, 1u);
    const uint64_t outs[6] = {uint64_t(d.node_bound) * 4, uint64_t(B) * 8, uint64_t(nmax) * 8, uint64_t(nmax) * 4,
                              prims * 16, prims * 24};
    for (int i = 0; i < 6; ++i) p.out_size[i] = outs[i];
    return PYRB_OK;
}

// Device pointers of a plan: scratch block at `scratch`, outputs given; fills the
// level descriptors.
void bind_plan(Plan& p, uint64_t scratch, const uint64_t outs[6], const Job& job, std::vector<LevelDesc>& levels) {
    BuildDesc& d = p.d;
    auto at = [&](uint64_t off) { return reinterpret_cast<void*>(scratch + off); };
    d.old_keys = reinterpret_cast<const uint64_t*>(job.old_keys);
    d.old_vals = reinterpret_cast<const uint32_t*>(job.old_vals);
    d.voxels = reinterpret_cast<const uint4*>(job.voxels);
    d.offsets = reinterpret_cast<const uint32_t*>(job.offsets);
    d.gen_counts = reinterpret_cast<const uint32_t*>(job.gen_counts);
    d.edits = reinterpret_cast<const uint4*>(job.edits);
    d.edit_offsets = reinterpret_cast<const uint32_t*>(job.edit_offsets);
    d.src_keys = reinterpret_cast<const uint64_t*>(job.src_keys);
    d.src_vals = reinterpret_cast<const uint32_t*>(job.src_vals);
    d.chunk_log2 = reinterpret_cast<const uint32_t*>(job.chunk_log2);
    d.voxel_offsets = reinterpret_cast<const uint32_t*>(job.voxel_offsets);
    d.edit_offsets2 = reinterpret_cast<const uint32_t*>(job.edit_offsets2);
    d.voxel_starts = reinterpret_cast<const uint64_t*>(job.voxel_starts);
    d.counters = static_cast<uint32_t*>(at(p.o_counters));
    d.hist = static_cast<uint32_t*>(at(p.o_hist));
    d.sort_status = static_cast<uint64_t*>(at(p.o_sort_status));
    d.uniq_status = static_cast<uint64_t*>(at(p.o_uniq_status));
    d.leafown_status = static_cast<uint64_t*>(at(p.o_leafown_status));
    d.leaf_table = static_cast<uint4*>(at(p.o_leaf_table));
    d.region_count = static_cast<uint32_t*>(at(p.o_regions));
    d.region_cursor = d.region_count + kMaxLeafRegions;
    d.region_zeroed = d.region_count + 2 * kMaxLeafRegions;
    // the sort buffers (or the cell grid) are dead once the unique voxels are out: N x
    // (kb + 4) bytes from k0 hold the B region-grouped masks, k1 their brick indices
    // (in the grid: 8 B per cell, at least 512 B per brick)
    if (p.grid || p.bucket) {
        d.grid_off = static_cast<uint64_t*>(at(p.o_grid_off));
        d.grid_count = static_cast<uint64_t*>(at(p.o_grid_count));
        d.grid_super = static_cast<uint64_t*>(at(p.o_grid_super));
        d.chunk_vstart = static_cast<uint32_t*>(at(p.o_chunk_vstart));
    }
    if (p.grid) {
        d.grid = static_cast<uint64_t*>(at(p.o_grid));
        d.pmask = d.grid;
        d.pidx = reinterpret_cast<uint32_t*>(d.grid + p.B);
    } else if (p.bucket) {
        d.bcount = static_cast<uint32_t*>(at(p.o_bcount));
        d.brec = static_cast<uint64_t*>(at(p.o_brec));
        d.bloc = static_cast<uint8_t*>(at(p.o_bloc));
        d.bsum = static_cast<uint64_t*>(at(p.o_bsum));
        // dead once the bricks are out: the records hold the region-grouped masks (8 B
        // per entry >= per brick), the counters their brick indices (4 B per brick position)
        d.pmask = d.brec;
        d.pidx = d.bcount;
    } else {
        d.pmask = static_cast<uint64_t*>(at(p.o_k0));
        d.pidx = static_cast<uint32_t*>(at(p.o_k1));
    }
    d.chunk_first = static_cast<uint32_t*>(at(p.o_chunk_first));
    d.roots = static_cast<uint32_t*>(at(p.o_roots));
    d.prim_start = static_cast<uint32_t*>(at(p.o_prim_start));
    d.seg_entry = static_cast<uint32_t*>(at(p.o_seg_entry));
    d.seg_tile = static_cast<uint32_t*>(at(p.o_seg_tile));
    if (!p.grid && !p.bucket) {
        d.kbuf[0] = at(p.o_k0);
        d.vbuf[0] = static_cast<uint32_t*>(at(p.o_v0));
        d.kbuf[1] = at(p.o_k1);
        d.vbuf[1] = static_cast<uint32_t*>(at(p.o_v1));
    }
    d.bkey = static_cast<uint64_t*>(at(p.o_bkey));
    d.bmask = static_cast<uint64_t*>(at(p.o_bmask));
    d.bfirst = static_cast<uint32_t*>(at(p.o_bfirst));
    d.binst = static_cast<uint8_t*>(at(p.o_binst));
    d.bdisp = static_cast<uint8_t*>(at(p.o_bdisp));
    d.bref = static_cast<uint32_t*>(at(p.o_bref));
    d.nodes = reinterpret_cast<uint32_t*>(outs[0]);
    d.leaves = reinterpret_cast<uint64_t*>(outs[1]);
    d.ukey = reinterpret_cast<uint64_t*>(outs[2]);
    d.uval = reinterpret_cast<uint32_t*>(outs[3]);
    d.prims = reinterpret_cast<uint8_t*>(outs[4]);
    d.aabbs = reinterpret_cast<float*>(outs[5]);

    levels.clear();
    for (uint32_t lv = 2; lv < d.log2; ++lv) {
        LevelDesc L;
        std::memset(&L, 0, sizeof(L));
        L.lv = lv;
        L.child_bound = lv == 2 ? p.B : p.P[lv - 1];
        L.parent_bound = p.P[lv];
        L.build_tiles = p.btiles[lv];
        L.own_tiles = p.otiles[lv];
        L.build_nb = p.bnb[lv];
        L.own_it = p.oit[lv];
        L.need_box = lv + 1 <= d.rt_log2 ? 1u : 0u;
        L.pcap = p.cap[lv];
        L.tile_ctr_build = kTileLevel0 + 2 * (lv - 2);
        L.tile_ctr_own = kTileLevel0 + 1 + 2 * (lv - 2);
        const int ps = (lv - 2) & 1;
        L.pkey = static_cast<uint64_t*>(at(p.o_set[ps][0]));
        L.pcnt = static_cast<uint32_t*>(at(p.o_set[ps][1]));
        L.pfirst = static_cast<uint32_t*>(at(p.o_set[ps][2]));
        L.pslot = static_cast<uint32_t*>(at(p.o_set[ps][3]));
        L.plo = static_cast<uint64_t*>(at(p.o_set[ps][4]));
        L.phi = static_cast<uint64_t*>(at(p.o_set[ps][5]));
        L.pwords = static_cast<uint32_t*>(at(p.o_set[ps][6]));
        L.cwords = static_cast<uint32_t*>(at(p.o_cwords));
        L.ptable = static_cast<uint4*>(at(p.o_table[lv]));
        L.build_status = static_cast<uint64_t*>(at(p.o_bstat[lv]));
        L.own_status = static_cast<uint64_t*>(at(p.o_ostat[lv]));
        if (lv == 2) {
            L.ckey = d.bkey;
            L.cmask = d.bmask;
            L.cfirst = d.bfirst;
            L.cslot = nullptr;  // brick references come from bref (and the leaf table)
            L.ctable = d.leaf_table;
        } else {
            const LevelDesc& C = levels.back();
            L.ckey = C.pkey;
            L.ccnt = C.pcnt;
            L.cfirst = C.pfirst;
            L.cslot = C.pslot;
            L.clo = C.plo;
            L.chi = C.phi;
            L.ctable = C.ptable;
        }
        levels.push_back(L);
    }
}

// The launches of a bound plan on `st` (the scratch is cleared here). Returns the
// number of kernels launched, or 0 with the CUDA error in *err.
uint32_t launch_plan(const Plan& p, const std::vector<LevelDesc>& levels, cudaStream_t st, cudaError_t* err) {
    const BuildDesc& d = p.d;
    Prof prof(st);
    uint8_t* base = reinterpret_cast<uint8_t*>(d.counters) - p.o_counters;
    *err = cudaMemsetAsync(base, 0, p.zero_bytes, st);
    if (*err == cudaSuccess) *err = cudaMemsetAsync(base + p.zero_bytes, 0xFF, p.ff_bytes, st);
    if (*err != cudaSuccess) return 0;
    prof.mark("memset");
    uint32_t launches = 0;
    launch(k_plan, 1, 1024, 0, st, d);
    ++launches;
    prof.mark("plan");
    if ((*err = cudaGetLastError()) != cudaSuccess) return 0;
    if (p.bucket) {
        launch(k_bkt_count, d.sort_tiles, kBlock, 0, st, d);
        prof.mark("bucket_count");
        launch(k_bkt_scan_tiles, d.bucket_scan_tiles, kBlock, 0, st, d);
        launch(k_bkt_scan_top, 1, kGridScanThreads, 0, st, d);
        launch(k_bkt_scan_apply, d.bucket_scan_tiles, kBlock, 0, st, d);
        prof.mark("bucket_scan");
        launch(k_bkt_scatter, d.sort_tiles, kBlock, 0, st, d);
        prof.mark("bucket_scatter");
        launch(k_grid_count<true>, d.grid_tiles, kBlock, 0, st, d);
        prof.mark("bucket_tile_count");
        if (!d.grid_fold) {
            launch(k_grid_scan, 1, kGridScanThreads, 0, st, d);
            prof.mark("grid_scan");
        }
        launch(k_grid_write<true>, d.grid_tiles, kBlock, 0, st, d);
        prof.mark("bucket_tile_write");
        launches += d.grid_fold ? 7 : 8;
        if (d.chunked) {
            launch(k_grid_chunks, std::max(std::min((p.K + kBlock - 1) / kBlock, 1024u), 1u), kBlock, 0, st, d);
            prof.mark("grid_chunks");
            ++launches;
        }
    } else if (p.grid) {
        launch(k_grid_scatter, d.sort_tiles, kBlock, 0, st, d);
        prof.mark("grid_scatter");
        launch(k_grid_count<false>, d.grid_tiles, kBlock, 0, st, d);
        prof.mark("grid_count");
        if (!d.grid_fold) {
            launch(k_grid_scan, 1, kGridScanThreads, 0, st, d);
            prof.mark("grid_scan");
        }
        launch(k_grid_write<false>, d.grid_tiles, kBlock, 0, st, d);
        prof.mark("grid_write");
        launches += d.grid_fold ? 3 : 4;
        if (d.chunked) {
            launch(k_grid_chunks, std::max(std::min((p.K + kBlock - 1) / kBlock, 1024u), 1u), kBlock, 0, st, d);
            prof.mark("grid_chunks");
            ++launches;
        }
    } else {
        if ((*err = launch_sort_any(p.rb, p.it, d, st, prof)) != cudaSuccess) return 0;
        launches += 3 + p.passes;
    }
    const uint32_t B = p.B;
    if (d.leaf_regions > 1) {
        launch(k_leaf_part, std::max(std::min((B + kBrickTile - 1) / kBrickTile, 148u * 8u), 1u), kBlock, 0, st, d);
        prof.mark("leaf_part");
        ++launches;
        const uint32_t S = d.leaf_cap / d.leaf_regions, nz = (S + kZeroSlots - 1) / kZeroSlots;
        launch(k_leaf_insert_regions, d.leaf_regions * (nz + 1) + (B + kInsTile - 1) / kInsTile, kBlock, 0, st, d);
    } else {
        launch(k_leaf_insert, leaf_insert_grid(d), kBlock, 0, st, d);
    }
    prof.mark("leaf_insert");
    launch(k_leaf_own, d.leafown_tiles, kBlock, 0, st, d);
    prof.mark("leaf_own");
    launches += 2;
    const uint32_t lv0 = tail_level(d.log2, B, p.P);
    launches += launch_levels(d, levels, lv0, make_tail(lv0, p.P, levels, d.leaf_table), st, prof);
    if (d.mode == kModeBatch && p.min_log2 < d.log2) {
        launch(k_batch_roots, std::max(std::min((p.K + 255) / 256, 1024u), 1u), 256, 0, st, d, d.log2);
        prof.mark("batch_roots");
        ++launches;
    }
    if ((*err = cudaGetLastError()) != cudaSuccess) return 0;
    return launches;
}

pyrb_result run_build(const pyrb_exec* e, const Job& job, pyrb_built* out, uint32_t* host_counts = nullptr) {
    if (!out) return fail(PYRB_ERROR_INVALID_ARGUMENT, "out is NULL");
    std::memset(out, 0, sizeof(*out));
    Plan p;
    pyrb_result r = plan_build(job, nullptr, p);
    if (r != PYRB_OK) return r;
    cudaStream_t st = e ? reinterpret_cast<cudaStream_t>(e->stream) : nullptr;
    Mem mem{e, st};

    // ---- allocations
    uint64_t scratch = mem.get(p.scratch_bytes);
    if (!scratch) return fail(PYRB_ERROR_OUT_OF_MEMORY, "device memory for the build scratch (%llu bytes)", (unsigned long long)p.scratch_bytes);
    uint64_t outs[6] = {};
    bool ok = true;
    for (int i = 0; i < 6; ++i) ok = (outs[i] = mem.get(p.out_size[i])) != 0 && ok;
    auto release_outputs = [&] {
        for (uint64_t q : outs) mem.put(q);
    };
    auto cleanup = [&] {
        release_outputs();
        mem.put(scratch);
    };
    if (!ok) {
        cleanup();
        return fail(PYRB_ERROR_OUT_OF_MEMORY, "device memory for the build outputs");
    }
    std::vector<LevelDesc> levels;
    bind_plan(p, scratch, outs, job, levels);
    const BuildDesc& d = p.d;
    const uint32_t K = p.K;

#define CUL(call)                                                                                 \
    do {                                                                                          \
        cudaError_t err_ = (call);                                                                \
        if (err_ != cudaSuccess) {                                                                \
            cleanup();                                                                            \
            return fail(PYRB_ERROR_CUDA, "%s: %s", #call, cudaGetErrorString(err_));              \
        }                                                                                         \
    } while (0)
    cudaError_t lerr = cudaSuccess;
    const uint32_t launches = launch_plan(p, levels, st, &lerr);
    CUL(lerr);

    const uint64_t scratch_bytes = p.scratch_bytes, out_bytes = p.out_bytes();
    auto fill_out = [&] {
        out->log2_size = d.log2;
        out->rt_log2 = d.rt_log2;
        out->nodes = outs[0];
        out->leaves = outs[1];
        out->keys = outs[2];
        out->attrs = outs[3];
        out->prims = outs[4];
        out->aabbs = outs[5];
    };
    auto fill_meta = [&](uint32_t* meta) {
        meta[0] = d.log2; meta[1] = d.rt_log2; meta[2] = p.passes; meta[3] = p.rb; meta[4] = launches;
        std::memcpy(meta + 5, &scratch_bytes, 8);
        std::memcpy(meta + 7, &out_bytes, 8);
    };
    // ---- asynchronous form: counts land in pinned host memory, no synchronisation
    if (host_counts) {
        CUL(cudaMemcpyAsync(host_counts, d.counters, kCtrCount * 4, cudaMemcpyDeviceToHost, st));
        if (p.chunked) {
            if (job.roots) CUL(cudaMemcpyAsync(job.roots, d.roots, uint64_t(K) * 4, cudaMemcpyDeviceToHost, st));
            if (job.first_voxel) CUL(cudaMemcpyAsync(job.first_voxel, d.chunk_first, uint64_t(K) * 4, cudaMemcpyDeviceToHost, st));
            if (job.first_prim) CUL(cudaMemcpyAsync(job.first_prim, d.prim_start, uint64_t(K) * 4, cudaMemcpyDeviceToHost, st));
        }
        mem.put(scratch);
        fill_meta(host_counts + kCtrCount);
        fill_out();
        return PYRB_OK;
    }
    // ---- read back
    uint32_t ctr[kCtrCount];
    CUL(cudaMemcpyAsync(ctr, d.counters, sizeof(ctr), cudaMemcpyDeviceToHost, st));
    if (p.chunked) {
        if (job.roots) CUL(cudaMemcpyAsync(job.roots, d.roots, uint64_t(K) * 4, cudaMemcpyDeviceToHost, st));
        if (job.first_voxel) CUL(cudaMemcpyAsync(job.first_voxel, d.chunk_first, uint64_t(K) * 4, cudaMemcpyDeviceToHost, st));
        if (job.first_prim) CUL(cudaMemcpyAsync(job.first_prim, d.prim_start, uint64_t(K) * 4, cudaMemcpyDeviceToHost, st));
    }
    CUL(cudaStreamSynchronize(st));
    mem.put(scratch);
    scratch = 0;
#undef CUL
    if (ctr[kCtrError]) {
        release_outputs();
        return device_error(ctr);
    }
    fill_out();
    fill_counts(ctr, out);
    uint32_t meta[16] = {};
    fill_meta(meta);
    fill_stats(ctr, meta);
    return PYRB_OK;
}

}  // namespace

namespace pyrb {
// The calling thread's error message, for the library's other translation units.
pyrb_result set_error(pyrb_result r, const char* msg) { return fail(r, "%s", msg); }
}  // namespace pyrb

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

PYRB_API pyrb_result pyrb_build(const pyrb_exec* e, uint32_t log2_size, uint32_t rt_log2_req, uint64_t old_keys,
                                uint64_t old_vals, uint32_t n_old, uint64_t edits, uint32_t n_new, pyrb_built* out) {
    if ((n_old && (!old_keys || !old_vals)) || (n_new && !edits))
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "NULL input pointer with a non-zero count");
    Job j;
    j.mode = kModePlain;
    j.log2 = log2_size;
    j.rt_req = rt_log2_req;
    j.old_keys = old_keys;
    j.old_vals = old_vals;
    j.n_old = n_old;
    j.voxels = edits;
    j.n_new = n_new;
    return run_build(e, j, out);
}

PYRB_API pyrb_result pyrb_build_chunks(const pyrb_exec* e, uint32_t log2_size, uint32_t rt_log2_req,
                                       const pyrb_chunk_batch* batch, uint32_t* roots, uint32_t* first_voxel,
                                       uint32_t* first_prim, pyrb_built* out) {
    if (!batch || batch->count == 0 || batch->capacity == 0)
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "empty chunk batch");
    if (!batch->offsets || (batch->total && !batch->voxels))
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "NULL chunk buffers");
    Job j;
    j.mode = kModeChunks;
    j.log2 = log2_size;
    j.rt_req = rt_log2_req;
    j.K = batch->count;
    j.capacity = batch->capacity;
    j.voxels = batch->voxels;
    j.offsets = batch->offsets;
    j.total = batch->total;
    j.roots = roots;
    j.first_voxel = first_voxel;
    j.first_prim = first_prim;
    return run_build(e, j, out);
}

static pyrb_result batch_job(const pyrb_batch* b, uint32_t rt_log2_req, uint32_t* roots, uint32_t* first_voxel,
                             uint32_t* first_prim, Job& j) {
    if (!b || b->count == 0) return fail(PYRB_ERROR_INVALID_ARGUMENT, "empty batch");
    if (!b->log2_host || !b->log2 || !b->voxel_offsets || (b->voxel_total && !b->voxels))
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "NULL batch buffers");
    if (b->edit_total && (!b->edits || !b->edit_offsets))
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "edit_total > 0 without edit buffers");
    uint32_t lmax = 0;
    for (uint32_t c = 0; c < b->count; ++c) lmax = std::max(lmax, b->log2_host[c]);
    j.mode = kModeBatch;
    j.log2 = lmax;
    j.rt_req = rt_log2_req;
    j.K = b->count;
    j.voxels = b->voxels;
    j.edits = b->edit_total ? b->edits : 0;
    j.chunk_log2_host = b->log2_host;
    j.chunk_log2 = b->log2;
    j.voxel_offsets = b->voxel_offsets;
    j.edit_offsets2 = b->edit_total ? b->edit_offsets : 0;
    j.voxel_starts = b->voxel_starts;
    j.voxel_total = b->voxel_total;
    j.edit_total = b->edit_total;
    j.roots = roots;
    j.first_voxel = first_voxel;
    j.first_prim = first_prim;
    return PYRB_OK;
}

PYRB_API pyrb_result pyrb_build_batch(const pyrb_exec* e, const pyrb_batch* batch, uint32_t rt_log2_req,
                                      uint32_t* roots, uint32_t* first_voxel, uint32_t* first_prim, pyrb_built* out) {
    Job j;
    pyrb_result r = batch_job(batch, rt_log2_req, roots, first_voxel, first_prim, j);
    return r != PYRB_OK ? r : run_build(e, j, out);
}

PYRB_API pyrb_result pyrb_build_batch_async(const pyrb_exec* e, const pyrb_batch* batch, uint32_t rt_log2_req,
                                            uint32_t* roots, uint32_t* first_voxel, uint32_t* first_prim,
                                            uint32_t* host_counts, pyrb_built* out) {
    if (!host_counts) return fail(PYRB_ERROR_INVALID_ARGUMENT, "host_counts is NULL");
    Job j;
    pyrb_result r = batch_job(batch, rt_log2_req, roots, first_voxel, first_prim, j);
    return r != PYRB_OK ? r : run_build(e, j, out, host_counts);
}

PYRB_API pyrb_result pyrb_build_chunks_edits(const pyrb_exec* e, uint32_t log2_size, uint32_t rt_log2_req,
                                             uint32_t count, uint32_t capacity, uint64_t voxels, uint64_t counts,
                                             uint64_t edits, uint64_t edit_offsets, uint32_t edit_total,
                                             uint32_t* roots, uint32_t* first_voxel, uint32_t* first_prim,
                                             pyrb_built* out) {
    if (count == 0 || capacity == 0) return fail(PYRB_ERROR_INVALID_ARGUMENT, "empty chunk batch");
    if (!voxels || !counts || !edit_offsets || (edit_total && !edits))
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "NULL chunk buffers");
    Job j;
    j.mode = kModeChunksEdits;
    j.log2 = log2_size;
    j.rt_req = rt_log2_req;
    j.K = count;
    j.capacity = capacity;
    j.voxels = voxels;
    j.gen_counts = counts;
    j.edits = edits;
    j.edit_offsets = edit_offsets;
    j.edit_total = edit_total;
    j.roots = roots;
    j.first_voxel = first_voxel;
    j.first_prim = first_prim;
    return run_build(e, j, out);
}

PYRB_API pyrb_result pyrb_downsample(const pyrb_exec* e, uint32_t log2_src, uint32_t rt_log2_req, uint64_t src_keys,
                                     uint64_t src_vals, uint32_t n_src, uint32_t shift, pyrb_built* out) {
    if (shift == 0 || shift + 3 > log2_src)
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "downsampling by 2^%u is not possible at 2^%u (result at least 2^3)",
                    shift, log2_src);
    if (n_src && (!src_keys || !src_vals)) return fail(PYRB_ERROR_INVALID_ARGUMENT, "NULL source buffers");
    Job j;
    j.mode = kModeDownsample;
    j.log2 = log2_src - shift;
    j.rt_req = rt_log2_req;
    j.src_keys = src_keys;
    j.src_vals = src_vals;
    j.n_new = n_src;
    j.shift = shift;
    return run_build(e, j, out);
}

PYRB_API pyrb_result pyrb_geometry_build(const pyrb_exec* e, uint32_t log2_size, uint32_t rt_log2_req,
                                         const void* voxels, uint32_t count, uint32_t flags, pyrb_built* out) {
    if (count && !voxels) return fail(PYRB_ERROR_INVALID_ARGUMENT, "voxels is NULL");
    if (!(flags & PYRB_BUILD_HOST_INPUT) || count == 0)
        return pyrb_build(e, log2_size, rt_log2_req, 0, 0, 0, reinterpret_cast<uint64_t>(voxels), count, out);
    cudaStream_t st = e ? reinterpret_cast<cudaStream_t>(e->stream) : nullptr;
    Mem mem{e, st};
    const uint64_t bytes = uint64_t(count) * 16;
    uint64_t dev = mem.get(bytes);
    if (!dev) return fail(PYRB_ERROR_OUT_OF_MEMORY, "device memory for the voxel upload (%llu bytes)", (unsigned long long)bytes);
    cudaError_t err = cudaMemcpyAsync(reinterpret_cast<void*>(dev), voxels, bytes, cudaMemcpyHostToDevice, st);
    if (err != cudaSuccess) {
        mem.put(dev);
        return fail(PYRB_ERROR_CUDA, "upload: %s", cudaGetErrorString(err));
    }
    pyrb_result r = pyrb_build(e, log2_size, rt_log2_req, 0, 0, 0, dev, count, out);
    mem.put(dev);
    return r;
}

PYRB_API void pyrb_built_free(const pyrb_exec* e, pyrb_built* b) {
    if (!b) return;
    cudaStream_t st = e ? reinterpret_cast<cudaStream_t>(e->stream) : nullptr;
    Mem mem{e, st};
    for (uint64_t p : {b->nodes, b->leaves, b->keys, b->attrs, b->prims, b->aabbs}) mem.put(p);
    std::memset(b, 0, sizeof(*b));
}

PYRB_API pyrb_result pyrb_build_async(const pyrb_exec* e, uint32_t log2_size, uint32_t rt_log2_req, uint64_t old_keys,
                                      uint64_t old_vals, uint32_t n_old, uint64_t edits, uint32_t n_new,
                                      uint32_t* host_counts, pyrb_built* out) {
    if (!host_counts) return fail(PYRB_ERROR_INVALID_ARGUMENT, "host_counts is NULL");
    if ((n_old && (!old_keys || !old_vals)) || (n_new && !edits))
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "NULL input pointer with a non-zero count");
    Job j;
    j.mode = kModePlain;
    j.log2 = log2_size;
    j.rt_req = rt_log2_req;
    j.old_keys = old_keys;
    j.old_vals = old_vals;
    j.n_old = n_old;
    j.voxels = edits;
    j.n_new = n_new;
    return run_build(e, j, out, host_counts);
}

PYRB_API pyrb_result pyrb_build_finish(const uint32_t* host_counts, pyrb_built* out) {
    if (!host_counts || !out) return fail(PYRB_ERROR_INVALID_ARGUMENT, "NULL argument");
    if (host_counts[kCtrError]) return device_error(host_counts);
    fill_counts(host_counts, out);
    fill_stats(host_counts, host_counts + kCtrCount);
    return PYRB_OK;
}

PYRB_API void pyrb_profile_enable(int on) { g_prof_on = on != 0; }

PYRB_API uint32_t pyrb_profile_read(float* ms, char* names, uint32_t name_len, uint32_t cap) {
    uint32_t n = uint32_t(g_prof_names.size());
    for (uint32_t i = 0; i < n && i < cap; ++i) {
        float t = 0;
        cudaEventElapsedTime(&t, g_prof_events[i], g_prof_events[i + 1]);
        if (ms) ms[i] = t;
        if (names && name_len) {
            snprintf(names + uint64_t(i) * name_len, name_len, "%s%s%u", g_prof_names[i].first,
                     g_prof_names[i].second || std::strcmp(g_prof_names[i].first, "sort_pass") == 0 ? ":" : "",
                     g_prof_names[i].second);
            if (!(g_prof_names[i].second || std::strcmp(g_prof_names[i].first, "sort_pass") == 0))
                snprintf(names + uint64_t(i) * name_len, name_len, "%s", g_prof_names[i].first);
        }
    }
    return n;
}

PYRB_API void pyrb_last_stats(pyrb_stats* out) {
    if (out) *out = g_stats;
}

PYRB_API const char* pyrb_error_message(void) { return g_msg; }

PYRB_API const char* pyrb_result_string(pyrb_result r) {
    switch (r) {
        case PYRB_OK: return "ok";
        case PYRB_ERROR_INVALID_ARGUMENT: return "invalid argument";
        case PYRB_ERROR_OUT_OF_MEMORY: return "out of memory";
        case PYRB_ERROR_CAPACITY: return "capacity exceeded";
        case PYRB_ERROR_CUDA: return "CUDA error";
        default: return "unknown result";
    }
}

PYRB_API pyrb_result pyrb_set_tuning(const pyrb_tuning* t) {
    if (!t) return fail(PYRB_ERROR_INVALID_ARGUMENT, "tuning is NULL");
    if ((t->radix_bits == 0) != (t->tile_keys == 0))
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "radix_bits and tile_keys are 0 together (automatic) or neither");
    if (t->radix_bits != 0 && t->radix_bits != 4 && (t->radix_bits < 8 || t->radix_bits > 11))
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "radix_bits must be 4, 8, 9, 10 or 11");
    if (t->tile_keys != 0 && t->tile_keys != 1024 && t->tile_keys != 2048 && t->tile_keys != 4096 && t->tile_keys != 8192)
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "tile_keys must be 1024, 2048, 4096 or 8192");
    if (t->tile_keys == 8192 && t->radix_bits != 8 && t->radix_bits != 9)
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "8192-key tiles take 8- or 9-bit digits");
    if (t->load_factor_pct < 25 || t->load_factor_pct > 90)
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "load_factor_pct must lie in [25, 90]");
    if (t->path > kPathBucket)
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "path must be 0 (automatic), 1 (sort), 2 (grid) or 3 (bucket)");
    g_radix_bits = t->radix_bits;
    g_tile_keys = t->tile_keys;
    g_load_pct = t->load_factor_pct;
    g_path = t->path;
    return PYRB_OK;
}

PYRB_API void pyrb_get_tuning(pyrb_tuning* t) {
    if (!t) return;
    t->radix_bits = g_radix_bits;
    t->tile_keys = g_tile_keys;
    t->load_factor_pct = g_load_pct;
    t->path = g_path;
}

// PYRD v1 (src/io.zig:88-129): 52-byte header, then nodes, leaves, attributes.
constexpr uint64_t kPyrdHeader = 4 + 4 * 4 + 8 * 4;

PYRB_API pyrb_result pyrb_pyrd_save(const pyrb_exec* e, const pyrb_built* b, void* out, uint64_t* size) {
    if (!b) return fail(PYRB_ERROR_INVALID_ARGUMENT, "built is NULL");
    if (!size) return fail(PYRB_ERROR_INVALID_ARGUMENT, "size is NULL");
    if (b->node_words == 0 || b->root + 1 >= b->node_words)
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "built has no root node (node_words %u, root %u)", b->node_words, b->root);
    const uint64_t nw = b->node_words, nl = b->leaf_count, na = b->voxel_count;
    const uint64_t need = kPyrdHeader + nw * 4 + nl * 8 + na * 4;
    if (out) {
        if (*size < need) return fail(PYRB_ERROR_INVALID_ARGUMENT, "buffer too small: %llu bytes needed",
                                      static_cast<unsigned long long>(need));
        cudaStream_t st = e ? reinterpret_cast<cudaStream_t>(e->stream) : nullptr;
        uint8_t* o = static_cast<uint8_t*>(out);
        uint8_t* body = o + kPyrdHeader;
        CU(cudaMemcpyAsync(body, reinterpret_cast<const void*>(b->nodes), nw * 4, cudaMemcpyDeviceToHost, st));
        if (nl) CU(cudaMemcpyAsync(body + nw * 4, reinterpret_cast<const void*>(b->leaves), nl * 8, cudaMemcpyDeviceToHost, st));
        if (na) CU(cudaMemcpyAsync(body + nw * 4 + nl * 8, reinterpret_cast<const void*>(b->attrs), na * 4,
                                   cudaMemcpyDeviceToHost, st));
        CU(cudaStreamSynchronize(st));
        uint32_t root_count = 0;
        std::memcpy(&root_count, body + (uint64_t(b->root) + 1) * 4, 4);
        std::memcpy(o, "PYRD", 4);
        const uint32_t h32[4] = {1u, b->log2_size, b->root, 1u};
        const uint64_t h64[4] = {root_count, nw, nl, na};
        std::memcpy(o + 4, h32, sizeof(h32));
        std::memcpy(o + 20, h64, sizeof(h64));
    }
    *size = need;
    return PYRB_OK;
}

PYRB_API pyrb_result pyrb_pyrd_load(const pyrb_exec* e, const void* data, uint64_t len, pyrb_built* out) {
    if (!out) return fail(PYRB_ERROR_INVALID_ARGUMENT, "out is NULL");
    std::memset(out, 0, sizeof(*out));
    if (!data) return fail(PYRB_ERROR_INVALID_ARGUMENT, "data is NULL");
    const uint8_t* d = static_cast<const uint8_t*>(data);
    if (len < kPyrdHeader || std::memcmp(d, "PYRD", 4) != 0) return fail(PYRB_ERROR_INVALID_ARGUMENT, "no valid DAG data");
    uint32_t h32[4];
    uint64_t h64[4];
    std::memcpy(h32, d + 4, sizeof(h32));
    std::memcpy(h64, d + 20, sizeof(h64));
    const uint32_t version = h32[0], log2 = h32[1], root = h32[2];
    const bool has_attrs = (h32[3] & 1) != 0;
    const uint64_t voxel_count = h64[0], nw = h64[1], nl = h64[2], na = h64[3];
    if (version != 1 || log2 < 3 || log2 > 20) return fail(PYRB_ERROR_INVALID_ARGUMENT, "no valid DAG data");
    // 32-bit counts in pyrb_built; the overflow-safe size check of io.load
    if (nw > 0xFFFFFFFFull || nl > 0xFFFFFFFFull || na > 0xFFFFFFFFull)
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "no valid DAG data");
    const uint64_t need = kPyrdHeader + nw * 4 + nl * 8 + na * 4;
    if (need > len || root >= nw || (has_attrs && na != voxel_count))
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "no valid DAG data");
    cudaStream_t st = e ? reinterpret_cast<cudaStream_t>(e->stream) : nullptr;
    Mem mem{e, st};
    pyrb_built r = {};
    r.log2_size = log2;
    r.root = root;
    r.node_words = uint32_t(nw);
    r.leaf_count = uint32_t(nl);
    r.voxel_count = uint32_t(has_attrs ? na : std::min<uint64_t>(voxel_count, 0xFFFFFFFFull));
    r.nodes = mem.get(nw * 4);
    r.leaves = nl ? mem.get(nl * 8) : 0;
    r.attrs = (has_attrs && na) ? mem.get(na * 4) : 0;
    if (!r.nodes || (nl && !r.leaves) || (has_attrs && na && !r.attrs)) {
        pyrb_built_free(e, &r);
        return fail(PYRB_ERROR_OUT_OF_MEMORY, "device memory for a loaded DAG (%llu bytes)",
                    static_cast<unsigned long long>(need));
    }
    const uint8_t* body = d + kPyrdHeader;
    cudaError_t err = cudaMemcpyAsync(reinterpret_cast<void*>(r.nodes), body, nw * 4, cudaMemcpyHostToDevice, st);
    if (err == cudaSuccess && nl)
        err = cudaMemcpyAsync(reinterpret_cast<void*>(r.leaves), body + nw * 4, nl * 8, cudaMemcpyHostToDevice, st);
    if (err == cudaSuccess && r.attrs)
        err = cudaMemcpyAsync(reinterpret_cast<void*>(r.attrs), body + nw * 4 + nl * 8, na * 4, cudaMemcpyHostToDevice, st);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st);
    if (err != cudaSuccess) {
        pyrb_built_free(e, &r);
        return fail(PYRB_ERROR_CUDA, "upload of a loaded DAG: %s", cudaGetErrorString(err));
    }
    *out = r;
    return PYRB_OK;
}

// ---------------------------------------------------------------------------
// Chunk attribute palettes (src/device/palette.zig, src/context.zig:1311-1360)
// ---------------------------------------------------------------------------
namespace {
// Device copies of the per-chunk host arrays plus the tile plan; freed stream-ordered.
struct PaletteJob {
    Mem mem;
    PaletteDesc p = {};
    uint64_t blocks[4] = {};
    uint32_t tiles = 0;
    pyrb_result setup(const uint32_t* first, uint32_t count) {
        std::vector<uint32_t> tile_of(count + 1);
        uint64_t t = 0;
        for (uint32_t c = 0; c < count; ++c) {
            if (first[c + 1] < first[c]) return fail(PYRB_ERROR_INVALID_ARGUMENT, "first[%u] > first[%u]", c, c + 1);
            tile_of[c] = uint32_t(t);
            // at least one tile: a chunk without voxels still gets its palette words
            t += std::max<uint64_t>((uint64_t(first[c + 1] - first[c]) + kPalTile - 1) / kPalTile, 1);
            if (t >= (uint64_t(1) << 31)) return fail(PYRB_ERROR_INVALID_ARGUMENT, "too many voxels");
        }
        tile_of[count] = uint32_t(t);
        tiles = uint32_t(t);
        blocks[0] = mem.get(uint64_t(count + 1) * 8);
        if (!blocks[0]) return fail(PYRB_ERROR_OUT_OF_MEMORY, "device memory for the palette plan");
        uint32_t* dfirst = reinterpret_cast<uint32_t*>(blocks[0]);
        CU(cudaMemcpyAsync(dfirst, first, uint64_t(count + 1) * 4, cudaMemcpyHostToDevice, mem.st));
        CU(cudaMemcpyAsync(dfirst + count + 1, tile_of.data(), uint64_t(count + 1) * 4, cudaMemcpyHostToDevice,
                           mem.st));
        CU(cudaStreamSynchronize(mem.st));  // the host vector goes out of scope
        p.first = dfirst;
        p.tile_of = dfirst + count + 1;
        p.count = count;
        return PYRB_OK;
    }
    uint32_t* take(int k, uint64_t bytes) {
        blocks[k] = mem.get(bytes);
        return reinterpret_cast<uint32_t*>(blocks[k]);
    }
    ~PaletteJob() {
        for (uint64_t b : blocks) mem.put(b);
    }
};
}  // namespace

PYRB_API pyrb_result pyrb_palette_scan(const pyrb_exec* e, uint64_t attrs, const uint32_t* first, uint32_t count,
                                       uint64_t palettes, uint32_t* counts) {
    if (!first || !counts || (count && !palettes)) return fail(PYRB_ERROR_INVALID_ARGUMENT, "NULL pointer");
    if (count == 0) return PYRB_OK;
    if (first[count] > first[0] && !attrs) return fail(PYRB_ERROR_INVALID_ARGUMENT, "attrs is NULL");
    PaletteJob j{Mem{e, e ? reinterpret_cast<cudaStream_t>(e->stream) : nullptr}};
    pyrb_result r = j.setup(first, count);
    if (r != PYRB_OK) return r;
    const cudaStream_t st = j.mem.st;
    j.p.attrs = reinterpret_cast<const uint32_t*>(attrs);
    uint32_t* tab = j.take(1, uint64_t(count) * kPalSlots * 8);
    uint32_t* small = j.take(2, uint64_t(count) * 8);
    if (!tab || !small) return fail(PYRB_ERROR_OUT_OF_MEMORY, "device memory for the palette tables");
    j.p.gval = tab;
    j.p.gfirst = tab + uint64_t(count) * kPalSlots;
    j.p.gflag = small;
    j.p.counts = small + count;
    j.p.palettes = reinterpret_cast<uint32_t*>(palettes);
    CU(cudaMemsetAsync(tab, 0xFF, uint64_t(count) * kPalSlots * 8, st));
    CU(cudaMemsetAsync(small, 0, uint64_t(count) * 4, st));
    launch(k_pal_collect, j.tiles, kBlock, 0, st, j.p);
    launch(k_pal_layout, (count + kBlock - 1) / kBlock, kBlock, 0, st, j.p);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(counts, j.p.counts, uint64_t(count) * 4, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    return PYRB_OK;
}

PYRB_API pyrb_result pyrb_palette_pack(const pyrb_exec* e, uint64_t attrs, const uint32_t* first, uint32_t count,
                                       uint64_t palettes, const uint32_t* counts, const uint32_t* dst, uint64_t pool) {
    if (!first || !counts || !dst || (count && (!palettes || !pool)))
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "NULL pointer");
    if (count == 0) return PYRB_OK;
    if (first[count] > first[0] && !attrs) return fail(PYRB_ERROR_INVALID_ARGUMENT, "attrs is NULL");
    PaletteJob j{Mem{e, e ? reinterpret_cast<cudaStream_t>(e->stream) : nullptr}};
    pyrb_result r = j.setup(first, count);
    if (r != PYRB_OK) return r;
    const cudaStream_t st = j.mem.st;
    uint32_t* small = j.take(1, uint64_t(count) * 8);
    if (!small) return fail(PYRB_ERROR_OUT_OF_MEMORY, "device memory for the palette plan");
    CU(cudaMemcpyAsync(small, counts, uint64_t(count) * 4, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(small + count, dst, uint64_t(count) * 4, cudaMemcpyHostToDevice, st));
    j.p.attrs = reinterpret_cast<const uint32_t*>(attrs);
    j.p.palettes = reinterpret_cast<uint32_t*>(palettes);
    j.p.counts = small;
    j.p.dst = small + count;
    j.p.pool = reinterpret_cast<uint32_t*>(pool);
    launch(k_pal_pack, j.tiles, kBlock, 0, st, j.p);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(st));
    return PYRB_OK;
}

// ---------------------------------------------------------------------------
// Path edits (src/device/pathedit.zig; host side of Context.pathEdit,
// src/context.zig:1093-1290, without its pool bookkeeping)
// ---------------------------------------------------------------------------
static_assert(sizeof(pyrb_path_edit_job) == sizeof(PathEditJob), "pyrb_path_edit_job layout");

PYRB_API pyrb_result pyrb_path_edit(const pyrb_exec* e, uint64_t nodes, uint64_t leaves, uint64_t attributes,
                                    pyrb_path_edit_job* jobs, uint32_t count, const uint32_t* edits,
                                    uint32_t n_edits) {
    if (count == 0) return PYRB_OK;
    if (!jobs || !nodes || !leaves || !attributes || (n_edits && !edits))
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "NULL pointer");
    uint32_t max_edits = 1;
    std::vector<uint32_t> attr_tile(count + 1), prim_tile(count + 1);
    uint64_t at = 0, pt = 0;
    for (uint32_t j = 0; j < count; ++j) {
        const pyrb_path_edit_job& jb = jobs[j];
        if (jb.edit_count > kPeMaxEdits)
            return fail(PYRB_ERROR_INVALID_ARGUMENT, "job %u: %u edits (at most %u per job)", j, jb.edit_count,
                        kPeMaxEdits);
        if (uint64_t(jb.edit_first) + jb.edit_count > n_edits)
            return fail(PYRB_ERROR_INVALID_ARGUMENT, "job %u: edits beyond the %u given", j, n_edits);
        if (jb.log2_size < 3 || jb.log2_size > 20 || jb.rt_log2 < 3 || jb.rt_log2 > jb.log2_size)
            return fail(PYRB_ERROR_INVALID_ARGUMENT, "job %u: log2_size %u / rt_log2 %u", j, jb.log2_size, jb.rt_log2);
        if (jb.node_arena < jb.node_offset || jb.leaf_arena < jb.leaf_offset)
            return fail(PYRB_ERROR_INVALID_ARGUMENT, "job %u: arena below the geometry", j);
        max_edits = std::max(max_edits, jb.edit_count);
        attr_tile[j] = uint32_t(at);
        prim_tile[j] = uint32_t(pt);
        // attribute slots of the job's target (32-bit values, or 8 indices per word)
        at += (uint64_t(jb.attr_count) + jb.edit_count + kPeTile - 1) / kPeTile;
        pt += (uint64_t(jb.prim_count) + kBlock - 1) / kBlock;
    }
    attr_tile[count] = uint32_t(at);
    prim_tile[count] = uint32_t(pt);
    if (at >= (uint64_t(1) << 31) || pt >= (uint64_t(1) << 31)) return fail(PYRB_ERROR_INVALID_ARGUMENT, "too many attributes");
    // Context.pathEdit: each job's edits stably ordered by brick, so that a brick is
    // one run (one new path per brick rather than per voxel)
    std::vector<uint32_t> sorted(uint64_t(std::max(n_edits, 1u)) * 4, 0);
    if (n_edits) std::memcpy(sorted.data(), edits, uint64_t(n_edits) * 16);
    for (uint32_t j = 0; j < count; ++j) {
        std::vector<std::array<uint32_t, 4>> v(jobs[j].edit_count);
        for (uint32_t k = 0; k < jobs[j].edit_count; ++k)
            std::memcpy(v[k].data(), edits + uint64_t(jobs[j].edit_first + k) * 4, 16);
        auto key = [](const std::array<uint32_t, 4>& a) {
            return (uint64_t(a[2] >> 2) << 42) | (uint64_t(a[1] >> 2) << 21) | uint64_t(a[0] >> 2);
        };
        std::stable_sort(v.begin(), v.end(), [&](const std::array<uint32_t, 4>& a, const std::array<uint32_t, 4>& b) {
            return key(a) < key(b);
        });
        for (uint32_t k = 0; k < jobs[j].edit_count; ++k)
            std::memcpy(sorted.data() + uint64_t(jobs[j].edit_first + k) * 4, v[k].data(), 16);
    }
    cudaStream_t st = e ? reinterpret_cast<cudaStream_t>(e->stream) : nullptr;
    Mem mem{e, st};
    const uint64_t jobs_bytes = uint64_t(count) * sizeof(PathEditJob);
    const uint64_t edit_bytes = uint64_t(std::max(n_edits, 1u)) * 16;
    const uint64_t plan_bytes = uint64_t(count + 1) * 8;
    const uint64_t block = mem.get(align_up(jobs_bytes, 256) + align_up(edit_bytes, 256) + plan_bytes);
    if (!block) return fail(PYRB_ERROR_OUT_OF_MEMORY, "device memory for the path edits");
    PathEditDesc p;
    p.nodes = reinterpret_cast<uint32_t*>(nodes);
    p.leaves = reinterpret_cast<uint64_t*>(leaves);
    p.attrs = reinterpret_cast<uint32_t*>(attributes);
    p.jobs = reinterpret_cast<PathEditJob*>(block);
    p.edits = reinterpret_cast<uint4*>(block + align_up(jobs_bytes, 256));
    uint32_t* plan = reinterpret_cast<uint32_t*>(block + align_up(jobs_bytes, 256) + align_up(edit_bytes, 256));
    p.attr_tile = plan;
    p.prim_tile = plan + count + 1;
    p.count = count;
    auto done = [&](pyrb_result r) {
        mem.put(block);
        return r;
    };
    cudaError_t err = cudaMemcpyAsync(p.jobs, jobs, jobs_bytes, cudaMemcpyHostToDevice, st);
    if (err == cudaSuccess) err = cudaMemcpyAsync(p.edits, sorted.data(), edit_bytes, cudaMemcpyHostToDevice, st);
    if (err == cudaSuccess) err = cudaMemcpyAsync(plan, attr_tile.data(), uint64_t(count + 1) * 4, cudaMemcpyHostToDevice, st);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(plan + count + 1, prim_tile.data(), uint64_t(count + 1) * 4, cudaMemcpyHostToDevice, st);
    if (err != cudaSuccess) return done(fail(PYRB_ERROR_CUDA, "path edit upload: %s", cudaGetErrorString(err)));
    const size_t ops_smem = size_t(max_edits) * 16;
    cudaFuncSetAttribute(k_path_attrs, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kPeMaxEdits * 16));
    launch(k_path_walk, (count + 3) / 4, 128, 0, st, p);
    if (at) launch(k_path_attrs, uint32_t(at), kBlock, ops_smem, st, p);
    if (pt) launch(k_path_boxes, uint32_t(pt), kBlock, 0, st, p);
    err = cudaGetLastError();
    if (err == cudaSuccess) err = cudaMemcpyAsync(jobs, p.jobs, jobs_bytes, cudaMemcpyDeviceToHost, st);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st);
    if (err != cudaSuccess) return done(fail(PYRB_ERROR_CUDA, "path edit: %s", cudaGetErrorString(err)));
    return done(PYRB_OK);
}

PYRB_API pyrb_result pyrb_build_memory(uint32_t log2_size, uint32_t rt_log2_req, uint32_t count,
                                       const uint32_t* chunk_log2, uint64_t entries, uint64_t* scratch_bytes,
                                       uint64_t* output_bytes) {
    if (count == 0) return fail(PYRB_ERROR_INVALID_ARGUMENT, "count is 0");
    if (entries >= (uint64_t(1) << 31))
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "too many entries for one build (%llu)", (unsigned long long)entries);
    Job j;
    j.K = count;
    j.rt_req = rt_log2_req;
    if (chunk_log2) {
        uint32_t lmax = 0;
        for (uint32_t c = 0; c < count; ++c) lmax = std::max(lmax, chunk_log2[c]);
        j.mode = kModeBatch;
        j.log2 = lmax;
        j.chunk_log2_host = chunk_log2;
        j.voxel_total = uint32_t(entries);
    } else if (count > 1) {
        j.mode = kModeChunks;
        j.log2 = log2_size;
        j.total = uint32_t(entries);
    } else {
        j.mode = kModePlain;
        j.log2 = log2_size;
        j.n_new = uint32_t(entries);
    }
    Plan p;
    pyrb_result r = plan_build(j, nullptr, p);
    if (r != PYRB_OK) return r;
    if (scratch_bytes) *scratch_bytes = p.scratch_bytes;
    if (output_bytes) *output_bytes = p.out_bytes();
    return PYRB_OK;
}

PYRB_API uint32_t pyrb_last_capacity_need(void) { return g_capacity_need; }

PYRB_API pyrb_result pyrb_selftest_wait_limit(const pyrb_exec* e, uint32_t which) {
    if (which > 1) return fail(PYRB_ERROR_INVALID_ARGUMENT, "which must be 0 or 1");
    cudaStream_t st = e ? reinterpret_cast<cudaStream_t>(e->stream) : nullptr;
    Mem mem{e, st};
    const uint64_t block = mem.get(1024);
    if (!block) return fail(PYRB_ERROR_OUT_OF_MEMORY, "device memory for the wait self-test");
    uint64_t* status = reinterpret_cast<uint64_t*>(block);
    uint32_t* counters = reinterpret_cast<uint32_t*>(block + 64);
    uint32_t ctr[kCtrCount] = {};
    cudaError_t err = cudaMemsetAsync(reinterpret_cast<void*>(block), 0, 1024, st);
    if (err == cudaSuccess) {
        k_selftest_wait<<<1, 32, 0, st>>>(status, counters, which);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpyAsync(ctr, counters, sizeof(ctr), cudaMemcpyDeviceToHost, st);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st);
    mem.put(block);
    if (err != cudaSuccess) return fail(PYRB_ERROR_CUDA, "wait self-test: %s", cudaGetErrorString(err));
    return ctr[kCtrError] ? device_error(ctr) : PYRB_OK;
}

PYRB_API uint32_t pyrb_version(void) { return (0u << 16) | 2u; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Build without any device allocation (pyrb_build_noalloc).
//
// Some callers cannot allocate device memory while they build: a render or frame
// loop must not call cudaMalloc (it synchronises the whole device and stalls the
// frame), and an engine whose device memory is budgeted up front has no allocator
// to offer for scratch. For them all scratch of the build lives in this fixed,
// file-scope device array; the caller brings input and output buffers. Every GPU
// that loads the library keeps the array until the process exits.
// ---------------------------------------------------------------------------
namespace {

constexpr uint64_t kStaticScratchBytes = 64ull << 20;   // 64 MiB per device
constexpr uint32_t kStaticMaxEntries = 1u << 20;        // input voxels per build
constexpr uint32_t kStaticMaxLog2 = 8;                  // edge 256

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_static_mu;
void* g_static_addr[64] = {};

// Device address of the array on the current device. The name g_static_scratch is
// only a host-side stand-in in host code; the first call per device (with that
// device current) resolves the real address with cudaGetSymbolAddress, and later
// calls reuse it. The address belongs to the device's primary context: after a
// cudaDeviceReset the library must be loaded again.
pyrb_result static_scratch(void** out) {
    int dev = 0;
    CU(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(PYRB_ERROR_CUDA, "device index %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (!g_static_addr[dev]) {
        void* p = nullptr;
        cudaError_t err = cudaGetSymbolAddress(&p, g_static_scratch);
        if (err != cudaSuccess || !p)
            return fail(PYRB_ERROR_CUDA, "cudaGetSymbolAddress(static scratch): %s", cudaGetErrorString(err));
        g_static_addr[dev] = p;
    }
    *out = g_static_addr[dev];
    return PYRB_OK;
}

}  // namespace

extern "C" {

PYRB_API pyrb_result pyrb_build_noalloc(void* stream, uint32_t log2_size, uint32_t rt_log2_req, uint64_t edits,
                                        uint32_t n_new, uint64_t nodes, uint32_t node_capacity, uint64_t leaves,
                                        uint32_t leaf_capacity, uint64_t keys, uint64_t attrs,
                                        uint32_t voxel_capacity, uint64_t prims, uint64_t aabbs,
                                        uint32_t prim_capacity, pyrb_built* out) {
    if (!out) return fail(PYRB_ERROR_INVALID_ARGUMENT, "out is NULL");
    std::memset(out, 0, sizeof(*out));
    if (log2_size < 3 || log2_size > kStaticMaxLog2)
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "pyrb_build_noalloc: log2_size must lie in [3, %u] (got %u)",
                    kStaticMaxLog2, log2_size);
    if (n_new > kStaticMaxEntries)
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "pyrb_build_noalloc: %u voxels exceed the fixed limit of %u", n_new,
                    kStaticMaxEntries);
    if (n_new && !edits) return fail(PYRB_ERROR_INVALID_ARGUMENT, "edits is NULL");
    if (!nodes || !leaves || !keys || !attrs || !prims || !aabbs)
        return fail(PYRB_ERROR_INVALID_ARGUMENT, "pyrb_build_noalloc: every output buffer is required");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    Job j;
    j.mode = kModePlain;
    j.log2 = log2_size;
    j.rt_req = rt_log2_req;
    j.voxels = edits;
    j.n_new = n_new;
    // one fixed tuning: the scratch bound below holds for it at every allowed size
    const Tune fixed{8, 4096, 50, kPathSort};
    Plan p;
    pyrb_result r = plan_build(j, &fixed, p);
    if (r != PYRB_OK) return r;
    const uint32_t prim_need = std::max(p.d.prim_bound, 1u);
    if (node_capacity < p.d.node_bound || leaf_capacity < p.B || voxel_capacity < p.nmax || prim_capacity < prim_need)
        return fail(PYRB_ERROR_INVALID_ARGUMENT,
                    "pyrb_build_noalloc: output buffers too small (need nodes %u words, leaves %u, keys/attrs %u, "
                    "prims %u)", p.d.node_bound, p.B, p.nmax, prim_need);
    if (p.scratch_bytes > kStaticScratchBytes)
        return fail(PYRB_ERROR_INVALID_ARGUMENT,
                    "pyrb_build_noalloc: this build needs %llu bytes of scratch, the fixed array holds %llu",
                    (unsigned long long)p.scratch_bytes, (unsigned long long)kStaticScratchBytes);

    void* base = nullptr;
    r = static_scratch(&base);
    if (r != PYRB_OK) return r;
    const uint64_t outs[6] = {nodes, leaves, keys, attrs, prims, aabbs};
    std::vector<LevelDesc> levels;
    bind_plan(p, reinterpret_cast<uint64_t>(base), outs, j, levels);
    // the array keeps the previous call's contents: launch_plan clears everything that
    // must start at zero (counters, histograms, look-back status, dedup tables) and the
    // 0xFF part before the first kernel
    cudaError_t err = cudaSuccess;
    const uint32_t launches = launch_plan(p, levels, st, &err);
    if (err != cudaSuccess) return fail(PYRB_ERROR_CUDA, "pyrb_build_noalloc: %s", cudaGetErrorString(err));
    uint32_t ctr[kCtrCount];
    CU(cudaMemcpyAsync(ctr, p.d.counters, sizeof(ctr), cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    if (ctr[kCtrError]) return device_error(ctr);
    out->log2_size = p.d.log2;
    out->rt_log2 = p.d.rt_log2;
    out->nodes = nodes;
    out->leaves = leaves;
    out->keys = keys;
    out->attrs = attrs;
    out->prims = prims;
    out->aabbs = aabbs;
    fill_counts(ctr, out);
    uint32_t meta[16] = {p.d.log2, p.d.rt_log2, p.passes, p.rb, launches};
    const uint64_t out_bytes = p.out_bytes();
    std::memcpy(meta + 5, &p.scratch_bytes, 8);
    std::memcpy(meta + 7, &out_bytes, 8);
    fill_stats(ctr, meta);
    return PYRB_OK;
}

}  // extern "C"
