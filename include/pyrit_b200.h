/* pyrit_b200 -- B200-native (sm_100a) sparse-voxel-DAG build for Pyrit.
 *
 * C ABI that replaces the GPU build seam of the reference, src/gpu_build.zig
 * (build :94-96, buildChunks :119-122, downsample :128-131, Built :26-47,
 * Exec :14-23). Plain pointers and sizes only; device buffers are passed as
 * 64-bit device addresses exactly like the reference's `u64` fields.
 *
 * Output layout (bit-exact with the reference GPU build):
 *   nodes   u32[node_words]  level by level (8^3 nodes first, root last); a node is
 *           [child mask, saturating voxel count, one ref per child]; refs of 8^3
 *           nodes are leaf indices, all others word offsets (src/device/dag.zig:1-16)
 *   leaves  u64[leaf_count]  unique 4^3 brick masks in first-occurrence Morton order
 *   keys    u64[voxel_count] sorted unique voxel keys (brick Morton << 6 | bit), with
 *           the chunk number above 3*log2_size bits in chunk batches
 *   attrs   u32[voxel_count] attributes in Morton (= depth-first) order
 *   prims   {u32 node, u32 attr_base, u64 cell}[prim_count], aabbs f32[prim_count][6]
 *           (src/device/types.zig:518-526) at edge 2^rt_log2
 * All output buffers belong to the caller; free them with pyrb_built_free.
 *
 * Thread safety: one build at a time per stream; different streams may build
 * concurrently. No call synchronises the device, only the caller's stream.
 */
#ifndef PYRIT_B200_H
#define PYRIT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define PYRB_API __declspec(dllexport)
#else
#define PYRB_API __attribute__((visibility("default")))
#endif

/* Result codes: the PyrResult values of include/pyrit.h:343-353 that the build can return. */
typedef int32_t pyrb_result;
#define PYRB_OK                      0
#define PYRB_ERROR_INVALID_ARGUMENT -1
#define PYRB_ERROR_OUT_OF_MEMORY    -3
#define PYRB_ERROR_CAPACITY         -4  /* world path: a chunk's generator count exceeds the capacity */
#define PYRB_ERROR_CUDA             -6

/* Memory and stream of a build (replaces gpu_build.Exec, src/gpu_build.zig:14-23).
 * alloc/free may be NULL: the library then allocates stream-ordered from its own
 * device memory pool (cudaMallocAsync on `stream`), which is what the reference's
 * Context.execOn does with cuMemAllocAsync (src/context.zig:873-911).
 * alloc returns 0 on failure. free must accept pointers returned by alloc. */
typedef struct pyrb_exec {
    void*    ctx;
    void*    stream;                                  /* cudaStream_t / CUstream; NULL = legacy default stream */
    uint64_t (*alloc)(void* ctx, uint64_t bytes);
    void     (*free)(void* ctx, uint64_t ptr);
} pyrb_exec;

/* gpu_build.Built (src/gpu_build.zig:26-47); all buffers are device memory owned by the caller. */
typedef struct pyrb_built {
    uint32_t log2_size;
    uint32_t rt_log2;
    uint64_t nodes;
    uint32_t node_words;
    uint32_t root;
    uint64_t leaves;
    uint32_t leaf_count;
    uint32_t reserved0;
    uint64_t keys;
    uint64_t attrs;
    uint32_t voxel_count;
    uint32_t reserved1;
    uint64_t prims;
    uint64_t aabbs;
    uint32_t prim_count;
    uint32_t reserved2;
} pyrb_built;

/* Build statistics of the last successful build on the calling thread. */
typedef struct pyrb_stats {
    uint32_t brick_count;            /* non-empty 4^3 bricks (B) */
    uint32_t level_parents[24];      /* P_l: parent nodes of level l before dedup (l = 2 .. log2-1) */
    uint32_t level_unique[24];       /* U_l: unique nodes of level l */
    uint32_t sort_passes;            /* radix passes of the onesweep sort (over the 3 log2 - 6 brick bits) */
    uint32_t radix_bits;             /* widest digit */
    uint32_t kernel_launches;        /* kernels launched by the build */
    uint32_t reserved;
    uint64_t scratch_bytes;          /* device scratch of the build (without outputs) */
    uint64_t output_bytes;           /* device bytes of the output buffers (upper bounds) */
} pyrb_stats;

/* gpu_build.build (src/gpu_build.zig:94-96): a DAG from n_old already sorted unique
 * voxels (old_keys u64 / old_vals u32, e.g. the previous version of an editable
 * geometry; copied, not consumed) and n_new entries `edits` (PyrVoxel[n_new],
 * {int32 x, y, z; uint32 attribute}) in any order. New entries override old ones,
 * the last of equal coordinates wins, attribute 0 deletes, coordinates outside
 * [0, 2^log2_size) are dropped. log2_size in [3, 20]; rt_log2_req is clamped to
 * [3, log2_size]. Synchronises `stream` once at the end to read the counts. */
PYRB_API pyrb_result pyrb_build(const pyrb_exec* e, uint32_t log2_size, uint32_t rt_log2_req,
                                uint64_t old_keys, uint64_t old_vals, uint32_t n_old,
                                uint64_t edits, uint32_t n_new, pyrb_built* out);

/* Asynchronous form of pyrb_build (no synchronisation at all): the counts are copied
 * into `host_counts` (pinned host memory, PYRB_COUNTS_WORDS u32) on the stream. Once
 * the stream has passed that copy, pyrb_build_finish fills the counts of `out`
 * (node_words, root, leaf_count, voxel_count, prim_count) and reports device-side
 * errors. The buffer pointers of `out` are valid immediately in stream order.
 * Scratch is released stream-ordered, so this form needs the default allocator or
 * stream-ordered alloc/free callbacks. */
#define PYRB_COUNTS_WORDS 176
PYRB_API pyrb_result pyrb_build_async(const pyrb_exec* e, uint32_t log2_size, uint32_t rt_log2_req,
                                      uint64_t old_keys, uint64_t old_vals, uint32_t n_old,
                                      uint64_t edits, uint32_t n_new, uint32_t* host_counts, pyrb_built* out);
PYRB_API pyrb_result pyrb_build_finish(const uint32_t* host_counts, pyrb_built* out);

/* gpu_build.ChunkBatch (src/gpu_build.zig:105-111): `voxels` holds `count` segments of
 * `capacity` PyrVoxels in chunk-local coordinates; segment c is filled up to
 * offsets[c+1] - offsets[c] (device u32[count+1], exclusive prefix sum), total = offsets[count]. */
typedef struct pyrb_chunk_batch {
    uint32_t count;
    uint32_t capacity;
    uint64_t voxels;
    uint64_t offsets;
    uint32_t total;
    uint32_t reserved;
} pyrb_chunk_batch;

/* gpu_build.buildChunks (src/gpu_build.zig:119-122): all chunks in one build sharing
 * node, leaf and attribute buffers (dedup across chunks per level). Host outputs
 * roots/first_voxel/first_prim (u32[count]; 0xFFFFFFFF = empty chunk). */
PYRB_API pyrb_result pyrb_build_chunks(const pyrb_exec* e, uint32_t log2_size, uint32_t rt_log2_req,
                                       const pyrb_chunk_batch* batch, uint32_t* roots, uint32_t* first_voxel,
                                       uint32_t* first_prim, pyrb_built* out);

/* World path with the pyr_world_edit overlay merged into the build
 * (replaces worldedit apply/compact/append, src/device/worldedit.zig:26-90, and the
 * buildChunks call of World.gpuWorkImpl, src/world.zig:984-1020). `counts` (device
 * u32[count]) are the generator's per-chunk counts (PyrWorldGenParams.counts);
 * `edits` (device PyrVoxel[]) hold each chunk's overlay entries in chunk-local
 * coordinates, chunk c at [edit_offsets[c], edit_offsets[c+1]) (device u32[count+1]);
 * edit_total = edit_offsets[count] (host copy, sizes the scratch).
 * Edits act as if applied after the generated voxels in list order: attribute 0
 * removes, anything else sets. Nothing is ever cut off: when a generator count
 * exceeds `capacity`, no result is kept and the call returns PYRB_ERROR_CAPACITY;
 * pyrb_last_capacity_need() then gives the largest count, so the host can grow the
 * capacity, generate again and retry, as the reference's world job does
 * (src/world.zig:968-996, growCapacity :850-879). */
PYRB_API pyrb_result pyrb_build_chunks_edits(const pyrb_exec* e, uint32_t log2_size, uint32_t rt_log2_req,
                                             uint32_t count, uint32_t capacity, uint64_t voxels, uint64_t counts,
                                             uint64_t edits, uint64_t edit_offsets, uint32_t edit_total,
                                             uint32_t* roots, uint32_t* first_voxel, uint32_t* first_prim,
                                             pyrb_built* out);

/* Batched build of many chunks of mixed edges in one pipeline run (the batched form
 * beside the reference's buildChunks, which needs one edge for all chunks). Chunk c
 * (edge 2^log2[c], log2 in [3, 10]) holds voxels[voxel_offsets[c] .. voxel_offsets[c+1])
 * in chunk-local coordinates, optionally followed by its overlay edits
 * edits[edit_offsets[c] .. edit_offsets[c+1]) (last entry wins, attribute 0 removes).
 * All chunks share one node/leaf/attribute buffer (nodes are deduplicated across
 * chunks). Keys carry the chunk number above 3 * max(log2) bits. Per chunk:
 * roots[c] (node offset of its root, 0xFFFFFFFF = empty), first_voxel[c] (first
 * attribute), first_prim[c] (first prim; prims are at edge 2^rt with
 * rt = clamp(rt_log2_req, 3, min(log2))). A chunk's voxel count is nodes[root + 1]. */
typedef struct pyrb_batch {
    uint32_t count;
    uint32_t reserved;
    const uint32_t* log2_host;   /* host u32[count] (sizes the scratch) */
    uint64_t log2;               /* device u32[count], same values */
    uint64_t voxels;             /* device PyrVoxel[voxel_total] */
    uint64_t voxel_offsets;      /* device u32[count+1] */
    uint64_t edits;              /* device PyrVoxel[edit_total] or 0 */
    uint64_t edit_offsets;       /* device u32[count+1] or 0 */
    uint32_t voxel_total;        /* host copy of voxel_offsets[count] */
    uint32_t edit_total;         /* host copy of edit_offsets[count] (0 = no edits) */
    uint64_t voxel_starts;       /* device u64[count] or 0: chunk c's voxels start at voxels[voxel_starts[c]]
                                    (its size stays voxel_offsets[c+1] - voxel_offsets[c]), so a batch can
                                    reference chunks in a resident pool without packing them */
} pyrb_batch;
PYRB_API pyrb_result pyrb_build_batch(const pyrb_exec* e, const pyrb_batch* batch, uint32_t rt_log2_req,
                                      uint32_t* roots, uint32_t* first_voxel, uint32_t* first_prim, pyrb_built* out);
/* Asynchronous form (see pyrb_build_async); roots/first_voxel/first_prim should be pinned. */
PYRB_API pyrb_result pyrb_build_batch_async(const pyrb_exec* e, const pyrb_batch* batch, uint32_t rt_log2_req,
                                            uint32_t* roots, uint32_t* first_voxel, uint32_t* first_prim,
                                            uint32_t* host_counts, pyrb_built* out);

/* gpu_build.downsample (src/gpu_build.zig:128-131): LOD of edge 2^(log2_src - shift)
 * from the sorted voxels of an editable geometry; per coarse cell the source voxel
 * with the largest key wins. shift >= 1 and shift + 3 <= log2_src. */
PYRB_API pyrb_result pyrb_downsample(const pyrb_exec* e, uint32_t log2_src, uint32_t rt_log2_req, uint64_t src_keys,
                                     uint64_t src_vals, uint32_t n_src, uint32_t shift, pyrb_built* out);

/* pyr_geometry_build's input handling (include/pyrit.h:464-466, src/context.zig:918-928):
 * like pyrb_build with n_old = 0, but with PYRB_BUILD_HOST_INPUT `voxels` is a host
 * pointer that is uploaded on the stream first. */
#define PYRB_BUILD_HOST_INPUT 0x1u
PYRB_API pyrb_result pyrb_geometry_build(const pyrb_exec* e, uint32_t log2_size, uint32_t rt_log2_req,
                                         const void* voxels, uint32_t count, uint32_t flags, pyrb_built* out);

/* Built.free (src/gpu_build.zig:42-46): frees the six output buffers (stream-ordered
 * with the default allocator) and zeroes `b`. */
PYRB_API void pyrb_built_free(const pyrb_exec* e, pyrb_built* b);

/* Copies the statistics of the calling thread's last successful build. */
PYRB_API void pyrb_last_stats(pyrb_stats* out);

/* Message of the calling thread's last error (diag.zig:17-38 / pyr_error_message). */
PYRB_API const char* pyrb_error_message(void);
PYRB_API const char* pyrb_result_string(pyrb_result r);

/* Tuning of the sort and the dedup tables (digit width 4, 8, 9, 10 or 11 bits; keys per
 * sort tile 1024, 2048 or 4096, or 8192 with 8- or 9-bit digits; both 0, the default:
 * chosen per build, 9 bits on 8192 entries where that takes one radix pass less than
 * 8 bits, else 8 bits on 4096; hash load factor in percent, 25..90) and of the way the
 * voxels are ordered (path: 0 automatic, the default -- for edges up to 2^10, a cell
 * grid in device memory for dense chunks with at most 4 cells per entry, else the radix
 * sort; 1 always the sort; 2 the grid wherever the edge allows it; 3 brick buckets, a
 * counting sort on the brick number followed by a per-brick cell grid in shared memory,
 * for edges up to 2^10 and at most 2^24 brick positions). The output never depends on
 * any of them. Applies to builds started afterwards on any thread. Returns
 * PYRB_ERROR_INVALID_ARGUMENT for unsupported values. */
typedef struct pyrb_tuning {
    uint32_t radix_bits;
    uint32_t tile_keys;
    uint32_t load_factor_pct;
    uint32_t path;
} pyrb_tuning;
PYRB_API pyrb_result pyrb_set_tuning(const pyrb_tuning* t);
PYRB_API void pyrb_get_tuning(pyrb_tuning* t);

/* Per-stage CUDA events of the calling thread's builds (off by default). After the
 * stream of the last build has synchronised, pyrb_profile_read returns the number of
 * stages and writes up to `cap` durations (ms) and NUL-terminated stage names
 * (`name_len` bytes each, e.g. "sort_pass:1", "node_build:3"). */
PYRB_API void pyrb_profile_enable(int on);
PYRB_API uint32_t pyrb_profile_read(float* ms, char* names, uint32_t name_len, uint32_t cap);

/* A plain build that allocates no device memory (no counterpart in the reference).
 * For callers that cannot allocate while they build: a render or frame loop must not
 * call cudaMalloc, which synchronises the whole device and stalls the frame, and an
 * engine whose device memory is budgeted up front has no allocator to hand over for
 * scratch. All scratch lives in a fixed 64 MiB device array inside the library (held
 * by every GPU that loads the library until the process exits); the caller passes the
 * input (device PyrVoxel[n_new]) and every output buffer (device memory) with its
 * capacity in elements. Limits: log2_size in [3, 8], n_new <= 2^20; larger requests
 * and too small outputs return PYRB_ERROR_INVALID_ARGUMENT with the sizes needed.
 * The first call on a device (with that device current) looks up the array's device
 * address with cudaGetSymbolAddress; make that first call before any stream capture.
 * The address is kept for the process (after cudaDeviceReset, load the library
 * again). All calls share the one array, which keeps the last call's contents (each
 * call clears what must start at zero): calls whose work overlaps on the GPU (other
 * streams, other threads) race and corrupt each other -- serialise them. The buffers
 * in `out` stay the caller's: never pass this pyrb_built to pyrb_built_free. Output
 * layout and values are identical to pyrb_build with n_old = 0; pyrb_last_stats
 * reports the call. Synchronises `stream` once at the end to read the counts. */
PYRB_API pyrb_result pyrb_build_noalloc(void* stream, uint32_t log2_size, uint32_t rt_log2_req, uint64_t edits,
                                        uint32_t n_new, uint64_t nodes, uint32_t node_capacity, uint64_t leaves,
                                        uint32_t leaf_capacity, uint64_t keys, uint64_t attrs,
                                        uint32_t voxel_capacity, uint64_t prims, uint64_t aabbs,
                                        uint32_t prim_capacity, pyrb_built* out);

/* PYRD v1 bytes of a built DAG: the download + save pair pyr_geometry_download /
 * pyr_dag_save (src/context.zig:1009-1031, src/root.zig:221-233, format src/io.zig:88-129).
 * Layout (little-endian): "PYRD", u32 version 1, log2_size, root, flags (bit 0:
 * attributes), u64 voxel_count (= nodes[root + 1], the root's saturated voxel count,
 * as the reference's download reads it), node_words, leaf_count, attr_count, then
 * nodes u32[], leaves u64[], attributes u32[]. Like pyr_dag_save, out == NULL only
 * sets *size; a buffer smaller than needed returns PYRB_ERROR_INVALID_ARGUMENT.
 * Copies on the exec's stream and synchronises it. */
PYRB_API pyrb_result pyrb_pyrd_save(const pyrb_exec* e, const pyrb_built* b, void* out, uint64_t* size);

/* pyr_dag_load (src/root.zig:235-244, io.load src/io.zig:131-160) onto the device: the
 * header is checked like the reference does (magic, version 1, log2_size in [3, 20],
 * sizes within `len`, root < node_words, attr_count == voxel_count when attributes are
 * present; otherwise PYRB_ERROR_INVALID_ARGUMENT "no valid DAG data"), then nodes, leaves
 * and attributes go into new device buffers of `out` (free with pyrb_built_free);
 * keys, prims and aabbs stay 0, voxel_count is the header's. */
PYRB_API pyrb_result pyrb_pyrd_load(const pyrb_exec* e, const void* data, uint64_t len, pyrb_built* out);

/* Chunk attribute palettes, the chunk-install step after a batch build
 * (src/device/palette.zig, src/context.zig:1311-1360): chunk c owns the attributes
 * attrs[first[c] .. first[c+1]) (device u32; first is a host u32[count+1], e.g. the
 * batch's first_voxel of its non-empty chunks followed by voxel_count).
 * pyrb_palette_scan: palettes (device u32[count][16]) receives up to 16 distinct
 * values per chunk in the reference's table order (64 slots, hash v * 0x9E3779B1 ^
 * h >> 15, linear probing, values inserted in order of first occurrence), padded with
 * the first value (0 for an empty chunk); counts (host u32[count]) the number of
 * distinct values, or 0xFFFFFFFF when there are more than 16 (the chunk keeps 32-bit
 * attributes). The value 0xFFFFFFFF never enters a palette (the reference's table
 * uses it as its empty marker). Synchronises the exec's stream. */
PYRB_API pyrb_result pyrb_palette_scan(const pyrb_exec* e, uint64_t attrs, const uint32_t* first, uint32_t count,
                                       uint64_t palettes, uint32_t* counts);
/* pyrb_palette_pack: writes chunk c at pool[dst[c] ..] (device u32 pool, host word
 * offsets dst[count]): for palette chunks the 16 palette words then one 4-bit index
 * per voxel (the first palette entry equal to its value), 8 per word, low nibble
 * first; for the others the attributes unchanged. The pool words of chunk c are
 * 16 + ceil(n/8) or n (context.zig:1345-1352). Synchronises the exec's stream. */
PYRB_API pyrb_result pyrb_palette_pack(const pyrb_exec* e, uint64_t attrs, const uint32_t* first, uint32_t count,
                                       uint64_t palettes, const uint32_t* counts, const uint32_t* dst, uint64_t pool);

/* Path edits (src/device/pathedit.zig; the kernel part of Context.pathEdit,
 * src/context.zig:1093-1290): set, change or remove voxels of a finished geometry
 * without rebuilding it. The brick of a change and the nodes above it are written as
 * copies into an arena above the geometry (everything else stays shared); the
 * attributes (depth-first order, 32-bit or the palette format) are rewritten from
 * attr_src into attr_a; RT prims get their new subtree node and attribute rank in
 * place, and their boxes are recomputed (with aabbs_keep they only grow, to the whole
 * cell). `nodes`, `leaves`, `attributes` are the device pools (u32, u64, u32) the
 * job offsets refer to; `edits` is a host array of n_edits {x, y, z, attribute}
 * (chunk coordinates; attribute 0 removes), job j owning [edit_first, +edit_count),
 * at most 4096 per job. Each job's edits are applied in order after a stable sort by
 * brick, as the reference's host does. The caller lays out the arenas and attribute
 * targets (node_cap >= edits * (levels * 10 + 4) + 8, leaf_cap >= edits, attr target
 * of attr_count + edits values) and keeps them from overlapping between jobs. The
 * out_* fields are written back into `jobs`: out_root, out_count (voxels after the
 * edits) and out_flags (PYRB_PATH_EDIT_*; REBUILD, EMPTY and OVERFLOW mean the job
 * must be rebuilt instead). Synchronises the exec's stream. */
#define PYRB_PATH_EDIT_REBUILD  0x1u
#define PYRB_PATH_EDIT_EMPTY    0x2u
#define PYRB_PATH_EDIT_OVERFLOW 0x4u
#define PYRB_PATH_EDIT_GREW     0x8u
typedef struct pyrb_path_edit_job {  /* the reference's PathEditJob, field for field */
    uint32_t node_offset, leaf_offset, root, log2_size;
    uint32_t attr_src, attr_count, attr_a, attr_b, attr_cap;
    uint32_t palette, pal_src, pal_dst;
    uint32_t node_arena, node_cap, leaf_arena, leaf_cap;
    uint32_t edit_first, edit_count, rt_log2, reserved0;
    uint64_t prims;                 /* device RtPrim[prim_count] (16 B: node, attr_base, cell) or 0 */
    uint32_t prim_count, reserved1;
    uint64_t aabbs;                 /* device float[prim_count][6] or 0 */
    uint32_t aabbs_keep;
    uint32_t out_root, out_count, out_attr_b, out_flags;
    uint32_t op, op_rank, op_attr;
} pyrb_path_edit_job;
PYRB_API pyrb_result pyrb_path_edit(const pyrb_exec* e, uint64_t nodes, uint64_t leaves, uint64_t attributes,
                                    pyrb_path_edit_job* jobs, uint32_t count, const uint32_t* edits,
                                    uint32_t n_edits);

/* Device memory a build would take, computed on the host without building (the upper
 * bounds the build allocates from): `entries` raw input entries (n_old + n_new for
 * pyrb_build; total for pyrb_build_chunks; count * capacity + edit_total for
 * pyrb_build_chunks_edits; voxel_total + edit_total for a batch) in `count` chunks of
 * edge 2^log2_size, or, when chunk_log2 (host u32[count]) is given, of edges
 * 2^chunk_log2[c] (a pyrb_build_batch; log2_size is ignored); rt_log2_req as the build
 * takes it (it sizes the prim outputs). Uses the current tuning.
 * scratch_bytes: freed when the build returns; output_bytes: the six output buffers.
 * The reference bounds its build scratch with a counting Exec (tests/cpu_test.zig:1559-1629). */
PYRB_API pyrb_result pyrb_build_memory(uint32_t log2_size, uint32_t rt_log2_req, uint32_t count,
                                       const uint32_t* chunk_log2, uint64_t entries, uint64_t* scratch_bytes,
                                       uint64_t* output_bytes);

/* Largest generator count of the calling thread's last PYRB_ERROR_CAPACITY result
 * (the capacity to grow to; src/world.zig:968-996), 0 if there was none. */
PYRB_API uint32_t pyrb_last_capacity_need(void);

/* Diagnostic of the device-side error path: runs one bounded wait that nothing ends
 * (which 0: the per-digit look-back of the sort passes; 1: the warp look-back of the
 * compaction kernels) on the exec's stream. The wait gives up after its poll limit
 * (about a second), sets the error word and returns, so the context stays usable; the
 * call returns what a build returns then: PYRB_ERROR_CUDA with the message "device-side
 * build error ... look-back wait limit". Synchronises the exec's stream. */
PYRB_API pyrb_result pyrb_selftest_wait_limit(const pyrb_exec* e, uint32_t which);

/* Served chunk builds: continuous batching of chunk-build requests on one GPU, the
 * served form beside the reference's streaming world job (World.gpuWorkImpl on its
 * worker thread, src/world.zig:937-1025, admission by free device memory :814-821,
 * LRU eviction of unused chunks, src/world_plan.zig:273-292). Requests name a chunk of
 * a device-resident pool of chunk voxel lists plus up to max_edits overlay edits
 * (host {x, y, z, attribute}; attribute 0 removes; the last entry of a coordinate
 * wins). A worker thread keeps up to max_inflight batches enqueued on the server's own
 * stream; whenever one completes, the requests that arrived meanwhile form the next
 * pyrb_build_batch (at most max_batch_requests and max_batch_entries voxels + edits;
 * a larger request runs alone). All scratch and results live in one device arena of
 * budget_bytes: a batch is admitted when the build's exact need (pyrb_build_memory)
 * fits, after evicting the least recently completed batches (those whose results were
 * all released first). A result stays valid until released or, when the arena is
 * full, evicted: copy out what must outlive that. Each result is bit-identical to the
 * same chunk built alone. */
typedef struct pyrb_server pyrb_server;
typedef struct pyrb_server_config {
    const uint32_t* pool_log2;    /* host u32[pool_count]: edge 2^log2 of every pool chunk, log2 in [3, 10] */
    const uint64_t* pool_starts;  /* host u64[pool_count]: first PyrVoxel of chunk c in pool_voxels */
    const uint32_t* pool_sizes;   /* host u32[pool_count]: PyrVoxels of chunk c (chunk-local coordinates) */
    uint64_t pool_voxels;         /* device PyrVoxel[]; must stay valid while the server lives */
    uint32_t pool_count;
    uint32_t rt_log2;             /* RT prim level of every build */
    uint64_t budget_bytes;        /* device arena for every batch's scratch and the results */
    uint64_t max_batch_entries;   /* voxels + edits of one batch */
    uint32_t max_batch_requests;
    uint32_t max_edits;           /* per request */
    uint32_t max_inflight;        /* batches enqueued on the GPU at once */
    uint32_t reserved;
} pyrb_server_config;
typedef struct pyrb_server_result {
    uint64_t id;                  /* the submitted id */
    int32_t status;               /* PYRB_OK, or the error of its batch */
    uint32_t root;                /* node offset of the chunk's root in batch.nodes; 0xFFFFFFFF: no voxels */
    uint32_t first_voxel;         /* its first key / attribute in batch.keys / batch.attrs */
    uint32_t first_prim;          /* its first prim in batch.prims / batch.aabbs */
    uint32_t voxel_count;
    uint32_t reserved;
    pyrb_built batch;             /* buffers of the batch that built it (shared; owned by the server) */
    double latency_ms;            /* submit -> the server saw its batch complete (host clock) */
} pyrb_server_result;
typedef struct pyrb_server_stats {
    uint64_t requests, batches, failed_batches, evictions, voxels, peak_bytes, arena_used;
    uint32_t max_batch_requests, pending, inflight, reserved;
} pyrb_server_stats;
/* Creates the server on the current device (allocates the arena and the staging
 * buffers once, starts the worker thread). */
PYRB_API pyrb_result pyrb_server_create(const pyrb_server_config* cfg, pyrb_server** out);
/* Queues a request (any thread). */
PYRB_API pyrb_result pyrb_server_submit(pyrb_server* s, uint64_t id, uint32_t chunk, const uint32_t* edits,
                                        uint32_t n_edits);
/* Copies up to `cap` finished results (in completion order) and removes them from the queue. */
PYRB_API uint32_t pyrb_server_poll(pyrb_server* s, pyrb_server_result* out, uint32_t cap);
/* The caller no longer needs result `id`; a batch is freed once all its results are released. */
PYRB_API pyrb_result pyrb_server_release(pyrb_server* s, uint64_t id);
PYRB_API void pyrb_server_get_stats(pyrb_server* s, pyrb_server_stats* out);
/* Waits (up to timeout_ms) until no request is pending or on the GPU. */
PYRB_API pyrb_result pyrb_server_drain(pyrb_server* s, uint32_t timeout_ms);
/* Stops the worker, waits for the GPU, frees everything (results included). */
PYRB_API void pyrb_server_destroy(pyrb_server* s);

/* Library version (major << 16 | minor). */
PYRB_API uint32_t pyrb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PYRIT_B200_H */
