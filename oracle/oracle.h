/* Oracle: CPU restatements of Pyrit's DAG-build algorithms.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA build in
 * pyrit_b200/. Only tests/, __graft_entry__.smoke() and the cpu_baseline leg of
 * bench.py load it; the product never links or calls it.
 *
 * Parity pinning: the reference (Zig 0.16) cannot be compiled or imported in
 * this environment, and it ships no golden files. The restatements are pinned
 * by the reference's own known-answer tests, restated in tests/test_oracle.py:
 *   src/dag_builder.zig:420-521 (morton KATs, empty, single voxel,
 *   dense == points == fn, period-8 dedup), src/rt_prims.zig:140-160 (exact
 *   prim cells, attr_base and AABBs), tests/cpu_test.zig:758-1060 (GPU
 *   algorithm vs CPU builder, edits vs rebuild, LOD vs largest key per cell,
 *   chunk batch == single build), and by agreement of the two independent
 *   restatements below (gbuild vs dag_builder) on leaves, attributes,
 *   voxel_count and the canonical node buffer.
 *
 * Three restatements:
 *   orc_gb_*   src/device/gbuild.zig ops sequenced like src/gpu_build.zig
 *              buildImpl, run one "thread" at a time like CpuExec.launchCpu
 *              (src/gpu_build.zig:366-414). Output layout = the GPU layout.
 *   orc_cpu_*  src/dag_builder.zig (streaming post-order builder with one
 *              node table shared by all levels).
 *   orc_we_*   src/device/worldedit.zig apply/compact/append.
 * plus a canonicaliser that relabels any DAG into level order.
 */
#ifndef PYRB_ORACLE_H
#define PYRB_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Result of a gbuild restatement: mirrors gpu_build.Built (src/gpu_build.zig:26-47)
 * with host arrays. Arrays are malloc'd; release with orc_built_free. */
typedef struct orc_built {
    uint32_t log2_size, rt_log2;
    uint32_t* nodes;   uint32_t node_words;  uint32_t root;
    uint64_t* leaves;  uint32_t leaf_count;
    uint64_t* keys;    uint32_t* attrs;      uint32_t voxel_count;
    uint8_t*  prims;   /* RtPrim[prim_count], 16 bytes each */
    float*    aabbs;   /* [prim_count][6] */
    uint32_t  prim_count;
    /* per-level statistics: parents (P_l) and unique nodes (U_l), l = 2..log2-1 */
    uint32_t  level_parents[24];
    uint32_t  level_unique[24];
    uint32_t  brick_count;
} orc_built;

/* gpu_build.build (src/gpu_build.zig:94-96). edits: int32/uint32 [n_new][4]. Returns 0 or -1. */
int orc_gb_build(uint32_t log2_size, uint32_t rt_log2_req, const uint64_t* old_keys, const uint32_t* old_vals,
                 uint32_t n_old, const uint32_t* edits, uint32_t n_new, orc_built* out);
/* gpu_build.buildChunks (src/gpu_build.zig:119-122). voxels: [count*capacity][4];
 * offsets: u32[count+1]. roots/first_voxel/first_prim: u32[count] outputs. */
int orc_gb_build_chunks(uint32_t log2_size, uint32_t rt_log2_req, uint32_t count, uint32_t capacity,
                        const uint32_t* voxels, const uint32_t* offsets, uint32_t* roots, uint32_t* first_voxel,
                        uint32_t* first_prim, orc_built* out);
/* gpu_build.downsample (src/gpu_build.zig:128-131). */
int orc_gb_downsample(uint32_t log2_src, uint32_t rt_log2_req, const uint64_t* src_keys, const uint32_t* src_vals,
                      uint32_t n_src, uint32_t shift, orc_built* out);
void orc_built_free(orc_built* b);

/* dag_builder.Dag (src/dag_builder.zig:18-31) with malloc'd arrays. */
typedef struct orc_dag {
    uint32_t log2_size, root;
    uint64_t voxel_count;
    uint32_t* nodes;  uint64_t node_words;
    uint64_t* leaves; uint64_t leaf_count;
    uint32_t* attrs;  uint64_t attr_count;   /* NULL when built without attributes */
} orc_dag;

/* buildPoints (src/dag_builder.zig:325-368): points int32/uint32 [n][4], every point
 * inside the volume and attribute != 0, else -1 (InvalidArgument). */
int orc_cpu_build_points(uint32_t log2_size, const uint32_t* points, uint64_t n, int store_attrs, orc_dag* out);
/* Edit overlay merged by a host hash map (last wins, attribute 0 removes), then
 * buildPoints (tests/cpu_test.zig:829-838). voxels [n][4], edits [m][4]. */
int orc_cpu_build_overlay(uint32_t log2_size, const uint32_t* voxels, uint64_t n, const uint32_t* edits, uint64_t m,
                          int store_attrs, orc_dag* out);
/* buildDense (src/dag_builder.zig:292-320): voxels[x + N*(y + N*z)], 0 = empty. */
int orc_cpu_build_dense(uint32_t log2_size, const uint32_t* voxels, int store_attrs, orc_dag* out);
/* buildFn (src/dag_builder.zig:373-412) over a dense lookup table (same octree walk). */
int orc_cpu_build_fn_dense(uint32_t log2_size, const uint32_t* voxels, int store_attrs, orc_dag* out);
void orc_dag_free(orc_dag* d);
/* Dag.lookup (src/dag_builder.zig:35-61); returns 0 for empty (attributes are != 0). */
uint32_t orc_lookup(uint32_t log2_size, const uint32_t* nodes, const uint64_t* leaves, const uint32_t* attrs,
                    uint32_t root, uint32_t x, uint32_t y, uint32_t z);
/* lookup for many points: pts [n][3] -> out[n] */
void orc_lookup_many(uint32_t log2_size, const uint32_t* nodes, const uint64_t* leaves, const uint32_t* attrs,
                     uint32_t root, const uint32_t* pts, uint64_t n, uint32_t* out);

/* Canonical level-order relabelling of a DAG reachable from `root`.
 * Level 2 nodes (children are leaves) first, then level 3, ..., root last; within a
 * level, first visit in depth-first child-index order (= Morton order of the cells).
 * Leaves keep their numbering. Writes at most cap words to out_nodes (pass NULL/0 to
 * query). Returns the canonical word count; *out_root = canonical root offset;
 * *shared_across_levels = number of node offsets reached at two or more levels
 * (the CPU builder's shared table can merge identical words across levels). */
uint64_t orc_canonicalize(uint32_t log2_size, const uint32_t* nodes, uint64_t node_words, uint32_t root,
                          uint32_t* out_nodes, uint64_t cap, uint32_t* out_root, uint64_t* shared_across_levels,
                          uint32_t* level_unique /* [24] or NULL */);

/* rt_prims.extract (src/rt_prims.zig:123-131): prims (16 B each) and aabbs [6] f32.
 * Returns the prim count; arrays malloc'd (free with orc_free). */
uint32_t orc_rt_prims_extract(const orc_dag* d, uint32_t requested_log2, uint8_t** prims, float** aabbs);

/* worldedit apply/compact/append (src/device/worldedit.zig:26-90) run sequentially.
 * voxels [count*capacity][4] (modified in place by apply), counts u32[count] in;
 * out_voxels [count*capacity][4], out_counts u32[count] out. */
void orc_we_apply_all(uint32_t count, uint32_t capacity, uint32_t* voxels, const uint32_t* counts,
                      const uint32_t* edits, const uint32_t* edit_offsets, uint32_t* out_voxels, uint32_t* out_counts);

/* PYRD v1 serialisation (src/io.zig:88-129). Returns the byte count; buf may be NULL. */
uint64_t orc_pyrd_save(uint32_t log2_size, uint32_t root, uint64_t voxel_count, const uint32_t* nodes,
                       uint64_t node_words, const uint64_t* leaves, uint64_t leaf_count, const uint32_t* attrs,
                       uint64_t attr_count, uint8_t* buf);

void orc_free(void* p);

/* Chunk attribute palettes (src/device/palette.zig), restated in palette_ref.cpp. */
void orc_palette_scan(const uint32_t* attrs, const uint32_t* first, uint32_t count, uint32_t* palettes,
                      uint32_t* counts);
uint64_t orc_palette_words(const uint32_t* first, uint32_t count, const uint32_t* counts, uint32_t* dst);
void orc_palette_pack(const uint32_t* attrs, const uint32_t* first, uint32_t count, const uint32_t* palettes,
                      const uint32_t* counts, const uint32_t* dst, uint32_t* pool);

/* Path edits (src/device/pathedit.zig), restated in pathedit_ref.cpp. The job is
 * the reference's PathEditJob (src/device/types.zig:613-658) field for field. */
typedef struct orc_rt_prim { uint32_t node, attr_base; uint64_t cell; } orc_rt_prim;
typedef struct orc_path_edit_job {
    uint32_t node_offset, leaf_offset, root, log2_size;
    uint32_t attr_src, attr_count, attr_a, attr_b, attr_cap;
    uint32_t palette, pal_src, pal_dst;
    uint32_t node_arena, node_cap, leaf_arena, leaf_cap;
    uint32_t edit_first, edit_count, rt_log2, reserved0;
    uint64_t prims;
    uint32_t prim_count, reserved1;
    uint64_t aabbs;
    uint32_t aabbs_keep;
    uint32_t out_root, out_count, out_attr_b, out_flags;
    uint32_t op, op_rank, op_attr;
} orc_path_edit_job;
void orc_path_edit_order(const orc_path_edit_job* jobs, uint32_t count, uint32_t (*edits)[4]);
void orc_path_edit(uint32_t* nodes, uint64_t* leaves, uint32_t* attrs, orc_path_edit_job* jobs, uint32_t count,
                   uint32_t (*edits)[4]);

#ifdef __cplusplus
}
#endif
#endif
