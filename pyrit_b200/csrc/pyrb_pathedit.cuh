// Path edits (src/device/pathedit.zig): voxels of a finished geometry are set,
// changed or removed without regenerating and rebuilding it. Only the path from
// the root to a changed brick is touched: the brick and the nodes above it are
// written as copies (new mask, voxel count and reference) into an arena above the
// geometry, everything else stays shared, so the node format and traversal are
// unchanged. Attributes are in depth-first order: an inserted or removed voxel
// shifts all later ones by one. RT prims point at subtrees: their node and the
// rank of their first voxel follow the change, and their boxes are recomputed.
//
// The reference runs one CTA per job and does everything of a job in it (thread 0
// walks, all threads then move the attributes). Here the three parts are three
// kernels over all jobs at once: the walks (one warp per job, its lane 0 walks: a
// job's changes depend on each other through the root), the attribute rewrite (one
// thread per output attribute over the whole GPU) and the boxes (one thread per
// prim). Every result equals the reference's job by job.
#pragma once

#include "pyrb_device.cuh"
#include "pyrb_internal.h"

namespace pyrb {

// The reference's PathEditJob (src/device/types.zig:613-658), field for field.
struct PathEditJob {
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
};
static_assert(sizeof(PathEditJob) == 136, "PathEditJob layout");

struct RtPrim {  // types.zig:518-525
    uint32_t node, attr_base;
    uint64_t cell;
};

constexpr uint32_t kPeOpNone = 0, kPeOpSet = 1, kPeOpInsert = 2, kPeOpRemove = 3;
constexpr uint32_t kPeRebuild = 0x1, kPeEmpty = 0x2, kPeOverflow = 0x4, kPeGrew = 0x8;
constexpr uint32_t kPeMaxEdits = 4096;   // types.path_edit_max_edits
constexpr uint32_t kPeTile = 2048;       // attributes per CTA of the rewrite

struct PathEditDesc {
    uint32_t* nodes;
    uint64_t* leaves;
    uint32_t* attrs;
    PathEditJob* jobs;
    uint4* edits;                // x, y, z, attribute; rewritten by the walk to (op, rank, value, 0)
    const uint32_t* attr_tile;   // [count + 1] first attribute tile of each job
    const uint32_t* prim_tile;   // [count + 1] first prim tile of each job
    uint32_t count;
};

__device__ __forceinline__ uint32_t pe_child_index(const uint32_t v[3], uint32_t s) {
    return ((v[0] >> s) & 1) | (((v[1] >> s) & 1) << 1) | (((v[2] >> s) & 1) << 2);
}
__device__ __forceinline__ uint64_t pe_morton(uint32_t x, uint32_t y, uint32_t z) {
    return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}

struct PeWalker {
    uint32_t* nodes;
    uint64_t* leaves;
    uint32_t node_next, node_end, leaf_next, leaf_end;
    bool overflow;
    __device__ bool alloc_node(uint32_t words, uint32_t* out) {
        if (node_next + words > node_end) { overflow = true; return false; }
        *out = node_next;
        node_next += words;
        return true;
    }
    __device__ bool alloc_leaf(uint32_t* out) {
        if (leaf_next >= leaf_end) { overflow = true; return false; }
        *out = leaf_next++;
        return true;
    }
};

struct PeWalk {
    uint32_t path[kMaxLevels + 2];
    uint32_t missing;
    uint64_t brick;
    uint32_t prefix;
};

// pathedit.zig:92-128: the path to the brick holding v and the rank of its first voxel
__device__ PeWalk pe_walk(const PeWalker& w, uint32_t root, uint32_t log2, const uint32_t v[3]) {
    PeWalk r;
    r.missing = 0;
    r.brick = 0;
    r.prefix = 0;
    uint32_t node = root, s = log2 - 1;
    while (true) {
        r.path[s] = node;
        const uint32_t mask = w.nodes[node] & 0xFF;
        const uint32_t ci = pe_child_index(v, s);
        const uint32_t before = __popc(mask & ((1u << ci) - 1));
        for (uint32_t k = 0; k < before; ++k) {
            const uint32_t ref = w.nodes[node + 2 + k];
            r.prefix += s == 2 ? uint32_t(__popcll(w.leaves[ref])) : w.nodes[ref + 1];
        }
        if (!(mask & (1u << ci))) { r.missing = s; return r; }
        const uint32_t ref = w.nodes[node + 2 + before];
        if (s == 2) { r.brick = w.leaves[ref]; return r; }
        node = ref;
        --s;
    }
}

// pathedit.zig:137-193: copies of the path with the new brick; false on arena overflow
__device__ bool pe_rewrite(PeWalker& w, const PeWalk& wk, uint32_t log2, uint32_t sub_level, const uint32_t v[3],
                           uint64_t new_brick, int32_t delta, bool* has_root, uint32_t* root, bool* has_sub,
                           uint32_t* sub) {
    bool has_child = false;
    uint32_t child = 0;
    if (new_brick != 0) {
        uint32_t l;
        if (!w.alloc_leaf(&l)) return false;
        w.leaves[l] = new_brick;
        child = l;
        has_child = true;
    }
    *has_sub = false;
    for (uint32_t s = 2; s < log2; ++s) {
        const uint32_t ci = pe_child_index(v, s), cbit = 1u << ci;
        const bool exists = wk.missing == 0 || s >= wk.missing;
        uint32_t mask = 0, count = 0, refs[8], n = 0;
        if (exists) {
            const uint32_t old = wk.path[s], om = w.nodes[old] & 0xFF;
            count = w.nodes[old + 1] + uint32_t(delta);
            uint32_t slot = 0;
            for (uint32_t k = 0; k < 8; ++k) {
                const uint32_t kb = 1u << k;
                if (k == ci) {
                    if (has_child) { refs[n++] = child; mask |= kb; }
                    if (om & kb) ++slot;
                } else if (om & kb) {
                    refs[n++] = w.nodes[old + 2 + slot];
                    ++slot;
                    mask |= kb;
                }
            }
        } else if (has_child) {
            mask = cbit;
            refs[0] = child;
            n = 1;
            count = uint32_t(delta);
        }
        if (mask == 0) {
            has_child = false;
        } else {
            uint32_t nn;
            if (!w.alloc_node(2 + n, &nn)) return false;
            w.nodes[nn] = mask;
            w.nodes[nn + 1] = count;
            for (uint32_t k = 0; k < n; ++k) w.nodes[nn + 2 + k] = refs[k];
            child = nn;
            has_child = true;
        }
        if (s + 1 == sub_level) { *has_sub = has_child; *sub = child; }
    }
    *has_root = has_child;
    *root = child;
    return true;
}

// pathedit.zig:489-534: prims follow the change of the brick at v
__device__ void pe_update_prims(PeWalker& w, const PathEditJob& job, const uint32_t v[3], int32_t delta, bool has_sub,
                                uint32_t sub, uint32_t* flags) {
    if (!job.prims) return;
    const uint64_t mc = pe_morton(v[0] >> job.rt_log2, v[1] >> job.rt_log2, v[2] >> job.rt_log2);
    RtPrim* prims = reinterpret_cast<RtPrim*>(job.prims);
    bool found = false;
    for (uint32_t k = 0; k < job.prim_count; ++k) {
        const uint64_t c = prims[k].cell;
        const uint64_t mp = pe_morton(uint32_t(c & 0x1FFFFF), uint32_t((c >> 21) & 0x1FFFFF), uint32_t((c >> 42) & 0x1FFFFF));
        if (mp == mc) {
            found = true;
            if (has_sub) {
                prims[k].node = sub;
            } else {
                uint32_t en;
                if (!w.alloc_node(2, &en)) {
                    *flags |= kPeOverflow;
                } else {
                    w.nodes[en] = 0;
                    w.nodes[en + 1] = 0;
                    prims[k].node = en;
                }
            }
        } else if (mp > mc) {
            prims[k].attr_base += uint32_t(delta);
        }
    }
    if (!found && has_sub) *flags |= kPeRebuild;
}

__device__ __forceinline__ PeWalker pe_walker(const PathEditDesc& p, const PathEditJob& job) {
    PeWalker w;
    w.nodes = p.nodes + job.node_offset;
    w.leaves = p.leaves + job.leaf_offset;
    w.node_next = job.node_arena - job.node_offset;
    w.node_end = job.node_arena - job.node_offset + job.node_cap;
    w.leaf_next = job.leaf_arena - job.leaf_offset;
    w.leaf_end = job.leaf_arena - job.leaf_offset + job.leaf_cap;
    w.overflow = false;
    return w;
}

// 1. One warp per job; lane 0 walks the job's bricks in order (pathedit.zig:283-368).
__global__ void __launch_bounds__(128) k_path_walk(PathEditDesc p) {
    grid_dep_wait();
    const uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (j >= p.count || (threadIdx.x & 31) != 0) return;
    PathEditJob& job = p.jobs[j];
    PeWalker w = pe_walker(p, job);
    uint4* edits = p.edits + job.edit_first;
    const uint32_t n_edits = job.edit_count;
    uint32_t pal[16];
    uint32_t n_pal = 0;
    if (job.palette) {
        for (uint32_t q = 0; q < 16; ++q) pal[q] = p.attrs[job.pal_src + q];
        n_pal = 1;
        while (n_pal < 16 && pal[n_pal] != pal[0]) ++n_pal;
    }
    uint32_t root = job.root, flags = 0, count = job.attr_count;
    uint32_t e = 0;
    while (e < n_edits) {
        const uint4 lead = edits[e];
        const uint32_t v0[3] = {lead.x, lead.y, lead.z};
        uint32_t end = e + 1;
        for (; end < n_edits; ++end) {
            const uint4 q = edits[end];
            if ((q.x >> 2) != (v0[0] >> 2) || (q.y >> 2) != (v0[1] >> 2) || (q.z >> 2) != (v0[2] >> 2)) break;
        }
        if (flags & (kPeEmpty | kPeOverflow)) {
            for (; e < end; ++e) edits[e] = make_uint4(kPeOpNone, 0, edits[e].w, 0);
            continue;
        }
        const PeWalk wk = pe_walk(w, root, job.log2_size, v0);
        uint64_t brick = wk.brick;
        int32_t delta = 0;
        for (; e < end; ++e) {
            const uint4 q = edits[e];
            const uint32_t bit = (q.x & 3) + 4 * (q.y & 3) + 16 * (q.z & 3);
            const uint64_t bm = uint64_t(1) << bit;
            const uint32_t rank = wk.prefix + uint32_t(__popcll(brick & (bm - 1)));
            const bool has = (brick & bm) != 0;
            uint32_t val = q.w;
            if (job.palette && q.w != 0) {
                uint32_t idx = 0;
                while (idx < n_pal && pal[idx] != val) ++idx;
                if (idx == n_pal) {
                    if (n_pal == 16) {
                        flags |= kPeOverflow;
                        edits[e] = make_uint4(0, 0, 0, 0);
                        continue;
                    }
                    pal[n_pal++] = val;
                }
                val = idx;
            }
            uint32_t op = kPeOpNone;
            if (q.w != 0 && has) op = kPeOpSet;
            if (q.w != 0 && !has) { op = kPeOpInsert; brick |= bm; delta += 1; }
            if (q.w == 0 && has) { op = kPeOpRemove; brick &= ~bm; delta -= 1; }
            edits[e] = make_uint4(op, rank, val, 0);
        }
        if (brick != wk.brick) {
            bool has_root, has_sub;
            uint32_t nr = 0, sub = 0;
            if (!pe_rewrite(w, wk, job.log2_size, job.rt_log2, v0, brick, delta, &has_root, &nr, &has_sub, &sub)) {
                flags |= kPeOverflow;
                continue;
            }
            if (has_root) root = nr; else flags |= kPeEmpty;
            count = uint32_t(int32_t(count) + delta);
            pe_update_prims(w, job, v0, delta, has_sub, sub, &flags);
        }
    }
    if (w.overflow) flags |= kPeOverflow;
    if (job.palette)
        for (uint32_t q = 0; q < 16; ++q) p.attrs[job.pal_dst + q] = q < n_pal ? pal[q] : pal[0];
    job.out_root = root;
    job.out_count = count;
    job.out_attr_b = 0;
    job.out_flags = flags;
}

// Where attribute i after all operations comes from (pathedit.zig:462-485): back
// through the job's operations, each maps an index after it to one before it.
__device__ __forceinline__ bool pe_source(const uint4* ops, uint32_t n, uint32_t i, uint32_t* val, uint32_t* idx_out) {
    uint32_t idx = i;
    for (uint32_t k = n; k > 0;) {
        --k;
        const uint4 o = ops[k];
        if (o.x == kPeOpInsert) {
            if (idx == o.y) { *val = o.z; return true; }
            if (idx > o.y) --idx;
        } else if (o.x == kPeOpRemove) {
            if (idx >= o.y) ++idx;
        } else if (o.x == kPeOpSet) {
            if (idx == o.y) { *val = o.z; return true; }
        }
    }
    *idx_out = idx;
    return false;
}

__device__ __forceinline__ uint32_t pe_job_of(const uint32_t* tile_of, uint32_t count, uint32_t tile) {
    uint32_t lo = 0, hi = count + 1;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(tile_of + mid) <= tile) lo = mid; else hi = mid;
    }
    return lo;
}

// 2. Attributes of every job, kPeTile outputs per CTA (pathedit.zig:370-425). The
// job's operations are staged in shared memory; 32-bit attributes are written one
// per thread, the palette format one index word (8 attributes) per thread.
__global__ void __launch_bounds__(kBlock) k_path_attrs(PathEditDesc p) {
    grid_dep_wait();
    extern __shared__ uint4 s_ops[];  // [largest edit_count of the jobs]
    const uint32_t tile = blockIdx.x;
    if (tile >= p.attr_tile[p.count]) return;
    const uint32_t j = pe_job_of(p.attr_tile, p.count, tile);
    const PathEditJob& job = p.jobs[j];
    if (job.out_flags & kPeEmpty) return;
    const uint32_t n_ops = min(job.edit_count, kPeMaxEdits);
    for (uint32_t k = threadIdx.x; k < n_ops; k += kBlock) s_ops[k] = p.edits[job.edit_first + k];
    __syncthreads();
    const uint32_t n_final = job.out_count;
    const uint32_t t0 = (tile - p.attr_tile[j]) * kPeTile;
    if (job.palette) {
        const uint32_t words = (n_final + 7) / 8;
        for (uint32_t wd = t0 / 8 + threadIdx.x; wd < min(words, (t0 + kPeTile) / 8); wd += kBlock) {
            uint32_t word = 0;
            for (uint32_t q = 0; q < 8; ++q) {
                const uint32_t i = wd * 8 + q;
                if (i >= n_final) break;
                uint32_t val = 0, idx = 0;
                const bool found = pe_source(s_ops, n_ops, i, &val, &idx);
                const uint32_t x = found ? val : (p.attrs[job.attr_src + (idx >> 3)] >> ((idx & 7) * 4)) & 15;
                word |= x << (q * 4);
            }
            p.attrs[job.attr_a + wd] = word;
        }
    } else {
        for (uint32_t i = t0 + threadIdx.x; i < min(n_final, t0 + kPeTile); i += kBlock) {
            uint32_t val = 0, idx = 0;
            const bool found = pe_source(s_ops, n_ops, i, &val, &idx);
            p.attrs[job.attr_a + i] = found ? val : p.attrs[job.attr_src + idx];
        }
    }
}

// pathedit.zig:198-236: tight box of a subtree in its own coordinates
__device__ void pe_subtree_box(const PeWalker& w, uint32_t node, uint32_t s_top, uint32_t lo[3], uint32_t hi[3]) {
    for (int a = 0; a < 3; ++a) { lo[a] = 0xFFFFFFFFu; hi[a] = 0; }
    struct Entry { uint32_t node, s, off[3]; };
    Entry stack[64];
    uint32_t sp = 1;
    stack[0] = {node, s_top, {0, 0, 0}};
    while (sp > 0) {
        const Entry e = stack[--sp];
        const uint32_t mask = w.nodes[e.node] & 0xFF, size = 1u << e.s;
        uint32_t slot = 0;
        for (uint32_t k = 0; k < 8; ++k) {
            if (!(mask & (1u << k))) continue;
            const uint32_t ref = w.nodes[e.node + 2 + slot];
            ++slot;
            const uint32_t off[3] = {e.off[0] + (k & 1) * size, e.off[1] + ((k >> 1) & 1) * size,
                                     e.off[2] + (k >> 2) * size};
            if (e.s == 2) {
                const uint64_t brick = w.leaves[ref];
                for (uint32_t b = 0; b < 64; ++b) {
                    if (!((brick >> b) & 1)) continue;
                    const uint32_t v[3] = {off[0] + (b & 3), off[1] + ((b >> 2) & 3), off[2] + (b >> 4)};
                    for (int a = 0; a < 3; ++a) {
                        lo[a] = min(lo[a], v[a]);
                        hi[a] = max(hi[a], v[a] + 1);
                    }
                }
            } else if (sp < 64) {
                stack[sp++] = {ref, e.s - 1, {off[0], off[1], off[2]}};
            }
        }
    }
}

// 3. Boxes of every prim of every job (pathedit.zig:427-459), one thread per prim.
__global__ void __launch_bounds__(kBlock) k_path_boxes(PathEditDesc p) {
    grid_dep_wait();
    const uint32_t tile = blockIdx.x;
    if (tile >= p.prim_tile[p.count]) return;
    const uint32_t j = pe_job_of(p.prim_tile, p.count, tile);
    PathEditJob& job = p.jobs[j];
    const uint32_t k = (tile - p.prim_tile[j]) * kBlock + threadIdx.x;
    if (!job.aabbs || !job.prims || k >= job.prim_count) return;
    const PeWalker w = pe_walker(p, job);
    const RtPrim* prims = reinterpret_cast<const RtPrim*>(job.prims);
    float* box_out = reinterpret_cast<float*>(job.aabbs) + uint64_t(k) * 6;
    const uint32_t size = 1u << job.rt_log2;
    const float eps = 1.0f / 256.0f;
    const uint64_t c = prims[k].cell;
    const uint32_t cell[3] = {uint32_t(c & 0x1FFFFF), uint32_t((c >> 21) & 0x1FFFFF), uint32_t((c >> 42) & 0x1FFFFF)};
    uint32_t lo[3], hi[3];
    pe_subtree_box(w, prims[k].node, job.rt_log2 - 1, lo, hi);
    if (lo[0] > hi[0]) { lo[0] = lo[1] = lo[2] = 0; hi[0] = hi[1] = hi[2] = 0; }
    float box[6];
    for (int a = 0; a < 3; ++a) {
        const float base = float(cell[a] * size);
        box[a] = __fsub_rn(__fadd_rn(base, float(lo[a])), eps);
        box[3 + a] = __fadd_rn(__fadd_rn(base, float(hi[a])), eps);
    }
    bool grew = false;
    if (!job.aabbs_keep) {
        for (int a = 0; a < 6; ++a) box_out[a] = box[a];
        grew = true;
    } else {
        bool inside = true;
        for (int a = 0; a < 3; ++a)
            if (box[a] < box_out[a] || box[3 + a] > box_out[3 + a]) inside = false;
        if (!inside) {
            for (int a = 0; a < 3; ++a) {
                const float base = float(cell[a] * size);
                box_out[a] = __fsub_rn(base, eps);
                box_out[3 + a] = __fadd_rn(__fadd_rn(base, float(size)), eps);
            }
            grew = true;
        }
    }
    if (grew) atomicOr(&job.out_flags, kPeGrew);
}

}  // namespace pyrb
