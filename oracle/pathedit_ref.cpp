// Oracle (test infrastructure only): CPU restatement of the reference's path edits,
// src/device/pathedit.zig (one job after the other, exactly as its thread 0 walks
// and its threads then rewrite the attributes and boxes), plus the host step of
// Context.pathEdit that orders each job's edits by brick (src/context.zig:1200-1211).
//
// A path edit changes voxels of a finished geometry without rebuilding it: the
// modified brick and the nodes above it are written as copies (with new mask, voxel
// count and reference) into an arena above the geometry; everything else stays
// shared. Attributes (depth-first order) are rewritten into a new buffer, RT prims
// get their new subtree node and shifted attribute rank, their boxes are recomputed.
#include <algorithm>
#include <array>
#include <cstdint>
#include <cstring>
#include <vector>

#include "oracle.h"

namespace {

constexpr uint32_t kOpNone = 0, kOpSet = 1, kOpInsert = 2, kOpRemove = 3;
constexpr uint32_t kRebuild = 0x1, kEmpty = 0x2, kOverflow = 0x4, kGrew = 0x8;
constexpr uint32_t kMaxLog2 = 20;

uint32_t bit_of(uint32_t v, uint32_t s) { return (v >> s) & 1; }
uint32_t child_index(const uint32_t v[3], uint32_t s) {
    return bit_of(v[0], s) | (bit_of(v[1], s) << 1) | (bit_of(v[2], s) << 2);
}
uint64_t morton(uint32_t x, uint32_t y, uint32_t z) {
    uint64_t m = 0;
    for (uint32_t b = 0; b < 21; ++b) {
        m |= uint64_t((x >> b) & 1) << (3 * b);
        m |= uint64_t((y >> b) & 1) << (3 * b + 1);
        m |= uint64_t((z >> b) & 1) << (3 * b + 2);
    }
    return m;
}
void unpack_cell(uint64_t c, uint32_t out[3]) {
    out[0] = uint32_t(c & 0x1FFFFF);
    out[1] = uint32_t((c >> 21) & 0x1FFFFF);
    out[2] = uint32_t((c >> 42) & 0x1FFFFF);
}
uint32_t popc32(uint32_t v) { return uint32_t(__builtin_popcount(v)); }
uint32_t popc64(uint64_t v) { return uint32_t(__builtin_popcountll(v)); }

struct Walker {  // pathedit.zig:63-89
    uint32_t* nodes;
    uint64_t* leaves;
    uint32_t node_next, node_end, leaf_next, leaf_end;
    bool overflow = false;
    bool alloc_node(uint32_t words, uint32_t* out) {
        if (node_next + words > node_end) { overflow = true; return false; }
        *out = node_next;
        node_next += words;
        return true;
    }
    bool alloc_leaf(uint32_t* out) {
        if (leaf_next >= leaf_end) { overflow = true; return false; }
        *out = leaf_next++;
        return true;
    }
};

struct Walk {  // pathedit.zig:92-128
    uint32_t path[kMaxLog2 + 1];
    uint32_t missing = 0;
    uint64_t brick = 0;
    uint32_t prefix = 0;
};

Walk walk(const Walker& w, uint32_t root, uint32_t log2, const uint32_t v[3]) {
    Walk r;
    uint32_t node = root, s = log2 - 1;
    while (true) {
        r.path[s] = node;
        const uint32_t mask = w.nodes[node] & 0xFF;
        const uint32_t ci = child_index(v, s);
        const uint32_t before = popc32(mask & ((1u << ci) - 1));
        for (uint32_t k = 0; k < before; ++k) {
            const uint32_t ref = w.nodes[node + 2 + k];
            r.prefix += s == 2 ? popc64(w.leaves[ref]) : w.nodes[ref + 1];
        }
        if (!(mask & (1u << ci))) { r.missing = s; return r; }
        const uint32_t ref = w.nodes[node + 2 + before];
        if (s == 2) { r.brick = w.leaves[ref]; return r; }
        node = ref;
        --s;
    }
}

// pathedit.zig:137-193; returns false on arena overflow
bool rewrite(Walker& w, const Walk& wk, uint32_t log2, uint32_t sub_level, const uint32_t v[3], uint64_t new_brick,
             int32_t delta, bool* has_root, uint32_t* root, bool* has_sub, uint32_t* sub) {
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
        const uint32_t ci = child_index(v, s), cbit = 1u << ci;
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

// pathedit.zig:198-236: tight box of the subtree `node` (level s_top) in its own coordinates
void subtree_box(const Walker& w, uint32_t node, uint32_t s_top, uint32_t lo[3], uint32_t hi[3]) {
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
                        lo[a] = std::min(lo[a], v[a]);
                        hi[a] = std::max(hi[a], v[a] + 1);
                    }
                }
            } else if (sp < 64) {
                stack[sp++] = {ref, e.s - 1, {off[0], off[1], off[2]}};
            }
        }
    }
}

// pathedit.zig:489-534
void update_prims(Walker& w, const orc_path_edit_job& job, const uint32_t v[3], int32_t delta, bool has_sub,
                  uint32_t sub, uint32_t* flags) {
    if (!job.prims) return;
    const uint32_t cell[3] = {v[0] >> job.rt_log2, v[1] >> job.rt_log2, v[2] >> job.rt_log2};
    const uint64_t mc = morton(cell[0], cell[1], cell[2]);
    orc_rt_prim* prims = reinterpret_cast<orc_rt_prim*>(job.prims);
    bool found = false;
    for (uint32_t k = 0; k < job.prim_count; ++k) {
        uint32_t pc[3];
        unpack_cell(prims[k].cell, pc);
        const uint64_t mp = morton(pc[0], pc[1], pc[2]);
        if (mp == mc) {
            found = true;
            if (has_sub) {
                prims[k].node = sub;
            } else {
                uint32_t en;
                if (!w.alloc_node(2, &en)) {
                    *flags |= kOverflow;
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
    if (!found && has_sub) *flags |= kRebuild;
}

struct Source { bool found; uint32_t val, idx; };
Source source_of(const uint32_t (*edits)[4], uint32_t first, uint32_t n_edits, uint32_t i) {  // pathedit.zig:462-485
    uint32_t idx = i;
    for (uint32_t k = n_edits; k > 0;) {
        --k;
        const uint32_t* o = edits[first + k];
        const uint32_t rank = o[1];
        switch (o[0]) {
            case kOpInsert:
                if (idx == rank) return {true, o[2], 0};
                if (idx > rank) --idx;
                break;
            case kOpRemove:
                if (idx >= rank) ++idx;
                break;
            case kOpSet:
                if (idx == rank) return {true, o[2], 0};
                break;
            default: break;
        }
    }
    return {false, 0, idx};
}

void run_job(uint32_t* nodes_pool, uint64_t* leaves_pool, uint32_t* attrs, orc_path_edit_job& job,
             uint32_t (*edits)[4]) {
    const uint32_t first = job.edit_first, n_edits = job.edit_count;
    Walker w;
    w.nodes = nodes_pool + job.node_offset;
    w.leaves = leaves_pool + job.leaf_offset;
    w.node_next = job.node_arena - job.node_offset;
    w.node_end = job.node_arena - job.node_offset + job.node_cap;
    w.leaf_next = job.leaf_arena - job.leaf_offset;
    w.leaf_end = job.leaf_arena - job.leaf_offset + job.leaf_cap;
    const uint32_t sub_level = job.rt_log2;

    // 0. palette
    uint32_t pal[16] = {};
    uint32_t n_pal = 0;
    if (job.palette) {
        for (uint32_t q = 0; q < 16; ++q) pal[q] = attrs[job.pal_src + q];
        n_pal = 1;
        while (n_pal < 16 && pal[n_pal] != pal[0]) ++n_pal;
    }
    // 1. tree, once per brick
    uint32_t root = job.root, flags = 0, count = job.attr_count;
    uint32_t e = 0;
    while (e < n_edits) {
        const uint32_t* lead = edits[first + e];
        const uint32_t v0[3] = {lead[0], lead[1], lead[2]};
        uint32_t end = e + 1;
        for (; end < n_edits; ++end) {
            const uint32_t* q = edits[first + end];
            if ((q[0] >> 2) != (v0[0] >> 2) || (q[1] >> 2) != (v0[1] >> 2) || (q[2] >> 2) != (v0[2] >> 2)) break;
        }
        if (flags & (kEmpty | kOverflow)) {
            for (; e < end; ++e) {
                const uint32_t a = edits[first + e][3];
                edits[first + e][0] = kOpNone; edits[first + e][1] = 0; edits[first + e][2] = a; edits[first + e][3] = 0;
            }
            continue;
        }
        const Walk wk = walk(w, root, job.log2_size, v0);
        uint64_t brick = wk.brick;
        int32_t delta = 0;
        for (; e < end; ++e) {
            uint32_t* q = edits[first + e];
            const uint32_t bit = (q[0] & 3) + 4 * (q[1] & 3) + 16 * (q[2] & 3);
            const uint64_t bm = uint64_t(1) << bit;
            const uint32_t rank = wk.prefix + popc64(brick & (bm - 1));
            const bool has = (brick & bm) != 0;
            uint32_t val = q[3];
            if (job.palette && q[3] != 0) {
                uint32_t idx = 0;
                while (idx < n_pal && pal[idx] != val) ++idx;
                if (idx == n_pal) {
                    if (n_pal == 16) {
                        flags |= kOverflow;
                        q[0] = q[1] = q[2] = q[3] = 0;
                        continue;
                    }
                    pal[n_pal++] = val;
                }
                val = idx;
            }
            uint32_t op = kOpNone;
            if (q[3] != 0 && has) op = kOpSet;
            if (q[3] != 0 && !has) { op = kOpInsert; brick |= bm; delta += 1; }
            if (q[3] == 0 && has) { op = kOpRemove; brick &= ~bm; delta -= 1; }
            q[0] = op; q[1] = rank; q[2] = val; q[3] = 0;
        }
        if (brick != wk.brick) {
            bool has_root, has_sub;
            uint32_t nr = 0, sub = 0;
            if (!rewrite(w, wk, job.log2_size, sub_level, v0, brick, delta, &has_root, &nr, &has_sub, &sub)) {
                flags |= kOverflow;
                continue;
            }
            if (has_root) root = nr; else flags |= kEmpty;
            count = uint32_t(int32_t(count) + delta);
            update_prims(w, job, v0, delta, has_sub, sub, &flags);
        }
    }
    if (w.overflow) flags |= kOverflow;
    if (job.palette)
        for (uint32_t q = 0; q < 16; ++q) attrs[job.pal_dst + q] = q < n_pal ? pal[q] : pal[0];
    job.out_root = root;
    job.out_count = count;
    job.out_attr_b = 0;
    job.out_flags = flags;

    // 2. attributes
    const uint32_t n_final = job.out_count;
    if (!(job.out_flags & kEmpty) && job.palette) {
        const uint32_t words = (n_final + 7) / 8;
        for (uint32_t wd = 0; wd < words; ++wd) {
            uint32_t word = 0;
            for (uint32_t j = 0; j < 8; ++j) {
                const uint32_t i = wd * 8 + j;
                if (i >= n_final) break;
                const Source s = source_of(edits, first, n_edits, i);
                const uint32_t idx = s.found ? s.val : (attrs[job.attr_src + (s.idx >> 3)] >> ((s.idx & 7) * 4)) & 15;
                word |= idx << (j * 4);
            }
            attrs[job.attr_a + wd] = word;
        }
    } else if (!(job.out_flags & kEmpty)) {
        // all sources are read before any target is written (the reference's threads
        // read attr_src while others write attr_a; the two never overlap)
        std::vector<uint32_t> out(n_final);
        for (uint32_t i = 0; i < n_final; ++i) {
            const Source s = source_of(edits, first, n_edits, i);
            out[i] = s.found ? s.val : attrs[job.attr_src + s.idx];
        }
        for (uint32_t i = 0; i < n_final; ++i) attrs[job.attr_a + i] = out[i];
    }

    // 3. boxes of all prims
    if (job.aabbs) {
        const orc_rt_prim* prims = reinterpret_cast<const orc_rt_prim*>(job.prims);
        float (*boxes)[6] = reinterpret_cast<float (*)[6]>(job.aabbs);
        const uint32_t size = 1u << job.rt_log2;
        const float eps = 1.0f / 256.0f;
        bool grew = false;
        for (uint32_t k = 0; k < job.prim_count; ++k) {
            uint32_t cell[3], lo[3], hi[3];
            unpack_cell(prims[k].cell, cell);
            subtree_box(w, prims[k].node, job.rt_log2 - 1, lo, hi);
            if (lo[0] > hi[0]) { lo[0] = lo[1] = lo[2] = 0; hi[0] = hi[1] = hi[2] = 0; }
            float box[6];
            for (int a = 0; a < 3; ++a) {
                const float base = float(cell[a] * size);
                box[a] = base + float(lo[a]) - eps;
                box[3 + a] = base + float(hi[a]) + eps;
            }
            if (!job.aabbs_keep) {
                std::memcpy(boxes[k], box, sizeof(box));
                grew = true;
            } else {
                bool inside = true;
                for (int a = 0; a < 3; ++a)
                    if (box[a] < boxes[k][a] || box[3 + a] > boxes[k][3 + a]) inside = false;
                if (!inside) {
                    for (int a = 0; a < 3; ++a) {
                        const float base = float(cell[a] * size);
                        boxes[k][a] = base - eps;
                        boxes[k][3 + a] = base + float(size) + eps;
                    }
                    grew = true;
                }
            }
        }
        if (grew) job.out_flags |= kGrew;
    }
}

}  // namespace

extern "C" {

void orc_path_edit_order(const orc_path_edit_job* jobs, uint32_t count, uint32_t (*edits)[4]) {
    // Context.pathEdit: per job a stable sort of its edits by brick
    for (uint32_t j = 0; j < count; ++j) {
        auto key = [](const uint32_t* a) {
            return (uint64_t(a[2] >> 2) << 42) | (uint64_t(a[1] >> 2) << 21) | uint64_t(a[0] >> 2);
        };
        std::vector<std::array<uint32_t, 4>> v(jobs[j].edit_count);
        for (uint32_t k = 0; k < jobs[j].edit_count; ++k)
            for (int c = 0; c < 4; ++c) v[k][c] = edits[jobs[j].edit_first + k][c];
        std::stable_sort(v.begin(), v.end(), [&](const std::array<uint32_t, 4>& a, const std::array<uint32_t, 4>& b) {
            return key(a.data()) < key(b.data());
        });
        for (uint32_t k = 0; k < jobs[j].edit_count; ++k)
            for (int c = 0; c < 4; ++c) edits[jobs[j].edit_first + k][c] = v[k][c];
    }
}

void orc_path_edit(uint32_t* nodes, uint64_t* leaves, uint32_t* attrs, orc_path_edit_job* jobs, uint32_t count,
                   uint32_t (*edits)[4]) {
    for (uint32_t j = 0; j < count; ++j) run_job(nodes, leaves, attrs, jobs[j], edits);
}

}  // extern "C"
