// Oracle (test infrastructure only): restatement of Pyrit's CPU DAG builder
// (src/dag_builder.zig), its lookup, rt_prims.extract (src/rt_prims.zig), the
// world edit overlay kernels (src/device/worldedit.zig) and the PYRD writer
// (src/io.zig), plus a canonical level-order relabelling used to compare node
// buffers written in different orders.
//
// Third-party arithmetic in the reference: Zig std Wyhash (dag_builder.zig:117),
// AutoHashMapUnmanaged (:177) and std.mem.sort (:342), Zig 0.16. None of them
// affects the output: the hash only places table slots (equality is a full
// word compare), and the sort uses the total order (key, input index). This
// restatement uses its own hash and std::sort on the same total order.
#include "oracle.h"

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <unordered_map>
#include <vector>

namespace {

constexpr uint32_t kMinLog2 = 3, kMaxLog2 = 20;  // dag_builder.zig:13-14

// Bit i of v -> bit 3i (dag_builder.zig:74-82) and inverse (:84-92)
uint64_t spread3(uint32_t v) {
    uint64_t x = v & 0x1FFFFFu;
    x = (x | (x << 32)) & 0x1F00000000FFFFull;
    x = (x | (x << 16)) & 0x1F0000FF0000FFull;
    x = (x | (x << 8)) & 0x100F00F00F00F00Full;
    x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}
uint32_t compact3(uint64_t v) {
    uint64_t x = v & 0x1249249249249249ull;
    x = (x | (x >> 2)) & 0x10C30C30C30C30C3ull;
    x = (x | (x >> 4)) & 0x100F00F00F00F00Full;
    x = (x | (x >> 8)) & 0x1F0000FF0000FFull;
    x = (x | (x >> 16)) & 0x1F00000000FFFFull;
    x = (x | (x >> 32)) & 0x1FFFFFull;
    return uint32_t(x);
}
inline uint64_t morton(uint32_t x, uint32_t y, uint32_t z) { return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2); }
inline uint32_t brick_bit(uint32_t lx, uint32_t ly, uint32_t lz) { return lx + 4 * ly + 16 * lz; }  // :64-66
inline uint32_t child_index(uint32_t x, uint32_t y, uint32_t z, uint32_t s) {                    // :68-71
    return ((x >> s) & 1) | (((y >> s) & 1) << 1) | (((z >> s) & 1) << 2);
}

uint64_t mix64(uint64_t x) {
    x ^= x >> 33; x *= 0xff51afd7ed558ccdull; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ull; x ^= x >> 33;
    return x;
}
uint64_t hash_words(const uint32_t* w, size_t n) {
    uint64_t h = 0x9E3779B97F4A7C15ull ^ n;
    for (size_t i = 0; i < n; ++i) h = mix64(h ^ w[i]) + i;
    return h;
}

// NodeTable (dag_builder.zig:107-155): open addressing over offsets into `nodes`,
// grown at 3/4 load, one table for all levels.
struct NodeTable {
    std::vector<uint32_t> slots;
    size_t used = 0;
    static constexpr uint32_t kEmpty = 0xFFFFFFFFu;
    static size_t node_len(const std::vector<uint32_t>& nodes, uint32_t off) { return 2 + __builtin_popcount(nodes[off] & 0xFF); }
    void grow(const std::vector<uint32_t>& nodes) {
        size_t cap = slots.empty() ? 1024 : slots.size() * 2;
        std::vector<uint32_t> ns(cap, kEmpty);
        for (uint32_t off : slots) {
            if (off == kEmpty) continue;
            size_t i = hash_words(&nodes[off], node_len(nodes, off)) & (cap - 1);
            while (ns[i] != kEmpty) i = (i + 1) & (cap - 1);
            ns[i] = off;
        }
        slots.swap(ns);
    }
    // intern (:139-154): offset of an identical node, else append `words`.
    uint32_t intern(std::vector<uint32_t>& nodes, const uint32_t* words, size_t n) {
        if ((used + 1) * 4 > slots.size() * 3) grow(nodes);
        size_t cap = slots.size();
        size_t i = hash_words(words, n) & (cap - 1);
        while (slots[i] != kEmpty) {
            uint32_t off = slots[i];
            size_t len = node_len(nodes, off);
            if (len == n && std::memcmp(&nodes[off], words, n * 4) == 0) return off;
            i = (i + 1) & (cap - 1);
        }
        uint32_t off = uint32_t(nodes.size());
        nodes.insert(nodes.end(), words, words + n);
        slots[i] = off;
        ++used;
        return off;
    }
};

struct Pending {  // dag_builder.zig:161-167
    bool valid = false;
    uint64_t key = 0;
    uint32_t mask = 0;
    uint64_t count = 0;
    uint32_t refs[8];
};

// Builder (dag_builder.zig:169-285): streaming bottom-up build from bricks in
// Morton order, one open node per level.
struct Builder {
    uint32_t log2_size;
    bool store_attrs;
    std::vector<uint32_t> nodes;
    std::vector<uint64_t> leaves;
    std::vector<uint32_t> attrs;
    NodeTable table;
    std::unordered_map<uint64_t, uint32_t> leaf_table;
    Pending pending[kMaxLog2];
    bool have_last = false;
    uint64_t last_brick = 0;
    uint64_t voxel_count = 0;
    bool bad = false;

    static void add_child(Pending& p, uint32_t idx, uint32_t ref, uint64_t count) {  // :214-220
        uint32_t pos = __builtin_popcount(p.mask);
        p.refs[pos] = ref;
        p.mask |= 1u << idx;
        p.count += count;
    }
    void finalize(uint32_t s) {  // :196-212
        Pending& p = pending[s];
        uint32_t words[10];
        uint32_t n = __builtin_popcount(p.mask);
        words[0] = p.mask;
        words[1] = uint32_t(std::min<uint64_t>(p.count, 0xFFFFFFFFull));
        std::memcpy(words + 2, p.refs, n * 4);
        uint32_t off = table.intern(nodes, words, 2 + n);
        if (s + 1 < log2_size) {
            add_child(pending[s + 1], uint32_t(p.key & 7), off, p.count);
        } else {
            pending[s].refs[0] = off;  // root
        }
        p.valid = false;
    }
    void add_brick(uint64_t m, uint64_t mask, const uint32_t* a) {  // :224-257
        if (have_last && m <= last_brick) { bad = true; return; }
        have_last = true;
        last_brick = m;
        uint32_t top = log2_size - 1;
        for (uint32_t s = 2; s <= top; ++s) {
            uint64_t key = m >> (3 * (s - 1));
            if (pending[s].valid && pending[s].key != key) finalize(s); else break;
        }
        for (uint32_t s = 2; s <= top; ++s) {
            if (!pending[s].valid) { pending[s] = Pending(); pending[s].valid = true; pending[s].key = m >> (3 * (s - 1)); }
        }
        auto it = leaf_table.find(mask);
        uint32_t li;
        if (it == leaf_table.end()) {
            li = uint32_t(leaves.size());
            leaf_table.emplace(mask, li);
            leaves.push_back(mask);
        } else {
            li = it->second;
        }
        uint32_t cnt = __builtin_popcountll(mask);
        add_child(pending[2], uint32_t(m & 7), li, cnt);
        voxel_count += cnt;
        if (store_attrs) attrs.insert(attrs.end(), a, a + cnt);
    }
    void finish(orc_dag* out) {  // :260-284
        uint32_t top = log2_size - 1;
        if (!pending[top].valid) { pending[top] = Pending(); pending[top].valid = true; pending[top].key = 0; }
        for (uint32_t s = 2; s <= top; ++s)
            if (pending[s].valid) finalize(s);
        out->log2_size = log2_size;
        out->root = pending[top].refs[0];
        out->voxel_count = voxel_count;
        out->node_words = nodes.size();
        out->nodes = (uint32_t*)std::malloc(std::max<size_t>(nodes.size(), 1) * 4);
        std::memcpy(out->nodes, nodes.data(), nodes.size() * 4);
        out->leaf_count = leaves.size();
        out->leaves = (uint64_t*)std::malloc(std::max<size_t>(leaves.size(), 1) * 8);
        std::memcpy(out->leaves, leaves.data(), leaves.size() * 8);
        if (store_attrs) {
            out->attr_count = attrs.size();
            out->attrs = (uint32_t*)std::malloc(std::max<size_t>(attrs.size(), 1) * 4);
            std::memcpy(out->attrs, attrs.data(), attrs.size() * 4);
        } else {
            out->attr_count = 0;
            out->attrs = nullptr;
        }
    }
};

struct Entry { uint64_t key; uint32_t order; uint32_t attr; };

// Octree walk of buildFn (dag_builder.zig:373-412) over a dense table.
void walk(Builder& b, const uint32_t* vox, uint32_t n, uint32_t x, uint32_t y, uint32_t z, uint32_t size) {
    if (size == 4) {
        uint32_t a[64];
        uint64_t mask = 0;
        uint32_t k = 0;
        for (uint32_t bit = 0; bit < 64; ++bit) {
            uint32_t v = vox[(x + (bit & 3)) + uint64_t(n) * ((y + ((bit >> 2) & 3)) + uint64_t(n) * (z + (bit >> 4)))];
            if (v != 0) { mask |= uint64_t(1) << bit; a[k++] = v; }
        }
        if (mask) b.add_brick(morton(x >> 2, y >> 2, z >> 2), mask, a);
        return;
    }
    uint32_t h = size / 2;
    for (uint32_t idx = 0; idx < 8; ++idx) walk(b, vox, n, x + (idx & 1) * h, y + ((idx >> 1) & 1) * h, z + (idx >> 2) * h, h);
}

}  // namespace

extern "C" {

int orc_cpu_build_points(uint32_t log2_size, const uint32_t* points, uint64_t n, int store_attrs, orc_dag* out) {
    std::memset(out, 0, sizeof(*out));
    if (log2_size < kMinLog2 || log2_size > kMaxLog2) return -1;
    Builder b;
    b.log2_size = log2_size;
    b.store_attrs = store_attrs != 0;
    int64_t nn = int64_t(1) << log2_size;
    std::vector<Entry> e(n);
    for (uint64_t i = 0; i < n; ++i) {  // :333-341
        const uint32_t* p = points + 4 * i;
        int32_t x = int32_t(p[0]), y = int32_t(p[1]), z = int32_t(p[2]);
        if (x < 0 || y < 0 || z < 0 || x >= nn || y >= nn || z >= nn || p[3] == 0) return -1;
        uint64_t brick = morton(uint32_t(x) >> 2, uint32_t(y) >> 2, uint32_t(z) >> 2);
        e[i] = {(brick << 6) | brick_bit(x & 3, y & 3, z & 3), uint32_t(i), p[3]};
    }
    std::sort(e.begin(), e.end(), [](const Entry& a, const Entry& c) {
        return a.key < c.key || (a.key == c.key && a.order < c.order);
    });
    uint32_t a[64];
    size_t i = 0;
    while (i < e.size()) {  // :348-366
        uint64_t brick = e[i].key >> 6, mask = 0;
        size_t k = 0;
        while (i < e.size() && (e[i].key >> 6) == brick) {
            uint64_t bm = uint64_t(1) << (e[i].key & 63);
            if (mask & bm) a[k - 1] = e[i].attr;  // duplicate: last wins
            else { mask |= bm; a[k++] = e[i].attr; }
            ++i;
        }
        b.add_brick(brick, mask, a);
    }
    if (b.bad) return -1;
    b.finish(out);
    return 0;
}

// Edit overlay on the CPU path: the edits are merged into the voxel list with a hash
// map (last entry wins, attribute 0 removes), then buildPoints runs on the result --
// how the reference's tests build the CPU side of an edited scene
// (tests/cpu_test.zig:829-838, tests/gpu_test.zig:686-700).
int orc_cpu_build_overlay(uint32_t log2_size, const uint32_t* voxels, uint64_t n, const uint32_t* edits, uint64_t m,
                          int store_attrs, orc_dag* out) {
    std::memset(out, 0, sizeof(*out));
    std::unordered_map<uint64_t, uint32_t> merged;
    merged.reserve(size_t((n + m) * 1.3));
    auto key = [](const uint32_t* p) { return uint64_t(p[0]) | (uint64_t(p[1]) << 21) | (uint64_t(p[2]) << 42); };
    for (uint64_t i = 0; i < n; ++i) merged[key(voxels + 4 * i)] = voxels[4 * i + 3];
    for (uint64_t i = 0; i < m; ++i) merged[key(edits + 4 * i)] = edits[4 * i + 3];
    std::vector<uint32_t> pts;
    pts.reserve(merged.size() * 4);
    for (const auto& kv : merged) {
        if (kv.second == 0) continue;
        pts.push_back(uint32_t(kv.first & 0x1FFFFF));
        pts.push_back(uint32_t((kv.first >> 21) & 0x1FFFFF));
        pts.push_back(uint32_t(kv.first >> 42));
        pts.push_back(kv.second);
    }
    return orc_cpu_build_points(log2_size, pts.data(), pts.size() / 4, store_attrs, out);
}

int orc_cpu_build_dense(uint32_t log2_size, const uint32_t* vox, int store_attrs, orc_dag* out) {  // :292-320
    std::memset(out, 0, sizeof(*out));
    if (log2_size < kMinLog2 || log2_size > kMaxLog2) return -1;
    Builder b;
    b.log2_size = log2_size;
    b.store_attrs = store_attrs != 0;
    uint64_t n = uint64_t(1) << log2_size;
    uint64_t bpa = n / 4, bc = bpa * bpa * bpa;
    uint32_t a[64];
    for (uint64_t m = 0; m < bc; ++m) {
        uint32_t c[3] = {compact3(m), compact3(m >> 1), compact3(m >> 2)};
        uint64_t mask = 0;
        uint32_t k = 0;
        for (uint32_t bit = 0; bit < 64; ++bit) {
            uint64_t x = c[0] * 4 + (bit & 3), y = c[1] * 4 + ((bit >> 2) & 3), z = c[2] * 4 + (bit >> 4);
            uint32_t v = vox[x + n * (y + n * z)];
            if (v) { mask |= uint64_t(1) << bit; a[k++] = v; }
        }
        if (mask) b.add_brick(m, mask, a);
    }
    b.finish(out);
    return 0;
}

int orc_cpu_build_fn_dense(uint32_t log2_size, const uint32_t* vox, int store_attrs, orc_dag* out) {
    std::memset(out, 0, sizeof(*out));
    if (log2_size < kMinLog2 || log2_size > kMaxLog2) return -1;
    Builder b;
    b.log2_size = log2_size;
    b.store_attrs = store_attrs != 0;
    walk(b, vox, 1u << log2_size, 0, 0, 0, 1u << log2_size);
    b.finish(out);
    return 0;
}

void orc_dag_free(orc_dag* d) {
    if (!d) return;
    std::free(d->nodes); std::free(d->leaves); std::free(d->attrs);
    std::memset(d, 0, sizeof(*d));
}

// Dag.lookup (dag_builder.zig:35-61): attribute rank from the voxel counts of the
// preceding siblings (children of 8^3 nodes are leaves: rank += popcount).
uint32_t orc_lookup(uint32_t log2_size, const uint32_t* nodes, const uint64_t* leaves, const uint32_t* attrs,
                    uint32_t root, uint32_t x, uint32_t y, uint32_t z) {
    uint32_t n = 1u << log2_size;
    if (x >= n || y >= n || z >= n) return 0;
    uint32_t node = root;
    uint64_t rank = 0;
    for (uint32_t s = log2_size - 1;; --s) {
        uint32_t mask = nodes[node] & 0xFF;
        uint32_t idx = child_index(x, y, z, s);
        if (((mask >> idx) & 1) == 0) return 0;
        uint32_t before = __builtin_popcount(mask & ((1u << idx) - 1));
        for (uint32_t k = 0; k < before; ++k) {
            uint32_t ref = nodes[node + 2 + k];
            rank += s == 2 ? uint64_t(__builtin_popcountll(leaves[ref])) : uint64_t(nodes[ref + 1]);
        }
        uint32_t child = nodes[node + 2 + before];
        if (s == 2) {
            uint64_t brick = leaves[child];
            uint32_t bit = brick_bit(x & 3, y & 3, z & 3);
            if (((brick >> bit) & 1) == 0) return 0;
            rank += __builtin_popcountll(brick & ((uint64_t(1) << bit) - 1));
            return attrs ? attrs[rank] : 1;
        }
        node = child;
    }
}

void orc_lookup_many(uint32_t log2_size, const uint32_t* nodes, const uint64_t* leaves, const uint32_t* attrs,
                     uint32_t root, const uint32_t* pts, uint64_t n, uint32_t* out) {
    for (uint64_t i = 0; i < n; ++i)
        out[i] = orc_lookup(log2_size, nodes, leaves, attrs, root, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
}

uint64_t orc_canonicalize(uint32_t log2_size, const uint32_t* nodes, uint64_t node_words, uint32_t root,
                          uint32_t* out_nodes, uint64_t cap, uint32_t* out_root, uint64_t* shared_across_levels,
                          uint32_t* level_unique) {
    (void)node_words;
    // level of a node = log2 of the child size (root level = log2_size - 1)
    uint32_t top = log2_size - 1;
    std::vector<std::vector<uint32_t>> order(top + 1);                  // per level: first-visit order of offsets
    std::vector<std::unordered_map<uint32_t, uint32_t>> index(top + 1);  // per level: offset -> canonical index
    std::unordered_map<uint32_t, uint32_t> level_of;
    uint64_t shared = 0;
    // depth-first in child-index order; visit(offset, level)
    struct Frame { uint32_t off, lv, k; };
    std::vector<Frame> st;
    auto enter = [&](uint32_t off, uint32_t lv) -> bool {
        auto& m = index[lv];
        if (m.count(off)) return false;
        m.emplace(off, uint32_t(order[lv].size()));
        order[lv].push_back(off);
        auto it = level_of.find(off);
        if (it == level_of.end()) level_of.emplace(off, lv);
        else if (it->second != lv && it->second != 0xFFFFFFFFu) { ++shared; it->second = 0xFFFFFFFFu; }
        return true;
    };
    enter(root, top);
    st.push_back({root, top, 0});
    while (!st.empty()) {
        Frame& f = st.back();
        uint32_t n = __builtin_popcount(nodes[f.off] & 0xFF);
        if (f.lv == 2 || f.k >= n) { st.pop_back(); continue; }
        uint32_t child = nodes[f.off + 2 + f.k];
        uint32_t clv = f.lv - 1;
        ++f.k;
        if (enter(child, clv)) st.push_back({child, clv, 0});
    }
    // canonical offsets: level 2 first
    std::vector<std::vector<uint32_t>> coff(top + 1);
    uint64_t w = 0;
    for (uint32_t lv = 2; lv <= top; ++lv) {
        coff[lv].resize(order[lv].size());
        for (size_t i = 0; i < order[lv].size(); ++i) {
            coff[lv][i] = uint32_t(w);
            w += 2 + __builtin_popcount(nodes[order[lv][i]] & 0xFF);
        }
        if (level_unique && lv < 24) level_unique[lv] = uint32_t(order[lv].size());
    }
    if (out_nodes && cap >= w) {
        for (uint32_t lv = 2; lv <= top; ++lv) {
            for (size_t i = 0; i < order[lv].size(); ++i) {
                uint32_t off = order[lv][i], dst = coff[lv][i];
                uint32_t n = __builtin_popcount(nodes[off] & 0xFF);
                out_nodes[dst] = nodes[off];
                out_nodes[dst + 1] = nodes[off + 1];
                for (uint32_t k = 0; k < n; ++k) {
                    uint32_t ref = nodes[off + 2 + k];
                    out_nodes[dst + 2 + k] = lv == 2 ? ref : coff[lv - 1][index[lv - 1][ref]];
                }
            }
        }
    }
    if (out_root) *out_root = coff[top].empty() ? 0 : coff[top][0];
    if (shared_across_levels) *shared_across_levels = shared;
    return w;
}

// rt_prims.extract (src/rt_prims.zig:30-131): one prim per occupied subtree of edge
// 2^k, tight voxel box, eps = 1/256, boxes cached per (node, level).
namespace {
struct Box { uint32_t mn[3], mx[3]; };
struct Extractor {
    const orc_dag* d;
    uint32_t k;
    std::unordered_map<uint64_t, Box> boxes;
    std::vector<uint8_t> prims;
    std::vector<float> aabbs;
    static Box empty() { return Box{{0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, {0, 0, 0}}; }
    static void merge(Box& a, const Box& b, const uint32_t off[3]) {
        for (int i = 0; i < 3; ++i) { a.mn[i] = std::min(a.mn[i], b.mn[i] + off[i]); a.mx[i] = std::max(a.mx[i], b.mx[i] + off[i]); }
    }
    static Box leaf_box(uint64_t mask) {
        Box b = empty();
        const uint32_t zero[3] = {0, 0, 0};
        for (uint64_t m = mask; m; m &= m - 1) {
            uint32_t bit = __builtin_ctzll(m);
            Box v{{bit & 3, (bit >> 2) & 3, bit >> 4}, {(bit & 3) + 1, ((bit >> 2) & 3) + 1, (bit >> 4) + 1}};
            merge(b, v, zero);
        }
        return b;
    }
    Box box(uint32_t node, uint32_t level) {
        uint64_t key = (uint64_t(level) << 32) | node;
        auto it = boxes.find(key);
        if (it != boxes.end()) return it->second;
        Box b = empty();
        uint32_t mask = d->nodes[node] & 0xFF, cs = 1u << (level - 1), j = 0;
        for (uint32_t idx = 0; idx < 8; ++idx) {
            if (!(mask & (1u << idx))) continue;
            uint32_t ref = d->nodes[node + 2 + j++];
            Box cb = level == 3 ? leaf_box(d->leaves[ref]) : box(ref, level - 1);
            uint32_t off[3] = {(idx & 1) * cs, ((idx >> 1) & 1) * cs, (idx >> 2) * cs};
            merge(b, cb, off);
        }
        boxes.emplace(key, b);
        return b;
    }
    void visit(uint32_t node, uint32_t level, const uint32_t origin[3], uint32_t rank) {
        if (level == k) {
            Box b = box(node, level);
            if (b.mn[0] >= b.mx[0]) return;
            uint64_t cell = uint64_t(origin[0] >> k) | (uint64_t(origin[1] >> k) << 21) | (uint64_t(origin[2] >> k) << 42);
            uint8_t rec[16];
            std::memcpy(rec, &node, 4);
            std::memcpy(rec + 4, &rank, 4);
            std::memcpy(rec + 8, &cell, 8);
            prims.insert(prims.end(), rec, rec + 16);
            const volatile float eps = 1.0f / 256.0f;
            float a[6];
            for (int i = 0; i < 3; ++i) {
                volatile float lo = float(origin[i] + b.mn[i]);
                volatile float hi = float(origin[i] + b.mx[i]);
                a[i] = lo - eps;
                a[3 + i] = hi + eps;
            }
            aabbs.insert(aabbs.end(), a, a + 6);
            return;
        }
        uint32_t mask = d->nodes[node] & 0xFF, cs = 1u << (level - 1), r = rank, j = 0;
        for (uint32_t idx = 0; idx < 8; ++idx) {
            if (!(mask & (1u << idx))) continue;
            uint32_t ref = d->nodes[node + 2 + j++];
            uint32_t o[3] = {origin[0] + (idx & 1) * cs, origin[1] + ((idx >> 1) & 1) * cs, origin[2] + (idx >> 2) * cs};
            visit(ref, level - 1, o, r);
            r += d->nodes[ref + 1];
        }
    }
};
}  // namespace

uint32_t orc_rt_prims_extract(const orc_dag* d, uint32_t requested_log2, uint8_t** prims, float** aabbs) {
    Extractor e;
    e.d = d;
    e.k = std::min(std::max(requested_log2, 3u), d->log2_size);
    const uint32_t o[3] = {0, 0, 0};
    e.visit(d->root, d->log2_size, o, 0);
    uint32_t n = uint32_t(e.prims.size() / 16);
    *prims = (uint8_t*)std::malloc(std::max<size_t>(e.prims.size(), 1));
    std::memcpy(*prims, e.prims.data(), e.prims.size());
    *aabbs = (float*)std::malloc(std::max<size_t>(e.aabbs.size(), 1) * 4);
    std::memcpy(*aabbs, e.aabbs.data(), e.aabbs.size() * 4);
    return n;
}

// worldedit.apply / compact / append (src/device/worldedit.zig:26-90), one
// "thread" at a time in index order (the GPU's atomicAdd order in compact is
// replaced by index order).
void orc_we_apply_all(uint32_t count, uint32_t capacity, uint32_t* voxels, const uint32_t* counts,
                      const uint32_t* edits, const uint32_t* edit_offsets, uint32_t* out_voxels, uint32_t* out_counts) {
    const uint32_t removed = 0xFFFFFFFFu;
    uint32_t n_edits = edit_offsets[count];
    std::vector<uint32_t> used(n_edits, 0);
    uint64_t cells = uint64_t(count) * capacity;
    for (uint64_t i = 0; i < cells; ++i) {  // apply :26-50
        uint32_t c = uint32_t(i / capacity), local = uint32_t(i % capacity);
        if (local >= counts[c]) continue;
        uint32_t* v = voxels + 4 * i;
        if (v[0] == removed) continue;
        for (uint32_t e = edit_offsets[c]; e < edit_offsets[c + 1]; ++e) {
            const uint32_t* q = edits + 4ull * e;
            if (q[0] == v[0] && q[1] == v[1] && q[2] == v[2]) {
                used[e] = 1;
                if (q[3] == 0) v[0] = removed; else v[3] = q[3];
            }
        }
    }
    std::memset(out_counts, 0, uint64_t(count) * 4);
    for (uint64_t i = 0; i < cells; ++i) {  // compact :53-67
        uint32_t c = uint32_t(i / capacity), local = uint32_t(i % capacity);
        if (local >= counts[c]) continue;
        const uint32_t* v = voxels + 4 * i;
        if (v[0] == removed) continue;
        uint32_t k = out_counts[c]++;
        if (k < capacity) std::memcpy(out_voxels + 4 * (uint64_t(c) * capacity + k), v, 16);
    }
    for (uint32_t i = 0; i < n_edits; ++i) {  // append :70-90
        if (used[i]) continue;
        const uint32_t* q = edits + 4ull * i;
        if (q[3] == 0) continue;
        uint32_t lo = 0, hi = count;
        while (lo + 1 < hi) {
            uint32_t mid = (lo + hi) / 2;
            if (edit_offsets[mid] <= i) lo = mid; else hi = mid;
        }
        uint32_t k = out_counts[lo]++;
        if (k < capacity) std::memcpy(out_voxels + 4 * (uint64_t(lo) * capacity + k), q, 16);
    }
}

// PYRD v1 (src/io.zig:88-129): "PYRD", version, log2, root, flags(bit0 attrs),
// voxel_count, node_words, leaf_count, attr_count (u64), then the arrays; little-endian.
uint64_t orc_pyrd_save(uint32_t log2_size, uint32_t root, uint64_t voxel_count, const uint32_t* nodes,
                       uint64_t node_words, const uint64_t* leaves, uint64_t leaf_count, const uint32_t* attrs,
                       uint64_t attr_count, uint8_t* buf) {
    const uint64_t header = 4 + 4 * 4 + 8 * 4;
    uint64_t na = attrs ? attr_count : 0;
    uint64_t size = header + node_words * 4 + leaf_count * 8 + na * 4;
    if (!buf) return size;
    std::memcpy(buf, "PYRD", 4);
    uint32_t h32[4] = {1, log2_size, root, attrs ? 1u : 0u};
    std::memcpy(buf + 4, h32, 16);
    uint64_t h64[4] = {voxel_count, node_words, leaf_count, na};
    std::memcpy(buf + 20, h64, 32);
    uint64_t o = header;
    std::memcpy(buf + o, nodes, node_words * 4); o += node_words * 4;
    std::memcpy(buf + o, leaves, leaf_count * 8); o += leaf_count * 8;
    if (na) std::memcpy(buf + o, attrs, na * 4);
    return size;
}

}  // extern "C"
