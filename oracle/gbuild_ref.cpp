// Oracle (test infrastructure only): sequential restatement of Pyrit's GPU
// DAG-build algorithm.
//
// Follows src/device/gbuild.zig (one function per op, run(p, i) for every
// "thread" i in order) sequenced exactly like buildImpl in src/gpu_build.zig:135-360,
// executed the way CpuExec.launchCpu does (src/gpu_build.zig:406-409):
// `for i in 0..threads: run(p, i)`. Scratch is poisoned with 0xCD like
// CpuExec.alloc (src/gpu_build.zig:384-390) so reads of unwritten memory show up.
//
// The output layout (level-by-level nodes, per-level dedup, owner = minimum
// index) is the reference GPU layout that the CUDA build must reproduce byte
// for byte.
#include "oracle.h"

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>

namespace {

// Op ids: src/device/gbuild.zig:21-50
enum Op : uint32_t {
    op_encode = 0, op_radix_hist, op_radix_scatter, op_scan_local, op_scan_totals, op_scan_add,
    op_unique_flags, op_unique_scatter, op_brick_heads, op_brick_build, op_leaf_insert, op_leaf_owner,
    op_leaf_first, op_leaf_write, op_node_heads, op_node_build, op_node_insert, op_node_owner,
    op_node_first, op_node_write, op_prim_setup, op_prim_emit, op_level_advance, op_finalize,
    op_hash_clear, op_downsample, op_pack_chunks, op_chunk_first, op_roots, op_prim_start
};

// Counter slots: src/device/gbuild.zig:53-62
enum { c_unique = 0, c_children, c_parents, c_leaves, c_cursor, c_scan, c_prims, c_root, c_tmp, c_count };

constexpr uint32_t scan_segment = 256;   // gbuild.zig:64
constexpr uint32_t no_slot = 0xFFFFFFFFu; // gbuild.zig:65
constexpr uint32_t node_stride = 10;     // gbuild.zig:66

// Host mirror of types.BuildParams (src/device/types.zig:758-823) with typed pointers.
struct P {
    uint32_t op, log2_size, rt_log2, level, pass, chunk, chunks, n_old, n_new, n_total;
    uint32_t scan_len_slot, scan_len, scan_result_slot, hash_cap;
    uint32_t* counts;
    const uint32_t* edits;
    uint64_t *keys_in, *keys_out;
    uint32_t *vals_in, *vals_out;
    uint32_t* hist; uint32_t* scan_data; uint32_t* scan_totals; uint32_t* flags;
    uint64_t* ukey; uint32_t* uval; uint64_t* masks;
    uint64_t* ch_key; uint32_t* ch_ref; uint32_t* ch_count; uint64_t* ch_lo; uint64_t* ch_hi;
    uint64_t* par_key; uint32_t* par_ref; uint32_t* par_count; uint64_t* par_lo; uint64_t* par_hi;
    uint32_t* node_tmp; uint32_t* node_len; uint64_t* hash_keys; uint32_t* hash_owner; uint32_t* slot;
    uint32_t* nodes_out; uint64_t* leaves_out; uint8_t* prims_out; float* aabbs_out;
    const uint64_t* src_keys; const uint32_t* src_vals; uint32_t shift;
    uint32_t chunk_bits, chunk_count, chunk_capacity;
    const uint32_t* chunk_offsets;
    uint32_t* chunk_first; uint32_t* roots_out; uint32_t* prim_start;
};

// localBits / keyBits / radixPasses: gbuild.zig:81-92
inline uint32_t local_bits(uint32_t log2) { return 3 * (log2 - 2) + 6; }
inline uint32_t key_bits(uint32_t log2, uint32_t cb) { return local_bits(log2) + cb + 1; }
inline uint32_t radix_passes(uint32_t log2, uint32_t cb) { return (key_bits(log2, cb) + 7) / 8; }
inline uint64_t invalid_key(const P& p) { return uint64_t(1) << (key_bits(p.log2_size, p.chunk_bits) - 1); }

// spread3 / compact3: gbuild.zig:103-121 (bit i of v -> bit 3i)
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
// localKey: gbuild.zig:98-101
inline uint64_t local_key(uint32_t x, uint32_t y, uint32_t z) {
    uint64_t brick = spread3(x >> 2) | (spread3(y >> 2) << 1) | (spread3(z >> 2) << 2);
    return (brick << 6) | ((x & 3) + 4 * (y & 3) + 16 * (z & 3));
}
// hash64 (splitmix64 finaliser): gbuild.zig:123-128
inline uint64_t hash64(uint64_t v) {
    uint64_t x = v + 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
// rt.packCell / unpackCell: src/device/rt.zig:16-22 (21 bits per axis)
inline uint64_t pack_cell(uint32_t x, uint32_t y, uint32_t z) {
    return uint64_t(x) | (uint64_t(y) << 21) | (uint64_t(z) << 42);
}
inline void unpack_cell(uint64_t c, uint32_t v[3]) {
    v[0] = uint32_t(c & 0x1FFFFF); v[1] = uint32_t((c >> 21) & 0x1FFFFF); v[2] = uint32_t(c >> 42);
}
// satAdd: gbuild.zig:139-142
inline uint32_t sat_add(uint32_t a, uint32_t b) { uint32_t r = a + b; return r < a ? 0xFFFFFFFFu : r; }

inline uint32_t scan_len(const P& p) { return p.scan_len_slot == no_slot ? p.scan_len : p.counts[p.scan_len_slot]; }

// --- ops -------------------------------------------------------------------

void encode(const P& p, uint32_t i) {  // gbuild.zig:184-199
    if (i >= p.n_new) return;
    const uint32_t* v = p.edits + 4ull * i;
    int32_t n = int32_t(1u << p.log2_size);
    int32_t x = int32_t(v[0]), y = int32_t(v[1]), z = int32_t(v[2]);
    uint32_t dst = p.n_old + i;
    if (x < 0 || y < 0 || z < 0 || x >= n || y >= n || z >= n) {
        p.keys_out[dst] = invalid_key(p);
        p.vals_out[dst] = 0;
        return;
    }
    p.keys_out[dst] = local_key(uint32_t(x), uint32_t(y), uint32_t(z));
    p.vals_out[dst] = v[3];
}

void pack_chunks(const P& p, uint32_t i) {  // gbuild.zig:203-230
    if (i >= p.n_total) return;
    const uint32_t* offs = p.chunk_offsets;
    uint32_t lo = 0, hi = p.chunk_count;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) / 2;
        if (offs[mid] <= i) lo = mid; else hi = mid;
    }
    uint32_t c = lo, j = i - offs[c];
    int32_t n = int32_t(1u << p.log2_size);
    uint64_t key = invalid_key(p);
    uint32_t val = 0;
    if (j < p.chunk_capacity) {
        const uint32_t* v = p.edits + 4ull * (uint64_t(c) * p.chunk_capacity + j);
        int32_t x = int32_t(v[0]), y = int32_t(v[1]), z = int32_t(v[2]);
        if (x >= 0 && y >= 0 && z >= 0 && x < n && y < n && z < n) {
            key = (uint64_t(c) << local_bits(p.log2_size)) | local_key(uint32_t(x), uint32_t(y), uint32_t(z));
            val = v[3];
        }
    }
    p.keys_out[i] = key;
    p.vals_out[i] = val;
}

inline uint32_t chunk_of(const P& p, uint64_t key) { return uint32_t(key >> local_bits(p.log2_size)); }

void chunk_first_op(const P& p, uint32_t i) {  // gbuild.zig:237-242
    if (i >= p.counts[c_unique]) return;
    uint32_t c = chunk_of(p, p.ukey[i]);
    if (i == 0 || chunk_of(p, p.ukey[i - 1]) != c) p.chunk_first[c] = i;
}

void roots_op(const P& p, uint32_t i) {  // gbuild.zig:245-248
    if (i >= p.counts[c_parents]) return;
    p.roots_out[uint32_t(p.par_key[i])] = p.par_ref[i];
}

void prim_start_op(const P& p, uint32_t i) {  // gbuild.zig:251-257
    if (i >= p.counts[c_parents]) return;
    uint32_t shift = 3 * (p.log2_size - p.rt_log2);
    uint32_t c = uint32_t(p.par_key[i] >> shift);
    if (i == 0 || (p.par_key[i - 1] >> shift) != c) p.prim_start[c] = i;
}

void downsample_op(const P& p, uint32_t i) {  // gbuild.zig:262-274
    if (i >= p.n_new) return;
    uint64_t key = p.src_keys[i];
    uint64_t brick = key >> 6;
    uint32_t bit = uint32_t(key & 63);
    uint32_t sh = p.shift;
    uint32_t x = ((compact3(brick) << 2) | (bit & 3)) >> sh;
    uint32_t y = ((compact3(brick >> 1) << 2) | ((bit >> 2) & 3)) >> sh;
    uint32_t z = ((compact3(brick >> 2) << 2) | (bit >> 4)) >> sh;
    uint64_t nb = spread3(x >> 2) | (spread3(y >> 2) << 1) | (spread3(z >> 2) << 2);
    p.keys_out[i] = (nb << 6) | ((x & 3) + 4 * (y & 3) + 16 * (z & 3));
    p.vals_out[i] = p.src_vals[i];
}

void radix_hist(const P& p, uint32_t c) {  // gbuild.zig:277-291
    if (c >= p.chunks) return;
    uint32_t shift = 8 * p.pass;
    for (uint32_t d = 0; d < 256; ++d) p.hist[d * p.chunks + c] = 0;
    uint32_t start = c * p.chunk, end = std::min(start + p.chunk, p.n_total);
    for (uint32_t k = start; k < end; ++k) p.hist[uint32_t((p.keys_in[k] >> shift) & 0xFF) * p.chunks + c] += 1;
}

void radix_scatter(const P& p, uint32_t c) {  // gbuild.zig:294-315
    if (c >= p.chunks) return;
    uint32_t shift = 8 * p.pass;
    uint32_t offs[256];
    for (uint32_t d = 0; d < 256; ++d) offs[d] = p.hist[d * p.chunks + c];
    uint32_t start = c * p.chunk, end = std::min(start + p.chunk, p.n_total);
    for (uint32_t k = start; k < end; ++k) {
        uint32_t d = uint32_t((p.keys_in[k] >> shift) & 0xFF);
        uint32_t dst = offs[d]++;
        p.keys_out[dst] = p.keys_in[k];
        p.vals_out[dst] = p.vals_in[k];
    }
}

void scan_local(const P& p, uint32_t t) {  // gbuild.zig:321-335
    uint32_t len = scan_len(p), start = t * scan_segment;
    if (start >= len) return;
    uint32_t end = std::min(start + scan_segment, len), sum = 0;
    for (uint32_t k = start; k < end; ++k) { uint32_t v = p.scan_data[k]; p.scan_data[k] = sum; sum += v; }
    p.scan_totals[t] = sum;
}

void scan_totals(const P& p) {  // gbuild.zig:337-349
    uint32_t len = scan_len(p), segs = (len + scan_segment - 1) / scan_segment, sum = 0;
    for (uint32_t k = 0; k < segs; ++k) { uint32_t v = p.scan_totals[k]; p.scan_totals[k] = sum; sum += v; }
    p.counts[p.scan_result_slot] = sum;
}

void scan_add(const P& p, uint32_t t) {  // gbuild.zig:351-360
    uint32_t len = scan_len(p), start = t * scan_segment;
    if (start >= len || t == 0) return;
    uint32_t add = p.scan_totals[t], end = std::min(start + scan_segment, len);
    for (uint32_t k = start; k < end; ++k) p.scan_data[k] += add;
}

bool keep(const P& p, uint32_t i) {  // gbuild.zig:366-372
    uint64_t k = p.keys_in[i];
    if (k & invalid_key(p)) return false;
    if (p.vals_in[i] == 0) return false;
    return i + 1 == p.n_total || p.keys_in[i + 1] != k;
}

void unique_flags(const P& p, uint32_t i) {  // gbuild.zig:374-381
    if (i >= p.n_total) return;
    bool last = i + 1 == p.n_total || p.keys_in[i + 1] != p.keys_in[i];
    bool valid = (p.keys_in[i] & invalid_key(p)) == 0 && p.vals_in[i] != 0;
    p.flags[i] = (last && valid) ? 1u : 0u;
}

void unique_scatter(const P& p, uint32_t i) {  // gbuild.zig:383-388
    if (i >= p.n_total || !keep(p, i)) return;
    uint32_t pos = p.flags[i];
    p.ukey[pos] = p.keys_in[i];
    p.uval[pos] = p.vals_in[i];
}

inline bool is_brick_head(const uint64_t* ukey, uint32_t i) { return i == 0 || (ukey[i] >> 6) != (ukey[i - 1] >> 6); }

void brick_heads(const P& p, uint32_t i) {  // gbuild.zig:398-401
    if (i >= p.counts[c_unique]) return;
    p.flags[i] = is_brick_head(p.ukey, i) ? 1u : 0u;
}

void brick_build(const P& p, uint32_t i) {  // gbuild.zig:403-428
    uint32_t u = p.counts[c_unique];
    if (i >= u || !is_brick_head(p.ukey, i)) return;
    uint32_t b = p.flags[i];
    uint64_t brick = p.ukey[i] >> 6, mask = 0;
    uint32_t lo[3] = {4, 4, 4}, hi[3] = {0, 0, 0};
    uint32_t j = i;
    for (; j < u && (p.ukey[j] >> 6) == brick; ++j) {
        uint32_t bit = uint32_t(p.ukey[j] & 63);
        mask |= uint64_t(1) << bit;
        uint32_t v[3] = {bit & 3, (bit >> 2) & 3, bit >> 4};
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], v[a]); hi[a] = std::max(hi[a], v[a] + 1); }
    }
    p.ch_key[b] = brick;
    p.masks[b] = mask;
    p.ch_count[b] = j - i;
    p.ch_lo[b] = pack_cell(lo[0], lo[1], lo[2]);
    p.ch_hi[b] = pack_cell(hi[0], hi[1], hi[2]);
}

void hash_clear(const P& p, uint32_t i) {  // gbuild.zig:430-434
    if (i >= p.hash_cap) return;
    p.hash_keys[i] = 0;
    p.hash_owner[i] = 0xFFFFFFFFu;
}

void leaf_insert(const P& p, uint32_t i) {  // gbuild.zig:436-447 (linear probing, CAS 0 -> mask)
    if (i >= p.counts[c_children]) return;
    uint64_t mask = p.masks[i];
    uint32_t m = p.hash_cap - 1, h = uint32_t(hash64(mask) & m);
    for (;; h = (h + 1) & m) {
        uint64_t prev = p.hash_keys[h];
        if (prev == 0) { p.hash_keys[h] = mask; break; }
        if (prev == mask) break;
    }
    p.slot[i] = h;
}

void owner_op(const P& p, uint32_t i, uint32_t count_slot) {  // gbuild.zig:450-454 (atomicMin)
    if (i >= p.counts[count_slot]) return;
    uint32_t s = p.slot[i];
    p.hash_owner[s] = std::min(p.hash_owner[s], i);
}

void leaf_first(const P& p, uint32_t i) {  // gbuild.zig:456-460
    if (i >= p.counts[c_children]) return;
    p.flags[i] = p.hash_owner[p.slot[i]] == i ? 1u : 0u;
}

void leaf_write(const P& p, uint32_t i) {  // gbuild.zig:462-469
    if (i >= p.counts[c_children]) return;
    uint32_t o = p.hash_owner[p.slot[i]];
    if (o == i) p.leaves_out[p.flags[i]] = p.masks[i];
    p.ch_ref[i] = p.flags[o];
}

inline bool is_node_head(const uint64_t* key, uint32_t i) { return i == 0 || (key[i] >> 3) != (key[i - 1] >> 3); }

void node_heads(const P& p, uint32_t i) {  // gbuild.zig:479-482
    if (i >= p.counts[c_children]) return;
    p.flags[i] = is_node_head(p.ch_key, i) ? 1u : 0u;
}

void node_build(const P& p, uint32_t i) {  // gbuild.zig:484-520
    uint32_t n = p.counts[c_children];
    if (i >= n || !is_node_head(p.ch_key, i)) return;
    uint32_t par = p.flags[i];
    uint64_t parent_key = p.ch_key[i] >> 3;
    uint32_t child_size = 1u << p.level;
    uint32_t* words = p.node_tmp + uint64_t(par) * node_stride;
    uint32_t mask = 0, count = 0, k = 0;
    uint32_t lo[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, hi[3] = {0, 0, 0};
    for (uint32_t j = i; j < n && (p.ch_key[j] >> 3) == parent_key; ++j) {
        uint32_t idx = uint32_t(p.ch_key[j] & 7);
        mask |= 1u << idx;
        words[2 + k] = p.ch_ref[j];
        ++k;
        count = sat_add(count, p.ch_count[j]);
        uint32_t off[3] = {(idx & 1) * child_size, ((idx >> 1) & 1) * child_size, (idx >> 2) * child_size};
        uint32_t clo[3], chi[3];
        unpack_cell(p.ch_lo[j], clo);
        unpack_cell(p.ch_hi[j], chi);
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], clo[a] + off[a]); hi[a] = std::max(hi[a], chi[a] + off[a]); }
    }
    words[0] = mask;
    words[1] = count;
    p.node_len[par] = 2 + k;
    p.par_key[par] = parent_key;
    p.par_count[par] = count;
    p.par_lo[par] = pack_cell(lo[0], lo[1], lo[2]);
    p.par_hi[par] = pack_cell(hi[0], hi[1], hi[2]);
}

inline const uint32_t* node_words(const P& p, uint32_t i, uint32_t* len) {  // gbuild.zig:522-525
    *len = p.node_len[i];
    return p.node_tmp + uint64_t(i) * node_stride;
}

void node_insert(const P& p, uint32_t i) {  // gbuild.zig:527-550 (table holds index + 1)
    if (i >= p.counts[c_parents]) return;
    uint32_t len;
    const uint32_t* w = node_words(p, i, &len);
    uint64_t h64 = len;
    for (uint32_t k = 0; k < len; ++k) h64 = hash64(h64 ^ w[k]);
    uint32_t m = p.hash_cap - 1, h = uint32_t(h64 & m);
    for (;; h = (h + 1) & m) {
        uint64_t prev = p.hash_keys[h];
        if (prev == 0) { p.hash_keys[h] = uint64_t(i) + 1; break; }
        uint32_t other = uint32_t(prev - 1), olen;
        const uint32_t* ow = node_words(p, other, &olen);
        if (olen == len && std::memcmp(ow, w, len * 4) == 0) break;
    }
    p.slot[i] = h;
}

void node_first(const P& p, uint32_t i) {  // gbuild.zig:552-557
    if (i >= p.counts[c_parents]) return;
    bool own = p.hash_owner[p.slot[i]] == i;
    p.flags[i] = own ? p.node_len[i] : 0;
}

void node_write(const P& p, uint32_t i) {  // gbuild.zig:559-571
    if (i >= p.counts[c_parents]) return;
    uint32_t o = p.hash_owner[p.slot[i]];
    uint32_t base = p.counts[c_cursor];
    if (o == i) {
        uint32_t len;
        const uint32_t* w = node_words(p, i, &len);
        std::memcpy(p.nodes_out + base + p.flags[i], w, len * 4);
    }
    p.par_ref[i] = base + p.flags[o];
}

void prim_setup(const P& p, uint32_t i) {  // gbuild.zig:574-577
    if (i >= p.counts[c_parents]) return;
    p.flags[i] = p.par_count[i];
}

void prim_emit(const P& p, uint32_t i) {  // gbuild.zig:579-605; f32 ops in the same order, no FMA
    uint32_t n = p.counts[c_parents];
    if (i >= n) return;
    uint64_t full_key = p.par_key[i];
    uint32_t local_shift = 3 * (p.log2_size - p.rt_log2);
    uint64_t key = full_key & ((uint64_t(1) << local_shift) - 1);
    uint32_t chunk = uint32_t(full_key >> local_shift);
    uint32_t cell[3] = {compact3(key), compact3(key >> 1), compact3(key >> 2)};
    uint32_t first = p.chunk_bits > 0 ? p.chunk_first[chunk] : 0;
    uint8_t* prim = p.prims_out + 16ull * i;
    uint32_t node = p.par_ref[i], attr_base = p.flags[i] - first;
    uint64_t pc = pack_cell(cell[0], cell[1], cell[2]);
    std::memcpy(prim, &node, 4);
    std::memcpy(prim + 4, &attr_base, 4);
    std::memcpy(prim + 8, &pc, 8);
    uint32_t size = 1u << p.rt_log2;
    uint32_t lo[3], hi[3];
    unpack_cell(p.par_lo[i], lo);
    unpack_cell(p.par_hi[i], hi);
    const volatile float eps = 1.0f / 256.0f;
    float* box = p.aabbs_out + 6ull * i;
    for (int a = 0; a < 3; ++a) {
        volatile float base = float(cell[a] * size);
        volatile float l = float(lo[a]);
        volatile float h = float(hi[a]);
        volatile float s0 = base + l;
        volatile float s1 = base + h;
        box[a] = s0 - eps;
        box[3 + a] = s1 + eps;
    }
    if (i == 0) p.counts[c_prims] = n;
}

void level_advance(const P& p) {  // gbuild.zig:607-612
    uint32_t* c = p.counts;
    c[c_cursor] += c[c_scan];
    c[c_children] = c[c_parents];
    if (p.level + 1 == p.log2_size) c[c_root] = c[c_parents] > 0 ? p.par_ref[0] : 0;
}

void finalize_op(const P& p) {  // gbuild.zig:615-624
    uint32_t* c = p.counts;
    if (c[c_unique] != 0) return;
    p.nodes_out[c[c_cursor]] = 0;
    p.nodes_out[c[c_cursor] + 1] = 0;
    c[c_root] = c[c_cursor];
    c[c_cursor] += 2;
    c[c_prims] = 0;
}

void run(const P& p, uint32_t i) {  // gbuild.zig:144-178
    switch (p.op) {
        case op_encode: encode(p, i); break;
        case op_radix_hist: radix_hist(p, i); break;
        case op_radix_scatter: radix_scatter(p, i); break;
        case op_scan_local: scan_local(p, i); break;
        case op_scan_totals: if (i == 0) scan_totals(p); break;
        case op_scan_add: scan_add(p, i); break;
        case op_unique_flags: unique_flags(p, i); break;
        case op_unique_scatter: unique_scatter(p, i); break;
        case op_brick_heads: brick_heads(p, i); break;
        case op_brick_build: brick_build(p, i); break;
        case op_leaf_insert: leaf_insert(p, i); break;
        case op_leaf_owner: owner_op(p, i, c_children); break;
        case op_leaf_first: leaf_first(p, i); break;
        case op_leaf_write: leaf_write(p, i); break;
        case op_node_heads: node_heads(p, i); break;
        case op_node_build: node_build(p, i); break;
        case op_node_insert: node_insert(p, i); break;
        case op_node_owner: owner_op(p, i, c_parents); break;
        case op_node_first: node_first(p, i); break;
        case op_node_write: node_write(p, i); break;
        case op_prim_setup: prim_setup(p, i); break;
        case op_prim_emit: prim_emit(p, i); break;
        case op_level_advance: if (i == 0) level_advance(p); break;
        case op_finalize: if (i == 0) finalize_op(p); break;
        case op_hash_clear: hash_clear(p, i); break;
        case op_downsample: downsample_op(p, i); break;
        case op_pack_chunks: pack_chunks(p, i); break;
        case op_chunk_first: chunk_first_op(p, i); break;
        case op_roots: roots_op(p, i); break;
        case op_prim_start: prim_start_op(p, i); break;
        default: break;
    }
}

// --- host sequencing (src/gpu_build.zig) ------------------------------------

// Scratch list with 0xCD poisoning (CpuExec.alloc, gpu_build.zig:384-390; Scratch :55-71).
struct Scratch {
    std::vector<void*> list;
    void* get(uint64_t bytes) {
        bytes = std::max<uint64_t>(bytes, 16);
        void* p = std::malloc(bytes);
        std::memset(p, 0xCD, bytes);
        list.push_back(p);
        return p;
    }
    ~Scratch() { for (void* p : list) std::free(p); }
};
void* out_alloc(uint64_t bytes) {
    bytes = std::max<uint64_t>(bytes, 16);
    void* p = std::malloc(bytes);
    std::memset(p, 0xCD, bytes);
    return p;
}

uint32_t next_pow2(uint64_t v) {  // gpu_build.zig:49-53
    uint64_t c = 1024;
    while (c < v) c *= 2;
    return uint32_t(c);
}

void launch(P& p, uint32_t op, uint32_t threads) {  // gpu_build.zig:73-76 + CpuExec.launchCpu
    p.op = op;
    threads = std::max(threads, 1u);
    for (uint32_t i = 0; i < threads; ++i) run(p, i);
}

void scan(P& p, uint32_t* data, uint32_t len_slot, uint32_t len, uint32_t upper, uint32_t result_slot) {  // :79-88
    p.scan_data = data;
    p.scan_len_slot = len_slot;
    p.scan_len = len;
    p.scan_result_slot = result_slot;
    uint32_t segs = (upper + scan_segment - 1) / scan_segment;
    launch(p, op_scan_local, segs);
    launch(p, op_scan_totals, 1);
    launch(p, op_scan_add, segs);
}

struct Downsample { const uint64_t* keys; const uint32_t* vals; uint32_t shift; };
struct Chunks { uint32_t count, capacity; const uint32_t* offsets; uint32_t* roots; uint32_t* first_voxel; uint32_t* first_prim; };

struct Level5 { uint64_t* key; uint32_t* ref; uint32_t* count; uint64_t* lo; uint64_t* hi; };

void set_level(P& p, const Level5& c, const Level5& q) {
    p.ch_key = c.key; p.ch_ref = c.ref; p.ch_count = c.count; p.ch_lo = c.lo; p.ch_hi = c.hi;
    p.par_key = q.key; p.par_ref = q.ref; p.par_count = q.count; p.par_lo = q.lo; p.par_hi = q.hi;
}

int build_impl(uint32_t log2_size, uint32_t rt_log2_req, const uint64_t* old_keys, const uint32_t* old_vals,
               uint32_t n_old, const uint32_t* edits, uint32_t n_new, const Downsample* ds, const Chunks* chunks,
               orc_built* out) {  // gpu_build.zig:135-360
    std::memset(out, 0, sizeof(*out));
    if (log2_size < 3 || log2_size > 20) return -1;
    uint32_t n_total = n_old + n_new;
    uint32_t nmax = std::max(n_total, 1u);
    uint32_t rt_log2 = std::min(std::max(rt_log2_req, 3u), log2_size);
    uint64_t chunk_factor = chunks ? chunks->count : 1;
    auto cells_at = [&](uint32_t lv, uint64_t factor, uint32_t cap) -> uint32_t {
        uint64_t per = uint64_t(1) << (3 * (log2_size - std::min(lv, log2_size)));
        return uint32_t(std::max<uint64_t>(std::min<uint64_t>(cap, per * factor), 1));
    };
    uint32_t n_brick = cells_at(2, chunk_factor, nmax);
    uint32_t n_node = cells_at(3, chunk_factor, nmax);

    Scratch s;
    P p;
    std::memset(&p, 0, sizeof(p));
    p.log2_size = log2_size;
    p.rt_log2 = rt_log2;
    p.n_old = n_old;
    p.n_new = n_new;
    p.n_total = n_total;
    if (chunks) {
        p.chunk_count = chunks->count;
        p.chunk_capacity = chunks->capacity;
        p.chunk_offsets = chunks->offsets;
        uint32_t bits = 0;
        while ((uint64_t(1) << bits) < chunks->count) ++bits;
        p.chunk_bits = bits;
        if (key_bits(log2_size, bits) > 64) return -1;
        uint64_t k = chunks->count;
        p.chunk_first = (uint32_t*)s.get(k * 4);
        p.roots_out = (uint32_t*)s.get(k * 4);
        p.prim_start = (uint32_t*)s.get(k * 4);
        std::memset(p.chunk_first, 0xFF, k * 4);
        std::memset(p.roots_out, 0xFF, k * 4);
        std::memset(p.prim_start, 0xFF, k * 4);
    }
    p.counts = (uint32_t*)s.get(c_count * 4);
    std::memset(p.counts, 0, c_count * 4);

    // 1. keys
    uint64_t* keys[2] = {(uint64_t*)s.get(uint64_t(nmax) * 8), (uint64_t*)s.get(uint64_t(nmax) * 8)};
    uint32_t* vals[2] = {(uint32_t*)s.get(uint64_t(nmax) * 4), (uint32_t*)s.get(uint64_t(nmax) * 4)};
    if (n_old > 0) {
        std::memcpy(keys[0], old_keys, uint64_t(n_old) * 8);
        std::memcpy(vals[0], old_vals, uint64_t(n_old) * 4);
    }
    p.edits = edits;
    p.keys_out = keys[0];
    p.vals_out = vals[0];
    if (chunks) {
        if (n_new > 0) launch(p, op_pack_chunks, n_new);
    } else if (ds) {
        p.src_keys = ds->keys;
        p.src_vals = ds->vals;
        p.shift = ds->shift;
        if (n_new > 0) launch(p, op_downsample, n_new);
    } else if (n_new > 0) {
        launch(p, op_encode, n_new);
    }

    // 2. radix sort, 8 bits per pass, 128 keys per "thread" (gpu_build.zig:200-222)
    p.chunk = 128;
    p.chunks = (nmax + p.chunk - 1) / p.chunk;
    p.hist = (uint32_t*)s.get(uint64_t(p.chunks) * 256 * 4);
    p.scan_totals = (uint32_t*)s.get(uint64_t((std::max(p.chunks * 256, nmax) + scan_segment - 1) / scan_segment) * 4 + 16);
    int cur = 0;
    for (uint32_t pass = 0; pass < radix_passes(log2_size, p.chunk_bits); ++pass) {
        p.pass = pass;
        p.keys_in = keys[cur];
        p.vals_in = vals[cur];
        p.keys_out = keys[cur ^ 1];
        p.vals_out = vals[cur ^ 1];
        launch(p, op_radix_hist, p.chunks);
        scan(p, p.hist, no_slot, p.chunks * 256, p.chunks * 256, c_scan);
        launch(p, op_radix_scatter, p.chunks);
        cur ^= 1;
    }
    p.keys_in = keys[cur];
    p.vals_in = vals[cur];

    // 3. unique voxels (gpu_build.zig:224-235)
    p.flags = (uint32_t*)s.get(uint64_t(nmax) * 4);
    launch(p, op_unique_flags, n_total);
    scan(p, p.flags, no_slot, n_total, nmax, c_unique);
    uint64_t* ukey = (uint64_t*)out_alloc(uint64_t(nmax) * 8);
    uint32_t* uval = (uint32_t*)out_alloc(uint64_t(nmax) * 4);
    p.ukey = ukey;
    p.uval = uval;
    launch(p, op_unique_scatter, n_total);
    if (chunks) launch(p, op_chunk_first, nmax);

    // 4. bricks (gpu_build.zig:237-262)
    Level5 ch = {(uint64_t*)s.get(uint64_t(n_brick) * 8), (uint32_t*)s.get(uint64_t(n_brick) * 4),
                 (uint32_t*)s.get(uint64_t(n_brick) * 4), (uint64_t*)s.get(uint64_t(n_brick) * 8),
                 (uint64_t*)s.get(uint64_t(n_brick) * 8)};
    p.ch_key = ch.key; p.ch_ref = ch.ref; p.ch_count = ch.count; p.ch_lo = ch.lo; p.ch_hi = ch.hi;
    p.masks = (uint64_t*)s.get(uint64_t(n_brick) * 8);
    launch(p, op_brick_heads, nmax);
    scan(p, p.flags, c_unique, 0, nmax, c_children);
    launch(p, op_brick_build, nmax);

    // the one read-back of the brick count (gpu_build.zig:264-272)
    uint32_t n_brick_real = std::max(p.counts[c_children], 1u);
    uint32_t n_node_real = std::min(n_brick_real, n_node);
    out->brick_count = p.counts[c_children];
    Level5 par = {(uint64_t*)s.get(uint64_t(n_node_real) * 8), (uint32_t*)s.get(uint64_t(n_node_real) * 4),
                  (uint32_t*)s.get(uint64_t(n_node_real) * 4), (uint64_t*)s.get(uint64_t(n_node_real) * 8),
                  (uint64_t*)s.get(uint64_t(n_node_real) * 8)};
    set_level(p, ch, par);

    // 5. leaf dedup (gpu_build.zig:274-289), load factor <= 0.8
    p.hash_cap = next_pow2(uint64_t(n_brick_real) * 5 / 4);
    p.hash_keys = (uint64_t*)s.get(uint64_t(p.hash_cap) * 8);
    p.hash_owner = (uint32_t*)s.get(uint64_t(p.hash_cap) * 4);
    p.slot = (uint32_t*)s.get(uint64_t(n_brick_real) * 4);
    uint64_t* leaves = (uint64_t*)out_alloc(uint64_t(n_brick_real) * 8);
    p.leaves_out = leaves;
    launch(p, op_hash_clear, p.hash_cap);
    launch(p, op_leaf_insert, nmax);
    launch(p, op_leaf_owner, nmax);
    launch(p, op_leaf_first, nmax);
    scan(p, p.flags, c_children, 0, nmax, c_leaves);
    launch(p, op_leaf_write, nmax);

    // 6. node levels (gpu_build.zig:291-336)
    uint64_t word_bound = 2, prim_bound = 1;
    for (uint32_t lv = 2; lv < log2_size; ++lv) {
        uint64_t cpa = uint64_t(1) << (log2_size - lv - 1);
        uint64_t cap = std::min<uint64_t>(n_brick_real, cpa * cpa * cpa * chunk_factor);
        word_bound += cap * node_stride;
        if (lv + 1 == rt_log2) prim_bound = std::max<uint64_t>(cap, 1);
    }
    uint32_t* nodes = (uint32_t*)out_alloc(word_bound * 4);
    uint8_t* prims = (uint8_t*)out_alloc(prim_bound * 16);
    float* aabbs = (float*)out_alloc(prim_bound * 24);
    p.nodes_out = nodes;
    p.prims_out = prims;
    p.aabbs_out = aabbs;
    p.node_tmp = (uint32_t*)s.get(uint64_t(n_node_real) * node_stride * 4);
    p.node_len = (uint32_t*)s.get(uint64_t(n_node_real) * 4);

    for (uint32_t lv = 2; lv < log2_size; ++lv) {
        p.level = lv;
        set_level(p, ch, par);
        launch(p, op_node_heads, nmax);
        scan(p, p.flags, c_children, 0, nmax, c_parents);
        launch(p, op_node_build, nmax);
        launch(p, op_hash_clear, p.hash_cap);
        launch(p, op_node_insert, nmax);
        launch(p, op_node_owner, nmax);
        launch(p, op_node_first, nmax);
        scan(p, p.flags, c_parents, 0, nmax, c_scan);
        launch(p, op_node_write, nmax);
        if (lv < 24) {
            out->level_parents[lv] = p.counts[c_parents];
            // unique nodes at this level = number of owners
            uint32_t u = 0;
            for (uint32_t i = 0; i < p.counts[c_parents]; ++i) u += p.hash_owner[p.slot[i]] == i;
            out->level_unique[lv] = u;
        }
        if (lv + 1 == rt_log2) {
            launch(p, op_prim_setup, nmax);
            scan(p, p.flags, c_parents, 0, nmax, c_tmp);
            launch(p, op_prim_emit, nmax);
            if (chunks) launch(p, op_prim_start, nmax);
        }
        if (chunks && lv + 1 == log2_size) launch(p, op_roots, nmax);
        launch(p, op_level_advance, 1);
        std::swap(ch, par);
    }
    launch(p, op_finalize, 1);

    uint32_t* c = p.counts;
    if (chunks) {
        std::memcpy(chunks->roots, p.roots_out, uint64_t(chunks->count) * 4);
        std::memcpy(chunks->first_voxel, p.chunk_first, uint64_t(chunks->count) * 4);
        std::memcpy(chunks->first_prim, p.prim_start, uint64_t(chunks->count) * 4);
    }
    out->log2_size = log2_size;
    out->rt_log2 = rt_log2;
    out->nodes = nodes;
    out->node_words = c[c_cursor];
    out->root = c[c_root];
    out->leaves = leaves;
    out->leaf_count = c[c_leaves];
    out->keys = ukey;
    out->attrs = uval;
    out->voxel_count = c[c_unique];
    out->prims = prims;
    out->aabbs = aabbs;
    out->prim_count = c[c_prims];
    return 0;
}

}  // namespace

extern "C" {

int orc_gb_build(uint32_t log2_size, uint32_t rt_log2_req, const uint64_t* old_keys, const uint32_t* old_vals,
                 uint32_t n_old, const uint32_t* edits, uint32_t n_new, orc_built* out) {
    return build_impl(log2_size, rt_log2_req, old_keys, old_vals, n_old, edits, n_new, nullptr, nullptr, out);
}

int orc_gb_build_chunks(uint32_t log2_size, uint32_t rt_log2_req, uint32_t count, uint32_t capacity,
                        const uint32_t* voxels, const uint32_t* offsets, uint32_t* roots, uint32_t* first_voxel,
                        uint32_t* first_prim, orc_built* out) {
    std::memset(out, 0, sizeof(*out));
    if (count == 0 || capacity == 0) return -1;  // gpu_build.zig:120
    Chunks c{count, capacity, offsets, roots, first_voxel, first_prim};
    return build_impl(log2_size, rt_log2_req, nullptr, nullptr, 0, voxels, offsets[count], nullptr, &c, out);
}

int orc_gb_downsample(uint32_t log2_src, uint32_t rt_log2_req, const uint64_t* src_keys, const uint32_t* src_vals,
                      uint32_t n_src, uint32_t shift, orc_built* out) {
    std::memset(out, 0, sizeof(*out));
    if (shift == 0 || shift + 3 > log2_src) return -1;  // gpu_build.zig:129
    Downsample d{src_keys, src_vals, shift};
    return build_impl(log2_src - shift, rt_log2_req, nullptr, nullptr, 0, nullptr, n_src, &d, nullptr, out);
}

void orc_built_free(orc_built* b) {
    if (!b) return;
    std::free(b->nodes); std::free(b->leaves); std::free(b->keys); std::free(b->attrs);
    std::free(b->prims); std::free(b->aabbs);
    std::memset(b, 0, sizeof(*b));
}

void orc_free(void* p) { std::free(p); }

}  // extern "C"
