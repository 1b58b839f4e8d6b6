// Oracle (test infrastructure only): CPU restatement of the reference's chunk
// attribute palettes, src/device/palette.zig, as CpuExec would run them: one chunk
// after the other, the voxels of a chunk inserted in order.
//
//   scan (palette.zig:55-104): distinct values of the chunk into a 64-slot table
//        (hash v * 0x9E3779B1 ^ h >> 15, linear probing, empty = 0xFFFFFFFF); the
//        17th distinct value (or a full table) marks the chunk "overflow"
//        (count 0xFFFFFFFF); otherwise the palette is the occupied slots in slot
//        order, padded to 16 entries with its first value (0 when empty).
//   pack (palette.zig:107-152): palette chunks -> 16 palette words then 4-bit
//        indices (first palette entry equal to the value), 8 per word, low nibble
//        first; overflow chunks -> the attributes unchanged.
#include <cstdint>
#include <cstring>

#include "oracle.h"

namespace {
constexpr uint32_t kSlots = 64, kMax = 16, kEmpty = 0xFFFFFFFFu, kOverflow = 0xFFFFFFFFu;
uint32_t pal_hash(uint32_t v) {  // palette.zig:34-38
    uint32_t h = v * 0x9E3779B1u;
    h ^= h >> 15;
    return h;
}
}  // namespace

extern "C" {

void orc_palette_scan(const uint32_t* attrs, const uint32_t* first, uint32_t count, uint32_t* palettes,
                      uint32_t* counts) {
    for (uint32_t c = 0; c < count; ++c) {
        uint32_t keys[kSlots];
        for (uint32_t k = 0; k < kSlots; ++k) keys[k] = kEmpty;
        uint32_t n_ins = 0;
        bool full = false;
        for (uint32_t i = first[c]; i < first[c + 1]; ++i) {
            const uint32_t v = attrs[i];
            uint32_t s = pal_hash(v) & (kSlots - 1), probes = 0;
            for (; probes < kSlots; ++probes) {
                if (keys[s] == v) break;
                if (keys[s] == kEmpty) {
                    keys[s] = v;
                    if (n_ins++ >= kMax) full = true;
                    break;
                }
                s = (s + 1) & (kSlots - 1);
            }
            if (probes == kSlots) full = true;
        }
        uint32_t* pal = palettes + uint64_t(c) * kMax;
        if (full || n_ins > kMax) {
            counts[c] = kOverflow;
            continue;
        }
        uint32_t n = 0;
        for (uint32_t q = 0; q < kSlots; ++q)
            if (keys[q] != kEmpty) pal[n++] = keys[q];
        for (; n < kMax; ++n) pal[n] = n_ins > 0 ? pal[0] : 0u;
        counts[c] = n_ins;
    }
}

uint64_t orc_palette_words(const uint32_t* first, uint32_t count, const uint32_t* counts, uint32_t* dst) {
    // context.zig:1345-1352: palette + indices, or 32 bits per voxel
    uint64_t w = 0;
    for (uint32_t c = 0; c < count; ++c) {
        const uint64_t n = first[c + 1] - first[c];
        if (dst) dst[c] = uint32_t(w);
        w += counts[c] != kOverflow ? kMax + (n + 7) / 8 : n;
    }
    return w;
}

void orc_palette_pack(const uint32_t* attrs, const uint32_t* first, uint32_t count, const uint32_t* palettes,
                      const uint32_t* counts, const uint32_t* dst, uint32_t* pool) {
    for (uint32_t c = 0; c < count; ++c) {
        const uint32_t lo = first[c], n = first[c + 1] - lo;
        uint32_t* out = pool + dst[c];
        if (counts[c] == kOverflow) {
            std::memcpy(out, attrs + lo, uint64_t(n) * 4);
            continue;
        }
        const uint32_t* pal = palettes + uint64_t(c) * kMax;
        for (uint32_t q = 0; q < kMax; ++q) out[q] = pal[q];
        for (uint32_t w = 0; w < (n + 7) / 8; ++w) {
            uint32_t word = 0;
            for (uint32_t j = 0; j < 8 && w * 8 + j < n; ++j) {
                const uint32_t v = attrs[lo + w * 8 + j];
                uint32_t idx = 0;
                for (uint32_t q = 0; q < kMax; ++q)
                    if (pal[q] == v) { idx = q; break; }
                word |= idx << (j * 4);
            }
            out[kMax + w] = word;
        }
    }
}

}  // extern "C"
