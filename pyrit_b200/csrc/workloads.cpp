// Seeded synthetic workloads (host side). See workloads.h for the definitions.
// Generation is split over z-slabs on all host threads; the output order is the
// scan order regardless of the thread count.
#include "workloads.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

namespace {

unsigned n_threads() {
    unsigned t = std::thread::hardware_concurrency();
    return t ? std::min(t, 64u) : 4u;
}

void parallel_for(uint32_t n, const std::function<void(uint32_t, uint32_t)>& fn) {
    unsigned t = std::min<unsigned>(n_threads(), std::max<uint32_t>(n, 1));
    std::vector<std::thread> th;
    for (unsigned k = 0; k < t; ++k) {
        uint32_t lo = uint32_t(uint64_t(n) * k / t), hi = uint32_t(uint64_t(n) * (k + 1) / t);
        th.emplace_back([=, &fn] { fn(lo, hi); });
    }
    for (auto& x : th) x.join();
}

// Generic dense generator: cell(x,y,z) -> attribute (0 = empty). Emits in scan order.
template <class F>
uint64_t emit_dense(uint32_t n, const F& cell, uint32_t* out, uint64_t cap) {
    std::vector<uint64_t> cnt(n + 1, 0);
    parallel_for(n, [&](uint32_t z0, uint32_t z1) {
        for (uint32_t z = z0; z < z1; ++z) {
            uint64_t c = 0;
            for (uint32_t y = 0; y < n; ++y)
                for (uint32_t x = 0; x < n; ++x) c += cell(x, y, z) != 0;
            cnt[z + 1] = c;
        }
    });
    for (uint32_t z = 0; z < n; ++z) cnt[z + 1] += cnt[z];
    uint64_t total = cnt[n];
    if (!out || cap < total) return total;
    parallel_for(n, [&](uint32_t z0, uint32_t z1) {
        for (uint32_t z = z0; z < z1; ++z) {
            uint32_t* o = out + 4 * cnt[z];
            for (uint32_t y = 0; y < n; ++y)
                for (uint32_t x = 0; x < n; ++x) {
                    uint32_t a = cell(x, y, z);
                    if (a) { o[0] = x; o[1] = y; o[2] = z; o[3] = a; o += 4; }
                }
        }
    });
    return total;
}

// Feistel permutation of [0, 2^(2*half)) keyed by seed; cycle-walk into [0, n).
uint64_t feistel(uint64_t v, uint32_t half, uint32_t seed) {
    uint64_t mask = (uint64_t(1) << half) - 1;
    uint64_t l = v >> half, r = v & mask;
    for (uint32_t round = 0; round < 4; ++round) {
        uint64_t f = wl_hash4(uint32_t(r), round, seed, 0xFE157E1u) & mask;
        uint64_t nl = r, nr = l ^ f;
        l = nl; r = nr;
    }
    return (l << half) | r;
}
uint64_t permute(uint64_t i, uint64_t n, uint32_t bits, uint32_t seed) {
    uint32_t half = (bits + 1) / 2;
    uint64_t v = feistel(i, half, seed);
    while (v >= n) v = feistel(v, half, seed);
    return v;
}

}  // namespace

extern "C" {

uint64_t wl_heightfield(uint32_t log2_size, uint32_t seed, uint32_t* out, uint64_t cap) {
    uint32_t n = 1u << log2_size;
    // height per column, heightfield coordinates x/32
    std::vector<int32_t> h(uint64_t(n) * n);
    parallel_for(n, [&](uint32_t z0, uint32_t z1) {
        for (uint32_t z = z0; z < z1; ++z)
            for (uint32_t x = 0; x < n; ++x)
                h[uint64_t(z) * n + x] = int32_t(wl_height_q16(int64_t(x) << 11, int64_t(z) << 11, seed) >> 16);
    });
    auto cell = [&](uint32_t x, uint32_t y, uint32_t z) -> uint32_t {
        int32_t hh = h[uint64_t(z) * n + x];
        return int32_t(y) < hh ? wl_layer_material(int32_t(y), hh) : 0u;
    };
    return emit_dense(n, cell, out, cap);
}

uint64_t wl_noise_grid(uint32_t log2_size, uint32_t seed, uint32_t* out, uint64_t cap, int32_t* threshold) {
    uint32_t n = 1u << log2_size;
    uint64_t cells = uint64_t(n) * n * n;
    std::vector<int32_t> v(cells);
    parallel_for(n, [&](uint32_t z0, uint32_t z1) {
        for (uint32_t z = z0; z < z1; ++z)
            for (uint32_t y = 0; y < n; ++y)
                for (uint32_t x = 0; x < n; ++x) v[(uint64_t(z) * n + y) * n + x] = wl_value3(x, y, z, seed);
    });
    // exact 70th percentile: value at rank floor(0.7 * cells) in ascending order
    const int32_t lo = -(1 << 17), hi = 1 << 17;
    std::vector<uint64_t> hist(uint64_t(hi - lo) + 1, 0);
    for (int32_t x : v) hist[uint64_t(std::min(std::max(x, lo), hi) - lo)]++;
    uint64_t rank = cells * 7 / 10, acc = 0;
    int32_t t = hi;
    for (uint64_t b = 0; b < hist.size(); ++b) {
        acc += hist[b];
        if (acc > rank) { t = int32_t(b) + lo; break; }
    }
    if (threshold) *threshold = t;
    auto cell = [&](uint32_t x, uint32_t y, uint32_t z) -> uint32_t {
        if (v[(uint64_t(z) * n + y) * n + x] <= t) return 0;
        return 1u + uint32_t(wl_hash4(x >> 3, y >> 3, z >> 3, seed ^ 0xB10C8u) % 8);
    };
    return emit_dense(n, cell, out, cap);
}

uint64_t wl_noise_edits(uint32_t log2_size, uint32_t seed, uint32_t* out, uint64_t cap) {
    uint32_t bits = 3 * log2_size;
    uint64_t cells = uint64_t(1) << bits;
    uint64_t count = cells / 200;  // 0.5 %
    if (!out || cap < count) return count;
    uint64_t mask = (uint64_t(1) << log2_size) - 1;
    for (uint64_t i = 0; i < count; ++i) {
        uint64_t pos = permute(i, cells, bits, seed ^ 0xED175u);
        uint64_t r = wl_hash4(uint32_t(i), uint32_t(i >> 32), seed, 0xED17u);
        uint32_t* o = out + 4 * i;
        o[0] = uint32_t(pos & mask);
        o[1] = uint32_t((pos >> log2_size) & mask);
        o[2] = uint32_t(pos >> (2 * log2_size));
        o[3] = (r & 1) ? 0u : 1u + uint32_t((r >> 8) % 8);
    }
    return count;
}

uint64_t wl_bernoulli_grid(uint32_t log2_size, uint32_t seed, uint32_t* out, uint64_t cap) {
    uint32_t n = 1u << log2_size;
    auto cell = [&](uint32_t x, uint32_t y, uint32_t z) -> uint32_t {
        uint64_t h = wl_hash4(x, y, z, seed);
        if (uint32_t(h >> 32) >= 644245094u) return 0;  // 0.15 * 2^32
        return 1u + uint32_t(uint32_t(h) % 255);
    };
    return emit_dense(n, cell, out, cap);
}

void wl_bernoulli_at(uint64_t n, const uint32_t* pts, uint32_t seed, uint32_t* out) {
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t h = wl_hash4(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], seed);
        out[i] = uint32_t(h >> 32) >= 644245094u ? 0u : 1u + uint32_t(uint32_t(h) % 255);
    }
}

uint64_t wl_uniform_edits(uint32_t log2_size, uint64_t count, uint32_t seed, uint32_t* out) {
    if (!out) return count;
    uint64_t mask = (uint64_t(1) << log2_size) - 1;
    for (uint64_t i = 0; i < count; ++i) {
        uint64_t a = wl_hash4(uint32_t(i), uint32_t(i >> 32), seed, 0xA11u);
        uint64_t b = wl_hash4(uint32_t(i), uint32_t(i >> 32), seed, 0xB22u);
        uint32_t* o = out + 4 * i;
        o[0] = uint32_t(a & mask);
        o[1] = uint32_t((a >> 21) & mask);
        o[2] = uint32_t((a >> 42) & mask);
        o[3] = (b & 1) ? 0u : 1u + uint32_t((b >> 8) % 255);
    }
    return count;
}

void wl_chunk_mix(uint32_t count, uint32_t seed, uint32_t* out_log2) {
    for (uint32_t k = 0; k < count; ++k) {
        uint32_t u = uint32_t(wl_hash4(k, seed, 0xC4u, 0x3u) % 10);
        out_log2[k] = u < 4 ? 5 : (u < 7 ? 6 : (u < 9 ? 7 : 8));
    }
}

uint64_t wl_mix_chunk(uint32_t index, uint32_t log2, uint32_t seed, uint32_t* out, uint64_t cap) {
    uint32_t e = 1u << log2;
    int64_t tx = index % 32, tz = index / 32;
    std::vector<int32_t> h(uint64_t(e) * e);
    for (uint32_t z = 0; z < e; ++z)
        for (uint32_t x = 0; x < e; ++x) {
            int64_t u = (tx << 17) + (int64_t(x) << (17 - log2)), v = (tz << 17) + (int64_t(z) << (17 - log2));
            h[uint64_t(z) * e + x] = int32_t((wl_height_q16(u, v, seed) * int64_t(e)) >> 22);
        }
    uint32_t nc = uint32_t(wl_hash4(index, seed, 0xCA7Eu, 0) % 21);
    std::vector<int32_t> cav(4 * nc);
    for (uint32_t k = 0; k < nc; ++k) {
        uint64_t a = wl_hash4(index, seed, 0xCA7Eu, k + 1);
        cav[4 * k] = int32_t(a % e);
        cav[4 * k + 1] = int32_t((a >> 16) % e);
        cav[4 * k + 2] = int32_t((a >> 32) % e);
        cav[4 * k + 3] = 3 + int32_t((a >> 48) % 10);
    }
    uint64_t c = 0;
    for (uint32_t z = 0; z < e; ++z)
        for (uint32_t y = 0; y < e; ++y)
            for (uint32_t x = 0; x < e; ++x) {
                int32_t hh = h[uint64_t(z) * e + x];
                if (int32_t(y) >= hh) continue;
                bool carved = false;
                for (uint32_t k = 0; k < nc && !carved; ++k) {
                    int32_t dx = int32_t(x) - cav[4 * k], dy = int32_t(y) - cav[4 * k + 1], dz = int32_t(z) - cav[4 * k + 2];
                    carved = dx * dx + dy * dy + dz * dz < cav[4 * k + 3] * cav[4 * k + 3];
                }
                if (carved) continue;
                if (out && c < cap) {
                    uint32_t* o = out + 4 * c;
                    o[0] = x; o[1] = y; o[2] = z; o[3] = wl_layer_material(int32_t(y), hh);
                }
                ++c;
            }
    return c;
}

uint64_t wl_chunk_edits(uint32_t log2, uint32_t n, uint32_t seed, uint32_t* out) {
    uint32_t mask = (1u << log2) - 1;
    for (uint32_t i = 0; i < n; ++i) {
        uint64_t a = wl_hash4(i, seed, 0xE0u, 1), b = wl_hash4(i, seed, 0xE0u, 2);
        uint32_t* o = out + 4ull * i;
        o[0] = uint32_t(a) & mask;
        o[1] = uint32_t(a >> 21) & mask;
        o[2] = uint32_t(a >> 42) & mask;
        o[3] = (b & 1) ? 0u : 1u + uint32_t((b >> 8) % 8);
    }
    return n;
}

uint32_t wl_attr_of(int32_t x, int32_t y, int32_t z) {  // tests/common.zig:14-19
    uint32_t h = (uint32_t(x) * 73856093u) ^ (uint32_t(y) * 19349663u) ^ (uint32_t(z) * 83492791u);
    h ^= h >> 13;
    h *= 0x5bd1e995u;
    return (h ^ (h >> 15)) | 1u;
}

void wl_scene_dense(uint32_t log2_size, uint32_t* dense) {  // tests/common.zig:24-35
    uint32_t nn = 1u << log2_size;
    volatile float n = float(nn);
    volatile float c = n * 0.5f;
    volatile float cx = c * 0.8f;
    volatile float r = n * 0.3f;
    volatile float r2 = r * r;
    for (uint32_t z = 0; z < nn; ++z)
        for (uint32_t y = 0; y < nn; ++y)
            for (uint32_t x = 0; x < nn; ++x) {
                volatile float fx = float(x), fy = float(y), fz = float(z);
                volatile float dx0 = fx + 0.5f, dy0 = fy + 0.5f, dz0 = fz + 0.5f;
                volatile float dx = dx0 - cx, dy = dy0 - c, dz = dz0 - c;
                volatile float sx = dx * dx, sy = dy * dy, sz = dz * dz;
                volatile float s1 = sx + sy;
                volatile float s = s1 + sz;
                uint32_t a = wl_attr_of(int32_t(x), int32_t(y), int32_t(z));
                bool in = s < r2;
                in = in || y < 3;
                in = in || (x % 16 == 3 && z % 16 == 5);
                in = in || a % 97 == 0;
                dense[x + uint64_t(nn) * (y + uint64_t(nn) * z)] = in ? a : 0u;
            }
}

void wl_poisson_arrivals(uint64_t n, double lambda, uint32_t seed, double* out) {
    double t = 0;
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t h = wl_hash4(uint32_t(i), uint32_t(i >> 32), seed, 0x9015u);
        double u = (double((h >> 11)) + 0.5) * (1.0 / 9007199254740992.0);
        t += -std::log(u) / lambda;
        out[i] = t;
    }
}

}  // extern "C"
