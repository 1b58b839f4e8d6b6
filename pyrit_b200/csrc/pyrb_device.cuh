// Device helpers of the DAG build: key arithmetic, status words of the
// decoupled look-back, block scans. sm_100a only.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pyrb_internal.h"

namespace pyrb {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kBlock = 256;
constexpr int kWarps = kBlock / 32;

// ---------------------------------------------------------------------------
// Key arithmetic. Same bit layout as the reference (src/device/gbuild.zig:98-121):
// key = (brick Morton << 6) | x&3 + 4(y&3) + 16(z&3), Morton interleaves x,y,z
// with x in the lowest bit. Written with PDEP-style masks of our own.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint64_t spread3(uint32_t v) {
    uint64_t x = v & 0x1FFFFFu;
    x = (x | (x << 32)) & 0x001F00000000FFFFull;
    x = (x | (x << 16)) & 0x001F0000FF0000FFull;
    x = (x | (x << 8)) & 0x100F00F00F00F00Full;
    x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}
__host__ __device__ __forceinline__ uint32_t compact3(uint64_t v) {
    uint64_t x = v & 0x1249249249249249ull;
    x = (x | (x >> 2)) & 0x10C30C30C30C30C3ull;
    x = (x | (x >> 4)) & 0x100F00F00F00F00Full;
    x = (x | (x >> 8)) & 0x001F0000FF0000FFull;
    x = (x | (x >> 16)) & 0x001F00000000FFFFull;
    x = (x | (x >> 32)) & 0x1FFFFFull;
    return uint32_t(x);
}
__host__ __device__ __forceinline__ uint64_t voxel_key(uint32_t x, uint32_t y, uint32_t z) {
    uint64_t brick = spread3(x >> 2) | (spread3(y >> 2) << 1) | (spread3(z >> 2) << 2);
    return (brick << 6) | ((x & 3) | ((y & 3) << 2) | ((z & 3) << 4));
}
// splitmix64 finaliser; only places table slots, never affects the output.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t v) {
    uint64_t x = v + 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
// rt.packCell layout (src/device/rt.zig:16-22): 21 bits per axis.
__host__ __device__ __forceinline__ uint64_t pack_cell(uint32_t x, uint32_t y, uint32_t z) {
    return uint64_t(x) | (uint64_t(y) << 21) | (uint64_t(z) << 42);
}
__host__ __device__ __forceinline__ uint32_t cell_x(uint64_t c) { return uint32_t(c & 0x1FFFFF); }
__host__ __device__ __forceinline__ uint32_t cell_y(uint64_t c) { return uint32_t((c >> 21) & 0x1FFFFF); }
__host__ __device__ __forceinline__ uint32_t cell_z(uint64_t c) { return uint32_t(c >> 42); }
__host__ __device__ __forceinline__ uint32_t sat_add(uint32_t a, uint32_t b) {
    uint32_t r = a + b;
    return r < a ? 0xFFFFFFFFu : r;
}
// Tight box of a 4^3 brick mask (min inclusive, max exclusive, per axis).
__device__ __forceinline__ void brick_box(uint64_t mask, uint64_t& lo, uint64_t& hi) {
    uint64_t zf = mask | (mask >> 32);
    uint32_t m16 = uint32_t((zf | (zf >> 16)) & 0xFFFF);       // OR over z: bits x + 4y
    uint32_t xs = (m16 | (m16 >> 8));
    xs = (xs | (xs >> 4)) & 0xF;                                 // x presence
    uint32_t ys = ((m16 & 0xF) ? 1u : 0u) | ((m16 & 0xF0) ? 2u : 0u) | ((m16 & 0xF00) ? 4u : 0u) |
                  ((m16 & 0xF000) ? 8u : 0u);
    uint32_t zs = ((mask & 0xFFFFull) ? 1u : 0u) | ((mask & 0xFFFF0000ull) ? 2u : 0u) |
                  ((mask & 0xFFFF00000000ull) ? 4u : 0u) | ((mask & 0xFFFF000000000000ull) ? 8u : 0u);
    lo = pack_cell(__ffs(xs) - 1, __ffs(ys) - 1, __ffs(zs) - 1);
    hi = pack_cell(32 - __clz(xs), 32 - __clz(ys), 32 - __clz(zs));
}

// ---------------------------------------------------------------------------
// Status words of the decoupled look-back: bits 62..63 flag, bits 0..61 value.
// ---------------------------------------------------------------------------
constexpr uint64_t kFlagAgg = 1ull << 62;
constexpr uint64_t kFlagInc = 2ull << 62;
constexpr uint64_t kValMask = (1ull << 62) - 1;
constexpr uint32_t kSpinLimit = 1u << 22;   // about a second with backoff; then error, never hang

__device__ __forceinline__ uint64_t ld_relaxed(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_relaxed32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint32_t ld_acquire32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
// Compare-and-swap with acquire-release ordering at device scope: the caller's
// earlier stores are visible to whoever observes the swapped value, and the value
// returned on failure comes with the other writer's earlier stores.
__device__ __forceinline__ uint32_t cas_acq_rel32(uint32_t* p, uint32_t cmp, uint32_t val) {
    uint32_t old;
    asm volatile("atom.acq_rel.gpu.global.cas.b32 %0, [%1], %2, %3;" : "=r"(old) : "l"(p), "r"(cmp), "r"(val) : "memory");
    return old;
}

// Look-back of one value by one thread (per digit in the sort) that inspects W
// predecessors per round: the W status loads are independent and in flight
// together. With hundreds of tiles in flight the nearest inclusive prefix is
// typically ~16 tiles back (measured at 1024^3), so a serial walk costs ~16 load
// latencies; wide windows cost status traffic (W x 8 B per digit per round) and
// registers: W = 2 measured best (1, 2, 3, 4, 8 and 16 tried). Tiles [first, tile) precede `tile`; status[first - 1]
// is never read. Returns the exclusive prefix and publishes the inclusive one; a
// predecessor that never publishes is waited for at most kSpinLimit polls, then
// err bit 0 is set.
template <int W>
__device__ __forceinline__ uint64_t lookback_window(uint64_t* status, uint32_t stride, uint32_t tile, uint32_t first,
                                                    uint64_t agg, uint32_t* err) {
    if (tile == first) {
        st_relaxed(status + uint64_t(tile) * stride, kFlagInc | agg);
        return 0;
    }
    uint64_t excl = 0;
    int64_t next = int64_t(tile) - 1;  // newest predecessor not yet added
    bool done = false;
    while (!done) {
        uint64_t s[W];
#pragma unroll
        for (int k = 0; k < W; ++k) {
            const int64_t t = next - k;
            s[k] = t >= int64_t(first) ? ld_relaxed(status + uint64_t(t) * stride) : kFlagInc;
        }
#pragma unroll
        for (int k = 0; k < W; ++k) {
            if (!done) {
                const int64_t t = next - k;
                uint64_t v = s[k];
                uint32_t spins = 0;
                while ((v >> 62) == 0) {
                    if (++spins > kSpinLimit) { atomicOr(err, kErrSpin); v = kFlagInc; break; }
                    if (spins > 8) __nanosleep(64);
                    v = ld_relaxed(status + uint64_t(t) * stride);
                }
                excl += v & kValMask;
                if ((v >> 62) == 2 || t == int64_t(first)) done = true;
            }
        }
        next -= W;
    }
    st_relaxed(status + uint64_t(tile) * stride, kFlagInc | (excl + agg));
    return excl;
}

// Warp-parallel look-back of a scalar (called by all 32 lanes of one warp; the
// aggregate must already be published with kFlagAgg unless tile == first).
// Each step inspects 32 predecessors at once.
__device__ __forceinline__ uint64_t lookback_warp(uint64_t* status, uint32_t tile, uint32_t first, uint64_t agg,
                                                  uint32_t* err) {
    const unsigned lane = threadIdx.x & 31;
    if (tile == first) {
        if (lane == 0) st_relaxed(status + tile, kFlagInc | agg);
        return 0;
    }
    uint64_t excl = 0;
    int64_t base = int64_t(tile) - 1;
    uint32_t spins = 0;
    while (true) {
        int64_t t = base - lane;
        uint64_t s = t >= int64_t(first) ? ld_relaxed(status + t) : kFlagInc;
        while (__any_sync(kFull, (s >> 62) == 0)) {
            if (++spins > kSpinLimit) {
                if ((s >> 62) == 0) { atomicOr(err, kErrSpin); s = kFlagInc; }
                break;
            }
            if (spins > 8) __nanosleep(64);
            if ((s >> 62) == 0) s = ld_relaxed(status + t);
        }
        unsigned inc = __ballot_sync(kFull, (s >> 62) == 2);
        uint64_t v = s & kValMask;
        if (inc) {
            unsigned stop = __ffs(inc) - 1;
            if (lane > stop) v = 0;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
        excl += v;
        if (inc) break;
        base -= 32;
    }
    if (lane == 0) st_relaxed(status + tile, kFlagInc | (excl + agg));
    return excl;
}

// Exclusive block scan of one u32 per thread (NW warps, kBlock threads by default).
// Returns the exclusive prefix; *total receives the block sum. Uses 2*NW+1 words of smem.
template <int NW = kWarps>
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* smem, uint32_t* total) {
    static_assert(NW <= 32, "one warp scans the warp sums");
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= unsigned(o)) x += y;
    }
    if (lane == 31) smem[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < unsigned(NW) ? smem[lane] : 0;
        uint32_t s = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(kFull, s, o);
            if (lane >= unsigned(o)) s += y;
        }
        if (lane < unsigned(NW)) smem[NW + lane] = s - w;
        if (lane == NW - 1) smem[2 * NW] = s;
    }
    __syncthreads();
    uint32_t r = smem[NW + warp] + x - v;
    *total = smem[2 * NW];
    __syncthreads();
    return r;
}

// The same scan with one barrier: every warp adds up the NW warp sums itself. The
// caller must not write smem[0, NW) again before every thread has returned (a second
// scan takes another buffer, or a barrier comes first).
template <int NW = kWarps>
__device__ __forceinline__ uint32_t block_excl_scan1(uint32_t v, uint32_t* smem, uint32_t* total) {
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= unsigned(o)) x += y;
    }
    if (lane == 31) smem[warp] = x;
    __syncthreads();
    uint32_t pre = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        const uint32_t s = smem[w];
        pre += unsigned(w) < warp ? s : 0u;
        tot += s;
    }
    *total = tot;
    return pre + x - v;
}

// 64-bit variant (two 31-bit fields packed are added together safely).
__device__ __forceinline__ uint64_t block_excl_scan64(uint64_t v, uint64_t* smem, uint64_t* total) {
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= unsigned(o)) x += y;
    }
    if (lane == 31) smem[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint64_t w = lane < unsigned(kWarps) ? smem[lane] : 0;
        uint64_t s = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(kFull, s, o);
            if (lane >= unsigned(o)) s += y;
        }
        if (lane < unsigned(kWarps)) smem[kWarps + lane] = s - w;
        if (lane == kWarps - 1) smem[2 * kWarps] = s;
    }
    __syncthreads();
    uint64_t r = smem[kWarps + warp] + x - v;
    *total = smem[2 * kWarps];
    __syncthreads();
    return r;
}

}  // namespace pyrb
