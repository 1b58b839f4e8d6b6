// Seeded synthetic workloads for the DAG build (integer / Q16.16 fixed point,
// so every platform produces the same voxel lists bit for bit).
//
// Voxel lists use Pyrit's PyrVoxel layout {int32 x, y, z; uint32 attribute}
// (include/pyrit.h:413-416). Edits use the same layout; attribute 0 removes.
//
//   heightfield 64^3 : h(x,z) = 32 + 12*fbm(x/32, z/32), fbm = 4-octave value
//                      noise (gain 1/2, lacunarity 2) normalised to [-1, 1];
//                      solid if y < h; material 1 top layer, 2 the next 3, 3 below.
//   noise 256^3      : 3-octave 3D value noise, base period 64; solid above the
//                      exact 70th percentile; material 1 + hash(8^3 block) mod 8;
//                      0.5% of the cells edited (distinct uniform positions,
//                      50/50 set/remove, set material 1..8), applied in list order.
//   chunk mix        : edge 32/64/128/256 with p .4/.3/.2/.1; heightfield content
//                      tiled by chunk and scaled to the edge; 0..20 spherical caves
//                      of radius 3..12 per chunk.
//   bernoulli 1024^3 : cell occupied iff hash < 0.15 * 2^32, material 1..255;
//                      10^6 uniform set/remove edits.
#ifndef PYRB_WORKLOADS_H
#define PYRB_WORKLOADS_H

#include <stdint.h>

#ifdef __CUDACC__
#define WL_FN __host__ __device__ __forceinline__
#else
#define WL_FN static inline
#endif

WL_FN uint64_t wl_mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
WL_FN uint64_t wl_hash4(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    return wl_mix64(((uint64_t)a << 32 | b) ^ wl_mix64(((uint64_t)c << 32 | d) ^ 0x5851F42D4C957F2Dull));
}
/* lattice value in [-65536, 65535] (Q16) */
WL_FN int32_t wl_lattice(uint32_t ix, uint32_t iy, uint32_t iz, uint32_t oct, uint32_t seed) {
    return (int32_t)(wl_hash4(ix, iy, iz, (oct << 24) ^ seed) >> 47) - 65536;
}
/* smoothstep 3f^2 - 2f^3 for f in [0, 65536) (Q16) */
WL_FN int64_t wl_smooth(int64_t f) {
    int64_t s = (f * f) >> 16;
    return (s * (3 * 65536 - 2 * f)) >> 16;
}
WL_FN int64_t wl_lerp(int64_t a, int64_t b, int64_t t) { return a + (((b - a) * t) >> 16); }

/* 2D value noise at Q16 coordinates (non-negative) */
WL_FN int64_t wl_noise2(int64_t px, int64_t pz, uint32_t oct, uint32_t seed) {
    uint32_t ix = (uint32_t)(px >> 16), iz = (uint32_t)(pz >> 16);
    int64_t tx = wl_smooth(px & 0xFFFF), tz = wl_smooth(pz & 0xFFFF);
    int64_t a = wl_lattice(ix, 0, iz, oct, seed), b = wl_lattice(ix + 1, 0, iz, oct, seed);
    int64_t c = wl_lattice(ix, 0, iz + 1, oct, seed), d = wl_lattice(ix + 1, 0, iz + 1, oct, seed);
    return wl_lerp(wl_lerp(a, b, tx), wl_lerp(c, d, tx), tz);
}
/* 4 octaves, gain 1/2, lacunarity 2, normalised by the amplitude sum 1.875 */
WL_FN int64_t wl_fbm2(int64_t u, int64_t v, uint32_t seed) {
    int64_t total = 0;
    for (uint32_t o = 0; o < 4; ++o) total += wl_noise2(u << o, v << o, o, seed) * (65536 >> o);
    return total / 122880;
}
/* heightfield in Q16 at Q16 coordinates: 32 + 12 * fbm */
WL_FN int64_t wl_height_q16(int64_t u, int64_t v, uint32_t seed) { return ((int64_t)32 << 16) + 12 * wl_fbm2(u, v, seed); }

/* material of a solid voxel at height y below surface height h (voxels) */
WL_FN uint32_t wl_layer_material(int32_t y, int32_t h) { return y == h - 1 ? 1u : (y >= h - 4 ? 2u : 3u); }

/* 3D value noise (3 octaves, base period 64) in Q16, range about [-65536, 65536] */
WL_FN int64_t wl_noise3(int64_t px, int64_t py, int64_t pz, uint32_t oct, uint32_t seed) {
    uint32_t ix = (uint32_t)(px >> 16), iy = (uint32_t)(py >> 16), iz = (uint32_t)(pz >> 16);
    int64_t tx = wl_smooth(px & 0xFFFF), ty = wl_smooth(py & 0xFFFF), tz = wl_smooth(pz & 0xFFFF);
    int64_t c000 = wl_lattice(ix, iy, iz, oct, seed), c100 = wl_lattice(ix + 1, iy, iz, oct, seed);
    int64_t c010 = wl_lattice(ix, iy + 1, iz, oct, seed), c110 = wl_lattice(ix + 1, iy + 1, iz, oct, seed);
    int64_t c001 = wl_lattice(ix, iy, iz + 1, oct, seed), c101 = wl_lattice(ix + 1, iy, iz + 1, oct, seed);
    int64_t c011 = wl_lattice(ix, iy + 1, iz + 1, oct, seed), c111 = wl_lattice(ix + 1, iy + 1, iz + 1, oct, seed);
    int64_t x00 = wl_lerp(c000, c100, tx), x10 = wl_lerp(c010, c110, tx);
    int64_t x01 = wl_lerp(c001, c101, tx), x11 = wl_lerp(c011, c111, tx);
    return wl_lerp(wl_lerp(x00, x10, ty), wl_lerp(x01, x11, ty), tz);
}
WL_FN int32_t wl_value3(uint32_t x, uint32_t y, uint32_t z, uint32_t seed) {
    int64_t px = (int64_t)x << 10, py = (int64_t)y << 10, pz = (int64_t)z << 10;  /* coordinate / 64 in Q16 */
    int64_t total = 0;
    for (uint32_t o = 0; o < 3; ++o) total += wl_noise3(px << o, py << o, pz << o, 16 + o, seed) * (65536 >> o);
    return (int32_t)(total / 114688);  /* amplitude sum 1.75 */
}

#ifdef __cplusplus
extern "C" {
#endif

/* All functions return the number of voxels (or edits) produced; with out == NULL
 * (or cap too small) they only count. Lists are in scan order (x fastest, then y, z). */
uint64_t wl_heightfield(uint32_t log2_size, uint32_t seed, uint32_t* out, uint64_t cap);
/* noise grid without edits; *threshold receives the 70th-percentile value used */
uint64_t wl_noise_grid(uint32_t log2_size, uint32_t seed, uint32_t* out, uint64_t cap, int32_t* threshold);
/* 0.5% distinct-position edits for a grid of edge 2^log2_size (list order = application order) */
uint64_t wl_noise_edits(uint32_t log2_size, uint32_t seed, uint32_t* out, uint64_t cap);
/* Bernoulli(0.15) grid, material 1..255 */
uint64_t wl_bernoulli_grid(uint32_t log2_size, uint32_t seed, uint32_t* out, uint64_t cap);
/* attribute of the Bernoulli grid at pts[n][3] (0 = empty) */
void wl_bernoulli_at(uint64_t n, const uint32_t* pts, uint32_t seed, uint32_t* out);
/* n uniform random set/remove edits, material 1..255 (positions may repeat) */
uint64_t wl_uniform_edits(uint32_t log2_size, uint64_t n, uint32_t seed, uint32_t* out);
/* chunk edges for the mix: out_log2[k] in {5,6,7,8} */
void wl_chunk_mix(uint32_t count, uint32_t seed, uint32_t* out_log2);
/* content of mix chunk `index` with edge 2^log2 */
uint64_t wl_mix_chunk(uint32_t index, uint32_t log2, uint32_t seed, uint32_t* out, uint64_t cap);
/* n uniform random set/remove edits in a chunk (material 1..8), per-request overlay */
uint64_t wl_chunk_edits(uint32_t log2, uint32_t n, uint32_t seed, uint32_t* out);
/* Dense test scene of the reference's tests (tests/common.zig:14-35: sphere, floor,
 * pillars, scattered voxels; attribute = attrOf), dense[x + N*(y + N*z)]. */
void wl_scene_dense(uint32_t log2_size, uint32_t* dense);
uint32_t wl_attr_of(int32_t x, int32_t y, int32_t z);
/* Poisson arrival times (seconds) at rate lambda */
void wl_poisson_arrivals(uint64_t n, double lambda, uint32_t seed, double* out);

#ifdef __cplusplus
}
#endif
#endif
