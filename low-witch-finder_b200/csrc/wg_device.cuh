// Device primitives for the Seed Check kernels: the game's RNGs, Perlin table
// construction and Perlin / Octave / DoublePerlin sampling in FP64.
//
// Every floating-point expression keeps the operation order of the reference
// (engine/tools/lysh/src/noise.c, caves.c, phase1.c) and the library is compiled with
// -fmad=false, so results are bit-identical to the reference CPU scanner built with
// -ffp-contract=off.
//
// Table layouts.  A Perlin permutation table is 256 bytes.  The hot kernels build 32
// tables per warp, one per lane, in a 8 KiB "bank-interleaved" block: byte k of lane L
// lives at ((k & ~3) * 32) + 4 L + (k & 3).  Every byte a lane touches is in bank L, so
// both the shuffle (random swap partner per lane) and later lookups by the same lane are
// free of bank conflicts.  Rare-path kernels use plain contiguous 256-byte tables.
#pragma once

#include <cstdint>

#include "wg_catalog.h"

namespace wg {

// ------------------------------------------------------------------------------------
// Xoroshiro128++ (engine/tools/lysh/src/rng.c:75-165)
// ------------------------------------------------------------------------------------
struct Xr {
    uint64_t lo, hi;
};

__device__ __forceinline__ uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

__device__ __forceinline__ uint64_t stafford13(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

__device__ __forceinline__ Xr xr_from_seed(uint64_t seed) {
    uint64_t l = seed ^ 0x6A09E667F3BCC909ULL;
    return Xr{stafford13(l), stafford13(l - 0x61C8864680B583EBULL)};
}

__device__ __forceinline__ Xr xr_make(uint64_t lo, uint64_t hi) {
    if ((lo | hi) == 0) {
        lo = 0x9E3779B97F4A7C15ULL;
        hi = 0x6A09E667F3BCC909ULL;
    }
    return Xr{lo, hi};
}

__device__ __forceinline__ uint64_t xr_next(Xr &s) {
    uint64_t lo = s.lo, hi = s.hi;
    uint64_t out = rotl64(lo + hi, 17) + lo;
    hi ^= lo;
    s.lo = rotl64(lo, 49) ^ hi ^ (hi << 21);
    s.hi = rotl64(hi, 28);
    return out;
}

// Java 17 nextInt(bound), Lemire's multiply-and-reject form.
__device__ __forceinline__ int xr_bounded(Xr &s, uint32_t bound) {
    uint64_t r = (uint64_t)(uint32_t)xr_next(s) * bound;
    if ((uint32_t)r < bound) {
        uint32_t m = (0u - bound) % bound;
        while ((uint32_t)r < m) r = (uint64_t)(uint32_t)xr_next(s) * bound;
    }
    return (int)(r >> 32);
}

__device__ __forceinline__ double xr_double(Xr &s) {
    return (double)(xr_next(s) >> 11) * 1.1102230246251565E-16;
}

// RNG of octave `p` (index into NoiseSpec octave arrays) of sub `sub` of noise `ns`,
// given the seed fork (the per-seed createRandomDeriver state).
__device__ __forceinline__ Xr octave_rng(const NoiseSpec &ns, Xr seed_fork, int sub, int p) {
    Xr noise = xr_make(ns.name_lo ^ seed_fork.lo, ns.name_hi ^ seed_fork.hi);
    uint64_t a = xr_next(noise), b = xr_next(noise);
    if (sub) {
        a = xr_next(noise);
        b = xr_next(noise);
    }
    Xr fork = xr_make(a, b);
    return xr_make(ns.oct_lo[p] ^ fork.lo, ns.oct_hi[p] ^ fork.hi);
}

__device__ __forceinline__ Xr seed_fork_of(uint64_t seed) {
    Xr r = xr_from_seed(seed);
    uint64_t a = xr_next(r), b = xr_next(r);
    return xr_make(a, b);
}

// ------------------------------------------------------------------------------------
// java.util.Random and swamp-hut placement (rng.c:187-227, structure.c:4-42)
// ------------------------------------------------------------------------------------
constexpr uint64_t kLcgMul = 0x5DEECE66DULL;
constexpr uint64_t kLcgMask = 0xFFFFFFFFFFFFULL;

__device__ __forceinline__ int lcg_bits(uint64_t &st, int bits) {
    st = (st * kLcgMul + 0xBULL) & kLcgMask;
    return (int)(uint32_t)(st >> (48 - bits));
}

__device__ __forceinline__ int lcg_int(uint64_t &st, int bound) {
    if ((bound & (bound - 1)) == 0) return (int)(((int64_t)bound * (int64_t)lcg_bits(st, 31)) >> 31);
    for (;;) {
        int u = lcg_bits(st, 31);
        int v = u % bound;
        if ((int32_t)((uint32_t)u - (uint32_t)v + (uint32_t)(bound - 1)) >= 0) return v;
    }
}

__device__ __forceinline__ uint64_t lcg_long(uint64_t &st) {
    uint64_t hi = (uint64_t)(uint32_t)lcg_bits(st, 32);
    int64_t lo = (int64_t)lcg_bits(st, 32);
    return (hi << 32) + (uint64_t)lo;
}

// Chunk of the swamp hut in region (rx, rz): spacing 32, separation 8.
__device__ __forceinline__ void hut_chunk(uint64_t seed, int rx, int rz, int salt, int &cx, int &cz) {
    uint64_t s = (uint64_t)(int64_t)rx * 341873128712ULL + (uint64_t)(int64_t)rz * 132897987541ULL + seed +
                 (uint64_t)(int64_t)salt;
    uint64_t st = (s ^ kLcgMul) & kLcgMask;
    int j = lcg_int(st, 24);
    int k = lcg_int(st, 24);
    cx = rx * 32 + j;
    cz = rz * 32 + k;
}

// Hut orientation, setLargeFeatureSeed + nextInt(4) (eval.c:41-50).
__device__ __forceinline__ int hut_dir(uint64_t seed, int hut_x, int hut_z) {
    uint64_t st = (seed ^ kLcgMul) & kLcgMask;
    uint64_t a = lcg_long(st);
    uint64_t b = lcg_long(st);
    uint64_t s = ((uint64_t)(int64_t)(hut_x >> 4) * a) ^ ((uint64_t)(int64_t)(hut_z >> 4) * b) ^ seed;
    st = (s ^ kLcgMul) & kLcgMask;
    return lcg_int(st, 4);
}

// splitmix64 with the golden-gamma pre-add (the reference's --seed-gen stream).
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// ------------------------------------------------------------------------------------
// Perlin permutation tables
// ------------------------------------------------------------------------------------
__device__ __forceinline__ int il_off(int k) { return ((k & 0xFC) << 5) | (k & 3); }

// Builds one Perlin sampler (3 nextDouble origins + 256-step shuffle, noise.c:61-78)
// into this lane's column of a bank-interleaved block; tb = block + 4 * lane.
__device__ __forceinline__ void perlin_build_il(uint8_t *tb, Xr r, double &ox, double &oy, double &oz) {
    ox = xr_double(r) * 256.0;
    oy = xr_double(r) * 256.0;
    oz = xr_double(r) * 256.0;
    uint32_t *w = reinterpret_cast<uint32_t *>(tb);
#pragma unroll 8
    for (int q = 0; q < 64; q++) w[q * 32] = 0x03020100u + 0x04040404u * (uint32_t)q;
#pragma unroll 4
    for (int i = 0; i < 256; i++) {
        int k = i + xr_bounded(r, (uint32_t)(256 - i));
        uint8_t *pi = tb + il_off(i);
        uint8_t *pk = tb + il_off(k);
        uint8_t a = *pi, b = *pk;
        *pi = b;
        *pk = a;
    }
}

// Same construction into a contiguous 256-byte table (rare-path kernels).
__device__ __forceinline__ void perlin_build_flat(uint8_t *t, Xr r, double &ox, double &oy, double &oz) {
    ox = xr_double(r) * 256.0;
    oy = xr_double(r) * 256.0;
    oz = xr_double(r) * 256.0;
    uint32_t *w = reinterpret_cast<uint32_t *>(t);
#pragma unroll 8
    for (int q = 0; q < 64; q++) w[q] = 0x03020100u + 0x04040404u * (uint32_t)q;
#pragma unroll 4
    for (int i = 0; i < 256; i++) {
        int k = i + xr_bounded(r, (uint32_t)(256 - i));
        uint8_t a = t[i], b = t[k];
        t[i] = b;
        t[k] = a;
    }
}

struct IlTable {
    const uint8_t *tb;  // block + 4 * lane
    __device__ __forceinline__ int operator()(int k) const { return tb[il_off(k)]; }
};
struct FlatTable {
    const uint8_t *t;
    __device__ __forceinline__ int operator()(int k) const { return t[k & 255]; }
};

// ------------------------------------------------------------------------------------
// Perlin sampling (noise.c:224-342)
// ------------------------------------------------------------------------------------
__device__ __forceinline__ double fade(double d) { return d * d * d * (d * (d * 6.0 - 15.0) + 10.0); }
__device__ __forceinline__ double lerp(double t, double a, double b) { return a + t * (b - a); }

// g * v for a gradient component g in {-1, 0, 1}: exactly the IEEE product (v, -v, or a
// zero carrying v's sign), written as bit operations.
__device__ __forceinline__ double gmul(double v, uint32_t h, uint32_t zero_mask, uint32_t neg_mask) {
    long long b = __double_as_longlong(v);
    long long keep = ((zero_mask >> h) & 1u) ? (long long)0x8000000000000000ULL : -1LL;
    long long flip = ((neg_mask >> h) & 1u) ? (long long)0x8000000000000000ULL : 0LL;
    return __longlong_as_double((b & keep) ^ flip);
}

// The game's 16-entry gradient table, as zero / negative bit masks per component.
constexpr uint32_t kGxZero = (1u << 8) | (1u << 9) | (1u << 10) | (1u << 11) | (1u << 13) | (1u << 15);
constexpr uint32_t kGxNeg = (1u << 1) | (1u << 3) | (1u << 5) | (1u << 7) | (1u << 14);
constexpr uint32_t kGyZero = (1u << 4) | (1u << 5) | (1u << 6) | (1u << 7);
constexpr uint32_t kGyNeg = (1u << 2) | (1u << 3) | (1u << 9) | (1u << 11) | (1u << 13) | (1u << 15);
constexpr uint32_t kGzZero = (1u << 0) | (1u << 1) | (1u << 2) | (1u << 3) | (1u << 12) | (1u << 14);
constexpr uint32_t kGzNeg = (1u << 6) | (1u << 7) | (1u << 10) | (1u << 11) | (1u << 15);

__device__ __forceinline__ double grad(int hash, double x, double y, double z) {
    uint32_t h = (uint32_t)hash & 15u;
    double gx = gmul(x, h, kGxZero, kGxNeg);
    double gy = gmul(y, h, kGyZero, kGyNeg);
    double gz = gmul(z, h, kGzZero, kGzNeg);
    return gx + gy + gz;
}

template <class T>
__device__ __forceinline__ double perlin_core(const T &P, int i, int j, int k, double x, double y, double y1,
                                              double z, double fx, double fy, double fz) {
    int a = P(i & 255), b = P((i + 1) & 255);
    int c = P((a + j) & 255), d = P((a + j + 1) & 255);
    int e = P((b + j) & 255), f = P((b + j + 1) & 255);
    double v000 = grad(P((c + k) & 255), x, y, z);
    double v100 = grad(P((e + k) & 255), x - 1, y, z);
    double v010 = grad(P((d + k) & 255), x, y1, z);
    double v110 = grad(P((f + k) & 255), x - 1, y1, z);
    double v001 = grad(P((c + k + 1) & 255), x, y, z - 1);
    double v101 = grad(P((e + k + 1) & 255), x - 1, y, z - 1);
    double v011 = grad(P((d + k + 1) & 255), x, y1, z - 1);
    double v111 = grad(P((f + k + 1) & 255), x - 1, y1, z - 1);
    double x00 = lerp(fx, v000, v100), x10 = lerp(fx, v010, v110);
    double x01 = lerp(fx, v001, v101), x11 = lerp(fx, v011, v111);
    return lerp(fz, lerp(fy, x00, x10), lerp(fy, x01, x11));
}

// MC maintainPrecision (noise.c:31-34); the identity inside +-1e7.
__device__ __forceinline__ double keep_precision(double v) {
    if (v > -1.0e7 && v < 1.0e7) return v;
    return v - (double)(long long)floor(v * 2.9802322387695312E-08 + 0.5) * 3.3554432E7;
}

// One Perlin sampler at y = 0; hy / fy are the y-origin fraction and its fade, jy its floor.
template <class T>
__device__ __forceinline__ double perlin_y0(const T &P, double ox, double oz, int jy, double hy, double fy, double x,
                                            double z) {
    double d = x + ox, f = z + oz;
    double fd = floor(d), ff = floor(f);
    int i = (int)fd, k = (int)ff;
    double g = d - i, l = f - k;
    return perlin_core(P, i, jy, k, g, hy, hy - 1.0, l, fade(g), fy, fade(l));
}

// One Perlin sampler in 3-D with y_scale = y_max = 0 (noise.c:246-261).
template <class T>
__device__ __forceinline__ double perlin_3d(const T &P, double ox, double oy, double oz, double x, double y,
                                            double z) {
    double d = x + ox, e = y + oy, f = z + oz;
    int i = (int)floor(d), j = (int)floor(e), k = (int)floor(f);
    double g = d - i, h = e - j, l = f - k;
    double hm = h - 0.0;
    return perlin_core(P, i, j, k, g, hm, hm - 1, l, fade(g), fade(h), fade(l));
}

constexpr double kDblScale = 1.0181268882175227;

// Java Math.min / Math.max with the signed-zero rules (mcmath.h).
__device__ __forceinline__ bool is_neg_zero(double v) {
    return __double_as_longlong(v) == (long long)0x8000000000000000ULL;
}
__device__ __forceinline__ double jmax(double a, double b) {
    if (a != a) return a;
    if (a == 0.0 && b == 0.0 && is_neg_zero(a)) return b;
    return (a >= b) ? a : b;
}
__device__ __forceinline__ double jmin(double a, double b) {
    if (a != a) return a;
    if (a == 0.0 && b == 0.0 && is_neg_zero(b)) return b;
    return (a <= b) ? a : b;
}
__device__ __forceinline__ double clampd(double v, double lo, double hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

}  // namespace wg
