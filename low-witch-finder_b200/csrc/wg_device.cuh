// Device primitives for the Seed Check kernels: the game's RNGs, Perlin table
// construction and Perlin / Octave / DoublePerlin sampling in FP64.
//
// Every floating-point expression keeps the operation order of the reference
// (engine/tools/lysh/src/noise.c, caves.c, phase1.c) and the library is compiled with
// -fmad=false, so results are bit-identical to the reference CPU scanner built with
// -ffp-contract=off.
//
// Table layouts.  A Perlin permutation table is 256 bytes.  The hot kernels keep the tables of
// one sampler slot for all the CTA's units in one byte-interleaved block of 256 rows: byte k of
// unit u sits at k * U + u (U = units per CTA).  Any lookup is then one multiply-add away from
// its index, and the 4-byte words of a row are shared by 4 units, so the random lookups of a
// warp spread over all banks (about 2-way conflicts).  Blocks are padded so that neighbouring
// slots start in different banks.  A bank-private layout (table c of each 32 in bank c only,
// conflict-free for any indices) was measured slower on the B200: its address arithmetic adds two
// integer operations to each access, and the table builds and samples are bound by issue and
// latency, not by shared-memory bandwidth (build alone 101.8 ms against 95.4 ms for 2^24 seeds).
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

// The same generator with the state as four 32-bit words, for the 256 nextInt(bound) draws of
// a Perlin shuffle: next32() returns only the low 32 bits of the output, which is all
// nextInt(bound) reads, and spells the 64-bit adds / rotates / shifts as 32-bit carry adds and
// funnel shifts.
struct Xr32 {
    uint32_t l0, l1, h0, h1;   // lo = (l1:l0), hi = (h1:h0)
    __device__ __forceinline__ explicit Xr32(const Xr &x)
        : l0((uint32_t)x.lo), l1((uint32_t)(x.lo >> 32)), h0((uint32_t)x.hi), h1((uint32_t)(x.hi >> 32)) {}
    __device__ __forceinline__ uint32_t next32() {
        uint32_t s0, s1;   // s = lo + hi
        asm("add.cc.u32 %0, %2, %3;\n\taddc.u32 %1, %4, %5;" : "=r"(s0), "=r"(s1) : "r"(l0), "r"(h0), "r"(l1), "r"(h1));
        const uint32_t out = __funnelshift_l(s1, s0, 17) + l0;            // low word of rotl(s, 17) + lo
        const uint32_t x0 = h0 ^ l0, x1 = h1 ^ l1;                          // hi ^= lo
        const uint32_t r0 = __funnelshift_r(l0, l1, 15), r1 = __funnelshift_r(l1, l0, 15);   // rotl(lo, 49)
        const uint32_t t0 = x0 << 21, t1 = __funnelshift_l(x0, x1, 21);   // hi << 21
        l0 = r0 ^ x0 ^ t0;
        l1 = r1 ^ x1 ^ t1;
        h0 = __funnelshift_l(x1, x0, 28);                                   // rotl(hi, 28)
        h1 = __funnelshift_l(x0, x1, 28);
        return out;
    }
    // Java 17 nextInt(bound): Lemire's multiply-and-reject on the low 32 bits.
    __device__ __forceinline__ uint32_t bounded(uint32_t bound) {
        uint32_t x = next32();
        uint32_t lo = x * bound, j = __umulhi(x, bound);
        if (lo < bound) {
            const uint32_t m = (0u - bound) % bound;
            while (lo < m) {
                x = next32();
                lo = x * bound;
                j = __umulhi(x, bound);
            }
        }
        return j;
    }
};

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
// Fills `nblocks` byte-interleaved blocks with the identity permutation: a block holds 256 rows
// of STRIDE bytes (one column per table), row k all equal to k, and blocks start PITCH bytes
// apart (PITCH - 256 * STRIDE bytes of padding shift consecutive blocks to other banks).
// Called by every thread of the CTA (thread tid of nthreads), followed by a barrier.
template <int STRIDE, int PITCH>
__device__ __forceinline__ void perm_blocks_init(uint8_t *base, int nblocks, int tid, int nthreads) {
    static_assert(STRIDE % 4 == 0 && PITCH % 4 == 0 && PITCH >= 256 * STRIDE, "rows must be whole words");
    constexpr int kRowWords = STRIDE / 4, kPitchWords = PITCH / 4;
    uint32_t *w = reinterpret_cast<uint32_t *>(base);
    for (int q = tid; q < nblocks * kPitchWords; q += nthreads) {
        const int in_block = q % kPitchWords;
        w[q] = (uint32_t)(in_block / kRowWords) * 0x01010101u;   // padding words get junk; never read
    }
}

// The 256-step Fisher-Yates shuffle of one Perlin sampler (noise.c:61-72) on an initialised
// column: byte k of this table is at t[k * STRIDE].  Draws the three origins first.
// Four steps at a time: the four draws are taken first with one combined check for Lemire's
// rare slow path (a low product word below the bound, probability < 2^-24 per draw); on that path
// the four steps' draws are taken again one by one with the exact rejection loop.  Either way the
// draws, and so the table, are those of the step-by-step shuffle; the common path is straight-line
// code in which the next draws overlap the swaps.
template <int STRIDE>
__device__ __forceinline__ void perlin_shuffle(uint8_t *t, Xr r, double &ox, double &oy, double &oz) {
    ox = xr_double(r) * 256.0;
    oy = xr_double(r) * 256.0;
    oz = xr_double(r) * 256.0;
    Xr32 q(r);
#pragma unroll 2
    for (int i = 0; i < 256; i += 4) {
        const Xr32 q0 = q;
        const uint32_t b0 = 256u - i, b1 = 255u - i, b2 = 254u - i, b3 = 253u - i;
        const uint32_t x0 = q.next32(), x1 = q.next32(), x2 = q.next32(), x3 = q.next32();
        uint32_t j0 = __umulhi(x0, b0), j1 = __umulhi(x1, b1), j2 = __umulhi(x2, b2), j3 = __umulhi(x3, b3);
        if ((x0 * b0 < b0) | (x1 * b1 < b1) | (x2 * b2 < b2) | (x3 * b3 < b3)) {
            q = q0;
            j0 = q.bounded(b0);
            j1 = q.bounded(b1);
            j2 = q.bounded(b2);
            j3 = q.bounded(b3);
        }
        const uint32_t js[4] = {j0, j1, j2, j3};
#pragma unroll
        for (int s = 0; s < 4; s++) {
            const int ii = i + s, k = ii + (int)js[s];
            const uint8_t a = t[ii * STRIDE], b = t[k * STRIDE];
            t[ii * STRIDE] = b;
            t[k * STRIDE] = a;
        }
    }
}

// The high 32-bit words of the doubles -1.0 / 0.0 / +1.0 of the game's 16-entry gradient table
// (noise.c:15-20), [component * 16 + hash], kept in shared memory by every sampling kernel: a
// warp's reads of one component touch at most 16 words in 16 distinct banks.
constexpr int kGradWords = 48;
__device__ __forceinline__ void fill_grad_table(uint32_t *gt, int tid);

// Table reader: byte k of a column with the given row stride, plus the gradient products.
template <int STRIDE>
struct ColTable {
    const uint8_t *t;
    const uint32_t *gt;
    __device__ __forceinline__ int operator()(int k) const { return t[k * STRIDE]; }
    // (double)g[0] * x + (double)g[1] * y + (double)g[2] * z, as the reference writes it
    __device__ __forceinline__ double grad(int hash, double x, double y, double z) const {
        const int h = hash & 15;
        return __hiloint2double((int)gt[h], 0) * x + __hiloint2double((int)gt[16 + h], 0) * y +
               __hiloint2double((int)gt[32 + h], 0) * z;
    }
};


// ------------------------------------------------------------------------------------
// Perlin sampling (noise.c:224-342)
// ------------------------------------------------------------------------------------
__device__ __forceinline__ double fade(double d) { return d * d * d * (d * (d * 6.0 - 15.0) + 10.0); }
__device__ __forceinline__ double lerp(double t, double a, double b) { return a + t * (b - a); }

// The game's 16-entry gradient table (noise.c:15-20) as 2-bit codes per component and hash:
// 0 = 0, 1 = +1, 3 = -1 (bits 2h..2h+1 of each constant).
__host__ __device__ constexpr uint32_t grad_codes(int c) {
    // rows: {gx, gy, gz} of hashes 0..15
    const int g[16][3] = {{1, 1, 0}, {-1, 1, 0}, {1, -1, 0}, {-1, -1, 0}, {1, 0, 1}, {-1, 0, 1},
                          {1, 0, -1}, {-1, 0, -1}, {0, 1, 1}, {0, -1, 1}, {0, 1, -1}, {0, -1, -1},
                          {1, 1, 0}, {0, -1, 1}, {-1, 1, 0}, {0, -1, -1}};
    uint32_t v = 0;
    for (int h = 0; h < 16; h++) v |= (uint32_t)(g[h][c] == 0 ? 0 : (g[h][c] > 0 ? 1 : 3)) << (2 * h);
    return v;
}

constexpr uint32_t kGradCodeX = grad_codes(0), kGradCodeY = grad_codes(1), kGradCodeZ = grad_codes(2);

__device__ __forceinline__ void fill_grad_table(uint32_t *gt, int tid) {
    if (tid < kGradWords) {
        const int c = tid / 16;
        const uint32_t codes = c == 0 ? kGradCodeX : (c == 1 ? kGradCodeY : kGradCodeZ);
        const uint32_t code = (codes >> (2 * (tid % 16))) & 3u;
        gt[tid] = code == 0 ? 0u : (code == 1 ? 0x3FF00000u : 0xBFF00000u);
    }
}

template <class T>
__device__ __forceinline__ double perlin_core(const T &P, int i, int j, int k, double x, double y, double y1,
                                              double z, double fx, double fy, double fz) {
    int a = P(i & 255), b = P((i + 1) & 255);
    int c = P((a + j) & 255), d = P((a + j + 1) & 255);
    int e = P((b + j) & 255), f = P((b + j + 1) & 255);
    double v000 = P.grad(P((c + k) & 255), x, y, z);
    double v100 = P.grad(P((e + k) & 255), x - 1, y, z);
    double v010 = P.grad(P((d + k) & 255), x, y1, z);
    double v110 = P.grad(P((f + k) & 255), x - 1, y1, z);
    double v001 = P.grad(P((c + k + 1) & 255), x, y, z - 1);
    double v101 = P.grad(P((e + k + 1) & 255), x - 1, y, z - 1);
    double v011 = P.grad(P((d + k + 1) & 255), x, y1, z - 1);
    double v111 = P.grad(P((f + k + 1) & 255), x - 1, y1, z - 1);
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
    // d - (double)(int)floor(d) == d - floor(d): |d| < 2^31 here, so the int round trip is exact
    double g = d - fd, l = f - ff;
    return perlin_core(P, i, jy, k, g, hy, hy - 1.0, l, fade(g), fy, fade(l));
}

// One Perlin sampler in 3-D with y_scale = y_max = 0 (noise.c:246-261).
template <class T>
__device__ __forceinline__ double perlin_3d(const T &P, double ox, double oy, double oz, double x, double y,
                                            double z) {
    double d = x + ox, e = y + oy, f = z + oz;
    double fd = floor(d), fe = floor(e), ff = floor(f);
    int i = (int)fd, j = (int)fe, k = (int)ff;
    double g = d - fd, h = e - fe, l = f - ff;
    double hm = h - 0.0;
    return perlin_core(P, i, j, k, g, hm, hm - 1, l, fade(g), fade(h), fade(l));
}

// ------------------------------------------------------------------------------------
// FP32 noise core (the climate samples of the FP32-plus-FP64-recheck path)
// ------------------------------------------------------------------------------------
// The coordinate reduction stays in FP64 exactly as above (d = x + ox, its floor and the
// fraction d - floor(d), which is exact), since a float cannot hold the fraction of a
// coordinate of magnitude ~1e5.  Everything after it works on values in [-2, 2] and runs in
// FP32 with the operation sequence below, whose error against the exact real-valued sample
// (the same lattice cell and hashes, exact fractions g, l and y origin hy) is bounded here.
// u = 2^-24 is the unit roundoff; "half-ulp" bounds a round-to-nearest result.
//
//  G = rn(g), L = rn(l), H = rn(hy) from exact doubles in [0, 1):      |err| <= u/2
//  G1 = G - 1 (exact for G >= 1/2, else rounds in (-1, -1/2]):          |err| <= u
//  FY = rn(fade(hy)) (fade taken in FP64):                             |err| <= u/2 + 2^-52
//  FX = fade_f32(G) evaluated as 1/2 + s (15/8 + s^2 (6 s^2 - 5)), s = G - 1/2:
//      s exact (Sterbenz) or within u/4; s^2 within u/8 (value <= 1/4); 6 s^2 - 5 in
//      [-5, -3.5] within u*4 * 1.19; the 15/8 step in [0.625, 1.875] within 2.81 u; the last
//      FMA within 1.41 u + u/2 of rounding; with fade' <= 1.875 carrying the u/2 input error
//      and the u/4 of s:  |FX - fade(g)| <= 3.32 u <= 4 u
//  corner dot (two +-1 components; the zero one adds nothing): one rounded add of two
//      coordinates, each within u, value <= 2:                          |err| <= 3 u
//  lerp(t, a, b) as (a - t a) + t b (two FMAs, each value <= 2 -> u of rounding each):
//      |err| <= max(err a, err b) + |t err| * |b - a| + 2 u, with |b - a| <= 4
//      x lerps: 3 u + 4 * 4 u + 2 u = 21 u;  y lerps: 21 u + 4 * u/2 + 2 u = 25 u;
//      z lerp: 25 u + 4 * 4 u + 2 u = 43 u   (T slightly above 1 after rounding: x 1.0001)
// So |FP32 sample - exact| <= 44 u = 2.62e-6 (kPerlinF32ErrUlps), and |sample| <= 2.  The
// FP64 sample of the reference order is within ~1e-14 of the exact value; the gates add that
// and the sums' own roundings (build_climate_steps).  No FMA contraction is left to the
// compiler: every FP32 operation below is an explicit intrinsic.
// Two FP32 lanes per instruction (PTX f32x2, sm_100): each lane is the scalar operation with its
// own round-to-nearest, so a packed step and two scalar steps give the same bits.
struct F2 {
    unsigned long long v;
};
__device__ __forceinline__ F2 f2(float a, float b) {
    F2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void f2_split(F2 r, float &a, float &b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r.v)); }
__device__ __forceinline__ F2 f2_fma(F2 a, F2 b, F2 c) {
    F2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return d;
}
__device__ __forceinline__ F2 f2_mul(F2 a, F2 b) {
    F2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
__device__ __forceinline__ F2 f2_add(F2 a, F2 b) {
    F2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
// fade_f32 on both lanes: 1/2 + s (15/8 + s^2 (6 s^2 - 5)), s = t - 1/2
__device__ __forceinline__ F2 fade_f32x2(F2 t) {
    const F2 s = f2_add(t, f2(-0.5f, -0.5f));
    const F2 s2 = f2_mul(s, s);
    const F2 p = f2_fma(f2(6.0f, 6.0f), s2, f2(-5.0f, -5.0f));
    const F2 q = f2_fma(s2, p, f2(1.875f, 1.875f));
    return f2_fma(s, q, f2(0.5f, 0.5f));
}
// lerp(t, a, b) = (a - t a) + t b on both lanes
__device__ __forceinline__ F2 lerp_f32x2(F2 t, F2 a, F2 b) {
    float t0, t1;
    f2_split(t, t0, t1);
    return f2_fma(t, b, f2_fma(f2(-t0, -t1), a, a));
}
__device__ __forceinline__ float lerp_f32(float t, float a, float b) {
    return __fmaf_rn(t, b, __fmaf_rn(-t, a, a));
}

// The game's 16 gradient vectors as floats, (x, z) pairs and the y components.  Each array is at
// most 128 bytes with one entry per hash, so a warp's reads of either (at most 16 distinct
// entries, in distinct banks) never conflict; one 16-byte (x, y, z, 0) vector per hash would
// span 256 bytes, where hashes h and h + 8 share banks.  Measured on the 9 x 9 workload: the
// climate kernel's FP32 core 5.5 % faster than with the 16-byte vectors.
struct GradF {
    float2 xz[16];
    float y[16];
};

// Table reader of the FP32 core.  Byte k of the table is at t[k * STRIDE] as in ColTable, and the
// table has a row 256 holding a copy of row 0 (written after the shuffle, in the slot block's
// padding), so that the pair P[k], P[(k + 1) & 255] is two loads from one address.
template <int STRIDE>
struct ColTableF {
    const uint8_t *t;
    const GradF *gf;
    __device__ __forceinline__ void pair(int k, int &lo, int &hi) const {
        const uint8_t *r = t + (k & 255) * STRIDE;
        lo = r[0];
        hi = r[STRIDE];
    }
    __device__ __forceinline__ float grad(int hash, float x, float y, float z) const {
        const int h = hash & 15;
        const float2 g = gf->xz[h];
        return __fmaf_rn(g.x, x, __fmaf_rn(gf->y[h], y, __fmul_rn(g.y, z)));
    }
};

__device__ __forceinline__ void fill_grad_table_f32(GradF *gf, int tid) {
    if (tid < 16) {
        float c[3];
        const uint32_t codes[3] = {kGradCodeX, kGradCodeY, kGradCodeZ};
        for (int q = 0; q < 3; q++) {
            const uint32_t code = (codes[q] >> (2 * tid)) & 3u;
            c[q] = code == 0 ? 0.0f : (code == 1 ? 1.0f : -1.0f);
        }
        gf->xz[tid] = make_float2(c[0], c[2]);
        gf->y[tid] = c[1];
    }
}

// One Perlin sampler at y = 0 in the FP32 core; hyf / fyf are rn(hy) and rn(fade(hy)) of the
// table's y origin fraction, jy its floor.  x, z are the FP64 sampling coordinates.  The corner
// values are paired along z, (v.0, v.1), so the x and y lerps and both fades run two lanes per
// instruction; every lane performs the operations the bound above counts.
template <class T>
__device__ __forceinline__ float perlin_y0_f32(const T &P, double ox, double oz, int jy, float hyf, float fyf,
                                               double x, double z) {
    const double d = x + ox, f = z + oz;
    const double fd = floor(d), ff = floor(f);
    const int i = (int)fd, k = (int)ff;
    const float g = __double2float_rn(d - fd), l = __double2float_rn(f - ff);
    const F2 gl = f2(g, l);
    float g1, l1;
    f2_split(f2_add(gl, f2(-1.0f, -1.0f)), g1, l1);   // g - 1, l - 1
    const float hy1 = __fsub_rn(hyf, 1.0f);
    int a, b, c, dd, e, ee;
    P.pair(i, a, b);
    P.pair(a + jy, c, dd);
    P.pair(b + jy, e, ee);
    int h000, h001, h100, h101, h010, h011, h110, h111;
    P.pair(c + k, h000, h001);
    P.pair(e + k, h100, h101);
    P.pair(dd + k, h010, h011);
    P.pair(ee + k, h110, h111);
    const F2 v00 = f2(P.grad(h000, g, hyf, l), P.grad(h001, g, hyf, l1));     // (v000, v001)
    const F2 v10 = f2(P.grad(h100, g1, hyf, l), P.grad(h101, g1, hyf, l1));   // (v100, v101)
    const F2 v01 = f2(P.grad(h010, g, hy1, l), P.grad(h011, g, hy1, l1));     // (v010, v011)
    const F2 v11 = f2(P.grad(h110, g1, hy1, l), P.grad(h111, g1, hy1, l1));   // (v110, v111)
    float fx, fz;
    f2_split(fade_f32x2(gl), fx, fz);
    const F2 x0 = lerp_f32x2(f2(fx, fx), v00, v10);    // (x00, x01)
    const F2 x1 = lerp_f32x2(f2(fx, fx), v01, v11);    // (x10, x11)
    float y0, y1;
    f2_split(lerp_f32x2(f2(fyf, fyf), x0, x1), y0, y1);
    return lerp_f32(fz, y0, y1);
}

// fade_f32 on one lane: 1/2 + s (15/8 + s^2 (6 s^2 - 5)), s = t - 1/2 (fade_f32x2's operations)
__device__ __forceinline__ float fade_f32(float t) {
    const float s = __fadd_rn(t, -0.5f);
    const float s2 = __fmul_rn(s, s);
    const float p = __fmaf_rn(6.0f, s2, -5.0f);
    const float q = __fmaf_rn(s2, p, 1.875f);
    return __fmaf_rn(s, q, 0.5f);
}

// One Perlin sampler in 3-D (y_scale = y_max = 0, noise.c:246-261) in the FP32 core: the three
// coordinate reductions in FP64 as perlin_3d (d = x + ox, its floor, the exact fraction), the rest
// in FP32 with perlin_y0_f32's operations, the y fraction H = rn(h) and its fade now per sample.
// Error against the exact sample (same lattice cell and hashes), in the terms of the bound above
// perlin_y0_f32: G, L, H within u/2 and G - 1, L - 1, H - 1 within u; FX, FY, FZ within 4 u; a
// corner dot within 3 u; x lerps 3 u + 4 * 4 u + 2 u = 21 u; y lerps 21 u + 4 * 4 u + 2 u = 39 u
// (the fade of y now carries 4 u instead of u/2); z lerp 39 u + 4 * 4 u + 2 u = 57 u.  So
// |FP32 sample - exact| <= 60 u (kPerlin3dF32ErrUlps) with |sample| <= 2.
template <class T>
__device__ __forceinline__ float perlin_3d_f32(const T &P, double ox, double oy, double oz, double x, double y,
                                               double z) {
    const double d = x + ox, e = y + oy, f = z + oz;
    const double fd = floor(d), fe = floor(e), ff = floor(f);
    const int i = (int)fd, j = (int)fe, k = (int)ff;
    const float g = __double2float_rn(d - fd), h = __double2float_rn(e - fe), l = __double2float_rn(f - ff);
    const F2 gl = f2(g, l);
    float g1, l1;
    f2_split(f2_add(gl, f2(-1.0f, -1.0f)), g1, l1);   // g - 1, l - 1
    const float h1 = __fsub_rn(h, 1.0f);
    int a, b, c, dd, ee, e2;
    P.pair(i, a, b);
    P.pair(a + j, c, dd);
    P.pair(b + j, ee, e2);
    int h000, h001, h100, h101, h010, h011, h110, h111;
    P.pair(c + k, h000, h001);
    P.pair(ee + k, h100, h101);
    P.pair(dd + k, h010, h011);
    P.pair(e2 + k, h110, h111);
    const F2 v00 = f2(P.grad(h000, g, h, l), P.grad(h001, g, h, l1));      // (v000, v001)
    const F2 v10 = f2(P.grad(h100, g1, h, l), P.grad(h101, g1, h, l1));    // (v100, v101)
    const F2 v01 = f2(P.grad(h010, g, h1, l), P.grad(h011, g, h1, l1));    // (v010, v011)
    const F2 v11 = f2(P.grad(h110, g1, h1, l), P.grad(h111, g1, h1, l1));  // (v110, v111)
    float fx, fz;
    f2_split(fade_f32x2(gl), fx, fz);
    const float fy = fade_f32(h);
    const F2 x0 = lerp_f32x2(f2(fx, fx), v00, v10);    // (x00, x01)
    const F2 x1 = lerp_f32x2(f2(fx, fx), v01, v11);    // (x10, x11)
    float y0, y1;
    f2_split(lerp_f32x2(f2(fy, fy), x0, x1), y0, y1);
    return lerp_f32(fz, y0, y1);
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
