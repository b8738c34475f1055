/* Test infrastructure only: the CPU oracle (the checker), never the product.
 *
 * Plain-C restatement of the reference's Seed Check phase 1 (lysh).  The arithmetic is
 * written out in the same operation order as the reference, because every floating-point
 * result must be bit-identical (compiled with -ffp-contract=off, like the reference).
 * Citations are to files under engine/tools/lysh/src/ unless stated otherwise.
 */
#include "witch_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* ------------------------------------------------------------------ */
/* seed stream: splitmix64 with the golden-gamma pre-add               */
/* engine/gpu/low54/device_construct.h:40-47, phase1_scan.cu:87         */
/* ------------------------------------------------------------------ */
uint64_t wo_splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

/* ------------------------------------------------------------------ */
/* MD5 (RFC 1321), used only to key the noise derivation (rng.c:13-73) */
/* ------------------------------------------------------------------ */
static uint32_t md5_k[64];
static const uint8_t md5_s[4][4] = {{7, 12, 17, 22}, {5, 9, 14, 20}, {4, 11, 16, 23}, {6, 10, 15, 21}};
static pthread_once_t md5_once = PTHREAD_ONCE_INIT;
static void md5_init_k(void) {
    for (int i = 0; i < 64; i++) md5_k[i] = (uint32_t)(fabs(sin((double)(i + 1))) * 4294967296.0);
}
static uint32_t rotl32(uint32_t x, int n) { return (x << n) | (x >> (32 - n)); }
static void md5_compress(uint32_t st[4], const uint8_t blk[64]) {
    uint32_t w[16];
    for (int i = 0; i < 16; i++)
        w[i] = (uint32_t)blk[4 * i] | ((uint32_t)blk[4 * i + 1] << 8) | ((uint32_t)blk[4 * i + 2] << 16) |
               ((uint32_t)blk[4 * i + 3] << 24);
    uint32_t a = st[0], b = st[1], c = st[2], d = st[3];
    for (int i = 0; i < 64; i++) {
        int round = i >> 4;
        uint32_t f;
        int g;
        switch (round) {
            case 0: f = (b & c) | (~b & d); g = i; break;
            case 1: f = (d & b) | (~d & c); g = (5 * i + 1) & 15; break;
            case 2: f = b ^ c ^ d; g = (3 * i + 5) & 15; break;
            default: f = c ^ (b | ~d); g = (7 * i) & 15; break;
        }
        uint32_t nb = b + rotl32(a + f + md5_k[i] + w[g], md5_s[round][i & 3]);
        a = d; d = c; c = b; b = nb;
    }
    st[0] += a; st[1] += b; st[2] += c; st[3] += d;
}
void wo_md5(const uint8_t *data, uint64_t len, uint8_t out[16]) {
    pthread_once(&md5_once, md5_init_k);
    uint32_t st[4] = {0x67452301u, 0xefcdab89u, 0x98badcfeu, 0x10325476u};
    uint64_t off = 0;
    for (; off + 64 <= len; off += 64) md5_compress(st, data + off);
    uint8_t tail[128];
    memset(tail, 0, sizeof(tail));
    uint64_t rem = len - off;
    memcpy(tail, data + off, rem);
    tail[rem] = 0x80;
    uint64_t tl = (rem + 9 <= 64) ? 64 : 128;
    uint64_t bits = len * 8;
    for (int i = 0; i < 8; i++) tail[tl - 8 + i] = (uint8_t)(bits >> (8 * i));
    md5_compress(st, tail);
    if (tl == 128) md5_compress(st, tail + 64);
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) out[4 * i + j] = (uint8_t)(st[i] >> (8 * j));
}

/* ------------------------------------------------------------------ */
/* Xoroshiro128++ family, bit-exact with the game (rng.c:75-185)       */
/* ------------------------------------------------------------------ */
typedef struct { uint64_t lo, hi; } xr_t;

static uint64_t stafford13(uint64_t z) {                       /* rng.c:76-80 */
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static void xr_seed(xr_t *s, uint64_t seed) {                  /* rng.c:82-87: upgradeSeedTo128bit */
    uint64_t l = seed ^ 0x6A09E667F3BCC909ULL;
    s->lo = stafford13(l);
    s->hi = stafford13(l - 0x61C8864680B583EBULL);
}
static void xr_set(xr_t *s, uint64_t lo, uint64_t hi) {        /* rng.c:89-96: zero-state sentinel */
    if ((lo | hi) == 0) { lo = 0x9E3779B97F4A7C15ULL; hi = 0x6A09E667F3BCC909ULL; }
    s->lo = lo; s->hi = hi;
}
static inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static inline uint64_t xr_next(xr_t *s) {                      /* rng.c:100-107 */
    uint64_t lo = s->lo, hi = s->hi;
    uint64_t out = rotl64(lo + hi, 17) + lo;
    hi ^= lo;
    s->lo = rotl64(lo, 49) ^ hi ^ (hi << 21);
    s->hi = rotl64(hi, 28);
    return out;
}
static inline int xr_bounded(xr_t *s, int bound) {             /* rng.c:116-130: Lemire rejection */
    uint64_t r = (xr_next(s) & 0xFFFFFFFFULL) * (uint64_t)(uint32_t)bound;
    if ((uint32_t)r < (uint32_t)bound) {
        uint32_t m = (uint32_t)(0u - (uint32_t)bound) % (uint32_t)bound;
        while ((uint32_t)r < m) r = (xr_next(s) & 0xFFFFFFFFULL) * (uint64_t)(uint32_t)bound;
    }
    return (int)(r >> 32);
}
static inline double xr_double(xr_t *s) {                      /* rng.c:137-139: top 53 bits */
    return (double)(xr_next(s) >> 11) * 1.1102230246251565E-16;
}
static void xr_fork(xr_t *out, xr_t *s) {                      /* rng.c:145-149: createRandomDeriver */
    uint64_t a = xr_next(s);
    uint64_t b = xr_next(s);
    xr_set(out, a, b);
}
static uint64_t be64(const uint8_t *p) {
    uint64_t v = 0;
    for (int i = 0; i < 8; i++) v = (v << 8) | p[i];
    return v;
}
static void xr_named(xr_t *out, const xr_t *s, const char *name) { /* rng.c:159-165: createRandom(String) */
    uint8_t h[16];
    wo_md5((const uint8_t *)name, strlen(name), h);
    xr_set(out, be64(h) ^ s->lo, be64(h + 8) ^ s->hi);
}

/* ------------------------------------------------------------------ */
/* java.util.Random (48-bit LCG) and structure placement               */
/* rng.c:187-227, structure.c:4-42                                     */
/* ------------------------------------------------------------------ */
#define LCG_MUL 0x5DEECE66DULL
#define LCG_MASK 0xFFFFFFFFFFFFULL
static inline int lcg_bits(uint64_t *st, int bits) {
    *st = (*st * LCG_MUL + 0xBULL) & LCG_MASK;
    return (int)(int32_t)(uint32_t)(*st >> (48 - bits));
}
static inline int lcg_int(uint64_t *st, int bound) {           /* JDK Random.nextInt(bound) */
    if ((bound & (bound - 1)) == 0)
        return (int)(((int64_t)bound * (int64_t)lcg_bits(st, 31)) >> 31);
    for (;;) {
        int u = lcg_bits(st, 31);
        int v = u % bound;
        /* Java evaluates u - v + (bound - 1) in wrapping 32-bit int arithmetic */
        if ((int32_t)((uint32_t)u - (uint32_t)v + (uint32_t)(bound - 1)) >= 0) return v;
    }
}
static inline uint64_t lcg_long(uint64_t *st) {                 /* rng.c:197-210: second half sign-extended */
    uint64_t hi = (uint64_t)(uint32_t)lcg_bits(st, 32);
    int64_t lo = (int64_t)lcg_bits(st, 32);
    return (hi << 32) + (uint64_t)lo;
}

void wo_hut_in_region(uint64_t seed, int rx, int rz, int salt, int *cx, int *cz) {
    uint64_t s = (uint64_t)rx * 341873128712ULL + (uint64_t)rz * 132897987541ULL + seed +
                 (uint64_t)(int64_t)salt;
    uint64_t st = (s ^ LCG_MUL) & LCG_MASK;
    int j = lcg_int(&st, 24);
    int k = lcg_int(&st, 24);
    *cx = rx * 32 + j;
    *cz = rz * 32 + k;
}

int wo_orientation(uint64_t seed, int hut_x, int hut_z) {      /* eval.c:41-50, structure.c:33-42 */
    uint64_t st = (seed ^ LCG_MUL) & LCG_MASK;
    uint64_t a = lcg_long(&st);
    uint64_t b = lcg_long(&st);
    uint64_t s = ((uint64_t)(int64_t)(hut_x >> 4) * a) ^ ((uint64_t)(int64_t)(hut_z >> 4) * b) ^ seed;
    st = (s ^ LCG_MUL) & LCG_MASK;
    return lcg_int(&st, 4);
}

/* ------------------------------------------------------------------ */
/* Noise parameter table (game data; the values of noise_table.h)      */
/* ------------------------------------------------------------------ */
typedef struct { const char *id; int first; int n; double amp[9]; } noise_def;
static const noise_def NOISES[] = {
    {"minecraft:temperature", -10, 6, {1.5, 0, 1, 0, 0, 0}},
    {"minecraft:continentalness", -9, 9, {1, 1, 2, 2, 2, 1, 1, 1, 1}},
    {"minecraft:erosion", -9, 5, {1, 1, 0, 1, 1}},
    {"minecraft:temperature_large", -12, 6, {1.5, 0, 1, 0, 0, 0}},
    {"minecraft:continentalness_large", -11, 9, {1, 1, 2, 2, 2, 1, 1, 1, 1}},
    {"minecraft:erosion_large", -11, 5, {1, 1, 0, 1, 1}},
    {"minecraft:ridge", -7, 6, {1, 2, 1, 0, 0, 0}},
    {"minecraft:aquifer_fluid_level_floodedness", -7, 1, {1}},
    {"minecraft:spaghetti_3d_1", -7, 1, {1}},
    {"minecraft:spaghetti_3d_2", -7, 1, {1}},
    {"minecraft:spaghetti_3d_rarity", -11, 1, {1}},
    {"minecraft:spaghetti_3d_thickness", -8, 1, {1}},
    {"minecraft:spaghetti_roughness", -5, 1, {1}},
    {"minecraft:spaghetti_roughness_modulator", -8, 1, {1}},
    {"minecraft:cave_entrance", -7, 3, {0.4, 0.5, 1}},
    {"minecraft:cave_layer", -8, 1, {1}},
    {"minecraft:cave_cheese", -8, 9, {0.5, 1, 2, 1, 2, 1, 0, 2, 0}},
};
#define N_NOISES ((int)(sizeof(NOISES) / sizeof(NOISES[0])))

/* ------------------------------------------------------------------ */
/* Perlin / Octave / DoublePerlin (noise.c:61-156)                     */
/* ------------------------------------------------------------------ */
#define MAXOCT 9
typedef struct {
    double ox, oy, oz;
    uint8_t perm[256];
    int present;
    int jy;                 /* y=0 constants (noise.c:73-77) */
    double hy, hy1, fy;
} perlin_t;
typedef struct {
    int n;
    double lac, per;
    double amp[MAXOCT];
    perlin_t oct[MAXOCT];
} octave_t;
typedef struct {
    double amplitude;
    octave_t sub[2];
} dbl_t;

static inline double fade(double d) { return d * d * d * (d * (d * 6.0 - 15.0) + 10.0); }

static void perlin_build(perlin_t *p, xr_t *r) {               /* noise.c:61-78 */
    p->ox = xr_double(r) * 256.0;
    p->oy = xr_double(r) * 256.0;
    p->oz = xr_double(r) * 256.0;
    for (int i = 0; i < 256; i++) p->perm[i] = (uint8_t)i;
    for (int i = 0; i < 256; i++) {
        int j = xr_bounded(r, 256 - i);
        uint8_t t = p->perm[i];
        p->perm[i] = p->perm[i + j];
        p->perm[i + j] = t;
    }
    p->present = 1;
    p->jy = (int)floor(p->oy);
    p->hy = p->oy - p->jy;
    p->hy1 = p->hy - 1.0;
    p->fy = fade(p->hy);
}

static void octave_build(octave_t *o, xr_t *r, const noise_def *d) { /* noise.c:80-109 */
    o->n = d->n;
    memcpy(o->amp, d->amp, sizeof(double) * (size_t)d->n);
    o->lac = pow(2.0, (double)d->first);
    o->per = pow(2.0, (double)(d->n - 1)) / (pow(2.0, (double)d->n) - 1.0);
    xr_t fork;
    xr_fork(&fork, r);
    for (int i = 0; i < d->n; i++) {
        o->oct[i].present = 0;
        if (d->amp[i] == 0.0) continue;
        char name[32];
        snprintf(name, sizeof(name), "octave_%d", d->first + i);
        xr_t per;
        xr_named(&per, &fork, name);
        perlin_build(&o->oct[i], &per);
    }
}

static const noise_def *find_noise(const char *id) {
    for (int i = 0; i < N_NOISES; i++)
        if (!strcmp(NOISES[i].id, id)) return &NOISES[i];
    return NULL;
}

static int dbl_build(dbl_t *dn, uint64_t seed, const char *id) { /* noise.c:111-143 */
    const noise_def *d = find_noise(id);
    if (!d) { memset(dn, 0, sizeof(*dn)); return -1; }
    xr_t r, fork, per;
    xr_seed(&r, seed);
    xr_fork(&fork, &r);
    xr_named(&per, &fork, d->id);
    octave_build(&dn->sub[0], &per, d);
    octave_build(&dn->sub[1], &per, d);
    int lo = -1, hi = -1;
    for (int i = 0; i < d->n; i++)
        if (d->amp[i] != 0.0) { if (lo < 0) lo = i; hi = i; }
    double span = (double)(hi - lo);
    dn->amplitude = 0.16666666666666666 / (0.1 * (1.0 + 1.0 / (span + 1.0)));
    return 0;
}

static inline double keep_precision(double v) {                /* noise.c:31-34 */
    if (v > -1.0e7 && v < 1.0e7) return v;
    return v - (double)(long)floor(v * 2.9802322387695312E-08 + 0.5) * 3.3554432E7;
}
static const int GRAD[16][3] = {
    {1, 1, 0}, {-1, 1, 0}, {1, -1, 0}, {-1, -1, 0}, {1, 0, 1}, {-1, 0, 1}, {1, 0, -1}, {-1, 0, -1},
    {0, 1, 1}, {0, -1, 1}, {0, 1, -1}, {0, -1, -1}, {1, 1, 0}, {0, -1, 1}, {-1, 1, 0}, {0, -1, -1}};
static inline double grad(int h, double x, double y, double z) { /* noise.c:52-55 */
    const int *g = GRAD[h & 15];
    return (double)g[0] * x + (double)g[1] * y + (double)g[2] * z;
}
static inline double lerp(double t, double a, double b) { return a + t * (b - a); }

/* The 8 corner gradients and trilinear blend (noise.c:224-244, 292-318). */
static inline double perlin_core(const uint8_t *P, int i, int j, int k, double x, double y, double y1,
                                 double z, double fx, double fy, double fz) {
    int a = P[i & 255], b = P[(i + 1) & 255];
    int c = P[(a + j) & 255], d = P[(a + j + 1) & 255];
    int e = P[(b + j) & 255], f = P[(b + j + 1) & 255];
    double v000 = grad(P[(c + k) & 255], x, y, z);
    double v100 = grad(P[(e + k) & 255], x - 1, y, z);
    double v010 = grad(P[(d + k) & 255], x, y1, z);
    double v110 = grad(P[(f + k) & 255], x - 1, y1, z);
    double v001 = grad(P[(c + k + 1) & 255], x, y, z - 1);
    double v101 = grad(P[(e + k + 1) & 255], x - 1, y, z - 1);
    double v011 = grad(P[(d + k + 1) & 255], x, y1, z - 1);
    double v111 = grad(P[(f + k + 1) & 255], x - 1, y1, z - 1);
    double x00 = lerp(fx, v000, v100), x10 = lerp(fx, v010, v110);
    double x01 = lerp(fx, v001, v101), x11 = lerp(fx, v011, v111);
    return lerp(fz, lerp(fy, x00, x10), lerp(fy, x01, x11));
}

static double perlin_y0(const perlin_t *p, double x, double z) {
    double d = x + p->ox, f = z + p->oz;
    int i = (int)floor(d), k = (int)floor(f);
    double g = d - i, l = f - k;
    return perlin_core(p->perm, i, p->jy, k, g, p->hy, p->hy1, l, fade(g), p->fy, fade(l));
}

static double perlin_3d(const perlin_t *p, double x, double y, double z) { /* noise.c:246-261, y_scale 0 */
    double d = x + p->ox, e = y + p->oy, f = z + p->oz;
    int i = (int)floor(d), j = (int)floor(e), k = (int)floor(f);
    double g = d - i, h = e - j, l = f - k;
    double hm = h - 0.0;
    return perlin_core(p->perm, i, j, k, g, hm, hm - 1, l, fade(g), fade(h), fade(l));
}

static double octave_y0(const octave_t *o, double x, double z) { /* noise.c:320-336 */
    double value = 0.0, lac = o->lac, per = o->per;
    for (int i = 0; i < o->n; i++) {
        if (o->oct[i].present) {
            double v = perlin_y0(&o->oct[i], keep_precision(x * lac), keep_precision(z * lac));
            value += (o->amp[i] * v) * per;
        }
        lac *= 2.0;
        per /= 2.0;
    }
    return value;
}

static double octave_3d(const octave_t *o, double x, double y, double z) { /* noise.c:263-281 */
    double value = 0.0, lac = o->lac, per = o->per;
    for (int i = 0; i < o->n; i++) {
        if (o->oct[i].present) {
            double v = perlin_3d(&o->oct[i], keep_precision(x * lac), keep_precision(y * lac),
                                 keep_precision(z * lac));
            value += (o->amp[i] * v) * per;
        }
        lac *= 2.0;
        per /= 2.0;
    }
    return value;
}

#define DSCALE 1.0181268882175227
static double dbl_y0(const dbl_t *dn, double x, double z) {    /* noise.c:338-342 */
    return (octave_y0(&dn->sub[0], x, z) + octave_y0(&dn->sub[1], x * DSCALE, z * DSCALE)) * dn->amplitude;
}
static double dbl_3d(const dbl_t *dn, double x, double y, double z) { /* noise.c:285-289 */
    return (octave_3d(&dn->sub[0], x, y, z) + octave_3d(&dn->sub[1], x * DSCALE, y * DSCALE, z * DSCALE)) *
           dn->amplitude;
}

/* Tiered erosion exit (noise.c:387-459): interleaved 0A,0B,1A,1B,... partial sums with
 * weight amp*persistence, compared (times the amplitude) against the tier thresholds after
 * evaluations 1..7.  Returns the tier that rejected, or -1 when the value reaches >= 0.55. */
static const double TIER_THR[7] = {0.05, 0.22, 0.42, 0.45, 0.49, 0.51, 0.55};
static int erosion_tiered(const dbl_t *dn, double x, double z) {
    const octave_t *a = &dn->sub[0], *b = &dn->sub[1];
    double sum = 0.0, lac_a = a->lac, per_a = a->per, lac_b = b->lac, per_b = b->per;
    int k = 0, next = 0;
    for (int i = 0; i < a->n; i++) {
        if (a->oct[i].present) {
            for (int s = 0; s < 2; s++) {
                const octave_t *o = s ? b : a;
                double sc = s ? DSCALE : 1.0;
                double xs = s ? lac_b : lac_a;
                double w = s ? b->amp[i] * per_b : a->amp[i] * per_a;
                double v = perlin_y0(&o->oct[i], keep_precision(x * sc * xs), keep_precision(z * sc * xs));
                sum += w * v;
                if (k == next + 1) {
                    if (sum * dn->amplitude < TIER_THR[next]) return next;
                    if (++next >= 7) return -1;
                }
                k++;
            }
        }
        lac_a *= 2.0; per_a /= 2.0;
        lac_b *= 2.0; per_b /= 2.0;
    }
    return -1;
}

/* ------------------------------------------------------------------ */
/* Java Math / MathHelper helpers (mcmath.h)                           */
/* ------------------------------------------------------------------ */
static inline int negzero(double v) { uint64_t b; memcpy(&b, &v, 8); return b == 0x8000000000000000ULL; }
static inline double jmax(double a, double b) {
    if (a != a) return a;
    if (a == 0.0 && b == 0.0 && negzero(a)) return b;
    return (a >= b) ? a : b;
}
static inline double jmin(double a, double b) {
    if (a != a) return a;
    if (a == 0.0 && b == 0.0 && negzero(b)) return b;
    return (a <= b) ? a : b;
}
static inline double clampd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* ------------------------------------------------------------------ */
/* Phase-1 state and the cave heuristics (caves.c:65-130)              */
/* ------------------------------------------------------------------ */
typedef struct {
    dbl_t erosion, temperature, ridge, continentalness;
    dbl_t entrance, rarity, thickness, sp1, sp2, rmod, rough, layer, cheese, flood;
} p1_t;

static void p1_build(p1_t *p, uint64_t seed, int large) {     /* phase1.c:11-17, climate.c:8-15, caves.c:65-77 */
    dbl_build(&p->erosion, seed, large ? "minecraft:erosion_large" : "minecraft:erosion");
    dbl_build(&p->temperature, seed, large ? "minecraft:temperature_large" : "minecraft:temperature");
    dbl_build(&p->continentalness, seed, large ? "minecraft:continentalness_large" : "minecraft:continentalness");
    dbl_build(&p->ridge, seed, "minecraft:ridge");
    dbl_build(&p->entrance, seed, "minecraft:cave_entrance");
    dbl_build(&p->rarity, seed, "minecraft:spaghetti_3d_rarity");
    dbl_build(&p->thickness, seed, "minecraft:spaghetti_3d_thickness");
    dbl_build(&p->sp1, seed, "minecraft:spaghetti_3d_1");
    dbl_build(&p->sp2, seed, "minecraft:spaghetti_3d_2");
    dbl_build(&p->rmod, seed, "minecraft:spaghetti_roughness_modulator");
    dbl_build(&p->rough, seed, "minecraft:spaghetti_roughness");
    dbl_build(&p->layer, seed, "minecraft:cave_layer");
    dbl_build(&p->cheese, seed, "minecraft:cave_cheese");
    dbl_build(&p->flood, seed, "minecraft:aquifer_fluid_level_floodedness");
}

static inline double tunnel_scale(double v) {                  /* caves.c:41-46 */
    if (v < -0.5) return 0.75;
    if (v < 0.0) return 1.0;
    if (v < 0.5) return 1.5;
    return 2.0;
}
static double spaghetti(const p1_t *c, int x, int y, int z) {  /* caves.c:83-104 */
    double e = tunnel_scale(dbl_3d(&c->rarity, (double)(x * 2), (double)y, (double)(z * 2)));
    double tv = dbl_3d(&c->thickness, (double)x, (double)y, (double)z);
    double h = lerp((tv - -1.0) / (1.0 - -1.0), 0.065, 0.088);
    double l = dbl_3d(&c->sp1, (double)x / e, (double)y / e, (double)z / e);
    double m = fabs(e * l) - h;
    double n = dbl_3d(&c->sp2, (double)x / e, (double)y / e, (double)z / e);
    double o = fabs(e * n) - h;
    double p = clampd(jmax(m, o), -1.0, 1.0);
    double mod = dbl_3d(&c->rmod, (double)x, (double)y, (double)z);
    double rgh = dbl_3d(&c->rough, (double)x, (double)y, (double)z);
    double q = (-0.05 + (-0.05 * mod)) * (-0.4 + fabs(rgh));
    return p + q;
}
static double entrance(const p1_t *c, int x, int y, int z) {   /* caves.c:106-113 */
    double ent = dbl_3d(&c->entrance, (double)x * 0.75, (double)y * 0.5, (double)z * 0.75);
    double t = (10.0 + (double)y) / 40.0;
    double cl = t < 0.0 ? 0.3 : (t > 1.0 ? 0.0 : lerp(t, 0.3, 0.0));
    double cc = ent + 0.37 + cl;
    return jmin(cc, spaghetti(c, x, y, z));
}
static double cheese(const p1_t *c, int x, int y, int z) {     /* caves.c:122-130 */
    double layer = dbl_3d(&c->layer, (double)x, (double)(int)((uint32_t)y * 8u), (double)z);
    double a = 4.0 * layer * layer;
    double raw = dbl_3d(&c->cheese, (double)x, (double)y * 0.6666666666666666, (double)z);
    return a + clampd(0.27 + raw, -1.0, 1.0);
}
static double flood(const p1_t *c, int hut_x, int hut_z, int y) { /* phase1.c:32-35 */
    return dbl_3d(&c->flood, (double)(hut_x + 3), (double)y * 0.67, (double)(hut_z + 3));
}
static double climate(const dbl_t *n, int hut_x, int hut_z) {  /* phase1.c:28-30 */
    return dbl_y0(n, (hut_x + 8) / 4.0, (hut_z + 8) / 4.0);
}

/* phase1.c:95-200: returns the reject code (10 = accept); *tier = erosion tier or -1. */
static int p1_check(const p1_t *p, const wo_opts *o, int hut_x, int hut_z, int maxh, int *tier) {
    *tier = -1;
    if (!o->single_biome) {
        int t = erosion_tiered(&p->erosion, (hut_x + 8) / 4.0, (hut_z + 8) / 4.0);
        if (t >= 0) { *tier = t; return 0; }
        double tp = climate(&p->temperature, hut_x, hut_z);
        if (o->mc_1_18_2) { if (tp < -0.45) return 1; }
        else if (tp > 0.2 || tp < -0.45) return 1;
        double r = climate(&p->ridge, hut_x, hut_z);
        if ((r > 0.42 && r < 0.91) || (r < -0.42 && r > -0.91)) return 2;
        if (!o->pre_26_2 && r <= -0.91) return 2;
    }
    int hx = hut_x + 3, hz = hut_z + 3;
    if (entrance(p, hx, 50, hz) >= 0) return 3;
    if (entrance(p, hx, 60, hz) >= 0) return 4;
    if (spaghetti(p, hx, maxh, hz) >= 0 && cheese(p, hx, maxh, hz) >= 0) return 5;
    int floor_y = (-40 < maxh) ? -40 : maxh;
    if (floor_y < -50) floor_y = -50;
    for (int y = 0; y >= floor_y; y -= 10)
        if (maxh < y && spaghetti(p, hx, y, hz) >= 0 && cheese(p, hx, y, hz) >= 0) return 6;
    for (int y = 10; y <= 40; y += 10)
        if (entrance(p, hx, y, hz) >= 0 && cheese(p, hx, y, hz) >= 0) return 7;
    if (!o->single_biome && climate(&p->continentalness, hut_x, hut_z) < -0.11) return 8;
    for (int y = maxh; y <= 60; y += 10)
        if (flood(p, hut_x, hut_z, y) > 0.41) return 9;
    return 10;
}

/* ------------------------------------------------------------------ */
/* exported entry points                                               */
/* ------------------------------------------------------------------ */
int wo_noise_dump(uint64_t seed, const char *id, double *head, int *present, double *origin,
                  unsigned char *perm) {
    dbl_t *dn = (dbl_t *)calloc(1, sizeof(dbl_t));
    if (!dn) return -1;
    if (dbl_build(dn, seed, id)) { free(dn); return -2; }
    head[0] = dn->amplitude;
    head[1] = dn->sub[0].lac; head[2] = dn->sub[0].per;
    head[3] = dn->sub[1].lac; head[4] = dn->sub[1].per;
    head[5] = dn->sub[0].n;
    for (int s = 0; s < 2; s++)
        for (int i = 0; i < 16; i++) {
            int k = s * 16 + i;
            const perlin_t *p = (i < MAXOCT) ? &dn->sub[s].oct[i] : NULL;
            int pr = (p && i < dn->sub[s].n) ? p->present : 0;
            present[k] = pr;
            origin[3 * k] = pr ? p->ox : 0.0;
            origin[3 * k + 1] = pr ? p->oy : 0.0;
            origin[3 * k + 2] = pr ? p->oz : 0.0;
            if (pr) memcpy(perm + 256 * k, p->perm, 256);
            else memset(perm + 256 * k, 0, 256);
        }
    free(dn);
    return 0;
}

long long wo_phase1_rect(uint64_t seed, const wo_opts *o, int max_height, int salt,
                         int rx0, int rx1, int rz0, int rz1,
                         signed char *codes, signed char *tiers, int *cx, int *cz) {
    p1_t *p = (p1_t *)malloc(sizeof(p1_t));
    if (!p) return -1;
    p1_build(p, seed, o->large_biomes);
    long long k = 0;
    for (int rz = rz0; rz < rz1; rz++)
        for (int rx = rx0; rx < rx1; rx++, k++) {
            int x, z, t;
            wo_hut_in_region(seed, rx, rz, salt ? salt : 14357620, &x, &z);
            int code = p1_check(p, o, x * 16, z * 16, max_height, &t);
            if (codes) codes[k] = (signed char)code;
            if (tiers) tiers[k] = (signed char)t;
            if (cx) cx[k] = x;
            if (cz) cz[k] = z;
        }
    free(p);
    return k;
}

int wo_probe(uint64_t seed, const wo_opts *o, int hut_x, int hut_z, int maxh, double *out) { /* phase1.c:47-87 */
    p1_t *p = (p1_t *)malloc(sizeof(p1_t));
    if (!p) return -1;
    p1_build(p, seed, o->large_biomes);
    int hx = hut_x + 3, hz = hut_z + 3, k = 0;
    out[k++] = climate(&p->erosion, hut_x, hut_z);
    out[k++] = climate(&p->temperature, hut_x, hut_z);
    out[k++] = climate(&p->ridge, hut_x, hut_z);
    out[k++] = climate(&p->continentalness, hut_x, hut_z);
    out[k++] = entrance(p, hx, 50, hz);
    out[k++] = entrance(p, hx, 60, hz);
    out[k++] = spaghetti(p, hx, maxh, hz);
    out[k++] = cheese(p, hx, maxh, hz);
    for (int y = 0; y >= -40; y -= 10) { out[k++] = spaghetti(p, hx, y, hz); out[k++] = cheese(p, hx, y, hz); }
    for (int y = 10; y <= 40; y += 10) { out[k++] = entrance(p, hx, y, hz); out[k++] = cheese(p, hx, y, hz); }
    for (int y = -50; y <= 60; y += 10) out[k++] = flood(p, hut_x, hut_z, y);
    free(p);
    return k;
}

typedef struct {
    const uint64_t *seeds;
    uint64_t gen_base;
    long long n;
    const wo_opts *o;
    int maxh, salt, rx0, rx1, rz0, rz1;
    wo_candidate *out;
    long long cap;
    long long found;
    long long next;
    long long hist[11];
    pthread_mutex_t mu;
} scan_job;

static void *scan_worker(void *arg) {
    scan_job *j = (scan_job *)arg;
    p1_t *p = (p1_t *)malloc(sizeof(p1_t));
    long long hist[11] = {0};
    for (;;) {
        pthread_mutex_lock(&j->mu);
        long long i = j->next++;
        pthread_mutex_unlock(&j->mu);
        if (i >= j->n || !p) break;
        uint64_t seed = j->seeds ? j->seeds[i] : wo_splitmix64(j->gen_base + (uint64_t)i);
        p1_build(p, seed, j->o->large_biomes);
        for (int rz = j->rz0; rz < j->rz1; rz++)
            for (int rx = j->rx0; rx < j->rx1; rx++) {
                int x, z, t;
                wo_hut_in_region(seed, rx, rz, j->salt ? j->salt : 14357620, &x, &z);
                int code = p1_check(p, j->o, x * 16, z * 16, j->maxh, &t);
                hist[code]++;
                if (code != 10) continue;
                pthread_mutex_lock(&j->mu);
                long long slot = j->found++;
                if (slot < j->cap && j->out) {
                    wo_candidate *c = &j->out[slot];
                    c->seed_index = (uint64_t)i; c->seed = (int64_t)seed;
                    c->rx = rx; c->rz = rz; c->chunk_x = x; c->chunk_z = z;
                }
                pthread_mutex_unlock(&j->mu);
            }
    }
    pthread_mutex_lock(&j->mu);
    for (int k = 0; k < 11; k++) j->hist[k] += hist[k];
    pthread_mutex_unlock(&j->mu);
    free(p);
    return NULL;
}

long long wo_scan_seeds(const uint64_t *seeds, uint64_t gen_base, long long n, const wo_opts *o,
                        int max_height, int salt, int rx0, int rx1, int rz0, int rz1, int threads,
                        wo_candidate *out, long long cap, long long *reject_hist) {
    scan_job j;
    memset(&j, 0, sizeof(j));
    j.seeds = seeds; j.gen_base = gen_base; j.n = n; j.o = o;
    j.maxh = max_height; j.salt = salt;
    j.rx0 = rx0; j.rx1 = rx1; j.rz0 = rz0; j.rz1 = rz1;
    j.out = out; j.cap = cap;
    pthread_mutex_init(&j.mu, NULL);
    if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (threads < 1) threads = 1;
    pthread_t *th = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    for (int t = 0; t < threads; t++) pthread_create(&th[t], NULL, scan_worker, &j);
    for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
    free(th);
    pthread_mutex_destroy(&j.mu);
    if (reject_hist) memcpy(reject_hist, j.hist, sizeof(j.hist));
    return j.found;
}

/* ------------------------------------------------------------------ */
/* Deep Dive: mineshaft start chunks under swamp huts                  */
/* engine/gpu/room_core.h:34-73 (setLargeFeatureSeed + nextDouble()    */
/* < 0.004), :146-175 (the region walk)                                */
/* ------------------------------------------------------------------ */
int wo_mineshaft_start(uint64_t s48, int cx, int cz, uint64_t *carver_out) {
    const uint64_t S = s48 & LCG_MASK;
    uint64_t st = (S ^ LCG_MUL) & LCG_MASK;
    const uint64_t a = lcg_long(&st);
    const uint64_t b = lcg_long(&st);
    const uint64_t carver =
        ((uint64_t)((int64_t)cx * (int64_t)a) ^ (uint64_t)((int64_t)cz * (int64_t)b) ^ S) & LCG_MASK;
    if (carver_out) *carver_out = carver;
    st = (carver ^ LCG_MUL) & LCG_MASK;
    const int64_t hi = (int64_t)(uint32_t)lcg_bits(&st, 26);
    const int64_t lo = (int64_t)(uint32_t)lcg_bits(&st, 27);
    return (double)((hi << 27) + lo) * 1.1102230246251565404e-16 < 0.004;
}

long long wo_deep_starts(const uint64_t *s48s, long long n, int rx0, int rx1, int rz0, int rz1, int64_t *out,
                         long long cap) {
    long long found = 0;
    for (long long i = 0; i < n; i++) {
        const uint64_t S = s48s[i] & LCG_MASK;
        for (int rz = rz0; rz < rz1; rz++)
            for (int rx = rx0; rx < rx1; rx++) {
                int cx, cz;
                uint64_t carver;
                wo_hut_in_region(S, rx, rz, 14357620, &cx, &cz);
                if (!wo_mineshaft_start(S, cx, cz, &carver)) continue;
                if (found < cap) {
                    int64_t *o = out + 6 * found;
                    o[0] = (int64_t)S; o[1] = rx; o[2] = rz; o[3] = cx; o[4] = cz; o[5] = (int64_t)carver;
                }
                found++;
            }
    }
    return found;
}

/* ------------------------------------------------------------------ */
/* Deep Dive solver: the structure seeds S (48 bits) whose swamp hut   */
/* in region (rx, rz) lies at chunk offsets (ox, oz) and whose         */
/* setLargeFeatureSeed state at that chunk equals a layout value X.    */
/* Equations: engine/gpu/solver_kernels.cuh:15-115; task space:        */
/* engine/gpu/taskspace.h.  Restated independently: the low 20 bits of */
/* the LCG state t = S ^ 0x5DEECE66D by exhaustion (pruned by the hut  */
/* offsets' low 3 bits and the equation's low bits), the upper 28 by a */
/* bit-serial lifting of the low-32-bit equation, then a full check.   */
/* ------------------------------------------------------------------ */
#define SOLVE_C0 14357620ULL
#define SOLVE_C1 341873128712ULL
#define SOLVE_C2 132897987541ULL
#define M20 0xFFFFFULL

uint64_t wo_region_const(int rx, int rz) {
    return (SOLVE_C0 + (uint64_t)(int64_t)rx * SOLVE_C1 + (uint64_t)(int64_t)rz * SOLVE_C2) & LCG_MASK;
}

/* taskspace.h:27: the 20-bit group scramble (the group -> residue map hunt.py's ranges name) */
uint32_t wo_perm_group(uint32_t p) {
    uint32_t x = (uint32_t)((p * 0x9E3779B1u) & 0xFFFFFu);
    x ^= x >> 9;
    x = (x * 0x85EBCA6Bu) & 0xFFFFFu;
    x ^= x >> 7;
    return x & 0xFFFFFu;
}

/* taskspace.h:12-18: the rx / rz ranges of a regime (both signs for 1 and 2) */
static int regime_ranges(int regime, int64_t lo[2], int64_t hi[2]) {
    if (regime == 0) { lo[0] = -16384; hi[0] = 16383; return 1; }
    if (regime == 1) { lo[0] = -32768; hi[0] = -16385; lo[1] = 16384; hi[1] = 32767; return 2; }
    lo[0] = -58593; hi[0] = -32769; lo[1] = 32768; hi[1] = 58593; return 2;
}

/* Regions of a regime whose region constant has low 20 bits c20 (taskspace.h:29-39), by
 * scanning rz for every rx (no modular inverse: an independent check of the GPU's). */
long long wo_group_regions(uint32_t c20, int regime_x, int regime_z, int32_t *rx_out, int32_t *rz_out, long long cap) {
    int64_t xl[2], xh[2], zl[2], zh[2];
    const int nx = regime_ranges(regime_x, xl, xh), nz = regime_ranges(regime_z, zl, zh);
    long long n = 0;
    for (int a = 0; a < nx; a++)
        for (int64_t rx = xl[a]; rx <= xh[a]; rx++) {
            const uint64_t base = (SOLVE_C0 + (uint64_t)rx * SOLVE_C1) & M20;
            for (int b = 0; b < nz; b++)
                for (int64_t rz = zl[b]; rz <= zh[b]; rz++) {
                    if (((base + (uint64_t)rz * SOLVE_C2) & M20) != c20) continue;
                    if (n < cap) { rx_out[n] = (int32_t)rx; rz_out[n] = (int32_t)rz; }
                    n++;
                }
        }
    return n;
}

/* The hut offsets of region constant creg under structure seed S (nextInt(24) twice, with the
 * JDK rejection): rcHutExact, engine/gpu/room_core.h:78-96. */
static void hut_offsets(uint64_t S, uint64_t creg, int *ox, int *oz) {
    uint64_t st = ((S + creg) ^ LCG_MUL) & LCG_MASK;
    *ox = lcg_int(&st, 24);
    *oz = lcg_int(&st, 24);
}

static uint64_t carver_state(uint64_t S, int cx, int cz) {
    uint64_t st = (S ^ LCG_MUL) & LCG_MASK;
    const uint64_t a = lcg_long(&st);
    const uint64_t b = lcg_long(&st);
    return ((uint64_t)((int64_t)cx * (int64_t)a) ^ (uint64_t)((int64_t)cz * (int64_t)b) ^ S) & LCG_MASK;
}

typedef struct {
    uint64_t X, creg, a2, k2, a4, k4;
    int cx, cz, ox, oz, m;
    uint64_t *out;
    long long n, cap;
} solve_ctx;

/* low 32 bits of (cx * a) ^ (cz * b) ^ S ^ X for the state t (only bits of t below 48 - 16
 * reach them): a and b agree with (A^2 t + K2) >> 16 and (A^4 t + K4) >> 16 in their low words */
static uint32_t eq_low(const solve_ctx *c, uint64_t t) {
    const uint32_t h2 = (uint32_t)((((c->a2 * t) + c->k2) & LCG_MASK) >> 16);
    const uint32_t h4 = (uint32_t)((((c->a4 * t) + c->k4) & LCG_MASK) >> 16);
    return ((uint32_t)c->cx * h2) ^ ((uint32_t)c->cz * h4) ^ (uint32_t)((t ^ LCG_MUL) & 0xFFFFFFFFu) ^ (uint32_t)c->X;
}

static void solve_verify(solve_ctx *c, uint64_t t) {
    const uint64_t S = (t ^ LCG_MUL) & LCG_MASK;
    if (carver_state(S, c->cx, c->cz) != c->X) return;
    int ox, oz;
    hut_offsets(S, c->creg, &ox, &oz);
    if (ox != c->ox || oz != c->oz) return;
    if (c->n < c->cap) c->out[c->n] = S;
    c->n++;
}

/* Bits of t below j are chosen and equation bits below j - 16 + m are zero.  Choosing bit j
 * settles equation bit j - 16 + m (the lowest bit the new term cx * A^2 * 2^(j-16) or
 * cz * A^4 * 2^(j-16) can reach); past bit 31 the remaining bits are free. */
static void solve_lift(solve_ctx *c, uint64_t t, int j) {
    const int kb = j - 16 + c->m;
    if (kb > 31) {
        for (uint64_t f = 0; f < (1ULL << (48 - j)); f++) solve_verify(c, t | (f << j));
        return;
    }
    for (uint64_t x = 0; x < 2; x++) {
        const uint64_t t1 = t | (x << j);
        if (!((eq_low(c, t1) >> kb) & 1u)) solve_lift(c, t1, j + 1);
    }
}

static int v2(uint32_t v) { int k = 0; if (!v) return 40; while (!(v & 1u)) { v >>= 1; k++; } return k; }

long long wo_solve_task(uint64_t X, int rx, int rz, int ox, int oz, uint64_t *out, long long cap) {
    solve_ctx c;
    memset(&c, 0, sizeof c);
    c.X = X & LCG_MASK;
    c.creg = wo_region_const(rx, rz);
    c.a2 = (LCG_MUL * LCG_MUL) & LCG_MASK;
    c.k2 = (0xBULL * (LCG_MUL + 1)) & LCG_MASK;
    c.a4 = (c.a2 * c.a2) & LCG_MASK;
    c.k4 = (0xBULL * (LCG_MUL * LCG_MUL * LCG_MUL + LCG_MUL * LCG_MUL + LCG_MUL + 1)) & LCG_MASK;
    c.cx = rx * 32 + ox;
    c.cz = rz * 32 + oz;
    c.ox = ox;
    c.oz = oz;
    const int vx = v2((uint32_t)c.cx), vz = v2((uint32_t)c.cz);
    c.m = vx < vz ? vx : vz;
    if (c.m > 8) return 0;   /* both offsets 0: no class (the reference's tiers leave it out) */
    c.out = out;
    c.cap = cap;
    const uint32_t low = (1u << (4 + c.m)) - 1u;
    for (uint64_t t20 = 0; t20 <= M20; t20++) {
        /* the hut offsets' low 3 bits come from state bits 17..19 of the region's first two draws */
        const uint64_t q0 = ((((t20 ^ LCG_MUL) & M20) + c.creg) ^ LCG_MUL) & M20;
        const uint64_t q1 = (q0 * LCG_MUL + 0xBULL) & M20;
        if ((int)(q1 >> 17) != (ox & 7)) continue;
        const uint64_t q2 = (q1 * LCG_MUL + 0xBULL) & M20;
        if ((int)(q2 >> 17) != (oz & 7)) continue;
        if (eq_low(&c, t20) & low) continue;
        solve_lift(&c, t20, 20);
    }
    return c.n;
}
