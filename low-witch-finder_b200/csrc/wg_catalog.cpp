// Host-side noise catalog; see wg_catalog.h.
#include "wg_catalog.h"

#include <cmath>
#include <cstdio>
#include <cstring>

namespace wg {

// The game's parameter table for the noises this engine samples (the values in the
// reference's engine/tools/lysh/src/noise_table.h: identifier, firstOctave, amplitudes).
static const NoiseDef kDefs[N_NOISE_COUNT] = {
    {"minecraft:erosion", -9, 5, {1, 1, 0, 1, 1}},
    {"minecraft:temperature", -10, 6, {1.5, 0, 1, 0, 0, 0}},
    {"minecraft:ridge", -7, 6, {1, 2, 1, 0, 0, 0}},
    {"minecraft:continentalness", -9, 9, {1, 1, 2, 2, 2, 1, 1, 1, 1}},
    {"minecraft:erosion_large", -11, 5, {1, 1, 0, 1, 1}},
    {"minecraft:temperature_large", -12, 6, {1.5, 0, 1, 0, 0, 0}},
    {"minecraft:continentalness_large", -11, 9, {1, 1, 2, 2, 2, 1, 1, 1, 1}},
    {"minecraft:cave_entrance", -7, 3, {0.4, 0.5, 1}},
    {"minecraft:spaghetti_3d_rarity", -11, 1, {1}},
    {"minecraft:spaghetti_3d_thickness", -8, 1, {1}},
    {"minecraft:spaghetti_3d_1", -7, 1, {1}},
    {"minecraft:spaghetti_3d_2", -7, 1, {1}},
    {"minecraft:spaghetti_roughness_modulator", -8, 1, {1}},
    {"minecraft:spaghetti_roughness", -5, 1, {1}},
    {"minecraft:cave_layer", -8, 1, {1}},
    {"minecraft:cave_cheese", -8, 9, {0.5, 1, 2, 1, 2, 1, 0, 2, 0}},
    {"minecraft:aquifer_fluid_level_floodedness", -7, 1, {1}},
};

const NoiseDef &noise_def(int id) { return kDefs[id]; }

static uint32_t rol(uint32_t x, int n) { return (x << n) | (x >> (32 - n)); }

void md5(const uint8_t *data, uint64_t len, uint8_t out[16]) {
    static const int S[4][4] = {{7, 12, 17, 22}, {5, 9, 14, 20}, {4, 11, 16, 23}, {6, 10, 15, 21}};
    uint32_t K[64];
    for (int i = 0; i < 64; i++) K[i] = (uint32_t)(std::fabs(std::sin((double)(i + 1))) * 4294967296.0);
    uint32_t h[4] = {0x67452301u, 0xefcdab89u, 0x98badcfeu, 0x10325476u};
    uint64_t nblk = (len + 9 + 63) / 64;
    for (uint64_t blk = 0; blk < nblk; blk++) {
        uint8_t b[64];
        for (int t = 0; t < 64; t++) {
            uint64_t pos = blk * 64 + (uint64_t)t;
            uint8_t v = 0;
            if (pos < len) v = data[pos];
            else if (pos == len) v = 0x80;
            else if (pos >= nblk * 64 - 8) v = (uint8_t)((len * 8) >> (8 * (pos - (nblk * 64 - 8))));
            b[t] = v;
        }
        uint32_t w[16];
        for (int t = 0; t < 16; t++)
            w[t] = (uint32_t)b[4 * t] | ((uint32_t)b[4 * t + 1] << 8) | ((uint32_t)b[4 * t + 2] << 16) |
                   ((uint32_t)b[4 * t + 3] << 24);
        uint32_t a = h[0], bb = h[1], c = h[2], d = h[3];
        for (int i = 0; i < 64; i++) {
            uint32_t f;
            int g;
            if (i < 16) { f = (bb & c) | (~bb & d); g = i; }
            else if (i < 32) { f = (d & bb) | (~d & c); g = (5 * i + 1) & 15; }
            else if (i < 48) { f = bb ^ c ^ d; g = (3 * i + 5) & 15; }
            else { f = c ^ (bb | ~d); g = (7 * i) & 15; }
            uint32_t nb = bb + rol(a + f + K[i] + w[g], S[i >> 4][i & 3]);
            a = d; d = c; c = bb; bb = nb;
        }
        h[0] += a; h[1] += bb; h[2] += c; h[3] += d;
    }
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) out[4 * i + j] = (uint8_t)(h[i] >> (8 * j));
}

static void digest_be(const char *s, uint64_t *lo, uint64_t *hi) {
    uint8_t d[16];
    md5((const uint8_t *)s, std::strlen(s), d);
    uint64_t a = 0, b = 0;
    for (int i = 0; i < 8; i++) a = (a << 8) | d[i];
    for (int i = 8; i < 16; i++) b = (b << 8) | d[i];
    *lo = a;
    *hi = b;
}

void build_noise_specs(NoiseSpec *specs) {
    for (int k = 0; k < N_NOISE_COUNT; k++) {
        const NoiseDef &d = kDefs[k];
        NoiseSpec &s = specs[k];
        std::memset(&s, 0, sizeof(s));
        digest_be(d.id, &s.name_lo, &s.name_hi);
        s.first_octave = d.first_octave;
        // Running lacunarity / persistence exactly as the octave loop computes them
        // (engine/tools/lysh/src/noise.c:85-86, 277-278): every slot doubles / halves,
        // including zero-amplitude slots.
        double lac = std::pow(2.0, (double)d.first_octave);
        double per = std::pow(2.0, (double)(d.n - 1)) / (std::pow(2.0, (double)d.n) - 1.0);
        int lo = -1, hi = -1, np = 0;
        for (int i = 0; i < d.n; i++) {
            if (d.amps[i] != 0.0) {
                char name[32];
                std::snprintf(name, sizeof(name), "octave_%d", d.first_octave + i);
                digest_be(name, &s.oct_lo[np], &s.oct_hi[np]);
                s.amp[np] = d.amps[i];
                s.lac[np] = lac;
                s.per[np] = per;
                s.octave[np] = i;
                np++;
                if (lo < 0) lo = i;
                hi = i;
            }
            lac *= 2.0;
            per /= 2.0;
        }
        s.npresent = np;
        double span = (double)(hi - lo);
        s.amplitude = 0.16666666666666666 / (0.1 * (1.0 + 1.0 / (span + 1.0)));
    }
}

}  // namespace wg
