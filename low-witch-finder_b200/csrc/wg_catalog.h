// Noise catalog: the game's DoublePerlin parameters for every noise on the Seed Check
// path, plus everything that can be derived from them once on the host (MD5 name digests,
// per-octave lacunarity / persistence, the DoublePerlin amplitude).  The device only ever
// sees the flattened NoiseSpec records below.
//
// Derivation chain restated here (engine/tools/lysh/src/noise.c:80-143, rng.c:145-165):
//   seed rng   = Xoroshiro128++(upgradeSeedTo128bit(worldSeed))
//   seed fork  = (next, next) of the seed rng                      (createRandomDeriver)
//   noise rng  = seed fork ^ MD5("minecraft:<name>")               (createRandom(String))
//   sub s fork = (next, next) of the noise rng, s = 0 then 1
//   octave rng = sub fork ^ MD5("octave_<firstOctave + i>")        for every non-zero amp
#pragma once

#include <cstdint>

namespace wg {

constexpr int kMaxOct = 9;

// Noise indices used by the kernels.  The *_LARGE entries replace erosion / temperature /
// continentalness under the LARGE_BIOMES preset (engine/tools/lysh/src/climate.c:8-15).
enum NoiseId : int {
    N_EROSION = 0,
    N_TEMPERATURE,
    N_RIDGE,
    N_CONTINENTALNESS,
    N_EROSION_LARGE,
    N_TEMPERATURE_LARGE,
    N_CONTINENTALNESS_LARGE,
    N_CAVE_ENTRANCE,
    N_SPAGHETTI_RARITY,
    N_SPAGHETTI_THICKNESS,
    N_SPAGHETTI_1,
    N_SPAGHETTI_2,
    N_ROUGHNESS_MODULATOR,
    N_ROUGHNESS,
    N_CAVE_LAYER,
    N_CAVE_CHEESE,
    N_FLOODEDNESS,
    N_NOISE_COUNT
};

// One DoublePerlin noise, flattened for the device.  Octave arrays list only the octaves
// whose amplitude is non-zero, in increasing octave order; lac/per are the running
// lacunarity / persistence values the game's octave loop holds at that octave.
struct NoiseSpec {
    uint64_t name_lo, name_hi;          // big-endian halves of MD5("minecraft:<name>")
    uint64_t oct_lo[kMaxOct];           // big-endian halves of MD5("octave_<n>")
    uint64_t oct_hi[kMaxOct];
    double amp[kMaxOct];
    double lac[kMaxOct];
    double per[kMaxOct];
    double amplitude;                    // 1/6 / (0.1 * (1 + 1/(span + 1)))
    int npresent;                        // non-zero amplitudes (octaves built per sub)
    int first_octave;
    int octave[kMaxOct];                 // slot index i of each present octave
};

// Fills specs[N_NOISE_COUNT].
void build_noise_specs(NoiseSpec *specs);

// RFC 1321 MD5 (used only for the name digests above).
void md5(const uint8_t *data, uint64_t len, uint8_t out[16]);

// The raw table entry (game data) a spec was built from.
struct NoiseDef {
    const char *id;
    int first_octave;
    int n;
    double amps[kMaxOct];
};
const NoiseDef &noise_def(int id);

}  // namespace wg
