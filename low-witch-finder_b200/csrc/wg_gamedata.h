// Game data tables the phase-2 kernels need, taken from the reference's generated headers when
// the library is built (never copied into this repository):
//
//   terrain spline tree   engine/tools/lysh/src/terrain_table.h  (offset / factor / peaks roots)
//   Mth.SIN table         engine/tools/lysh/src/sin_table.h      (65,536 floats)
//   biome R-trees         engine/tools/lysh/src/biome_trees.h    (one tree per game version)
//   noise parameters      engine/tools/lysh/src/noise_table.h    (firstOctave + amplitudes)
//
// wg_gamedata.cpp is compiled with -I pointing at the reference's lysh sources.  A build
// without them defines WG_NO_GAMEDATA and every phase-2 entry point then fails with a clear
// error instead of computing anything.
#pragma once

#include <cstdint>

namespace wg {

// One spline node (terrain_table.h's lysh_spline_node, field for field).
struct SplineNode {
    int kind;      // 0 = spline with n points, 1 = constant
    int coord;     // 0 continentalness, 1 erosion, 2 normalized weirdness, 3 weirdness
    int n;         // number of points
    int loc;       // first location in the float pool
    int der;       // first derivative in the float pool
    int child;     // first child index in the child pool
    float constant;
};

struct BiomeTree {
    const int16_t *range;    // 12 values per node: (min, max) of the six climate parameters
    const uint8_t *kids;     // child count per node (0 = leaf)
    const uint8_t *biome;    // biome id of a leaf
    const uint16_t *end;     // index just past the node's subtree
    int n_nodes;
};

// One noise parameter set (noise_table.h's lysh_noise_def, field for field).
struct GameNoise {
    const char *id;
    int first_octave;
    int n;
    const double *amps;
};

constexpr int kBiomeTrees = 8;
constexpr int kSinEntries = 65536;

struct GameData {
    bool available;
    const SplineNode *nodes;
    int n_nodes;
    const float *floats;
    int n_floats;
    const int *child;
    int n_child;
    int root_offset, root_factor, root_peak;
    const float *sin_table;  // kSinEntries
    BiomeTree trees[kBiomeTrees];
    const GameNoise *noises;
    int n_noises;
};

const GameData &game_data();

}  // namespace wg
