// Build-time game data; see wg_gamedata.h.  With WG_NO_GAMEDATA (the reference's lysh sources
// were not found when the library was built) the tables are absent and available == false.
#include "wg_gamedata.h"

#include <cstddef>
#include <cstring>

#ifndef WG_NO_GAMEDATA
#include <stdint.h>
#include <string.h>

#include "biome_trees.h"
#include "noise_table.h"
#include "sin_table.h"
#include "terrain_table.h"
#endif

namespace wg {

#ifndef WG_NO_GAMEDATA
static_assert(sizeof(lysh_spline_node) == sizeof(SplineNode), "spline node layout");
static_assert(offsetof(lysh_spline_node, constant) == offsetof(SplineNode, constant), "spline node layout");
static_assert(sizeof(lysh_noise_def) == sizeof(GameNoise), "noise def layout");
static_assert(offsetof(lysh_noise_def, amps) == offsetof(GameNoise, amps), "noise def layout");

#define WG_TREE(k)                                                                                  \
    BiomeTree {                                                                                     \
        &gtree##k##_range[0][0], gtree##k##_kids, gtree##k##_biome, gtree##k##_end,                  \
            (int)(sizeof(gtree##k##_kids) / sizeof(gtree##k##_kids[0]))                             \
    }

static GameData make_game_data() {
    GameData g;
    std::memset(&g, 0, sizeof(g));
    g.available = true;
    g.nodes = reinterpret_cast<const SplineNode *>(LYSH_TERRAIN_NODES);
    g.n_nodes = (int)(sizeof(LYSH_TERRAIN_NODES) / sizeof(LYSH_TERRAIN_NODES[0]));
    g.floats = LYSH_TERRAIN_FLOATS;
    g.n_floats = (int)(sizeof(LYSH_TERRAIN_FLOATS) / sizeof(LYSH_TERRAIN_FLOATS[0]));
    g.child = LYSH_TERRAIN_CHILD;
    g.n_child = (int)(sizeof(LYSH_TERRAIN_CHILD) / sizeof(LYSH_TERRAIN_CHILD[0]));
    g.root_offset = LYSH_TERRAIN_SURFACE_OFFSET;
    g.root_factor = LYSH_TERRAIN_SURFACE_FACTOR;
    g.root_peak = LYSH_TERRAIN_SURFACE_PEAK;
    g.sin_table = LYSH_MC_SIN;
    static_assert(LYSH_TREE_COUNT == kBiomeTrees, "biome tree count");
    const BiomeTree t[kBiomeTrees] = {WG_TREE(0), WG_TREE(1), WG_TREE(2), WG_TREE(3),
                                      WG_TREE(4), WG_TREE(5), WG_TREE(6), WG_TREE(7)};
    for (int k = 0; k < kBiomeTrees; k++) g.trees[k] = t[k];
    g.noises = reinterpret_cast<const GameNoise *>(LYSH_NOISE_TABLE);
    g.n_noises = (int)LYSH_NOISE_TABLE_N;
    return g;
}
#undef WG_TREE
#else
static GameData make_game_data() {
    GameData g;
    std::memset(&g, 0, sizeof(g));
    g.available = false;
    return g;
}
#endif

const GameData &game_data() {
    static const GameData g = make_game_data();
    return g;
}

}  // namespace wg
