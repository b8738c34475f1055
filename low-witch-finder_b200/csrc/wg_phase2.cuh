// Phase 2 (the confirmation of a phase-1 survivor) on the GPU: shared definitions between the
// kernels (wg_phase2.cu) and the host engine (wg_p2engine.cu).
//
// Phase 2 restates lysh_eval_hut (engine/tools/lysh/src/eval.c:121-242) for one hut at a time:
// orientation, the real biome gate at the chunk centre, the aquifer flood test of the 63
// footprint columns at y = 62, and the footprint's post-carver surface heights.  Everything it
// reads lies in ONE chunk, the hut's (the footprint starts at the chunk origin and is at most
// 9 blocks wide), so the work is organised per "job" = (world seed, hut chunk):
//
//   world     all Perlin tables of one seed that phase 2 samples: 31 DoublePerlin noises and
//             the 40 legacy octaves of the blended base noise (~50 KB in HBM); one thread per
//             table (p2_legacy_kernel walks the blended noise's shared RNG stream first).
//   grid      the chunk's `interpolated` corner columns: 5 x 5 columns x 49 cell heights of
//             the base density and the three interpolated noodle children.
//   aquifer   the chunk's 3 x 35 x 3 aquifer cells (anchor position + fluid status) and
//             skipSamplingAboveY, all computed up front (the reference memoises them lazily;
//             the values are the same).
//   carve     the 289-origin cave / canyon carver walk over the chunk (cell states in shared
//             memory; every ellipsoid's cells carved by the warp's lanes in parallel).
//   finish    biome gate, wet columns, pre- and post-carver heights, the verdict.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "wg_device.cuh"
#include "wg_gamedata.h"

namespace wg {

// DoublePerlin noises phase 2 samples.  The four climate noises with a *_large variant take
// that variant's parameters under LARGE_BIOMES.
enum P2Noise : int {
    Q_OFFSET = 0,
    Q_CONT,
    Q_EROSION,
    Q_RIDGE,
    Q_TEMPERATURE,
    Q_VEGETATION,
    Q_JAGGED,
    Q_ENTRANCE,
    Q_ROUGH,
    Q_ROUGH_MOD,
    Q_SP3D_1,
    Q_SP3D_2,
    Q_SP3D_RARITY,
    Q_SP3D_THICK,
    Q_SP2D,
    Q_SP2D_ELEV,
    Q_SP2D_MOD,
    Q_SP2D_THICK,
    Q_PILLAR,
    Q_PILLAR_RARE,
    Q_PILLAR_THICK,
    Q_LAYER,
    Q_CHEESE,
    Q_NOODLE,
    Q_NOODLE_THICK,
    Q_NOODLE_RA,
    Q_NOODLE_RB,
    Q_AQ_BARRIER,
    Q_AQ_FLOOD,
    Q_AQ_SPREAD,
    Q_AQ_LAVA,
    Q_COUNT
};

constexpr int kP2MaxOct = 16;
constexpr int kLegacyPerlins = 40;   // blended noise: min limit 16, max limit 16, main 8

// Sampling parameters of one noise (present octaves only, increasing octave order).
struct P2Spec {
    double amp[kP2MaxOct], lac[kP2MaxOct], per[kP2MaxOct];
    double amplitude;
    int npresent;
    int first_slot;   // world slot of (sub 0, octave 0); sub 1 follows at first_slot + npresent
};

// Name digests for building one noise's tables.
struct P2Digest {
    uint64_t name_lo, name_hi;
    uint64_t oct_lo[kP2MaxOct], oct_hi[kP2MaxOct];
};

struct P2Perlin {
    double ox, oy, oz;
    uint8_t perm[256];
};

// Seed-independent phase-2 tables, one copy per device (global memory).
struct P2Tables {
    P2Spec spec[2][Q_COUNT];       // [large biomes][noise]
    P2Digest digest[2][Q_COUNT];
    uint64_t terrain_lo, terrain_hi;   // MD5("minecraft:terrain"): the blended noise's random
    uint64_t aquifer_lo, aquifer_hi;   // MD5("minecraft:aquifer"): the aquifer's positional random
    int n_slots;                   // DoublePerlin slots; the legacy octaves follow
    int16_t slot_noise[256];       // per slot: noise, sub, present-octave index
    int8_t slot_sub[256];
    int8_t slot_oct[256];
    // game data (wg_gamedata.h), device copies
    const SplineNode *nodes;
    const float *floats;
    const int *child;
    int root_offset, root_factor, root_peak;
    // Mth.SIN as a quarter wave: entries 0..16384 (padded to kSinQuarterPad); the host checks that
    // they and sin_half_turn (entry 32768) rebuild all 65,536 entries bit for bit
    // the legacy octaves' start-state jumps: for octave k, 128 rows of two words whose parity with
    // the 128-bit Xoroshiro state (lo = bits 0..63) gives bit b of the state 259 k steps later
    const uint64_t *legacy_jump;
    const float *sin_quarter;
    float sin_half_turn;
    BiomeTree trees[kBiomeTrees];
};

constexpr int kSinQuarter = 16385, kSinQuarterPad = 16388;   // padded to whole 16-byte vectors
constexpr int kWorldSlotsMax = 192;
constexpr int kSplineDepth = 8;   // deepest spline nesting the evaluator holds (the game's is 5)
constexpr int kTreeDepth = 16;    // deepest biome R-tree the search holds

// One seed's phase-2 noise state.
struct P2World {
    uint64_t seed;
    int large;
    int pad;
    uint64_t aq_rand_lo, aq_rand_hi;          // the aquifer's positional random factory
    Xr legacy_rng[kLegacyPerlins];            // start states of the legacy octaves
    P2Perlin perl[kWorldSlotsMax];
};

// The chunk's interpolation grid and aquifer cells.
constexpr int kGridCols = 25;     // 5 x 5 corner columns, index gx * 5 + gz
constexpr int kGridYs = 49;       // y = -64 + 8 i
constexpr int kAqX = 3, kAqY = 35, kAqZ = 3, kAqCells = kAqX * kAqY * kAqZ;
constexpr int kCarveCells = 384 * 16 * 16;
// Column tops (lysh_preliminary_surface_level, a function of the quart column) around a chunk:
// quart x from 4 * chunk_x - 16, quart z from 4 * chunk_z - 8.  That covers the aquifer cells'
// 13 surface samples, the skipSamplingAboveY span and the flood test of a hut in the chunk.
constexpr int kTopX = 27, kTopZ = 19;

enum : int { BS_SOLID = 0, BS_AIR = 1, BS_WATER = 2, BS_LAVA = 3 };   // lysh_block_state order
enum : int { CV_UNCHANGED = 0, CV_AIR = 1, CV_WATER = 2, CV_LAVA = 3 };

struct P2Chunk {
    int world;                     // index into the world array
    int chunk_x, chunk_z;
    int max_psl;                   // highest column top around the chunk (INT_MIN before p2_tops_kernel)
    int min_gx, min_gy, min_gz;
    int carved;                    // cells[] holds the carver result
    double main[kGridCols][kGridYs];
    double noodle[3][kGridCols][kGridYs];
    int64_t aq_loc[kAqCells];
    int32_t aq_level[kAqCells];
    uint8_t aq_type[kAqCells];
    int16_t tops[kTopZ][kTopX];    // column tops, quart x - (4 * chunk_x - 16), quart z - (4 * chunk_z - 8)
    alignas(16) uint8_t cells[kCarveCells];   // CV_* per block, index (lz << 4 | lx) | (y + 64) << 8; copied as words
    // per block of the chunk (index as cells): the pre-carver state (lysh_phase2_block_at) in the
    // low nibble, the aquifer substance at density 0 in the high one (BS_* codes)
    alignas(16) uint8_t states[kCarveCells];
};
static_assert(offsetof(P2Chunk, cells) % 16 == 0, "carve cells are copied as 32-bit words");
static_assert(offsetof(P2Perlin, perm) % 4 == 0, "tables are written as 32-bit words");

// One hut to confirm and its result (the fields of lysh_hut_result, engine/tools/lysh/src/eval.h:63-85).
struct P2Hut {
    int job;                       // P2Chunk index
    int hut_x, hut_z;
    int max_y;
};

struct P2Result {
    int32_t hut_x, hut_z, rx, rz, dir, axis_z, size_x, size_z;
    int32_t avg_y, wet_columns, flooded, all_dry, ok, reject;
    int32_t biome_ok, biome_winner, biome_qx, biome_qy, biome_qz, biome_occ_y;
    int64_t sum_h;
    int64_t biome_t[6];
};

// Point probes (the parity interface); kinds for p2_probe_kernel.
enum : int {
    PR_BASE_NOISE = 0,   // blended base noise at block (x, y, z)
    PR_DENSITY_RAW,      // lysh_phase2_density_raw_at
    PR_COLUMN_TOP,       // lysh_preliminary_surface_level (x, z)
    PR_CONTINENTALNESS,  // terrain info at biome (x >> 2, z >> 2)
    PR_EROSION,
    PR_WEIRDNESS,
    PR_OFFSET_261,       // TerrainNoisePoint offset / factor / peaks (26.1 semantics)
    PR_FACTOR_261,
    PR_PEAKS_261,
    PR_FLUID,            // computeFluid(x, y, z): level * 4 + type
    PR_DENSITY,          // lysh_phase2_density_at (chunk job of (x, z))
    PR_BLOCK,            // lysh_phase2_block_at   (chunk job)
    PR_HEIGHT_PRE,       // lysh_phase2_height_pre_carver (chunk job)
    PR_HEIGHT,           // lysh_phase2_height (chunk job, carved)
    PR_GRID_MAIN,        // the chunk grid's stored corner value at the cell holding (x, y, z)
    PR_KINDS
};

void p2_launch_legacy(const P2Tables *T, P2World *worlds, int n_worlds, cudaStream_t s);
void p2_launch_build(const P2Tables *T, P2World *worlds, int n_worlds, cudaStream_t s);
void p2_launch_grid(const P2Tables *T, const P2World *worlds, P2Chunk *jobs, int n_jobs, cudaStream_t s);
void p2_launch_aquifer(const P2Tables *T, const P2World *worlds, P2Chunk *jobs, int n_jobs, cudaStream_t s);
void p2_launch_states(const P2Tables *T, const P2World *worlds, P2Chunk *jobs, int n_jobs, cudaStream_t s);
void p2_launch_carve(const P2Tables *T, const P2World *worlds, P2Chunk *jobs, int n_jobs, cudaStream_t s);
void p2_launch_finish(const P2Tables *T, const P2World *worlds, const P2Chunk *jobs, const P2Hut *huts,
                      int n_huts, int tree, P2Result *out, cudaStream_t s);
// Points: (world, x, y, z, job) per probe; out one double per point.
void p2_launch_probe(const P2Tables *T, const P2World *worlds, const P2Chunk *jobs, const int32_t *pts,
                     int n_pts, int kind, double *out, cudaStream_t s);

// biome_map raster and chunk-list passes (one world: worlds[0]).
void p2_launch_biome_map(const P2Tables *T, const P2World *worlds, int tree, int64_t x0, int64_t z0, int w, int h,
                         int step, int ss, int y, uint8_t *out, cudaStream_t s);
void p2_launch_biome_chunks(const P2Tables *T, const P2World *worlds, int tree, const int32_t *cx, const int32_t *cz,
                            int n, uint8_t *out, uint8_t *need, cudaStream_t s);
// Biome winner per point (world, x, z, y) of pts (4 ints per point): the finisher's biome_at.
void p2_launch_biome_points(const P2Tables *T, const P2World *worlds, int tree, const int32_t *pts, int n,
                            int32_t *out, cudaStream_t s);

}  // namespace wg
