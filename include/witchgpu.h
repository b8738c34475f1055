/* witchgpu.h -- C ABI of the B200 Seed Check engine (libwitchgpu.so).
 *
 * Plain C types only: opaque engine handle, caller-owned buffers, int status returns
 * (WG_OK = 0), no exit() inside the library.  One engine owns one CUDA context binding,
 * one stream and its work buffers; an engine is not thread-safe (use one per thread),
 * matching the one-ctx-per-thread rule of the reference's lysh API
 * (engine/tools/lysh/src/eval.h:40-47).
 *
 * Each entry point names the reference interface it replaces.
 */
#ifndef WITCHGPU_H
#define WITCHGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define WG_OK           0
#define WG_ERR_ARG      1   /* invalid argument (empty rect, null buffer, unknown name) */
#define WG_ERR_CUDA     2   /* a CUDA call failed; wg_engine_error() has the message */
#define WG_ERR_NOMEM    3   /* device or host allocation failed */
#define WG_ERR_CAPACITY 4   /* a work list stayed full even at the smallest batch */
#define WG_ERR_NODEV    5   /* no CUDA device / the requested device is absent */

typedef struct wg_engine wg_engine;

/* Version / preset bits; field-for-field the layout of lysh_phase1_opts
 * (engine/tools/lysh/src/phase1.h:45-57).  All-zero = 26.2 rules, NORMAL preset. */
typedef struct {
    int mc_1_18_2;      /* temperature gate: lower bound only */
    int single_biome;   /* SINGLE_BIOME preset: climate / continentalness gates skipped */
    int pre_26_2;       /* 1 = rules before 26.2 (no ridge <= -0.91 rejection) */
    int large_biomes;   /* LARGE_BIOMES preset: *_large climate noises */
    int biome_tree;     /* 0 = chosen from the bits above, else 1 + biome tree index */
} wg_opts;

/* One phase-1 survivor: a (seed, swamp-hut region) that passed every phase-1 gate.
 * The hut's block position is (chunk_x * 16, chunk_z * 16). */
typedef struct {
    uint64_t seed_index;   /* index of the seed in the request (list position / generator step) */
    int64_t seed;          /* world seed */
    int32_t rx, rz;        /* region */
    int32_t chunk_x, chunk_z;
} wg_candidate;

/* Funnel and timing of one Seed Check request. */
typedef struct {
    int64_t scanned;              /* (seed, region) checks */
    int64_t accepted;             /* phase-1 survivors */
    int64_t climate_survivors;    /* passed erosion / temperature / ridge */
    int64_t deep_candidates;      /* also passed Entrance(50) and Entrance(60) */
    int64_t reject_hist[11];      /* per LYSH_P1_REJECT_* code; [10] = accepted */
    int64_t tier_hist[7];         /* erosion tier that rejected (lysh's tier histogram) */
    int64_t batches;              /* device batches run */
    int64_t retries;              /* batches re-run smaller after a full work list */
    int64_t kernel_launches[3];   /* climate, entrance, ladder kernel launches */
    double kernel_ms[3];          /* their summed device time (CUDA events around each launch) */
    double gpu_ms;                /* device time of the whole call, CUDA events on its stream */
    double wall_ms;               /* host wall time of the call */
    int64_t rechecks;             /* FP32 noise core: climate gate decisions re-taken in FP64 */
    int64_t records;              /* seed units with climate survivors (tables the entrance kernel builds / 18) */
} wg_scan_stats;

/* Create an engine on CUDA device `device`: context binding, stream, noise tables and work
 * buffers.  Replaces phase1_scan's allocateBuffers() and its one-context-per-process
 * set-up (engine/gpu/low54/phase1_scan.cu:825-866, :1492-1513). */
int wg_engine_open(int device, wg_engine **out);

/* Release everything wg_engine_open made (phase1_scan.cu:868-879).  NULL is a no-op. */
void wg_engine_close(wg_engine *e);

/* Message of the engine's last failure ("" if none). */
const char *wg_engine_error(const wg_engine *e);

/* Noise core of the phase-1 gates.
 *   WG_NOISE_FP32 (the default): the climate gates' samples (erosion tiers, temperature, ridge)
 *     in FP32 after an FP64 coordinate reduction, gates decided from the FP32 sums outside a
 *     derived error band and re-taken in FP64 inside it, so every verdict equals the FP64 path's;
 *     wg_scan_stats.rechecks counts the re-takes.  The cave gates sample in FP64.
 *   WG_NOISE_FP64: every sample in FP64 in the reference's operation order.
 *   WG_NOISE_FP32_CAVES: WG_NOISE_FP32 plus the entrance gate's 3-D cave samples in FP32 (the
 *     tunnel-scale interval and Entrance(50) / Entrance(60) re-taken in FP64 inside their error
 *     bands).  Same verdicts; not the default because on a B200 it is slower at 9 x 9 regions per
 *     seed (the FP64 pipe is not what bounds that kernel) and only slightly faster on whole-world
 *     scans.
 *   WG_NOISE_FP32_RECHECK_ALL: WG_NOISE_FP32_CAVES with every gate re-taken in FP64, a check mode
 *     that runs the recheck paths on every decision (slow; for tests of those paths).
 * The reference has the same choice as a build flag, without the recheck
 * (PHASE1_FP32_CORE, engine/gpu/low54/device_noise.h:132-160).  WG_ERR_ARG for other values. */
#define WG_NOISE_FP32 0
#define WG_NOISE_FP64 1
#define WG_NOISE_FP32_RECHECK_ALL 2
#define WG_NOISE_FP32_CAVES 3
int wg_engine_set_noise_core(wg_engine *e, int core);

/* The FP32 core's measured error: out64[b * n_points + i] = the y = 0 DoublePerlin value of climate
 * noise `noise` in world seeds[b] at noise-space point (xz[2i], 0, xz[2i + 1]) in FP64 (the
 * reference's lysh_dblnoise_sample_y0, engine/tools/lysh/src/noise.c:320-342), out32[...] = the
 * same value from the FP32 core's samples.  noise: 0 erosion, 1 temperature, 2 ridge,
 * 3 continentalness, 4 erosion_large, 5 temperature_large, 6 continentalness_large.  Host
 * buffers; n_seeds * n_points <= 2^26. */
int wg_noise_probe(wg_engine *e, const int64_t *seeds, uint64_t n_seeds, int noise, const double *xz,
                   uint64_t n_points, double *out32, double *out64);

/* The same for the 3-D cave noises the entrance gate samples in the FP32 core: out64[...] = the
 * DoublePerlin value of `noise` in world seeds[b] at noise-space point (xyz[3i], xyz[3i + 1],
 * xyz[3i + 2]) in FP64 (the reference's lysh_dblnoise_sample, engine/tools/lysh/src/noise.c:263-289),
 * out32[...] = the same value from the FP32 core's octave samples.  noise: 7 cave_entrance,
 * 8 spaghetti_rarity, 9 spaghetti_thickness, 10 spaghetti_3d_1, 11 spaghetti_3d_2,
 * 12 roughness_modulator, 13 roughness.  Host buffers; n_seeds * n_points <= 2^26. */
int wg_noise_probe_3d(wg_engine *e, const int64_t *seeds, uint64_t n_seeds, int noise, const double *xyz,
                      uint64_t n_points, double *out32, double *out64);

/* lysh's --version / --preset names -> option bits
 * (engine/tools/lysh/src/main.c:104-132).  0 on success, WG_ERR_ARG if unknown.  Each sets only
 * its own fields (version: mc_1_18_2, pre_26_2, biome_tree; preset: single_biome, large_biomes),
 * so start from a zeroed wg_opts. */
int wg_parse_version(const char *name, wg_opts *opts);
int wg_parse_preset(const char *name, wg_opts *opts);

/* Seed Check phase 1 over every seed x every region of [rx0,rx1) x [rz0,rz1).
 * Seeds are seeds[0..n_seeds) (host memory) or, when seeds is NULL, the generator
 * splitmix64(gen_base + i) of phase1_scan's --seed-gen.  Writes up to `cap` survivors to
 * `out` (host memory), sorted by (seed_index, rz, rx); *n_out = the number found, which may
 * exceed cap (then only the first cap are written).  `stats` may be NULL.
 * Replaces phase1_scan's runScan() batch loop (phase1_scan.cu:881-1342) and the phase-1
 * pass of lysh_scan_rect (engine/tools/lysh/src/search.c:198-265); the survivor set is
 * exactly lysh_phase1_check_ex's (phase1.c:130-200), without the GPU density prefilter. */
int wg_seed_check(wg_engine *e, const int64_t *seeds, uint64_t gen_base, uint64_t n_seeds,
                  const wg_opts *opts, int max_height, int salt,
                  int rx0, int rx1, int rz0, int rz1,
                  wg_candidate *out, uint64_t cap, uint64_t *n_out, wg_scan_stats *stats);

/* Same request with device-resident buffers: d_seeds (device, or NULL for the generator)
 * and d_out (device, unsorted).  All work is enqueued on `stream` (a cudaStream_t; NULL =
 * the engine's own stream), so events the caller records on that stream bracket it.  The
 * call returns when the work is complete. */
int wg_seed_check_device(wg_engine *e, const int64_t *d_seeds, uint64_t gen_base, uint64_t n_seeds,
                         const wg_opts *opts, int max_height, int salt,
                         int rx0, int rx1, int rz0, int rz1,
                         wg_candidate *d_out, uint64_t cap, uint64_t *n_out, wg_scan_stats *stats,
                         void *stream);

/* Per-region phase-1 verdicts for parity checks: codes / tiers (host, n_seeds * R entries,
 * seed-major, rz outer, rx inner) receive the LYSH_P1_REJECT_* code and the erosion tier
 * (-1 if none) of every (seed, region), as lysh_phase1_check_ex reports them
 * (phase1.c:130-200, search.c:148-160). */
int wg_phase1_codes(wg_engine *e, const int64_t *seeds, uint64_t gen_base, uint64_t n_seeds,
                    const wg_opts *opts, int max_height, int salt,
                    int rx0, int rx1, int rz0, int rz1, int8_t *codes, int8_t *tiers);

/* Seed Check phase 1 that allocates nothing, for callers that cannot call cudaMalloc: a
 * process whose device memory belongs to another allocator (a framework's caching allocator,
 * a serving loop with a fixed budget), or a latency-critical stream on which cudaMalloc /
 * cudaFree could synchronize the device or fail under fragmentation.  No counterpart in the
 * reference.
 *
 * The caller passes device buffers: d_seeds (or NULL for splitmix64(gen_base + i)) and d_out
 * (room for `cap` candidates, unsorted); *n_out (host) receives the number found, which may
 * exceed cap (only cap are written).  Work runs on `stream` (NULL = the default stream) and
 * the call returns when it is done.  The current CUDA device is used.
 *
 * Limits: n_seeds <= 65,536 and at most 4,096 regions per seed per call, else WG_ERR_CAPACITY;
 * WG_ERR_CAPACITY also when a call's climate survivors exceed 1,048,576 (or its unit records
 * 131,072, or its deep candidates 65,536).  Unlike wg_seed_check_device, a full list is not
 * re-run in smaller pieces, so the practical size is set by the climate survivors: about 1.7 %
 * of regions pass the climate gates at the usual rules, so keep n_seeds * regions below about
 * 2^20 / 0.017 = 6e7 checks per call (about 15,000 seeds on a full 64 x 64 rect, 65,536 seeds up
 * to ~900 regions).  The work lists live in one 6 MiB file-scope __device__ array that every GPU
 * loading the library holds until the process exits.  The first call on a device uploads the
 * noise tables and looks up that array's address, so make it before any stream capture.  Every
 * call is synchronous: it waits for its stream and reads the list counters back to the host.
 * All calls share the array: calls that overlap on the GPU (other streams or host threads) race
 * on it. */
int wg_seed_check_noalloc(const int64_t *d_seeds, uint64_t gen_base, uint32_t n_seeds,
                          const wg_opts *opts, int max_height, int salt,
                          int rx0, int rx1, int rz0, int rz1,
                          wg_candidate *d_out, uint32_t cap, uint32_t *n_out, void *stream);

/* ---------------- phase 2: confirmation of a hut (lysh_eval_hut) ---------------- */

/* One confirmed (or rejected) hut: the fields of lysh_hut_result
 * (engine/tools/lysh/src/eval.h:63-85), same meanings and units. */
typedef struct {
    int32_t hut_x, hut_z;        /* hut origin (block), = chunk * 16 */
    int32_t rx, rz;              /* its region (floorDiv by 32 chunks) */
    int32_t dir;                 /* orientation: 0 N, 1 E, 2 S, 3 W */
    int32_t axis_z;              /* 1 -> footprint 7 (x) by 9 (z), 0 -> 9 by 7 */
    int32_t size_x, size_z;
    int32_t avg_y;               /* post-carver footprint height sum / 63 (truncated) */
    int32_t wet_columns;         /* footprint columns with water above y = 62 */
    int32_t flooded, all_dry;    /* wet_columns == 63 / == 0 */
    int32_t ok;                  /* biome ok && !flooded && avg_y <= max_y */
    int32_t reject;              /* 0 ok, 1 avg_y > max_y, 2 flooded, 3 biome */
    int32_t biome_ok, biome_winner;
    int32_t biome_qx, biome_qy, biome_qz, biome_occ_y;
    int64_t sum_h;               /* footprint height sum (pre-carver when the flood short-circuit applied) */
    int64_t biome_t[6];          /* quantized temperature, humidity, continentalness, erosion, depth, weirdness */
} wg_hut_result;

/* Phase 2 for n huts: hut i of world seed seeds[i] at block (hut_x[i], hut_z[i]) (the
 * chunk origin of a phase-1 survivor), judged against max_y.  out[0..n) receives
 * lysh_eval_hut's result for each (engine/tools/lysh/src/eval.c:121-242): orientation,
 * the real biome gate at the chunk centre, the y = 62 aquifer flood test of the 63 footprint
 * columns, the post-carver footprint heights.  The search context's version and preset come
 * from opts (eval.c:70-107).  Replaces lysh_eval_hut and the `lysh hut` confirmations
 * hunt.py spawns per candidate. */
int wg_eval_huts(wg_engine *e, const int64_t *seeds, const int32_t *hut_x, const int32_t *hut_z, uint64_t n,
                 const wg_opts *opts, int max_y, wg_hut_result *out);

/* Counts of a graded scan: lysh_hut_grade (engine/tools/lysh/src/eval.h:100-114). */
typedef struct {
    int64_t scanned;             /* regions scanned */
    int64_t evaluated;           /* phase-1 survivors judged by phase 2 */
    int64_t accepted;
    int64_t rejected_y, rejected_flood, rejected_biome;
    int32_t hits_written;        /* rows written to hits */
    double ms;                   /* wall time of the call */
    double p2_ms;                /* of which phase 2 */
} wg_hut_grade;

#define WG_HUT_GRADE_INTS 12

/* Phase 1 + phase 2 over [rx0,rx1) x [rz0,rz1) for one seed: lysh_grade_scan
 * (engine/tools/lysh/src/eval.c:481-492, session band :405-477).  hits (may be NULL) receives
 * up to hits_cap rows of WG_HUT_GRADE_INTS ints for the accepted huts, in region order
 * (rz outer, rx inner): hutX, hutZ, rx, rz, dir, avg_y, flooded, ok, wet_columns, size_x,
 * size_z, reject (eval.c:258-271). */
int wg_grade_scan(wg_engine *e, int64_t seed, const wg_opts *opts, int max_height,
                  int rx0, int rx1, int rz0, int rz1, int salt, int max_y,
                  int32_t *hits, int32_t hits_cap, wg_hut_grade *grade);

/* Phase-2 parity probes: out[i] = the value of `kind` at block (xyz[3i], xyz[3i+1],
 * xyz[3i+2]) in world `seed` (y ignored where the quantity is per column).  Kinds and the
 * reference function each one equals:
 *   0 blended base noise                lysh_interp_calculate_noise_261   interp_noise.c:100
 *   1 density before interpolation      lysh_phase2_density_raw_at        phase2.c:151
 *   2 preliminary surface level         lysh_preliminary_surface_level    column_top.c:94
 *   3/4/5 continentalness / erosion / weirdness at biome (x>>2, z>>2)     terrain.c:22
 *   6/7/8 terrain offset / factor / peaks (26.1 ridges_folded)            spline.c:112
 *   9 computeFluid: level * 4 + type (0 solid, 1 air, 2 water, 3 lava)    aquifer.c:327
 *   10 interpolated final density       lysh_phase2_density_at            phase2.c:161
 *   11 block state before carvers       lysh_phase2_block_at              phase2.c:309
 *   12 surface height before carvers    lysh_phase2_height_pre_carver     phase2.c:318
 *   13 surface height after carvers     lysh_phase2_height                phase2.c:438
 *   14 the chunk's stored `interpolated` corner value for the cell holding the point, i.e.
 *      kind 1 at ((x >> 2) * 4, -64 + 8 * ((y + 64) >> 3), (z >> 2) * 4)  phase2.c:73-96 */
int wg_p2_probe(wg_engine *e, int64_t seed, const wg_opts *opts, int kind, const int32_t *xyz, uint64_t n,
                double *out);

/* ---------------- Deep Dive: mineshaft starts under swamp huts ---------------- */

/* A swamp hut whose chunk is also a mineshaft start chunk, for a 48-bit structure seed. */
typedef struct {
    uint64_t seed_index;         /* index of the structure seed in the request (list position / base offset) */
    int64_t s48;                 /* structure seed (the world seed's low 48 bits) */
    int32_t rx, rz;              /* hut region */
    int32_t chunk_x, chunk_z;    /* hut chunk = mineshaft start chunk */
    int64_t carver;              /* setLargeFeatureSeed state of that chunk (48 bits) */
} wg_deep_start;

/* The region walk of the Deep Dive solver: for every structure seed s48[0..n) (or, when s48 is
 * NULL, s48_base + i) and every region of [rx0,rx1) x [rz0,rz1), the region's swamp-hut chunk
 * and whether a mineshaft starts there (setLargeFeatureSeed + nextDouble() < 0.004).  Writes the
 * first cap hits of the (seed_index, rz, rx) order to out (host); *n_out = the number found (may
 * exceed cap: call again with a bigger buffer for the rest).  Replaces the
 * room walk of hut_lookup_v4 (rcWalkStep / walkStepCarver / rcIsStartS0,
 * engine/gpu/room_core.h:40-175, engine/gpu/hut_lookup_v4_source.cu:47-75): the forward
 * direction; the layout-catalogue direction is wg_deep_solve. */
int wg_deep_starts(wg_engine *e, const int64_t *s48, int64_t s48_base, uint64_t n,
                   int rx0, int rx1, int rz0, int rz1, wg_deep_start *out, uint64_t cap, uint64_t *n_out);

/* A hut on a mineshaft start chunk whose carver state is a catalogued layout. */
typedef struct {
    uint64_t seed_index;         /* index of the structure seed in the request */
    int64_t s48;                 /* structure seed */
    int32_t rx, rz;              /* hut region */
    int32_t chunk_x, chunk_z;    /* hut chunk = mineshaft start chunk */
    int64_t carver;              /* its setLargeFeatureSeed state = the catalogued layout */
    uint32_t value;              /* that layout's catalogue value (air above the hut floor: hi | lo << 10) */
    uint32_t pad;
} wg_sweep_match;

/* The Deep Dive forward sweep with the layout-catalogue probe (hut_lookup_v4 without --solve:
 * sweepProbeKernel, engine/gpu/hut_lookup_v4_source.cu:77-99, driven per structure seed at
 * :1504-1530): for every structure seed s48[0..n) (or, when s48 is NULL, s48_base + i) and every
 * region of [rx0,rx1) x [rz0,rz1), the region's swamp-hut chunk, whether a mineshaft starts there,
 * and for each start whether its carver state is one of layouts[0..n_layouts) (values[k] is layout
 * k's catalogue value; values may be NULL).  out receives the first cap matches sorted by
 * (seed_index, rz, rx); *n_out = all of them (WG_ERR_CAPACITY past 2^20 in one call); starts (may
 * be NULL) receives each structure seed's number of starts. */
int wg_deep_sweep(wg_engine *e, const uint64_t *layouts, const uint32_t *values, uint64_t n_layouts,
                  const int64_t *s48, int64_t s48_base, uint64_t n, int rx0, int rx1, int rz0, int rz1,
                  wg_sweep_match *out, uint64_t cap, uint64_t *n_out, uint64_t *starts);

/* The Deep Dive terrain stage (hut_lookup_v4 --spots, engine/gpu/hut_lookup_v4_source.cu:1262-1290):
 * for each spot (s48[i], chunk_x[i], chunk_z[i]), the 65,536 world seeds (u << 48) | s48[i],
 * u = 0..65535, through the phase-1 gates (lysh_phase1_check_ex at max_height) at the spot's
 * region.  Writes the surviving (seed, region) of every spot whose hut lies in the spot chunk to
 * out (host, up to cap, sorted; seed_index = i * 65536 + u); *n_out = the number found.  Spots
 * that are not mineshaft start chunks are skipped and counted in *not_start (may be NULL), as
 * hut_lookup_v4 reports them. */
int wg_deep_spots(wg_engine *e, const int64_t *s48, const int32_t *chunk_x, const int32_t *chunk_z, uint64_t n_spots,
                  const wg_opts *opts, int max_height, wg_candidate *out, uint64_t cap, uint64_t *n_out,
                  uint64_t *not_start);

/* ---------------- the mineshaft finisher (hunt.py finish_row) ---------------- */

/* One piece of a mineshaft tree, as `mstree` prints it (engine/tools/mstree/mstree.cpp:17-33):
 * kind 'R' room, 'C' corridor, 'X' / 'Y' one- / two-storey crossing, 'S' stairs; the inclusive
 * block box; facing 0 N, 1 S, 2 W, 3 E (-1 for the room); the parent's index (-1 for the room);
 * rails on a corridor. */
typedef struct {
    int32_t kind, x0, y0, z0, x1, y1, z1, facing, parent, rails;
} wg_ms_piece;

/* The mineshaft tree of world seed ws at chunk (chunk_x, chunk_z) (mstree <ws> <cx> <cz>): the
 * start test, MineShaftPieces generation and the move below sea level.  Writes up to cap pieces
 * (at most 512 exist), *n_out = their number, *room_floor = the room's floor y.  Returns
 * WG_ERR_ARG when the chunk is not a mineshaft start (mstree's exit 3), WG_ERR_CAPACITY when the
 * tree exceeds the generator's 512 pieces, 16 open pieces or byte-range boxes (the reference
 * reports those trees as failed too). */
int wg_mineshaft_tree(wg_engine *e, int64_t ws, int32_t chunk_x, int32_t chunk_z, wg_ms_piece *out, uint32_t cap,
                      uint32_t *n_out, int32_t *room_floor);

/* The finisher's measurements of one Deep Dive survivor (world seed, hut chunk): everything
 * hunt.py's finish_row (hunt.py:277-333) reads from lysh hut, mstree, biome_at, msroom and
 * skyscan.  Heights and floors are block y; the footprint is the 7 x 9 blocks at the chunk origin
 * (finish_row runs msroom with MC_SHAPE=79 and skyscan with 7 x 9). */
typedef struct {
    int32_t hut_x, hut_z;          /* 16 * chunk */
    int32_t verdict_ok;            /* lysh hut --max-y 100 --phase2-max-y 100: ACCEPT */
    int32_t avg_y;                 /* its floor */
    int32_t tree_status;           /* 0 tree built, 1 not a mineshaft start, 2 tree too large */
    int32_t pieces, room_floor;    /* mstree: pieces, the room's floor (its first line's y) */
    int32_t biome[2];              /* biome_at --ms --y room_floor: 1.21.5 tree, 26.2 tree (BIOME_26) */
    int32_t nat;                   /* msroom EXACT: the footprint floor without the mineshaft */
    int32_t top[2], refused[2];    /* msroom EXACT: top0 / top1 floors and refused pieces */
    int32_t no_guard[2];           /* msroom EXACT: ng0 / ng1 floors (liquid guard off) */
    int64_t sum_nat, sum_top[2], sum_no_guard[2];   /* the footprint height sums behind them */
    /* skyscan --list over the footprint: height sum (mean = sum / 63), min, max, columns at or
     * below -54, lava and solid blocks from y -59 up to each surface, the corner heights, columns
     * above -53 */
    int64_t scan_sum;
    int32_t scan_min, scan_max, le54, lava, solid, nw, ne, sw, se, above53;
} wg_finish_row;

/* The finisher over n survivors (ws[i], chunk_x[i], chunk_z[i]) on the GPU: lysh's hut verdict,
 * the mineshaft tree, the deep-dark biomes at the room floor, the carved floors and the footprint
 * scan, written to out[i].  Rows whose chunk is no start or whose tree failed carry tree_status
 * and no floors.  hunt.py turns a row into its result line only when verdict_ok, tree_status 0,
 * not both biomes deep dark (183) and top[1] <= its min_r. */
int wg_finish_rows(wg_engine *e, const int64_t *ws, const int32_t *chunk_x, const int32_t *chunk_z, uint64_t n,
                   wg_finish_row *out);

/* ---------------- biome map ---------------- */

/* biome_map's raster (engine/tools/mineshaft/biome_map.c): w x h bytes (z outer, x inner; w, h
 * <= 4096), cell (i, j) = the blocks [x0 + i step, x0 + (i+1) step) x [z0 + j step, ...); each of
 * its ss x ss sample points (ss 1..4) gives the biome at the middle of the chunk holding it with the
 * surface at y + 1 (lysh_swamp_hut_biome_ok); the cell is the dominant biome, a swamp winning at a
 * quarter of the samples.  opts selects the biome tree (wg_parse_version). */
int wg_biome_map(wg_engine *e, int64_t seed, const wg_opts *opts, int64_t x0, int64_t z0, int w, int h, int step,
                 int ss, int y, uint8_t *out);

/* biome_map --stdin: the biome the witch-hut test sees at each chunk (cx[i], cz[i]): the middle
 * column at six fixed surface heights, and where they disagree about a swamp, at the chunk's
 * real pre-carver surface (biome_map.c:38-52). */
int wg_biome_chunks(wg_engine *e, int64_t seed, const wg_opts *opts, const int32_t *cx, const int32_t *cz,
                    uint64_t n, uint8_t *out);

/* ---------------- Deep Dive solver: structure seeds for a mineshaft layout ---------------- */

/* One plan line (the reference's plan.txt: "X regime class ..."): the setLargeFeatureSeed state
 * wanted at the hut chunk (a catalogued mineshaft layout), the region regime on each axis
 * (0: |r| <= 16383, 1: 16384..32767, 2: 32768..58593, both signs) and the chunk-offset class
 * (1 "odd": one offset odd; 2 "u2": both even, 2-adic valuations differ; 3 "eq": equal
 * valuations, not both 0). */
typedef struct {
    uint64_t layout;
    int32_t regime_x, regime_z;
    int32_t tier;
    int32_t pad;
} wg_solve_bundle;

/* A structure seed whose swamp hut (chunk_x, chunk_z) has that layout's carver state. */
typedef struct {
    uint64_t s48;
    int32_t chunk_x, chunk_z;
    uint64_t layout;
    uint64_t group;          /* the group it was found in (bundle << 20 | group within the bundle) */
} wg_solve_hit;

typedef struct {
    uint64_t groups, regions, tasks;
    uint64_t candidates;     /* low-20-bit candidates lifted (sum over tasks of their list length) */
    uint64_t hits;
    uint64_t host_check_failures;   /* hits dropped by the host's forward check (expected 0) */
    double gpu_ms, wall_ms;
} wg_solve_stats;

/* Groups [first_group, first_group + n_groups) of the bundles (group g: bundle g >> 20, residue
 * class scramble(g & 0xFFFFF) of the region constant's low 20 bits): every (region, chunk offset)
 * task of the group solved for all structure seeds.  Hits sorted by (group, s48, chunk_x, chunk_z);
 * *n_out = all, at most cap written.  Replaces hut_lookup_v4 --solve-only --solve5 --plan
 * (engine/gpu/hut_lookup_v4_source.cu:1293-1380; equations solver_kernels.cuh, solver_fused.cuh;
 * task space taskspace.h). */
int wg_deep_solve(wg_engine *e, const wg_solve_bundle *bundles, uint64_t n_bundles, uint64_t first_group,
                  uint64_t n_groups, wg_solve_hit *out, uint64_t cap, uint64_t *n_out, wg_solve_stats *stats);

/* The same solve for explicit tasks: region (rx[i], rz[i]) with chunk offsets (ox[i], oz[i]) in
 * 0..23, not both 0; hits' group = the task index.  hut_lookup_v4 --solve --tasks-file. */
int wg_deep_solve_tasks(wg_engine *e, uint64_t layout, const int32_t *rx, const int32_t *rz, const int32_t *ox,
                        const int32_t *oz, uint64_t n, wg_solve_hit *out, uint64_t cap, uint64_t *n_out);

/* ---------------- job server: batched and streamed Seed Check jobs ---------------- */

/* One Seed Check job: seeds[0..n_seeds) (copied at submit) or, when seeds is NULL,
 * splitmix64(gen_base + i); every seed x every region of [rx0,rx1) x [rz0,rz1) at max_height. */
typedef struct {
    const int64_t *seeds;
    uint64_t gen_base;
    uint64_t n_seeds;
    int rx0, rx1, rz0, rz1;
    int max_height;
    int salt;                    /* 0 = the swamp-hut salt */
    wg_opts opts;
} wg_job;

typedef struct {
    int32_t done;                /* 1 when the job's survivors are ready */
    int32_t status;              /* WG_OK, or the error the job ended with */
    uint64_t found;              /* phase-1 survivors */
    double queue_ms;             /* submit -> start of the batch that ran it */
    double latency_ms;           /* submit -> done */
    uint64_t batch_jobs;         /* jobs flattened into that batch (the job included) */
} wg_job_status;

/* How wg_seed_check_jobs runs: 1 (the default) = every job's seeds resident at once and the whole
 * job list as one CUDA graph launch, whose device-side loop takes slices of units off a queue,
 * runs the phase-1 kernels on each and appends the survivors, with no host synchronisation
 * between slices (it falls back to 0 when the seeds exceed 2^27); 0 = the host batch loop.  The
 * reference has no batched-job path. */
int wg_engine_set_job_queue(wg_engine *e, int device_queue);

/* Autotuned job settings: for each job class (regions per seed up to max_regions[k]) the regions
 * per work unit, and the (seed, region) checks per queue slice, each the fastest of the candidates
 * timed on the device on probe jobs of that class (seed counts log-uniform 1..4,096; a window's
 * time is the best of three runs after a warm-up, a budget's the best of two).  The
 * reference tunes its scanner per GPU with a measured sweep (hunt.py:927-1019). */
typedef struct {
    uint32_t max_regions[4];          /* class k: rects of up to this many regions (class 3: any) */
    uint32_t window[4];               /* regions per unit chosen for the class */
    uint32_t window_candidates[4][4]; /* the windows timed (0 = none) */
    double window_ms[4][4];           /* their device time on the class's probe jobs */
    uint64_t budget;                  /* (seed, region) checks per queue slice chosen */
    uint64_t budget_candidates[3];
    double budget_ms[3];              /* device time of all classes' probe jobs at each budget */
} wg_tune_report;

/* Times the candidates on this engine's GPU (a few seconds) and keeps the fastest settings for the
 * engine's later wg_seed_check_jobs calls; report (may be NULL) receives the measurements. */
int wg_engine_tune(wg_engine *e, wg_tune_report *report);

/* Sets the job settings directly (e.g. from a saved tuning): window[4] regions per unit per class
 * (NULL or 0 = the default rule: a whole seed up to 4,096 regions, else 2,048), budget checks per
 * slice (0 = 2^27). */
int wg_engine_set_tuning(wg_engine *e, const uint32_t *window, uint64_t budget);

/* Many Seed Check jobs at once (uneven seed counts, rects and floors), flattened into shared
 * device batches: every batch covers slices of several jobs through the kernels' job table.
 * Survivors are written job by job (job order, then seed_index, rz, rx; seed_index is the seed's
 * position in its job); job_found[i] (if not NULL) = job i's count; *n_out = all, at most cap
 * written.  Each job's survivors equal wg_seed_check on that job alone.  The reference has one
 * job per phase1_scan request (engine/gpu/low54/phase1_scan.cu:1328-1387). */
int wg_seed_check_jobs(wg_engine *e, const wg_job *jobs, uint64_t n_jobs, wg_candidate *out, uint64_t cap,
                       uint64_t *n_out, uint64_t *job_found, wg_scan_stats *stats);

typedef struct wg_server wg_server;

/* A job server on CUDA device `device`: one worker thread with its own engine takes the queued
 * jobs, flattens every queued job with the same rect, max_height, salt and rules into one
 * request (their seed lists concatenated), runs it, and hands each job its survivors.  Seeds
 * of queued jobs stay in host memory until their batch runs (max_queued_seeds bounds them;
 * submit returns WG_ERR_CAPACITY beyond it).  The reference has no job server; lysh's
 * session API (engine/tools/lysh/src/eval.h:180-205) and hunt.py's worker protocol
 * (hunt.py:1276-1332) are the interfaces it batches. */
int wg_server_open(int device, uint64_t max_queued_seeds, wg_server **out);

/* Server settings (all-zero = the defaults of wg_server_open). */
typedef struct {
    uint64_t max_queued_seeds;   /* host-queued seeds at most (0 = 2^30) */
    uint64_t arena_seeds;        /* device seed slots (0 = a quarter of the free HBM, at most 2^28);
                                    a job with more seeds is refused at submit (WG_ERR_CAPACITY) */
    uint64_t batch_checks;       /* (seed, region) checks per batch (0 = 2^25) */
    uint64_t fail_job;           /* host-side fault injection for tests: every batch that holds the
                                    job with this id fails before launch (0 = none) */
} wg_server_config;

/* wg_server_open with explicit settings.  A failed batch fails no job by itself while the engine
 * still works: its jobs run again one at a time, and only a job that fails alone ends with the
 * error (wg_job_status.status); the others' results are those they get alone.  A broken CUDA
 * context ends every job, queued ones included. */
int wg_server_open_config(int device, const wg_server_config *cfg, wg_server **out);

/* Queue a job; *job_id identifies it.  Non-blocking. */
int wg_server_submit(wg_server *s, const wg_job *job, uint64_t *job_id);

/* The job's status; when wait_ms > 0, waits up to that long for it to finish. */
int wg_server_poll(wg_server *s, uint64_t job_id, int wait_ms, wg_job_status *st);

/* A finished job's survivors (sorted by seed_index within the job, then rz, rx; seed_index is
 * the seed's position in the job); *n_out = all of them, at most cap written.  The job's
 * results are released once they have all been taken. */
int wg_server_take(wg_server *s, uint64_t job_id, wg_candidate *out, uint64_t cap, uint64_t *n_out);

/* The server's totals so far: batches, kernel launches and device times, (seed, region) checks
 * and survivors of the finished jobs. */
int wg_server_stats(wg_server *s, wg_scan_stats *st);

/* Stop the worker (finishing the batch in flight) and release everything; jobs not finished
 * are dropped. */
void wg_server_close(wg_server *s);

#ifdef __cplusplus
}
#endif

#endif /* WITCHGPU_H */
