// Seed Check phase 1 on the GPU: the shared definitions between the kernels
// (wg_phase1.cu) and the host engine (wg_engine.cu).
//
// Phase 1 restates lysh_phase1_check_ex (engine/tools/lysh/src/phase1.c:130-200) per
// (seed, region) and is split into three kernels by how often each stage is reached:
//
//   climate  every seed     builds the 18 climate Perlins of 16 units per CTA in shared
//                           memory, runs the tiered erosion / temperature / ridge gates for
//                           every region, and emits per-unit records of the survivors
//                           (~1.7% of regions at 9x9).
//   entrance seeds with     builds the 18 Perlins of cave_entrance + the spaghetti set for
//            survivors      16 records per CTA, evaluates Entrance(50) and Entrance(60)
//                           (97% of climate survivors stop here).
// Both hot kernels use ~100 KiB of shared memory, so two CTAs share an SM and one CTA's table
// build overlaps the other's evaluation.
//   ladder   the rest       one 64-thread CTA per remaining candidate builds all 54 cave /
//                           continent / floodedness Perlins (54 of its 64 threads build, ~10 CTAs
//                           per SM) and finishes the ladder in lysh's order.
#pragma once

#include <cstdint>

#include "wg_catalog.h"

namespace wg {

// Reject codes, identical to LYSH_P1_REJECT_* (engine/tools/lysh/src/phase1.h:61-74).
enum : int {
    P1_EROSION = 0,
    P1_TEMPERATURE = 1,
    P1_RIDGE = 2,
    P1_ENTRANCE_50 = 3,
    P1_ENTRANCE_60 = 4,
    P1_CAVE_AT_MAXH = 5,
    P1_LADDER_NEG = 6,
    P1_LADDER_POS = 7,
    P1_CONTINENTALNESS = 8,
    P1_FLOODEDNESS = 9,
    P1_ACCEPT = 10,
    P1_KINDS = 11
};
constexpr int kTiers = 7;

constexpr int kUnits = 16;          // units (climate) or records (entrance) per CTA
constexpr int kSlotsA = 18;         // erosion 8 + temperature 4 + ridge 6
constexpr int kSlotsB = 18;         // cave_entrance 6 + six one-octave spaghetti noises x 2
constexpr int kSlotsC = 54;         // kSlotsB + cave_layer 2 + cave_cheese 14 + continentalness 18 + floodedness 2
constexpr int kThreadsA = kSlotsA * kUnits;   // one thread per (slot, unit) table
constexpr int kThreadsB = kSlotsB * kUnits;
constexpr int kThreadsC = 64;
constexpr int kRecordCap = 64;      // survivors held per unit record in the climate kernel
constexpr int kChunk = 96;          // regions per unit whose hut positions are staged at a time

// Counter block written by the kernels (one per engine, reset per batch).
enum : int {
    CNT_RECORDS = 0,   // per-seed survivor records emitted by the climate kernel
    CNT_SURVIVORS,     // climate survivors (entries of surv_region)
    CNT_DEEP,          // candidates that passed Entrance(50) and Entrance(60)
    CNT_FINAL,         // phase-1 survivors
    CNT_OVERFLOW,      // bit 0 records/survivors, bit 1 deep list, bit 2 final list
    CNT_RECHECK,       // FP32 noise core: gate decisions re-taken in FP64 (value inside the error band)
    CNT_WORDS = 8
};

// Final phase-1 survivor; the layout of wg_candidate in include/witchgpu.h.
struct Candidate {
    uint64_t seed_index;
    int64_t seed;
    int32_t rx, rz;
    int32_t chunk_x, chunk_z;
};

// Work is cut into "units": unit u of a request is (seed u / n_win, region window
// u % n_win); a window is `win` consecutive regions of the rect (rz outer, rx inner).  One
// lane of the climate kernel owns one unit, so a request with few seeds and a huge rect
// (a whole-world scan of one seed) fills the GPU as well as many seeds x 9x9 regions.
//
// Jobs mode flattens many Seed Check jobs, each with its own rect and floor, into one batch:
// entry k of the job table covers the global units [unit0, next entry's unit0) and maps them
// to units first, first + 1, ... of one job (so a batch can take any slice of a job).
struct JobGeom {
    uint64_t unit0;        // first global unit of this entry (entries sorted by unit0, none empty)
    uint64_t first;        // the job's unit index of that first unit
    uint64_t seed0;        // global seed index of the job's seed 0 (index into BatchArgs::seeds)
    uint64_t n_win;        // windows per seed of the job
    uint64_t n_regions;    // regions per seed (rw * rh)
    uint32_t win;          // regions per window
    int32_t rx0, rz0, rw;  // the job's region rect origin and width
    int32_t max_height;    // the job's gate floor
    int32_t pad;
};
static_assert(sizeof(JobGeom) == 64, "job table entry layout");

// Everything a phase-1 batch needs (device pointers only).
struct BatchArgs {
    const int64_t *seeds;         // all request seeds (global seed index), or nullptr: splitmix64(gen_base + i)
    uint64_t gen_base;
    uint64_t unit0;               // global index of the batch's first unit
    uint32_t n_units;             // units in this batch
    uint32_t win;                 // regions per window
    uint64_t n_win;               // windows per seed
    uint64_t n_regions;           // regions per seed (rw * rh)
    int rx0, rz0, rw, rh;         // region rect origin and size
    int salt;
    int max_height;
    int mc_1_18_2, pre_26_2, single_biome, large_biomes;
    int fp32_core;                // 1: climate samples in FP32, FP64 recheck inside the error band;
                                  // 3: also the entrance gate's cave samples; 2: as 3, every gate
                                  // re-taken in FP64; 0: FP64
    int small_coords;             // every climate coordinate of the batch lies inside
                                  // maintainPrecision's identity range (coords_small)

    uint32_t *rec_unit;           // [cap_rec] batch-local unit of each record
    uint32_t *rec_off;            // [cap_rec] first entry in surv_region
    uint32_t *rec_cnt;            // [cap_rec]
    uint32_t *surv_region;        // [cap_surv] region offset inside the unit's window
    uint32_t *deep;               // [cap_deep * 2] (batch-local unit, region offset)
    Candidate *out;               // [cap_out] phase-1 survivors of this batch
    uint32_t cap_rec, cap_surv, cap_deep, cap_out;
    uint32_t *counters;           // [CNT_WORDS], zeroed per batch
    unsigned long long *hist;     // [P1_KINDS + kTiers] funnel + erosion tier histogram, zeroed per batch
    int8_t *codes;                // optional [n_seeds * n_regions] reject code per (seed, region)
    int8_t *tiers;                // optional, same shape: erosion tier (-1 if none)

    // Optional spots mode (the Deep Dive terrain stage): seed g is the world seed
    // (g & 0xFFFF) << 48 | spot_s48[g >> 16], one of the 65,536 upper-bit variants of a 48-bit
    // structure seed, and its rect is shifted by the spot's region (spot_rx, spot_rz)[g >> 16].
    const int64_t *spot_s48 = nullptr;
    const int32_t *spot_rx = nullptr, *spot_rz = nullptr;

    // Optional jobs mode: the batch's units are resolved through this table (rect, window and
    // max_height per job; seeds from `seeds`); unit0 .. unit0 + n_units are global units of it.
    const JobGeom *jobs = nullptr;
    uint32_t n_jobs = 0;

    // Optional device work queue (wg_queue.cu): when set, the batch's unit0 and n_units are read
    // from dyn[0], dyn[1] at kernel start instead of the fields above (a graph replays the same
    // launches while a device kernel moves the batch along the queue); n_units above is then the
    // largest batch the launch geometry covers.
    const uint64_t *dyn = nullptr;
};

// The batch range of a launch: dyn when set, else the launch's own fields.
__device__ __forceinline__ void batch_range(BatchArgs &a) {
    if (a.dyn) {
        a.unit0 = a.dyn[0];
        a.n_units = (uint32_t)a.dyn[1];
    }
}

// One evaluation step of the climate state machine (a single y=0 Perlin sample).  The last
// four fields serve the FP32 noise core: cf = (float)(c1 * c2), and for a tier step the band
// [lo, hi) of partial sums (in sum space, i.e. before the amplitude) inside which an FP32
// partial sum cannot decide the tier; err is the bound on |FP32 partial sum - FP64 partial sum|
// after this step.
struct ClimateStep {
    double sc, lac, c1, c2, thr, amp;
    int slot, act, tier, pad;
    float cf, lo, hi, err;
};

// Undecidable bands of the FP32 core for the temperature and ridge gates, in sum space
// (the DoublePerlin's octave sum before the amplitude): t_*[0] around -0.45, t_*[1] around 0.2;
// r_*[0..3] around -0.91, -0.42, 0.42, 0.91.  A total in [lo, hi) is re-taken in FP64.
struct F32Bands {
    float t_lo[2], t_hi[2];
    float r_lo[4], r_hi[4];
};

// Bound on |FP32 Perlin sample - exact sample| of perlin_y0_f32 (wg_device.cuh), in units of
// 2^-24; derived operation by operation in the comment above perlin_y0_f32.
constexpr double kPerlinF32ErrUlps = 44.0;
// The same bound for the 3-D sample perlin_3d_f32 (the cave noises of the entrance kernel).
constexpr double kPerlin3dF32ErrUlps = 60.0;
enum : int { ACT_NONE = 0, ACT_TIER, ACT_TIER_LAST, ACT_END_SUB_A, ACT_TEMPERATURE, ACT_RIDGE };
constexpr int kClimateSteps = kSlotsA;

// Host: the 18-step climate sequence for one preset, with the FP32 core's error bands
// (wg_engine.cu); the temperature / ridge bands of the same preset.
void build_climate_steps(const NoiseSpec *specs, int erosion, int temperature, ClimateStep *steps);
F32Bands build_f32_bands(const ClimateStep *steps);
// Host: builds the noise parameters, climate steps and FP32 bands of both presets and uploads
// them to the current device's constant memory (upload_tables).
void upload_phase1_tables();
// Host: whether every climate sampling coordinate of regions with rx, rz in [lo, hi] (inclusive)
// stays inside maintainPrecision's identity range (|v| < 1e7): a climate point is 4 * chunk + 2 with
// |chunk| <= 32 |r| + 23, scaled by at most 1.0181268882175227 and the largest climate lacunarity.
bool coords_small(int64_t lo, int64_t hi);

// An item of the breadth-first climate stage for one-region units: the unit, its partial sums.
struct SpotItem {
    uint32_t unit, pad;
    double sum, sum_a;
};

// Launchers (wg_phase1.cu).
void upload_tables(const NoiseSpec *specs, const ClimateStep *steps_normal, const ClimateStep *steps_large,
                   const F32Bands *bands);
void launch_climate(const BatchArgs &a, cudaStream_t s);
void launch_entrance(const BatchArgs &a, int grid, cudaStream_t s);
void launch_ladder(const BatchArgs &a, int grid, cudaStream_t s);
// Sets the kernels' shared-memory limits and the ladder's resident-block count on the current
// device, so that the launch functions make no further runtime calls (a stream capture may follow).
void prepare_phase1_launches();
size_t climate_smem_bytes(bool fp32_core);
// The climate stage of a batch whose units have one region each (spots mode), breadth first over
// two item lists of `cap` entries (counts: 2 words, device); climate survivors become records.
void launch_spot_climate(const BatchArgs &a, SpotItem *list0, SpotItem *list1, uint32_t *counts, uint32_t cap,
                         int sm_count, cudaStream_t s);
size_t spot_smem_bytes();
size_t entrance_smem_bytes();
// The FP32 core's error probe: noise `noise` (NoiseId) of seed d_seeds[b] at y = 0 and the n_points
// (x, z) of d_xz, FP32 core -> d_out32[b * n_points + i], FP64 -> d_out64[...].
void launch_noise_probe(const int64_t *d_seeds, uint32_t n_seeds, int noise, const double *d_xz, uint32_t n_points,
                        double *d_out32, double *d_out64, cudaStream_t s);
// The same for a 3-D cave noise of the entrance kernel (N_CAVE_ENTRANCE .. N_ROUGHNESS) at the
// points d_xyz (x, y, z triples): the FP32 core's samples summed in FP64, and the FP64 value.
void launch_noise_probe3d(const int64_t *d_seeds, uint32_t n_seeds, int noise, const double *d_xyz,
                          uint32_t n_points, double *d_out32, double *d_out64, cudaStream_t s);

}  // namespace wg
