// Seed Check phase-1 kernels; see wg_phase1.cuh for the pipeline.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <type_traits>

#include "wg_device.cuh"
#include "wg_phase1.cuh"

namespace wg {

namespace cg = cooperative_groups;

__constant__ NoiseSpec c_noise[N_NOISE_COUNT];
__constant__ ClimateStep c_steps[2][kClimateSteps];     // [large_biomes][step]
__constant__ int8_t c_slot_a[2][kSlotsA][3];             // climate slots: noise, sub, octave
__constant__ int8_t c_slot_c[2][kSlotsC][3];             // cave slots (the entrance kernel uses the first 18)
__constant__ F32Bands c_bands[2];                        // [large_biomes] FP32 core: temperature / ridge bands

// Slot bases of each noise inside the cave slot set (sub 0 octaves, then sub 1 octaves).
constexpr int kBaseEntrance = 0, kBaseRarity = 6, kBaseThickness = 8, kBaseSp1 = 10, kBaseSp2 = 12;
constexpr int kBaseRmod = 14, kBaseRough = 16, kBaseLayer = 18, kBaseCheese = 20, kBaseCont = 34;
constexpr int kBaseFlood = 52;

static void fill_slots(int8_t (*dst)[3], const NoiseSpec *specs, const int *noises, int nn, int expect) {
    int s = 0;
    for (int q = 0; q < nn; q++) {
        int np = specs[noises[q]].npresent;
        for (int sub = 0; sub < 2; sub++)
            for (int p = 0; p < np; p++) {
                dst[s][0] = (int8_t)noises[q];
                dst[s][1] = (int8_t)sub;
                dst[s][2] = (int8_t)p;
                s++;
            }
    }
    (void)expect;
}

void upload_tables(const NoiseSpec *specs, const ClimateStep *steps_normal, const ClimateStep *steps_large,
                   const F32Bands *bands) {
    cudaMemcpyToSymbol(c_noise, specs, sizeof(NoiseSpec) * N_NOISE_COUNT);
    cudaMemcpyToSymbol(c_bands, bands, sizeof(F32Bands) * 2);
    ClimateStep st[2][kClimateSteps];
    for (int i = 0; i < kClimateSteps; i++) {
        st[0][i] = steps_normal[i];
        st[1][i] = steps_large[i];
    }
    cudaMemcpyToSymbol(c_steps, st, sizeof(st));
    int8_t sa[2][kSlotsA][3], sc[2][kSlotsC][3];
    for (int lg = 0; lg < 2; lg++) {
        int na[3] = {lg ? N_EROSION_LARGE : N_EROSION, lg ? N_TEMPERATURE_LARGE : N_TEMPERATURE, N_RIDGE};
        fill_slots(sa[lg], specs, na, 3, kSlotsA);
        int nc[11] = {N_CAVE_ENTRANCE, N_SPAGHETTI_RARITY, N_SPAGHETTI_THICKNESS, N_SPAGHETTI_1, N_SPAGHETTI_2,
                      N_ROUGHNESS_MODULATOR, N_ROUGHNESS, N_CAVE_LAYER, N_CAVE_CHEESE,
                      lg ? N_CONTINENTALNESS_LARGE : N_CONTINENTALNESS, N_FLOODEDNESS};
        fill_slots(sc[lg], specs, nc, 11, kSlotsC);
    }
    cudaMemcpyToSymbol(c_slot_a, sa, sizeof(sa));
    cudaMemcpyToSymbol(c_slot_c, sc, sizeof(sc));
}

// ------------------------------------------------------------------------------------
// helpers
// ------------------------------------------------------------------------------------
// Global seed index and region of a batch-local unit / window offset.
__device__ __forceinline__ uint64_t unit_seed_index(const BatchArgs &a, uint32_t u) { return (a.unit0 + u) / a.n_win; }
__device__ __forceinline__ uint64_t unit_window(const BatchArgs &a, uint32_t u) { return (a.unit0 + u) % a.n_win; }
__device__ __forceinline__ uint64_t seed_value(const BatchArgs &a, uint64_t g) {
    if (a.spot_s48) return ((g & 0xFFFFull) << 48) | ((uint64_t)a.spot_s48[g >> 16] & 0xFFFFFFFFFFFFull);
    return a.seeds ? (uint64_t)a.seeds[g] : splitmix64(a.gen_base + g);
}
// Rect origin of seed g (shifted to the seed's spot region in spots mode).
__device__ __forceinline__ int rect_x0(const BatchArgs &a, uint64_t g) { return a.spot_rx ? a.rx0 + a.spot_rx[g >> 16] : a.rx0; }
__device__ __forceinline__ int rect_z0(const BatchArgs &a, uint64_t g) { return a.spot_rz ? a.rz0 + a.spot_rz[g >> 16] : a.rz0; }
// Everything about a batch-local unit: its seed, its window and the rect it walks.
struct UnitPos {
    uint64_t g;        // global seed index
    uint64_t rbase;    // first region of the window (index into the rect, rz outer, rx inner)
    uint32_t len;      // regions in the window
    int rx0, rz0, rw;  // the rect the window lies in
    int max_height;
};
__device__ __forceinline__ UnitPos unit_pos(const BatchArgs &a, uint32_t u) {
    UnitPos p;
    if (a.jobs) {
        // the last table entry whose first global unit is <= this unit
        const uint64_t ul = a.unit0 + u;
        uint32_t lo = 0, hi = a.n_jobs - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (a.jobs[mid].unit0 <= ul) lo = mid;
            else hi = mid - 1;
        }
        const JobGeom &j = a.jobs[lo];
        const uint64_t loc = ul - j.unit0 + j.first;
        p.g = j.seed0 + loc / j.n_win;
        p.rbase = (loc % j.n_win) * j.win;
        const uint64_t left = j.n_regions - p.rbase;
        p.len = (uint32_t)(left < j.win ? left : j.win);
        p.rx0 = j.rx0;
        p.rz0 = j.rz0;
        p.rw = j.rw;
        p.max_height = j.max_height;
        return p;
    }
    p.g = unit_seed_index(a, u);
    p.rbase = unit_window(a, u) * a.win;
    const uint64_t left = a.n_regions - p.rbase;
    p.len = (uint32_t)(left < a.win ? left : a.win);
    p.rx0 = rect_x0(a, p.g);
    p.rz0 = rect_z0(a, p.g);
    p.rw = a.rw;
    p.max_height = a.max_height;
    return p;
}
// Region (rx, rz) of region index r of a unit's rect (rz outer, rx inner: search.c:148-149).
__device__ __forceinline__ void unit_region_xz(const UnitPos &p, uint64_t r, int &rx, int &rz) {
    rz = p.rz0 + (int)(r / (uint64_t)p.rw);
    rx = p.rx0 + (int)(r % (uint64_t)p.rw);
}

__device__ __forceinline__ void note_code(const BatchArgs &a, uint64_t g, uint64_t r, int code, int tier) {
    if (a.codes) {
        size_t at = (size_t)g * (size_t)a.n_regions + (size_t)r;
        a.codes[at] = (int8_t)code;
        a.tiers[at] = (int8_t)tier;
    }
}

// Bytes between consecutive slot blocks: 256 rows of kUnits columns plus 16 bytes, so the two
// slots a warp builds at once (one per half-warp) sit 4 banks apart.
constexpr int kPitch = 256 * kUnits + 16;
// The ladder kernel keeps its 54 tables as columns of one block (pitch 56 bytes per row).
constexpr int kLadderStride = 56;

// Table sources: where a sampler's permutation table and origin live.
struct SrcCols {  // byte-interleaved blocks of kUnits columns, origins [slot][unit]
    const uint8_t *perm;
    const double *ox, *oy, *oz;
    const uint32_t *gt;
    int unit;
    __device__ __forceinline__ double p3(int slot, double x, double y, double z) const {
        ColTable<kUnits> T{perm + slot * kPitch + unit, gt};
        int o = slot * kUnits + unit;
        return perlin_3d(T, ox[o], oy[o], oz[o], x, y, z);
    }
};
struct SrcColsF {  // the same columns read by the FP32 core (row 256 of every column = row 0)
    const uint8_t *perm;
    const double *ox, *oy, *oz;
    const GradF *gf;
    int unit;
    __device__ __forceinline__ float p3(int slot, double x, double y, double z) const {
        ColTableF<kUnits> T{perm + slot * kPitch + unit, gf};
        int o = slot * kUnits + unit;
        return perlin_3d_f32(T, ox[o], oy[o], oz[o], x, y, z);
    }
};
struct SrcFlat {  // the ladder's block: table of slot s in column s, origins [slot][3]
    const uint8_t *perm;
    const double *org;
    const uint32_t *gt;
    __device__ __forceinline__ double p3(int slot, double x, double y, double z) const {
        ColTable<kLadderStride> T{perm + slot, gt};
        return perlin_3d(T, org[3 * slot], org[3 * slot + 1], org[3 * slot + 2], x, y, z);
    }
};

// DoublePerlinNoiseSampler.sample (noise.c:263-289).
template <class S>
__device__ double dbl3d(const S &src, int noise, int base, double x, double y, double z) {
    const NoiseSpec &ns = c_noise[noise];
    const int np = ns.npresent;
    double a = 0.0;
    for (int p = 0; p < np; p++) {
        double l = ns.lac[p];
        double v = src.p3(base + p, keep_precision(x * l), keep_precision(y * l), keep_precision(z * l));
        a += (ns.amp[p] * v) * ns.per[p];
    }
    double xs = x * kDblScale, ys = y * kDblScale, zs = z * kDblScale;
    double b = 0.0;
    for (int p = 0; p < np; p++) {
        double l = ns.lac[p];
        double v = src.p3(base + np + p, keep_precision(xs * l), keep_precision(ys * l), keep_precision(zs * l));
        b += (ns.amp[p] * v) * ns.per[p];
    }
    return (a + b) * ns.amplitude;
}

// SearchCoords cave heuristics (caves.c:41-130).
__device__ __forceinline__ double tunnel_scale(double v) {
    if (v < -0.5) return 0.75;
    if (v < 0.0) return 1.0;
    if (v < 0.5) return 1.5;
    return 2.0;
}

template <class S>
__device__ double spaghetti(const S &src, int x, int y, int z) {
    double e = tunnel_scale(dbl3d(src, N_SPAGHETTI_RARITY, kBaseRarity, (double)(int)((uint32_t)x * 2u), (double)y,
                                  (double)(int)((uint32_t)z * 2u)));
    double tv = dbl3d(src, N_SPAGHETTI_THICKNESS, kBaseThickness, (double)x, (double)y, (double)z);
    double h = lerp((tv - -1.0) / (1.0 - -1.0), 0.065, 0.088);
    double l = dbl3d(src, N_SPAGHETTI_1, kBaseSp1, (double)x / e, (double)y / e, (double)z / e);
    double m = fabs(e * l) - h;
    double n = dbl3d(src, N_SPAGHETTI_2, kBaseSp2, (double)x / e, (double)y / e, (double)z / e);
    double o = fabs(e * n) - h;
    double p = clampd(jmax(m, o), -1.0, 1.0);
    double mod = dbl3d(src, N_ROUGHNESS_MODULATOR, kBaseRmod, (double)x, (double)y, (double)z);
    double rgh = dbl3d(src, N_ROUGHNESS, kBaseRough, (double)x, (double)y, (double)z);
    double q = (-0.05 + (-0.05 * mod)) * (-0.4 + fabs(rgh));
    return p + q;
}

template <class S>
__device__ double entrance(const S &src, int x, int y, int z) {
    double ent = dbl3d(src, N_CAVE_ENTRANCE, kBaseEntrance, (double)x * 0.75, (double)y * 0.5, (double)z * 0.75);
    double t = (10.0 + (double)y) / 40.0;
    double cl = t < 0.0 ? 0.3 : (t > 1.0 ? 0.0 : lerp(t, 0.3, 0.0));
    double cc = ent + 0.37 + cl;
    return jmin(cc, spaghetti(src, x, y, z));
}

template <class S>
__device__ double cheese(const S &src, int x, int y, int z) {
    double layer = dbl3d(src, N_CAVE_LAYER, kBaseLayer, (double)x, (double)(int)((uint32_t)y * 8u), (double)z);
    double av = 4.0 * layer * layer;
    double raw = dbl3d(src, N_CAVE_CHEESE, kBaseCheese, (double)x, (double)y * 0.6666666666666666, (double)z);
    return av + clampd(0.27 + raw, -1.0, 1.0);
}

// FP32 core: the reference's FP64 values, for an entrance decision or a tunnel-scale interval
// whose FP32-core value lies inside its error band (kept out of line: the rare path).
__device__ __noinline__ double entrance64(SrcCols src, int x, int y, int z) { return entrance(src, x, y, z); }
__device__ __noinline__ double rarity64(SrcCols src, int x, int y, int z) {
    return dbl3d(src, N_SPAGHETTI_RARITY, kBaseRarity, (double)(int)((uint32_t)x * 2u), (double)y,
                 (double)(int)((uint32_t)z * 2u));
}

// ------------------------------------------------------------------------------------
// climate kernel
// ------------------------------------------------------------------------------------
// Step parameters are stored field by field (structure of arrays): threads sit at different
// steps, and consecutive 8-byte entries fall in different banks.
struct ClimateSteps {
    double sc[kClimateSteps], lac[kClimateSteps], c1[kClimateSteps], c2[kClimateSteps];
    double thr[kClimateSteps], amp[kClimateSteps];
    int slot[kClimateSteps], act[kClimateSteps], tier[kClimateSteps];
    float cf[kClimateSteps], lo[kClimateSteps], hi[kClimateSteps];   // FP32 core (ClimateStep)
};

// Per-table y origin: the FP64 path keeps hy and fade(hy) as doubles; the FP32 core keeps hy as a
// double (for its FP64 rechecks, which recompute fade(hy) in the reference's order) and
// rn(hy), rn(fade(hy)) as floats.
template <bool F32>
struct TableY {
    double hy[kSlotsA * kUnits], fy[kSlotsA * kUnits];
    __device__ __forceinline__ double fy64(int o) const { return fy[o]; }
};
template <>
struct TableY<true> {
    double hy[kSlotsA * kUnits];
    float hyf[kSlotsA * kUnits], fyf[kSlotsA * kUnits];
    __device__ __forceinline__ double fy64(int o) const { return fade(hy[o]); }
};

constexpr int kClimateWarps = kThreadsA / 32;
constexpr int kWarpList = 112;   // tier-0 survivors a warp carries (a warp has <= 192 regions a chunk, ~43 % pass)

template <bool F32>
struct ClimateSmem {
    using Real = typename std::conditional<F32, float, double>::type;
    uint8_t perm[kSlotsA * kPitch];           // slot s, row k, unit u at s * kPitch + k * kUnits + u
    double ox[kSlotsA * kUnits], oz[kSlotsA * kUnits];
    TableY<F32> ty;
    int jy[kSlotsA * kUnits];
    int2 pos[kChunk * kUnits];                 // hut chunk (cx, cz) of window offset c0 + j, unit u
    // each warp's survivors of the chunk (unit << 16 | (j - c0)) and their erosion partial sums:
    // the tier-0 survivors of the warp's own regions, compacted in place after every later step
    uint32_t wl[kClimateWarps][kWarpList];
    Real wsum[kClimateWarps][kWarpList];
    uint32_t surv[kUnits * kRecordCap];
    uint32_t cnt[kUnits];
    uint32_t len[kUnits];                      // regions in the unit's window (0: past the batch)
    uint64_t g[kUnits], rbase[kUnits], seed[kUnits];   // seed index, first region, world seed
    uint32_t col0[kUnits];                     // column of the unit's first region in its rect row
    int row0[kUnits];                          // rz of the unit's first region
    int rx0u[kUnits];                          // rect x origin of the unit's seed
    uint32_t rwu[kUnits];                      // rect width of the unit's job
    unsigned int hist[P1_KINDS + kTiers];
    uint32_t grad[kGradWords];
    GradF gf;                                  // FP32 core: the gradient vectors as floats
    ClimateSteps steps;
};

size_t climate_smem_bytes(bool fp32_core) { return fp32_core ? sizeof(ClimateSmem<true>) : sizeof(ClimateSmem<false>); }

// A record holding one survivor, for a unit whose shared list is full.
__device__ void emit_single(const BatchArgs &a, uint32_t u, uint32_t off_in_win) {
    uint32_t ri = atomicAdd(&a.counters[CNT_RECORDS], 1u);
    uint32_t off = atomicAdd(&a.counters[CNT_SURVIVORS], 1u);
    if (ri < a.cap_rec && off < a.cap_surv) {
        a.rec_unit[ri] = u;
        a.rec_off[ri] = off;
        a.rec_cnt[ri] = 1;
        a.surv_region[off] = off_in_win;
    } else {
        if (ri < a.cap_rec) a.rec_cnt[ri] = 0;  // a reserved record is never left stale
        atomicOr(&a.counters[CNT_OVERFLOW], 1u);
    }
}

template <class Sm>
__device__ __forceinline__ void keep_survivor(Sm &S, const BatchArgs &a, int iu, uint32_t j) {
    uint32_t q = atomicAdd(&S.cnt[iu], 1u);
    if (q < kRecordCap) S.surv[iu * kRecordCap + q] = j;
    else emit_single(a, blockIdx.x * kUnits + (uint32_t)iu, j);
}

template <class Sm>
__device__ __forceinline__ void climate_reject(Sm &S, const BatchArgs &a, int iu, uint32_t j, int code, int tier) {
    atomicAdd(&S.hist[code], 1u);
    if (tier >= 0) atomicAdd(&S.hist[P1_KINDS + tier], 1u);
    note_code(a, S.g[iu], S.rbase[iu] + j, code, tier);
}

// Erosion rejections are counted per thread in registers (16-bit fields, tiers 0-3 and 4-6) and
// added to the histogram once at the end; a shared counter hit by most lanes of a warp at once
// would serialise.  A field cannot overflow: per chunk a thread rejects at most 6 regions in the
// tier-0 pass, at most 4 in each of the 6 later erosion steps (a warp's list holds <= kWarpList
// = 112 regions, 4 rounds of 32) and at most 6 in its own walks of a full list's overflow, over at
// most 43 chunks (4,096 / 96).
struct TierCounts {
    uint64_t lo = 0, hi = 0;
    __device__ __forceinline__ void add(int tier) {
        if (tier < 4) lo += 1ull << (16 * tier);
        else hi += 1ull << (16 * (tier - 4));
    }
    __device__ __forceinline__ uint32_t get(int tier) const {
        return (uint32_t)(((tier < 4 ? lo : hi) >> (16 * (tier & 3))) & 0xFFFFu);
    }
};

template <class Sm>
__device__ __forceinline__ void erosion_reject(const Sm &S, const BatchArgs &a, TierCounts &tc, int iu, uint32_t j,
                                               int tier) {
    tc.add(tier);
    note_code(a, S.g[iu], S.rbase[iu] + j, P1_EROSION, tier);
}

// One y = 0 Perlin sample of climate step k for unit iu at climate point (xc, zc), in FP64 with
// the reference's operations (the FP64 path, and the FP32 core's rechecks).
template <class Sm>
__device__ __forceinline__ double climate_sample(const Sm &S, int iu, int k, double xc, double zc) {
    const ClimateSteps &st = S.steps;
    const int slot = st.slot[k];
    const int o = slot * kUnits + iu;
    const double sc = st.sc[k], lac = st.lac[k];
    ColTable<kUnits> T{S.perm + slot * kPitch + iu, S.grad};
    return perlin_y0(T, S.ox[o], S.oz[o], S.jy[o], S.ty.hy[o], S.ty.fy64(o), keep_precision((xc * sc) * lac),
                     keep_precision((zc * sc) * lac));
}

// The same sample in the FP32 core (coordinates reduced in FP64, the rest in FP32).  SMALL: the
// host has shown every coordinate of the batch to lie inside maintainPrecision's identity range
// (BatchArgs::small_coords), so the check is left out and the sample is one branch-free block.
template <bool SMALL>
__device__ __forceinline__ float climate_sample_f32(const ClimateSmem<true> &S, int iu, int k, double xc, double zc) {
    const ClimateSteps &st = S.steps;
    const int slot = st.slot[k];
    const int o = slot * kUnits + iu;
    const double sc = st.sc[k], lac = st.lac[k];
    ColTableF<kUnits> T{S.perm + slot * kPitch + iu, &S.gf};
    const double x = (xc * sc) * lac, z = (zc * sc) * lac;
    return perlin_y0_f32(T, S.ox[o], S.oz[o], S.jy[o], S.ty.hyf[o], S.ty.fyf[o], SMALL ? x : keep_precision(x),
                         SMALL ? z : keep_precision(z));
}

// One climate step's table of one unit with its parameters held in registers: the tier-0 pass
// samples the same two tables for every region a thread takes (a thread's unit is tid % kUnits in
// every trip), so their origins, y terms and step constants are read from shared memory once.
struct Y0Table {
    const uint8_t *col;
    double ox, oz, sc, lac;
    int jy;
    float hyf, fyf;
};
__device__ __forceinline__ Y0Table y0_table(const ClimateSmem<true> &S, int iu, int k) {
    const ClimateSteps &st = S.steps;
    const int slot = st.slot[k], o = slot * kUnits + iu;
    return Y0Table{S.perm + slot * kPitch + iu, S.ox[o], S.oz[o], st.sc[k], st.lac[k], S.jy[o], S.ty.hyf[o],
                   S.ty.fyf[o]};
}
// climate_sample_f32 from a Y0Table: the same operations on the same values.
template <bool SMALL>
__device__ __forceinline__ float climate_sample_f32(const ClimateSmem<true> &S, const Y0Table &y, double xc, double zc) {
    ColTableF<kUnits> T{y.col, &S.gf};
    const double x = (xc * y.sc) * y.lac, z = (zc * y.sc) * y.lac;
    return perlin_y0_f32(T, y.ox, y.oz, y.jy, y.hyf, y.fyf, SMALL ? x : keep_precision(x),
                         SMALL ? z : keep_precision(z));
}

// FP64 octave sum of climate steps [k0, k1] in the reference's order (sum += (c1 * v) * c2):
// the exact partial sum an FP32 recheck decides on.
template <class Sm>
__device__ __noinline__ double climate_sum64(const Sm &S, int iu, int k0, int k1, double xc, double zc) {
    const ClimateSteps &st = S.steps;
    double sum = 0.0;
    for (int k = k0; k <= k1; k++) sum += (st.c1[k] * climate_sample(S, iu, k, xc, zc)) * st.c2[k];
    return sum;
}

// FP64 DoublePerlin value of a temperature / ridge noise whose steps are k0 .. k0 + n - 1 (sub A,
// then sub B; ACT_END_SUB_A closes sub A), as the state machine combines it.
template <class Sm>
__device__ __noinline__ double climate_value64(const Sm &S, int iu, int k0, int n, double xc, double zc) {
    const ClimateSteps &st = S.steps;
    double sum = 0.0, sum_a = 0.0;
    for (int p = 0; p < n; p++) {
        const int k = k0 + p;
        sum += (st.c1[k] * climate_sample(S, iu, k, xc, zc)) * st.c2[k];
        if (st.act[k] == ACT_END_SUB_A) {
            sum_a = sum;
            sum = 0.0;
        }
    }
    return (sum_a + sum) * st.amp[k0 + n - 1];
}

template <class Sm>
__device__ __forceinline__ void climate_point(const Sm &S, int iu, uint32_t jl, double &xc, double &zc) {
    const int2 c = S.pos[jl * kUnits + iu];
    xc = (c.x * 16 + 8) * 0.25;   // exact: an integer over 4
    zc = (c.y * 16 + 8) * 0.25;
}

// The climate steps from step k0 for one region (e = unit << 16 | offset in the chunk), one Perlin
// sample per loop trip, run by one thread: the path for a tier-0 survivor that finds its warp's
// list full.  Always FP64 (the FP32 core enters it with k0 = 0 and recomputes the partial sum
// exactly).
template <class Sm>
__device__ void climate_rest(Sm &S, const BatchArgs &a, TierCounts &tc, uint32_t e, uint32_t c0, int k0, double sum,
                             double xc, double zc) {
    const ClimateSteps &st = S.steps;
    const int iu = (int)(e >> 16);
    const uint32_t j = c0 + (e & 0xFFFFu);
    double sum_a = 0.0;
    for (int k = k0; k < kClimateSteps; k++) {
        const double v = climate_sample(S, iu, k, xc, zc);
        sum += (st.c1[k] * v) * st.c2[k];
        switch (st.act[k]) {
            case ACT_TIER:
                if (sum * st.amp[k] < st.thr[k]) {
                    erosion_reject(S, a, tc, iu, j, st.tier[k]);
                    return;
                }
                break;
            case ACT_TIER_LAST:
                if (sum * st.amp[k] < st.thr[k]) {
                    erosion_reject(S, a, tc, iu, j, st.tier[k]);
                    return;
                }
                sum = 0.0;   // temperature and ridge follow here
                break;
            case ACT_END_SUB_A:
                sum_a = sum;
                sum = 0.0;
                break;
            case ACT_TEMPERATURE: {
                double t = (sum_a + sum) * st.amp[k];
                bool bad = a.mc_1_18_2 ? (t < -0.45) : (t > 0.2 || t < -0.45);
                if (bad) {
                    climate_reject(S, a, iu, j, P1_TEMPERATURE, -1);
                    return;
                }
                sum = 0.0;
                break;
            }
            case ACT_RIDGE: {
                double rg = (sum_a + sum) * st.amp[k];
                if ((rg > 0.42 && rg < 0.91) || (rg < -0.42 && rg > -0.91) || (!a.pre_26_2 && rg <= -0.91))
                    climate_reject(S, a, iu, j, P1_RIDGE, -1);
                else
                    keep_survivor(S, a, iu, j);   // climate survivor, not yet a verdict
                return;
            }
            default:
                break;
        }
    }
}

// Thread t owns table (slot t / kUnits, unit t % kUnits) during the build.  The evaluation of a
// chunk of regions runs in phases separated by barriers: (1) tier 0 (samples 0A, 0B) for every
// region, a uniform loop that rejects ~57 %; (2) the remaining erosion tiers for the survivors,
// taken from a shared list by any thread; (3) temperature and (4) ridge for the ~5 % that pass
// erosion, one sample per thread, summed per region in the reference's order.
//
// F32 (the FP32 noise core): every sample of the four phases is taken in FP32 (perlin_y0_f32)
// and the partial sums are carried in FP32.  A gate decides from the FP32 value when it lies
// outside the step's error band ([lo, hi) around the threshold in sum space, from the derived
// bound); inside the band the thread recomputes that region's samples in FP64 in the reference's
// order and decides exactly as the FP64 path does.  So every decision, and with it the reject
// codes, tier histogram and survivor set, equals the FP64 path's.
template <bool F32, bool SMALL>
__global__ void __launch_bounds__(kThreadsA, 2) climate_kernel(BatchArgs a) {
    using Real = typename ClimateSmem<F32>::Real;
    extern __shared__ __align__(16) uint8_t smem_raw[];
    ClimateSmem<F32> &S = *reinterpret_cast<ClimateSmem<F32> *>(smem_raw);
    batch_range(a);
    if (blockIdx.x * kUnits >= a.n_units) return;   // past this batch (a launch sized for a larger one)
    const int tid = threadIdx.x;
    const int my_slot = tid / kUnits, uu = tid % kUnits;
    const int large = a.large_biomes ? 1 : 0;
    uint32_t rechecks = 0;
    const bool all_rechecks = F32 && a.fp32_core == 2;   // every FP32 gate re-taken in FP64 (a check mode)
    if (tid < P1_KINDS + kTiers) S.hist[tid] = 0;
    fill_grad_table(S.grad, tid);
    if (F32) fill_grad_table_f32(&S.gf, tid);
    if (tid < kClimateSteps) {
        const ClimateStep &c = c_steps[large][tid];
        S.steps.sc[tid] = c.sc;
        S.steps.lac[tid] = c.lac;
        S.steps.c1[tid] = c.c1;
        S.steps.c2[tid] = c.c2;
        S.steps.thr[tid] = c.thr;
        S.steps.amp[tid] = c.amp;
        S.steps.slot[tid] = c.slot;
        S.steps.act[tid] = c.act;
        S.steps.tier[tid] = c.tier;
        S.steps.cf[tid] = c.cf;
        S.steps.lo[tid] = c.lo;
        S.steps.hi[tid] = c.hi;
    }

    const uint32_t u = blockIdx.x * kUnits + (uint32_t)uu;
    const bool valid = u < a.n_units;
    UnitPos up{};
    up.rw = 1;
    if (valid) up = unit_pos(a, u);
    const uint64_t g = up.g;
    const uint64_t seed = valid ? seed_value(a, g) : 0;
    const uint32_t len = valid ? up.len : 0;
    if (tid < kUnits) {
        S.cnt[tid] = 0;
        S.len[tid] = len;
        S.g[tid] = g;
        S.rbase[tid] = up.rbase;
        S.seed[tid] = seed;
        S.col0[tid] = (uint32_t)(up.rbase % (uint64_t)up.rw);
        S.row0[tid] = up.rz0 + (int)(up.rbase / (uint64_t)up.rw);
        S.rx0u[tid] = up.rx0;
        S.rwu[tid] = (uint32_t)up.rw;
    }
    TierCounts tc;

    // ---- build: every thread shuffles one table ----
    if (!a.single_biome) {
        perm_blocks_init<kUnits, kPitch>(S.perm, kSlotsA, tid, kThreadsA);
        __syncthreads();
        if (valid) {
            const int noise = c_slot_a[large][my_slot][0], sub = c_slot_a[large][my_slot][1],
                      p = c_slot_a[large][my_slot][2];
            Xr r = octave_rng(c_noise[noise], seed_fork_of(seed), sub, p);
            double ox, oy, oz;
            uint8_t *col = S.perm + my_slot * kPitch + uu;
            perlin_shuffle<kUnits>(col, r, ox, oy, oz);
            col[256 * kUnits] = col[0];   // row 256 = row 0, in the slot's padding (ColTableF)
            const int o = my_slot * kUnits + uu;
            int jy = (int)floor(oy);
            double hy = oy - jy;
            S.ox[o] = ox;
            S.oz[o] = oz;
            S.ty.hy[o] = hy;
            if constexpr (F32) {
                S.ty.hyf[o] = __double2float_rn(hy);
                S.ty.fyf[o] = __double2float_rn(fade(hy));
            } else {
                S.ty.fy[o] = fade(hy);
            }
            S.jy[o] = jy;
        }
    }
    __shared__ uint32_t max_len;
    if (tid == 0) max_len = 0;
    __syncthreads();
    if (valid && tid < kUnits) atomicMax(&max_len, len);
    __syncthreads();
    const uint32_t cta_len = max_len;
    const ClimateSteps &st = S.steps;

    // The regions of a chunk are evaluated warp by warp: a warp stages the hut chunks of its own
    // regions (q = tid + r * kThreadsA), takes tier 0 for them, and carries its tier-0 survivors
    // through the remaining erosion tiers, temperature and ridge in its own list, synchronising
    // with __syncwarp only: no step of one warp waits for another warp.
    const int warp = tid >> 5, lane = tid & 31;
    uint32_t *const wl = S.wl[warp];
    Real *const wsum = S.wsum[warp];
    const unsigned lanes_below = (1u << lane) - 1u;
    constexpr int kT0 = 8, kR0 = 12;   // first temperature / ridge step
    for (uint32_t c0 = 0; c0 < cta_len; c0 += kChunk) {
        // ---- stage the hut chunks of this warp's regions (j < len: c0 + q / kUnits < c0 + kChunk) ----
        for (int q = tid; q < kChunk * kUnits; q += kThreadsA) {
            const int qu = q % kUnits;
            const uint32_t j = c0 + (uint32_t)(q / kUnits);
            if (j >= S.len[qu]) continue;
            const uint32_t t = S.col0[qu] + j;   // region offset from the unit's first row start
            const uint32_t rw = S.rwu[qu];
            const int rz = S.row0[qu] + (int)(t / rw), rx = S.rx0u[qu] + (int)(t % rw);
            int cx, cz;
            hut_chunk(S.seed[qu], rx, rz, a.salt, cx, cz);
            S.pos[q] = make_int2(cx, cz);
        }

        // ---- tier 0 for every region: samples 0A and 0B with loop-invariant parameters ----
        uint32_t wcount = 0;   // the warp's list length, the same in every lane
        {
            const int nq = kUnits * kChunk;
            // The trips are warp-uniform (every lane takes kTrips of them, a lane past its unit's
            // regions with valid = false), so the append needs one ballot and a list length held
            // in registers.
            constexpr int kTrips = (kUnits * kChunk + kThreadsA - 1) / kThreadsA;
            static_assert(kThreadsA % kUnits == 0, "a thread's unit must be the same in every trip");
            const int iu = tid % kUnits;
            const uint32_t len = S.len[iu];
            // the decision's bookkeeping: warp-aggregated append of a survivor to the warp's list
            auto tier0_decide = [&](bool valid, uint32_t jl, Real sum, bool pass, double xc, double zc) {
                const uint32_t j = c0 + jl;
                const unsigned m = __ballot_sync(0xFFFFFFFFu, valid && pass);
                const uint32_t base = wcount;
                wcount += (uint32_t)__popc(m);
                if (!valid) return;
                if (!pass) {
                    erosion_reject(S, a, tc, iu, j, st.tier[1]);
                } else {
                    const uint32_t t = base + (uint32_t)__popc(m & lanes_below);
                    if (t < kWarpList) {
                        wl[t] = ((uint32_t)iu << 16) | jl;
                        wsum[t] = sum;
                    } else if (F32) {
                        // list full: this thread walks the region through the rest itself, in FP64
                        climate_rest(S, a, tc, ((uint32_t)iu << 16) | jl, c0, 0, 0.0, xc, zc);
                    } else {
                        climate_rest(S, a, tc, ((uint32_t)iu << 16) | jl, c0, 2, (double)sum, xc, zc);
                    }
                }
            };
            if (a.single_biome) {   // phase1.c:96: the climate gates are skipped
                for (int q = tid; q < nq; q += kThreadsA) {
                    const int iu = q % kUnits;
                    const uint32_t j = c0 + (uint32_t)(q / kUnits);
                    if (j < S.len[iu]) keep_survivor(S, a, iu, j);
                }
            } else if constexpr (F32) {
                const Y0Table y0a = y0_table(S, iu, 0), y0b = y0_table(S, iu, 1);
                const float cf0 = st.cf[0], cf1 = st.cf[1], lo1 = st.lo[1], hi1 = st.hi[1];
#pragma unroll 1   // one copy of the sample code: the chunk loop cycles through every phase
                for (int r = 0; r < kTrips; r++) {
                    const int q = tid + r * kThreadsA;
                    const uint32_t jl = (uint32_t)(q / kUnits);
                    const bool valid = q < nq && c0 + jl < len;
                    if (__ballot_sync(0xFFFFFFFFu, valid) == 0u) continue;   // the whole warp is past its regions
                    double xc = 0.0, zc = 0.0;
                    float sum = 0.0f;
                    bool pass = false;
                    if (valid) {
                        climate_point(S, iu, jl, xc, zc);
                        sum = __fmul_rn(cf0, climate_sample_f32<SMALL>(S, y0a, xc, zc));
                        sum = __fmaf_rn(cf1, climate_sample_f32<SMALL>(S, y0b, xc, zc), sum);
                        if (!all_rechecks && sum < lo1) {
                            pass = false;
                        } else if (!all_rechecks && sum >= hi1) {
                            pass = true;
                        } else {   // inside the error band: decide in FP64
                            rechecks++;
                            pass = !(climate_sum64(S, iu, 0, 1, xc, zc) * st.amp[1] < st.thr[1]);
                        }
                    }
                    tier0_decide(valid, jl, sum, pass, xc, zc);
                }
            } else {
#pragma unroll 1   // one copy of the sample code: the chunk loop cycles through every phase
                for (int r = 0; r < kTrips; r++) {
                    const int q = tid + r * kThreadsA;
                    const uint32_t jl = (uint32_t)(q / kUnits);
                    const bool valid = q < nq && c0 + jl < len;
                    if (__ballot_sync(0xFFFFFFFFu, valid) == 0u) continue;   // the whole warp is past its regions
                    double xc = 0.0, zc = 0.0, sum = 0.0;
                    bool pass = false;
                    if (valid) {
                        climate_point(S, iu, jl, xc, zc);
                        sum += (st.c1[0] * climate_sample(S, iu, 0, xc, zc)) * st.c2[0];
                        sum += (st.c1[1] * climate_sample(S, iu, 1, xc, zc)) * st.c2[1];
                        pass = !(sum * st.amp[1] < st.thr[1]);
                    }
                    tier0_decide(valid, jl, sum, pass, xc, zc);
                }
            }
        }
        __syncwarp();   // the list's entries are visible to the whole warp
        uint32_t n = min(wcount, (uint32_t)kWarpList);

        // ---- the remaining erosion tiers, breadth first over the warp's list: every listed region
        // takes erosion step k (one sample with the step's slot and constants), its tier check, and
        // the survivors are compacted in place for step k + 1 ----
        if (!a.single_biome) {
#pragma unroll 1
            for (int k = 2; n && k < kClimateSteps && st.act[k] != ACT_NONE && st.act[k] <= ACT_TIER_LAST; k++) {
                const double c1 = st.c1[k], c2 = st.c2[k], amp = st.amp[k], thr = st.thr[k];
                const float cf = st.cf[k], lo = st.lo[k], hi = st.hi[k];
                const int tier = st.tier[k];
                // rounds of 32 items, compacted as they go: round b's survivors land at
                // [nn, nn + kept) <= b + 32, on items every lane has read already (__syncwarp
                // between the reads and the writes), never on a later round's items
                uint32_t nn = 0;
#pragma unroll 1
                for (uint32_t b = 0; b < n; b += 32) {
                    const uint32_t q = b + (uint32_t)lane;
                    bool keep = false;
                    uint32_t e = 0;
                    Real sum = 0;
                    if (q < n) {
                        e = wl[q];
                        const int iu = (int)(e >> 16);
                        double xc, zc;
                        climate_point(S, iu, e & 0xFFFFu, xc, zc);
                        bool reject;
                        if constexpr (F32) {
                            sum = __fmaf_rn(cf, climate_sample_f32<SMALL>(S, iu, k, xc, zc), wsum[q]);
                            if (!all_rechecks && sum < lo) {
                                reject = true;
                            } else if (!all_rechecks && sum >= hi) {
                                reject = false;
                            } else {   // inside the error band: the exact partial sum of steps 0..k
                                rechecks++;
                                reject = climate_sum64(S, iu, 0, k, xc, zc) * amp < thr;
                            }
                        } else {
                            sum = wsum[q];
                            sum += (c1 * climate_sample(S, iu, k, xc, zc)) * c2;
                            reject = sum * amp < thr;
                        }
                        if (reject) erosion_reject(S, a, tc, iu, c0 + (e & 0xFFFFu), tier);
                        else keep = true;
                    }
                    const unsigned m = __ballot_sync(0xFFFFFFFFu, keep);
                    __syncwarp();   // every lane has read its item of this round
                    if (keep) {
                        const uint32_t at = nn + (uint32_t)__popc(m & lanes_below);
                        wl[at] = e;
                        wsum[at] = sum;
                    }
                    nn += (uint32_t)__popc(m);
                }
                __syncwarp();   // the compacted list is complete
                n = nn;
            }
        } else {
            n = 0;
        }

        // ---- temperature for the warp's erosion survivors: four lanes per region, one sample each,
        // summed in the reference's order by the first of the four; survivors compacted in place ----
        uint32_t nr = 0;
        for (uint32_t base = 0; base < n; base += 8) {
            const uint32_t i = base + (uint32_t)(lane >> 2);
            const int p = lane & 3;
            const bool have = i < n;
            const uint32_t e = have ? wl[i] : 0u;
            const int iu = (int)(e >> 16);
            double xc = 0.0, zc = 0.0;
            Real v = 0;
            if (have) {
                climate_point(S, iu, e & 0xFFFFu, xc, zc);
                if constexpr (F32) v = climate_sample_f32<SMALL>(S, iu, kT0 + p, xc, zc);
                else v = climate_sample(S, iu, kT0 + p, xc, zc);
            }
            const Real vs[4] = {v, __shfl_down_sync(0xFFFFFFFFu, v, 1), __shfl_down_sync(0xFFFFFFFFu, v, 2),
                                __shfl_down_sync(0xFFFFFFFFu, v, 3)};
            bool keep = false;
            if (have && p == 0) {
                bool bad;
                if constexpr (F32) {
                    float sum = 0.0f;
                    for (int q = 0; q < 4; q++) sum = __fmaf_rn(st.cf[kT0 + q], vs[q], sum);
                    const F32Bands &B = c_bands[large];
                    if (all_rechecks || (sum >= B.t_lo[0] && sum < B.t_hi[0]) || (sum >= B.t_lo[1] && sum < B.t_hi[1])) {
                        rechecks++;
                        const double t = climate_value64(S, iu, kT0, 4, xc, zc);
                        bad = a.mc_1_18_2 ? (t < -0.45) : (t > 0.2 || t < -0.45);
                    } else {
                        const bool low = sum < B.t_lo[0], high = sum >= B.t_hi[1];   // t < -0.45, t > 0.2
                        bad = a.mc_1_18_2 ? low : (low || high);
                    }
                } else {
                    double sum = 0.0, sum_a = 0.0;
                    for (int q = 0; q < 4; q++) {   // the state machine's accumulation, steps kT0..kT0+3
                        const int k = kT0 + q;
                        sum += (st.c1[k] * vs[q]) * st.c2[k];
                        if (st.act[k] == ACT_END_SUB_A) {
                            sum_a = sum;
                            sum = 0.0;
                        }
                    }
                    const double t = (sum_a + sum) * st.amp[kT0 + 3];
                    bad = a.mc_1_18_2 ? (t < -0.45) : (t > 0.2 || t < -0.45);
                }
                if (bad) climate_reject(S, a, iu, c0 + (e & 0xFFFFu), P1_TEMPERATURE, -1);
                else keep = true;
            }
            const unsigned m = __ballot_sync(0xFFFFFFFFu, keep);
            __syncwarp();   // this round's reads are done before its survivors are written
            if (keep) wl[nr + (uint32_t)__popc(m & lanes_below)] = e;
            nr += (uint32_t)__popc(m);
        }
        __syncwarp();

        // ---- ridge for those that passed temperature: six lanes per region (lanes 0-29) ----
        for (uint32_t base = 0; base < nr; base += 5) {
            const uint32_t i = base + (uint32_t)(lane / 6);
            const int p = lane % 6;
            const bool have = lane < 30 && i < nr;
            const uint32_t e = have ? wl[i] : 0u;
            const int iu = (int)(e >> 16);
            double xc = 0.0, zc = 0.0;
            Real v = 0;
            if (have) {
                climate_point(S, iu, e & 0xFFFFu, xc, zc);
                if constexpr (F32) v = climate_sample_f32<SMALL>(S, iu, kR0 + p, xc, zc);
                else v = climate_sample(S, iu, kR0 + p, xc, zc);
            }
            const Real vs[6] = {v,
                                __shfl_down_sync(0xFFFFFFFFu, v, 1),
                                __shfl_down_sync(0xFFFFFFFFu, v, 2),
                                __shfl_down_sync(0xFFFFFFFFu, v, 3),
                                __shfl_down_sync(0xFFFFFFFFu, v, 4),
                                __shfl_down_sync(0xFFFFFFFFu, v, 5)};
            if (have && p == 0) {
                const uint32_t j = c0 + (e & 0xFFFFu);
                bool bad;
                if constexpr (F32) {
                    float sum = 0.0f;
                    for (int q = 0; q < 6; q++) sum = __fmaf_rn(st.cf[kR0 + q], vs[q], sum);
                    const F32Bands &B = c_bands[large];
                    bool inside = all_rechecks;
                    for (int q = 0; q < 4; q++) inside |= sum >= B.r_lo[q] && sum < B.r_hi[q];
                    if (inside) {
                        rechecks++;
                        const double rg = climate_value64(S, iu, kR0, 6, xc, zc);
                        bad = (rg > 0.42 && rg < 0.91) || (rg < -0.42 && rg > -0.91) || (!a.pre_26_2 && rg <= -0.91);
                    } else {
                        // above[q]: the ridge value lies above threshold q (-0.91, -0.42, 0.42, 0.91)
                        const bool a0 = sum >= B.r_hi[0], a1 = sum >= B.r_hi[1], a2 = sum >= B.r_hi[2],
                                   a3 = sum >= B.r_hi[3];
                        bad = (a2 && !a3) || (!a1 && a0) || (!a.pre_26_2 && !a0);
                    }
                } else {
                    double sum = 0.0, sum_a = 0.0;
                    for (int q = 0; q < 6; q++) {
                        const int k = kR0 + q;
                        sum += (st.c1[k] * vs[q]) * st.c2[k];
                        if (st.act[k] == ACT_END_SUB_A) {
                            sum_a = sum;
                            sum = 0.0;
                        }
                    }
                    const double rg = (sum_a + sum) * st.amp[kR0 + 5];
                    bad = (rg > 0.42 && rg < 0.91) || (rg < -0.42 && rg > -0.91) || (!a.pre_26_2 && rg <= -0.91);
                }
                if (bad) climate_reject(S, a, iu, j, P1_RIDGE, -1);
                else keep_survivor(S, a, iu, j);
            }
        }
        __syncwarp();   // the list and the staged positions are free for the next chunk
    }
    __syncthreads();   // every warp's survivors are in the units' lists
    if constexpr (F32) {
        const uint32_t n = __reduce_add_sync(0xFFFFFFFFu, rechecks);
        if ((tid & 31) == 0 && n) atomicAdd(&a.counters[CNT_RECHECK], n);
    }

    // ---- erosion rejections counted in registers: one warp sum per tier ----
    {
        uint32_t total = 0;
        for (int t = 0; t < kTiers; t++) {
            const uint32_t v = __reduce_add_sync(0xFFFFFFFFu, tc.get(t));
            total += v;
            if ((tid & 31) == 0 && v) atomicAdd(&S.hist[P1_KINDS + t], v);
        }
        if ((tid & 31) == 0 && total) atomicAdd(&S.hist[P1_EROSION], total);
    }
    __syncthreads();

    // ---- one record per unit with survivors ----
    if (tid < kUnits && valid) {
        uint32_t n = min(S.cnt[tid], (uint32_t)kRecordCap);
        if (n) {
            uint32_t ri = atomicAdd(&a.counters[CNT_RECORDS], 1u);
            uint32_t off = atomicAdd(&a.counters[CNT_SURVIVORS], n);
            if (ri < a.cap_rec && off + n <= a.cap_surv) {
                a.rec_unit[ri] = u;
                a.rec_off[ri] = off;
                a.rec_cnt[ri] = n;
                for (uint32_t q = 0; q < n; q++) a.surv_region[off + q] = S.surv[tid * kRecordCap + q];
            } else {
                if (ri < a.cap_rec) a.rec_cnt[ri] = 0;
                atomicOr(&a.counters[CNT_OVERFLOW], 1u);
            }
        }
    }
    if (tid < P1_KINDS + kTiers && S.hist[tid]) atomicAdd(&a.hist[tid], (unsigned long long)S.hist[tid]);
}

// cudaFuncSetAttribute applies to the device current at the call, so it is made once per device.
template <class K>
static void allow_dynamic_smem(K kernel, size_t bytes, unsigned long long &done_mask) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && (done_mask >> dev) & 1ull) return;
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (dev >= 0 && dev < 64) done_mask |= 1ull << dev;
}

static unsigned long long g_smem_done64 = 0, g_smem_done32 = 0, g_smem_done32s = 0, g_smem_done_ent = 0,
                          g_smem_done_ent32 = 0;

void launch_climate(const BatchArgs &a, cudaStream_t s) {
    int grid = (int)((a.n_units + kUnits - 1) / kUnits);
    if (a.fp32_core && a.small_coords) {
        allow_dynamic_smem(climate_kernel<true, true>, sizeof(ClimateSmem<true>), g_smem_done32s);
        climate_kernel<true, true><<<grid, kThreadsA, sizeof(ClimateSmem<true>), s>>>(a);
    } else if (a.fp32_core) {
        allow_dynamic_smem(climate_kernel<true, false>, sizeof(ClimateSmem<true>), g_smem_done32);
        climate_kernel<true, false><<<grid, kThreadsA, sizeof(ClimateSmem<true>), s>>>(a);
    } else {
        allow_dynamic_smem(climate_kernel<false, false>, sizeof(ClimateSmem<false>), g_smem_done64);
        climate_kernel<false, false><<<grid, kThreadsA, sizeof(ClimateSmem<false>), s>>>(a);
    }
}

// ------------------------------------------------------------------------------------
// Noise probe: one y = 0 DoublePerlin noise of one world seed per CTA, sampled at a list of
// points both in FP64 (the reference's order, noise.c:320-342) and in the FP32 core (the
// samples of perlin_y0_f32 summed as the climate kernel sums them, times the amplitude): the
// measured error of the FP32 core.
// ------------------------------------------------------------------------------------
constexpr int kProbeThreads = 256;
constexpr int kProbeStride = 20;   // bytes per table row: one column per table (<= 18 tables)

__global__ void __launch_bounds__(kProbeThreads) noise_probe_kernel(const int64_t *seeds, int noise, const double *xz,
                                                                     uint32_t n_points, double *out32, double *out64) {
    __shared__ __align__(16) uint8_t perm[257 * kProbeStride];   // row 256 = row 0 (ColTableF)
    __shared__ double ox[2 * kMaxOct], oz[2 * kMaxOct], hy[2 * kMaxOct], fy[2 * kMaxOct];
    __shared__ float hyf[2 * kMaxOct], fyf[2 * kMaxOct];
    __shared__ int jy[2 * kMaxOct];
    __shared__ uint32_t grad[kGradWords];
    __shared__ GradF gf;
    const int t = threadIdx.x;
    const NoiseSpec &ns = c_noise[noise];
    const int np = ns.npresent;
    const uint64_t seed = (uint64_t)seeds[blockIdx.x];
    fill_grad_table(grad, t);
    fill_grad_table_f32(&gf, t);
    perm_blocks_init<kProbeStride, 257 * kProbeStride>(perm, 1, t, kProbeThreads);
    __syncthreads();
    if (t < 2 * np) {
        Xr r = octave_rng(ns, seed_fork_of(seed), t / np, t % np);
        double x0, y0, z0;
        perlin_shuffle<kProbeStride>(perm + t, r, x0, y0, z0);
        perm[256 * kProbeStride + t] = perm[t];
        const int j = (int)floor(y0);
        const double h = y0 - j;
        ox[t] = x0;
        oz[t] = z0;
        jy[t] = j;
        hy[t] = h;
        fy[t] = fade(h);
        hyf[t] = __double2float_rn(h);
        fyf[t] = __double2float_rn(fade(h));
    }
    __syncthreads();
    for (uint32_t i = t; i < n_points; i += kProbeThreads) {
        const double x = xz[2 * i], z = xz[2 * i + 1];
        double a = 0.0, b = 0.0;
        float s = 0.0f;
        for (int q = 0; q < 2 * np; q++) {
            const int p = q % np;
            const double sc = q < np ? 1.0 : kDblScale, l = ns.lac[p];
            const double px = keep_precision((x * sc) * l), pz = keep_precision((z * sc) * l);
            const ColTable<kProbeStride> T{perm + q, grad};
            const ColTableF<kProbeStride> TF{perm + q, &gf};
            const double v = perlin_y0(T, ox[q], oz[q], jy[q], hy[q], fy[q], px, pz);
            if (q < np) a += (ns.amp[p] * v) * ns.per[p];
            else b += (ns.amp[p] * v) * ns.per[p];
            s = __fmaf_rn((float)(ns.amp[p] * ns.per[p]), perlin_y0_f32(TF, ox[q], oz[q], jy[q], hyf[q], fyf[q], px, pz), s);
        }
        const size_t o = (size_t)blockIdx.x * n_points + i;
        out64[o] = (a + b) * ns.amplitude;
        out32[o] = (double)s * ns.amplitude;
    }
}

void launch_noise_probe(const int64_t *d_seeds, uint32_t n_seeds, int noise, const double *d_xz, uint32_t n_points,
                        double *d_out32, double *d_out64, cudaStream_t s) {
    noise_probe_kernel<<<n_seeds, kProbeThreads, 0, s>>>(d_seeds, noise, d_xz, n_points, d_out32, d_out64);
}

// The same probe for the entrance kernel's 3-D cave noises: DoublePerlin `noise` of seeds[b] at
// the points xyz, in FP64 in the reference's order (dbl3d, noise.c:263-289) and from the FP32
// core's samples (perlin_3d_f32) summed in FP64 as the entrance kernel sums them.
__global__ void __launch_bounds__(kProbeThreads) noise_probe3d_kernel(const int64_t *seeds, int noise,
                                                                       const double *xyz, uint32_t n_points,
                                                                       double *out32, double *out64) {
    __shared__ __align__(16) uint8_t perm[257 * kProbeStride];   // row 256 = row 0 (ColTableF)
    __shared__ double ox[2 * kMaxOct], oy[2 * kMaxOct], oz[2 * kMaxOct];
    __shared__ uint32_t grad[kGradWords];
    __shared__ GradF gf;
    const int t = threadIdx.x;
    const NoiseSpec &ns = c_noise[noise];
    const int np = ns.npresent;
    const uint64_t seed = (uint64_t)seeds[blockIdx.x];
    fill_grad_table(grad, t);
    fill_grad_table_f32(&gf, t);
    perm_blocks_init<kProbeStride, 257 * kProbeStride>(perm, 1, t, kProbeThreads);
    __syncthreads();
    if (t < 2 * np) {
        Xr r = octave_rng(ns, seed_fork_of(seed), t / np, t % np);
        double x0, y0, z0;
        perlin_shuffle<kProbeStride>(perm + t, r, x0, y0, z0);
        perm[256 * kProbeStride + t] = perm[t];
        ox[t] = x0;
        oy[t] = y0;
        oz[t] = z0;
    }
    __syncthreads();
    for (uint32_t i = t; i < n_points; i += kProbeThreads) {
        const double x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
        double a = 0.0, b = 0.0, a32 = 0.0, b32 = 0.0;
        for (int q = 0; q < 2 * np; q++) {
            const int p = q % np;
            const double l = ns.lac[p];
            const double bx = q < np ? x : x * kDblScale, by = q < np ? y : y * kDblScale,
                         bz = q < np ? z : z * kDblScale;
            const double px = keep_precision(bx * l), py = keep_precision(by * l), pz = keep_precision(bz * l);
            const ColTable<kProbeStride> T{perm + q, grad};
            const ColTableF<kProbeStride> TF{perm + q, &gf};
            const double v = perlin_3d(T, ox[q], oy[q], oz[q], px, py, pz);
            const double v32 = (double)perlin_3d_f32(TF, ox[q], oy[q], oz[q], px, py, pz);
            if (q < np) {
                a += (ns.amp[p] * v) * ns.per[p];
                a32 += (ns.amp[p] * v32) * ns.per[p];
            } else {
                b += (ns.amp[p] * v) * ns.per[p];
                b32 += (ns.amp[p] * v32) * ns.per[p];
            }
        }
        const size_t o = (size_t)blockIdx.x * n_points + i;
        out64[o] = (a + b) * ns.amplitude;
        out32[o] = (a32 + b32) * ns.amplitude;
    }
}

void launch_noise_probe3d(const int64_t *d_seeds, uint32_t n_seeds, int noise, const double *d_xyz,
                          uint32_t n_points, double *d_out32, double *d_out64, cudaStream_t s) {
    noise_probe3d_kernel<<<n_seeds, kProbeThreads, 0, s>>>(d_seeds, noise, d_xyz, n_points, d_out32, d_out64);
}

// ------------------------------------------------------------------------------------
// Climate stage for one-region units (the Deep Dive terrain stage: 65,536 upper-bit variants of
// a spot, each a different world seed over one region).  The climate kernel builds all 18 climate
// tables of a unit because a 9 x 9 unit needs nearly all of them; a one-region unit needs the two
// tier-0 tables and then one more per erosion step it reaches (about 3.2 of 18 on average), and
// each step samples only its own octave.  So the stage runs breadth first over lists in HBM:
// tier 0 for every unit, then one kernel per erosion step over the survivors of the step before
// (one table per item, the partial sum carried in the item), then temperature and ridge for the
// erosion survivors; ridge survivors become unit records for the entrance kernel as usual.
// A thread owns one byte column of its block's table area and builds one table at a time there.
// ------------------------------------------------------------------------------------
constexpr int kSpotThreads = 256;
constexpr int kSpotStride = kSpotThreads + 16;   // bytes per table row: one column per thread

struct SpotSmem {
    uint8_t perm[256 * kSpotStride];
    uint32_t grad[kGradWords];
};

// Builds, in this thread's column, the table of climate step k of `seed` and samples it at the
// unit's climate point (xc, zc) (climate_sample for a single table).
__device__ double spot_sample(SpotSmem &S, int large, int k, uint64_t seed, double xc, double zc) {
    const ClimateStep &cs = c_steps[large][k];
    const int slot = cs.slot;
    uint8_t *col = S.perm + threadIdx.x;
    for (int i = 0; i < 256; i++) col[i * kSpotStride] = (uint8_t)i;
    Xr r = octave_rng(c_noise[c_slot_a[large][slot][0]], seed_fork_of(seed), c_slot_a[large][slot][1],
                      c_slot_a[large][slot][2]);
    double ox, oy, oz;
    perlin_shuffle<kSpotStride>(col, r, ox, oy, oz);
    const int jy = (int)floor(oy);
    const double hy = oy - jy;
    const ColTable<kSpotStride> T{col, S.grad};
    return perlin_y0(T, ox, oz, jy, hy, fade(hy), keep_precision((xc * cs.sc) * cs.lac),
                     keep_precision((zc * cs.sc) * cs.lac));
}

// The unit's world seed and climate point (its only region's hut chunk middle).
__device__ __forceinline__ uint64_t spot_point(const BatchArgs &a, uint32_t u, double &xc, double &zc) {
    const UnitPos up = unit_pos(a, u);
    const uint64_t seed = seed_value(a, up.g);
    int cx, cz;
    hut_chunk(seed, up.rx0, up.rz0, a.salt, cx, cz);
    xc = (cx * 16 + 8) * 0.25;   // exact: an integer over 4
    zc = (cz * 16 + 8) * 0.25;
    return seed;
}

__device__ __forceinline__ void spot_append(SpotItem *out, uint32_t *out_n, uint32_t cap, bool keep, const SpotItem &it,
                                            uint32_t *overflow) {
    cg::coalesced_group grp = cg::coalesced_threads();
    const unsigned m = grp.ballot(keep);
    uint32_t base = 0;
    if (grp.thread_rank() == 0 && m) base = atomicAdd(out_n, (uint32_t)__popc(m));
    base = grp.shfl(base, 0);
    if (keep) {
        const uint32_t at = base + (uint32_t)__popc(m & ((1u << grp.thread_rank()) - 1u));
        if (at < cap) out[at] = it;
        else atomicOr(overflow, 1u);
    }
}

__device__ __forceinline__ void spot_count(unsigned long long *hist, int idx, uint32_t n) {
    const uint32_t tot = __reduce_add_sync(0xFFFFFFFFu, n);
    if ((threadIdx.x & 31) == 0 && tot) atomicAdd(&hist[idx], (unsigned long long)tot);
}

// Tier 0: lanes 2i and 2i+1 build octaves 0A and 0B of one unit; the even lane sums them in the
// reference's order and applies the tier-0 threshold.
__global__ void __launch_bounds__(kSpotThreads) spot_tier0_kernel(BatchArgs a, SpotItem *out, uint32_t *out_n,
                                                                  uint32_t cap) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    SpotSmem &S = *reinterpret_cast<SpotSmem *>(smem_raw);
    fill_grad_table(S.grad, threadIdx.x);
    __syncthreads();
    const int large = a.large_biomes ? 1 : 0;
    const ClimateStep &s0 = c_steps[large][0], &s1 = c_steps[large][1];
    uint32_t rejected = 0;
    const uint64_t tasks = 2ull * a.n_units;
    for (uint64_t base = (uint64_t)blockIdx.x * kSpotThreads; base < tasks; base += (uint64_t)gridDim.x * kSpotThreads) {
        const uint64_t task = base + threadIdx.x;
        const bool valid = task < tasks;
        const uint32_t u = (uint32_t)(task >> 1);
        double v = 0.0;
        if (valid) {
            double xc, zc;
            const uint64_t seed = spot_point(a, u, xc, zc);
            v = spot_sample(S, large, (int)(task & 1), seed, xc, zc);
        }
        const double v1 = __shfl_down_sync(0xFFFFFFFFu, v, 1);
        bool keep = false;
        SpotItem it{u, 0u, 0.0, 0.0};
        if (valid && !(task & 1)) {
            double sum = 0.0;
            sum += (s0.c1 * v) * s0.c2;
            sum += (s1.c1 * v1) * s1.c2;
            if (sum * s1.amp < s1.thr) rejected++;
            else {
                keep = true;
                it.sum = sum;
            }
        }
        spot_append(out, out_n, cap, keep, it, &a.counters[CNT_OVERFLOW]);
    }
    spot_count(a.hist, P1_KINDS + s1.tier, rejected);
    spot_count(a.hist, P1_EROSION, rejected);
}

// Climate steps [k0, k1) for every listed item, one table at a time per item, in the state
// machine's order (erosion tier checks, the A/B split, temperature, ridge).  Items that pass the
// last erosion tier or temperature go to `out` for the next stage; ridge survivors become unit
// records (CNT_RECORDS / CNT_SURVIVORS, one region each) for the entrance kernel.
__global__ void __launch_bounds__(kSpotThreads) spot_steps_kernel(BatchArgs a, int k0, int k1, const SpotItem *in,
                                                                  const uint32_t *in_n, SpotItem *out, uint32_t *out_n,
                                                                  uint32_t cap) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    SpotSmem &S = *reinterpret_cast<SpotSmem *>(smem_raw);
    fill_grad_table(S.grad, threadIdx.x);
    __syncthreads();
    const int large = a.large_biomes ? 1 : 0;
    const uint32_t n = min(*in_n, cap);
    uint32_t rej_tier = 0, rej_temp = 0, rej_ridge = 0;
    for (uint32_t base = blockIdx.x * kSpotThreads; base < n; base += gridDim.x * kSpotThreads) {
        const uint32_t e = base + threadIdx.x;
        bool keep = false;
        SpotItem it{0u, 0u, 0.0, 0.0};
        if (e < n) {
            it = in[e];
            double xc, zc;
            const uint64_t seed = spot_point(a, it.unit, xc, zc);
            double sum = it.sum, sum_a = it.sum_a;
            bool alive = true;
            for (int k = k0; k < k1 && alive; k++) {
                const ClimateStep &cs = c_steps[large][k];
                sum += (cs.c1 * spot_sample(S, large, k, seed, xc, zc)) * cs.c2;
                switch (cs.act) {
                    case ACT_TIER:
                    case ACT_TIER_LAST:
                        if (sum * cs.amp < cs.thr) {
                            alive = false;
                            rej_tier++;
                        } else if (cs.act == ACT_TIER_LAST) {
                            sum = 0.0;
                        }
                        break;
                    case ACT_END_SUB_A:
                        sum_a = sum;
                        sum = 0.0;
                        break;
                    case ACT_TEMPERATURE: {
                        const double t = (sum_a + sum) * cs.amp;
                        const bool bad = a.mc_1_18_2 ? (t < -0.45) : (t > 0.2 || t < -0.45);
                        if (bad) {
                            alive = false;
                            rej_temp++;
                        }
                        sum = 0.0;
                        sum_a = 0.0;
                        break;
                    }
                    case ACT_RIDGE: {
                        const double rg = (sum_a + sum) * cs.amp;
                        if ((rg > 0.42 && rg < 0.91) || (rg < -0.42 && rg > -0.91) || (!a.pre_26_2 && rg <= -0.91)) {
                            alive = false;
                            rej_ridge++;
                        } else {
                            emit_single(a, it.unit, 0u);   // climate survivor: a record of one region
                        }
                        alive = false;   // ridge is the last climate step
                        break;
                    }
                    default:
                        break;
                }
            }
            if (alive) {
                keep = true;
                it.sum = sum;
                it.sum_a = sum_a;
            }
        }
        spot_append(out, out_n, cap, keep, it, &a.counters[CNT_OVERFLOW]);
    }
    // a step kernel over erosion steps checks one tier (the caller runs one step per launch there)
    if (k1 <= 8) {
        spot_count(a.hist, P1_KINDS + (k1 - 2), rej_tier);
        spot_count(a.hist, P1_EROSION, rej_tier);
    }
    spot_count(a.hist, P1_TEMPERATURE, rej_temp);
    spot_count(a.hist, P1_RIDGE, rej_ridge);
}

size_t spot_smem_bytes() { return sizeof(SpotSmem); }

void launch_spot_climate(const BatchArgs &a, SpotItem *list0, SpotItem *list1, uint32_t *counts, uint32_t cap,
                         int sm_count, cudaStream_t s) {
    static unsigned long long done0 = 0, done1 = 0;
    allow_dynamic_smem(spot_tier0_kernel, sizeof(SpotSmem), done0);
    allow_dynamic_smem(spot_steps_kernel, sizeof(SpotSmem), done1);
    const int grid = sm_count * 3;   // three 70 KB blocks per SM
    SpotItem *lists[2] = {list0, list1};
    cudaMemsetAsync(counts, 0, sizeof(uint32_t) * 2, s);
    spot_tier0_kernel<<<grid, kSpotThreads, sizeof(SpotSmem), s>>>(a, lists[0], &counts[0], cap);
    int cur = 0;
    // erosion steps 2..7, one launch each; then temperature (8..11) and ridge (12..17)
    const int bounds[][2] = {{2, 3}, {3, 4}, {4, 5}, {5, 6}, {6, 7}, {7, 8}, {8, 12}, {12, 18}};
    for (const auto &b : bounds) {
        cudaMemsetAsync(&counts[cur ^ 1], 0, sizeof(uint32_t), s);
        spot_steps_kernel<<<grid, kSpotThreads, sizeof(SpotSmem), s>>>(a, b[0], b[1], lists[cur], &counts[cur],
                                                                       lists[cur ^ 1], &counts[cur ^ 1], cap);
        cur ^= 1;
    }
}

// ------------------------------------------------------------------------------------
// entrance kernel: Entrance(50) / Entrance(60) for every climate survivor
//
// Thread t builds table (slot t / kUnits, record t % kUnits).  Afterwards it samples only that
// table, for up to kEntChunk survivors of its record at y = 50 and y = 60, into shared memory;
// the tunnel scale e (from the rarity slots) is formed between the two sampling rounds, because
// spaghetti_3d_1/2 are sampled at (x/e, y/e, z/e).  One pass then sums the samples in the
// reference's order (DoublePerlin: sub 0 octaves, then sub 1, times the amplitude;
// caves.c:83-113).  Entrance(60) is computed for every survivor but only decides those with
// Entrance(50) < 0, as in lysh.
// ------------------------------------------------------------------------------------
constexpr int kEntFlat = 64;                   // survivors evaluated per round of a tile
constexpr int kEntList = kUnits * kRecordCap;  // survivors a tile can hold

// The entrance kernel's DoublePerlin noises, in the order of EntranceSmem::err.
constexpr int kEntNoises = 7;
enum : int { EN_ENTRANCE = 0, EN_RARITY, EN_THICKNESS, EN_SP1, EN_SP2, EN_RMOD, EN_ROUGH };
__device__ __forceinline__ int ent_noise(int i) {
    return i == EN_ENTRANCE ? N_CAVE_ENTRANCE
           : i == EN_RARITY ? N_SPAGHETTI_RARITY
           : i == EN_THICKNESS ? N_SPAGHETTI_THICKNESS
           : i == EN_SP1 ? N_SPAGHETTI_1
           : i == EN_SP2 ? N_SPAGHETTI_2
           : i == EN_RMOD ? N_ROUGHNESS_MODULATOR : N_ROUGHNESS;
}

// FP32 core: bound on |value - reference value| of a DoublePerlin whose octave samples each carry
// at most kPerlin3dF32ErrUlps * 2^-24 (perlin_3d_f32) and are summed in FP64 in the reference's
// order: value = (sum_a + sum_b) * amplitude with sum = sum_p (amp_p * v_p) * per_p, so the error is
// at most |amplitude| * 2 * sum_p |amp_p * per_p| times the sample bound, plus 1e-12 for the FP64
// roundings of both sides.
__device__ double dp_err_f32(int noise) {
    const NoiseSpec &ns = c_noise[noise];
    double w = 0.0;
    for (int p = 0; p < ns.npresent; p++) w += fabs(ns.amp[p] * ns.per[p]);
    return 2.0 * fabs(ns.amplitude) * w * (kPerlin3dF32ErrUlps / 16777216.0) + 1e-12;
}

struct EntranceSmem {
    uint8_t perm[kSlotsB * kPitch];
    double ox[kSlotsB * kUnits], oy[kSlotsB * kUnits], oz[kSlotsB * kUnits];
    double val[kSlotsB][2][kEntFlat];     // [slot][y=50,60][survivor]
    double tun[2][kEntFlat];              // tunnel scale e per survivor and height
    int hx[kEntFlat], hz[kEntFlat];       // sampling block of each survivor
    uint32_t emap[kEntList];              // tile survivor list: record << 16 | index in its record
    uint64_t rseed[kUnits], rg[kUnits], rbase[kUnits];
    uint32_t runit[kUnits], roff[kUnits];
    int rrx0[kUnits], rrz0[kUnits], rrw[kUnits];   // rect of each record's unit
    unsigned int hist[P1_KINDS];
    unsigned int n_list;
    uint32_t grad[kGradWords];
    GradF gf;                             // FP32 core: the gradient vectors as floats
    double err[kEntNoises];               // FP32 core: bound on each DoublePerlin value (ent_noise order)
    double slot_lac[kSlotsB];             // per slot: the octave's lacunarity, noise id, sub
    int slot_noise[kSlotsB], slot_sub[kSlotsB];
};

size_t entrance_smem_bytes() { return sizeof(EntranceSmem); }

// Base (unscaled) sampling point of cave noise `noise` at block (x, y, z); e = tunnel scale.
__device__ __forceinline__ void cave_point(int noise, int x, int y, int z, double e, double &px, double &py,
                                           double &pz) {
    switch (noise) {
        case N_CAVE_ENTRANCE:
            px = (double)x * 0.75; py = (double)y * 0.5; pz = (double)z * 0.75;
            break;
        case N_SPAGHETTI_RARITY:
            px = (double)(int)((uint32_t)x * 2u); py = (double)y; pz = (double)(int)((uint32_t)z * 2u);
            break;
        case N_SPAGHETTI_1:
        case N_SPAGHETTI_2:
            px = (double)x / e; py = (double)y / e; pz = (double)z / e;
            break;
        default:
            px = (double)x; py = (double)y; pz = (double)z;
            break;
    }
}

// One octave of one sub-sampler of a DoublePerlin at a base point (noise.c:263-289 inner step);
// l is that octave's lacunarity.
template <class Src>
__device__ __forceinline__ double slot_sample(const Src &src, int slot, int sub, double l, double px, double py,
                                              double pz) {
    if (sub) {
        px = px * kDblScale;
        py = py * kDblScale;
        pz = pz * kDblScale;
    }
    return src.p3(slot, keep_precision(px * l), keep_precision(py * l), keep_precision(pz * l));
}

// DoublePerlin value from its per-octave samples stored at val[base .. base + 2 np).
__device__ __forceinline__ double combine(const EntranceSmem &S, int noise, int base, int h, int e) {
    const NoiseSpec &ns = c_noise[noise];
    const int np = ns.npresent;
    double a = 0.0, b = 0.0;
    for (int p = 0; p < np; p++) a += (ns.amp[p] * S.val[base + p][h][e]) * ns.per[p];
    for (int p = 0; p < np; p++) b += (ns.amp[p] * S.val[base + np + p][h][e]) * ns.per[p];
    return (a + b) * ns.amplitude;
}

// Slots that do not depend on the tunnel scale (everything but spaghetti_3d_1 / _2).
__device__ __forceinline__ int free_slot(int i) { return i < kBaseSp1 ? i : i + 4; }

// Thread t builds table (slot t / kUnits, record t % kUnits).  The tile's survivors are then
// listed, and every Perlin sample they need — per survivor, slot and height (y = 50, 60) — is an
// independent task spread over all threads: round 1 the 14 slots that do not depend on the
// tunnel scale e, then e from the rarity samples, round 2 spaghetti_3d_1 / _2 at (x/e, y/e, z/e).
// One pass sums the samples in the reference's order (DoublePerlin: sub 0 octaves, then sub 1,
// times the amplitude; caves.c:83-113).  Entrance(60) is computed for every survivor but only
// decides those with Entrance(50) < 0, as in lysh.
template <bool F32>
__global__ void __launch_bounds__(kThreadsB, 2) entrance_kernel(BatchArgs a) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    EntranceSmem &S = *reinterpret_cast<EntranceSmem *>(smem_raw);
    batch_range(a);
    const int tid = threadIdx.x;
    const int my_slot = tid / kUnits, rr = tid % kUnits;
    const bool all_rechecks = F32 && a.fp32_core == 2;   // every FP32 decision re-taken in FP64 (a check mode)
    uint32_t rechecks = 0;
    if (tid < P1_KINDS) S.hist[tid] = 0;
    fill_grad_table(S.grad, tid);
    if (F32) {
        fill_grad_table_f32(&S.gf, tid);
        if (tid < kEntNoises) S.err[tid] = dp_err_f32(ent_noise(tid));
    }
    if (tid < kSlotsB) {
        const int noise = c_slot_c[0][tid][0];
        S.slot_noise[tid] = noise;
        S.slot_sub[tid] = c_slot_c[0][tid][1];
        S.slot_lac[tid] = c_noise[noise].lac[c_slot_c[0][tid][2]];
    }
    // A full list means the host discards this batch and re-runs it smaller.
    if (a.counters[CNT_OVERFLOW]) return;
    const uint32_t n_rec = min(a.counters[CNT_RECORDS], a.cap_rec);
    const uint32_t n_tiles = (n_rec + kUnits - 1) / kUnits;
    const int my_noise = c_slot_c[0][my_slot][0], my_sub = c_slot_c[0][my_slot][1], my_p = c_slot_c[0][my_slot][2];
    for (uint32_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const uint32_t ri = tile * kUnits + (uint32_t)rr;
        perm_blocks_init<kUnits, kPitch>(S.perm, kSlotsB, tid, kThreadsB);
        __syncthreads();
        uint32_t cnt = 0;
        if (ri < n_rec) {
            const uint32_t u = a.rec_unit[ri], off = a.rec_off[ri];
            cnt = a.rec_cnt[ri];
            if (u >= a.n_units || off >= a.cap_surv || cnt > a.cap_surv - off || cnt > kRecordCap) cnt = 0;
            const UnitPos up = unit_pos(a, u);
            const uint64_t g = up.g;
            const uint64_t seed = seed_value(a, g);
            if (my_slot == 0) {
                S.rseed[rr] = seed;
                S.rg[rr] = g;
                S.rbase[rr] = up.rbase;
                S.runit[rr] = u;
                S.roff[rr] = off;
                S.rrx0[rr] = up.rx0;
                S.rrz0[rr] = up.rz0;
                S.rrw[rr] = up.rw;
            }
            if (cnt) {
                Xr r = octave_rng(c_noise[my_noise], seed_fork_of(seed), my_sub, my_p);
                double ox, oy, oz;
                uint8_t *col = S.perm + my_slot * kPitch + rr;
                perlin_shuffle<kUnits>(col, r, ox, oy, oz);
                col[256 * kUnits] = col[0];   // row 256 = row 0, in the slot's padding (ColTableF)
                const int o = my_slot * kUnits + rr;
                S.ox[o] = ox;
                S.oy[o] = oy;
                S.oz[o] = oz;
            }
        }
        if (tid == 0) S.n_list = 0;
        __syncthreads();
        // list this tile's survivors
        if (my_slot == 0 && cnt) {
            const uint32_t at = atomicAdd(&S.n_list, cnt);
            for (uint32_t j = 0; j < cnt; j++) S.emap[at + j] = ((uint32_t)rr << 16) | j;
        }
        __syncthreads();
        const uint32_t n_list = S.n_list;
        for (uint32_t e0 = 0; e0 < n_list; e0 += kEntFlat) {
            const uint32_t m = min((uint32_t)kEntFlat, n_list - e0);
            for (uint32_t e = tid; e < m; e += kThreadsB) {
                const uint32_t em = S.emap[e0 + e];
                const int r2 = (int)(em >> 16);
                const uint32_t jr = a.surv_region[S.roff[r2] + (em & 0xFFFFu)];
                const uint64_t reg = S.rbase[r2] + jr;
                const int rz = S.rrz0[r2] + (int)(reg / (uint64_t)S.rrw[r2]);
                const int rx = S.rrx0[r2] + (int)(reg % (uint64_t)S.rrw[r2]);
                int cx, cz;
                hut_chunk(S.rseed[r2], rx, rz, a.salt, cx, cz);
                S.hx[e] = cx * 16 + 3;
                S.hz[e] = cz * 16 + 3;
            }
            __syncthreads();
            // round 1: 14 slots x 2 heights per survivor
            for (uint32_t t = tid; t < m * 28; t += kThreadsB) {
                const uint32_t e = t / 28, rem = t % 28;
                const int slot = free_slot((int)(rem >> 1)), h = (int)(rem & 1);
                const int r2 = (int)(S.emap[e0 + e] >> 16);
                double px, py, pz;
                cave_point(S.slot_noise[slot], S.hx[e], h ? 60 : 50, S.hz[e], 1.0, px, py, pz);
                if constexpr (F32) {
                    const SrcColsF src{S.perm, S.ox, S.oy, S.oz, &S.gf, r2};
                    S.val[slot][h][e] = slot_sample(src, slot, S.slot_sub[slot], S.slot_lac[slot], px, py, pz);
                } else {
                    const SrcCols src{S.perm, S.ox, S.oy, S.oz, S.grad, r2};
                    S.val[slot][h][e] = slot_sample(src, slot, S.slot_sub[slot], S.slot_lac[slot], px, py, pz);
                }
            }
            __syncthreads();
            for (uint32_t t = tid; t < m * 2; t += kThreadsB) {
                const uint32_t e = t >> 1;
                const int h = (int)(t & 1);
                double rar = combine(S, N_SPAGHETTI_RARITY, kBaseRarity, h, (int)e);
                if (F32) {   // the interval of the tunnel scale must be the reference's
                    const double er = S.err[EN_RARITY];
                    if (all_rechecks || fabs(rar + 0.5) <= er || fabs(rar) <= er || fabs(rar - 0.5) <= er) {
                        rechecks++;
                        const SrcCols src{S.perm, S.ox, S.oy, S.oz, S.grad, (int)(S.emap[e0 + e] >> 16)};
                        rar = rarity64(src, S.hx[e], h ? 60 : 50, S.hz[e]);
                    }
                }
                S.tun[h][e] = tunnel_scale(rar);
            }
            __syncthreads();
            // round 2: spaghetti_3d_1 / _2 (4 slots) x 2 heights per survivor
            for (uint32_t t = tid; t < m * 8; t += kThreadsB) {
                const uint32_t e = t / 8, rem = t % 8;
                const int slot = kBaseSp1 + (int)(rem >> 1), h = (int)(rem & 1);
                const int r2 = (int)(S.emap[e0 + e] >> 16);
                double px, py, pz;
                cave_point(S.slot_noise[slot], S.hx[e], h ? 60 : 50, S.hz[e], S.tun[h][e], px, py, pz);
                if constexpr (F32) {
                    const SrcColsF src{S.perm, S.ox, S.oy, S.oz, &S.gf, r2};
                    S.val[slot][h][e] = slot_sample(src, slot, S.slot_sub[slot], S.slot_lac[slot], px, py, pz);
                } else {
                    const SrcCols src{S.perm, S.ox, S.oy, S.oz, S.grad, r2};
                    S.val[slot][h][e] = slot_sample(src, slot, S.slot_sub[slot], S.slot_lac[slot], px, py, pz);
                }
            }
            __syncthreads();
            // the six DoublePerlin values per survivor and height, one per thread, each summed in
            // the reference's order and stored over its own first slot's sample (a task reads and
            // writes only its own noise's slots)
            for (uint32_t t = tid; t < m * 12; t += kThreadsB) {
                const uint32_t e = t / 12, rem = t % 12;
                const int h = (int)(rem & 1), k = (int)(rem >> 1);
                const int noise = k == 0 ? N_CAVE_ENTRANCE
                                  : k == 1 ? N_SPAGHETTI_THICKNESS
                                  : k == 2 ? N_SPAGHETTI_1
                                  : k == 3 ? N_SPAGHETTI_2
                                  : k == 4 ? N_ROUGHNESS_MODULATOR : N_ROUGHNESS;
                const int base = k == 0 ? kBaseEntrance
                                 : k == 1 ? kBaseThickness
                                 : k == 2 ? kBaseSp1
                                 : k == 3 ? kBaseSp2
                                 : k == 4 ? kBaseRmod : kBaseRough;
                const double v = combine(S, noise, base, h, (int)e);
                S.val[base][h][e] = v;
            }
            __syncthreads();
            // decide in the reference's order
            for (uint32_t e = tid; e < m; e += kThreadsB) {
                double ent_v[2];
                for (int h = 0; h < 2; h++) {
                    const int y = h ? 60 : 50;
                    const double te = S.tun[h][e];
                    double ent = S.val[kBaseEntrance][h][e];
                    double t = (10.0 + (double)y) / 40.0;
                    double cl = t < 0.0 ? 0.3 : (t > 1.0 ? 0.0 : lerp(t, 0.3, 0.0));
                    double cc = ent + 0.37 + cl;
                    double tv = S.val[kBaseThickness][h][e];
                    double hh = lerp((tv - -1.0) / (1.0 - -1.0), 0.065, 0.088);
                    double l = S.val[kBaseSp1][h][e];
                    double mm = fabs(te * l) - hh;
                    double n = S.val[kBaseSp2][h][e];
                    double o = fabs(te * n) - hh;
                    double pp = clampd(jmax(mm, o), -1.0, 1.0);
                    double mod = S.val[kBaseRmod][h][e];
                    double rgh = S.val[kBaseRough][h][e];
                    double q = (-0.05 + (-0.05 * mod)) * (-0.4 + fabs(rgh));
                    ent_v[h] = jmin(cc, pp + q);
                    if (F32) {
                        // the inputs carry at most S.err; the formula's slopes: cc 1 in ent; hh
                        // 0.023 / 2 in tv; |te l| te in l (te exact); q 0.05 |-0.4 + |rgh|| in mod
                        // and 0.05 |1 + mod| in rgh; max, min, clamp and |.| 1
                        const double e_hh = 0.0115 * S.err[EN_THICKNESS];
                        const double e_pp = fmax(te * S.err[EN_SP1], te * S.err[EN_SP2]) + e_hh;
                        const double e_q = 0.05 * S.err[EN_RMOD] * (fabs(-0.4 + fabs(rgh)) + S.err[EN_ROUGH]) +
                                           0.05 * (1.0 + fabs(mod) + S.err[EN_RMOD]) * S.err[EN_ROUGH];
                        const double bound = fmax(S.err[EN_ENTRANCE], e_pp + e_q) * 1.000001 + 1e-12;
                        if (all_rechecks || fabs(ent_v[h]) <= bound) {   // inside the band: the reference's value
                            rechecks++;
                            const SrcCols src{S.perm, S.ox, S.oy, S.oz, S.grad, (int)(S.emap[e0 + e] >> 16)};
                            ent_v[h] = entrance64(src, S.hx[e], y, S.hz[e]);
                        }
                    }
                }
                const uint32_t em = S.emap[e0 + e];
                const int r2 = (int)(em >> 16);
                const uint32_t jr = a.surv_region[S.roff[r2] + (em & 0xFFFFu)];
                int code = -1;
                if (ent_v[0] >= 0) code = P1_ENTRANCE_50;
                else if (ent_v[1] >= 0) code = P1_ENTRANCE_60;
                if (code >= 0) {
                    atomicAdd(&S.hist[code], 1u);
                    note_code(a, S.rg[r2], S.rbase[r2] + jr, code, -1);
                } else {
                    uint32_t di = atomicAdd(&a.counters[CNT_DEEP], 1u);
                    if (di < a.cap_deep) {
                        a.deep[2 * di] = S.runit[r2];
                        a.deep[2 * di + 1] = jr;
                    } else {
                        atomicOr(&a.counters[CNT_OVERFLOW], 2u);
                    }
                }
            }
            __syncthreads();
        }
    }
    if (F32) {
        const uint32_t n = __reduce_add_sync(0xFFFFFFFFu, rechecks);
        if ((tid & 31) == 0 && n) atomicAdd(&a.counters[CNT_RECHECK], n);
    }
    __syncthreads();
    if (tid < P1_KINDS && S.hist[tid]) atomicAdd(&a.hist[tid], (unsigned long long)S.hist[tid]);
}

// grid <= 0: one CTA per tile the batch can produce (records <= units, and <= the list's capacity;
// a CTA past the batch's tiles returns at once).  Separate CTAs start their table builds at
// different times, so the two on an SM are seldom in the same phase: one's build fills the issue
// slots the other's latency-bound sampling leaves free, which persistent CTAs started together
// did not do.  The kernel still loops over tiles with a grid stride, so any grid is correct.
void launch_entrance(const BatchArgs &a, int grid, cudaStream_t s) {
    if (grid <= 0) {
        const uint64_t recs = a.n_units < a.cap_rec ? a.n_units : a.cap_rec;
        grid = (int)((recs + kUnits - 1) / kUnits);
        if (grid < 1) grid = 1;
    }
    if (a.fp32_core >= 2) {   // the cave samples in the FP32 core (WG_NOISE_FP32_CAVES, the check mode)
        allow_dynamic_smem(entrance_kernel<true>, sizeof(EntranceSmem), g_smem_done_ent32);
        entrance_kernel<true><<<grid, kThreadsB, sizeof(EntranceSmem), s>>>(a);
    } else {
        allow_dynamic_smem(entrance_kernel<false>, sizeof(EntranceSmem), g_smem_done_ent);
        entrance_kernel<false><<<grid, kThreadsB, sizeof(EntranceSmem), s>>>(a);
    }
}

// ------------------------------------------------------------------------------------
// ladder kernel: the rest of lysh_phase1_check_ex for candidates past Entrance(60)
//
// One CTA per candidate.  After its 54 tables are built, every Perlin sample the remaining
// ladder can read is computed in parallel (round 1: everything but spaghetti_3d_1/2; then the
// tunnel scale per height; round 2: spaghetti_3d_1/2), and one thread walks lysh's ladder in order
// over the stored samples.  Samples the ladder ends up not reading change nothing.
// ------------------------------------------------------------------------------------
constexpr int kLadderHeights = 12;   // maxHeight, the y <= 0 ladder (<= 6), y = 10..40
constexpr int kFloodHeights = 16;

struct LadderSmem {
    uint8_t perm[256 * kLadderStride];       // slot s, row k at k * kLadderStride + s
    double org[kSlotsC * 3];
    double val[kSlotsC][kLadderHeights];     // [slot][height index]
    double fval[2][kFloodHeights];           // floodedness samples
    double tun[kLadderHeights];
    int ys[kLadderHeights];
    uint32_t grad[kGradWords];
};

// Octave-sum of noise `noise` (slots base .. base + 2 np) over stored samples v[slot * stride].
__device__ __forceinline__ double combine_vals(int noise, const double *v, int stride) {
    const NoiseSpec &ns = c_noise[noise];
    const int np = ns.npresent;
    double a = 0.0, b = 0.0;
    for (int p = 0; p < np; p++) a += (ns.amp[p] * v[p * stride]) * ns.per[p];
    for (int p = 0; p < np; p++) b += (ns.amp[p] * v[(np + p) * stride]) * ns.per[p];
    return (a + b) * ns.amplitude;
}

__global__ void __launch_bounds__(kThreadsC, 10) ladder_kernel(BatchArgs a) {
    __shared__ __align__(16) LadderSmem S;
    batch_range(a);
    const int t = threadIdx.x;
    const int large = a.large_biomes ? 1 : 0;
    const int cont_noise = large ? N_CONTINENTALNESS_LARGE : N_CONTINENTALNESS;
    if (a.counters[CNT_OVERFLOW]) return;
    const uint32_t n_deep = min(a.counters[CNT_DEEP], a.cap_deep);
    fill_grad_table(S.grad, t);
    const SrcFlat src{S.perm, S.org, S.grad};

    for (uint32_t q = blockIdx.x; q < n_deep; q += gridDim.x) {
        const uint32_t u = a.deep[2 * q], jr = a.deep[2 * q + 1];
        const UnitPos up = unit_pos(a, u);
        const uint64_t g = up.g;
        const uint64_t r = up.rbase + jr;
        const uint64_t seed = seed_value(a, g);
        int rx, rz, cx, cz;
        unit_region_xz(up, r, rx, rz);
        hut_chunk(seed, rx, rz, a.salt, cx, cz);
        // heights: [0] maxHeight, then y = 0, -10, ... >= ladderFloor with maxHeight < y, then
        // 10..40 (S.ys is rewritten only after the previous candidate's closing barrier)
        const int mh = up.max_height;
        int floor_y = (-40 < mh) ? -40 : mh;
        if (floor_y < -50) floor_y = -50;
        int nh = 0;
        if (t == 0) S.ys[nh] = mh;
        nh++;
        for (int y = 0; y >= floor_y; y -= 10)
            if (mh < y) {
                if (t == 0) S.ys[nh] = y;
                nh++;
            }
        const int first_pos = nh;
        for (int y = 10; y <= 40; y += 10) {
            if (t == 0) S.ys[nh] = y;
            nh++;
        }
        const long long nf_ll = mh > 60 ? 0 : ((long long)60 - mh) / 10 + 1;
        const int nf = nf_ll > kFloodHeights ? 0 : (int)nf_ll;   // more: sampled one by one at the end
        const int hut_x = cx * 16, hut_z = cz * 16;
        const int hx = hut_x + 3, hz = hut_z + 3;
        perm_blocks_init<kLadderStride, 256 * kLadderStride>(S.perm, 1, t, kThreadsC);
        __syncthreads();
        if (t < kSlotsC) {
            const int noise = c_slot_c[large][t][0], sub = c_slot_c[large][t][1], p = c_slot_c[large][t][2];
            Xr rng = octave_rng(c_noise[noise], seed_fork_of(seed), sub, p);
            double ox, oy, oz;
            perlin_shuffle<kLadderStride>(S.perm + t, rng, ox, oy, oz);
            S.org[3 * t] = ox;
            S.org[3 * t + 1] = oy;
            S.org[3 * t + 2] = oz;
        }
        __syncthreads();
        // round 1: per height, rarity .. rough minus spaghetti_3d_1/2 (8 slots), cave_layer and
        // cave_cheese (16 slots); cave_entrance (6 slots) at y = 10..40; continentalness; flood
        const int n_a = nh * 24, n_b = (nh - first_pos) * 6, n_c = 18, n_d = nf * 2;
        for (int k = t; k < n_a + n_b + n_c + n_d; k += kThreadsC) {
            int slot, hi = 0;
            double px, py, pz;
            if (k < n_a) {
                hi = k / 24;
                const int s24 = k % 24;
                slot = s24 < 4 ? kBaseRarity + s24 : (s24 < 8 ? kBaseRmod + (s24 - 4) : kBaseLayer + (s24 - 8));
                const int y = S.ys[hi];
                if (slot < kBaseRmod || slot >= kBaseLayer) {
                    if (slot < kBaseThickness) {   // rarity at (x*2, y, z*2)
                        px = (double)(int)((uint32_t)hx * 2u); py = (double)y; pz = (double)(int)((uint32_t)hz * 2u);
                    } else if (slot < kBaseSp1) {  // thickness
                        px = (double)hx; py = (double)y; pz = (double)hz;
                    } else if (slot < kBaseCheese) {   // cave_layer at (x, y*8, z)
                        px = (double)hx; py = (double)(int)((uint32_t)y * 8u); pz = (double)hz;
                    } else {                           // cave_cheese at (x, y*2/3, z)
                        px = (double)hx; py = (double)y * 0.6666666666666666; pz = (double)hz;
                    }
                } else {                               // roughness modulator / roughness
                    px = (double)hx; py = (double)y; pz = (double)hz;
                }
            } else if (k < n_a + n_b) {
                const int kk = k - n_a;
                hi = first_pos + kk / 6;
                slot = kBaseEntrance + kk % 6;
                const int y = S.ys[hi];
                px = (double)hx * 0.75; py = (double)y * 0.5; pz = (double)hz * 0.75;
            } else if (k < n_a + n_b + n_c) {
                slot = kBaseCont + (k - n_a - n_b);
                px = (hut_x + 8) / 4.0; py = 0.0; pz = (hut_z + 8) / 4.0;
            } else {
                const int kk = k - n_a - n_b - n_c;
                hi = kk >> 1;
                slot = kBaseFlood + (kk & 1);
                px = (double)(hut_x + 3); py = (double)(mh + 10 * hi) * 0.67; pz = (double)(hut_z + 3);
            }
            const int noise = c_slot_c[large][slot][0], sub = c_slot_c[large][slot][1], p = c_slot_c[large][slot][2];
            const double v = slot_sample(src, slot, sub, c_noise[noise].lac[p], px, py, pz);
            if (slot >= kBaseFlood) S.fval[slot - kBaseFlood][hi] = v;
            else S.val[slot][hi] = v;
        }
        __syncthreads();
        if (t < nh) S.tun[t] = tunnel_scale(combine_vals(N_SPAGHETTI_RARITY, &S.val[kBaseRarity][t], kLadderHeights));
        __syncthreads();
        // round 2: spaghetti_3d_1 / _2 at (x/e, y/e, z/e)
        for (int k = t; k < nh * 4; k += kThreadsC) {
            const int hi = k >> 2, slot = kBaseSp1 + (k & 3);
            const double e = S.tun[hi], y = (double)S.ys[hi];
            const int noise = c_slot_c[large][slot][0], sub = c_slot_c[large][slot][1], p = c_slot_c[large][slot][2];
            S.val[slot][hi] = slot_sample(src, slot, sub, c_noise[noise].lac[p], (double)hx / e, y / e, (double)hz / e);
        }
        __syncthreads();
        if (t == 0) {
            // lysh_phase1_check_ex from the cave at maxHeight on (phase1.c:149-199)
            auto spag = [&](int hi) {
                const double e = S.tun[hi];
                const double tv = combine_vals(N_SPAGHETTI_THICKNESS, &S.val[kBaseThickness][hi], kLadderHeights);
                const double h = lerp((tv - -1.0) / (1.0 - -1.0), 0.065, 0.088);
                const double l = combine_vals(N_SPAGHETTI_1, &S.val[kBaseSp1][hi], kLadderHeights);
                const double m = fabs(e * l) - h;
                const double n = combine_vals(N_SPAGHETTI_2, &S.val[kBaseSp2][hi], kLadderHeights);
                const double o = fabs(e * n) - h;
                const double pp = clampd(jmax(m, o), -1.0, 1.0);
                const double mod = combine_vals(N_ROUGHNESS_MODULATOR, &S.val[kBaseRmod][hi], kLadderHeights);
                const double rgh = combine_vals(N_ROUGHNESS, &S.val[kBaseRough][hi], kLadderHeights);
                const double qq = (-0.05 + (-0.05 * mod)) * (-0.4 + fabs(rgh));
                return pp + qq;
            };
            auto chz = [&](int hi) {
                const double layer = combine_vals(N_CAVE_LAYER, &S.val[kBaseLayer][hi], kLadderHeights);
                const double av = 4.0 * layer * layer;
                const double raw = combine_vals(N_CAVE_CHEESE, &S.val[kBaseCheese][hi], kLadderHeights);
                return av + clampd(0.27 + raw, -1.0, 1.0);
            };
            int code = P1_ACCEPT;
            if (spag(0) >= 0 && chz(0) >= 0) code = P1_CAVE_AT_MAXH;
            if (code == P1_ACCEPT)
                for (int hi = 1; hi < first_pos; hi++)
                    if (spag(hi) >= 0 && chz(hi) >= 0) {
                        code = P1_LADDER_NEG;
                        break;
                    }
            if (code == P1_ACCEPT)
                for (int hi = first_pos; hi < nh; hi++) {
                    const int y = S.ys[hi];
                    const double ent = combine_vals(N_CAVE_ENTRANCE, &S.val[kBaseEntrance][hi], kLadderHeights);
                    const double tt = (10.0 + (double)y) / 40.0;
                    const double cl = tt < 0.0 ? 0.3 : (tt > 1.0 ? 0.0 : lerp(tt, 0.3, 0.0));
                    const double cc = ent + 0.37 + cl;
                    if (jmin(cc, spag(hi)) >= 0 && chz(hi) >= 0) {
                        code = P1_LADDER_POS;
                        break;
                    }
                }
            if (code == P1_ACCEPT && !a.single_biome) {
                // the y = 0 climate sample equals the 3-D sample at y = 0 bit for bit
                const double c = combine_vals(cont_noise, &S.val[kBaseCont][0], kLadderHeights);
                if (c < -0.11) code = P1_CONTINENTALNESS;
            }
            if (code == P1_ACCEPT) {
                if (nf_ll <= kFloodHeights) {
                    for (int fi = 0; fi < nf; fi++)
                        if (combine_vals(N_FLOODEDNESS, &S.fval[0][fi], kFloodHeights) > 0.41) {
                            code = P1_FLOODEDNESS;
                            break;
                        }
                } else {
                    for (long long y = mh; y <= 60; y += 10) {
                        const double f = dbl3d(src, N_FLOODEDNESS, kBaseFlood, (double)(hut_x + 3),
                                               (double)y * 0.67, (double)(hut_z + 3));
                        if (f > 0.41) {
                            code = P1_FLOODEDNESS;
                            break;
                        }
                    }
                }
            }
            atomicAdd(&a.hist[code], 1ull);
            note_code(a, g, r, code, -1);
            if (code == P1_ACCEPT) {
                uint32_t oi = atomicAdd(&a.counters[CNT_FINAL], 1u);
                if (oi < a.cap_out) {
                    Candidate c;
                    c.seed_index = g;
                    c.seed = (int64_t)seed;
                    c.rx = rx;
                    c.rz = rz;
                    c.chunk_x = cx;
                    c.chunk_z = cz;
                    a.out[oi] = c;
                } else {
                    atomicOr(&a.counters[CNT_OVERFLOW], 4u);
                }
            }
        }
        __syncthreads();
    }
}

// grid <= 0: as many blocks as are resident at once (the kernel loops over candidates, so blocks
// beyond the resident count would only form a second, mostly idle wave)
static int g_ladder_per_sm = 0, g_ladder_sms = 0;

static void ladder_geometry() {
    if (g_ladder_per_sm) return;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_ladder_sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_ladder_per_sm, ladder_kernel, kThreadsC, 0);
    if (g_ladder_per_sm < 1) g_ladder_per_sm = 1;
}

void launch_ladder(const BatchArgs &a, int grid, cudaStream_t s) {
    if (grid <= 0) {
        ladder_geometry();
        grid = g_ladder_sms * g_ladder_per_sm;
    }
    ladder_kernel<<<grid, kThreadsC, 0, s>>>(a);
}

void prepare_phase1_launches() {
    allow_dynamic_smem(climate_kernel<true, true>, sizeof(ClimateSmem<true>), g_smem_done32s);
    allow_dynamic_smem(climate_kernel<true, false>, sizeof(ClimateSmem<true>), g_smem_done32);
    allow_dynamic_smem(climate_kernel<false, false>, sizeof(ClimateSmem<false>), g_smem_done64);
    allow_dynamic_smem(entrance_kernel<false>, sizeof(EntranceSmem), g_smem_done_ent);
    allow_dynamic_smem(entrance_kernel<true>, sizeof(EntranceSmem), g_smem_done_ent32);
    ladder_geometry();
}

}  // namespace wg
