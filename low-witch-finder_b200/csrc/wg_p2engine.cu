// Host side of phase 2 (include/witchgpu.h: wg_eval_huts, wg_grade_scan, wg_p2_probe): the
// seed-independent tables, grouping huts into worlds (seeds) and jobs (seed, hut chunk), and the
// kernel sequence legacy -> build -> grid -> aquifer -> carve -> finish (wg_phase2.cuh).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <utility>
#include <vector>

#include "../../include/witchgpu.h"
#include "wg_catalog.h"
#include "wg_engine_impl.h"
#include "wg_gamedata.h"
#include "wg_phase2.cuh"

using namespace wg;

#define P2_CUDA(call, what)                                             \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) return eng->fail(WG_ERR_CUDA, what, e_); \
    } while (0)

namespace {

// Identifiers of the noises phase 2 samples (the reference's terrain.c:8-16, biome.c:82-89,
// density.c:28-55, aquifer.c:121-124), and the LARGE_BIOMES replacements.
const char *const kQNames[Q_COUNT] = {
    "minecraft:offset",
    "minecraft:continentalness",
    "minecraft:erosion",
    "minecraft:ridge",
    "minecraft:temperature",
    "minecraft:vegetation",
    "minecraft:jagged",
    "minecraft:cave_entrance",
    "minecraft:spaghetti_roughness",
    "minecraft:spaghetti_roughness_modulator",
    "minecraft:spaghetti_3d_1",
    "minecraft:spaghetti_3d_2",
    "minecraft:spaghetti_3d_rarity",
    "minecraft:spaghetti_3d_thickness",
    "minecraft:spaghetti_2d",
    "minecraft:spaghetti_2d_elevation",
    "minecraft:spaghetti_2d_modulator",
    "minecraft:spaghetti_2d_thickness",
    "minecraft:pillar",
    "minecraft:pillar_rareness",
    "minecraft:pillar_thickness",
    "minecraft:cave_layer",
    "minecraft:cave_cheese",
    "minecraft:noodle",
    "minecraft:noodle_thickness",
    "minecraft:noodle_ridge_a",
    "minecraft:noodle_ridge_b",
    "minecraft:aquifer_barrier",
    "minecraft:aquifer_fluid_level_floodedness",
    "minecraft:aquifer_fluid_level_spread",
    "minecraft:aquifer_lava",
};

const char *large_name(int q) {
    switch (q) {
        case Q_CONT: return "minecraft:continentalness_large";
        case Q_EROSION: return "minecraft:erosion_large";
        case Q_TEMPERATURE: return "minecraft:temperature_large";
        case Q_VEGETATION: return "minecraft:vegetation_large";
        default: return kQNames[q];
    }
}

void digest(const char *s, uint64_t &lo, uint64_t &hi) {
    uint8_t d[16];
    md5((const uint8_t *)s, std::strlen(s), d);
    lo = hi = 0;
    for (int i = 0; i < 8; i++) lo = (lo << 8) | d[i];
    for (int i = 8; i < 16; i++) hi = (hi << 8) | d[i];
}

const GameNoise *find_noise(const GameData &g, const char *id) {
    for (int i = 0; i < g.n_noises; i++)
        if (!std::strcmp(g.noises[i].id, id)) return &g.noises[i];
    return nullptr;
}

// Spec + digests of one noise (noise.c:75-143: running lacunarity 2^firstOctave and
// persistence 2^(n-1) / (2^n - 1) over every slot, octave names "octave_<firstOctave + i>",
// amplitude 1/6 / (0.1 * (1 + 1 / (span + 1)))).
bool make_spec(const GameNoise &n, P2Spec &s, P2Digest &d) {
    std::memset(&s, 0, sizeof s);
    std::memset(&d, 0, sizeof d);
    if (n.n > kP2MaxOct) return false;
    digest(n.id, d.name_lo, d.name_hi);
    double lac = std::pow(2.0, (double)n.first_octave);
    double per = std::pow(2.0, (double)(n.n - 1)) / (std::pow(2.0, (double)n.n) - 1.0);
    int lo = -1, hi = -1, np = 0;
    for (int i = 0; i < n.n; i++) {
        if (n.amps[i] != 0.0) {
            char name[32];
            std::snprintf(name, sizeof name, "octave_%d", n.first_octave + i);
            digest(name, d.oct_lo[np], d.oct_hi[np]);
            s.amp[np] = n.amps[i];
            s.lac[np] = lac;
            s.per[np] = per;
            np++;
            if (lo < 0) lo = i;
            hi = i;
        }
        lac *= 2.0;
        per /= 2.0;
    }
    s.npresent = np;
    const double span = (double)(hi - lo);
    s.amplitude = 0.16666666666666666 / (0.1 * (1.0 + 1.0 / (span + 1.0)));
    return np > 0;
}

template <class T>
int upload(wg_engine *eng, const T *src, size_t count, const T **dst) {
    void *p = nullptr;
    P2_CUDA(cudaMalloc(&p, sizeof(T) * count), "alloc game data");
    eng->p2_game.push_back(p);
    P2_CUDA(cudaMemcpy(p, src, sizeof(T) * count, cudaMemcpyHostToDevice), "upload game data");
    *dst = static_cast<const T *>(p);
    return WG_OK;
}

// Nesting depth of a spline node / an R-tree node (the device evaluators use fixed stacks).
int spline_depth(const GameData &g, int node) {
    const SplineNode &n = g.nodes[node];
    if (n.kind == 1) return 1;
    int d = 0;
    for (int k = 0; k < n.n; k++) d = std::max(d, spline_depth(g, g.child[n.child + k]));
    return d + 1;
}
int tree_depth(const BiomeTree &t, int node) {
    if (t.kids[node] == 0) return 1;
    int d = 0, c = node + 1;
    for (int k = 0; k < t.kids[node]; k++, c = t.end[c]) d = std::max(d, tree_depth(t, c));
    return d + 1;
}

int ensure_tables(wg_engine *eng) {
    if (eng->p2_tables) return WG_OK;
    const GameData &g = game_data();
    if (!g.available)
        return eng->fail(WG_ERR_ARG, "phase 2 needs the game data tables, which were not found when the library was "
                                     "built (set LYSH to the reference's engine/tools/lysh/src and rebuild)");
    if (spline_depth(g, g.root_offset) > kSplineDepth || spline_depth(g, g.root_factor) > kSplineDepth ||
        spline_depth(g, g.root_peak) > kSplineDepth)
        return eng->fail(WG_ERR_ARG, "phase 2: terrain spline nests deeper than the device evaluator holds");
    for (int k = 0; k < kBiomeTrees; k++)
        if (tree_depth(g.trees[k], 0) > kTreeDepth)
            return eng->fail(WG_ERR_ARG, "phase 2: biome tree nests deeper than the device search holds");
    std::vector<P2Tables> hv(1);
    P2Tables *h = hv.data();
    std::memset(h, 0, sizeof *h);
    for (int v = 0; v < 2; v++)
        for (int q = 0; q < Q_COUNT; q++) {
            const char *id = v ? large_name(q) : kQNames[q];
            const GameNoise *n = find_noise(g, id);
            if (!n || !make_spec(*n, h->spec[v][q], h->digest[v][q]))
                return eng->fail(WG_ERR_ARG, "phase 2: noise missing from the game data table");
        }
    int slot = 0;
    for (int q = 0; q < Q_COUNT; q++) {
        const int np = h->spec[0][q].npresent;
        if (h->spec[1][q].npresent != np || slot + 2 * np > kWorldSlotsMax)
            return eng->fail(WG_ERR_ARG, "phase 2: noise table layout");
        h->spec[0][q].first_slot = h->spec[1][q].first_slot = slot;
        for (int sub = 0; sub < 2; sub++)
            for (int p = 0; p < np; p++, slot++) {
                h->slot_noise[slot] = (int16_t)q;
                h->slot_sub[slot] = (int8_t)sub;
                h->slot_oct[slot] = (int8_t)p;
            }
    }
    h->n_slots = slot;
    if (slot + kLegacyPerlins > kWorldSlotsMax) return eng->fail(WG_ERR_ARG, "phase 2: world slots");
    digest("minecraft:terrain", h->terrain_lo, h->terrain_hi);
    digest("minecraft:aquifer", h->aquifer_lo, h->aquifer_hi);
    int rc = upload(eng, g.nodes, (size_t)g.n_nodes, &h->nodes);
    if (!rc) rc = upload(eng, g.floats, (size_t)g.n_floats, &h->floats);
    if (!rc) rc = upload(eng, g.child, (size_t)g.n_child, &h->child);
    if (!rc) {   // legacy octave k starts 259 k Xoroshiro steps in, when no earlier bounded draw rejects
        const auto step = [](uint64_t &lo, uint64_t &hi) {
            const uint64_t x = hi ^ lo;
            lo = ((lo << 49) | (lo >> 15)) ^ x ^ (x << 21);
            hi = (x << 28) | (x >> 36);
        };
        std::vector<uint64_t> jumps((size_t)kLegacyPerlins * 128 * 2, 0);
        uint64_t clo[128], chi[128];   // column j: the image of basis vector j
        for (int j = 0; j < 128; j++) {
            clo[j] = j < 64 ? 1ULL << j : 0;
            chi[j] = j < 64 ? 0 : 1ULL << (j - 64);
        }
        for (int k = 0; k < kLegacyPerlins; k++) {
            for (int b = 0; b < 128; b++)
                for (int j = 0; j < 128; j++) {
                    const uint64_t bit = b < 64 ? (clo[j] >> b) & 1 : (chi[j] >> (b - 64)) & 1;
                    jumps[((size_t)k * 128 + b) * 2 + (j >> 6)] |= bit << (j & 63);
                }
            for (int j = 0; j < 128; j++)
                for (int n = 0; n < 259; n++) step(clo[j], chi[j]);
        }
        rc = upload(eng, jumps.data(), jumps.size(), &h->legacy_jump);
    }
    if (!rc) {   // the sine table as a quarter wave, checked against the full table
        std::vector<float> quarter(kSinQuarterPad, 0.0f);
        for (int i = 0; i < kSinQuarter; i++) quarter[i] = g.sin_table[i];
        h->sin_half_turn = g.sin_table[32768];
        for (int i = 0; i < kSinEntries; i++) {
            const int hh = i & 32767, k = hh <= 16384 ? hh : 32768 - hh;
            float v = (i & 32768) ? -quarter[k] : quarter[k];
            if (i == 32768) v = h->sin_half_turn;
            uint32_t a, b;
            std::memcpy(&a, &v, 4);
            std::memcpy(&b, &g.sin_table[i], 4);
            if (a != b) return eng->fail(WG_ERR_ARG, "phase 2: sine table is not a quarter wave");
        }
        rc = upload(eng, quarter.data(), quarter.size(), &h->sin_quarter);
    }
    h->root_offset = g.root_offset;
    h->root_factor = g.root_factor;
    h->root_peak = g.root_peak;
    for (int k = 0; k < kBiomeTrees && !rc; k++) {
        const BiomeTree &t = g.trees[k];
        BiomeTree &d = h->trees[k];
        d.n_nodes = t.n_nodes;
        rc = upload(eng, t.range, (size_t)t.n_nodes * 12, &d.range);
        if (!rc) rc = upload(eng, t.kids, (size_t)t.n_nodes, &d.kids);
        if (!rc) rc = upload(eng, t.biome, (size_t)t.n_nodes, &d.biome);
        if (!rc) rc = upload(eng, t.end, (size_t)t.n_nodes, &d.end);
    }
    if (rc) return rc;
    void *p = nullptr;
    P2_CUDA(cudaMalloc(&p, sizeof(P2Tables)), "alloc phase-2 tables");
    eng->p2_tables = static_cast<P2Tables *>(p);
    P2_CUDA(cudaMemcpy(p, h, sizeof(P2Tables), cudaMemcpyHostToDevice), "upload phase-2 tables");
    return WG_OK;
}

template <class T>
int grow(wg_engine *eng, T **buf, int &cap, int need) {
    if (need <= cap) return WG_OK;
    cudaFree(*buf);
    *buf = nullptr;
    cap = 0;
    const int n = std::max(need, 16);
    P2_CUDA(cudaMalloc((void **)buf, sizeof(T) * (size_t)n), "alloc phase-2 buffers");
    cap = n;
    return WG_OK;
}

// Biome tree of a search context (eval.c:100-107).
int tree_for(const wg_opts &o) {
    if (o.biome_tree > 0) return std::min(o.biome_tree - 1, kBiomeTrees - 1);
    if (o.mc_1_18_2) return 0;    // "1.18.2"
    if (o.pre_26_2) return 5;     // "1.21.5"
    return 6;                     // "26.2"
}

constexpr int kJobsPerBatch = 512;

struct JobKey {
    int world, cx, cz;
    bool operator<(const JobKey &o) const {
        if (world != o.world) return world < o.world;
        if (cx != o.cx) return cx < o.cx;
        return cz < o.cz;
    }
};

// Builds the worlds of `seeds` and the chunk state of `jobs` (world index, chunk) on the device.
int prepare(wg_engine *eng, const std::vector<uint64_t> &seeds, int large, const std::vector<JobKey> &jobs,
            bool carve) {
    int rc = grow(eng, &eng->p2_worlds, eng->p2_world_cap, (int)seeds.size());
    if (!rc) rc = grow(eng, &eng->p2_jobs, eng->p2_job_cap, (int)jobs.size());
    if (rc) return rc;
    struct WorldHead {
        uint64_t seed;
        int large, pad;
    };
    std::vector<WorldHead> wh(seeds.size());
    for (size_t i = 0; i < seeds.size(); i++) wh[i] = WorldHead{seeds[i], large, 0};
    P2_CUDA(cudaMemcpy2DAsync(eng->p2_worlds, sizeof(P2World), wh.data(), sizeof(WorldHead), sizeof(WorldHead),
                              wh.size(), cudaMemcpyHostToDevice, eng->stream),
            "upload worlds");
    struct JobHead {
        int world, chunk_x, chunk_z, max_psl, min_gx, min_gy, min_gz, carved;
    };
    std::vector<JobHead> jh(jobs.size());
    for (size_t i = 0; i < jobs.size(); i++)
        jh[i] = JobHead{jobs[i].world, jobs[i].cx, jobs[i].cz, INT_MIN, 0, 0, 0, 0};
    if (!jobs.empty())
        P2_CUDA(cudaMemcpy2DAsync(eng->p2_jobs, sizeof(P2Chunk), jh.data(), sizeof(JobHead), sizeof(JobHead),
                                  jh.size(), cudaMemcpyHostToDevice, eng->stream),
                "upload jobs");
    p2_launch_legacy(eng->p2_tables, eng->p2_worlds, (int)seeds.size(), eng->stream);
    p2_launch_build(eng->p2_tables, eng->p2_worlds, (int)seeds.size(), eng->stream);
    if (!jobs.empty()) {
        p2_launch_grid(eng->p2_tables, eng->p2_worlds, eng->p2_jobs, (int)jobs.size(), eng->stream);
        p2_launch_aquifer(eng->p2_tables, eng->p2_worlds, eng->p2_jobs, (int)jobs.size(), eng->stream);
        p2_launch_states(eng->p2_tables, eng->p2_worlds, eng->p2_jobs, (int)jobs.size(), eng->stream);
        if (carve) p2_launch_carve(eng->p2_tables, eng->p2_worlds, eng->p2_jobs, (int)jobs.size(), eng->stream);
    }
    P2_CUDA(cudaGetLastError(), "phase-2 launch");
    return WG_OK;
}

// Phase 2 for huts[first, first + n), which hold at most kJobsPerBatch distinct (seed, chunk) jobs.
int eval_batch(wg_engine *eng, const int64_t *seeds, const int32_t *hx, const int32_t *hz, uint64_t first, uint64_t n,
               const wg_opts &o, int max_y, wg_hut_result *out) {
    std::map<uint64_t, int> world_of;
    std::vector<uint64_t> wseeds;
    std::map<JobKey, int> job_of;
    std::vector<JobKey> jobs;
    std::vector<P2Hut> huts(n);
    for (uint64_t i = 0; i < n; i++) {
        const uint64_t s = (uint64_t)seeds[first + i];
        auto w = world_of.find(s);
        int wi;
        if (w == world_of.end()) {
            wi = (int)wseeds.size();
            world_of[s] = wi;
            wseeds.push_back(s);
        } else {
            wi = w->second;
        }
        const JobKey k{wi, hx[first + i] >> 4, hz[first + i] >> 4};
        auto j = job_of.find(k);
        int ji;
        if (j == job_of.end()) {
            ji = (int)jobs.size();
            job_of[k] = ji;
            jobs.push_back(k);
        } else {
            ji = j->second;
        }
        huts[i] = P2Hut{ji, hx[first + i], hz[first + i], max_y};
    }
    int rc = prepare(eng, wseeds, o.large_biomes ? 1 : 0, jobs, true);
    if (!rc) rc = grow(eng, &eng->p2_huts, eng->p2_hut_cap, (int)n);
    if (!rc) rc = grow(eng, &eng->p2_results, eng->p2_result_cap, (int)n);
    if (rc) return rc;
    P2_CUDA(cudaMemcpyAsync(eng->p2_huts, huts.data(), sizeof(P2Hut) * n, cudaMemcpyHostToDevice, eng->stream),
            "upload huts");
    p2_launch_finish(eng->p2_tables, eng->p2_worlds, eng->p2_jobs, eng->p2_huts, (int)n, tree_for(o),
                     eng->p2_results, eng->stream);
    P2_CUDA(cudaGetLastError(), "phase-2 finish");
    static_assert(sizeof(wg_hut_result) == sizeof(P2Result), "hut result layout");
    P2_CUDA(cudaMemcpyAsync(out + first, eng->p2_results, sizeof(P2Result) * n, cudaMemcpyDeviceToHost, eng->stream),
            "copy results");
    P2_CUDA(cudaStreamSynchronize(eng->stream), "phase 2");
    return WG_OK;
}

int eval_huts(wg_engine *eng, const int64_t *seeds, const int32_t *hx, const int32_t *hz, uint64_t n, const wg_opts &o,
              int max_y, wg_hut_result *out) {
    int rc = ensure_tables(eng);
    if (rc) return rc;
    uint64_t first = 0;
    while (first < n) {   // batches of at most kJobsPerBatch distinct chunks
        std::map<std::pair<uint64_t, std::pair<int, int>>, int> seen;
        uint64_t count = 0;
        while (first + count < n) {
            auto key = std::make_pair((uint64_t)seeds[first + count],
                                      std::make_pair(hx[first + count] >> 4, hz[first + count] >> 4));
            if (!seen.count(key)) {
                if ((int)seen.size() == kJobsPerBatch) break;
                seen[key] = 1;
            }
            count++;
        }
        rc = eval_batch(eng, seeds, hx, hz, first, count, o, max_y, out);
        if (rc) return rc;
        first += count;
    }
    return WG_OK;
}

}  // namespace

int wg::p2_prepare_chunks(wg_engine *eng, const std::vector<uint64_t> &seeds, int large, const std::vector<int> &world,
                          const std::vector<int> &cx, const std::vector<int> &cz) {
    if (world.size() > (size_t)kJobsPerBatch || cx.size() != world.size() || cz.size() != world.size())
        return eng->fail(WG_ERR_ARG, "phase-2 chunks: more than 512 chunks per call");
    int rc = ensure_tables(eng);
    if (rc) return rc;
    std::vector<JobKey> jobs(world.size());
    for (size_t i = 0; i < world.size(); i++) jobs[i] = JobKey{world[i], cx[i], cz[i]};
    return prepare(eng, seeds, large, jobs, true);
}

void p2_release(wg_engine *eng) {
    for (void *p : eng->p2_game) cudaFree(p);
    eng->p2_game.clear();
    cudaFree(eng->p2_tables);
    cudaFree(eng->p2_worlds);
    cudaFree(eng->p2_jobs);
    cudaFree(eng->p2_huts);
    cudaFree(eng->p2_results);
    cudaFree(eng->p2_pts);
    cudaFree(eng->p2_vals);
    eng->p2_tables = nullptr;
    eng->p2_worlds = nullptr;
    eng->p2_jobs = nullptr;
    eng->p2_huts = nullptr;
    eng->p2_results = nullptr;
    eng->p2_pts = nullptr;
    eng->p2_vals = nullptr;
    eng->p2_world_cap = eng->p2_job_cap = eng->p2_hut_cap = eng->p2_result_cap = eng->p2_pt_cap = eng->p2_val_cap = 0;
}

extern "C" {

int wg_eval_huts(wg_engine *eng, const int64_t *seeds, const int32_t *hut_x, const int32_t *hut_z, uint64_t n,
                 const wg_opts *opts, int max_y, wg_hut_result *out) {
    if (!eng || (n && (!seeds || !hut_x || !hut_z || !out))) return WG_ERR_ARG;
    if (n == 0) return WG_OK;
    P2_CUDA(cudaSetDevice(eng->device), "cudaSetDevice");
    wg_opts o;
    std::memset(&o, 0, sizeof o);
    if (opts) o = *opts;
    return eval_huts(eng, seeds, hut_x, hut_z, n, o, max_y, out);
}

int wg_grade_scan(wg_engine *eng, int64_t seed, const wg_opts *opts, int max_height, int rx0, int rx1, int rz0,
                  int rz1, int salt, int max_y, int32_t *hits, int32_t hits_cap, wg_hut_grade *grade) {
    if (!eng || rx1 <= rx0 || rz1 <= rz0 || (hits_cap > 0 && !hits)) return WG_ERR_ARG;
    auto t0 = std::chrono::steady_clock::now();
    wg_opts o;
    std::memset(&o, 0, sizeof o);
    if (opts) o = *opts;
    // phase 1: every survivor of the rect, sorted (rz, rx)
    uint64_t found = 0;
    int rc = wg_seed_check(eng, &seed, 0, 1, &o, max_height, salt, rx0, rx1, rz0, rz1, nullptr, 0, &found, nullptr);
    if (rc) return rc;
    std::vector<wg_candidate> cand(found);
    if (found) {
        uint64_t again = 0;
        rc = wg_seed_check(eng, &seed, 0, 1, &o, max_height, salt, rx0, rx1, rz0, rz1, cand.data(), found, &again,
                           nullptr);
        if (rc) return rc;
    }
    // phase 2 on the survivors
    std::vector<int64_t> seeds(found, seed);
    std::vector<int32_t> hx(found), hz(found);
    for (uint64_t i = 0; i < found; i++) {
        hx[i] = cand[i].chunk_x * 16;
        hz[i] = cand[i].chunk_z * 16;
    }
    std::vector<wg_hut_result> res(found);
    auto t1 = std::chrono::steady_clock::now();
    if (found) {
        P2_CUDA(cudaSetDevice(eng->device), "cudaSetDevice");
        rc = eval_huts(eng, seeds.data(), hx.data(), hz.data(), found, o, max_y, res.data());
        if (rc) return rc;
    }
    auto t2 = std::chrono::steady_clock::now();
    wg_hut_grade g;
    std::memset(&g, 0, sizeof g);
    g.scanned = (int64_t)((int64_t)rx1 - rx0) * (int64_t)((int64_t)rz1 - rz0);
    g.evaluated = (int64_t)found;
    int32_t written = 0;
    for (uint64_t i = 0; i < found; i++) {
        const wg_hut_result &r = res[i];
        if (r.ok) {
            g.accepted++;
            if (hits && written < hits_cap) {
                int32_t *d = hits + (size_t)written * WG_HUT_GRADE_INTS;
                d[0] = r.hut_x; d[1] = r.hut_z; d[2] = r.rx; d[3] = r.rz; d[4] = r.dir; d[5] = r.avg_y;
                d[6] = r.flooded; d[7] = r.ok; d[8] = r.wet_columns; d[9] = r.size_x; d[10] = r.size_z;
                d[11] = r.reject;
                written++;
            }
        } else if (r.reject == 3) {
            g.rejected_biome++;
        } else if (r.reject == 1) {
            g.rejected_y++;
        } else if (r.reject == 2) {
            g.rejected_flood++;
        }
    }
    g.hits_written = written;
    g.p2_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
    g.ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (grade) *grade = g;
    return WG_OK;
}

int wg_p2_probe(wg_engine *eng, int64_t seed, const wg_opts *opts, int kind, const int32_t *xyz, uint64_t n,
                double *out) {
    if (!eng || kind < 0 || kind >= PR_KINDS || (n && (!xyz || !out))) return WG_ERR_ARG;
    if (n == 0) return WG_OK;
    if (n > (1u << 24)) return WG_ERR_CAPACITY;
    P2_CUDA(cudaSetDevice(eng->device), "cudaSetDevice");
    int rc = ensure_tables(eng);
    if (rc) return rc;
    wg_opts o;
    std::memset(&o, 0, sizeof o);
    if (opts) o = *opts;
    const bool per_chunk = kind >= PR_DENSITY;
    uint64_t first = 0;
    while (first < n) {   // points of at most kJobsPerBatch chunks per pass
        std::map<JobKey, int> job_of;
        std::vector<JobKey> jobs;
        std::vector<int32_t> pts;
        uint64_t count = 0;
        while (first + count < n) {
            const int32_t *p = xyz + 3 * (first + count);
            int ji = 0;
            if (per_chunk) {
                const JobKey k{0, p[0] >> 4, p[2] >> 4};
                auto it = job_of.find(k);
                if (it == job_of.end()) {
                    if ((int)jobs.size() == kJobsPerBatch) break;
                    ji = (int)jobs.size();
                    job_of[k] = ji;
                    jobs.push_back(k);
                } else {
                    ji = it->second;
                }
            }
            pts.insert(pts.end(), {0, p[0], p[1], p[2], ji});
            count++;
        }
        std::vector<uint64_t> ws(1, (uint64_t)seed);
        rc = prepare(eng, ws, o.large_biomes ? 1 : 0, jobs, kind == PR_HEIGHT);
        if (!rc) rc = grow(eng, &eng->p2_pts, eng->p2_pt_cap, (int)(5 * count));
        if (!rc) rc = grow(eng, &eng->p2_vals, eng->p2_val_cap, (int)count);
        if (rc) return rc;
        P2_CUDA(cudaMemcpyAsync(eng->p2_pts, pts.data(), sizeof(int32_t) * pts.size(), cudaMemcpyHostToDevice,
                                eng->stream),
                "upload probes");
        p2_launch_probe(eng->p2_tables, eng->p2_worlds, eng->p2_jobs, eng->p2_pts, (int)count, kind, eng->p2_vals,
                        eng->stream);
        P2_CUDA(cudaGetLastError(), "probe launch");
        P2_CUDA(cudaMemcpyAsync(out + first, eng->p2_vals, sizeof(double) * count, cudaMemcpyDeviceToHost,
                                eng->stream),
                "copy probes");
        P2_CUDA(cudaStreamSynchronize(eng->stream), "probes");
        first += count;
    }
    return WG_OK;
}

int wg_biome_map(wg_engine *eng, int64_t seed, const wg_opts *opts, int64_t x0, int64_t z0, int w, int h, int step,
                 int ss, int y, uint8_t *out) {
    if (!eng || !out || w <= 0 || h <= 0 || w > 4096 || h > 4096 || step < 1 || ss < 1 || ss > 4) return WG_ERR_ARG;
    P2_CUDA(cudaSetDevice(eng->device), "cudaSetDevice");
    wg_opts o;
    std::memset(&o, 0, sizeof o);
    if (opts) o = *opts;
    int rc = ensure_tables(eng);
    if (rc) return rc;
    rc = prepare(eng, std::vector<uint64_t>{(uint64_t)seed}, o.large_biomes ? 1 : 0, std::vector<JobKey>{}, false);
    if (rc) return rc;
    const size_t cells = (size_t)w * (size_t)h;
    uint8_t *d_out = nullptr;
    P2_CUDA(cudaMalloc(&d_out, cells), "biome map buffer");
    p2_launch_biome_map(eng->p2_tables, eng->p2_worlds, tree_for(o), x0, z0, w, h, step, ss, y, d_out, eng->stream);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, cells, cudaMemcpyDeviceToHost, eng->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(eng->stream);
    cudaFree(d_out);
    if (e != cudaSuccess) return eng->fail(WG_ERR_CUDA, "biome map", e);
    return WG_OK;
}

int wg_biome_chunks(wg_engine *eng, int64_t seed, const wg_opts *opts, const int32_t *cx, const int32_t *cz,
                    uint64_t n, uint8_t *out) {
    if (!eng || (n && (!cx || !cz || !out))) return WG_ERR_ARG;
    if (n == 0) return WG_OK;
    if (n > (1u << 24)) return WG_ERR_CAPACITY;
    P2_CUDA(cudaSetDevice(eng->device), "cudaSetDevice");
    wg_opts o;
    std::memset(&o, 0, sizeof o);
    if (opts) o = *opts;
    int rc = ensure_tables(eng);
    if (rc) return rc;
    rc = prepare(eng, std::vector<uint64_t>{(uint64_t)seed}, o.large_biomes ? 1 : 0, std::vector<JobKey>{}, false);
    if (rc) return rc;
    int32_t *d_xz = nullptr;
    uint8_t *d_out = nullptr;
    std::vector<uint8_t> need(n);
    cudaError_t e = cudaMalloc(&d_xz, sizeof(int32_t) * 2 * n);
    if (e == cudaSuccess) e = cudaMalloc(&d_out, 2 * n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_xz, cx, sizeof(int32_t) * n, cudaMemcpyHostToDevice, eng->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_xz + n, cz, sizeof(int32_t) * n, cudaMemcpyHostToDevice, eng->stream);
    if (e == cudaSuccess) {
        p2_launch_biome_chunks(eng->p2_tables, eng->p2_worlds, tree_for(o), d_xz, d_xz + n, (int)n, d_out, d_out + n,
                               eng->stream);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, n, cudaMemcpyDeviceToHost, eng->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(need.data(), d_out + n, n, cudaMemcpyDeviceToHost, eng->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(eng->stream);
    cudaFree(d_xz);
    cudaFree(d_out);
    if (e != cudaSuccess) return eng->fail(WG_ERR_CUDA, "biome chunks", e);
    // chunks on a swamp's edge: the biome with the real (pre-carver) surface of the chunk's middle,
    // which the phase-2 path computes for a hut at the chunk origin
    std::vector<int64_t> seeds;
    std::vector<int32_t> hx, hz;
    std::vector<uint64_t> at;
    for (uint64_t k = 0; k < n; k++)
        if (need[k]) {
            seeds.push_back(seed);
            hx.push_back(cx[k] * 16);
            hz.push_back(cz[k] * 16);
            at.push_back(k);
        }
    if (!at.empty()) {
        std::vector<wg_hut_result> r(at.size());
        rc = eval_huts(eng, seeds.data(), hx.data(), hz.data(), at.size(), o, -64, r.data());
        if (rc) return rc;
        for (size_t q = 0; q < at.size(); q++) out[at[q]] = (uint8_t)(r[q].biome_winner & 0xFF);
    }
    return WG_OK;
}

}  // extern "C"
