// The engine object behind include/witchgpu.h (private to the library).
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <string>
#include <vector>

#include "../../include/witchgpu.h"
#include "wg_phase1.cuh"

namespace wg {
struct P2Tables;
struct P2World;
struct P2Chunk;
struct P2Hut;
struct P2Result;
struct QueueRes;
}  // namespace wg

struct wg_engine {
    int device = 0;
    int sm_count = 148;
    int fp32_core = 1;   // 1 FP32 core with FP64 rechecks, 3 also the cave samples, 0 FP64, 2 as 3 re-taking every gate
    int job_queue = 1;   // wg_seed_check_jobs through the device work queue (1) or the host batch loop (0)
    // autotuned job settings (wg_engine_tune): regions per unit per job class (0 = window_for's
    // rule) and (seed, region) checks per queue slice (0 = kWorkPerBatch)
    uint32_t tuned_win[4] = {0, 0, 0, 0};
    uint64_t tuned_budget = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaStream_t copy_stream = nullptr;   // host seed uploads of wg_seed_check, one batch ahead
    cudaEvent_t ev_up = nullptr;          // recorded after the last upload enqueued
    std::string err;

    uint32_t *rec_unit = nullptr, *rec_off = nullptr, *rec_cnt = nullptr, *surv = nullptr, *deep = nullptr;
    wg::Candidate *out = nullptr;
    uint32_t *counters = nullptr;
    unsigned long long *hist = nullptr;
    uint32_t *h_counters = nullptr;         // pinned
    unsigned long long *h_hist = nullptr;   // pinned
    cudaEvent_t kev[4] = {nullptr, nullptr, nullptr, nullptr};   // around the three kernels of a batch
    int64_t *d_seed_list = nullptr;
    uint64_t d_seed_cap = 0;
    // breadth-first climate stage of one-region batches: two item lists and their counts
    wg::SpotItem *spot_items[2] = {nullptr, nullptr};
    uint32_t *spot_counts = nullptr;

    // phase 2 (wg_p2engine.cu): device tables, grow-only work buffers
    wg::P2Tables *p2_tables = nullptr;
    std::vector<void *> p2_game;          // device copies of the game data tables
    wg::P2World *p2_worlds = nullptr;
    wg::P2Chunk *p2_jobs = nullptr;
    wg::P2Hut *p2_huts = nullptr;
    wg::P2Result *p2_results = nullptr;
    int32_t *p2_pts = nullptr;
    double *p2_vals = nullptr;
    // Deep Dive solver (wg_solve.cu): its device tables and work buffers
    struct SolveState *solve = nullptr;
    // Deep Dive region walk (wg_deep.cu): its grow-only work buffers
    struct WalkState *walk = nullptr;
    // device work queue of batched jobs (wg_queue.cu): its state and output buffer
    wg::QueueRes *queue = nullptr;
    // mineshaft finisher (wg_finish.cu): its grow-only buffers
    struct FinishState *finish = nullptr;

    int p2_world_cap = 0, p2_job_cap = 0, p2_hut_cap = 0, p2_result_cap = 0, p2_pt_cap = 0, p2_val_cap = 0;

    int fail(int code, const char *what, cudaError_t e = cudaSuccess) {
        char buf[512];
        if (e != cudaSuccess) std::snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
        else std::snprintf(buf, sizeof buf, "%s", what);
        err = buf;
        return code;
    }
};

// Frees the phase-2 state of an engine (called by wg_engine_close).
void p2_release(wg_engine *eng);
// Frees the Deep Dive solver state of an engine (called by wg_engine_close).
void solve_release(wg_engine *eng);
// Frees the region walk's buffers of an engine (called by wg_engine_close).
void walk_release(wg_engine *eng);
// Frees the finisher's buffers of an engine (called by wg_engine_close).
void finish_release(wg_engine *eng);

namespace wg {

// Phase-2 state of up to 512 chunks (wg_p2engine.cu): the seed-independent tables, the worlds of
// `seeds` (large biomes or not) and, per chunk i (world index world[i], chunk cx[i], cz[i]), its
// grid, aquifer, block states and carver result in eng->p2_worlds / eng->p2_jobs, chunk i at
// index i.  Asynchronous on eng->stream.
int p2_prepare_chunks(wg_engine *eng, const std::vector<uint64_t> &seeds, int large, const std::vector<int> &world,
                      const std::vector<int> &cx, const std::vector<int> &cz);

// Per-batch work budget: (seed, region) checks per batch and units per batch, and the sizes of
// the engine's phase-1 work lists.
constexpr uint64_t kWorkPerBatch = 1ull << 27;
constexpr uint32_t kMaxUnits = 1u << 20;
constexpr uint32_t kCapRec = kMaxUnits + (1u << 16);
constexpr uint32_t kCapSurv = 1u << 23;
constexpr uint32_t kCapDeep = 1u << 20;
constexpr uint32_t kCapOut = 1u << 20;
// Units per batch of the breadth-first one-region climate stage (its item lists are this long;
// its climate survivors, ~1.7 %, stay far below the record capacity).
constexpr uint32_t kSpotUnits = 1u << 22;

// Whether a batch takes the breadth-first one-region climate stage.
inline bool spot_path(bool jobs, uint64_t win, bool codes, bool single_biome) {
    return !jobs && win == 1 && !codes && !single_biome;
}

// Regions per unit window: a whole seed when its rect is small, else 2048-region windows.
uint32_t window_for(uint64_t n_regions);

// Job classes of the autotuner by regions per seed: <= 16, <= 256, <= 4096, more.
constexpr uint64_t kJobClassMax[4] = {16, 256, 4096, ~0ull};
inline int job_class(uint64_t n_regions) {
    int c = 0;
    while (c < 3 && n_regions > kJobClassMax[c]) c++;
    return c;
}
// A job's window: the engine's tuned value for its class, else window_for's rule.
inline uint32_t job_window(const wg_engine *eng, uint64_t n_regions) {
    const uint32_t w = eng ? eng->tuned_win[job_class(n_regions)] : 0u;
    if (!w) return window_for(n_regions);
    return (uint32_t)(n_regions < w ? n_regions : w);
}

// One phase-1 request over one rect (wg_engine.cu).
struct Request {
    const int64_t *d_seeds;   // device seeds or nullptr (generator)
    uint64_t gen_base;
    uint64_t n_seeds;
    wg_opts opts;
    int max_height, salt;
    int rx0, rx1, rz0, rz1;
    int8_t *d_codes, *d_tiers;   // optional per-region verdicts (device)
    const int64_t *d_spot_s48;   // optional spots mode (BatchArgs::spot_s48 and the spot regions)
    const int32_t *d_spot_rx, *d_spot_rz;
    const int64_t *h_seeds;      // optional host seeds: run_request uploads each batch's seeds into
                                 // d_seeds on the copy stream while the batch before it runs
};

struct Sink {            // where phase-1 survivors go after each batch
    std::vector<Candidate> *host = nullptr;
    Candidate *dev = nullptr;
    uint64_t dev_cap = 0;
    uint64_t found = 0;
};

// The BatchArgs fields every batch of an engine shares (work lists, counters, rules, salt).
BatchArgs base_args(wg_engine *eng, const wg_opts &opts, int salt);
// Runs units [unit0, unit0 + n_units) of `proto` (three kernels, one sync), halving on overflow.
int run_batch(wg_engine *eng, const BatchArgs &proto, uint64_t unit0, uint32_t n_units, Sink &sink,
              wg_scan_stats &st);
int run_request(wg_engine *eng, const Request &rq, Sink &sink, wg_scan_stats &st);

}  // namespace wg
