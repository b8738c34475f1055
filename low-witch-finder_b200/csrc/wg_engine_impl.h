// The engine object behind include/witchgpu.h (private to the library).
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <string>
#include <vector>

#include "wg_phase1.cuh"

namespace wg {
struct P2Tables;
struct P2World;
struct P2Chunk;
struct P2Hut;
struct P2Result;
}  // namespace wg

struct wg_engine {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
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

    // phase 2 (wg_p2engine.cu): device tables, grow-only work buffers
    wg::P2Tables *p2_tables = nullptr;
    std::vector<void *> p2_game;          // device copies of the game data tables
    wg::P2World *p2_worlds = nullptr;
    wg::P2Chunk *p2_jobs = nullptr;
    wg::P2Hut *p2_huts = nullptr;
    wg::P2Result *p2_results = nullptr;
    int32_t *p2_pts = nullptr;
    double *p2_vals = nullptr;
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
