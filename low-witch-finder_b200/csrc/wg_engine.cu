// Host engine behind include/witchgpu.h: batch planning, device work buffers, the
// three-kernel phase-1 pipeline per batch, overflow retry and the funnel statistics.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/witchgpu.h"
#include "wg_catalog.h"
#include "wg_deep.cuh"
#include "wg_engine_impl.h"
#include "wg_phase1.cuh"
#include "wg_queue.h"

using namespace wg;

// Regions per unit window: a whole seed when its rect is small, else 2048-region windows.
uint32_t wg::window_for(uint64_t n_regions) { return n_regions <= 4096 ? (uint32_t)n_regions : 2048u; }

// Climate evaluation steps (see ClimateStep): the tiered erosion sequence
// (engine/tools/lysh/src/noise.c:387-459) followed by plain y=0 DoublePerlin samples of
// temperature and ridge (noise.c:320-342).
void wg::build_climate_steps(const NoiseSpec *specs, int erosion, int temperature, ClimateStep *st) {
    static const double thr[7] = {0.05, 0.22, 0.42, 0.45, 0.49, 0.51, 0.55};
    std::memset(st, 0, sizeof(ClimateStep) * kClimateSteps);
    const NoiseSpec &e = specs[erosion];
    int k = 0;
    for (int p = 0; p < e.npresent; p++)
        for (int sub = 0; sub < 2; sub++, k++) {
            ClimateStep &s = st[k];
            s.slot = sub * e.npresent + p;
            s.sc = sub ? 1.0181268882175227 : 1.0;
            s.lac = e.lac[p];
            s.c1 = e.amp[p] * e.per[p];
            s.c2 = 1.0;
            s.amp = e.amplitude;
            if (k >= 1) {
                s.act = (k == 7) ? ACT_TIER_LAST : ACT_TIER;
                s.tier = k - 1;
                s.thr = thr[k - 1];
            }
        }
    int base = 2 * e.npresent;
    const int plain[2] = {temperature, N_RIDGE};
    for (int q = 0; q < 2; q++) {
        const NoiseSpec &n = specs[plain[q]];
        for (int sub = 0; sub < 2; sub++)
            for (int p = 0; p < n.npresent; p++, k++) {
                ClimateStep &s = st[k];
                s.slot = base + sub * n.npresent + p;
                s.sc = sub ? 1.0181268882175227 : 1.0;
                s.lac = n.lac[p];
                s.c1 = n.amp[p];
                s.c2 = n.per[p];
                s.amp = n.amplitude;
                if (p == n.npresent - 1) s.act = sub ? (q == 0 ? ACT_TEMPERATURE : ACT_RIDGE) : ACT_END_SUB_A;
            }
        base += 2 * n.npresent;
    }
    // FP32 core: each running FP32 sum (erosion over steps 0..7; temperature 8..11; ridge 12..17,
    // each from zero) is s_k = fma(cf_k, v_k, s_{k-1}) with |v_k - exact sample| <= eps (the
    // Perlin bound) and |exact sample| <= 2.  Per step the error grows by
    //   |c_k| (eps + 2.01 u)          (the sample's error and cf_k = rn(c_k), c_k = c1 * c2)
    // + 2.01 u sum_{i<=k} |c_i|       (the FMA's rounding of a partial sum of that magnitude),
    // u = 2^-24.  The band half-width is twice that bound plus 1e-10, which covers the FP64
    // path's own distance from the exact value (~1e-13) and the rounding of sum * amp against
    // the threshold.
    const double u = 1.0 / 16777216.0, eps = kPerlinF32ErrUlps * u, vmax = 2.01;
    double err = 0.0, mag = 0.0;
    for (int i = 0; i < kClimateSteps; i++) {
        ClimateStep &s = st[i];
        if (i == 0 || i == 8 || i == 12) err = mag = 0.0;   // a new running sum starts
        const double c = s.c1 * s.c2;
        mag += std::fabs(c);
        err += std::fabs(c) * (eps + vmax * u) + vmax * u * mag;
        s.cf = (float)c;
        s.err = (float)(2.0 * err + 1e-10);
        if (s.act == ACT_TIER || s.act == ACT_TIER_LAST) {
            const double center = s.thr / s.amp, half = 2.0 * err + 1e-10;
            s.lo = std::nextafter((float)(center - half), -INFINITY);
            s.hi = std::nextafter((float)(center + half), INFINITY);
        }
    }
}

F32Bands wg::build_f32_bands(const ClimateStep *st) {
    F32Bands b;
    const double t_amp = st[11].amp, r_amp = st[17].amp, t_half = st[11].err, r_half = st[17].err;
    const double t_thr[2] = {-0.45, 0.2}, r_thr[4] = {-0.91, -0.42, 0.42, 0.91};
    for (int i = 0; i < 2; i++) {
        b.t_lo[i] = std::nextafter((float)(t_thr[i] / t_amp - t_half), -INFINITY);
        b.t_hi[i] = std::nextafter((float)(t_thr[i] / t_amp + t_half), INFINITY);
    }
    for (int i = 0; i < 4; i++) {
        b.r_lo[i] = std::nextafter((float)(r_thr[i] / r_amp - r_half), -INFINITY);
        b.r_hi[i] = std::nextafter((float)(r_thr[i] / r_amp + r_half), INFINITY);
    }
    return b;
}

namespace {
double g_climate_lac_max = 1.0;   // the largest lacunarity of a climate step (both presets)
}

bool wg::coords_small(int64_t lo, int64_t hi) {
    const double r = (double)std::max<int64_t>(std::llabs(lo), std::llabs(hi));
    return (4.0 * (32.0 * r + 23.0) + 2.0) * 1.02 * g_climate_lac_max < 0.99e7;
}

void wg::upload_phase1_tables() {
    NoiseSpec specs[N_NOISE_COUNT];
    build_noise_specs(specs);
    ClimateStep normal[kClimateSteps], large[kClimateSteps];
    build_climate_steps(specs, N_EROSION, N_TEMPERATURE, normal);
    build_climate_steps(specs, N_EROSION_LARGE, N_TEMPERATURE_LARGE, large);
    double lac = 0.0;
    for (int k = 0; k < kClimateSteps; k++) lac = std::max(lac, std::max(normal[k].lac, large[k].lac));
    g_climate_lac_max = lac;
    const F32Bands bands[2] = {build_f32_bands(normal), build_f32_bands(large)};
    upload_tables(specs, normal, large, bands);
}

#define WG_CUDA(call, what)                                        \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return eng->fail(WG_ERR_CUDA, what, e_); \
    } while (0)

namespace wg {

int run_batch(wg_engine *eng, const BatchArgs &proto, uint64_t unit0, uint32_t n_units, Sink &sink,
              wg_scan_stats &st) {
    BatchArgs a = proto;
    a.unit0 = unit0;
    a.n_units = n_units;
    WG_CUDA(cudaMemsetAsync(eng->counters, 0, sizeof(uint32_t) * CNT_WORDS, eng->stream), "memset counters");
    WG_CUDA(cudaMemsetAsync(eng->hist, 0, sizeof(unsigned long long) * (P1_KINDS + kTiers), eng->stream),
            "memset hist");
    WG_CUDA(cudaEventRecord(eng->kev[0], eng->stream), "event");
    // one region per unit: the climate tables are built lazily, breadth first
    if (spot_path(a.jobs != nullptr, a.win, a.codes != nullptr, a.single_biome != 0)) {
        if (!eng->spot_counts) {
            WG_CUDA(cudaMalloc(&eng->spot_items[0], sizeof(SpotItem) * kSpotUnits), "alloc");
            WG_CUDA(cudaMalloc(&eng->spot_items[1], sizeof(SpotItem) * kSpotUnits), "alloc");
            WG_CUDA(cudaMalloc(&eng->spot_counts, sizeof(uint32_t) * 2), "alloc");
        }
        launch_spot_climate(a, eng->spot_items[0], eng->spot_items[1], eng->spot_counts, kSpotUnits, eng->sm_count,
                            eng->stream);
    } else {
        launch_climate(a, eng->stream);
    }
    WG_CUDA(cudaEventRecord(eng->kev[1], eng->stream), "event");
    launch_entrance(a, 0, eng->stream);
    WG_CUDA(cudaEventRecord(eng->kev[2], eng->stream), "event");
    launch_ladder(a, 0, eng->stream);
    WG_CUDA(cudaEventRecord(eng->kev[3], eng->stream), "event");
    WG_CUDA(cudaGetLastError(), "kernel launch");
    WG_CUDA(cudaMemcpyAsync(eng->h_counters, eng->counters, sizeof(uint32_t) * CNT_WORDS, cudaMemcpyDeviceToHost,
                            eng->stream),
            "copy counters");
    WG_CUDA(cudaMemcpyAsync(eng->h_hist, eng->hist, sizeof(unsigned long long) * (P1_KINDS + kTiers),
                            cudaMemcpyDeviceToHost, eng->stream),
            "copy hist");
    WG_CUDA(cudaStreamSynchronize(eng->stream), "batch");
    st.batches++;
    for (int k = 0; k < 3; k++) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, eng->kev[k], eng->kev[k + 1]);
        st.kernel_ms[k] += ms;
        st.kernel_launches[k]++;
    }
    if (eng->h_counters[CNT_OVERFLOW]) {
        if (n_units <= 32) return eng->fail(WG_ERR_CAPACITY, "phase-1 work list full even for 32 units");
        st.retries++;
        uint32_t half = n_units / 2;
        int rc = run_batch(eng, proto, unit0, half, sink, st);
        if (rc) return rc;
        return run_batch(eng, proto, unit0 + half, n_units - half, sink, st);
    }
    for (int i = 0; i < P1_KINDS; i++) st.reject_hist[i] += (int64_t)eng->h_hist[i];
    for (int i = 0; i < kTiers; i++) st.tier_hist[i] += (int64_t)eng->h_hist[P1_KINDS + i];
    st.climate_survivors += eng->h_counters[CNT_SURVIVORS];
    st.rechecks += eng->h_counters[CNT_RECHECK];
    st.records += eng->h_counters[CNT_RECORDS];
    st.deep_candidates += eng->h_counters[CNT_DEEP];
    uint32_t nf = eng->h_counters[CNT_FINAL];
    if (nf) {
        if (sink.host) {
            size_t at = sink.host->size();
            sink.host->resize(at + nf);
            WG_CUDA(cudaMemcpy(sink.host->data() + at, eng->out, sizeof(Candidate) * nf, cudaMemcpyDeviceToHost),
                    "copy survivors");
        } else if (sink.dev && sink.found < sink.dev_cap) {
            uint64_t n = std::min<uint64_t>(nf, sink.dev_cap - sink.found);
            WG_CUDA(cudaMemcpyAsync(sink.dev + sink.found, eng->out, sizeof(Candidate) * n, cudaMemcpyDeviceToDevice,
                                    eng->stream),
                    "copy survivors");
        }
    }
    sink.found += nf;
    return WG_OK;
}

BatchArgs base_args(wg_engine *eng, const wg_opts &opts, int salt) {
    BatchArgs a;
    std::memset(&a, 0, sizeof a);
    a.salt = salt ? salt : 14357620;
    a.mc_1_18_2 = opts.mc_1_18_2;
    a.pre_26_2 = opts.pre_26_2;
    a.single_biome = opts.single_biome;
    a.large_biomes = opts.large_biomes;
    a.fp32_core = eng->fp32_core;
    a.rec_unit = eng->rec_unit;
    a.rec_off = eng->rec_off;
    a.rec_cnt = eng->rec_cnt;
    a.surv_region = eng->surv;
    a.deep = eng->deep;
    a.out = eng->out;
    a.cap_rec = kCapRec;
    a.cap_surv = kCapSurv;
    a.cap_deep = kCapDeep;
    a.cap_out = kCapOut;
    a.counters = eng->counters;
    a.hist = eng->hist;
    return a;
}

int run_request(wg_engine *eng, const Request &rq, Sink &sink, wg_scan_stats &st) {
    if (rq.rx1 <= rq.rx0 || rq.rz1 <= rq.rz0 || rq.n_seeds == 0) return eng->fail(WG_ERR_ARG, "empty request");
    const uint64_t rw = (uint64_t)((int64_t)rq.rx1 - rq.rx0), rh = (uint64_t)((int64_t)rq.rz1 - rq.rz0);
    const uint64_t n_regions = rw * rh;
    const uint32_t win = window_for(n_regions);
    const uint64_t n_win = (n_regions + win - 1) / win;
    const uint64_t units = rq.n_seeds * n_win;

    BatchArgs a = base_args(eng, rq.opts, rq.salt);
    a.seeds = rq.d_seeds;
    a.gen_base = rq.gen_base;
    a.win = win;
    a.n_win = n_win;
    a.n_regions = n_regions;
    a.rx0 = rq.rx0;
    a.rz0 = rq.rz0;
    a.rw = (int)rw;
    a.rh = (int)rh;
    a.max_height = rq.max_height;
    a.codes = rq.d_codes;
    a.tiers = rq.d_tiers;
    a.spot_s48 = rq.d_spot_s48;
    a.spot_rx = rq.d_spot_rx;
    a.spot_rz = rq.d_spot_rz;
    // spots shift the rect by their own regions: only plain requests are proved small
    a.small_coords = !rq.d_spot_s48 && coords_small(std::min(rq.rx0, rq.rz0), std::max(rq.rx1, rq.rz1) - 1ll) ? 1 : 0;

    uint64_t per_batch = std::min<uint64_t>(kMaxUnits, std::max<uint64_t>(32, kWorkPerBatch / win));
    if (rq.opts.single_biome)  // every region survives the climate stage
        per_batch = std::min<uint64_t>(per_batch, std::max<uint64_t>(32, kCapSurv / 2 / win));
    if (spot_path(false, win, rq.d_codes != nullptr, rq.opts.single_biome != 0)) per_batch = kSpotUnits;
    st.scanned = (int64_t)(rq.n_seeds * n_regions);
    // host seeds: the seeds of units [0, units_end) enqueued on the copy stream, ev_up after them
    uint64_t uploaded = 0;
    auto upload_to = [&](uint64_t units_end) -> int {
        const uint64_t need = std::min<uint64_t>(rq.n_seeds, (units_end + n_win - 1) / n_win);
        if (need <= uploaded) return WG_OK;
        WG_CUDA(cudaMemcpyAsync(const_cast<int64_t *>(rq.d_seeds) + uploaded, rq.h_seeds + uploaded,
                                sizeof(int64_t) * (need - uploaded), cudaMemcpyHostToDevice, eng->copy_stream),
                "upload seeds");
        WG_CUDA(cudaEventRecord(eng->ev_up, eng->copy_stream), "event");
        uploaded = need;
        return WG_OK;
    };
    for (uint64_t u0 = 0; u0 < units; u0 += per_batch) {
        uint32_t n = (uint32_t)std::min<uint64_t>(per_batch, units - u0);
        if (rq.h_seeds) {
            int rc = upload_to(u0 + n);   // this batch's seeds (enqueued during the batch before, except the first)
            if (rc) return rc;
            WG_CUDA(cudaStreamWaitEvent(eng->stream, eng->ev_up, 0), "wait for the seed upload");
            rc = upload_to(u0 + n + per_batch);   // the next batch's, while this one runs
            if (rc) return rc;
        }
        int rc = run_batch(eng, a, u0, n, sink, st);
        if (rc) return rc;
    }
    st.accepted = (int64_t)sink.found;
    return WG_OK;
}

}  // namespace wg

namespace {

int reserve_seeds(wg_engine *eng, uint64_t n) {
    if (n > eng->d_seed_cap) {
        if (eng->d_seed_list) cudaFree(eng->d_seed_list);
        eng->d_seed_list = nullptr;
        eng->d_seed_cap = 0;
        WG_CUDA(cudaMalloc(&eng->d_seed_list, sizeof(int64_t) * n), "alloc seed list");
        eng->d_seed_cap = n;
    }
    return WG_OK;
}

int stage_seeds(wg_engine *eng, const int64_t *seeds, uint64_t n, const int64_t **d_seeds) {
    *d_seeds = nullptr;
    if (!seeds) return WG_OK;
    if (n > eng->d_seed_cap) {
        if (eng->d_seed_list) cudaFree(eng->d_seed_list);
        eng->d_seed_list = nullptr;
        eng->d_seed_cap = 0;
        WG_CUDA(cudaMalloc(&eng->d_seed_list, sizeof(int64_t) * n), "alloc seed list");
        eng->d_seed_cap = n;
    }
    WG_CUDA(cudaMemcpyAsync(eng->d_seed_list, seeds, sizeof(int64_t) * n, cudaMemcpyHostToDevice, eng->stream),
            "upload seeds");
    *d_seeds = eng->d_seed_list;
    return WG_OK;
}

Request make_request(const wg_opts *opts, uint64_t gen_base, uint64_t n_seeds, int max_height, int salt, int rx0,
                     int rx1, int rz0, int rz1) {
    Request rq;
    std::memset(&rq, 0, sizeof rq);
    if (opts) rq.opts = *opts;
    rq.gen_base = gen_base;
    rq.n_seeds = n_seeds;
    rq.max_height = max_height;
    rq.salt = salt;
    rq.rx0 = rx0;
    rq.rx1 = rx1;
    rq.rz0 = rz0;
    rq.rz1 = rz1;
    return rq;
}

// Version names with a biome tree (the reference's biome_trees.h version table): tree
// index, 1.18 rules, pre-26.2 rules.
struct VersionName {
    const char *name;
    int tree, is_118, pre_262;
};
const VersionName kVersions[] = {
    {"1.18", 0, 1, 1},   {"1.18.1", 0, 1, 1},  {"1.18.2", 0, 1, 1},  {"1.19", 1, 0, 1},    {"1.19.2", 1, 0, 1},
    {"1.19.3", 2, 0, 1}, {"1.19.4", 2, 0, 1},  {"1.20", 3, 0, 1},    {"1.20.1", 3, 0, 1},  {"1.20.2", 3, 0, 1},
    {"1.20.4", 3, 0, 1}, {"1.20.5", 3, 0, 1},  {"1.20.6", 3, 0, 1},  {"1.21", 3, 0, 1},    {"1.21.1", 3, 0, 1},
    {"1.21.2", 3, 0, 1}, {"1.21.3", 3, 0, 1},  {"1.21.4", 4, 0, 1},  {"1.21.5", 5, 0, 1},  {"1.21.8", 5, 0, 1},
    {"1.21.11", 5, 0, 1}, {"26.1", 5, 0, 1},   {"26.2", 6, 0, 0},    {"26.3", 7, 0, 0},
};

}  // namespace

extern "C" {

int wg_parse_version(const char *s, wg_opts *o) {
    if (!s || !o) return WG_ERR_ARG;
    for (const VersionName &v : kVersions)
        if (!std::strcmp(v.name, s)) {
            o->mc_1_18_2 = v.is_118;
            o->pre_26_2 = v.pre_262;
            o->biome_tree = v.tree + 1;
            return WG_OK;
        }
    static const char *v118[] = {"1.18.x", nullptr};
    static const char *vpre[] = {"1.19.x", "1.20.x", "1.21.x~26.1", "1.21.5~26.1", "1.19.x~26.1", nullptr};
    for (int i = 0; v118[i]; i++)
        if (!std::strcmp(s, v118[i])) { o->mc_1_18_2 = 1; o->pre_26_2 = 1; return WG_OK; }
    for (int i = 0; vpre[i]; i++)
        if (!std::strcmp(s, vpre[i])) { o->mc_1_18_2 = 0; o->pre_26_2 = 1; return WG_OK; }
    if (!std::strcmp(s, "26.2~26.3")) { o->mc_1_18_2 = 0; o->pre_26_2 = 0; return WG_OK; }
    return WG_ERR_ARG;
}

int wg_parse_preset(const char *s, wg_opts *o) {
    if (!s || !o) return WG_ERR_ARG;
    if (!std::strcmp(s, "NORMAL")) return WG_OK;
    if (!std::strcmp(s, "LARGE_BIOMES")) { o->large_biomes = 1; return WG_OK; }
    if (!std::strcmp(s, "SINGLE_BIOME")) { o->single_biome = 1; return WG_OK; }
    return WG_ERR_ARG;
}

int wg_engine_open(int device, wg_engine **out) {
    if (!out) return WG_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0 || device < 0 || device >= ndev) return WG_ERR_NODEV;
    wg_engine *eng = new (std::nothrow) wg_engine();
    if (!eng) return WG_ERR_NOMEM;
    eng->device = device;
    int rc = [&]() -> int {
        WG_CUDA(cudaSetDevice(device), "cudaSetDevice");
        WG_CUDA(cudaDeviceGetAttribute(&eng->sm_count, cudaDevAttrMultiProcessorCount, device), "device attr");
        WG_CUDA(cudaStreamCreateWithFlags(&eng->stream, cudaStreamNonBlocking), "stream");
        WG_CUDA(cudaEventCreate(&eng->ev0), "event");
        WG_CUDA(cudaEventCreate(&eng->ev1), "event");
        WG_CUDA(cudaStreamCreateWithFlags(&eng->copy_stream, cudaStreamNonBlocking), "stream");
        WG_CUDA(cudaEventCreateWithFlags(&eng->ev_up, cudaEventDisableTiming), "event");
        for (int k = 0; k < 4; k++) WG_CUDA(cudaEventCreate(&eng->kev[k]), "event");
        upload_phase1_tables();
        WG_CUDA(cudaGetLastError(), "upload tables");
        WG_CUDA(cudaMalloc(&eng->rec_unit, sizeof(uint32_t) * kCapRec), "alloc");
        WG_CUDA(cudaMalloc(&eng->rec_off, sizeof(uint32_t) * kCapRec), "alloc");
        WG_CUDA(cudaMalloc(&eng->rec_cnt, sizeof(uint32_t) * kCapRec), "alloc");
        WG_CUDA(cudaMalloc(&eng->surv, sizeof(uint32_t) * kCapSurv), "alloc");
        WG_CUDA(cudaMalloc(&eng->deep, sizeof(uint32_t) * 2 * kCapDeep), "alloc");
        WG_CUDA(cudaMalloc(&eng->out, sizeof(Candidate) * kCapOut), "alloc");
        WG_CUDA(cudaMalloc(&eng->counters, sizeof(uint32_t) * CNT_WORDS), "alloc");
        WG_CUDA(cudaMalloc(&eng->hist, sizeof(unsigned long long) * (P1_KINDS + kTiers)), "alloc");
        WG_CUDA(cudaMallocHost(&eng->h_counters, sizeof(uint32_t) * CNT_WORDS), "alloc");
        WG_CUDA(cudaMallocHost(&eng->h_hist, sizeof(unsigned long long) * (P1_KINDS + kTiers)), "alloc");
        return WG_OK;
    }();
    if (rc) {
        wg_engine_close(eng);
        return rc;
    }
    *out = eng;
    return WG_OK;
}

void wg_engine_close(wg_engine *eng) {
    if (!eng) return;
    cudaSetDevice(eng->device);
    if (eng->stream) cudaStreamSynchronize(eng->stream);
    cudaFree(eng->rec_unit);
    cudaFree(eng->rec_off);
    cudaFree(eng->rec_cnt);
    cudaFree(eng->surv);
    cudaFree(eng->deep);
    cudaFree(eng->out);
    cudaFree(eng->counters);
    cudaFree(eng->hist);
    cudaFree(eng->d_seed_list);
    cudaFree(eng->spot_items[0]);
    cudaFree(eng->spot_items[1]);
    cudaFree(eng->spot_counts);
    p2_release(eng);
    solve_release(eng);
    walk_release(eng);
    queue_release(eng);
    finish_release(eng);
    cudaFreeHost(eng->h_counters);
    cudaFreeHost(eng->h_hist);
    if (eng->ev0) cudaEventDestroy(eng->ev0);
    if (eng->ev1) cudaEventDestroy(eng->ev1);
    for (int k = 0; k < 4; k++)
        if (eng->kev[k]) cudaEventDestroy(eng->kev[k]);
    if (eng->ev_up) cudaEventDestroy(eng->ev_up);
    if (eng->copy_stream) cudaStreamDestroy(eng->copy_stream);
    if (eng->stream) cudaStreamDestroy(eng->stream);
    delete eng;
}

const char *wg_engine_error(const wg_engine *eng) { return eng ? eng->err.c_str() : "no engine"; }

// wg_noise_probe / wg_noise_probe_3d: dims = 2 (x, z points, y = 0 climate noises) or 3 (x, y, z
// points, the entrance kernel's cave noises).
static int noise_probe(wg_engine *eng, const int64_t *seeds, uint64_t n_seeds, int noise, const double *pts,
                       uint64_t n_points, double *out32, double *out64, int dims) {
    const bool ok_noise = dims == 2 ? (noise >= 0 && noise <= N_CONTINENTALNESS_LARGE)
                                    : (noise >= N_CAVE_ENTRANCE && noise <= N_ROUGHNESS);
    if (!eng || !seeds || !pts || !out32 || !out64 || n_seeds == 0 || n_points == 0 || !ok_noise ||
        n_seeds > (1u << 20) || n_points > (1u << 20) || n_seeds * n_points > (1ull << 26))
        return eng ? eng->fail(WG_ERR_ARG, "noise probe: bad noise id or sizes") : WG_ERR_ARG;
    WG_CUDA(cudaSetDevice(eng->device), "cudaSetDevice");
    int64_t *d_seeds = nullptr;
    double *d_pts = nullptr, *d_out = nullptr;
    const size_t n_out = (size_t)(n_seeds * n_points);
    int rc = [&]() -> int {
        WG_CUDA(cudaMalloc(&d_seeds, sizeof(int64_t) * n_seeds), "alloc");
        WG_CUDA(cudaMalloc(&d_pts, sizeof(double) * dims * n_points), "alloc");
        WG_CUDA(cudaMalloc(&d_out, sizeof(double) * 2 * n_out), "alloc");
        WG_CUDA(cudaMemcpyAsync(d_seeds, seeds, sizeof(int64_t) * n_seeds, cudaMemcpyHostToDevice, eng->stream),
                "copy");
        WG_CUDA(cudaMemcpyAsync(d_pts, pts, sizeof(double) * dims * n_points, cudaMemcpyHostToDevice, eng->stream),
                "copy");
        if (dims == 2)
            launch_noise_probe(d_seeds, (uint32_t)n_seeds, noise, d_pts, (uint32_t)n_points, d_out, d_out + n_out,
                               eng->stream);
        else
            launch_noise_probe3d(d_seeds, (uint32_t)n_seeds, noise, d_pts, (uint32_t)n_points, d_out, d_out + n_out,
                                 eng->stream);
        WG_CUDA(cudaGetLastError(), "noise probe launch");
        WG_CUDA(cudaMemcpyAsync(out32, d_out, sizeof(double) * n_out, cudaMemcpyDeviceToHost, eng->stream), "copy");
        WG_CUDA(cudaMemcpyAsync(out64, d_out + n_out, sizeof(double) * n_out, cudaMemcpyDeviceToHost, eng->stream),
                "copy");
        WG_CUDA(cudaStreamSynchronize(eng->stream), "noise probe");
        return WG_OK;
    }();
    cudaFree(d_seeds);
    cudaFree(d_pts);
    cudaFree(d_out);
    return rc;
}

int wg_noise_probe(wg_engine *eng, const int64_t *seeds, uint64_t n_seeds, int noise, const double *xz,
                   uint64_t n_points, double *out32, double *out64) {
    return noise_probe(eng, seeds, n_seeds, noise, xz, n_points, out32, out64, 2);
}

int wg_noise_probe_3d(wg_engine *eng, const int64_t *seeds, uint64_t n_seeds, int noise, const double *xyz,
                      uint64_t n_points, double *out32, double *out64) {
    return noise_probe(eng, seeds, n_seeds, noise, xyz, n_points, out32, out64, 3);
}

int wg_engine_set_noise_core(wg_engine *eng, int core) {
    if (!eng || (core != WG_NOISE_FP32 && core != WG_NOISE_FP64 && core != WG_NOISE_FP32_RECHECK_ALL &&
                 core != WG_NOISE_FP32_CAVES))
        return WG_ERR_ARG;
    eng->fp32_core = core == WG_NOISE_FP64 ? 0 : (core == WG_NOISE_FP32 ? 1 : (core == WG_NOISE_FP32_CAVES ? 3 : 2));
    return WG_OK;
}

int wg_seed_check(wg_engine *eng, const int64_t *seeds, uint64_t gen_base, uint64_t n_seeds, const wg_opts *opts,
                  int max_height, int salt, int rx0, int rx1, int rz0, int rz1, wg_candidate *out, uint64_t cap,
                  uint64_t *n_out, wg_scan_stats *stats) {
    if (!eng || (cap && !out)) return WG_ERR_ARG;
    auto t0 = std::chrono::steady_clock::now();
    WG_CUDA(cudaSetDevice(eng->device), "cudaSetDevice");
    Request rq = make_request(opts, gen_base, n_seeds, max_height, salt, rx0, rx1, rz0, rz1);
    // the seeds go up batch by batch, each upload overlapping the batch before it (run_request)
    int rc = reserve_seeds(eng, seeds ? n_seeds : 0);
    if (rc) return rc;
    if (seeds) {
        rq.d_seeds = eng->d_seed_list;
        rq.h_seeds = seeds;
    }
    wg_scan_stats st;
    std::memset(&st, 0, sizeof st);
    std::vector<Candidate> found;
    Sink sink;
    sink.host = &found;
    WG_CUDA(cudaEventRecord(eng->ev0, eng->stream), "event");
    rc = run_request(eng, rq, sink, st);
    if (rc) return rc;
    WG_CUDA(cudaEventRecord(eng->ev1, eng->stream), "event");
    WG_CUDA(cudaEventSynchronize(eng->ev1), "event");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, eng->ev0, eng->ev1);
    std::sort(found.begin(), found.end(), [](const Candidate &x, const Candidate &y) {
        if (x.seed_index != y.seed_index) return x.seed_index < y.seed_index;
        if (x.rz != y.rz) return x.rz < y.rz;
        return x.rx < y.rx;
    });
    uint64_t n = std::min<uint64_t>(cap, found.size());
    for (uint64_t i = 0; i < n; i++) {
        const Candidate &c = found[i];
        out[i].seed_index = c.seed_index;
        out[i].seed = c.seed;
        out[i].rx = c.rx;
        out[i].rz = c.rz;
        out[i].chunk_x = c.chunk_x;
        out[i].chunk_z = c.chunk_z;
    }
    if (n_out) *n_out = found.size();
    st.gpu_ms = ms;
    st.wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (stats) *stats = st;
    return WG_OK;
}

int wg_seed_check_device(wg_engine *eng, const int64_t *d_seeds, uint64_t gen_base, uint64_t n_seeds,
                         const wg_opts *opts, int max_height, int salt, int rx0, int rx1, int rz0, int rz1,
                         wg_candidate *d_out, uint64_t cap, uint64_t *n_out, wg_scan_stats *stats, void *stream) {
    if (!eng || (cap && !d_out)) return WG_ERR_ARG;
    static_assert(sizeof(wg_candidate) == sizeof(Candidate), "candidate layout");
    auto t0 = std::chrono::steady_clock::now();
    WG_CUDA(cudaSetDevice(eng->device), "cudaSetDevice");
    // Run on the caller's stream for this call, so the caller's events bracket the work.
    struct StreamSwap {
        wg_engine *e;
        cudaStream_t saved;
        ~StreamSwap() { e->stream = saved; }
    } swap{eng, eng->stream};
    if (stream) eng->stream = (cudaStream_t)stream;
    Request rq = make_request(opts, gen_base, n_seeds, max_height, salt, rx0, rx1, rz0, rz1);
    rq.d_seeds = d_seeds;
    wg_scan_stats st;
    std::memset(&st, 0, sizeof st);
    Sink sink;
    sink.dev = reinterpret_cast<Candidate *>(d_out);
    sink.dev_cap = cap;
    WG_CUDA(cudaEventRecord(eng->ev0, eng->stream), "event");
    int rc = run_request(eng, rq, sink, st);
    if (rc) return rc;
    WG_CUDA(cudaEventRecord(eng->ev1, eng->stream), "event");
    WG_CUDA(cudaEventSynchronize(eng->ev1), "event");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, eng->ev0, eng->ev1);
    if (n_out) *n_out = sink.found;
    st.gpu_ms = ms;
    st.wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (stats) *stats = st;
    return WG_OK;
}

int wg_phase1_codes(wg_engine *eng, const int64_t *seeds, uint64_t gen_base, uint64_t n_seeds, const wg_opts *opts,
                    int max_height, int salt, int rx0, int rx1, int rz0, int rz1, int8_t *codes, int8_t *tiers) {
    if (!eng || !codes || !tiers || rx1 <= rx0 || rz1 <= rz0) return WG_ERR_ARG;
    WG_CUDA(cudaSetDevice(eng->device), "cudaSetDevice");
    const uint64_t total = n_seeds * (uint64_t)((int64_t)rx1 - rx0) * (uint64_t)((int64_t)rz1 - rz0);
    Request rq = make_request(opts, gen_base, n_seeds, max_height, salt, rx0, rx1, rz0, rz1);
    int rc = stage_seeds(eng, seeds, n_seeds, &rq.d_seeds);
    if (rc) return rc;
    int8_t *dc = nullptr, *dt = nullptr;
    WG_CUDA(cudaMalloc(&dc, total), "alloc codes");
    if (cudaMalloc(&dt, total) != cudaSuccess) {
        cudaFree(dc);
        return eng->fail(WG_ERR_NOMEM, "alloc tiers");
    }
    cudaMemsetAsync(dc, -1, total, eng->stream);
    cudaMemsetAsync(dt, -1, total, eng->stream);
    rq.d_codes = dc;
    rq.d_tiers = dt;
    wg_scan_stats st;
    std::memset(&st, 0, sizeof st);
    std::vector<Candidate> found;
    Sink sink;
    sink.host = &found;
    rc = run_request(eng, rq, sink, st);
    if (!rc) {
        cudaError_t e1 = cudaMemcpy(codes, dc, total, cudaMemcpyDeviceToHost);
        cudaError_t e2 = cudaMemcpy(tiers, dt, total, cudaMemcpyDeviceToHost);
        if (e1 != cudaSuccess || e2 != cudaSuccess) rc = eng->fail(WG_ERR_CUDA, "copy codes", e1 ? e1 : e2);
    }
    cudaFree(dc);
    cudaFree(dt);
    return rc;
}

int wg_deep_spots(wg_engine *eng, const int64_t *s48, const int32_t *chunk_x, const int32_t *chunk_z,
                  uint64_t n_spots, const wg_opts *opts, int max_height, wg_candidate *out, uint64_t cap,
                  uint64_t *n_out, uint64_t *not_start) {
    if (!eng || (n_spots && (!s48 || !chunk_x || !chunk_z)) || (cap && !out)) return WG_ERR_ARG;
    if (n_spots > (1ull << 16)) return WG_ERR_CAPACITY;   // 2^32 world seeds per call at most
    WG_CUDA(cudaSetDevice(eng->device), "cudaSetDevice");
    // keep the spots that are mineshaft start chunks (hut_lookup_v4 --spots skips the others)
    std::vector<int64_t> ks;
    std::vector<int32_t> krx, krz;
    std::vector<uint64_t> kidx;
    uint64_t bad = 0;
    for (uint64_t i = 0; i < n_spots; i++) {
        const DeepCtx c = deep_ctx((uint64_t)s48[i]);
        if (!deep_is_start(deep_carver(c, chunk_x[i], chunk_z[i]))) {
            bad++;
            continue;
        }
        ks.push_back((int64_t)c.s48);
        krx.push_back(chunk_x[i] >> 5);   // floorDiv by 32 chunks
        krz.push_back(chunk_z[i] >> 5);
        kidx.push_back(i);
    }
    if (not_start) *not_start = bad;
    if (n_out) *n_out = 0;
    if (ks.empty()) return WG_OK;
    const uint64_t nk = ks.size();
    int64_t *d_s = nullptr;
    int32_t *d_x = nullptr, *d_z = nullptr;
    cudaError_t e = cudaMalloc(&d_s, sizeof(int64_t) * nk);
    if (e == cudaSuccess) e = cudaMalloc(&d_x, sizeof(int32_t) * nk);
    if (e == cudaSuccess) e = cudaMalloc(&d_z, sizeof(int32_t) * nk);
    if (e == cudaSuccess) e = cudaMemcpy(d_s, ks.data(), sizeof(int64_t) * nk, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_x, krx.data(), sizeof(int32_t) * nk, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_z, krz.data(), sizeof(int32_t) * nk, cudaMemcpyHostToDevice);
    int rc = WG_OK;
    std::vector<Candidate> found;
    if (e != cudaSuccess) {
        rc = eng->fail(WG_ERR_CUDA, "deep spots upload", e);
    } else {
        Request rq = make_request(opts, 0, nk << 16, max_height, 0, 0, 1, 0, 1);
        rq.d_spot_s48 = d_s;
        rq.d_spot_rx = d_x;
        rq.d_spot_rz = d_z;
        wg_scan_stats st;
        std::memset(&st, 0, sizeof st);
        Sink sink;
        sink.host = &found;
        rc = run_request(eng, rq, sink, st);
    }
    cudaFree(d_s);
    cudaFree(d_x);
    cudaFree(d_z);
    if (rc) return rc;
    // survivors whose hut is the spot chunk, renumbered by the caller's spot index
    std::vector<wg_candidate> keep;
    for (const Candidate &c : found) {
        const uint64_t k = c.seed_index >> 16, u = c.seed_index & 0xFFFF;
        const uint64_t i = kidx[k];
        if (c.chunk_x != chunk_x[i] || c.chunk_z != chunk_z[i]) continue;
        wg_candidate w;
        w.seed_index = (i << 16) | u;
        w.seed = c.seed;
        w.rx = c.rx;
        w.rz = c.rz;
        w.chunk_x = c.chunk_x;
        w.chunk_z = c.chunk_z;
        keep.push_back(w);
    }
    std::sort(keep.begin(), keep.end(),
              [](const wg_candidate &x, const wg_candidate &y) { return x.seed_index < y.seed_index; });
    const uint64_t nw = std::min<uint64_t>(cap, keep.size());
    for (uint64_t i = 0; i < nw; i++) out[i] = keep[i];
    if (n_out) *n_out = keep.size();
    return WG_OK;
}

}  // extern "C"
