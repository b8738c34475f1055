// Seed Check phase 1 for callers that cannot allocate device memory.
//
// Some callers own every byte of device memory through their own allocator — a framework
// process whose caching allocator must not be bypassed, or a serving loop with a fixed memory
// budget — and some cannot afford cudaMalloc / cudaFree on their hot path, because those calls
// can synchronize the whole device and can fail under fragmentation.  wg_seed_check_noalloc
// serves them: the caller passes the seeds and the output buffer, and the work lists the three
// phase-1 kernels need (unit records, climate survivors, deep candidates, counters) live in
// one file-scope __device__ array of fixed size instead of engine-allocated buffers.
//
// The array is part of the library's device image: every GPU that loads libwitchgpu.so holds
// its kNoAllocScratchBytes until the process exits.  All calls share it and it keeps the
// previous call's contents, so each call clears the counters it relies on; two calls that run
// at the same time on the GPU (different streams or host threads) race on it.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/witchgpu.h"
#include "wg_catalog.h"
#include "wg_phase1.cuh"

using namespace wg;

namespace {

constexpr uint32_t kNaMaxSeeds = 65536;        // seeds per call
constexpr uint32_t kNaMaxRegions = 4096;       // regions per seed (one window per seed)
constexpr uint32_t kNaRecords = 1u << 17;
constexpr uint32_t kNaSurvivors = 1u << 20;
constexpr uint32_t kNaDeep = 1u << 16;

// Byte layout of the scratch array (every block starts on a 256-byte boundary).
constexpr size_t kOffCounters = 0;
constexpr size_t kOffHist = 256;
constexpr size_t kOffRecUnit = 512;
constexpr size_t kOffRecOff = kOffRecUnit + sizeof(uint32_t) * kNaRecords;
constexpr size_t kOffRecCnt = kOffRecOff + sizeof(uint32_t) * kNaRecords;
constexpr size_t kOffSurv = kOffRecCnt + sizeof(uint32_t) * kNaRecords;
constexpr size_t kOffDeep = kOffSurv + sizeof(uint32_t) * kNaSurvivors;
constexpr size_t kNoAllocScratchBytes = kOffDeep + 2 * sizeof(uint32_t) * kNaDeep;   // 6 MiB + 512 B
static_assert(kOffRecOff % 256 == 0 && kOffRecCnt % 256 == 0 && kOffSurv % 256 == 0 && kOffDeep % 256 == 0,
              "scratch blocks must stay 256-byte aligned");

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

// Per-device set-up, done by the first call on each device with that device current: the
// noise tables go to the device's constant memory and the scratch array's device address is
// looked up (host code may not use g_noalloc_scratch itself: on the host that name is only a
// stand-in symbol, not a device address).
constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned char *g_scratch_ptr[kMaxDevices] = {};
int g_sm_count[kMaxDevices] = {};

int setup_device(int dev) {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (g_scratch_ptr[dev]) return WG_OK;
    upload_phase1_tables();
    if (cudaGetLastError() != cudaSuccess) return WG_ERR_CUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return WG_ERR_CUDA;
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return WG_ERR_CUDA;
    g_sm_count[dev] = sms;
    g_scratch_ptr[dev] = static_cast<unsigned char *>(p);
    return WG_OK;
}

}  // namespace

extern "C" int wg_seed_check_noalloc(const int64_t *d_seeds, uint64_t gen_base, uint32_t n_seeds,
                                     const wg_opts *opts, int max_height, int salt, int rx0, int rx1, int rz0,
                                     int rz1, wg_candidate *d_out, uint32_t cap, uint32_t *n_out, void *stream) {
    if (!n_out || (cap && !d_out) || n_seeds == 0 || rx1 <= rx0 || rz1 <= rz0) return WG_ERR_ARG;
    const uint64_t rw = (uint64_t)((int64_t)rx1 - rx0), rh = (uint64_t)((int64_t)rz1 - rz0);
    if (n_seeds > kNaMaxSeeds || rw * rh > kNaMaxRegions) return WG_ERR_CAPACITY;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return WG_ERR_NODEV;
    if (dev < 0 || dev >= kMaxDevices) return WG_ERR_NODEV;
    int rc = setup_device(dev);
    if (rc) return rc;
    unsigned char *base = g_scratch_ptr[dev];
    cudaStream_t s = (cudaStream_t)stream;

    BatchArgs a{};
    a.seeds = d_seeds;
    a.gen_base = gen_base;
    a.unit0 = 0;
    a.n_units = n_seeds;
    a.win = (uint32_t)(rw * rh);
    a.n_win = 1;
    a.n_regions = rw * rh;
    a.rx0 = rx0;
    a.rz0 = rz0;
    a.rw = (int)rw;
    a.rh = (int)rh;
    a.salt = salt ? salt : 14357620;
    a.max_height = max_height;
    if (opts) {
        a.mc_1_18_2 = opts->mc_1_18_2;
        a.pre_26_2 = opts->pre_26_2;
        a.single_biome = opts->single_biome;
        a.large_biomes = opts->large_biomes;
    }
    a.fp32_core = 1;   // the engine's default noise core
    a.small_coords = coords_small(std::min(rx0, rz0), std::max(rx1, rz1) - 1ll) ? 1 : 0;
    a.counters = reinterpret_cast<uint32_t *>(base + kOffCounters);
    a.hist = reinterpret_cast<unsigned long long *>(base + kOffHist);
    a.rec_unit = reinterpret_cast<uint32_t *>(base + kOffRecUnit);
    a.rec_off = reinterpret_cast<uint32_t *>(base + kOffRecOff);
    a.rec_cnt = reinterpret_cast<uint32_t *>(base + kOffRecCnt);
    a.surv_region = reinterpret_cast<uint32_t *>(base + kOffSurv);
    a.deep = reinterpret_cast<uint32_t *>(base + kOffDeep);
    a.out = reinterpret_cast<Candidate *>(d_out);
    a.cap_rec = kNaRecords;
    a.cap_surv = kNaSurvivors;
    a.cap_deep = kNaDeep;
    a.cap_out = cap;

    // The array still holds the previous call's lists; only the counters and the funnel must
    // start from zero (the lists are written before they are read).
    if (cudaMemsetAsync(base, 0, kOffRecUnit, s) != cudaSuccess) return WG_ERR_CUDA;
    launch_climate(a, s);
    launch_entrance(a, g_sm_count[dev] * 2, s);
    launch_ladder(a, 0, s);
    if (cudaGetLastError() != cudaSuccess) return WG_ERR_CUDA;
    uint32_t counters[CNT_WORDS];
    if (cudaMemcpyAsync(counters, a.counters, sizeof counters, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return WG_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return WG_ERR_CUDA;
    if (counters[CNT_OVERFLOW] & 3u) return WG_ERR_CAPACITY;   // a scratch list was full
    *n_out = counters[CNT_FINAL];                               // may exceed cap: only cap written
    return WG_OK;
}
