// Deep Dive region walk (wg_deep_starts): for structure seeds x a region rect, the swamp-hut chunk
// of every region and whether a mineshaft starts in it (the forward direction of the reference's
// room walker, engine/gpu/room_core.h:146-175).  Integer LCG work only: one thread walks a strip
// of 64 regions along rx.  The hits come out in (seed, rz, rx) order without a sort: a counting
// pass, a prefix over the block totals, and a writing pass that walks again and stores each hit
// at its place.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/witchgpu.h"
#include "wg_deep.cuh"
#include "wg_device.cuh"
#include "wg_engine_impl.h"

using namespace wg;

namespace {

struct DeepHit {
    uint64_t seed_index;
    int64_t s48;
    int32_t rx, rz, chunk_x, chunk_z;
    int64_t carver;
};
static_assert(sizeof(DeepHit) == sizeof(wg_deep_start), "deep start layout");

constexpr int kDeepThreads = 256;
constexpr int kDeepCols = 64;                     // rx columns one thread walks
constexpr uint64_t kDeepPassTasks = 1ull << 24;   // tasks per pass: 65,536 blocks

// Task t = (seed i, row rz, strip of kDeepCols columns), strips fastest, so that walking the
// tasks in order and each strip along rx visits the regions in the output order (seed, rz, rx).
struct WalkGeom {
    const int64_t *s48s;
    uint64_t s48_base, n_seeds;
    int rx0, rw, rz0, rh, strips;
};

template <class F>
__device__ __forceinline__ void walk_task(const WalkGeom &G, uint64_t t, F &&on_start) {
    const int strip = (int)(t % (uint64_t)G.strips);
    const uint64_t rest = t / (uint64_t)G.strips;
    const int row = (int)(rest % (uint64_t)G.rh);
    const uint64_t i = rest / (uint64_t)G.rh;
    if (i >= G.n_seeds) return;
    const uint64_t s48 = (G.s48s ? (uint64_t)G.s48s[i] : G.s48_base + i) & kDeepMask48;
    const DeepCtx c = deep_ctx(s48);
    const int rz = G.rz0 + row;
    const int xa = G.rx0 + strip * kDeepCols, xb = min(G.rx0 + G.rw, xa + kDeepCols);
    for (int rx = xa; rx < xb; rx++) {
        int cx, cz;
        hut_chunk(s48, rx, rz, 14357620, cx, cz);
        const uint64_t carver = deep_carver(c, cx, cz);
        if (deep_is_start(carver)) on_start(i, s48, rx, rz, cx, cz, carver);
    }
}

// Pass 1: each task's number of starts (at most kDeepCols, one byte) and each block's total.
__global__ void __launch_bounds__(kDeepThreads) walk_count_kernel(WalkGeom G, uint64_t t0, uint64_t n_tasks,
                                                                  uint8_t *__restrict__ counts,
                                                                  uint32_t *__restrict__ block_sums) {
    const uint64_t k = (uint64_t)blockIdx.x * kDeepThreads + threadIdx.x;
    uint32_t n = 0;
    if (k < n_tasks) {
        walk_task(G, t0 + k, [&](uint64_t, uint64_t, int, int, int, int, uint64_t) { n++; });
        counts[k] = (uint8_t)n;
    }
    const uint32_t w = __reduce_add_sync(0xFFFFFFFFu, n);
    __shared__ uint32_t warp_sums[kDeepThreads / 32];
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x / 32] = w;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t tot = 0;
        for (int q = 0; q < kDeepThreads / 32; q++) tot += warp_sums[q];
        block_sums[blockIdx.x] = tot;
    }
}

// Pass 2 (one block): exclusive prefix of the block totals on top of the starts of earlier passes
// (*total), which it then advances.
__global__ void __launch_bounds__(1024) walk_scan_kernel(const uint32_t *__restrict__ block_sums, uint32_t n_blocks,
                                                         uint64_t *__restrict__ block_base,
                                                         unsigned long long *__restrict__ total) {
    __shared__ unsigned long long part[1024];
    const uint32_t per = (n_blocks + 1023) / 1024, b0 = threadIdx.x * per, b1 = min(n_blocks, b0 + per);
    unsigned long long s = 0;
    for (uint32_t b = b0; b < b1; b++) s += block_sums[b];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1) {   // inclusive scan of the 1,024 partial sums
        const unsigned long long v = threadIdx.x >= (unsigned)d ? part[threadIdx.x - d] : 0ull;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    unsigned long long base = *total + part[threadIdx.x] - s;
    for (uint32_t b = b0; b < b1; b++) {
        block_base[b] = base;
        base += block_sums[b];
    }
    __syncthreads();
    if (threadIdx.x == 1023) *total += part[1023];
}

// Pass 3: each task writes its starts at its place in the output order (those past cap are
// counted but not written).
__global__ void __launch_bounds__(kDeepThreads) walk_write_kernel(WalkGeom G, uint64_t t0, uint64_t n_tasks,
                                                                  const uint8_t *__restrict__ counts,
                                                                  const uint64_t *__restrict__ block_base,
                                                                  DeepHit *__restrict__ out, uint64_t cap) {
    const uint64_t k = (uint64_t)blockIdx.x * kDeepThreads + threadIdx.x;
    const uint32_t n = k < n_tasks ? counts[k] : 0u;
    // exclusive prefix of n within the block
    const int lane = threadIdx.x & 31, wid = threadIdx.x / 32;
    uint32_t incl = n;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (lane >= d) incl += v;
    }
    __shared__ uint32_t warp_sums[kDeepThreads / 32];
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    uint32_t before = 0;
    for (int q = 0; q < wid; q++) before += warp_sums[q];
    if (!n) return;
    uint64_t at = block_base[blockIdx.x] + before + incl - n;
    walk_task(G, t0 + k, [&](uint64_t i, uint64_t s48, int rx, int rz, int cx, int cz, uint64_t carver) {
        if (at < cap) out[at] = DeepHit{i, (int64_t)s48, rx, rz, cx, cz, (int64_t)carver};
        at++;
    });
}

// ------------------------------------------------------------------------------------
// Forward sweep with the layout-catalogue probe (wg_deep_sweep): every region of the rect for every
// structure seed, its hut chunk, the start test, and for each start whether its carver state is a
// catalogued layout (the reference's forward mode, engine/gpu/hut_lookup_v4_source.cu:77-99 and
// :1504-1530).  A thread walks one rx column over kSweepRows rows of rz, stepping the region seed
// and the carver's z term by constants per row instead of recomputing them.
// ------------------------------------------------------------------------------------
constexpr int kSweepRows = 64;
constexpr uint64_t kSweepPassTasks = 1ull << 24;
constexpr uint64_t kRegionMulX = 341873128712ull, kRegionMulZ = 132897987541ull;
constexpr uint32_t kHutDrawLimit = 2147483640u;   // nextInt(24) re-draws a 31-bit value at or above this
constexpr uint64_t kStartHiBound = 268435;        // floor(0.004 * 2^53 / 2^27): the start test's first draw

struct SweepMatch {
    uint64_t seed_index;
    int64_t s48;
    int32_t rx, rz, chunk_x, chunk_z;
    int64_t carver;
    uint32_t value, pad;
};
static_assert(sizeof(SweepMatch) == sizeof(wg_sweep_match), "sweep match layout");

struct SweepGeom {
    const int64_t *s48s;
    uint64_t s48_base, n_seeds;
    int rx0, rw, rz0, rh, segs;          // segs: row segments of kSweepRows per column
    const uint64_t *keys;                // catalogued layouts, sorted ascending
    const uint32_t *vals;
    uint32_t n_keys;
};

// Index of carver in the sorted catalogue, or -1.
__device__ __forceinline__ int catalogue_find(const SweepGeom &G, uint64_t carver) {
    uint32_t lo = 0, hi = G.n_keys;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (G.keys[mid] < carver) lo = mid + 1;
        else hi = mid;
    }
    return (lo < G.n_keys && G.keys[lo] == carver) ? (int)lo : -1;
}

// nextInt(24) of a java.util.Random state right after setSeed: the state after the draw, the value
// in v; false when the 31-bit draw falls in the re-draw range (the caller takes the exact path).
__device__ __forceinline__ bool draw24(uint64_t &st, int &v) {
    st = deep_step(st);
    const uint32_t u = (uint32_t)(st >> 17);
    v = (int)(u % 24u);
    return u < kHutDrawLimit;
}

__global__ void __launch_bounds__(kDeepThreads) sweep_kernel(SweepGeom G, uint64_t t0, uint64_t n_tasks,
                                                             unsigned long long *__restrict__ starts,
                                                             SweepMatch *__restrict__ out,
                                                             unsigned long long *__restrict__ n_out, uint64_t cap) {
    const uint64_t k = (uint64_t)blockIdx.x * kDeepThreads + threadIdx.x;
    uint32_t n_starts = 0;
    uint64_t i = 0;
    if (k < n_tasks) {
        const uint64_t t = t0 + k;
        const int col = (int)(t % (uint64_t)G.rw);
        const uint64_t rest = t / (uint64_t)G.rw;
        const int seg = (int)(rest % (uint64_t)G.segs);
        i = rest / (uint64_t)G.segs;
        const uint64_t s48 = (G.s48s ? (uint64_t)G.s48s[i] : G.s48_base + i) & kDeepMask48;
        const DeepCtx c = deep_ctx(s48);
        const int rx = G.rx0 + col;
        const int za = G.rz0 + seg * kSweepRows, zb = min(G.rz0 + G.rh, za + kSweepRows);
        // region seed (low 48 bits suffice: setSeed masks to 48 bits) and the carver's row terms
        uint64_t rs = (uint64_t)(int64_t)rx * kRegionMulX + (uint64_t)(int64_t)za * kRegionMulZ + s48 + 14357620ull;
        const uint64_t px = (uint64_t)((int64_t)rx * 32) * (uint64_t)c.a;
        uint64_t pz = (uint64_t)((int64_t)za * 32) * (uint64_t)c.b;
#pragma unroll 4   // rows are independent apart from the two running sums: four in flight (4 structure seeds over the whole world: 156.5 vs 159.9 ms)
        for (int rz = za; rz < zb; rz++) {
            uint64_t st = (rs ^ kDeepMul) & kDeepMask48;
            int j, m;
            const bool ok1 = draw24(st, j), ok2 = draw24(st, m);
            int cx = rx * 32 + j, cz = rz * 32 + m;
            uint64_t carver;
            if (ok1 && ok2) {
                carver = ((px + (uint64_t)(int64_t)j * (uint64_t)c.a) ^ (pz + (uint64_t)(int64_t)m * (uint64_t)c.b) ^ s48) &
                         kDeepMask48;
            } else {   // a re-draw: the exact placement
                hut_chunk(s48, rx, rz, 14357620, cx, cz);
                carver = deep_carver(c, cx, cz);
            }
            const uint64_t s1 = deep_step((carver ^ kDeepMul) & kDeepMask48);
            const uint64_t hi = s1 >> 22;
            const bool start = hi < kStartHiBound || (hi == kStartHiBound && deep_is_start(carver));
            if (start) {
                n_starts++;
                const int at = catalogue_find(G, carver);
                if (at >= 0) {
                    const unsigned long long slot = atomicAdd(n_out, 1ull);
                    if (slot < cap) out[slot] = SweepMatch{i, (int64_t)s48, rx, rz, cx, cz, (int64_t)carver, G.vals[at], 0u};
                }
            }
            rs += kRegionMulZ;
            pz += 32ull * (uint64_t)c.b;
        }
    }
    // starts per structure seed: one warp sum when the warp's lanes share a seed (lanes past the
    // tasks count nothing); a warp that straddles two seeds adds lane by lane
    const uint64_t i0 = __shfl_sync(0xFFFFFFFFu, i, 0);
    if (__all_sync(0xFFFFFFFFu, k >= n_tasks || i == i0)) {
        const uint32_t tot = __reduce_add_sync(0xFFFFFFFFu, n_starts);
        if ((threadIdx.x & 31) == 0 && tot) atomicAdd(&starts[i0], (unsigned long long)tot);
    } else if (k < n_tasks && n_starts) {
        atomicAdd(&starts[i], (unsigned long long)n_starts);
    }
}

#define DEEP_CUDA(call, what)                                           \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) return eng->fail(WG_ERR_CUDA, what, e_); \
    } while (0)

}  // namespace

struct WalkState {
    int64_t *s48 = nullptr;
    DeepHit *out = nullptr;
    uint8_t *counts = nullptr;
    uint32_t *block_sums = nullptr;
    uint64_t *block_base = nullptr;
    unsigned long long *total = nullptr;
    uint64_t cap_s48 = 0, cap_out = 0;
    // forward sweep: catalogue, per-seed start counts, matches
    uint64_t *keys = nullptr;
    uint32_t *vals = nullptr;
    unsigned long long *starts = nullptr, *n_match = nullptr;
    SweepMatch *match = nullptr;
    uint64_t cap_keys = 0, cap_starts = 0;
};

void walk_release(wg_engine *eng) {
    WalkState *w = eng->walk;
    if (!w) return;
    cudaFree(w->s48);
    cudaFree(w->out);
    cudaFree(w->counts);
    cudaFree(w->block_sums);
    cudaFree(w->block_base);
    cudaFree(w->total);
    cudaFree(w->keys);
    cudaFree(w->vals);
    cudaFree(w->starts);
    cudaFree(w->n_match);
    cudaFree(w->match);
    delete w;
    eng->walk = nullptr;
}

namespace {
constexpr uint64_t kSweepMatchCap = 1u << 20;

int walk_state(wg_engine *eng) {
    if (eng->walk) return WG_OK;
    eng->walk = new (std::nothrow) WalkState();
    if (!eng->walk) return eng->fail(WG_ERR_NOMEM, "deep walk state");
    WalkState &w0 = *eng->walk;
    DEEP_CUDA(cudaMalloc(&w0.counts, kDeepPassTasks), "deep starts buffers");
    DEEP_CUDA(cudaMalloc(&w0.block_sums, sizeof(uint32_t) * (kDeepPassTasks / kDeepThreads)), "deep starts buffers");
    DEEP_CUDA(cudaMalloc(&w0.block_base, sizeof(uint64_t) * (kDeepPassTasks / kDeepThreads)), "deep starts buffers");
    DEEP_CUDA(cudaMalloc(&w0.total, sizeof(unsigned long long)), "deep starts buffers");
    return WG_OK;
}

int upload_seeds(wg_engine *eng, WalkState &w, const int64_t *s48, uint64_t n) {
    if (!s48) return WG_OK;
    if (n > w.cap_s48) {
        cudaFree(w.s48);
        w.s48 = nullptr;
        w.cap_s48 = 0;
        DEEP_CUDA(cudaMalloc(&w.s48, sizeof(int64_t) * n), "deep seeds");
        w.cap_s48 = n;
    }
    DEEP_CUDA(cudaMemcpyAsync(w.s48, s48, sizeof(int64_t) * n, cudaMemcpyHostToDevice, eng->stream), "upload seeds");
    return WG_OK;
}
}  // namespace

extern "C" int wg_deep_sweep(wg_engine *eng, const uint64_t *layouts, const uint32_t *values, uint64_t n_layouts,
                             const int64_t *s48, int64_t s48_base, uint64_t n, int rx0, int rx1, int rz0, int rz1,
                             wg_sweep_match *out, uint64_t cap, uint64_t *n_out, uint64_t *starts) {
    if (!eng || !layouts || n_layouts == 0 || n_layouts > (1u << 24) || rx1 <= rx0 || rz1 <= rz0 || n == 0 ||
        (cap && !out))
        return eng ? eng->fail(WG_ERR_ARG, "deep sweep: bad arguments") : WG_ERR_ARG;
    const int64_t rw = (int64_t)rx1 - rx0, rh = (int64_t)rz1 - rz0;
    if (rw > (1 << 24) || rh > (1 << 24) || n > (1u << 24)) return eng->fail(WG_ERR_ARG, "deep sweep: rect or seed count too large");
    DEEP_CUDA(cudaSetDevice(eng->device), "cudaSetDevice");
    int rc = walk_state(eng);
    if (rc) return rc;
    WalkState &w = *eng->walk;
    cudaStream_t st = eng->stream;
    // the catalogue, sorted by layout (values follow), duplicates keep their first value
    std::vector<std::pair<uint64_t, uint32_t>> cat(n_layouts);
    for (uint64_t q = 0; q < n_layouts; q++) cat[q] = {layouts[q] & kDeepMask48, values ? values[q] : 0u};
    std::stable_sort(cat.begin(), cat.end(), [](const auto &x, const auto &y) { return x.first < y.first; });
    cat.erase(std::unique(cat.begin(), cat.end(), [](const auto &x, const auto &y) { return x.first == y.first; }),
              cat.end());
    std::vector<uint64_t> keys(cat.size());
    std::vector<uint32_t> vals(cat.size());
    for (size_t q = 0; q < cat.size(); q++) {
        keys[q] = cat[q].first;
        vals[q] = cat[q].second;
    }
    if (keys.size() > w.cap_keys) {
        cudaFree(w.keys);
        cudaFree(w.vals);
        w.keys = nullptr;
        w.vals = nullptr;
        w.cap_keys = 0;
        DEEP_CUDA(cudaMalloc(&w.keys, sizeof(uint64_t) * keys.size()), "sweep catalogue");
        DEEP_CUDA(cudaMalloc(&w.vals, sizeof(uint32_t) * keys.size()), "sweep catalogue");
        w.cap_keys = keys.size();
    }
    if (n > w.cap_starts) {
        cudaFree(w.starts);
        w.starts = nullptr;
        w.cap_starts = 0;
        DEEP_CUDA(cudaMalloc(&w.starts, sizeof(unsigned long long) * n), "sweep start counts");
        w.cap_starts = n;
    }
    if (!w.match) {
        DEEP_CUDA(cudaMalloc(&w.match, sizeof(SweepMatch) * kSweepMatchCap), "sweep matches");
        DEEP_CUDA(cudaMalloc(&w.n_match, sizeof(unsigned long long)), "sweep matches");
    }
    DEEP_CUDA(cudaMemcpyAsync(w.keys, keys.data(), sizeof(uint64_t) * keys.size(), cudaMemcpyHostToDevice, st), "upload");
    DEEP_CUDA(cudaMemcpyAsync(w.vals, vals.data(), sizeof(uint32_t) * vals.size(), cudaMemcpyHostToDevice, st), "upload");
    rc = upload_seeds(eng, w, s48, n);
    if (rc) return rc;
    DEEP_CUDA(cudaMemsetAsync(w.starts, 0, sizeof(unsigned long long) * n, st), "memset");
    DEEP_CUDA(cudaMemsetAsync(w.n_match, 0, sizeof(unsigned long long), st), "memset");
    SweepGeom G;
    G.s48s = s48 ? w.s48 : nullptr;
    G.s48_base = (uint64_t)s48_base;
    G.n_seeds = n;
    G.rx0 = rx0;
    G.rw = (int)rw;
    G.rz0 = rz0;
    G.rh = (int)rh;
    G.segs = (int)((rh + kSweepRows - 1) / kSweepRows);
    G.keys = w.keys;
    G.vals = w.vals;
    G.n_keys = (uint32_t)keys.size();
    const uint64_t n_tasks = n * (uint64_t)G.segs * (uint64_t)G.rw;
    for (uint64_t t0 = 0; t0 < n_tasks; t0 += kSweepPassTasks) {
        const uint64_t m = std::min<uint64_t>(kSweepPassTasks, n_tasks - t0);
        sweep_kernel<<<(uint32_t)((m + kDeepThreads - 1) / kDeepThreads), kDeepThreads, 0, st>>>(
            G, t0, m, w.starts, w.match, w.n_match, kSweepMatchCap);
        DEEP_CUDA(cudaGetLastError(), "deep sweep launch");
    }
    unsigned long long found = 0;
    DEEP_CUDA(cudaMemcpyAsync(&found, w.n_match, sizeof(found), cudaMemcpyDeviceToHost, st), "read count");
    std::vector<unsigned long long> st_counts(starts ? n : 0);
    if (starts)
        DEEP_CUDA(cudaMemcpyAsync(st_counts.data(), w.starts, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost, st),
                  "read starts");
    DEEP_CUDA(cudaStreamSynchronize(st), "deep sweep");
    if (found > kSweepMatchCap) return eng->fail(WG_ERR_CAPACITY, "deep sweep: more than 2^20 catalogue matches in one call");
    std::vector<SweepMatch> m(found);
    if (found) DEEP_CUDA(cudaMemcpy(m.data(), w.match, sizeof(SweepMatch) * found, cudaMemcpyDeviceToHost), "copy matches");
    std::sort(m.begin(), m.end(), [](const SweepMatch &x, const SweepMatch &y) {
        return x.seed_index != y.seed_index ? x.seed_index < y.seed_index : (x.rz != y.rz ? x.rz < y.rz : x.rx < y.rx);
    });
    const uint64_t nw = std::min<uint64_t>(cap, found);
    if (nw) std::memcpy(out, m.data(), sizeof(SweepMatch) * nw);
    if (n_out) *n_out = found;
    for (uint64_t q = 0; q < (starts ? n : 0); q++) starts[q] = st_counts[q];
    return WG_OK;
}

extern "C" int wg_deep_starts(wg_engine *eng, const int64_t *s48, int64_t s48_base, uint64_t n, int rx0, int rx1,
                              int rz0, int rz1, wg_deep_start *out, uint64_t cap, uint64_t *n_out) {
    if (!eng || rx1 <= rx0 || rz1 <= rz0 || n == 0 || (cap && !out)) return WG_ERR_ARG;
    const int64_t rw = (int64_t)rx1 - rx0, rh = (int64_t)rz1 - rz0;
    if (rw > (1 << 24) || rh > (1 << 24)) return WG_ERR_ARG;
    DEEP_CUDA(cudaSetDevice(eng->device), "cudaSetDevice");
    if (!eng->walk) {
        eng->walk = new (std::nothrow) WalkState();
        if (!eng->walk) return eng->fail(WG_ERR_NOMEM, "deep starts state");
        WalkState &w0 = *eng->walk;
        DEEP_CUDA(cudaMalloc(&w0.counts, kDeepPassTasks), "deep starts buffers");
        DEEP_CUDA(cudaMalloc(&w0.block_sums, sizeof(uint32_t) * (kDeepPassTasks / kDeepThreads)), "deep starts buffers");
        DEEP_CUDA(cudaMalloc(&w0.block_base, sizeof(uint64_t) * (kDeepPassTasks / kDeepThreads)), "deep starts buffers");
        DEEP_CUDA(cudaMalloc(&w0.total, sizeof(unsigned long long)), "deep starts buffers");
    }
    WalkState &w = *eng->walk;
    // the device hit list holds the first cap starts of the output order (at least one slot)
    const uint64_t dcap = std::min<uint64_t>(std::max<uint64_t>(cap, 1), 1u << 24);
    if (dcap > w.cap_out) {
        cudaFree(w.out);
        w.out = nullptr;
        w.cap_out = 0;
        DEEP_CUDA(cudaMalloc(&w.out, sizeof(DeepHit) * dcap), "deep starts hit list");
        w.cap_out = dcap;
    }
    if (s48 && n > w.cap_s48) {
        cudaFree(w.s48);
        w.s48 = nullptr;
        w.cap_s48 = 0;
        DEEP_CUDA(cudaMalloc(&w.s48, sizeof(int64_t) * n), "deep starts seeds");
        w.cap_s48 = n;
    }
    cudaStream_t st = eng->stream;
    if (s48) DEEP_CUDA(cudaMemcpyAsync(w.s48, s48, sizeof(int64_t) * n, cudaMemcpyHostToDevice, st), "upload seeds");
    DEEP_CUDA(cudaMemsetAsync(w.total, 0, sizeof(unsigned long long), st), "memset");
    WalkGeom G;
    G.s48s = s48 ? w.s48 : nullptr;
    G.s48_base = (uint64_t)s48_base;
    G.n_seeds = n;
    G.rx0 = rx0;
    G.rw = (int)rw;
    G.rz0 = rz0;
    G.rh = (int)rh;
    G.strips = (int)((rw + kDeepCols - 1) / kDeepCols);
    const uint64_t n_tasks = n * (uint64_t)rh * (uint64_t)G.strips;
    for (uint64_t t0 = 0; t0 < n_tasks; t0 += kDeepPassTasks) {
        const uint64_t m = std::min<uint64_t>(kDeepPassTasks, n_tasks - t0);
        const uint32_t blocks = (uint32_t)((m + kDeepThreads - 1) / kDeepThreads);
        walk_count_kernel<<<blocks, kDeepThreads, 0, st>>>(G, t0, m, w.counts, w.block_sums);
        walk_scan_kernel<<<1, 1024, 0, st>>>(w.block_sums, blocks, w.block_base, w.total);
        walk_write_kernel<<<blocks, kDeepThreads, 0, st>>>(G, t0, m, w.counts, w.block_base, w.out, dcap);
        DEEP_CUDA(cudaGetLastError(), "deep starts launch");
    }
    unsigned long long found = 0;
    DEEP_CUDA(cudaMemcpyAsync(&found, w.total, sizeof(found), cudaMemcpyDeviceToHost, st), "read count");
    DEEP_CUDA(cudaStreamSynchronize(st), "deep starts");
    if (found > dcap && cap > dcap) return eng->fail(WG_ERR_CAPACITY, "deep starts: more than 2^24 hits in one call");
    const uint64_t nw = std::min<uint64_t>(cap, found);
    if (nw) DEEP_CUDA(cudaMemcpy(out, w.out, sizeof(DeepHit) * nw, cudaMemcpyDeviceToHost), "copy hits");
    if (n_out) *n_out = found;
    return WG_OK;
}
