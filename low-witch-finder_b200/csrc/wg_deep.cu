// Deep Dive region walk (wg_deep_starts): for structure seeds x a region rect, the swamp-hut chunk
// of every region and whether a mineshaft starts in it.  Integer LCG work only: one thread walks
// one (seed, rx) column of regions along rz, as the reference's room walker does
// (engine/gpu/room_core.h:146-175): the region seed advances by 132897987541 per row and the
// chunk products cx * a, cz * b are formed from the hut offsets.
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
constexpr int kDeepRowsPerThread = 64;   // rz rows one thread walks

__global__ void __launch_bounds__(kDeepThreads) deep_starts_kernel(const int64_t *__restrict__ s48s, uint64_t s48_base,
                                                                   uint64_t n_seeds, int rx0, int rw, int rz0, int rh,
                                                                   uint64_t n_tasks, DeepHit *out, uint32_t cap,
                                                                   unsigned long long *count) {
    const int strips = (rh + kDeepRowsPerThread - 1) / kDeepRowsPerThread;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n_tasks;
         t += (uint64_t)gridDim.x * blockDim.x) {
        // task = (seed, strip, column): neighbouring threads take neighbouring columns of one strip
        const int col = (int)(t % (uint64_t)rw);
        const uint64_t rest = t / (uint64_t)rw;
        const int strip = (int)(rest % (uint64_t)strips);
        const uint64_t i = rest / (uint64_t)strips;
        if (i >= n_seeds) continue;
        const uint64_t s48 = (s48s ? (uint64_t)s48s[i] : s48_base + i) & kDeepMask48;
        const DeepCtx c = deep_ctx(s48);
        const int rx = rx0 + col;
        const int za = rz0 + strip * kDeepRowsPerThread;
        const int zb = min(rz0 + rh, za + kDeepRowsPerThread);
        for (int rz = za; rz < zb; rz++) {
            int cx, cz;
            hut_chunk(s48, rx, rz, 14357620, cx, cz);
            const uint64_t carver = deep_carver(c, cx, cz);
            if (!deep_is_start(carver)) continue;
            const unsigned long long k = atomicAdd(count, 1ull);
            if (k < cap) out[k] = DeepHit{i, (int64_t)s48, rx, rz, cx, cz, (int64_t)carver};
        }
    }
}

#define DEEP_CUDA(call, what)                                           \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) return eng->fail(WG_ERR_CUDA, what, e_); \
    } while (0)

}  // namespace

extern "C" int wg_deep_starts(wg_engine *eng, const int64_t *s48, int64_t s48_base, uint64_t n, int rx0, int rx1,
                              int rz0, int rz1, wg_deep_start *out, uint64_t cap, uint64_t *n_out) {
    if (!eng || rx1 <= rx0 || rz1 <= rz0 || n == 0 || (cap && !out)) return WG_ERR_ARG;
    const int64_t rw = (int64_t)rx1 - rx0, rh = (int64_t)rz1 - rz0;
    if (rw > (1 << 24) || rh > (1 << 24)) return WG_ERR_ARG;
    DEEP_CUDA(cudaSetDevice(eng->device), "cudaSetDevice");
    const uint64_t strips = (uint64_t)((rh + kDeepRowsPerThread - 1) / kDeepRowsPerThread);
    const uint64_t n_tasks = n * strips * (uint64_t)rw;
    // device buffers: the seed list, the hit list (room for cap hits, at least one) and the count
    const uint32_t dcap = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(cap, 1), 1u << 24);
    int64_t *d_s48 = nullptr;
    DeepHit *d_out = nullptr;
    unsigned long long *d_count = nullptr;
    int rc = WG_OK;
    cudaError_t e = cudaSuccess;
    if (s48) e = cudaMalloc(&d_s48, sizeof(int64_t) * n);
    if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(DeepHit) * dcap);
    if (e == cudaSuccess) e = cudaMalloc(&d_count, sizeof(unsigned long long));
    if (e == cudaSuccess && s48)
        e = cudaMemcpyAsync(d_s48, s48, sizeof(int64_t) * n, cudaMemcpyHostToDevice, eng->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), eng->stream);
    unsigned long long found = 0;
    if (e == cudaSuccess) {
        const uint64_t blocks = std::min<uint64_t>((n_tasks + kDeepThreads - 1) / kDeepThreads,
                                                   (uint64_t)eng->sm_count * 64);
        deep_starts_kernel<<<(unsigned)blocks, kDeepThreads, 0, eng->stream>>>(
            d_s48, (uint64_t)s48_base, n, rx0, (int)rw, rz0, (int)rh, n_tasks, d_out, dcap, d_count);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&found, d_count, sizeof(unsigned long long), cudaMemcpyDeviceToHost, eng->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(eng->stream);
    std::vector<DeepHit> hits;
    if (e == cudaSuccess && found) {
        hits.resize(std::min<uint64_t>(found, dcap));
        e = cudaMemcpy(hits.data(), d_out, sizeof(DeepHit) * hits.size(), cudaMemcpyDeviceToHost);
    }
    if (e != cudaSuccess) rc = eng->fail(WG_ERR_CUDA, "deep starts", e);
    cudaFree(d_s48);
    cudaFree(d_out);
    cudaFree(d_count);
    if (rc) return rc;
    if (found > dcap && cap > dcap) return eng->fail(WG_ERR_CAPACITY, "deep starts: more than 2^24 hits in one call");
    std::sort(hits.begin(), hits.end(), [](const DeepHit &x, const DeepHit &y) {
        if (x.seed_index != y.seed_index) return x.seed_index < y.seed_index;
        if (x.rz != y.rz) return x.rz < y.rz;
        return x.rx < y.rx;
    });
    // Only the first cap of the sorted order are wanted; when more than cap were found, the
    // device kept an arbitrary cap of them, so the caller is told the total and retries bigger.
    const uint64_t nw = std::min<uint64_t>(cap, hits.size());
    if (nw) std::memcpy(out, hits.data(), sizeof(DeepHit) * nw);
    if (n_out) *n_out = found;
    return WG_OK;
}
