// Deep Dive solver: for a mineshaft layout X (a catalogued setLargeFeatureSeed state), the
// structure seeds S whose swamp hut in region (rx, rz) lies at chunk offsets (ox, oz) and whose
// state at that chunk, setLargeFeatureSeed(S, cx, cz), equals X.  The reference's equations are
// engine/gpu/solver_kernels.cuh:15-115 and solver_fused.cuh; its task space (groups of regions by
// the low 20 bits of the region constant, regimes, offset classes) is engine/gpu/taskspace.h.
//
// Let t = S ^ 0x5DEECE66D be the LCG state after setSeed(S) and h2, h4 the low words of the two
// nextLong() draws a, b.  The low 32 bits of the carver state are (cx h2) ^ (cz h4) ^ S, and
// h2 = ((A^2 t + K2) >> 16) mod 2^32 (h4 with A^4, K4): adding 2^j to t (j >= 16) adds
// (A^2 << (j - 16)) to h2.  So with m = min(v2(cx), v2(cz)), state bit j first reaches equation
// bit j - 16 + m, and the equation can be lifted bit by bit:
//   * lists: per (group, key) the low-20-bit states t20 whose hut offsets have the right low 3
//     bits (state bits 17..19 of the region's first two draws) and whose equation bits
//     0 .. 3 + m are already zero; key = (cx, cz) mod 2^(4+m), which fixes those bits;
//   * chain: per task (region, offset) one warp, each lane lifts the upper 28 state bits of one
//     list entry.  When v2(cx) != v2(cz) each equation bit has one solution and the lift runs
//     four bits per step (lift_chunks); when v2(cx) == v2(cz) state bit j does not reach
//     equation bit j - 16 + m, so a nibble of the equation has 0 to 16 solutions and the lift is
//     a depth-first search over nibbles (lift_eq).  Past equation bit 31 the remaining top bits
//     are enumerated and every completion is checked in full (48-bit carver state, hut offsets
//     with the JDK rejection).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <vector>

#include "../../include/witchgpu.h"
#include "wg_engine_impl.h"

namespace {

constexpr uint64_t kA = 0x5DEECE66Dull, kC = 0xBull, kM48 = 0xFFFFFFFFFFFFull, kM20 = 0xFFFFFull;
constexpr uint64_t kA2 = (kA * kA) & kM48;
constexpr uint64_t kK2 = (kC * (kA + 1)) & kM48;
constexpr uint64_t kA4 = (kA2 * kA2) & kM48;
constexpr uint64_t kK4 = (kC * (kA * kA * kA + kA * kA + kA + 1)) & kM48;
constexpr uint64_t kA3 = (kA2 * kA) & kM48;
constexpr uint64_t kK3 = (kC * (kA * kA + kA + 1)) & kM48;
constexpr uint64_t kSalt = 14357620ull, kRX = 341873128712ull, kRZ = 132897987541ull;
constexpr int kRadius = 58593;
constexpr uint32_t kListCap = 1536;     // t20 entries per (group, key) list (mean 1,024 at m = 0)
constexpr uint32_t kGroupsPerBatch = 16;
constexpr uint32_t kHitCap = 1u << 20;
constexpr int kChainThreads = 256;
constexpr int kLiftTable = 8 * 16 * 16;    // nibble lift table (bytes)
constexpr int kEqTable = 8 * 16 * 16 * 2;  // nibble solution masks of the v2(cx) == v2(cz) lift (bytes)

// One group slot of a batch: its regions, offsets, key table and first task.
struct SolveSlot {
    uint64_t group;          // group id reported with hits
    uint64_t task_begin;     // first task of the slot (prefix over the batch's slots)
    uint32_t c20;            // low 20 bits of the region constant shared by the slot's regions
    uint32_t reg_begin, reg_count;
    uint32_t off_begin, off_count;
    uint32_t key_begin, key_count;   // keys[key_begin ..), lists [list_begin + k]
    uint32_t map_begin;      // keymap[map_begin + o * 64 + (rx & 7) * 8 + (rz & 7)] = key index
    uint32_t list_begin;
    uint32_t pad;
};

struct SolveKey {            // (cx, cz) mod 2^(4 + m)
    uint32_t cxm, czm;
    int32_t m, pad;
};

struct SolveHitDev {
    uint64_t s48;
    int32_t cx, cz;
    uint64_t layout, group;
};
static_assert(sizeof(SolveHitDev) == sizeof(wg_solve_hit), "solve hit layout");

enum : int { SCNT_HITS = 0, SCNT_OVERFLOW = 1, SCNT_CANDIDATES = 2, SCNT_WORDS = 4 };

__host__ __device__ __forceinline__ uint64_t region_const(int rx, int rz) {
    return (kSalt + (uint64_t)(int64_t)rx * kRX + (uint64_t)(int64_t)rz * kRZ) & kM48;
}

__host__ __device__ __forceinline__ int v2_of(uint32_t v) {
#ifdef __CUDA_ARCH__
    return v ? __ffs((int)v) - 1 : 40;
#else
    return v ? __builtin_ctz(v) : 40;
#endif
}

// v2(cx) == v2(cz) for cx = 32 rx + ox, cz = 32 rz + oz with 0 <= ox, oz < 24, not both 0.
__host__ __device__ __forceinline__ bool offsets_eq(int ox, int oz) {
    return ox != 0 && oz != 0 && v2_of((uint32_t)ox) == v2_of((uint32_t)oz);
}

// Equation bits of t (low 32): (cx h2) ^ (cz h4) ^ S ^ X.
__device__ __forceinline__ uint32_t eq_word(uint64_t t, uint32_t cx, uint32_t cz, uint32_t xs) {
    const uint32_t h2 = (uint32_t)((((kA2 * t) + kK2) & kM48) >> 16);
    const uint32_t h4 = (uint32_t)((((kA4 * t) + kK4) & kM48) >> 16);
    return (cx * h2) ^ (cz * h4) ^ (uint32_t)t ^ xs;   // xs = X ^ A (low words): S = t ^ A
}

__device__ __forceinline__ int lcg_next_int24(uint64_t &s) {
    for (;;) {
        s = (s * kA + kC) & kM48;
        const int bits = (int)(s >> 17), val = bits % 24;
        if ((int)((uint32_t)bits - (uint32_t)val + 23u) >= 0) return val;
    }
}

// Full check of a structure seed: the carver state at (cx, cz) and the hut offsets of the region.
__device__ __forceinline__ bool solve_check(uint64_t S, int cx, int cz, uint64_t X, uint64_t creg, int ox, int oz) {
    uint64_t s = (S ^ kA) & kM48;
    int32_t h[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        s = (s * kA + kC) & kM48;
        h[k] = (int32_t)(s >> 16);
    }
    const uint64_t a = ((uint64_t)(int64_t)h[0] << 32) + (uint64_t)(int64_t)h[1];
    const uint64_t b = ((uint64_t)(int64_t)h[2] << 32) + (uint64_t)(int64_t)h[3];
    const uint64_t carver = ((uint64_t)((int64_t)cx * (int64_t)a) ^ (uint64_t)((int64_t)cz * (int64_t)b) ^ S) & kM48;
    if (carver != X) return false;
    uint64_t r = ((S + creg) ^ kA) & kM48;
    if (lcg_next_int24(r) != ox) return false;
    return lcg_next_int24(r) == oz;
}

struct ChainTask {
    int cx, cz, ox, oz, m;
    bool eq;
    uint64_t creg, X, group;
};

__device__ __forceinline__ void emit_hit(const ChainTask &T, uint64_t S, SolveHitDev *hits, uint32_t cap,
                                         unsigned long long *cnt) {
    const unsigned long long k = atomicAdd(&cnt[SCNT_HITS], 1ull);
    if (k < cap) hits[k] = SolveHitDev{S, T.cx, T.cz, T.X, T.group};
    else atomicOr(&cnt[SCNT_OVERFLOW], 2ull);
}

// v2(cx) != v2(cz), four state bits per step.  Divide the equation by 2^m and call "o" the term
// whose multiplier is odd after that (cx h2 if v2(cx) = m, else cz h4) and "e" the other.  With
// z = o (the odd term's value) as the unknown instead of the upper state bits u: 16 u =
// (z - o0) / (odd multiplier) = V, and e = Kq + rho z with rho = (even multiplier) / (odd
// multiplier), an even number.  The equation z ^ (Kq + rho z) ^ Y = 0, where Y = (S ^ X) >> m
// holds u only as V << 16 (bits known from lower nibbles), is triangular in z nibble by nibble:
// nibble k solves zk ^ ((Aq_k + rho zk) mod 16) = Y_k, Aq = Kq + rho z<k, one lookup in a
// 2,048-entry table [rho mod 16 / 2][Aq_k][Y_k].  The top m bits of u are free.
struct ChunkTask {
    uint32_t inv, rho, coef_o_x;   // 1 / odd multiplier, rho, 1 if the odd term is cx h2
    const uint8_t *row;            // table row for rho mod 16
};

__device__ __forceinline__ uint32_t inverse_u32(uint32_t a) {   // a odd
    uint32_t x = a;
#pragma unroll
    for (int i = 0; i < 5; i++) x *= 2u - a * x;
    return x;
}

// Full check of t = t20 | u << 20 (u: 28 bits).  The 48-bit carver state from 32-bit words: the
// draws' low words h2, h4 move by (A^2 << 4) u and (A^4 << 4) u; only the low 16 bits of the high
// words h1, h3 reach bit 47 of a, b, and those are bits 16..31 of A t + C, A^3 t + K3, which the
// state's low word alone decides.
__device__ __forceinline__ void check_u(const ChainTask &T, uint32_t t20, uint32_t h2, uint32_t h4, uint32_t u,
                                        SolveHitDev *hits, uint32_t cap, unsigned long long *cnt) {
    const uint32_t t32 = t20 | (u << 20);
    const uint32_t h2u = h2 + (uint32_t)(kA2 << 4) * u, h4u = h4 + (uint32_t)(kA4 << 4) * u;
    const uint32_t h1lo = (((uint32_t)kA * t32 + (uint32_t)kC) >> 16) & 0xFFFFu;
    const uint32_t h3lo = (((uint32_t)kA3 * t32 + (uint32_t)kK3) >> 16) & 0xFFFFu;
    const uint64_t a = ((uint64_t)h1lo << 32) + (uint64_t)(int64_t)(int32_t)h2u;
    const uint64_t b = ((uint64_t)h3lo << 32) + (uint64_t)(int64_t)(int32_t)h4u;
    const uint64_t S = ((((uint64_t)(u >> 12)) << 32) | t32) ^ (kA & kM48);
    const uint64_t carver =
        ((uint64_t)((int64_t)T.cx * (int64_t)a) ^ (uint64_t)((int64_t)T.cz * (int64_t)b) ^ S) & kM48;
    if (carver != T.X) return;
    if (solve_check(S, T.cx, T.cz, T.X, T.creg, T.ox, T.oz)) emit_hit(T, S, hits, cap, cnt);
}

__device__ void lift_chunks(const ChainTask &T, const ChunkTask &N, uint32_t t20, SolveHitDev *hits, uint32_t cap,
                             unsigned long long *cnt) {
    const uint32_t cx = (uint32_t)T.cx, cz = (uint32_t)T.cz, m = (uint32_t)T.m;
    const uint32_t h2 = (uint32_t)((((kA2 * t20) + kK2) & kM48) >> 16);
    const uint32_t h4 = (uint32_t)((((kA4 * t20) + kK4) & kM48) >> 16);
    const uint32_t P = cx * h2, Q = cz * h4;
    const uint32_t o0 = (N.coef_o_x ? P : Q) >> m, e0 = (N.coef_o_x ? Q : P) >> m;
    const uint32_t s0 = t20 ^ (uint32_t)kA, x32 = (uint32_t)T.X;
    const uint32_t kq = e0 - N.rho * o0;
    uint32_t z = o0 & 15u;   // nibble 0 is o0's: u only enters from bit 4 (16 u)
#pragma unroll
    for (int k = 4; k < 32; k += 4) {
        const uint32_t V = (z - o0) * N.inv;
        const uint32_t Y = ((s0 ^ (V << 16)) ^ x32) >> m;
        const uint32_t Aq = kq + N.rho * z;
        z |= (uint32_t)N.row[(((Aq >> k) & 15u) << 4) | ((Y >> k) & 15u)] << k;
    }
    const uint32_t u0 = (((z - o0) * N.inv) >> 4) & ((1u << (28 - m)) - 1u);
    for (uint32_t f = 0; f < (1u << m); f++) check_u(T, t20, h2, h4, u0 | (f << (28 - m)), hits, cap, cnt);
}

// v2(cx) == v2(cz): the same substitution with o = cx h2 leaves rho = (cz A^4) / (cx A^2) odd, and
// then z ^ ((Aq + rho z) mod 16) no longer determines z's nibble: its bit 0 equals Aq's (a check on
// the lower nibbles) and its bits 1..3 constrain the nibble's bits 0..2, so a nibble has 0 to 16
// solutions.  They come as a 16-bit mask from a 4 KB table [rho mod 16 / 2][Aq_k][Y_k], and the
// seven nibbles above the list's are searched depth first with one mask per level.  Equation bits
// past 31 - m do not exist: at the top nibble the mask is the union over them, so every remaining
// u is enumerated there.
__device__ __forceinline__ uint32_t eq_mask(const uint16_t *row, uint32_t Aq, uint32_t Y, int k, int valid) {
    const uint32_t a = (Aq >> k) & 15u, y = (Y >> k) & 15u;
    if (valid >= 4) return row[(a << 4) | y];
    uint32_t mk = 0;   // union over the equation bits that do not exist
    const uint32_t keep = (1u << valid) - 1u;
    for (uint32_t yy = 0; yy < 16; yy++)
        if (((yy ^ y) & keep) == 0) mk |= row[(a << 4) | yy];
    return mk;
}

// The per-candidate constants of the search: the draws' low words at t20, the odd term o0, and
// Kq = e0 - rho o0 (rho = (cz A^4) / (cx A^2), odd).
struct EqCand {
    uint32_t h2, h4, o0, kq, s0;
};

__device__ __forceinline__ EqCand eq_cand(const ChainTask &T, const ChunkTask &N, uint32_t t20) {
    EqCand c;
    c.h2 = (uint32_t)((((kA2 * t20) + kK2) & kM48) >> 16);
    c.h4 = (uint32_t)((((kA4 * t20) + kK4) & kM48) >> 16);
    c.o0 = ((uint32_t)T.cx * c.h2) >> T.m;
    c.kq = (((uint32_t)T.cz * c.h4) >> T.m) - N.rho * c.o0;
    c.s0 = t20 ^ (uint32_t)kA;
    return c;
}

// Solutions of the nibble at level L (bits 4 + 4L .. 7 + 4L) given z's lower nibbles.  Y's nibble
// reads V bits up to 4L + m - 9 < 4 + 4L (m <= 4), all set already.
__device__ __forceinline__ uint32_t eq_level(const ChainTask &T, const ChunkTask &N, const uint16_t *row,
                                             const EqCand &c, uint32_t z, int L) {
    const int k = 4 + 4 * L;
    const uint32_t V = (z - c.o0) * N.inv;
    const uint32_t Y = ((c.s0 ^ (V << 16)) ^ (uint32_t)T.X) >> T.m;
    return eq_mask(row, c.kq + N.rho * z, Y, k, 32 - T.m - k);
}

// Depth-first search below node (z, L0): z holds the nibbles under level L0.
__device__ void lift_eq_from(const ChainTask &T, const ChunkTask &N, const uint16_t *row, uint32_t t20,
                             const EqCand &c, uint32_t z, int L0, SolveHitDev *hits, uint32_t cap,
                             unsigned long long *cnt) {
    uint32_t masks[7];
    int L = L0;
    masks[L] = eq_level(T, N, row, c, z, L);
    for (;;) {
        if (!masks[L]) {
            if (--L < L0) return;
            continue;
        }
        const int k = 4 + 4 * L;
        const uint32_t v = (uint32_t)__ffs((int)masks[L]) - 1u;
        masks[L] &= masks[L] - 1u;
        z = (z & ((1u << k) - 1u)) | (v << k);
        if (L == 6) {
            check_u(T, t20, c.h2, c.h4, ((z - c.o0) * N.inv) >> 4, hits, cap, cnt);
            continue;
        }
        L++;
        masks[L] = eq_level(T, N, row, c, z, L);
    }
}

// One eq task, level by level across the warp: each lane's own search tree has a different size
// (0 to 16 solutions per nibble), so instead of a search per lane the warp keeps the nodes of a
// level in a shared queue and every lane expands queue entries; 32 list entries start a round.
// A node whose children do not fit in the next level's queue is searched depth first by its lane.
constexpr int kEqQueue = 256;
constexpr uint32_t kEqNone = 0xFFFFFFFFu;   // queue slot reserved by a node that did not fit

__device__ void eq_task(const ChainTask &T, const ChunkTask &N, const uint16_t *row, const uint32_t *list,
                        uint32_t n, SolveHitDev *hits, uint32_t cap, unsigned long long *cnt) {
    __shared__ uint2 queue[kChainThreads / 32][2][kEqQueue];   // (t20, z) per node
    __shared__ uint32_t qcount[kChainThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x / 32;
    for (uint32_t base = 0; base < n; base += 32) {
        uint2 *cur = queue[wid][0], *nxt = queue[wid][1];
        const uint32_t c0 = min(32u, n - base);
        if ((uint32_t)lane < c0) {
            const uint32_t t20 = list[base + lane];
            cur[lane] = make_uint2(t20, eq_cand(T, N, t20).o0 & 15u);
        }
        uint32_t count = c0;
        for (int L = 0; L < 7 && count; L++) {
            if (lane == 0) qcount[wid] = 0;
            __syncwarp();
            const int k = 4 + 4 * L;
            for (uint32_t i = (uint32_t)lane; i < count; i += 32) {
                const uint2 nd = cur[i];
                if (nd.x == kEqNone) continue;
                const EqCand c = eq_cand(T, N, nd.x);
                uint32_t mk = eq_level(T, N, row, c, nd.y, L);
                if (!mk) continue;
                if (L == 6) {
                    for (; mk; mk &= mk - 1u) {
                        const uint32_t z = nd.y | (((uint32_t)__ffs((int)mk) - 1u) << k);
                        check_u(T, nd.x, c.h2, c.h4, ((z - c.o0) * N.inv) >> 4, hits, cap, cnt);
                    }
                    continue;
                }
                const uint32_t pc = (uint32_t)__popc(mk);
                uint32_t at = atomicAdd(&qcount[wid], pc);
                if (at + pc <= (uint32_t)kEqQueue) {
                    for (; mk; mk &= mk - 1u)
                        nxt[at++] = make_uint2(nd.x, nd.y | (((uint32_t)__ffs((int)mk) - 1u) << k));
                } else {
                    for (uint32_t q = at; q < (uint32_t)kEqQueue && q < at + pc; q++) nxt[q] = make_uint2(kEqNone, 0u);
                    for (; mk; mk &= mk - 1u)
                        lift_eq_from(T, N, row, nd.x, c, nd.y | (((uint32_t)__ffs((int)mk) - 1u) << k), L + 1, hits,
                                     cap, cnt);
                }
            }
            __syncwarp();
            count = min(qcount[wid], (uint32_t)kEqQueue);
            uint2 *t = cur;
            cur = nxt;
            nxt = t;
            __syncwarp();
        }
    }
}

// grid (key, slot): the list of (slot, key) from the t20 candidates of the key's hut offsets.
__global__ void __launch_bounds__(256) solve_lists_kernel(const SolveSlot *__restrict__ slots,
                                                          const SolveKey *__restrict__ keys,
                                                          const uint32_t *__restrict__ hq,
                                                          const uint32_t *__restrict__ hq_off, uint64_t X,
                                                          uint32_t *__restrict__ lists, uint32_t *__restrict__ counts,
                                                          unsigned long long *cnt) {
    const SolveSlot &sl = slots[blockIdx.y];
    if (blockIdx.x >= sl.key_count) return;
    const SolveKey K = keys[sl.key_begin + blockIdx.x];
    const uint32_t li = sl.list_begin + blockIdx.x;
    const uint32_t hkey = ((K.cxm & 7u) << 3) | (K.czm & 7u);
    const uint32_t lo = hq_off[hkey], hi = hq_off[hkey + 1];
    const uint32_t low = (1u << (4 + K.m)) - 1u, xs = (uint32_t)(X ^ kA), a20 = (uint32_t)(kA & kM20);
    __shared__ uint32_t n;
    if (threadIdx.x == 0) n = 0;
    __syncthreads();
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        // region state q0 = ((S + creg) ^ A) mod 2^20  ->  t20 = ((q0 ^ A) - creg) ^ A
        const uint32_t q0 = hq[i];
        const uint32_t t20 = (((q0 ^ a20) - sl.c20) & (uint32_t)kM20) ^ a20;
        if (eq_word(t20, K.cxm, K.czm, xs) & low) continue;
        const uint32_t k = atomicAdd(&n, 1u);
        if (k < kListCap) lists[(size_t)li * kListCap + k] = t20;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        counts[li] = min(n, kListCap);
        if (n > kListCap) atomicOr(&cnt[SCNT_OVERFLOW], 1ull);
    }
}

// One warp per task (slot, region, offset); lanes take the task's list entries.
template <bool EQ>
__global__ void __launch_bounds__(kChainThreads, EQ ? 4 : 6) solve_chain_kernel(
    const SolveSlot *__restrict__ slots, uint32_t n_slots, uint64_t n_tasks, const int2 *__restrict__ regions,
    const int2 *__restrict__ offsets, const uint32_t *__restrict__ keymap, const uint32_t *__restrict__ lists,
    const uint32_t *__restrict__ counts, const uint8_t *__restrict__ nib, uint64_t X, SolveHitDev *hits,
    uint32_t hit_cap, unsigned long long *cnt) {
    // the class's table: the nibble lift's (2 KB) or the solution masks (4 KB, after it in `nib`)
    constexpr int kTab = EQ ? kEqTable : kLiftTable;
    __shared__ __align__(16) uint8_t tab[kTab];
    const uint8_t *src = nib + (EQ ? kLiftTable : 0);
    for (int i = threadIdx.x; i < kTab / 16; i += kChainThreads) ((uint4 *)tab)[i] = ((const uint4 *)src)[i];
    __syncthreads();
    const uint16_t *eqtab = reinterpret_cast<const uint16_t *>(tab);
    const int lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (kChainThreads / 32);
    unsigned long long lifted = 0;
    for (uint64_t w = (uint64_t)blockIdx.x * (kChainThreads / 32) + threadIdx.x / 32; w < n_tasks; w += warps) {
        uint32_t lo = 0, hi = n_slots - 1;   // last slot whose first task is <= w
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (slots[mid].task_begin <= w) lo = mid;
            else hi = mid - 1;
        }
        const SolveSlot &sl = slots[lo];
        const uint64_t local = w - sl.task_begin;
        const uint32_t o = (uint32_t)(local / sl.reg_count), r = (uint32_t)(local % sl.reg_count);
        const int2 O = offsets[sl.off_begin + o];
        // the class follows from the offsets (0 < offset < 24, so v2(cx) = v2(ox) unless ox = 0)
        if (offsets_eq(O.x, O.y) != EQ) continue;
        const int2 R = regions[sl.reg_begin + r];
        ChainTask T;
        T.ox = O.x;
        T.oz = O.y;
        T.cx = R.x * 32 + O.x;
        T.cz = R.y * 32 + O.y;
        const int vx = v2_of((uint32_t)T.cx), vz = v2_of((uint32_t)T.cz);
        T.m = min(vx, vz);
        T.eq = vx == vz;
        T.creg = region_const(R.x, R.y);
        T.X = X;
        T.group = sl.group;
        const uint32_t k = keymap[sl.map_begin + o * 64 + (uint32_t)(R.x & 7) * 8 + (uint32_t)(R.y & 7)];
        const uint32_t li = sl.list_begin + k;
        const uint32_t n = counts[li];
        const uint32_t *list = lists + (size_t)li * kListCap;
        if (lane == 0) lifted += n;
        if constexpr (EQ) {
            ChunkTask N;
            const uint32_t co = ((uint32_t)T.cx * (uint32_t)kA2) >> T.m, ce = ((uint32_t)T.cz * (uint32_t)kA4) >> T.m;
            N.coef_o_x = 1u;
            N.inv = inverse_u32(co);
            N.rho = ce * N.inv;
            N.row = nullptr;
            eq_task(T, N, eqtab + ((N.rho & 15u) >> 1) * 256, list, n, hits, hit_cap, cnt);
        } else {
            ChunkTask N;
            const uint32_t cxa = (uint32_t)T.cx * (uint32_t)kA2, cza = (uint32_t)T.cz * (uint32_t)kA4;
            N.coef_o_x = vx < vz ? 1u : 0u;
            const uint32_t co = (N.coef_o_x ? cxa : cza) >> T.m, ce = (N.coef_o_x ? cza : cxa) >> T.m;
            N.inv = inverse_u32(co);
            N.rho = ce * N.inv;
            N.row = tab + ((N.rho & 15u) >> 1) * 256;
            for (uint32_t i = lane; i < n; i += 32) lift_chunks(T, N, list[i], hits, hit_cap, cnt);
        }
    }
    if (lane == 0 && lifted) atomicAdd(&cnt[SCNT_CANDIDATES], lifted);
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
struct SolveState {
    uint32_t *hq = nullptr, *hq_off = nullptr;   // region states q0 (mod 2^20) grouped by hut key
    uint8_t *nib = nullptr;   // [rho mod 16 / 2][a][y] -> x with x ^ ((a + rho x) mod 16) = y (rho even), then the odd-rho masks
    SolveSlot *slots = nullptr;
    SolveKey *keys = nullptr;
    uint32_t *keymap = nullptr, *lists = nullptr, *counts = nullptr;
    int2 *regions = nullptr, *offsets = nullptr;
    SolveHitDev *hits = nullptr;
    unsigned long long *cnt = nullptr;
    size_t cap_slots = 0, cap_keys = 0, cap_map = 0, cap_lists = 0, cap_regions = 0, cap_offsets = 0;
};

void solve_release(wg_engine *eng) {
    SolveState *s = eng->solve;
    if (!s) return;
    void *ptrs[] = {s->hq, s->hq_off, s->nib, s->slots, s->keys, s->keymap, s->lists, s->counts, s->regions, s->offsets,
                    s->hits, s->cnt};
    for (void *p : ptrs) cudaFree(p);
    delete s;
    eng->solve = nullptr;
}

namespace {

#define SOLVE_CUDA(call, what)                                          \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) return eng->fail(WG_ERR_CUDA, what, e_); \
    } while (0)

template <class T>
int grow(wg_engine *eng, T *&p, size_t &cap, size_t n, const char *what) {
    if (n <= cap) return WG_OK;
    cudaFree(p);
    p = nullptr;
    cap = 0;
    const size_t c = std::max<size_t>(n, 64);
    cudaError_t e = cudaMalloc(&p, sizeof(T) * c);
    if (e != cudaSuccess) return eng->fail(WG_ERR_NOMEM, what, e);
    cap = c;
    return WG_OK;
}

int solve_state(wg_engine *eng, SolveState **out) {
    if (!eng->solve) {
        SolveState *s = new SolveState();
        eng->solve = s;
        // the 2^20 region states q0 sorted by the low 3 bits of the two hut draws they give:
        // q1 = A q0 + C, q2 = A q1 + C (mod 2^20), key = ((q1 >> 17) << 3) | (q2 >> 17)
        std::vector<uint32_t> key(1u << 20), list(1u << 20), off(65, 0);
        for (uint32_t q = 0; q < (1u << 20); q++) {
            const uint64_t q1 = ((uint64_t)q * kA + kC) & kM20, q2 = (q1 * kA + kC) & kM20;
            key[q] = (uint32_t)(((q1 >> 17) << 3) | (q2 >> 17));
            off[key[q] + 1]++;
        }
        for (int k = 0; k < 64; k++) off[k + 1] += off[k];
        std::vector<uint32_t> fill(off.begin(), off.end() - 1);
        for (uint32_t q = 0; q < (1u << 20); q++) list[fill[key[q]]++] = q;
        SOLVE_CUDA(cudaMalloc(&s->hq, sizeof(uint32_t) << 20), "solver tables");
        SOLVE_CUDA(cudaMalloc(&s->hq_off, sizeof(uint32_t) * 65), "solver tables");
        SOLVE_CUDA(cudaMalloc(&s->hits, sizeof(SolveHitDev) * kHitCap), "solver hits");
        SOLVE_CUDA(cudaMalloc(&s->cnt, sizeof(unsigned long long) * SCNT_WORDS), "solver counters");
        SOLVE_CUDA(cudaMemcpy(s->hq, list.data(), sizeof(uint32_t) << 20, cudaMemcpyHostToDevice), "solver tables");
        SOLVE_CUDA(cudaMemcpy(s->hq_off, off.data(), sizeof(uint32_t) * 65, cudaMemcpyHostToDevice), "solver tables");
        // the nibble step's solutions, by search: x ^ ((a + 2r x) mod 16) is a bijection of x
        std::vector<uint8_t> nib(kLiftTable + kEqTable, 0);
        for (int r = 0; r < 8; r++)
            for (int a = 0; a < 16; a++)
                for (int x = 0; x < 16; x++) nib[r * 256 + a * 16 + (x ^ ((a + 2 * r * x) & 15))] = (uint8_t)x;
        // and the masks of x with x ^ ((a + rho x) mod 16) = y for odd rho = 2r + 1
        std::vector<uint16_t> eqm(kEqTable / 2, 0);
        for (int r = 0; r < 8; r++)
            for (int a = 0; a < 16; a++)
                for (int x = 0; x < 16; x++) eqm[r * 256 + a * 16 + (x ^ ((a + (2 * r + 1) * x) & 15))] |= (uint16_t)(1u << x);
        std::memcpy(nib.data() + kLiftTable, eqm.data(), kEqTable);
        SOLVE_CUDA(cudaMalloc(&s->nib, kLiftTable + kEqTable), "solver tables");
        SOLVE_CUDA(cudaMemcpy(s->nib, nib.data(), kLiftTable + kEqTable, cudaMemcpyHostToDevice), "solver tables");
    }
    *out = eng->solve;
    return WG_OK;
}

// taskspace.h:12-18: the rx / rz ranges of a regime.
int regime_ranges(int regime, int64_t lo[2], int64_t hi[2]) {
    if (regime == 0) {
        lo[0] = -16384;
        hi[0] = 16383;
        return 1;
    }
    if (regime == 1) {
        lo[0] = -32768, hi[0] = -16385, lo[1] = 16384, hi[1] = 32767;
        return 2;
    }
    lo[0] = -kRadius, hi[0] = -32769, lo[1] = 32768, hi[1] = kRadius;
    return 2;
}

// taskspace.h:27: the scramble from a group's index to the residue class it covers.
uint32_t perm_group(uint32_t p) {
    uint32_t x = (p * 0x9E3779B1u) & 0xFFFFFu;
    x ^= x >> 9;
    x = (x * 0x85EBCA6Bu) & 0xFFFFFu;
    x ^= x >> 7;
    return x & 0xFFFFFu;
}

uint32_t inverse_mod_2_20(uint32_t b) {   // b odd; Newton's iteration doubles the correct bits
    uint32_t x = b;
    for (int i = 0; i < 5; i++) x *= 2u - b * x;
    return x & 0xFFFFFu;
}

// The regime's regions whose region constant is c20 mod 2^20: for each rx the one rz residue
// (the z multiplier is odd, so invertible mod 2^20), kept if it names a region inside the range.
void group_regions(uint32_t c20, int rgx, int rgz, std::vector<int2> &out) {
    int64_t xl[2], xh[2], zl[2], zh[2];
    const int nx = regime_ranges(rgx, xl, xh), nz = regime_ranges(rgz, zl, zh);
    const uint32_t inv = inverse_mod_2_20((uint32_t)(kRZ & kM20)), c1 = (uint32_t)(kRX & kM20),
                   c0 = (uint32_t)(kSalt & kM20);
    for (int a = 0; a < nx; a++)
        for (int64_t rx = xl[a]; rx <= xh[a]; rx++) {
            const uint32_t rem = (c20 - c0 - (uint32_t)rx * c1) & 0xFFFFFu;
            const uint32_t r = (rem * inv) & 0xFFFFFu;
            int64_t rz;
            if (r <= (uint32_t)kRadius) rz = r;
            else if (r >= (1u << 20) - (uint32_t)kRadius) rz = (int64_t)r - (1 << 20);
            else continue;
            bool in = false;
            for (int b = 0; b < nz; b++) in |= rz >= zl[b] && rz <= zh[b];
            if (in) out.push_back(make_int2((int)rx, (int)rz));
        }
}

int v2_host(int v) { return v ? __builtin_ctz((uint32_t)v) : 40; }

// The chunk offsets of an offset class (taskspace.h / solver_fused.cuh:23-31): 1 = the 2-adic
// valuations of ox and oz differ and the smaller is 0, 2 = differ with the smaller >= 1,
// 3 = equal (and not both 0).
void tier_offsets(int tier, std::vector<int2> &out) {
    for (int a = 0; a < 24; a++)
        for (int b = 0; b < 24; b++) {
            const int va = a ? v2_host(a) : 99, vb = b ? v2_host(b) : 99, m = std::min(va, vb);
            const bool t1 = va != vb && m == 0, t2 = va != vb && m >= 1, t3 = va == vb && va < 99;
            if ((tier == 1 && t1) || (tier == 2 && t2) || (tier == 3 && t3)) out.push_back(make_int2(a, b));
        }
}

SolveKey key_of(int cx, int cz) {
    const int vx = v2_host(cx), vz = v2_host(cz), m = std::min(vx, vz);
    const uint32_t mask = (1u << (4 + m)) - 1u;
    return SolveKey{(uint32_t)cx & mask, (uint32_t)cz & mask, m, 0};
}

// Key table and the (offset, rx mod 8, rz mod 8) -> key map of an offset list.
void build_keys(const std::vector<int2> &offs, std::vector<SolveKey> &keys, std::vector<uint32_t> &map) {
    std::map<std::tuple<int, uint32_t, uint32_t>, uint32_t> index;
    map.assign(offs.size() * 64, 0);
    for (size_t o = 0; o < offs.size(); o++)
        for (int a = 0; a < 8; a++)
            for (int b = 0; b < 8; b++) {
                const SolveKey k = key_of(32 * a + offs[o].x, 32 * b + offs[o].y);
                auto it = index.find({k.m, k.cxm, k.czm});
                if (it == index.end()) {
                    it = index.emplace(std::make_tuple(k.m, k.cxm, k.czm), (uint32_t)keys.size()).first;
                    keys.push_back(k);
                }
                map[o * 64 + a * 8 + b] = it->second;
            }
}

bool host_hit_ok(const SolveHitDev &h, bool need_start) {
    // the forward computation the reference's host thread repeats: the carver state, the hut's
    // exact chunk (room_core.h rcHutExact) and (for a catalogued layout) that the layout state
    // starts a mineshaft
    const uint64_t S = h.s48 & kM48;
    uint64_t s = (S ^ kA) & kM48;
    int32_t v[4];
    for (int k = 0; k < 4; k++) {
        s = (s * kA + kC) & kM48;
        v[k] = (int32_t)(s >> 16);
    }
    const uint64_t a = ((uint64_t)(int64_t)v[0] << 32) + (uint64_t)(int64_t)v[1];
    const uint64_t b = ((uint64_t)(int64_t)v[2] << 32) + (uint64_t)(int64_t)v[3];
    if ((((uint64_t)((int64_t)h.cx * (int64_t)a) ^ (uint64_t)((int64_t)h.cz * (int64_t)b) ^ S) & kM48) != h.layout)
        return false;
    const int rx = h.cx >> 5, rz = h.cz >> 5;
    uint64_t r = ((S + region_const(rx, rz)) ^ kA) & kM48;
    int off[2];
    for (int k = 0; k < 2; k++)
        for (;;) {
            r = (r * kA + kC) & kM48;
            const int bits = (int)(r >> 17), val = bits % 24;
            if ((int)((uint32_t)bits - (uint32_t)val + 23u) >= 0) {
                off[k] = val;
                break;
            }
        }
    if (rx * 32 + off[0] != h.cx || rz * 32 + off[1] != h.cz) return false;
    if (!need_start) return true;
    uint64_t q = (h.layout ^ kA) & kM48;
    q = (q * kA + kC) & kM48;
    const int64_t hi = (int64_t)(q >> 22);
    q = (q * kA + kC) & kM48;
    const int64_t lo = (int64_t)(q >> 21);
    return (double)((hi << 27) + lo) * 1.1102230246251565404e-16 < 0.004;
}

// One batch: lists for every (slot, key), then the chain over every task; hits appended to `out`.
int run_solve_batch(wg_engine *eng, SolveState *st, uint64_t X, const std::vector<SolveSlot> &slots,
                    const std::vector<SolveKey> &keys, const std::vector<uint32_t> &map,
                    const std::vector<int2> &regions, const std::vector<int2> &offs, uint32_t n_lists,
                    uint32_t max_keys, uint64_t n_tasks, std::vector<SolveHitDev> &out, wg_solve_stats &ss) {
    int rc = grow(eng, st->slots, st->cap_slots, slots.size(), "solver slots");
    if (!rc) rc = grow(eng, st->keys, st->cap_keys, keys.size(), "solver keys");
    if (!rc) rc = grow(eng, st->keymap, st->cap_map, map.size(), "solver key map");
    if (!rc) rc = grow(eng, st->regions, st->cap_regions, std::max<size_t>(regions.size(), 1), "solver regions");
    if (!rc) rc = grow(eng, st->offsets, st->cap_offsets, offs.size(), "solver offsets");
    if (!rc && (size_t)n_lists * kListCap > st->cap_lists) {
        cudaFree(st->lists);
        cudaFree(st->counts);
        st->lists = nullptr;
        st->counts = nullptr;
        st->cap_lists = 0;
        cudaError_t e = cudaMalloc(&st->lists, sizeof(uint32_t) * kListCap * (size_t)n_lists);
        if (e == cudaSuccess) e = cudaMalloc(&st->counts, sizeof(uint32_t) * n_lists);
        if (e != cudaSuccess) return eng->fail(WG_ERR_NOMEM, "solver lists", e);
        st->cap_lists = (size_t)n_lists * kListCap;
    }
    if (rc) return rc;
    cudaStream_t s = eng->stream;
    SOLVE_CUDA(cudaMemcpyAsync(st->slots, slots.data(), sizeof(SolveSlot) * slots.size(), cudaMemcpyHostToDevice, s), "upload");
    SOLVE_CUDA(cudaMemcpyAsync(st->keys, keys.data(), sizeof(SolveKey) * keys.size(), cudaMemcpyHostToDevice, s), "upload");
    SOLVE_CUDA(cudaMemcpyAsync(st->keymap, map.data(), sizeof(uint32_t) * map.size(), cudaMemcpyHostToDevice, s), "upload");
    if (!regions.empty())
        SOLVE_CUDA(cudaMemcpyAsync(st->regions, regions.data(), sizeof(int2) * regions.size(), cudaMemcpyHostToDevice, s),
                   "upload");
    SOLVE_CUDA(cudaMemcpyAsync(st->offsets, offs.data(), sizeof(int2) * offs.size(), cudaMemcpyHostToDevice, s), "upload");
    SOLVE_CUDA(cudaMemsetAsync(st->cnt, 0, sizeof(unsigned long long) * SCNT_WORDS, s), "memset");
    SOLVE_CUDA(cudaEventRecord(eng->ev0, s), "event");
    solve_lists_kernel<<<dim3(max_keys, (unsigned)slots.size()), 256, 0, s>>>(st->slots, st->keys, st->hq, st->hq_off, X,
                                                                             st->lists, st->counts, st->cnt);
    if (n_tasks) {
        // one kernel per offset class present (the equal-valuation class has its own search); as
        // many blocks as are resident at once: the kernel loops over tasks, so more would only
        // form a second, mostly idle wave
        bool has_eq = false, has_other = false;
        for (const int2 &o : offs) (offsets_eq(o.x, o.y) ? has_eq : has_other) = true;
        static int per_sm[2] = {0, 0};
        for (int eq = 0; eq < 2; eq++) {
            if (!(eq ? has_eq : has_other)) continue;
            if (!per_sm[eq]) {
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &per_sm[eq], eq ? solve_chain_kernel<true> : solve_chain_kernel<false>, kChainThreads, 0);
                if (per_sm[eq] < 1) per_sm[eq] = 1;
            }
            const uint64_t blocks = std::min<uint64_t>((n_tasks + (kChainThreads / 32) - 1) / (kChainThreads / 32),
                                                       (uint64_t)eng->sm_count * per_sm[eq]);
            (eq ? solve_chain_kernel<true> : solve_chain_kernel<false>)<<<(unsigned)blocks, kChainThreads, 0, s>>>(
                st->slots, (uint32_t)slots.size(), n_tasks, st->regions, st->offsets, st->keymap, st->lists,
                st->counts, st->nib, X, st->hits, kHitCap, st->cnt);
        }
    }
    SOLVE_CUDA(cudaGetLastError(), "solver launch");
    SOLVE_CUDA(cudaEventRecord(eng->ev1, s), "event");
    unsigned long long c[SCNT_WORDS];
    SOLVE_CUDA(cudaMemcpyAsync(c, st->cnt, sizeof c, cudaMemcpyDeviceToHost, s), "read counters");
    SOLVE_CUDA(cudaStreamSynchronize(s), "solver batch");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, eng->ev0, eng->ev1);
    ss.gpu_ms += ms;
    if (c[SCNT_OVERFLOW] & 1ull) return eng->fail(WG_ERR_CAPACITY, "solver: a candidate list outgrew its capacity");
    if (c[SCNT_OVERFLOW] & 2ull) return eng->fail(WG_ERR_CAPACITY, "solver: more hits in one batch than the hit buffer holds");
    ss.candidates += c[SCNT_CANDIDATES];
    const size_t at = out.size();
    out.resize(at + c[SCNT_HITS]);
    if (c[SCNT_HITS])
        SOLVE_CUDA(cudaMemcpy(out.data() + at, st->hits, sizeof(SolveHitDev) * c[SCNT_HITS], cudaMemcpyDeviceToHost),
                   "copy hits");
    return WG_OK;
}

int finish_hits(std::vector<SolveHitDev> &hits, bool need_start, wg_solve_hit *out, uint64_t cap, uint64_t *n_out,
                wg_solve_stats &ss) {
    std::sort(hits.begin(), hits.end(), [](const SolveHitDev &a, const SolveHitDev &b) {
        if (a.group != b.group) return a.group < b.group;
        if (a.s48 != b.s48) return a.s48 < b.s48;
        if (a.cx != b.cx) return a.cx < b.cx;
        return a.cz < b.cz;
    });
    hits.erase(std::unique(hits.begin(), hits.end(),
                           [](const SolveHitDev &a, const SolveHitDev &b) {
                               return a.group == b.group && a.s48 == b.s48 && a.cx == b.cx && a.cz == b.cz;
                           }),
               hits.end());
    uint64_t n = 0;
    for (const SolveHitDev &h : hits) {
        if (!host_hit_ok(h, need_start)) {
            ss.host_check_failures++;
            continue;
        }
        if (n < cap) std::memcpy(&out[n], &h, sizeof h);
        n++;
    }
    ss.hits = n;
    if (n_out) *n_out = n;
    return WG_OK;
}

}  // namespace

extern "C" int wg_deep_solve(wg_engine *eng, const wg_solve_bundle *bundles, uint64_t n_bundles, uint64_t first_group,
                             uint64_t n_groups, wg_solve_hit *out, uint64_t cap, uint64_t *n_out, wg_solve_stats *stats) {
    if (!eng || !bundles || n_bundles == 0 || (cap && !out)) return WG_ERR_ARG;
    if (first_group + n_groups > (n_bundles << 20) || first_group + n_groups < first_group) return WG_ERR_ARG;
    for (uint64_t b = 0; b < n_bundles; b++) {
        const wg_solve_bundle &B = bundles[b];
        if (B.tier < 1 || B.tier > 3 || B.regime_x < 0 || B.regime_x > 2 || B.regime_z < 0 || B.regime_z > 2)
            return eng->fail(WG_ERR_ARG, "solver: bad bundle (tier 1..3, regimes 0..2)");
    }
    const auto t0 = std::chrono::steady_clock::now();
    SOLVE_CUDA(cudaSetDevice(eng->device), "cudaSetDevice");
    SolveState *st = nullptr;
    int rc = solve_state(eng, &st);
    if (rc) return rc;
    wg_solve_stats ss;
    std::memset(&ss, 0, sizeof ss);
    std::vector<SolveHitDev> hits;
    uint64_t g = first_group;
    const uint64_t g_end = first_group + n_groups;
    int64_t cur_bundle = -1;
    std::vector<int2> offs;
    std::vector<SolveKey> keys;
    std::vector<uint32_t> map;
    while (g < g_end) {
        const uint64_t b = g >> 20;
        const wg_solve_bundle &B = bundles[b];
        if ((int64_t)b != cur_bundle) {
            offs.clear();
            keys.clear();
            tier_offsets(B.tier, offs);
            build_keys(offs, keys, map);
            cur_bundle = (int64_t)b;
        }
        const uint64_t batch_end = std::min<uint64_t>({g_end, (b + 1) << 20, g + kGroupsPerBatch});
        std::vector<SolveSlot> slots;
        std::vector<int2> regions;
        uint64_t tasks = 0;
        for (uint64_t q = g; q < batch_end; q++) {
            SolveSlot sl;
            std::memset(&sl, 0, sizeof sl);
            sl.group = q;
            sl.c20 = perm_group((uint32_t)(q & kM20));
            sl.reg_begin = (uint32_t)regions.size();
            group_regions(sl.c20, B.regime_x, B.regime_z, regions);
            sl.reg_count = (uint32_t)(regions.size() - sl.reg_begin);
            if (!sl.reg_count) continue;   // no task
            sl.off_begin = 0;
            sl.off_count = (uint32_t)offs.size();
            sl.key_begin = 0;
            sl.key_count = (uint32_t)keys.size();
            sl.map_begin = 0;
            sl.list_begin = (uint32_t)(slots.size() * keys.size());
            sl.task_begin = tasks;
            tasks += (uint64_t)sl.reg_count * sl.off_count;
            slots.push_back(sl);
        }
        ss.groups += batch_end - g;
        ss.regions += regions.size();
        ss.tasks += tasks;
        if (!slots.empty()) {
            rc = run_solve_batch(eng, st, B.layout & kM48, slots, keys, map, regions, offs,
                                 (uint32_t)(slots.size() * keys.size()), (uint32_t)keys.size(), tasks, hits, ss);
            if (rc) return rc;
        }
        g = batch_end;
    }
    rc = finish_hits(hits, true, out, cap, n_out, ss);
    ss.wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (stats) *stats = ss;
    return rc;
}

extern "C" int wg_deep_solve_tasks(wg_engine *eng, uint64_t layout, const int32_t *rx, const int32_t *rz,
                                   const int32_t *ox, const int32_t *oz, uint64_t n, wg_solve_hit *out, uint64_t cap,
                                   uint64_t *n_out) {
    if (!eng || (n && (!rx || !rz || !ox || !oz)) || (cap && !out)) return WG_ERR_ARG;
    for (uint64_t i = 0; i < n; i++)
        if (ox[i] < 0 || ox[i] > 23 || oz[i] < 0 || oz[i] > 23 || (ox[i] == 0 && oz[i] == 0) || rx[i] < -kRadius ||
            rx[i] > kRadius || rz[i] < -kRadius || rz[i] > kRadius)
            return eng->fail(WG_ERR_ARG, "solver task: offsets 0..23 (not both 0), regions within +-58593");
    SOLVE_CUDA(cudaSetDevice(eng->device), "cudaSetDevice");
    SolveState *st = nullptr;
    int rc = solve_state(eng, &st);
    if (rc) return rc;
    wg_solve_stats ss;
    std::memset(&ss, 0, sizeof ss);
    std::vector<SolveHitDev> hits;
    for (uint64_t i0 = 0; i0 < n; i0 += 4096) {   // each task is its own slot with one key
        const uint64_t i1 = std::min<uint64_t>(n, i0 + 4096);
        std::vector<SolveSlot> slots;
        std::vector<SolveKey> keys;
        std::vector<uint32_t> map;
        std::vector<int2> regions, offs;
        for (uint64_t i = i0; i < i1; i++) {
            SolveSlot sl;
            std::memset(&sl, 0, sizeof sl);
            const uint32_t k = (uint32_t)(i - i0);
            sl.group = i;
            sl.c20 = (uint32_t)(region_const(rx[i], rz[i]) & kM20);
            sl.reg_begin = k;
            sl.reg_count = 1;
            sl.off_begin = k;
            sl.off_count = 1;
            sl.key_begin = k;
            sl.key_count = 1;
            sl.map_begin = k * 64;
            sl.list_begin = k;
            sl.task_begin = k;
            slots.push_back(sl);
            regions.push_back(make_int2(rx[i], rz[i]));
            offs.push_back(make_int2(ox[i], oz[i]));
            keys.push_back(key_of(rx[i] * 32 + ox[i], rz[i] * 32 + oz[i]));
            map.insert(map.end(), 64, 0u);
        }
        rc = run_solve_batch(eng, st, layout & kM48, slots, keys, map, regions, offs, (uint32_t)slots.size(), 1,
                             slots.size(), hits, ss);
        if (rc) return rc;
    }
    return finish_hits(hits, false, out, cap, n_out, ss);
}
