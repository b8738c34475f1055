// Deep Dive (mineshaft starts under swamp huts): the structure-side primitives shared by the room
// walk kernel (wg_deep.cu) and the host code (the spot check of wg_deep_spots).
//
// A mineshaft starts in chunk (cx, cz) of structure seed S when, after setLargeFeatureSeed
// (setSeed(S); a = nextLong(); b = nextLong(); setSeed(cx * a ^ cz * b ^ S)), nextDouble() < 0.004
// (engine/gpu/room_core.h:34-73).  Everything here depends on the seed's low 48 bits only.
#pragma once

#include <cstdint>

namespace wg {

constexpr uint64_t kDeepMask48 = 0xFFFFFFFFFFFFull;
constexpr uint64_t kDeepMul = 0x5DEECE66Dull;
constexpr double kMineshaftP = 0.004;

// (a, b): the two nextLong() draws of setSeed(S).
struct DeepCtx {
    uint64_t s48;
    int64_t a, b;
};

__host__ __device__ __forceinline__ uint64_t deep_step(uint64_t s) { return (s * kDeepMul + 0xBull) & kDeepMask48; }

__host__ __device__ __forceinline__ int64_t deep_next_long(uint64_t &s) {
    s = deep_step(s);
    const uint64_t hi = (uint64_t)(uint32_t)(int32_t)(s >> 16);
    s = deep_step(s);
    const int64_t lo = (int64_t)(int32_t)(uint32_t)(s >> 16);
    return (int64_t)((hi << 32) + (uint64_t)lo);
}

__host__ __device__ __forceinline__ DeepCtx deep_ctx(uint64_t s48) {
    DeepCtx c;
    c.s48 = s48 & kDeepMask48;
    uint64_t s = (c.s48 ^ kDeepMul) & kDeepMask48;
    c.a = deep_next_long(s);
    c.b = deep_next_long(s);
    return c;
}

// setLargeFeatureSeed state of chunk (cx, cz), 48 bits.
__host__ __device__ __forceinline__ uint64_t deep_carver(const DeepCtx &c, int32_t cx, int32_t cz) {
    return ((uint64_t)((int64_t)cx * c.a) ^ (uint64_t)((int64_t)cz * c.b) ^ c.s48) & kDeepMask48;
}

// nextDouble() < 0.004 after setSeed(carver): ((next(26) << 27) + next(27)) * 2^-53.
__host__ __device__ __forceinline__ bool deep_is_start(uint64_t carver) {
    uint64_t s = (carver ^ kDeepMul) & kDeepMask48;
    s = deep_step(s);
    const int64_t hi = (int64_t)(s >> 22);
    s = deep_step(s);
    const int64_t lo = (int64_t)(s >> 21);
    return (double)((hi << 27) + lo) * 1.1102230246251565404e-16 < kMineshaftP;
}

}  // namespace wg
