// Whole-world mineshaft-start counts of the reference's Deep Dive region walk, on the CPU.
//
// Fixture generator only (run by make_golden_sweep.py --cpu, which compiles this file against the
// reference's engine/gpu/room_core.h where it lies): for each structure seed given on the command
// line it walks every hut region of the +-30M world (rx, rz in [-58593, 58593]) with the header's
// rcWalkInit / rcWalkStep, as the reference's sweepProbeKernel does
// (engine/gpu/hut_lookup_v4_source.cu:47-99), and prints
//
//   seed <s48> starts <count>
//   redraw_start <s48> <rx> <rz> <chunk x> <chunk z>     one per start whose region re-draws nextInt(24)
//
// The header's exact hut placement (rcHutExact, room_core.h:86-105) tests its re-draw condition in
// signed 32-bit arithmetic that overflows exactly when a re-draw is due; built with plain -O2 the
// compiler may assume no overflow and drop the loop, built with -fwrapv the loop runs as in
// java.util.Random.nextInt.  The generator builds this file both ways.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "room_core.h"

namespace {

// java.util.Random: setSeed(s48), then two nextLong() draws (the carver's a and b).
RoomCtx make_ctx(int64_t s48) {
    uint64_t s = ((uint64_t)s48 ^ RC_LCG_MULT) & RC_LCG_MASK;
    auto next32 = [&]() {
        s = (s * RC_LCG_MULT + RC_LCG_ADD) & RC_LCG_MASK;
        return (int64_t)(int32_t)(uint32_t)(s >> 16);
    };
    RoomCtx c;
    c.seed = s48;
    const int64_t a_hi = next32(), a_lo = next32();
    c.a = (int64_t)((uint64_t)a_hi << 32) + a_lo;
    const int64_t b_hi = next32(), b_lo = next32();
    c.b = (int64_t)((uint64_t)b_hi << 32) + b_lo;
    c.hiReject = (int32_t)std::ceil(RC_MINESHAFT_P * 67108864.0);
    c.hiAcceptBelow = (int32_t)std::floor(RC_MINESHAFT_P * 67108864.0);
    return c;
}

// True when one of the region's two nextInt(24) draws is re-drawn by java.util.Random.
bool redraws(uint64_t region_seed) {
    uint64_t s = (region_seed ^ RC_LCG_MULT) & RC_LCG_MASK;
    bool any = false;
    for (int k = 0; k < 2; k++) {
        s = (s * RC_LCG_MULT + RC_LCG_ADD) & RC_LCG_MASK;
        any |= (uint32_t)(s >> 17) >= 2147483640u;
    }
    return any;
}

struct Hit {
    int rx, rz, cx, cz;
};

}  // namespace

int main(int argc, char **argv) {
    const int radius = 58593;
    for (int q = 1; q < argc; q++) {
        const int64_t s48 = (int64_t)(std::strtoull(argv[q], nullptr, 10) & RC_LCG_MASK);
        const RoomCtx c = make_ctx(s48);
        const uint64_t K = rcWalkK(c);
        long long total = 0;
        std::vector<Hit> hits;
#pragma omp parallel for reduction(+ : total) schedule(dynamic, 64)
        for (int rx = -radius; rx <= radius; rx++) {
            RoomWalker w;
            rcWalkInit(w, c, rx, -radius);
            for (int rz = -radius; rz <= radius; rz++) {
                const uint64_t rs = w.rs;
                int32_t cx, cz;
                if (!rcWalkStep(w, c, K, &cx, &cz)) continue;
                total++;
                if (redraws(rs)) {
#pragma omp critical
                    hits.push_back(Hit{rx, rz, cx, cz});
                }
            }
        }
        std::printf("seed %lld starts %lld\n", (long long)s48, total);
        for (const Hit &h : hits) std::printf("redraw_start %lld %d %d %d %d\n", (long long)s48, h.rx, h.rz, h.cx, h.cz);
        std::fflush(stdout);
    }
    return 0;
}
