// Test infrastructure only (the checker, never the product).
//
// The reference's own Deep Dive room walk (engine/gpu/room_core.h, host-callable inline
// functions), compiled from that header where it lies by oracle/Makefile into
// oracle/_ref/libroom_ref.so.  This file only calls the header's functions:
//   rcWalkInit / rcWalkStep / rcWalkK   the incremental region walk (room_core.h:146-175)
//   rcIsStart / rcCarverSeed            the start test of one chunk (room_core.h:34-73)
#include <cmath>
#include <cstdint>

#include "room_core.h"

static RoomCtx make_ctx(int64_t s48) {
    // hut_lookup_v4's makeCtx (engine/gpu/hut_lookup_v4_source.cu:767-773): setSeed + two nextLong
    uint64_t s = ((uint64_t)s48 ^ RC_LCG_MULT) & RC_LCG_MASK;
    auto next = [&](int bits) {
        s = (s * RC_LCG_MULT + RC_LCG_ADD) & RC_LCG_MASK;
        return (int32_t)(s >> (48 - bits));
    };
    auto next_long = [&]() {
        int64_t hi = (int64_t)next(32);
        int64_t lo = (int64_t)next(32);
        return (int64_t)((uint64_t)hi << 32) + lo;
    };
    RoomCtx c;
    c.seed = s48;
    c.a = next_long();
    c.b = next_long();
    c.hiReject = (int32_t)std::ceil(RC_MINESHAFT_P * 67108864.0);
    c.hiAcceptBelow = (int32_t)std::floor(RC_MINESHAFT_P * 67108864.0);
    return c;
}

extern "C" {

int roomh_is_start(int64_t s48, int cx, int cz) {
    const RoomCtx c = make_ctx(s48 & (int64_t)RC_LCG_MASK);
    return rcIsStart(c, cx, cz) ? 1 : 0;
}

// rows of 5 int64: s48, rx, rz, cx, cz; seed-major, rz outer, rx inner (the walker runs along rz
// per rx column, so the rows are gathered per column and emitted in that order afterwards).
long long roomh_walk(const int64_t *s48s, long long n, int rx0, int rx1, int rz0, int rz1, int64_t *out, long long cap) {
    long long found = 0;
    const int rw = rx1 - rx0, rh = rz1 - rz0;
    for (long long i = 0; i < n; i++) {
        const int64_t S = s48s[i] & (int64_t)RC_LCG_MASK;
        const RoomCtx c = make_ctx(S);
        const uint64_t K = rcWalkK(c);
        // start flags per (rz, rx), filled column by column
        unsigned char *flag = new unsigned char[(size_t)rw * rh];
        int32_t *hx = new int32_t[(size_t)rw * rh], *hz = new int32_t[(size_t)rw * rh];
        for (int rx = rx0; rx < rx1; rx++) {
            RoomWalker w;
            rcWalkInit(w, c, rx, rz0);
            for (int rz = rz0; rz < rz1; rz++) {
                int32_t cx, cz;
                const bool st = rcWalkStep(w, c, K, &cx, &cz);
                const size_t k = (size_t)(rz - rz0) * rw + (rx - rx0);
                flag[k] = st;
                hx[k] = cx;
                hz[k] = cz;
            }
        }
        for (int rz = rz0; rz < rz1; rz++)
            for (int rx = rx0; rx < rx1; rx++) {
                const size_t k = (size_t)(rz - rz0) * rw + (rx - rx0);
                if (!flag[k]) continue;
                if (found < cap) {
                    int64_t *o = out + 5 * found;
                    o[0] = S; o[1] = rx; o[2] = rz; o[3] = hx[k]; o[4] = hz[k];
                }
                found++;
            }
        delete[] flag;
        delete[] hx;
        delete[] hz;
    }
    return found;
}

}  // extern "C"
