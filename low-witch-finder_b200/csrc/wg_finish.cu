// The mineshaft finisher (hunt.py finish_row, hunt.py:277-333) for a batch of Deep Dive
// survivors on the GPU: per survivor (world seed, hut chunk) the hut's phase-2 verdict at the
// ceiling 100, the mineshaft's piece tree (mstree), the hut floor once the mineshaft's room and
// tunnels are carved into the chunk (msroom's EXACT line), the footprint scan (skyscan --list) and
// the deep-dark test at the room floor (biome_at --ms).
//
// Reference tools restated here, by file:
//   engine/tools/mstree/mstree.cpp:10-54, mineshaft_tree.h, mineshaft_tree_iter.h
//        start test, MineShaftPieces generation (depth first, the iterative runner's child
//        order), the move below sea level, the piece list mstree prints
//   engine/tools/mineshaft/mineshaft_carve.h:1-238, msroom.c:84-170
//        the carving model of the pieces in the hut's chunk (fills, the room's dome, floor
//        planks, pillars, rails, the liquid guard) and the footprint heights
//   engine/tools/mineshaft/skyscan.c:26-58   the footprint scan of --list mode
//   engine/tools/mineshaft/biome_at.c:31-39  the biome at the room floor (--ms)
//
// Work layout: one thread per survivor builds its tree (a few hundred java.util.Random draws and
// overlap tests against at most 512 boxes; survivors are rare, so this is not the cost); the
// phase-2 chunk state (the same kernels as wg_eval_huts: world tables, grid, aquifer, block
// states, carvers) gives the block state after carvers of every block of the hut's chunk; one
// CTA per (survivor, carving pass) applies the pieces to a 16 x 16 x 140 block window in shared
// memory, each piece's boxes filled by all threads.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <map>
#include <vector>

#include "../../include/witchgpu.h"
#include "wg_engine_impl.h"
#include "wg_phase2.cuh"

namespace wg {
namespace {

// ------------------------------------------------------------------------------------
// The piece tree (mstree)
// ------------------------------------------------------------------------------------
constexpr int kMsMaxPieces = 512;   // pieces per tree (the reference's MT_MAXP)
constexpr int kMsMaxFrames = 16;    // open pieces on the generation stack (its MT_MAXF)
constexpr uint64_t kMsMul = 0x5DEECE66Dull, kMsMask = 0xFFFFFFFFFFFFull;

enum : int { MS_ROOM = 0, MS_CORRIDOR = 1, MS_CROSSING = 2, MS_STAIRS = 3 };
enum : int { MS_N = 0, MS_S = 1, MS_W = 2, MS_E = 3 };
// tree status (mineshaft_tree_iter.h mtRunFinish): generated, or not a start / out of range
enum : int { MS_OK = 0, MS_NOT_START = 1, MS_TOO_LARGE = 2 };

struct MsPiece {
    int x0, y0, z0, x1, y1, z1;
    int type, facing, depth, rails, parent;
};

// java.util.Random over a 48-bit state.
struct JRand {
    uint64_t s;
    __device__ int next(int bits) {
        s = (s * kMsMul + 0xBull) & kMsMask;
        return (int)(int64_t)(s >> (48 - bits));
    }
    __device__ int next_int(int bound) {
        if ((bound & -bound) == bound) return (int)(((int64_t)bound * (int64_t)next(31)) >> 31);
        for (;;) {
            const int bits = next(31), val = bits % bound;
            if ((int32_t)((uint32_t)bits - (uint32_t)val + (uint32_t)(bound - 1)) >= 0) return val;
        }
    }
    __device__ bool next_bool() { return next(1) != 0; }
    __device__ int64_t next_long() {
        const int64_t hi = (int64_t)next(32);
        const int64_t lo = (int64_t)next(32);
        return (int64_t)((uint64_t)hi << 32) + lo;
    }
};

// A child request: the corner (i, j, k) a new piece grows from, its direction and the parent's depth.
struct MsReq {
    int i, j, k, dir, depth;
};

// An open piece on the stack and where its child enumeration stands.
struct MsFrame {
    int x0, y0, z0, x1, y1, z1;
    int type, facing, depth, idx;
    int phase, k, side, jj;
};

struct MsTree {
    JRand r;
    MsPiece *p;       // this tree's piece array (global memory)
    int n, sx, sz, min_y, max_y, too_large;
};

__device__ __forceinline__ bool fits8(int v) { return v >= -128 && v <= 127; }

// Whether box b overlaps a piece already placed (inclusive bounds).  The reference packs piece
// coordinates relative to the room corner (sx, 50, sz) into bytes and calls a tree whose boxes do
// not fit out of range; the same test is kept so that such trees are reported, not answered.
__device__ bool ms_overlaps(MsTree &t, int x0, int y0, int z0, int x1, int y1, int z1) {
    if (!(fits8(x0 - t.sx) && fits8(z0 - t.sz) && fits8(x1 - t.sx) && fits8(z1 - t.sz) && fits8(y0 - 50) &&
          fits8(y1 - 50))) {
        t.too_large = 1;
        return false;
    }
    for (int q = t.n - 1; q >= 0; q--) {
        const MsPiece &a = t.p[q];
        if (a.x1 >= x0 && a.x0 <= x1 && a.z1 >= z0 && a.z0 <= z1 && a.y1 >= y0 && a.y0 <= y1) return true;
    }
    return false;
}

__device__ void ms_push(MsTree &t, const MsPiece &a) {
    if (!(fits8(a.x0 - t.sx) && fits8(a.z0 - t.sz) && fits8(a.x1 - t.sx) && fits8(a.z1 - t.sz) && fits8(a.y0 - 50) &&
          fits8(a.y1 - 50)))
        t.too_large = 1;
    t.p[t.n++] = a;
    t.min_y = min(t.min_y, a.y0);
    t.max_y = max(t.max_y, a.y1);
}

__device__ MsFrame ms_frame(const MsPiece &p, int idx) {
    MsFrame f;
    f.x0 = p.x0;
    f.y0 = p.y0;
    f.z0 = p.z0;
    f.x1 = p.x1;
    f.y1 = p.y1;
    f.z1 = p.z1;
    f.type = p.type;
    f.facing = p.facing;
    f.depth = p.depth;
    f.idx = idx;
    f.phase = f.k = f.side = 0;
    const int j = (p.y1 - p.y0 + 1) - 3 - 1;
    f.jj = j <= 0 ? 1 : j;
    return f;
}

__device__ __forceinline__ MsReq ms_req(int i, int j, int k, int dir, int depth) { return MsReq{i, j, k, dir, depth}; }

// The next child request of an open piece (MineShaftRoom / Corridor / Crossing / Stairs
// addChildren, one request per call, drawing exactly the random numbers the recursive form draws
// before each child), or false when the piece has no more.
__device__ bool ms_next_child(MsTree &t, MsFrame &f, MsReq &r) {
    switch (f.type) {
        case MS_STAIRS: {
            if (f.phase) return false;
            f.phase = 1;
            switch (f.facing) {
                case MS_S: r = ms_req(f.x0, f.y0, f.z1 + 1, MS_S, f.depth); break;
                case MS_W: r = ms_req(f.x0 - 1, f.y0, f.z0, MS_W, f.depth); break;
                case MS_E: r = ms_req(f.x1 + 1, f.y0, f.z0, MS_E, f.depth); break;
                default: r = ms_req(f.x0, f.y0, f.z0 - 1, MS_N, f.depth); break;
            }
            return true;
        }
        case MS_CROSSING: {
            while (f.phase < 7) {
                const int ph = f.phase++;
                if (ph < 3) {
                    // three exits at floor level: ahead and to both sides of the entry direction
                    const int fwd_n = f.z0 - 1, fwd_s = f.z1 + 1, side_w = f.x0 - 1, side_e = f.x1 + 1;
                    int i = f.x0 + 1, k = f.z0 + 1, dir = MS_N;
                    switch (f.facing) {
                        case MS_S:
                            if (ph == 0) { i = f.x0 + 1; k = fwd_s; dir = MS_S; }
                            else if (ph == 1) { i = side_w; k = f.z0 + 1; dir = MS_W; }
                            else { i = side_e; k = f.z0 + 1; dir = MS_E; }
                            break;
                        case MS_W:
                            if (ph == 0) { i = f.x0 + 1; k = fwd_n; dir = MS_N; }
                            else if (ph == 1) { i = f.x0 + 1; k = fwd_s; dir = MS_S; }
                            else { i = side_w; k = f.z0 + 1; dir = MS_W; }
                            break;
                        case MS_E:
                            if (ph == 0) { i = f.x0 + 1; k = fwd_n; dir = MS_N; }
                            else if (ph == 1) { i = f.x0 + 1; k = fwd_s; dir = MS_S; }
                            else { i = side_e; k = f.z0 + 1; dir = MS_E; }
                            break;
                        default:
                            if (ph == 0) { i = f.x0 + 1; k = fwd_n; dir = MS_N; }
                            else if (ph == 1) { i = side_w; k = f.z0 + 1; dir = MS_W; }
                            else { i = side_e; k = f.z0 + 1; dir = MS_E; }
                            break;
                    }
                    r = ms_req(i, f.y0, k, dir, f.depth);
                    return true;
                }
                if (f.y1 - f.y0 + 1 <= 3) {   // a one-storey crossing has no upper exits
                    f.phase = 7;
                    return false;
                }
                if (!t.r.next_bool()) continue;
                const int q = ph - 3, y = f.y0 + 3 + 1;
                if (q == 0) r = ms_req(f.x0 + 1, y, f.z0 - 1, MS_N, f.depth);
                else if (q == 1) r = ms_req(f.x0 - 1, y, f.z0 + 1, MS_W, f.depth);
                else if (q == 2) r = ms_req(f.x1 + 1, y, f.z0 + 1, MS_E, f.depth);
                else r = ms_req(f.x0 + 1, y, f.z1 + 1, MS_S, f.depth);
                return true;
            }
            return false;
        }
        case MS_CORRIDOR: {
            const bool along_x = f.facing == MS_W || f.facing == MS_E;
            if (f.phase == 0) {   // the corridor's continuation: ahead (j <= 1) or turning
                const int j = t.r.next_int(4);
                const int y = f.y0 - 1 + t.r.next_int(3);
                int i, k, dir;
                switch (f.facing) {
                    case MS_S:
                        if (j <= 1) { i = f.x0; k = f.z1 + 1; dir = MS_S; }
                        else if (j == 2) { i = f.x0 - 1; k = f.z1 - 3; dir = MS_W; }
                        else { i = f.x1 + 1; k = f.z1 - 3; dir = MS_E; }
                        break;
                    case MS_W:
                        if (j <= 1) { i = f.x0 - 1; k = f.z0; dir = MS_W; }
                        else if (j == 2) { i = f.x0; k = f.z0 - 1; dir = MS_N; }
                        else { i = f.x0; k = f.z1 + 1; dir = MS_S; }
                        break;
                    case MS_E:
                        if (j <= 1) { i = f.x1 + 1; k = f.z0; dir = MS_E; }
                        else if (j == 2) { i = f.x1 - 3; k = f.z0 - 1; dir = MS_N; }
                        else { i = f.x1 - 3; k = f.z1 + 1; dir = MS_S; }
                        break;
                    default:
                        if (j <= 1) { i = f.x0; k = f.z0 - 1; dir = MS_N; }
                        else if (j == 2) { i = f.x0 - 1; k = f.z0; dir = MS_W; }
                        else { i = f.x1 + 1; k = f.z0; dir = MS_E; }
                        break;
                }
                r = ms_req(i, y, k, dir, f.depth);
                f.phase = 1;
                return true;
            }
            if (f.phase == 1) {   // then side branches every 5 blocks, while the depth allows
                if (f.depth >= 8) {
                    f.phase = 9;
                    return false;
                }
                f.k = (along_x ? f.x0 : f.z0) + 3;
            } else if (f.phase == 2) {
                f.k += 5;
            } else {
                return false;
            }
            const int lim = along_x ? f.x1 : f.z1;
            while (f.k + 3 <= lim) {
                const int l = t.r.next_int(5);
                if (l <= 1) {
                    if (along_x) r = ms_req(f.k, f.y0, l == 0 ? f.z0 - 1 : f.z1 + 1, l == 0 ? MS_N : MS_S, f.depth + 1);
                    else r = ms_req(l == 0 ? f.x0 - 1 : f.x1 + 1, f.y0, f.k, l == 0 ? MS_W : MS_E, f.depth + 1);
                    f.phase = 2;
                    return true;
                }
                f.k += 5;
            }
            f.phase = 9;
            return false;
        }
        default: {   // the room: exits along its four walls at random offsets and heights
            const int xs = f.x1 - f.x0 + 1, zs = f.z1 - f.z0 + 1;
            while (f.side < 4) {
                const int span = f.side < 2 ? xs : zs;
                if (f.phase == 0) f.k = 0;
                else f.k += 4;
                if (f.k >= span) {
                    f.side++;
                    f.phase = 0;
                    continue;
                }
                f.k += t.r.next_int(span);
                if (f.k + 3 > span) {
                    f.side++;
                    f.phase = 0;
                    continue;
                }
                const int y = f.y0 + t.r.next_int(f.jj) + 1;
                switch (f.side) {
                    case 0: r = ms_req(f.x0 + f.k, y, f.z0 - 1, MS_N, f.depth); break;
                    case 1: r = ms_req(f.x0 + f.k, y, f.z1 + 1, MS_S, f.depth); break;
                    case 2: r = ms_req(f.x0 - 1, y, f.z0 + f.k, MS_W, f.depth); break;
                    default: r = ms_req(f.x1 + 1, y, f.z0 + f.k, MS_E, f.depth); break;
                }
                f.phase = 1;
                return true;
            }
            return false;
        }
    }
}

// The piece a child request makes, or false (MineShaftPieces.generateAndAddPiece: depth <= 8,
// within 80 blocks of the room corner; 80 % corridor, 10 % stairs, 20 % crossing by nextInt(100),
// each fitted to the first of its candidate boxes that overlaps no placed piece).
__device__ bool ms_attempt(MsTree &t, const MsReq &q, MsPiece &np) {
    if (!(q.depth <= 8 && abs(q.i - t.sx) <= 80 && abs(q.k - t.sz) <= 80)) return false;
    const int i = q.i, j = q.j, k = q.k, dir = q.dir;
    np.depth = q.depth + 1;
    np.facing = dir;
    np.rails = 0;
    const int m = t.r.next_int(100);
    int x0 = i, y0 = j, z0 = k, x1 = i, y1 = j + 2, z1 = k;
    if (m >= 80) {   // crossing, one or two storeys
        np.type = MS_CROSSING;
        if (t.r.next_int(4) == 0) y1 += 4;
        switch (dir) {
            case MS_S: x0 = i - 1; x1 = i + 3; z1 = k + 4; break;
            case MS_W: x0 = i - 4; z0 = k - 1; z1 = k + 3; break;
            case MS_E: x1 = i + 4; z0 = k - 1; z1 = k + 3; break;
            default: x0 = i - 1; x1 = i + 3; z0 = k - 4; break;
        }
        if (ms_overlaps(t, x0, y0, z0, x1, y1, z1)) return false;
    } else if (m >= 70) {   // stairs: 9 long, down 5
        np.type = MS_STAIRS;
        y0 = j - 5;
        switch (dir) {
            case MS_S: x1 = i + 2; z1 = k + 8; break;
            case MS_W: x0 = i - 8; z1 = k + 2; break;
            case MS_E: x1 = i + 8; z1 = k + 2; break;
            default: x1 = i + 2; z0 = k - 8; break;
        }
        if (ms_overlaps(t, x0, y0, z0, x1, y1, z1)) return false;
    } else {   // corridor: the longest of 5 * (2..4) blocks that fits
        np.type = MS_CORRIDOR;
        int len;
        for (len = t.r.next_int(3) + 2; len > 0; --len) {
            const int mm = len * 5;
            switch (dir) {
                case MS_S: x1 = i + 2; z1 = k + mm - 1; break;
                case MS_W: x0 = i - (mm - 1); z1 = k + 2; break;
                case MS_E: x1 = i + mm - 1; z1 = k + 2; break;
                default: x1 = i + 2; z0 = k - (mm - 1); break;
            }
            if (!ms_overlaps(t, x0, y0, z0, x1, y1, z1)) break;
        }
        if (len <= 0) return false;
        np.rails = t.r.next_int(3) == 0 ? 1 : 0;
        if (!np.rails) (void)t.r.next_int(23);   // the spider-corridor draw
    }
    np.x0 = x0;
    np.y0 = y0;
    np.z0 = z0;
    np.x1 = x1;
    np.y1 = y1;
    np.z1 = z1;
    return true;
}

// True when the carver state X (setLargeFeatureSeed of the chunk) starts a mineshaft:
// nextDouble() < 0.004 (mstree.cpp:10-15).
__device__ bool ms_start(uint64_t X) {
    uint64_t s = (X ^ kMsMul) & kMsMask;
    s = (s * kMsMul + 0xBull) & kMsMask;
    const uint64_t a = s >> 22;
    s = (s * kMsMul + 0xBull) & kMsMask;
    const uint64_t b = s >> 21;
    return (double)((a << 27) + b) * 1.1102230246251565e-16 < 0.004;
}

struct MsInfo {
    int status, n, floor, pad;
};

// One thread per survivor: the start test, then the tree generated depth first from the room
// (mineshaft_tree_iter.h mtRunInit / mtRunStep / mtRunFinish), then every piece moved down so the
// tree lies below sea level (StructurePiecesBuilder.moveBelowSeaLevel(63, -64, random, 10)).
__global__ void ms_tree_kernel(const int64_t *__restrict__ ws, const int32_t *__restrict__ cxs,
                               const int32_t *__restrict__ czs, int n, MsPiece *__restrict__ pieces,
                               MsInfo *__restrict__ info) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    MsInfo &out = info[row];
    out.n = 0;
    out.floor = 0;
    const uint64_t s48 = (uint64_t)ws[row] & kMsMask;
    const int cx = cxs[row], cz = czs[row];
    JRand jr{(s48 ^ kMsMul) & kMsMask};
    const int64_t a = jr.next_long(), b = jr.next_long();
    const uint64_t X = (uint64_t)(((int64_t)cx * a) ^ ((int64_t)cz * b) ^ (int64_t)s48) & kMsMask;
    if (!ms_start(X)) {
        out.status = MS_NOT_START;
        return;
    }
    MsTree t;
    t.r.s = (X ^ kMsMul) & kMsMask;
    t.p = pieces + (size_t)row * kMsMaxPieces;
    t.n = 0;
    t.too_large = 0;
    t.min_y = INT_MAX;
    t.max_y = INT_MIN;
    (void)t.r.next(26);   // the start test's nextDouble
    (void)t.r.next(27);
    MsPiece room;
    room.type = MS_ROOM;
    room.facing = -1;
    room.depth = 0;
    room.rails = 0;
    room.parent = -1;
    room.x0 = cx * 16 + 2;
    room.y0 = 50;
    room.z0 = cz * 16 + 2;
    room.x1 = room.x0 + 7 + t.r.next_int(6);
    room.y1 = 54 + t.r.next_int(6);
    room.z1 = room.z0 + 7 + t.r.next_int(6);
    t.sx = room.x0;
    t.sz = room.z0;
    ms_push(t, room);
    MsFrame st[kMsMaxFrames];
    int sp = 0;
    st[sp++] = ms_frame(room, 0);
    bool failed = false;
    while (sp > 0) {
        MsFrame &f = st[sp - 1];
        MsReq q;
        if (!ms_next_child(t, f, q)) {
            --sp;
            continue;
        }
        MsPiece np;
        if (!ms_attempt(t, q, np)) continue;
        if (t.n >= kMsMaxPieces || sp >= kMsMaxFrames) {
            failed = true;
            break;
        }
        np.parent = f.idx;
        ms_push(t, np);
        st[sp] = ms_frame(np, t.n - 1);
        sp++;
    }
    if (failed || t.too_large) {
        out.status = MS_TOO_LARGE;
        out.n = t.n;
        return;
    }
    const int span = t.max_y - t.min_y + 1;
    int l = span - 64 + 1;
    if (l < 53) l += t.r.next_int(53 - l);
    const int m = l - t.max_y;
    for (int q = 0; q < t.n; q++) {
        t.p[q].y0 += m;
        t.p[q].y1 += m;
    }
    out.status = MS_OK;
    out.n = t.n;
    out.floor = 50 + m;
}

// ------------------------------------------------------------------------------------
// Carving the pieces into the hut's chunk (msroom)
// ------------------------------------------------------------------------------------
// The block window of the carving model: the chunk's 16 x 16 columns, y -64 .. 75
// (mineshaft_carve.h MC_Y0 / MC_YN); outside it every block keeps its state after carvers.
constexpr int kMcY0 = -64, kMcYN = 140, kMcTop = kMcY0 + kMcYN - 1;
constexpr int kMcCells = 16 * 16 * kMcYN;
// Window cell values: untouched, carved to air, a placed solid block (plank or pillar), a rail.
enum : uint8_t { MC_NATURAL = 0, MC_CARVED = 1, MC_PLACED = 2, MC_RAIL = 3 };
// Block states the model reads (msroom.c natcb plus the rail): solid, air, water, lava, rail.
enum : int { ST_SOLID = 0, ST_AIR = 1, ST_WATER = 2, ST_LAVA = 3, ST_RAIL = 4 };
constexpr int kCarveThreads = 256;
constexpr int kFootW = 7, kFootD = 9;   // the footprint finish_row measures (MC_SHAPE=79: 7 x 9)

// Block state after the carvers of block (x, y, z) of the job's chunk (lysh carved_state_at).
__device__ __forceinline__ int natural_state(const P2Chunk &J, int x, int y, int z) {
    if (y < -64 || y > 319) return ST_AIR;   // outside the chunk's 384 levels (never read by the model)
    const int ci = ((z & 15) << 4) | (x & 15) | ((y + 64) << 8);
    const uint8_t cv = J.cells[ci];
    return cv != CV_UNCHANGED ? (int)cv : (int)(J.states[ci] & 15u);
}

struct McWin {
    uint8_t *w;           // kMcCells window values (shared memory)
    const P2Chunk *J;
    int cx0, cz0;
    __device__ __forceinline__ int index(int x, int y, int z) const {
        return ((x - cx0) * 16 + (z - cz0)) * kMcYN + (y - kMcY0);
    }
    __device__ __forceinline__ bool inside(int x, int y, int z) const {
        return x >= cx0 && x <= cx0 + 15 && z >= cz0 && z <= cz0 + 15 && y >= kMcY0 && y <= kMcTop;
    }
    __device__ int state(int x, int y, int z) const {
        if (inside(x, y, z)) {
            const uint8_t v = w[index(x, y, z)];
            if (v == MC_PLACED) return ST_SOLID;
            if (v == MC_RAIL) return ST_RAIL;
            if (v == MC_CARVED) return ST_AIR;
        }
        return natural_state(*J, x, y, z);
    }
    __device__ bool liquid(int x, int y, int z) const {
        const int s = state(x, y, z);
        return s == ST_WATER || s == ST_LAVA;
    }
    // a solid block in column (x, z) from y up to the window's top (mc_solidFrom)
    __device__ bool solid_from(int x, int y, int z) const {
        for (int yy = max(y, kMcY0); yy <= kMcTop; yy++)
            if (state(x, yy, z) == ST_SOLID) return true;
        return false;
    }
    __device__ void place(int x, int y, int z) {
        if (inside(x, y, z)) w[index(x, y, z)] = MC_PLACED;
    }
};

// Every cell of box (x0..x1, y0..y1, z0..z1), clipped to the window, carved to air; the CTA's
// threads share the cells.  Called by all threads.
__device__ void mc_fill(McWin &M, int x0, int y0, int z0, int x1, int y1, int z1) {
    x0 = max(x0, M.cx0);
    z0 = max(z0, M.cz0);
    x1 = min(x1, M.cx0 + 15);
    z1 = min(z1, M.cz0 + 15);
    y0 = max(y0, kMcY0);
    y1 = min(y1, kMcTop);
    if (x1 < x0 || y1 < y0 || z1 < z0) return;
    const int nx = x1 - x0 + 1, ny = y1 - y0 + 1, nz = z1 - z0 + 1;
    for (int q = threadIdx.x; q < nx * ny * nz; q += blockDim.x) {
        const int y = y0 + q % ny, z = z0 + (q / ny) % nz, x = x0 + q / (ny * nz);
        M.w[M.index(x, y, z)] = MC_CARVED;
    }
}

// True (in every thread) when a face of the box grown by one block, clipped to the chunk and to
// y -64 .. 319, touches water or lava (mc_guard; StructurePiece.isInInvalidLocation).
__device__ bool mc_guard(const McWin &M, const MsPiece &p) {
    const int i = max(p.x0 - 1, M.cx0), j = max(p.y0 - 1, -64), k = max(p.z0 - 1, M.cz0);
    const int l = min(p.x1 + 1, M.cx0 + 15), m = min(p.y1 + 1, 319), n = min(p.z1 + 1, M.cz0 + 15);
    const int ax = l - i + 1, ay = m - j + 1, az = n - k + 1;
    const int fa = ax * az, fb = ax * ay, fc = az * ay;   // per face pair: y-faces, z-faces, x-faces
    int hit = 0;
    for (int q = threadIdx.x; q < 2 * (fa + fb + fc) && !hit; q += blockDim.x) {
        int r = q;
        if (r < 2 * fa) {
            const int o = i + (r >> 1) / az, pz = k + (r >> 1) % az;
            hit = M.liquid(o, (r & 1) ? m : j, pz);
        } else if ((r -= 2 * fa) < 2 * fb) {
            const int o = i + (r >> 1) / ay, py = j + (r >> 1) % ay;
            hit = M.liquid(o, py, (r & 1) ? n : k);
        } else {
            r -= 2 * fb;
            const int o = k + (r >> 1) / ay, py = j + (r >> 1) % ay;
            hit = M.liquid((r & 1) ? l : i, py, o);
        }
    }
    return __syncthreads_or(hit) != 0;
}

// Floor planks under a piece (mc_floorFill): in each of the piece's columns inside the chunk, an
// air block under the floor gets a plank when the column has a solid block at or above the floor.
__device__ void mc_floor(McWin &M, const MsPiece &p) {
    const int x0 = max(p.x0, M.cx0), x1 = min(p.x1, M.cx0 + 15), z0 = max(p.z0, M.cz0), z1 = min(p.z1, M.cz0 + 15);
    if (x1 < x0 || z1 < z0) return;
    const int nz = z1 - z0 + 1;
    for (int q = threadIdx.x; q < (x1 - x0 + 1) * nz; q += blockDim.x) {
        const int x = x0 + q / nz, z = z0 + q % nz;
        if (M.state(x, p.y0 - 1, z) == ST_AIR && M.solid_from(x, p.y0, z)) M.place(x, p.y0 - 1, z);
    }
}

// Rails along a corridor's middle (mc_rails, top layer 0): where the block under the floor is
// solid and the floor block is air.
__device__ void mc_rails(McWin &M, const MsPiece &p) {
    const bool along_z = (p.x1 - p.x0) == 2;
    const int n = along_z ? p.z1 - p.z0 + 1 : p.x1 - p.x0 + 1;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int x = along_z ? p.x0 + 1 : p.x0 + i, z = along_z ? p.z0 + i : p.z0 + 1;
        if (x < M.cx0 || x > M.cx0 + 15 || z < M.cz0 || z > M.cz0 + 15) continue;
        if (M.state(x, p.y0 - 1, z) != ST_SOLID) continue;
        if (M.state(x, p.y0, z) == ST_AIR && M.inside(x, p.y0, z)) M.w[M.index(x, p.y0, z)] = MC_RAIL;
    }
}

// The room's dome above its 3-block floor layer: the cells of the ellipsoid
// dx^2 + dy^2 + dz^2 <= 1.05 in float arithmetic (the model's mc_dome_eps), carved.
__device__ void mc_dome(McWin &M, const MsPiece &p) {
    const float W = (float)(p.x1 - p.x0 + 1), H = (float)(p.y1 - (p.y0 + 4) + 1), D = (float)(p.z1 - p.z0 + 1);
    const float cx = __fadd_rn(__int2float_rn(p.x0), __fdiv_rn(W, 2.0f));
    const float cz = __fadd_rn(__int2float_rn(p.z0), __fdiv_rn(D, 2.0f));
    const float hw = __fmul_rn(W, 0.5f), hd = __fmul_rn(D, 0.5f);
    const int ny = p.y1 - (p.y0 + 4) + 1, nx = p.x1 - p.x0 + 1, nz = p.z1 - p.z0 + 1;
    if (ny <= 0) return;
    for (int q = threadIdx.x; q < ny * nx * nz; q += blockDim.x) {
        const int y = p.y0 + 4 + q / (nx * nz), x = p.x0 + (q / nz) % nx, z = p.z0 + q % nz;
        const float dy = __fdiv_rn((float)(y - (p.y0 + 4)), H);
        const float dx = __fdiv_rn(__fsub_rn(__int2float_rn(x), cx), hw);
        const float dz = __fdiv_rn(__fsub_rn(__int2float_rn(z), cz), hd);
        const float r2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
        if (r2 <= 1.05f && M.inside(x, y, z)) M.w[M.index(x, y, z)] = MC_CARVED;
    }
}

// One carving pass of one survivor: the pieces applied in order to the chunk's window with the top
// layer 0 or 1 and the liquid guard on or off (msroom.c:131-163), then the footprint's surface
// heights (mc_height: the highest block that is not air, plus one) summed.
// Pass p of row r: top = p & 1, guard = !(p >> 1).  Out: [row][pass] = (height sum, refused).
__global__ void __launch_bounds__(kCarveThreads) ms_carve_kernel(const P2Chunk *__restrict__ jobs,
                                                                 const int32_t *__restrict__ job_of,
                                                                 const int32_t *__restrict__ hx,
                                                                 const int32_t *__restrict__ hz,
                                                                 const MsPiece *__restrict__ pieces,
                                                                 const MsInfo *__restrict__ info,
                                                                 long long *__restrict__ sums,
                                                                 int32_t *__restrict__ refused) {
    extern __shared__ uint8_t win[];
    __shared__ long long hsum;
    __shared__ int nref;
    const int row = blockIdx.x >> 2, pass = blockIdx.x & 3;
    const int top = pass & 1;
    const bool guard = (pass >> 1) == 0;
    if (info[row].status != MS_OK) {
        if (threadIdx.x == 0) {
            sums[blockIdx.x] = 0;
            refused[blockIdx.x] = 0;
        }
        return;
    }
    McWin M;
    M.w = win;
    M.J = &jobs[job_of[row]];
    M.cx0 = hx[row] & ~15;
    M.cz0 = hz[row] & ~15;
    for (int q = threadIdx.x; q < kMcCells; q += blockDim.x) win[q] = MC_NATURAL;
    if (threadIdx.x == 0) {
        hsum = 0;
        nref = 0;
    }
    __syncthreads();
    const MsPiece *pc = pieces + (size_t)row * kMsMaxPieces;
    const int n = info[row].n;
    for (int idx = 0; idx < n; idx++) {
        const MsPiece p = pc[idx];
        if (p.x1 < M.cx0 || p.x0 > M.cx0 + 15 || p.z1 < M.cz0 || p.z0 > M.cz0 + 15) continue;
        if (guard && mc_guard(M, p)) {
            if (threadIdx.x == 0) nref++;
            __syncthreads();
            continue;
        }
        const bool two_storey = p.y1 - p.y0 + 1 > 3;
        switch (p.type) {
            case MS_ROOM: {
                mc_fill(M, p.x0, p.y0 + 1, p.z0, p.x1, min(p.y0 + 3, p.y1), p.z1);
                // each direct child's entrance through the room's wall (the top 3 layers of the child)
                for (int c = 1; c < n; c++) {
                    const MsPiece ch = pc[c];
                    if (ch.parent != 0) continue;
                    int ex0 = ch.x0, ex1 = ch.x1, ez0 = ch.z0, ez1 = ch.z1;
                    if (ch.facing == MS_N) { ez0 = p.z0; ez1 = p.z0 + 1; }
                    else if (ch.facing == MS_S) { ez0 = p.z1 - 1; ez1 = p.z1; }
                    else if (ch.facing == MS_W) { ex0 = p.x0; ex1 = p.x0 + 1; }
                    else { ex0 = p.x1 - 1; ex1 = p.x1; }
                    mc_fill(M, ex0, ch.y1 - 2, ez0, ex1, ch.y1, ez1);
                }
                mc_dome(M, p);
                break;
            }
            case MS_CORRIDOR:
                mc_fill(M, p.x0, p.y0, p.z0, p.x1, p.y0 + 1, p.z1);
                if (top) mc_fill(M, p.x0, p.y0 + 2, p.z0, p.x1, p.y0 + 2, p.z1);
                __syncthreads();
                mc_floor(M, p);
                __syncthreads();
                if (p.rails && !top) mc_rails(M, p);
                break;
            case MS_CROSSING: {
                if (two_storey) {
                    mc_fill(M, p.x0 + 1, p.y0, p.z0, p.x1 - 1, p.y0 + 2, p.z1);
                    mc_fill(M, p.x0, p.y0, p.z0 + 1, p.x1, p.y0 + 2, p.z1 - 1);
                    mc_fill(M, p.x0 + 1, p.y1 - 2, p.z0, p.x1 - 1, p.y1, p.z1);
                    mc_fill(M, p.x0, p.y1 - 2, p.z0 + 1, p.x1, p.y1, p.z1 - 1);
                    mc_fill(M, p.x0 + 1, p.y0 + 3, p.z0 + 1, p.x1 - 1, p.y0 + 3, p.z1 - 1);
                } else {
                    mc_fill(M, p.x0 + 1, p.y0, p.z0, p.x1 - 1, p.y1, p.z1);
                    mc_fill(M, p.x0, p.y0, p.z0 + 1, p.x1, p.y1, p.z1 - 1);
                }
                __syncthreads();
                // the four pillars, where the block above the crossing is not air
                if (threadIdx.x < 4) {
                    const int px = (threadIdx.x & 2) ? p.x1 - 1 : p.x0 + 1, pz = (threadIdx.x & 1) ? p.z1 - 1 : p.z0 + 1;
                    if (px >= M.cx0 && px <= M.cx0 + 15 && pz >= M.cz0 && pz <= M.cz0 + 15 &&
                        M.state(px, p.y1 + 1, pz) != ST_AIR)
                        for (int y = p.y0; y <= p.y1; y++) M.place(px, y, pz);
                }
                __syncthreads();
                mc_floor(M, p);
                break;
            }
            default: {   // stairs: nine slices stepping down along the facing
                const int lo[9] = {5, 5, 4, 3, 2, 1, 1, 0, 0}, hi[9] = {7, 7, 7, 6, 5, 4, 3, 2, 2};
                for (int lz = 0; lz < 9; lz++) {
                    int xa = p.x0, xb = p.x1, za = p.z0, zb = p.z1;
                    if (p.facing == MS_N) za = zb = p.z1 - lz;
                    else if (p.facing == MS_S) za = zb = p.z0 + lz;
                    else if (p.facing == MS_W) xa = xb = p.x1 - lz;
                    else xa = xb = p.x0 + lz;
                    mc_fill(M, xa, p.y0 + lo[lz], za, xb, p.y0 + hi[lz], zb);
                }
                break;
            }
        }
        __syncthreads();
    }
    // footprint heights: column (hx + dx, hz + dz), dx < 7, dz < 9
    if (threadIdx.x < kFootW * kFootD) {
        const int x = hx[row] + threadIdx.x / kFootD, z = hz[row] + threadIdx.x % kFootD;
        int h = -64;
        for (int y = 319; y >= -64; y--)
            if (M.state(x, y, z) != ST_AIR) {
                h = y + 1;
                break;
            }
        atomicAdd((unsigned long long *)&hsum, (unsigned long long)(long long)h);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        sums[blockIdx.x] = hsum;
        refused[blockIdx.x] = guard ? nref : 0;
    }
}

// ------------------------------------------------------------------------------------
// The footprint scan (skyscan --list) and the plain floor (msroom's "nat")
// ------------------------------------------------------------------------------------
// Per survivor, over the 7 x 9 footprint at (hx, hz): each column's surface height after the
// carvers (lysh_phase2_height) and, from y = -59 (the corridor top skyscan counts from) up to it,
// the lava and solid blocks.  One CTA of 64 threads per survivor, one column per thread.
struct ScanOut {
    long long sum;
    int32_t min, max, le54, lava, solid, nw, ne, sw, se, above53, pad;
};

__global__ void __launch_bounds__(64) ms_scan_kernel(const P2Chunk *__restrict__ jobs, const int32_t *__restrict__ job_of,
                                                     const int32_t *__restrict__ hx, const int32_t *__restrict__ hz,
                                                     ScanOut *__restrict__ out) {
    __shared__ int hs[64], lv[64], so[64];
    const int row = blockIdx.x, t = threadIdx.x;
    const P2Chunk &J = jobs[job_of[row]];
    if (t < kFootW * kFootD) {
        const int dx = t / kFootD, dz = t % kFootD, x = hx[row] + dx, z = hz[row] + dz;
        int h = -64;
        for (int y = 319; y >= -64; y--)
            if (natural_state(J, x, y, z) != ST_AIR) {
                h = y + 1;
                break;
            }
        int lava = 0, solid = 0;
        for (int y = -59; y < h; y++) {
            const int s = natural_state(J, x, y, z);
            if (s == ST_LAVA) lava++;
            else if (s == ST_SOLID) solid++;
        }
        hs[t] = h;
        lv[t] = lava;
        so[t] = solid;
    }
    __syncthreads();
    if (t != 0) return;
    ScanOut o;
    o.sum = 0;
    o.min = 1000;
    o.max = -1000;
    o.le54 = o.lava = o.solid = o.above53 = 0;
    o.pad = 0;
    for (int c = 0; c < kFootW * kFootD; c++) {
        const int h = hs[c];
        o.sum += h;
        o.min = min(o.min, h);
        o.max = max(o.max, h);
        o.le54 += h <= -54;
        o.above53 += h > -53;
        o.lava += lv[c];
        o.solid += so[c];
    }
    o.nw = hs[0];                                   // (dx, dz) = (0, 0)
    o.ne = hs[(kFootW - 1) * kFootD];               // (6, 0)
    o.sw = hs[kFootD - 1];                          // (0, 8)
    o.se = hs[(kFootW - 1) * kFootD + kFootD - 1];  // (6, 8)
    out[row] = o;
}

}  // namespace
}  // namespace wg

// ------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------
using namespace wg;

// The finisher's device buffers, grown to the largest batch seen (rows per batch <= 512, the
// phase-2 chunk batch).
struct FinishState {
    int64_t *ws = nullptr;
    int32_t *cx = nullptr, *cz = nullptr, *hx = nullptr, *hz = nullptr, *job_of = nullptr;
    MsPiece *pieces = nullptr;
    MsInfo *info = nullptr;
    long long *sums = nullptr;
    int32_t *refused = nullptr;
    ScanOut *scan = nullptr;
    int32_t *bpts = nullptr, *bout = nullptr;
    int cap = 0;
};

void finish_release(wg_engine *eng) {
    FinishState *f = eng->finish;
    if (!f) return;
    cudaFree(f->ws);
    cudaFree(f->cx);
    cudaFree(f->cz);
    cudaFree(f->hx);
    cudaFree(f->hz);
    cudaFree(f->job_of);
    cudaFree(f->pieces);
    cudaFree(f->info);
    cudaFree(f->sums);
    cudaFree(f->refused);
    cudaFree(f->scan);
    cudaFree(f->bpts);
    cudaFree(f->bout);
    delete f;
    eng->finish = nullptr;
}

#define FIN_CUDA(call, what)                                            \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) return eng->fail(WG_ERR_CUDA, what, e_); \
    } while (0)

namespace {

constexpr int kFinishBatch = 512;          // rows per batch: the phase-2 chunk batch
constexpr int kTreeBiome = 5, kTreeBiome26 = 6;   // R-trees of 1.19.x~26.1 and of 26.2 (BIOME_26)

int finish_state(wg_engine *eng, int need) {
    if (!eng->finish) {
        eng->finish = new (std::nothrow) FinishState();
        if (!eng->finish) return eng->fail(WG_ERR_NOMEM, "finisher state");
    }
    if (need <= eng->finish->cap) return WG_OK;
    const size_t n = (size_t)need;
    finish_release(eng);
    eng->finish = new (std::nothrow) FinishState();
    if (!eng->finish) return eng->fail(WG_ERR_NOMEM, "finisher state");
    FinishState &g = *eng->finish;
    FIN_CUDA(cudaMalloc(&g.ws, sizeof(int64_t) * n), "finisher buffers");
    FIN_CUDA(cudaMalloc(&g.cx, sizeof(int32_t) * n), "finisher buffers");
    FIN_CUDA(cudaMalloc(&g.cz, sizeof(int32_t) * n), "finisher buffers");
    FIN_CUDA(cudaMalloc(&g.hx, sizeof(int32_t) * n), "finisher buffers");
    FIN_CUDA(cudaMalloc(&g.hz, sizeof(int32_t) * n), "finisher buffers");
    FIN_CUDA(cudaMalloc(&g.job_of, sizeof(int32_t) * n), "finisher buffers");
    FIN_CUDA(cudaMalloc(&g.pieces, sizeof(MsPiece) * kMsMaxPieces * n), "finisher buffers");
    FIN_CUDA(cudaMalloc(&g.info, sizeof(MsInfo) * n), "finisher buffers");
    FIN_CUDA(cudaMalloc(&g.sums, sizeof(long long) * 4 * n), "finisher buffers");
    FIN_CUDA(cudaMalloc(&g.refused, sizeof(int32_t) * 4 * n), "finisher buffers");
    FIN_CUDA(cudaMalloc(&g.scan, sizeof(ScanOut) * n), "finisher buffers");
    FIN_CUDA(cudaMalloc(&g.bpts, sizeof(int32_t) * 4 * n), "finisher buffers");
    FIN_CUDA(cudaMalloc(&g.bout, sizeof(int32_t) * 2 * n), "finisher buffers");
    g.cap = need;
    return WG_OK;
}

// Trees of rows [0, m) of the batch already uploaded to f.ws / f.cx / f.cz.
int run_trees(wg_engine *eng, int m, std::vector<MsInfo> &info) {
    FinishState &f = *eng->finish;
    ms_tree_kernel<<<(m + 127) / 128, 128, 0, eng->stream>>>(f.ws, f.cx, f.cz, m, f.pieces, f.info);
    FIN_CUDA(cudaGetLastError(), "mineshaft tree launch");
    info.resize(m);
    FIN_CUDA(cudaMemcpyAsync(info.data(), f.info, sizeof(MsInfo) * m, cudaMemcpyDeviceToHost, eng->stream),
             "copy tree status");
    FIN_CUDA(cudaStreamSynchronize(eng->stream), "mineshaft trees");
    return WG_OK;
}

int upload_rows(wg_engine *eng, const int64_t *ws, const int32_t *cx, const int32_t *cz, int m) {
    FinishState &f = *eng->finish;
    std::vector<int32_t> hx(m), hz(m);
    for (int i = 0; i < m; i++) {
        hx[i] = cx[i] * 16;
        hz[i] = cz[i] * 16;
    }
    cudaStream_t s = eng->stream;
    FIN_CUDA(cudaMemcpyAsync(f.ws, ws, sizeof(int64_t) * m, cudaMemcpyHostToDevice, s), "upload rows");
    FIN_CUDA(cudaMemcpyAsync(f.cx, cx, sizeof(int32_t) * m, cudaMemcpyHostToDevice, s), "upload rows");
    FIN_CUDA(cudaMemcpyAsync(f.cz, cz, sizeof(int32_t) * m, cudaMemcpyHostToDevice, s), "upload rows");
    FIN_CUDA(cudaMemcpyAsync(f.hx, hx.data(), sizeof(int32_t) * m, cudaMemcpyHostToDevice, s), "upload rows");
    FIN_CUDA(cudaMemcpyAsync(f.hz, hz.data(), sizeof(int32_t) * m, cudaMemcpyHostToDevice, s), "upload rows");
    FIN_CUDA(cudaStreamSynchronize(s), "upload rows");   // hx / hz are host temporaries
    return WG_OK;
}

}  // namespace

extern "C" int wg_mineshaft_tree(wg_engine *eng, int64_t ws, int32_t chunk_x, int32_t chunk_z, wg_ms_piece *out,
                                 uint32_t cap, uint32_t *n_out, int32_t *room_floor) {
    if (!eng || (cap && !out)) return WG_ERR_ARG;
    FIN_CUDA(cudaSetDevice(eng->device), "cudaSetDevice");
    int rc = finish_state(eng, 1);
    if (rc) return rc;
    rc = upload_rows(eng, &ws, &chunk_x, &chunk_z, 1);
    if (rc) return rc;
    std::vector<MsInfo> info;
    rc = run_trees(eng, 1, info);
    if (rc) return rc;
    if (info[0].status == MS_NOT_START) return eng->fail(WG_ERR_ARG, "mineshaft tree: the chunk is not a mineshaft start");
    if (info[0].status != MS_OK) return eng->fail(WG_ERR_CAPACITY, "mineshaft tree: the tree exceeds the generator's limits");
    std::vector<MsPiece> p(info[0].n);
    FIN_CUDA(cudaMemcpy(p.data(), eng->finish->pieces, sizeof(MsPiece) * p.size(), cudaMemcpyDeviceToHost),
             "copy tree");
    for (uint32_t q = 0; q < (uint32_t)p.size() && q < cap; q++) {
        const MsPiece &a = p[q];
        const int kind = a.type == MS_ROOM ? 'R'
                         : a.type == MS_CORRIDOR ? 'C'
                         : a.type == MS_CROSSING ? (a.y1 - a.y0 + 1 > 3 ? 'Y' : 'X')
                                                 : 'S';
        out[q] = wg_ms_piece{kind, a.x0, a.y0, a.z0, a.x1, a.y1, a.z1, a.facing, a.parent, a.rails};
    }
    if (n_out) *n_out = (uint32_t)p.size();
    if (room_floor) *room_floor = info[0].floor;
    return WG_OK;
}

extern "C" int wg_finish_rows(wg_engine *eng, const int64_t *ws, const int32_t *chunk_x, const int32_t *chunk_z,
                              uint64_t n, wg_finish_row *out) {
    if (!eng || (n && (!ws || !chunk_x || !chunk_z || !out))) return WG_ERR_ARG;
    if (n == 0) return WG_OK;
    FIN_CUDA(cudaSetDevice(eng->device), "cudaSetDevice");
    std::memset(out, 0, sizeof(wg_finish_row) * n);
    // lysh hut --max-y 100 --phase2-max-y 100 --version 1.19.x~26.1 (hunt.py:279-284)
    {
        std::vector<int32_t> hx(n), hz(n);
        for (uint64_t i = 0; i < n; i++) {
            hx[i] = chunk_x[i] * 16;
            hz[i] = chunk_z[i] * 16;
        }
        std::vector<wg_hut_result> hr(n);
        wg_opts o;
        std::memset(&o, 0, sizeof o);
        o.pre_26_2 = 1;
        int rc = wg_eval_huts(eng, ws, hx.data(), hz.data(), n, &o, 100, hr.data());
        if (rc) return rc;
        for (uint64_t i = 0; i < n; i++) {
            out[i].hut_x = hx[i];
            out[i].hut_z = hz[i];
            out[i].verdict_ok = hr[i].ok;
            out[i].avg_y = hr[i].avg_y;
        }
    }
    int rc = finish_state(eng, (int)std::min<uint64_t>(n, kFinishBatch));
    if (rc) return rc;
    FinishState &f = *eng->finish;
    cudaStream_t s = eng->stream;
    for (uint64_t first = 0; first < n; first += kFinishBatch) {
        const int m = (int)std::min<uint64_t>(kFinishBatch, n - first);
        rc = upload_rows(eng, ws + first, chunk_x + first, chunk_z + first, m);
        if (rc) return rc;
        std::vector<MsInfo> info;
        rc = run_trees(eng, m, info);
        if (rc) return rc;
        // the hut chunks' phase-2 state: one world per distinct seed, one chunk per row
        std::map<uint64_t, int> world_of;
        std::vector<uint64_t> seeds;
        std::vector<int> world(m), cxs(m), czs(m), job_of(m);
        for (int i = 0; i < m; i++) {
            const uint64_t sd = (uint64_t)ws[first + i];
            auto it = world_of.find(sd);
            if (it == world_of.end()) it = world_of.emplace(sd, (int)seeds.size()).first, seeds.push_back(sd);
            world[i] = it->second;
            cxs[i] = chunk_x[first + i];
            czs[i] = chunk_z[first + i];
            job_of[i] = i;
        }
        rc = p2_prepare_chunks(eng, seeds, 0, world, cxs, czs);
        if (rc) return rc;
        FIN_CUDA(cudaMemcpyAsync(f.job_of, job_of.data(), sizeof(int32_t) * m, cudaMemcpyHostToDevice, s), "upload");
        ms_carve_kernel<<<4 * m, kCarveThreads, kMcCells, s>>>(eng->p2_jobs, f.job_of, f.hx, f.hz, f.pieces, f.info,
                                                               f.sums, f.refused);
        ms_scan_kernel<<<m, 64, 0, s>>>(eng->p2_jobs, f.job_of, f.hx, f.hz, f.scan);
        FIN_CUDA(cudaGetLastError(), "finisher launch");
        // biome_at --ms --y room_floor: the middle of the chunk north of the start, y = the floor
        std::vector<int32_t> bp(4 * (size_t)m, 0);
        for (int i = 0; i < m; i++) {
            const int x = chunk_x[first + i] * 16, z = chunk_z[first + i] * 16 - 8;
            bp[4 * i] = world[i];
            bp[4 * i + 1] = (x >> 4) * 16 + 8;
            bp[4 * i + 2] = (z >> 4) * 16 + 8;
            bp[4 * i + 3] = info[i].floor;
        }
        FIN_CUDA(cudaMemcpyAsync(f.bpts, bp.data(), sizeof(int32_t) * 4 * m, cudaMemcpyHostToDevice, s), "upload");
        p2_launch_biome_points(eng->p2_tables, eng->p2_worlds, kTreeBiome, f.bpts, m, f.bout, s);
        p2_launch_biome_points(eng->p2_tables, eng->p2_worlds, kTreeBiome26, f.bpts, m, f.bout + m, s);
        FIN_CUDA(cudaGetLastError(), "finisher biome launch");
        std::vector<long long> sums(4 * (size_t)m);
        std::vector<int32_t> refused(4 * (size_t)m), biome(2 * (size_t)m);
        std::vector<ScanOut> scan(m);
        FIN_CUDA(cudaMemcpyAsync(sums.data(), f.sums, sizeof(long long) * 4 * m, cudaMemcpyDeviceToHost, s), "copy");
        FIN_CUDA(cudaMemcpyAsync(refused.data(), f.refused, sizeof(int32_t) * 4 * m, cudaMemcpyDeviceToHost, s), "copy");
        FIN_CUDA(cudaMemcpyAsync(biome.data(), f.bout, sizeof(int32_t) * 2 * m, cudaMemcpyDeviceToHost, s), "copy");
        FIN_CUDA(cudaMemcpyAsync(scan.data(), f.scan, sizeof(ScanOut) * m, cudaMemcpyDeviceToHost, s), "copy");
        FIN_CUDA(cudaStreamSynchronize(s), "finisher");
        for (int i = 0; i < m; i++) {
            wg_finish_row &r = out[first + i];
            const ScanOut &o = scan[i];
            r.tree_status = info[i].status;
            r.pieces = info[i].n;
            r.room_floor = info[i].floor;
            r.scan_sum = o.sum;
            r.scan_min = o.min;
            r.scan_max = o.max;
            r.le54 = o.le54;
            r.lava = o.lava;
            r.solid = o.solid;
            r.nw = o.nw;
            r.ne = o.ne;
            r.sw = o.sw;
            r.se = o.se;
            r.above53 = o.above53;
            r.sum_nat = o.sum;
            r.nat = (int32_t)(o.sum / 63);
            if (info[i].status != MS_OK) continue;
            r.biome[0] = biome[i];
            r.biome[1] = biome[m + i];
            for (int top = 0; top < 2; top++) {
                r.sum_top[top] = sums[4 * i + top];
                r.top[top] = (int32_t)(sums[4 * i + top] / 63);
                r.refused[top] = refused[4 * i + top];
                r.sum_no_guard[top] = sums[4 * i + 2 + top];
                r.no_guard[top] = (int32_t)(sums[4 * i + 2 + top] / 63);
            }
        }
    }
    return WG_OK;
}
