// hut_lookup: drop-in for the two Deep Dive commands hunt.py runs through the reference's GPU
// engine (hut_lookup_v4, engine/gpu/hut_lookup_v4_source.cu:777-841 flags), on top of
// libwitchgpu.so:
//
//   solver   --catalog C --solve-only --solve5 --plan P --first-index F --count N
//            [--regime XZ] [--dump-hits H] [--out O] [--quiet]          (hunt.py:947-952)
//            hits "S,chunkX,chunkZ,layoutX,1" to H; the summary line "solve: ..." on stdout
//            (:1373-1380); exit 1 when a hit fails the host's forward check, as there
//   terrain  --catalog C --spots SP [--max-height -54] --out O [--batch B] [--quiet]
//            (hunt.py:954-957): "S chunkX chunkZ" lines; the world seeds (u << 48) | S48 that
//            pass the phase-1 gates at the spot region whose hut is the spot chunk, as
//            "seed,chunkX,chunkZ,layoutX,airHi,airLo" rows appended to O (header when empty);
//            exit 1 when a spot is not a mineshaft start chunk (:1262-1290)
//   forward  --catalog C --first-index F --count N [--max-height -54] [--out O] [--quiet]
//            (the reference's default mode, :1504-1533): structure seed
//            s48 = (index * 0x9E3779B97F4A7D + 0x2545F4914F6CDD) mod 2^48 for each index of the range
//            (:27-29, :1505); every hut region of the +-30M world (radius 58,593) swept for huts on
//            mineshaft start chunks whose carver state is a catalogued layout (wg_deep_sweep); each
//            match's 65,536 world seeds through the terrain stage as in --spots; the reference's
//            per-seed line on stderr and its summary line on stdout
//
//   finish   --finish ROWS [--min-r R]
//            the mineshaft finisher over terrain-stage rows "seed,chunkX,chunkZ[,layoutX,airHi,airLo]"
//            (a header line is skipped): per row what hunt.py's finish_row computes through lysh,
//            mstree, biome_at, msroom and skyscan (hunt.py:277-333), here one wg_finish_rows call for
//            all rows; the result line of each accepted row on stdout, in finish_row's format, and a
//            summary on stderr
//
// The tuning flags of the reference (--fused-*, --task-batch, --ero-*, --batch, --u-*) are
// accepted and change nothing: the solver and the gates here are exact.  The terrain gates are
// lysh's phase 1 (lysh_phase1_check_ex) at --max-height with the hunt driver's version
// (1.19.x~26.1), the same rule the spot fixtures pin.
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <chrono>
#include <map>
#include <string>
#include <vector>

#include "../../include/witchgpu.h"

namespace {

// The terrain stage of one call's spots: survivors appended to `out` as the reference's rows.
// Returns the survivor count, or -1 on failure; *not_start counts spots that are not start chunks.
long long terrain_rows(wg_engine *eng, const std::vector<int64_t> &s48, const std::vector<int32_t> &cx,
                       const std::vector<int32_t> &cz, const std::vector<uint64_t> &layout,
                       const std::vector<uint32_t> &value, int max_h, FILE *out, uint64_t *not_start);

bool read_catalog(const char *path, std::map<uint64_t, std::pair<unsigned, unsigned>> &cat) {
    FILE *f = std::fopen(path, "r");
    if (!f) return false;
    char ln[1024];
    while (std::fgets(ln, sizeof ln, f)) {
        if (ln[0] == '#' || ln[0] == '\n') continue;
        unsigned long long x;
        double hi, lo;
        if (std::sscanf(ln, "%llu %lf %lf", &x, &hi, &lo) != 3) continue;
        cat[x & 0xFFFFFFFFFFFFull] = {(unsigned)hi & 0x3FF, (unsigned)lo & 0x3FF};
    }
    std::fclose(f);
    return true;
}

// The spot's setLargeFeatureSeed state, the reference's layoutX column for a spot: setSeed(S),
// a = nextLong(), b = nextLong(), (cx a) ^ (cz b) ^ S (room_core.h:55-58).
uint64_t carver_state(uint64_t s48, int cx, int cz) {
    const uint64_t A = 0x5DEECE66Dull, M = 0xFFFFFFFFFFFFull;
    uint64_t s = (s48 ^ A) & M;
    int32_t h[4];
    for (int k = 0; k < 4; k++) {
        s = (s * A + 0xBull) & M;
        h[k] = (int32_t)(s >> 16);
    }
    const uint64_t a = ((uint64_t)(int64_t)h[0] << 32) + (uint64_t)(int64_t)h[1];
    const uint64_t b = ((uint64_t)(int64_t)h[2] << 32) + (uint64_t)(int64_t)h[3];
    return ((uint64_t)((int64_t)cx * (int64_t)a) ^ (uint64_t)((int64_t)cz * (int64_t)b) ^ s48) & M;
}

int tier_of(const char *cls) {
    if (!std::strcmp(cls, "odd")) return 1;
    if (!std::strcmp(cls, "u2")) return 2;
    if (!std::strcmp(cls, "eq")) return 3;
    return 0;
}

int fail(const char *msg) {
    std::fprintf(stderr, "%s\n", msg);
    return 2;
}

long long terrain_rows(wg_engine *eng, const std::vector<int64_t> &s48, const std::vector<int32_t> &cx,
                       const std::vector<int32_t> &cz, const std::vector<uint64_t> &layout,
                       const std::vector<uint32_t> &value, int max_h, FILE *out, uint64_t *not_start) {
    wg_opts o{};   // wg_parse_version sets the version bits only; NORMAL preset
    wg_parse_version("1.19.x~26.1", &o);
    long long total = 0;
    *not_start = 0;
    for (size_t i0 = 0; i0 < s48.size(); i0 += 4096) {
        const size_t n = std::min<size_t>(4096, s48.size() - i0);
        std::vector<wg_candidate> c(1 << 16);
        uint64_t got = 0, bad = 0;
        int rc;
        for (;;) {
            rc = wg_deep_spots(eng, s48.data() + i0, cx.data() + i0, cz.data() + i0, n, &o, max_h, c.data(), c.size(),
                               &got, &bad);
            if (rc || got <= c.size()) break;
            c.resize(got);
        }
        if (rc) {
            std::fprintf(stderr, "terrain stage failed: %s\n", wg_engine_error(eng));
            return -1;
        }
        *not_start += bad;
        for (uint64_t k = 0; k < got; k++) {
            const size_t spot = i0 + (size_t)(c[k].seed_index >> 16);
            std::fprintf(out, "%lld,%d,%d,%llu,%u,%u\n", (long long)c[k].seed, cx[spot], cz[spot],
                         (unsigned long long)layout[spot], value[spot] & 0x3FF, (value[spot] >> 10) & 0x3FF);
            total++;
        }
    }
    return total;
}

}  // namespace

namespace {

// One terrain-stage row for the finisher.
struct FinishIn {
    int64_t ws;
    int32_t cx, cz;
    std::string layout, hi, lo;
};

// --finish: the result line of every accepted row, exactly as finish_row prints it:
// "%4d  terrain %4s  refused %2s  if-none-refused %4s  NW %4s  max %4s  lava %4s  air %s/%s  biome %s
//  layout %s  seed %s  /tp %d %d %d" (hunt.py:329-331), where the floor is msroom's top1, "refused"
// its first (top0) count, "if-none-refused" ng1, NW / max / lava skyscan's, biome the 1.21.5-tree
// biome at the room floor.  A row is rejected when lysh does not accept the hut at 100, the chunk is
// no mineshaft start, the room floor is deep dark in both biome sets, or the floor is above min_r.
int run_finish(wg_engine *eng, const char *path, int min_r) {
    FILE *f = std::fopen(path, "r");
    if (!f) {
        std::fprintf(stderr, "cannot read %s\n", path);
        return 1;
    }
    std::vector<FinishIn> rows;
    char ln[512];
    while (std::fgets(ln, sizeof ln, f)) {
        if (!(ln[0] == '-' || (ln[0] >= '0' && ln[0] <= '9'))) continue;   // header or blank
        std::vector<std::string> t;
        std::string cur;
        for (const char *p = ln; *p && *p != '\n' && *p != '\r'; p++) {
            if (*p == ',' || *p == ' ' || *p == '\t') {
                if (!cur.empty()) t.push_back(cur);
                cur.clear();
            } else {
                cur += *p;
            }
        }
        if (!cur.empty()) t.push_back(cur);
        if (t.size() < 3) continue;
        FinishIn r;
        r.ws = std::strtoll(t[0].c_str(), nullptr, 10);
        r.cx = (int32_t)std::atoi(t[1].c_str());
        r.cz = (int32_t)std::atoi(t[2].c_str());
        r.layout = t.size() > 3 ? t[3] : "0";
        r.hi = t.size() > 4 ? t[4] : "0";
        r.lo = t.size() > 5 ? t[5] : "0";
        rows.push_back(r);
    }
    std::fclose(f);
    std::vector<int64_t> ws(rows.size());
    std::vector<int32_t> cx(rows.size()), cz(rows.size());
    for (size_t i = 0; i < rows.size(); i++) {
        ws[i] = rows[i].ws;
        cx[i] = rows[i].cx;
        cz[i] = rows[i].cz;
    }
    std::vector<wg_finish_row> out(rows.size());
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = wg_finish_rows(eng, ws.data(), cx.data(), cz.data(), rows.size(), out.data());
    if (rc) {
        std::fprintf(stderr, "wg_finish_rows: %s\n", wg_engine_error(eng));
        return 1;
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    size_t kept = 0;
    for (size_t i = 0; i < rows.size(); i++) {
        const wg_finish_row &r = out[i];
        if (!r.verdict_ok || r.tree_status != 0) continue;
        if (r.biome[0] == 183 && r.biome[1] == 183) continue;   // deep dark in both sets: no mineshaft
        if (r.top[1] > min_r) continue;
        kept++;
        std::printf("%4d  terrain %4d  refused %2d  if-none-refused %4d  NW %4d  max %4d  lava %4d  air %s/%s  "
                    "biome %d  layout %s  seed %" PRId64 "  /tp %d %d %d\n",
                    r.top[1], r.nat, r.refused[0], r.no_guard[1], r.nw, r.scan_max, r.lava, rows[i].hi.c_str(),
                    rows[i].lo.c_str(), r.biome[0], rows[i].layout.c_str(), rows[i].ws, r.hut_x, r.top[1], r.hut_z);
    }
    std::fprintf(stderr, "finish: %zu rows, %zu accepted, %.3f s\n", rows.size(), kept, secs);
    return 0;
}

}  // namespace

int main(int argc, char **argv) {
    const char *cat_path = nullptr, *plan_path = nullptr, *spots_path = nullptr, *hits_path = nullptr;
    const char *finish_path = nullptr;
    int min_r = 999;
    const char *out_path = "hut_lookup_out.csv";
    long long first = 0, count = 1;
    int regx = -1, regz = -1, max_h = -54;
    bool solve5 = false, quiet = false, solve_flag = false;
    for (int i = 1; i < argc; i++) {
        const char *a = argv[i];
        auto val = [&]() -> const char * { return i + 1 < argc ? argv[++i] : nullptr; };
        if (!std::strcmp(a, "--catalog")) cat_path = val();
        else if (!std::strcmp(a, "--plan")) plan_path = val();
        else if (!std::strcmp(a, "--spots")) spots_path = val();
        else if (!std::strcmp(a, "--finish")) finish_path = val();
        else if (!std::strcmp(a, "--min-r")) { const char *v = val(); if (v) min_r = std::atoi(v); }
        else if (!std::strcmp(a, "--dump-hits")) hits_path = val();
        else if (!std::strcmp(a, "--out")) out_path = val();
        else if (!std::strcmp(a, "--first-index")) { const char *v = val(); if (v) first = std::atoll(v); }
        else if (!std::strcmp(a, "--count")) { const char *v = val(); if (v) count = std::atoll(v); }
        else if (!std::strcmp(a, "--max-height")) { const char *v = val(); if (v) max_h = std::atoi(v); }
        else if (!std::strcmp(a, "--regime")) {
            const char *v = val();
            if (!v || std::strlen(v) != 2 || v[0] < '0' || v[0] > '2' || v[1] < '0' || v[1] > '2')
                return fail("--regime XZ: two digits 0 (exact), 1 (mid), 2 (far)");
            regx = v[0] - '0';
            regz = v[1] - '0';
        } else if (!std::strcmp(a, "--far")) regx = regz = 2;
        else if (!std::strcmp(a, "--solve5")) solve5 = true;
        else if (!std::strcmp(a, "--quiet")) quiet = true;
        else if (!std::strcmp(a, "--solve-only") || !std::strcmp(a, "--solve")) solve_flag = true;
        else if (!std::strcmp(a, "--ero-split") || !std::strcmp(a, "--timing") || !std::strcmp(a, "--no-async"))
            ;
        else if (!std::strncmp(a, "--fused-", 8) || !std::strncmp(a, "--ero-", 6) || !std::strcmp(a, "--task-batch") ||
                 !std::strcmp(a, "--batch") || !std::strcmp(a, "--u-lo") || !std::strcmp(a, "--u-hi") ||
                 !std::strcmp(a, "--u-batch") || !std::strcmp(a, "--min-air") || !std::strcmp(a, "--cols")) {
            if (!val()) return fail("missing value");
        } else {
            std::fprintf(stderr, "unknown arg %s\n", a);
            return 2;
        }
    }
    if (finish_path) {
        wg_engine *feng = nullptr;
        if (wg_engine_open(0, &feng)) {
            std::fprintf(stderr, "no GPU engine\n");
            return 1;
        }
        const int frc = run_finish(feng, finish_path, min_r);
        wg_engine_close(feng);
        return frc;
    }
    if (!cat_path) return fail("usage: hut_lookup --catalog cat.txt (--solve-only --solve5 --plan P | --spots S) ...");
    std::map<uint64_t, std::pair<unsigned, unsigned>> cat;
    if (!read_catalog(cat_path, cat)) { std::fprintf(stderr, "cannot read %s\n", cat_path); return 1; }

    wg_engine *eng = nullptr;
    int rc = wg_engine_open(0, &eng);
    if (rc) { std::fprintf(stderr, "no GPU engine (status %d)\n", rc); return 1; }

    if (spots_path) {
        FILE *sf = std::fopen(spots_path, "r");
        if (!sf) { std::fprintf(stderr, "cannot read %s\n", spots_path); wg_engine_close(eng); return 1; }
        std::vector<int64_t> s48;
        std::vector<int32_t> cx, cz;
        char ln[512];
        while (std::fgets(ln, sizeof ln, sf)) {
            long long S;
            int x, z;
            if (ln[0] == '#' || std::sscanf(ln, "%lld %d %d", &S, &x, &z) != 3) continue;
            s48.push_back((int64_t)((uint64_t)S & 0xFFFFFFFFFFFFull));
            cx.push_back(x);
            cz.push_back(z);
        }
        std::fclose(sf);
        FILE *out = std::fopen(out_path, "a");
        if (!out) { std::fprintf(stderr, "cannot write %s\n", out_path); wg_engine_close(eng); return 1; }
        std::fseek(out, 0, SEEK_END);
        if (std::ftell(out) == 0) std::fprintf(out, "seed,chunkX,chunkZ,layoutX,airHi,airLo\n");
        std::vector<uint64_t> layout(s48.size());
        std::vector<uint32_t> zero(s48.size(), 0);
        for (size_t i = 0; i < s48.size(); i++) layout[i] = carver_state((uint64_t)s48[i], cx[i], cz[i]);
        uint64_t bad_all = 0;
        const auto t0 = std::chrono::steady_clock::now();
        const long long total = terrain_rows(eng, s48, cx, cz, layout, zero, max_h, out, &bad_all);
        std::fclose(out);
        if (bad_all) std::fprintf(stderr, "*** %llu spots are not mineshaft start chunks\n", (unsigned long long)bad_all);
        const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::printf("spots: %zu spots (%llu not a start), %llu terrain survivors -> %s; terrain %.3f s (%.1f ms per spot)\n",
                    s48.size(), (unsigned long long)bad_all, (unsigned long long)std::max(0LL, total), out_path, secs,
                    s48.empty() ? 0.0 : 1e3 * secs / (double)s48.size());
        wg_engine_close(eng);
        return total < 0 ? 1 : (bad_all ? 1 : 0);
    }

    if (!solve5 && !solve_flag) {
        // forward mode: sweep the world per structure seed, probe the catalogue, terrain-check the matches
        if (first < 0 || count < 1) { wg_engine_close(eng); return fail("--first-index >= 0 and --count >= 1"); }
        std::vector<uint64_t> keys;
        std::vector<uint32_t> vals;
        for (const auto &kv : cat) {
            keys.push_back(kv.first);
            vals.push_back(kv.second.first | (kv.second.second << 10));
        }
        if (keys.empty()) { wg_engine_close(eng); return fail("empty catalogue"); }
        if (!quiet) std::printf("catalogue: %zu layouts\n", keys.size());
        FILE *out = std::fopen(out_path, "a");
        if (!out) { std::fprintf(stderr, "cannot write %s\n", out_path); wg_engine_close(eng); return 1; }
        std::fseek(out, 0, SEEK_END);
        if (std::ftell(out) == 0) std::fprintf(out, "seed,chunkX,chunkZ,layoutX,airHi,airLo\n");
        const auto t0 = std::chrono::steady_clock::now();
        auto wall = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
        unsigned long long tot_matches = 0, tot_surv = 0;
        int status = 0;
        std::vector<wg_sweep_match> m(1 << 12);
        for (long long si = 0; si < count && !status; si++) {
            const int64_t s48 = (int64_t)(((uint64_t)(first + si) * 0x9E3779B97F4A7DULL + 0x2545F4914F6CDDULL) &
                                          0xFFFFFFFFFFFFull);
            uint64_t got = 0, starts = 0;
            for (;;) {
                rc = wg_deep_sweep(eng, keys.data(), vals.data(), keys.size(), &s48, 0, 1, -58593, 58594, -58593, 58594,
                                   m.data(), m.size(), &got, &starts);
                if (rc || got <= m.size()) break;
                m.resize(got);
            }
            if (rc) { std::fprintf(stderr, "sweep failed: %s\n", wg_engine_error(eng)); status = 1; break; }
            std::vector<int64_t> ss(got, s48);
            std::vector<int32_t> mx(got), mz(got);
            std::vector<uint64_t> lay(got);
            std::vector<uint32_t> val(got);
            for (uint64_t k = 0; k < got; k++) {
                mx[k] = m[k].chunk_x;
                mz[k] = m[k].chunk_z;
                lay[k] = (uint64_t)m[k].carver;
                val[k] = m[k].value;
            }
            uint64_t bad = 0;
            const long long surv = got ? terrain_rows(eng, ss, mx, mz, lay, val, max_h, out, &bad) : 0;
            if (surv < 0) { status = 1; break; }
            std::fflush(out);
            tot_matches += got;
            tot_surv += (unsigned long long)surv;
            if (!quiet)
                std::fprintf(stderr, "S48 %lld (index %lld): %llu hut starts, %llu catalogue matches, %llu terrain survivors | %.1f s\n",
                             (long long)s48, first + si, (unsigned long long)starts, (unsigned long long)got,
                             (unsigned long long)surv, wall());
        }
        std::fclose(out);
        std::printf("done:%lld structure seeds, %llu matches, %llu survivors -> %s (%.1f s, %.2f s per structure seed)\n",
                    count, tot_matches, tot_surv, out_path, wall(), wall() / (double)count);
        wg_engine_close(eng);
        return status;
    }
    if (!solve5) { wg_engine_close(eng); return fail("--solve / --solve-only need --solve5 here"); }
    std::vector<wg_solve_bundle> bundles;
    if (plan_path) {
        FILE *pf = std::fopen(plan_path, "r");
        if (!pf) { std::fprintf(stderr, "cannot read plan %s\n", plan_path); wg_engine_close(eng); return 1; }
        char ln[1024];
        while (std::fgets(ln, sizeof ln, pf)) {
            if (ln[0] == '#' || ln[0] == '\n') continue;
            unsigned long long x;
            char rg[8], cls[16] = "odd";
            if (std::sscanf(ln, "%llu %7s %15s", &x, rg, cls) < 2 || std::strlen(rg) != 2 || rg[0] < '0' || rg[0] > '2' ||
                rg[1] < '0' || rg[1] > '2') {
                std::fprintf(stderr, "bad plan line: %s", ln);
                std::fclose(pf);
                wg_engine_close(eng);
                return 2;
            }
            const int t = tier_of(cls);
            if (!t) { std::fprintf(stderr, "plan class '%s' unknown (odd | u2 | eq)\n", cls); std::fclose(pf); wg_engine_close(eng); return 2; }
            wg_solve_bundle b;
            std::memset(&b, 0, sizeof b);
            b.layout = x & 0xFFFFFFFFFFFFull;
            b.regime_x = rg[0] - '0';
            b.regime_z = rg[1] - '0';
            b.tier = t;
            bundles.push_back(b);
        }
        std::fclose(pf);
    } else {
        if (regx < 0) { wg_engine_close(eng); return fail("--solve5 needs --regime XZ (or --plan)"); }
        for (const auto &kv : cat) {
            wg_solve_bundle b;
            std::memset(&b, 0, sizeof b);
            b.layout = kv.first;
            b.regime_x = regx;
            b.regime_z = regz;
            b.tier = 1;
            bundles.push_back(b);
        }
    }
    if (bundles.empty()) { wg_engine_close(eng); return fail("no bundles"); }
    if (first < 0 || count < 1 || (unsigned long long)(first + count) > ((unsigned long long)bundles.size() << 20)) {
        std::fprintf(stderr, "group range %lld..%lld outside the %zu bundles x 2^20 groups\n", first, first + count,
                     bundles.size());
        wg_engine_close(eng);
        return 2;
    }
    FILE *hf = hits_path ? std::fopen(hits_path, "w") : nullptr;
    if (hits_path && !hf) { std::fprintf(stderr, "cannot write %s\n", hits_path); wg_engine_close(eng); return 1; }
    wg_solve_stats tot;
    std::memset(&tot, 0, sizeof tot);
    std::vector<wg_solve_hit> hits(1 << 16);
    for (long long g = first; g < first + count && rc == WG_OK;) {
        const long long n = std::min<long long>(256, first + count - g);
        wg_solve_stats st;
        uint64_t got = 0;
        for (;;) {
            rc = wg_deep_solve(eng, bundles.data(), bundles.size(), (uint64_t)g, (uint64_t)n, hits.data(), hits.size(),
                               &got, &st);
            if (rc || got <= hits.size()) break;
            hits.resize(got);
        }
        if (rc) { std::fprintf(stderr, "solver failed: %s\n", wg_engine_error(eng)); break; }
        for (uint64_t k = 0; k < got && hf; k++)
            std::fprintf(hf, "%llu,%d,%d,%llu,1\n", (unsigned long long)hits[k].s48, hits[k].chunk_x, hits[k].chunk_z,
                         (unsigned long long)hits[k].layout);
        tot.groups += st.groups;
        tot.tasks += st.tasks;
        tot.hits += st.hits;
        tot.host_check_failures += st.host_check_failures;
        tot.gpu_ms += st.gpu_ms;
        tot.wall_ms += st.wall_ms;
        if (!quiet)
            std::fprintf(stderr, "groups %lld..%lld: %llu hits | %.1f s\n", first, g + n,
                         (unsigned long long)tot.hits, tot.wall_ms / 1e3);
        g += n;
    }
    if (hf) std::fclose(hf);
    std::printf("solve: %llu tasks in %llu groups, %llu hits (%.4f per task), host-check failures %llu\n",
                (unsigned long long)tot.tasks, (unsigned long long)tot.groups, (unsigned long long)tot.hits,
                tot.tasks ? (double)tot.hits / (double)tot.tasks : 0.0, (unsigned long long)tot.host_check_failures);
    std::printf("solve times: device %.3f s; wall %.3f s (%.4f us per task wall)\n", tot.gpu_ms / 1e3,
                tot.wall_ms / 1e3, tot.tasks ? 1e3 * tot.wall_ms / (double)tot.tasks : 0.0);
    wg_engine_close(eng);
    if (rc) return 1;
    return tot.host_check_failures ? 1 : 0;
}
