// phase1_scan: drop-in replacement for the reference GPU scanner's command-line and
// --worker contract (engine/gpu/low54/phase1_scan.cu:561-601 usage, :641-759 flags,
// :1328-1339 CSV, :1365-1387 worker loop), on top of libwitchgpu.so.
//
// Differences a caller can observe:
//   * The rows written are the exact hit set: lysh's phase-1 survivors (lysh_phase1_check_ex)
//     confirmed by lysh's phase 2 (lysh_eval_hut: biome gate, flood test, post-carver footprint
//     heights) at --phase2-max-y (default: --max-height as given, before the clamp below, as
//     lysh scan's default), on the GPU through wg_eval_huts.  The 6th CSV column (the reference's
//     gpuEst) holds the hut's floor y, avg_y.  hunt.py reads the first three columns and
//     re-confirms each row with `lysh hut` at its ceiling (<= -50, hunt.py:1347-1349), which
//     accepts a subset of these rows, so its results are those of the phase-1 superset with one
//     `lysh hut` per hit instead of one per candidate.  --phase1-candidates writes the phase-1
//     superset instead, with "nan" in the 6th column.  There is no lossy density prefilter, so
//     --no-density-prefilter / --climate-gate / --no-climate-gate / --block are accepted and
//     change nothing.
//   * --max-height is clamped like lysh's phase1CheckHeight (-50 / -54 -> -50,
//     engine/tools/lysh/src/main.c:135-137).
//   * --version / --preset take lysh's names (default 1.19.x~26.1, the hunt driver's);
//     --v26-2 selects the 26.2 ridge rule as before.
//   * --self-test re-checks sampled regions of the request's first 16 seeds (the reference's
//     sampling, up to 20,000 regions per seed at a fixed stride, phase1_scan.cu:1289-1326) through
//     the engine's plain FP64 noise core and compares each verdict with the scan's phase-1
//     survivor list (the FP32 core's); prints the reference's summary line and fails the request
//     (rc 1) on any mismatch.
//   * --quad-bases sweeps (base, high 16 bits) as the reference does (:64-86, :700-724):
//     index i of the request is the seed bases[g >> 16] | (g & 0xffff) << 48 with
//     g = offset * 65536 + i; the seeds are expanded on the host in slices.  Combining it
//     with --seed / --seed-list / --seed-gen is an error here (the reference ignores them).
//   * --max-hut-dist D (with --gate-center-x / -z) keeps the candidates whose reported
//     position (16 chunkX, 16 chunkZ) lies within D blocks of the centre (:241-292, :340-349);
//     D < 0 (the default) turns the gate off.
//   * --require-all-regions keeps a seed's candidates only when every region of the rect
//     passes the three climate gates (:145-181) -- here lysh's erosion / temperature / ridge
//     verdicts, so the SINGLE_BIOME and 1.18.2 rules follow lysh.
#include <cctype>
#include <algorithm>
#include <chrono>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/witchgpu.h"

namespace {

struct Params {
    std::vector<int64_t> seeds;
    bool gen = false;
    uint64_t gen_base = 0;
    long long gen_count = 0;
    int min_rx = -128, max_rx = 128, min_rz = -128, max_rz = 128;
    int max_height = -40;
    wg_opts opts{};
    std::string out_path;
    std::string quad_path;              // --quad-bases
    std::vector<uint64_t> quad_bases;
    long long quad_offset = 0, quad_limit = 0;
    long long max_hut_dist = -1;        // --max-hut-dist; < 0 = no position gate
    int gate_x = 0, gate_z = 0;
    bool require_all = false;
    bool phase1_only = false;           // --phase1-candidates: write the phase-1 survivors unconfirmed
    bool have_p2_max_y = false;         // --phase2-max-y given
    int p2_max_y = -40;                 // phase-2 ceiling (default: --max-height before the clamp)
    bool self_test = false;
};

uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// Seeds of a --quad-bases request: request index i -> bases[g >> 16] | (g & 0xffff) << 48,
// g = offset * 65536 + i (phase1_scan.cu:79-86).
int64_t quad_seed(const Params &p, uint64_t i) {
    const uint64_t g = (uint64_t)p.quad_offset * 65536ull + i;
    return (int64_t)(p.quad_bases[g >> 16] | ((g & 0xFFFFull) << 48));
}

bool load_quad_bases(Params &p) {
    std::ifstream f(p.quad_path);
    if (!f) {
        std::fprintf(stderr, "cannot open --quad-bases %s\n", p.quad_path.c_str());
        return false;
    }
    unsigned long long v;
    while (f >> v) p.quad_bases.push_back(v);
    if (p.quad_bases.empty()) {
        std::fprintf(stderr, "--quad-bases file had no seeds\n");
        return false;
    }
    if (p.quad_offset < 0 || (size_t)p.quad_offset >= p.quad_bases.size()) {
        std::fprintf(stderr, "--quad-base-offset out of range\n");
        return false;
    }
    const long long avail = (long long)p.quad_bases.size() - p.quad_offset;
    if (p.quad_limit <= 0 || p.quad_limit > avail) p.quad_limit = avail;
    if (p.quad_limit > 32767) {   // the reference's per-request cap (2^31 seeds)
        std::fprintf(stderr, "--quad-base-limit capped at 32767\n");
        p.quad_limit = 32767;
    }
    return true;
}

bool read_seed_list(const char *path, std::vector<int64_t> &out) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return false;
    std::string buf;
    char tmp[1 << 16];
    size_t n;
    while ((n = std::fread(tmp, 1, sizeof tmp, f)) > 0) buf.append(tmp, n);
    std::fclose(f);
    const char *p = buf.c_str(), *end = p + buf.size();
    while (p < end) {
        while (p < end && !(std::isdigit((unsigned char)*p) || *p == '-')) p++;
        if (p >= end) break;
        char *next = nullptr;
        unsigned long long v = std::strtoull(p, &next, 10);  // unsigned and signed decimal spellings
        if (next == p) { p++; continue; }
        out.push_back((int64_t)v);
        p = next;
    }
    return true;
}

bool parse(const std::vector<std::string> &t, Params &p) {
    p.opts = wg_opts{};
    wg_parse_version("1.19.x~26.1", &p.opts);
    bool ok = true;
    size_t i = 0;
    auto next = [&](const char *what) -> std::string {
        if (i + 1 >= t.size()) {
            std::fprintf(stderr, "missing value for %s\n", what);
            ok = false;
            return std::string();
        }
        return t[++i];
    };
    for (; i < t.size() && ok; i++) {
        const std::string &a = t[i];
        if (a == "--seed") p.seeds.push_back((int64_t)std::strtoull(next("--seed").c_str(), nullptr, 10));
        else if (a == "--seed-list") {
            std::string path = next("--seed-list");
            if (ok && !read_seed_list(path.c_str(), p.seeds)) {
                std::fprintf(stderr, "cannot open seed list %s\n", path.c_str());
                ok = false;
            }
        } else if (a == "--seed-gen") {
            std::string b = next("--seed-gen (base)");
            std::string c = ok ? next("--seed-gen (count)") : std::string();
            if (ok) {
                p.gen = true;
                p.gen_base = std::strtoull(b.c_str(), nullptr, 10);
                p.gen_count = std::atoll(c.c_str());
            }
        } else if (a == "--min-region-x") p.min_rx = std::atoi(next(a.c_str()).c_str());
        else if (a == "--max-region-x") p.max_rx = std::atoi(next(a.c_str()).c_str());
        else if (a == "--min-region-z") p.min_rz = std::atoi(next(a.c_str()).c_str());
        else if (a == "--max-region-z") p.max_rz = std::atoi(next(a.c_str()).c_str());
        else if (a == "--max-height") p.max_height = std::atoi(next(a.c_str()).c_str());
        else if (a == "--v26-2") p.opts.pre_26_2 = 0;
        else if (a == "--version") {
            std::string v = next(a.c_str());
            if (ok && wg_parse_version(v.c_str(), &p.opts)) {
                std::fprintf(stderr, "bad --version %s\n", v.c_str());
                ok = false;
            }
        } else if (a == "--preset") {
            std::string v = next(a.c_str());
            if (ok && wg_parse_preset(v.c_str(), &p.opts)) {
                std::fprintf(stderr, "bad --preset %s\n", v.c_str());
                ok = false;
            }
        } else if (a == "--out") p.out_path = next(a.c_str());
        else if (a == "--block") (void)next(a.c_str());
        else if (a == "--self-test") p.self_test = true;
        else if (a == "--phase1-candidates") p.phase1_only = true;
        else if (a == "--phase2-max-y") {
            p.p2_max_y = std::atoi(next(a.c_str()).c_str());
            p.have_p2_max_y = true;
        } else if (a == "--no-density-prefilter" || a == "--climate-gate" || a == "--no-climate-gate" ||
                   a == "--worker") {
        } else if (a == "--quad-bases") p.quad_path = next(a.c_str());
        else if (a == "--quad-base-offset") p.quad_offset = std::atoll(next(a.c_str()).c_str());
        else if (a == "--quad-base-limit") p.quad_limit = std::atoll(next(a.c_str()).c_str());
        else if (a == "--max-hut-dist") p.max_hut_dist = std::atoll(next(a.c_str()).c_str());
        else if (a == "--gate-center-x") p.gate_x = std::atoi(next(a.c_str()).c_str());
        else if (a == "--gate-center-z") p.gate_z = std::atoi(next(a.c_str()).c_str());
        else if (a == "--require-all-regions") p.require_all = true;
        else {
            std::fprintf(stderr, "unknown argument: %s\n", a.c_str());
            ok = false;
        }
    }
    if (!ok) return false;
    if (!p.quad_path.empty()) {
        if (p.gen || !p.seeds.empty()) {
            std::fprintf(stderr, "--quad-bases cannot be combined with --seed/--seed-list/--seed-gen\n");
            return false;
        }
        if (!load_quad_bases(p)) return false;
    }
    if (p.gen && !p.seeds.empty()) {
        std::fprintf(stderr, "--seed-gen cannot be combined with --seed/--seed-list\n");
        return false;
    }
    if (p.gen && p.gen_count <= 0) {
        std::fprintf(stderr, "--seed-gen count must be positive\n");
        return false;
    }
    if (!p.gen && p.seeds.empty() && p.quad_bases.empty()) {
        std::fprintf(stderr, "no seeds given\n");
        return false;
    }
    if (p.max_rx <= p.min_rx || p.max_rz <= p.min_rz) {
        std::fprintf(stderr, "empty region range\n");
        return false;
    }
    if (!p.have_p2_max_y) p.p2_max_y = p.max_height;
    if (p.max_height < -50) p.max_height = -50;
    return true;
}

// One wg_seed_check call; the output grows until it holds every candidate.  The candidates
// are appended to `out` with their seed_index shifted by `index0`.
bool check_seeds(wg_engine *eng, const Params &p, const int64_t *seeds, uint64_t gen_base, uint64_t n,
                 uint64_t index0, std::vector<wg_candidate> &out, int64_t &scanned) {
    std::vector<wg_candidate> buf;
    uint64_t cap = 1u << 16, found = 0;
    wg_scan_stats st{};
    for (;;) {
        buf.resize(cap);
        int rc = wg_seed_check(eng, seeds, gen_base, n, &p.opts, p.max_height, 0, p.min_rx, p.max_rx, p.min_rz,
                               p.max_rz, buf.data(), cap, &found, &st);
        if (rc) {
            std::fprintf(stderr, "scan failed (%d): %s\n", rc, wg_engine_error(eng));
            return false;
        }
        if (found <= cap) break;
        cap = found;
    }
    for (uint64_t k = 0; k < found; k++) {
        buf[k].seed_index += index0;
        out.push_back(buf[k]);
    }
    scanned += st.scanned;
    return true;
}

// --max-hut-dist: the reported position (16 chunkX, 16 chunkZ) within D blocks of the centre
// (phase1_scan.cu:340-349).
bool within_gate(const Params &p, const wg_candidate &c) {
    if (p.max_hut_dist < 0) return true;
    const long long dx = 16LL * c.chunk_x - p.gate_x, dz = 16LL * c.chunk_z - p.gate_z;
    return dx * dx + dz * dz <= p.max_hut_dist * p.max_hut_dist;
}

// --require-all-regions: keeps the candidates of the seeds whose every region of the rect
// passes erosion, temperature and ridge (phase1_scan.cu:145-181).  Only seeds that have a
// candidate can qualify, so only those are re-checked, region by region, through
// wg_phase1_codes (codes 0..2 are the three climate rejections).
bool all_regions_filter(wg_engine *eng, const Params &p, std::vector<wg_candidate> &cands) {
    std::vector<int64_t> seeds;
    for (const wg_candidate &c : cands) seeds.push_back(c.seed);
    std::sort(seeds.begin(), seeds.end());
    seeds.erase(std::unique(seeds.begin(), seeds.end()), seeds.end());
    const uint64_t R = (uint64_t)(p.max_rx - p.min_rx) * (uint64_t)(p.max_rz - p.min_rz);
    const uint64_t per = std::max<uint64_t>(1, (1ull << 26) / R);
    std::vector<char> good(seeds.size(), 0);
    std::vector<int8_t> codes, tiers;
    for (uint64_t k0 = 0; k0 < seeds.size(); k0 += per) {
        const uint64_t n = std::min<uint64_t>(per, seeds.size() - k0);
        codes.assign(n * R, -1);
        tiers.assign(n * R, -1);
        int rc = wg_phase1_codes(eng, seeds.data() + k0, 0, n, &p.opts, p.max_height, 0, p.min_rx, p.max_rx,
                                 p.min_rz, p.max_rz, codes.data(), tiers.data());
        if (rc) {
            std::fprintf(stderr, "all-regions check failed (%d): %s\n", rc, wg_engine_error(eng));
            return false;
        }
        for (uint64_t i = 0; i < n; i++) {
            const int8_t *c = codes.data() + i * R;
            good[k0 + i] = std::all_of(c, c + R, [](int8_t v) { return v > 2; });
        }
    }
    std::vector<wg_candidate> kept;
    for (const wg_candidate &c : cands) {
        const size_t at = (size_t)(std::lower_bound(seeds.begin(), seeds.end(), c.seed) - seeds.begin());
        if (good[at]) kept.push_back(c);
    }
    cands.swap(kept);
    return true;
}

// The world seed of request index i.
int64_t request_seed(const Params &p, uint64_t i) {
    if (!p.quad_bases.empty()) return quad_seed(p, i);
    if (p.gen) return (int64_t)splitmix64(p.gen_base + i);
    return p.seeds[i];
}

// --self-test: sampled regions of the first 16 seeds re-checked through the FP64 noise core, one
// one-region job each, against the scan's phase-1 survivors `cands` (phase1_scan.cu:1289-1326).
// Returns the number of mismatches, or -1 if the check itself failed.
long long self_test(wg_engine *eng, const Params &p, uint64_t n_seeds, const std::vector<wg_candidate> &cands) {
    const uint64_t rw = (uint64_t)(p.max_rx - p.min_rx), rh = (uint64_t)(p.max_rz - p.min_rz);
    const uint64_t total = rw * rh, step = total > 20000 ? total / 20000 : 1;
    const uint64_t ns = std::min<uint64_t>(n_seeds, 16);
    std::vector<int64_t> seeds(ns);
    std::vector<wg_job> jobs;
    for (uint64_t s = 0; s < ns; s++) {
        seeds[s] = request_seed(p, s);
        for (uint64_t idx = 0; idx < total; idx += step) {
            wg_job j{};
            j.seeds = &seeds[s];
            j.n_seeds = 1;
            j.rx0 = p.min_rx + (int)(idx % rw);
            j.rz0 = p.min_rz + (int)(idx / rw);
            j.rx1 = j.rx0 + 1;
            j.rz1 = j.rz0 + 1;
            j.max_height = p.max_height;
            j.opts = p.opts;
            jobs.push_back(j);
        }
    }
    std::vector<uint64_t> job_found(jobs.size(), 0);
    std::vector<wg_candidate> got(jobs.size() + 1);
    uint64_t n_got = 0;
    wg_engine_set_noise_core(eng, WG_NOISE_FP64);
    const int rc = wg_seed_check_jobs(eng, jobs.data(), jobs.size(), got.data(), got.size(), &n_got,
                                      job_found.data(), nullptr);
    wg_engine_set_noise_core(eng, WG_NOISE_FP32);
    if (rc) {
        std::fprintf(stderr, "self-test scan failed (%d): %s\n", rc, wg_engine_error(eng));
        return -1;
    }
    std::vector<std::pair<int64_t, std::pair<int, int>>> hits;   // (seed index, (rx, rz)) of the scan
    for (const wg_candidate &c : cands)
        if (c.seed_index < ns) hits.push_back({(int64_t)c.seed_index, {c.rx, c.rz}});
    std::sort(hits.begin(), hits.end());
    long long mismatches = 0;
    for (size_t k = 0; k < jobs.size(); k++) {
        const int64_t s = (int64_t)(k / ((total + step - 1) / step));
        const bool dev = std::binary_search(hits.begin(), hits.end(), std::make_pair(s, std::make_pair(jobs[k].rx0, jobs[k].rz0)));
        const bool fp64 = job_found[k] != 0;
        if (dev != fp64) {
            if (mismatches < 5)
                std::printf("  MISMATCH seed=%" PRId64 " region(%d,%d): scan=%d fp64=%d\n", seeds[s], jobs[k].rx0,
                            jobs[k].rz0, (int)dev, (int)fp64);
            mismatches++;
        }
    }
    std::printf("self-test: checked %zu sampled regions across %" PRIu64 " seed(s), %lld mismatches -> %s\n",
                jobs.size(), ns, mismatches, mismatches == 0 ? "PASS" : "FAIL");
    return mismatches;
}

// Phase 2 for the phase-1 survivors: keeps the huts lysh_eval_hut accepts at the ceiling, with
// their floor y.
bool confirm(wg_engine *eng, const Params &p, std::vector<wg_candidate> &cands, std::vector<int> &floor_y) {
    floor_y.clear();
    if (cands.empty()) return true;
    std::vector<int64_t> seeds(cands.size());
    std::vector<int32_t> hx(cands.size()), hz(cands.size());
    for (size_t i = 0; i < cands.size(); i++) {
        seeds[i] = cands[i].seed;
        hx[i] = cands[i].chunk_x * 16;
        hz[i] = cands[i].chunk_z * 16;
    }
    std::vector<wg_hut_result> res(cands.size());
    const int rc = wg_eval_huts(eng, seeds.data(), hx.data(), hz.data(), cands.size(), &p.opts, p.p2_max_y, res.data());
    if (rc) {
        std::fprintf(stderr, "phase 2 failed (%d): %s\n", rc, wg_engine_error(eng));
        return false;
    }
    std::vector<wg_candidate> kept;
    for (size_t i = 0; i < cands.size(); i++)
        if (res[i].ok) {
            kept.push_back(cands[i]);
            floor_y.push_back(res[i].avg_y);
        }
    cands.swap(kept);
    return true;
}

int run_scan(wg_engine *eng, const Params &p) {
    const bool quad = !p.quad_bases.empty();
    const uint64_t n = quad ? (uint64_t)p.quad_limit * 65536ull : p.gen ? (uint64_t)p.gen_count : p.seeds.size();
    std::vector<wg_candidate> out;
    std::vector<int> floor_y;
    int64_t scanned = 0;
    auto t0 = std::chrono::steady_clock::now();
    if (quad) {
        // 2^31 seeds at most per request: expanded and checked in slices of 2^22
        constexpr uint64_t kSlice = 1ull << 22;
        std::vector<int64_t> slice;
        for (uint64_t i0 = 0; i0 < n; i0 += kSlice) {
            const uint64_t m = std::min(kSlice, n - i0);
            slice.resize(m);
            for (uint64_t i = 0; i < m; i++) slice[i] = quad_seed(p, i0 + i);
            if (!check_seeds(eng, p, slice.data(), 0, m, i0, out, scanned)) return 1;
        }
    } else if (!check_seeds(eng, p, p.gen ? nullptr : p.seeds.data(), p.gen_base, n, 0, out, scanned)) {
        return 1;
    }
    long long mismatches = 0;
    if (p.self_test && (mismatches = self_test(eng, p, n, out)) < 0) return 1;
    if (p.max_hut_dist >= 0)
        out.erase(std::remove_if(out.begin(), out.end(), [&](const wg_candidate &c) { return !within_gate(p, c); }),
                  out.end());
    if (p.require_all && !out.empty() && !all_regions_filter(eng, p, out)) return 1;
    const uint64_t phase1 = out.size();
    if (!p.phase1_only && !confirm(eng, p, out, floor_y)) return 1;
    const uint64_t found = out.size();
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("kernel: %.3f s  candidates=%" PRIu64 "  (%.2f M region-seed-checks/s across %" PRIu64 " seed(s))\n",
                secs, found, secs > 0 ? (double)scanned / secs / 1e6 : 0.0, n);
    if (!p.phase1_only)
        std::printf("phase 2: %" PRIu64 " phase-1 survivors, %" PRIu64 " huts with floor <= %d\n", phase1, found,
                    p.p2_max_y);
    if (!p.out_path.empty()) {
        FILE *f = std::fopen(p.out_path.c_str(), "w");
        if (!f) {
            std::fprintf(stderr, "cannot write %s\n", p.out_path.c_str());
            return 1;
        }
        std::fprintf(f, "seed,chunkX,chunkZ,blockX,blockZ,gpuEst\n");
        for (size_t i = 0; i < out.size(); i++) {
            const wg_candidate &c = out[i];
            std::fprintf(f, "%" PRId64 ",%d,%d,%d,%d,", c.seed, c.chunk_x, c.chunk_z, c.chunk_x * 16, c.chunk_z * 16);
            if (p.phase1_only) std::fprintf(f, "nan\n");
            else std::fprintf(f, "%d\n", floor_y[i]);
        }
        std::fclose(f);
        std::printf("wrote %zu candidates to %s\n", out.size(), p.out_path.c_str());
    }
    if (mismatches) {
        std::fprintf(stderr, "self-test FAILED\n");
        return 1;
    }
    return 0;
}

std::vector<std::string> tokenize(std::string line) {
    if (line.size() >= 3 && (unsigned char)line[0] == 0xEF && (unsigned char)line[1] == 0xBB &&
        (unsigned char)line[2] == 0xBF)
        line.erase(0, 3);
    std::vector<std::string> out;
    std::istringstream iss(line);
    std::string tok;
    while (iss >> tok) out.push_back(tok);
    return out;
}

void usage() {
    std::printf(
        "usage: phase1_scan --seed <n> [--seed <n> ...] [--seed-list <file>] [options]\n"
        "       phase1_scan --seed-gen <base> <count> [options]\n"
        "       phase1_scan --worker\n"
        "  --min-region-x/--max-region-x/--min-region-z/--max-region-z <n>  rect, max exclusive (default +-128)\n"
        "  --max-height <n>     phase-1 maxHeight, default -40 (-50/-54 -> -50)\n"
        "  --version <v>        lysh version name (default 1.19.x~26.1); --v26-2 = 26.2 ridge rule\n"
        "  --preset <p>         NORMAL | LARGE_BIOMES | SINGLE_BIOME\n"
        "  --out <file>         CSV seed,chunkX,chunkZ,blockX,blockZ,gpuEst (gpuEst = the hut's floor y)\n"
        "  --phase2-max-y <y>   phase-2 ceiling: keep huts with floor <= y (default --max-height)\n"
        "  --phase1-candidates  write every phase-1 survivor (unconfirmed, gpuEst nan)\n"
        "  --self-test          re-check sampled regions through the FP64 noise core; rc 1 on a mismatch\n"
        "  --quad-bases <file>  sweep every base x its 65,536 high-16-bit variants\n"
        "  --quad-base-offset <n> / --quad-base-limit <n>  slice of the base list (limit <= 32767)\n"
        "  --max-hut-dist <d>   keep huts within d blocks of --gate-center-x/--gate-center-z\n"
        "  --require-all-regions  a seed needs every region to pass the climate gates\n"
        "  --device <n>         CUDA device (default 0)\n"
        "  --worker             read one request per stdin line; ===WORKER_READY===, ===SCAN_DONE rc=N===\n");
}

}  // namespace

int main(int argc, char **argv) {
    std::setvbuf(stdout, nullptr, _IOLBF, 1024);
    std::vector<std::string> tokens;
    int device = 0;
    bool worker = false;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        if (a == "--device" && i + 1 < argc) { device = std::atoi(argv[++i]); continue; }
        if (a == "--worker") worker = true;
        if (a == "--help" || a == "-h") { usage(); return 0; }
        tokens.push_back(a);
    }
    if (!worker && tokens.empty()) { usage(); return 2; }
    Params p;
    if (!worker && !parse(tokens, p)) { usage(); return 2; }
    wg_engine *eng = nullptr;
    int rc = wg_engine_open(device, &eng);
    if (rc) {
        std::fprintf(stderr, "cannot open the GPU engine on device %d (status %d)\n", device, rc);
        return 1;
    }
    if (!worker) {
        rc = run_scan(eng, p);
        wg_engine_close(eng);
        return rc;
    }
    std::printf("===WORKER_READY===\n");
    std::fflush(stdout);
    std::string line;
    while (std::getline(std::cin, line)) {
        if (line.empty()) continue;
        Params q;
        if (!parse(tokenize(line), q)) {
            std::printf("===SCAN_ERROR: bad request line===\n");
            std::fflush(stdout);
            continue;
        }
        int r = run_scan(eng, q);
        std::printf("===SCAN_DONE rc=%d===\n", r);
        std::fflush(stdout);
    }
    wg_engine_close(eng);
    return 0;
}
