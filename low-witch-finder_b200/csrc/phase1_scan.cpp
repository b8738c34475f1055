// phase1_scan: drop-in replacement for the reference GPU scanner's command-line and
// --worker contract (engine/gpu/low54/phase1_scan.cu:561-601 usage, :641-759 flags,
// :1328-1339 CSV, :1365-1387 worker loop), on top of libwitchgpu.so.
//
// Differences a caller can observe:
//   * The candidate set is exactly lysh's phase-1 survivor set (lysh_phase1_check_ex),
//     not the reference GPU scanner's superset; there is no lossy density prefilter, so
//     --no-density-prefilter / --climate-gate / --no-climate-gate / --block are accepted
//     and change nothing.
//   * --max-height is clamped like lysh's phase1CheckHeight (-50 / -54 -> -50,
//     engine/tools/lysh/src/main.c:135-137).
//   * --version / --preset take lysh's names (default 1.19.x~26.1, the hunt driver's);
//     --v26-2 selects the 26.2 ridge rule as before.
//   * The 6th CSV column (gpuEst) is "nan": the reference's prefilter estimate does not exist.
//   * --quad-bases / --require-all-regions / --max-hut-dist / --gate-center-* are refused
//     with a clear error (not part of the Seed Check path).
#include <cctype>
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
};

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
        else if (a == "--self-test" || a == "--no-density-prefilter" || a == "--climate-gate" ||
                 a == "--no-climate-gate" || a == "--worker") {
        } else if (a == "--quad-bases" || a == "--quad-base-offset" || a == "--quad-base-limit" ||
                   a == "--require-all-regions" || a == "--max-hut-dist" || a == "--gate-center-x" ||
                   a == "--gate-center-z") {
            std::fprintf(stderr, "unsupported option %s (not part of the Seed Check path)\n", a.c_str());
            ok = false;
        } else {
            std::fprintf(stderr, "unknown argument: %s\n", a.c_str());
            ok = false;
        }
    }
    if (!ok) return false;
    if (p.gen && !p.seeds.empty()) {
        std::fprintf(stderr, "--seed-gen cannot be combined with --seed/--seed-list\n");
        return false;
    }
    if (p.gen && p.gen_count <= 0) {
        std::fprintf(stderr, "--seed-gen count must be positive\n");
        return false;
    }
    if (!p.gen && p.seeds.empty()) {
        std::fprintf(stderr, "no seeds given\n");
        return false;
    }
    if (p.max_rx <= p.min_rx || p.max_rz <= p.min_rz) {
        std::fprintf(stderr, "empty region range\n");
        return false;
    }
    if (p.max_height < -50) p.max_height = -50;
    return true;
}

int run_scan(wg_engine *eng, const Params &p) {
    uint64_t n = p.gen ? (uint64_t)p.gen_count : p.seeds.size();
    std::vector<wg_candidate> out;
    uint64_t cap = 1u << 16, found = 0;
    wg_scan_stats st{};
    auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        out.resize(cap);
        int rc = wg_seed_check(eng, p.gen ? nullptr : p.seeds.data(), p.gen_base, n, &p.opts, p.max_height, 0,
                               p.min_rx, p.max_rx, p.min_rz, p.max_rz, out.data(), cap, &found, &st);
        if (rc) {
            std::fprintf(stderr, "scan failed (%d): %s\n", rc, wg_engine_error(eng));
            return 1;
        }
        if (found <= cap) break;
        cap = found;
    }
    out.resize(found);
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("kernel: %.3f s  candidates=%" PRIu64 "  (%.2f M region-seed-checks/s across %" PRIu64 " seed(s))\n",
                secs, found, secs > 0 ? (double)st.scanned / secs / 1e6 : 0.0, n);
    if (!p.out_path.empty()) {
        FILE *f = std::fopen(p.out_path.c_str(), "w");
        if (!f) {
            std::fprintf(stderr, "cannot write %s\n", p.out_path.c_str());
            return 1;
        }
        std::fprintf(f, "seed,chunkX,chunkZ,blockX,blockZ,gpuEst\n");
        for (const wg_candidate &c : out)
            std::fprintf(f, "%" PRId64 ",%d,%d,%d,%d,nan\n", c.seed, c.chunk_x, c.chunk_z, c.chunk_x * 16,
                         c.chunk_z * 16);
        std::fclose(f);
        std::printf("wrote %zu candidates to %s\n", out.size(), p.out_path.c_str());
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
        "  --out <file>         CSV seed,chunkX,chunkZ,blockX,blockZ,gpuEst\n"
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
