// biome_map: drop-in for the map tab's biome raster tool (engine/tools/mineshaft/biome_map.c,
// usage at :1-20, arguments :54-86) on top of libwitchgpu.so, with the same flags, limits,
// exit codes and raw-byte output:
//
//   biome_map --seed S --x0 X --z0 Z --w W --h H [--step B] [--ss K] [--ver V] [--y Y]
//   biome_map --seed S --stdin [--ver V] [--y Y]          ("cx cz" lines in, one byte each out)
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/witchgpu.h"

int main(int argc, char **argv) {
    long long seed = 0, x0 = 0, z0 = 0;
    int w = 0, h = 0, step = 16, have = 0, from_stdin = 0, ss = 1, y = 63;
    const char *ver = "26.3";
    for (int i = 1; i < argc; i++) {
        if (!std::strcmp(argv[i], "--seed") && i + 1 < argc) { seed = std::atoll(argv[++i]); have |= 1; }
        else if (!std::strcmp(argv[i], "--x0") && i + 1 < argc) { x0 = std::atoll(argv[++i]); have |= 2; }
        else if (!std::strcmp(argv[i], "--z0") && i + 1 < argc) { z0 = std::atoll(argv[++i]); have |= 4; }
        else if (!std::strcmp(argv[i], "--w") && i + 1 < argc) { w = std::atoi(argv[++i]); have |= 8; }
        else if (!std::strcmp(argv[i], "--h") && i + 1 < argc) { h = std::atoi(argv[++i]); have |= 16; }
        else if (!std::strcmp(argv[i], "--step") && i + 1 < argc) step = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--ss") && i + 1 < argc) ss = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--ver") && i + 1 < argc) ver = argv[++i];
        else if (!std::strcmp(argv[i], "--y") && i + 1 < argc) y = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--stdin")) { from_stdin = 1; have |= 30; }
        else { std::fprintf(stderr, "biome_map: unknown arg %s\n", argv[i]); return 2; }
    }
    if (from_stdin) w = h = 1;
    if (have != 31 || w <= 0 || h <= 0 || w > 4096 || h > 4096 || step < 1 || ss < 1 || ss > 4) {
        std::fprintf(stderr, "usage: biome_map --seed S (--x0 X --z0 Z --w W --h H [--step B] [--ss 1..4] | --stdin) "
                             "[--ver 1.18.2|1.19.3|...|26.3] [--y Y]\n");
        return 2;
    }
    wg_opts o;
    std::memset(&o, 0, sizeof o);
    if (wg_parse_version(ver, &o) != WG_OK || o.biome_tree == 0) {
        std::fprintf(stderr, "biome_map: --ver must be a game version such as 1.18.2, 1.19.3, 1.21.4 or 26.3\n");
        return 2;
    }
    wg_engine *eng = nullptr;
    if (wg_engine_open(0, &eng) != WG_OK) { std::fprintf(stderr, "biome_map: no GPU engine\n"); return 1; }
    int rc = WG_OK;
    if (from_stdin) {
        std::vector<int32_t> cx, cz;
        long long a, b;
        while (std::scanf("%lld %lld", &a, &b) == 2) {
            cx.push_back((int32_t)a);
            cz.push_back((int32_t)b);
        }
        std::vector<uint8_t> out(cx.size());
        if (!cx.empty()) rc = wg_biome_chunks(eng, seed, &o, cx.data(), cz.data(), cx.size(), out.data());
        if (rc == WG_OK && !out.empty() && std::fwrite(out.data(), 1, out.size(), stdout) != out.size()) rc = WG_ERR_ARG;
    } else {
        std::vector<uint8_t> out((size_t)w * (size_t)h);
        rc = wg_biome_map(eng, seed, &o, x0, z0, w, h, step, ss, y, out.data());
        if (rc == WG_OK && std::fwrite(out.data(), 1, out.size(), stdout) != out.size()) rc = WG_ERR_ARG;
    }
    if (rc != WG_OK) std::fprintf(stderr, "biome_map: %s\n", wg_engine_error(eng));
    wg_engine_close(eng);
    return rc == WG_OK ? 0 : 1;
}
