/* Test infrastructure only (the checker, never the product).
 *
 * Flat, ctypes-friendly wrappers around the reference's own lysh library, compiled from the
 * reference sources by oracle/Makefile into oracle/_ref/liblysh_ref.so.  Every function here
 * only calls lysh's public entry points; no world-generation arithmetic lives in this file.
 *
 *   lysh_phase1_init / lysh_phase1_check_ex / lysh_phase1_probe   engine/tools/lysh/src/phase1.c:11,130,47
 *   lysh_swamp_hut_in_region                                      engine/tools/lysh/src/structure.c:14
 *   lysh_dblnoise_from_seed_id                                    engine/tools/lysh/src/noise.c:145
 *   lysh_search_ctx_init / lysh_eval_hut / lysh_grade_scan        engine/tools/lysh/src/eval.c:70,121,481
 *   lysh_scan_rect (phase-1 only, no phase-2 hook)                engine/tools/lysh/src/search.c:198
 */
#include <limits.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "biome.h"
#include "column_top.h"
#include "eval.h"
#include "noise.h"
#include "phase1.h"
#include "phase2.h"
#include "search.h"
#include "structure.h"

static lysh_phase1_opts mk_opts(int mc118, int pre262, int large, int single, int tree) {
    lysh_phase1_opts o;
    memset(&o, 0, sizeof(o));
    o.mc_1_18_2 = mc118;
    o.pre_26_2 = pre262;
    o.large_biomes = large;
    o.single_biome = single;
    o.biome_tree = tree;
    return o;
}

/* Version string -> option bits, the same name table `lysh --version` accepts
 * (engine/tools/lysh/src/main.c:104-125).  Returns 0 on success. */
int refh_parse_version(const char *s, int *mc118, int *pre262, int *tree) {
    int tr, is118, pre;
    *tree = 0;
    if (!lysh_biome_version(s, &tr, &is118, &pre)) {
        *mc118 = is118; *pre262 = pre; *tree = tr + 1;
        return 0;
    }
    const char *v118[] = {"1.18.2", "1.18", "1.18.x", "1.18.1", NULL};
    const char *vpre[] = {"1.19.2", "1.19", "1.19.x", "1.20.1", "1.20", "1.20.x", "1.21", "1.21.1",
                          "1.21.x~26.1", "1.21.5~26.1", "1.19.x~26.1", "26.1", NULL};
    for (int i = 0; v118[i]; i++) if (!strcmp(s, v118[i])) { *mc118 = 1; *pre262 = 1; return 0; }
    for (int i = 0; vpre[i]; i++) if (!strcmp(s, vpre[i])) { *mc118 = 0; *pre262 = 1; return 0; }
    if (!strcmp(s, "26.2") || !strcmp(s, "26.2~26.3")) { *mc118 = 0; *pre262 = 0; return 0; }
    if (!strcmp(s, "26.3")) {
        *mc118 = 0; *pre262 = 0;
        lysh_biome_version("26.3", &tr, NULL, NULL);
        *tree = tr + 1;
        return 0;
    }
    return 1;
}

int refh_hut_in_region(uint64_t seed, int rx, int rz, int salt, int *cx, int *cz) {
    lysh_chunkpos p = lysh_swamp_hut_in_region(seed, rx, rz, salt ? salt : LYSH_SWAMP_HUT_SALT);
    *cx = p.chunkX;
    *cz = p.chunkZ;
    return 0;
}

int refh_hut_orientation(uint64_t seed, int hut_x, int hut_z) {
    return lysh_hut_orientation(seed, hut_x, hut_z);
}

/* Phase-1 verdict of every region of [rx0,rx1) x [rz0,rz1), rz outer and rx inner (the
 * enumeration order of search.c:148-149).  codes[k] = LYSH_P1_* reject code (10 = accept),
 * tiers[k] = erosion tier that rejected early (-1 if none), cx/cz = hut chunk. */
long long refh_phase1_rect(uint64_t seed, int mc118, int pre262, int large, int single, int tree,
                           int max_height, int salt, int rx0, int rx1, int rz0, int rz1,
                           signed char *codes, signed char *tiers, int *cx, int *cz) {
    lysh_phase1_opts o = mk_opts(mc118, pre262, large, single, tree);
    lysh_phase1 *p = (lysh_phase1 *)malloc(sizeof(lysh_phase1));
    if (!p) return -1;
    lysh_phase1_init(p, seed, &o);
    long long k = 0;
    for (int rz = rz0; rz < rz1; rz++) {
        for (int rx = rx0; rx < rx1; rx++) {
            lysh_chunkpos pos = lysh_swamp_hut_in_region(seed, rx, rz, salt ? salt : LYSH_SWAMP_HUT_SALT);
            long long hist[LYSH_TIER_MAX];
            memset(hist, 0, sizeof(hist));
            lysh_phase1_result r;
            r.reject = -1;
            lysh_phase1_check_ex(p, &o, pos.chunkX * 16, pos.chunkZ * 16, max_height, &r, hist);
            int t = -1;
            for (int i = 0; i < LYSH_TIER_MAX; i++) if (hist[i]) t = i;
            if (codes) codes[k] = (signed char)r.reject;
            if (tiers) tiers[k] = (signed char)t;
            if (cx) cx[k] = pos.chunkX;
            if (cz) cz[k] = pos.chunkZ;
            k++;
        }
    }
    free(p);
    return k;
}

/* The 38 raw probe doubles at one hut (phase1.c:47-87 order). */
int refh_probe(uint64_t seed, int mc118, int pre262, int large, int single, int tree,
               int hut_x, int hut_z, int max_height, double *out) {
    lysh_phase1_opts o = mk_opts(mc118, pre262, large, single, tree);
    lysh_phase1 *p = (lysh_phase1 *)malloc(sizeof(lysh_phase1));
    if (!p) return -1;
    lysh_phase1_init(p, seed, &o);
    lysh_phase1_probe(p, hut_x, hut_z, max_height, out);
    free(p);
    return LYSH_P1_PROBE_N;
}

/* One DoublePerlin noise's constructed state: for sub s (0/1) and octave slot i (< 16):
 * present[s*16+i], origin[(s*16+i)*3 + {0,1,2}], perm[(s*16+i)*256 + k]; head[] =
 * {amplitude, lacunarity0, persistence0, lacunarity1, persistence1, n}. */
int refh_noise_dump(uint64_t seed, const char *id, double *head, int *present, double *origin,
                    unsigned char *perm) {
    lysh_dblnoise *dn = (lysh_dblnoise *)malloc(sizeof(lysh_dblnoise));
    if (!dn) return -1;
    lysh_dblnoise_from_seed_id(dn, seed, id);
    head[0] = dn->amplitude;
    head[1] = dn->sub[0].lacunarity;
    head[2] = dn->sub[0].persistence;
    head[3] = dn->sub[1].lacunarity;
    head[4] = dn->sub[1].persistence;
    head[5] = dn->sub[0].n;
    for (int s = 0; s < 2; s++) {
        for (int i = 0; i < LYSH_MAX_OCT; i++) {
            const lysh_perlin *pl = &dn->sub[s].oct[i];
            int k = s * LYSH_MAX_OCT + i;
            present[k] = (i < dn->sub[s].n) ? pl->present : 0;
            origin[k * 3 + 0] = present[k] ? pl->ox : 0.0;
            origin[k * 3 + 1] = present[k] ? pl->oy : 0.0;
            origin[k * 3 + 2] = present[k] ? pl->oz : 0.0;
            memcpy(perm + (size_t)k * 256, pl->perm, 256);
            if (!present[k]) memset(perm + (size_t)k * 256, 0, 256);
        }
    }
    free(dn);
    return 0;
}

/* ---------------- phase 2: one search ctx per handle ---------------- */
void *refh_ctx_new(uint64_t seed, int mc118, int pre262, int large, int single, int tree, int max_height) {
    lysh_phase1_opts o = mk_opts(mc118, pre262, large, single, tree);
    lysh_search_ctx *ctx = (lysh_search_ctx *)calloc(1, sizeof(lysh_search_ctx));
    if (!ctx) return NULL;
    lysh_search_ctx_init(ctx, seed, &o, max_height);
    return ctx;
}

void refh_ctx_free(void *h) {
    if (!h) return;
    lysh_search_ctx_free((lysh_search_ctx *)h);
    free(h);
}

/* lysh_eval_hut -> out[24]:
 * 0 dir 1 size_x 2 size_z 3 avg_y 4 sum_h 5 wet 6 flooded 7 ok 8 reject 9 biome_ok 10 winner
 * 11 qx 12 qy 13 qz 14 occ_y 15..20 t[6] 21 rx 22 rz 23 all_dry */
void refh_ctx_eval(void *h, int hut_x, int hut_z, int max_y, long long *out) {
    lysh_hut_result r = lysh_eval_hut((lysh_search_ctx *)h, hut_x, hut_z, max_y);
    out[0] = r.dir; out[1] = r.size_x; out[2] = r.size_z; out[3] = r.avg_y; out[4] = r.sum_h;
    out[5] = r.wet_columns; out[6] = r.flooded; out[7] = r.ok; out[8] = r.reject;
    out[9] = r.biome_ok; out[10] = r.biome_winner; out[11] = r.biome_qx; out[12] = r.biome_qy;
    out[13] = r.biome_qz; out[14] = r.biome_occ_y;
    for (int i = 0; i < 6; i++) out[15 + i] = r.biome_t[i];
    out[21] = r.rx; out[22] = r.rz; out[23] = r.all_dry;
}

int refh_ctx_height(void *h, int x, int z, int carved) {
    lysh_search_ctx *c = (lysh_search_ctx *)h;
    return carved ? lysh_phase2_height(&c->p2, x, z) : lysh_phase2_height_pre_carver(&c->p2, x, z);
}

double refh_ctx_density(void *h, int x, int y, int z) {
    lysh_search_ctx *c = (lysh_search_ctx *)h;
    return lysh_phase2_density_at(&c->p2, x, y, z);
}

int refh_ctx_block(void *h, int x, int y, int z) {
    lysh_search_ctx *c = (lysh_search_ctx *)h;
    return (int)lysh_phase2_block_at(&c->p2, x, y, z);
}

/* Phase-2 probes, kind for kind the ones the GPU engine's wg_p2_probe answers:
 *   0 lysh_interp_calculate_noise_261 (interp_noise.c:100)   1 lysh_phase2_density_raw_at (phase2.c:151)
 *   2 lysh_preliminary_surface_level (column_top.c:94)       3/4/5 terrain info cont / erosion / weirdness
 *   6/7/8 terrain point offset / factor / peaks (26.1)        9 computeFluid: level * 4 + type (aquifer.c:327)
 *   10 lysh_phase2_density_at  11 lysh_phase2_block_at  12 height before carvers  13 height after carvers */
void refh_ctx_probe(void *h, int kind, const int *xyz, long long n, double *out) {
    lysh_search_ctx *c = (lysh_search_ctx *)h;
    for (long long i = 0; i < n; i++) {
        const int x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
        double v = 0.0;
        lysh_terrain_info ti;
        switch (kind) {
            case 0: v = lysh_interp_calculate_noise_261(&c->p2.interp, x, y, z); break;
            case 1: v = lysh_phase2_density_raw_at(&c->p2, x, y, z); break;
            case 2: v = (double)lysh_preliminary_surface_level(&c->p2.terrain, x, z); break;
            case 3: case 4: case 5: case 6: case 7: case 8:
                lysh_terrain_info_at(&c->p2.terrain, x >> 2, z >> 2, &ti);
                v = kind == 3 ? ti.continentalness : kind == 4 ? ti.erosion : kind == 5 ? ti.weirdness
                  : kind == 6 ? (double)ti.point.offset : kind == 7 ? (double)ti.point.factor
                  : (double)ti.point.peaks;
                break;
            case 9: {
                int level;
                lysh_block_state type;
                lysh_aquifer_compute_fluid(&c->p2.aquifer, x, y, z, &level, &type);
                v = (double)level * 4.0 + (double)type;
                break;
            }
            case 10: v = lysh_phase2_density_at(&c->p2, x, y, z); break;
            case 11: v = (double)lysh_phase2_block_at(&c->p2, x, y, z); break;
            case 12: v = (double)lysh_phase2_height_pre_carver(&c->p2, x, z); break;
            case 13: v = (double)lysh_phase2_height(&c->p2, x, z); break;
            default: break;
        }
        out[i] = v;
    }
}

/* lysh_grade_scan: phase 1 + phase 2 over a rect for one seed.  stats[0..6] =
 * scanned, evaluated, accepted, rejected_y, rejected_flood, rejected_biome, hits_written. */
void refh_grade_scan(uint64_t seed, int mc118, int pre262, int large, int single, int tree,
                     int max_height, int rx0, int rx1, int rz0, int rz1, int salt, int threads,
                     int max_y, int *hits, int cap, long long *stats) {
    lysh_phase1_opts o = mk_opts(mc118, pre262, large, single, tree);
    lysh_hut_grade g;
    memset(&g, 0, sizeof(g));
    g.hits = hits;
    g.hits_cap = cap;
    lysh_grade_scan(seed, &o, max_height, rx0, rx1, rz0, rz1, salt ? salt : LYSH_SWAMP_HUT_SALT,
                    threads, max_y, &g);
    stats[0] = g.scanned; stats[1] = g.evaluated; stats[2] = g.accepted; stats[3] = g.rejected_y;
    stats[4] = g.rejected_flood; stats[5] = g.rejected_biome; stats[6] = g.hits_written;
}

/* ---------------- timed CPU baseline: many seeds, all host threads ----------------
 * Each seed runs lysh's own phase-1 scan (lysh_scan_rect without a phase-2 hook: one
 * lysh_phase1_init per seed, then every region through lysh_phase1_check_ex), one seed per
 * worker at a time; seeds are handed out dynamically.  accepted[i] = phase-1 survivors. */
typedef struct {
    const uint64_t *seeds;
    long long n;
    lysh_phase1_opts o;
    int max_height, salt, rx0, rx1, rz0, rz1;
    long long *accepted;
    long long next;
    pthread_mutex_t mu;
} seeds_job;

static void *seeds_worker(void *arg) {
    seeds_job *j = (seeds_job *)arg;
    for (;;) {
        pthread_mutex_lock(&j->mu);
        long long i = j->next++;
        pthread_mutex_unlock(&j->mu);
        if (i >= j->n) break;
        lysh_scan_opts so;
        memset(&so, 0, sizeof(so));
        so.seed = j->seeds[i];
        so.opts = j->o;
        so.max_height = j->max_height;
        so.salt = j->salt ? j->salt : LYSH_SWAMP_HUT_SALT;
        so.threads = 1;
        lysh_scan_result res;
        lysh_scan_rect(&so, j->rx0, j->rx1, j->rz0, j->rz1, &res);
        if (j->accepted) j->accepted[i] = res.accepted;
    }
    return NULL;
}

double refh_phase1_seeds(const uint64_t *seeds, long long n, int mc118, int pre262, int large,
                         int single, int tree, int max_height, int salt, int rx0, int rx1,
                         int rz0, int rz1, int threads, long long *accepted) {
    seeds_job j;
    memset(&j, 0, sizeof(j));
    j.seeds = seeds; j.n = n; j.o = mk_opts(mc118, pre262, large, single, tree);
    j.max_height = max_height; j.salt = salt;
    j.rx0 = rx0; j.rx1 = rx1; j.rz0 = rz0; j.rz1 = rz1;
    j.accepted = accepted;
    pthread_mutex_init(&j.mu, NULL);
    if (threads < 1) threads = lysh_cpu_count();
    pthread_t *th = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    for (int t = 0; t < threads; t++) pthread_create(&th[t], NULL, seeds_worker, &j);
    for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
    clock_gettime(CLOCK_MONOTONIC, &t1);
    free(th);
    pthread_mutex_destroy(&j.mu);
    return (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
}

int refh_cpu_count(void) { return lysh_cpu_count(); }
