/* Test infrastructure only: the CPU oracle (the checker), never the product.
 *
 * A plain-C restatement of the reference's Seed Check phase-1 path (lysh):
 * Java-LCG swamp-hut region placement, Xoroshiro128++ noise derivation, Perlin /
 * Octave / DoublePerlin construction and sampling, the tiered erosion gate, the
 * climate gates and the cave / continentalness / floodedness ladder.  Each function in
 * witch_oracle.c cites the reference file:line it restates.  Only tests/, the smoke
 * check and bench.py's CPU baseline load this library.
 */
#ifndef WITCH_ORACLE_H
#define WITCH_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Version / preset bits, same meaning as lysh_phase1_opts (engine/tools/lysh/src/phase1.h:45-57). */
typedef struct {
    int mc_1_18_2;
    int single_biome;
    int pre_26_2;
    int large_biomes;
} wo_opts;

/* One phase-1 survivor. */
typedef struct {
    uint64_t seed_index;
    int64_t seed;
    int32_t rx, rz;
    int32_t chunk_x, chunk_z;
} wo_candidate;

uint64_t wo_splitmix64(uint64_t x);
void wo_md5(const uint8_t *data, uint64_t len, uint8_t out[16]);
void wo_hut_in_region(uint64_t seed, int rx, int rz, int salt, int *cx, int *cz);
int wo_orientation(uint64_t seed, int hut_x, int hut_z);

/* Same layout as the reference harness's refh_noise_dump. */
int wo_noise_dump(uint64_t seed, const char *id, double *head, int *present, double *origin,
                  unsigned char *perm);

/* Per-region phase-1 verdicts over a rect, rz outer / rx inner. */
long long wo_phase1_rect(uint64_t seed, const wo_opts *o, int max_height, int salt,
                         int rx0, int rx1, int rz0, int rz1,
                         signed char *codes, signed char *tiers, int *cx, int *cz);

/* The 38 fixed-order probe doubles. */
/* Deep Dive (engine/gpu/room_core.h): is chunk (cx, cz) a mineshaft start of structure seed
 * s48; and every region of a rect whose swamp-hut chunk is one, as rows (s48, rx, rz, cx, cz,
 * carver), seed-major, rz outer, rx inner.  Returns the number found (rows beyond cap unwritten). */
int wo_mineshaft_start(uint64_t s48, int cx, int cz, uint64_t *carver_out);
long long wo_deep_starts(const uint64_t *s48s, long long n, int rx0, int rx1, int rz0, int rz1, int64_t *out,
                         long long cap);

int wo_probe(uint64_t seed, const wo_opts *o, int hut_x, int hut_z, int max_height, double *out);

/* Phase-1 survivors of many seeds over one rect (threads <= 0: all cores).  Seeds are
 * seeds[i] when seeds != NULL, else splitmix64(gen_base + i).  Writes up to cap
 * survivors (unordered across seeds, rz/rx order within a seed), returns the total found
 * (which may exceed cap).  reject_hist (11 entries, may be NULL) receives the funnel. */
long long wo_scan_seeds(const uint64_t *seeds, uint64_t gen_base, long long n, const wo_opts *o,
                        int max_height, int salt, int rx0, int rx1, int rz0, int rz1, int threads,
                        wo_candidate *out, long long cap, long long *reject_hist);


/* Deep Dive solver (engine/gpu/solver_kernels.cuh, taskspace.h) */
uint64_t wo_region_const(int rx, int rz);
uint32_t wo_perm_group(uint32_t p);
long long wo_group_regions(uint32_t c20, int regime_x, int regime_z, int32_t *rx_out, int32_t *rz_out, long long cap);
long long wo_solve_task(uint64_t X, int rx, int rz, int ox, int oz, uint64_t *out, long long cap);

#ifdef __cplusplus
}
#endif

#endif
