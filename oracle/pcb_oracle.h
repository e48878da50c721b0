/* CPU oracle for the pcbroute search back end -- TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load this library, and only as the
 * checker (or the timed CPU baseline); the product path never calls it.
 *
 * It restates, in plain C and single-threaded exact arithmetic, what one gpu_solve() call of pcbroute computes
 * (src/gpu.cu:550-622 with src/gpu.cu:78-115 for the cost resolution and src/gpu.cu:122-363 for the relaxation
 * rule), under the fixed-point contract written at the top of include/pcbg.h. Where the reference GPU code
 * relaxes with float sweeps whose result depends on the sweep schedule, the oracle computes the unique integer
 * least fixed point with Dijkstra's algorithm; the B200 kernels must reproduce it bit for bit.
 *
 * Parity pin: the reference's tests hold no distance fields or paths for this path (tests/test_gpu_gate.py only
 * checks that the GPU is used and the board completes). The oracle is pinned by (a) the reference router itself:
 * linked with this oracle as its gpu.h back end (oracle/Makefile) it passes the reference's own GPU gate checks,
 * and with --gpu-pops 0 it writes sessions byte-identical to the unmodified reference binary; (b) a brute-force
 * Bellman-Ford in the test suite; (c) committed golden fixtures (tests/golden/) generated by this oracle.
 */
#ifndef PCB_ORACLE_H
#define PCB_ORACLE_H

#include "../include/pcbg.h"

#ifdef __cplusplus
extern "C" {
#endif

/* "unreached" and the saturation value of 64-bit distances (a byte pattern, as on the device) */
#define PCBO_INF64 0x7F7F7F7F7F7F7F7Full
/* a move whose 16 x cost reaches this is impassable */
#define PCBO_WLIM 4611686018427387904.0f

/* Fixed-point weight of a move into a state of cost factor cf with move factor fac (PCBO_INF64: impassable). */
uint64_t pcbo_weight(float cf, float fac);
/* Fixed-point cost of a start of float cost g0. */
uint64_t pcbo_start_d(float g0);
/* fac[l][m] of a query: fl(len[m] * dirf[l][m]). */
void pcbo_factors(float step, const float dirf[8][8], float fac[8][8]);

/* Resolve the costs of the rectangle [rx0, rx0 + rw) x [ry0, ry0 + rh) of the query's window, as the reference's
 * prep_cf / prep_v kernels do after the own-copper overrides (src/gpu.cu:78-115, 460-478): dense outputs
 * cf[l][j][i], flags[l][j][i] (bit0 a via may land, bit1 target), vcf[j][i] (NULL to skip). */
void pcbo_resolve(const pcbg_query* q, int rx0, int ry0, int rw, int rh, float* cf, uint8_t* flags, float* vcf);

/* Exact least fixed point over a resolved dense rectangle. starts: rect states and fixed-point costs (the least
 * per state counts). dist: nl*rh*rw 64-bit distances (PCBO_INF64 unreached). Returns best rect state or -1, and
 * its cost in *best_d. When a target is reached, the search stops once it has settled every state at or below the
 * target's cost (the part of the field a solve reports); states above it keep upper bounds. */
int64_t pcbo_dijkstra(int rw, int rh, int nl, const float fac[8][8], const float* cf, const uint8_t* flags,
                      const float* vcf, int64_t n_starts, const uint32_t* start_idx, const uint64_t* start_d,
                      uint64_t* dist, uint64_t* best_d);

/* Walk-back over an exact field from `best` to a start (src/router.cpp:1615-1679 order): at each state stop if it
 * is a start at its own start cost, else step to the first predecessor, moves 0-7 then via layers ascending, whose
 * distance plus the move's weight equals this state's. Writes rect states, best first. Returns the states written,
 * 0 if best < 0, -1 if no predecessor exists or the walk exceeds cap. */
int64_t pcbo_walkback(int rw, int rh, int nl, const float fac[8][8], const float* cf, const uint8_t* flags,
                      const float* vcf, int64_t n_starts, const uint32_t* start_idx, const uint64_t* start_d,
                      const uint64_t* dist, int64_t best, uint32_t* path, int64_t cap);

/* The reported float field of a solved rectangle: d / 16 where d <= d(best) (every reached state if best < 0). */
void pcbo_report(int64_t n, const uint64_t* dist, int64_t best, uint64_t best_d, float* out);

/* One whole gpu_solve(): rectangle growth from the start/target box with the octile stop (src/gpu.cu:575-619),
 * each rectangle resolved and solved exactly. out->d is malloc'd (free with pcbo_free). Returns tries (>= 1)
 * or -1 (no starts or no targets). */
int pcbo_solve(const pcbg_query* q, pcbg_result* out);
void pcbo_free(float* p);
/* The state cap of one rectangle (gpu_configure's max_states; 0: none). A rectangle over it makes pcbo_solve
 * return -1, as the back end does (src/gpu.cu:426). */
void pcbo_set_max_states(size_t n);

/* The congestion cost maps of every class (src/router.cpp:386-405 with own = 0; rebuild_costs 409-420):
 * st/oc/ov [k][l][n], vst [k][n], hist [l][n], gnd[l] (NULL entries or NULL: no ground factor);
 * outputs cst [k][l][n], vcst [k][n]. */
void pcbo_costs_rebuild(int n, int nl, int nclasses, const uint16_t* st, const uint8_t* oc, const uint8_t* ov,
                        const uint16_t* vst, const float* hist, const float* const* gnd, float pres, int hard,
                        float* cst, float* vcst);

/* A resolved dense search for the multi-search CPU baseline. */
typedef struct pcbo_search {
    int rw, rh, nl;
    float fac[8][8];
    const float* cf;
    const uint8_t* flags;
    const float* vcf;
    int64_t n_starts;
    const uint32_t* start_idx;
    const uint64_t* start_d;
    int64_t best;
    uint64_t best_d;
    int64_t settled;            /* states at or below best_d (every reached state when no target is reached) */
} pcbo_search;
/* Solve n searches on `threads` host threads (one search per thread at a time, taken in array order). */
void pcbo_solve_many(pcbo_search* s, int n, int threads);

#ifdef __cplusplus
}
#endif

#endif
