/* pcbg -- C ABI of the B200 search back end for pcbroute.
 *
 * Plain pointers and sizes only. Two layers:
 *   1. pcbg_solve(): one search exactly as pcbroute's gpu_solve() takes it (src/gpu.h:10-57), with the
 *      GpuQuery vectors flattened into (index, value, count) arrays. gpu_api.cpp implements gpu.h on top of it,
 *      so a ctypes / cgo / JNI binding sees the same contract as the router does.
 *   2. pcbg_solve_batch(): many searches whose costs are already resolved in device memory, solved in one
 *      persistent launch (no counterpart in the reference, which launches ~27 kernels per sweep per search;
 *      it replaces the per-search sweep loop of src/gpu.cu:493-524 for a whole round of searches).
 *
 * Arithmetic contract (shared bit for bit with the CPU oracle):
 *   - a move into state q in direction m costs W = rint(16 * fl(cf(q) * fac[l][m])) fixed-point units, where
 *     fac[l][m] = fl(len[m] * dirf[l][m]), len = step (m < 4) or fl(step * sqrt 2) (m >= 4), and fl() is one IEEE
 *     single-precision multiply; cf >= 1e30 (or a product whose 16x is >= 2^63) is impassable;
 *   - a via into layer l at cell c costs rint(16 * vcf(c)), vcf = fl(resolved via factor * via_cost);
 *   - a start costs ceil(16 * g0) (0 if g0 <= 0);
 *   - distances are exact integer least fixed points; the reported field is d / 16 for every state with
 *     d <= d(best) (all reached states when no target is reached) and 1e30 elsewhere; best is the target
 *     state minimising (d, state index).
 */
#ifndef PCBG_H
#define PCBG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PCBG_SCALE 16          /* fixed-point units per length unit of GpuQuery::step */
#define PCBG_INF_F 1e30f       /* "not reached" / "blocked" as the router reads it */

/* return codes (besides the >= 1 round count of a converged solve) */
#define PCBG_ERR_FAIL (-1)     /* solve failed: the caller carries on without the GPU (src/gpu.h:55-57) */
#define PCBG_ERR_BUSY (-3)     /* every slot busy and wait == 0 */

/* A search request. Mirrors GpuQuery (src/gpu.h:10-36); the three std::vector members become index/value/count
 * triples. All pointers are host pointers borrowed for the duration of the call. */
typedef struct pcbg_query {
    int32_t nx, ny, nl;
    int32_t wi0, wj0, ww, wh;
    uint16_t me;
    float via_cost, step;
    float dirf[8][8];
    uint8_t lay[8];
    const float* cst[8];
    const uint16_t* st[8];
    const float* vcst;
    const uint16_t* vst;
    const uint64_t* tbit;
    const uint32_t* own_cf_idx;
    const float* own_cf_val;
    int64_t n_own_cf;
    const uint32_t* own_vcf_idx;
    const float* own_vcf_val;
    int64_t n_own_vcf;
    const uint32_t* start_idx;
    const float* start_val;
    int64_t n_starts;
    const uint8_t* prior;
    int32_t pi0, pj0, pw, ph, pnl;
    const int32_t* pcol;
    const int32_t* prow;
    int32_t play[8];
    float mlf[256];
    uint8_t mthr;
    uint8_t corridor;
} pcbg_query;

/* The solution of one search. Mirrors GpuOut (src/gpu.h:39-50) plus diagnostics. `d` is a pinned host buffer
 * owned by the library (nl * rh * rw floats, [l][j][i]); give it back with pcbg_host_release(d, cap). */
typedef struct pcbg_result {
    int32_t rx0, ry0, rw, rh, nl, ww, wh;
    int64_t best;
    float* d;
    size_t cap;
    int32_t rounds;        /* persistent-kernel relaxation rounds of the last rectangle */
    int32_t tries;         /* rectangles solved (the window grows while a cheaper path may lie outside) */
    int32_t wide;          /* 1 if 64-bit distances were needed */
    int64_t tile_visits;   /* tiles relaxed in the last rectangle */
    double ub;             /* cost of the best target (1e30 if none) */
} pcbg_result;

/* src/gpu.h:52 (gpu_available): 1 if a device is present and the kernels load. */
int pcbg_available(void);
/* src/gpu.h:53-54 (gpu_configure): concurrent solve slots (before first use) and the state cap per solve. */
void pcbg_configure(int slots, size_t max_states);
/* src/gpu.h:55-57 (gpu_solve): >= 1 rounds on success, PCBG_ERR_FAIL, or PCBG_ERR_BUSY. Thread-safe. */
int pcbg_solve(const pcbg_query* q, pcbg_result* out, int wait);
/* src/gpu.cu:393-407 (GpuOut::reserve / ~GpuOut): pinned output buffers from a pool. */
float* pcbg_host_acquire(size_t n, size_t* cap);
void pcbg_host_release(float* p, size_t cap);
/* Text of the last failure on this thread ("" if none). */
const char* pcbg_last_error(void);

/* ---- batched device API --------------------------------------------------------------------------------- */

/* One search whose costs are resolved on the device. Device arrays are pitched: state (l, j, i) sits at
 * (l * hpad + j) * pitch + i, with pitch and hpad multiples of 32 and padding cells impassable (cf >= 1e30,
 * flags 0, vcf >= 1e30). */
typedef struct pcbg_search {
    int32_t rw, rh, nl;
    int32_t pitch, hpad;
    float fac[8][8];            /* fl(len[m] * dirf[l][m]) */
    const float* cf;            /* device [nl][hpad][pitch] resolved step cost factor */
    const uint8_t* flags;       /* device [nl][hpad][pitch] bit0 via may land, bit1 target */
    const float* vcf;           /* device [hpad][pitch] resolved via cost, or NULL for no vias */
    const uint32_t* start_idx;  /* device rect states (l * rh + j) * rw + i */
    const uint64_t* start_d;    /* device fixed-point start costs */
    int32_t n_starts;
    float* out;                 /* device [nl][rh][rw] reported field, or NULL */
    uint32_t* path;             /* device, or NULL: the walk-back from best to a start (rect states, best first) */
    int32_t path_cap;           /* capacity of path, in states */
    int32_t* path_len;          /* device: states written; 0 if no target was reached, -1 if no walk fits path_cap */
    /* results */
    int64_t best;               /* rect state of the cheapest target, -1 if none */
    uint64_t best_d;            /* its fixed-point cost */
    int32_t status;             /* 0 ok, 1 needed 64-bit distances (solved again wide), < 0 error */
    int32_t rounds;
} pcbg_search;

/* Solve n searches in one persistent launch on `stream` (a cudaStream_t, NULL for the legacy stream). Scratch
 * (distances, tile worklists) comes from the library's device arena. Returns 0 or PCBG_ERR_FAIL. Blocks until
 * the results are in the structs. */
int pcbg_solve_batch(pcbg_search* s, int32_t n, void* stream);

/* Largest search (padded states, nl * hpad * pitch) pcbg_solve_noalloc accepts. */
#define PCBG_NOALLOC_MAX_STATES 2097152

/* Solve one resolved device search without allocating any memory. No counterpart in the reference.
 *
 * Some callers cannot call cudaMalloc / cudaFree:
 *   - a host process whose device memory is owned by another allocator, for example a framework's caching pool or
 *     a fixed per-process budget, so that any memory outside it is refused;
 *   - a host thread that must not stall its peers: cudaFree waits for all work on the device, so the batch path's
 *     growing arena can pause every other router thread's searches at an unpredictable moment.
 * This entry point takes the same pcbg_search as pcbg_solve_batch: inputs, starts and the optional output field
 * are still the caller's. All scratch (distances, tile stamps and worklists, descriptors) lives in one static
 * device array, sized for PCBG_NOALLOC_MAX_STATES padded states. That is about 16.1 MiB, and every GPU that
 * loads the library holds it until the process exits. Larger searches return PCBG_ERR_FAIL with the reason in
 * pcbg_last_error(). The call itself makes no cudaMalloc, cudaFree or allocating library call.
 *
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress). Make that first call
 * before any stream capture. Every call shares the one array and clears what it needs at the start. Calls
 * whose GPU work overlaps would race on the array, so this function serialises calls within the process and
 * returns only when its work on `stream` is done. Returns 0 (results in *s, as pcbg_solve_batch) or
 * PCBG_ERR_FAIL. */
int pcbg_solve_noalloc(pcbg_search* s, void* stream);

/* Counters of the last batch solved on this thread (for throughput and roofline accounting): tile visits, the sum
 * over visits of the search's layer count (each layer of a visit stages 32 x 32 states), relaxation rounds, the
 * device time of the relaxation launches in ms (CUDA events on the launch stream), and kernels launched. */
int64_t pcbg_last_batch_tile_visits(void);
int64_t pcbg_last_batch_layer_visits(void);
int32_t pcbg_last_batch_rounds(void);
float pcbg_last_batch_kernel_ms(void);
int32_t pcbg_last_batch_launches(void);
int64_t pcbg_last_batch_local_iters(void);   /* sum over tile visits of local relaxation iterations */
/* Ordered rounds of the last batch: tiles listed for a round and passed on to a later one, and tiles dropped because
 * every improvement that listed them lies above the search's best target. */
int64_t pcbg_last_batch_deferred(void);
int64_t pcbg_last_batch_dropped(void);
/* States the last batch reported: at or below each search's best target's cost (every reached state of a search
 * that reached no target). */
int64_t pcbg_last_batch_settled(void);
/* Share of the relaxation launches' block time spent visiting tiles (SM cycles, summed over blocks); the rest is the
 * round filters and the waits at grid barriers for a round's last visits. */
float pcbg_last_batch_busy_frac(void);
/* Order in which an ordered round's visits are taken: 0 as listed, 1 the lower half of each search's band first,
 * 2 the tiles of the searches with the most layers first (a value outside 0-2 selects it). Results are the same for
 * every order. Default 2, or PCBG_VISIT_ORDER from the environment. */
void pcbg_set_visit_order(int32_t order);
int32_t pcbg_visit_order(void);

/* Scheduling of the relaxation rounds (no reference counterpart; the reference sweeps whole windows, src/gpu.cu:
 * 493-524). A queued tile carries the least distance among the edge improvements that queued it; with band B > 0 a
 * round of a search visits only the tiles keyed within B weight scales of the least key queued for it (the weight
 * scale: the mean straight-move weight of the search's cheapest well-filled tile), defers the rest to a later round
 * and drops tiles keyed above the best target found. B = 0 visits every queued tile each round. Results are the
 * same for every B; only the work changes. Default (a value < 0): the autotuned band of the batch's class, or before
 * any tuning 0 for batches of fewer than 16 tiles per resident block and 32 for larger ones. */
void pcbg_set_round_band(int32_t band);
int32_t pcbg_round_band(void);     /* the band of the last batch solved on this thread */
/* The schedule autotuner: for each layer-count class (1-2, 3-4, 5-6, 7-8 layers) and batch class (0: fewer than 16
 * tiles per resident block, as a router's concurrent searches; 1: more, as a round of the batched microbenchmark)
 * it solves seeded searches on `stream` under every round band (0, 8, 16, 32, 64, 128) and kernel build (2 or 3 blocks
 * per SM), and keeps the fastest for every later launch of that class (pcbg_set_round_band still overrides the band).
 * Writes one entry per class (up to cap) and returns how many, or PCBG_ERR_FAIL. Takes a few seconds. */
typedef struct pcbg_tune_entry {
    int32_t layers_lo, layers_hi, batch_class;
    int32_t band, blocks_per_sm;      /* the schedule chosen */
    float ms, ms_untuned;             /* its relaxation time, and the untuned rule's (band 16, 2 / 3 blocks) */
    int32_t searches, rw, rh, nl;     /* the timed batch */
} pcbg_tune_entry;
int32_t pcbg_autotune(void* stream, pcbg_tune_entry* out, int32_t cap);
/* The same on the caller's own batch (as pcbg_solve_batch takes it; it is solved 24 times): the fastest schedule
 * becomes the one of the batch's class, for callers whose batches repeat in shape. Returns 1 (entry in *out, rw / rh
 * 0 for a mixed batch) or PCBG_ERR_FAIL. */
int32_t pcbg_autotune_batch(pcbg_search* s, int32_t n, void* stream, pcbg_tune_entry* out);
/* Resident blocks per SM of the last batch's relaxation launch on this thread. */
int32_t pcbg_last_batch_blocks_per_sm(void);

/* Cap on the relaxation rounds of one launch (default 2^20; a value < 1 restores it). A launch that reaches the cap
 * stops and its solve returns PCBG_ERR_FAIL: a bounded device loop, which tests lower to see the error path. */
void pcbg_set_max_rounds(int32_t rounds);

/* ---- device mirror of the router's cost grids (extends src/gpu.h; replaces the per-solve uploads of
 * src/gpu.cu:432-439) -----------------------------------------------------------------------------------------------
 * A router that reports its cost-grid changes keeps a copy of each net class's grids in HBM; gpu_solve / pcbg_solve
 * then copy a search's rectangle device to device instead of from host memory. The grids are the router's own host
 * arrays (RClass, src/router.cpp:197-211), layer-major [l][j * nx + i]; the back end page-locks them in place and
 * remembers the pointers, which must stay valid while the class is mirrored.
 *   pcbg_mirror_class   after rebuild_costs (src/router.cpp:409-420): every grid of class cls is copied up (the
 *                       owner grids st / vst on the first call only: they do not change after set-up). oc / ov /
 *                       hist may be NULL (only the learned scheduler's features read them).
 *   pcbg_mirror_spans   after refresh_costs(id, spans) (src/router.cpp:1880-1890): the cells of the spans (j, i0, i1
 *                       triples) of cost grid kind 0 (cst[layer]) or 1 (vcst), and of the occupancy grid the stamp
 *                       changed (oc[layer] / ov[layer]), are copied up. A class that is not mirrored is ignored.
 *   pcbg_mirror_history after count_conflicts marked history (src/router.cpp:1970-1999).
 * Each call returns once the device copy is current. Returns 0 or PCBG_ERR_FAIL. */
int pcbg_mirror_class(int32_t cls, int32_t nx, int32_t ny, int32_t nl, const float* const* cst, const float* vcst,
                      const uint16_t* const* st, const uint16_t* vst, const uint8_t* const* oc,
                      const uint8_t* const* ov, const float* const* hist);
int pcbg_mirror_spans(int32_t cls, int32_t kind, int32_t layer, const int32_t* spans, int32_t nspans);
int pcbg_mirror_history(int32_t cls);
/* The mirrored cost grids of a class, for checks: cst [nl][ny * nx], vcst, oc, ov [nl][ny * nx] (any may be NULL). */
int pcbg_mirror_download(int32_t cls, float* cst, float* vcst, uint8_t* oc, uint8_t* ov);

/* ---- the round batcher (no reference counterpart) -----------------------------------------------------------
 * pcbg_solve / gpu_solve calls that run concurrently, from the router's worker threads (src/router.cpp:2187-2235
 * runs T of them ahead of the commit point), are solved together: each prepares its inputs on its own slot
 * stream, then the searches queued at that moment run in one persistent relaxation launch. The leader waits for
 * searches still preparing at most a window that tunes itself between 50 and 2000 microseconds: waits that bring no
 * search in shrink it, waits that do widen it. pcbg_batch_window(us) fixes it at `us` (0: never wait); a negative
 * value returns to the tuned window. Results never depend on the grouping. pcbg_batcher_stats reports the launches
 * made and the searches they solved since the library loaded. */
void pcbg_batch_window(int32_t us);
void pcbg_batcher_stats(int64_t* batches, int64_t* searches);

/* ---- device-resident congestion cost maps (src/router.cpp:197-211, 383-420, 1880-1999) ---------------------- */

/* The cost maps the searches read, kept in HBM and updated in place: per class k, the static owner grids st[l] / vst
 * (0 free, 0xFFFF blocked, else the owning net + 1), the other nets' occupancy oc[l] / ov[l] (u8 counts), the
 * history hist[l] (shared by the classes) and an optional ground-pour factor per layer; outputs cst[l] / vcst
 * (RClass::cst / vcst). All host arrays are layer-major [l][j * nx + i]. */
typedef struct pcbg_costs pcbg_costs;
pcbg_costs* pcbg_costs_create(int32_t nx, int32_t ny, int32_t nl, int32_t nclasses);
void pcbg_costs_destroy(pcbg_costs* h);
int pcbg_costs_set_static(pcbg_costs* h, int32_t cls, const uint16_t* st, const uint16_t* vst);
int pcbg_costs_set_occupancy(pcbg_costs* h, int32_t cls, const uint8_t* oc, const uint8_t* ov);
int pcbg_costs_set_history(pcbg_costs* h, const float* hist);
int pcbg_costs_set_ground(pcbg_costs* h, int32_t layer, const float* fac);   /* NULL: none on that layer */
/* rebuild_costs(pres, hard) (src/router.cpp:409-420): every cost of every class. */
int pcbg_costs_rebuild(pcbg_costs* h, float pres, int32_t hard);
/* A commit's stamp of one grid (class cls, kind 0 track / 1 via, layer): occupancy +1 (sign > 0, saturating at 255)
 * or -1 over the spans (j, i0, i1 triples, non-overlapping as the router merges them), then the costs of those cells
 * recomputed with the last rebuild's pres / hard (stamp + refresh_costs, src/router.cpp:1880-1963). */
int pcbg_costs_stamp(pcbg_costs* h, int32_t cls, int32_t kind, int32_t layer, const int32_t* spans, int32_t nspans,
                     int32_t sign);
/* count_conflicts(mark_hist) (src/router.cpp:1970-1999): hist += inc at the listed states l * nx * ny + cell, in
 * list order. */
int pcbg_costs_add_history(pcbg_costs* h, const uint32_t* states, int32_t m, float inc);
int pcbg_costs_download(pcbg_costs* h, int32_t cls, float* cst, float* vcst);
int pcbg_costs_download_history(pcbg_costs* h, float* hist);
/* Device pointer of a class's map (layer -1: the via map), for searches that read costs in place. */
const float* pcbg_costs_device_map(pcbg_costs* h, int32_t cls, int32_t layer);
/* Mean device time (ms, CUDA events) of `reps` full rebuilds. */
float pcbg_costs_time_rebuild(pcbg_costs* h, float pres, int32_t hard, int32_t reps);

/* ---- speculative negotiation rounds on the device (src/router.cpp:2096-2242, route_waves) ----------------------
 * A fixed order of nets is routed against a cost board (pcbg_costs, one class). The nets a policy picks from the
 * lookahead window of the commit point are searched together in one persistent launch, walked back on the device,
 * and committed in order: a net is accepted if no commit since its search started crossed a block (8 x 8 cells)
 * of its window, else it is searched again (a wasted search). Every policy gives the paths of the sequential one. */
typedef struct pcbg_net {
    int32_t x0, y0, x1, y1;     /* search window [x0, x1) x [y0, y1) on the board */
    uint32_t src, tgt;          /* board states l * nx * ny + y * nx + x, inside the window */
} pcbg_net;

typedef struct pcbg_spec_stats {
    int64_t searches;           /* searches run, speculative ones included */
    int64_t wasted;             /* searches thrown away at commit */
    int64_t batches;            /* persistent launches */
    int64_t commits;
    int64_t conflicts;          /* nets whose path shares a state with another net's path */
    double search_ms;           /* host time in the batched searches (resolve, launch, walk-back, paths read) */
    double total_ms;
    double relax_ms;            /* device time of the relaxation launches (CUDA events) */
} pcbg_spec_stats;

typedef struct pcbg_spec pcbg_spec;

#define PCBG_SPEC_SEQUENTIAL 0  /* one net per launch: the order's own result */
#define PCBG_SPEC_PLAIN 1       /* every open net of the lookahead window (route_waves' workers) */
#define PCBG_SPEC_LEARNED 2     /* the nets the attached scheduler picks; PLAIN when none is attached */

/* Learned batch composition: given the commit point and the open candidates of the window (ascending), set
 * pick[k] != 0 for the candidates to search now (the net at the commit point is always searched). Returns 0. */
typedef int (*pcbg_spec_scheduler)(void* user, pcbg_spec* s, int32_t cursor, const int32_t* cand, int32_t n,
                                   int32_t* pick);
/* Called before each search with the commit point: the nets [cursor, net) are not committed yet. */
typedef void (*pcbg_spec_observer)(void* user, pcbg_spec* s, int32_t cursor, int32_t net);

pcbg_spec* pcbg_spec_create(pcbg_costs* costs, int32_t cls, const pcbg_net* nets, int32_t n, float via_cost);
void pcbg_spec_destroy(pcbg_spec* s);
void pcbg_spec_set_scheduler(pcbg_spec* s, pcbg_spec_scheduler f, void* user);
void pcbg_spec_set_observer(pcbg_spec* s, pcbg_spec_observer f, void* user);
/* One rip-up-and-reroute iteration at present-congestion factor pres: lift every path, rebuild the costs, route
 * all nets in order with the policy (width: the lookahead, adapted as route_waves does). */
int pcbg_spec_iterate(pcbg_spec* s, float pres, int32_t policy, int32_t width, pcbg_spec_stats* st);
/* A net's committed path (board states, target first); returns its length. */
int32_t pcbg_spec_path(pcbg_spec* s, int32_t net, uint32_t* states, int32_t cap);
/* History += inc on every state two or more paths share (count_conflicts); returns how many. */
int32_t pcbg_spec_add_history(pcbg_spec* s, float inc);
/* 1 if a path through these board states would invalidate a search of net's window, else 0. */
int32_t pcbg_spec_window_reads(pcbg_spec* s, int32_t net, const uint32_t* states, int32_t m);

/* The engine's nets, board size and cost board (for schedulers). */
int pcbg_spec_net(pcbg_spec* s, int32_t k, pcbg_net* out);
void pcbg_spec_board(pcbg_spec* s, int32_t* nx, int32_t* ny, int32_t* nl);
int pcbg_spec_costs(pcbg_spec* s, pcbg_costs** costs, int32_t* cls);

/* ---- the learned speculation scheduler (no reference counterpart) --------------------------------------------
 * A conflict predictor: a 3-layer MLP (PCBG_SCHED_FEATURES -> 128 -> 128 -> 1, BF16 operands, FP32 accumulation)
 * over per-pair features of (searched net i, earlier uncommitted net j): 32 x 32 occupancy and history rasters of
 * j's window, an 8 x 8 mask of i's window in it, and 64 box-overlap / pin scalars. Attached to a pcbg_spec it
 * searches net i with the others of the window only while 1 - prod_j (1 - p_ij) < threshold; the plain batching is
 * its fallback. Attached as a logger to plain rounds it records the features of every speculative pair; after the
 * round pcbg_sched_label sets each pair's label (did j's committed path cross a block of i's window) and
 * pcbg_sched_train fits the network on the GPU with its own forward / backward kernels and Adam. */
#define PCBG_SCHED_FEATURES 2176
#define PCBG_SCHED_HIDDEN 128
typedef struct pcbg_sched pcbg_sched;
pcbg_sched* pcbg_sched_create(uint64_t seed);
void pcbg_sched_destroy(pcbg_sched* s);
void pcbg_sched_attach(pcbg_sched* s, pcbg_spec* spec, float threshold);
void pcbg_sched_attach_logger(pcbg_sched* s, pcbg_spec* spec);
/* Labels of the pairs logged since the last call, from spec's committed paths; returns the positives. */
int64_t pcbg_sched_label(pcbg_sched* s, pcbg_spec* spec);
int64_t pcbg_sched_log_size(pcbg_sched* s, int64_t* positives);
int pcbg_sched_train(pcbg_sched* s, int32_t epochs, float lr, int32_t batch, uint64_t seed, float* loss);
void pcbg_sched_counts(pcbg_sched* s, int64_t* scored, int64_t* deferred);
/* The network on host arrays. Parameters are packed f32: W1 [128][2176], W2 [128][128], b1, b2, w3 [128], b3.
 * x: B rows of 2176 bf16 bit patterns, B a multiple of 64. */
int64_t pcbg_sched_nparams(pcbg_sched* s);
int pcbg_sched_get_params(pcbg_sched* s, float* out);
int pcbg_sched_set_params(pcbg_sched* s, const float* in);
int pcbg_sched_forward_host(pcbg_sched* s, const uint16_t* x, int32_t B, float* p);
/* Gradients of sum_b w_b BCE(z_b, y_b) / sum_b w_b, packed like the parameters, and that loss. */
int pcbg_sched_grad_host(pcbg_sched* s, const uint16_t* x, const float* y, const float* w, int32_t B, float* grad,
                         float* loss);

/* Append labelled pairs (x: n rows of PCBG_SCHED_FEATURES bf16 bit patterns, y: n labels 0 / 1) to the
 * scheduler's conflict log, e.g. the logs a router wrote in log mode (below), before pcbg_sched_train. */
int pcbg_sched_add_log_host(pcbg_sched* s, const uint16_t* x, const float* y, int64_t n);

/* ---- the learned scheduler inside pcbroute's own router (route_waves, src/router.cpp:2119-2242) -------------
 * A router built with the hooks of baseline/router_hooks.h calls these from route_waves (no reference
 * counterpart: the reference takes the next net whenever a worker is free, src/router.cpp:2172-2178). Positions are
 * places in the call's commit order. The mode comes from the environment: PCBG_SCHED=log with PCBG_SCHED_LOG=<file>
 * appends the labelled (searched net, uncommitted earlier net) pairs of every speculative search to the file
 * (records: int64 rows, rows x PCBG_SCHED_FEATURES bf16, rows u8 labels); PCBG_SCHED=learned with
 * PCBG_SCHED_MODEL=<file> (pcbg_sched_get_params' floats) defers a speculative search while its predicted risk is at
 * or above PCBG_SCHED_THRESHOLD (default 0.5). Anything else: off, the router's own choice. Features are read from
 * the mirrored grids of class 0 (pcbg_mirror_class). */
typedef struct pcbg_rnet {
    int32_t x0, y0, x1, y1;     /* the net's search window on the board, in cells: [x0, x1) x [y0, y1) */
    float sx, sy, tx, ty;       /* two pin positions, in cells */
} pcbg_rnet;
typedef struct pcbg_rsched_stats {
    int64_t calls, searches, speculative, commits, wasted, scored, deferred, logged, positives;
} pcbg_rsched_stats;
int32_t pcbg_rsched_mode(void);                       /* 0 off, 1 log, 2 learned */
void pcbg_rsched_begin(int32_t n);                    /* a route_waves call over n nets */
void pcbg_rsched_net(int32_t pos, const pcbg_rnet* net);
/* 1 if a worker may search position pos now (the commit point is `cursor`, `version` commits were made). */
int32_t pcbg_rsched_allow(int32_t pos, int32_t cursor, int64_t version);
void pcbg_rsched_started(int32_t pos, int32_t cursor, int64_t version);
void pcbg_rsched_committed(int32_t pos, int64_t commit_index);
/* The verdict on position pos's search: accepted, and which commits made since it started changed a block it read. */
void pcbg_rsched_verdict(int32_t pos, int32_t accepted, const int64_t* hit_commits, int32_t nhit);
void pcbg_rsched_end(void);
void pcbg_rsched_get_stats(pcbg_rsched_stats* out);

/* ---- seeded synthetic search generator (the batched-search microbenchmark workload) ----------------------- */

/* Fill a pitched search with the seeded workload: per (layer, cell) cost 1 + (h % 16), about 15 % of cells
 * blocked in value-noise blobs (drawn per layer), via cost `via` per cell, flags, one source and one
 * target picked among free cells. cf/flags/vcf are the pcbg_search device arrays; src/tgt receive the rect
 * states chosen (device int64 each). Deterministic in (seed). */
int pcbg_synth_search(uint64_t seed, int32_t rw, int32_t rh, int32_t nl, int32_t pitch, int32_t hpad, float via,
                      float* cf, uint8_t* flags, float* vcf, int64_t* src_tgt, void* stream);
/* The same search into dense host arrays (cf/flags [nl][rh][rw], vcf [rh][rw]) on `threads` host threads. */
int pcbg_synth_search_host(uint64_t seed, int32_t rw, int32_t rh, int32_t nl, float via, float* cf, uint8_t* flags,
                           float* vcf, int64_t* src_tgt, int32_t threads);

#ifdef __cplusplus
}
#endif

#endif /* PCBG_H */
