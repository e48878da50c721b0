// Internal declarations shared by the pcbg engine sources (not part of the C ABI).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <vector>

#include "pcbg.h"

namespace pcbg {

// Tile geometry of the relaxation kernel: 32 x 32 cells, every layer of the search (up to 8).
constexpr int TILE = 32;
constexpr int MAX_LAYERS = 8;

// Fixed-point limits. INF is a byte pattern so that cudaMemset(0x7F) fills "unreached"; a finite weight is below
// WLIM so that d + w never wraps (d <= INF, w < 2^31 resp. 2^63) and min(v, d + w) <= v <= INF.
constexpr uint32_t INF32 = 0x7F7F7F7Fu;
constexpr uint64_t INF64 = 0x7F7F7F7F7F7F7F7Full;
constexpr float WLIM32 = 2130706432.0f;               // 2^31 - 2^24
constexpr float WLIM64 = 4611686018427387904.0f;      // 2^62

// Per-search device descriptor of the relaxation kernel.
//   mode 1 (joint): the moves of a layer fall into weight classes x (moves 0, 1), y (2, 3), diagonal (4-7) with
//     one factor each; a visit stages one integer weight plane per class (K = 2 when x and y share a factor on
//     every layer, else 3: plane_h / plane_v / plane_d) and relaxes all layers of a line jointly.
//   mode 0 (general): any per-move factors and 64-bit distances; per-layer scans with weights computed per move.
struct SDev {
    int rw, rh, nl, pitch, hpad, ntx, nty, mode;
    int K, plane_h, plane_v, plane_d;
    float fac[MAX_LAYERS][8];
    float maxfac[MAX_LAYERS];
    const float* cf;
    const uint8_t* fl;
    const float* vcf;
    void* dist;
    uint32_t* stamp;
    uint32_t* sides;   // per tile: which halo sides changed since its last visit (bit 8: everything)
    uint32_t* tkey;    // per tile: least improved edge distance that queued it since its last visit (all ones: none)
    float* out;
    uint32_t* path;    // walk-back output (or null), capacity path_cap; its length goes to *path_len
    int* path_len;
    int path_cap;
};

// Per-search statistics written by the kernels.
struct SStat {
    unsigned long long ub;        // least target distance seen (all ones: none)
    unsigned long long maxw;      // largest finite weight met in visited tiles
    unsigned long long best;      // rect state of the cheapest target (all ones: none)
    unsigned long long maxd;      // largest finite distance in the field
    unsigned int need_wide;       // a finite weight does not fit 32-bit arithmetic
    unsigned int wscale;          // least mean straight-move weight over the well-filled tiles visited (all ones: none)
    unsigned int kmin[3];         // per rotating round: least key of the tiles queued for it (all ones: none)
    unsigned int settled;         // states reported: at or below the best target's cost (all reached when none)
};

// Search handed to the batch solver (host side).
struct BatchItem {
    int rw, rh, nl, pitch, hpad;
    float fac[MAX_LAYERS][8];
    const float* cf;
    const uint8_t* fl;
    const float* vcf;
    const uint32_t* start_idx;   // device, rect states
    const uint64_t* start_d;     // device
    int n_starts;
    float* out;
    uint32_t* path;              // device, or null: walk-back from best to a start
    int path_cap;
    int* path_len;               // device
    // results
    int64_t best;
    uint64_t best_d;
    int status;
    int rounds;
};

// Solve a batch on `stream` (blocks until done). Returns 0 or -1 (error text in last_error()).
int solve_batch(BatchItem* items, int n, cudaStream_t stream);

void set_error(const std::string& s);
const std::string& last_error();

// Round / tile-visit counters of the last batch on this thread.
struct BatchStats {
    int rounds = 0;
    long long tile_visits = 0;     // tile visits (each stages and relaxes every layer of a 32 x 32 tile)
    long long layer_visits = 0;    // sum over visits of the search's layer count
    float kernel_ms = 0.f;         // device time of the relaxation launches (CUDA events on the launch stream)
    int launches = 0;              // kernels this library launched for the batch
    long long local_iters = 0;     // sum over tile visits of the local relaxation iterations
    long long deferred = 0;        // ordered rounds: tiles listed for a round and passed on to the next one
    long long dropped = 0;         // ordered rounds: tiles dropped because nothing that queued them can matter
    long long settled = 0;         // states at or below their search's best target's cost (all reached when none)
    long long busy_cycles = 0;     // relaxation launches: SM cycles the blocks spent visiting tiles, summed
    long long block_cycles = 0;    // and the SM cycles they were resident (visiting, filtering, at grid barriers)
    int band = 0;                  // round band of the (last) relaxation launch
    int blocks_per_sm = 0;         // resident blocks per SM of its build
};
BatchStats& last_stats();

// The round batcher (batcher.cpp): concurrent searches solved in one relaxation launch. A search calls
// batcher_enter() before it prepares its inputs, then either batcher_submit() (blocks until its batch is solved) or,
// on an error before submitting, batcher_leave().
struct BatchResult {
    int rc = 0;                 // solve_batch's return for the batch
    std::string error;          // its error text when rc != 0
    long long tile_visits = 0;  // of the whole batch
    int batch_size = 0;         // searches solved in the same launch
    float kernel_ms = 0.f;      // relaxation launch time of the batch
};
void batcher_enter();
void batcher_leave();
int batcher_submit(BatchItem& item, BatchResult& res);
void batcher_window(int us);
void batcher_stats(long long* batches, long long* searches);

// Device planes of one class of a cost board (costs.cu), for kernels outside it that read the board in place.
struct CostPlanes {
    int nx, ny, nl;
    const float* cst[MAX_LAYERS];
    const float* vcst;
    const uint8_t* oc[MAX_LAYERS];
    const uint8_t* ov[MAX_LAYERS];
    const float* hist[MAX_LAYERS];
};
bool cost_planes(pcbg_costs* h, int cls, CostPlanes& out);

// The router's cost grids mirrored in device memory (mirror.cu). mirror_lookup: the device planes of the mirrored
// class whose host grids the query points at (false: not mirrored). mirror_planes: a mirrored class as cost planes.
struct MirrorView {
    const float* cst[MAX_LAYERS];
    const uint16_t* st[MAX_LAYERS];
    const float* vcst;
    const uint16_t* vst;
};
bool mirror_lookup(const pcbg_query& q, MirrorView& v);
bool mirror_planes(int cls, CostPlanes& out);

// The conflict predictor's network (mlp.cu): D0 inputs (two 32 x 32 rasters, an 8 x 8 overlap mask, 64 scalars),
// two hidden layers of MLP_H, one logit. BF16 operands, FP32 accumulation, FP32 master weights under Adam.
constexpr int MLP_D0 = 2 * 1024 + 64 + 64, MLP_H = 128;
struct Mlp {
    // f32 parameters, packed: W1 [H][D0], W2 [H][H], b1 [H], b2 [H], w3 [H], b3
    size_t nparams = 0;
    float *master = nullptr, *grad = nullptr, *m1 = nullptr, *m2 = nullptr;
    __nv_bfloat16 *w1b = nullptr, *w2b = nullptr, *w2t = nullptr;
    // activations of the last forward (capacity cap rows)
    int cap = 0;
    __nv_bfloat16 *h1 = nullptr, *h1t = nullptr, *h2 = nullptr, *dz2 = nullptr, *dz2t = nullptr, *dz1 = nullptr,
                  *dz1t = nullptr, *xt = nullptr;
    float *z3 = nullptr, *lossd = nullptr;
    int step = 0;
    std::vector<void*> owned;
    ~Mlp();
    bool init(uint64_t seed);
    int set_params(const float* host);
    int refresh_bf16(cudaStream_t s);
    bool reserve(int B);
    // x [B][D0] bf16 on the device, B a multiple of 64; p (device, may be null): sigmoid of the logits
    int forward(cudaStream_t s, const __nv_bfloat16* x, int B, float* p);
    // after forward on the same x: gradients of sum_b w[b] * BCE(z3[b], y[b]) / wsum into grad; loss (host) if set
    int backward(cudaStream_t s, const __nv_bfloat16* x, const float* y, const float* w, float wsum, int B, float* loss);
    int adam(cudaStream_t s, float lr);
};

// Side of the square cell blocks by which speculative rounds track what a search read and a commit changed.
constexpr int SPEC_BLOCK = 8;

inline size_t round_up(size_t x, size_t m) { return (x + m - 1) / m * m; }

}  // namespace pcbg
