// Exact multi-layer grid shortest paths on sm_100a: the relaxation engine behind gpu_solve and pcbg_solve_batch.
//
// The reference (src/gpu.cu:122-363, 488-524) relaxes a search window with 8 directional min-plus sweeps plus a
// via pass, 27 launches and one host sync per sweep, until nothing changes. Here the same relaxation rule
// (a move into a state costs its factor times the move's length and direction factor; vias land only where a via
// may, src/gpu.cu:154-155, 332-350) is solved to its exact integer least fixed point by a tiled worklist:
//
//   * the window is cut into 32 x 32-cell tiles holding every layer; a tile visit stages the tile's distances
//     (with a one-cell halo from its neighbours), integer move weights, via weights and via/target masks in shared
//     memory and relaxes them to a local fixed point;
//   * the local relaxation scans lines (rows, columns, both diagonals) with all layers of a line in one thread,
//     mixing vias at every cell of the line, so a path that changes layers along a straight run settles in one
//     pass; the forward and backward walks of a line run on two threads at once, and only lines through cells that
//     went down are walked again; all walks of an iteration run concurrently, with shared-memory atomicMin updates
//     so that every stored value only decreases;
//   * a tile whose edge cell improved below the staged value of an adjacent cell of a neighbour (and not above the
//     best target found so far) queues that neighbour for the next round;
//   * one persistent cooperative launch runs all rounds of all searches of a batch, with a bounded software grid
//     barrier between rounds, so a whole round of searches with uneven windows and layer counts shares the GPU;
//   * rounds go in distance order per search (delta-stepping at tile granularity): a queued tile carries a key,
//     the least improved edge distance that queued it, and a round visits only the tiles whose key lies within a
//     band of the search's least key; the others wait for a later round, and tiles keyed above the search's best
//     target are dropped. Tiles visited concurrently in one round read each other's old edges, so an unordered
//     round revisits a tile each time a wave of improvements crosses it; the band keeps the visits near the front;
//   * within a round the visits of the searches with the most layers start first (they take longest, and a round
//     ends with its last visit), so the short visits fill the end of the round.
//
// Exactness: distances are fixed-point integers (pcbg.h); min-plus over integers is exact and associative, so the
// least fixed point is unique and any monotone schedule reaches it. A visit ends only after a full pass changed
// nothing, and a neighbour is skipped only when no edge value can lower its adjacent cells; improvements above the
// best target are not propagated (no path through them can matter), and a queued tile is dropped only when every
// improvement that queued it lies above the best target. Deferring a tile to a later round changes only the order. The epilogue reports every state at or below
// the best target's cost, and those are exact.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "pcbg_internal.h"

namespace pcbg {

namespace {

constexpr int NT = 384;                 // threads per tile block: 12 warps, one per line and direction
constexpr int HS = TILE + 2;            // tile side with halo
constexpr int DSTR = TILE + 3;          // shared row stride of distances (odd: conflict-free row, column, diagonal)
constexpr int CSTR = TILE + 1;          // shared row stride of per-state and per-cell arrays
constexpr int LS = HS * DSTR;           // distance plane stride (one layer)
constexpr int WLS = TILE * CSTR;        // weight plane stride (one layer)
constexpr int MAX_IT = 64;              // local iterations before a tile is re-queued instead
constexpr long long BAR_SPIN_LIMIT = 1ll << 24;   // polls (with __nanosleep) before a barrier wait gives up

constexpr uint32_t KEY_NONE = 0xFFFFFFFFu;   // tile key / round minimum: nothing queued

// control words of a batch: per rotating round the queued count and the next item taken; per round parity the
// counts of the round's visit list filled from its front and from its back, and the next item taken (ordered rounds)
// (C_WIDEN: the doublings of the band the next ordered round uses)
enum { C_CNT = 0, C_NEXT = 3, C_BAR = 6, C_GEN = 7, C_ERR = 8, C_ROUNDS = 9, C_VCNT = 10, C_VNEXT = 12, C_WIDEN = 14,
       C_BCNT = 16, C_N = 18 };
constexpr unsigned int MAX_WIDEN = 12;   // band x 4096: wider than any search's key range, i.e. unordered
enum { ERR_BARRIER = 1, ERR_ROUNDS = 2, ERR_OVERFLOW = 4 };
// counters of a launch: tile visits, layer visits, local iterations, tiles deferred to a later round, tiles dropped,
// SM cycles the blocks spent visiting tiles, SM cycles the blocks were resident (both summed over blocks)
constexpr int NVIS = 7;
// order of an ordered round's visit list: 0 as filtered, 1 the lower half of each search's band first, 2 the tiles
// of the searches with the most layers first
enum { ORDER_FIFO = 0, ORDER_KEY = 1, ORDER_LAYERS = 2 };

template <typename DT> struct Lim;
template <> struct Lim<uint32_t> {
    static constexpr uint32_t INF = INF32;
    __device__ static float wlim() { return WLIM32; }
    __device__ static uint32_t cvt(float y) { return __float2uint_rn(y); }
};
template <> struct Lim<uint64_t> {
    static constexpr uint64_t INF = INF64;
    __device__ static float wlim() { return WLIM64; }
    __device__ static uint64_t cvt(float y) { return __float2ull_rn(y); }
};

// Fixed-point weight of entering a state of cost factor cf by a move of factor fac (pcbg.h; oracle pcbo_weight).
template <typename DT> __device__ __forceinline__ DT qweight(float cf, float fac) {
    const float y = __fmul_rn(__fmul_rn(cf, fac), 16.0f);
    if (!(cf < 1e30f) || !(y < Lim<DT>::wlim())) return Lim<DT>::INF;
    if (!(y > 0.0f)) return DT(0);
    return Lim<DT>::cvt(y);
}

template <typename DT> __device__ __forceinline__ DT dmin(DT a, DT b) { return a < b ? a : b; }
__device__ __forceinline__ void atomic_min_d(uint32_t* p, uint32_t v) { atomicMin(reinterpret_cast<unsigned int*>(p), v); }
__device__ __forceinline__ void atomic_min_d(uint64_t* p, uint64_t v) {
    atomicMin(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
}

struct SolveArgs {
    const SDev* S;
    SStat* st;
    int n;
    int nlmax;
    int kmax;                     // weight planes of joint-mode searches (0: none in the batch)
    unsigned long long* wl;       // 3 rotating worklists of `cap` items: (search << 32) | tile
    unsigned long long* vl;       // ordered rounds: the items of the current round that are visited (cap items)
    unsigned int cap;
    unsigned int* ctl;
    unsigned long long* visits;   // NVIS counters
    int max_rounds;
    int ordered;                  // 1: rounds in distance bands (32-bit distances only), 0: every queued tile
    unsigned int band;            // band width of an ordered round, in multiples of the search's weight scale
    int order;                    // ORDER_*: which visits of an ordered round go to the front of its list
};

// Key of an improvement: its distance, as 32 bits (64-bit distances run unordered and only need "some key").
template <typename DT> __device__ __forceinline__ uint32_t key_of(DT v) {
    return static_cast<unsigned long long>(v) < KEY_NONE ? uint32_t(v) : KEY_NONE - 1;
}

// Shared memory of a visit. d: distances with halo [nl][HS][DSTR]; w: joint mode, K integer weight planes
// [K][nl][TILE][CSTR] (general mode: float cost factors [nl][TILE][CSTR]); v: via weight per cell; e: staged edge
// values [nl][4][TILE]; m: via-landing and target layer masks per cell (u32).
struct Lay {
    size_t d, w, v, e, m, total;
};
// wbytes: bytes per state of the w region (joint: K u16 planes, at least one float plane for the fallback)
__host__ __device__ inline int joint_wbytes(int K) { return 2 * K > 4 ? 2 * K : 4; }
__host__ __device__ inline Lay layout(int nlm, int wbytes, size_t dsz) {
    Lay L;
    size_t o = 0;
    L.d = o; o += size_t(nlm) * LS * dsz; o = (o + 15) & ~size_t(15);
    L.w = o; o += size_t(wbytes) * nlm * WLS; o = (o + 15) & ~size_t(15);
    L.v = o; o += size_t(WLS) * dsz; o = (o + 15) & ~size_t(15);
    L.e = o; o += size_t(nlm) * 4 * TILE * dsz; o = (o + 15) & ~size_t(15);
    L.m = o; o += size_t(2) * WLS * 4; o = (o + 15) & ~size_t(15);
    L.total = o;
    return L;
}
__host__ __device__ inline Lay layout_for(int nlm, int kmax, size_t dsz, int mode) {
    // one dynamic allocation serves both modes: the larger of the two layouts, same offsets per mode
    return mode ? layout(nlm, joint_wbytes(kmax), 4) : layout(nlm, 4, dsz);
}

// Software grid barrier with a bounded wait: every block of the cooperative launch is resident, so the wait ends
// unless something is badly wrong; then it records ERR_BARRIER and returns instead of spinning forever.
__device__ void grid_barrier(unsigned int* ctl, unsigned int nblocks) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* gen = ctl + C_GEN;
        const unsigned int g = *gen;
        __threadfence();
        const unsigned int arrived = atomicAdd(ctl + C_BAR, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(ctl + C_BAR, 0u);
            __threadfence();
            atomicAdd(ctl + C_GEN, 1u);
        } else {
            long long spins = 0;
            while (*gen == g) {
                if (++spins > BAR_SPIN_LIMIT) { atomicOr(ctl + C_ERR, unsigned(ERR_BARRIER)); break; }
                __nanosleep(128);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

__device__ __forceinline__ void enqueue(const SolveArgs& a, const SDev& S, int s, int tile, int next_round) {
    const unsigned int old = atomicMax(S.stamp + tile, unsigned(next_round));
    if (old >= unsigned(next_round)) return;  // already queued for that round
    const int buf = next_round % 3;
    const unsigned int pos = atomicAdd(a.ctl + C_CNT + buf, 1u);
    if (pos < a.cap) a.wl[size_t(buf) * a.cap + pos] = (static_cast<unsigned long long>(s) << 32) | unsigned(tile);
    else atomicOr(a.ctl + C_ERR, unsigned(ERR_OVERFLOW));
}

// Queue a tile for next_round with the key of what queued it: the tile's key and the round's least key for the
// search both take the minimum before the tile is listed (the key counts even when the tile is listed already).
__device__ __forceinline__ void queue_tile(const SolveArgs& a, const SDev& S, int s, int tile, int next_round,
                                           uint32_t key) {
    if (a.ordered) {
        atomicMin(S.tkey + tile, key);
        atomicMin(&a.st[s].kmin[next_round % 3], key);
    }
    enqueue(a, S, s, tile, next_round);
}

struct VisitShared {
    unsigned int marks, any, wide, iters, sides;
    unsigned int kvis;             // the tile's key when the visit took it (ordered rounds)
    unsigned int mkey[8];          // per neighbour marked: least improved edge value that marked it
    unsigned int wcnt;             // finite straight-move weights staged, and their sum (ordered rounds)
    unsigned long long tmin, wmax, wsum;
};

// Halo sides of a tile, as neighbour directions: 0 L, 1 R, 2 T, 3 B, 4 TL, 5 TR, 6 BL, 7 BR; SIDE_ALL: the interior
// itself changed (a start was written, or the last visit stopped early), every line must be walked.
constexpr unsigned SIDE_ALL = 1u << 8;
__device__ __forceinline__ unsigned opposite_side(int b) {
    const int opp[8] = {1, 0, 3, 2, 7, 6, 5, 4};
    return 1u << opp[b];
}

// The lines whose end cells lie on the given halo sides (their first iteration's dirty set), as 6 words (rows,
// columns, diagonals e + 31 in 2 words, anti-diagonals s in 2 words). A line reads the halo only at its two ends:
// rows at columns -1 / 32, columns at rows -1 / 32, diagonal e at (e, 0) - (1, 1) and its far end, anti-diagonal s
// at (s - lo + 1, lo - 1) and (lo - 1, s - lo + 1).
__device__ __forceinline__ void side_lines(unsigned sides, uint32_t (&w)[6]) {
    for (int k = 0; k < 6; ++k) w[k] = 0;
    if (sides & SIDE_ALL) {
        w[0] = w[1] = w[2] = w[4] = 0xFFFFFFFFu;
        w[3] = w[5] = 0x7FFFFFFFu;
        return;
    }
    const uint32_t LO = 0xFFFFFFFFu;                         // bits 0..31 of a 63-bit set
    const uint32_t HI0 = 0x80000000u, HI1 = 0x7FFFFFFFu;     // bits 31..62
    if (sides & 1u) { w[0] = LO; w[2] |= LO; w[4] |= LO; }                                // left
    if (sides & 2u) { w[0] = LO; w[2] |= HI0; w[3] |= HI1; w[4] |= HI0; w[5] |= HI1; }   // right
    if (sides & 4u) { w[1] = LO; w[2] |= HI0; w[3] |= HI1; w[4] |= LO; }                 // top
    if (sides & 8u) { w[1] = LO; w[2] |= LO; w[4] |= HI0; w[5] |= HI1; }                 // bottom
    if (sides & (16u | 128u)) w[2] |= HI0;                                               // corners TL, BR: diagonal 0
    if (sides & (32u | 64u)) w[4] |= HI0;                                                // corners TR, BL: anti-diagonal 31
}

// ---- staging shared by both modes ----

// Staging is latency-bound: a visit's loads come from L2 or HBM, and a block has few warps. Each thread therefore
// issues a whole chunk of independent loads before it stores any of them.
constexpr int STAGE_CHUNK = 4;

template <typename DT>
__device__ void stage_dist(const SDev& S, DT* dS, int x0, int y0) {
    const DT* dist = reinterpret_cast<const DT*>(S.dist);
    const int total = S.nl * HS * HS;
    for (int base = threadIdx.x; base < total; base += NT * STAGE_CHUNK) {
        DT v[STAGE_CHUNK];
        #pragma unroll
        for (int u = 0; u < STAGE_CHUNK; ++u) {
            const int idx = base + u * NT;
            const int l = idx / (HS * HS), rem = idx % (HS * HS), r = rem / HS, c = rem % HS;
            const int gy = y0 + r - 1, gx = x0 + c - 1;
            v[u] = Lim<DT>::INF;
            // distances are written by other blocks during the launch: read them at L2, never from this SM's L1
            if (idx < total && gy >= 0 && gy < S.hpad && gx >= 0 && gx < S.pitch)
                v[u] = __ldcg(dist + (size_t(l) * S.hpad + gy) * S.pitch + gx);
        }
        #pragma unroll
        for (int u = 0; u < STAGE_CHUNK; ++u) {
            const int idx = base + u * NT;
            if (idx >= total) break;
            const int l = idx / (HS * HS), rem = idx % (HS * HS), r = rem / HS, c = rem % HS;
            dS[l * LS + r * DSTR + c] = v[u];
        }
    }
}

// 32-bit distances: 16-byte loads. A staged row spans columns x0 - 1 .. x0 + 32; the aligned words x0 - 4 .. x0 + 35
// cover it in 10 loads, and words outside the field (left of column 0, right of the pitch, rows off the field)
// stay unreached.
template <>
__device__ void stage_dist<uint32_t>(const SDev& S, uint32_t* dS, int x0, int y0) {
    const uint32_t* dist = reinterpret_cast<const uint32_t*>(S.dist);
    constexpr int G = 10;   // 16-byte groups per staged row
    const int total = S.nl * HS * G;
    for (int base = threadIdx.x; base < total; base += NT * STAGE_CHUNK) {
        uint4 v[STAGE_CHUNK];
        #pragma unroll
        for (int u = 0; u < STAGE_CHUNK; ++u) {
            const int it = base + u * NT;
            const int l = it / (HS * G), rem = it % (HS * G), r = rem / G, g = rem % G;
            const int gy = y0 + r - 1, gx = x0 - 4 + 4 * g;
            v[u] = make_uint4(INF32, INF32, INF32, INF32);
            if (it < total && gy >= 0 && gy < S.hpad && gx >= 0 && gx + 4 <= S.pitch)
                v[u] = __ldcg(reinterpret_cast<const uint4*>(dist + (size_t(l) * S.hpad + gy) * S.pitch + gx));
        }
        #pragma unroll
        for (int u = 0; u < STAGE_CHUNK; ++u) {
            const int it = base + u * NT;
            if (it >= total) break;
            const int l = it / (HS * G), rem = it % (HS * G), r = rem / G, g = rem % G;
            const uint32_t w[4] = {v[u].x, v[u].y, v[u].z, v[u].w};
            #pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int c = 4 * g + e - 3;   // staged column: word x0 - 4 + 4g + e is column c - 1 of the tile
                if (c >= 0 && c < HS) dS[l * LS + r * DSTR + c] = w[e];
            }
        }
    }
}

// via weight per cell and the via-landing / target layer masks; 4 cells per thread-step (the flags of 4 cells are
// one 32-bit word per layer, the via costs one 128-bit word), all layers' words loaded before any is used
template <typename DT>
__device__ void stage_cells(const SDev& S, DT* vS, uint32_t* vokS, uint32_t* tgS, int x0, int y0, bool& wide,
                            unsigned long long& wmax) {
    for (int g = threadIdx.x; g < TILE * TILE / 4; g += NT) {
        const int r = g >> 3, c0 = (g & 7) * 4;
        uint32_t fw[MAX_LAYERS];
        #pragma unroll
        for (int l = 0; l < MAX_LAYERS; ++l)
            fw[l] = l < S.nl ? *reinterpret_cast<const uint32_t*>(S.fl + (size_t(l) * S.hpad + y0 + r) * S.pitch + x0 + c0) : 0u;
        float4 vv = make_float4(1e30f, 1e30f, 1e30f, 1e30f);
        if (S.vcf) vv = *reinterpret_cast<const float4*>(S.vcf + size_t(y0 + r) * S.pitch + x0 + c0);
        const float vc[4] = {vv.x, vv.y, vv.z, vv.w};
        #pragma unroll
        for (int e = 0; e < 4; ++e) {
            DT wv = Lim<DT>::INF;
            const float v = vc[e];
            if (v < 1e30f) {
                const float y = __fmul_rn(v, 16.0f);
                if (!(y < Lim<DT>::wlim())) wide = true;
                else { wv = qweight<DT>(v, 1.0f); wmax = max(wmax, static_cast<unsigned long long>(wv)); }
            }
            vS[r * CSTR + c0 + e] = wv;
            unsigned int vm = 0, tm = 0;
            #pragma unroll
            for (int l = 0; l < MAX_LAYERS; ++l) {
                const unsigned f = (fw[l] >> (8 * e)) & 0xFFu;
                vm |= (f & 1u) << l;
                tm |= ((f >> 1) & 1u) << l;
            }
            vokS[r * CSTR + c0 + e] = vm;
            tgS[r * CSTR + c0 + e] = tm;
        }
    }
}

// edge cell k of side (0 left, 1 right, 2 top, 3 bottom) in tile coordinates
__device__ __forceinline__ void edge_rc(int side, int k, int& r, int& c) {
    r = side <= 1 ? k : (side == 2 ? 0 : TILE - 1);
    c = side == 0 ? 0 : (side == 1 ? TILE - 1 : k);
}

template <typename DT>
__device__ void save_edges(const SDev& S, const DT* dS, DT* eS) {
    for (int idx = threadIdx.x; idx < S.nl * 4 * TILE; idx += NT) {
        const int l = idx / (4 * TILE), side = (idx / TILE) & 3, k = idx % TILE;
        int r, c;
        edge_rc(side, k, r, c);
        eS[idx] = dS[l * LS + (r + 1) * DSTR + c + 1];
    }
}

// ---- joint-layer line scans (mode 1) ----

// One cell of a line: every layer's move from the previous cell of the line, then vias among the layers.
template <int NL>
__device__ __forceinline__ void jstep(uint32_t* dS, const uint16_t* wP, const uint32_t* vS, const uint32_t* vokS,
                                      int dofs, int wofs, uint32_t (&prev)[NL], int& ch) {
    uint32_t v[NL], c[NL];
    uint32_t m = INF32;
    #pragma unroll
    for (int l = 0; l < NL; ++l) {
        v[l] = dS[l * LS + dofs];
        const uint32_t w16 = wP[l * WLS + wofs];
        c[l] = min(v[l], prev[l] + (w16 == 0xFFFFu ? INF32 : w16));   // 0xFFFF: impassable
        m = min(m, c[l]);
    }
    const uint32_t mv = m + vS[wofs];
    const uint32_t vm = vokS[wofs];
    uint32_t any = 0;
    #pragma unroll
    for (int l = 0; l < NL; ++l) {
        c[l] = ((vm >> l) & 1u) ? min(c[l], mv) : c[l];
        any |= uint32_t(c[l] < v[l]);
        atomicMin(dS + l * LS + dofs, c[l]);   // unconditional: a min that lowers nothing is harmless, and cheaper
                                               // than an atomic predicated on c < v
        prev[l] = c[l];
    }
    ch = int(any);
}

// A line of the tile walked forward then backward: cell k at distance offset d0 + k * ds and weight offset
// w0 + k * ws, k < len; pf / pb: the halo cells before the first / after the last cell. One call site per thread
// and no unrolling: the walk is inlined once per layer count, which keeps the kernel in the instruction cache.
// Returns the positions k at which any layer's cost went down.
template <int NL>
__device__ __forceinline__ uint32_t walk_line(uint32_t* dS, const uint16_t* wP, const uint32_t* vS, const uint32_t* vokS,
                                              int d0, int ds, int w0, int ws, int len, int pf, int pb, int dir) {
    // one direction per walker: a shortest path never turns back along a line, so the forward and the backward
    // walks of a line are independent and run on two threads at once
    uint32_t moved = 0;
    int ch;
    uint32_t prev[NL];
    const int start = dir ? pb : pf;
    #pragma unroll
    for (int l = 0; l < NL; ++l) prev[l] = dS[l * LS + start];
    const int k0 = dir ? len - 1 : 0, step = dir ? -1 : 1;
    for (int t = 0, k = k0; t < len; ++t, k += step) {
        jstep<NL>(dS, wP, vS, vokS, d0 + k * ds, w0 + k * ws, prev, ch);
        moved |= uint32_t(ch) << k;
    }
    return moved;
}

// bit k of x to bit 2k (32 -> 64 bits)
__device__ __forceinline__ uint64_t spread2(uint32_t x) {
    uint64_t v = x;
    v = (v | (v << 16)) & 0x0000FFFF0000FFFFull;
    v = (v | (v << 8)) & 0x00FF00FF00FF00FFull;
    v = (v | (v << 4)) & 0x0F0F0F0F0F0F0F0Full;
    v = (v | (v << 2)) & 0x3333333333333333ull;
    v = (v | (v << 1)) & 0x5555555555555555ull;
    return v;
}

// Line ids of a tile: 0-31 rows r, 32-63 columns c, 64-126 main diagonals i - j = e (id 95 + e), 127-189
// anti-diagonals i + j = s (id 127 + s). Dirty sets are 6 words: rows, columns, 2 x diagonals, 2 x anti-diagonals.
constexpr int NLINES = 190;

// Walk line `id`, then add to `mark` every line through a cell whose cost went down (its own included).
template <int NL>
__device__ __forceinline__ bool walk_id(const SDev& S, uint32_t* dS, const uint16_t* wS, const uint32_t* vS,
                                        const uint32_t* vokS, int id, int dir, uint32_t (&mark)[6]) {
    int plane, d0, ds, w0, ws, len, pf, pb;
    int fam, a0 = 0, b0 = 0;
    if (id < 32) {
        const int r = id;
        fam = 0; a0 = r;
        plane = S.plane_h; d0 = (r + 1) * DSTR + 1; ds = 1; w0 = r * CSTR; ws = 1; len = TILE;
        pf = (r + 1) * DSTR; pb = (r + 1) * DSTR + TILE + 1;
    } else if (id < 64) {
        const int c = id - 32;
        fam = 1; a0 = c;
        plane = S.plane_v; d0 = DSTR + c + 1; ds = DSTR; w0 = c; ws = CSTR; len = TILE;
        pf = c + 1; pb = (TILE + 1) * DSTR + c + 1;
    } else if (id < 127) {
        const int e = id - 95;
        const int i0 = e > 0 ? e : 0, j0 = e < 0 ? -e : 0;
        fam = 2; a0 = i0; b0 = j0;
        plane = S.plane_d; len = TILE - (e < 0 ? -e : e);
        d0 = (j0 + 1) * DSTR + i0 + 1; ds = DSTR + 1; w0 = j0 * CSTR + i0; ws = CSTR + 1;
        pf = j0 * DSTR + i0; pb = (j0 + len + 1) * DSTR + i0 + len + 1;
    } else {
        const int s = id - 127;
        const int lo = s > TILE - 1 ? s - (TILE - 1) : 0;
        fam = 3; a0 = s; b0 = lo;
        plane = S.plane_d; len = TILE - (s > TILE - 1 ? s - (TILE - 1) : (TILE - 1) - s);
        d0 = (lo + 1) * DSTR + (s - lo) + 1; ds = DSTR - 1; w0 = lo * CSTR + (s - lo); ws = CSTR - 1;
        pf = lo * DSTR + (s - lo + 2); pb = (s - lo + 2) * DSTR + lo;
    }
    const uint32_t M = walk_line<NL>(dS, wS + plane * S.nl * WLS, vS, vokS, d0, ds, w0, ws, len, pf, pb, dir);
    if (!M) return false;
    uint64_t d1 = 0, d2 = 0;
    if (fam == 0) {            // row r, cell (r, k): column k, diagonal k - r, anti-diagonal r + k
        mark[0] |= 1u << a0;
        mark[1] |= M;
        d1 = uint64_t(M) << (TILE - 1 - a0);
        d2 = uint64_t(M) << a0;
    } else if (fam == 1) {     // column c, cell (k, c): row k, diagonal c - k, anti-diagonal k + c
        mark[1] |= 1u << a0;
        mark[0] |= M;
        d1 = uint64_t(__brev(M)) << a0;
        d2 = uint64_t(M) << a0;
    } else if (fam == 2) {     // diagonal from (i0, j0), cell (j0 + k, i0 + k): anti-diagonal i0 + j0 + 2k
        const int e = id - 95;
        d1 = 1ull << (e + TILE - 1);
        mark[0] |= M << b0;
        mark[1] |= M << a0;
        d2 = spread2(M) << (a0 + b0);
    } else {                   // anti-diagonal s, cell (lo + k, s - lo - k): diagonal s - 2 lo - 2k
        const int s = a0, lo = b0;
        d2 = 1ull << s;
        mark[0] |= M << lo;
        mark[1] |= __brev(M) >> (TILE - 1 - (s - lo));
        d1 = spread2(__brev(M)) >> (TILE - 1 - s + 2 * lo);
    }
    mark[2] |= uint32_t(d1);
    mark[3] |= uint32_t(d1 >> 32);
    mark[4] |= uint32_t(d2);
    mark[5] |= uint32_t(d2 >> 32);
    return true;
}

// Position of set bit k (counted from 0) of x; x has more than k set bits.
__device__ __forceinline__ int select_bit(uint32_t x, int k) {
    int pos = 0, c;
    c = __popc(x & 0xFFFFu); if (k >= c) { k -= c; x >>= 16; pos += 16; }
    c = __popc(x & 0xFFu);   if (k >= c) { k -= c; x >>= 8;  pos += 8; }
    c = __popc(x & 0xFu);    if (k >= c) { k -= c; x >>= 4;  pos += 4; }
    c = __popc(x & 0x3u);    if (k >= c) { k -= c; x >>= 2;  pos += 2; }
    return pos + (k >= int(x & 1u) ? 1 : 0);
}

// Relax a tile to its local fixed point. The lines whose end cells read a changed halo side start dirty (every
// line after a start was written or a visit stopped early). Each iteration walks every dirty line both ways, one
// walk unit per thread, packed onto the fewest warps, and marks the lines through the cells that went down, the
// walked line included (its other direction may have passed those cells before they went down). The visit ends
// after an iteration with no dirty line, i.e. after a pass in which no line changed anything.
//
// One block barrier per iteration. The dirty sets rotate through three buffers: an iteration reads one, ORs its
// marks into the next, and clears the third, which the previous iteration read and the next one writes. With P
// dirty lines, thread t < P walks the t-th dirty line forward and thread P + t walks it backward; each thread
// finds its line by popcounts over the 6 words, so the units need no compacted list.
template <int NL>
__device__ int relax_joint(const SDev& S, uint32_t* dS, const uint16_t* wS, const uint32_t* vS, const uint32_t* vokS,
                           VisitShared& sh, bool& requeue) {
    __shared__ uint32_t dirty[3][6];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        uint32_t w[6];
        side_lines(sh.sides, w);
        for (int k = 0; k < 6; ++k) { dirty[0][k] = w[k]; dirty[1][k] = 0; dirty[2][k] = 0; }
    }
    int cur = 0, nxt = 1, old = 2;
    for (int it = 0;; ++it) {
        __syncthreads();
        uint32_t w[6];
        int pc[6], P = 0;
        #pragma unroll
        for (int k = 0; k < 6; ++k) {
            w[k] = dirty[cur][k];
            pc[k] = __popc(w[k]);
            P += pc[k];
        }
        if (P == 0) return it;
        if (tid < 6) dirty[old][tid] = 0;
        const int total = 2 * P;
        uint32_t mark[6] = {0, 0, 0, 0, 0, 0};
        bool changed = false;
        if (tid < total) {
            const int dir = tid < P ? 0 : 1;
            int k = dir ? tid - P : tid, base = 0;
            uint32_t x = w[0];
            if (k >= pc[0]) { k -= pc[0]; base = 32; x = w[1];
                if (k >= pc[1]) { k -= pc[1]; base = 64; x = w[2];
                    if (k >= pc[2]) { k -= pc[2]; base = 96; x = w[3];
                        if (k >= pc[3]) { k -= pc[3]; base = 127; x = w[4];
                            if (k >= pc[4]) { k -= pc[4]; base = 159; x = w[5]; } } } } }
            changed = walk_id<NL>(S, dS, wS, vS, vokS, base + select_bit(x, k), dir, mark);
        }
        if (warp * 32 < total) {
            #pragma unroll
            for (int q = 0; q < 6; ++q) {
                const uint32_t m = __reduce_or_sync(0xFFFFFFFFu, mark[q]);
                if (lane == 0 && m) atomicOr(&dirty[nxt][q], m);
            }
            if (__any_sync(0xFFFFFFFFu, changed) && lane == 0) sh.any = 1;
        }
        if (it + 1 >= MAX_IT) {
            __syncthreads();
            bool left = false;
            if (tid < 6) left = dirty[nxt][tid] != 0;
            if (__syncthreads_or(left)) requeue = true;
            return it + 1;
        }
        const int t = cur; cur = nxt; nxt = old; old = t;
    }
}

// ---- per-layer scans with weights computed per move (mode 0: any factors, 64-bit distances) ----

template <typename DT>
__device__ int relax_general(const SDev& S, DT* dS, const float* cS, const DT* vS, const uint32_t* vokS,
                             VisitShared& sh, bool& requeue) {
    const int tid = threadIdx.x, nl = S.nl;
    for (int it = 0;; ++it) {
        int ch = 0;
        for (int line = tid; line < nl * TILE; line += NT) {      // rows: +x, -x
            const int l = line >> 5, r = line & 31;
            DT* row = dS + l * LS + (r + 1) * DSTR;
            const float* crow = cS + l * WLS + r * CSTR;
            DT prev = row[0];
            for (int k = 0; k < TILE; ++k) {
                const DT v = row[k + 1], n = dmin(v, prev + qweight<DT>(crow[k], S.fac[l][0]));
                if (n < v) { row[k + 1] = n; ch = 1; }
                prev = n;
            }
            prev = row[TILE + 1];
            for (int k = TILE - 1; k >= 0; --k) {
                const DT v = row[k + 1], n = dmin(v, prev + qweight<DT>(crow[k], S.fac[l][1]));
                if (n < v) { row[k + 1] = n; ch = 1; }
                prev = n;
            }
        }
        __syncthreads();
        for (int line = tid; line < nl * TILE; line += NT) {      // columns: +y, -y
            const int l = line >> 5, c = line & 31;
            DT* col = dS + l * LS + c + 1;
            const float* ccol = cS + l * WLS + c;
            DT prev = col[0];
            for (int k = 0; k < TILE; ++k) {
                const DT v = col[(k + 1) * DSTR], n = dmin(v, prev + qweight<DT>(ccol[k * CSTR], S.fac[l][2]));
                if (n < v) { col[(k + 1) * DSTR] = n; ch = 1; }
                prev = n;
            }
            prev = col[(TILE + 1) * DSTR];
            for (int k = TILE - 1; k >= 0; --k) {
                const DT v = col[(k + 1) * DSTR], n = dmin(v, prev + qweight<DT>(ccol[k * CSTR], S.fac[l][3]));
                if (n < v) { col[(k + 1) * DSTR] = n; ch = 1; }
                prev = n;
            }
        }
        __syncthreads();
        for (int line = tid; line < nl * (2 * TILE - 1); line += NT) {   // i - j = e: (+,+), (-,-)
            const int l = line / (2 * TILE - 1), e = line % (2 * TILE - 1) - (TILE - 1);
            const int i0 = e > 0 ? e : 0, j0 = e < 0 ? -e : 0, len = TILE - (e < 0 ? -e : e);
            DT* base = dS + l * LS;
            const float* cb = cS + l * WLS;
            DT prev = base[j0 * DSTR + i0];
            for (int k = 0; k < len; ++k) {
                DT* p = base + (j0 + k + 1) * DSTR + i0 + k + 1;
                const DT v = *p, n = dmin(v, prev + qweight<DT>(cb[(j0 + k) * CSTR + i0 + k], S.fac[l][4]));
                if (n < v) { *p = n; ch = 1; }
                prev = n;
            }
            prev = base[(j0 + len + 1) * DSTR + i0 + len + 1];
            for (int k = len - 1; k >= 0; --k) {
                DT* p = base + (j0 + k + 1) * DSTR + i0 + k + 1;
                const DT v = *p, n = dmin(v, prev + qweight<DT>(cb[(j0 + k) * CSTR + i0 + k], S.fac[l][7]));
                if (n < v) { *p = n; ch = 1; }
                prev = n;
            }
        }
        __syncthreads();
        for (int line = tid; line < nl * (2 * TILE - 1); line += NT) {   // i + j = s: (-,+), (+,-)
            const int l = line / (2 * TILE - 1), s = line % (2 * TILE - 1);
            const int lo = s > TILE - 1 ? s - (TILE - 1) : 0;
            const int len = TILE - (s > TILE - 1 ? s - (TILE - 1) : (TILE - 1) - s);
            DT* base = dS + l * LS;
            const float* cb = cS + l * WLS;
            DT prev = base[lo * DSTR + (s - lo + 2)];
            for (int k = 0; k < len; ++k) {
                const int j = lo + k, i = s - j;
                DT* p = base + (j + 1) * DSTR + i + 1;
                const DT v = *p, n = dmin(v, prev + qweight<DT>(cb[j * CSTR + i], S.fac[l][6]));
                if (n < v) { *p = n; ch = 1; }
                prev = n;
            }
            prev = base[(s - lo + 2) * DSTR + lo];
            for (int k = 0; k < len; ++k) {
                const int i = lo + k, j = s - i;
                DT* p = base + (j + 1) * DSTR + i + 1;
                const DT v = *p, n = dmin(v, prev + qweight<DT>(cb[j * CSTR + i], S.fac[l][5]));
                if (n < v) { *p = n; ch = 1; }
                prev = n;
            }
        }
        __syncthreads();
        for (int cell = tid; cell < TILE * TILE; cell += NT) {           // vias
            const int r = cell >> 5, c = cell & 31;
            const DT wv = vS[r * CSTR + c];
            const uint32_t vm = vokS[r * CSTR + c];
            if (wv >= Lim<DT>::INF || !vm) continue;
            DT best = Lim<DT>::INF;
            for (int l = 0; l < nl; ++l) best = dmin(best, dS[l * LS + (r + 1) * DSTR + c + 1]);
            if (best >= Lim<DT>::INF) continue;
            const DT n = best + wv;
            for (int l = 0; l < nl; ++l) {
                if (!((vm >> l) & 1)) continue;
                DT* p = dS + l * LS + (r + 1) * DSTR + c + 1;
                if (n < *p) { *p = n; ch = 1; }
            }
        }
        const int any = __syncthreads_or(ch);
        if (!any) return it + 1;
        if (tid == 0) sh.any = 1;
        if (it + 1 >= MAX_IT) { requeue = true; return it + 1; }
    }
}

// ---- one tile visit ----

template <typename DT>
__device__ void visit_tile(const SolveArgs& a, int s, int tile, int round, unsigned char* smem) {
    const SDev& S = a.S[s];
    const int tid = threadIdx.x;
    const int nl = S.nl, pitch = S.pitch, hpad = S.hpad;
    const int tx = tile % S.ntx, ty = tile / S.ntx;
    const int x0 = tx * TILE, y0 = ty * TILE;
    const bool joint = sizeof(DT) == 4 && S.mode == 1;
    const Lay L = layout_for(a.nlmax, a.kmax, sizeof(DT), joint ? 1 : 0);
    DT* dS = reinterpret_cast<DT*>(smem + L.d);
    DT* vS = reinterpret_cast<DT*>(smem + L.v);
    DT* eS = reinterpret_cast<DT*>(smem + L.e);
    uint32_t* vokS = reinterpret_cast<uint32_t*>(smem + L.m);
    uint32_t* tgS = vokS + WLS;
    __shared__ VisitShared sh;
    const DT INF = Lim<DT>::INF;
    if (tid == 0) {
        sh.marks = 0; sh.any = 0; sh.wide = 0; sh.iters = 0; sh.tmin = ~0ull; sh.wmax = 0;
        sh.wcnt = 0; sh.wsum = 0;
        for (int b = 0; b < 8; ++b) sh.mkey[b] = KEY_NONE;
        // The key that queued the tile and which halo sides changed since the last visit, taken before the halo is
        // read, so that a neighbour that marks us afterwards has also queued us for the next round with its key.
        // The key goes first: a marking neighbour sets its side bit before it lowers the key (with a fence between),
        // so a visit that takes a mark's key also takes that mark's side bit, and a round that finds the key gone
        // may skip the tile (its marks were all consumed by a visit that walked their sides).
        sh.kvis = a.ordered ? atomicExch(S.tkey + tile, KEY_NONE) : KEY_NONE;
        __threadfence();
        sh.sides = atomicExch(S.sides + tile, 0u);
        __threadfence();   // the halo reads below come after the exchange that saw the neighbours' marks
    }
    __syncthreads();

    // ---- stage
    stage_dist<DT>(S, dS, x0, y0);
    unsigned long long wmax = 0, wsum = 0;
    unsigned int wcnt = 0;
    bool wide = false;
    bool fallback = false;   // joint search whose weights do not fit 16 bits in this tile: general relaxation
    if (joint) {
        // integer weights of the x, y and diagonal move classes of every state, 16 bits each (0xFFFF impassable)
        uint16_t* wS = reinterpret_cast<uint16_t*>(smem + L.w);
        bool big = false;
        auto w16 = [&](uint32_t w) -> uint16_t {
            if (w >= INF32) return 0xFFFFu;
            if (w >= 0xFFFFu) { big = true; return 0xFFFEu; }
            return uint16_t(w);
        };
        constexpr int WCH = 4;
        const int groups = nl * TILE * TILE / 4;   // 4 cells of one row and layer per 128-bit load
        for (int base = tid; base < groups; base += NT * WCH) {
            float4 q4[WCH];
            #pragma unroll
            for (int u = 0; u < WCH; ++u) {
                const int g = base + u * NT;
                if (g < groups) {
                    const int l = g >> 8, r = (g >> 3) & 31, c0 = (g & 7) * 4;
                    q4[u] = *reinterpret_cast<const float4*>(S.cf + (size_t(l) * hpad + y0 + r) * pitch + x0 + c0);
                }
            }
            #pragma unroll
            for (int u = 0; u < WCH; ++u) {
                const int g = base + u * NT;
                if (g >= groups) break;
                const int l = g >> 8, r = (g >> 3) & 31, c0 = (g & 7) * 4;
                const float cv[4] = {q4[u].x, q4[u].y, q4[u].z, q4[u].w};
                #pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const float cf = cv[e];
                    if (cf < 1e30f && !(__fmul_rn(__fmul_rn(cf, S.maxfac[l]), 16.0f) < WLIM32)) wide = true;
                    const uint32_t wx = qweight<uint32_t>(cf, S.fac[l][0]), wy = qweight<uint32_t>(cf, S.fac[l][2]);
                    const uint32_t wd = qweight<uint32_t>(cf, S.fac[l][4]);
                    if (wx < INF32) { wsum += wx; ++wcnt; }
                    const int o = l * WLS + r * CSTR + c0 + e;
                    wS[o] = w16(wx);
                    if (S.K == 3) wS[nl * WLS + o] = w16(wy);
                    wS[(S.K - 1) * nl * WLS + o] = w16(wd);
                    if (cf < 1e30f) {
                        const uint32_t mw = max(max(wx < INF32 ? wx : 0u, wy < INF32 ? wy : 0u), wd < INF32 ? wd : 0u);
                        wmax = max(wmax, static_cast<unsigned long long>(mw));
                    }
                }
            }
        }
        fallback = __syncthreads_or(big);
        if (fallback) {  // the same region now holds the float cost factors of the general relaxation
            float* cS = reinterpret_cast<float*>(smem + L.w);
            for (int idx = tid; idx < nl * TILE * TILE; idx += NT) {
                const int l = idx >> 10, r = (idx >> 5) & 31, c = idx & 31;
                cS[l * WLS + r * CSTR + c] = S.cf[(size_t(l) * hpad + y0 + r) * pitch + x0 + c];
            }
        }
    } else {
        float* cS = reinterpret_cast<float*>(smem + L.w);
        for (int idx = tid; idx < nl * TILE * TILE; idx += NT) {
            const int l = idx >> 10, r = (idx >> 5) & 31, c = idx & 31;
            const float cf = S.cf[(size_t(l) * hpad + y0 + r) * pitch + x0 + c];
            cS[l * WLS + r * CSTR + c] = cf;
            if (cf < 1e30f) {
                const float y = __fmul_rn(__fmul_rn(cf, S.maxfac[l]), 16.0f);
                if (!(y < Lim<DT>::wlim())) wide = true;
                else wmax = max(wmax, static_cast<unsigned long long>(qweight<DT>(cf, S.maxfac[l])));
                if (a.ordered) {
                    const uint32_t wx = qweight<uint32_t>(cf, S.fac[l][0]);
                    if (wx < INF32) { wsum += wx; ++wcnt; }
                }
            }
        }
    }
    stage_cells<DT>(S, vS, vokS, tgS, x0, y0, wide, wmax);
    __syncthreads();
    save_edges<DT>(S, dS, eS);
    if (wide) atomicOr(&sh.wide, 1u);
    if (wmax) atomicMax(&sh.wmax, wmax);
    if (a.ordered && wcnt) { atomicAdd(&sh.wcnt, wcnt); atomicAdd(&sh.wsum, wsum); }
    __syncthreads();
    // the search's weight scale (ordered rounds): the least mean straight-move weight of a well-filled tile, i.e.
    // what a step through open board costs, whatever the congested or blocked parts cost
    if (a.ordered && tid == 0 && sh.wcnt >= 128) {
        const unsigned long long mean = sh.wsum / sh.wcnt;
        atomicMin(&a.st[s].wscale, mean < KEY_NONE ? unsigned(mean) : KEY_NONE - 1);
    }

    // ---- relax to a local fixed point
    bool requeue = false;
    int iters;
    if (joint && !fallback) {
        const uint16_t* wS = reinterpret_cast<const uint16_t*>(smem + L.w);
        uint32_t* d32 = reinterpret_cast<uint32_t*>(dS);
        const uint32_t* v32 = reinterpret_cast<const uint32_t*>(vS);
        switch (nl) {
            case 1: iters = relax_joint<1>(S, d32, wS, v32, vokS, sh, requeue); break;
            case 2: iters = relax_joint<2>(S, d32, wS, v32, vokS, sh, requeue); break;
            case 3: iters = relax_joint<3>(S, d32, wS, v32, vokS, sh, requeue); break;
            case 4: iters = relax_joint<4>(S, d32, wS, v32, vokS, sh, requeue); break;
            case 5: iters = relax_joint<5>(S, d32, wS, v32, vokS, sh, requeue); break;
            case 6: iters = relax_joint<6>(S, d32, wS, v32, vokS, sh, requeue); break;
            case 7: iters = relax_joint<7>(S, d32, wS, v32, vokS, sh, requeue); break;
            default: iters = relax_joint<8>(S, d32, wS, v32, vokS, sh, requeue); break;
        }
    } else {
        iters = relax_general<DT>(S, dS, reinterpret_cast<const float*>(smem + L.w), vS, vokS, sh, requeue);
    }
    __syncthreads();

    // ---- targets of the tile: least distance into the search's bound
    const unsigned long long ub_now = *reinterpret_cast<volatile unsigned long long*>(&a.st[s].ub);
    {
        unsigned long long tmin = ~0ull;
        for (int cell = tid; cell < TILE * TILE; cell += NT) {
            const int r = cell >> 5, c = cell & 31;
            const uint32_t tm = tgS[r * CSTR + c];
            if (!tm) continue;
            for (int l = 0; l < nl; ++l)
                if ((tm >> l) & 1) {
                    const DT v = dS[l * LS + (r + 1) * DSTR + c + 1];
                    if (v < INF) tmin = min(tmin, static_cast<unsigned long long>(v));
                }
        }
        if (tmin != ~0ull) atomicMin(&sh.tmin, tmin);
    }
    __syncthreads();
    const unsigned long long ub = min(ub_now, sh.tmin);
    if (sh.any) {
        DT* distw = reinterpret_cast<DT*>(S.dist);
        if constexpr (sizeof(DT) == 4) {   // 16-byte stores: 4 cells of a row per store
            for (int g = tid; g < nl * TILE * TILE / 4; g += NT) {
                const int l = g >> 8, r = (g >> 3) & 31, c0 = (g & 7) * 4;
                const DT* src = dS + l * LS + (r + 1) * DSTR + c0 + 1;
                *reinterpret_cast<uint4*>(distw + (size_t(l) * hpad + y0 + r) * pitch + x0 + c0) =
                    make_uint4(src[0], src[1], src[2], src[3]);
            }
        } else {
            for (int idx = tid; idx < nl * TILE * TILE; idx += NT) {
                const int l = idx >> 10, r = (idx >> 5) & 31, c = idx & 31;
                distw[(size_t(l) * hpad + y0 + r) * pitch + x0 + c] = dS[l * LS + (r + 1) * DSTR + c + 1];
            }
        }
        // an edge cell that improved (to at most the bound) below an adjacent neighbour cell's staged value:
        // that neighbour looks again. bits: 0 L, 1 R, 2 T, 3 B, 4 TL, 5 TR, 6 BL, 7 BR
        // A warp's 32 consecutive entries are the 32 cells of one side of one layer (the loop bound and NT are
        // multiples of 32), so the warp reduces its marks, and in ordered rounds their keys, before shared atomics.
        unsigned int marks = 0;
        for (int idx = tid; idx < nl * 4 * TILE; idx += NT) {
            const int l = idx / (4 * TILE), side = (idx / TILE) & 3, k = idx % TILE;
            int r, c;
            edge_rc(side, k, r, c);
            const DT v = dS[l * LS + (r + 1) * DSTR + c + 1];
            unsigned int bits = 0;
            if (v < eS[idx] && static_cast<unsigned long long>(v) <= ub) {
                const DT* hb = dS + l * LS;
                // the three halo cells across this side, and the neighbour tile each belongs to
                for (int t = -1; t <= 1; ++t) {
                    int hr, hc, bit;
                    if (side == 0 || side == 1) {
                        hr = r + t; hc = side == 0 ? -1 : TILE;
                        bit = hr < 0 ? (side == 0 ? 4 : 5) : hr >= TILE ? (side == 0 ? 6 : 7) : side;
                    } else {
                        hc = c + t; hr = side == 2 ? -1 : TILE;
                        bit = hc < 0 ? (side == 2 ? 4 : 6) : hc >= TILE ? (side == 2 ? 5 : 7) : side;
                    }
                    if (v < hb[(hr + 1) * DSTR + hc + 1]) bits |= 1u << bit;
                }
            }
            const unsigned int wbits = __reduce_or_sync(0xFFFFFFFFu, bits);
            marks |= wbits;
            if (a.ordered && wbits) {
                const uint32_t key = key_of<DT>(v);
                for (unsigned int rest = wbits; rest; rest &= rest - 1) {
                    const int b = __ffs(rest) - 1;
                    const uint32_t kb = __reduce_min_sync(0xFFFFFFFFu, ((bits >> b) & 1u) ? key : KEY_NONE);
                    if ((tid & 31) == 0) atomicMin(&sh.mkey[b], kb);
                }
            }
        }
        if (marks && (tid & 31) == 0) atomicOr(&sh.marks, marks);
        __threadfence();   // the written distances are visible device-wide before any neighbour is marked
    }
    if (tid == 0) sh.iters = unsigned(iters);
    __syncthreads();
    // lanes 0-7 of warp 0 queue the marked neighbours, lane 8 the tile itself when its visit stopped early, lane 0
    // updates the search's bound and counters
    if (tid == 0) {
        SStat& st = a.st[s];
        if (sh.tmin != ~0ull && sh.tmin < ub_now) atomicMin(&st.ub, sh.tmin);
        if (sh.wmax) atomicMax(&st.maxw, sh.wmax);
        if (sh.wide) atomicOr(&st.need_wide, 1u);
        atomicAdd(a.visits, 1ull);
        atomicAdd(a.visits + 1, static_cast<unsigned long long>(nl));
        atomicAdd(a.visits + 2, static_cast<unsigned long long>(sh.iters));
    }
    if (tid < 8 && ((sh.marks >> tid) & 1u)) {
        const int b = tid;
        const int DXs[8] = {-1, 1, 0, 0, -1, 1, -1, 1}, DYs[8] = {0, 0, -1, 1, -1, -1, 1, 1};
        const int nx = tx + DXs[b], ny = ty + DYs[b];
        if (nx >= 0 && ny >= 0 && nx < S.ntx && ny < S.nty) {
            atomicOr(S.sides + ny * S.ntx + nx, opposite_side(b));   // the side of the neighbour facing us
            __threadfence();                                           // the side bit before the key (see above)
            queue_tile(a, S, s, ny * S.ntx + nx, round + 1, sh.mkey[b]);
        }
    }
    if (tid == 8 && requeue) {
        atomicOr(S.sides + tile, SIDE_ALL);
        __threadfence();
        queue_tile(a, S, s, tile, round + 1, sh.kvis == KEY_NONE ? 0u : sh.kvis);
    }
    __syncthreads();
}

// Two builds of the kernel: MINB = 2 blocks per SM with up to 80 registers a thread, or MINB = 3 within 56
// registers (the 32-bit build spills 124 bytes). A third resident block fills more of the time that warps wait at the
// local-iteration barrier, but each block runs slower; relax_launch takes it only for batches with many tiles.
template <typename DT, int MINB>
__global__ void __launch_bounds__(NT, MINB) relax_kernel(SolveArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ unsigned int sh_item_hi, sh_item_lo, sh_stop;
    __shared__ long long sh_t0, sh_tv, sh_busy;   // SM clock at start and at the current visit; cycles visiting
    const unsigned int nblocks = gridDim.x;
    const int tid = threadIdx.x;
    if (tid == 0) { sh_t0 = clock64(); sh_busy = 0; }
    int round = 1;
    for (;; ++round) {
        const int buf = round % 3;
        const unsigned int n = *reinterpret_cast<volatile unsigned int*>(a.ctl + C_CNT + buf);
        const unsigned int cnt = n < a.cap ? n : a.cap;
        // The items visited this round and where the blocks take them from: the round's list itself, or (ordered
        // rounds) the visit list that the filter below builds from it.
        const unsigned long long* items = a.wl + size_t(buf) * a.cap;
        unsigned int* next = a.ctl + C_NEXT + buf;
        unsigned int vcnt = cnt, vfront = cnt;
        if (a.ordered) {
            // Filter, all threads of the grid over the round's list. A tile whose key is gone was visited after it
            // was listed (its improvements with it); one keyed above the search's best target has nothing that
            // can matter; one keyed above the search's band waits for a later round (listed again, its key and
            // the next round's least key kept). The rest make the visit list.
            const int vp = round & 1;
            const unsigned int widen = *reinterpret_cast<volatile unsigned int*>(a.ctl + C_WIDEN);
            const unsigned long long band = static_cast<unsigned long long>(a.band) << widen;
            if (blockIdx.x == 0 && tid == 0) {
                a.ctl[C_VCNT + (vp ^ 1)] = 0;
                a.ctl[C_BCNT + (vp ^ 1)] = 0;
                a.ctl[C_VNEXT + (vp ^ 1)] = 0;
            }
            for (int q = blockIdx.x * NT + tid; q < a.n; q += nblocks * NT) a.st[q].kmin[(round + 2) % 3] = KEY_NONE;
            unsigned int deferred = 0, dropped = 0;
            for (unsigned int k = blockIdx.x * NT + tid; k < cnt; k += nblocks * NT) {
                const unsigned long long it = __ldcg(items + k);
                const int s = int(it >> 32), tile = int(it & 0xFFFFFFFFu);
                const SDev& S = a.S[s];
                const uint32_t key = __ldcg(S.tkey + tile);
                if (key == KEY_NONE) continue;
                const SStat& st = a.st[s];
                const unsigned long long ub = *reinterpret_cast<const volatile unsigned long long*>(&st.ub);
                if (key > ub) { ++dropped; continue; }
                const uint32_t km = *reinterpret_cast<const volatile unsigned int*>(&st.kmin[buf]);
                const uint32_t ws = *reinterpret_cast<const volatile unsigned int*>(&st.wscale);
                const unsigned long long thr = ws == KEY_NONE || km == KEY_NONE
                    ? ~0ull : static_cast<unsigned long long>(km) + static_cast<unsigned long long>(ws) * band;
                if (key > thr) {
                    queue_tile(a, S, s, tile, round + 1, key);
                    ++deferred;
                    continue;
                }
                // Front or back of the visit list; blocks take the front first, then the back from its end. Each
                // listed item is placed at most once, so the two parts (at most cnt <= cap items) never meet.
                bool front = true;
                if (a.order == ORDER_KEY)
                    front = thr == ~0ull || key <= km ||
                            2ull * (key - km) <= static_cast<unsigned long long>(ws) * band;
                else if (a.order == ORDER_LAYERS)
                    front = 2 * S.nl > a.nlmax;
                if (front) {
                    const unsigned int pos = atomicAdd(a.ctl + C_VCNT + vp, 1u);
                    a.vl[pos] = it;
                } else {
                    const unsigned int pos = atomicAdd(a.ctl + C_BCNT + vp, 1u);
                    a.vl[a.cap - 1u - pos] = it;
                }
            }
            deferred = __reduce_add_sync(0xFFFFFFFFu, deferred);
            dropped = __reduce_add_sync(0xFFFFFFFFu, dropped);
            if ((tid & 31) == 0 && deferred) atomicAdd(a.visits + 3, static_cast<unsigned long long>(deferred));
            if ((tid & 31) == 0 && dropped) atomicAdd(a.visits + 4, static_cast<unsigned long long>(dropped));
            grid_barrier(a.ctl, nblocks);
            items = a.vl;
            next = a.ctl + C_VNEXT + vp;
            vfront = *reinterpret_cast<volatile unsigned int*>(a.ctl + C_VCNT + vp);
            vcnt = vfront + *reinterpret_cast<volatile unsigned int*>(a.ctl + C_BCNT + vp);
            // A round whose visit list cannot keep every block busy widens the next round's band (doubling it, up
            // to unordered); a round with far more tiles than blocks narrows it again. Read by every block only
            // after the end-of-round barrier, so the whole grid uses one band per round.
            if (blockIdx.x == 0 && tid == 0) {
                unsigned int w = widen;
                if (vcnt < 2 * nblocks) w = w < MAX_WIDEN ? w + 1 : w;
                else if (vcnt > 16 * nblocks && w > 0) w -= 1;
                a.ctl[C_WIDEN] = w;
            }
        }
        for (;;) {
            if (tid == 0) {
                const unsigned int k = atomicAdd(next, 1u);
                if (k < vcnt) {
                    // written last round, or by the filter (the back part from the list's end)
                    const unsigned long long it = __ldcg(items + (k < vfront ? k : a.cap - 1u - (k - vfront)));
                    sh_item_hi = unsigned(it >> 32);
                    sh_item_lo = unsigned(it & 0xFFFFFFFFu);
                } else {
                    sh_item_hi = 0xFFFFFFFFu;
                }
            }
            __syncthreads();
            const unsigned int hi = sh_item_hi, lo = sh_item_lo;
            __syncthreads();
            if (hi == 0xFFFFFFFFu) break;
            if (tid == 0) sh_tv = clock64();
            visit_tile<DT>(a, int(hi), int(lo), round, smem);   // ends with a block barrier
            if (tid == 0) sh_busy += clock64() - sh_tv;
        }
        // the list consumed last round is free: clear it for the round after next
        if (blockIdx.x == 0 && tid == 0) {
            const int fb = (round + 2) % 3;
            a.ctl[C_CNT + fb] = 0;
            a.ctl[C_NEXT + fb] = 0;
        }
        grid_barrier(a.ctl, nblocks);
        if (tid == 0) {
            const unsigned int err = *reinterpret_cast<volatile unsigned int*>(a.ctl + C_ERR);
            const unsigned int nn = *reinterpret_cast<volatile unsigned int*>(a.ctl + C_CNT + (round + 1) % 3);
            sh_stop = (err != 0 || nn == 0) ? 1u : 0u;
            if (!sh_stop && round >= a.max_rounds) {
                atomicOr(a.ctl + C_ERR, unsigned(ERR_ROUNDS));
                sh_stop = 1u;
            }
        }
        __syncthreads();
        if (sh_stop) break;
    }
    if (blockIdx.x == 0 && tid == 0) a.ctl[C_ROUNDS] = unsigned(round);
    if (tid == 0) {
        atomicAdd(a.visits + 5, static_cast<unsigned long long>(sh_busy));
        atomicAdd(a.visits + 6, static_cast<unsigned long long>(clock64() - sh_t0));
    }
}

// starts: distance init (least per state) and the first round's tiles. A start's value is written here, not by a
// visit, so no visit sees it "improve": the tile holding it and all 8 neighbours (which read it through their
// halo) are queued.
template <typename DT>
__global__ void seed_kernel(SolveArgs a, const uint32_t* const* sidx, const uint64_t* const* sd, const int* ns) {
    const int s = blockIdx.x;
    const SDev& S = a.S[s];
    DT* dist = reinterpret_cast<DT*>(S.dist);
    const size_t RN = size_t(S.rw) * S.rh;
    for (int k = threadIdx.x; k < ns[s]; k += blockDim.x) {
        const uint32_t q = sidx[s][k];
        const int l = int(q / RN), rem = int(q % RN), j = rem / S.rw, i = rem % S.rw;
        if (l >= S.nl) continue;
        uint64_t v = sd[s][k];
        if (v >= uint64_t(Lim<DT>::INF)) continue;
        atomic_min_d(dist + (size_t(l) * S.hpad + j) * S.pitch + i, DT(v));
        const int tx = i / TILE, ty = j / TILE;
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const int nx = tx + dx, ny = ty + dy;
                if (nx >= 0 && ny >= 0 && nx < S.ntx && ny < S.nty) {
                    atomicOr(S.sides + ny * S.ntx + nx, SIDE_ALL);
                    queue_tile(a, S, s, ny * S.ntx + nx, 1, key_of<DT>(DT(v)));
                }
            }
    }
}

// report: the cheapest target (least state index among those at the bound), the field, the largest distance
template <typename DT>
__global__ void report_kernel(const SDev* Sv, SStat* stv) {
    const int s = blockIdx.y;
    const SDev& S = Sv[s];
    SStat& st = stv[s];
    const DT INF = Lim<DT>::INF;
    const DT* dist = reinterpret_cast<const DT*>(S.dist);
    const unsigned long long ub = st.ub;
    const bool have = ub < static_cast<unsigned long long>(INF);
    const size_t RN = size_t(S.rw) * S.rh, N = RN * S.nl;
    unsigned long long bidx = ~0ull, maxd = 0;
    unsigned int low = 0;
    for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < N; q += size_t(gridDim.x) * blockDim.x) {
        const int l = int(q / RN), rem = int(q % RN), j = rem / S.rw, i = rem % S.rw;
        const size_t p = (size_t(l) * S.hpad + j) * S.pitch + i;
        const DT d = dist[p];
        const bool rep = d < INF && (!have || static_cast<unsigned long long>(d) <= ub);
        if (d < INF) {
            maxd = max(maxd, static_cast<unsigned long long>(d));
            if (have && (S.fl[p] & 2) && static_cast<unsigned long long>(d) == ub) bidx = min(bidx, static_cast<unsigned long long>(q));
        }
        low += rep ? 1u : 0u;
        if (S.out) S.out[q] = rep ? __ull2float_rn(d) * 0.0625f : 1e30f;
    }
    for (int o = 16; o; o >>= 1) {
        bidx = min(bidx, __shfl_xor_sync(0xFFFFFFFFu, bidx, o));
        maxd = max(maxd, __shfl_xor_sync(0xFFFFFFFFu, maxd, o));
        low += __shfl_xor_sync(0xFFFFFFFFu, low, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (bidx != ~0ull) atomicMin(&st.best, bidx);
        if (maxd) atomicMax(&st.maxd, maxd);
        if (low) atomicAdd(&st.settled, low);
    }
}

// Walk-back from the best target to a start over the exact field, one warp per search. At each state q: stop if q
// is a start at its own start cost; else step to the first predecessor p, in the order moves 0-7 then via layers
// ascending (the router's walk-back order, src/router.cpp:1615-1679), with d(p) + w(p -> q) == d(q). Every state
// on the walk has d <= d(best), where the field is exact, so the walk is the oracle's. Lanes 0-7 test the moves,
// 8-15 the via layers, 16-31 the start list.
template <typename DT>
__global__ void walkback_kernel(const SDev* Sv, const SStat* stv, const uint32_t* const* sidx, const uint64_t* const* sd,
                                const int* ns) {
    const int s = blockIdx.x, lane = threadIdx.x;
    const SDev& S = Sv[s];
    if (!S.path) return;
    const SStat& st = stv[s];
    const DT INF = Lim<DT>::INF;
    if (st.best == ~0ull || st.ub >= static_cast<unsigned long long>(INF)) {
        if (lane == 0) *S.path_len = 0;
        return;
    }
    const int MX[8] = {1, -1, 0, 0, 1, 1, -1, -1}, MY[8] = {0, 0, 1, -1, 1, -1, 1, -1};
    const DT* dist = reinterpret_cast<const DT*>(S.dist);
    const size_t RN = size_t(S.rw) * S.rh;
    auto at = [&](int l, int j, int i) { return (size_t(l) * S.hpad + j) * S.pitch + i; };
    unsigned long long q = st.best;
    int n = 0, result = -1;
    for (; n < S.path_cap; ++n) {
        const int l = int(q / RN), rem = int(q % RN), j = rem / S.rw, i = rem % S.rw;
        const size_t pq = at(l, j, i);
        const DT dq = dist[pq];
        if (lane == 0) S.path[n] = uint32_t(q);
        bool hit = false, start = false;
        unsigned long long cand = 0;
        if (lane < 8) {
            const int pi = i - MX[lane], pj = j - MY[lane];
            if (pi >= 0 && pj >= 0 && pi < S.rw && pj < S.rh) {
                const DT w = qweight<DT>(S.cf[pq], S.fac[l][lane]);
                const DT dp = dist[at(l, pj, pi)];
                hit = w < INF && dp < INF && dp + w == dq;
                cand = size_t(l) * RN + size_t(pj) * S.rw + pi;
            }
        } else if (lane < 16) {
            const int l2 = lane - 8;
            if (S.vcf && l2 < S.nl && l2 != l && (S.fl[pq] & 1)) {
                const DT w = qweight<DT>(S.vcf[size_t(j) * S.pitch + i], 1.0f);
                const DT dp = dist[at(l2, j, i)];
                hit = w < INF && dp < INF && dp + w == dq;
                cand = size_t(l2) * RN + size_t(j) * S.rw + i;
            }
        } else {
            for (int k = lane - 16; k < ns[s]; k += 16)
                if (sidx[s][k] == uint32_t(q) && sd[s][k] < uint64_t(INF) && DT(sd[s][k]) == dq) start = true;
        }
        if (__any_sync(0xFFFFFFFFu, start)) { result = n + 1; break; }
        const unsigned b = __ballot_sync(0xFFFFFFFFu, hit);
        if (!b) break;
        q = __shfl_sync(0xFFFFFFFFu, cand, __ffs(b) - 1);
    }
    if (lane == 0) *S.path_len = result;
}

// ---- device arena (grow-only; all batch solves are serialised by g_mu) ----

std::mutex g_mu;

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    bool need(size_t n) {
        if (cap >= n) return true;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t c = n + n / 8 + 256;
        if (cudaMalloc(&p, c) != cudaSuccess) { p = nullptr; return false; }
        cap = c;
        return true;
    }
};

struct Arena {
    DevBuf dist, stamp, tkey, wl, vl, sdev, sstat, ctl, visits, sptr;
} g_arena;

// Round cap of a launch: a bound on the device loop, which tests lower (pcbg_set_max_rounds, or PCBG_MAX_ROUNDS in
// the environment of a process such as the router) to see a launch stop with ERR_ROUNDS and its caller fall back.
int max_rounds_from_env() {
    const char* e = std::getenv("PCBG_MAX_ROUNDS");
    const int v = e ? std::atoi(e) : 0;
    return v >= 1 ? v : (1 << 20);
}
int g_max_rounds = max_rounds_from_env();

// Order of an ordered round's visit list (ORDER_*): pcbg_set_visit_order, or PCBG_VISIT_ORDER in the environment.
// Default: the searches with the most layers first. Their visits take longest, and a round ends when its last visit
// does, so taking them first leaves the short visits to fill the end of the round (longest-first list scheduling).
int visit_order_from_env() {
    const char* e = std::getenv("PCBG_VISIT_ORDER");
    const int v = e ? std::atoi(e) : -1;
    return v >= ORDER_FIFO && v <= ORDER_LAYERS ? v : ORDER_LAYERS;
}
int g_order = visit_order_from_env();

thread_local std::string t_err;
thread_local BatchStats t_stats;
cudaEvent_t g_ev0 = nullptr, g_ev1 = nullptr;

// pinned host staging of a batch's descriptors and results (batches are serialised by g_mu)
struct HostStage {
    unsigned char* p = nullptr;
    size_t cap = 0;
} g_hstage;

bool host_stage(size_t n) {
    if (g_hstage.cap >= n) return true;
    if (g_hstage.p) cudaFreeHost(g_hstage.p);
    g_hstage.p = nullptr;
    g_hstage.cap = 0;
    const size_t c = n + n / 2 + 4096;
    if (cudaHostAlloc(reinterpret_cast<void**>(&g_hstage.p), c, cudaHostAllocDefault) != cudaSuccess) return false;
    g_hstage.cap = c;
    return true;
}

template <typename DT, int MINB> int blocks_per_sm(size_t smem) {
    if (cudaFuncSetAttribute(relax_kernel<DT, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
        return -1;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, relax_kernel<DT, MINB>, NT, smem) != cudaSuccess) return -1;
    return per_sm;
}

// The relax kernel build for a launch over `tiles` tiles with `smem` bytes of dynamic shared memory, and how many of
// its blocks are resident on the device at once (<= 0: none can be). The 3-block build pays only when rounds queue
// far more tiles than blocks: a batch of at least 16 tiles per resident block (a 512-search wave of the
// microbenchmark has about 170 K tiles; one search or a speculative round a few thousand at most).
struct RelaxLaunch {
    void* fn;
    int resident;
};
int sm_count() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms > 0 ? sms : 1;
}

// minb: the build asked for (3 or 2 blocks per SM; 0: the untuned rule, 3 for batches of at least 16 tiles per
// resident block). A 3-block build whose shared memory does not fit 3 blocks falls back to the 2-block one.
template <typename DT> RelaxLaunch relax_launch(size_t smem, size_t tiles, int minb = 0) {
    const int sms = sm_count();
    if (minb == 3 || (minb == 0 && tiles >= size_t(16) * 3 * sms)) {
        const int p3 = blocks_per_sm<DT, 3>(smem);
        if (p3 >= 3) return {reinterpret_cast<void*>(relax_kernel<DT, 3>), p3 * sms};
    }
    const int p2 = blocks_per_sm<DT, 2>(smem);
    return {reinterpret_cast<void*>(relax_kernel<DT, 2>), p2 < 0 ? -1 : p2 * sms};
}

// ---- relaxation schedules: the round band and the kernel build of a launch, per layer-count class (1-2, 3-4, 5-6,
// 7-8 layers) and batch class (fewer, or at least, 16 tiles per resident block of the 3-block build)

struct Schedule {
    int band;
    int minb;
};
struct TuneTable {
    bool set[4][2] = {};
    Schedule s[4][2];
    float ms[4][2];
    float ms_untuned[4][2];
};
TuneTable g_tune;
int g_band_user = -1;                 // pcbg_set_round_band: one band for every launch (-1: tuned or default)
constexpr int DEFAULT_BAND = 16;    // the band the untuned rule of the first ordered kernel used (reported as "untuned")
const Schedule* g_force = nullptr;    // the autotuner's candidate while it times one

int layer_class(int nl) { return std::min(3, std::max(0, (nl - 1) / 2)); }
int size_class(size_t tiles) { return tiles >= size_t(16) * 3 * sm_count() ? 1 : 0; }

// Before (or without) a tuning run: what the tuner chose on a B200 for most classes: small batches unordered on the
// 2-block build, large ones with a band of 32.
Schedule schedule_for(int nl, size_t tiles) {
    if (g_force) return *g_force;
    Schedule sc = size_class(tiles) ? Schedule{32, 0} : Schedule{0, 2};
    if (g_tune.set[layer_class(nl)][size_class(tiles)]) sc = g_tune.s[layer_class(nl)][size_class(tiles)];
    if (g_band_user >= 0) sc.band = g_band_user;
    return sc;
}

// joint mode needs one factor per move class on every layer (true of every query the router builds)
void classify(SDev& S) {
    bool ok = true, xy = true;
    for (int l = 0; l < S.nl; ++l) {
        const float* f = S.fac[l];
        ok &= f[0] == f[1] && f[2] == f[3] && f[4] == f[5] && f[4] == f[6] && f[4] == f[7];
        xy &= f[0] == f[2];
    }
    S.mode = ok ? 1 : 0;
    S.K = xy ? 2 : 3;
    S.plane_h = 0;
    S.plane_v = xy ? 0 : 1;
    S.plane_d = S.K - 1;
}

// Solve items[idx[0..m)] with DT distances.
void init_stat(SStat& x) {
    x.ub = ~0ull; x.maxw = 0; x.best = ~0ull; x.maxd = 0; x.need_wide = 0;
    x.wscale = KEY_NONE; x.kmin[0] = x.kmin[1] = x.kmin[2] = KEY_NONE; x.settled = 0;
}

template <typename DT>
int run_batch(BatchItem* items, const std::vector<int>& idx, cudaStream_t stream, BatchStats& bs, int band) {
    const int m = int(idx.size());
    std::vector<SDev> sd(m);
    std::vector<size_t> doff(m), toff(m);
    size_t dbytes = 0, tiles = 0;
    int nlmax = 1, kmax = 0;
    bool any_general = false, any_path = false;
    for (int k = 0; k < m; ++k) {
        const BatchItem& b = items[idx[k]];
        SDev& S = sd[k];
        memset(&S, 0, sizeof(S));
        S.rw = b.rw; S.rh = b.rh; S.nl = b.nl; S.pitch = b.pitch; S.hpad = b.hpad;
        S.ntx = b.pitch / TILE; S.nty = b.hpad / TILE;
        for (int l = 0; l < MAX_LAYERS; ++l) {
            float mf = 0.f;
            for (int d = 0; d < 8; ++d) { S.fac[l][d] = b.fac[l][d]; if (l < b.nl) mf = std::max(mf, b.fac[l][d]); }
            S.maxfac[l] = mf;
        }
        classify(S);
        if (sizeof(DT) != 4) S.mode = 0;
        if (S.mode) kmax = std::max(kmax, S.K);
        else any_general = true;
        S.cf = b.cf; S.fl = b.fl; S.vcf = b.vcf; S.out = b.out;
        S.path = b.path; S.path_len = b.path_len; S.path_cap = b.path_cap;
        if (b.path) any_path = true;
        doff[k] = dbytes;
        dbytes += round_up(size_t(b.nl) * b.hpad * b.pitch * sizeof(DT), 256);
        toff[k] = tiles;
        tiles += size_t(S.ntx) * S.nty;
        nlmax = std::max(nlmax, b.nl);
    }
    size_t smem = 0;
    if (kmax) smem = std::max(smem, layout(nlmax, joint_wbytes(kmax), 4).total);
    if (any_general) smem = std::max(smem, layout(nlmax, 4, sizeof(DT)).total);
    Arena& A = g_arena;
    const unsigned int cap = unsigned(std::max<size_t>(tiles, 1));
    if (!A.dist.need(dbytes) || !A.stamp.need(tiles * 8 + 8) || !A.tkey.need(tiles * 4 + 4) ||
        !A.wl.need(size_t(3) * cap * 8) || !A.vl.need(size_t(cap) * 8) ||
        !A.sdev.need(sizeof(SDev) * m) || !A.sstat.need(sizeof(SStat) * m) || !A.ctl.need(C_N * 4) ||
        !A.visits.need(NVIS * 8) || !A.sptr.need(size_t(m) * (8 + 8 + 4) + 64)) {
        t_err = "device allocation failed";
        return -1;
    }
    for (int k = 0; k < m; ++k) {
        sd[k].dist = static_cast<unsigned char*>(A.dist.p) + doff[k];
        sd[k].stamp = static_cast<uint32_t*>(A.stamp.p) + toff[k];
        sd[k].sides = static_cast<uint32_t*>(A.stamp.p) + tiles + toff[k];
        sd[k].tkey = static_cast<uint32_t*>(A.tkey.p) + toff[k];
    }
    // the batch's descriptors, initial stats and start lists go up from pinned staging (asynchronous copies; a copy
    // from pageable memory would go through the driver's bounce buffer one call at a time)
    const size_t h_sd = 0, h_st = round_up(sizeof(SDev) * m, 16), h_sp = h_st + round_up(sizeof(SStat) * m, 16);
    const size_t h_res = h_sp + round_up(size_t(m) * 20, 16), h_ctl = h_res + round_up(sizeof(SStat) * m, 16);
    const size_t h_vis = h_ctl + round_up(C_N * 4, 16), h_end = h_vis + NVIS * 8;
    if (!host_stage(h_end)) { t_err = "pinned allocation failed"; return -1; }
    unsigned char* hs = g_hstage.p;
    memcpy(hs + h_sd, sd.data(), sizeof(SDev) * m);
    SStat* st0 = reinterpret_cast<SStat*>(hs + h_st);
    for (int k = 0; k < m; ++k) {
        init_stat(st0[k]);
        reinterpret_cast<const uint32_t**>(hs + h_sp)[k] = items[idx[k]].start_idx;
        reinterpret_cast<const uint64_t**>(hs + h_sp + size_t(m) * 8)[k] = items[idx[k]].start_d;
        reinterpret_cast<int*>(hs + h_sp + size_t(m) * 16)[k] = items[idx[k]].n_starts;
    }
    unsigned char* sp = static_cast<unsigned char*>(A.sptr.p);
    const uint32_t* const* d_sip = reinterpret_cast<const uint32_t* const*>(sp);
    const uint64_t* const* d_sdp = reinterpret_cast<const uint64_t* const*>(sp + size_t(m) * 8);
    const int* d_ns = reinterpret_cast<const int*>(sp + size_t(m) * 16);
    cudaMemcpyAsync(A.sdev.p, hs + h_sd, sizeof(SDev) * m, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(A.sstat.p, hs + h_st, sizeof(SStat) * m, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(sp, hs + h_sp, size_t(m) * 20, cudaMemcpyHostToDevice, stream);
    cudaMemsetAsync(A.dist.p, 0x7F, dbytes, stream);
    cudaMemsetAsync(A.stamp.p, 0, tiles * 8 + 8, stream);
    cudaMemsetAsync(A.tkey.p, 0xFF, tiles * 4 + 4, stream);
    cudaMemsetAsync(A.ctl.p, 0, C_N * 4, stream);
    cudaMemsetAsync(A.visits.p, 0, NVIS * 8, stream);
    SolveArgs a;
    a.S = static_cast<const SDev*>(A.sdev.p);
    a.st = static_cast<SStat*>(A.sstat.p);
    a.n = m;
    a.nlmax = nlmax;
    a.kmax = kmax;
    a.wl = static_cast<unsigned long long*>(A.wl.p);
    a.vl = static_cast<unsigned long long*>(A.vl.p);
    a.cap = cap;
    a.ctl = static_cast<unsigned int*>(A.ctl.p);
    a.visits = static_cast<unsigned long long*>(A.visits.p);
    const Schedule sc = schedule_for(nlmax, tiles);
    if (sizeof(DT) != 4) band = 0;
    else if (band < 0) band = sc.band;
    a.max_rounds = g_max_rounds;
    a.band = unsigned(band);
    a.ordered = band > 0 ? 1 : 0;
    a.order = g_order;
    seed_kernel<DT><<<m, 128, 0, stream>>>(a, d_sip, d_sdp, d_ns);
    const RelaxLaunch R = relax_launch<DT>(smem, tiles, sc.minb);
    bs.band = band;
    bs.blocks_per_sm = R.resident / sm_count();
    if (R.resident <= 0) { t_err = "relax kernel cannot be resident"; return -1; }
    // a round visits each queued tile once: more blocks than tiles would only wait at the grid barriers
    const int blocks = int(std::min<size_t>(size_t(R.resident), std::max<size_t>(tiles, 1)));
    void* args[] = {&a};
    if (!g_ev0) { cudaEventCreate(&g_ev0); cudaEventCreate(&g_ev1); }
    cudaEventRecord(g_ev0, stream);
    cudaError_t e = cudaLaunchCooperativeKernel(R.fn, dim3(blocks), dim3(NT), args, smem, stream);
    if (e != cudaSuccess) { t_err = std::string("cooperative launch: ") + cudaGetErrorString(e); return -1; }
    cudaEventRecord(g_ev1, stream);
    report_kernel<DT><<<dim3(32, m), 256, 0, stream>>>(a.S, a.st);
    bs.launches += 3;
    if (any_path) {
        walkback_kernel<DT><<<m, 32, 0, stream>>>(a.S, a.st, d_sip, d_sdp, d_ns);
        bs.launches += 1;
    }
    const SStat* st = reinterpret_cast<const SStat*>(hs + h_res);
    const unsigned int* ctl = reinterpret_cast<const unsigned int*>(hs + h_ctl);
    const unsigned long long* visits = reinterpret_cast<const unsigned long long*>(hs + h_vis);
    cudaMemcpyAsync(hs + h_res, A.sstat.p, sizeof(SStat) * m, cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(hs + h_ctl, A.ctl.p, C_N * 4, cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(hs + h_vis, A.visits.p, NVIS * 8, cudaMemcpyDeviceToHost, stream);
    e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) { t_err = std::string("batch solve: ") + cudaGetErrorString(e); return -1; }
    if (ctl[C_ERR]) {
        t_err = "batch solve aborted (error bits " + std::to_string(ctl[C_ERR]) + ")";
        return -1;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g_ev0, g_ev1);
    bs.kernel_ms += ms;
    bs.rounds += int(ctl[C_ROUNDS]);
    bs.tile_visits += (long long)visits[0];
    bs.layer_visits += (long long)visits[1];
    bs.local_iters += (long long)visits[2];
    bs.deferred += (long long)visits[3];
    bs.dropped += (long long)visits[4];
    bs.busy_cycles += (long long)visits[5];
    bs.block_cycles += (long long)visits[6];
    const int rounds_out = int(ctl[C_ROUNDS]);
    const unsigned long long INF = static_cast<unsigned long long>(Lim<DT>::INF);
    for (int k = 0; k < m; ++k) {
        BatchItem& b = items[idx[k]];
        const SStat& x = st[k];
        const bool have = x.ub < INF;
        b.best = have && x.best != ~0ull ? int64_t(x.best) : -1;
        b.best_d = have ? x.ub : INF64;
        b.rounds = rounds_out;
        // exactness of 32-bit arithmetic: a dropped weight or sum matters only if nothing at or below it was found
        bool redo = false;
        if (sizeof(DT) == 4) {
            if (x.need_wide && (!have || x.ub >= static_cast<unsigned long long>(WLIM32))) redo = true;
            if (!have && x.maxd + x.maxw >= INF) redo = true;
        }
        b.status = redo ? 1 : 0;
        if (!redo) bs.settled += x.settled;
    }
    return 0;
}

}  // namespace

void set_error(const std::string& s) { t_err = s; }
const std::string& last_error() { return t_err; }
BatchStats& last_stats() { return t_stats; }

int solve_batch_locked(BatchItem* items, int n, cudaStream_t stream);

int solve_batch(BatchItem* items, int n, cudaStream_t stream) {
    std::lock_guard<std::mutex> g(g_mu);
    return solve_batch_locked(items, n, stream);
}

int solve_batch_locked(BatchItem* items, int n, cudaStream_t stream) {
    t_stats = BatchStats{};
    if (n <= 0) return 0;
    for (int k = 0; k < n; ++k) {
        const BatchItem& b = items[k];
        if (b.nl < 1 || b.nl > MAX_LAYERS || b.rw < 1 || b.rh < 1 || b.pitch % TILE || b.hpad % TILE || b.pitch < b.rw ||
            b.hpad < b.rh) {
            t_err = "bad search geometry";
            return -1;
        }
    }
    std::vector<int> all(n);
    for (int k = 0; k < n; ++k) all[k] = k;
    if (run_batch<uint32_t>(items, all, stream, t_stats, -1) != 0) return -1;
    std::vector<int> wide;
    for (int k = 0; k < n; ++k)
        if (items[k].status == 1) wide.push_back(k);
    if (!wide.empty()) {
        if (run_batch<uint64_t>(items, wide, stream, t_stats, 0) != 0) return -1;
        for (int k : wide) items[k].status = 1;
    }
    return 0;
}

}  // namespace pcbg

// ---- C ABI: batched device searches ----

extern "C" int pcbg_solve_batch(pcbg_search* s, int32_t n, void* stream) {
    std::vector<pcbg::BatchItem> it(n > 0 ? n : 0);
    for (int k = 0; k < n; ++k) {
        pcbg::BatchItem& b = it[k];
        const pcbg_search& q = s[k];
        b.rw = q.rw; b.rh = q.rh; b.nl = q.nl; b.pitch = q.pitch; b.hpad = q.hpad;
        memcpy(b.fac, q.fac, sizeof(b.fac));
        b.cf = q.cf; b.fl = q.flags; b.vcf = q.vcf;
        b.start_idx = q.start_idx; b.start_d = q.start_d; b.n_starts = q.n_starts;
        b.out = q.out;
        b.path = q.path; b.path_cap = q.path_cap; b.path_len = q.path_len;
    }
    const int r = pcbg::solve_batch(it.data(), n, static_cast<cudaStream_t>(stream));
    if (r != 0) return PCBG_ERR_FAIL;
    for (int k = 0; k < n; ++k) {
        s[k].best = it[k].best;
        s[k].best_d = it[k].best_d;
        s[k].status = it[k].status;
        s[k].rounds = it[k].rounds;
    }
    return 0;
}

extern "C" int64_t pcbg_last_batch_tile_visits(void) { return pcbg::last_stats().tile_visits; }
extern "C" int32_t pcbg_last_batch_rounds(void) { return pcbg::last_stats().rounds; }
extern "C" int64_t pcbg_last_batch_layer_visits(void) { return pcbg::last_stats().layer_visits; }
extern "C" float pcbg_last_batch_kernel_ms(void) { return pcbg::last_stats().kernel_ms; }
extern "C" int32_t pcbg_last_batch_launches(void) { return pcbg::last_stats().launches; }
extern "C" int64_t pcbg_last_batch_local_iters(void) { return pcbg::last_stats().local_iters; }
extern "C" int64_t pcbg_last_batch_deferred(void) { return pcbg::last_stats().deferred; }
extern "C" int64_t pcbg_last_batch_dropped(void) { return pcbg::last_stats().dropped; }
extern "C" int64_t pcbg_last_batch_settled(void) { return pcbg::last_stats().settled; }
extern "C" float pcbg_last_batch_busy_frac(void) {
    const pcbg::BatchStats& b = pcbg::last_stats();
    return b.block_cycles > 0 ? float(double(b.busy_cycles) / double(b.block_cycles)) : 0.f;
}
extern "C" void pcbg_set_visit_order(int32_t order) {
    std::lock_guard<std::mutex> g(pcbg::g_mu);
    pcbg::g_order = order >= pcbg::ORDER_FIFO && order <= pcbg::ORDER_LAYERS ? order : pcbg::ORDER_LAYERS;
}
extern "C" int32_t pcbg_visit_order(void) {
    std::lock_guard<std::mutex> g(pcbg::g_mu);
    return pcbg::g_order;
}

extern "C" void pcbg_set_round_band(int32_t band) {
    std::lock_guard<std::mutex> g(pcbg::g_mu);
    pcbg::g_band_user = band < 0 ? -1 : band;
}
extern "C" int32_t pcbg_round_band(void) { return pcbg::last_stats().band; }
extern "C" int32_t pcbg_last_batch_blocks_per_sm(void) { return pcbg::last_stats().blocks_per_sm; }

extern "C" void pcbg_set_max_rounds(int32_t rounds) {
    std::lock_guard<std::mutex> g(pcbg::g_mu);
    pcbg::g_max_rounds = rounds < 1 ? (1 << 20) : rounds;
}

// ---- pcbg_solve_noalloc: one search with all scratch in a static device array ----
//
// For callers that cannot allocate device memory. Everything the batch path takes from its grow-only arena
// (distances, tile stamps, keys, worklists, descriptors, control words) is carved here from one file-scope array of
// fixed size instead, and the host side uses only stack storage.

static __device__ __align__(256) unsigned char pcbg_noalloc_scratch[
    PCBG_NOALLOC_MAX_STATES * 8 +                                                  // distances, room for 64-bit
    (PCBG_NOALLOC_MAX_STATES / (pcbg::TILE * pcbg::TILE)) * (8 + 4 + 3 * 8 + 8) +  // tile stamps + sides, keys,
                                                                                   // 3 worklists, visit list
    4096];                                                                          // descriptors, control words

namespace pcbg {
namespace {

constexpr size_t NA_TILES = PCBG_NOALLOC_MAX_STATES / (TILE * TILE);
constexpr size_t NA_DIST = size_t(PCBG_NOALLOC_MAX_STATES) * 8;
constexpr size_t NA_STAMP = NA_DIST;                       // stamps, then sides
constexpr size_t NA_TKEY = NA_STAMP + NA_TILES * 8;
constexpr size_t NA_WL = NA_TKEY + NA_TILES * 4;
constexpr size_t NA_VL = NA_WL + NA_TILES * 3 * 8;
constexpr size_t NA_SMALL = NA_VL + NA_TILES * 8;
// offsets in the small area after the lists
constexpr size_t NA_SDEV = 0, NA_SSTAT = 1024, NA_CTL = 1088, NA_VIS = 1168, NA_SPTR = 1232;
static_assert(sizeof(SDev) <= NA_SSTAT - NA_SDEV && sizeof(SStat) <= NA_CTL - NA_SSTAT &&
              C_N * 4 <= NA_VIS - NA_CTL && NVIS * 8 <= NA_SPTR - NA_VIS && NA_SPTR + 24 <= 4096,
              "no-alloc small area layout");
static_assert(NA_SMALL + 4096 == sizeof(pcbg_noalloc_scratch), "no-alloc scratch layout");

std::mutex g_na_mu;
void* g_na_base[64] = {};

// error text without heap allocation: the thread's message buffer is reserved during set-up
void na_error(const char* fmt, const char* a = "", long long x = 0, long long y = 0) {
    char buf[200];
    snprintf(buf, sizeof(buf), fmt, a, x, y);
    t_err.assign(buf);
}

// device address of the static scratch on the current device (looked up once per device)
unsigned char* na_base() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) { na_error("no current device%s"); return nullptr; }
    std::lock_guard<std::mutex> g(g_na_mu);
    if (!g_na_base[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, pcbg_noalloc_scratch);
        if (e != cudaSuccess || !p) { na_error("cudaGetSymbolAddress: %s", cudaGetErrorString(e)); return nullptr; }
        g_na_base[dev] = p;
    }
    return static_cast<unsigned char*>(g_na_base[dev]);
}

template <typename DT>
int na_run(pcbg_search* q, unsigned char* base, cudaStream_t stream, int band, int minb) {
    SDev S;
    memset(&S, 0, sizeof(S));
    S.rw = q->rw; S.rh = q->rh; S.nl = q->nl; S.pitch = q->pitch; S.hpad = q->hpad;
    S.ntx = q->pitch / TILE; S.nty = q->hpad / TILE;
    for (int l = 0; l < MAX_LAYERS; ++l) {
        float mf = 0.f;
        for (int d = 0; d < 8; ++d) { S.fac[l][d] = q->fac[l][d]; if (l < q->nl) mf = std::max(mf, q->fac[l][d]); }
        S.maxfac[l] = mf;
    }
    classify(S);
    if (sizeof(DT) != 4) S.mode = 0;
    S.cf = q->cf; S.fl = q->flags; S.vcf = q->vcf; S.out = q->out;
    S.path = q->path; S.path_len = q->path_len; S.path_cap = q->path_cap;
    const size_t states = size_t(q->nl) * q->hpad * q->pitch, tiles = size_t(S.ntx) * S.nty;
    // the launch shape first: nothing is queued on the stream unless the relaxation can be launched
    const size_t smem = S.mode ? layout(q->nl, joint_wbytes(S.K), 4).total : layout(q->nl, 4, sizeof(DT)).total;
    const RelaxLaunch R = relax_launch<DT>(smem, tiles, minb);
    if (R.resident <= 0) { na_error("relax kernel cannot be resident%s"); return -1; }
    // a round visits each queued tile once: more blocks than tiles would only wait at the grid barriers
    const int blocks = int(std::min<size_t>(size_t(R.resident), std::max<size_t>(tiles, 1)));
    unsigned char* small = base + NA_SMALL;
    S.dist = base;
    S.stamp = reinterpret_cast<uint32_t*>(base + NA_STAMP);
    S.sides = S.stamp + NA_TILES;
    S.tkey = reinterpret_cast<uint32_t*>(base + NA_TKEY);
    SStat st0;
    init_stat(st0);
    const void* sptr[2] = {q->start_idx, q->start_d};
    const int ns = q->n_starts;
    cudaMemcpyAsync(small + NA_SDEV, &S, sizeof(S), cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(small + NA_SSTAT, &st0, sizeof(st0), cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(small + NA_SPTR, sptr, sizeof(sptr), cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(small + NA_SPTR + 16, &ns, sizeof(ns), cudaMemcpyHostToDevice, stream);
    // the array keeps the previous call's contents: clear what must start unreached / zero / keyless
    cudaMemsetAsync(base, 0x7F, states * sizeof(DT), stream);
    cudaMemsetAsync(base + NA_STAMP, 0, tiles * 4, stream);
    cudaMemsetAsync(base + NA_STAMP + NA_TILES * 4, 0, tiles * 4, stream);
    cudaMemsetAsync(base + NA_TKEY, 0xFF, tiles * 4, stream);
    cudaMemsetAsync(small + NA_CTL, 0, C_N * 4, stream);
    cudaMemsetAsync(small + NA_VIS, 0, NVIS * 8, stream);
    SolveArgs a;
    a.S = reinterpret_cast<const SDev*>(small + NA_SDEV);
    a.st = reinterpret_cast<SStat*>(small + NA_SSTAT);
    a.n = 1;
    a.nlmax = q->nl;
    a.kmax = S.mode ? S.K : 0;
    a.wl = reinterpret_cast<unsigned long long*>(base + NA_WL);
    a.vl = reinterpret_cast<unsigned long long*>(base + NA_VL);
    a.cap = unsigned(tiles);
    a.ctl = reinterpret_cast<unsigned int*>(small + NA_CTL);
    a.visits = reinterpret_cast<unsigned long long*>(small + NA_VIS);
    a.max_rounds = g_max_rounds;
    a.band = unsigned(band);
    a.ordered = sizeof(DT) == 4 && band > 0 ? 1 : 0;
    a.order = g_order;
    const uint32_t* const* sip = reinterpret_cast<const uint32_t* const*>(small + NA_SPTR);
    const uint64_t* const* sdp = reinterpret_cast<const uint64_t* const*>(small + NA_SPTR + 8);
    const int* nsp = reinterpret_cast<const int*>(small + NA_SPTR + 16);
    seed_kernel<DT><<<1, 128, 0, stream>>>(a, sip, sdp, nsp);
    void* args[] = {&a};
    cudaError_t e = cudaLaunchCooperativeKernel(R.fn, dim3(blocks), dim3(NT), args, smem, stream);
    if (e != cudaSuccess) {
        // the copies, clears and seeds queued above must be done before another call can reuse the array
        cudaStreamSynchronize(stream);
        na_error("cooperative launch: %s", cudaGetErrorString(e));
        return -1;
    }
    report_kernel<DT><<<dim3(32, 1), 256, 0, stream>>>(a.S, a.st);
    if (q->path) walkback_kernel<DT><<<1, 32, 0, stream>>>(a.S, a.st, sip, sdp, nsp);
    SStat x;
    unsigned int ctl[C_N];
    cudaMemcpyAsync(&x, small + NA_SSTAT, sizeof(x), cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(ctl, small + NA_CTL, sizeof(ctl), cudaMemcpyDeviceToHost, stream);
    e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) { na_error("no-alloc solve: %s", cudaGetErrorString(e)); return -1; }
    if (ctl[C_ERR]) { na_error("no-alloc solve aborted (error bits %s%lld)", "", (long long)ctl[C_ERR]); return -1; }
    const unsigned long long INF = static_cast<unsigned long long>(Lim<DT>::INF);
    const bool have = x.ub < INF;
    q->best = have && x.best != ~0ull ? int64_t(x.best) : -1;
    q->best_d = have ? x.ub : INF64;
    q->rounds = int(ctl[C_ROUNDS]);
    bool redo = false;
    if (sizeof(DT) == 4) {
        if (x.need_wide && (!have || x.ub >= static_cast<unsigned long long>(WLIM32))) redo = true;
        if (!have && x.maxd + x.maxw >= INF) redo = true;
    }
    q->status = redo ? 1 : 0;
    return 0;
}

}  // namespace
}  // namespace pcbg

extern "C" int pcbg_solve_noalloc(pcbg_search* s, void* stream) {
    using namespace pcbg;
    if (t_err.capacity() < 256) t_err.reserve(256);  // set-up, first call on this thread
    if (!s || s->nl < 1 || s->nl > MAX_LAYERS || s->rw < 1 || s->rh < 1 || s->pitch % TILE || s->hpad % TILE ||
        s->pitch < s->rw || s->hpad < s->rh) {
        na_error("bad search geometry%s");
        return PCBG_ERR_FAIL;
    }
    const size_t states = size_t(s->nl) * s->hpad * s->pitch;
    if (states > size_t(PCBG_NOALLOC_MAX_STATES)) {
        na_error("search of %s%lld padded states exceeds the no-alloc limit of %lld states", "", (long long)states,
                 (long long)PCBG_NOALLOC_MAX_STATES);
        return PCBG_ERR_FAIL;
    }
    unsigned char* base = na_base();
    if (!base) return PCBG_ERR_FAIL;
    std::lock_guard<std::mutex> g(g_mu);  // one solve at a time in this process: calls share the array
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const Schedule sc = schedule_for(s->nl, size_t(s->pitch / TILE) * (s->hpad / TILE));
    if (na_run<uint32_t>(s, base, st, sc.band, sc.minb) != 0) return PCBG_ERR_FAIL;
    if (s->status == 1) {
        if (na_run<uint64_t>(s, base, st, 0, sc.minb) != 0) return PCBG_ERR_FAIL;
        s->status = 1;
    }
    return 0;
}

// ---- the schedule autotuner ----
//
// For each layer-count class (searches of 2, 4, 6, 8 layers) and batch class (two searches of 1024 x 768, the size
// of a router's few concurrent searches; and enough 512 x 512 searches for at least 16 tiles per resident block, a
// round of the batched microbenchmark), the seeded generator's searches are solved under every schedule: round
// band 0 (every queued tile each round), 8, 16, 32, 64, 128 weight scales, and the 2- and 3-blocks-per-SM builds. The
// fastest relaxation (least device time of two launches) becomes the class's schedule for every later launch.
// Results never depend on the schedule; only the time does.

extern "C" int32_t pcbg_autotune(void* stream, pcbg_tune_entry* out, int32_t cap) {
    using namespace pcbg;
    std::lock_guard<std::mutex> g(g_mu);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int sms = sm_count();
    const int bands[] = {0, 8, 16, 32, 64, 128};
    const int nls[4] = {2, 4, 6, 8};
    TuneTable T;
    int written = 0;
    for (int lc = 0; lc < 4; ++lc)
        for (int sc = 0; sc < 2; ++sc) {
            const int nl = nls[lc];
            const int rw = sc ? 512 : 1024, rh = sc ? 512 : 768;
            const int n = sc ? int((size_t(16) * 3 * sms + 255) / 256 * 11 / 10) : 2;
            const size_t plane = size_t(rw) * rh, PN = plane * nl;
            // one allocation: per search cf, flags, vcf, the generator's source / target, the start cost
            const size_t per = PN * 4 + PN + plane * 4 + 16 + 16;
            unsigned char* buf = nullptr;
            if (cudaMalloc(&buf, per * n) != cudaSuccess) { set_error("autotune allocation failed"); return PCBG_ERR_FAIL; }
            std::vector<BatchItem> items(n);
            bool ok = true;
            for (int k = 0; k < n && ok; ++k) {
                unsigned char* b = buf + per * k;
                float* cf = reinterpret_cast<float*>(b);
                uint8_t* fl = b + PN * 4;
                float* vcf = reinterpret_cast<float*>(b + PN * 5);
                int64_t* stt = reinterpret_cast<int64_t*>(b + PN * 5 + plane * 4);
                uint64_t* sd = reinterpret_cast<uint64_t*>(stt + 2);
                ok = pcbg_synth_search(0xA0707E00ull + 97 * k + lc * 7 + sc, rw, rh, nl, rw, rh, 8.0f + float(k % 25),
                                       cf, fl, vcf, stt, st) == 0;
                cudaMemsetAsync(sd, 0, 8, st);
                BatchItem& it = items[k];
                memset(&it, 0, sizeof(it));
                it.rw = rw; it.rh = rh; it.nl = nl; it.pitch = rw; it.hpad = rh;
                for (int l = 0; l < MAX_LAYERS; ++l)
                    for (int m = 0; m < 8; ++m) it.fac[l][m] = m < 4 ? 1.0f : 1.41421354f;
                it.cf = cf; it.fl = fl; it.vcf = vcf;
                // the start: the generator's source, a rect state in the low word of its int64 (little endian); a
                // source that could not be placed (-1) is beyond the search and seeds nothing
                it.start_idx = reinterpret_cast<const uint32_t*>(stt);
                it.start_d = sd;
                it.n_starts = 1;
            }
            if (!ok || cudaStreamSynchronize(st) != cudaSuccess) {
                cudaFree(buf);
                set_error("autotune search generation failed");
                return PCBG_ERR_FAIL;
            }
            float best_ms = 1e30f, untuned_ms = 1e30f;
            Schedule best{DEFAULT_BAND, 0};
            for (int band : bands)
                for (int minb = 2; minb <= 3; ++minb) {
                    const Schedule cand{band, minb};
                    g_force = &cand;
                    float ms = 1e30f;
                    for (int rep = 0; rep < 2; ++rep) {
                        if (solve_batch_locked(items.data(), n, st) != 0) { ms = 1e30f; break; }
                        ms = std::min(ms, t_stats.kernel_ms);
                    }
                    g_force = nullptr;
                    if (ms < best_ms) { best_ms = ms; best = cand; }
                    if (band == DEFAULT_BAND && minb == (sc ? 3 : 2)) untuned_ms = ms;
                }
            cudaFree(buf);
            T.s[lc][sc] = best;
            T.set[lc][sc] = true;
            T.ms[lc][sc] = best_ms;
            T.ms_untuned[lc][sc] = untuned_ms;
            if (out && written < cap) {
                pcbg_tune_entry& e = out[written++];
                e.layers_lo = 2 * lc + 1; e.layers_hi = 2 * lc + 2; e.batch_class = sc;
                e.band = best.band; e.blocks_per_sm = best.minb;
                e.ms = best_ms; e.ms_untuned = untuned_ms;
                e.searches = n; e.rw = rw; e.rh = rh; e.nl = nl;
            }
        }
    g_tune = T;
    return written;
}

// Tune on the caller's own batch: every schedule is timed on it (the fastest of two launches each), and the best
// becomes the schedule of its class (its largest layer count, and whether it holds at least 16 tiles per resident
// block). For a caller whose batches repeat in shape, such as the microbenchmark's waves.
extern "C" int32_t pcbg_autotune_batch(pcbg_search* s, int32_t n, void* stream, pcbg_tune_entry* out) {
    using namespace pcbg;
    if (n <= 0) return 0;
    std::vector<BatchItem> items(n);
    int nlmax = 1;
    size_t tiles = 0;
    for (int k = 0; k < n; ++k) {
        BatchItem& b = items[k];
        const pcbg_search& q = s[k];
        memset(&b, 0, sizeof(b));
        b.rw = q.rw; b.rh = q.rh; b.nl = q.nl; b.pitch = q.pitch; b.hpad = q.hpad;
        memcpy(b.fac, q.fac, sizeof(b.fac));
        b.cf = q.cf; b.fl = q.flags; b.vcf = q.vcf;
        b.start_idx = q.start_idx; b.start_d = q.start_d; b.n_starts = q.n_starts;
        b.out = q.out;
        nlmax = std::max(nlmax, q.nl);
        tiles += size_t(q.pitch / TILE) * (q.hpad / TILE);
    }
    std::lock_guard<std::mutex> g(g_mu);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int bands[] = {0, 8, 16, 32, 64, 128};
    float best_ms = 1e30f, untuned_ms = 1e30f;
    Schedule best{DEFAULT_BAND, 0};
    for (int band : bands)
        for (int minb = 2; minb <= 3; ++minb) {
            const Schedule cand{band, minb};
            g_force = &cand;
            float ms = 1e30f;
            for (int rep = 0; rep < 2; ++rep) {
                if (solve_batch_locked(items.data(), n, st) != 0) { g_force = nullptr; return PCBG_ERR_FAIL; }
                ms = std::min(ms, t_stats.kernel_ms);
            }
            g_force = nullptr;
            if (ms < best_ms) { best_ms = ms; best = cand; }
            if (band == DEFAULT_BAND && minb == 3) untuned_ms = ms;
        }
    const int lc = layer_class(nlmax), sc = size_class(tiles);
    g_tune.s[lc][sc] = best;
    g_tune.set[lc][sc] = true;
    g_tune.ms[lc][sc] = best_ms;
    g_tune.ms_untuned[lc][sc] = untuned_ms;
    if (out) {
        out->layers_lo = 2 * lc + 1; out->layers_hi = 2 * lc + 2; out->batch_class = sc;
        out->band = best.band; out->blocks_per_sm = best.minb;
        out->ms = best_ms; out->ms_untuned = untuned_ms;
        out->searches = n; out->rw = 0; out->rh = 0; out->nl = nlmax;
    }
    return 1;
}
