// Exact multi-layer grid shortest paths on sm_100a: the relaxation engine behind gpu_solve and pcbg_solve_batch.
//
// The reference (src/gpu.cu:122-363, 488-524) relaxes a search window with 8 directional min-plus sweeps plus a
// via pass, 27 launches and one host sync per sweep, until nothing changes. Here the same relaxation rule
// (move into a state costs its factor times the move's length and direction factor, vias land only where a via
// may, src/gpu.cu:154-155, 332-350) is solved to its exact integer least fixed point by a tiled worklist:
//
//   * the window is cut into 32 x 32-cell tiles holding every layer; a tile visit stages the tile's distances
//     (with a one-cell halo from its neighbours), cost factors, via costs and via/target masks in shared memory
//     and relaxes them to a local fixed point (directional line scans +x/-x, +y/-y, both diagonals, vias);
//   * a tile whose edge cells improved (to a cost not above the best target found so far) queues the neighbours
//     that read those cells for the next round;
//   * one persistent cooperative launch runs all rounds of all searches of a batch, with a bounded software
//     grid barrier between rounds, so a whole round of searches with uneven windows shares the GPU.
//
// Exactness: distances are fixed-point integers (pcbg.h), min-plus over integers is exact and associative, so
// the least fixed point is unique and independent of the tile order; every state whose least cost is at most the
// best target's is exact (the dirty rule only drops improvements above the best target, which cannot lie on a
// path that matters), and the epilogue reports exactly those.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "pcbg_internal.h"

namespace pcbg {

namespace {

constexpr int NT = 256;                 // threads per tile block
constexpr int HS = TILE + 2;            // tile side with halo
constexpr int DSTR = TILE + 3;          // shared row stride of distances (odd: conflict-free row and column scans)
constexpr int CSTR = TILE + 1;          // shared row stride of cost factors / per-cell arrays
constexpr int MAX_IT = 64;              // local iterations before a tile is re-queued instead
constexpr long long BAR_SPIN_LIMIT = 1ll << 24;   // polls (with __nanosleep) before a barrier wait gives up

// control words of a batch
enum { C_CNT = 0, C_NEXT = 3, C_BAR = 6, C_GEN = 7, C_ERR = 8, C_ROUNDS = 9, C_OVF = 10, C_N = 16 };
enum { ERR_BARRIER = 1, ERR_ROUNDS = 2, ERR_OVERFLOW = 4 };

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
    unsigned long long* wl;       // 3 rotating worklists of `cap` items: (search << 32) | tile
    unsigned int cap;
    unsigned int* ctl;
    unsigned long long* visits;
    int max_rounds;
};

struct SmemLayout {
    size_t d, c, w, e, m, total;
};
__host__ __device__ inline SmemLayout smem_layout(int nlm, size_t dsz) {
    SmemLayout L;
    size_t o = 0;
    L.d = o; o += size_t(nlm) * HS * DSTR * dsz; o = (o + 15) & ~size_t(15);
    L.c = o; o += size_t(nlm) * TILE * CSTR * 4; o = (o + 15) & ~size_t(15);
    L.w = o; o += size_t(TILE) * CSTR * dsz; o = (o + 15) & ~size_t(15);
    L.e = o; o += size_t(nlm) * 4 * TILE * dsz; o = (o + 15) & ~size_t(15);
    L.m = o; o += size_t(2) * TILE * CSTR; o = (o + 15) & ~size_t(15);
    L.total = o;
    return L;
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

// One tile visit: stage, relax to a local fixed point, write back, queue neighbours, report targets.
template <typename DT>
__device__ void visit_tile(const SolveArgs& a, int s, int tile, int round, unsigned char* smem) {
    const SDev& S = a.S[s];
    const int tid = threadIdx.x;
    const int nl = S.nl, pitch = S.pitch, hpad = S.hpad;
    const int tx = tile % S.ntx, ty = tile / S.ntx;
    const int x0 = tx * TILE, y0 = ty * TILE;
    const SmemLayout L = smem_layout(a.nlmax, sizeof(DT));
    DT* dS = reinterpret_cast<DT*>(smem + L.d);
    float* cS = reinterpret_cast<float*>(smem + L.c);
    DT* wS = reinterpret_cast<DT*>(smem + L.w);
    DT* eS = reinterpret_cast<DT*>(smem + L.e);
    uint8_t* vokS = smem + L.m;
    uint8_t* tgS = vokS + TILE * CSTR;
    __shared__ unsigned int sh_marks, sh_any;
    __shared__ unsigned long long sh_tmin, sh_wmax;
    __shared__ unsigned int sh_wide;
    const DT INF = Lim<DT>::INF;
    const DT* dist = reinterpret_cast<const DT*>(S.dist);
    DT* distw = reinterpret_cast<DT*>(S.dist);
    if (tid == 0) { sh_marks = 0; sh_any = 0; sh_tmin = ~0ull; sh_wmax = 0; sh_wide = 0; }

    // ---- stage: distances with halo
    for (int idx = tid; idx < nl * HS * HS; idx += NT) {
        const int l = idx / (HS * HS), rem = idx % (HS * HS), r = rem / HS, c = rem % HS;
        const int gy = y0 + r - 1, gx = x0 + c - 1;
        DT v = INF;
        if (gy >= 0 && gy < hpad && gx >= 0 && gx < pitch) v = dist[(size_t(l) * hpad + gy) * pitch + gx];
        dS[(l * HS + r) * DSTR + c] = v;
    }
    // cost factors; the largest weight any move into a staged state can take decides whether 32-bit
    // arithmetic is exact for this search
    unsigned long long wmax = 0;
    bool wide = false;
    for (int idx = tid; idx < nl * TILE * TILE; idx += NT) {
        const int l = idx >> 10, r = (idx >> 5) & 31, c = idx & 31;
        const float cf = S.cf[(size_t(l) * hpad + y0 + r) * pitch + x0 + c];
        cS[(l * TILE + r) * CSTR + c] = cf;
        if (cf < 1e30f) {
            const float y = __fmul_rn(__fmul_rn(cf, S.maxfac[l]), 16.0f);
            if (!(y < Lim<DT>::wlim())) wide = true;
            else wmax = max(wmax, static_cast<unsigned long long>(qweight<DT>(cf, S.maxfac[l])));
        }
    }
    // per cell: via weight and the via-landing / target masks over the layers
    for (int cell = tid; cell < TILE * TILE; cell += NT) {
        const int r = cell >> 5, c = cell & 31;
        DT wv = INF;
        if (S.vcf) {
            const float v = S.vcf[size_t(y0 + r) * pitch + x0 + c];
            if (v < 1e30f) {
                const float y = __fmul_rn(v, 16.0f);
                if (!(y < Lim<DT>::wlim())) wide = true;
                else { wv = qweight<DT>(v, 1.0f); wmax = max(wmax, static_cast<unsigned long long>(wv)); }
            }
        }
        wS[r * CSTR + c] = wv;
        unsigned int vm = 0, tm = 0;
        for (int l = 0; l < nl; ++l) {
            const uint8_t f = S.fl[(size_t(l) * hpad + y0 + r) * pitch + x0 + c];
            vm |= unsigned(f & 1) << l;
            tm |= unsigned((f >> 1) & 1) << l;
        }
        vokS[r * CSTR + c] = uint8_t(vm);
        tgS[r * CSTR + c] = uint8_t(tm);
    }
    __syncthreads();
    // original edge values (to tell which neighbours must look again)
    for (int idx = tid; idx < nl * 4 * TILE; idx += NT) {
        const int l = idx / (4 * TILE), side = (idx / TILE) & 3, k = idx % TILE;
        const int r = side == 0 ? k : side == 1 ? k : side == 2 ? 0 : TILE - 1;
        const int c = side == 0 ? 0 : side == 1 ? TILE - 1 : k;
        eS[idx] = dS[(l * HS + r + 1) * DSTR + c + 1];
    }
    if (wide) atomicOr(&sh_wide, 1u);
    if (wmax) atomicMax(&sh_wmax, wmax);
    __syncthreads();

    // ---- relax to a local fixed point
    bool requeue = false;
    for (int it = 0;; ++it) {
        int ch = 0;
        // +x then -x along rows: one thread per (layer, row)
        {
            const int l = tid >> 5, r = tid & 31;
            if (l < nl) {
                DT* row = dS + (l * HS + r + 1) * DSTR;
                const float* crow = cS + (l * TILE + r) * CSTR;
                const float f0 = S.fac[l][0], f1 = S.fac[l][1];
                DT prev = row[0];
                #pragma unroll 8
                for (int k = 0; k < TILE; ++k) {
                    const DT v = row[k + 1], n = dmin(v, prev + qweight<DT>(crow[k], f0));
                    if (n < v) { row[k + 1] = n; ch = 1; }
                    prev = n;
                }
                prev = row[TILE + 1];
                #pragma unroll 8
                for (int k = TILE - 1; k >= 0; --k) {
                    const DT v = row[k + 1], n = dmin(v, prev + qweight<DT>(crow[k], f1));
                    if (n < v) { row[k + 1] = n; ch = 1; }
                    prev = n;
                }
            }
        }
        __syncthreads();
        // +y then -y along columns: one thread per (layer, column)
        {
            const int l = tid >> 5, c = tid & 31;
            if (l < nl) {
                DT* col = dS + l * HS * DSTR + c + 1;
                const float* ccol = cS + l * TILE * CSTR + c;
                const float f2 = S.fac[l][2], f3 = S.fac[l][3];
                DT prev = col[0];
                #pragma unroll 8
                for (int k = 0; k < TILE; ++k) {
                    const DT v = col[(k + 1) * DSTR], n = dmin(v, prev + qweight<DT>(ccol[k * CSTR], f2));
                    if (n < v) { col[(k + 1) * DSTR] = n; ch = 1; }
                    prev = n;
                }
                prev = col[(TILE + 1) * DSTR];
                #pragma unroll 8
                for (int k = TILE - 1; k >= 0; --k) {
                    const DT v = col[(k + 1) * DSTR], n = dmin(v, prev + qweight<DT>(ccol[k * CSTR], f3));
                    if (n < v) { col[(k + 1) * DSTR] = n; ch = 1; }
                    prev = n;
                }
            }
        }
        __syncthreads();
        // main diagonals i - j = e: (+,+) forward, (-,-) backward
        for (int line = tid; line < nl * (2 * TILE - 1); line += NT) {
            const int l = line / (2 * TILE - 1), e = line % (2 * TILE - 1) - (TILE - 1);
            const int i0 = e > 0 ? e : 0, j0 = e < 0 ? -e : 0, len = TILE - (e < 0 ? -e : e);
            DT* base = dS + l * HS * DSTR;
            const float* cb = cS + l * TILE * CSTR;
            const float f4 = S.fac[l][4], f7 = S.fac[l][7];
            DT prev = base[j0 * DSTR + i0];  // (i0 - 1, j0 - 1) in halo coordinates
            for (int k = 0; k < len; ++k) {
                const int i = i0 + k, j = j0 + k;
                DT* p = base + (j + 1) * DSTR + i + 1;
                const DT v = *p, n = dmin(v, prev + qweight<DT>(cb[j * CSTR + i], f4));
                if (n < v) { *p = n; ch = 1; }
                prev = n;
            }
            prev = base[(j0 + len + 1) * DSTR + i0 + len + 1];
            for (int k = len - 1; k >= 0; --k) {
                const int i = i0 + k, j = j0 + k;
                DT* p = base + (j + 1) * DSTR + i + 1;
                const DT v = *p, n = dmin(v, prev + qweight<DT>(cb[j * CSTR + i], f7));
                if (n < v) { *p = n; ch = 1; }
                prev = n;
            }
        }
        __syncthreads();
        // anti-diagonals i + j = s: (-,+) with j increasing, (+,-) with i increasing
        for (int line = tid; line < nl * (2 * TILE - 1); line += NT) {
            const int l = line / (2 * TILE - 1), sdx = line % (2 * TILE - 1);
            const int lo = sdx > TILE - 1 ? sdx - (TILE - 1) : 0, len = TILE - (sdx > TILE - 1 ? sdx - (TILE - 1) : (TILE - 1) - sdx);
            DT* base = dS + l * HS * DSTR;
            const float* cb = cS + l * TILE * CSTR;
            const float f5 = S.fac[l][5], f6 = S.fac[l][6];
            // (-,+): q = (i, j) from p = (i + 1, j - 1); cells j = lo .. lo + len - 1, i = sdx - j
            {
                DT prev = base[lo * DSTR + (sdx - lo + 1) + 1];
                for (int k = 0; k < len; ++k) {
                    const int j = lo + k, i = sdx - j;
                    DT* p = base + (j + 1) * DSTR + i + 1;
                    const DT v = *p, n = dmin(v, prev + qweight<DT>(cb[j * CSTR + i], f6));
                    if (n < v) { *p = n; ch = 1; }
                    prev = n;
                }
            }
            // (+,-): q = (i, j) from p = (i - 1, j + 1); cells i = lo .. lo + len - 1, j = sdx - i
            {
                DT prev = base[(sdx - lo + 1 + 1) * DSTR + lo];
                for (int k = 0; k < len; ++k) {
                    const int i = lo + k, j = sdx - i;
                    DT* p = base + (j + 1) * DSTR + i + 1;
                    const DT v = *p, n = dmin(v, prev + qweight<DT>(cb[j * CSTR + i], f5));
                    if (n < v) { *p = n; ch = 1; }
                    prev = n;
                }
            }
        }
        __syncthreads();
        // vias: from the cheapest layer of a cell to every layer a via may land on
        for (int cell = tid; cell < TILE * TILE; cell += NT) {
            const int r = cell >> 5, c = cell & 31;
            const DT wv = wS[r * CSTR + c];
            if (wv >= INF) continue;
            const unsigned int vm = vokS[r * CSTR + c];
            if (!vm) continue;
            DT best = INF;
            for (int l = 0; l < nl; ++l) best = dmin(best, dS[(l * HS + r + 1) * DSTR + c + 1]);
            if (best >= INF) continue;
            const DT n = best + wv;
            for (int l = 0; l < nl; ++l) {
                if (!((vm >> l) & 1)) continue;
                DT* p = dS + (l * HS + r + 1) * DSTR + c + 1;
                if (n < *p) { *p = n; ch = 1; }
            }
        }
        const int any = __syncthreads_or(ch);
        if (!any) break;
        if (tid == 0) sh_any = 1;
        if (it + 1 >= MAX_IT) { requeue = true; break; }
    }
    __syncthreads();

    // ---- targets of the tile: least (distance) into the search's bound
    const unsigned long long ub_now = *reinterpret_cast<volatile unsigned long long*>(&a.st[s].ub);
    {
        unsigned long long tmin = ~0ull;
        for (int cell = tid; cell < TILE * TILE; cell += NT) {
            const int r = cell >> 5, c = cell & 31;
            const unsigned int tm = tgS[r * CSTR + c];
            if (!tm) continue;
            for (int l = 0; l < nl; ++l)
                if ((tm >> l) & 1) {
                    const DT v = dS[(l * HS + r + 1) * DSTR + c + 1];
                    if (v < INF) tmin = min(tmin, static_cast<unsigned long long>(v));
                }
        }
        if (tmin != ~0ull) atomicMin(&sh_tmin, tmin);
    }
    __syncthreads();
    const unsigned long long ub = min(ub_now, sh_tmin);
    if (sh_any) {
        // write back the interior
        for (int idx = tid; idx < nl * TILE * TILE; idx += NT) {
            const int l = idx >> 10, r = (idx >> 5) & 31, c = idx & 31;
            distw[(size_t(l) * hpad + y0 + r) * pitch + x0 + c] = dS[(l * HS + r + 1) * DSTR + c + 1];
        }
        // edges that improved to at most the bound: the neighbours reading them look again
        unsigned int marks = 0;
        for (int idx = tid; idx < nl * 4 * TILE; idx += NT) {
            const int l = idx / (4 * TILE), side = (idx / TILE) & 3, k = idx % TILE;
            const int r = side == 0 ? k : side == 1 ? k : side == 2 ? 0 : TILE - 1;
            const int c = side == 0 ? 0 : side == 1 ? TILE - 1 : k;
            const DT v = dS[(l * HS + r + 1) * DSTR + c + 1];
            if (!(v < eS[idx]) || static_cast<unsigned long long>(v) > ub) continue;
            // bits: 0 L, 1 R, 2 T, 3 B, 4 TL, 5 TR, 6 BL, 7 BR
            if (side == 0) { marks |= 1u; if (k == 0) marks |= 16u; if (k == TILE - 1) marks |= 64u; }
            else if (side == 1) { marks |= 2u; if (k == 0) marks |= 32u; if (k == TILE - 1) marks |= 128u; }
            else if (side == 2) marks |= 4u;
            else marks |= 8u;
        }
        if (marks) atomicOr(&sh_marks, marks);
    }
    __syncthreads();
    if (tid == 0) {
        SStat& st = a.st[s];
        if (sh_tmin != ~0ull && sh_tmin < ub_now) atomicMin(&st.ub, sh_tmin);
        if (sh_wmax) atomicMax(&st.maxw, sh_wmax);
        if (sh_wide) atomicOr(&st.need_wide, 1u);
        const unsigned int m = sh_marks;
        const int DXs[8] = {-1, 1, 0, 0, -1, 1, -1, 1}, DYs[8] = {0, 0, -1, 1, -1, -1, 1, 1};
        for (int b = 0; b < 8; ++b) {
            if (!((m >> b) & 1)) continue;
            const int nx = tx + DXs[b], ny = ty + DYs[b];
            if (nx < 0 || ny < 0 || nx >= S.ntx || ny >= S.nty) continue;
            enqueue(a, S, s, ny * S.ntx + nx, round + 1);
        }
        if (requeue) enqueue(a, S, s, tile, round + 1);
        atomicAdd(a.visits, 1ull);
    }
    __syncthreads();
}

template <typename DT>
__global__ void __launch_bounds__(NT) relax_kernel(SolveArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ unsigned int sh_item_hi, sh_item_lo, sh_stop;
    const unsigned int nblocks = gridDim.x;
    int round = 1;
    for (;; ++round) {
        const int buf = round % 3;
        const unsigned int n = *reinterpret_cast<volatile unsigned int*>(a.ctl + C_CNT + buf);
        const unsigned int cnt = n < a.cap ? n : a.cap;
        for (;;) {
            if (threadIdx.x == 0) {
                const unsigned int k = atomicAdd(a.ctl + C_NEXT + buf, 1u);
                if (k < cnt) {
                    const unsigned long long it = a.wl[size_t(buf) * a.cap + k];
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
            visit_tile<DT>(a, int(hi), int(lo), round, smem);
        }
        // the list consumed last round is free: clear it for the round after next
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            const int fb = (round + 2) % 3;
            a.ctl[C_CNT + fb] = 0;
            a.ctl[C_NEXT + fb] = 0;
        }
        grid_barrier(a.ctl, nblocks);
        if (threadIdx.x == 0) {
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
    if (blockIdx.x == 0 && threadIdx.x == 0) a.ctl[C_ROUNDS] = unsigned(round);
}

// starts: distance init (least per state) and the first round's tiles
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
        enqueue(a, S, s, (j / TILE) * S.ntx + i / TILE, 1);
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
    for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < N; q += size_t(gridDim.x) * blockDim.x) {
        const int l = int(q / RN), rem = int(q % RN), j = rem / S.rw, i = rem % S.rw;
        const size_t p = (size_t(l) * S.hpad + j) * S.pitch + i;
        const DT d = dist[p];
        if (d < INF) {
            maxd = max(maxd, static_cast<unsigned long long>(d));
            if (have && (S.fl[p] & 2) && static_cast<unsigned long long>(d) == ub) bidx = min(bidx, static_cast<unsigned long long>(q));
        }
        if (S.out) S.out[q] = (d < INF && (!have || static_cast<unsigned long long>(d) <= ub)) ? __ull2float_rn(d) * 0.0625f : 1e30f;
    }
    for (int o = 16; o; o >>= 1) {
        bidx = min(bidx, __shfl_xor_sync(0xFFFFFFFFu, bidx, o));
        maxd = max(maxd, __shfl_xor_sync(0xFFFFFFFFu, maxd, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (bidx != ~0ull) atomicMin(&st.best, bidx);
        if (maxd) atomicMax(&st.maxd, maxd);
    }
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
    DevBuf dist, stamp, wl, sdev, sstat, ctl, visits, sptr;
    std::vector<unsigned char> hbuf;
} g_arena;

thread_local std::string t_err;
thread_local BatchStats t_stats;

template <typename DT> int occupancy_blocks(int nlmax, size_t* smem_out) {
    const size_t smem = smem_layout(nlmax, sizeof(DT)).total;
    *smem_out = smem;
    if (cudaFuncSetAttribute(relax_kernel<DT>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess) return -1;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, relax_kernel<DT>, NT, smem) != cudaSuccess) return -1;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return per_sm * sms;
}

// Solve items[idx[0..m)] with DT distances. dist scratch per item at doff[k] (bytes).
template <typename DT>
int run_batch(BatchItem* items, const std::vector<int>& idx, cudaStream_t stream, int& rounds_out, long long& visits_out) {
    const int m = int(idx.size());
    std::vector<SDev> sd(m);
    std::vector<size_t> doff(m), toff(m);
    size_t dbytes = 0, tiles = 0;
    int nlmax = 1;
    for (int k = 0; k < m; ++k) {
        const BatchItem& b = items[idx[k]];
        SDev& S = sd[k];
        memset(&S, 0, sizeof(S));
        S.rw = b.rw; S.rh = b.rh; S.nl = b.nl; S.pitch = b.pitch; S.hpad = b.hpad;
        S.ntx = b.pitch / TILE; S.nty = b.hpad / TILE;
        for (int l = 0; l < MAX_LAYERS; ++l) {
            float mf = 0.f;
            for (int d = 0; d < 8; ++d) { S.fac[l][d] = b.fac[l][d]; mf = std::max(mf, b.fac[l][d]); }
            S.maxfac[l] = mf;
        }
        S.cf = b.cf; S.fl = b.fl; S.vcf = b.vcf; S.out = b.out;
        doff[k] = dbytes;
        dbytes += round_up(size_t(b.nl) * b.hpad * b.pitch * sizeof(DT), 256);
        toff[k] = tiles;
        tiles += size_t(S.ntx) * S.nty;
        nlmax = std::max(nlmax, b.nl);
    }
    Arena& A = g_arena;
    const unsigned int cap = unsigned(std::max<size_t>(tiles, 1));
    if (!A.dist.need(dbytes) || !A.stamp.need(tiles * 4 + 4) || !A.wl.need(size_t(3) * cap * 8) ||
        !A.sdev.need(sizeof(SDev) * m) || !A.sstat.need(sizeof(SStat) * m) || !A.ctl.need(C_N * 4) ||
        !A.visits.need(8) || !A.sptr.need(size_t(m) * (8 + 8 + 4) + 64)) {
        t_err = "device allocation failed";
        return -1;
    }
    for (int k = 0; k < m; ++k) {
        sd[k].dist = static_cast<unsigned char*>(A.dist.p) + doff[k];
        sd[k].stamp = static_cast<uint32_t*>(A.stamp.p) + toff[k];
    }
    // host-side arrays for the start pointers
    std::vector<const uint32_t*> sip(m);
    std::vector<const uint64_t*> sdp(m);
    std::vector<int> nsv(m);
    for (int k = 0; k < m; ++k) { sip[k] = items[idx[k]].start_idx; sdp[k] = items[idx[k]].start_d; nsv[k] = items[idx[k]].n_starts; }
    unsigned char* sp = static_cast<unsigned char*>(A.sptr.p);
    const uint32_t* const* d_sip = reinterpret_cast<const uint32_t* const*>(sp);
    const uint64_t* const* d_sdp = reinterpret_cast<const uint64_t* const*>(sp + size_t(m) * 8);
    const int* d_ns = reinterpret_cast<const int*>(sp + size_t(m) * 16);
    std::vector<SStat> st0(m);
    for (auto& x : st0) { x.ub = ~0ull; x.maxw = 0; x.best = ~0ull; x.maxd = 0; x.need_wide = 0; x.pad = 0; }
    cudaMemcpyAsync(A.sdev.p, sd.data(), sizeof(SDev) * m, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(A.sstat.p, st0.data(), sizeof(SStat) * m, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(sp, sip.data(), size_t(m) * 8, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(sp + size_t(m) * 8, sdp.data(), size_t(m) * 8, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(sp + size_t(m) * 16, nsv.data(), size_t(m) * 4, cudaMemcpyHostToDevice, stream);
    cudaMemsetAsync(A.dist.p, 0x7F, dbytes, stream);
    cudaMemsetAsync(A.stamp.p, 0, tiles * 4 + 4, stream);
    cudaMemsetAsync(A.ctl.p, 0, C_N * 4, stream);
    cudaMemsetAsync(A.visits.p, 0, 8, stream);
    SolveArgs a;
    a.S = static_cast<const SDev*>(A.sdev.p);
    a.st = static_cast<SStat*>(A.sstat.p);
    a.n = m;
    a.nlmax = nlmax;
    a.wl = static_cast<unsigned long long*>(A.wl.p);
    a.cap = cap;
    a.ctl = static_cast<unsigned int*>(A.ctl.p);
    a.visits = static_cast<unsigned long long*>(A.visits.p);
    a.max_rounds = 1 << 20;
    seed_kernel<DT><<<m, 128, 0, stream>>>(a, d_sip, d_sdp, d_ns);
    size_t smem = 0;
    const int blocks = occupancy_blocks<DT>(nlmax, &smem);
    if (blocks <= 0) { t_err = "relax kernel cannot be resident"; return -1; }
    void* args[] = {&a};
    cudaError_t e = cudaLaunchCooperativeKernel(reinterpret_cast<void*>(relax_kernel<DT>), dim3(blocks), dim3(NT), args, smem, stream);
    if (e != cudaSuccess) { t_err = std::string("cooperative launch: ") + cudaGetErrorString(e); return -1; }
    report_kernel<DT><<<dim3(32, m), 256, 0, stream>>>(a.S, a.st);
    std::vector<SStat> st(m);
    unsigned int ctl[C_N];
    unsigned long long visits = 0;
    cudaMemcpyAsync(st.data(), A.sstat.p, sizeof(SStat) * m, cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(ctl, A.ctl.p, sizeof(ctl), cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(&visits, A.visits.p, 8, cudaMemcpyDeviceToHost, stream);
    e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) { t_err = std::string("batch solve: ") + cudaGetErrorString(e); return -1; }
    if (ctl[C_ERR]) {
        t_err = "batch solve aborted (error bits " + std::to_string(ctl[C_ERR]) + ")";
        return -1;
    }
    rounds_out = int(ctl[C_ROUNDS]);
    visits_out = (long long)visits;
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
    }
    return 0;
}

}  // namespace

void set_error(const std::string& s) { t_err = s; }
const std::string& last_error() { return t_err; }
BatchStats& last_stats() { return t_stats; }

int solve_batch(BatchItem* items, int n, cudaStream_t stream) {
    std::lock_guard<std::mutex> g(g_mu);
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
    int rounds = 0;
    long long visits = 0;
    if (run_batch<uint32_t>(items, all, stream, rounds, visits) != 0) return -1;
    t_stats.rounds = rounds;
    t_stats.tile_visits = visits;
    std::vector<int> wide;
    for (int k = 0; k < n; ++k)
        if (items[k].status == 1) wide.push_back(k);
    if (!wide.empty()) {
        if (run_batch<uint64_t>(items, wide, stream, rounds, visits) != 0) return -1;
        t_stats.rounds += rounds;
        t_stats.tile_visits += visits;
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
