// pcbg_solve(): one pcbroute search exactly as gpu_solve() receives it (src/gpu.h:10-57), on the B200 engine.
//
// Per rectangle of the window: the class's cost maps are copied in (src/gpu.cu:432-439), the net's own-copper
// overrides scattered (src/gpu.cu:460-476), every state's cost factor resolved on the device as the CPU search
// sees it (src/gpu.cu:78-115: own copper by owner id, the learned prior's factor and corridor, where a via may
// land, the target bits), and the relaxation engine of solver.cu solves it exactly. The rectangle grows from the
// start/target box by 80 x 3^k cells until an octile lower bound shows that nothing outside it can beat the best
// target (src/gpu.cu:575-619); the touched-block bookkeeping of the router depends on that rectangle, so the rule
// is kept as the reference has it.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstring>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <thread>
#include <vector>

#include "pcbg_internal.h"

namespace pcbg {
namespace {

constexpr float FINF = 1e30f;

struct QParams {
    int rw, rh, nl, pitch, hpad;
    int rx0, ry0, ww, wh;      // rectangle in the window, window size (for the target bits)
    uint16_t me;
    float via_cost;
    uint8_t lay[MAX_LAYERS];
    int play[MAX_LAYERS];
    int has_prior, corridor, mthr;
    int pi0, pj0, pw, ph;
};

// src/gpu.cu:78-105 (prep_cf) + 107-115 (prep_v): resolve one pitched state (and, on layer 0, its cell's via)
__global__ void resolve_kernel(QParams p, float* cf, const uint16_t* st, uint8_t* fl, float* vcf, const uint16_t* vst,
                               const uint64_t* tbit, const uint8_t* prior, const int* pcol, const int* prow,
                               const float* mlf) {
    const size_t plane = size_t(p.hpad) * p.pitch;
    const size_t total = plane * p.nl;
    for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < total; q += size_t(gridDim.x) * blockDim.x) {
        const int l = int(q / plane);
        const size_t rem = q % plane;
        const int j = int(rem / p.pitch), i = int(rem % p.pitch);
        if (j >= p.rh || i >= p.rw) {
            cf[q] = FINF;
            fl[q] = 0;
            if (l == 0 && vcf) vcf[rem] = FINF;
            continue;
        }
        const size_t ws = (size_t(l) * p.wh + (p.ry0 + j)) * p.ww + (p.rx0 + i);
        const bool tg = (tbit[ws >> 6] >> (ws & 63)) & 1;
        const float v = cf[q];
        const uint16_t o = st[q];
        float r;
        if (!p.lay[l] || !(v < FINF)) r = FINF;
        else if (v < 0.f) r = o == p.me ? -v : FINF;
        else r = v;
        int pv = 255;
        if (p.has_prior && p.lay[l]) {
            const int pl = p.play[l];
            if (pl >= 0) {
                const int x = pcol[i] - p.pi0, y = prow[j] - p.pj0;
                pv = (x < 0 || y < 0 || x >= p.pw || y >= p.ph) ? 0 : prior[(size_t(pl) * p.ph + y) * p.pw + x];
            }
            if (p.corridor && pv < p.mthr && !tg) r = FINF;
            else if (r < FINF) r = __fmul_rn(r, mlf[pv]);
        }
        cf[q] = r;
        const bool vok = p.lay[l] ? ((o == 0 || o == p.me) && (!p.corridor || tg || pv >= p.mthr)) : tg;
        fl[q] = uint8_t((vok ? 1 : 0) | (tg ? 2 : 0));
        if (l == 0 && vcf) {
            const float vv = vcf[rem];
            const uint16_t vo = vst[rem];
            const float vr = !(vv < FINF) ? FINF : vv < 0.f ? (vo == p.me ? -vv : FINF) : vv;
            vcf[rem] = vr < FINF ? __fmul_rn(vr, p.via_cost) : FINF;
        }
    }
}

__global__ void scatter_kernel(float* dst, const uint32_t* idx, const float* val, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) dst[idx[k]] = val[k];
}

template <class T> struct DBuf {
    T* p = nullptr;
    size_t cap = 0;
    bool need(size_t n) {
        if (n == 0) n = 1;
        if (cap >= n) return true;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        const size_t c = n + n / 8;
        if (cudaMalloc(&p, c * sizeof(T)) != cudaSuccess) { p = nullptr; return false; }
        cap = c;
        return true;
    }
};

// One slot: a stream and the device buffers of one search's inputs. As in the reference (src/gpu.cu:37-58), a
// worker thread holds a slot for the whole search, and `slots` searches prepare their inputs concurrently; their
// relaxations then run together through the round batcher (batcher.cpp).
struct Slot {
    cudaStream_t stream = nullptr;
    bool busy = false;
    DBuf<float> cf, vcf, out, lval;
    DBuf<uint16_t> st, vst;
    DBuf<uint8_t> fl, prior;
    DBuf<uint64_t> tbit, sd;
    DBuf<int> pcol, prow;
    DBuf<float> mlf;
    DBuf<uint32_t> lidx, sidx;
    unsigned char* stage = nullptr;   // pinned host staging of a rectangle's cost maps
    size_t stage_cap = 0;
};

// Grow-only pinned staging buffer of a slot.
bool stage_need(Slot& E, size_t n) {
    if (E.stage_cap >= n) return true;
    if (E.stage) cudaFreeHost(E.stage);
    E.stage = nullptr;
    E.stage_cap = 0;
    const size_t c = n + n / 4 + 4096;
    if (cudaHostAlloc(reinterpret_cast<void**>(&E.stage), c, cudaHostAllocDefault) != cudaSuccess) { E.stage = nullptr; return false; }
    E.stage_cap = c;
    return true;
}

// Rows [y0, y0 + rh) x columns [x0, x0 + rw) of a row-major host grid of row length nx, packed with row pitch
// `pitch` into dst.
template <class T>
void pack_rows(T* dst, const T* src, size_t nx, size_t hoff, int rw, int j0, int j1, int pitch) {
    for (int j = j0; j < j1; ++j) memcpy(dst + size_t(j) * pitch, src + hoff + size_t(j) * nx, size_t(rw) * sizeof(T));
}

std::mutex g_cfg_mu;
int g_slots = 4;
size_t g_maxn = size_t(48) << 20;
int g_ok = -1;
std::once_flag g_once;
std::vector<Slot*> g_slot_v;            // made on first use; never freed (the library lives as long as the process)
std::mutex g_slot_mu;
std::condition_variable g_slot_cv;

std::mutex g_pool_mu;
std::vector<std::pair<float*, size_t>> g_pool;

float fac_len(float step, int m) { return m < 4 ? step : float(double(step) * std::sqrt(2.0)); }

uint64_t start_fixed(float g0) {
    const float y = g0 * 16.0f;
    if (!(y > 0.0f)) return 0;
    if (!(y < WLIM64)) return INF64;
    return uint64_t(std::ceil(y));
}

#define CK(x)                                                             \
    do {                                                                  \
        cudaError_t e_ = (x);                                             \
        if (e_ != cudaSuccess) { set_error(std::string(#x) + ": " + cudaGetErrorString(e_)); return -1; } \
    } while (0)

double now_s() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

// Where one search's time went (printed per search when PCBG_TIMES is set, like the reference's GPU_TIMES).
struct SearchTimes {
    double prep = 0, batch = 0, out = 0, kernel_ms = 0;
    int batch_size = 0;
};

// Solve one rectangle. Fills best (window state or -1), ub (float cost of best, 1e30 if none), and out->d.
int solve_rect(Slot& E, const pcbg_query& q, int rx0, int ry0, int rw, int rh, pcbg_result* out, int64_t& best, float& ub,
               SearchTimes& tm) {
    const double t0 = now_s();
    const int nl = q.nl;
    const size_t RN = size_t(rw) * rh, N = RN * nl;
    if (N > g_maxn) { set_error("window over the state cap"); return -1; }
    // until it joins the batcher's queue, this search counts as one the batch leader waits for
    batcher_enter();
    struct Preparing {
        bool on = true;
        ~Preparing() { if (on) batcher_leave(); }
    } preparing;
    const int pitch = int(round_up(rw, TILE)), hpad = int(round_up(rh, TILE));
    const size_t plane = size_t(pitch) * hpad, PN = plane * nl;
    const bool vias = q.via_cost >= 0;
    if (!E.cf.need(PN) || !E.st.need(PN) || !E.fl.need(PN) || !E.vcf.need(plane) || !E.vst.need(plane) || !E.out.need(N) ||
        !E.pcol.need(rw) || !E.prow.need(rh)) {
        set_error("device allocation failed");
        return -1;
    }
    cudaStream_t S = E.stream;
    const size_t hoff = size_t(q.wj0 + ry0) * q.nx + (q.wi0 + rx0);
    // The rectangle's rows of the host cost maps are packed into pinned staging, then copied with one DMA per grid:
    // a strided copy from pageable memory moves row by row through the driver's own staging and runs several
    // times slower. Rows keep the device pitch, so each grid is one contiguous copy (padding cells are written by
    // the resolve kernel).
    const size_t rows = size_t(rh) * pitch;
    const size_t grid_bytes = rows * 6, total = grid_bytes * size_t(nl + (vias ? 1 : 0));
    const int ngrids = nl + (vias ? 1 : 0);
    MirrorView mv;
    const bool mirrored = mirror_lookup(q, mv);
    if (mirrored) {
        // the class's grids are in HBM already: the rectangle is copied device to device
        for (int l = 0; l < ngrids; ++l) {
            float* dc = l < nl ? E.cf.p + size_t(l) * plane : E.vcf.p;
            uint16_t* ds = l < nl ? E.st.p + size_t(l) * plane : E.vst.p;
            const float* sc = (l < nl ? mv.cst[l] : mv.vcst) + hoff;
            const uint16_t* ss = (l < nl ? mv.st[l] : mv.vst) + hoff;
            CK(cudaMemcpy2DAsync(dc, size_t(pitch) * 4, sc, size_t(q.nx) * 4, size_t(rw) * 4, rh, cudaMemcpyDeviceToDevice, S));
            CK(cudaMemcpy2DAsync(ds, size_t(pitch) * 2, ss, size_t(q.nx) * 2, size_t(rw) * 2, rh, cudaMemcpyDeviceToDevice, S));
        }
    }
    if (!mirrored && !stage_need(E, total)) { set_error("pinned allocation failed"); return -1; }
    auto pack = [&](int j0, int j1) {
        for (int l = 0; l < ngrids; ++l) {
            pack_rows(reinterpret_cast<float*>(E.stage + size_t(l) * grid_bytes), l < nl ? q.cst[l] : q.vcst,
                      size_t(q.nx), hoff, rw, j0, j1, pitch);
            pack_rows(reinterpret_cast<uint16_t*>(E.stage + size_t(l) * grid_bytes + rows * 4), l < nl ? q.st[l] : q.vst,
                      size_t(q.nx), hoff, rw, j0, j1, pitch);
        }
    };
    // a whole-board rectangle packs tens of MB: split its rows over a few threads
    const int nth = total > (size_t(16) << 20) ? 4 : 1;
    if (mirrored) {
    } else if (nth == 1) {
        pack(0, rh);
    } else {
        std::vector<std::thread> th;
        for (int t = 1; t < nth; ++t) th.emplace_back(pack, rh * t / nth, rh * (t + 1) / nth);
        pack(0, rh / nth);
        for (auto& x : th) x.join();
    }
    for (int l = 0; l < ngrids && !mirrored; ++l) {
        float* hc = reinterpret_cast<float*>(E.stage + size_t(l) * grid_bytes);
        uint16_t* hs = reinterpret_cast<uint16_t*>(E.stage + size_t(l) * grid_bytes + rows * 4);
        float* dc = l < nl ? E.cf.p + size_t(l) * plane : E.vcf.p;
        uint16_t* ds = l < nl ? E.st.p + size_t(l) * plane : E.vst.p;
        CK(cudaMemcpyAsync(dc, hc, rows * 4, cudaMemcpyHostToDevice, S));
        CK(cudaMemcpyAsync(ds, hs, rows * 2, cudaMemcpyHostToDevice, S));
    }
    if (q.prior) {
        CK(cudaMemcpyAsync(E.pcol.p, q.pcol + q.wi0 + rx0, size_t(rw) * 4, cudaMemcpyHostToDevice, S));
        CK(cudaMemcpyAsync(E.prow.p, q.prow + q.wj0 + ry0, size_t(rh) * 4, cudaMemcpyHostToDevice, S));
    }
    // own-copper overrides: window states / cells -> pitched indices of this rectangle
    const size_t FWN = size_t(q.ww) * q.wh;
    std::vector<uint32_t> li;
    std::vector<float> lv;
    auto scatter = [&](const uint32_t* idx, const float* val, int64_t n, bool cells, float* dst) -> int {
        li.clear();
        lv.clear();
        for (int64_t k = 0; k < n; ++k) {
            const size_t w = idx[k], l = cells ? 0 : w / FWN, c = w % FWN;
            const int i = int(c % q.ww) - rx0, j = int(c / q.ww) - ry0;
            if (i < 0 || j < 0 || i >= rw || j >= rh || l >= size_t(nl)) continue;
            li.push_back(uint32_t(l * plane + size_t(j) * pitch + i));
            lv.push_back(val[k]);
        }
        if (li.empty()) return 0;
        if (!E.lidx.need(li.size()) || !E.lval.need(li.size())) { set_error("device allocation failed"); return -1; }
        CK(cudaMemcpyAsync(E.lidx.p, li.data(), li.size() * 4, cudaMemcpyHostToDevice, S));
        CK(cudaMemcpyAsync(E.lval.p, lv.data(), lv.size() * 4, cudaMemcpyHostToDevice, S));
        scatter_kernel<<<unsigned((li.size() + 255) / 256), 256, 0, S>>>(dst, E.lidx.p, E.lval.p, int(li.size()));
        CK(cudaStreamSynchronize(S));  // the host lists are reused
        return 0;
    };
    if (scatter(q.own_cf_idx, q.own_cf_val, q.n_own_cf, false, E.cf.p) < 0) return -1;
    if (vias && scatter(q.own_vcf_idx, q.own_vcf_val, q.n_own_vcf, true, E.vcf.p) < 0) return -1;
    QParams p;
    memset(&p, 0, sizeof(p));
    p.rw = rw; p.rh = rh; p.nl = nl; p.pitch = pitch; p.hpad = hpad;
    p.rx0 = rx0; p.ry0 = ry0; p.ww = q.ww; p.wh = q.wh;
    p.me = q.me; p.via_cost = q.via_cost;
    for (int l = 0; l < MAX_LAYERS; ++l) { p.lay[l] = q.lay[l]; p.play[l] = q.play[l]; }
    p.has_prior = q.prior != nullptr; p.corridor = q.corridor; p.mthr = q.mthr;
    p.pi0 = q.pi0; p.pj0 = q.pj0; p.pw = q.pw; p.ph = q.ph;
    {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const size_t blocks = std::min<size_t>((PN + 255) / 256, size_t(sms) * 16);
        resolve_kernel<<<unsigned(blocks), 256, 0, S>>>(p, E.cf.p, E.st.p, E.fl.p, vias ? E.vcf.p : nullptr, E.vst.p, E.tbit.p,
                                                         E.prior.p, E.pcol.p, E.prow.p, E.mlf.p);
        CK(cudaGetLastError());
    }
    // starts: window states -> rect states, fixed-point costs
    std::vector<uint32_t> si;
    std::vector<uint64_t> sv;
    for (int64_t k = 0; k < q.n_starts; ++k) {
        const size_t w = q.start_idx[k], l = w / FWN, c = w % FWN;
        const int i = int(c % q.ww) - rx0, j = int(c / q.ww) - ry0;
        if (i < 0 || j < 0 || i >= rw || j >= rh || l >= size_t(nl)) continue;
        si.push_back(uint32_t(l * RN + size_t(j) * rw + i));
        sv.push_back(start_fixed(q.start_val[k]));
    }
    if (!E.sidx.need(si.size()) || !E.sd.need(sv.size())) { set_error("device allocation failed"); return -1; }
    if (!si.empty()) {
        CK(cudaMemcpyAsync(E.sidx.p, si.data(), si.size() * 4, cudaMemcpyHostToDevice, S));
        CK(cudaMemcpyAsync(E.sd.p, sv.data(), sv.size() * 8, cudaMemcpyHostToDevice, S));
    }
    BatchItem b;
    memset(&b, 0, sizeof(b));
    b.rw = rw; b.rh = rh; b.nl = nl; b.pitch = pitch; b.hpad = hpad;
    for (int l = 0; l < MAX_LAYERS; ++l)
        for (int m = 0; m < 8; ++m) b.fac[l][m] = l < 8 ? fac_len(q.step, m) * q.dirf[l][m] : 0.f;
    b.cf = E.cf.p; b.fl = E.fl.p; b.vcf = vias ? E.vcf.p : nullptr;
    b.start_idx = E.sidx.p; b.start_d = E.sd.p; b.n_starts = int(si.size());
    b.out = E.out.p;
    CK(cudaStreamSynchronize(S));   // the inputs are on the device before the batch launch reads them
    BatchResult br;
    preparing.on = false;
    const double t1 = now_s();
    if (batcher_submit(b, br) != 0) { set_error(br.error); return -1; }
    const double t2 = now_s();
    // the field, into a pinned buffer from the pool
    float* d = out->d;
    size_t cap = out->cap;
    if (!d || cap < N) {
        if (d) pcbg_host_release(d, cap);
        d = pcbg_host_acquire(N, &cap);
        out->d = d;
        out->cap = cap;
        if (!d) { set_error("pinned allocation failed"); return -1; }
    }
    CK(cudaMemcpyAsync(d, E.out.p, N * 4, cudaMemcpyDeviceToHost, S));
    CK(cudaStreamSynchronize(S));
    const double t3 = now_s();
    tm.prep += t1 - t0;
    tm.batch += t2 - t1;
    tm.out += t3 - t2;
    tm.kernel_ms += br.kernel_ms;
    tm.batch_size = std::max(tm.batch_size, br.batch_size);
    best = -1;
    ub = FINF;
    if (b.best >= 0) {
        const size_t l = size_t(b.best) / RN, c = size_t(b.best) % RN;
        best = int64_t((l * q.wh + (c / rw + ry0)) * q.ww + (c % rw + rx0));
        ub = float(b.best_d) * 0.0625f;
    }
    out->rx0 = rx0; out->ry0 = ry0; out->rw = rw; out->rh = rh; out->nl = nl; out->ww = q.ww; out->wh = q.wh;
    out->best = best;
    out->rounds = b.rounds;
    out->wide = b.status == 1;
    out->tile_visits = br.tile_visits;
    out->ub = ub;
    return 0;
}

bool probe_device() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return false;
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, resolve_kernel) != cudaSuccess) return false;  // no sm_100a image for this device
    return true;
}

}  // namespace
}  // namespace pcbg

using namespace pcbg;

extern "C" int pcbg_available(void) {
    std::call_once(g_once, [] { g_ok = probe_device() ? 1 : 0; });
    return g_ok;
}

extern "C" void pcbg_configure(int slots, size_t max_states) {
    std::lock_guard<std::mutex> g(g_cfg_mu);
    g_slots = std::max(1, slots);
    if (max_states) g_maxn = max_states;
}

extern "C" const char* pcbg_last_error(void) { return last_error().c_str(); }

extern "C" float* pcbg_host_acquire(size_t n, size_t* cap) {
    {
        std::lock_guard<std::mutex> g(g_pool_mu);
        for (size_t k = 0; k < g_pool.size(); ++k)
            if (g_pool[k].second >= n) {
                float* p = g_pool[k].first;
                *cap = g_pool[k].second;
                g_pool.erase(g_pool.begin() + long(k));
                return p;
            }
    }
    const size_t c = n + n / 4 + 1;
    float* p = nullptr;
    if (cudaHostAlloc(reinterpret_cast<void**>(&p), c * sizeof(float), cudaHostAllocDefault) != cudaSuccess) {
        *cap = 0;
        return nullptr;
    }
    *cap = c;
    return p;
}

extern "C" void pcbg_host_release(float* p, size_t cap) {
    if (!p) return;
    std::lock_guard<std::mutex> g(g_pool_mu);
    g_pool.push_back({p, cap});
}

// Host-side fault injection, for tests of the caller's fallback (the router carries on with its CPU search when
// gpu_solve returns -1, src/router.cpp:1598, 1691-1700). PCBG_FAIL_SOLVE=k makes the k-th call of this process
// (counting from 1) fail before it touches the device; PCBG_FAIL_SOLVE=k:p also fails every p-th call after it.
// Nothing is injected on the device.
namespace {
struct FailPlan {
    long long first = 0, every = 0;
    FailPlan() {
        const char* e = std::getenv("PCBG_FAIL_SOLVE");
        if (!e) return;
        char* end = nullptr;
        first = std::strtoll(e, &end, 10);
        if (end && *end == ':') every = std::strtoll(end + 1, nullptr, 10);
    }
};
std::atomic<long long> g_solve_calls{0};
bool injected_failure() {
    static const FailPlan plan;
    if (plan.first <= 0) return false;
    const long long n = ++g_solve_calls;
    return n == plan.first || (plan.every > 0 && n > plan.first && (n - plan.first) % plan.every == 0);
}
}  // namespace

extern "C" int pcbg_solve(const pcbg_query* qp, pcbg_result* out, int wait) {
    if (injected_failure()) { set_error("injected failure (PCBG_FAIL_SOLVE)"); return PCBG_ERR_FAIL; }
    if (!pcbg_available()) { set_error("no usable device"); return PCBG_ERR_FAIL; }
    const pcbg_query& q = *qp;
    if (q.nl < 1 || q.nl > MAX_LAYERS || q.ww < 1 || q.wh < 1) { set_error("bad query"); return PCBG_ERR_FAIL; }
    Slot* sp = nullptr;
    {
        std::unique_lock<std::mutex> lk(g_slot_mu);
        if (g_slot_v.empty()) {
            std::lock_guard<std::mutex> g(g_cfg_mu);
            for (int k = 0; k < g_slots; ++k) g_slot_v.push_back(new Slot());
        }
        auto free_slot = [&]() -> Slot* {
            for (Slot* c : g_slot_v)
                if (!c->busy) return c;
            return nullptr;
        };
        sp = free_slot();
        if (!sp && !wait) return PCBG_ERR_BUSY;
        while (!sp) {
            g_slot_cv.wait(lk);
            sp = free_slot();
        }
        sp->busy = true;
    }
    struct Release {
        Slot* s;
        ~Release() {
            {
                std::lock_guard<std::mutex> g(g_slot_mu);
                s->busy = false;
            }
            g_slot_cv.notify_one();
        }
    } release{sp};
    Slot& E = *sp;
    if (!E.stream && cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("stream creation failed");
        return PCBG_ERR_FAIL;
    }
    set_error("");
    const size_t FWN = size_t(q.ww) * q.wh, WS = FWN * q.nl, WB = WS / 64 + 1;
    cudaStream_t S = E.stream;
    // shared by every rectangle: the target bits, the prior map and its factor table
    if (!E.tbit.need(WB) || !E.mlf.need(256)) { set_error("device allocation failed"); return PCBG_ERR_FAIL; }
    if (cudaMemcpyAsync(E.tbit.p, q.tbit, WB * 8, cudaMemcpyHostToDevice, S) != cudaSuccess) return PCBG_ERR_FAIL;
    if (q.prior) {
        const size_t pn = size_t(q.pw) * q.ph * q.pnl;
        if (!E.prior.need(pn)) { set_error("device allocation failed"); return PCBG_ERR_FAIL; }
        if (cudaMemcpyAsync(E.prior.p, q.prior, pn, cudaMemcpyHostToDevice, S) != cudaSuccess) return PCBG_ERR_FAIL;
        if (cudaMemcpyAsync(E.mlf.p, q.mlf, 256 * 4, cudaMemcpyHostToDevice, S) != cudaSuccess) return PCBG_ERR_FAIL;
    }
    // box of the starts and of the targets; a path of cost ub only crosses cells whose octile distance from the
    // starts plus to the targets is at most ub (src/gpu.cu:575-598)
    int sx0 = INT_MAX, sy0 = INT_MAX, sx1 = -1, sy1 = -1, tx0 = INT_MAX, ty0 = INT_MAX, tx1 = -1, ty1 = -1;
    for (int64_t k = 0; k < q.n_starts; ++k) {
        const size_t c = q.start_idx[k] % FWN;
        const int i = int(c % q.ww), j = int(c / q.ww);
        sx0 = std::min(sx0, i); sx1 = std::max(sx1, i); sy0 = std::min(sy0, j); sy1 = std::max(sy1, j);
    }
    for (size_t w = 0; w < WB; ++w) {
        uint64_t b = q.tbit[w];
        while (b) {
            const int k = __builtin_ctzll(b);
            b &= b - 1;
            const size_t st = w * 64 + size_t(k);
            if (st >= WS) continue;
            const size_t c = st % FWN;
            const int i = int(c % q.ww), j = int(c / q.ww);
            tx0 = std::min(tx0, i); tx1 = std::max(tx1, i); ty0 = std::min(ty0, j); ty1 = std::max(ty1, j);
        }
    }
    if (sx1 < 0 || tx1 < 0) { set_error("no starts or no targets"); return PCBG_ERR_FAIL; }
    float minfac = 1.f;
    for (int l = 0; l < q.nl; ++l)
        if (q.lay[l])
            for (int m = 0; m < 8; ++m) minfac = std::min(minfac, q.dirf[l][m]);
    const double unit = double(q.step) * minfac;
    auto oct = [&](int i, int j, int x0, int y0, int x1, int y1) {
        const double dx = std::max({0.0, double(x0) - i, double(i) - x1}), dy = std::max({0.0, double(y0) - j, double(j) - y1});
        return unit * (std::max(dx, dy) + 0.41421356 * std::min(dx, dy));
    };
    auto lb = [&](int i, int j) { return oct(i, j, sx0, sy0, sx1, sy1) + oct(i, j, tx0, ty0, tx1, ty1); };
    const int hx0 = std::min(sx0, tx0), hy0 = std::min(sy0, ty0), hx1 = std::max(sx1, tx1), hy1 = std::max(sy1, ty1);
    int M = 80, tries = 0;
    SearchTimes tm;
    const double t_start = now_s();
    out->best = -1;
    for (;; M *= 3, ++tries) {
        int rx0 = std::max(0, hx0 - M), ry0 = std::max(0, hy0 - M);
        int rx1 = std::min(q.ww, hx1 + M + 1), ry1 = std::min(q.wh, hy1 + M + 1);
        if (tries == 0 && double(rx1 - rx0) * (ry1 - ry0) > 0.5 * double(q.ww) * q.wh) { rx0 = ry0 = 0; rx1 = q.ww; ry1 = q.wh; }
        const bool full = rx0 == 0 && ry0 == 0 && rx1 == q.ww && ry1 == q.wh;
        int64_t best = -1;
        float ub = FINF;
        if (solve_rect(E, q, rx0, ry0, rx1 - rx0, ry1 - ry0, out, best, ub, tm) != 0) return PCBG_ERR_FAIL;
        if (full) break;
        if (ub < FINF * 0.5f) {
            const double lim = double(ub) * 1.0001 + 1e-3;
            double mn = 1e300;
            if (rx0 > 0) for (int j = 0; j < q.wh; ++j) mn = std::min(mn, lb(rx0 - 1, j));
            if (rx1 < q.ww) for (int j = 0; j < q.wh; ++j) mn = std::min(mn, lb(rx1, j));
            if (ry0 > 0) for (int i = 0; i < q.ww; ++i) mn = std::min(mn, lb(i, ry0 - 1));
            if (ry1 < q.wh) for (int i = 0; i < q.ww; ++i) mn = std::min(mn, lb(i, ry1));
            if (mn > lim) break;
        }
    }
    out->tries = tries + 1;
    static const bool report = std::getenv("PCBG_TIMES") != nullptr;
    if (report)
        std::fprintf(stderr,
                     "pcbg: window %dx%dx%d rect %dx%d (%d tries) prep %.2f ms, batch %.2f ms (%d searches, relax %.2f ms), "
                     "field %.2f ms, total %.2f ms\n",
                     q.ww, q.wh, q.nl, out->rw, out->rh, tries + 1, tm.prep * 1e3, tm.batch * 1e3, tm.batch_size,
                     tm.kernel_ms, tm.out * 1e3, (now_s() - t_start) * 1e3);
    return std::max(1, out->rounds);
}
