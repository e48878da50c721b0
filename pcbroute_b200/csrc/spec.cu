// Speculative negotiation rounds on the device: pcbroute's route_waves (src/router.cpp:2096-2242), restated for
// batched searches.
//
// route_waves routes a fixed order of nets with T worker threads that run ahead of the commit point. Each worker
// searches the next net against the board as committed so far. A net is committed once every net before it is. It
// is accepted if no commit since its search started touched a block of cells the search read; otherwise it is
// searched again (a wasted search). The result is exactly that of routing the nets one by one in this order,
// whatever the timing, and the lookahead adapts to the rejections (+1 per accept up to 2T, x3/4 per rejection down
// to 2).
//
// Here the T workers become one batch: the nets the policy picks from the lookahead window are searched together
// in one persistent relaxation launch, against the device cost board (costs.cu), and walked back on the device.
// Commits then run in order on the host, stamping each accepted path into the board's occupancy (costs_stamp:
// occupancy and the costs of those cells). A search reads its whole window, so a commit invalidates every later
// search whose window covers one of the BS x BS blocks the committed path crosses.
//
// An iteration is PathFinder's rip-up and reroute: every net's previous path is lifted, the costs are rebuilt with
// the iteration's present-congestion factor, and the nets are routed in order. Policies choose only which nets are
// searched together; the commit order and the acceptance test are fixed, so every policy gives the same paths as
// the sequential one (one search per launch, never rejected).
#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "pcbg_internal.h"

namespace pcbg {
namespace {

constexpr int BS = SPEC_BLOCK;   // cells per side of a touched block

struct WinDesc {
    int x0, y0, rw, rh, pitch, hpad;
    size_t off_state, off_cell;    // into the batch's pitched cf / flags and vcf arrays
    uint32_t tgt;                  // rect state of the target
};

// The window of each search, resolved from the class's cost maps: a step cost factor where the map is a free,
// finite cost (own-copper and blocked cells are impassable to these nets), a via landing wherever the layer is
// passable, the target bit, and the via cost times via_cost.
__global__ void spec_resolve_kernel(CostPlanes P, const WinDesc* wd, int nl, float via_cost, float* cf, uint8_t* fl,
                                    float* vcf) {
    const WinDesc W = wd[blockIdx.y];
    const size_t plane = size_t(W.hpad) * W.pitch, total = plane * nl;
    for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < total; q += size_t(gridDim.x) * blockDim.x) {
        const int l = int(q / plane);
        const size_t rem = q % plane;
        const int j = int(rem / W.pitch), i = int(rem % W.pitch);
        float c = 1e30f, v = 1e30f;
        uint8_t f = 0;
        if (i < W.rw && j < W.rh) {
            const size_t cell = size_t(W.y0 + j) * P.nx + (W.x0 + i);
            const float x = P.cst[l][cell];
            if (x > 0.f && x < 1e30f) { c = x; f = 1; }
            const uint32_t rs = uint32_t((size_t(l) * W.rh + j) * W.rw + i);
            if (rs == W.tgt) f |= 2;
            if (l == 0) {
                const float y = P.vcst[cell];
                if (y > 0.f && y < 1e30f && via_cost >= 0.f) v = __fmul_rn(y, via_cost);
            }
        }
        cf[W.off_state + q] = c;
        fl[W.off_state + q] = f;
        if (l == 0) vcf[W.off_cell + rem] = v;
    }
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
        const size_t c = n + n / 4;
        if (cudaMalloc(&p, c * sizeof(T)) != cudaSuccess) { p = nullptr; return false; }
        cap = c;
        return true;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

double now_s() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

}  // namespace
}  // namespace pcbg

struct pcbg_spec {
    pcbg_costs* costs = nullptr;
    int cls = 0;
    pcbg::CostPlanes P{};
    float via_cost = 0.f;
    float fac[pcbg::MAX_LAYERS][8];
    std::vector<pcbg_net> nets;
    std::vector<std::vector<uint32_t>> path;     // committed paths, board states, target first
    cudaStream_t stream = nullptr;
    pcbg::DBuf<float> cf, vcf;
    pcbg::DBuf<uint8_t> fl;
    pcbg::DBuf<uint32_t> si, pbuf;
    pcbg::DBuf<uint64_t> sd;
    pcbg::DBuf<int> plen;
    pcbg::DBuf<pcbg::WinDesc> wd;
    unsigned char* hpin = nullptr;               // pinned staging of a batch's uploads and of its paths
    size_t hpin_cap = 0;
    pcbg_spec_scheduler sched = nullptr;        // learned batch composition (PCBG_SPEC_LEARNED)
    void* sched_user = nullptr;
    pcbg_spec_observer observer = nullptr;      // called once per speculative search (conflict logs)
    void* observer_user = nullptr;
};

namespace pcbg {
namespace {

int bw_of(const pcbg_spec* S) { return (S->P.nx + BS - 1) / BS; }

bool pinned(pcbg_spec* S, size_t n) {
    if (S->hpin_cap >= n) return true;
    if (S->hpin) cudaFreeHost(S->hpin);
    S->hpin = nullptr;
    S->hpin_cap = 0;
    const size_t c = n + n / 2 + 4096;
    if (cudaHostAlloc(reinterpret_cast<void**>(&S->hpin), c, cudaHostAllocDefault) != cudaSuccess) return false;
    S->hpin_cap = c;
    return true;
}

// Search nets B (indices) in one batch; paths come back as board states, target first (empty: no path).
int run_searches(pcbg_spec* S, const std::vector<int>& B, std::vector<std::vector<uint32_t>>& out, double& ms,
                 double& relax_ms) {
    const double t0 = now_s();
    const int n = int(B.size()), nl = S->P.nl;
    std::vector<WinDesc> wd(n);
    size_t states = 0, cells = 0;
    for (int k = 0; k < n; ++k) {
        const pcbg_net& N = S->nets[B[k]];
        WinDesc& W = wd[k];
        W.x0 = N.x0; W.y0 = N.y0; W.rw = N.x1 - N.x0; W.rh = N.y1 - N.y0;
        W.pitch = int(round_up(W.rw, TILE)); W.hpad = int(round_up(W.rh, TILE));
        W.off_state = states; W.off_cell = cells;
        states += size_t(W.pitch) * W.hpad * nl;
        cells += size_t(W.pitch) * W.hpad;
        const size_t board = size_t(S->P.nx) * S->P.ny;
        const int tl = int(N.tgt / board), tc = int(N.tgt % board), ty = tc / S->P.nx, tx = tc % S->P.nx;
        W.tgt = uint32_t((size_t(tl) * W.rh + (ty - N.y0)) * W.rw + (tx - N.x0));
    }
    if (!S->cf.need(states) || !S->fl.need(states) || !S->vcf.need(cells) || !S->pbuf.need(states) ||
        !S->plen.need(n) || !S->si.need(n) || !S->sd.need(n) || !S->wd.need(n)) {
        set_error("device allocation failed");
        return -1;
    }
    // uploads from pinned staging: window descriptors, then start states, then start costs (all zero)
    const size_t o_si = round_up(n * sizeof(WinDesc), 16), o_sd = o_si + round_up(size_t(n) * 4, 16);
    const size_t o_pl = o_sd + size_t(n) * 8;
    if (!pinned(S, o_pl + size_t(n) * 4)) { set_error("pinned allocation failed"); return -1; }
    memcpy(S->hpin, wd.data(), n * sizeof(WinDesc));
    uint32_t* si = reinterpret_cast<uint32_t*>(S->hpin + o_si);
    uint64_t* sd = reinterpret_cast<uint64_t*>(S->hpin + o_sd);
    const size_t board = size_t(S->P.nx) * S->P.ny;
    for (int k = 0; k < n; ++k) {
        const pcbg_net& N = S->nets[B[k]];
        const int sl = int(N.src / board), sc = int(N.src % board), sy = sc / S->P.nx, sx = sc % S->P.nx;
        si[k] = uint32_t((size_t(sl) * wd[k].rh + (sy - N.y0)) * wd[k].rw + (sx - N.x0));
        sd[k] = 0;
    }
    cudaStream_t st = S->stream;
    cudaMemcpyAsync(S->wd.p, S->hpin, n * sizeof(WinDesc), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(S->si.p, si, n * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(S->sd.p, sd, n * 8, cudaMemcpyHostToDevice, st);
    spec_resolve_kernel<<<dim3(64, n), 256, 0, st>>>(S->P, S->wd.p, nl, S->via_cost, S->cf.p, S->fl.p, S->vcf.p);
    if (cudaGetLastError() != cudaSuccess) {   // the batch launch follows on the same stream
        set_error("window resolve failed");
        return -1;
    }
    std::vector<BatchItem> items(n);
    size_t poff = 0;
    std::vector<size_t> poffs(n);
    for (int k = 0; k < n; ++k) {
        BatchItem& b = items[k];
        memset(&b, 0, sizeof(b));
        const WinDesc& W = wd[k];
        b.rw = W.rw; b.rh = W.rh; b.nl = nl; b.pitch = W.pitch; b.hpad = W.hpad;
        memcpy(b.fac, S->fac, sizeof(b.fac));
        b.cf = S->cf.p + W.off_state; b.fl = S->fl.p + W.off_state;
        b.vcf = S->via_cost >= 0.f ? S->vcf.p + W.off_cell : nullptr;
        b.start_idx = S->si.p + k; b.start_d = S->sd.p + k; b.n_starts = 1;
        b.out = nullptr;
        b.path = S->pbuf.p + poff; b.path_cap = int(size_t(W.rw) * W.rh * nl); b.path_len = S->plen.p + k;
        poffs[k] = poff;
        poff += size_t(W.rw) * W.rh * nl;
    }
    if (solve_batch(items.data(), n, st) != 0) return -1;
    relax_ms += last_stats().kernel_ms;
    // path lengths, then every path, into pinned staging
    std::vector<int> plen(n);
    cudaMemcpyAsync(S->hpin + o_pl, S->plen.p, n * 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) { set_error("path read failed"); return -1; }
    memcpy(plen.data(), S->hpin + o_pl, n * 4);
    size_t total = 0;
    std::vector<size_t> hoff(n);
    for (int k = 0; k < n; ++k) {
        if (plen[k] < 0) { set_error("walk-back failed"); return -1; }
        hoff[k] = total;
        total += size_t(plen[k]);
    }
    if (!pinned(S, total * 4 + 16)) { set_error("pinned allocation failed"); return -1; }
    uint32_t* hp = reinterpret_cast<uint32_t*>(S->hpin);
    for (int k = 0; k < n; ++k)
        if (plen[k]) cudaMemcpyAsync(hp + hoff[k], S->pbuf.p + poffs[k], size_t(plen[k]) * 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) { set_error("path read failed"); return -1; }
    out.assign(n, {});
    for (int k = 0; k < n; ++k) {
        const WinDesc& W = wd[k];
        const size_t RN = size_t(W.rw) * W.rh;
        out[k].reserve(size_t(plen[k]));
        for (int q = 0; q < plen[k]; ++q) {
            const uint32_t r = hp[hoff[k] + q];
            const size_t l = r / RN, c = r % RN;
            const int j = int(c / W.rw), i = int(c % W.rw);
            out[k].push_back(uint32_t(l * board + size_t(W.y0 + j) * S->P.nx + (W.x0 + i)));
        }
    }
    ms += (now_s() - t0) * 1e3;
    return 0;
}

// Stamp (sign +1) or lift (-1) a path: track occupancy on each state's layer, via occupancy at each layer change
// (on the lower layer). Spans per (kind, layer), merged per row.
int stamp_path(pcbg_spec* S, const std::vector<uint32_t>& p, int sign) {
    const int nl = S->P.nl, nx = S->P.nx;
    const size_t board = size_t(nx) * S->P.ny;
    std::vector<std::vector<std::pair<int, int>>> cells(2 * nl);   // (row, col) per (kind, layer)
    for (size_t k = 0; k < p.size(); ++k) {
        const int l = int(p[k] / board), c = int(p[k] % board);
        cells[l].push_back({c / nx, c % nx});
        if (k + 1 < p.size()) {
            const int l2 = int(p[k + 1] / board), c2 = int(p[k + 1] % board);
            if (l2 != l && c2 == c) cells[nl + std::min(l, l2)].push_back({c / nx, c % nx});
        }
    }
    for (int g = 0; g < 2 * nl; ++g) {
        auto& v = cells[g];
        if (v.empty()) continue;
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        std::vector<int32_t> spans;
        for (size_t a = 0; a < v.size();) {
            size_t b = a;
            while (b + 1 < v.size() && v[b + 1].first == v[a].first && v[b + 1].second == v[b].second + 1) ++b;
            spans.push_back(v[a].first);
            spans.push_back(v[a].second);
            spans.push_back(v[b].second);
            a = b + 1;
        }
        if (pcbg_costs_stamp(S->costs, S->cls, g < nl ? 0 : 1, g % nl, spans.data(), int32_t(spans.size() / 3), sign) != 0)
            return -1;
    }
    return 0;
}

// the blocks a committed path crosses (any layer)
std::vector<uint32_t> blocks_of(const pcbg_spec* S, const std::vector<uint32_t>& p) {
    const size_t board = size_t(S->P.nx) * S->P.ny;
    const int bw = bw_of(S);
    std::vector<uint32_t> b;
    b.reserve(p.size());
    for (uint32_t s : p) {
        const int c = int(s % board), y = c / S->P.nx, x = c % S->P.nx;
        b.push_back(uint32_t((y / BS) * bw + x / BS));
    }
    std::sort(b.begin(), b.end());
    b.erase(std::unique(b.begin(), b.end()), b.end());
    return b;
}

bool window_reads(const pcbg_spec* S, const pcbg_net& N, const std::vector<uint32_t>& blocks) {
    const int bw = bw_of(S);
    const int bx0 = N.x0 / BS, bx1 = (N.x1 - 1) / BS, by0 = N.y0 / BS, by1 = (N.y1 - 1) / BS;
    for (uint32_t b : blocks) {
        const int by = int(b) / bw, bx = int(b) % bw;
        if (bx >= bx0 && bx <= bx1 && by >= by0 && by <= by1) return true;
    }
    return false;
}

}  // namespace
}  // namespace pcbg

using namespace pcbg;

extern "C" pcbg_spec* pcbg_spec_create(pcbg_costs* costs, int32_t cls, const pcbg_net* nets, int32_t n, float via_cost) {
    CostPlanes P;
    if (!costs || n < 0 || !cost_planes(costs, cls, P)) { set_error("bad cost board or class"); return nullptr; }
    const size_t board = size_t(P.nx) * P.ny;
    for (int k = 0; k < n; ++k) {
        const pcbg_net& N = nets[k];
        bool ok = N.x0 >= 0 && N.y0 >= 0 && N.x1 <= P.nx && N.y1 <= P.ny && N.x0 < N.x1 && N.y0 < N.y1;
        for (uint32_t s : {N.src, N.tgt}) {
            if (!ok) break;
            const size_t l = s / board, c = s % board;
            const int y = int(c / P.nx), x = int(c % P.nx);
            ok = l < size_t(P.nl) && x >= N.x0 && x < N.x1 && y >= N.y0 && y < N.y1;
        }
        if (!ok) { set_error("net " + std::to_string(k) + ": window or pins outside the board"); return nullptr; }
    }
    pcbg_spec* S = new pcbg_spec();
    S->costs = costs;
    S->cls = cls;
    S->P = P;
    S->via_cost = via_cost;
    const float diag = float(std::sqrt(2.0));
    for (int l = 0; l < MAX_LAYERS; ++l)
        for (int m = 0; m < 8; ++m) S->fac[l][m] = m < 4 ? 1.0f : diag;
    S->nets.assign(nets, nets + n);
    S->path.assign(n, {});
    if (cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete S;
        set_error("stream creation failed");
        return nullptr;
    }
    return S;
}

extern "C" void pcbg_spec_destroy(pcbg_spec* S) {
    if (!S) return;
    cudaStreamSynchronize(S->stream);
    S->cf.release(); S->vcf.release(); S->fl.release(); S->si.release(); S->pbuf.release();
    S->sd.release(); S->plen.release(); S->wd.release();
    if (S->hpin) cudaFreeHost(S->hpin);
    cudaStreamDestroy(S->stream);
    delete S;
}

extern "C" void pcbg_spec_set_scheduler(pcbg_spec* S, pcbg_spec_scheduler f, void* user) {
    S->sched = f;
    S->sched_user = user;
}

extern "C" void pcbg_spec_set_observer(pcbg_spec* S, pcbg_spec_observer f, void* user) {
    S->observer = f;
    S->observer_user = user;
}

extern "C" int pcbg_spec_iterate(pcbg_spec* S, float pres, int32_t policy, int32_t width, pcbg_spec_stats* st) {
    if (!S || width < 1 || policy < PCBG_SPEC_SEQUENTIAL || policy > PCBG_SPEC_LEARNED) { set_error("bad arguments"); return PCBG_ERR_FAIL; }
    if (policy == PCBG_SPEC_LEARNED && !S->sched) policy = PCBG_SPEC_PLAIN;   // the plain batching is the fallback
    const double t0 = now_s();
    pcbg_spec_stats z;
    memset(&z, 0, sizeof(z));
    // rip up every net, then the costs of this iteration
    for (auto& p : S->path)
        if (!p.empty() && stamp_path(S, p, -1) != 0) return PCBG_ERR_FAIL;
    if (pcbg_costs_rebuild(S->costs, pres, 0) != 0) return PCBG_ERR_FAIL;
    const int n = int(S->nets.size());
    for (auto& p : S->path) p.clear();
    std::vector<char> done(n, 0);
    std::vector<size_t> startver(n, 0);
    std::vector<std::vector<uint32_t>> pending(n);
    std::vector<std::vector<uint32_t>> commits;
    size_t lookahead = size_t(policy == PCBG_SPEC_SEQUENTIAL ? 1 : width);
    int cursor = 0;
    std::vector<int32_t> cand, pick;
    while (cursor < n) {
        // the nets this launch searches: not searched yet (or rejected), within the lookahead of the commit point
        cand.clear();
        for (int i = cursor; i < n && size_t(i) < size_t(cursor) + lookahead; ++i)
            if (!done[i]) cand.push_back(i);
        std::vector<int> B;
        if (policy == PCBG_SPEC_LEARNED && cand.size() > 1) {
            pick.assign(cand.size(), 0);
            if (S->sched(S->sched_user, S, cursor, cand.data(), int32_t(cand.size()), pick.data()) != 0) return PCBG_ERR_FAIL;
            for (size_t k = 0; k < cand.size(); ++k)
                if (pick[k] || cand[k] == cursor) B.push_back(cand[k]);
        } else {
            B.assign(cand.begin(), cand.end());
        }
        if (S->observer)
            for (int i : B) S->observer(S->observer_user, S, cursor, i);
        std::vector<std::vector<uint32_t>> res;
        if (run_searches(S, B, res, z.search_ms, z.relax_ms) != 0) return PCBG_ERR_FAIL;
        ++z.batches;
        z.searches += int64_t(B.size());
        for (size_t k = 0; k < B.size(); ++k) {
            pending[B[k]] = std::move(res[k]);
            startver[B[k]] = commits.size();
            done[B[k]] = 1;
        }
        while (cursor < n && done[cursor]) {
            const int c = cursor;
            bool fine = true;
            for (size_t v = startver[c]; v < commits.size() && fine; ++v)
                if (window_reads(S, S->nets[c], commits[v])) fine = false;
            if (fine) {
                if (!pending[c].empty() && stamp_path(S, pending[c], +1) != 0) return PCBG_ERR_FAIL;
                commits.push_back(blocks_of(S, pending[c]));
                S->path[c] = std::move(pending[c]);
                ++cursor;
                ++z.commits;
                if (policy != PCBG_SPEC_SEQUENTIAL) lookahead = std::min(size_t(width) * 2, lookahead + 1);
            } else {
                ++z.wasted;
                done[c] = 0;
                if (policy != PCBG_SPEC_SEQUENTIAL) lookahead = std::max<size_t>(2, lookahead * 3 / 4);
                break;
            }
        }
    }
    // nets whose paths share a state with another net's
    std::vector<std::pair<uint32_t, int>> all;
    for (int k = 0; k < n; ++k)
        for (uint32_t s : S->path[k]) all.push_back({s, k});
    std::sort(all.begin(), all.end());
    std::vector<char> hit(n, 0);
    for (size_t a = 0; a + 1 < all.size(); ++a)
        if (all[a].first == all[a + 1].first && all[a].second != all[a + 1].second) hit[all[a].second] = hit[all[a + 1].second] = 1;
    for (char h : hit) z.conflicts += h;
    z.total_ms = (now_s() - t0) * 1e3;
    if (st) *st = z;
    return 0;
}

extern "C" int32_t pcbg_spec_path(pcbg_spec* S, int32_t net, uint32_t* states, int32_t cap) {
    if (!S || net < 0 || net >= int32_t(S->nets.size())) return PCBG_ERR_FAIL;
    const auto& p = S->path[net];
    if (states) std::copy(p.begin(), p.begin() + std::min<size_t>(p.size(), size_t(std::max(cap, 0))), states);
    return int32_t(p.size());
}

extern "C" int32_t pcbg_spec_add_history(pcbg_spec* S, float inc) {
    if (!S) return PCBG_ERR_FAIL;
    std::vector<uint32_t> all;
    for (auto& p : S->path) {
        std::vector<uint32_t> u(p);
        std::sort(u.begin(), u.end());
        u.erase(std::unique(u.begin(), u.end()), u.end());
        all.insert(all.end(), u.begin(), u.end());
    }
    std::sort(all.begin(), all.end());
    std::vector<uint32_t> over;
    for (size_t a = 0; a < all.size();) {
        size_t b = a;
        while (b < all.size() && all[b] == all[a]) ++b;
        if (b - a > 1) over.push_back(all[a]);
        a = b;
    }
    if (!over.empty() && pcbg_costs_add_history(S->costs, over.data(), int32_t(over.size()), inc) != 0) return PCBG_ERR_FAIL;
    return int32_t(over.size());
}

extern "C" int32_t pcbg_spec_window_reads(pcbg_spec* S, int32_t net, const uint32_t* states, int32_t m) {
    if (!S || net < 0 || net >= int32_t(S->nets.size()) || m < 0) return PCBG_ERR_FAIL;
    std::vector<uint32_t> p(states, states + m);
    return window_reads(S, S->nets[net], blocks_of(S, p)) ? 1 : 0;
}

extern "C" int pcbg_spec_net(pcbg_spec* S, int32_t k, pcbg_net* out) {
    if (!S || k < 0 || k >= int32_t(S->nets.size())) return PCBG_ERR_FAIL;
    *out = S->nets[k];
    return 0;
}

extern "C" void pcbg_spec_board(pcbg_spec* S, int32_t* nx, int32_t* ny, int32_t* nl) {
    if (nx) *nx = S->P.nx;
    if (ny) *ny = S->P.ny;
    if (nl) *nl = S->P.nl;
}

extern "C" int pcbg_spec_costs(pcbg_spec* S, pcbg_costs** costs, int32_t* cls) {
    if (!S) return PCBG_ERR_FAIL;
    *costs = S->costs;
    *cls = S->cls;
    return 0;
}
