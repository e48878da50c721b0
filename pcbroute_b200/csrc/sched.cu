// The learned speculation scheduler: a conflict predictor that picks which nets of the lookahead window are searched
// together, so that fewer speculative searches are thrown away at the fixed-order commit.
//
// A speculative search of net i is wasted when a net j committed before it, and not yet committed when i was
// searched, lays its path through a block of i's window (the acceptance test of src/router.cpp:2211-2216). The
// predictor estimates that event per pair (i, j) from:
//   * 32 x 32 rasters of j's window, sampled from the board as it is at the search: the occupancy (tracks and vias,
//     all layers) and the history (all layers);
//   * an 8 x 8 mask of where i's window lies within j's window;
//   * 64 scalars of box overlap and pin geometry (overlap fractions, how much of j's pin-to-pin segment crosses i's
//     window, pin positions, sizes, order gap, occupancy and history inside the overlap).
// Net i's risk is 1 - prod_j (1 - p_ij) over the uncommitted nets before it; the scheduler searches i now when the
// risk is below a threshold, otherwise it waits until those nets are committed. The net at the commit point is always
// searched, and the commit order and acceptance test are untouched, so the paths do not change.
//
// Conflict logs: attached as an observer to plain speculative rounds, the scheduler records the features of every
// (searched net, earlier uncommitted net) pair at search time; after the round the labels come from the committed
// paths. Training runs the MLP's own forward and backward kernels (mlp.cu) with Adam, on the GPU.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "pcbg_internal.h"

namespace pcbg {
namespace {

struct PairDesc {
    int ix0, iy0, ix1, iy1;     // window of the searched net i
    int jx0, jy0, jx1, jy1;     // window of the earlier net j
    float jsx, jsy, jtx, jty;   // j's pins
    float gap;                  // i - j
};

constexpr int RS = 32;   // raster side
constexpr int MS = 8;    // mask side

// One block per pair: features into X[pair][MLP_D0] (bf16).
__global__ void __launch_bounds__(256) pair_features_kernel(CostPlanes P, const PairDesc* pd, __nv_bfloat16* X) {
    const PairDesc d = pd[blockIdx.x];
    __nv_bfloat16* x = X + size_t(blockIdx.x) * MLP_D0;
    __shared__ float red[4][256];
    const float jw = float(d.jx1 - d.jx0), jh = float(d.jy1 - d.jy0);
    float so = 0.f, sh = 0.f, sio = 0.f, sih = 0.f;   // sums over the raster, and over its part inside i's window
    for (int k = threadIdx.x; k < RS * RS; k += blockDim.x) {
        const int u = k % RS, v = k / RS;
        const int cx = min(d.jx1 - 1, d.jx0 + int((u + 0.5f) * jw / RS));
        const int cy = min(d.jy1 - 1, d.jy0 + int((v + 0.5f) * jh / RS));
        const size_t c = size_t(cy) * P.nx + cx;
        float occ = 0.f, hs = 0.f;
        for (int l = 0; l < P.nl; ++l) {
            occ += float(P.oc[l][c]) + float(P.ov[l][c]);
            hs += P.hist[l][c];
        }
        const float fo = fminf(occ, 8.f) * 0.25f, fh = fminf(hs / float(P.nl), 16.f) * 0.25f;
        x[k] = __float2bfloat16_rn(fo);
        x[RS * RS + k] = __float2bfloat16_rn(fh);
        so += fo;
        sh += fh;
        if (cx >= d.ix0 && cx < d.ix1 && cy >= d.iy0 && cy < d.iy1) {
            sio += fo;
            sih += fh;
        }
    }
    if (threadIdx.x < MS * MS) {
        const int u = threadIdx.x % MS, v = threadIdx.x / MS;
        const float cx = d.jx0 + (u + 0.5f) * jw / MS, cy = d.jy0 + (v + 0.5f) * jh / MS;
        const bool in = cx >= d.ix0 && cx < d.ix1 && cy >= d.iy0 && cy < d.iy1;
        x[2 * RS * RS + threadIdx.x] = __float2bfloat16_rn(in ? 1.f : 0.f);
    }
    red[0][threadIdx.x] = so;
    red[1][threadIdx.x] = sh;
    red[2][threadIdx.x] = sio;
    red[3][threadIdx.x] = sih;
    __syncthreads();
    for (int o = 128; o; o >>= 1) {
        if (threadIdx.x < o)
            for (int r = 0; r < 4; ++r) red[r][threadIdx.x] += red[r][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x < 64) {
        const int f = threadIdx.x;
        const float ox0 = fmaxf(d.ix0, d.jx0), ox1 = fminf(d.ix1, d.jx1), oy0 = fmaxf(d.iy0, d.jy0), oy1 = fminf(d.iy1, d.jy1);
        const float ow = fmaxf(0.f, ox1 - ox0), oh = fmaxf(0.f, oy1 - oy0), oa = ow * oh;
        const float ia = float(d.ix1 - d.ix0) * float(d.iy1 - d.iy0), ja = jw * jh;
        // j's pin-to-pin segment against i's window, 64 samples
        int inside = 0;
        float dmin = 1e30f;
        const float icx = 0.5f * (d.ix0 + d.ix1), icy = 0.5f * (d.iy0 + d.iy1);
        for (int s = 0; s < 64; ++s) {
            const float t = (s + 0.5f) / 64.f;
            const float px = d.jsx + t * (d.jtx - d.jsx), py = d.jsy + t * (d.jty - d.jsy);
            inside += (px >= d.ix0 && px < d.ix1 && py >= d.iy0 && py < d.iy1);
            dmin = fminf(dmin, sqrtf((px - icx) * (px - icx) + (py - icy) * (py - icy)));
        }
        const float idiag = sqrtf(ia) + 1.f;
        const float seg = sqrtf((d.jtx - d.jsx) * (d.jtx - d.jsx) + (d.jty - d.jsy) * (d.jty - d.jsy));
        const bool sin_ = d.jsx >= d.ix0 && d.jsx < d.ix1 && d.jsy >= d.iy0 && d.jsy < d.iy1;
        const bool tin = d.jtx >= d.ix0 && d.jtx < d.ix1 && d.jty >= d.iy0 && d.jty < d.iy1;
        const float nin = fmaxf(1.f, oa / fmaxf(ja, 1.f) * RS * RS);
        float v = 0.f;
        switch (f) {
            case 0: v = oa / fmaxf(ia, 1.f); break;
            case 1: v = oa / fmaxf(ja, 1.f); break;
            case 2: v = inside / 64.f; break;
            case 3: v = inside > 0 ? 1.f : 0.f; break;
            case 4: v = sin_ ? 1.f : 0.f; break;
            case 5: v = tin ? 1.f : 0.f; break;
            case 6: v = fminf(dmin / idiag, 4.f); break;
            case 7: v = log2f(fmaxf(ia, 1.f)) / 16.f; break;
            case 8: v = log2f(fmaxf(ja, 1.f)) / 16.f; break;
            case 9: v = fminf(d.gap, 64.f) / 32.f; break;
            case 10: v = red[2][0] / nin; break;
            case 11: v = red[3][0] / nin; break;
            case 12: v = red[0][0] / (RS * RS); break;
            case 13: v = red[1][0] / (RS * RS); break;
            case 14: v = fminf(seg, 512.f) / 128.f; break;
            case 15: v = 1.f; break;
            case 16: v = (d.jsx - icx) / idiag; break;
            case 17: v = (d.jsy - icy) / idiag; break;
            case 18: v = (d.jtx - icx) / idiag; break;
            case 19: v = (d.jty - icy) / idiag; break;
            default: v = 0.f;
        }
        x[2 * RS * RS + MS * MS + f] = __float2bfloat16_rn(v);
    }
}

// rows idx[0..n) of X into Y (n rows), zero rows up to m
__global__ void gather_rows_kernel(const __nv_bfloat16* X, const int* idx, int n, int m, __nv_bfloat16* Y) {
    const int r = blockIdx.x;
    const uint4 z = make_uint4(0, 0, 0, 0);
    const uint4* src = r < n ? reinterpret_cast<const uint4*>(X + size_t(idx[r]) * MLP_D0) : nullptr;
    uint4* dst = reinterpret_cast<uint4*>(Y + size_t(r) * MLP_D0);
    for (int k = threadIdx.x; k < MLP_D0 / 8; k += blockDim.x) dst[k] = src ? src[k] : z;
    (void)m;
}

}  // namespace
}  // namespace pcbg

using namespace pcbg;

struct pcbg_sched {
    Mlp net;
    cudaStream_t stream = nullptr;
    float threshold = 0.5f;
    // conflict log: features on the device, pair geometry and labels on the host
    __nv_bfloat16* X = nullptr;
    size_t xcap = 0, nlog = 0;
    std::vector<int> li, lj;        // logged pairs (net i searched, earlier net j), in log order
    std::vector<float> label;       // 0 / 1, filled by pcbg_sched_label (NaN until then)
    size_t labelled = 0;
    // scratch
    PairDesc* pd = nullptr;
    size_t pdcap = 0;
    __nv_bfloat16* xb = nullptr;    // a batch of features
    size_t xbcap = 0;
    float *yb = nullptr, *wb = nullptr, *pb = nullptr;
    int* ib = nullptr;
    size_t ybcap = 0, wbcap = 0, pbcap = 0, ibcap = 0;
    int64_t scored = 0, deferred = 0;
};

namespace {

template <class T> bool grow(T*& p, size_t& cap, size_t n) {
    if (cap >= n) return true;
    const size_t c = std::max(n, cap * 2);
    T* q = nullptr;
    if (cudaMalloc(&q, c * sizeof(T)) != cudaSuccess) return false;
    if (p) {
        cudaDeviceSynchronize();   // kernels still writing the old buffer run on non-blocking streams
        cudaMemcpy(q, p, cap * sizeof(T), cudaMemcpyDeviceToDevice);
        cudaFree(p);
    }
    p = q;
    cap = c;
    return true;
}

bool pair_of(pcbg_spec* s, int i, int j, int nx, PairDesc& d) {
    pcbg_net a, b;
    if (pcbg_spec_net(s, i, &a) != 0 || pcbg_spec_net(s, j, &b) != 0) return false;
    d.ix0 = a.x0; d.iy0 = a.y0; d.ix1 = a.x1; d.iy1 = a.y1;
    d.jx0 = b.x0; d.jy0 = b.y0; d.jx1 = b.x1; d.jy1 = b.y1;
    int32_t nxv = 0, nyv = 0;
    pcbg_spec_board(s, &nxv, &nyv, nullptr);
    const size_t board = size_t(nxv) * nyv;
    const int sc = int(b.src % board), tc = int(b.tgt % board);
    d.jsx = float(sc % nx); d.jsy = float(sc / nx);
    d.jtx = float(tc % nx); d.jty = float(tc / nx);
    d.gap = float(i - j);
    return true;
}

// Whether net j's path can invalidate a search of net i at all: a path stays inside its own window, and a commit
// invalidates i only through blocks of i's window, so pairs whose windows share no block never conflict.
bool blocks_meet(pcbg_spec* s, int i, int j) {
    pcbg_net a, b;
    if (pcbg_spec_net(s, i, &a) != 0 || pcbg_spec_net(s, j, &b) != 0) return true;
    const int B = SPEC_BLOCK;
    return a.x0 / B <= (b.x1 - 1) / B && b.x0 / B <= (a.x1 - 1) / B && a.y0 / B <= (b.y1 - 1) / B &&
           b.y0 / B <= (a.y1 - 1) / B;
}

// features of pairs into X rows [row0, row0 + n) (stream-ordered on the scheduler's stream)
int features(pcbg_sched* S, pcbg_spec* s, const std::vector<PairDesc>& pds, __nv_bfloat16* X) {
    if (pds.empty()) return 0;
    CostPlanes P;
    pcbg_costs* costs = nullptr;
    int32_t cls = 0;
    if (pcbg_spec_costs(s, &costs, &cls) != 0 || !cost_planes(costs, cls, P)) return -1;
    if (!grow(S->pd, S->pdcap, pds.size())) return -1;
    cudaMemcpyAsync(S->pd, pds.data(), pds.size() * sizeof(PairDesc), cudaMemcpyHostToDevice, S->stream);
    pair_features_kernel<<<unsigned(pds.size()), 256, 0, S->stream>>>(P, S->pd, X);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int sched_pick(void* user, pcbg_spec* s, int32_t cursor, const int32_t* cand, int32_t n, int32_t* pick) {
    pcbg_sched* S = static_cast<pcbg_sched*>(user);
    int32_t nx = 0, ny = 0;
    pcbg_spec_board(s, &nx, &ny, nullptr);
    std::vector<PairDesc> pds;
    std::vector<int> owner;
    for (int k = 0; k < n; ++k) {
        const int i = cand[k];
        for (int j = cursor; j < i; ++j) {
            if (!blocks_meet(s, i, j)) continue;   // p_ij = 0
            PairDesc d;
            if (!pair_of(s, i, j, nx, d)) return -1;
            pds.push_back(d);
            owner.push_back(k);
        }
    }
    for (int k = 0; k < n; ++k) pick[k] = cand[k] == cursor ? 1 : 0;
    if (pds.empty()) {   // no open net shares a block with an uncommitted one: all are safe
        for (int k = 0; k < n; ++k) pick[k] = 1;
        return 0;
    }
    const size_t B = round_up(pds.size(), 64);
    if (!grow(S->xb, S->xbcap, B * MLP_D0) || !grow(S->pb, S->pbcap, B)) return -1;
    cudaMemsetAsync(S->xb, 0, B * MLP_D0 * 2, S->stream);
    if (features(S, s, pds, S->xb) != 0) return -1;
    if (S->net.forward(S->stream, S->xb, int(B), S->pb) != 0) return -1;
    std::vector<float> p(pds.size());
    cudaMemcpyAsync(p.data(), S->pb, p.size() * 4, cudaMemcpyDeviceToHost, S->stream);
    if (cudaStreamSynchronize(S->stream) != cudaSuccess) return -1;
    std::vector<double> keep(n, 1.0);
    for (size_t q = 0; q < pds.size(); ++q) keep[owner[q]] *= 1.0 - double(p[q]);
    for (int k = 0; k < n; ++k) {
        if (cand[k] == cursor) continue;
        ++S->scored;
        if (1.0 - keep[k] < double(S->threshold)) pick[k] = 1;
        else ++S->deferred;
    }
    return 0;
}

void sched_log(void* user, pcbg_spec* s, int32_t cursor, int32_t net) {
    pcbg_sched* S = static_cast<pcbg_sched*>(user);
    if (net <= cursor) return;
    int32_t nx = 0, ny = 0;
    pcbg_spec_board(s, &nx, &ny, nullptr);
    std::vector<PairDesc> pds;
    for (int j = cursor; j < net; ++j) {
        if (!blocks_meet(s, net, j)) continue;   // never a conflict: not logged
        PairDesc d;
        if (!pair_of(s, net, j, nx, d)) return;
        pds.push_back(d);
        S->li.push_back(net);
        S->lj.push_back(j);
        S->label.push_back(std::nanf(""));
    }
    if (!grow(S->X, S->xcap, (S->nlog + pds.size()) * MLP_D0)) {
        set_error("conflict log allocation failed");
        S->li.resize(S->nlog); S->lj.resize(S->nlog); S->label.resize(S->nlog);
        return;
    }
    if (features(S, s, pds, S->X + S->nlog * MLP_D0) != 0) {
        S->li.resize(S->nlog); S->lj.resize(S->nlog); S->label.resize(S->nlog);
        return;
    }
    S->nlog += pds.size();
}

}  // namespace

extern "C" pcbg_sched* pcbg_sched_create(uint64_t seed) {
    pcbg_sched* S = new pcbg_sched();
    if (!S->net.init(seed) || cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete S;
        set_error("scheduler allocation failed");
        return nullptr;
    }
    return S;
}

extern "C" void pcbg_sched_destroy(pcbg_sched* S) {
    if (!S) return;
    cudaStreamSynchronize(S->stream);
    for (void* p : {static_cast<void*>(S->X), static_cast<void*>(S->pd), static_cast<void*>(S->xb),
                    static_cast<void*>(S->yb), static_cast<void*>(S->wb), static_cast<void*>(S->pb),
                    static_cast<void*>(S->ib)})
        if (p) cudaFree(p);
    cudaStreamDestroy(S->stream);
    delete S;
}

extern "C" void pcbg_sched_attach(pcbg_sched* S, pcbg_spec* s, float threshold) {
    S->threshold = threshold;
    pcbg_spec_set_scheduler(s, sched_pick, S);
}

extern "C" void pcbg_sched_attach_logger(pcbg_sched* S, pcbg_spec* s) { pcbg_spec_set_observer(s, sched_log, S); }

extern "C" int64_t pcbg_sched_label(pcbg_sched* S, pcbg_spec* s) {
    int64_t pos = 0;
    std::vector<std::vector<uint32_t>> paths;
    for (size_t q = S->labelled; q < S->nlog; ++q) {
        const int j = S->lj[q];
        const int32_t n = pcbg_spec_path(s, j, nullptr, 0);
        std::vector<uint32_t> p(std::max(n, 0));
        if (n > 0) pcbg_spec_path(s, j, p.data(), n);
        const int32_t r = pcbg_spec_window_reads(s, S->li[q], p.data(), int32_t(p.size()));
        if (r < 0) return PCBG_ERR_FAIL;
        S->label[q] = float(r);
        pos += r;
    }
    S->labelled = S->nlog;
    return pos;
}

extern "C" int64_t pcbg_sched_log_size(pcbg_sched* S, int64_t* positives) {
    int64_t p = 0;
    for (size_t q = 0; q < S->labelled; ++q) p += S->label[q] > 0.5f;
    if (positives) *positives = p;
    return int64_t(S->labelled);
}

extern "C" int pcbg_sched_train(pcbg_sched* S, int32_t epochs, float lr, int32_t batch, uint64_t seed, float* loss_out) {
    const size_t n = S->labelled;
    if (n == 0 || batch < 64 || batch % 64) { set_error("nothing labelled, or batch not a multiple of 64"); return PCBG_ERR_FAIL; }
    if (!grow(S->xb, S->xbcap, size_t(batch) * MLP_D0) || !grow(S->yb, S->ybcap, size_t(batch)) ||
        !grow(S->wb, S->wbcap, size_t(batch)) || !grow(S->ib, S->ibcap, size_t(batch)))
        return PCBG_ERR_FAIL;
    // positives and negatives weighted to equal total weight
    size_t npos = 0;
    for (size_t q = 0; q < n; ++q) npos += S->label[q] > 0.5f;
    const float wpos = npos ? float(n) / (2.f * npos) : 1.f, wneg = npos < n ? float(n) / (2.f * (n - npos)) : 1.f;
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    uint64_t st = seed;
    auto rnd = [&]() {
        st = st * 6364136223846793005ull + 1442695040888963407ull;
        return st >> 33;
    };
    float last = 0.f;
    std::vector<float> y(batch), w(batch);
    for (int e = 0; e < epochs; ++e) {
        for (size_t k = n - 1; k > 0; --k) std::swap(order[k], order[rnd() % (k + 1)]);
        double esum = 0.0;
        int nb = 0;
        for (size_t b0 = 0; b0 < n; b0 += size_t(batch)) {
            const int m = int(std::min<size_t>(batch, n - b0));
            float wsum = 0.f;
            for (int r = 0; r < batch; ++r) {
                if (r < m) {
                    const float lab = S->label[order[b0 + r]];
                    y[r] = lab;
                    w[r] = lab > 0.5f ? wpos : wneg;
                    wsum += w[r];
                } else {
                    y[r] = 0.f;
                    w[r] = 0.f;
                }
            }
            cudaMemcpyAsync(S->ib, order.data() + b0, size_t(m) * 4, cudaMemcpyHostToDevice, S->stream);
            cudaMemcpyAsync(S->yb, y.data(), size_t(batch) * 4, cudaMemcpyHostToDevice, S->stream);
            cudaMemcpyAsync(S->wb, w.data(), size_t(batch) * 4, cudaMemcpyHostToDevice, S->stream);
            gather_rows_kernel<<<batch, 128, 0, S->stream>>>(S->X, S->ib, m, batch, S->xb);
            float loss = 0.f;
            if (S->net.forward(S->stream, S->xb, batch, nullptr) != 0) return PCBG_ERR_FAIL;
            if (S->net.backward(S->stream, S->xb, S->yb, S->wb, wsum, batch, &loss) != 0) return PCBG_ERR_FAIL;
            if (S->net.adam(S->stream, lr) != 0) return PCBG_ERR_FAIL;
            if (cudaStreamSynchronize(S->stream) != cudaSuccess) return PCBG_ERR_FAIL;
            esum += loss;
            ++nb;
        }
        last = float(esum / std::max(nb, 1));
    }
    if (loss_out) *loss_out = last;
    return 0;
}

extern "C" void pcbg_sched_counts(pcbg_sched* S, int64_t* scored, int64_t* deferred) {
    if (scored) *scored = S->scored;
    if (deferred) *deferred = S->deferred;
}

// ---- host-array entry points of the network (the gradient check against the CPU oracle) ----

extern "C" int64_t pcbg_sched_nparams(pcbg_sched* S) { return int64_t(S->net.nparams); }

extern "C" int pcbg_sched_get_params(pcbg_sched* S, float* out) {
    return cudaMemcpy(out, S->net.master, S->net.nparams * 4, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : PCBG_ERR_FAIL;
}

extern "C" int pcbg_sched_set_params(pcbg_sched* S, const float* in) { return S->net.set_params(in) == 0 ? 0 : PCBG_ERR_FAIL; }

/* x: B rows of MLP_D0 bf16 bit patterns (B a multiple of 64). p: B probabilities. */
extern "C" int pcbg_sched_forward_host(pcbg_sched* S, const uint16_t* x, int32_t B, float* p) {
    if (B <= 0 || B % 64 || !grow(S->xb, S->xbcap, size_t(B) * MLP_D0) || !grow(S->pb, S->pbcap, size_t(B))) return PCBG_ERR_FAIL;
    cudaMemcpyAsync(S->xb, x, size_t(B) * MLP_D0 * 2, cudaMemcpyHostToDevice, S->stream);
    if (S->net.forward(S->stream, S->xb, B, S->pb) != 0) return PCBG_ERR_FAIL;
    cudaMemcpyAsync(p, S->pb, size_t(B) * 4, cudaMemcpyDeviceToHost, S->stream);
    return cudaStreamSynchronize(S->stream) == cudaSuccess ? 0 : PCBG_ERR_FAIL;
}

/* Gradients (packed like the parameters) of sum_b w_b BCE(z_b, y_b) / sum_b w_b, and that loss. */
extern "C" int pcbg_sched_grad_host(pcbg_sched* S, const uint16_t* x, const float* y, const float* w, int32_t B,
                                    float* grad, float* loss) {
    if (B <= 0 || B % 64) return PCBG_ERR_FAIL;
    if (!grow(S->xb, S->xbcap, size_t(B) * MLP_D0) || !grow(S->yb, S->ybcap, size_t(B)) || !grow(S->wb, S->wbcap, size_t(B)))
        return PCBG_ERR_FAIL;
    float* yd = S->yb;
    float* wd = S->wb;
    float wsum = 0.f;
    for (int b = 0; b < B; ++b) wsum += w[b];
    cudaMemcpyAsync(S->xb, x, size_t(B) * MLP_D0 * 2, cudaMemcpyHostToDevice, S->stream);
    cudaMemcpyAsync(yd, y, size_t(B) * 4, cudaMemcpyHostToDevice, S->stream);
    cudaMemcpyAsync(wd, w, size_t(B) * 4, cudaMemcpyHostToDevice, S->stream);
    int rc = S->net.forward(S->stream, S->xb, B, nullptr);
    if (rc == 0) rc = S->net.backward(S->stream, S->xb, yd, wd, wsum, B, loss);
    if (rc == 0 && cudaMemcpyAsync(grad, S->net.grad, S->net.nparams * 4, cudaMemcpyDeviceToHost, S->stream) != cudaSuccess) rc = -1;
    if (cudaStreamSynchronize(S->stream) != cudaSuccess) rc = -1;
    return rc == 0 ? 0 : PCBG_ERR_FAIL;
}

// ---- the learned scheduler inside pcbroute's own router (route_waves, src/router.cpp:2119-2242) ----
//
// The router's worker takes the next net of the commit order within the lookahead (src/router.cpp:2172-2178); a
// search is wasted when a commit made after it started changes a 16 x 16 block it read (src/router.cpp:2200-2216).
// A router built with the hooks (baseline/router_hooks.h) reports, per route_waves call, each net's search window
// and pins, the start of each search, each commit and each verdict. In log mode the scheduler records the features
// of every (searched net, uncommitted earlier net) pair at search start and labels them at the verdict: positive
// when the earlier net's commit changed a block the search read. In learned mode it lets a worker start net i ahead
// of the commit point only while the predicted risk 1 - prod_j (1 - p_ij) stays below the threshold; the net at
// the commit point is always searched, and the commit order and check are the router's own, so the session cannot
// change. Mode, model and log files come from the environment:
//   PCBG_SCHED=log|learned, PCBG_SCHED_LOG=<file> (log mode: labelled pairs appended), PCBG_SCHED_MODEL=<file>
//   (learned mode: parameters as written by pcbg_sched_get_params), PCBG_SCHED_THRESHOLD (default 0.5).

namespace {

constexpr int RBS = 16;   // the router's block side (src/router.cpp:404)

struct RPair {
    int i, j;
    int64_t row;   // row of the pending log
};

struct RSched {
    std::mutex mu;
    int mode = -1;             // 0 off, 1 log, 2 learned
    float threshold = 0.5f;
    std::string log_path;
    pcbg_sched* S = nullptr;
    std::vector<pcbg_rnet> nets;
    std::vector<int64_t> commit_of;   // per position: index of the commit that committed it (-1: none yet)
    std::vector<RPair> pending;       // logged pairs awaiting their verdict
    __nv_bfloat16* X = nullptr;       // pending features (device)
    size_t xcap = 0, nx_rows = 0;
    std::vector<uint16_t> out_x;      // labelled rows not yet written
    std::vector<uint8_t> out_y;
    int64_t cache_pos = -1, cache_ver = -1, cache_cur = -1;
    int cache_val = 1;
    uint64_t rng = 0x9E3779B97F4A7C15ull;
    pcbg_rsched_stats st{};
};

RSched g_rs;

void rs_init() {
    if (g_rs.mode >= 0) return;
    g_rs.mode = 0;
    const char* m = std::getenv("PCBG_SCHED");
    if (!m) return;
    const std::string mode(m);
    if (const char* t = std::getenv("PCBG_SCHED_THRESHOLD")) g_rs.threshold = float(std::atof(t));
    // a scheduler asked for but not usable leaves the router's own speculation, and says so once
    auto off = [](const char* why, const char* what) {
        std::fprintf(stderr, "pcbg: PCBG_SCHED=%s: %s; speculation stays the router's own\n", what, why);
    };
    if (mode == "log") {
        const char* p = std::getenv("PCBG_SCHED_LOG");
        if (!p) return off("PCBG_SCHED_LOG is not set", "log");
        g_rs.log_path = p;
        g_rs.S = pcbg_sched_create(1);
        if (!g_rs.S) return off("the predictor could not be created on the device", "log");
        g_rs.mode = 1;
    } else if (mode == "learned") {
        const char* p = std::getenv("PCBG_SCHED_MODEL");
        if (!p) return off("PCBG_SCHED_MODEL is not set", "learned");
        g_rs.S = pcbg_sched_create(1);
        if (!g_rs.S) return off("the predictor could not be created on the device", "learned");
        std::vector<float> w(g_rs.S->net.nparams);
        FILE* f = std::fopen(p, "rb");
        if (!f) return off("the model file cannot be opened", "learned");
        const size_t got = std::fread(w.data(), 4, w.size(), f);
        std::fclose(f);
        if (got != w.size()) return off("the model file holds fewer parameters than the predictor", "learned");
        if (pcbg_sched_set_params(g_rs.S, w.data()) != 0) return off("the parameters could not be loaded", "learned");
        g_rs.mode = 2;
    } else {
        off("unknown mode (log or learned)", m);
    }
}

bool rs_blocks_meet(const pcbg_rnet& a, const pcbg_rnet& b) {
    return a.x0 / RBS <= (b.x1 - 1) / RBS && b.x0 / RBS <= (a.x1 - 1) / RBS && a.y0 / RBS <= (b.y1 - 1) / RBS &&
           b.y0 / RBS <= (a.y1 - 1) / RBS;
}

PairDesc rs_pair(int i, int j) {
    const pcbg_rnet &a = g_rs.nets[i], &b = g_rs.nets[j];
    PairDesc d;
    d.ix0 = a.x0; d.iy0 = a.y0; d.ix1 = a.x1; d.iy1 = a.y1;
    d.jx0 = b.x0; d.jy0 = b.y0; d.jx1 = b.x1; d.jy1 = b.y1;
    d.jsx = b.sx; d.jsy = b.sy; d.jtx = b.tx; d.jty = b.ty;
    d.gap = float(i - j);
    return d;
}

// features of pairs (i, j) for j in js into X (stream-ordered on the scheduler's stream)
int rs_features(const std::vector<PairDesc>& pds, __nv_bfloat16* X) {
    CostPlanes P;
    if (!mirror_planes(0, P)) return -1;
    pcbg_sched* S = g_rs.S;
    if (!grow(S->pd, S->pdcap, pds.size())) return -1;
    cudaMemcpyAsync(S->pd, pds.data(), pds.size() * sizeof(PairDesc), cudaMemcpyHostToDevice, S->stream);
    pair_features_kernel<<<unsigned(pds.size()), 256, 0, S->stream>>>(P, S->pd, X);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

void rs_flush() {
    if (g_rs.mode != 1 || g_rs.out_y.empty()) return;
    FILE* f = std::fopen(g_rs.log_path.c_str(), "ab");
    if (!f) return;
    // record: int64 rows, then rows x MLP_D0 bf16, then rows labels (u8)
    const int64_t rows = int64_t(g_rs.out_y.size());
    std::fwrite(&rows, 8, 1, f);
    std::fwrite(g_rs.out_x.data(), 2, g_rs.out_x.size(), f);
    std::fwrite(g_rs.out_y.data(), 1, g_rs.out_y.size(), f);
    std::fclose(f);
    g_rs.out_x.clear();
    g_rs.out_y.clear();
}

}  // namespace

extern "C" int pcbg_rsched_mode(void) {
    std::lock_guard<std::mutex> g(g_rs.mu);
    rs_init();
    return g_rs.mode;
}

extern "C" void pcbg_rsched_begin(int32_t n) {
    std::lock_guard<std::mutex> g(g_rs.mu);
    rs_init();
    g_rs.nets.assign(n > 0 ? n : 0, pcbg_rnet{});
    g_rs.commit_of.assign(n > 0 ? n : 0, -1);
    g_rs.pending.clear();
    g_rs.nx_rows = 0;
    g_rs.cache_pos = -1;
    ++g_rs.st.calls;
}

extern "C" void pcbg_rsched_net(int32_t pos, const pcbg_rnet* net) {
    std::lock_guard<std::mutex> g(g_rs.mu);
    if (pos >= 0 && pos < int(g_rs.nets.size()) && net) g_rs.nets[pos] = *net;
}

extern "C" int32_t pcbg_rsched_allow(int32_t pos, int32_t cursor, int64_t version) {
    std::lock_guard<std::mutex> g(g_rs.mu);
    if (g_rs.mode != 2 || pos <= cursor || pos >= int(g_rs.nets.size())) return 1;
    if (g_rs.cache_pos == pos && g_rs.cache_ver == version && g_rs.cache_cur == cursor) return g_rs.cache_val;
    std::vector<PairDesc> pds;
    for (int j = cursor; j < pos; ++j)
        if (rs_blocks_meet(g_rs.nets[pos], g_rs.nets[j])) pds.push_back(rs_pair(pos, j));
    int allow = 1;
    if (!pds.empty()) {
        pcbg_sched* S = g_rs.S;
        const size_t B = round_up(pds.size(), 64);
        if (!grow(S->xb, S->xbcap, B * MLP_D0) || !grow(S->pb, S->pbcap, B)) return 1;
        cudaMemsetAsync(S->xb, 0, B * MLP_D0 * 2, S->stream);
        if (rs_features(pds, S->xb) != 0 || S->net.forward(S->stream, S->xb, int(B), S->pb) != 0) return 1;
        std::vector<float> p(pds.size());
        cudaMemcpyAsync(p.data(), S->pb, p.size() * 4, cudaMemcpyDeviceToHost, S->stream);
        if (cudaStreamSynchronize(S->stream) != cudaSuccess) return 1;
        double keep = 1.0;
        for (float x : p) keep *= 1.0 - double(x);
        allow = 1.0 - keep < double(g_rs.threshold) ? 1 : 0;
        ++g_rs.st.scored;
        if (!allow) ++g_rs.st.deferred;
    }
    g_rs.cache_pos = pos; g_rs.cache_ver = version; g_rs.cache_cur = cursor; g_rs.cache_val = allow;
    return allow;
}

extern "C" void pcbg_rsched_started(int32_t pos, int32_t cursor, int64_t version) {
    (void)version;
    std::lock_guard<std::mutex> g(g_rs.mu);
    ++g_rs.st.searches;
    if (pos > cursor) ++g_rs.st.speculative;
    if (g_rs.mode != 1 || pos <= cursor || pos >= int(g_rs.nets.size())) return;
    std::vector<PairDesc> pds;
    std::vector<int> js;
    for (int j = cursor; j < pos; ++j)
        if (rs_blocks_meet(g_rs.nets[pos], g_rs.nets[j])) { pds.push_back(rs_pair(pos, j)); js.push_back(j); }
    if (pds.empty()) return;
    if (!grow(g_rs.X, g_rs.xcap, (g_rs.nx_rows + pds.size()) * MLP_D0)) return;
    if (rs_features(pds, g_rs.X + g_rs.nx_rows * MLP_D0) != 0) return;
    for (size_t k = 0; k < js.size(); ++k) g_rs.pending.push_back({pos, js[k], int64_t(g_rs.nx_rows + k)});
    g_rs.nx_rows += pds.size();
}

extern "C" void pcbg_rsched_committed(int32_t pos, int64_t commit_index) {
    std::lock_guard<std::mutex> g(g_rs.mu);
    if (pos >= 0 && pos < int(g_rs.commit_of.size())) g_rs.commit_of[pos] = commit_index;
    ++g_rs.st.commits;
}

extern "C" void pcbg_rsched_verdict(int32_t pos, int32_t accepted, const int64_t* hit_commits, int32_t nhit) {
    std::lock_guard<std::mutex> g(g_rs.mu);
    if (!accepted) ++g_rs.st.wasted;
    if (g_rs.mode != 1) return;
    std::vector<RPair> rest;
    std::vector<std::pair<int64_t, uint8_t>> lab;
    for (const RPair& p : g_rs.pending) {
        if (p.i != pos) { rest.push_back(p); continue; }
        const int64_t c = p.j < int(g_rs.commit_of.size()) ? g_rs.commit_of[p.j] : -1;
        bool hit = false;
        for (int k = 0; k < nhit && !hit; ++k) hit = hit_commits[k] == c;
        // negatives are sampled (1 in 4) to bound the log; positives are all kept
        g_rs.rng = g_rs.rng * 6364136223846793005ull + 1442695040888963407ull;
        if (!hit && (g_rs.rng >> 33) % 4 != 0) continue;
        lab.push_back({p.row, uint8_t(hit ? 1 : 0)});
    }
    g_rs.pending.swap(rest);
    if (lab.empty()) return;
    const size_t old = g_rs.out_x.size();
    g_rs.out_x.resize(old + lab.size() * MLP_D0);
    cudaStreamSynchronize(g_rs.S->stream);
    for (size_t k = 0; k < lab.size(); ++k) {
        cudaMemcpy(g_rs.out_x.data() + old + k * MLP_D0, g_rs.X + size_t(lab[k].first) * MLP_D0, MLP_D0 * 2,
                   cudaMemcpyDeviceToHost);
        g_rs.out_y.push_back(lab[k].second);
        g_rs.st.logged += 1;
        g_rs.st.positives += lab[k].second;
    }
    if (g_rs.out_y.size() >= 4096) rs_flush();
}

extern "C" void pcbg_rsched_end(void) {
    std::lock_guard<std::mutex> g(g_rs.mu);
    rs_flush();
    g_rs.pending.clear();
    g_rs.nx_rows = 0;
}

extern "C" void pcbg_rsched_get_stats(pcbg_rsched_stats* out) {
    std::lock_guard<std::mutex> g(g_rs.mu);
    if (out) *out = g_rs.st;
}

extern "C" int pcbg_sched_add_log_host(pcbg_sched* S, const uint16_t* x, const float* y, int64_t n) {
    if (n <= 0) return 0;
    if (S->labelled != S->nlog) { set_error("unlabelled pairs pending"); return PCBG_ERR_FAIL; }
    if (!grow(S->X, S->xcap, (S->nlog + size_t(n)) * MLP_D0)) return PCBG_ERR_FAIL;
    if (cudaMemcpy(S->X + S->nlog * MLP_D0, x, size_t(n) * MLP_D0 * 2, cudaMemcpyHostToDevice) != cudaSuccess)
        return PCBG_ERR_FAIL;
    for (int64_t k = 0; k < n; ++k) {
        S->li.push_back(-1);
        S->lj.push_back(-1);
        S->label.push_back(y[k]);
    }
    S->nlog += size_t(n);
    S->labelled = S->nlog;
    return 0;
}
