// Device-resident congestion cost maps: the present / history cost update of PathFinder on the B200.
//
// pcbroute keeps, per net class, the cost a search reads at every (layer, cell) and at every via cell
// (RClass::cst / vcst, src/router.cpp:197-211). They follow from the static owner grids, the other nets' occupancy,
// the history and the present-congestion factor:
//   track:  INF if static-blocked (or occupied while legalising), else ((1 + hist) * (1 + pres * occ)) * gnd,
//           negated where the cell is some net's own copper                           (cost_xp, router.cpp:386-394)
//   via:    INF likewise, else (1 + sum_l hist / NL) * (1 + pres * sum_l ov), negated on own copper
//                                                                                     (vcost_xp, router.cpp:396-405)
// rebuild_costs recomputes every cell each round on one host thread per (class, layer) (router.cpp:409-420);
// refresh_costs recomputes the cells a commit stamped (router.cpp:1880-1890); count_conflicts adds the history
// increment on conflicting path cells (router.cpp:1970-1999). Here all of it stays in HBM:
//   * costs_rebuild_kernel: one pass, 8 cells per thread with 128-bit loads and stores, every class per thread so
//     the history / ground planes shared by the classes are read once;
//   * costs_stamp_kernel: occupancy +-1 over uploaded spans and the refresh of those cells, in one launch;
//   * costs_history_kernel: history += increment at listed path states.
// The float operations are the reference's, in its order, one IEEE operation at a time (no contraction), so the
// maps are bit-identical to the host router's.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "pcbg_internal.h"

namespace pcbg {
namespace {

constexpr float CINF = 1e30f;
constexpr uint16_t FREE = 0, BLOCK = 0xFFFF;

struct CostDev {
    int n, nl, nclasses, has_gnd;
    // per class: [nl][n] / [n] device planes
    const uint16_t* st[MAX_LAYERS * 8];
    uint8_t* oc[MAX_LAYERS * 8];
    uint8_t* ov[MAX_LAYERS * 8];
    float* cst[MAX_LAYERS * 8];
    const uint16_t* vst[8];
    float* vcst[8];
    const float* hist[MAX_LAYERS];
    const float* gnd[MAX_LAYERS];     // null: no ground factor on that layer
};

// src/router.cpp:386-394 with own = 0
__device__ __forceinline__ float cost_track(uint16_t s, int occ, float h, const float* gnd, size_t c, float pres, int hard) {
    if (s == BLOCK) return CINF;
    if (hard && occ > 0) return CINF;
    const float a = __fadd_rn(1.f, h);
    const float b = __fadd_rn(1.f, __fmul_rn(pres, float(occ > 0 ? occ : 0)));
    float v = __fmul_rn(a, b);
    if (gnd) v = __fmul_rn(v, gnd[c]);
    return s == FREE ? v : -v;
}

// src/router.cpp:396-405 with own = 0
__device__ __forceinline__ float cost_via(const CostDev& D, int k, size_t c, float pres, int hard) {
    const uint16_t s = D.vst[k][c];
    if (s == BLOCK) return CINF;
    int occ = 0;
    float hs = 0.f;
    for (int l = 0; l < D.nl; ++l) {
        occ += D.ov[k * MAX_LAYERS + l][c];
        hs = __fadd_rn(hs, D.hist[l][c]);
    }
    if (hard && occ > 0) return CINF;
    const float a = __fadd_rn(1.f, __fdiv_rn(hs, float(D.nl)));
    const float b = __fadd_rn(1.f, __fmul_rn(pres, float(occ > 0 ? occ : 0)));
    const float v = __fmul_rn(a, b);
    return s == FREE ? v : -v;
}

// via cost of one cell from its summed history and via occupancy (src/router.cpp:396-405 with own = 0)
__device__ __forceinline__ float via_of(uint16_t s, int occ, float a, float pres, int hard) {
    if (s == BLOCK) return CINF;
    if (hard && occ > 0) return CINF;
    const float v = __fmul_rn(a, __fadd_rn(1.f, __fmul_rn(pres, float(occ > 0 ? occ : 0))));
    return s == FREE ? v : -v;
}

// Every cell of every class, 4 cells per thread and one pass: the history of every layer is loaded once (128-bit)
// and serves both the track costs of its layer and the via costs' layer sum. Per class, the owners (64-bit, 4
// cells) and occupancy (32-bit, 4 cells) of every layer and the via grids are loaded before any cost is computed,
// so a thread keeps them all in flight at once. The history sum runs in layer order, as vcost_xp does.
__global__ void __launch_bounds__(256) costs_rebuild_kernel(CostDev D, float pres, int hard) {
    const size_t n = size_t(D.n);
    const int nl = D.nl, nc = D.nclasses;
    const size_t quads = (n + 3) / 4;
    for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < quads; q += size_t(gridDim.x) * blockDim.x) {
        const size_t c0 = q * 4;
        if (c0 + 4 > n) {   // ragged end of the board
            for (size_t c = c0; c < n; ++c) {
                float hsum = 0.f;
                for (int l = 0; l < nl; ++l) hsum = __fadd_rn(hsum, D.hist[l][c]);
                const float a = __fadd_rn(1.f, __fdiv_rn(hsum, float(nl)));
                for (int k = 0; k < nc; ++k) {
                    int occ = 0;
                    for (int l = 0; l < nl; ++l) {
                        const int id = k * MAX_LAYERS + l;
                        D.cst[id][c] = cost_track(D.st[id][c], D.oc[id][c], D.hist[l][c], D.gnd[l], c, pres, hard);
                        occ += D.ov[id][c];
                    }
                    D.vcst[k][c] = via_of(D.vst[k][c], occ, a, pres, hard);
                }
            }
            continue;
        }
        float4 hv[MAX_LAYERS];
        #pragma unroll
        for (int l = 0; l < MAX_LAYERS; ++l)
            if (l < nl) hv[l] = __ldcs(reinterpret_cast<const float4*>(D.hist[l] + c0));
        float hs[4] = {0.f, 0.f, 0.f, 0.f};
        #pragma unroll
        for (int l = 0; l < MAX_LAYERS; ++l)
            if (l < nl) {
                hs[0] = __fadd_rn(hs[0], hv[l].x);
                hs[1] = __fadd_rn(hs[1], hv[l].y);
                hs[2] = __fadd_rn(hs[2], hv[l].z);
                hs[3] = __fadd_rn(hs[3], hv[l].w);
            }
        float a[4];
        #pragma unroll
        for (int e = 0; e < 4; ++e) a[e] = __fadd_rn(1.f, __fdiv_rn(hs[e], float(nl)));
        for (int k = 0; k < nc; ++k) {
            uint2 sv[MAX_LAYERS];
            uint32_t oc[MAX_LAYERS], ow[MAX_LAYERS];
            #pragma unroll
            for (int l = 0; l < MAX_LAYERS; ++l)
                if (l < nl) {
                    const int id = k * MAX_LAYERS + l;
                    sv[l] = __ldcs(reinterpret_cast<const uint2*>(D.st[id] + c0));
                    oc[l] = __ldcs(reinterpret_cast<const uint32_t*>(D.oc[id] + c0));
                    ow[l] = __ldcs(reinterpret_cast<const uint32_t*>(D.ov[id] + c0));
                }
            const uint2 vv = __ldcs(reinterpret_cast<const uint2*>(D.vst[k] + c0));
            int occ[4] = {0, 0, 0, 0};
            #pragma unroll
            for (int l = 0; l < MAX_LAYERS; ++l)
                if (l < nl) {
                    const float h[4] = {hv[l].x, hv[l].y, hv[l].z, hv[l].w};
                    const uint16_t st[4] = {uint16_t(sv[l].x), uint16_t(sv[l].x >> 16), uint16_t(sv[l].y), uint16_t(sv[l].y >> 16)};
                    const uint8_t o[4] = {uint8_t(oc[l]), uint8_t(oc[l] >> 8), uint8_t(oc[l] >> 16), uint8_t(oc[l] >> 24)};
                    float out[4];
                    #pragma unroll
                    for (int e = 0; e < 4; ++e) out[e] = cost_track(st[e], o[e], h[e], D.gnd[l], c0 + e, pres, hard);
                    __stcs(reinterpret_cast<float4*>(D.cst[k * MAX_LAYERS + l] + c0), make_float4(out[0], out[1], out[2], out[3]));
                    occ[0] += int(ow[l] & 0xFF);
                    occ[1] += int((ow[l] >> 8) & 0xFF);
                    occ[2] += int((ow[l] >> 16) & 0xFF);
                    occ[3] += int(ow[l] >> 24);
                }
            const uint16_t vs[4] = {uint16_t(vv.x), uint16_t(vv.x >> 16), uint16_t(vv.y), uint16_t(vv.y >> 16)};
            __stcs(reinterpret_cast<float4*>(D.vcst[k] + c0),
                   make_float4(via_of(vs[0], occ[0], a[0], pres, hard), via_of(vs[1], occ[1], a[1], pres, hard),
                               via_of(vs[2], occ[2], a[2], pres, hard), via_of(vs[3], occ[3], a[3], pres, hard)));
        }
    }
}

// spans (j, i0, i1) of one grid (class k, kind 0 track / 1 via, layer l): occupancy +-1 then refresh
// (src/router.cpp:1892-1963 apply + 1880-1890)
__global__ void costs_stamp_kernel(CostDev D, int k, int kind, int l, const int* spans, int nspans, int nx, int sign,
                                   float pres, int hard) {
    for (int s = blockIdx.x; s < nspans; s += gridDim.x) {
        const int j = spans[3 * s], i0 = spans[3 * s + 1], i1 = spans[3 * s + 2];
        for (int i = i0 + threadIdx.x; i <= i1; i += blockDim.x) {
            const size_t c = size_t(j) * nx + i;
            uint8_t* g = kind ? D.ov[k * MAX_LAYERS + l] : D.oc[k * MAX_LAYERS + l];
            const uint8_t v = g[c];
            g[c] = sign < 0 ? uint8_t(v - 1) : (v < 255 ? uint8_t(v + 1) : v);
        }
    }
}

__global__ void costs_refresh_kernel(CostDev D, int k, int kind, int l, const int* spans, int nspans, int nx, float pres,
                                     int hard) {
    for (int s = blockIdx.x; s < nspans; s += gridDim.x) {
        const int j = spans[3 * s], i0 = spans[3 * s + 1], i1 = spans[3 * s + 2];
        for (int i = i0 + threadIdx.x; i <= i1; i += blockDim.x) {
            const size_t c = size_t(j) * nx + i;
            const int id = k * MAX_LAYERS + l;
            if (kind) D.vcst[k][c] = cost_via(D, k, c, pres, hard);
            else D.cst[id][c] = cost_track(D.st[id][c], D.oc[id][c], D.hist[l][c], D.gnd[l], c, pres, hard);
        }
    }
}

// hist[l][c] += inc at the listed states (l * n + c), in list order (src/router.cpp:1983)
__global__ void costs_history_kernel(float* const* hist, const uint32_t* states, int m, size_t n, float inc) {
    // one thread walks the list: repeated states must add in order, exactly as the host loop does
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int k = 0; k < m; ++k) {
        const uint32_t q = states[k];
        float* h = hist[q / n];
        const size_t c = q % n;
        h[c] = __fadd_rn(h[c], inc);
    }
}

}  // namespace
}  // namespace pcbg

// ---- C ABI ----

struct pcbg_costs {
    pcbg::CostDev D;
    std::vector<void*> owned;
    cudaStream_t stream = nullptr;
    int nx = 0, ny = 0;
    float* hist_ptrs_dev = nullptr;
    int* spans_dev = nullptr;
    size_t spans_cap = 0;
    uint32_t* states_dev = nullptr;
    size_t states_cap = 0;
    float pres = 0.f;
    int hard = 0;
};

namespace {

template <class T> T* dalloc(pcbg_costs* h, size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return nullptr;
    h->owned.push_back(p);
    return static_cast<T*>(p);
}

bool fail(const char* what) {
    pcbg::set_error(what);
    return false;
}

}  // namespace

extern "C" pcbg_costs* pcbg_costs_create(int32_t nx, int32_t ny, int32_t nl, int32_t nclasses) {
    if (nx < 1 || ny < 1 || nl < 1 || nl > pcbg::MAX_LAYERS || nclasses < 1 || nclasses > 8) {
        pcbg::set_error("bad cost board geometry");
        return nullptr;
    }
    pcbg_costs* h = new pcbg_costs();
    memset(&h->D, 0, sizeof(h->D));
    h->nx = nx;
    h->ny = ny;
    const size_t n = size_t(nx) * ny;
    h->D.n = int(n);
    h->D.nl = nl;
    h->D.nclasses = nclasses;
    bool ok = true;
    for (int k = 0; k < nclasses && ok; ++k) {
        for (int l = 0; l < nl && ok; ++l) {
            const int id = k * pcbg::MAX_LAYERS + l;
            uint16_t* st = dalloc<uint16_t>(h, n);
            uint8_t* oc = dalloc<uint8_t>(h, n);
            uint8_t* ov = dalloc<uint8_t>(h, n);
            float* cst = dalloc<float>(h, n);
            ok = st && oc && ov && cst;
            if (!ok) break;
            cudaMemset(st, 0, n * 2);
            cudaMemset(oc, 0, n);
            cudaMemset(ov, 0, n);
            h->D.st[id] = st; h->D.oc[id] = oc; h->D.ov[id] = ov; h->D.cst[id] = cst;
        }
        uint16_t* vst = dalloc<uint16_t>(h, n);
        float* vcst = dalloc<float>(h, n);
        ok = ok && vst && vcst;
        if (ok) { cudaMemset(vst, 0, n * 2); h->D.vst[k] = vst; h->D.vcst[k] = vcst; }
    }
    for (int l = 0; l < nl && ok; ++l) {
        float* hs = dalloc<float>(h, n);
        ok = hs != nullptr;
        if (ok) { cudaMemset(hs, 0, n * 4); h->D.hist[l] = hs; }
    }
    float** hp = ok ? reinterpret_cast<float**>(dalloc<float*>(h, pcbg::MAX_LAYERS)) : nullptr;
    ok = ok && hp;
    if (ok) {
        cudaMemcpy(hp, h->D.hist, sizeof(h->D.hist), cudaMemcpyHostToDevice);
        h->hist_ptrs_dev = reinterpret_cast<float*>(hp);
    }
    if (!ok || cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        for (void* p : h->owned) cudaFree(p);
        delete h;
        pcbg::set_error("cost board allocation failed");
        return nullptr;
    }
    return h;
}

extern "C" void pcbg_costs_destroy(pcbg_costs* h) {
    if (!h) return;
    cudaStreamSynchronize(h->stream);
    for (void* p : h->owned) cudaFree(p);
    cudaStreamDestroy(h->stream);
    delete h;
}

extern "C" int pcbg_costs_set_static(pcbg_costs* h, int32_t cls, const uint16_t* st, const uint16_t* vst) {
    if (!h || cls < 0 || cls >= h->D.nclasses) return PCBG_ERR_FAIL;
    const size_t n = size_t(h->D.n);
    for (int l = 0; l < h->D.nl; ++l)
        if (cudaMemcpy(const_cast<uint16_t*>(h->D.st[cls * pcbg::MAX_LAYERS + l]), st + l * n, n * 2, cudaMemcpyHostToDevice) !=
            cudaSuccess)
            return PCBG_ERR_FAIL;
    if (cudaMemcpy(const_cast<uint16_t*>(h->D.vst[cls]), vst, n * 2, cudaMemcpyHostToDevice) != cudaSuccess) return PCBG_ERR_FAIL;
    return 0;
}

extern "C" int pcbg_costs_set_occupancy(pcbg_costs* h, int32_t cls, const uint8_t* oc, const uint8_t* ov) {
    if (!h || cls < 0 || cls >= h->D.nclasses) return PCBG_ERR_FAIL;
    const size_t n = size_t(h->D.n);
    for (int l = 0; l < h->D.nl; ++l) {
        const int id = cls * pcbg::MAX_LAYERS + l;
        if (cudaMemcpy(h->D.oc[id], oc + l * n, n, cudaMemcpyHostToDevice) != cudaSuccess) return PCBG_ERR_FAIL;
        if (cudaMemcpy(h->D.ov[id], ov + l * n, n, cudaMemcpyHostToDevice) != cudaSuccess) return PCBG_ERR_FAIL;
    }
    return 0;
}

extern "C" int pcbg_costs_set_history(pcbg_costs* h, const float* hist) {
    if (!h) return PCBG_ERR_FAIL;
    const size_t n = size_t(h->D.n);
    for (int l = 0; l < h->D.nl; ++l)
        if (cudaMemcpy(const_cast<float*>(h->D.hist[l]), hist + l * n, n * 4, cudaMemcpyHostToDevice) != cudaSuccess)
            return PCBG_ERR_FAIL;
    return 0;
}

extern "C" int pcbg_costs_set_ground(pcbg_costs* h, int32_t layer, const float* fac) {
    if (!h || layer < 0 || layer >= h->D.nl) return PCBG_ERR_FAIL;
    const size_t n = size_t(h->D.n);
    if (!fac) { h->D.gnd[layer] = nullptr; return 0; }
    float* g = const_cast<float*>(h->D.gnd[layer]);
    if (!g) {
        g = dalloc<float>(h, n);
        if (!g) return PCBG_ERR_FAIL;
        h->D.gnd[layer] = g;
    }
    return cudaMemcpy(g, fac, n * 4, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : PCBG_ERR_FAIL;
}

extern "C" int pcbg_costs_rebuild(pcbg_costs* h, float pres, int32_t hard) {
    if (!h) return PCBG_ERR_FAIL;
    h->pres = pres;
    h->hard = hard;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    pcbg::costs_rebuild_kernel<<<unsigned(sms * 8), 256, 0, h->stream>>>(h->D, pres, hard);
    if (cudaGetLastError() != cudaSuccess) return PCBG_ERR_FAIL;
    return cudaStreamSynchronize(h->stream) == cudaSuccess ? 0 : PCBG_ERR_FAIL;
}

extern "C" int pcbg_costs_stamp(pcbg_costs* h, int32_t cls, int32_t kind, int32_t layer, const int32_t* spans,
                                int32_t nspans, int32_t sign) {
    if (!h || cls < 0 || cls >= h->D.nclasses || layer < 0 || layer >= h->D.nl || nspans < 0) return PCBG_ERR_FAIL;
    if (nspans == 0) return 0;
    for (int s = 0; s < nspans; ++s) {
        const int j = spans[3 * s], i0 = spans[3 * s + 1], i1 = spans[3 * s + 2];
        if (j < 0 || j >= h->ny || i0 < 0 || i1 >= h->nx || i0 > i1) { pcbg::set_error("span outside the board"); return PCBG_ERR_FAIL; }
    }
    {
        // the spans' cells are updated in parallel: each cell may appear once (the router's stamps are merged)
        std::vector<std::pair<int, int>> order(nspans);
        for (int s = 0; s < nspans; ++s) order[s] = {spans[3 * s] * 0 + s, s};
        std::sort(order.begin(), order.end(), [&](const std::pair<int, int>& a, const std::pair<int, int>& b) {
            const int* x = spans + 3 * a.second;
            const int* y = spans + 3 * b.second;
            return x[0] < y[0] || (x[0] == y[0] && x[1] < y[1]);
        });
        for (int s = 1; s < nspans; ++s) {
            const int* x = spans + 3 * order[s - 1].second;
            const int* y = spans + 3 * order[s].second;
            if (x[0] == y[0] && y[1] <= x[2]) { pcbg::set_error("overlapping spans"); return PCBG_ERR_FAIL; }
        }
    }
    if (h->spans_cap < size_t(nspans)) {
        int* p = dalloc<int>(h, size_t(nspans) * 3 * 2);
        if (!p) return PCBG_ERR_FAIL;
        h->spans_dev = p;
        h->spans_cap = size_t(nspans) * 2;
    }
    if (cudaMemcpyAsync(h->spans_dev, spans, size_t(nspans) * 12, cudaMemcpyHostToDevice, h->stream) != cudaSuccess) return PCBG_ERR_FAIL;
    const unsigned blocks = unsigned(std::min(nspans, 4096));
    pcbg::costs_stamp_kernel<<<blocks, 64, 0, h->stream>>>(h->D, cls, kind, layer, h->spans_dev, nspans, h->nx, sign, h->pres, h->hard);
    pcbg::costs_refresh_kernel<<<blocks, 64, 0, h->stream>>>(h->D, cls, kind, layer, h->spans_dev, nspans, h->nx, h->pres, h->hard);
    if (cudaGetLastError() != cudaSuccess) return PCBG_ERR_FAIL;
    return cudaStreamSynchronize(h->stream) == cudaSuccess ? 0 : PCBG_ERR_FAIL;
}

extern "C" int pcbg_costs_add_history(pcbg_costs* h, const uint32_t* states, int32_t m, float inc) {
    if (!h || m < 0) return PCBG_ERR_FAIL;
    if (m == 0) return 0;
    const size_t n = size_t(h->D.n);
    for (int k = 0; k < m; ++k)
        if (states[k] >= n * size_t(h->D.nl)) { pcbg::set_error("history state outside the board"); return PCBG_ERR_FAIL; }
    if (h->states_cap < size_t(m)) {
        uint32_t* p = dalloc<uint32_t>(h, size_t(m) * 2);
        if (!p) return PCBG_ERR_FAIL;
        h->states_dev = p;
        h->states_cap = size_t(m) * 2;
    }
    if (cudaMemcpyAsync(h->states_dev, states, size_t(m) * 4, cudaMemcpyHostToDevice, h->stream) != cudaSuccess) return PCBG_ERR_FAIL;
    pcbg::costs_history_kernel<<<1, 32, 0, h->stream>>>(reinterpret_cast<float* const*>(h->hist_ptrs_dev), h->states_dev, m, n, inc);
    if (cudaGetLastError() != cudaSuccess) return PCBG_ERR_FAIL;
    return cudaStreamSynchronize(h->stream) == cudaSuccess ? 0 : PCBG_ERR_FAIL;
}

extern "C" int pcbg_costs_download(pcbg_costs* h, int32_t cls, float* cst, float* vcst) {
    if (!h || cls < 0 || cls >= h->D.nclasses) return PCBG_ERR_FAIL;
    const size_t n = size_t(h->D.n);
    for (int l = 0; l < h->D.nl; ++l)
        if (cst && cudaMemcpy(cst + l * n, h->D.cst[cls * pcbg::MAX_LAYERS + l], n * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
            return PCBG_ERR_FAIL;
    if (vcst && cudaMemcpy(vcst, h->D.vcst[cls], n * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return PCBG_ERR_FAIL;
    return 0;
}

extern "C" int pcbg_costs_download_history(pcbg_costs* h, float* hist) {
    if (!h) return PCBG_ERR_FAIL;
    const size_t n = size_t(h->D.n);
    for (int l = 0; l < h->D.nl; ++l)
        if (cudaMemcpy(hist + l * n, h->D.hist[l], n * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return PCBG_ERR_FAIL;
    return 0;
}

bool pcbg::cost_planes(pcbg_costs* h, int cls, CostPlanes& o) {
    if (!h || cls < 0 || cls >= h->D.nclasses) return false;
    memset(&o, 0, sizeof(o));
    o.nx = h->nx;
    o.ny = h->ny;
    o.nl = h->D.nl;
    for (int l = 0; l < h->D.nl; ++l) {
        const int id = cls * pcbg::MAX_LAYERS + l;
        o.cst[l] = h->D.cst[id];
        o.oc[l] = h->D.oc[id];
        o.ov[l] = h->D.ov[id];
        o.hist[l] = h->D.hist[l];
    }
    o.vcst = h->D.vcst[cls];
    return true;
}

extern "C" const float* pcbg_costs_device_map(pcbg_costs* h, int32_t cls, int32_t layer) {
    if (!h || cls < 0 || cls >= h->D.nclasses || layer < -1 || layer >= h->D.nl) return nullptr;
    return layer < 0 ? h->D.vcst[cls] : h->D.cst[cls * pcbg::MAX_LAYERS + layer];
}

extern "C" float pcbg_costs_time_rebuild(pcbg_costs* h, float pres, int32_t hard, int32_t reps) {
    if (!h || reps < 1) return -1.f;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    pcbg::costs_rebuild_kernel<<<unsigned(sms * 8), 256, 0, h->stream>>>(h->D, pres, hard);  // warm
    cudaEventRecord(a, h->stream);
    for (int r = 0; r < reps; ++r) pcbg::costs_rebuild_kernel<<<unsigned(sms * 8), 256, 0, h->stream>>>(h->D, pres, hard);
    cudaEventRecord(b, h->stream);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    h->pres = pres;
    h->hard = hard;
    return ms / reps;
}
