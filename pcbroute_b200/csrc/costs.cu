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

// every cell of every class: 8 cells per thread (128-bit loads of st/hist/gnd and stores of cst)
__global__ void costs_rebuild_kernel(CostDev D, float pres, int hard) {
    const size_t n = size_t(D.n);
    const size_t groups = (n + 7) / 8;
    for (size_t g = size_t(blockIdx.x) * blockDim.x + threadIdx.x; g < groups * D.nl; g += size_t(gridDim.x) * blockDim.x) {
        const int l = int(g / groups);
        const size_t c0 = (g % groups) * 8;
        const bool full = c0 + 8 <= n;
        float h[8], gf[8];
        if (full) {
            const float4* hp = reinterpret_cast<const float4*>(D.hist[l] + c0);
            const float4 h0 = hp[0], h1 = hp[1];
            h[0] = h0.x; h[1] = h0.y; h[2] = h0.z; h[3] = h0.w; h[4] = h1.x; h[5] = h1.y; h[6] = h1.z; h[7] = h1.w;
        } else {
            for (int e = 0; e < 8; ++e) h[e] = c0 + e < n ? D.hist[l][c0 + e] : 0.f;
        }
        for (int k = 0; k < D.nclasses; ++k) {
            const int id = k * MAX_LAYERS + l;
            float out[8];
            if (full) {
                const uint4 sv = *reinterpret_cast<const uint4*>(D.st[id] + c0);
                const uint2 ov = *reinterpret_cast<const uint2*>(D.oc[id] + c0);
                const uint16_t s[8] = {uint16_t(sv.x), uint16_t(sv.x >> 16), uint16_t(sv.y), uint16_t(sv.y >> 16),
                                       uint16_t(sv.z), uint16_t(sv.z >> 16), uint16_t(sv.w), uint16_t(sv.w >> 16)};
                const uint8_t o[8] = {uint8_t(ov.x), uint8_t(ov.x >> 8), uint8_t(ov.x >> 16), uint8_t(ov.x >> 24),
                                      uint8_t(ov.y), uint8_t(ov.y >> 8), uint8_t(ov.y >> 16), uint8_t(ov.y >> 24)};
                #pragma unroll
                for (int e = 0; e < 8; ++e) out[e] = cost_track(s[e], o[e], h[e], D.gnd[l], c0 + e, pres, hard);
                float4* op = reinterpret_cast<float4*>(D.cst[id] + c0);
                op[0] = make_float4(out[0], out[1], out[2], out[3]);
                op[1] = make_float4(out[4], out[5], out[6], out[7]);
            } else {
                for (size_t c = c0; c < n; ++c)
                    D.cst[id][c] = cost_track(D.st[id][c], D.oc[id][c], D.hist[l][c], D.gnd[l], c, pres, hard);
            }
        }
        (void)gf;
    }
    // via maps: one cell per thread; the layer sum of the history is shared by the classes (summed in layer
    // order, as vcost_xp does)
    for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x) {
        float hs = 0.f;
        for (int l = 0; l < D.nl; ++l) hs = __fadd_rn(hs, D.hist[l][c]);
        const float a = __fadd_rn(1.f, __fdiv_rn(hs, float(D.nl)));
        for (int k = 0; k < D.nclasses; ++k) {
            const uint16_t s = D.vst[k][c];
            float v = CINF;
            if (s != BLOCK) {
                int occ = 0;
                for (int l = 0; l < D.nl; ++l) occ += D.ov[k * MAX_LAYERS + l][c];
                if (!(hard && occ > 0)) {
                    v = __fmul_rn(a, __fadd_rn(1.f, __fmul_rn(pres, float(occ > 0 ? occ : 0))));
                    if (s != FREE) v = -v;
                }
            }
            D.vcst[k][c] = v;
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
