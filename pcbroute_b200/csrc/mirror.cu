// Device mirror of the router's cost grids (the boundary extension pcbg_grid_sync of the drop-in back end).
//
// The reference back end copies a search's rectangle of the class's cost and owner grids from host memory on every
// solve (src/gpu.cu:432-439): on large boards that upload, not the relaxation, is most of a search's time. A router
// that tells the back end when it changes those grids keeps a copy of them in HBM instead:
//   * after rebuild_costs (src/router.cpp:409-420) it hands over every grid of a class: cost and via cost (RClass::
//     cst / vcst), the static owner grids (st / vst, uploaded once), the occupancy (oc / ov) and the history;
//   * after each refresh_costs (src/router.cpp:1880-1890, called by every stamp and rip-up of a commit) it names the
//     spans that changed, and those cells of the cost grid and of the stamped occupancy grid are copied up.
// Both calls return once the device copy is current, so a search that starts after them reads what they wrote. A
// query whose grid pointers are a mirrored class's (gpu_solve passes RClass::cst[l].data() and friends) then takes
// its rectangle from the mirror with device-to-device copies. A commit that runs while a search copies its
// rectangle can be seen half-applied, exactly as a search reading the host grids would see it; the router's commit
// check rejects such a search whenever the commit touched a block it read (src/router.cpp:2200-2216).
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "pcbg_internal.h"

namespace pcbg {
namespace {

struct MirrorClass {
    bool on = false;
    int nx = 0, ny = 0, nl = 0;
    // host grids (the router's own vectors), page-locked in place so that copies run at full link speed
    const float* h_cst[MAX_LAYERS] = {};
    const float* h_vcst = nullptr;
    const uint16_t* h_st[MAX_LAYERS] = {};
    const uint16_t* h_vst = nullptr;
    const uint8_t* h_oc[MAX_LAYERS] = {};
    const uint8_t* h_ov[MAX_LAYERS] = {};
    const float* h_hist[MAX_LAYERS] = {};
    // device copies: [l][ny * nx] planes
    float* cst = nullptr;
    float* vcst = nullptr;
    uint16_t* st = nullptr;
    uint16_t* vst = nullptr;
    uint8_t* oc = nullptr;
    uint8_t* ov = nullptr;
    float* hist = nullptr;
};

std::mutex g_mu_m;
std::vector<MirrorClass> g_cls;
cudaStream_t g_ms = nullptr;
std::vector<void*> g_registered;
// span staging: packed values and their cell indices, pinned
struct SpanStage {
    unsigned char* h = nullptr;
    size_t cap = 0;
    unsigned char* d = nullptr;
    size_t dcap = 0;
} g_ss;

void pin(const void* p, size_t bytes) {
    if (!p || !bytes) return;
    void* q = const_cast<void*>(p);
    if (std::find(g_registered.begin(), g_registered.end(), q) != g_registered.end()) return;
    // memory that is already page-locked (or that the driver refuses to lock) is still copied, only slower
    if (cudaHostRegister(q, bytes, cudaHostRegisterDefault) == cudaSuccess) g_registered.push_back(q);
    else cudaGetLastError();
}

template <class T> bool dalloc(T*& p, size_t n) {
    if (p) return true;
    return cudaMalloc(&p, n * sizeof(T)) == cudaSuccess;
}

// Scatter packed values into a plane: (index, value) pairs of one element type.
template <class T>
__global__ void span_scatter_kernel(T* dst, const uint32_t* idx, const T* val, int n) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) dst[idx[k]] = val[k];
}

int fail(const char* what) {
    set_error(std::string("mirror: ") + what);
    return PCBG_ERR_FAIL;
}

}  // namespace

bool mirror_lookup(const pcbg_query& q, MirrorView& v) {
    std::lock_guard<std::mutex> g(g_mu_m);
    for (const MirrorClass& M : g_cls) {
        if (!M.on || M.nx != q.nx || M.ny != q.ny || M.nl != q.nl || M.h_cst[0] != q.cst[0]) continue;
        bool all = M.h_vcst == q.vcst && M.h_vst == q.vst;
        for (int l = 0; l < q.nl; ++l) all = all && M.h_cst[l] == q.cst[l] && M.h_st[l] == q.st[l];
        if (!all) continue;
        const size_t n = size_t(M.nx) * M.ny;
        for (int l = 0; l < MAX_LAYERS; ++l) {
            v.cst[l] = l < M.nl ? M.cst + l * n : nullptr;
            v.st[l] = l < M.nl ? M.st + l * n : nullptr;
        }
        v.vcst = M.vcst;
        v.vst = M.vst;
        return true;
    }
    return false;
}

bool mirror_planes(int cls, CostPlanes& out) {
    std::lock_guard<std::mutex> g(g_mu_m);
    if (cls < 0 || cls >= int(g_cls.size()) || !g_cls[cls].on) return false;
    const MirrorClass& M = g_cls[cls];
    const size_t n = size_t(M.nx) * M.ny;
    out.nx = M.nx; out.ny = M.ny; out.nl = M.nl;
    for (int l = 0; l < MAX_LAYERS; ++l) {
        out.cst[l] = l < M.nl ? M.cst + l * n : nullptr;
        out.oc[l] = l < M.nl ? M.oc + l * n : nullptr;
        out.ov[l] = l < M.nl ? M.ov + l * n : nullptr;
        out.hist[l] = l < M.nl ? M.hist + l * n : nullptr;
    }
    out.vcst = M.vcst;
    return true;
}

}  // namespace pcbg

using namespace pcbg;

extern "C" int pcbg_mirror_class(int32_t cls, int32_t nx, int32_t ny, int32_t nl, const float* const* cst,
                                 const float* vcst, const uint16_t* const* st, const uint16_t* vst,
                                 const uint8_t* const* oc, const uint8_t* const* ov, const float* const* hist) {
    if (cls < 0 || cls > 63 || nx < 1 || ny < 1 || nl < 1 || nl > MAX_LAYERS || !cst || !st || !vcst || !vst)
        return fail("bad class description");
    std::lock_guard<std::mutex> g(g_mu_m);
    if (!g_ms && cudaStreamCreateWithFlags(&g_ms, cudaStreamNonBlocking) != cudaSuccess) return fail("stream");
    if (int(g_cls.size()) <= cls) g_cls.resize(cls + 1);
    MirrorClass& M = g_cls[cls];
    const size_t n = size_t(nx) * ny;
    if (M.on && (M.nx != nx || M.ny != ny || M.nl != nl)) return fail("board size changed");
    const bool first = !M.on;
    if (first) {
        M.nx = nx; M.ny = ny; M.nl = nl;
        if (!dalloc(M.cst, n * nl) || !dalloc(M.vcst, n) || !dalloc(M.st, n * nl) || !dalloc(M.vst, n) ||
            !dalloc(M.oc, n * nl) || !dalloc(M.ov, n * nl) || !dalloc(M.hist, n * nl))
            return fail("device allocation failed");
        cudaMemsetAsync(M.oc, 0, n * nl, g_ms);
        cudaMemsetAsync(M.ov, 0, n * nl, g_ms);
        cudaMemsetAsync(M.hist, 0, n * nl * 4, g_ms);
    }
    for (int l = 0; l < nl; ++l) {
        M.h_cst[l] = cst[l];
        M.h_st[l] = st[l];
        M.h_oc[l] = oc ? oc[l] : nullptr;
        M.h_ov[l] = ov ? ov[l] : nullptr;
        M.h_hist[l] = hist ? hist[l] : nullptr;
        pin(cst[l], n * 4);
        if (oc) pin(oc[l], n);
        if (ov) pin(ov[l], n);
        if (hist) pin(hist[l], n * 4);
    }
    M.h_vcst = vcst;
    M.h_vst = vst;
    pin(vcst, n * 4);
    // the owner grids are static after the router's set-up: once
    if (first) {
        for (int l = 0; l < nl; ++l)
            if (cudaMemcpyAsync(M.st + l * n, st[l], n * 2, cudaMemcpyHostToDevice, g_ms) != cudaSuccess) return fail("copy");
        if (cudaMemcpyAsync(M.vst, vst, n * 2, cudaMemcpyHostToDevice, g_ms) != cudaSuccess) return fail("copy");
    }
    for (int l = 0; l < nl; ++l) {
        if (cudaMemcpyAsync(M.cst + l * n, cst[l], n * 4, cudaMemcpyHostToDevice, g_ms) != cudaSuccess) return fail("copy");
        if (oc && cudaMemcpyAsync(M.oc + l * n, oc[l], n, cudaMemcpyHostToDevice, g_ms) != cudaSuccess) return fail("copy");
        if (ov && cudaMemcpyAsync(M.ov + l * n, ov[l], n, cudaMemcpyHostToDevice, g_ms) != cudaSuccess) return fail("copy");
        if (hist && cudaMemcpyAsync(M.hist + l * n, hist[l], n * 4, cudaMemcpyHostToDevice, g_ms) != cudaSuccess)
            return fail("copy");
    }
    if (cudaMemcpyAsync(M.vcst, vcst, n * 4, cudaMemcpyHostToDevice, g_ms) != cudaSuccess) return fail("copy");
    if (cudaStreamSynchronize(g_ms) != cudaSuccess) return fail("copy");
    M.on = true;
    return 0;
}

extern "C" int pcbg_mirror_spans(int32_t cls, int32_t kind, int32_t layer, const int32_t* spans, int32_t nspans) {
    std::lock_guard<std::mutex> g(g_mu_m);
    if (cls < 0 || cls >= int(g_cls.size()) || !g_cls[cls].on) return 0;   // not mirrored: nothing to keep current
    MirrorClass& M = g_cls[cls];
    if (layer < 0 || layer >= M.nl || kind < 0 || kind > 1) return fail("bad grid");
    if (nspans <= 0) return 0;
    // cells of the spans, clipped to the board
    size_t cells = 0;
    for (int k = 0; k < nspans; ++k) {
        const int j = spans[3 * k], i0 = std::max(0, spans[3 * k + 1]), i1 = std::min(M.nx - 1, spans[3 * k + 2]);
        if (j >= 0 && j < M.ny && i1 >= i0) cells += size_t(i1 - i0 + 1);
    }
    if (!cells) return 0;
    const size_t n = size_t(M.nx) * M.ny;
    const float* hc = kind ? M.h_vcst : M.h_cst[layer];
    const uint8_t* ho = kind ? M.h_ov[layer] : M.h_oc[layer];
    float* dc = kind ? M.vcst : M.cst + size_t(layer) * n;
    uint8_t* dov = kind ? M.ov + size_t(layer) * n : M.oc + size_t(layer) * n;
    // staging: indices (4 B), cost values (4 B), occupancy values (1 B) per cell
    const size_t need = cells * 9 + 64;
    if (g_ss.cap < need) {
        if (g_ss.h) cudaFreeHost(g_ss.h);
        if (g_ss.d) cudaFree(g_ss.d);
        g_ss.h = nullptr; g_ss.d = nullptr; g_ss.cap = g_ss.dcap = 0;
        const size_t c = need * 2;
        if (cudaHostAlloc(reinterpret_cast<void**>(&g_ss.h), c, cudaHostAllocDefault) != cudaSuccess) return fail("pinned");
        if (cudaMalloc(&g_ss.d, c) != cudaSuccess) return fail("device allocation failed");
        g_ss.cap = g_ss.dcap = c;
    }
    uint32_t* hi = reinterpret_cast<uint32_t*>(g_ss.h);
    float* hv = reinterpret_cast<float*>(g_ss.h + cells * 4);
    uint8_t* hb = g_ss.h + cells * 8;
    size_t o = 0;
    for (int k = 0; k < nspans; ++k) {
        const int j = spans[3 * k], i0 = std::max(0, spans[3 * k + 1]), i1 = std::min(M.nx - 1, spans[3 * k + 2]);
        if (j < 0 || j >= M.ny || i1 < i0) continue;
        const size_t base = size_t(j) * M.nx, len = size_t(i1 - i0 + 1);
        memcpy(hv + o, hc + base + i0, len * 4);
        if (ho) memcpy(hb + o, ho + base + i0, len);
        for (size_t t = 0; t < len; ++t) hi[o + t] = uint32_t(base + i0 + t);
        o += len;
    }
    if (cudaMemcpyAsync(g_ss.d, g_ss.h, cells * 9, cudaMemcpyHostToDevice, g_ms) != cudaSuccess) return fail("copy");
    const uint32_t* di = reinterpret_cast<const uint32_t*>(g_ss.d);
    const int blocks = int(std::min<size_t>((cells + 255) / 256, 1024));
    span_scatter_kernel<float><<<blocks, 256, 0, g_ms>>>(dc, di, reinterpret_cast<const float*>(g_ss.d + cells * 4),
                                                         int(cells));
    if (ho) span_scatter_kernel<uint8_t><<<blocks, 256, 0, g_ms>>>(dov, di, g_ss.d + cells * 8, int(cells));
    if (cudaStreamSynchronize(g_ms) != cudaSuccess) return fail("span update");
    return 0;
}

extern "C" int pcbg_mirror_history(int32_t cls) {
    std::lock_guard<std::mutex> g(g_mu_m);
    if (cls < 0 || cls >= int(g_cls.size()) || !g_cls[cls].on) return 0;
    MirrorClass& M = g_cls[cls];
    const size_t n = size_t(M.nx) * M.ny;
    for (int l = 0; l < M.nl; ++l)
        if (M.h_hist[l] && cudaMemcpyAsync(M.hist + l * n, M.h_hist[l], n * 4, cudaMemcpyHostToDevice, g_ms) != cudaSuccess)
            return fail("copy");
    return cudaStreamSynchronize(g_ms) == cudaSuccess ? 0 : fail("copy");
}

extern "C" int pcbg_mirror_download(int32_t cls, float* cst, float* vcst, uint8_t* oc, uint8_t* ov) {
    std::lock_guard<std::mutex> g(g_mu_m);
    if (cls < 0 || cls >= int(g_cls.size()) || !g_cls[cls].on) return fail("class not mirrored");
    MirrorClass& M = g_cls[cls];
    const size_t n = size_t(M.nx) * M.ny;
    if (cst && cudaMemcpy(cst, M.cst, n * M.nl * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return fail("copy");
    if (vcst && cudaMemcpy(vcst, M.vcst, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return fail("copy");
    if (oc && cudaMemcpy(oc, M.oc, n * M.nl, cudaMemcpyDeviceToHost) != cudaSuccess) return fail("copy");
    if (ov && cudaMemcpy(ov, M.ov, n * M.nl, cudaMemcpyDeviceToHost) != cudaSuccess) return fail("copy");
    return 0;
}
