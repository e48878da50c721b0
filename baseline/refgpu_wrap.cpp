// A C entry point around pcbroute's own CUDA back end (src/gpu.cu, built unchanged beside this file by
// baseline/Makefile), so that the same searches can be timed through it and through libpcbgpu: one search over a
// whole window given as dense host arrays, exactly as gpu_solve receives it from the router (src/gpu.h:10-57).
#include <chrono>
#include <cstdint>
#include <cstring>

#include "gpu.h"

extern "C" int refgpu_solve_dense(int rw, int rh, int nl, const float* cst, const uint16_t* st, const float* vcst,
                                  const uint16_t* vst, const uint64_t* tbit, uint32_t src, float via_cost,
                                  int64_t* best, double* seconds) {
    if (!gpu_available() || nl < 1 || nl > 8) return -1;
    GpuQuery q;
    q.nx = rw; q.ny = rh; q.NL = nl;
    q.wi0 = 0; q.wj0 = 0; q.ww = rw; q.wh = rh;
    q.me = 1;
    q.via_cost = via_cost;
    q.step = 1.0f;
    for (int l = 0; l < 8; ++l) {
        for (int m = 0; m < 8; ++m) q.dirf[l][m] = 1.0f;
        q.lay[l] = l < nl ? 1 : 0;
        q.cst[l] = l < nl ? cst + size_t(l) * rw * rh : nullptr;
        q.st[l] = l < nl ? st + size_t(l) * rw * rh : nullptr;
        q.play[l] = -1;
    }
    q.vcst = vcst;
    q.vst = vst;
    q.tbit = tbit;
    q.starts.push_back({src, 0.0f});
    const auto t0 = std::chrono::steady_clock::now();
    GpuOut out;
    const int r = gpu_solve(q, out, true);
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *best = out.best;
    return r;
}

// The same search with a given diagonal direction factor, returning the solved rectangle (rx0, ry0, rw, rh) and its
// field (nl * rh * rw floats, the GpuOut layout) for comparison with another back end. Returns gpu_solve's code,
// or -2 when the field does not fit `cap`.
extern "C" int refgpu_solve_field(int rw, int rh, int nl, const float* cst, const uint16_t* st, const float* vcst,
                                  const uint16_t* vst, const uint64_t* tbit, uint32_t src, float via_cost,
                                  float dirf_diag, int32_t* rect, float* field, int64_t cap, int64_t* best) {
    if (!gpu_available() || nl < 1 || nl > 8) return -1;
    GpuQuery q;
    q.nx = rw; q.ny = rh; q.NL = nl;
    q.wi0 = 0; q.wj0 = 0; q.ww = rw; q.wh = rh;
    q.me = 1;
    q.via_cost = via_cost;
    q.step = 1.0f;
    for (int l = 0; l < 8; ++l) {
        for (int m = 0; m < 8; ++m) q.dirf[l][m] = m < 4 ? 1.0f : dirf_diag;
        q.lay[l] = l < nl ? 1 : 0;
        q.cst[l] = l < nl ? cst + size_t(l) * rw * rh : nullptr;
        q.st[l] = l < nl ? st + size_t(l) * rw * rh : nullptr;
        q.play[l] = -1;
    }
    q.vcst = vcst;
    q.vst = vst;
    q.tbit = tbit;
    q.starts.push_back({src, 0.0f});
    GpuOut out;
    const int r = gpu_solve(q, out, true);
    *best = out.best;
    rect[0] = out.rx0; rect[1] = out.ry0; rect[2] = out.rw; rect[3] = out.rh;
    if (r < 1) return r;
    const int64_t n = int64_t(out.rw) * out.rh * nl;
    if (n > cap) return -2;
    std::memcpy(field, out.d, size_t(n) * sizeof(float));
    return r;
}
