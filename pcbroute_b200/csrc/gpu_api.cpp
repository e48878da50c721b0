// pcbroute's gpu.h (src/gpu.h:10-57) implemented over the pcbg C ABI: the drop-in replacement for src/gpu.cu.
// The router objects built with -DPCB_GPU link against libpcbgpu.so unchanged.
#include "gpu.h"

#include <cstring>
#include <vector>

#include "pcbg.h"

namespace {

// GpuQuery's vectors of (index, value) pairs as the two arrays pcbg_query takes
struct Flat {
    std::vector<uint32_t> idx;
    std::vector<float> val;
    explicit Flat(const std::vector<std::pair<uint32_t, float>>& v) {
        idx.reserve(v.size());
        val.reserve(v.size());
        for (const auto& p : v) {
            idx.push_back(p.first);
            val.push_back(p.second);
        }
    }
};

}  // namespace

// src/gpu.cu:383-391
bool gpu_available() { return pcbg_available() != 0; }

// src/gpu.cu:377-381
void gpu_configure(int slots, size_t max_states) { pcbg_configure(slots, max_states); }

// src/gpu.cu:393-403: a pinned buffer of at least n floats, from the pool
void GpuOut::reserve(size_t n) {
    if (d && cap >= n) return;
    if (d) pcbg_host_release(d, cap);
    d = pcbg_host_acquire(n, &cap);
    if (!d) cap = 0;
}

// src/gpu.cu:405-407
GpuOut::~GpuOut() {
    if (d) pcbg_host_release(d, cap);
}

// src/gpu.cu:409-416: cost of a window state (1e30 outside the solved rectangle)
float GpuOut::operator()(int64_t q) const {
    const int64_t WN = int64_t(ww) * wh;
    const int l = int(q / WN);
    const int64_t c = q % WN;
    const int i = int(c % ww) - rx0, j = int(c / ww) - ry0;
    if (i < 0 || j < 0 || i >= rw || j >= rh) return 1e30f;
    return d[(size_t(l) * rh + j) * rw + i];
}

// src/gpu.cu:550-622
int gpu_solve(const GpuQuery& q, GpuOut& out, bool wait) {
    if (q.NL < 1 || q.NL > 8) return -1;
    const Flat own(q.own_cf), ownv(q.own_vcf), st(q.starts);
    pcbg_query p;
    std::memset(&p, 0, sizeof(p));
    p.nx = q.nx; p.ny = q.ny; p.nl = q.NL;
    p.wi0 = q.wi0; p.wj0 = q.wj0; p.ww = q.ww; p.wh = q.wh;
    p.me = q.me; p.via_cost = q.via_cost; p.step = q.step;
    std::memcpy(p.dirf, q.dirf, sizeof(p.dirf));
    for (int l = 0; l < 8; ++l) {
        p.lay[l] = q.lay[l];
        p.play[l] = q.play[l];
        p.cst[l] = l < q.NL ? q.cst[l] : nullptr;
        p.st[l] = l < q.NL ? q.st[l] : nullptr;
    }
    p.vcst = q.vcst; p.vst = q.vst; p.tbit = q.tbit;
    p.own_cf_idx = own.idx.data(); p.own_cf_val = own.val.data(); p.n_own_cf = int64_t(own.idx.size());
    p.own_vcf_idx = ownv.idx.data(); p.own_vcf_val = ownv.val.data(); p.n_own_vcf = int64_t(ownv.idx.size());
    p.start_idx = st.idx.data(); p.start_val = st.val.data(); p.n_starts = int64_t(st.idx.size());
    p.prior = q.prior; p.pi0 = q.pi0; p.pj0 = q.pj0; p.pw = q.pw; p.ph = q.ph; p.pnl = q.pnl;
    p.pcol = q.pcol; p.prow = q.prow;
    std::memcpy(p.mlf, q.mlf, sizeof(p.mlf));
    p.mthr = q.mthr; p.corridor = q.corridor ? 1 : 0;
    pcbg_result r;
    std::memset(&r, 0, sizeof(r));
    r.d = out.d;
    r.cap = out.cap;
    const int rc = pcbg_solve(&p, &r, wait ? 1 : 0);
    // the output buffer may have been replaced even on failure: keep ownership consistent
    out.d = r.d;
    out.cap = r.cap;
    if (rc < 0) return rc;
    out.rx0 = r.rx0; out.ry0 = r.ry0; out.rw = r.rw; out.rh = r.rh; out.NL = r.nl; out.ww = r.ww; out.wh = r.wh;
    out.best = r.best;
    return rc;
}
