// gpu.h (src/gpu.h:10-57) implemented by the CPU oracle -- TEST INFRASTRUCTURE ONLY.
//
// Linked with pcbroute's own router objects (oracle/Makefile), it makes "the reference router with an exact search
// back end": the router-level oracle against which the B200 build's sessions are compared byte for byte.
#include "gpu.h"

#include <atomic>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "pcb_oracle.h"

bool gpu_available() { return true; }

void gpu_configure(int slots, size_t max_states) {
    (void)slots;
    pcbo_set_max_states(max_states);
}

GpuOut::~GpuOut() { std::free(d); }

void GpuOut::reserve(size_t n) {
    if (d && cap >= n) return;
    std::free(d);
    d = static_cast<float*>(std::malloc(n * sizeof(float)));
    cap = d ? n : 0;
}

float GpuOut::operator()(int64_t q) const {
    const int64_t WN = int64_t(ww) * wh;
    const int l = int(q / WN);
    const int64_t c = q % WN;
    const int i = int(c % ww) - rx0, j = int(c / ww) - ry0;
    if (i < 0 || j < 0 || i >= rw || j >= rh) return 1e30f;
    return d[(size_t(l) * rh + j) * rw + i];
}

// The back end's host-side fault injection, restated: PCBG_FAIL_SOLVE=k[:p] fails the k-th call (and every p-th
// after it), so the oracle router and the B200 router fall back to the CPU search on the same searches.
struct FailPlan {
    long long first = 0, every = 0;
    FailPlan() {
        if (const char* e = std::getenv("PCBG_FAIL_SOLVE")) {
            char* end = nullptr;
            first = std::strtoll(e, &end, 10);
            if (end && *end == ':') every = std::strtoll(end + 1, nullptr, 10);
        }
    }
};
static std::atomic<long long> g_calls{0};
static bool injected_failure() {
    static const FailPlan plan;
    if (plan.first <= 0) return false;
    const long long n = ++g_calls;
    return n == plan.first || (plan.every > 0 && n > plan.first && (n - plan.first) % plan.every == 0);
}

int gpu_solve(const GpuQuery& q, GpuOut& out, bool wait) {
    (void)wait;
    if (injected_failure()) return -1;
    if (q.NL < 1 || q.NL > 8) return -1;
    auto flat = [](const std::vector<std::pair<uint32_t, float>>& v, std::vector<uint32_t>& i, std::vector<float>& x) {
        for (const auto& p : v) { i.push_back(p.first); x.push_back(p.second); }
    };
    std::vector<uint32_t> oi, vi, si;
    std::vector<float> ov, vv, sv;
    flat(q.own_cf, oi, ov);
    flat(q.own_vcf, vi, vv);
    flat(q.starts, si, sv);
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
    p.own_cf_idx = oi.data(); p.own_cf_val = ov.data(); p.n_own_cf = int64_t(oi.size());
    p.own_vcf_idx = vi.data(); p.own_vcf_val = vv.data(); p.n_own_vcf = int64_t(vi.size());
    p.start_idx = si.data(); p.start_val = sv.data(); p.n_starts = int64_t(si.size());
    p.prior = q.prior; p.pi0 = q.pi0; p.pj0 = q.pj0; p.pw = q.pw; p.ph = q.ph; p.pnl = q.pnl;
    p.pcol = q.pcol; p.prow = q.prow;
    std::memcpy(p.mlf, q.mlf, sizeof(p.mlf));
    p.mthr = q.mthr; p.corridor = q.corridor ? 1 : 0;
    pcbg_result r;
    std::memset(&r, 0, sizeof(r));
    const int rc = pcbo_solve(&p, &r);
    if (rc < 0) return -1;
    std::free(out.d);
    out.d = r.d;
    out.cap = r.cap;
    out.rx0 = r.rx0; out.ry0 = r.ry0; out.rw = r.rw; out.rh = r.rh; out.NL = r.nl; out.ww = r.ww; out.wh = r.wh;
    out.best = r.best;
    return rc;
}
