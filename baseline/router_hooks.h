// Hooks that let pcbroute's own router drive the B200 back end's extensions: the device mirror of the cost grids
// and the learned speculation scheduler (include/pcbg.h). This header is force-included (-include) when
// baseline/patch_router.py's copy of src/router.cpp is compiled; the patch adds one call per hook site:
//
//   pcbgh_rebuilt       end of rebuild_costs (src/router.cpp:409-420): mirror every grid of every class
//   pcbgh_refreshed     end of refresh_costs (src/router.cpp:1880-1890): mirror the spans a stamp changed
//   pcbgh_begin         route_waves (src/router.cpp:2119), once the call's commit order is fixed: the nets' windows
//   pcbgh_allow         the worker's wait for the next net (src/router.cpp:2172-2175): may it start now?
//   pcbgh_started       a worker took a net (src/router.cpp:2176-2181)
//   pcbgh_verdict       the commit check of the net at the commit point (src/router.cpp:2200-2205)
//   pcbgh_commit        a commit was made (src/router.cpp:2210)
//   pcbgh_end           route_waves returns
//
// Every hook reads state the router already has and changes none of it, except that pcbgh_allow can make a worker
// wait for the next commit instead of starting a speculative search; the router's fixed commit order and its
// check decide every result, so the session is the same whatever the hooks answer. PCBG_MIRROR=0 in the
// environment turns the mirror off; the scheduler is off unless PCBG_SCHED is set (include/pcbg.h).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <vector>

#include "pcbg.h"

inline bool pcbgh_mirror_on() {
    static const bool on = [] {
        const char* e = std::getenv("PCBG_MIRROR");
        return !(e && e[0] == '0');
    }();
    return on;
}

template <class RC>
void pcbgh_rebuilt(std::vector<RC>& rcs, std::vector<std::vector<float>>& hist, int NL, int nx, int ny) {
    if (!pcbgh_mirror_on()) return;
    for (size_t k = 0; k < rcs.size(); ++k) {
        RC& R = rcs[k];
        if (R.cst.empty()) continue;
        const float* cst[8] = {};
        const uint16_t* st[8] = {};
        const uint8_t* oc[8] = {};
        const uint8_t* ov[8] = {};
        const float* hs[8] = {};
        for (int l = 0; l < NL && l < 8; ++l) {
            cst[l] = R.cst[l].data();
            st[l] = R.st[l].data();
            oc[l] = R.oc[l].data();
            ov[l] = R.ov[l].data();
            hs[l] = l < int(hist.size()) && !hist[l].empty() ? hist[l].data() : nullptr;
        }
        const bool have_hist = !hist.empty() && !hist[0].empty();
        pcbg_mirror_class(int32_t(k), nx, ny, NL, cst, R.vcst.data(), st, R.vst.data(), oc, ov, have_hist ? hs : nullptr);
    }
}

template <class SP>
void pcbgh_refreshed(size_t k, size_t kind, size_t l, const std::vector<SP>& spans) {
    if (!pcbgh_mirror_on() || spans.empty()) return;
    thread_local std::vector<int32_t> tri;
    tri.clear();
    for (const SP& s : spans) {
        tri.push_back(int32_t(s.j));
        tri.push_back(int32_t(s.i0));
        tri.push_back(int32_t(s.i1));
    }
    pcbg_mirror_spans(int32_t(k), int32_t(kind), int32_t(l), tri.data(), int32_t(spans.size()));
}

// A net's search window as route_job's first stage opens it (J.box grown by o.window, src/router.cpp:1294), in
// cells, and two corners of its pin box as its "pins".
template <class G, class B>
pcbg_rnet pcbgh_rnet(const G& g, const B& box, double margin) {
    auto cx = [&](double x) { return int(std::floor((x - g.x0) / g.s)); };
    auto cy = [&](double y) { return int(std::floor((y - g.y0) / g.s)); };
    pcbg_rnet r;
    r.x0 = std::max(0, cx(box.x0 - margin));
    r.y0 = std::max(0, cy(box.y0 - margin));
    r.x1 = std::min(g.nx, cx(box.x1 + margin) + 1);
    r.y1 = std::min(g.ny, cy(box.y1 + margin) + 1);
    if (r.x1 <= r.x0) r.x1 = std::min(g.nx, r.x0 + 1);
    if (r.y1 <= r.y0) r.y1 = std::min(g.ny, r.y0 + 1);
    r.sx = float((box.x0 - g.x0) / g.s);
    r.sy = float((box.y0 - g.y0) / g.s);
    r.tx = float((box.x1 - g.x0) / g.s);
    r.ty = float((box.y1 - g.y0) / g.s);
    return r;
}

inline bool pcbgh_sched_on() {
    static const bool on = pcbg_rsched_mode() != 0;
    return on;
}

template <class JOBS, class G>
void pcbgh_begin(const std::vector<int>& order, const JOBS& jobs, const G& g, double window) {
    if (!pcbgh_sched_on()) return;
    pcbg_rsched_begin(int32_t(order.size()));
    for (size_t p = 0; p < order.size(); ++p) {
        const pcbg_rnet r = pcbgh_rnet(g, jobs[order[p]].box, window);
        pcbg_rsched_net(int32_t(p), &r);
    }
}

inline bool pcbgh_allow(size_t pos, size_t cursor, size_t version) {
    if (!pcbgh_sched_on() || pos <= cursor) return true;
    return pcbg_rsched_allow(int32_t(pos), int32_t(cursor), int64_t(version)) != 0;
}

inline void pcbgh_started(size_t pos, size_t cursor, size_t version) {
    if (pcbgh_sched_on()) pcbg_rsched_started(int32_t(pos), int32_t(cursor), int64_t(version));
}

// The commits since the search at pos started that changed a block it read (the router's own test,
// src/router.cpp:2200-2205, run over every commit instead of stopping at the first).
template <class C>
void pcbgh_verdict(size_t pos, bool fine, size_t startver, const std::vector<std::vector<uint32_t>>& commits,
                   const C& touch, const C& touchv, size_t split) {
    if (!pcbgh_sched_on()) return;
    thread_local std::vector<int64_t> hits;
    hits.clear();
    for (size_t c = startver; c < commits.size(); ++c)
        for (uint32_t b : commits[c])
            if (b < split ? touch[b] : touchv[b - split]) { hits.push_back(int64_t(c)); break; }
    pcbg_rsched_verdict(int32_t(pos), fine ? 1 : 0, hits.data(), int32_t(hits.size()));
}

inline void pcbgh_commit(size_t pos, size_t index) {
    if (pcbgh_sched_on()) pcbg_rsched_committed(int32_t(pos), int64_t(index));
}

inline void pcbgh_end() {
    if (pcbgh_sched_on()) pcbg_rsched_end();
}
