"""Test infrastructure only (never used by the product path): the sequential meaning of a speculative negotiation
iteration, restated on the CPU with the oracle's own pieces.

pcbroute's route_waves commits nets in a fixed order and accepts a speculative search only when no earlier commit
changed what it read, so its result is that of routing the nets one by one (src/router.cpp:2096-2118). This file
routes them one by one:

  * the cost maps from the oracle's cost_xp / vcost_xp restatement (pcbo_costs_rebuild, src/router.cpp:383-420),
    rebuilt before every net from the static grids, the occupancy and the history;
  * each net's window resolved the way csrc/spec.cu resolves it (free finite costs pass; via cost times via_cost;
    a via lands wherever the layer passes; the target bit);
  * the oracle's exact Dijkstra and walk-back (pcbo_dijkstra, pcbo_walkback);
  * the path stamped into the occupancy: +1 track occupancy per state on its layer, +1 via occupancy on the lower
    layer at every layer change (the stamp of src/router.cpp:1892-1963);
  * between iterations, rip-up of every path, and history += inc on every state two or more paths share
    (count_conflicts, src/router.cpp:1970-1999).
"""
from __future__ import annotations

import numpy as np

from oracle import oracle

CINF = np.float32(1e30)


def _fac(nl: int) -> np.ndarray:
    f = np.ones((8, 8), np.float32)
    f[:, 4:] = np.float32(np.sqrt(2.0))
    return f


def _stamp(b, oc, ov, path, sign):
    board = b["n"]
    for k, s in enumerate(path):
        l, c = divmod(int(s), board)
        oc[0, l, c] = np.uint8(int(oc[0, l, c]) + sign)
        if k + 1 < len(path):
            l2, c2 = divmod(int(path[k + 1]), board)
            if l2 != l and c2 == c:
                lo = min(l, l2)
                ov[0, lo, c] = np.uint8(int(ov[0, lo, c]) + sign)


def route_net(b, cst, vcst, net, via_cost):
    nx, nl, board = b["nx"], b["nl"], b["n"]
    x0, y0, x1, y1, src, tgt = net
    rw, rh = x1 - x0, y1 - y0
    win = cst[0].reshape(nl, b["ny"], nx)[:, y0:y1, x0:x1]
    cf = np.where((win > 0) & (win < CINF), win, CINF).astype(np.float32)
    fl = ((win > 0) & (win < CINF)).astype(np.uint8)
    tl, tc = divmod(tgt, board)
    fl[tl, tc // nx - y0, tc % nx - x0] |= 2
    vw = vcst[0].reshape(b["ny"], nx)[y0:y1, x0:x1]
    vcf = np.where((vw > 0) & (vw < CINF), vw * np.float32(via_cost), CINF).astype(np.float32)
    sl, sc = divmod(src, board)
    si = np.array([(sl * rh + (sc // nx - y0)) * rw + (sc % nx - x0)], np.uint32)
    sd = np.zeros(1, np.uint64)
    fac = _fac(nl)
    dist, best, _ = oracle.dijkstra(fac, cf, fl, vcf, si, sd)
    rect = oracle.walkback(fac, cf, fl, vcf, si, sd, dist, best)
    assert rect is not None
    out = []
    for r in rect:
        l, c = divmod(int(r), rw * rh)
        out.append(l * board + (y0 + c // rw) * nx + (x0 + c % rw))
    return np.array(out, np.uint32)


def negotiate(b: dict, iters: int, hist_inc: float = 1.0, via_cost: float = 4.0, pres_of=None) -> list[np.ndarray]:
    nl, n = b["nl"], b["n"]
    st = b["st"][None].astype(np.uint16)
    vst = b["vst"][None].astype(np.uint16)
    oc = np.zeros((1, nl, n), np.uint8)
    ov = np.zeros((1, nl, n), np.uint8)
    hist = np.zeros((nl, n), np.float32)
    paths = [np.zeros(0, np.uint32) for _ in b["nets"]]
    for it in range(iters):
        pres = pres_of(it)
        for p in paths:
            _stamp(b, oc, ov, p, -1)
        paths = []
        for net in b["nets"]:
            cst, vcst = oracle.costs_rebuild(st, oc, ov, vst, hist, None, pres, False)
            p = route_net(b, cst, vcst, net, via_cost)
            _stamp(b, oc, ov, p, +1)
            paths.append(p)
        if it + 1 < iters:
            allp = np.concatenate([np.unique(p) for p in paths]) if paths else np.zeros(0, np.uint32)
            vals, counts = np.unique(allp, return_counts=True)
            for s in vals[counts > 1]:
                l, c = divmod(int(s), n)
                hist[l, c] = np.float32(hist[l, c] + np.float32(hist_inc))
    return paths
