"""Speculative negotiation rounds on the B200 (csrc/spec.cu): the Python side of pcbg_spec_* and its board generator.

A `Round` owns a device cost board (one class) and a fixed order of nets. `iterate()` is one rip-up-and-reroute
iteration of PathFinder, routed the way pcbroute's route_waves routes a wave (src/router.cpp:2096-2242): nets
searched ahead of the commit point, committed in order, searched again when a commit changed their window.

`spec_board()` makes the seeded boards the speculation tests and the scheduler's training use: obstacle blobs on
every layer, two-pin nets with pins on the top layer, windows = the pins' box plus a margin.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

SEQUENTIAL, PLAIN, LEARNED = 0, 1, 2


def spec_board(seed: int, nx: int = 192, ny: int = 160, nl: int = 4, nnets: int = 96, margin: int = 12,
               span: tuple[int, int] = (16, 90), block: float = 0.12) -> dict:
    """Seeded board: static grids (0 free, 0xFFFF blocked) with blob obstacles, and nets (window, src, tgt).
    Pins are free cells of layer 0; a pin's cell stays free on every layer so that vias can leave it."""
    rng = np.random.default_rng(seed)
    n = nx * ny
    yy, xx = np.mgrid[0:ny, 0:nx]
    st = np.zeros((nl, n), np.uint16)
    for l in range(nl):
        field = np.zeros((ny, nx), np.float32)
        for _ in range(max(4, n // 900)):
            cx, cy, r = rng.uniform(0, nx), rng.uniform(0, ny), rng.uniform(2, 9)
            field += np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2 * r * r)).astype(np.float32)
        thr = np.quantile(field, 1.0 - block)
        st[l][(field >= thr).reshape(-1)] = 0xFFFF
    nets = []
    used = set()
    board = n
    tries = 0
    while len(nets) < nnets and tries < 100000:
        tries += 1
        sx, sy = int(rng.integers(1, nx - 1)), int(rng.integers(1, ny - 1))
        d = int(rng.integers(span[0], span[1]))
        ang = rng.uniform(0, 2 * np.pi)
        tx, ty = int(round(sx + d * np.cos(ang))), int(round(sy + d * np.sin(ang)))
        if not (1 <= tx < nx - 1 and 1 <= ty < ny - 1):
            continue
        cs, ct = sy * nx + sx, ty * nx + tx
        if cs in used or ct in used or cs == ct:
            continue
        if st[0, cs] or st[0, ct]:
            continue
        used.update((cs, ct))
        x0, x1 = max(0, min(sx, tx) - margin), min(nx, max(sx, tx) + margin + 1)
        y0, y1 = max(0, min(sy, ty) - margin), min(ny, max(sy, ty) + margin + 1)
        nets.append((x0, y0, x1, y1, cs, ct))
    for (_, _, _, _, cs, ct) in nets:
        st[:, cs] = 0
        st[:, ct] = 0
    vst = np.where((st == 0xFFFF).all(axis=0), 0xFFFF, 0).astype(np.uint16)
    return dict(nx=nx, ny=ny, nl=nl, n=n, st=st, vst=vst, nets=nets, board=board, seed=seed)


class Round:
    """pcbg_costs (one class) + pcbg_spec over a spec_board()."""

    def __init__(self, b: dict, via_cost: float = 4.0):
        self.lib = _lib.load()
        L = self.lib
        self.b = b
        self.h = L.pcbg_costs_create(b["nx"], b["ny"], b["nl"], 1)
        if not self.h:
            raise RuntimeError(_lib.last_error())
        st = np.ascontiguousarray(b["st"], np.uint16)
        vst = np.ascontiguousarray(b["vst"], np.uint16)
        if L.pcbg_costs_set_static(self.h, 0, st.ctypes.data, vst.ctypes.data) != 0:
            raise RuntimeError(_lib.last_error())
        arr = (_lib.Net * len(b["nets"]))()
        for k, (x0, y0, x1, y1, s, t) in enumerate(b["nets"]):
            arr[k].x0, arr[k].y0, arr[k].x1, arr[k].y1, arr[k].src, arr[k].tgt = x0, y0, x1, y1, s, t
        self.s = L.pcbg_spec_create(self.h, 0, arr, len(b["nets"]), via_cost)
        if not self.s:
            raise RuntimeError(_lib.last_error())
        self._keep = []

    def set_scheduler(self, fn):
        """fn(cursor, cand list) -> list of picked candidates (ints); a Python callback for tests."""
        def cb(user, spec, cursor, cand, n, pick):
            chosen = set(fn(int(cursor), [int(cand[k]) for k in range(n)]))
            for k in range(n):
                pick[k] = 1 if int(cand[k]) in chosen else 0
            return 0
        f = _lib.SCHEDULER(cb)
        self._keep.append(f)
        self.lib.pcbg_spec_set_scheduler(self.s, f, None)

    def set_scheduler_ptr(self, fn_ptr: int, user: int):
        f = C.cast(C.c_void_p(fn_ptr), _lib.SCHEDULER)
        self._keep.append(f)
        self.lib.pcbg_spec_set_scheduler(self.s, f, C.c_void_p(user))

    def iterate(self, pres: float, policy: int, width: int) -> dict:
        st = _lib.SpecStats()
        if self.lib.pcbg_spec_iterate(self.s, pres, policy, width, C.byref(st)) != 0:
            raise RuntimeError(_lib.last_error())
        return {k: getattr(st, k) for k, _ in _lib.SpecStats._fields_}

    def paths(self) -> list[np.ndarray]:
        out = []
        for k in range(len(self.b["nets"])):
            n = self.lib.pcbg_spec_path(self.s, k, None, 0)
            a = np.empty(max(n, 0), np.uint32)
            if n > 0:
                self.lib.pcbg_spec_path(self.s, k, a.ctypes.data, n)
            out.append(a)
        return out

    def add_history(self, inc: float) -> int:
        r = self.lib.pcbg_spec_add_history(self.s, inc)
        if r < 0:
            raise RuntimeError(_lib.last_error())
        return r

    def close(self):
        if self.s:
            self.lib.pcbg_spec_destroy(self.s)
            self.s = None
        if self.h:
            self.lib.pcbg_costs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pres_of(it: int) -> float:
    """Present-congestion factor of iteration it: 0.5, growing x1.6 per iteration (pcbroute's log shows 0.50,
    0.80, 1.28, ...)."""
    return 0.5 * 1.6 ** it


def negotiate(b: dict, iters: int, policy: int, width: int, hist_inc: float = 1.0, scheduler=None,
              via_cost: float = 4.0) -> tuple[list[np.ndarray], list[dict]]:
    """`iters` iterations of rip-up and reroute with history between them; returns the final paths and the
    per-iteration stats."""
    r = Round(b, via_cost)
    try:
        if scheduler is not None:
            scheduler(r)
        stats = []
        for it in range(iters):
            s = r.iterate(pres_of(it), policy, width)
            stats.append(s)
            if it + 1 < iters:
                r.add_history(hist_inc)
        return r.paths(), stats
    finally:
        r.close()
