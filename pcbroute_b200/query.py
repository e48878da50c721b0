"""Python mirror of pcbroute's GpuQuery / GpuOut / gpu_solve (src/gpu.h:10-57) over the pcbg C ABI.

A GpuQuery holds numpy arrays for the full-grid cost maps and the window's target bits, and the (index, value)
lists the router builds in gpu_finish (src/router.cpp:1527-1584). gpu_solve() fills a GpuOut with the solved
rectangle, the best target and the reported field, with the reference's return convention (>= 1 on success,
-1 failure, -3 busy). The call goes through libpcbgpu.so; there is no CPU path here.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib

SQRT2 = float(np.sqrt(np.float64(2.0)))


def _ptr(a: np.ndarray | None) -> int | None:
    return None if a is None else a.ctypes.data


@dataclass
class GpuQuery:
    """src/gpu.h:10-36. cst/st: [NL, ny * nx] (layer-major); vcst/vst: [ny * nx]; tbit: uint64 words over the
    window states l * ww * wh + j * ww + i."""
    nx: int
    ny: int
    NL: int
    wi0: int
    wj0: int
    ww: int
    wh: int
    me: int
    via_cost: float
    step: float
    dirf: np.ndarray                      # [8, 8] float32
    lay: np.ndarray                       # [8] uint8
    cst: np.ndarray                       # [NL, ny * nx] float32
    st: np.ndarray                        # [NL, ny * nx] uint16
    vcst: np.ndarray                      # [ny * nx] float32
    vst: np.ndarray                       # [ny * nx] uint16
    tbit: np.ndarray                      # uint64
    own_cf: list = field(default_factory=list)
    own_vcf: list = field(default_factory=list)
    starts: list = field(default_factory=list)
    prior: np.ndarray | None = None       # [pnl, ph, pw] uint8
    pi0: int = 0
    pj0: int = 0
    pcol: np.ndarray | None = None        # [nx] int32
    prow: np.ndarray | None = None        # [ny] int32
    play: np.ndarray | None = None        # [8] int32
    mlf: np.ndarray | None = None         # [256] float32
    mthr: int = 0
    corridor: bool = False

    def window_states(self) -> int:
        return self.ww * self.wh * self.NL

    def to_c(self) -> tuple[_lib.Query, list]:
        """The pcbg_query struct and the arrays it points into (keep them alive during the call)."""
        keep = []
        q = _lib.Query()
        q.nx, q.ny, q.nl = self.nx, self.ny, self.NL
        q.wi0, q.wj0, q.ww, q.wh = self.wi0, self.wj0, self.ww, self.wh
        q.me = self.me
        q.via_cost, q.step = self.via_cost, self.step
        d = np.ascontiguousarray(self.dirf, dtype=np.float32).reshape(8, 8)
        for l in range(8):
            for m in range(8):
                q.dirf[l][m] = float(d[l, m])
            q.lay[l] = int(self.lay[l])
        cst = np.ascontiguousarray(self.cst, dtype=np.float32)
        st = np.ascontiguousarray(self.st, dtype=np.uint16)
        keep += [cst, st]
        for l in range(self.NL):
            q.cst[l] = cst[l].ctypes.data
            q.st[l] = st[l].ctypes.data
        vcst = np.ascontiguousarray(self.vcst, dtype=np.float32)
        vst = np.ascontiguousarray(self.vst, dtype=np.uint16)
        tbit = np.ascontiguousarray(self.tbit, dtype=np.uint64)
        keep += [vcst, vst, tbit]
        q.vcst, q.vst, q.tbit = _ptr(vcst), _ptr(vst), _ptr(tbit)

        def pairs(lst):
            idx = np.array([p[0] for p in lst], dtype=np.uint32)
            val = np.array([p[1] for p in lst], dtype=np.float32)
            keep.extend([idx, val])
            return _ptr(idx) if len(lst) else None, _ptr(val) if len(lst) else None, len(lst)

        q.own_cf_idx, q.own_cf_val, q.n_own_cf = pairs(self.own_cf)
        q.own_vcf_idx, q.own_vcf_val, q.n_own_vcf = pairs(self.own_vcf)
        q.start_idx, q.start_val, q.n_starts = pairs(self.starts)
        play = self.play if self.play is not None else -np.ones(8, np.int32)
        for l in range(8):
            q.play[l] = int(play[l])
        mlf = self.mlf if self.mlf is not None else np.ones(256, np.float32)
        for v in range(256):
            q.mlf[v] = float(mlf[v])
        if self.prior is not None:
            prior = np.ascontiguousarray(self.prior, dtype=np.uint8)
            pcol = np.ascontiguousarray(self.pcol, dtype=np.int32)
            prow = np.ascontiguousarray(self.prow, dtype=np.int32)
            keep += [prior, pcol, prow]
            q.prior, q.pcol, q.prow = _ptr(prior), _ptr(pcol), _ptr(prow)
            q.pnl, q.ph, q.pw = prior.shape
            q.pi0, q.pj0 = self.pi0, self.pj0
        q.mthr = self.mthr
        q.corridor = 1 if self.corridor else 0
        return q, keep


@dataclass
class GpuOut:
    """src/gpu.h:39-50, with the field copied out of the pinned buffer as a numpy array [NL, rh, rw]."""
    rx0: int = 0
    ry0: int = 0
    rw: int = 0
    rh: int = 0
    NL: int = 0
    ww: int = 0
    wh: int = 0
    best: int = -1
    d: np.ndarray | None = None
    rounds: int = 0
    tries: int = 0
    wide: bool = False
    tile_visits: int = 0
    ub: float = 1e30

    def __call__(self, q: int) -> float:
        """Cost of a window state (1e30 outside the solved rectangle), as GpuOut::operator() (src/gpu.cu:409-416)."""
        wn = self.ww * self.wh
        l, c = divmod(q, wn)
        i, j = c % self.ww - self.rx0, c // self.ww - self.ry0
        if i < 0 or j < 0 or i >= self.rw or j >= self.rh:
            return 1e30
        return float(self.d[l, j, i])


def available() -> bool:
    return bool(_lib.load().pcbg_available())


def configure(slots: int, max_states: int) -> None:
    _lib.load().pcbg_configure(slots, max_states)


def gpu_solve(q: GpuQuery, out: GpuOut, wait: bool = True) -> int:
    """src/gpu.h:55-57. Returns the rounds taken (>= 1), -1 on failure, -3 if busy and not waiting."""
    lib = _lib.load()
    cq, keep = q.to_c()
    r = _lib.Result()
    rc = lib.pcbg_solve(C.byref(cq), C.byref(r), 1 if wait else 0)
    del keep
    try:
        if rc < 0:
            return rc
        n = r.rw * r.rh * r.nl
        arr = np.ctypeslib.as_array(r.d, shape=(n,)).copy().reshape(r.nl, r.rh, r.rw)
        out.rx0, out.ry0, out.rw, out.rh, out.NL, out.ww, out.wh = r.rx0, r.ry0, r.rw, r.rh, r.nl, r.ww, r.wh
        out.best, out.d = int(r.best), arr
        out.rounds, out.tries, out.wide, out.tile_visits, out.ub = r.rounds, r.tries, bool(r.wide), r.tile_visits, r.ub
        return rc
    finally:
        if r.d:
            lib.pcbg_host_release(r.d, r.cap)
