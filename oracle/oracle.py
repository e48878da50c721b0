"""ctypes wrapper of the C oracle (oracle/_build/libpcboracle.so) -- TEST INFRASTRUCTURE ONLY.

solve() restates one gpu_solve() call of pcbroute (src/gpu.cu:550-622) exactly; dijkstra() solves a resolved
dense rectangle; weight() / start_d() expose the fixed-point rules of include/pcbg.h.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libpcboracle.so")
INF64 = 0x7F7F7F7F7F7F7F7F

_lib = None


class _Search(C.Structure):
    _fields_ = [
        ("rw", C.c_int), ("rh", C.c_int), ("nl", C.c_int),
        ("fac", (C.c_float * 8) * 8),
        ("cf", C.c_void_p), ("flags", C.c_void_p), ("vcf", C.c_void_p),
        ("n_starts", C.c_int64), ("start_idx", C.c_void_p), ("start_d", C.c_void_p),
        ("best", C.c_int64), ("best_d", C.c_uint64), ("settled", C.c_int64),
    ]


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            import sys
            sys.path.insert(0, os.path.dirname(HERE))
            from pcbroute_b200 import build
            build.build_oracle()
        L = C.CDLL(LIB_PATH)
        from pcbroute_b200 import _lib as plib
        L.pcbo_weight.argtypes = [C.c_float, C.c_float]
        L.pcbo_weight.restype = C.c_uint64
        L.pcbo_start_d.argtypes = [C.c_float]
        L.pcbo_start_d.restype = C.c_uint64
        L.pcbo_solve.argtypes = [C.POINTER(plib.Query), C.POINTER(plib.Result)]
        L.pcbo_solve.restype = C.c_int
        L.pcbo_free.argtypes = [C.c_void_p]
        L.pcbo_dijkstra.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64)]
        L.pcbo_dijkstra.restype = C.c_int64
        L.pcbo_walkback.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64]
        L.pcbo_walkback.restype = C.c_int64
        L.pcbo_report.argtypes = [C.c_int64, C.c_void_p, C.c_int64, C.c_uint64, C.c_void_p]
        L.pcbo_resolve.argtypes = [C.POINTER(plib.Query), C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                   C.c_void_p]
        L.pcbo_solve_many.argtypes = [C.POINTER(_Search), C.c_int, C.c_int]
        _lib = L
    return _lib


def weight(cf: float, fac: float) -> int:
    return int(lib().pcbo_weight(cf, fac))


def start_d(g0: float) -> int:
    return int(lib().pcbo_start_d(g0))


def factors(step: float, dirf: np.ndarray) -> np.ndarray:
    ln = np.array([step] * 4 + [np.float32(np.float64(step) * np.sqrt(2.0))] * 4, np.float32)
    return (ln[None, :] * np.asarray(dirf, np.float32).reshape(8, 8)).astype(np.float32)


def solve(q):
    """One gpu_solve() of pcbroute_b200.query.GpuQuery q: returns a pcbroute_b200.query.GpuOut (field as numpy)."""
    from pcbroute_b200.query import GpuOut
    from pcbroute_b200 import _lib as plib
    cq, keep = q.to_c()
    r = plib.Result()
    rc = lib().pcbo_solve(C.byref(cq), C.byref(r))
    del keep
    out = GpuOut()
    if rc < 0:
        return rc, out
    n = r.rw * r.rh * r.nl
    out.d = np.ctypeslib.as_array(r.d, shape=(n,)).copy().reshape(r.nl, r.rh, r.rw)
    lib().pcbo_free(C.cast(r.d, C.c_void_p))
    out.rx0, out.ry0, out.rw, out.rh, out.NL, out.ww, out.wh = r.rx0, r.ry0, r.rw, r.rh, r.nl, r.ww, r.wh
    out.best, out.tries, out.ub = int(r.best), r.tries, r.ub
    return rc, out


def resolve(q, rx0: int, ry0: int, rw: int, rh: int, vias: bool = True):
    """Resolved dense cf [nl, rh, rw], flags, vcf [rh, rw] of a rectangle of q's window."""
    cq, keep = q.to_c()
    cf = np.empty((q.NL, rh, rw), np.float32)
    fl = np.empty((q.NL, rh, rw), np.uint8)
    vcf = np.empty((rh, rw), np.float32) if vias else None
    lib().pcbo_resolve(C.byref(cq), rx0, ry0, rw, rh, cf.ctypes.data, fl.ctypes.data,
                       vcf.ctypes.data if vcf is not None else None)
    del keep
    return cf, fl, vcf


def dijkstra(fac: np.ndarray, cf: np.ndarray, flags: np.ndarray, vcf, start_idx, start_dv):
    """Exact distances (uint64 [nl, rh, rw]) of a resolved dense rectangle, best rect state, best cost."""
    nl, rh, rw = cf.shape
    fac = np.ascontiguousarray(fac, np.float32)
    cf = np.ascontiguousarray(cf, np.float32)
    flags = np.ascontiguousarray(flags, np.uint8)
    vcf = None if vcf is None else np.ascontiguousarray(vcf, np.float32)
    si = np.ascontiguousarray(start_idx, np.uint32)
    sd = np.ascontiguousarray(start_dv, np.uint64)
    dist = np.empty((nl, rh, rw), np.uint64)
    bd = C.c_uint64(0)
    best = lib().pcbo_dijkstra(rw, rh, nl, fac.ctypes.data, cf.ctypes.data, flags.ctypes.data,
                               None if vcf is None else vcf.ctypes.data, len(si), si.ctypes.data, sd.ctypes.data,
                               dist.ctypes.data, C.byref(bd))
    return dist, int(best), int(bd.value)


def walkback(fac: np.ndarray, cf: np.ndarray, flags: np.ndarray, vcf, start_idx, start_dv, dist: np.ndarray, best: int,
             cap: int = 1 << 20) -> np.ndarray | None:
    """Path (rect states, best first) of pcbo_walkback, [] if best < 0, None if the walk fails."""
    nl, rh, rw = cf.shape
    fac = np.ascontiguousarray(fac, np.float32)
    cf = np.ascontiguousarray(cf, np.float32)
    flags = np.ascontiguousarray(flags, np.uint8)
    vcf = None if vcf is None else np.ascontiguousarray(vcf, np.float32)
    si = np.ascontiguousarray(start_idx, np.uint32)
    sd = np.ascontiguousarray(start_dv, np.uint64)
    d = np.ascontiguousarray(dist, np.uint64)
    path = np.empty(cap, np.uint32)
    n = lib().pcbo_walkback(rw, rh, nl, fac.ctypes.data, cf.ctypes.data, flags.ctypes.data,
                            None if vcf is None else vcf.ctypes.data, len(si), si.ctypes.data, sd.ctypes.data,
                            d.ctypes.data, best, path.ctypes.data, cap)
    return None if n < 0 else path[:n].copy()


def report(dist: np.ndarray, best: int, best_d: int) -> np.ndarray:
    out = np.empty(dist.shape, np.float32)
    d = np.ascontiguousarray(dist, np.uint64)
    lib().pcbo_report(d.size, d.ctypes.data, best, best_d, out.ctypes.data)
    return out


def solve_many(searches: list[dict], threads: int) -> list[tuple[int, int, int]]:
    """Solve resolved dense searches on host threads (taken in list order). Each dict: fac, cf, flags, vcf,
    start_idx, start_d. Returns (best, best_d, settled) per search: settled counts the states at or below best_d
    (every reached state when no target is reached)."""
    arr = (_Search * len(searches))()
    keep = []
    for k, s in enumerate(searches):
        nl, rh, rw = s["cf"].shape
        a = arr[k]
        a.rw, a.rh, a.nl = rw, rh, nl
        fac = np.ascontiguousarray(s["fac"], np.float32)
        for l in range(8):
            for m in range(8):
                a.fac[l][m] = float(fac[l, m])
        cf = np.ascontiguousarray(s["cf"], np.float32)
        fl = np.ascontiguousarray(s["flags"], np.uint8)
        vcf = None if s["vcf"] is None else np.ascontiguousarray(s["vcf"], np.float32)
        si = np.ascontiguousarray(s["start_idx"], np.uint32)
        sd = np.ascontiguousarray(s["start_d"], np.uint64)
        keep += [cf, fl, vcf, si, sd]
        a.cf, a.flags = cf.ctypes.data, fl.ctypes.data
        a.vcf = None if vcf is None else vcf.ctypes.data
        a.n_starts, a.start_idx, a.start_d = len(si), si.ctypes.data, sd.ctypes.data
    lib().pcbo_solve_many(arr, len(searches), threads)
    return [(int(arr[k].best), int(arr[k].best_d), int(arr[k].settled)) for k in range(len(searches))]


def costs_rebuild(st, oc, ov, vst, hist, gnd, pres: float, hard: bool):
    """Cost maps of every class (src/router.cpp:386-405): st/oc/ov [k, l, n], vst [k, n], hist [l, n],
    gnd: list per layer of [n] float32 or None. Returns cst [k, l, n], vcst [k, n]."""
    k, nl, n = st.shape
    L = lib()
    L.pcbo_costs_rebuild.argtypes = [C.c_int] * 3 + [C.c_void_p] * 6 + [C.c_float, C.c_int, C.c_void_p, C.c_void_p]
    st = np.ascontiguousarray(st, np.uint16)
    oc = np.ascontiguousarray(oc, np.uint8)
    ov = np.ascontiguousarray(ov, np.uint8)
    vst = np.ascontiguousarray(vst, np.uint16)
    hist = np.ascontiguousarray(hist, np.float32)
    gk = [None if g is None else np.ascontiguousarray(g, np.float32) for g in (gnd or [None] * nl)]
    gp = (C.c_void_p * nl)(*[None if g is None else g.ctypes.data for g in gk])
    cst = np.empty((k, nl, n), np.float32)
    vcst = np.empty((k, n), np.float32)
    L.pcbo_costs_rebuild(n, nl, k, st.ctypes.data, oc.ctypes.data, ov.ctypes.data, vst.ctypes.data, hist.ctypes.data,
                         C.cast(gp, C.c_void_p), pres, 1 if hard else 0, cst.ctypes.data, vcst.ctypes.data)
    return cst, vcst
