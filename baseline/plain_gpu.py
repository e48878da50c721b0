"""The plain GPU back end against this one, search by search, on the batched-search microbenchmark's own searches.

Each arm solves the same first N searches of the workload (seed 20261203; windows 64-2048 cells per side, 2-6
layers) through the one-search `gpu_solve` contract, from dense host arrays, with the upload, the solve and the
field download inside the timed call:

  ref    pcbroute's src/gpu.cu built for sm_100a (baseline/_ref/librefgpu.so, refgpu_solve_dense)
  b200   this library's pcbg_solve (the gpu.h path the router links)

The reference back end sweeps in float and this one relaxes in exact integers, so only the best targets' positions
are compared, not the fields. Each arm runs in its own process; one JSON line per arm:

    python baseline/plain_gpu.py --arm ref --searches 48
    python baseline/plain_gpu.py --arm b200 --searches 48
"""
import argparse
import ctypes as C
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from pcbroute_b200 import _lib, query, synth  # noqa: E402

SEED = 20261203


def make(lib, k, sizes):
    rw, rh, nl, via, sseed = sizes[k]
    n = rw * rh
    cf = np.empty(nl * n, np.float32)
    fl = np.empty(nl * n, np.uint8)
    vcf = np.empty(n, np.float32)
    st = np.zeros(2, np.int64)
    rc = lib.pcbg_synth_search_host(sseed, rw, rh, nl, via, cf.ctypes.data, fl.ctypes.data, vcf.ctypes.data,
                                    st.ctypes.data, os.cpu_count() or 1)
    assert rc == 0
    src, tgt = int(st[0]), int(st[1])
    tbit = np.zeros(nl * n // 64 + 1, np.uint64)
    if tgt >= 0:
        tbit[tgt >> 6] |= np.uint64(1) << np.uint64(tgt & 63)
    return dict(rw=rw, rh=rh, nl=nl, via=via, cst=cf, st=np.zeros(nl * n, np.uint16), vcst=np.ones(n, np.float32),
                vst=np.zeros(n, np.uint16), tbit=tbit, src=src, tgt=tgt, states=nl * n)


def run_ref(s, ref):
    best = C.c_int64(-1)
    secs = C.c_double(0)
    r = ref.refgpu_solve_dense(s["rw"], s["rh"], s["nl"], s["cst"].ctypes.data, s["st"].ctypes.data,
                               s["vcst"].ctypes.data, s["vst"].ctypes.data, s["tbit"].ctypes.data, s["src"],
                               C.c_float(s["via"]), C.byref(best), C.byref(secs))
    return r, int(best.value), float(secs.value)


def run_b200(s, lib):
    import time
    nl = s["nl"]
    dirf = np.ones((8, 8), np.float32)
    lay = np.array([1 if l < nl else 0 for l in range(8)], np.uint8)
    q = query.GpuQuery(nx=s["rw"], ny=s["rh"], NL=nl, wi0=0, wj0=0, ww=s["rw"], wh=s["rh"], me=1, via_cost=s["via"],
                       step=1.0, dirf=dirf, lay=lay, cst=s["cst"].reshape(nl, -1), st=s["st"].reshape(nl, -1),
                       vcst=s["vcst"], vst=s["vst"], tbit=s["tbit"], starts=[(s["src"], 0.0)])
    cq, keep = q.to_c()
    r = _lib.Result()
    t0 = time.perf_counter()
    rc = lib.pcbg_solve(C.byref(cq), C.byref(r), 1)
    secs = time.perf_counter() - t0
    best = int(r.best)
    if r.d:
        lib.pcbg_host_release(r.d, r.cap)
    del keep
    return rc, best, secs


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--arm", choices=["ref", "b200"], required=True)
    ap.add_argument("--searches", type=int, default=48)
    ap.add_argument("--max-states", type=int, default=48 << 20, help="skip searches above this many states")
    a = ap.parse_args()
    lib = _lib.load()
    ref = None
    if a.arm == "ref":
        ref = C.CDLL(os.path.join(ROOT, "baseline", "_ref", "librefgpu.so"))
        ref.refgpu_solve_dense.restype = C.c_int
        ref.refgpu_solve_dense.argtypes = [C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 5 + \
            [C.c_uint32, C.c_float, C.POINTER(C.c_int64), C.POINTER(C.c_double)]
    sizes = synth.microbench_sizes(SEED, a.searches)
    solve = (lambda s: run_ref(s, ref)) if ref else (lambda s: run_b200(s, lib))
    solve(make(lib, 0, sizes))   # warm-up: context, module load, first allocations
    states = secs = 0.0
    n = failed = 0
    bests = []
    for k in range(a.searches):
        if sizes[k][0] * sizes[k][1] * sizes[k][2] > a.max_states:
            continue
        s = make(lib, k, sizes)
        rc, best, t = solve(s)
        if rc < 0:
            failed += 1
            continue
        states += s["states"]
        secs += t
        n += 1
        bests.append(best == s["tgt"] if s["tgt"] >= 0 else best < 0)
    print(json.dumps({"arm": a.arm, "searches": n, "failed": failed, "states": int(states), "seconds": round(secs, 3),
                      "gcell_relax_s": round(9.0 * states / secs / 1e9, 4) if secs else None,
                      "best_is_the_target": sum(bests), "workload": f"first {a.searches} microbenchmark searches"}))


if __name__ == "__main__":
    main()
