"""The oracle pinned to pcbroute's own search back end: src/gpu.cu, built unchanged for sm_100a by
baseline/Makefile into baseline/_ref/librefgpu.so (src/gpu.cu:422-622, reached through refgpu_solve_field in
baseline/refgpu_wrap.cpp).

The reference relaxes in float and the oracle in fixed point (a move weight is rint(16 * cf * fac)), so the two
fields agree to the fixed point's quantization, and exactly where the quantization is exact:

  * unit diagonals: with the diagonal direction factor fl(1/sqrt 2), every move of the microbenchmark's integer
    costs weighs an integer in both back ends (the reference's factor rounds to 1 - 6e-8), so the fields agree to
    the reference's float rounding: a relative 1e-5;
  * sqrt 2 diagonals (the workload as benchmarked): each move's fixed-point weight is within 1/32 of the float one
    and every move costs at least 1, so a path of cost D differs by at most D / 32 between the two. The test checks
    that bound, and that the mean relative difference stays far below it.

Compared: the solved rectangle (the same growth rule, src/gpu.cu:575-619), the best target, and the field on every
state below the best target's cost (the reference prunes relaxations at its bound, src/gpu.cu:353-363, so states
at or above it are not settled there).
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import oracle
from pcbroute_b200 import query, synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "baseline", "_ref", "librefgpu.so")
INV_SQRT2 = float(np.float32(1.0) / np.float32(np.sqrt(2.0)))


def _ref():
    if not os.path.exists(REF_LIB):
        pytest.skip("baseline/_ref/librefgpu.so not built (needs the pcbroute sources at build time)")
    lib = C.CDLL(REF_LIB)
    lib.refgpu_solve_field.restype = C.c_int
    lib.refgpu_solve_field.argtypes = [C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 5 + \
        [C.c_uint32, C.c_float, C.c_float, C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]
    return lib


def _searches(n, max_states):
    sizes = synth.microbench_sizes(20261203, 4096)
    out = []
    for k, (rw, rh, nl, via, seed) in enumerate(sizes):
        if rw * rh * nl <= max_states:
            out.append((rw, rh, nl, via, seed))
        if len(out) == n:
            break
    return out


def _solve_both(ref, rw, rh, nl, via, seed, diag):
    cf, fl, vcf, src, tgt = synth.search_arrays(seed, rw, rh, nl, via)
    n = rw * rh
    cst = np.ascontiguousarray(cf.reshape(nl, n))
    st = np.zeros((nl, n), np.uint16)
    vcst = np.ones(n, np.float32)
    vst = np.zeros(n, np.uint16)
    tbit = np.zeros(nl * n // 64 + 1, np.uint64)
    tbit[tgt >> 6] |= np.uint64(1) << np.uint64(tgt & 63)
    field = np.empty(nl * n, np.float32)
    rect = np.zeros(4, np.int32)
    best = C.c_int64(-1)
    rc = ref.refgpu_solve_field(rw, rh, nl, cst.ctypes.data, st.ctypes.data, vcst.ctypes.data, vst.ctypes.data,
                                tbit.ctypes.data, src, via, diag, rect.ctypes.data, field.ctypes.data, field.size,
                                C.byref(best))
    assert rc >= 1, rc
    dirf = np.ones((8, 8), np.float32)
    dirf[:, 4:] = diag
    lay = np.array([1 if l < nl else 0 for l in range(8)], np.uint8)
    q = query.GpuQuery(nx=rw, ny=rh, NL=nl, wi0=0, wj0=0, ww=rw, wh=rh, me=1, via_cost=via, step=1.0, dirf=dirf,
                       lay=lay, cst=cst, st=st, vcst=vcst, vst=vst, tbit=tbit, starts=[(src, 0.0)])
    orc, o = oracle.solve(q)
    assert orc >= 1
    r = dict(rect=tuple(int(x) for x in rect), best=int(best.value),
             d=field[:nl * rect[2] * rect[3]].reshape(nl, rect[3], rect[2]))
    return r, o


@pytest.mark.parametrize("diag", ["unit", "sqrt2"])
def test_reference_backend_fields_match_the_oracle(diag):
    ref = _ref()
    dval = INV_SQRT2 if diag == "unit" else 1.0
    same_rect = compared = 0
    rel_sum, rel_n = 0.0, 0
    cases = _searches(20, 3_000_000)
    for (rw, rh, nl, via, seed) in cases:
        r, o = _solve_both(ref, rw, rh, nl, via, seed, dval)
        if r["rect"] != (o.rx0, o.ry0, o.rw, o.rh):
            continue
        same_rect += 1
        assert r["best"] == o.best, (rw, rh, nl, r["best"], o.best)
        ub_o = float(o.ub)
        ub_r = float(r["d"].reshape(-1)[_rect_index(o, o.best)])
        low = o.d < min(ub_o, ub_r) * (1 - 1e-4)
        a, b = o.d[low].astype(np.float64), r["d"][low].astype(np.float64)
        rel = np.abs(a - b) / np.maximum(a, 1.0)
        if diag == "unit":
            assert rel.max(initial=0) <= 1e-5, (rw, rh, nl, rel.max())
            assert abs(ub_r - ub_o) <= 1e-5 * ub_o
        else:
            assert rel.max(initial=0) <= 1.0 / 32, (rw, rh, nl, rel.max())
        rel_sum += rel.sum()
        rel_n += rel.size
        compared += 1
    # the growth rule is the same; only a float / fixed-point tie at the octile bound could change a rectangle
    assert same_rect >= 0.9 * len(cases), (same_rect, len(cases))
    assert compared and rel_n
    if diag == "sqrt2":
        assert rel_sum / rel_n < 2e-3, rel_sum / rel_n


def _rect_index(o, best):
    """Index into the rectangle field of window state `best`."""
    wn = o.ww * o.wh
    l, c = divmod(best, wn)
    i, j = c % o.ww - o.rx0, c // o.ww - o.ry0
    return (l * o.rh + j) * o.rw + i
