"""Device-resident congestion cost maps (csrc/costs.cu) against the oracle's restatement of pcbroute's cost_xp /
vcost_xp (src/router.cpp:386-405), bit for bit: full rebuilds, commit stamps (occupancy +-1 and refresh over spans)
and history increments (count_conflicts, src/router.cpp:1970-1999)."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle
from pcbroute_b200 import _lib


def board(seed, nx=97, ny=61, nl=3, ncls=2, ground=True):
    rng = np.random.default_rng(seed)
    n = nx * ny
    st = np.zeros((ncls, nl, n), np.uint16)
    st[rng.random(st.shape) < 0.1] = 0xFFFF
    own = rng.random(st.shape) < 0.1
    st[own] = rng.integers(1, 30, size=int(own.sum())).astype(np.uint16)
    vst = np.zeros((ncls, n), np.uint16)
    vst[rng.random(vst.shape) < 0.1] = 0xFFFF
    vown = rng.random(vst.shape) < 0.08
    vst[vown] = rng.integers(1, 30, size=int(vown.sum())).astype(np.uint16)
    oc = rng.integers(0, 4, size=(ncls, nl, n)).astype(np.uint8) * (rng.random((ncls, nl, n)) < 0.3)
    ov = rng.integers(0, 3, size=(ncls, nl, n)).astype(np.uint8) * (rng.random((ncls, nl, n)) < 0.2)
    hist = (rng.random((nl, n)) * rng.integers(0, 5, size=(nl, n))).astype(np.float32)
    gnd = [None] * nl
    if ground:
        gnd[nl // 2] = np.where(rng.random(n) < 0.5, np.float32(2.5), np.float32(1.0)).astype(np.float32)
    return dict(nx=nx, ny=ny, nl=nl, ncls=ncls, st=st, vst=vst, oc=oc.astype(np.uint8), ov=ov.astype(np.uint8),
                hist=hist, gnd=gnd)


def numpy_costs(b, pres, hard):
    """Independent restatement of cost_xp / vcost_xp in float32 numpy (one IEEE op per step)."""
    st, oc, ov, vst, hist = b["st"], b["oc"].astype(np.int64), b["ov"].astype(np.int64), b["vst"], b["hist"]
    one = np.float32(1)
    pres = np.float32(pres)
    cst = np.empty(st.shape, np.float32)
    for k in range(st.shape[0]):
        for l in range(st.shape[1]):
            occ = oc[k, l]
            v = (one + hist[l]) * (one + pres * np.maximum(occ, 0).astype(np.float32))
            if b["gnd"][l] is not None:
                v = v * b["gnd"][l]
            v = np.where(st[k, l] == 0, v, -v)
            v = np.where((st[k, l] == 0xFFFF) | ((occ > 0) & hard), np.float32(1e30), v)
            cst[k, l] = v.astype(np.float32)
    vcst = np.empty(vst.shape, np.float32)
    hs = np.zeros(hist.shape[1], np.float32)
    for l in range(hist.shape[0]):
        hs = (hs + hist[l]).astype(np.float32)
    for k in range(st.shape[0]):
        occ = ov[k].sum(axis=0)
        v = (one + hs / np.float32(hist.shape[0])) * (one + pres * np.maximum(occ, 0).astype(np.float32))
        v = np.where(vst[k] == 0, v, -v)
        vcst[k] = np.where((vst[k] == 0xFFFF) | ((occ > 0) & hard), np.float32(1e30), v).astype(np.float32)
    return cst, vcst


def oracle_costs(b, pres, hard):
    return oracle.costs_rebuild(b["st"], b["oc"], b["ov"], b["vst"], b["hist"], b["gnd"], pres, hard)


@pytest.mark.parametrize("seed,pres,hard", [(1, 0.5, False), (2, 7.25, False), (3, 1e4, False), (4, 3.0, True)])
def test_oracle_costs_match_numpy_restatement(seed, pres, hard):
    b = board(seed)
    c1, v1 = oracle_costs(b, pres, hard)
    c2, v2 = numpy_costs(b, pres, hard)
    assert np.array_equal(c1.view(np.uint32), c2.view(np.uint32))
    assert np.array_equal(v1.view(np.uint32), v2.view(np.uint32))


class Dev:
    def __init__(self, b):
        self.lib = _lib.load()
        self.b = b
        self.h = self.lib.pcbg_costs_create(b["nx"], b["ny"], b["nl"], b["ncls"])
        assert self.h, _lib.last_error()
        for k in range(b["ncls"]):
            assert self.lib.pcbg_costs_set_static(self.h, k, b["st"][k].ctypes.data, b["vst"][k].ctypes.data) == 0
            assert self.lib.pcbg_costs_set_occupancy(self.h, k, b["oc"][k].ctypes.data, b["ov"][k].ctypes.data) == 0
        assert self.lib.pcbg_costs_set_history(self.h, b["hist"].ctypes.data) == 0
        for l, g in enumerate(b["gnd"]):
            if g is not None:
                assert self.lib.pcbg_costs_set_ground(self.h, l, g.ctypes.data) == 0

    def maps(self):
        b = self.b
        n = b["nx"] * b["ny"]
        cst = np.empty((b["ncls"], b["nl"], n), np.float32)
        vcst = np.empty((b["ncls"], n), np.float32)
        for k in range(b["ncls"]):
            assert self.lib.pcbg_costs_download(self.h, k, cst[k].ctypes.data, vcst[k].ctypes.data) == 0
        return cst, vcst

    def close(self):
        self.lib.pcbg_costs_destroy(self.h)


def _same(a, b):
    return np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("seed,pres,hard", [(11, 0.5, False), (12, 37.5, False), (13, 1e4, False), (14, 2.0, True)])
def test_device_rebuild_matches_oracle(gpu, seed, pres, hard):
    b = board(seed, nx=203 + seed, ny=77, nl=2 + seed % 3, ncls=1 + seed % 3)
    d = Dev(b)
    try:
        assert d.lib.pcbg_costs_rebuild(d.h, pres, int(hard)) == 0
        c, v = d.maps()
        c2, v2 = oracle_costs(b, pres, hard)
        assert _same(c, c2) and _same(v, v2)
    finally:
        d.close()


@pytest.mark.gpu
def test_device_stamps_and_history_match_oracle(gpu):
    """Commits stamp occupancy spans (+1 and later -1), the history grows on conflicting states (some repeated):
    after each step the device maps equal the oracle's maps of the updated board."""
    rng = np.random.default_rng(21)
    b = board(21, nx=150, ny=90, nl=3, ncls=2)
    d = Dev(b)
    try:
        pres, hard = 3.5, False
        assert d.lib.pcbg_costs_rebuild(d.h, pres, 0) == 0
        nx, ny, n = b["nx"], b["ny"], b["nx"] * b["ny"]
        stamped = []
        for step in range(6):
            k, kind, l = int(rng.integers(0, 2)), int(rng.integers(0, 2)), int(rng.integers(0, 3))
            rows = rng.choice(ny, size=12, replace=False)
            spans = []
            for j in rows:
                i0 = int(rng.integers(0, nx - 20))
                spans += [int(j), i0, i0 + int(rng.integers(0, 19))]
            sp = np.array(spans, np.int32)
            sign = 1 if step < 4 else -1
            if sign < 0:
                k, kind, l, sp = stamped[step - 4]
            assert d.lib.pcbg_costs_stamp(d.h, k, kind, l, sp.ctypes.data, len(sp) // 3, sign) == 0, _lib.last_error()
            stamped.append((k, kind, l, sp))
            g = b["ov"] if kind else b["oc"]
            for j, i0, i1 in sp.reshape(-1, 3):
                cells = g[k, l, j * nx + i0: j * nx + i1 + 1].astype(np.int64)
                g[k, l, j * nx + i0: j * nx + i1 + 1] = (np.minimum(cells + 1, 255) if sign > 0 else cells - 1) % 256
            # the device refreshed only the stamped cells with the rebuild's pres; compare those cells and the rest
            c, v = d.maps()
            c2, v2 = oracle_costs(b, pres, hard)
            assert _same(c, c2) and _same(v, v2), step
        states = rng.integers(0, n * b["nl"], size=400).astype(np.uint32)
        states = np.concatenate([states, states[:50]])       # repeated states add twice, in order
        assert d.lib.pcbg_costs_add_history(d.h, states.ctypes.data, len(states), np.float32(0.75)) == 0
        for q in states:
            b["hist"][q // n, q % n] = np.float32(b["hist"][q // n, q % n] + np.float32(0.75))
        hist = np.empty_like(b["hist"])
        assert d.lib.pcbg_costs_download_history(d.h, hist.ctypes.data) == 0
        assert _same(hist, b["hist"])
        pres = 5.25
        assert d.lib.pcbg_costs_rebuild(d.h, pres, 0) == 0
        c, v = d.maps()
        c2, v2 = oracle_costs(b, pres, hard)
        assert _same(c, c2) and _same(v, v2)
    finally:
        d.close()


@pytest.mark.gpu
def test_device_stamp_rejects_overlapping_spans(gpu):
    b = board(31, nx=64, ny=32, nl=2, ncls=1)
    d = Dev(b)
    try:
        sp = np.array([3, 10, 20, 3, 15, 30], np.int32)
        assert d.lib.pcbg_costs_stamp(d.h, 0, 0, 0, sp.ctypes.data, 2, 1) == -1
        assert "overlapping" in _lib.last_error()
    finally:
        d.close()
