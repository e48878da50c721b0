"""The CPU oracle on its own: fixed-point rules, Dijkstra against brute-force Bellman-Ford, cost resolution
against an independent numpy restatement of the reference's prep kernels, and the solve contract."""
import numpy as np
import pytest

from oracle import oracle as O
from pcbroute_b200 import synth

INF = O.INF64
DX = [1, -1, 0, 0, 1, 1, -1, -1]
DY = [0, 0, 1, -1, 1, -1, 1, -1]


def test_weight_rules():
    assert O.weight(1.0, 50.0) == 800
    assert O.weight(2.0, np.float32(50.0 * np.float32(np.sqrt(2.0)))) == int(np.rint(np.float32(2.0) * np.float32(70.71068) * 16))
    assert O.weight(1e30, 1.0) == INF
    assert O.weight(float("inf"), 1.0) == INF
    assert O.weight(0.0, 50.0) == 0
    assert O.weight(1.03125, 1.0) == 16 * 1 + 0  # 16.5 rounds half to even
    assert O.weight(1.09375, 1.0) == 18          # 17.5 -> 18
    assert O.weight(3e17, 16.0) == INF           # 16 * x >= 2^62
    assert O.start_d(0.0) == 0 and O.start_d(-5.0) == 0
    assert O.start_d(1.0) == 16 and O.start_d(1.01) == 17


def _bellman_ford(fac, cf, fl, vcf, si, sd):
    nl, rh, rw = cf.shape
    d = np.full((nl, rh, rw), INF, dtype=object)
    for s, v in zip(si, sd):
        l, c = divmod(int(s), rw * rh)
        d[l, c // rw, c % rw] = min(d[l, c // rw, c % rw], int(v))
    changed = True
    while changed:
        changed = False
        for l in range(nl):
            for j in range(rh):
                for i in range(rw):
                    best = d[l, j, i]
                    for m in range(8):
                        pi, pj = i - DX[m], j - DY[m]
                        if 0 <= pi < rw and 0 <= pj < rh and d[l, pj, pi] < INF:
                            w = O.weight(float(cf[l, j, i]), float(fac[l, m]))
                            if w < INF:
                                best = min(best, d[l, pj, pi] + w)
                    if vcf is not None and fl[l, j, i] & 1:
                        wv = O.weight(float(vcf[j, i]), 1.0)
                        if wv < INF:
                            for l2 in range(nl):
                                if l2 != l and d[l2, j, i] < INF:
                                    best = min(best, d[l2, j, i] + wv)
                    if best < d[l, j, i]:
                        d[l, j, i] = best
                        changed = True
    return d


@pytest.mark.parametrize("case", range(16))
def test_dijkstra_is_the_least_fixed_point(case):
    rng = np.random.default_rng(case)
    nl, rh, rw = int(rng.integers(1, 4)), int(rng.integers(1, 9)), int(rng.integers(1, 9))
    cf = (1 + rng.random((nl, rh, rw)) * 5).astype(np.float32)
    cf[rng.random(cf.shape) < 0.2] = 1e30
    fl = (rng.random((nl, rh, rw)) < 0.8).astype(np.uint8) | ((rng.random((nl, rh, rw)) < 0.1).astype(np.uint8) << 1)
    vcf = (rng.random((rh, rw)) * 300).astype(np.float32) if case % 3 else None
    fac = O.factors(50.0, np.where(rng.random((8, 8)) < 0.5, 1.0, 1.5).astype(np.float32))
    ns = int(rng.integers(1, 3))
    si = rng.integers(0, nl * rh * rw, ns).astype(np.uint32)
    sd = rng.integers(0, 2000, ns).astype(np.uint64)
    dist, best, bd = O.dijkstra(fac, cf, fl, vcf, si, sd)
    ref = _bellman_ford(fac, cf, fl, vcf, si, sd)
    d = dist.astype(object)
    if best < 0:
        assert (d == ref).all()
    else:
        # the search stops at the best target: exact at or below its cost, upper bounds above it
        low = ref <= bd
        assert (d[low] == ref[low]).all()
        assert (d[~low] > bd).all()
    tg = [(int(ref[s]), k) for k, s in enumerate(np.ndindex(ref.shape)) if fl[s] & 2 and ref[s] < INF]
    if tg:
        assert (bd, best) == min(tg)
    else:
        assert best == -1


def _resolve_numpy(q, rx0, ry0, rw, rh):
    """Independent restatement of src/gpu.cu:78-115 after the own-copper scatters (src/gpu.cu:460-478)."""
    nl = q.NL
    cf = np.empty((nl, rh, rw), np.float32)
    fl = np.empty((nl, rh, rw), np.uint8)
    jj, ii = np.mgrid[0:rh, 0:rw]
    gx, gy = q.wi0 + rx0 + ii, q.wj0 + ry0 + jj
    h = gy * q.nx + gx
    fwn = q.ww * q.wh
    own = {}
    for w, v in q.own_cf:
        l, c = divmod(w, fwn)
        i, j = c % q.ww - rx0, c // q.ww - ry0
        if 0 <= i < rw and 0 <= j < rh:
            own[(l, j, i)] = np.float32(v)
    for l in range(nl):
        v = q.cst[l][h].copy()
        for (ll, j, i), val in own.items():
            if ll == l:
                v[j, i] = val
        o = q.st[l][h]
        ws = (l * q.wh + ry0 + jj) * q.ww + rx0 + ii
        tg = ((q.tbit[ws >> 6] >> (ws & 63).astype(np.uint64)) & np.uint64(1)).astype(bool)
        with np.errstate(invalid="ignore", over="ignore"):
            r = np.where(~(v < 1e30) | (not q.lay[l]), np.float32(1e30),
                         np.where(v < 0, np.where(o == q.me, -v, np.float32(1e30)), v)).astype(np.float32)
        pv = np.full((rh, rw), 255)
        if q.prior is not None and q.lay[l]:
            pl = q.play[l]
            if pl >= 0:
                x, y = q.pcol[gx] - q.pi0, q.prow[gy] - q.pj0
                inb = (x >= 0) & (y >= 0) & (x < q.prior.shape[2]) & (y < q.prior.shape[1])
                pv = np.where(inb, q.prior[pl][np.clip(y, 0, q.prior.shape[1] - 1), np.clip(x, 0, q.prior.shape[2] - 1)], 0)
            cut = q.corridor & (pv < q.mthr) & ~tg
            with np.errstate(over="ignore"):
                r = np.where(cut, np.float32(1e30), np.where(r < 1e30, (r * q.mlf[pv]).astype(np.float32), r))
        cf[l] = r
        if q.lay[l]:
            vok = ((o == 0) | (o == q.me)) & (~np.bool_(q.corridor) | tg | (pv >= q.mthr))
        else:
            vok = tg
        fl[l] = vok.astype(np.uint8) | (tg.astype(np.uint8) << 1)
    return cf, fl


@pytest.mark.parametrize("seed", range(8))
def test_resolve_matches_independent_restatement(seed):
    q = synth.random_query(seed, nx=50, ny=40, nl=3, prior=seed % 2 == 1, corridor=seed % 4 == 1,
                           unusable_layer=seed % 3 == 0)
    rx0, ry0 = 3, 2
    rw, rh = q.ww - 5, q.wh - 4
    cf, fl, _ = O.resolve(q, rx0, ry0, rw, rh)
    cf2, fl2 = _resolve_numpy(q, rx0, ry0, rw, rh)
    assert np.array_equal(cf.view(np.uint32), cf2.view(np.uint32))
    assert np.array_equal(fl, fl2)


@pytest.mark.parametrize("seed", range(6))
def test_solve_contract(seed):
    """The reported field: best is a target at the least target cost, every finite value <= that cost, and every
    reported state satisfies the relaxation equation (it is reached by its cheapest predecessor)."""
    q = synth.random_query(40 + seed, nx=70, ny=60, nl=3, prior=seed % 2 == 0)
    rc, out = O.solve(q)
    assert rc >= 1
    assert out.best >= 0
    fwn = q.ww * q.wh
    l, c = divmod(out.best, fwn)
    assert (int(q.tbit[out.best >> 6]) >> (out.best & 63)) & 1
    bestv = out.d[l, c // q.ww - out.ry0, c % q.ww - out.rx0]
    fin = out.d[out.d < 1e29]
    assert fin.max() <= bestv
    assert np.float32(out.ub) == bestv


def test_golden_fixtures():
    """The oracle still produces the committed golden outputs (tests/golden/make_golden.py)."""
    import os
    from tests.golden import make_golden
    path = os.path.join(os.path.dirname(__file__), "golden", "oracle_golden.npz")
    g = np.load(path)
    for name, q in make_golden.cases():
        rc, out = O.solve(q)
        assert rc >= 1
        assert np.array_equal(g[name + "_rect"], np.array([out.rx0, out.ry0, out.rw, out.rh, out.best, out.tries])), name
        assert make_golden.digest(out.d) == str(g[name + "_digest"]), name


@pytest.mark.parametrize("seed", range(4))
def test_walkback_is_a_shortest_path(seed):
    """pcbo_walkback: consecutive states are one move or one via apart, each step's weight is exactly the distance
    difference, the walk starts at the best target and ends at a start at its start cost."""
    rw, rh, nl = 40 + 7 * seed, 33 + 5 * seed, 2 + seed % 3
    cf, fl, vcf, src, tgt = synth.search_arrays(300 + seed, rw, rh, nl, 12.0)
    fac = synth.microbench_factors(nl)
    si = np.array([src], np.uint32)
    sd = np.zeros(1, np.uint64)
    dist, best, bd = O.dijkstra(fac, cf, fl, vcf, si, sd)
    path = O.walkback(fac, cf, fl, vcf, si, sd, dist, best)
    if best < 0:
        assert path is not None and len(path) == 0
        return
    assert path is not None and path[0] == best and path[-1] == src
    d = dist.reshape(-1)
    RN = rw * rh
    for q, p in zip(path[:-1], path[1:]):
        lq, cq = divmod(int(q), RN)
        lp, cp = divmod(int(p), RN)
        jq, iq = divmod(cq, rw)
        jp, ip = divmod(cp, rw)
        if lq == lp:
            m = [k for k in range(8) if (iq - ip, jq - jp) == (DX[k], DY[k])]
            assert len(m) == 1
            w = O.weight(float(cf.reshape(-1)[q]), float(fac[lq, m[0]]))
        else:
            assert cq == cp and fl.reshape(-1)[q] & 1
            w = O.weight(float(vcf.reshape(-1)[cq]), 1.0)
        assert int(d[p]) + w == int(d[q])
