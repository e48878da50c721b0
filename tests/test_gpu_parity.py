"""Parity of the sm_100a back end with the CPU oracle: bit-exact fields, best targets, rectangles.

Every test here runs the CUDA kernels through the C ABI (libpcbgpu.so) and checks the result against
oracle/oracle.py on the same seeded inputs.
"""
import ctypes as C

import numpy as np
import pytest

from pcbroute_b200 import _lib, query, synth
from oracle import oracle

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def make_device_search(seed, rw, rh, nl, via):
    """Generate one microbenchmark search on the device (pitched) and return tensors + numpy copies."""
    torch = _torch()
    pitch, hpad = -(-rw // 32) * 32, -(-rh // 32) * 32
    cf = torch.empty(nl * hpad * pitch, dtype=torch.float32, device="cuda")
    fl = torch.empty(nl * hpad * pitch, dtype=torch.uint8, device="cuda")
    vcf = torch.empty(hpad * pitch, dtype=torch.float32, device="cuda")
    st = torch.empty(2, dtype=torch.int64, device="cuda")
    rc = _lib.load().pcbg_synth_search(seed, rw, rh, nl, pitch, hpad, via, cf.data_ptr(), fl.data_ptr(),
                                       vcf.data_ptr(), st.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    return dict(rw=rw, rh=rh, nl=nl, pitch=pitch, hpad=hpad, via=via, seed=seed, cf=cf, fl=fl, vcf=vcf, st=st)


def dense(t, nl, hpad, pitch, rh, rw):
    return t.cpu().numpy().reshape(nl, hpad, pitch)[:, :rh, :rw]


@pytest.mark.parametrize("rw,rh,nl", [(64, 64, 2), (97, 45, 3), (200, 130, 6), (31, 257, 4), (33, 33, 8)])
def test_device_generator_matches_numpy(gpu, rw, rh, nl):
    s = make_device_search(1234 + rw, rw, rh, nl, 17.0)
    cf, fl, vcf, src, tgt = synth.search_arrays(1234 + rw, rw, rh, nl, 17.0)
    dcf = dense(s["cf"], nl, s["hpad"], s["pitch"], rh, rw)
    dfl = dense(s["fl"], nl, s["hpad"], s["pitch"], rh, rw)
    assert np.array_equal(dcf.view(np.uint32), cf.view(np.uint32))
    assert np.array_equal(dfl, fl)
    assert np.array_equal(s["vcf"].cpu().numpy().reshape(s["hpad"], s["pitch"])[:rh, :rw], vcf)
    assert tuple(s["st"].cpu().tolist()) == (src, tgt)
    # padding is impassable
    full = s["cf"].cpu().numpy().reshape(nl, s["hpad"], s["pitch"])
    assert (full[:, rh:, :] >= 1e30).all() and (full[:, :, rw:] >= 1e30).all()


def run_batch(searches, with_out=True, with_path=False):
    torch = _torch()
    lib = _lib.load()
    arr = (_lib.Search * len(searches))()
    keep = []
    for k, s in enumerate(searches):
        a = arr[k]
        a.rw, a.rh, a.nl, a.pitch, a.hpad = s["rw"], s["rh"], s["nl"], s["pitch"], s["hpad"]
        fac = synth.microbench_factors(s["nl"])
        for l in range(8):
            for m in range(8):
                a.fac[l][m] = float(fac[l, m])
        a.cf, a.flags, a.vcf = s["cf"].data_ptr(), s["fl"].data_ptr(), s["vcf"].data_ptr()
        src = int(s["st"][0].item())
        si = torch.tensor([max(src, 0)], dtype=torch.int32, device="cuda")
        sd = torch.zeros(1, dtype=torch.int64, device="cuda")
        keep += [si, sd]
        a.start_idx, a.start_d, a.n_starts = si.data_ptr(), sd.data_ptr(), 1 if src >= 0 else 0
        if with_out:
            out = torch.empty(s["nl"] * s["rh"] * s["rw"], dtype=torch.float32, device="cuda")
            keep.append(out)
            s["out"] = out
            a.out = out.data_ptr()
        else:
            a.out = None
        if with_path:
            cap = 4 * (s["rw"] + s["rh"]) * s["nl"] + 64
            path = torch.empty(cap, dtype=torch.int32, device="cuda")
            plen = torch.zeros(1, dtype=torch.int32, device="cuda")
            keep += [path, plen]
            s["path"], s["plen"] = path, plen
            a.path, a.path_cap, a.path_len = path.data_ptr(), cap, plen.data_ptr()
    rc = lib.pcbg_solve_batch(arr, len(searches), None)
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    return arr


def oracle_of(s):
    cf, fl, vcf, src, tgt = synth.search_arrays(s["seed"], s["rw"], s["rh"], s["nl"], s["via"])
    fac = synth.microbench_factors(s["nl"])
    si = np.array([src] if src >= 0 else [], np.uint32)
    sd = np.zeros(len(si), np.uint64)
    dist, best, bd = oracle.dijkstra(fac, cf, fl, vcf, si, sd)
    return oracle.report(dist, best, bd), best, bd


def test_batch_matches_oracle(gpu):
    rng = np.random.default_rng(5)
    searches = []
    for k in range(24):
        rw, rh = int(rng.integers(20, 320)), int(rng.integers(20, 320))
        nl = int(rng.integers(2, 7))
        searches.append(make_device_search(9000 + k, rw, rh, nl, float(rng.integers(8, 33))))
    arr = run_batch(searches)
    for k, s in enumerate(searches):
        field, best, bd = oracle_of(s)
        assert arr[k].best == best, (k, arr[k].best, best)
        if best >= 0:
            assert arr[k].best_d == bd
        got = s["out"].cpu().numpy().reshape(s["nl"], s["rh"], s["rw"])
        assert np.array_equal(got.view(np.uint32), field.view(np.uint32)), k


def test_large_batch_matches_oracle(gpu):
    """A batch of at least 48 tiles per SM: the solver then runs its 3-blocks-per-SM build of the relax kernel (taken
    for batches of 16 or more tiles per resident block), which smaller batches never reach."""
    torch = _torch()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    side = 960                                     # 30 x 30 tiles per search
    n = -(-48 * sms // (30 * 30)) + 1
    searches = [make_device_search(9500 + k, side, side, 2, 20.0) for k in range(n)]
    arr = run_batch(searches)
    for k, s in enumerate(searches):
        field, best, bd = oracle_of(s)
        assert arr[k].best == best, (k, arr[k].best, best)
        if best >= 0:
            assert arr[k].best_d == bd
        got = s["out"].cpu().numpy().reshape(s["nl"], s["rh"], s["rw"])
        assert np.array_equal(got.view(np.uint32), field.view(np.uint32)), k


def _oracle_many(searches, threads=None):
    """oracle_of over many searches on host threads (the C oracle releases the GIL)."""
    import os
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(threads or os.cpu_count() or 1) as ex:
        return list(ex.map(oracle_of, searches))


def _check_fields(searches, arr, refs, tag):
    for k, (s, (field, best, bd)) in enumerate(zip(searches, refs)):
        assert arr[k].best == best, (tag, k, arr[k].best, best)
        if best >= 0:
            assert arr[k].best_d == bd, (tag, k)
        got = s["out"].cpu().numpy().reshape(s["nl"], s["rh"], s["rw"])
        assert np.array_equal(got.view(np.uint32), field.view(np.uint32)), (tag, k)
        del s["out"]


def test_largest_microbenchmark_searches_match_oracle(gpu):
    """The 8 largest searches of the benchmarked workload (windows up to 2047 x 2047 with up to 6 layers, 32-bit
    distances near their largest values) in one launch, large enough for the 3-blocks-per-SM build: fields, best
    targets and their costs equal the oracle's bit for bit."""
    sizes = synth.microbench_sizes(20261203, 4096)
    big = sorted(range(len(sizes)), key=lambda k: -sizes[k][0] * sizes[k][1] * sizes[k][2])[:8]
    assert max(sizes[k][0] for k in big) >= 1800 and max(sizes[k][2] for k in big) == 6
    searches = [make_device_search(sizes[k][4], sizes[k][0], sizes[k][1], sizes[k][2], sizes[k][3]) for k in big]
    arr = run_batch(searches)
    refs = _oracle_many(searches)
    _check_fields(searches, arr, refs, "largest")


def test_eight_layer_searches_match_oracle(gpu):
    """8-layer windows of 1024 x 1024 and more (the most shared memory per visit) against the oracle."""
    searches = [make_device_search(9800 + k, rw, rh, 8, via)
                for k, (rw, rh, via) in enumerate([(1024, 1024, 12.0), (1200, 1100, 30.0)])]
    arr = run_batch(searches)
    _check_fields(searches, arr, _oracle_many(searches), "8 layers")


@pytest.mark.parametrize("band", [0, 1, 4, 64])
def test_round_band_changes_work_not_results(gpu, band):
    """Ordered rounds (pcbg_set_round_band) change which tiles a round visits, never the fixed point: every band,
    0 (every queued tile each round) included, gives the oracle's fields and best targets."""
    lib = _lib.load()
    rng = np.random.default_rng(77)
    searches = []
    for k in range(10):
        rw, rh = int(rng.integers(60, 700)), int(rng.integers(60, 700))
        searches.append(make_device_search(9700 + k, rw, rh, int(rng.integers(2, 7)), float(rng.integers(8, 33))))
    lib.pcbg_set_round_band(band)
    try:
        arr = run_batch(searches)
        deferred = lib.pcbg_last_batch_deferred()
    finally:
        lib.pcbg_set_round_band(-1)   # back to the tuned / default band
    if band == 0:
        assert deferred == 0
    for k, s in enumerate(searches):
        field, best, bd = oracle_of(s)
        assert arr[k].best == best, (band, k, arr[k].best, best)
        if best >= 0:
            assert arr[k].best_d == bd
        got = s["out"].cpu().numpy().reshape(s["nl"], s["rh"], s["rw"])
        assert np.array_equal(got.view(np.uint32), field.view(np.uint32)), (band, k)


@pytest.mark.parametrize("order", [0, 1, 2])
def test_visit_order_changes_work_not_results(gpu, order):
    """The order of an ordered round's visits (pcbg_set_visit_order: as listed, the lower half of each search's band
    first, the searches with the most layers first) changes which visits see which neighbours' results, never the
    fixed point. The visit list's two-ended filling is checked with a narrow band (many deferred tiles, rounds of
    both parts) on searches of 2 to 6 layers; the busy share is a fraction."""
    lib = _lib.load()
    rng = np.random.default_rng(78)
    searches = []
    for k in range(12):
        rw, rh = int(rng.integers(100, 900)), int(rng.integers(100, 900))
        searches.append(make_device_search(9600 + k, rw, rh, int(rng.integers(2, 7)), float(rng.integers(8, 33))))
    prev = lib.pcbg_visit_order()
    lib.pcbg_set_round_band(4)
    lib.pcbg_set_visit_order(order)
    try:
        assert lib.pcbg_visit_order() == order
        arr = run_batch(searches)
        busy = lib.pcbg_last_batch_busy_frac()
        assert lib.pcbg_last_batch_deferred() > 0
    finally:
        lib.pcbg_set_round_band(-1)
        lib.pcbg_set_visit_order(prev)
    assert 0.0 < busy <= 1.0, busy
    _check_fields(searches, arr, _oracle_many(searches), f"order {order}")


def test_walkback_matches_oracle(gpu):
    """The device walk-back (one warp per search, after the relaxation) equals the oracle's walk over its exact
    field: the same states in the same order, best target first, ending on the start."""
    rng = np.random.default_rng(11)
    searches = []
    for k in range(16):
        rw, rh = int(rng.integers(20, 260)), int(rng.integers(20, 260))
        searches.append(make_device_search(4200 + k, rw, rh, int(rng.integers(2, 7)), float(rng.integers(8, 33))))
    arr = run_batch(searches, with_path=True)
    walked = 0
    for k, s in enumerate(searches):
        cf, fl, vcf, src, tgt = synth.search_arrays(s["seed"], s["rw"], s["rh"], s["nl"], s["via"])
        fac = synth.microbench_factors(s["nl"])
        si = np.array([src] if src >= 0 else [], np.uint32)
        sd = np.zeros(len(si), np.uint64)
        dist, best, bd = oracle.dijkstra(fac, cf, fl, vcf, si, sd)
        ref = oracle.walkback(fac, cf, fl, vcf, si, sd, dist, best)
        n = int(s["plen"].item())
        assert ref is not None
        assert n == len(ref), (k, n, len(ref))
        got = s["path"][:n].cpu().numpy().view(np.uint32)
        assert np.array_equal(got, ref), k
        walked += n > 0
    assert walked >= 10


def test_batch_without_field_output(gpu):
    searches = [make_device_search(77 + k, 150 + 13 * k, 90 + 7 * k, 3, 12.0) for k in range(4)]
    arr = run_batch(searches, with_out=False)
    for k, s in enumerate(searches):
        _, best, bd = oracle_of(s)
        assert (arr[k].best, arr[k].best_d if best >= 0 else 0) == (best, bd if best >= 0 else 0)


def _cmp_query(q):
    out = query.GpuOut()
    rc = query.gpu_solve(q, out)
    orc, ref = oracle.solve(q)
    if orc < 0:
        assert rc == -1
        return out, ref
    assert rc >= 1, _lib.last_error()
    assert (out.rx0, out.ry0, out.rw, out.rh, out.NL, out.ww, out.wh) == \
        (ref.rx0, ref.ry0, ref.rw, ref.rh, ref.NL, ref.ww, ref.wh)
    assert out.best == ref.best
    assert out.tries == ref.tries
    assert np.array_equal(out.d.view(np.uint32), ref.d.view(np.uint32))
    return out, ref


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("opts", [
    dict(),
    dict(prior=True),
    dict(prior=True, corridor=True),
    dict(vias=False),
    dict(unusable_layer=True),
    dict(own=False, n_starts=1, n_targets=1),
])
def test_query_matches_oracle(gpu, seed, opts):
    q = synth.random_query(100 + seed, nx=120, ny=100, nl=3 + seed % 3, **opts)
    _cmp_query(q)


@pytest.mark.parametrize("seed", range(4))
def test_query_free_direction_factors(gpu, seed):
    """A factor per move (no x / y / diagonal classes): the general per-layer relaxation."""
    _cmp_query(synth.random_query(500 + seed, nx=110, ny=90, nl=2 + seed, free_dirf=True))


@pytest.mark.parametrize("seed", range(3))
def test_query_large_costs(gpu, seed):
    """Cost factors up to 3e5 (16 x weights far above 65535 but inside 32-bit arithmetic): tiles holding them are
    relaxed by the general path, the others by the 16-bit joint path, in the same solve."""
    _cmp_query(synth.random_query(700 + seed, nx=130, ny=100, nl=3, big_costs=True))


@pytest.mark.parametrize("corner", [(31, 31), (32, 32), (31, 32), (0, 31), (63, 0), (32, 5), (5, 63)])
def test_start_on_tile_edges(gpu, corner):
    """Starts on tile edges and corners: the tiles around a start must all relax from it."""
    i, j = corner
    q = synth.random_query(600 + i + 7 * j, nx=100, ny=100, nl=2, window=(0, 0, 100, 100), n_starts=1, n_targets=2,
                           own=False)
    q.starts = [(j * q.ww + i, 0.0)]
    _cmp_query(q)


def test_batch_mixes_joint_and_general_searches(gpu):
    """One persistent launch holding searches of both relaxation modes and different layer counts."""
    torch = _torch()
    lib = _lib.load()
    searches = [make_device_search(4000 + k, 70 + 31 * k, 50 + 17 * k, 2 + k % 5, 9.0) for k in range(6)]
    arr = (_lib.Search * len(searches))()
    keep, facs = [], []
    rng = np.random.default_rng(3)
    for k, s in enumerate(searches):
        a = arr[k]
        a.rw, a.rh, a.nl, a.pitch, a.hpad = s["rw"], s["rh"], s["nl"], s["pitch"], s["hpad"]
        fac = synth.microbench_factors(s["nl"])
        if k % 2:  # per-move factors: general mode
            fac = (fac * (1.0 + rng.integers(0, 4, size=(8, 8)) * 0.25)).astype(np.float32)
        facs.append(fac)
        for l in range(8):
            for m in range(8):
                a.fac[l][m] = float(fac[l, m])
        a.cf, a.flags, a.vcf = s["cf"].data_ptr(), s["fl"].data_ptr(), s["vcf"].data_ptr()
        si = s["st"][:1].to(torch.int32)
        sd = torch.zeros(1, dtype=torch.int64, device="cuda")
        out = torch.empty(s["nl"] * s["rh"] * s["rw"], dtype=torch.float32, device="cuda")
        keep += [si, sd, out]
        s["out"] = out
        a.start_idx, a.start_d, a.n_starts, a.out = si.data_ptr(), sd.data_ptr(), 1, out.data_ptr()
    assert lib.pcbg_solve_batch(arr, len(arr), None) == 0, _lib.last_error()
    torch.cuda.synchronize()
    for k, s in enumerate(searches):
        cf, fl, vcf, src, tgt = synth.search_arrays(s["seed"], s["rw"], s["rh"], s["nl"], s["via"])
        dist, best, bd = oracle.dijkstra(facs[k], cf, fl, vcf, np.array([src], np.uint32), np.zeros(1, np.uint64))
        field = oracle.report(dist, best, bd)
        assert arr[k].best == best
        got = s["out"].cpu().numpy().reshape(s["nl"], s["rh"], s["rw"])
        assert np.array_equal(got.view(np.uint32), field.view(np.uint32)), k


@pytest.mark.parametrize("seed", range(4))
def test_query_rectangle_growth(gpu, seed):
    """Windows much larger than the start/target box: the solved rectangle grows by 80 x 3^k cells."""
    rng = np.random.default_rng(seed)
    q = synth.random_query(300 + seed, nx=900, ny=700, nl=2, window=(10, 20, 880, 670), n_starts=1, n_targets=2)
    # put the starts and targets close together so the first rectangle is small
    fwn = q.ww * q.wh
    cx, cy = int(rng.integers(200, 600)), int(rng.integers(150, 450))
    q.starts = [((cy * q.ww + cx), 0.0)]
    q.tbit[:] = 0
    for dx, dy in [(int(rng.integers(5, 60)), int(rng.integers(-40, 40))), (-30, 25)]:
        t = (cy + dy) * q.ww + cx + dx + fwn * int(rng.integers(0, 2))
        q.tbit[t >> 6] |= np.uint64(1) << np.uint64(t & 63)
    out, ref = _cmp_query(q)
    assert ref.rw < q.ww or ref.rh < q.wh  # a proper sub-rectangle was enough


def test_unreachable_target(gpu):
    q = synth.random_query(7, nx=80, ny=60, nl=2, n_starts=1, n_targets=1, vias=False, own=False)
    fwn = q.ww * q.wh
    # wall the target in on both layers (blocked ring)
    t = (q.wh // 2) * q.ww + q.ww // 2
    q.tbit[:] = 0
    q.tbit[t >> 6] |= np.uint64(1) << np.uint64(t & 63)
    for l in range(2):
        for dj in range(-2, 3):
            for di in range(-2, 3):
                if max(abs(di), abs(dj)) == 2:
                    c = (q.wj0 + q.wh // 2 + dj) * q.nx + q.wi0 + q.ww // 2 + di
                    q.cst[l, c] = 1e30
    q.starts = [(0 * fwn + 3 * q.ww + 3, 0.0)]
    out, ref = _cmp_query(q)
    assert out.best == -1 and ref.best == -1


def test_start_on_target(gpu):
    q = synth.random_query(8, nx=70, ny=50, nl=2, n_starts=1, n_targets=1, own=False)
    q.tbit[:] = 0
    s = q.starts[0][0]
    q.tbit[s >> 6] |= np.uint64(1) << np.uint64(s & 63)
    out, ref = _cmp_query(q)
    assert out.best == s


@pytest.mark.parametrize("ww,wh,nl", [(1, 1, 2), (33, 1, 1), (1, 65, 3), (45, 37, 8)])
def test_odd_windows(gpu, ww, wh, nl):
    q = synth.random_query(9 + ww + wh, nx=ww + 10, ny=wh + 10, nl=nl, window=(5, 5, ww, wh), n_starts=1,
                           n_targets=1, own=False)
    _cmp_query(q)


def test_wide_distances(gpu):
    """A target reachable only across very expensive cells: 32-bit weights overflow, the 64-bit pass takes over."""
    q = synth.random_query(21, nx=100, ny=40, nl=1, window=(0, 0, 100, 40), n_starts=1, n_targets=1, vias=False,
                           own=False)
    q.cst[:] = np.abs(q.cst[:]).clip(1, 4).astype(np.float32)
    q.st[:] = 0
    # a wall at x = 50 of cost 5e6 (16 * 70 * 5e6 > 2^31)
    for j in range(40):
        q.cst[0, j * 100 + 50] = np.float32(5e6)
    q.starts = [(20 * 100 + 10, 0.0)]
    q.tbit[:] = 0
    t = 20 * 100 + 90
    q.tbit[t >> 6] |= np.uint64(1) << np.uint64(t & 63)
    out, ref = _cmp_query(q)
    assert out.wide and out.best == t and ref.ub > 5e6


def test_concurrent_queries_are_batched_and_exact(gpu):
    """Queries from 8 threads at once (the router's worker threads) run through the round batcher: the launches
    solve several searches each, and every result is the oracle's, whatever the grouping."""
    import threading
    lib = _lib.load()
    qs = [synth.random_query(700 + k, nx=150, ny=110, nl=2 + k % 5, prior=k % 3 == 0) for k in range(24)]
    refs = [oracle.solve(q) for q in qs]
    b0, s0 = C.c_int64(), C.c_int64()
    lib.pcbg_batcher_stats(C.byref(b0), C.byref(s0))
    outs = [None] * len(qs)
    errs = []

    def work(w):
        try:
            for k in range(w, len(qs), 8):
                out = query.GpuOut()
                outs[k] = (query.gpu_solve(qs[k], out), out)
        except Exception as e:  # surfaced below
            errs.append(e)

    ts = [threading.Thread(target=work, args=(w,)) for w in range(8)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errs, errs
    b1, s1 = C.c_int64(), C.c_int64()
    lib.pcbg_batcher_stats(C.byref(b1), C.byref(s1))
    searches, batches = s1.value - s0.value, b1.value - b0.value
    assert searches >= len(qs)
    assert batches < searches, (batches, searches)    # some launches solved more than one search
    for (rc, out), (orc, ref) in zip(outs, refs):
        if orc < 0:
            assert rc == -1
            continue
        assert rc >= 1
        assert (out.rx0, out.ry0, out.rw, out.rh, out.best, out.tries) == \
            (ref.rx0, ref.ry0, ref.rw, ref.rh, ref.best, ref.tries)
        assert np.array_equal(out.d.view(np.uint32), ref.d.view(np.uint32))


def test_round_cap_stops_the_launch_and_the_device_stays_usable(gpu):
    """The relaxation's round loop is bounded (pcbg_set_max_rounds lowers the bound): a launch that reaches it stops,
    the solve returns PCBG_ERR_FAIL with the error bit of the round cap (ERR_ROUNDS = 2), and the next solve on the
    same context is exact again."""
    lib = _lib.load()
    s = make_device_search(9900, 900, 700, 4, 20.0)
    lib.pcbg_set_max_rounds(2)
    try:
        arr = (_lib.Search * 1)()
        torch = _torch()
        a = arr[0]
        a.rw, a.rh, a.nl, a.pitch, a.hpad = s["rw"], s["rh"], s["nl"], s["pitch"], s["hpad"]
        fac = synth.microbench_factors(s["nl"])
        for l in range(8):
            for m in range(8):
                a.fac[l][m] = float(fac[l, m])
        a.cf, a.flags, a.vcf = s["cf"].data_ptr(), s["fl"].data_ptr(), s["vcf"].data_ptr()
        si = s["st"][:1].to(torch.int32)
        sd = torch.zeros(1, dtype=torch.int64, device="cuda")
        a.start_idx, a.start_d, a.n_starts = si.data_ptr(), sd.data_ptr(), 1
        assert lib.pcbg_solve_batch(arr, 1, None) == -1
        assert "error bits 2" in _lib.last_error(), _lib.last_error()
    finally:
        lib.pcbg_set_max_rounds(0)
    arr = run_batch([s])
    field, best, bd = oracle_of(s)
    assert arr[0].best == best
    got = s["out"].cpu().numpy().reshape(s["nl"], s["rh"], s["rw"])
    assert np.array_equal(got.view(np.uint32), field.view(np.uint32))


def test_autotuned_schedule_keeps_results(gpu):
    """pcbg_autotune_batch times every schedule on a batch and keeps the fastest for its class; the solves that then
    take the tuned schedule still give the oracle's fields."""
    lib = _lib.load()
    searches = [make_device_search(9950 + k, 300 + 40 * k, 260, 2 + k % 5, 14.0) for k in range(6)]
    arr = run_batch(searches)
    e = _lib.TuneEntry()
    assert lib.pcbg_autotune_batch(arr, len(searches), None, C.byref(e)) == 1, _lib.last_error()
    assert e.band in (0, 8, 16, 32, 64, 128) and e.blocks_per_sm in (2, 3) and e.ms > 0
    arr = run_batch(searches)
    assert lib.pcbg_round_band() == e.band
    for k, s in enumerate(searches):
        field, best, bd = oracle_of(s)
        assert arr[k].best == best
        got = s["out"].cpu().numpy().reshape(s["nl"], s["rh"], s["rw"])
        assert np.array_equal(got.view(np.uint32), field.view(np.uint32)), k
