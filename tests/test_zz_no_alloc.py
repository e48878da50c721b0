"""pcbg_solve_noalloc: the entry point for callers that cannot allocate device memory.

Callers whose device memory belongs to another allocator, or whose threads must not be stalled by cudaFree,
call pcbg_solve_noalloc. It keeps its scratch in a static device array, so it must give exactly what
pcbg_solve_batch (which allocates from its own arena) gives for the same search, and both must equal the CPU
oracle. These tests check that on two calls in a row with different searches, since the second call reuses the
array the first one left behind; that the walk-back it is asked for is the batch path's; that repeated calls leave
the device's free memory unchanged; and that a search above the stated limit is refused with a message. This file
is collected last.
"""
import numpy as np
import pytest

from oracle import oracle
from pcbroute_b200 import _lib, synth

pytestmark = pytest.mark.gpu


def _search(torch, seed, rw, rh, nl, via):
    lib = _lib.load()
    pitch, hpad = -(-rw // 32) * 32, -(-rh // 32) * 32
    t = dict(cf=torch.empty(nl * hpad * pitch, dtype=torch.float32, device="cuda"),
             fl=torch.empty(nl * hpad * pitch, dtype=torch.uint8, device="cuda"),
             vcf=torch.empty(hpad * pitch, dtype=torch.float32, device="cuda"),
             st=torch.empty(2, dtype=torch.int64, device="cuda"))
    assert lib.pcbg_synth_search(seed, rw, rh, nl, pitch, hpad, via, t["cf"].data_ptr(), t["fl"].data_ptr(),
                                 t["vcf"].data_ptr(), t["st"].data_ptr(), None) == 0
    t["si"] = t["st"][:1].to(torch.int32)
    t["sd"] = torch.zeros(1, dtype=torch.int64, device="cuda")
    n = rw * rh * nl
    t["out"] = torch.full((n,), -1.0, dtype=torch.float32, device="cuda")
    cap = 4 * (rw + rh) * nl + 64
    t["path"] = torch.zeros(cap, dtype=torch.int32, device="cuda")
    t["plen"] = torch.full((1,), -7, dtype=torch.int32, device="cuda")
    arr = (_lib.Search * 1)()
    a = arr[0]
    a.rw, a.rh, a.nl, a.pitch, a.hpad = rw, rh, nl, pitch, hpad
    fac = synth.microbench_factors(nl)
    for l in range(8):
        for m in range(8):
            a.fac[l][m] = float(fac[l, m])
    a.cf, a.flags, a.vcf = t["cf"].data_ptr(), t["fl"].data_ptr(), t["vcf"].data_ptr()
    a.start_idx, a.start_d, a.n_starts = t["si"].data_ptr(), t["sd"].data_ptr(), 1
    a.out = t["out"].data_ptr()
    a.path, a.path_cap, a.path_len = t["path"].data_ptr(), cap, t["plen"].data_ptr()
    return arr, t


def _solve(torch, noalloc, arr, t):
    lib = _lib.load()
    t["out"].fill_(-1.0)
    t["path"].zero_()
    t["plen"].fill_(-7)
    torch.cuda.synchronize()
    rc = lib.pcbg_solve_noalloc(arr, None) if noalloc else lib.pcbg_solve_batch(arr, 1, None)
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    plen = int(t["plen"].item())
    path = t["path"][:max(plen, 0)].cpu().numpy().copy()
    return t["out"].cpu().numpy().copy(), arr[0].best, arr[0].best_d, arr[0].status, plen, path


CASES = [(7001, 700, 520, 5, 12.0), (7002, 230, 170, 3, 20.0)]


def test_noalloc_matches_the_allocating_entry_point_and_the_oracle_on_two_calls_in_a_row():
    import torch
    assert torch.cuda.is_available()
    # the second search is smaller than the first: what call 1 left in the array must not leak into call 2
    made = [_search(torch, *c) for c in CASES]
    refs = [_solve(torch, False, arr, t) for (arr, t) in made]
    gots = [_solve(torch, True, arr, t) for (arr, t) in made]   # two no-alloc calls in a row
    for c, ref, got in zip(CASES, refs, gots):
        assert got[1:4] == ref[1:4], (c, got[1:4], ref[1:4])
        assert got[1] >= 0
        # exact: the arithmetic is integer, the tolerance is zero
        assert np.array_equal(got[0].view(np.uint32), ref[0].view(np.uint32)), c
        # the walk-back the caller asked for: written, and the batch path's state for state
        assert got[4] > 0 and got[4] == ref[4], (c, got[4], ref[4])
        assert np.array_equal(got[5], ref[5]), c
        # and the oracle's field and best target
        seed, rw, rh, nl, via = c
        cf, fl, vcf, src, tgt = synth.search_arrays(seed, rw, rh, nl, via)
        dist, best, bd = oracle.dijkstra(synth.microbench_factors(nl), cf, fl, vcf, np.array([src], np.uint32),
                                         np.zeros(1, np.uint64))
        assert got[1] == best and got[2] == bd, (c, got[1:3], best, bd)
        field = oracle.report(dist, best, bd)
        assert np.array_equal(got[0].view(np.uint32), field.reshape(-1).view(np.uint32)), c
        assert int(got[5][0]) == best and int(got[5][-1]) == src


def test_noalloc_calls_leave_free_device_memory_unchanged():
    import torch
    made = [_search(torch, *c) for c in CASES]
    for arr, t in made:                       # warm-up: every kernel this path launches is loaded
        _solve(torch, True, arr, t)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    lib = _lib.load()
    for _ in range(3):
        for arr, _t in made:
            assert lib.pcbg_solve_noalloc(arr, None) == 0, _lib.last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_refuses_searches_above_its_limit():
    import torch
    lib = _lib.load()
    arr, t = _search(torch, 7003, 64, 64, 2, 10.0)
    arr[0].rw, arr[0].rh, arr[0].pitch, arr[0].hpad = 2048, 1056, 2048, 1056   # 2 x 2048 x 1056 > 2^21
    arr[0].out = None
    arr[0].path = None
    assert lib.pcbg_solve_noalloc(arr, None) == -1
    assert "exceeds the no-alloc limit" in _lib.last_error()
